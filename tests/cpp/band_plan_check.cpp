// Test driver: the coarser levels' bands of a banded encode (band_plan.h follow_bands) on
// seeded random parent maps. Checks, per case: a parent's band is the latest band of its
// children (0 without children), so no brick runs before a child it reads; the order lists
// every brick once, by band, keeping brick order within a band; band g is exactly
// order[cuts[g], cuts[g + 1]). Prints "ok <cases>" or the first failure; exit code 0 on success.
#include "band_plan.h"

#include <cstdio>
#include <random>
#include <vector>

using namespace idx2g;

int main()
{
  std::mt19937 rng(5);
  int cases = 0;
  for (int t = 0; t < 400; ++t)
  {
    const int nbands = 1 + (int)(rng() % 17);
    const int nparents = (int)(rng() % 300);
    const int nchild = (int)(rng() % 2400);
    std::vector<int> cb((size_t)nchild), cp((size_t)nchild);
    for (int j = 0; j < nchild; ++j)
    {
      cb[(size_t)j] = (int)(rng() % (unsigned)nbands);
      // mostly valid parents, some none or out of range
      const unsigned r = rng() % 20;
      cp[(size_t)j] = r == 0 ? -1 : (r == 1 ? nparents + (int)(rng() % 5) : (nparents ? (int)(rng() % (unsigned)nparents) : -1));
    }
    const level_bands lb = follow_bands(cb, cp, nparents, nbands);
    std::vector<int> want((size_t)nparents, 0);
    for (int j = 0; j < nchild; ++j)
      if (cp[(size_t)j] >= 0 && cp[(size_t)j] < nparents && cb[(size_t)j] > want[(size_t)cp[(size_t)j]])
        want[(size_t)cp[(size_t)j]] = cb[(size_t)j];
    if (lb.band != want)
    {
      std::printf("FAIL band case %d\n", t);
      return 1;
    }
    if ((int)lb.order.size() != nparents || (int)lb.cuts.size() != nbands + 1 || lb.cuts[0] != 0 ||
        lb.cuts[(size_t)nbands] != nparents)
    {
      std::printf("FAIL shape case %d\n", t);
      return 1;
    }
    std::vector<int> seen((size_t)nparents, 0);
    for (int g = 0; g < nbands; ++g)
      for (int i = lb.cuts[(size_t)g]; i < lb.cuts[(size_t)g + 1]; ++i)
      {
        const int p = lb.order[(size_t)i];
        if (p < 0 || p >= nparents || seen[(size_t)p]++ || lb.band[(size_t)p] != g ||
            (i > lb.cuts[(size_t)g] && lb.order[(size_t)i - 1] > p))
        {
          std::printf("FAIL order case %d band %d index %d\n", t, g, i);
          return 1;
        }
      }
    ++cases;
  }
  std::printf("ok %d\n", cases);
  return 0;
}
