// Bands of the coarser levels of an encode whose level 0 runs in bands (the field arriving
// band by band from host memory): a brick of level l + 1 can run once every brick that hands
// it its low band (its children on level l) has run, so its band is the latest band among its
// children's. Host-only; used by the level-0 streamed encode (encode.cu) and tested on the CPU.
#pragma once

#include <algorithm>
#include <vector>

namespace idx2g
{

struct level_bands
{
  std::vector<int> band;   // per brick of the level: the band after which it can run
  std::vector<int> order;  // the level's bricks by band (stable: brick order within a band)
  std::vector<int> cuts;   // nbands + 1 entries: band g is order[cuts[g], cuts[g + 1])
};

// child_band[j], child_parent[j]: the band of brick j of the finer level and the index of its
// parent on this level (-1 or out of range: none); nparents bricks on this level, nbands bands.
// A brick without children gets band 0.
inline level_bands follow_bands(const std::vector<int>& child_band, const std::vector<int>& child_parent, int nparents,
                                int nbands)
{
  level_bands r;
  const size_t n = nparents > 0 ? (size_t)nparents : 0;
  r.band.assign(n, 0);
  for (size_t j = 0; j < child_band.size() && j < child_parent.size(); ++j)
  {
    const int p = child_parent[j];
    if (p >= 0 && (size_t)p < n && child_band[j] > r.band[(size_t)p])
      r.band[(size_t)p] = child_band[j];
  }
  r.order.resize(n);
  for (size_t i = 0; i < n; ++i)
    r.order[i] = (int)i;
  std::stable_sort(r.order.begin(), r.order.end(),
                   [&](int x, int y) { return r.band[(size_t)x] < r.band[(size_t)y]; });
  r.cuts.assign((size_t)(nbands > 0 ? nbands : 0) + 1, (int)n);
  size_t i = 0;
  for (int g = 0; g <= nbands; ++g)
  {
    while (i < n && r.band[(size_t)r.order[i]] < g)
      ++i;
    r.cuts[(size_t)g] = (int)i;
  }
  return r;
}

} // namespace idx2g
