// Test driver: the table form of the linear brick index (format.h brick_linearizer) against
// linear_brick for every brick of every level, and for coordinates past the tables, of the
// configurations read from stdin (nx ny nz bx by bz levels per line). Prints one line per
// configuration: "ok <bricks checked>" or "FAIL <level> <x> <y> <z>".
#include "format.h"

#include <cstdio>
#include <iostream>
#include <sstream>

using namespace idx2g;

int main()
{
  std::string line;
  int fails = 0;
  while (std::getline(std::cin, line))
  {
    std::istringstream is(line);
    params p;
    is >> p.dims.x >> p.dims.y >> p.dims.z >> p.brick_dims.x >> p.brick_dims.y >> p.brick_dims.z >> p.num_levels;
    p.type = dtype::float32;
    p.tolerance = 1e-3;
    p.name = "kat";
    p.field = "kat";
    dataset_format f;
    if (finalize(&f, &p) != 0)
    {
      std::printf("FAIL finalize\n");
      ++fails;
      continue;
    }
    long long n = 0;
    bool ok = true;
    for (int l = 0; l < f.nlevels && ok; ++l)
    {
      const v3 nb = f.nbricks3[(size_t)l];
      const brick_linearizer lin(f, l, nb);
      for (int z = 0; z <= nb.z && ok; ++z)  // (one past the tables on each axis)
        for (int y = 0; y <= nb.y && ok; ++y)
          for (int x = 0; x <= nb.x && ok; ++x)
          {
            const v3 b(x, y, z);
            ++n;
            if (lin(b) != linear_brick(f, l, b))
            {
              std::printf("FAIL %d %d %d %d\n", l, x, y, z);
              ok = false;
              ++fails;
            }
          }
    }
    if (ok)
      std::printf("ok %lld\n", n);
  }
  return fails;
}
