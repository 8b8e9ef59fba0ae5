// Test driver: prints the library's Finalize-derived tables (host format code) for
// the configurations read from stdin, one line per configuration, in the layout of
// the reference harness's ref_finalize. Built and run by tests/test_format.py.
//
// input lines:  nx ny nz dtype(0|1) bx by bz levels bricks_per_chunk chunks_per_file files_per_dir
// output lines: code nlevels gx gy gz | i32 x (40*L) | u64 x (6*L) | strings (3*L)
#include "format.h"

#include <cstdio>
#include <iostream>
#include <sstream>

using namespace idx2g;

int main()
{
  std::string line;
  while (std::getline(std::cin, line))
  {
    std::istringstream is(line);
    params p;
    int dt;
    is >> p.dims.x >> p.dims.y >> p.dims.z >> dt >> p.brick_dims.x >> p.brick_dims.y >> p.brick_dims.z >>
      p.num_levels >> p.bricks_per_chunk >> p.chunks_per_file >> p.files_per_dir;
    p.type = dt == 0 ? dtype::float32 : dtype::float64;
    p.tolerance = 1e-3;
    p.name = "kat";
    p.field = "kat";
    dataset_format f;
    int code = finalize(&f, &p);
    std::ostringstream o;
    o << code;
    if (code == 0)
    {
      int L = f.nlevels;
      o << " " << L << " " << f.group_brick3.x << " " << f.group_brick3.y << " " << f.group_brick3.z << " |";
      for (int l = 0; l < L; ++l)
      {
        int v[40] = {};
        for (int d = 0; d < 3; ++d)
        {
          v[0 + d] = f.nbricks3[l][d];
          v[3 + d] = f.bricks_per_chunk3[l][d];
          v[6 + d] = f.chunks_per_file3[l][d];
          v[9 + d] = f.nchunks3[l][d];
          v[12 + d] = f.nfiles3[l][d];
        }
        v[15] = f.bricks_per_chunk[l];
        v[16] = f.chunks_per_file[l];
        v[17] = f.bricks_per_file[l];
        v[18] = (int)f.bricks_order_str[l].size();
        v[19] = (int)f.files_dirs_depth[l].size();
        for (size_t k = 0; k < f.files_dirs_depth[l].size() && k < 4; ++k)
          v[20 + k] = f.files_dirs_depth[l][k];
        v[24] = (int)f.chunks_order_str[l].size();
        v[25] = (int)f.files_order_str[l].size();
        for (int k = 0; k < 40; ++k)
          o << " " << v[k];
      }
      o << " |";
      for (int l = 0; l < L; ++l)
        o << " " << f.bricks_order[l] << " " << f.bricks_order_in_chunk[l] << " " << f.chunks_order_in_file[l]
          << " " << f.chunks_order[l] << " " << f.files_order[l] << " " << f.transform_order;
      o << " |";
      for (int l = 0; l < L; ++l)
        o << " " << (f.bricks_order_str[l].empty() ? "-" : f.bricks_order_str[l]) << " "
          << (f.chunks_order_str[l].empty() ? "-" : f.chunks_order_str[l]) << " "
          << (f.files_order_str[l].empty() ? "-" : f.files_order_str[l]);
    }
    std::cout << o.str() << "\n";
  }
  return 0;
}
