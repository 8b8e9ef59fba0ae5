// Test driver: runs the library's encode plan and packer (host C++) with the
// oracle's CPU brick coder as the device stage, so that the packing logic can
// be compared with the reference's files on a machine without a GPU.
// Built and run by tests/test_packer_cpu.py.
//
//   oracle_encode <raw> <nx> <ny> <nz> <float32|float64> <levels> <tol> <out_dir>
//                 <name> <field> [bx by bz] [bricks_per_chunk chunks_per_file files_per_dir]
#include "encoder.h"
#include "format.h"
#include "oracle_coder.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace idx2g;

int main(int argc, char** argv)
{
  if (argc < 11)
  {
    fprintf(stderr, "usage: oracle_encode raw nx ny nz dtype levels tol out_dir name field [bx by bz] "
                    "[bricks_per_chunk chunks_per_file files_per_dir]\n");
    return 2;
  }
  params p;
  p.dims = v3(atoi(argv[2]), atoi(argv[3]), atoi(argv[4]));
  p.type = strcmp(argv[5], "float32") == 0 ? dtype::float32 : dtype::float64;
  p.num_levels = atoi(argv[6]);
  p.tolerance = atof(argv[7]);
  p.out_dir = argv[8];
  p.name = argv[9];
  p.field = argv[10];
  if (argc >= 14)
    p.brick_dims = v3(atoi(argv[11]), atoi(argv[12]), atoi(argv[13]));
  if (argc >= 17)
  {
    p.bricks_per_chunk = atoi(argv[14]);
    p.chunks_per_file = atoi(argv[15]);
    p.files_per_dir = atoi(argv[16]);
  }
  dataset_format f;
  int e = finalize(&f, &p);
  if (e)
  {
    fprintf(stderr, "finalize error %d\n", e);
    return 10 + e;
  }
  size_t n = (size_t)prod(p.dims);
  size_t es = p.type == dtype::float32 ? 4 : 8;
  std::vector<uint8_t> raw(n * es);
  FILE* fp = fopen(argv[1], "rb");
  if (!fp || fread(raw.data(), 1, raw.size(), fp) != raw.size())
  {
    fprintf(stderr, "cannot read %s\n", argv[1]);
    return 3;
  }
  fclose(fp);
  oracle_coder coder(f, raw.data());
  e = encode_dataset(&f, &p, &coder, nullptr, true, nullptr);
  if (e)
  {
    fprintf(stderr, "encode error %d\n", e);
    return 10 + e;
  }
  return 0;
}
