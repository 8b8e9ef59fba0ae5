// Test driver: runs the library's encode plan and packer (host C++) with the
// oracle's CPU brick coder as the device stage, so that the packing logic can
// be compared with the reference's files on a machine without a GPU.
// Built and run by tests/test_packer_cpu.py. With ORACLE_DPACK=1 in the environment the
// regions are packed by the device packer's host stages with its kernels restated on the host
// (dpack_emul.h) instead of the host packer.
//
//   oracle_encode <raw> <nx> <ny> <nz> <float32|float64> <levels> <tol> <out_dir>
//                 <name> <field> [bx by bz] [bricks_per_chunk chunks_per_file files_per_dir]
#include "dpack.h"
#include "dpack_emul.h"
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
  const char* dp = getenv("ORACLE_DPACK");
  if (dp && dp[0] == '1')
  {
    encode_plan plan;
    e = make_encode_plan(f, &plan);
    std::vector<level_output> outs;
    if (!e)
      e = encode_levels(&f, &coder, &outs, plan);
    if (e)
    {
      fprintf(stderr, "encode error %d\n", e);
      return 10 + e;
    }
    if (!device_pack_applies(f, plan))
    {
      fprintf(stderr, "device packer not applicable\n");
      return 5;
    }
    std::vector<std::vector<int>> nexps;
    for (const level_output& o : outs)
      nexps.push_back(o.nexps);
    dpack_plan P;
    e = dpack_make_plan(f, plan, nexps, &P);
    std::vector<dpack_key> keys;
    std::vector<int> kmin;
    if (!e && emul::pack_keys(f, P, outs, &keys, &kmin))
    {
      fprintf(stderr, "device packer key window exceeded\n");
      return 6;
    }
    packed_dataset pd;
    dpack_layout L;
    if (!e)
      e = dpack_make_layout(f, P, keys, kmin, &L, &pd);
    std::vector<uint8_t> image, exps;
    if (!e)
    {
      emul::pack_write(P, outs, keys, kmin, L, &image, &exps);
      e = dpack_finish(f, P, L, image.data(), exps.data(), &pd);
    }
    if (!e)
      e = write_dataset(&f, &p, pd.files, pack_stats_text(pd.stats), nullptr, true, nullptr, nullptr, 0.0);
  }
  else
    e = encode_dataset(&f, &p, &coder, nullptr, true, nullptr);
  if (e)
  {
    fprintf(stderr, "encode error %d\n", e);
    return 10 + e;
  }
  return 0;
}
