// Sharded encode with the oracle's CPU brick coder (test infrastructure): the library's shard
// plan, header payload and per-shard packing/writing (idx2_b200/csrc/shard.cpp) driven by
// tests/test_shard_cpu.py from several processes that exchange the payloads through
// torch.distributed (gloo).
#include "encoder.h"
#include "format.h"
#include "oracle_coder.h"
#include "shard.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

using namespace idx2g;

namespace
{

struct job
{
  params p;
  dataset_format f;
  encode_plan plan;
  shard_plan sp;
  std::vector<uint8_t> raw;
  std::unique_ptr<oracle_coder> coder;
  std::vector<level_output> outs;
  std::vector<uint8_t> headers;
  double vmin = 0, vmax = 0;
};

} // namespace

extern "C"
{

// Plan shard `shard` of nshards for a raw field (x fastest) and code its bricks. Returns a
// handle (null on error, *err set).
void* oshard_begin(const char* raw_path, int nx, int ny, int nz, int f32, int levels, double tol, const char* out_dir,
                   const char* name, const char* field, int shard, int nshards, int* err)
{
  std::unique_ptr<job> j(new job);
  j->p.dims = v3(nx, ny, nz);
  j->p.type = f32 ? dtype::float32 : dtype::float64;
  j->p.num_levels = levels;
  j->p.tolerance = tol;
  j->p.out_dir = out_dir;
  j->p.name = name;
  j->p.field = field;
  if (nz == 1)
    j->p.brick_dims = v3(32, 32, 1);
  *err = finalize(&j->f, &j->p);
  if (*err)
    return nullptr;
  *err = make_encode_plan(j->f, &j->plan);
  if (!*err)
    *err = make_shard_plan(j->f, j->plan, nshards, shard, &j->sp);
  if (*err)
    return nullptr;
  const size_t bytes = (size_t)nx * ny * nz * (f32 ? 4 : 8);
  j->raw.resize(bytes);
  FILE* fp = fopen(raw_path, "rb");
  if (!fp || fread(j->raw.data(), 1, bytes, fp) != bytes)
  {
    if (fp)
      fclose(fp);
    *err = FileReadFailed;
    return nullptr;
  }
  fclose(fp);
  j->coder.reset(new oracle_coder(j->f, j->raw.data()));
  *err = encode_levels(&j->f, j->coder.get(), &j->outs, j->sp.local);
  if (!*err)
    *err = shard_headers(j->f, j->plan, j->sp, j->outs, &j->headers);
  if (*err)
    return nullptr;
  j->vmin = j->f.value_min;
  j->vmax = j->f.value_max;
  return j.release();
}

size_t oshard_headers(void* h, const void** p)
{
  job* j = (job*)h;
  *p = j->headers.data();
  return j->headers.size();
}

void oshard_range(void* h, double* vmin, double* vmax)
{
  *vmin = ((job*)h)->vmin;
  *vmax = ((job*)h)->vmax;
}

void oshard_region(void* h, int* from3, int* dims3)
{
  const extent& r = ((job*)h)->sp.region;
  from3[0] = r.from.x;
  from3[1] = r.from.y;
  from3[2] = r.from.z;
  dims3[0] = r.dims.x;
  dims3[1] = r.dims.y;
  dims3[2] = r.dims.z;
}

int oshard_finish(void* h, const void* const* headers, const size_t* sizes, double vmin, double vmax)
{
  job* j = (job*)h;
  j->f.value_min = vmin;
  j->f.value_max = vmax;
  std::vector<const uint8_t*> b((size_t)j->sp.nshards);
  std::vector<size_t> n((size_t)j->sp.nshards);
  for (int s = 0; s < j->sp.nshards; ++s)
  {
    b[(size_t)s] = (const uint8_t*)headers[s];
    n[(size_t)s] = sizes[s];
  }
  return pack_shard(&j->f, &j->p, j->plan, j->sp, j->outs, b, n, nullptr);
}

void oshard_free(void* h) { delete (job*)h; }

} // extern "C"
