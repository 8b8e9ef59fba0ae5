// C ABI of the library (include/idx2g.h).
#include "../../include/idx2g.h"

#include "decode_device.h"
#include "decoder.h"
#include "device.h"
#include "dpack_device.h"
#include "encoder.h"
#include "format.h"
#include "shard.h"
#include "trace.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <atomic>
#include <thread>
#include <vector>

using namespace idx2g;

struct idx2g_ctx
{
  device_ctx d;
};

namespace
{

void to_params(const idx2g_params* in, params* p)
{
  p->name = in->name;
  p->field = in->field;
  p->dims = v3(in->dims[0], in->dims[1], in->dims[2]);
  p->type = in->dtype == IDX2G_FLOAT32 ? dtype::float32 : dtype::float64;
  p->brick_dims = v3(in->brick_dims[0], in->brick_dims[1], in->brick_dims[2]);
  p->num_levels = in->num_levels;
  p->tolerance = in->tolerance;
  p->bricks_per_chunk = in->bricks_per_chunk;
  p->chunks_per_file = in->chunks_per_file;
  p->files_per_dir = in->files_per_dir;
  p->bit_planes_per_chunk = in->bit_planes_per_chunk;
  p->bit_planes_per_file = in->bit_planes_per_file;
  p->version[0] = in->version[0];
  p->version[1] = in->version[1];
  p->out_dir = in->out_dir[0] ? in->out_dir : ".";
  p->input_file = in->input_file;
  p->in_dir = in->in_dir[0] ? in->in_dir : ".";
  p->has_extent = in->has_extent != 0;
  if (p->has_extent)
  {
    v3 f(in->first[0], in->first[1], in->first[2]);
    v3 l(in->last[0], in->last[1], in->last[2]);
    p->decode_extent.from = f;
    p->decode_extent.dims = l - f + v3(1);
  }
  p->downsampling = v3(in->downsampling[0], in->downsampling[1], in->downsampling[2]);
  p->decode_tolerance = in->decode_tolerance;
}

} // namespace

extern "C"
{

IDX2G_API void idx2g_params_init(idx2g_params* p)
{
  memset(p, 0, sizeof *p);
  p->dtype = IDX2G_FLOAT64;
  p->brick_dims[0] = p->brick_dims[1] = p->brick_dims[2] = 32;
  p->bricks_per_chunk = 4096;
  p->chunks_per_file = 64;
  p->files_per_dir = 64;
  p->bit_planes_per_chunk = 1;
  p->bit_planes_per_file = 16;
  p->version[0] = 1;
  p->version[1] = 0;
  strcpy(p->out_dir, ".");
  strcpy(p->in_dir, ".");
}

IDX2G_API const char* idx2g_error_string(int code)
{
  static const char* names[] = { "NoError", "UnknownError", "SizeZero", "SizeTooSmall",
                                 "SizeMismatched", "DimensionMismatched", "DimensionsTooMany",
                                 "AttributeNotFound", "OptionNotSupported", "TypeNotSupported",
                                 "FileCreateFailed", "FileReadFailed", "FileWriteFailed",
                                 "FileOpenFailed", "FileCloseFailed", "FileSeekFailed",
                                 "FileTellFailed", "ParseFailed", "OutOfMemory", "DimensionsRepeated",
                                 "DimensionTooSmall", "BrickSizeNotPowerOfTwo", "BrickSizeTooBig",
                                 "TooManyLevels", "TooManyTransformPassesPerLevel",
                                 "TooManyLevelsOrTransformPasses", "TooManyBricksPerFile",
                                 "TooManyFilesPerDir", "NotSupportedInVersion",
                                 "CannotCreateDirectory", "SyntaxError", "TooManyBricksPerChunk",
                                 "TooManyChunksPerFile", "ChunksPerFileNotPowerOf2",
                                 "BricksPerChunkNotPowerOf2", "ChunkNotFound", "BrickNotFound",
                                 "FileNotFound", "UnsupportedScheme" };
  if (code >= 0 && code < (int)(sizeof names / sizeof names[0]))
    return names[code];
  switch (code)
  {
    case CudaError:
      return "CudaError";
    case InvalidArgument:
      return "InvalidArgument";
    case DeviceStreamOverflow:
      return "DeviceStreamOverflow";
    case CorruptStream:
      return "CorruptStream";
    case ScratchTooSmall:
      return "ScratchTooSmall";
    default:
      return "Unknown";
  }
}

IDX2G_API const char* idx2g_version(void) { return "idx2g 0.1 (sm_100a)"; }

IDX2G_API int idx2g_ctx_create(int device, void* stream, idx2g_ctx** out)
{
  if (!out)
    return InvalidArgument;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0)
    return CudaError;
  if (cudaSetDevice(device) != cudaSuccess)
    return CudaError;
  idx2g_ctx* c = new (std::nothrow) idx2g_ctx;
  if (!c)
    return OutOfMemory;
  c->d.device = device;
  cudaDeviceGetAttribute(&c->d.num_sms, cudaDevAttrMultiProcessorCount, device);
  if (stream)
  {
    c->d.stream = (cudaStream_t)stream;
    c->d.own_stream = false;
  }
  else
  {
    if (cudaStreamCreateWithFlags(&c->d.stream, cudaStreamNonBlocking) != cudaSuccess)
    {
      delete c;
      return CudaError;
    }
    c->d.own_stream = true;
  }
  cudaEventCreate(&c->d.ev0);
  cudaEventCreate(&c->d.ev1);
  // the allocation-free decode's fixed array is taken here, not at its first call
  if (noalloc_prepare(device) != NoError)
  {
    idx2g_ctx_destroy(c);
    return CudaError;
  }
  *out = c;
  return NoError;
}

IDX2G_API long long idx2g_ctx_launches(const idx2g_ctx* c) { return c ? c->d.launches : 0; }

IDX2G_API int idx2g_ctx_destroy(idx2g_ctx* c)
{
  if (!c)
    return NoError;
  cudaSetDevice(c->d.device);
  if (c->d.stream)
    cudaStreamSynchronize(c->d.stream);
  c->d.release();
  if (c->d.own_stream && c->d.stream)
    cudaStreamDestroy(c->d.stream);
  trim_dataset_pool(c->d.device);
  delete c;
  return NoError;
}

IDX2G_API int idx2g_check_params(const idx2g_params* in)
{
  if (!in)
    return InvalidArgument;
  params p;
  to_params(in, &p);
  dataset_format f;
  return finalize(&f, &p);
}

IDX2G_API int idx2g_encode(idx2g_ctx* c, const idx2g_params* in, const void* field,
                           int field_on_device, idx2g_encode_info* info)
{
  if (!c || !in || !field)
    return InvalidArgument;
  cudaSetDevice(c->d.device);
  params p;
  to_params(in, &p);
  dataset_format f;
  int e = finalize(&f, &p);
  if (e)
    return e;
  const bool f32 = p.type == dtype::float32;
  const size_t bytes = (size_t)prod(p.dims) * (f32 ? 4 : 8);
  auto t0 = std::chrono::steady_clock::now();
  const void* d_field = field;
  const void* host_field = nullptr;
  if (!field_on_device)
  {
    // the field goes to a device buffer of the context's workspace (kept across calls); from
    // pinned memory, a 3D field is copied in bands that overlap level 0's launches
    void* staged = c->d.ws("enc.field", bytes);
    if (!staged)
      return OutOfMemory;
    cudaPointerAttributes pa;
    const bool pinned = cudaPointerGetAttributes(&pa, field) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (pinned && p.dims.z > 1 && c->d.copies())
      host_field = field;
    else
      cudaMemcpyAsync(staged, field, bytes, cudaMemcpyHostToDevice, c->d.stream);
    d_field = staged;
  }
  encode_timing tm;
  long long stream_bytes = 0, exp_bytes = 0;
  double kms = 0;
  long long launches = 0;
  std::vector<float> lms;
  std::vector<long long> lbytes;
  {
    gpu_coder coder(&c->d, f, d_field, f32);
    coder.set_host_field(host_field);
    const std::shared_ptr<const encode_plan> plan = c->d.plan_for(f, &e);
    if (!plan)
      return e;
    // packed on the device where the plan allows it (every plan of the reference's brick
    // orders does); IDX2G_HOST_PACK=1 packs on the host
    static const bool host_pack = [] {
      const char* v = std::getenv("IDX2G_HOST_PACK");
      return v && v[0] == '1';
    }();
    if (!host_pack && device_pack_applies(f, *plan))
      e = encode_dataset_dpack(&c->d, &f, &p, &coder, &tm, plan, c->d.file_hint(f));
    else
      e = encode_dataset(&f, &p, &coder, nullptr, true, &tm, plan.get(), c->d.file_hint(f));
    if (!e)
      c->d.set_file_hint(f, tm.level_file_bytes);
    stream_bytes = coder.stream_bytes();
    exp_bytes = coder.exp_bytes();
    kms = coder.kernel_ms();
    launches = coder.kernel_launches();
    lms = coder.level_ms();
    lbytes = coder.level_bytes();
  }
  if (e)
    return e;
  auto t1 = std::chrono::steady_clock::now();
  (void)t0;
  (void)t1;
  if (info)
  {
    memset(info, 0, sizeof *info);
    info->kernel_ms = kms;
    info->device_s = tm.device_s;
    info->pack_s = tm.pack_s;
    info->write_s = tm.write_s;
    info->stream_bytes = stream_bytes;
    info->exp_bytes = exp_bytes;
    info->file_bytes = (long long)tm.file_bytes;
    info->kernel_launches = launches;
    info->value_min = f.value_min;
    info->value_max = f.value_max;
    info->num_levels = (int)lms.size();
    for (size_t i = 0; i < lms.size() && i < 16; ++i)
    {
      info->level_kernel_ms[i] = lms[i];
      info->level_out_bytes[i] = lbytes[i];
    }
  }
  return NoError;
}

IDX2G_API int idx2g_encode_device(idx2g_ctx* c, const idx2g_params* in, const void* d_field,
                                  idx2g_encode_info* info)
{
  if (!c || !in || !d_field)
    return InvalidArgument;
  cudaSetDevice(c->d.device);
  params p;
  to_params(in, &p);
  dataset_format f;
  int e = finalize(&f, &p);
  if (e)
    return e;
  gpu_coder coder(&c->d, f, d_field, p.type == dtype::float32);
  coder.set_keep_device(true);
  std::vector<level_output> outs;
  auto t0 = std::chrono::steady_clock::now();
  const std::shared_ptr<const encode_plan> plan = c->d.plan_for(f, &e);
  if (!plan)
    return e;
  e = encode_levels(&f, &coder, &outs, *plan);
  auto t1 = std::chrono::steady_clock::now();
  if (e)
    return e;
  if (info)
  {
    memset(info, 0, sizeof *info);
    info->kernel_ms = coder.kernel_ms();
    info->device_s = std::chrono::duration<double>(t1 - t0).count();
    info->stream_bytes = coder.stream_bytes();
    info->exp_bytes = coder.exp_bytes();
    info->kernel_launches = coder.kernel_launches();
    info->value_min = f.value_min;
    info->value_max = f.value_max;
    info->num_levels = (int)coder.level_ms().size();
    for (size_t i = 0; i < coder.level_ms().size() && i < 16; ++i)
    {
      info->level_kernel_ms[i] = coder.level_ms()[i];
      info->level_out_bytes[i] = coder.level_bytes()[i];
    }
  }
  return NoError;
}

namespace
{

// A sharded encode between idx2g_encode_shard and idx2g_encode_shard_finish.
struct shard_job
{
  params p;
  dataset_format f;
  std::shared_ptr<const encode_plan> plan;
  shard_plan sp;
  std::unique_ptr<gpu_coder> coder;
  std::vector<level_output> outs;
  std::vector<uint8_t> headers;
  double device_s = 0;
};

int shard_setup(const idx2g_params* in, int shard, int nshards, params* p, dataset_format* f,
                encode_plan* own_plan, shard_plan* sp)
{
  to_params(in, p);
  int e = finalize(f, p);
  if (e)
    return e;
  e = make_encode_plan(*f, own_plan);
  if (e)
    return e;
  return make_shard_plan(*f, *own_plan, nshards, shard, sp);
}

} // namespace

IDX2G_API int idx2g_shard_region(const idx2g_params* in, int shard, int nshards, int from3[3], int dims3[3])
{
  if (!in || !from3 || !dims3)
    return InvalidArgument;
  params p;
  dataset_format f;
  encode_plan plan;
  shard_plan sp;
  int e = shard_setup(in, shard, nshards, &p, &f, &plan, &sp);
  if (e)
    return e;
  for (int k = 0; k < 3; ++k)
  {
    from3[k] = k == 0 ? sp.region.from.x : k == 1 ? sp.region.from.y : sp.region.from.z;
    dims3[k] = k == 0 ? sp.region.dims.x : k == 1 ? sp.region.dims.y : sp.region.dims.z;
  }
  return NoError;
}

IDX2G_API int idx2g_encode_shard(idx2g_ctx* c, const idx2g_params* in, const void* d_field, const int origin3[3],
                                 const int dims3[3], int shard, int nshards, int flags, const void** headers,
                                 size_t* header_bytes, double* vmin, double* vmax, idx2g_encode_info* info)
{
  const bool device_only = (flags & IDX2G_SHARD_DEVICE_ONLY) != 0;
  if (!c || !in || !d_field || !origin3 || !dims3 || (!device_only && (!headers || !header_bytes)))
    return InvalidArgument;
  cudaSetDevice(c->d.device);
  c->d.shard.reset();
  auto job = std::make_shared<shard_job>();
  to_params(in, &job->p);
  int e = finalize(&job->f, &job->p);
  if (e)
    return e;
  job->plan = c->d.plan_for(job->f, &e);
  if (!job->plan)
    return e;
  e = make_shard_plan(job->f, *job->plan, nshards, shard, &job->sp);
  if (e)
    return e;
  // the buffer must hold the shard's region, from a brick-aligned origin
  const v3 o(origin3[0], origin3[1], origin3[2]), d(dims3[0], dims3[1], dims3[2]);
  const extent& r = job->sp.region;
  const v3 bd = job->f.brick_dims;
  if (o.x % bd.x || o.y % bd.y || o.z % bd.z || o.x > r.from.x || o.y > r.from.y || o.z > r.from.z ||
      o.x + d.x < r.from.x + r.dims.x || o.y + d.y < r.from.y + r.dims.y || o.z + d.z < r.from.z + r.dims.z)
    return InvalidArgument;
  job->coder.reset(new gpu_coder(&c->d, job->f, d_field, job->p.type == dtype::float32));
  job->coder->set_field_region(o, d);
  job->coder->set_keep_device(device_only);
  const auto t0 = std::chrono::steady_clock::now();
  e = encode_levels(&job->f, job->coder.get(), &job->outs, job->sp.local);
  if (e)
    return e;
  job->device_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (!device_only)
  {
    e = shard_headers(job->f, *job->plan, job->sp, job->outs, &job->headers);
    if (e)
      return e;
    *headers = job->headers.data();
    *header_bytes = job->headers.size();
  }
  if (vmin)
    *vmin = job->f.value_min;
  if (vmax)
    *vmax = job->f.value_max;
  if (info)
  {
    memset(info, 0, sizeof *info);
    info->kernel_ms = job->coder->kernel_ms();
    info->device_s = job->device_s;
    info->stream_bytes = job->coder->stream_bytes();
    info->exp_bytes = job->coder->exp_bytes();
    info->kernel_launches = job->coder->kernel_launches();
    info->value_min = job->f.value_min;
    info->value_max = job->f.value_max;
    info->num_levels = (int)job->coder->level_ms().size();
    for (size_t i = 0; i < job->coder->level_ms().size() && i < 16; ++i)
    {
      info->level_kernel_ms[i] = job->coder->level_ms()[i];
      info->level_out_bytes[i] = job->coder->level_bytes()[i];
    }
  }
  if (!device_only)
    c->d.shard = job;
  return NoError;
}

IDX2G_API int idx2g_encode_shard_finish(idx2g_ctx* c, const idx2g_params* in, int shard, int nshards,
                                        const void* const* headers, const size_t* header_bytes, double vmin,
                                        double vmax, idx2g_encode_info* info)
{
  if (!c || !in || !headers || !header_bytes)
    return InvalidArgument;
  std::shared_ptr<shard_job> job = std::static_pointer_cast<shard_job>(c->d.shard);
  if (!job || job->sp.shard != shard || job->sp.nshards != nshards)
    return InvalidArgument;  // no idx2g_encode_shard of this shard before
  c->d.shard.reset();
  job->f.value_min = vmin;
  job->f.value_max = vmax;
  std::vector<const uint8_t*> blobs((size_t)nshards);
  std::vector<size_t> sizes((size_t)nshards);
  for (int s = 0; s < nshards; ++s)
  {
    blobs[(size_t)s] = (const uint8_t*)headers[s];
    sizes[(size_t)s] = header_bytes[s];
  }
  encode_timing tm;
  const int e = pack_shard(&job->f, &job->p, *job->plan, job->sp, job->outs, blobs, sizes, &tm);
  if (info)
  {
    info->pack_s = tm.pack_s;
    info->write_s = tm.write_s;
    info->file_bytes = (long long)tm.file_bytes;
  }
  return e;
}

IDX2G_API int idx2g_encode_batch(idx2g_ctx* c, const idx2g_params* in, const void* const* fields, int n,
                                 int fields_on_device, int flags, idx2g_encode_info* infos)
{
  if (!c || !in || !fields || n < 0)
    return InvalidArgument;
  if (n == 0)
    return NoError;
  cudaSetDevice(c->d.device);
  cudaStream_t st = c->d.stream;
  const auto t0 = std::chrono::steady_clock::now();
  stage_timer tt;
  std::vector<params> ps((size_t)n);
  std::vector<dataset_format> fs((size_t)n);
  std::vector<std::shared_ptr<const encode_plan>> plans((size_t)n);  // held for the whole call
  std::vector<std::vector<level_output>> outs((size_t)n);
  size_t host_bytes = 0;
  long long total_bricks = 0;
  int nf64 = 0;
  for (int i = 0; i < n; ++i)
  {
    if (!fields[i])
      return InvalidArgument;
    to_params(in + i, &ps[(size_t)i]);
    int e = finalize(&fs[(size_t)i], &ps[(size_t)i]);
    if (e)
      return e;
    plans[(size_t)i] = c->d.plan_for(fs[(size_t)i], &e);
    if (!plans[(size_t)i])
      return e;
    host_bytes += (((size_t)prod(ps[(size_t)i].dims) * (ps[(size_t)i].type == dtype::float32 ? 4 : 8)) + 255) &
                  ~(size_t)255;
    total_bricks += (long long)plans[(size_t)i]->levels[0].size();
    nf64 += ps[(size_t)i].type == dtype::float64;
  }
  tt.lap("batch.plans");
  // fields to the device (one staging buffer of the context's workspace)
  std::vector<const void*> dptr((size_t)n);
  if (!fields_on_device)
  {
    uint8_t* staged = (uint8_t*)c->d.ws("enc.batchfields", host_bytes);
    if (!staged)
      return OutOfMemory;
    size_t at = 0;
    for (int i = 0; i < n; ++i)
    {
      const size_t b = (size_t)prod(ps[(size_t)i].dims) * (ps[(size_t)i].type == dtype::float32 ? 4 : 8);
      cudaMemcpyAsync(staged + at, fields[i], b, cudaMemcpyHostToDevice, st);
      dptr[(size_t)i] = staged + at;
      at += (b + 255) & ~(size_t)255;
    }
  }
  else
    for (int i = 0; i < n; ++i)
      dptr[(size_t)i] = fields[i];
  std::vector<batch_field> bf((size_t)n);
  for (int i = 0; i < n; ++i)
  {
    bf[(size_t)i].f = &fs[(size_t)i];
    bf[(size_t)i].plan = plans[(size_t)i].get();
    bf[(size_t)i].d_field = dptr[(size_t)i];
    bf[(size_t)i].f32 = ps[(size_t)i].type == dtype::float32;
    bf[(size_t)i].outs = &outs[(size_t)i];
  }
  const bool graph = (flags & IDX2G_BATCH_GRAPH) != 0;
  const bool device_only = (flags & IDX2G_BATCH_DEVICE_ONLY) != 0;
  batch_tuning tune;
  if (flags & IDX2G_BATCH_AUTOTUNE)
  {
    // the launch shape is timed once per batch signature and remembered by the context
    char key[96];
    snprintf(key, sizeof key, "%d/%lld/%d", n, total_bricks, nf64);
    auto it = c->d.tuned.find(key);
    if (it == c->d.tuned.end())
    {
      // candidates: the global-slot kernel at 1 CTA per SM and at as many as can reside, and
      // the 3D bricks in shared memory over CTA pairs (the 2D bricks then on the slot kernel)
      const batch_tuning cands[3] = { { 1, 0 }, { 0, 0 }, { 0, 1 } };
      double best = 1e300;
      int best_code = 0;
      for (const batch_tuning& cand : cands)
      {
        if (cand.split == 1 && !split_kernel_available())
          continue;
        std::vector<batch_field> trial = bf;
        std::vector<std::vector<level_output>> touts((size_t)n);
        for (int i = 0; i < n; ++i)
          trial[(size_t)i].outs = &touts[(size_t)i];
        batch_encoder te(&c->d, &trial, "b");
        int e = te.prepare(cand);
        if (!e)
          e = te.run_all(graph, true);
        if (e)
          return e;
        if (te.kernel_ms() < best)
        {
          best = te.kernel_ms();
          best_code = cand.ctas_per_sm + 10 * cand.split;
        }
      }
      it = c->d.tuned.emplace(key, best_code).first;
    }
    tune.ctas_per_sm = it->second % 10;
    tune.split = it->second / 10;
  }
  tt.lap("batch.tune");
  batch_encoder enc(&c->d, &bf, "b");
  int e = enc.prepare(tune);
  tt.lap("batch.prepare");
  if (!e)
    e = enc.run_all(graph, device_only);
  if (e)
    return e;
  tt.lap("batch.run");
  const auto t1 = std::chrono::steady_clock::now();
  for (int i = 0; i < n; ++i)
  {
    fs[(size_t)i].value_min = bf[(size_t)i].vmin;
    fs[(size_t)i].value_max = bf[(size_t)i].vmax;
  }
  std::vector<encode_timing> tm((size_t)n);
  if (!device_only)
  {
    // packing and files, several fields at a time
    std::atomic<int> next{ 0 }, err{ 0 };
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt ? (nt > 16 ? 16 : nt) : 4;
    if ((int)nt > n)
      nt = (unsigned)n;
    auto work = [&]() {
      for (int i; (i = next.fetch_add(1)) < n;)
      {
        const int r = pack_dataset(&fs[(size_t)i], &ps[(size_t)i], *plans[(size_t)i], outs[(size_t)i], nullptr,
                                   true, &tm[(size_t)i]);
        if (r)
          err = r;
      }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t)
      th.emplace_back(work);
    work();
    for (auto& t : th)
      t.join();
    if (err)
      return err;
  }
  if (infos)
  {
    const double dev_s = std::chrono::duration<double>(t1 - t0).count();
    for (int i = 0; i < n; ++i)
    {
      idx2g_encode_info* info = infos + i;
      memset(info, 0, sizeof *info);
      info->kernel_ms = enc.kernel_ms();
      info->device_s = dev_s;
      info->pack_s = tm[(size_t)i].pack_s;
      info->write_s = tm[(size_t)i].write_s;
      info->exp_bytes = bf[(size_t)i].exp_bytes;
      info->file_bytes = (long long)tm[(size_t)i].file_bytes;
      info->kernel_launches = enc.launches();
      info->value_min = fs[(size_t)i].value_min;
      info->value_max = fs[(size_t)i].value_max;
      info->num_levels = fs[(size_t)i].nlevels;
    }
  }
  return NoError;
}

IDX2G_API int idx2g_dataset_open(idx2g_ctx* c, const idx2g_params* in, idx2g_dataset** ds)
{
  if (!c || !in || !ds)
    return InvalidArgument;
  params p;
  to_params(in, &p);
  return dataset_open(&c->d, p, (dataset_handle**)ds);
}

IDX2G_API int idx2g_output_grid(const idx2g_dataset* ds, const idx2g_params* in, int from3[3],
                                int dims3[3], int strd3[3])
{
  if (!ds || !in)
    return InvalidArgument;
  params p;
  to_params(in, &p);
  grid g;
  int e = dataset_output_grid((const dataset_handle*)ds, p, &g);
  if (e)
    return e;
  for (int d = 0; d < 3; ++d)
  {
    from3[d] = g.from[d];
    dims3[d] = g.dims[d];
    strd3[d] = g.strd[d];
  }
  return NoError;
}

IDX2G_API int idx2g_decode(idx2g_ctx* c, idx2g_dataset* ds, const idx2g_params* in, void* out,
                           size_t out_bytes, int out_on_device, double* kernel_ms)
{
  if (!c || !ds || !in || !out)
    return InvalidArgument;
  params p;
  to_params(in, &p);
  return dataset_decode(&c->d, (dataset_handle*)ds, p, out, out_bytes, out_on_device != 0, kernel_ms);
}

IDX2G_API int idx2g_decode_batch(idx2g_ctx* c, idx2g_dataset* ds, const idx2g_params* in, int n,
                                 void* const* outs, const size_t* out_bytes, int out_on_device, double* kernel_ms)
{
  if (!c || !ds || !in || !outs || !out_bytes || n < 0)
    return InvalidArgument;
  std::vector<params> ps((size_t)n);
  for (int i = 0; i < n; ++i)
  {
    if (!outs[i])
      return InvalidArgument;
    to_params(in + i, &ps[(size_t)i]);
  }
  return dataset_decode_batch(&c->d, (dataset_handle*)ds, ps.data(), n, outs, out_bytes, out_on_device != 0,
                              kernel_ms);
}

IDX2G_API long long idx2g_coeff_count(const idx2g_params* in)
{
  if (!in)
    return -1;
  params p;
  to_params(in, &p);
  dataset_format f;
  if (finalize(&f, &p))
    return -1;
  return synth_coeff_count(f);
}

IDX2G_API int idx2g_decode_brick_map(idx2g_ctx* c, idx2g_dataset* ds, const idx2g_params* in, const char* path,
                                     double* kernel_ms)
{
  if (!c || !ds || !in || !path)
    return InvalidArgument;
  params p;
  to_params(in, &p);
  return dataset_decode_brick_map(&c->d, (dataset_handle*)ds, p, path, kernel_ms);
}

IDX2G_API int idx2g_coeffs(idx2g_ctx* c, idx2g_dataset* ds, const idx2g_params* in, void* d_coeffs, size_t bytes,
                           double* kernel_ms)
{
  if (!c || !ds || !in || !d_coeffs)
    return InvalidArgument;
  params p;
  to_params(in, &p);
  return dataset_coeffs(&c->d, (dataset_handle*)ds, p, d_coeffs, bytes, kernel_ms);
}

static int synth_call(idx2g_ctx* c, const idx2g_params* in, int nbatch, const void* src, void* dst, bool adjoint,
                      double* kernel_ms)
{
  if (!c || !in || !src || !dst || nbatch < 1)
    return InvalidArgument;
  params p;
  to_params(in, &p);
  dataset_format f;
  int e = finalize(&f, &p);
  if (e)
    return e;
  return synth(&c->d, f, nbatch, src, dst, adjoint, kernel_ms);
}

IDX2G_API int idx2g_synth(idx2g_ctx* c, const idx2g_params* in, int nbatch, const void* d_coeffs, void* d_grid,
                          double* kernel_ms)
{
  return synth_call(c, in, nbatch, d_coeffs, d_grid, false, kernel_ms);
}

IDX2G_API int idx2g_synth_adjoint(idx2g_ctx* c, const idx2g_params* in, int nbatch, const void* d_grid_grad,
                                  void* d_coeff_grad, double* kernel_ms)
{
  return synth_call(c, in, nbatch, d_grid_grad, d_coeff_grad, true, kernel_ms);
}

// Allocation-free decode (include/idx2g.h): for callers that cannot allocate device memory at
// decode time; all temporaries are in the fixed scratch array of decode.cu.
IDX2G_API int idx2g_decode_noalloc(idx2g_ctx* c, idx2g_dataset* ds, const idx2g_params* in, void* d_out,
                                   size_t out_bytes, double* kernel_ms)
{
  if (!c || !ds || !in || !d_out)
    return InvalidArgument;
  params p;
  to_params(in, &p);
  return dataset_decode_noalloc(&c->d, (dataset_handle*)ds, p, d_out, out_bytes, kernel_ms);
}

IDX2G_API int idx2g_dataset_close(idx2g_dataset* ds)
{
  dataset_close((dataset_handle*)ds);
  return NoError;
}

IDX2G_API int idx2g_dataset_info(const idx2g_dataset* ds, char* name, char* field, int dims3[3],
                                 int* dt, int* num_levels, double* tolerance, long long* resident)
{
  if (!ds)
    return InvalidArgument;
  const dataset_format& f = dataset_fmt((const dataset_handle*)ds);
  if (name)
    snprintf(name, 64, "%s", f.name.c_str());
  if (field)
    snprintf(field, 64, "%s", f.field.c_str());
  if (dims3)
  {
    dims3[0] = f.dims.x;
    dims3[1] = f.dims.y;
    dims3[2] = f.dims.z;
  }
  if (dt)
    *dt = f.type == dtype::float32 ? IDX2G_FLOAT32 : IDX2G_FLOAT64;
  if (num_levels)
    *num_levels = f.nlevels;
  if (tolerance)
    *tolerance = f.tolerance;
  if (resident)
    *resident = (long long)dataset_resident_bytes((const dataset_handle*)ds);
  return NoError;
}

} // extern "C"
