// CUDA context and the device stages of the encoder / decoder.
#pragma once

#include "encoder.h"

#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace idx2g
{

// One context per thread; all work is ordered on `stream`. The context owns a
// grow-only workspace of named device buffers reused across calls, so repeated
// encodes / decodes do not allocate.
struct device_ctx
{
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> evpool;  // timing events of calls that time several launches
  // streams for host copies that overlap the kernels of `stream`, one per direction (created
  // on first use)
  cudaStream_t copy_stream = nullptr, copy_out_stream = nullptr;
  cudaStream_t copies()
  {
    if (!copy_stream && cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking) != cudaSuccess)
      copy_stream = nullptr;
    return copy_stream;
  }
  cudaStream_t copies_out()
  {
    if (!copy_out_stream && cudaStreamCreateWithFlags(&copy_out_stream, cudaStreamNonBlocking) != cudaSuccess)
      copy_out_stream = nullptr;
    return copy_out_stream;
  }
  long long launches = 0;  // kernels launched on this context so far
  // batched encode: the launch shape chosen per batch signature (CTAs per SM + 10 * split kernel)
  std::map<std::string, int> tuned;
  std::shared_ptr<void> shard;       // a sharded encode between its two calls (api.cpp)
  std::shared_ptr<void> dpack;       // the device packer's tables of the last plan (dpack_host.cpp)
  // instantiated CUDA graphs of batched encodes, by batch tag: the launches they were captured
  // from (a byte image of every launch's arguments) and the executable graph
  struct cached_graph
  {
    std::string launches;            // signature of the captured launches
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;           // kernels the graph launches
  };
  std::map<std::string, cached_graph> graphs;
  // Encode plans by format: the brick order and the EncodeSubband events depend only on the
  // dims, the brick dims and the number of levels, so repeated encodes of fields of one shape
  // (the time steps of a simulation) plan once.
  // Callers hold the returned pointer for as long as they use the plan: the cache keeps the
  // plans of the last shapes up to 256 MB of plan tables (IDX2G_PLAN_CACHE_MB overrides it; a
  // batch of many small shapes, or a few 1024^3 ones) and may drop one while an earlier
  // holder still uses it.
  std::map<std::string, std::shared_ptr<const encode_plan>> plans;
  std::vector<std::string> plan_order;  // keys, oldest first
  size_t plan_bytes = 0;
  static size_t plan_size(const encode_plan& p)
  {
    size_t b = p.events.size() * sizeof(encode_event) + 256;
    for (const auto& l : p.levels)
      b += l.size() * sizeof(brick_entry);
    return b;
  }
  static std::string plan_key(const dataset_format& f)
  {
    char key[128];
    snprintf(key, sizeof key, "%d %d %d/%d %d %d/%d", f.dims.x, f.dims.y, f.dims.z, f.brick_dims.x, f.brick_dims.y,
             f.brick_dims.z, f.nlevels);
    return key;
  }
  std::shared_ptr<const encode_plan> plan_for(const dataset_format& f, int* err)
  {
    const std::string key = plan_key(f);
    auto it = plans.find(key);
    if (it != plans.end())
      return it->second;
    std::shared_ptr<encode_plan> pl = std::make_shared<encode_plan>();
    *err = make_encode_plan(f, pl.get());
    if (*err)
      return nullptr;
    const size_t sz = plan_size(*pl);
    const char* mb = std::getenv("IDX2G_PLAN_CACHE_MB");
    const size_t kBudget = (mb ? (size_t)std::strtoull(mb, nullptr, 10) : (size_t)256) << 20;
    size_t drop = 0;
    while (drop < plan_order.size() && plan_bytes + sz > kBudget)
    {
      auto old = plans.find(plan_order[drop]);
      if (old != plans.end())
      {
        plan_bytes -= plan_size(*old->second);
        plans.erase(old);
      }
      ++drop;
    }
    plan_order.erase(plan_order.begin(), plan_order.begin() + (long)drop);
    plans[key] = pl;
    plan_order.push_back(key);
    plan_bytes += sz;
    return pl;
  }
  // Bytes of each level's data file in the last encode of a shape (by plan_key): the next
  // encode of that shape has the file system allocate about as many pages while its device
  // stage runs (a guess only: the writer sets every file's size and writes every byte).
  std::map<std::string, std::vector<unsigned long long>> file_hints;
  const std::vector<unsigned long long>* file_hint(const dataset_format& f)
  {
    auto it = file_hints.find(plan_key(f));
    return it == file_hints.end() ? nullptr : &it->second;
  }
  void set_file_hint(const dataset_format& f, const std::vector<unsigned long long>& sizes)
  {
    const std::string key = plan_key(f);
    if (sizes.empty())
    {
      file_hints.erase(key);
      return;
    }
    if (file_hints.size() >= 16 && !file_hints.count(key))
      file_hints.erase(file_hints.begin());
    file_hints[key] = sizes;
  }

  struct buf
  {
    void* p = nullptr;
    size_t n = 0;
    size_t dirty = 0;  // bytes that may be non-zero (for ws_zeroed)
  };
  std::map<std::string, buf> bufs;

  // Buffer of at least `bytes` bytes (contents unspecified).
  void* ws(const std::string& name, size_t bytes)
  {
    buf& b = bufs[name];
    if (b.n < bytes || !b.p)
    {
      // a buffer that has to grow again grows by half at least, so a run of growing requests
      // (serving batches of rising size) reallocates a logarithmic number of times
      size_t want = bytes + bytes / 8 + 256;
      if (b.n && want < b.n + b.n / 2)
        want = b.n + b.n / 2;
      if (b.p)
        cudaFree(b.p);
      b.p = nullptr;
      b.n = 0;
      if (cudaMalloc(&b.p, want) != cudaSuccess)
        return nullptr;
      b.n = want;
      b.dirty = want;
    }
    return b.p;
  }
  // Buffer of at least `bytes` bytes, all zero (only the previously used prefix is cleared).
  void* ws_zeroed(const std::string& name, size_t bytes)
  {
    void* p = ws(name, bytes);
    if (!p)
      return nullptr;
    buf& b = bufs[name];
    if (b.dirty)
      cudaMemsetAsync(b.p, 0, b.dirty, stream);
    b.dirty = 0;
    return p;
  }
  size_t ws_size(const std::string& name)
  {
    auto it = bufs.find(name);
    return it == bufs.end() ? 0 : it->second.n;
  }
  void ws_mark_dirty(const std::string& name, size_t bytes)
  {
    buf& b = bufs[name];
    size_t d = bytes + 64 < b.n ? bytes + 64 : b.n;
    if (d > b.dirty)
      b.dirty = d;
  }
  // Pinned host buffer of at least `bytes` bytes (grow-only, kept across calls).
  std::map<std::string, buf> pins;
  size_t pinned_size(const std::string& name)
  {
    auto it = pins.find(name);
    return it == pins.end() ? 0 : it->second.n;
  }
  void* pinned(const std::string& name, size_t bytes)
  {
    buf& b = pins[name];
    if (b.n < bytes || !b.p)
    {
      if (b.p)
        cudaFreeHost(b.p);
      b.p = nullptr;
      b.n = 0;
      size_t want = bytes + bytes / 4 + 4096;
      if (cudaMallocHost(&b.p, want) != cudaSuccess)
        return nullptr;
      b.n = want;
    }
    return b.p;
  }
  // Timing event i of the pool (created on first use), or null.
  cudaEvent_t ev(size_t i)
  {
    while (evpool.size() <= i)
    {
      cudaEvent_t e = nullptr;
      if (cudaEventCreate(&e) != cudaSuccess)
        return nullptr;
      evpool.push_back(e);
    }
    return evpool[i];
  }
  void release()
  {
    for (auto& kv : graphs)
      if (kv.second.exec)
        cudaGraphExecDestroy(kv.second.exec);
    graphs.clear();
    for (cudaStream_t* s : { &copy_stream, &copy_out_stream })
      if (*s)
      {
        cudaStreamSynchronize(*s);
        cudaStreamDestroy(*s);
        *s = nullptr;
      }
    for (cudaEvent_t e : evpool)
      cudaEventDestroy(e);
    evpool.clear();
    for (auto& kv : bufs)
      if (kv.second.p)
        cudaFree(kv.second.p);
    bufs.clear();
    for (auto& kv : pins)
      if (kv.second.p)
        cudaFreeHost(kv.second.p);
    pins.clear();
    if (ev0)
      cudaEventDestroy(ev0);
    if (ev1)
      cudaEventDestroy(ev1);
    ev0 = ev1 = nullptr;
  }
};

// Waits for a stream when it goes out of scope: a call that has copies of a caller's host
// buffer in flight on a side stream returns only after them, on its error paths too.
struct stream_fence
{
  cudaStream_t s = nullptr;
  ~stream_fence()
  {
    if (s)
      cudaStreamSynchronize(s);
  }
};

// One field of a device encode (a launch may cover the bricks of many fields).
struct batch_field
{
  const dataset_format* f = nullptr;
  const encode_plan* plan = nullptr;
  const void* d_field = nullptr;  // device pointer
  bool f32 = true;
  // the samples d_field holds: [field_origin, field_origin + field_dims) of the dataset
  // (field_dims 0: the whole dataset); the origin is a multiple of the brick size
  v3 field_origin, field_dims;
  std::vector<level_output>* outs = nullptr;  // receives one entry per level
  double vmin = 1.7976931348623157e308, vmax = -1.7976931348623157e308;
  long long stream_bytes = 0, exp_bytes = 0;
  std::vector<float> level_ms;
  std::vector<long long> level_bytes;
};

// Launch shape of the device encode.
struct batch_tuning
{
  int ctas_per_sm = 0;  // global-slot kernel: CTAs per SM, 0 as many as can reside
  // 3D bricks in shared memory over 2-CTA clusters (k_encode_split): 1 on, 0 off, -1 the
  // library's default; the environment variable IDX2G_ENC_SPLIT (0 or 1) overrides either
  int split = -1;
};

// Whether the split encode kernel (3D bricks in shared memory over CTA pairs) can be offered to
// the batch tuner on this device (encode.cu).
bool split_kernel_available();

// The device stage for a set of fields: per level, one launch of the encode kernel over the
// bricks of every field that has the level. Levels can be enqueued one by one (with the
// results read back after each), or all at once, optionally captured in a CUDA graph.
class batch_encoder
{
public:
  batch_encoder(device_ctx* ctx, std::vector<batch_field>* fields, const std::string& tag);
  ~batch_encoder();
  int prepare(const batch_tuning& t);
  int nlevels() const { return (int)levels_.size(); }
  int enqueue_level(int l);
  // Level 0 of one 3D field whose samples are in pinned host memory: bands of brick rows are
  // copied to `staged` on the context's copy stream, each band's launch waits for its copy
  // only. *nbands: launches made (timed by event pairs 2g, 2g + 1 of the context's pool).
  // The coarser levels go in bands as well, between level 0's: a brick as soon as the band
  // holding the last of its children has run (levels that are launched so: followed()).
  int enqueue_level0_streamed(const void* host, void* staged, int* nbands);
  // Whether level l was launched with level 0's bands, and its launches' time once they ran.
  bool followed(int l) const { return l > 0 && (size_t)l < follow_events_.size() && !follow_events_[(size_t)l].empty(); }
  float followed_ms(int l) const;
  // While the bands of enqueue_level0_streamed run: as each band ends, its stream bytes go to
  // the level's pinned host buffer on the copy-out stream (when the buffer is already large
  // enough), so that collect_level finds them there.
  void stream_out_level0(int nbands);
  // Wait for level l, relaunch it with more room if its streams overflowed, read back the
  // region offsets and streams (unless keep_device) into the fields' level outputs.
  int collect_level(int l, bool keep_device);
  // Every level: enqueued back to back (in one CUDA graph if use_graph), then collected.
  int run_all(bool use_graph, bool keep_device);
  double kernel_ms() const { return kernel_ms_; }
  void add_kernel_ms(double ms) { kernel_ms_ += ms; }
  long long launches() const { return launches_; }
  // A collected level's regions on the device (one field's batch): stream and region offsets
  // (index brick * 8 + subband), valid while the encoder and its context's workspaces live.
  void device_level(int l, const uint8_t** stream, const unsigned long long** offset) const;
  // A level collected with keep_device: its offsets and streams read back into o (one
  // field's batch), as collect_level does without keep_device.
  int copy_level_out(int l, level_output* o);

  struct level_launch;

private:
  device_ctx* ctx_;
  std::vector<batch_field>* fields_;
  std::string tag_;
  batch_tuning tune_;
  std::vector<std::unique_ptr<level_launch>> levels_;
  std::vector<std::vector<int>> follow_events_;  // per level: event pairs of its band launches
  double kernel_ms_ = 0;
  long long launches_ = 0;
  long long graph_launches_ = 0;  // kernels in the cached graph of this batch's launches
};

// Device brick coder for one field (brick_coder interface): a batch of one.
class gpu_coder : public brick_coder
{
public:
  gpu_coder(device_ctx* ctx, const dataset_format& f, const void* d_field, bool field_f32);
  ~gpu_coder() override;
  int run_level(int level, const encode_plan& plan, level_output* out) override;
  void value_range(double* vmin, double* vmax) override;
  // Leave the coder output on the device (no copies for the packer).
  void set_keep_device(bool v) { keep_device_ = v; }
  // The field's samples are in pinned host memory `host`; d_field (given at construction) is
  // the device buffer they go to, copied while level 0 runs.
  void set_host_field(const void* host) { host_field_ = host; }
  // d_field holds only the samples [origin, origin + dims) of the dataset (a shard's region;
  // origin a multiple of the brick size)
  void set_field_region(v3 origin, v3 dims)
  {
    fields_[0].field_origin = origin;
    fields_[0].field_dims = dims;
  }
  double kernel_ms() const { return enc_ ? enc_->kernel_ms() : 0.0; }
  long long kernel_launches() const { return enc_ ? enc_->launches() : 0; }
  // After a keep_device encode: the levels' regions on the device, or read back into outs
  // (whose nexps are set).
  void device_level(int l, const uint8_t** stream, const unsigned long long** offset) const
  {
    enc_->device_level(l, stream, offset);
  }
  int copy_level_out(int l, level_output* o) { return enc_->copy_level_out(l, o); }
  long long stream_bytes() const { return fields_[0].stream_bytes; }
  long long exp_bytes() const { return fields_[0].exp_bytes; }
  const std::vector<float>& level_ms() const { return fields_[0].level_ms; }
  const std::vector<long long>& level_bytes() const { return fields_[0].level_bytes; }

private:
  device_ctx* ctx_;
  const dataset_format& f_;
  bool keep_device_ = false;
  const void* host_field_ = nullptr;
  std::vector<level_output> outs_;
  std::vector<batch_field> fields_;
  std::unique_ptr<batch_encoder> enc_;
};

} // namespace idx2g
