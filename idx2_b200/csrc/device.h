// CUDA context and the device stages of the encoder / decoder.
#pragma once

#include "encoder.h"

#include <cuda_runtime.h>
#include <map>
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
  long long launches = 0;  // kernels launched on this context so far

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
      if (b.p)
        cudaFree(b.p);
      b.p = nullptr;
      b.n = 0;
      size_t want = bytes + bytes / 8 + 256;
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
  void release()
  {
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

// Device brick coder: transforms and codes every brick of a level in one launch.
class gpu_coder : public brick_coder
{
public:
  gpu_coder(device_ctx* ctx, const dataset_format& f, const void* d_field, bool field_f32);
  ~gpu_coder() override;
  int run_level(int level, const encode_plan& plan, level_output* out) override;
  void value_range(double* vmin, double* vmax) override;
  // Leave the coder output on the device (no copies for the packer).
  void set_keep_device(bool v) { keep_device_ = v; }
  double kernel_ms() const { return kernel_ms_; }
  long long kernel_launches() const { return launches_; }
  long long stream_bytes() const { return stream_bytes_; }
  long long exp_bytes() const { return exp_bytes_; }
  const std::vector<float>& level_ms() const { return level_ms_; }
  const std::vector<long long>& level_bytes() const { return level_bytes_; }

private:
  device_ctx* ctx_;
  const dataset_format& f_;
  const void* d_field_;
  bool field_f32_;
  bool keep_device_ = false;
  const double* in_bricks_ = nullptr;
  double vmin_ = 1.7976931348623157e308, vmax_ = -1.7976931348623157e308;
  double kernel_ms_ = 0;
  long long launches_ = 0, stream_bytes_ = 0, exp_bytes_ = 0;
  std::vector<float> level_ms_;
  std::vector<long long> level_bytes_;
};

} // namespace idx2g
