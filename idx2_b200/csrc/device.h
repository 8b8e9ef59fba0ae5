// CUDA context and the device stages of the encoder / decoder.
#pragma once

#include "encoder.h"

#include <cuda_runtime.h>
#include <vector>

namespace idx2g
{

// One context per thread; all work is ordered on `stream`.
struct device_ctx
{
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
};

// Device brick coder: transforms and codes every brick of a level in one launch.
class gpu_coder : public brick_coder
{
public:
  gpu_coder(device_ctx* ctx, const dataset_format& f, const void* d_field, bool field_f32);
  ~gpu_coder() override;
  int run_level(int level, const encode_plan& plan, level_output* out) override;
  void value_range(double* vmin, double* vmax) override;
  double kernel_ms() const { return kernel_ms_; }
  long long kernel_launches() const { return launches_; }
  long long stream_bytes() const { return stream_bytes_; }
  long long exp_bytes() const { return exp_bytes_; }

private:
  void* dev_alloc(size_t bytes);
  device_ctx* ctx_;
  const dataset_format& f_;
  const void* d_field_;
  bool field_f32_;
  const double* in_bricks_ = nullptr;
  std::vector<void*> owned_;
  double vmin_ = 1.7976931348623157e308, vmax_ = -1.7976931348623157e308;
  double kernel_ms_ = 0;
  long long launches_ = 0, stream_bytes_ = 0, exp_bytes_ = 0;
};

} // namespace idx2g
