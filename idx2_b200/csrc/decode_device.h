// Device side of the decoder: resident dataset tables and the per-level decode launch.
#pragma once

#include "device.h"
#include "encoder.h"
#include "format.h"

#include <vector>

namespace idx2g
{

// One brick of a decode request.
struct decode_brick
{
  long long flat;  // row in the flat (level, brick) tables
  int parent;      // index of the parent in the previous (coarser) decoded level, -1 if none
  int pos[3];      // position inside the parent
  // output copy (only on the output level): brick-local source grid and output grid
  int src_from[3], src_strd[3], dims[3], dst_from[3], dst_strd[3];
};

struct decode_level
{
  int level = 0;
  int mask = 0;
  bool is_output = false;
  int spacing[8][3] = {};
  int nblocks[8] = {};
  uint64_t geom[8][kMaxBlocksPerSubband] = {};
  double inv_weight[8] = {};
  int norm_mask = 0;
  std::vector<decode_brick> bricks;
};

struct decode_request
{
  int nlevels = 1, nsb = 8;
  bool is2d = false, f32 = false;
  int etol = 0;
  v3 out_from, out_dims, out_strd;
  std::vector<decode_level> levels;  // coarsest first
};

class decode_device
{
public:
  ~decode_device();
  int upload(device_ctx* ctx, const std::vector<int16_t>& exps, const std::vector<int32_t>& kmin,
             const std::vector<int32_t>& n, const std::vector<uint64_t>& first,
             const std::vector<uint64_t>& off, const uint8_t* blob, size_t blob_bytes);
  int decode(device_ctx* ctx, const decode_request& rq, void* out, size_t out_bytes, bool out_on_device,
             double* kernel_ms);
  // Allocation-free decode into a device buffer: every temporary lives in a fixed static
  // device array of decode.cu (limits and semantics there and in include/idx2g.h).
  int decode_noalloc(device_ctx* ctx, const decode_request& rq, void* d_out, size_t out_bytes,
                     double* kernel_ms);
  size_t resident_bytes() const { return resident_; }

private:
  int16_t* exps_ = nullptr;
  int32_t* kmin_ = nullptr;
  int32_t* n_ = nullptr;
  unsigned long long* first_ = nullptr;
  unsigned long long* off_ = nullptr;
  uint8_t* blob_ = nullptr;
  size_t blob_bytes_ = 0;
  size_t resident_ = 0;
};

} // namespace idx2g
