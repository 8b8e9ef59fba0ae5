// Device side of the decoder: resident dataset tables and the per-level decode launch.
#pragma once

#include "device.h"
#include "encoder.h"
#include "format.h"

#include <vector>

namespace idx2g
{

// One brick of a decode launch.
struct decode_brick
{
  long long flat;  // row in the flat (level, brick) tables
  int parent;      // the parent's store index in the previous (coarser) launch, -1 if none
  int pos[3];      // position inside the parent
  // output copy (only on the output level): brick-local source grid and output grid
  int src_from[3], src_strd[3], dims[3], dst_from[3], dst_strd[3];
  int req;         // entry of the launch's request table
  int store;       // index in the launch's array of kept bricks (-1: output brick)
};

// What one request needs on one level (a launch may serve the bricks of many requests).
struct decode_target
{
  int mask;           // decoded subbands
  int is_output;      // the request's finest level: bricks go to the output grid
  int etol;           // Exponent(tolerance)
  int pad;
  int spacing[8][3];  // per subband: blocks not on this spacing are skipped (BypassDecode)
  void* out;          // output grid (device)
  int out_dims[3];
  int pad2;
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
  std::vector<v3> b3;  // brick coordinates of `bricks` (host side)
};

struct decode_request
{
  int nlevels = 1, nsb = 8;
  bool is2d = false, f32 = false;
  int etol = 0;
  int bpc = 1;  // BitPlanesPerChunk of the dataset
  v3 out_from, out_dims, out_strd;
  std::vector<decode_level> levels;  // coarsest first
};

// Brick-map mode (the reference's HashMap output, Core/idx2Decode.cpp:446-477): every decoded
// level's bricks are kept on the device (subband-major, in plan order) with a significance flag
// per brick (a block of a subband > 0, or of the coarsest level, was decoded).
struct decode_keep
{
  std::vector<const double*> bricks;     // per level l: [plan bricks][33^3] or null (not decoded)
  std::vector<std::vector<int>> sig;     // per level l: significance per plan brick
};

// A part of a kept brick copied out by gather_bricks: samples [from, from + dims) of the
// brick at src, x fastest, to out (elements).
struct brick_piece
{
  const double* src;
  int from[3], dims[3];
  long long out;
};

// A bit-plane chunk of an opened dataset, as the file tails locate it (host).
struct index_chunk
{
  unsigned long long off, size;  // bytes of the chunk in the blob
  int level, subband, bpkey, pad_;
};

class decode_device
{
public:
  ~decode_device();
  // Opening a dataset: alloc() the per-(brick, subband) tables of nslots entries and the blob,
  // upload_blob() each range of the files as it is read (any thread), build_index() once the
  // exponents are on the host (waits for every copy).
  int alloc(device_ctx* ctx, size_t nslots, size_t blob_bytes);
  void upload_blob(device_ctx* ctx, const uint8_t* src, size_t offset, size_t bytes);
  // The channel tables, built on the device (after every upload_blob): the chunk
  // headers in the blob (Core/idx2Decode.cpp:507 DecompressChunk: varbyte NBricks, the first
  // brick as a varbyte then unary gaps, varbyte sizes) are read a warp per chunk and a lane per
  // brick, twice:
  // the key range of every (brick, subband) slot, an exclusive scan of the slots' key counts,
  // then each brick's data offset. brick_map: per level (from level_base[l], level_size[l]
  // entries) the flat brick of each linear brick index, or -1. Then the exponents go up.
  int build_index(device_ctx* ctx, const std::vector<index_chunk>& chunks, const std::vector<int>& brick_map,
                  const std::vector<long long>& level_base, const std::vector<int>& level_size, int nsb,
                  const int16_t* exps, size_t* nchan);
  int decode(device_ctx* ctx, const decode_request& rq, void* out, size_t out_bytes, bool out_on_device,
             double* kernel_ms);
  // Several requests on this dataset at once: per level one launch (of each kernel) over the
  // bricks of every request that decodes the level. outs[i] receives request i's grid.
  // coeff_out (coefficient mode, one full-field request): the dequantised coefficients of every
  // brick (levels finest first, bricks row-major, 33^3 each) in place of the grid.
  // keep (brick-map mode, one full-field request): every level's bricks kept, see decode_keep.
  int decode_batch(device_ctx* ctx, const std::vector<const decode_request*>& rqs, void* const* outs,
                   const size_t* out_bytes, bool out_on_device, double* kernel_ms, void* coeff_out = nullptr,
                   decode_keep* keep = nullptr);
  // Copy pieces of kept bricks (subband-major) into a host buffer of `total` doubles.
  static int gather_bricks(device_ctx* ctx, const std::vector<brick_piece>& pieces, bool is2d, size_t total,
                           double* host_out);
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
  size_t nslots_ = 0;
  int device_ = 0;
  size_t resident_ = 0;
};

// Give the device memory that no open dataset holds back to the driver.
void trim_dataset_pool(int device);

// Loads the decode kernels into the current context and resolves the allocation-free
// decode's scratch array there (called when a context is created on the device).
int noalloc_prepare(int device);

} // namespace idx2g
