// Device packer, device side: the kernel launches and the encode path around them (dpack.h).
#pragma once

#include "device.h"
#include "dpack.h"

namespace idx2g
{

// One level's coder output on the device: the stream of regions and the region offset of
// every (brick, subband) (index brick * 8 + subband).
struct device_level_stream
{
  const uint8_t* stream = nullptr;
  const unsigned long long* offset = nullptr;
  int nsb = 0;
  std::vector<int> nexps;  // per subband
};

// per (segment, key slot): running totals of the key's pairs (order-free atomics)
struct dpack_acc
{
  unsigned n, szb;
  int first, last;  // first / last event of the segment with bytes for the key
  unsigned long long db;
};

constexpr int kPackSub = 256;  // events of a sub-range

// per (segment, key, sub-range): the key's varbyte-size and data bytes in the sub-range, then
// (after the ranks pass) those of the segment's earlier sub-ranges
struct dpack_sub
{
  unsigned long long vb, data;
};

struct dpack_args
{
  const dpack_segment* segs;
  int nseg;
  const dpack_event* evs;
  int nev;
  // per event: its region, key window and the start of its key offsets in kb
  unsigned long long* ev_region;  // byte address of the region
  int* ev_kmin;
  int* ev_nkeys;
  unsigned long long* ev_kb;
  uint32_t* kb;                   // per event and key: the key stream's byte offset in the region's streams
  unsigned long long kb_cap;      // entries of kb
  unsigned long long* cursor;     // kb entries taken
  int* seg_kmax;                  // [nseg]
  dpack_acc* acc;                 // [nseg][kSegKeys]
  // sub-ranges of kPackSub events of a segment (a CTA each in the totals and write passes)
  const int4* subs;               // (segment, first event, end event, index of the sub-range in its segment)
  int nsub;
  const int* seg_sub0;            // [nseg]: the segment's first entry of sub_acc (x kSegKeys)
  dpack_sub* sub_acc;             // per (segment, key, sub-range): totals, then exclusive prefixes
  const uint8_t* streams[16];
  const unsigned long long* offsets[16];
  int etol, end_bp, bpc, exp_bytes;  // exp_bytes: 1 (float32) or 2 (float64)
  int* seg_kmin;                     // [nseg]: key of slot 0 (or a large value: no keys)
  dpack_key* keys;                   // [nseg][kSegKeys]
  const unsigned long long* chunk_off;  // [nseg][kSegKeys]: first byte of the chunk in image
  uint32_t* image;                   // zeroed
  uint8_t* exps;                     // raw exponents of every segment
  int* error;                        // 1: a segment spans more than kSegKeys keys, 2: kb too small
};

void dpack_launch_keys(const dpack_args& a, int grid, cudaStream_t st);
void dpack_launch_write(const dpack_args& a, int grid, cudaStream_t st);

// Packs the levels' regions on ctx's device. Returns NoError, or NotApplicable when a segment
// holds more keys than the kernels' window (the caller then packs on the host).
constexpr int kDpackNotApplicable = -2;
// The plan's segment tables are made and uploaded once and kept on the context for the next
// encode of the same plan.
// on_image (may be empty): called once the image's copy to the host is under way, with the
// layout, the host image and the function that waits for a part of it to arrive.
using image_hook = std::function<void(const dpack_layout&, const uint8_t*, const ready_fn&)>;
int device_pack(device_ctx* ctx, const dataset_format& f, const std::shared_ptr<const encode_plan>& plan,
                const std::vector<device_level_stream>& levels, packed_dataset* out,
                const image_hook& on_image = image_hook());

// encode_dataset with the device packer: every level coded with its regions kept on the
// device, packed there, and the files written. When the packer does not take a segment (more
// keys than its window), the regions are read back and packed on the host instead.
// timing: device_s the coding, pack_s the packing (with the copy of the chunk sections to the
// host), write_s the files.
int encode_dataset_dpack(device_ctx* ctx, dataset_format* f, params* p, gpu_coder* coder, encode_timing* timing,
                         const std::shared_ptr<const encode_plan>& plan,
                         const std::vector<unsigned long long>* prealloc);

} // namespace idx2g
