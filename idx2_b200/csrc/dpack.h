// Device packer: the chunk assembly of the encode (Core/idx2Encode.cpp:84-137
// EncodeBrickSubbandMetadata, Core/idx2Write.cpp:38-386 WriteChunk / FlushChunks /
// WriteChunkExponents / FlushChunkExponents) as a scan-then-scatter over the coder's regions
// while they are still on the device.
//
// The channels of one (level, subband) see that subband's bricks in encode order; a chunk is
// one channel's data over one range of BricksPerChunk bricks. When the bricks of every
// (level, subband) arrive in chunk order (the encode order makes them so), a channel's data in
// a chunk is exactly the (brick, key) pairs of that range with bytes for the key, in encode
// order, and the sequential state machine's flushes follow from per-chunk facts alone: a
// channel enters a chunk at the first brick of the range with bytes for it (at its place in
// that brick's first-touch order of keys), which writes the data it held, and what it holds
// at the end is written by FlushChunks in channel-key order. So:
//   the key pass (dpack.cu), over every event at once with a warp each: its region's key
//     window and key-stream offsets, its segment's key range, then per key of the
//     (level, subband, chunk) segment its brick count, first / last brick, byte and
//     varbyte-size totals (atomics, order-free); then a CTA per segment finds the event and
//     touch rank at which each key enters the chunk;
//   the host orders the chunks by their flush stamps, assigns file offsets, builds the file
//     tails and the statistics (no brick data touched);
//   k_pack_write (a CTA per segment, a warp per chunk): exclusive scans over the segment's
//     bricks in encode order give each pair's place; the chunk header (varbyte NBricks, the
//     first brick as a varbyte then unary gaps, varbyte sizes) and the pairs' channel bytes
//     are scattered into the file images, and the raw exponents of the segment into the
//     exponent buffer (compressed with zstd on the host).
// The files equal the host packer's (packer.cpp) byte for byte.
#pragma once

#include "encoder.h"
#include "packer.h"

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace idx2g
{

// The packed dataset: file contents (chunk sections pointing into `image`, tails owned) and
// the statistics, as the host packer's files() / stats().
struct packed_dataset
{
  std::map<std::string, file_buffer> files;
  pack_stats stats;
  const uint8_t* image = nullptr;  // pinned host copy of the chunk sections
  std::vector<std::vector<uint8_t>> exps_z;
  // waits until the bytes [p, p + n) of the image have arrived (set by the device packer,
  // whose copy of the image runs on while the files are being written)
  std::function<void(const uint8_t*, size_t)> ready;
};

// Whether the device packer takes this plan (every (level, subband)'s bricks in chunk order,
// bricks increasing inside every chunk); otherwise the host packer runs.
bool device_pack_applies(const dataset_format& f, const encode_plan& plan);

// ---------------------------------------------------------------------------
// kernel tables (dpack.cu) and the host stages around the kernels (dpack_plan.cpp), which
// the CPU tests also drive with the kernels' work done on the host
// ---------------------------------------------------------------------------
constexpr int kSegKeys = 256;  // keys of one segment (key window of its chunks)

struct dpack_segment
{
  int level, subband, nexps;
  int ev0, ev1;  // events [ev0, ev1) of the event table
  int pad_;
  unsigned long long exp_off;  // first byte of the segment's raw exponents
};

struct dpack_event
{
  unsigned long long linear;  // linear brick index on the level
  unsigned gevent;            // index in the encode's event order
  int brick;                  // brick index in the level's list (region offset lookup)
  int seg;                    // its segment
  int pad_;
};

// per (segment, key slot); n = 0: the key has no bytes in the segment
struct dpack_key
{
  unsigned n, sizes_bytes, enter_event, enter_rank;
  unsigned long long first_brick, last_brick, data_bytes;
};

// Segments of the plan: per (level, subband), in order of first appearance, its events cut
// at chunk changes; raw exponent offsets per segment.
struct dpack_plan
{
  std::vector<dpack_segment> segs;
  std::vector<dpack_event> evs;
  std::vector<u64> seg_chunk;
  std::vector<std::pair<int, int>> groups;             // (level, subband)
  std::vector<std::pair<size_t, size_t>> group_segs;  // [first, last) segment of each group
  unsigned long long exp_total = 0;
  int exp_bytes = 1;
};
// nexps[level][subband]: blocks per subband
int dpack_make_plan(const dataset_format& f, const encode_plan& plan, const std::vector<std::vector<int>>& nexps,
                    dpack_plan* P);

// The chunk section of the files: every chunk's first byte in the image (per segment and key
// slot, ~0: none), the image size, each file's span of it.
struct dpack_layout
{
  std::vector<unsigned long long> chunk_off;
  unsigned long long total = 0;
  std::map<std::string, std::pair<unsigned long long, unsigned long long>> file_span;
};
// From the key pass's output: chunk flush stamps, file order and offsets; out receives the
// files' chunk tables (sizes, addresses) and the bit-plane statistics.
int dpack_make_layout(const dataset_format& f, const dpack_plan& P, const std::vector<dpack_key>& keys,
                      const std::vector<int>& kmin, dpack_layout* L, packed_dataset* out);
// From k_pack_write's output (host copies of the image and of the raw exponents): exponent
// chunks (zstd), file contents and tails, the remaining statistics.
int dpack_finish(const dataset_format& f, const dpack_plan& P, const dpack_layout& L, const uint8_t* image,
                 const uint8_t* exps, packed_dataset* out);

} // namespace idx2g
