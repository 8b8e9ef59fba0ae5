// Chunk/file packer: turns per-(brick, subband) coder output into the on-disk
// layout of the reference (Core/idx2Write.cpp, Core/idx2Encode.cpp:41-137,
// Core/idx2Encode.cpp:233-249).  The GPU produces, for every brick and subband,
// the block exponents and one byte-aligned bit stream per bit-plane channel;
// the packer replays the reference's channel / chunk / file state machine over
// those results in the reference's encode order, so chunk contents and chunk
// order inside each file are the reference's.
//
// Brick data is never copied while packing: channels and files hold references
// (segments) into the coder output, which must outlive the packer; files are
// written from their segment lists.
#pragma once

#include "format.h"

#include <cstdint>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace idx2g
{

// LSB-first bit writer with the reference's byte layout (Core/BitStream.h).
struct bit_writer
{
  std::vector<uint8_t> bytes;
  uint64_t nbits = 0;
  void put(uint64_t v, int n);    // n <= 57
  void put_varbyte(uint64_t v);   // Core/VarInt.h:14
  void put_unary(uint64_t v);     // Core/VarInt.h:82
  size_t size() const { return (size_t)((nbits + 7) / 8); }
  void clear()
  {
    bytes.clear();
    nbits = 0;
  }
};

// Output of the block coder for one (brick, subband).
struct subband_result
{
  int level = 0;
  u64 brick = 0;  // linear brick index on its level
  int subband = 0;
  const int16_t* exps = nullptr;  // coded blocks, Morton order
  int nexps = 0;
  int kmin = 1, kmax = 0;            // bit-plane channel keys present (kmin > kmax: none)
  const uint32_t* sizes = nullptr;   // bytes per key, index key - kmin (0: absent)
  const uint8_t* bytes = nullptr;    // channel streams back to back, ascending key order; null
                                     // for another shard's brick (its segments stay null)
};

struct pack_stats
{
  struct acc
  {
    double s = 0, ssq = 0;
    long long n = 0;
    void add(double v)
    {
      s += v;
      ssq += v * v;
      ++n;
    }
    double avg() const { return s / (double)n; }
    double sd() const;
  };
  acc bit_plane_chunks, brick_deltas, brick_sizes, chunk_sizes, chunk_addrs_raw, chunk_addrs_z,
    exp_chunks_raw, exp_chunks_z, exp_chunk_sizes, exp_addrs_raw, exp_addrs_z;
};

struct segment
{
  const uint8_t* p;
  size_t n;
};

// Consecutive segments of a file: a whole bit-plane chunk (header, then its bricks' data),
// or one piece of the tail.
struct segment_run
{
  const segment* seg;
  size_t nseg;
  size_t bytes;
};

struct file_buffer
{
  std::vector<segment_run> parts;                   // file content, in order
  std::deque<std::vector<uint8_t>> owned;           // bytes the parts point into
  std::deque<segment> singles;                      // the segments of one-segment runs
  size_t nbytes = 0;
  bit_writer chunk_sizes;                           // varbyte sizes of bit-plane chunks
  std::vector<u64> chunk_addrs;                     // chunk addresses
  bool has_chunks = false;
  std::vector<segment> exp_parts;                   // compressed exponent chunks
  std::vector<u64> exp_addrs;
  bool has_exps = false;
  void append_owned(std::vector<uint8_t>&& v);
  void append_ref(const uint8_t* p, size_t n);
  // n segments that stay in place while the file is alive
  void append_run(const segment* s, size_t n, size_t bytes);
  template <typename F>
  void for_each_segment(F&& fn) const
  {
    for (const segment_run& r : parts)
      for (size_t k = 0; k < r.nseg; ++k)
        fn(r.seg[k]);
  }
};

// The packer records the (brick, subband) results in the reference's encode order and, at
// finish, replays the channel state machine of every (level, subband) on its own thread:
// channels of different (level, subband) never interact, and each chunk write is stamped
// with its place in the sequential order (event index, then rank inside the event; the final
// flushes after every event, in the reference's flush order), so the merged chunk order in
// every file and the order of the statistics are those of a sequential pass.
class packer
{
public:
  packer(const dataset_format& f, double tolerance);
  ~packer();
  // One EncodeSubband call of the reference (Core/idx2Encode.cpp:261); r's arrays must
  // outlive the packer.
  int add(const subband_result& r);
  // add() of every result, in order
  int add_all(std::vector<subband_result>&& rs);
  // Channel / chunk state machine, FlushChunks + FlushChunkExponents (Core/idx2Write.cpp:317,
  // :121), file assembly.
  int finish();
  std::map<std::string, file_buffer>& files() { return files_; }
  const pack_stats& stats() const { return stats_; }
  // The statistics block the reference appends to the metadata file (Core/idx2Write.cpp:389).
  std::string stats_text() const;

  struct group;  // the channels of one (level, subband)

private:
  const dataset_format& f_;
  double tol_;
  int etol_;
  std::vector<subband_result> events_;
  std::map<std::string, file_buffer> files_;
  std::vector<std::unique_ptr<group>> groups_;
  pack_stats stats_;
};

// The statistics block the reference appends to the metadata file (Core/idx2Write.cpp:389).
std::string pack_stats_text(const pack_stats& s);

// zstd level 1: frames byte-identical to the reference's zstd 1.4.5 (zstd_frame.cpp); the
// decompression goes through the system libzstd (loaded at run time; any version reads them).
int zstd_compress(const uint8_t* src, size_t n, std::vector<uint8_t>* out);
int zstd_decompress(const uint8_t* src, size_t n, std::vector<uint8_t>* out);
const char* zstd_version();

// plane loop bound shared with the device coder (Core/idx2Encode.cpp:195-206)
inline bool plane_coded(int bp, int emax, int etol, int bpc)
{
  int realbp = bp + emax;
  bool too_high = 64 - 6 > realbp - etol + 1;
  return !(too_high && ((realbp + 1024) % bpc) == 0);
}
int exponent_f64(double v);

// Called before the bytes [p, p + n) of a part are read: waits until they are in place
// (parts whose bytes are still arriving, e.g. from the device).
using ready_fn = std::function<void(const uint8_t* p, size_t n)>;

// Write files from their parts (creating directories), with several threads.
int write_files(const std::vector<std::pair<std::string, const file_buffer*>>& files, const ready_fn* ready = nullptr);

} // namespace idx2g
