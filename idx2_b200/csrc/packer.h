// Chunk/file packer: turns per-(brick, subband) coder output into the on-disk
// layout of the reference (Core/idx2Write.cpp, Core/idx2Encode.cpp:41-137,
// Core/idx2Encode.cpp:233-249).  The GPU produces, for every brick and subband,
// the block exponents and one byte-aligned bit stream per bit-plane channel;
// the packer replays the reference's channel / chunk / file state machine over
// those results in the reference's encode order, so chunk contents and chunk
// order inside each file are the reference's.
#pragma once

#include "format.h"

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace idx2g
{

// LSB-first bit writer with the reference's byte layout (Core/BitStream.h).
struct bit_writer
{
  std::vector<uint8_t> bytes;
  uint64_t nbits = 0;
  void put(uint64_t v, int n);
  void put_varbyte(uint64_t v);  // Core/VarInt.h:14
  void put_unary(uint64_t v);    // Core/VarInt.h:82
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
  const uint8_t* bytes = nullptr;    // channel streams back to back, ascending key order
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

struct file_buffer
{
  std::vector<uint8_t> data;        // chunks in write order (then metadata at flush)
  bit_writer chunk_sizes;           // varbyte sizes of bit-plane chunks
  std::vector<u64> chunk_addrs;     // chunk addresses
  bool has_chunks = false;
  std::vector<uint8_t> exp_data;    // zstd-compressed exponent chunks
  bit_writer exp_sizes;
  std::vector<u64> exp_addrs;
  bool has_exps = false;
};

class packer
{
public:
  packer(const dataset_format& f, double tolerance);
  // One EncodeSubband call of the reference (Core/idx2Encode.cpp:261).
  int add(const subband_result& r);
  // FlushChunks + FlushChunkExponents (Core/idx2Write.cpp:317, :121); fills files.
  int finish();
  std::map<std::string, file_buffer>& files() { return files_; }
  const pack_stats& stats() const { return stats_; }
  // The statistics block the reference appends to the metadata file (Core/idx2Write.cpp:389).
  std::string stats_text() const;

private:
  struct channel
  {
    bit_writer deltas, sizes;
    std::vector<uint8_t> bricks;
    u64 last_chunk = 0, last_brick = 0;
    int nbricks = 0;
  };
  struct sub_channel
  {
    std::vector<uint8_t> brick_exps;
    u64 last_chunk = 0, last_brick = 0;
  };
  void write_chunk(channel& c, int level, int subband, int bpkey);
  void write_chunk_exps(sub_channel& s, int level, int subband);
  void first_touch_order(const subband_result& r, std::vector<int>* keys) const;

  const dataset_format& f_;
  double tol_;
  int etol_;
  std::map<uint32_t, channel> channels_;  // ordered by channel key
  std::map<std::pair<int, int>, sub_channel> subs_;
  std::map<std::string, file_buffer> files_;
  pack_stats stats_;
};

// zstd level 1 through the system libzstd (loaded at run time).
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

} // namespace idx2g
