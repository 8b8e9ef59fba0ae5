// Encode driver: the order in which the reference encodes bricks and subbands,
// the level-by-level device stage, and the final packing into files.
//
// The reference encodes depth-first: for every level-0 brick in traversal order
// it transforms the brick, and while emitting subband 0 it hands the low band to
// the parent, encoding the parent as soon as its last child arrives
// (Core/idx2Encode.cpp:276-340, :395-426).  Here the same recursion only fixes the
// ORDER: the device stage transforms and codes all bricks of one level at once,
// and the packer replays the (level, brick, subband) events afterwards.
#pragma once

#include "format.h"
#include "packer.h"

#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <thread>
#include <vector>

namespace idx2g
{

struct brick_entry
{
  v3 brick3;           // brick coordinates on its level
  u64 linear = 0;      // GetLinearBrick
  v3 valid;            // ExtentLocal dims: valid samples inside the 32^3 brick
  int parent = -1;     // index of the parent in the next level's list
  v3 pos_in_parent;    // LocalBrickPos3
  int nchildren = 0;   // for parents: NChildrenMax
};

struct encode_event
{
  int level, brick, subband;
};

struct encode_plan
{
  std::vector<std::vector<brick_entry>> levels;  // per level, in encode order
  std::vector<encode_event> events;              // EncodeSubband calls in order
};

int make_encode_plan(const dataset_format& f, encode_plan* plan);

// Block geometry of one subband: the coded blocks in the reference's Morton walk
// (Core/idx2Encode.cpp:157-174), packed as d3 (offset / 4) and block dims.
struct block_geom
{
  uint8_t dx, dy, dz;  // block offset in units of 4 samples
  uint8_t bx, by, bz;  // block dims (1..4)
  uint16_t code;       // Morton code
};
// Geometry of the coded blocks of subband sb at a level; skips CodedInNextLevel blocks.
void subband_blocks(const dataset_format& f, int level, int sb, std::vector<block_geom>* out);

// Coder output of one level, in host memory.
constexpr int kMaxBlocksPerSubband = 128;  // >= 125 (5^3)
constexpr int kKeyWindow = 128;            // channel keys per (brick, subband)

// The coder output of one (brick, subband) is a self-describing region of the level's
// stream, 4-byte aligned:
//   int32 kmin, int32 nkeys                       channel keys kmin .. kmin + nkeys - 1
//   int16 exps[nexps], padded to 4 bytes          block exponents, coded blocks in Morton order
//   uint32 sizes[nkeys]                           bytes of each channel stream (0: absent)
//   channel streams back to back, ascending key, each byte-aligned; padded to 4 bytes
struct region_view
{
  int kmin = 1, kmax = 0;
  const int16_t* exps = nullptr;
  const uint32_t* sizes = nullptr;
  const uint8_t* bytes = nullptr;
};
inline size_t region_header_bytes(int nexps, int nkeys)
{
  return 8 + (((size_t)nexps * 2 + 3) & ~(size_t)3) + (size_t)nkeys * 4;
}
inline region_view view_region(const uint8_t* r, int nexps)
{
  region_view v;
  int32_t kmin, nkeys;
  memcpy(&kmin, r, 4);
  memcpy(&nkeys, r + 4, 4);
  v.kmin = nkeys > 0 ? kmin : 1;
  v.kmax = nkeys > 0 ? kmin + nkeys - 1 : 0;
  v.exps = reinterpret_cast<const int16_t*>(r + 8);
  v.sizes = reinterpret_cast<const uint32_t*>(r + 8 + (((size_t)nexps * 2 + 3) & ~(size_t)3));
  v.bytes = r + region_header_bytes(nexps, nkeys > 0 ? nkeys : 0);
  return v;
}

struct level_output
{
  int nbricks = 0, nsb = 0;
  std::vector<int> nexps;        // per subband (identical for every brick of the level)
  std::vector<uint64_t> offset;  // [brick][sb] byte offset of the region in stream
  std::vector<uint8_t> stream;   // the regions (or, when ext_stream is set, in that buffer)
  const uint8_t* ext_stream = nullptr;
  const uint8_t* bytes() const { return ext_stream ? ext_stream : stream.data(); }
};

// A device (or test) stage that transforms and codes every brick of a level.
class brick_coder
{
public:
  virtual ~brick_coder() = default;
  // Runs level `level` for `bricks` (encode order). Level 0 reads the input field;
  // level > 0 reads the parent bricks assembled by the previous level's run.
  virtual int run_level(int level, const encode_plan& plan, level_output* out) = 0;
  // min / max over the input field (valid after level 0)
  virtual void value_range(double* vmin, double* vmax) = 0;
};

struct encode_timing
{
  double device_s = 0, pack_s = 0, write_s = 0;
  unsigned long long file_bytes = 0;  // data files + metadata file
  int nfiles = 0;
  // bytes of every level's data file when each level has exactly one (else empty)
  std::vector<unsigned long long> level_file_bytes;
};

// Full encode: plan, device stage for every level, packing, files (Core/idx2Encode.cpp:390).
// files (may be null) receives path -> bytes; write_files controls whether they are
// written to disk (several files at a time).
// plan (may be null): the format's encode plan, made here when null.
// prealloc (may be null): expected bytes of each level's data file (one file per level, such as
// the sizes of the previous encode of this shape); the file system allocates their pages on a
// thread of its own while the device stage runs.
int encode_dataset(dataset_format* f, params* p, brick_coder* coder,
                   std::map<std::string, std::vector<uint8_t>>* files, bool write_files,
                   encode_timing* timing, const encode_plan* plan = nullptr,
                   const std::vector<unsigned long long>* prealloc = nullptr);

// Packing and files for the device stage's outputs (the second half of encode_dataset).
// before_write (may be null) is joined before the first file is opened.
int pack_dataset(const dataset_format* f, const params* p, const encode_plan& plan,
                 const std::vector<level_output>& outs, std::map<std::string, std::vector<uint8_t>>* files,
                 bool write_files, encode_timing* timing, std::thread* before_write = nullptr);

// The second half of pack_dataset: the metadata file (format text + stats) and the data
// files from their parts; files / write_files / timing / before_write as pack_dataset.
struct file_buffer;
// ready (may be null): waited on before a part's bytes are read (write_files).
int write_dataset(const dataset_format* f, const params* p, std::map<std::string, file_buffer>& data,
                  const std::string& stats, std::map<std::string, std::vector<uint8_t>>* files, bool write_files,
                  encode_timing* timing, std::thread* before_write, double pack_s,
                  const std::function<void(const uint8_t*, size_t)>* ready = nullptr);

// Bytes of every level's data file into timing->level_file_bytes, when each level has
// exactly one (else empty).
void note_level_files(const dataset_format& f, const encode_plan& plan, const std::map<std::string, file_buffer>& data,
                      encode_timing* timing);

// Allocate the pages of each level's data file (sizes[l] bytes, file size unchanged) on a new
// thread; levels with fewer than 64 MB are left alone.
std::thread preallocate_files(const dataset_format& f, const encode_plan& plan,
                              const std::vector<unsigned long long>& sizes);

// The device stage only: every level through the coder, with the given plan.
int encode_levels(dataset_format* f, brick_coder* coder, std::vector<level_output>* outs, const encode_plan& plan);

int write_file(const std::string& path, const std::vector<uint8_t>& data);
int make_dirs_for(const std::string& path);

} // namespace idx2g
