// Host-side description of an idx2 dataset: parameters, the derived brick /
// chunk / file orders, subband geometry and file naming.  This is the
// equivalent of the reference's idx2_file after Finalize
// (Core/idx2Common.h:111-184, Core/idx2Common.cpp:726).  It is pure host
// C++ with no CUDA dependency; the encoder/decoder drivers and the CLI use it.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace idx2g
{

using u64 = uint64_t;
using i64 = int64_t;

// Error codes: the reference's idx2_CommonErrs (Core/ErrorCodes.h:6-10) followed by
// idx2_err_code (Core/idx2Common.h:36-56); the numeric values are those of the
// reference's idx2_Enum, so a caller can compare them directly.
enum err : int
{
  NoError = 0,
  UnknownError,
  SizeZero,
  SizeTooSmall,
  SizeMismatched,
  DimensionMismatched,
  DimensionsTooMany,
  AttributeNotFound,
  OptionNotSupported,
  TypeNotSupported,
  FileCreateFailed,
  FileReadFailed,
  FileWriteFailed,
  FileOpenFailed,
  FileCloseFailed,
  FileSeekFailed,
  FileTellFailed,
  ParseFailed,
  OutOfMemory,
  DimensionsRepeated,
  DimensionTooSmall,
  BrickSizeNotPowerOfTwo,
  BrickSizeTooBig,
  TooManyLevels,
  TooManyTransformPassesPerLevel,
  TooManyLevelsOrTransformPasses,
  TooManyBricksPerFile,
  TooManyFilesPerDir,
  NotSupportedInVersion,
  CannotCreateDirectory,
  SyntaxError,
  TooManyBricksPerChunk,
  TooManyChunksPerFile,
  ChunksPerFileNotPowerOf2,
  BricksPerChunkNotPowerOf2,
  ChunkNotFound,
  BrickNotFound,
  FileNotFound,
  UnsupportedScheme,
  // codes of this library (no reference counterpart)
  CudaError = 100,
  InvalidArgument = 101,
  DeviceStreamOverflow = 102,
  CorruptStream = 103,
  ScratchTooSmall = 104,  // request larger than the allocation-free decode's fixed scratch
};

struct v3
{
  int x = 0, y = 0, z = 0;
  v3() = default;
  constexpr v3(int a, int b, int c) : x(a), y(b), z(c) {}
  explicit constexpr v3(int a) : x(a), y(a), z(a) {}
  int& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  int operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  bool operator==(const v3& o) const { return x == o.x && y == o.y && z == o.z; }
  bool operator!=(const v3& o) const { return !(*this == o); }
};
inline v3 operator+(v3 a, v3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline v3 operator-(v3 a, v3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline v3 operator*(v3 a, v3 b) { return { a.x * b.x, a.y * b.y, a.z * b.z }; }
inline v3 operator/(v3 a, v3 b) { return { a.x / b.x, a.y / b.y, a.z / b.z }; }
inline v3 operator%(v3 a, v3 b) { return { a.x % b.x, a.y % b.y, a.z % b.z }; }
inline v3 vmin(v3 a, v3 b)
{
  return { a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z };
}
inline v3 vmax(v3 a, v3 b)
{
  return { a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z };
}
inline bool all_lt(v3 a, v3 b) { return a.x < b.x && a.y < b.y && a.z < b.z; }
inline bool all_le(v3 a, v3 b) { return a.x <= b.x && a.y <= b.y && a.z <= b.z; }
inline i64 prod(v3 a) { return (i64)a.x * a.y * a.z; }

// [from, from + dims) box of samples (or bricks); grids add a stride.
struct extent
{
  v3 from, dims;
  v3 last() const { return from + dims - v3(1); }
  v3 to() const { return from + dims; }
};
struct grid
{
  v3 from, dims, strd{ 1, 1, 1 };
};

int log2_floor(i64 v);
int log2_ceil(i64 v);
bool is_pow2(i64 v);

extent crop(const extent& a, const extent& b);
grid crop(const grid& a, const grid& b);
grid relative(const grid& a, const grid& b);

enum class dtype : int
{
  float32 = 0,
  float64 = 1
};

// Transform orders are base-4 strings of X/Y/Z/+ with the first character in the
// lowest bits (Core/Wavelet.cpp:407-460).
u64 encode_order(const std::string& s);
std::string decode_order(u64 order);
std::string decode_order_for_dims(u64 order, v3 n3);
int decode_order_passes(u64 order, int passes, std::string* out);

struct subband
{
  grid g;        // inside the extended brick (33^3 or 33x33x1)
  v3 low_high;   // 1 = high-pass along that axis
  v3 level_rev;  // Level3Rev of the reference (1 for low, 0 for high with one pass)
};

// Parameters as the reference's params struct (Core/idx2Common.h:74-108).
struct params
{
  std::string name, field;
  v3 dims{ 0, 0, 0 };
  dtype type = dtype::float64;
  v3 brick_dims{ 32, 32, 32 };
  int num_levels = 0;
  double tolerance = 0;
  int bricks_per_chunk = 4096;
  int chunks_per_file = 64;
  int files_per_dir = 64;
  int bit_planes_per_chunk = 1;
  int bit_planes_per_file = 16;
  int version[2] = { 1, 0 };
  std::string out_dir = ".";
  // decode
  std::string input_file;
  std::string in_dir = ".";
  bool has_extent = false;
  extent decode_extent;
  v3 downsampling{ 0, 0, 0 };
  double decode_tolerance = 0;
};

// The finalised dataset description (the reference's idx2_file).
struct dataset_format
{
  std::string name, field, dir;
  v3 dims{ 256, 256, 256 };
  dtype type = dtype::float64;
  v3 brick_dims{ 32, 32, 32 };
  v3 brick_dims_ext{ 33, 33, 33 };
  v3 block_dims{ 4, 4, 4 };
  v3 downsampling{ 0, 0, 0 };
  int version[2] = { 1, 0 };
  u64 transform_order = 0;
  std::string transform_order_full;
  int nlevels = 1;
  double tolerance = 0;
  int files_per_dir = 512;
  int bricks_per_chunk_in = 4096;
  int chunks_per_file_in = 64;
  int bit_planes_per_chunk = 1;
  int bit_planes_per_file = 32;
  v3 group_brick3;
  double value_min = 0, value_max = 0;

  std::vector<subband> subbands;         // extended brick (33)
  std::vector<subband> subbands_nonext;  // non-extended brick (32)
  std::vector<v3> nbricks3, nchunks3, nfiles3, bricks_per_chunk3, chunks_per_file3;
  std::vector<std::string> bricks_order_str, chunks_order_str, files_order_str;
  std::vector<u64> bricks_order, bricks_order_in_chunk, chunks_order_in_file, chunks_order,
    files_order;
  std::vector<int> bricks_per_chunk, chunks_per_file, bricks_per_file;
  std::vector<std::vector<int>> files_dirs_depth;
  std::vector<uint8_t> decode_masks;             // per level
  std::vector<std::vector<v3>> decode_spacings;  // per level, per subband

  bool is2d() const { return brick_dims.z == 1; }
  int nsubbands() const { return (int)subbands.size(); }
};

// Set the fields from params (Applications/idx2App.cpp:217 SetParams) and finalise
// (Core/idx2Common.cpp:726 Finalize). Returns an err code.
int finalize(dataset_format* f, params* p);
// Finalise a format that was read from a metadata file (decode side, idx2.cpp:23 Init).
int finalize_read(dataset_format* f, params* p);

// Linear brick index on a level (Core/idx2Lookup.cpp:13 GetLinearBrick).
u64 linear_brick(const dataset_format& f, int level, v3 brick3);
// linear_brick of a level by table: the index interleaves the axes' bits, so it is the OR of
// one entry per axis (tables for coordinates below n[d]; larger ones fall back to the loop).
struct brick_linearizer
{
  const dataset_format* f = nullptr;
  int level = 0;
  std::vector<u64> t[3];
  brick_linearizer(const dataset_format& fmt, int l, v3 n);
  u64 operator()(v3 b) const
  {
    if ((unsigned)b.x < t[0].size() && (unsigned)b.y < t[1].size() && (unsigned)b.z < t[2].size())
      return t[0][(size_t)b.x] | t[1][(size_t)b.y] | t[2][(size_t)b.z];
    return linear_brick(*f, level, b);
  }
};
v3 spatial_brick(const dataset_format& f, int level, u64 linear);

// Addresses (Core/idx2Lookup.h:16-59).
inline u64 get_address(u64 brick, int brick_shift, int level, int subband, int bit_plane)
{
  return ((u64)level << 60) + ((brick >> brick_shift) << 18) + ((u64)(subband << 12)) +
         ((u64)bit_plane & 0xFFF);
}
u64 chunk_address(const dataset_format& f, u64 brick, int level, int subband, int bpkey);
u64 file_address(const dataset_format& f, u64 brick, int level);
std::string file_path(const dataset_format& f, u64 brick, int level);
inline uint32_t channel_key(int bpkey, int level, int subband)
{
  return ((uint32_t)bpkey << 16) + ((uint32_t)subband << 4) + (uint32_t)level;
}

// Output grid of a decode (Core/idx2Common.cpp:772 GetGrid).
grid output_grid(const dataset_format& f, const extent& ext);

// Metadata file (Core/idx2Common.cpp:150 WriteMetaFile, :183 ReadMetaFileFromBuffer).
std::string meta_text(const dataset_format& f, const params& p);
int parse_meta(const std::string& text, dataset_format* f);

// Depth-first traversal over a power-of-two box, in the order given by a transform
// order (Core/idx2Common.h:318-462 idx2_*Traverse). body(from3, address,
// item_in_parent, items_before) is called for each unit cell that intersects ext.
struct traverse_item
{
  v3 from3;
  u64 address = 0;
  int item_in_parent = 0;  // BrickInChunk / ChunkInFile
  i64 items_before = 0;    // NBricksBefore / NChunksBefore
};
template <typename F>
void traverse(u64 order, v3 from3, v3 dims3, const extent& ext, const extent& ext2, F&& body);

// Subband normalisation weights of one level (Core/Wavelet.cpp:111-137): w[s] for the nsubbands
// subbands; mask has bit s set where the weight applies (all but subband 0 below the coarsest).
void level_weights(const dataset_format& f, int level, double w[8], int* mask);

} // namespace idx2g

#include "format_traverse.h"
