// Level-1 zstd frame compressor whose frames are byte-identical to those of zstd 1.4.5's
// ZSTD_compress(dst, cap, src, n, 1), the call the reference makes for exponent chunks and
// chunk-address tables (Core/idx2Encode.cpp:23-37 CompressBufZstd, vendored zstd 1.4.5 at
// Core/zstd/zstd.h:73-75). zstd's format fixes how a frame decodes, not which frame a
// compressor writes; byte parity of the data files therefore needs the same match finder,
// entropy-table choices and block decisions as that release, which this file restates:
// the fast strategy's double-position hash search with repeat offsets, Huffman literals
// (tree, height limit, weight header, 1 or 4 streams, table reuse across blocks), FSE tables
// for literal lengths / match lengths / offsets (default, RLE or normalised counts), and the
// raw / RLE / compressed block choice. Pure host C++; decompression stays with any zstd
// library (the format is version independent).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace idx2g
{
namespace zstd145
{

// Upper bound of a frame's size for n input bytes (the format's compress bound).
size_t compress_bound(size_t n);

// One frame of src[0, n) at level 1, appended to out (out is cleared first). n = 0 gives
// the empty frame.
void compress(const uint8_t* src, size_t n, std::vector<uint8_t>* out);

} // namespace zstd145
} // namespace idx2g
