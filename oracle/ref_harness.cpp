// Known-answer harness around the reference idx2 library (test infrastructure).
//
// Compiled by oracle/Makefile against the reference sources read in place; the
// result (oracle/_ref/libidx2_ref_harness.so) is loaded only by tests/ and by
// tests/golden/make_golden.py to pin the C restatement and the CUDA library.
// Every entry point calls the reference's own functions; nothing here restates
// an algorithm.
#include "idx2.h"
#include "Core/Zfp.h"
#include "Core/Function.h"
#include "Core/VarInt.h"
#include "Core/BitStream.h"
#include "Core/Wavelet.h"
#include "Core/idx2Lookup.h"

#include <string.h>

// the reference's vendored zstd 1.4.5 (compiled into the reference library)
extern "C" size_t ZSTD_compress(void* dst, size_t cap, const void* src, size_t n, int level);
extern "C" size_t ZSTD_compressBound(size_t n);

using namespace idx2;

namespace
{

// Finalize an idx2_file the way idx2App does (Applications/idx2App.cpp:217 SetParams).
int
SetUp(idx2_file* F, params* P, int nx, int ny, int nz, int dtype_code, int bx, int by, int bz,
      int nlevels, double tol, int bricks_per_chunk, int chunks_per_file, int files_per_dir,
      int bit_planes_per_chunk)
{
  snprintf(P->Meta.Name, sizeof(P->Meta.Name), "%s", "kat");
  snprintf(P->Meta.Field, sizeof(P->Meta.Field), "%s", "kat");
  P->Meta.Dims3 = v3i(nx, ny, nz);
  P->Meta.DType = dtype_code == 0 ? dtype::float32 : dtype::float64;
  P->BrickDims3 = v3i(bx, by, bz);
  P->NLevels = nlevels;
  P->Tolerance = tol;
  P->BricksPerChunk = bricks_per_chunk;
  P->ChunksPerFile = chunks_per_file;
  P->FilesPerDir = files_per_dir;
  P->BitPlanesPerChunk = bit_planes_per_chunk;
  SetName(F, P->Meta.Name);
  SetField(F, P->Meta.Field);
  SetVersion(F, P->Version);
  SetDimensions(F, P->Meta.Dims3);
  SetDataType(F, P->Meta.DType);
  SetBrickSize(F, P->BrickDims3);
  SetBricksPerChunk(F, P->BricksPerChunk);
  SetChunksPerFile(F, P->ChunksPerFile);
  SetBitPlanesPerChunk(F, P->BitPlanesPerChunk);
  SetNumLevels(F, (i8)P->NLevels);
  SetTolerance(F, P->Tolerance);
  SetFilesPerDirectory(F, P->FilesPerDir);
  SetDir(F, ".");
  auto Err = Finalize(F, P);
  return (int)Err.Code;
}

} // namespace

extern "C"
{

/* Finalize-derived format tables for one configuration.
   out_i32 layout per level L (stride 40):
     [0..2] NBricks3, [3..5] BricksPerChunk3s, [6..8] ChunksPerFile3s, [9..11] NChunks3,
     [12..14] NFiles3, [15] BricksPerChunk, [16] ChunksPerFile, [17] BricksPerFile,
     [18] BricksOrderStr.Len, [19] FilesDirsDepth.Len, [20..23] FilesDirsDepth,
     [24] ChunksOrderStr.Len, [25] FilesOrderStr.Len
   out_u64 per level (stride 6): BricksOrder, BricksOrderInChunk, ChunksOrderInFile,
     ChunksOrder, FilesOrder, TransformOrder
   out_str per level (stride 128*3): BricksOrderStr, ChunksOrderStr, FilesOrderStr.
   Returns the reference error code (0 = NoError). */
int
ref_finalize(int nx, int ny, int nz, int dtype_code, int bx, int by, int bz, int nlevels,
             double tol, int bricks_per_chunk, int chunks_per_file, int files_per_dir,
             int bit_planes_per_chunk, int* out_nlevels, int* out_i32, unsigned long long* out_u64,
             char* out_str, int* out_group3)
{
  idx2_file F;
  params P;
  int Code = SetUp(&F, &P, nx, ny, nz, dtype_code, bx, by, bz, nlevels, tol, bricks_per_chunk,
                   chunks_per_file, files_per_dir, bit_planes_per_chunk);
  if (Code != 0)
    return Code;
  *out_nlevels = F.NLevels;
  for (int D = 0; D < 3; ++D)
    out_group3[D] = F.GroupBrick3[D];
  for (int L = 0; L < F.NLevels; ++L)
  {
    int* O = out_i32 + 40 * L;
    for (int D = 0; D < 3; ++D)
    {
      O[0 + D] = F.NBricks3[L][D];
      O[3 + D] = F.BricksPerChunk3s[L][D];
      O[6 + D] = F.ChunksPerFile3s[L][D];
      O[9 + D] = F.NChunks3[L][D];
      O[12 + D] = F.NFiles3[L][D];
    }
    O[15] = F.BricksPerChunk[L];
    O[16] = F.ChunksPerFile[L];
    O[17] = F.BricksPerFile[L];
    O[18] = F.BricksOrderStr[L].Len;
    O[19] = F.FilesDirsDepth[L].Len;
    for (int K = 0; K < F.FilesDirsDepth[L].Len && K < 4; ++K)
      O[20 + K] = F.FilesDirsDepth[L][K];
    O[24] = F.ChunksOrderStr[L].Len;
    O[25] = F.FilesOrderStr[L].Len;
    unsigned long long* U = out_u64 + 6 * L;
    U[0] = F.BricksOrder[L];
    U[1] = F.BricksOrderInChunk[L];
    U[2] = F.ChunksOrderInFile[L];
    U[3] = F.ChunksOrder[L];
    U[4] = F.FilesOrder[L];
    U[5] = F.TransformOrder;
    char* S = out_str + 384 * L;
    memcpy(S, F.BricksOrderStr[L].Data, F.BricksOrderStr[L].Len);
    memcpy(S + 128, F.ChunksOrderStr[L].Data, F.ChunksOrderStr[L].Len);
    memcpy(S + 256, F.FilesOrderStr[L].Data, F.FilesOrderStr[L].Len);
  }
  Dealloc(&F);
  return 0;
}

/* Decode-side subband masks and spacings (Core/idx2Common.cpp:403 BuildSubbands with a
   downsampling factor). out_masks[L]; out_spacing[(L*8+Sb)*3+D]. */
int
ref_decode_masks(int nx, int ny, int nz, int bx, int by, int bz, int nlevels, int dsx, int dsy,
                 int dsz, int* out_masks, int* out_spacing)
{
  idx2_file F;
  params P;
  SetDownsamplingFactor(&F, v3i(dsx, dsy, dsz));
  P.DownsamplingFactor3 = v3i(dsx, dsy, dsz);
  int Code = SetUp(&F, &P, nx, ny, nz, 1, bx, by, bz, nlevels, 1e-3, 4096, 64, 64, 1);
  if (Code != 0)
    return Code;
  for (int L = 0; L < F.NLevels; ++L)
  {
    out_masks[L] = F.DecodeSubbandMasks[L];
    for (int Sb = 0; Sb < (int)Size(F.Subbands); ++Sb)
      for (int D = 0; D < 3; ++D)
        out_spacing[(L * 8 + Sb) * 3 + D] = F.DecodeSubbandSpacings[L][Sb][D];
  }
  Dealloc(&F);
  return 0;
}

/* Brick forward transform exactly as EncodeBrick does it (Core/idx2Encode.cpp:291-295):
   ExtrapolateCdf53 on the valid dims, then one-level ForwardCdf53 with normalisation.
   bz == 1 selects 2D bricks (32x32x1 -> 33x33x1). The brick buffer is nx*ny*nz doubles
   with nx=ny=33 and nz=33 (3D) or 1 (2D), x fastest. */
int
ref_brick_forward(double* brick, int bz, int vx, int vy, int vz, int level, int coarsest)
{
  idx2_file F;
  params P;
  int Code = SetUp(&F, &P, 256, 256, bz == 1 ? 1 : 256, 1, 32, 32, bz, 2, 1e-3, 4096, 64, 64, 1);
  if (Code != 0)
    return Code;
  volume Vol(buffer((byte*)brick, Prod(F.BrickDimsExt3) * (i64)sizeof(f64)), F.BrickDimsExt3,
             dtype::float64);
  ExtrapolateCdf53(v3i(vx, vy, vz), F.TransformOrder, &Vol);
  ForwardCdf53(F.BrickDimsExt3, level, F.Subbands, F.TransformDetails, &Vol, coarsest != 0);
  Dealloc(&F);
  return 0;
}

/* Only the extrapolation round trip (Core/Wavelet.cpp:68). */
int
ref_brick_extrapolate(double* brick, int bz, int vx, int vy, int vz)
{
  idx2_file F;
  params P;
  int Code = SetUp(&F, &P, 256, 256, bz == 1 ? 1 : 256, 1, 32, 32, bz, 2, 1e-3, 4096, 64, 64, 1);
  if (Code != 0)
    return Code;
  volume Vol(buffer((byte*)brick, Prod(F.BrickDimsExt3) * (i64)sizeof(f64)), F.BrickDimsExt3,
             dtype::float64);
  ExtrapolateCdf53(v3i(vx, vy, vz), F.TransformOrder, &Vol);
  Dealloc(&F);
  return 0;
}

/* Brick inverse transform as DecodeBrick does it (Core/idx2Decode.cpp:316-317). */
int
ref_brick_inverse(double* brick, int bz, int level, int coarsest)
{
  idx2_file F;
  params P;
  int Code = SetUp(&F, &P, 256, 256, bz == 1 ? 1 : 256, 1, 32, 32, bz, 2, 1e-3, 4096, 64, 64, 1);
  if (Code != 0)
    return Code;
  volume Vol(buffer((byte*)brick, Prod(F.BrickDimsExt3) * (i64)sizeof(f64)), F.BrickDimsExt3,
             dtype::float64);
  InverseCdf53(F.BrickDimsExt3, level, F.Subbands, F.TransformDetails, &Vol, coarsest != 0);
  Dealloc(&F);
  return 0;
}

/* One block through QuantizeF32/F64, ForwardZfp, ForwardShuffle and the bit-plane loop of
   EncodeSubbandBlocks (Core/idx2Encode.cpp:176-254), each plane coded into its own stream.
   vals: 4^ndims doubles. Outputs: emax, ucoeffs[4^ndims] (shuffled negabinary), and for each
   coded plane k (in coding order): plane_bp[k], plane_nin[k], plane_bits[k] (bit length) and
   plane_words[k*4..k*4+3] (the bits, LSB first). Returns the number of coded planes. */
int
ref_block_encode(const double* vals, int ndims, int is_f32, double tol, int bpc, int* emax,
                 unsigned long long* ucoeffs, int* plane_bp, int* plane_nin, int* plane_bits,
                 unsigned long long* plane_words)
{
  const i8 NBitPlanes = 64;
  const int NVals = 1 << (2 * ndims);
  const i8 Prec = NBitPlanes - 1 - ndims;
  f64 BlockFloats[64];
  u64 BlockUInts[64];
  for (int I = 0; I < NVals; ++I)
    BlockFloats[I] = vals[I];
  buffer_t BufFloats(BlockFloats, NVals);
  buffer_t BufInts((i64*)BlockFloats, NVals);
  const i16 EMax = !is_f32 ? (i16)QuantizeF64(Prec, BufFloats, &BufInts)
                           : (i16)QuantizeF32(Prec, BufFloats, &BufInts);
  ForwardZfp((i64*)BlockFloats, ndims);
  ForwardShuffle((i64*)BlockFloats, BlockUInts, ndims);
  *emax = EMax;
  for (int I = 0; I < NVals; ++I)
    ucoeffs[I] = BlockUInts[I];
  i8 N = 0;
  i8 EndBitPlane = Min(i8(is_f32 ? 32 : 64), NBitPlanes);
  int K = 0;
  for (int Bp = NBitPlanes - 1; Bp >= NBitPlanes - EndBitPlane; --Bp)
  {
    i16 RealBp = Bp + EMax;
    bool TooHighPrecision = NBitPlanes - 6 > RealBp - Exponent(tol) + 1;
    if (TooHighPrecision && (RealBp + BitPlaneKeyBias_) % bpc == 0)
      break;
    bitstream Bs;
    InitWrite(&Bs, 256);
    plane_bp[K] = Bp;
    plane_nin[K] = N;
    Encode(BlockUInts, NVals, Bp, N, &Bs);
    plane_bits[K] = (int)BitSize(Bs);
    Flush(&Bs);
    memset(plane_words + 4 * K, 0, 32);
    memcpy(plane_words + 4 * K, Bs.Stream.Data, Size(Bs));
    Dealloc(&Bs);
    ++K;
  }
  return K;
}

/* Decode the coded planes of one block back to the dequantised doubles, mirroring
   DecodeSubband's per-block tail (Core/idx2Decode.cpp:141-227) with every plane read from its
   own stream. Returns 0. */
int
ref_block_decode(int ndims, int emax, int nplanes, const int* plane_bp,
                 const unsigned long long* plane_words, double* out_vals)
{
  const int NVals = 1 << (2 * ndims);
  const int Prec = 64 - 1 - ndims;
  u64 BlockUInts[64] = {};
  f64 BlockFloats[64];
  i8 N = 0;
  for (int K = 0; K < nplanes; ++K)
  {
    u64 Words[5] = { plane_words[4 * K], plane_words[4 * K + 1], plane_words[4 * K + 2],
                     plane_words[4 * K + 3], 0 };
    bitstream Bs;
    InitRead(&Bs, buffer((byte*)Words, sizeof(Words)));
    Decode(BlockUInts, NVals, plane_bp[K], N, &Bs, false);
  }
  buffer_t BufFloats(BlockFloats, NVals);
  buffer_t BufInts((i64*)BlockFloats, NVals);
  InverseShuffle(BlockUInts, (i64*)BlockFloats, ndims);
  InverseZfp((i64*)BlockFloats, ndims);
  Dequantize(emax, Prec, BufInts, &BufFloats);
  for (int I = 0; I < NVals; ++I)
    out_vals[I] = BlockFloats[I];
  return 0;
}

/* Variable-length integer codes (Core/VarInt.h:14,82): writes varbyte(vals[i]) for
   i < n_var, then unary(vals[i]) for the rest, into one stream. Returns the bit length. */
long long
ref_varint_stream(const unsigned long long* vals, int n_var, int n_total, unsigned char* out,
                  long long out_cap)
{
  bitstream Bs;
  InitWrite(&Bs, out_cap + 64);
  for (int I = 0; I < n_total; ++I)
  {
    GrowToAccomodate(&Bs, 64 + (I < n_var ? 0 : (i64)(vals[I] / 8)));
    if (I < n_var)
      WriteVarByte(&Bs, vals[I]);
    else
      WriteUnary(&Bs, (u32)vals[I]);
  }
  long long Bits = BitSize(Bs);
  Flush(&Bs);
  memcpy(out, Bs.Stream.Data, Min((i64)out_cap, Size(Bs)));
  Dealloc(&Bs);
  return Bits;
}

/* Morton helpers (Core/BitOps.h:249,282). */
unsigned int
ref_encode_morton3(unsigned int x, unsigned int y, unsigned int z)
{
  return EncodeMorton3(v3<u32>(x, y, z));
}

/* Output grid of a decode request (Core/idx2Common.cpp:772 GetGrid). out: from3, dims3,
   strd3. */
int
ref_output_grid(int nx, int ny, int nz, int bx, int by, int bz, int nlevels, int fx, int fy,
                int fz, int lx, int ly, int lz, int dsx, int dsy, int dsz, int* out9)
{
  idx2_file F;
  params P;
  SetDownsamplingFactor(&F, v3i(dsx, dsy, dsz));
  P.DownsamplingFactor3 = v3i(dsx, dsy, dsz);
  int Code = SetUp(&F, &P, nx, ny, nz, 1, bx, by, bz, nlevels, 1e-3, 4096, 64, 64, 1);
  if (Code != 0)
    return Code;
  extent Ext(v3i(fx, fy, fz), v3i(lx - fx + 1, ly - fy + 1, lz - fz + 1));
  grid G = GetGrid(F, Ext);
  v3i A = From(G), B = Dims(G), C = Strd(G);
  for (int D = 0; D < 3; ++D)
  {
    out9[D] = A[D];
    out9[3 + D] = B[D];
    out9[6 + D] = C[D];
  }
  Dealloc(&F);
  return 0;
}

/* The reference's exponent-chunk / address-table compression (Core/idx2Encode.cpp:23
   CompressBufZstd): ZSTD_compress at level 1 of the vendored zstd 1.4.5. Returns the frame size
   (0 for an empty input, as CompressBufZstd writes nothing then). */
size_t
ref_zstd_compress(const void* src, size_t n, void* dst, size_t cap)
{
  if (n == 0)
    return 0;
  if (cap < ZSTD_compressBound(n))
    return 0;
  return ZSTD_compress(dst, cap, src, n, 1);
}

size_t
ref_zstd_bound(size_t n)
{
  return ZSTD_compressBound(n);
}

} // extern "C"
