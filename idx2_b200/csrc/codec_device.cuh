// Device-side building blocks of the idx2 brick codec for sm_100a.
//
// Arithmetic follows the reference operation for operation (FP64 lifting in the
// reference's order, integer zfp lifting, negabinary shuffle), so results are
// bit-identical to the CPU implementation; the file is compiled with
// --fmad=false so no expression is contracted into an FMA.
#pragma once

#include <cstdint>

namespace idx2g
{
namespace dev
{

constexpr int kExt = 33;           // extended brick side (32 + 1)
constexpr int kBrick3D = 33 * 33 * 33;
constexpr int kBrick2D = 33 * 33;

struct dgrid
{
  int from[3], dims[3], strd[3];
};

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

// One CDF5/3 lifting sweep along axis a over the lines of grid G, split over the
// threads of the CTA (Core/Wavelet.h:178 FLiftCdf53, :250 ILiftCdf53, lift_option
// Normal). Each thread runs whole lines in the reference's sample order.
inline __device__ void lift_sweep(double* F, const int N[3], const dgrid& G, const int M[3], int a,
                           bool forward)
{
  const int P = G.from[a], D = G.dims[a], S = G.strd[a];
  if (D == 1)
    return;
  const int b = a == 0 ? 1 : 0;
  const int c = a == 2 ? 1 : 2;
  const int st[3] = { 1, N[0], N[0] * N[1] };
  const int x0 = imin(P + S * D, M[a]);
  const int x1 = imin(P + S * (D - 1), M[a]);
  const int x2 = P + S * (D - 2);
  const int x3 = P + S * (D - 3);
  const bool ext = (D % 2) == 0;
  const int s = st[a];
  const int nlines = G.dims[b] * G.dims[c];
  for (int li = threadIdx.x; li < nlines; li += blockDim.x)
  {
    const int u = G.from[b] + (li % G.dims[b]) * G.strd[b];
    const int v = G.from[c] + (li / G.dims[b]) * G.strd[c];
    double* L = F + imin(u, M[b]) * st[b] + imin(v, M[c]) * st[c];
#define AT(t) L[(t) * s]
    if (forward)
    {
      if (ext)
      {
        double A = AT(x2), B = AT(x1);
        AT(x0) = __dsub_rn(__dmul_rn(2.0, B), A);
      }
      for (int x = P + S; x < P + S * (D - 2); x += 2 * S)
        AT(x) = __dsub_rn(AT(x), __dmul_rn(__dadd_rn(AT(x - S), AT(x + S)), 0.5));
      if (!ext)
        AT(x2) = __dsub_rn(AT(x2), __dmul_rn(__dadd_rn(AT(x1), AT(x3)), 0.5));
      else if (x1 < M[a])
        AT(x1) = 0;
      for (int x = P + S; x < P + S * (D - 2); x += 2 * S)
      {
        double V = __dmul_rn(AT(x), 0.25);
        AT(x - S) = __dadd_rn(AT(x - S), V);
        AT(x + S) = __dadd_rn(AT(x + S), V);
      }
      if (!ext)
      {
        double V = __dmul_rn(AT(x2), 0.25);
        AT(x3) = __dadd_rn(AT(x3), V);
        AT(x1) = __dadd_rn(AT(x1), V);
      }
    }
    else
    {
      for (int x = P + S; x < P + S * (D - 2); x += 2 * S)
      {
        double V = __dmul_rn(AT(x), 0.25);
        AT(x - S) = __dsub_rn(AT(x - S), V);
        AT(x + S) = __dsub_rn(AT(x + S), V);
      }
      if (!ext)
      {
        double V = __dmul_rn(AT(x2), 0.25);
        AT(x3) = __dsub_rn(AT(x3), V);
        AT(x1) = __dsub_rn(AT(x1), V);
      }
      else
      {
        double A = AT(x0), B = AT(x2);
        AT(x1) = __dmul_rn(__dadd_rn(A, B), 0.5);
      }
      for (int x = P + S; x < P + S * (D - 2); x += 2 * S)
        AT(x) = __dadd_rn(AT(x), __dmul_rn(__dadd_rn(AT(x - S), AT(x + S)), 0.5));
      if (!ext)
        AT(x2) = __dadd_rn(AT(x2), __dmul_rn(__dadd_rn(AT(x1), AT(x3)), 0.5));
    }
#undef AT
  }
}

// One CDF5/3 line held in registers: samples at positions k*S (k < D) plus, for even D,
// the extrapolated sample in slot D. Same operations and order as lift_sweep (the reference's
// clamps to M never apply to the grids of the brick transforms: every position is <= 32).
template <bool FWD>
__device__ __forceinline__ void lift_regs(double (&v)[33], int D)
{
  const bool ext = (D % 2) == 0;
  if (FWD)
  {
    if (ext)
    {
#pragma unroll
      for (int k = 2; k < 33; ++k)
        if (k == D)
          v[k] = __dsub_rn(__dmul_rn(2.0, v[k - 1]), v[k - 2]);
    }
#pragma unroll
    for (int k = 1; k < 31; k += 2)
      if (k < D - 2)
        v[k] = __dsub_rn(v[k], __dmul_rn(__dadd_rn(v[k - 1], v[k + 1]), 0.5));
#pragma unroll
    for (int k = 1; k < 32; ++k)
    {
      if (!ext && k == D - 2)
        v[k] = __dsub_rn(v[k], __dmul_rn(__dadd_rn(v[k + 1], v[k - 1]), 0.5));
      if (ext && k == D - 1)
        v[k] = 0.0;
    }
#pragma unroll
    for (int k = 1; k < 31; k += 2)
      if (k < D - 2)
      {
        double V = __dmul_rn(v[k], 0.25);
        v[k - 1] = __dadd_rn(v[k - 1], V);
        v[k + 1] = __dadd_rn(v[k + 1], V);
      }
    if (!ext)
    {
#pragma unroll
      for (int k = 1; k < 32; ++k)
        if (k == D - 2)
        {
          double V = __dmul_rn(v[k], 0.25);
          v[k - 1] = __dadd_rn(v[k - 1], V);
          v[k + 1] = __dadd_rn(v[k + 1], V);
        }
    }
  }
  else
  {
#pragma unroll
    for (int k = 1; k < 31; k += 2)
      if (k < D - 2)
      {
        double V = __dmul_rn(v[k], 0.25);
        v[k - 1] = __dsub_rn(v[k - 1], V);
        v[k + 1] = __dsub_rn(v[k + 1], V);
      }
#pragma unroll
    for (int k = 1; k < 32; ++k)
    {
      if (!ext && k == D - 2)
      {
        double V = __dmul_rn(v[k], 0.25);
        v[k - 1] = __dsub_rn(v[k - 1], V);
        v[k + 1] = __dsub_rn(v[k + 1], V);
      }
      if (ext && k == D - 1)
        v[k] = __dmul_rn(__dadd_rn(v[k + 1], v[k - 1]), 0.5);
    }
#pragma unroll
    for (int k = 1; k < 31; k += 2)
      if (k < D - 2)
        v[k] = __dadd_rn(v[k], __dmul_rn(__dadd_rn(v[k - 1], v[k + 1]), 0.5));
    if (!ext)
    {
#pragma unroll
      for (int k = 1; k < 32; ++k)
        if (k == D - 2)
          v[k] = __dadd_rn(v[k], __dmul_rn(__dadd_rn(v[k + 1], v[k - 1]), 0.5));
    }
  }
}

// One line with a compile-time length D: load, lift in registers, store. The inverse reads
// the extrapolated slot D of an even-length line, the forward writes it.
template <int D, bool FWD>
__device__ __forceinline__ void lift_line_fixed(double* L, int s)
{
  constexpr bool ext = (D % 2) == 0;
  constexpr int nload = D + (ext && !FWD ? 1 : 0);
  constexpr int nstore = D + (ext && FWD ? 1 : 0);
  double v[33];
#pragma unroll
  for (int k = 0; k < 33; ++k)
    v[k] = k < nload ? L[k * s] : 0.0;
  lift_regs<FWD>(v, D);
#pragma unroll
  for (int k = 0; k < nstore; ++k)
    L[k * s] = v[k];
}

// The same with a compile-time stride (immediate offsets, no address registers).
template <int D, bool FWD, int STRIDE>
__device__ __forceinline__ void lift_line_strided(double* L)
{
  constexpr bool ext = (D % 2) == 0;
  constexpr int nload = D + (ext && !FWD ? 1 : 0);
  constexpr int nstore = D + (ext && FWD ? 1 : 0);
  double v[33];
#pragma unroll
  for (int k = 0; k < 33; ++k)
    v[k] = k < nload ? L[k * STRIDE] : 0.0;
  lift_regs<FWD>(v, D);
#pragma unroll
  for (int k = 0; k < nstore; ++k)
    L[k * STRIDE] = v[k];
}

// The lines of a sweep with a compile-time length and stride: line li starts at
// (li % ub) * sb + (li / ub) * sc.
template <int D, bool FWD, int STRIDE>
__device__ __forceinline__ void sweep_strided(double* F, int nlines, int ub, int sb, int sc)
{
  for (int li = threadIdx.x; li < nlines; li += blockDim.x)
    lift_line_strided<D, FWD, STRIDE>(F + (li % ub) * sb + (li / ub) * sc);
}

template <bool FWD>
__device__ __noinline__ void lift_line(double* L, int s, int D)
{
  switch (D)
  {
#define IDX2G_LIFT_CASE(n) \
  case n:                  \
    lift_line_fixed<n, FWD>(L, s); \
    break;
    IDX2G_LIFT_CASE(2) IDX2G_LIFT_CASE(3) IDX2G_LIFT_CASE(4) IDX2G_LIFT_CASE(5) IDX2G_LIFT_CASE(6)
    IDX2G_LIFT_CASE(7) IDX2G_LIFT_CASE(8) IDX2G_LIFT_CASE(9) IDX2G_LIFT_CASE(10) IDX2G_LIFT_CASE(11)
    IDX2G_LIFT_CASE(12) IDX2G_LIFT_CASE(13) IDX2G_LIFT_CASE(14) IDX2G_LIFT_CASE(15) IDX2G_LIFT_CASE(16)
    IDX2G_LIFT_CASE(17) IDX2G_LIFT_CASE(18) IDX2G_LIFT_CASE(19) IDX2G_LIFT_CASE(20) IDX2G_LIFT_CASE(21)
    IDX2G_LIFT_CASE(22) IDX2G_LIFT_CASE(23) IDX2G_LIFT_CASE(24) IDX2G_LIFT_CASE(25) IDX2G_LIFT_CASE(26)
    IDX2G_LIFT_CASE(27) IDX2G_LIFT_CASE(28) IDX2G_LIFT_CASE(29) IDX2G_LIFT_CASE(30) IDX2G_LIFT_CASE(31)
    IDX2G_LIFT_CASE(32) IDX2G_LIFT_CASE(33)
#undef IDX2G_LIFT_CASE
    default:
      break;
  }
}

// A lifting sweep over the lines of G with each line in registers.
template <bool FWD>
__device__ void lift_sweep_regs(double* F, const int N[3], const dgrid& G, int a)
{
  const int D = G.dims[a], S = G.strd[a];
  if (D == 1)
    return;
  const int b = a == 0 ? 1 : 0;
  const int c = a == 2 ? 1 : 2;
  const int st[3] = { 1, N[0], N[0] * N[1] };
  const int s = st[a] * S;
  const int nlines = G.dims[b] * G.dims[c];
  // The first-level sweeps of 33^3 bricks (line lengths 32 and 33 with strides 1, 33, 1089)
  // run with compile-time strides; other sweeps (edge bricks) go through the out-of-line switch.
  if (S == 1 && N[0] == 33 && N[1] == 33 && (D == 32 || D == 33))
  {
    const int ub = G.dims[b], sb = G.strd[b] * st[b], sc = G.strd[c] * st[c];
    if (D == 33)
    {
      if (a == 0)
        sweep_strided<33, FWD, 1>(F, nlines, ub, sb, sc);
      else if (a == 1)
        sweep_strided<33, FWD, 33>(F, nlines, ub, sb, sc);
      else
        sweep_strided<33, FWD, 1089>(F, nlines, ub, sb, sc);
    }
    else
    {
      if (a == 0)
        sweep_strided<32, FWD, 1>(F, nlines, ub, sb, sc);
      else if (a == 1)
        sweep_strided<32, FWD, 33>(F, nlines, ub, sb, sc);
      else
        sweep_strided<32, FWD, 1089>(F, nlines, ub, sb, sc);
    }
    return;
  }
  for (int li = threadIdx.x; li < nlines; li += blockDim.x)
  {
    const int u = (li % G.dims[b]) * G.strd[b];
    const int w = (li / G.dims[b]) * G.strd[c];
    lift_line<FWD>(F + u * st[b] + w * st[c], s, D);
  }
}

// The grid sequence of the multi-level transform on the first dims3 samples
// (Core/Wavelet.cpp:210 ForwardCdf53 / :304 InverseCdf53 with a transform order).
struct lift_stack
{
  dgrid g[16];
  int8_t axis[16];
  int n;
  int coarse;  // first sweep of the second level: from there on every position is even
};

inline __device__ void build_stack(const int dims3[3], int nlevels, uint64_t order, lift_stack* st)
{
  int level = 0;
  uint64_t prev = order;
  int D3[3] = { dims3[0], dims3[1], dims3[2] };
  int R3[3] = { dims3[0], dims3[1], dims3[2] };
  int S3[3] = { 1, 1, 1 };
  dgrid G;
  for (int k = 0; k < 3; ++k)
  {
    G.from[k] = 0;
    G.dims[k] = dims3[k];
    G.strd[k] = 1;
  }
  st->n = 0;
  st->coarse = -1;
  while (level < nlevels)
  {
    int d = (int)(order & 3);
    order >>= 2;
    if (d == 3)
    {
      if (level == 0)
        st->coarse = st->n;
      if (order == 3)
        order = prev;
      else
        prev = order;
      for (int k = 0; k < 3; ++k)
      {
        G.strd[k] = S3[k];
        G.dims[k] = D3[k];
        R3[k] = D3[k];
      }
      ++level;
    }
    else
    {
      if (st->n < 16)
      {
        st->g[st->n] = G;
        st->axis[st->n] = (int8_t)d;
        ++st->n;
      }
      R3[d] = D3[d] + (D3[d] % 2 == 0);
      for (int k = 0; k < 3; ++k)
        G.dims[k] = R3[k];
      D3[d] = (R3[d] + 1) >> 1;
      S3[d] <<= 1;
    }
  }
  if (st->coarse < 0)
    st->coarse = st->n;
}

// A grid of even positions mapped onto the half-resolution lattice (position p -> p / 2);
// axes of one sample keep stride 1.
__device__ __forceinline__ dgrid half_grid(const dgrid& g)
{
  dgrid h;
  for (int k = 0; k < 3; ++k)
  {
    h.from[k] = g.from[k] >> 1;
    h.dims[k] = g.dims[k];
    h.strd[k] = g.strd[k] >= 2 ? g.strd[k] >> 1 : 1;
  }
  return h;
}

// Core/Math.h:524 Exponent<f64>, via the IEEE exponent field (glibc frexp semantics:
// infinities and NaNs give 0).
__device__ __forceinline__ int exponent_f64(double v)
{
  if (v == 0)
    return -1023;
  long long bits = __double_as_longlong(v);
  int e = (int)((bits >> 52) & 0x7ff);
  if (e == 0x7ff)
    return 0;
  if (e == 0)
    return -1022;  // denormal: frexp gives <= -1022, clamped to 1 - bias
  return e - 1022;
}

__device__ __forceinline__ int exponent_f32(float v)
{
  if (v == 0)
    return -127;
  int bits = __float_as_int(v);
  int e = (bits >> 23) & 0xff;
  if (e == 0xff)
    return 0;
  if (e == 0)
    return -126;
  return e - 126;
}

// 2^k as a double (ldexp(1, k)).
__device__ __forceinline__ double pow2(int k)
{
  if (k > 1023)
    return __longlong_as_double(0x7ff0000000000000ll);
  if (k >= -1022)
    return __longlong_as_double((long long)(k + 1023) << 52);
  if (k >= -1074)
    return __longlong_as_double(1ll << (k + 1074));
  return 0.0;
}

// Truncating double -> int64 with the x86 cvttsd2si result for NaN / out of range.
__device__ __forceinline__ long long trunc_i64(double v)
{
  if (!(v < 9223372036854775808.0 && v >= -9223372036854775808.0))
    return (long long)0x8000000000000000ull;
  return __double2ll_rz(v);
}

// zfp 4-point lifting (Core/Zfp.h:145 FLift, :181 ILift), on four elements anywhere.
__device__ __forceinline__ void fwd_lift4_at(long long* p0, long long* p1, long long* p2, long long* p3)
{
  long long x = *p0, y = *p1, z = *p2, w = *p3;
  x += w;
  x >>= 1;
  w -= x;
  z += y;
  z >>= 1;
  y -= z;
  x += z;
  x >>= 1;
  z -= x;
  w += y;
  w >>= 1;
  y -= w;
  w += y >> 1;
  y -= w >> 1;
  *p0 = x;
  *p1 = y;
  *p2 = z;
  *p3 = w;
}

__device__ __forceinline__ void fwd_lift4(long long* p, int s) { fwd_lift4_at(p, p + s, p + 2 * s, p + 3 * s); }

__device__ __forceinline__ void inv_lift4_at(long long* p0, long long* p1, long long* p2, long long* p3)
{
  long long x = *p0, y = *p1, z = *p2, w = *p3;
  y += w >> 1;
  w -= y >> 1;
  y += w;
  w = (long long)((unsigned long long)w << 1);
  w -= y;
  z += x;
  x = (long long)((unsigned long long)x << 1);
  x -= z;
  y += z;
  z = (long long)((unsigned long long)z << 1);
  z -= y;
  w += x;
  x = (long long)((unsigned long long)x << 1);
  x -= w;
  *p0 = x;
  *p1 = y;
  *p2 = z;
  *p3 = w;
}

__device__ __forceinline__ void inv_lift4(long long* p, int s) { inv_lift4_at(p, p + s, p + 2 * s, p + 3 * s); }

// 32 x 32 bit-matrix transpose across a warp: lane r holds row r; afterwards lane c holds
// column c (bit r of the result = bit c of row r). Five exchange rounds of halving blocks.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane)
{
  const uint32_t m[5] = { 0x0000ffffu, 0x00ff00ffu, 0x0f0f0f0fu, 0x33333333u, 0x55555555u };
#pragma unroll
  for (int i = 0; i < 5; ++i)
  {
    const int j = 16 >> i;
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? ((x & ~m[i]) | ((y & ~m[i]) >> j)) : ((x & m[i]) | ((y & m[i]) << j));
  }
  return x;
}

// Warp-cooperative forward zfp transform of one block held in shared memory
// (Core/Zfp.h:262 ForwardZfp(P, D)): lines of each pass go to different lanes.
__device__ __forceinline__ void warp_fwd_zfp(long long* q, int nd, int lane)
{
  if (nd == 3)
  {
    if (lane < 16)
      fwd_lift4(q + 4 * (lane & 3) + 16 * (lane >> 2), 1);
    __syncwarp();
    if (lane < 16)
      fwd_lift4(q + 16 * (lane & 3) + (lane >> 2), 4);
    __syncwarp();
    if (lane < 16)
      fwd_lift4(q + (lane & 3) + 4 * (lane >> 2), 16);
    __syncwarp();
  }
  else if (nd == 2)
  {
    if (lane < 4)
      fwd_lift4(q + 4 * lane, 1);
    __syncwarp();
    if (lane < 4)
      fwd_lift4(q + lane, 4);
    __syncwarp();
  }
  else if (nd == 1)
  {
    if (lane == 0)
      fwd_lift4(q, 1);
    __syncwarp();
  }
}

__device__ __forceinline__ void warp_inv_zfp(long long* q, int nd, int lane)
{
  if (nd == 3)
  {
    if (lane < 16)
      inv_lift4(q + (lane & 3) + 4 * (lane >> 2), 16);
    __syncwarp();
    if (lane < 16)
      inv_lift4(q + 16 * (lane & 3) + (lane >> 2), 4);
    __syncwarp();
    if (lane < 16)
      inv_lift4(q + 4 * (lane & 3) + 16 * (lane >> 2), 1);
    __syncwarp();
  }
  else if (nd == 2)
  {
    if (lane < 4)
      inv_lift4(q + lane, 4);
    __syncwarp();
    if (lane < 4)
      inv_lift4(q + 4 * lane, 1);
    __syncwarp();
  }
  else if (nd == 1)
  {
    if (lane == 0)
      inv_lift4(q, 1);
    __syncwarp();
  }
}

constexpr unsigned long long kNegaMask = 0xaaaaaaaaaaaaaaaaull;

// Coefficient order by total sequency (Core/Zfp.h:419 Perm3, :498 Perm2), as flat
// indices x + 4y + 16z into the block.
static __constant__ uint8_t kPerm3d[64] = {
  0,  1,  4,  16, 20, 17, 5,  2,  8,  32, 21, 6,  18, 24, 9,  33, 36, 3,  12, 48, 22, 25,
  37, 40, 34, 10, 7,  19, 28, 13, 49, 52, 41, 38, 26, 23, 29, 53, 11, 35, 44, 14, 50, 56,
  42, 27, 39, 45, 30, 54, 57, 60, 51, 15, 43, 46, 58, 61, 55, 31, 62, 59, 47, 63
};
static __constant__ uint8_t kPerm2d[16] = { 0, 1, 4, 5, 2, 8, 6, 9, 3, 12, 10, 7, 13, 11, 14, 15 };

__device__ __forceinline__ int perm(int nd, int i)
{
  return nd == 3 ? (int)kPerm3d[i] : (nd == 2 ? (int)kPerm2d[i] : i);
}

// Number of coded planes of a block (Core/idx2Encode.cpp:195-206, BitPlanesPerChunk 1):
// planes 63 .. lowbp with lowbp = max(64 - EndBitPlane, 57 + Exponent(tol) - EMax).
__device__ __forceinline__ int coded_planes(int emax, int etol, int end_bp)
{
  int low = 57 + etol - emax;
  int lim = 64 - end_bp;
  low = low > lim ? low : lim;
  return low <= 63 ? 64 - low : 0;
}

// Number of coded planes of a block with BitPlanesPerChunk bpc (Core/idx2Encode.cpp:195-206,
// Core/idx2Decode.cpp:144-162): planes from 63 down, stopping at the first plane past the
// tolerance whose key value RealBp + 1024 is a multiple of bpc; the channel key of plane Bp is
// (Bp + EMax + 1024) / bpc.
__device__ __forceinline__ int coded_planes(int emax, int etol, int end_bp, int bpc)
{
  if (bpc == 1)
    return coded_planes(emax, etol, end_bp);
  int np = 0;
  for (int bp = 63; bp >= 64 - end_bp; --bp)
  {
    const int realbp = bp + emax;
    if (58 > realbp - etol + 1 && ((realbp + 1024) % bpc) == 0)
      break;
    ++np;
  }
  return np;
}

// Channel key of plane kk (0 = plane 63) of a block whose top plane has key value top =
// EMax + 63 + 1024.
__device__ __forceinline__ int plane_key(int top, int kk, int bpc)
{
  return bpc == 1 ? top - kk : (top - kk) / bpc;  // (the common case without a division)
}

// Planes [kk0, kk1] of a block (np coded planes, top as above) that are in channel key; empty
// when kk0 > kk1. Key values of coded planes are non-negative (checked by the kernels).
__device__ __forceinline__ void key_planes(int top, int np, int key, int bpc, int& kk0, int& kk1)
{
  kk1 = top - key * bpc;
  kk0 = kk1 - (bpc - 1);
  kk0 = kk0 < 0 ? 0 : kk0;
  kk1 = kk1 > np - 1 ? np - 1 : kk1;
}

// Bit length of one plane of the group-test coder (Core/Zfp.h:771 Encode<u64>) with
// nin significant coefficients before the plane and plane bits x.
__device__ __forceinline__ int plane_bits(unsigned long long x, int nin, int nvals)
{
  unsigned long long r = nin < 64 ? (x >> nin) : 0ull;
  if (r == 0)
    return nin + (nin < nvals ? 1 : 0);
  int k = __popcll(r);
  int s = 63 - __clzll(x);
  return k + s + (s < nvals - 1 ? 2 : 0);
}

__device__ __forceinline__ int plane_nout(unsigned long long x, int nin)
{
  int m = x ? 64 - __clzll(x) : 0;
  return m > nin ? m : nin;
}

// OR nbits (<= 32) of v into a zero-initialised bit stream at bit position pos.
__device__ __forceinline__ void or_bits(uint32_t* words, unsigned long long pos, uint32_t v, int n)
{
  if (n <= 0 || v == 0)
    return;
  if (n < 32)
    v &= (1u << n) - 1u;
  unsigned long long w = pos >> 5;
  int sh = (int)(pos & 31);
  atomicOr(words + w, v << sh);
  if (sh + n > 32)
    atomicOr(words + w + 1, v >> (32 - sh));
}

// Write the bits of one plane (Core/Zfp.h:771 Encode<u64>) at bit position pos of a
// zero-initialised stream. Only one-bits are stored.
inline __device__ void write_plane(uint32_t* words, unsigned long long pos, unsigned long long x, int nin,
                            int nvals)
{
  // raw bits of the already significant coefficients
  int n = nin;
  for (int i = 0; i < n; i += 32)
  {
    int m = n - i < 32 ? n - i : 32;
    or_bits(words, pos + (unsigned long long)i, (uint32_t)(x >> i), m);
  }
  pos += (unsigned long long)n;
  unsigned long long r = n < 64 ? (x >> n) : 0ull;
  while (n < nvals)
  {
    if (r == 0)
    {
      pos += 1;  // group bit 0
      break;
    }
    or_bits(words, pos, 1u, 1);  // group bit 1
    pos += 1;
    int t = __ffsll((long long)r) - 1;
    int s = n + t;
    if (s < nvals - 1)
    {
      pos += (unsigned long long)t;  // t zero bits
      or_bits(words, pos, 1u, 1);
      pos += 1;
      n = s + 1;
      r = (t + 1 < 64) ? (r >> (t + 1)) : 0ull;
    }
    else
    {
      pos += (unsigned long long)t;  // zeros up to the last coefficient, which is implied
      n = nvals;
      r = 0;
    }
  }
}

// 192-bit little-endian bit string in three words.
struct bits192
{
  unsigned long long w0 = 0, w1 = 0, w2 = 0;
  __device__ __forceinline__ void set(int p)
  {
    if (p < 64)
      w0 |= 1ull << p;
    else if (p < 128)
      w1 |= 1ull << (p - 64);
    else
      w2 |= 1ull << (p - 128);
  }
  // bits [b, b + 32), b >= 0
  __device__ __forceinline__ uint32_t get32(int b) const
  {
    const int k = b >> 6, o = b & 63;
    const unsigned long long lo = k == 0 ? w0 : (k == 1 ? w1 : (k == 2 ? w2 : 0ull));
    const unsigned long long hi = k == 0 ? w1 : (k == 1 ? w2 : 0ull);
    return (uint32_t)(o ? ((lo >> o) | (hi << (64 - o))) : lo);
  }
};

// The code of one bit plane (Core/Zfp.h:771 Encode<u64>) built in registers: the first nin
// bits of x raw, then for every further one-bit a group bit 1, the zero bits up to it and
// the one-bit itself (implied when it is the last coefficient), then a group bit 0 while
// coefficients remain. At most 64 + 2 * 64 + 1 bits; returns the length.
__device__ __forceinline__ int plane_code(unsigned long long x, int nin, int nvals, bits192* c)
{
  c->w0 = nin >= 64 ? x : (x & ((1ull << nin) - 1ull));
  c->w1 = c->w2 = 0;
  int len = nin, n = nin;
  unsigned long long r = n < 64 ? (x >> n) : 0ull;
  while (n < nvals)
  {
    if (r == 0)
    {
      len += 1;
      break;
    }
    c->set(len);
    len += 1;
    const int t = __ffsll((long long)r) - 1;
    const int s = n + t;
    len += t;
    if (s < nvals - 1)
    {
      c->set(len);
      len += 1;
      n = s + 1;
      r = (t + 1 < 64) ? (r >> (t + 1)) : 0ull;
    }
    else
    {
      n = nvals;
      r = 0;
    }
  }
  return len;
}

// OR a code of len bits into a zero-initialised word stream at bit position pos.
__device__ __forceinline__ void or_code(uint32_t* words, unsigned long long pos, const bits192& c, int len)
{
  if (len <= 0)
    return;
  uint32_t* w = words + (pos >> 5);
  const int sh = (int)(pos & 31);
  const uint32_t first = (uint32_t)(c.w0 << sh);
  if (first)
    atomicOr(w, first);
  const int nw = (sh + len + 31) >> 5;
  for (int i = 1; i < nw; ++i)
  {
    const uint32_t v = c.get32(32 * i - sh);
    if (v)
      atomicOr(w + i, v);
  }
}

// Distributed shared memory of a thread-block cluster: the 32-bit shared::cluster address of
// a location of CTA `rank`'s shared memory (the same variable as `p` in this CTA), and loads /
// stores through it.
__device__ __forceinline__ unsigned cluster_addr(const void* p, int rank)
{
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n"
               : "=r"(r)
               : "r"((unsigned)__cvta_generic_to_shared(p)), "r"(rank));
  return r;
}

template <typename T>
__device__ __forceinline__ T ld_cluster(unsigned addr)
{
  T v;
  if constexpr (sizeof(T) == 4)
    asm volatile("ld.shared::cluster.f32 %0, [%1];\n" : "=f"(v) : "r"(addr) : "memory");
  else
    asm volatile("ld.shared::cluster.f64 %0, [%1];\n" : "=d"(v) : "r"(addr) : "memory");
  return v;
}

template <typename T>
__device__ __forceinline__ void st_cluster(unsigned addr, T v)
{
  if constexpr (sizeof(T) == 4)
    asm volatile("st.shared::cluster.f32 [%0], %1;\n" ::"r"(addr), "f"(v) : "memory");
  else
    asm volatile("st.shared::cluster.f64 [%0], %1;\n" ::"r"(addr), "d"(v) : "memory");
}

} // namespace dev
} // namespace idx2g
