// Encode kernels for sm_100a and the device stage of the encoder.
//
// One persistent CTA per brick slot runs the whole per-brick pipeline of the
// reference (Core/idx2Encode.cpp:276-335 EncodeBrick and :141-256
// EncodeSubbandBlocks):
//   A  gather the brick (level 0: from the field, widened to FP64; level > 0: the
//      parent brick assembled by the children) into the CTA's FP64 slot,
//   B  extrapolation round trip + one-level CDF5/3 + subband normalisation,
//   C  hand the low band to the parent brick of the next level,
//   D  per subband: warp-per-block exponent / quantise / zfp / shuffle, bit planes
//      by warp ballot, closed-form plane lengths, per-channel scan, bit scatter.
// The channel streams of a (brick, subband) are placed with one atomic cursor
// bump; the host packer reads them back by offset.
#include "codec_device.cuh"
#include "device.h"
#include "band_plan.h"
#include "encoder.h"
#include "trace.h"

#include <cooperative_groups.h>
#include <cuda.h>  // CUtensorMap (the encoder is reached through the runtime's entry point)

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace idx2g
{

namespace
{

// Per-phase cycle counters of thread 0 of every CTA, for profiling builds only
// (-DIDX2G_PHASE_TIMING); compiled out otherwise.
#ifdef IDX2G_PHASE_TIMING
__device__ unsigned long long g_phase_cycles[16];
struct phase_acc
{
  long long ph[16];
  long long t;
};
#define ENC_PHASE_INIT phase_acc pacc_ = {};
#define ENC_PHASE_START \
  if (threadIdx.x == 0) \
    pacc_.t = clock64();
#define ENC_PHASE(k)                 \
  if (threadIdx.x == 0)              \
  {                                  \
    const long long t_ = clock64();  \
    pacc_.ph[k] += t_ - pacc_.t;     \
    pacc_.t = t_;                    \
  }
#define ENC_PHASE_FLUSH            \
  if (threadIdx.x == 0)            \
    for (int k = 0; k < 16; ++k)   \
      atomicAdd(&g_phase_cycles[k], (unsigned long long)pacc_.ph[k]);
#else
struct phase_acc
{
};
#define ENC_PHASE_INIT phase_acc pacc_;
#define ENC_PHASE_START
#define ENC_PHASE(k)
#define ENC_PHASE_FLUSH
#endif

// CTA size: 256 threads with two CTAs per SM, or 512 with one (IDX2G_ENC_THREADS)
#ifndef IDX2G_ENC_THREADS
#define IDX2G_ENC_THREADS 256
#endif
constexpr int kThreads = IDX2G_ENC_THREADS;
constexpr int kWarps = kThreads / 32;
#ifndef IDX2G_ENC_CTAS
#define IDX2G_ENC_CTAS (IDX2G_ENC_THREADS >= 512 ? 1 : 2)
#endif
constexpr int kCtasPerSm = IDX2G_ENC_CTAS;
// per-block zfp scratch, one padding word after every 4 (conflict-free 4-point passes)
constexpr int kQStride = 80;
__device__ __forceinline__ int qpad(int i) { return i + (i >> 2); }
// plane-major (plane, block) tables of a subband, rows padded against bank conflicts
constexpr int kRowX = kMaxBlocksPerSubband + 1;    // unsigned long long
constexpr int kRowOff = kMaxBlocksPerSubband + 2;  // uint16_t
constexpr int kRowNin = kMaxBlocksPerSubband + 4;  // uint8_t
constexpr unsigned kStageBytes = 8192;
constexpr int kGz = 4;  // z-planes per chunk of the level-0 gather

struct enc_brick
{
  int b3[3];      // brick coordinates (level 0: field origin = b3 * 32)
  int valid[3];   // valid dims
  int parent;     // parent index in the next level's brick list, -1 if none
  int pos[3];     // position inside the parent (0/1 per axis)
  int field;      // entry of the launch's field table
};

// Per-field parameters of one level (a launch may cover the bricks of many fields).
struct enc_field
{
  int is2d, f32_exp, etol, end_bp, nsb;
  uint64_t order;
  const void* field;
  int field_f32;
  long long fdims[3];
  const uint64_t* geom;      // [nsb][kMaxBlocksPerSubband]
  const int* nblocks;        // [nsb]
  double weight[8];
  int norm_mask;
  int bpc;                   // BitPlanesPerChunk: bit planes per channel key
  int pad_;
  const CUtensorMap* tmap;   // level 0: the field as a 3D tensor (boxes of 32 x 32 x kGz), or null
};

constexpr int kNB3 = 33 * 33 * 33;  // brick stride of slots and parent arrays (2D bricks use 33^2)

struct enc_args
{
  int level, nbricks;
  int first, last;    // the launch codes entries [first, last) of the brick list, or of `order`
  const int* order;   // null, or the brick of each entry
  int planes;  // plane capacity per block in shared memory (32 or 64)
  const enc_field* fields;
  const enc_brick* bricks;
  const double* in_bricks;   // level > 0: [nbricks][kNB3] assembled parents
  double* slots;             // [gridDim][kNB3]
  double* parent_bricks;     // [nparents][kNB3] (zeroed), null on the coarsest level
  unsigned long long* offset;  // [nbricks][8] region offsets
  uint32_t* stream;
  unsigned long long cap_bytes;
  unsigned long long* cursor;
  int* error;
  double* bmin;
  double* bmax;
};

// shared memory layout: this struct, then the per-(plane, block) tables of one subband
// sized by the number of planes a block can have (32 for float32 data, 64 for float64):
//   unsigned long long X[P][kRowX]   plane bit masks
//   uint16_t off[P][kRowOff]         plane bit lengths, then bit offsets in the channel
//   uint8_t nin[P][kRowNin]          significant coefficients before the plane
template <int NT>
struct enc_smem_t
{
  static constexpr int W = NT / 32;
  long long q[W][2][kQStride];  // per-warp scratch of two blocks
  int16_t emax[kMaxBlocksPerSubband];
  int16_t ktop[kMaxBlocksPerSubband];
  uint8_t np[kMaxBlocksPerSubband];
  uint8_t nvals_log[kMaxBlocksPerSubband];
  uint8_t perm3[64];
  uint8_t perm2[16];
  uint32_t key_bits[kKeyWindow];
  uint32_t key_base[kKeyWindow];
  uint32_t stage[kStageBytes / 4];  // one (brick, subband) region being assembled
  unsigned alloc, hdr;
  enc_field fp;  // parameters of the current brick's field
  dev::lift_stack stack;
  double red[2][W];
  int kmin, kmax;
  unsigned long long region;
  int ok;
  unsigned long long tma_bar[2];  // completion of the gather's two chunk buffers (TMA path)
};
using enc_smem = enc_smem_t<kThreads>;

inline size_t enc_smem_bytes(int planes)
{
  // the coding tables, which also hold the 17^3 even lattice during the transform
  const size_t tables = (size_t)planes * ((size_t)kRowX * 8 + (size_t)kRowOff * 2 + (size_t)kRowNin);
  const size_t lattice = (size_t)17 * 17 * 17 * 8;
  // the level-0 gather with its first sweeps: one chunk buffer and a 4-plane FP64 band
  const size_t band = (size_t)kGz * 32 * 32 * (planes == 32 ? 4 : 8) + (size_t)kGz * 33 * 33 * 8;
  size_t space = tables > lattice ? tables : lattice;
  space = space > band ? space : band;
  return ((sizeof(enc_smem) + 127) & ~(size_t)127) + space;
}

template <int CPS>
__global__ void __launch_bounds__(kThreads, CPS) k_encode_level(const enc_args a);

// The encode kernel compiled for kCtasPerSm CTAs per SM, or (three) for three CTAs of 256
// threads per SM (80 registers): the same code; the second suits the level-0 launch of a
// large field, whose many bricks keep the third CTA busy.
constexpr bool kThreeCtas = kThreads == 256;
using enc_kernel_fn = void (*)(const enc_args);
inline enc_kernel_fn enc_kernel(bool three)
{
  if constexpr (kThreeCtas)
    return three ? k_encode_level<3> : k_encode_level<kCtasPerSm>;
  return k_encode_level<kCtasPerSm>;
}

// Resident CTAs of the encode kernel per SM with `smem` bytes of dynamic shared memory on the
// current device (at least 1, at most the kernel's launch bound).
inline int enc_occupancy(size_t smem, bool three = false)
{
  int n = 0;
  const enc_kernel_fn k = enc_kernel(three);
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kThreads, smem) != cudaSuccess)
  {
    cudaGetLastError();
    n = 1;
  }
  n = n < 1 ? 1 : n;
  const int cap = three && kThreeCtas ? 3 : kCtasPerSm;
  return n < cap ? n : cap;
}

__device__ __forceinline__ void unpack_geom(uint64_t g, int d3[3], int bd[3])
{
  d3[0] = (int)(g & 0xff) * 4;
  d3[1] = (int)((g >> 8) & 0xff) * 4;
  d3[2] = (int)((g >> 16) & 0xff) * 4;
  bd[0] = (int)((g >> 24) & 0xff);
  bd[1] = (int)((g >> 32) & 0xff);
  bd[2] = (int)((g >> 40) & 0xff);
}

__device__ __forceinline__ void subband_grid(int is2d, int s, int from[3], int dims[3], int strd[3])
{
  int h[3] = { 0, 0, 0 };
  if (is2d)
  {
    h[0] = (s >> 1) & 1;
    h[1] = s & 1;
  }
  else
  {
    h[0] = (s >> 2) & 1;
    h[1] = (s >> 1) & 1;
    h[2] = s & 1;
  }
  for (int k = 0; k < 3; ++k)
  {
    if (is2d && k == 2)
    {
      from[k] = 0;
      dims[k] = 1;
      strd[k] = 1;
    }
    else
    {
      from[k] = h[k];
      dims[k] = h[k] ? 16 : 17;
      strd[k] = 2;
    }
  }
}

__device__ __forceinline__ double warp_max(double v)
{
  for (int o = 16; o > 0; o >>= 1)
  {
    double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = v < w ? w : v;
  }
  return v;
}

// L2 prefetch of the field rows a level-0 brick will gather.
__device__ __forceinline__ void prefetch_rows(const enc_field& a, const enc_brick& b)
{
  const int vx = b.valid[0], vy = b.valid[1], vz = b.valid[2];
  const int esz = a.field_f32 ? 4 : 8;
  const long long gx0 = (long long)b.b3[0] * 32, gy0 = (long long)b.b3[1] * 32,
                  gz0 = (long long)b.b3[2] * (a.is2d ? 1 : 32);
  for (int r = threadIdx.x; r < vy * vz; r += blockDim.x)
  {
    const int y = r % vy, z = r / vy;
    const char* p = (const char*)a.field + (((gz0 + z) * a.fdims[1] + gy0 + y) * a.fdims[0] + gx0) * esz;
    const char* q = p + (size_t)vx * esz - 1;
    for (const char* c = p; c <= q; c += 128)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(c));
    if ((((uintptr_t)q) >> 7) != (((uintptr_t)p + (((uintptr_t)(q - p)) & ~(uintptr_t)127)) >> 7))
      asm volatile("prefetch.global.L2 [%0];" ::"l"(q));
  }
}

// One zfp 4-point lifting line (Core/Zfp.h:145 FLift) on the padded per-block scratch:
// elements i, i + s, i + 2s, i + 3s of the block.
__device__ __forceinline__ void lift4_padded(long long* q, int i, int s)
{
  dev::fwd_lift4_at(q + qpad(i), q + qpad(i + s), q + qpad(i + 2 * s), q + qpad(i + 3 * s));
}

// Offset in the brick of sample j of a block (block dims are 4 or 1 per axis since the
// subbands of a 33^3 brick are 17 or 16 wide).
__device__ __forceinline__ int block_sample(int base, int lx, int ly, int j, int sy, int sz)
{
  const int x = j & lx;
  const int y = (j >> (lx ? 2 : 0)) & ly;
  const int z = j >> ((lx ? 2 : 0) + (ly ? 2 : 0));
  return base + 2 * x + sy * y + sz * z;
}

struct block_info
{
  int base, lx, ly, nd;
};

__device__ __forceinline__ block_info block_at(const uint64_t* geom, int b, const int from[3], int is2d,
                                              bool zsplit = false)
{
  int d3[3], bd[3];
  unpack_geom(geom[b], d3, bd);
  block_info bi;
  // zsplit: the subband's planes (z = from[2] + 2k) are packed, plane k at k * 33 * 33
  const int zp = is2d ? 0 : (zsplit ? d3[2] : from[2] + 2 * d3[2]);
  bi.base = zp * 33 * 33 + (from[1] + 2 * d3[1]) * 33 + from[0] + 2 * d3[0];
  bi.lx = bd[0] > 1 ? 3 : 0;
  bi.ly = bd[1] > 1 ? 3 : 0;
  bi.nd = (bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1);
  return bi;
}

// Block coding of subband s of brick bi, its samples at F in the 33^3 layout (SZ: the stride
// between the subband's z-planes), or, with zsplit, with the subband's planes (one z parity)
// packed one after the other (SZ = 33 * 33):
// exponents, quantisation, zfp, shuffle, bit planes, channel scans, the region's
// allocation and the bit scatter (Core/idx2Encode.cpp:141-256 EncodeSubbandBlocks).
template <int NT>
__device__ __forceinline__ void code_subband(const enc_args& a, enc_smem_t<NT>& sm, unsigned long long* const Xp,
                                             uint16_t* const OFF, uint8_t* const NIN, const int P,
                                             const double* const F, const int SZ, const bool zsplit, const int bi,
                                             const int s, phase_acc& pacc_)
{
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const enc_field& fp = sm.fp;
  int from[3], dims[3], strd[3];
  subband_grid(fp.is2d, s, from, dims, strd);
  const int nb = fp.nblocks[s];
  const uint64_t* geom = fp.geom + (size_t)s * kMaxBlocksPerSubband;
  const size_t bs = (size_t)bi * 8 + (size_t)s;

  // D1: a warp codes two blocks (lanes own samples j and j + 32 of each): exponent,
  // quantisation, zfp transform, shuffle, bit-plane masks by ballot; then the
  // significance chain and the plane lengths, lane-parallel over the planes.
  // The samples of the warp's next pair are loaded while the current pair is coded.
  const int npairs = (nb + 1) >> 1;
  double cv[4];
  block_info cA, cB;
  auto load_pair = [&](int pr, double v[4], block_info& A, block_info& B) {
    const int b0 = 2 * pr, b1 = 2 * pr + 1;
    A = block_at(geom, b0, from, fp.is2d, zsplit);
    const bool hb = b1 < nb;
    B = hb ? block_at(geom, b1, from, fp.is2d, zsplit) : A;
    const int nvA = 1 << (2 * A.nd), nvB = hb ? 1 << (2 * B.nd) : 0;
    v[0] = lane < nvA ? F[block_sample(A.base, A.lx, A.ly, lane, 66, SZ)] : 0.0;
    v[1] = lane + 32 < nvA ? F[block_sample(A.base, A.lx, A.ly, lane + 32, 66, SZ)] : 0.0;
    v[2] = lane < nvB ? F[block_sample(B.base, B.lx, B.ly, lane, 66, SZ)] : 0.0;
    v[3] = lane + 32 < nvB ? F[block_sample(B.base, B.lx, B.ly, lane + 32, 66, SZ)] : 0.0;
  };
  if (warp < npairs)
    load_pair(warp, cv, cA, cB);
  for (int pr = warp; pr < npairs; pr += NW)
  {
    double nv_[4] = { 0, 0, 0, 0 };
    block_info nA = cA, nB = cB;
    if (pr + NW < npairs)
      load_pair(pr + NW, nv_, nA, nB);
    const int bA = 2 * pr, bB = 2 * pr + 1;
    const bool hasB = bB < nb;
    const int ndA = cA.nd, ndB = hasB ? cB.nd : 0;
    const int nvA = 1 << (2 * ndA), nvB = hasB ? 1 << (2 * ndB) : 0;
    // block maxima
    double mA = fabs(cv[0]), mB = fabs(cv[2]);
    {
      const double m1 = fabs(cv[1]), m3 = fabs(cv[3]);
      mA = mA < m1 ? m1 : mA;
      mB = mB < m3 ? m3 : mB;
    }
    mA = warp_max(mA);
    mB = warp_max(mB);
    const int eA = fp.f32_exp ? dev::exponent_f32(__double2float_rn(mA)) : dev::exponent_f64(mA);
    const int eB = fp.f32_exp ? dev::exponent_f32(__double2float_rn(mB)) : dev::exponent_f64(mB);
    const double sA = dev::pow2(63 - ndA - 1 - eA), sB = dev::pow2(63 - ndB - 1 - eB);
    long long* qA = sm.q[warp][0];
    long long* qB = sm.q[warp][1];
    if (lane < nvA)
      qA[qpad(lane)] = dev::trunc_i64(__dmul_rn(sA, cv[0]));
    if (lane + 32 < nvA)
      qA[qpad(lane + 32)] = dev::trunc_i64(__dmul_rn(sA, cv[1]));
    if (lane < nvB)
      qB[qpad(lane)] = dev::trunc_i64(__dmul_rn(sB, cv[2]));
    if (lane + 32 < nvB)
      qB[qpad(lane + 32)] = dev::trunc_i64(__dmul_rn(sB, cv[3]));
    __syncwarp();
    // zfp transform (Core/Zfp.h:262): the 16 lines of a pass of block A on lanes 0-15,
    // of block B on lanes 16-31
    {
      // (the halves share no data: each synchronises on its own 16 lanes)
      const int h = lane >> 4, l = lane & 15;
      const unsigned hm = h ? 0xffff0000u : 0x0000ffffu;
      long long* q = h ? qB : qA;
      const int nd = h ? ndB : ndA;
      if (nd == 3)
      {
        lift4_padded(q, 4 * (l & 3) + 16 * (l >> 2), 1);
        __syncwarp(hm);
        lift4_padded(q, 16 * (l & 3) + (l >> 2), 4);
        __syncwarp(hm);
        lift4_padded(q, (l & 3) + 4 * (l >> 2), 16);
      }
      else if (nd == 2)
      {
        if (l < 4)
          lift4_padded(q, 4 * l, 1);
        __syncwarp(hm);
        if (l < 4)
          lift4_padded(q, l, 4);
      }
      else if (nd == 1)
      {
        if (l == 0)
          lift4_padded(q, 0, 1);
      }
      __syncwarp();
    }
    // shuffle to sequency order, negabinary (Core/Zfp.h:419-520)
    auto permj = [&](int nd, int j) -> int {
      return nd == 3 ? (int)sm.perm3[j] : (nd == 2 ? (int)sm.perm2[j & 15] : j);
    };
    unsigned long long uA0 = 0, uA1 = 0, uB0 = 0, uB1 = 0;
    if (lane < nvA)
      uA0 = ((unsigned long long)qA[qpad(permj(ndA, lane))] + dev::kNegaMask) ^ dev::kNegaMask;
    if (lane + 32 < nvA)
      uA1 = ((unsigned long long)qA[qpad(permj(ndA, lane + 32))] + dev::kNegaMask) ^ dev::kNegaMask;
    if (lane < nvB)
      uB0 = ((unsigned long long)qB[qpad(permj(ndB, lane))] + dev::kNegaMask) ^ dev::kNegaMask;
    if (lane + 32 < nvB)
      uB1 = ((unsigned long long)qB[qpad(permj(ndB, lane + 32))] + dev::kNegaMask) ^ dev::kNegaMask;
    __syncwarp();
    int npA = dev::coded_planes(eA, fp.etol, fp.end_bp, fp.bpc);
    int npB = hasB ? dev::coded_planes(eB, fp.etol, fp.end_bp, fp.bpc) : 0;
    if (npA > P || npB > P)
    {
      // more planes than the tables hold (a float64 block in a 32-plane launch): the level is
      // coded again by a launch with room for them; this one's output is void
      if (lane == 0)
        atomicExch(a.error, 8);
      npA = npA < P ? npA : P;
      npB = npB < P ? npB : P;
    }
    const int npM = npA > npB ? npA : npB;
    unsigned long long* XA = Xp + bA;  // plane k at XA[k * kRowX]
    unsigned long long* XB = Xp + bB;
    if (lane == 0)
    {
      sm.emax[bA] = (int16_t)eA;
      sm.ktop[bA] = (int16_t)(eA + 63 + 1024);
      sm.np[bA] = (uint8_t)npA;
      sm.nvals_log[bA] = (uint8_t)(2 * ndA);
    }
    if (lane == 1 && hasB)
    {
      sm.emax[bB] = (int16_t)eB;
      sm.ktop[bB] = (int16_t)(eB + 63 + 1024);
      sm.np[bB] = (uint8_t)npB;
      sm.nvals_log[bB] = (uint8_t)(2 * ndB);
    }
    // Bit planes by warp transposes: transposing the high words of (uA0 | uA1) gives lane c
    // the mask of plane k = 31 - c (bit 63 - k of every coefficient), the low words planes
    // 32..63 (k = 63 - c). Then the significance chain (Core/Zfp.h:771): nin(k) = max over
    // planes k' < k of the highest one-bit + 1, a suffix maximum over the lanes; and the
    // plane lengths.
    {
      int carryA = 0, carryB = 0;
      const int ngroups = npM > 32 ? 2 : 1;
      for (int g = 0; g < ngroups; ++g)
      {
        const int sh = g ? 0 : 32;
        const int k = 31 - lane + 32 * g;
        unsigned long long xa =
          (unsigned long long)dev::warp_transpose32((uint32_t)(uA0 >> sh), lane) |
          ((unsigned long long)dev::warp_transpose32((uint32_t)(uA1 >> sh), lane) << 32);
        unsigned long long xb =
          (unsigned long long)dev::warp_transpose32((uint32_t)(uB0 >> sh), lane) |
          ((unsigned long long)dev::warp_transpose32((uint32_t)(uB1 >> sh), lane) << 32);
        xa = k < npA ? xa : 0ull;
        xb = k < npB ? xb : 0ull;
        if (k < npA)
          XA[k * kRowX] = xa;
        if (k < npB)
          XB[k * kRowX] = xb;
        // inclusive maximum over planes <= k, i.e. over lanes >= lane
        int ia = xa ? 64 - __clzll(xa) : 0, ib = xb ? 64 - __clzll(xb) : 0;
        for (int o = 1; o < 32; o <<= 1)
        {
          const int ta = __shfl_down_sync(0xffffffffu, ia, o), tb = __shfl_down_sync(0xffffffffu, ib, o);
          if (lane + o < 32)
          {
            ia = ia > ta ? ia : ta;
            ib = ib > tb ? ib : tb;
          }
        }
        int ea = __shfl_down_sync(0xffffffffu, ia, 1), eb = __shfl_down_sync(0xffffffffu, ib, 1);
        ea = lane < 31 ? ea : 0;
        eb = lane < 31 ? eb : 0;
        const int nA_ = ea > carryA ? ea : carryA, nB_ = eb > carryB ? eb : carryB;
        if (k < npA)
        {
          NIN[k * kRowNin + bA] = (uint8_t)nA_;
          OFF[k * kRowOff + bA] = (uint16_t)dev::plane_bits(xa, nA_, nvA);
        }
        if (k < npB)
        {
          NIN[k * kRowNin + bB] = (uint8_t)nB_;
          OFF[k * kRowOff + bB] = (uint16_t)dev::plane_bits(xb, nB_, nvB);
        }
        const int ta = __shfl_sync(0xffffffffu, ia, 0), tb = __shfl_sync(0xffffffffu, ib, 0);
        carryA = carryA > ta ? carryA : ta;
        carryB = carryB > tb ? carryB : tb;
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
      cv[i] = nv_[i];
    cA = nA;
    cB = nB;
  }
  __syncthreads();
  ENC_PHASE(10)

  // key range of the subband
  if (warp == 0)
  {
    int lo = 1 << 30, hi = -(1 << 30);
    for (int b = lane; b < nb; b += 32)
    {
      const int n = sm.np[b];
      if (!n)
        continue;
      const int t = sm.ktop[b];
      if (t - n + 1 < 0)
        atomicExch(a.error, 1);  // negative key value: a tolerance below 2^-1070 (unsupported)
      const int kl = dev::plane_key(t, n - 1, fp.bpc), kh = dev::plane_key(t, 0, fp.bpc);
      lo = kl < lo ? kl : lo;
      hi = kh > hi ? kh : hi;
    }
    for (int o = 16; o > 0; o >>= 1)
    {
      const int l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
      lo = l2 < lo ? l2 : lo;
      hi = h2 > hi ? h2 : hi;
    }
    if (lane == 0)
    {
      if (hi < lo)
      {
        lo = 1;
        hi = 0;
      }
      sm.kmin = lo;
      sm.kmax = hi;
      sm.ok = (hi - lo + 1) <= kKeyWindow;
      if (!sm.ok)
        atomicExch(a.error, 1);
    }
  }
  __syncthreads();
  const int kmin = sm.kmin, kmax = sm.kmax;
  const int nkeys = sm.ok ? kmax - kmin + 1 : 0;
  ENC_PHASE(11)

  // D3: per channel key (a warp each), bit offsets in the channel's stream: blocks in
  // Morton order, within a block its planes of the key top-down (one plane per key when
  // BitPlanesPerChunk is 1); an exclusive scan of the plane lengths, in place
  for (int t = warp; t < nkeys && fp.bpc == 1; t += NW)
  {
    // one plane per key: plane ktop - key of each block
    const int key = kmin + t;
    uint32_t carry = 0;
    for (int b0 = 0; b0 < nb; b0 += 32)
    {
      const int b = b0 + lane;
      int kk = b < nb ? sm.ktop[b] - key : -1;
      kk = (kk >= 0 && b < nb && kk < sm.np[b]) ? kk : -1;
      const uint32_t v = kk >= 0 ? OFF[kk * kRowOff + b] : 0u;
      uint32_t inc = v;
      for (int o = 1; o < 32; o <<= 1)
      {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
          inc += y;
      }
      if (kk >= 0)
        OFF[kk * kRowOff + b] = (uint16_t)(carry + inc - v);
      carry += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0)
      sm.key_bits[t] = carry;
  }
  for (int t = warp; t < nkeys && fp.bpc > 1; t += NW)
  {
    const int key = kmin + t;
    uint32_t carry = 0;
    for (int b0 = 0; b0 < nb; b0 += 32)
    {
      const int b = b0 + lane;
      int kk0 = 1, kk1 = 0;
      if (b < nb && sm.np[b])
        dev::key_planes(sm.ktop[b], sm.np[b], key, fp.bpc, kk0, kk1);
      uint32_t v = 0;
      for (int kk = kk0; kk <= kk1; ++kk)
        v += OFF[kk * kRowOff + b];
      uint32_t inc = v;
      for (int o = 1; o < 32; o <<= 1)
      {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
          inc += y;
      }
      uint32_t run = carry + inc - v;
      for (int kk = kk0; kk <= kk1; ++kk)
      {
        const uint32_t len = OFF[kk * kRowOff + b];
        OFF[kk * kRowOff + b] = (uint16_t)run;
        run += len;
      }
      carry += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0)
    {
      sm.key_bits[t] = carry;
      if (carry > 65535u)
        atomicExch(a.error, 1);  // offsets are 16-bit: a key stream of more than 65535 bits
    }
  }
  __syncthreads();
  ENC_PHASE(12)

  // D4: channel byte bases and the region of this (brick, subband)
  // (regions are whole 32-bit words so every CTA owns the words it writes)
  if (warp == 0)
  {
    uint32_t v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
      const int t = lane * 4 + i;
      v[i] = t < nkeys ? (sm.key_bits[t] + 7u) / 8u : 0u;
    }
    const uint32_t tot = v[0] + v[1] + v[2] + v[3];
    uint32_t inc = tot;
    for (int o = 1; o < 32; o <<= 1)
    {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o)
        inc += y;
    }
    uint32_t acc = inc - tot;
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
      const int t = lane * 4 + i;
      if (t < nkeys)
        sm.key_base[t] = acc;
      acc += v[i];
    }
    const uint32_t base = __shfl_sync(0xffffffffu, inc, 31);
    if (lane == 0)
    {
      // region: header (kmin, nkeys), exponents, channel sizes, channel streams
      const unsigned hdr = 8u + ((2u * (unsigned)nb + 3u) & ~3u) + 4u * (unsigned)nkeys;
      const unsigned alloc = hdr + ((base + 3u) & ~3u);
      unsigned long long region = atomicAdd(a.cursor, (unsigned long long)alloc);
      if (region + alloc > a.cap_bytes)
        atomicExch(a.error, 2);
      sm.region = region;
      sm.alloc = alloc;
      sm.hdr = hdr;
      a.offset[bs] = region;
    }
  }
  __syncthreads();
  const unsigned long long region = sm.region;
  const unsigned alloc = sm.alloc;
  const unsigned hdr = sm.hdr;
  const bool fits = region + alloc <= a.cap_bytes;
  ENC_PHASE(13)

  // D5: the plane codes, built in registers and ORed into shared memory when the region
  // is small enough, else straight into the (zeroed) global region; then the region is
  // stored with plain writes
  if (fits && alloc)
  {
    const bool staged = alloc <= kStageBytes;
    uint32_t* words = staged ? sm.stage : a.stream + region / 4;
    for (unsigned i = tid; i < alloc / 4; i += NT)
      words[i] = 0u;
    __syncthreads();
    if (tid == 0)
    {
      words[0] = (uint32_t)(nkeys ? kmin : 1);
      words[1] = (uint32_t)nkeys;
    }
    uint16_t* ew = reinterpret_cast<uint16_t*>(words + 2);
    for (int b = tid; b < nb; b += NT)
      ew[b] = (uint16_t)sm.emax[b];
    uint32_t* sw = words + 2 + ((2u * (unsigned)nb + 3u) >> 2);
    for (int t = tid; t < nkeys; t += NT)
      sw[t] = (sm.key_bits[t] + 7) / 8;
    for (int idx = tid; idx < P * kMaxBlocksPerSubband; idx += NT)
    {
      const int b = idx & (kMaxBlocksPerSubband - 1), kk = idx / kMaxBlocksPerSubband;
      if (b >= nb || kk >= sm.np[b])
        continue;
      const int t = dev::plane_key(sm.ktop[b], kk, fp.bpc) - kmin;
      const unsigned long long pos = ((unsigned long long)hdr + sm.key_base[t]) * 8ull +
                                     (unsigned long long)OFF[kk * kRowOff + b];
      dev::bits192 c;
      const int len =
        dev::plane_code(Xp[kk * kRowX + b], NIN[kk * kRowNin + b], 1 << sm.nvals_log[b], &c);
      dev::or_code(words, pos, c, len);
    }
    __syncthreads();
    if (staged)
    {
      uint32_t* dst = a.stream + region / 4;
      for (unsigned i = tid; i < alloc / 4; i += NT)
        __stcs(dst + i, sm.stage[i]);
    }
  }
  __syncthreads();
  ENC_PHASE(14)
}

template <int CPS>
__global__ void __launch_bounds__(kThreads, CPS) k_encode_level(const enc_args a)
{
  extern __shared__ __align__(128) unsigned char smem_raw[];
  enc_smem& sm = *reinterpret_cast<enc_smem*>(smem_raw);
  const int P = a.planes;
  // the tables start 128-byte aligned: the gather's chunk buffers there are TMA destinations
  unsigned long long* const Xp =
    reinterpret_cast<unsigned long long*>(smem_raw + ((sizeof(enc_smem) + 127) & ~(size_t)127));
  uint16_t* const OFF = reinterpret_cast<uint16_t*>(Xp + (size_t)kRowX * P);
  uint8_t* const NIN = reinterpret_cast<uint8_t*>(OFF + (size_t)kRowOff * P);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* F = a.slots + (size_t)blockIdx.x * (size_t)kNB3;
  if (tid < 64)
    sm.perm3[tid] = dev::perm(3, tid);
  if (tid < 16)
    sm.perm2[tid] = dev::perm(2, tid);
  if (tid == 0 && a.level == 0)
  {
    const unsigned b0 = (unsigned)__cvta_generic_to_shared(&sm.tma_bar[0]);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b0 + 8u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  unsigned tma_parity = 0;  // bit b: phase parity of chunk buffer b's next completion
  ENC_PHASE_INIT

  for (int it = a.first + (int)blockIdx.x; it < a.last; it += gridDim.x)
  {
    const int bi = a.order ? a.order[it] : it;
    const enc_brick& br = a.bricks[bi];
    {
      // the field's parameters to shared memory (read often, and across barriers)
      static_assert(sizeof(enc_field) % 4 == 0, "enc_field is copied as words");
      const uint32_t* src = reinterpret_cast<const uint32_t*>(a.fields + br.field);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sm.fp);
      for (int i = tid; i < (int)(sizeof(enc_field) / 4); i += kThreads)
        dst[i] = src[i];
    }
    __syncthreads();
    const enc_field& fp = sm.fp;
    const int N[3] = { 33, 33, fp.is2d ? 1 : 33 };
    const int NB = N[0] * N[1] * N[2];
    const int SZ = fp.is2d ? 0 : 2 * 33 * 33;  // sample stride along z inside a subband
    // the extrapolation's sweeps on the valid dims (Core/Wavelet.cpp:68)
    if (tid == 0)
      dev::build_stack(br.valid, 5, fp.order, &sm.stack);
    __syncthreads();
    auto level_one = [&](const dev::dgrid& g) {
      return g.from[0] == 0 && g.from[1] == 0 && g.from[2] == 0 && g.strd[0] == 1 && g.strd[1] == 1 && g.strd[2] == 1;
    };
    // A level-0 brick read through TMA whose first two sweeps are X and Y (in either order)
    // takes them during the gather, on each chunk of planes in shared memory
    const bool gather_xy = a.level == 0 && fp.tmap != nullptr && !fp.is2d && sm.stack.coarse >= 2 &&
                           sm.stack.axis[0] + sm.stack.axis[1] == 1 && level_one(sm.stack.g[0]) &&
                           level_one(sm.stack.g[1]);
    ENC_PHASE_START
    // ---------------- A: gather ----------------
    if (a.level == 0 && gather_xy)
    {
      // one chunk buffer: the copy of chunk c + 1 runs while chunk c's sweeps do
      const int vx = br.valid[0], vy = br.valid[1], vz = br.valid[2];
      double mn = 1.7976931348623157e308, mx = -1.7976931348623157e308;
      const long long gx0 = (long long)br.b3[0] * 32, gy0 = (long long)br.b3[1] * 32, gz0 = (long long)br.b3[2] * 32;
      const int esz = fp.field_f32 ? 4 : 8;
      unsigned char* const stage = reinterpret_cast<unsigned char*>(Xp);
      const unsigned box_bytes = (unsigned)(kGz * 32 * 32 * esz);
      double* const T = reinterpret_cast<double*>(stage + box_bytes);  // kGz x 33 x 33
      const unsigned s0 = (unsigned)__cvta_generic_to_shared(stage);
      const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.tma_bar[0]);
      const int nch = (33 + kGz - 1) / kGz;
      auto issue = [&](int c) {
        if (tid == 0 && c < nch && c * kGz < vz)
        {
          asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(box_bytes) : "memory");
          asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
                       " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(s0),
                       "l"(fp.tmap), "r"((int)gx0), "r"((int)gy0), "r"((int)(gz0 + c * kGz)), "r"(bar)
                       : "memory");
        }
      };
      // a first-level forward sweep (lift_sweep_regs<true>) restricted to planes [z0, z0 + nz)
      auto band_sweep = [&](const dev::dgrid& G, int ax, int z0, int nz) {
        const int D = G.dims[ax];
        const int nu = G.dims[1 - ax];
        const int zhi = z0 + nz < G.dims[2] ? z0 + nz : G.dims[2];
        if (D == 1 || zhi <= z0)
          return;
        const int su = ax == 0 ? 33 : 1;
        for (int li = tid; li < nu * (zhi - z0); li += kThreads)
        {
          double* L = T + (li / nu) * 33 * 33 + (li % nu) * su;
          if (D == 32)
            ax == 0 ? dev::lift_line_strided<32, true, 1>(L) : dev::lift_line_strided<32, true, 33>(L);
          else if (D == 33)
            ax == 0 ? dev::lift_line_strided<33, true, 1>(L) : dev::lift_line_strided<33, true, 33>(L);
          else
            dev::lift_line<true>(L, ax == 0 ? 1 : 33, D);
        }
      };
      issue(0);
      for (int c = 0; c < nch; ++c)
      {
        const int z0 = c * kGz;
        const int nz = 33 - z0 < kGz ? 33 - z0 : kGz;
        int ok = 1;
        if (z0 < vz)
        {
          const unsigned par = tma_parity & 1u;
          ok = 0;
          for (int it = 0; it < (1 << 22) && !ok; ++it)
            asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                         " selp.u32 %0, 1, 0, p;\n}\n"
                         : "=r"(ok)
                         : "r"(bar), "r"(par)
                         : "memory");
          tma_parity ^= 1u;
        }
        if (!__syncthreads_and(ok))
        {
          if (tid == 0)
          {
            // a lost copy: report it, wait (bounded) for it once more, end this CTA
            atomicExch(a.error, 4);
            int done = 0;
            for (int it = 0; it < (1 << 22) && !done; ++it)
              asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                           " selp.u32 %0, 1, 0, p;\n}\n"
                           : "=r"(done)
                           : "r"(bar), "r"((tma_parity & 1u) ^ 1u)
                           : "memory");
          }
          return;
        }
        for (int i = tid; i < nz * 33 * 33; i += kThreads)
        {
          const int x = i % 33, row = i / 33, y = row % 33, zz = row / 33, z = z0 + zz;
          const bool in = x < vx && y < vy && z < vz;
          double v = 0.0;
          if (in)
            v = fp.field_f32 ? (double)reinterpret_cast<const float*>(stage)[(zz * 32 + y) * 32 + x]
                             : reinterpret_cast<const double*>(stage)[(zz * 32 + y) * 32 + x];
          T[i] = v;
          if (in)
          {
            mn = v < mn ? v : mn;
            mx = mx < v ? v : mx;
          }
        }
        __syncthreads();
        issue(c + 1);
        band_sweep(sm.stack.g[0], sm.stack.axis[0], z0, nz);
        __syncthreads();
        band_sweep(sm.stack.g[1], sm.stack.axis[1], z0, nz);
        __syncthreads();
        double* dst = F + (size_t)z0 * 33 * 33;
        for (int i = tid; i < nz * 33 * 33; i += kThreads)
          dst[i] = T[i];
        __syncthreads();
      }
      for (int o = 16; o > 0; o >>= 1)
      {
        double w1 = __shfl_xor_sync(0xffffffffu, mn, o), w2 = __shfl_xor_sync(0xffffffffu, mx, o);
        mn = w1 < mn ? w1 : mn;
        mx = mx < w2 ? w2 : mx;
      }
      if (lane == 0)
      {
        sm.red[0][warp] = mn;
        sm.red[1][warp] = mx;
      }
      __syncthreads();
      if (tid == 0)
      {
        for (int w = 1; w < kWarps; ++w)
        {
          mn = sm.red[0][w] < mn ? sm.red[0][w] : mn;
          mx = mx < sm.red[1][w] ? sm.red[1][w] : mx;
        }
        a.bmin[bi] = mn;
        a.bmax[bi] = mx;
      }
    }
    else if (a.level == 0)
    {
      const int vx = br.valid[0], vy = br.valid[1], vz = br.valid[2];
      double mn = 1.7976931348623157e308, mx = -1.7976931348623157e308;
      const long long gx0 = (long long)br.b3[0] * 32, gy0 = (long long)br.b3[1] * 32,
                      gz0 = (long long)br.b3[2] * (fp.is2d ? 1 : 32);
      // The brick's samples come through shared memory in chunks of kGz z-planes,
      // double-buffered in the coding tables' space (idle here): asynchronous copies of chunk
      // c + 1 are in flight while chunk c is widened into the brick; samples outside the
      // valid region (and the x = 32, y = 32, z = 32 faces) are zero.
      // With a tensor map (the usual case), one thread loads each chunk as one bulk tensor copy
      // (TMA) of a 32 x 32 x kGz box completing on an mbarrier; samples past the volume's
      // edge arrive as zeros, planes of the next brick are loaded and not used.
      const int esz = fp.field_f32 ? 4 : 8;
      unsigned char* const stage = reinterpret_cast<unsigned char*>(Xp);
      const unsigned stage_bytes = (unsigned)(kGz * 32 * 32 * esz);
      const unsigned box_bytes = (unsigned)((fp.is2d ? 1 : kGz) * 32 * 32 * esz);
      const int nch = (N[2] + kGz - 1) / kGz;
      const bool tma = fp.tmap != nullptr;
      auto issue = [&](int c) {
        const int z0 = c * kGz;
        const int nz = vz - z0 < kGz ? vz - z0 : kGz;
        const unsigned s0 = (unsigned)__cvta_generic_to_shared(stage) + (unsigned)(c & 1) * stage_bytes;
        if (tma)
        {
          if (tid == 0 && nz > 0)
          {
            const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.tma_bar[c & 1]);
            // the buffer was last written and read by ordinary accesses
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(box_bytes)
                         : "memory");
            asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
                         " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(s0),
                         "l"(fp.tmap), "r"((int)gx0), "r"((int)gy0), "r"((int)(gz0 + z0)), "r"(bar)
                         : "memory");
          }
          return;
        }
        for (int i = tid; i < nz * vy * 32; i += kThreads)
        {
          const int x = i & 31, row = i >> 5, y = row % vy, zz = row / vy;
          if (x >= vx)
            continue;
          const long long src = ((gz0 + z0 + zz) * fp.fdims[1] + gy0 + y) * fp.fdims[0] + gx0 + x;
          const unsigned d = s0 + (unsigned)(((zz * 32 + y) * 32 + x) * esz);
          if (fp.field_f32)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"((const float*)fp.field + src)
                         : "memory");
          else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"((const double*)fp.field + src)
                         : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
      };
      // chunk c in shared memory; false (in every thread) if its bulk copy did not complete
      // within the wait's bound (the copy then counts as lost)
      auto wait_chunk = [&](int c) -> bool {
        if (!tma)
        {
          if (c + 1 < nch)
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
          else
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
          __syncthreads();
          return true;
        }
        int ok = 1;
        if (c * kGz < vz)
        {
          const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.tma_bar[c & 1]);
          const unsigned par = (tma_parity >> (c & 1)) & 1u;
          ok = 0;
          for (int it = 0; it < (1 << 22) && !ok; ++it)
            asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                         " selp.u32 %0, 1, 0, p;\n}\n"
                         : "=r"(ok)
                         : "r"(bar), "r"(par)
                         : "memory");
          tma_parity ^= 1u << (c & 1);
        }
        return __syncthreads_and(ok) != 0;
      };
      issue(0);
      for (int c = 0; c < nch; ++c)
      {
        if (c + 1 < nch)
          issue(c + 1);
        if (!wait_chunk(c))
        {
          // a lost copy: report it and end this CTA (uniformly) after a bounded wait for the
          // copies still in flight
          if (tid == 0)
          {
            atomicExch(a.error, 4);
            for (int k = c; k <= c + 1 && k < nch; ++k)
            {
              if (k * kGz >= vz)
                continue;
              const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.tma_bar[k & 1]);
              const unsigned par = k == c ? ((tma_parity >> (k & 1)) & 1u) ^ 1u : (tma_parity >> (k & 1)) & 1u;
              int ok = 0;
              for (int it = 0; it < (1 << 22) && !ok; ++it)
                asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                             " selp.u32 %0, 1, 0, p;\n}\n"
                             : "=r"(ok)
                             : "r"(bar), "r"(par)
                             : "memory");
            }
          }
          return;
        }
        const unsigned char* buf = stage + (size_t)(c & 1) * stage_bytes;
        const int z0 = c * kGz;
        const int nz = N[2] - z0 < kGz ? N[2] - z0 : kGz;
        for (int i = tid; i < nz * 33 * 33; i += kThreads)
        {
          const int x = i % 33, row = i / 33, y = row % 33, zz = row / 33, z = z0 + zz;
          const bool in = x < vx && y < vy && z < vz;
          double v = 0.0;
          if (in)
            v = fp.field_f32 ? (double)reinterpret_cast<const float*>(buf)[(zz * 32 + y) * 32 + x]
                             : reinterpret_cast<const double*>(buf)[(zz * 32 + y) * 32 + x];
          F[(z * 33 + y) * 33 + x] = v;
          if (in)
          {
            mn = v < mn ? v : mn;
            mx = mx < v ? v : mx;
          }
        }
        __syncthreads();  // the buffer is refilled by the next chunk but one
      }
      for (int o = 16; o > 0; o >>= 1)
      {
        double w1 = __shfl_xor_sync(0xffffffffu, mn, o), w2 = __shfl_xor_sync(0xffffffffu, mx, o);
        mn = w1 < mn ? w1 : mn;
        mx = mx < w2 ? w2 : mx;
      }
      if (lane == 0)
      {
        sm.red[0][warp] = mn;
        sm.red[1][warp] = mx;
      }
      __syncthreads();
      if (tid == 0)
      {
        for (int w = 1; w < kWarps; ++w)
        {
          mn = sm.red[0][w] < mn ? sm.red[0][w] : mn;
          mx = mx < sm.red[1][w] ? sm.red[1][w] : mx;
        }
        a.bmin[bi] = mn;
        a.bmax[bi] = mx;
      }
    }
    else
    {
      // (bricks are NB = 33^3 doubles, an odd count: only 8-byte alignment is guaranteed)
      const double* src = a.in_bricks + (size_t)bi * (size_t)kNB3;
      for (int i = tid; i < NB; i += kThreads)
        F[i] = __ldcs(src + i);
    }
    __syncthreads();
    ENC_PHASE(0)

    // ---------------- B: transform ----------------
    {
      // extrapolation round trip (Core/Wavelet.cpp:68): forward on the valid dims, then the
      // inverse on the 33^3 grid except its last sweep (X at full resolution), which is fused
      // with the first sweep of the real transform below
      // The sweeps from the second level on touch only the even positions: the forward
      // sweeps of levels 2.. and the inverse ones back to level 2 run on the 17^3 even
      // lattice copied into shared memory (the coding tables' space, idle here), lifted in
      // place sample by sample.
      double* S = reinterpret_cast<double*>(Xp);
      const int NS[3] = { 17, 17, fp.is2d ? 1 : 17 };
      const int nsub = NS[0] * NS[1] * NS[2];
      const int nf = sm.stack.n, cf = sm.stack.coarse;
      for (int i = gather_xy ? 2 : 0; i < cf; ++i)
      {
        dev::lift_sweep_regs<true>(F, N, sm.stack.g[i], sm.stack.axis[i]);
        __syncthreads();
        if (i == 0)
        {
          ENC_PHASE(1)
        }
      }
      ENC_PHASE(2)
      for (int i = tid; i < nsub; i += kThreads)
      {
        const int x = i % 17, y = (i / 17) % 17, z = i / 289;
        S[i] = F[(2 * z * 33 + 2 * y) * 33 + 2 * x];
      }
      __syncthreads();
      for (int i = cf; i < nf; ++i)
      {
        dev::lift_sweep(S, NS, dev::half_grid(sm.stack.g[i]), NS, sm.stack.axis[i], true);
        __syncthreads();
      }
      ENC_PHASE(3)
      if (tid == 0)
        dev::build_stack(N, 5, fp.order, &sm.stack);
      __syncthreads();
      const int ni = sm.stack.n, ci = sm.stack.coarse;
      for (int i = ni - 1; i >= ci; --i)
      {
        dev::lift_sweep(S, NS, dev::half_grid(sm.stack.g[i]), NS, sm.stack.axis[i], false);
        __syncthreads();
      }
      for (int i = tid; i < nsub; i += kThreads)
      {
        const int x = i % 17, y = (i / 17) % 17, z = i / 289;
        F[(2 * z * 33 + 2 * y) * 33 + 2 * x] = S[i];
      }
      __syncthreads();
      ENC_PHASE(4)
      // With the first level's sweeps in Z, Y, X order on the whole 33^3 brick (the usual
      // transform order), the sweeps that stay inside z-planes -- the inverse Y, the inverse
      // then forward X, and the forward Y -- run on bands of kPlanes z-planes in shared
      // memory (the coding tables' space, idle here): one read and one write of the brick
      // instead of three of each. The same line functions run on the same values.
      auto full33 = [&](const dev::dgrid& g) {
        return g.from[0] == 0 && g.from[1] == 0 && g.from[2] == 0 && g.dims[0] == 33 && g.dims[1] == 33 &&
               g.dims[2] == 33 && g.strd[0] == 1 && g.strd[1] == 1 && g.strd[2] == 1;
      };
      const bool planar = !fp.is2d && ci == 3 && sm.stack.axis[2] == 2 && sm.stack.axis[1] == 1 &&
                          sm.stack.axis[0] == 0 && full33(sm.stack.g[2]) && full33(sm.stack.g[1]);
      for (int i = ci - 1; i >= (planar ? 2 : 1); --i)
      {
        dev::lift_sweep_regs<false>(F, N, sm.stack.g[i], sm.stack.axis[i]);
        __syncthreads();
      }
      ENC_PHASE(5)
      if (planar)
      {
        constexpr int kPlanes = 4;  // 4 x 33 x 33 doubles: 34.8 KB, within the tables' space
        double* T = reinterpret_cast<double*>(Xp);
        for (int z0 = 0; z0 < 33; z0 += kPlanes)
        {
          const int nzc = 33 - z0 < kPlanes ? 33 - z0 : kPlanes;
          const int n = nzc * 33 * 33;
          const double* src = F + (size_t)z0 * 33 * 33;
          for (int i = tid; i < n; i += kThreads)
            T[i] = src[i];
          __syncthreads();
          // inverse Y (columns of each plane)
          for (int li = tid; li < 33 * nzc; li += kThreads)
            dev::lift_line_strided<33, false, 33>(T + (li / 33) * 33 * 33 + li % 33);
          __syncthreads();
          // inverse X (D = 33) then forward X of the one-level transform (Core/Wavelet.cpp:81)
          for (int li = tid; li < 33 * nzc; li += kThreads)
          {
            double* row = T + li * 33;
            double v[33];
#pragma unroll
            for (int k = 0; k < 33; ++k)
              v[k] = row[k];
            dev::lift_regs<false>(v, 33);
            dev::lift_regs<true>(v, 33);
#pragma unroll
            for (int k = 0; k < 33; ++k)
              row[k] = v[k];
          }
          __syncthreads();
          // forward Y
          for (int li = tid; li < 33 * nzc; li += kThreads)
          {
            double* col = T + (li / 33) * 33 * 33 + li % 33;
            double v[33];
#pragma unroll
            for (int k = 0; k < 33; ++k)
              v[k] = col[k * 33];
            dev::lift_regs<true>(v, 33);
#pragma unroll
            for (int k = 0; k < 33; ++k)
              col[k * 33] = v[k];
          }
          __syncthreads();
          double* dst = F + (size_t)z0 * 33 * 33;
          for (int i = tid; i < n; i += kThreads)
            dst[i] = T[i];
          __syncthreads();
        }
      }
      // inverse X (D = 33) then forward X of the one-level transform (Core/Wavelet.cpp:81)
      for (int li = tid; !planar && li < 33 * N[2]; li += kThreads)
      {
        double* row = F + li * 33;
        double v[33];
#pragma unroll
        for (int k = 0; k < 33; ++k)
          v[k] = row[k];
        dev::lift_regs<false>(v, 33);
        dev::lift_regs<true>(v, 33);
#pragma unroll
        for (int k = 0; k < 33; ++k)
          row[k] = v[k];
      }
      __syncthreads();
      ENC_PHASE(6)
      // forward Y (done above for planar bricks), and forward Z; subband normalisation applied
      // as the last sweep stores (Core/Wavelet.cpp:111-137)
      for (int li = tid; !planar && li < 33 * N[2]; li += kThreads)
      {
        const int x = li % 33, z = li / 33;
        double* col = F + z * 33 * 33 + x;
        double v[33];
#pragma unroll
        for (int k = 0; k < 33; ++k)
          v[k] = col[k * 33];
        dev::lift_regs<true>(v, 33);
#pragma unroll
        for (int k = 0; k < 33; ++k)
        {
          double f = v[k];
          if (fp.is2d)
          {
            const int s = ((x & 1) << 1) | (k & 1);
            f = ((fp.norm_mask >> s) & 1) ? __dmul_rn(f, fp.weight[s]) : f;
          }
          col[k * 33] = f;
        }
      }
      __syncthreads();
      ENC_PHASE(7)
      if (!fp.is2d)
      {
        for (int li = tid; li < 33 * 33; li += kThreads)
        {
          const int x = li % 33, y = li / 33;
          double* col = F + y * 33 + x;
          double v[33];
#pragma unroll
          for (int k = 0; k < 33; ++k)
            v[k] = col[k * 33 * 33];
          dev::lift_regs<true>(v, 33);
#pragma unroll
          for (int k = 0; k < 33; ++k)
          {
            const int s = ((x & 1) << 2) | ((y & 1) << 1) | (k & 1);
            col[k * 33 * 33] = ((fp.norm_mask >> s) & 1) ? __dmul_rn(v[k], fp.weight[s]) : v[k];
          }
        }
        __syncthreads();
      }
    }
    ENC_PHASE(8)

    // ---------------- C: low band to the parent ----------------
    if (a.parent_bricks && br.parent >= 0)
    {
      double* P = a.parent_bricks + (size_t)br.parent * (size_t)kNB3;
      const int nz = fp.is2d ? 1 : 16;
      for (int i = tid; i < 16 * 16 * nz; i += kThreads)
      {
        int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        int cz = fp.is2d ? 0 : 2 * z;
        __stcs(P + ((br.pos[2] * nz + z) * 33 + (br.pos[1] * 16 + y)) * 33 + (br.pos[0] * 16 + x),
               F[(cz * 33 + 2 * y) * 33 + 2 * x]);
      }
    }
    ENC_PHASE(9)

    // ---------------- D: block coding per subband ----------------
    for (int s = 0; s < fp.nsb; ++s)
    {
      // towards the end of the brick, ask L2 for the rows of this CTA's next brick
      if (a.level == 0 && s == (fp.nsb * 5) / 8 && it + (int)gridDim.x < a.last)
      {
        const int nx = a.order ? a.order[it + gridDim.x] : it + (int)gridDim.x;
        prefetch_rows(a.fields[a.bricks[nx].field], a.bricks[nx]);
      }
      code_subband<kThreads>(a, sm, Xp, OFF, NIN, P, F, SZ, false, bi, s, pacc_);
    }
  }
  ENC_PHASE_FLUSH
}

namespace cg = cooperative_groups;
#include "encode_split.cuh"

} // namespace

// ---------------------------------------------------------------------------
// device stage
// ---------------------------------------------------------------------------

struct batch_encoder::level_launch
{
  int level = 0;
  std::vector<enc_brick> bricks;
  std::vector<enc_field> fields;  // geom / nblocks device pointers filled by prepare
  std::vector<uint64_t> geom;     // [layout][8][kMaxBlocksPerSubband]
  std::vector<int> nblocks;       // [layout][8]
  std::vector<int> layout;        // field table entry -> its block layout
  std::vector<int> field_job;     // field table entry -> index in the batch
  std::vector<int> job_first;     // batch index -> first brick (-1: no such level)
  int nparents = 0;
  int planes = 32;
  int grid = 1;
  bool split = false;  // k_encode_split for the 3D bricks (bricks in shared memory)
  bool three = false;  // the three-CTA build of k_encode_level
  int split_grid = 2;
  // a level with 2D and 3D bricks: the 3D bricks (split_order) go to k_encode_split, the 2D
  // ones (slot_order) to k_encode_level
  std::vector<int> split_order, slot_order;
  int* d_split_order = nullptr;
  int* d_slot_order = nullptr;
  size_t smem = 0;
  unsigned long long cap = 0;
  enc_brick* d_bricks = nullptr;
  enc_field* d_fields = nullptr;
  uint64_t* d_geom = nullptr;
  int* d_nblocks = nullptr;
  unsigned long long* d_off = nullptr;
  unsigned long long* d_misc = nullptr;
  double* d_bmin = nullptr;
  double* d_bmax = nullptr;
  double* d_parents = nullptr;
  std::string sname;
  enc_args args;
  unsigned long long prefetched = 0;  // stream bytes copied to the pinned buffer while running
};

batch_encoder::batch_encoder(device_ctx* ctx, std::vector<batch_field>* fields, const std::string& tag)
  : ctx_(ctx), fields_(fields), tag_(tag)
{
}

batch_encoder::~batch_encoder() = default;

namespace
{

using encode_tiled_fn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                     const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

encode_tiled_fn tensor_map_encoder()
{
  static encode_tiled_fn fn = []() -> encode_tiled_fn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
    {
      cudaGetLastError();
      return nullptr;
    }
    return (encode_tiled_fn)p;
  }();
  return fn;
}

// The field of f as a 3D tensor (x fastest) read in boxes of 32 x 32 x kGz samples (one plane
// for 2D fields). TMA wants the base address and the row and plane pitches in multiples of 16
// bytes; fields that do not have them are gathered with ordinary copies. Box origins are
// brick origins, multiples of 32 samples along x: 16-byte aligned for either sample type.
bool field_tensor_map(const enc_field& f, CUtensorMap* map)
{
  encode_tiled_fn enc = tensor_map_encoder();
  const size_t esz = f.field_f32 ? 4 : 8;
  if (!enc || !f.field || ((uintptr_t)f.field & 15) || ((size_t)f.fdims[0] * esz) % 16 ||
      f.fdims[0] < 1 || f.fdims[1] < 1 || f.fdims[2] < 1 || f.fdims[0] > (1ll << 31) || f.fdims[1] > (1ll << 31) ||
      f.fdims[2] > (1ll << 31))
    return false;
  const cuuint64_t dims[3] = { (cuuint64_t)f.fdims[0], (cuuint64_t)f.fdims[1], (cuuint64_t)f.fdims[2] };
  const cuuint64_t pitch[2] = { (cuuint64_t)f.fdims[0] * esz, (cuuint64_t)f.fdims[0] * (cuuint64_t)f.fdims[1] * esz };
  const cuuint32_t box[3] = { 32, 32, (cuuint32_t)(f.is2d ? 1 : kGz) };
  const cuuint32_t estr[3] = { 1, 1, 1 };
  memset(map, 0, sizeof *map);
  return enc(map, f.field_f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
             const_cast<void*>(f.field), dims, pitch, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

} // namespace

namespace
{

// Clusters of k_encode_split that fit on the device at once (0: the kernel cannot run; its
// shared memory is set once per process).
int split_clusters()
{
  static int n = [] {
    const size_t smem = split_smem_bytes();
    if (cudaFuncSetAttribute(k_encode_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    {
      cudaGetLastError();
      return 0;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(sms > 1 ? sms & ~1 : 2));
    cfg.blockDim = dim3(kSplitThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = 2;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_encode_split, &cfg) != cudaSuccess)
    {
      cudaGetLastError();
      return 0;
    }
    return clusters;
  }();
  return n;
}

// Whether the 3D bricks of a launch go to k_encode_split: IDX2G_ENC_SPLIT=0 / 1 decides, else
// the tuning's choice, else the library's default.
bool split_wanted(const batch_tuning& t)
{
  const char* env = std::getenv("IDX2G_ENC_SPLIT");
  if (env && (env[0] == '0' || env[0] == '1'))
    return env[0] == '1';
  if (t.split >= 0)
    return t.split == 1;
  return kSplitByDefault;
}

} // namespace

bool split_kernel_available() { return kSplitOffered && split_clusters() > 0; }

int batch_encoder::prepare(const batch_tuning& t)
{
  tune_ = t;
  std::vector<batch_field>& J = *fields_;
  int L = 0;
  for (batch_field& j : J)
  {
    const dataset_format& f = *j.f;
    if (f.bit_planes_per_chunk < 1 || f.bit_planes_per_chunk > 8)
      return OptionNotSupported;  // keys of coded planes stay non-negative up to 8 planes per key
    if (f.brick_dims.x != 32 || f.brick_dims.y != 32 || (f.brick_dims.z != 32 && f.brick_dims.z != 1))
      return OptionNotSupported;
    L = f.nlevels > L ? f.nlevels : L;
    j.outs->assign((size_t)f.nlevels, level_output());
    j.level_ms.assign((size_t)f.nlevels, 0.f);
    j.level_bytes.assign((size_t)f.nlevels, 0);
  }
  // first brick of every field in every level's launch
  std::vector<std::vector<int>> first((size_t)L + 1, std::vector<int>(J.size(), -1));
  std::vector<int> count((size_t)L + 1, 0);
  for (int l = 0; l < L; ++l)
    for (size_t j = 0; j < J.size(); ++j)
      if (l < J[j].f->nlevels)
      {
        first[(size_t)l][j] = count[(size_t)l];
        count[(size_t)l] += (int)J[j].plan->levels[(size_t)l].size();
      }
  levels_.clear();
  cudaStream_t st = ctx_->stream;
  size_t max_grid = 1;
  for (int l = 0; l < L; ++l)
  {
    levels_.emplace_back(new level_launch());
    level_launch& ll = *levels_.back();
    ll.level = l;
    ll.job_first = first[(size_t)l];
    ll.nparents = count[(size_t)l + 1];
    unsigned long long cap = 16ull << 20;
    // block geometry tables: one per distinct subband layout (2D or 3D, brick and block dims,
    // coarsest level or not), shared by the fields that have it
    std::map<std::string, int> layouts;
    std::vector<int>& field_layout = ll.layout;
    for (size_t j = 0; j < J.size(); ++j)
    {
      const dataset_format& f = *J[j].f;
      if (l >= f.nlevels)
        continue;
      const int fi = (int)ll.fields.size();
      enc_field ef;
      memset(&ef, 0, sizeof ef);
      ef.is2d = f.is2d();
      ef.f32_exp = f.type == dtype::float32;
      ef.etol = exponent_f64(f.tolerance);
      ef.end_bp = f.type == dtype::float32 ? 32 : 64;
      ef.nsb = f.nsubbands();
      ef.order = f.transform_order;
      ef.field = J[j].d_field;
      ef.field_f32 = J[j].f32;
      const v3 fd = J[j].field_dims.x > 0 ? J[j].field_dims : f.dims;
      ef.fdims[0] = fd.x;
      ef.fdims[1] = fd.y;
      ef.fdims[2] = fd.z;
      level_weights(f, l, ef.weight, &ef.norm_mask);
      ef.bpc = f.bit_planes_per_chunk;
      if (ef.end_bp == 64)
        ll.planes = 64;
      ll.fields.push_back(ef);
      ll.field_job.push_back((int)j);
      char lk[96];
      snprintf(lk, sizeof lk, "%d %d %d %d/%d %d %d/%d", (int)ef.is2d, f.brick_dims_ext.x, f.brick_dims_ext.y,
               f.brick_dims_ext.z, f.block_dims.x, f.block_dims.y, f.block_dims.z, (int)(l + 1 < f.nlevels));
      auto li = layouts.find(lk);
      if (li == layouts.end())
      {
        const int slot = (int)layouts.size();
        li = layouts.emplace(lk, slot).first;
        ll.geom.resize((size_t)(slot + 1) * 8 * kMaxBlocksPerSubband, 0);
        ll.nblocks.resize((size_t)(slot + 1) * 8, 0);
        for (int sb = 0; sb < ef.nsb; ++sb)
        {
          std::vector<block_geom> g;
          subband_blocks(f, l, sb, &g);
          ll.nblocks[(size_t)slot * 8 + (size_t)sb] = (int)g.size();
          for (size_t b = 0; b < g.size(); ++b)
            ll.geom[((size_t)slot * 8 + (size_t)sb) * kMaxBlocksPerSubband + b] =
              (uint64_t)g[b].dx | ((uint64_t)g[b].dy << 8) | ((uint64_t)g[b].dz << 16) |
              ((uint64_t)g[b].bx << 24) | ((uint64_t)g[b].by << 32) | ((uint64_t)g[b].bz << 40);
        }
      }
      field_layout.push_back(li->second);
      const std::vector<brick_entry>& bricks = J[j].plan->levels[(size_t)l];
      const bool has_parent = l + 1 < f.nlevels;
      // level 0 reads the field: brick coordinates relative to the samples the buffer holds
      const v3 ob = l == 0 ? J[j].field_origin / f.brick_dims : v3(0);
      for (const brick_entry& e : bricks)
        ll.bricks.push_back(enc_brick{ { e.brick3.x - ob.x, e.brick3.y - ob.y, e.brick3.z - ob.z },
                                       { e.valid.x, e.valid.y, e.valid.z },
                                       has_parent ? first[(size_t)l + 1][j] + e.parent : -1,
                                       { e.pos_in_parent.x, e.pos_in_parent.y, e.pos_in_parent.z },
                                       fi });
      const unsigned long long NB = (unsigned long long)(ef.is2d ? 33 * 33 : kNB3);
      cap += (unsigned long long)bricks.size() * NB * 2ull;
    }
    const int nbr = (int)ll.bricks.size();
    // CTAs per SM: as many as the level's shared memory and the kernel's registers let reside
    // (or fewer, when the tuning asks), so that no CTA of the grid waits for a place
    // the level-0 launch of many bricks takes the three-CTA build when three CTAs fit
    ll.three = kThreeCtas && l == 0 && tune_.ctas_per_sm == 0 && nbr >= 6 * ctx_->num_sms &&
               enc_occupancy(enc_smem_bytes(ll.planes), true) >= 3;
    const int occ = enc_occupancy(enc_smem_bytes(ll.planes), ll.three);
    const int cps = tune_.ctas_per_sm > 0 && tune_.ctas_per_sm < occ ? tune_.ctas_per_sm : occ;
    const int lim = cps * ctx_->num_sms;
    ll.grid = nbr < lim ? (nbr > 0 ? nbr : 1) : lim;
    {
      // the 3D bricks go to the split kernel when it is wanted and the device runs it
      ll.split_order.clear();
      ll.slot_order.clear();
      for (int i = 0; i < nbr; ++i)
        (ll.fields[(size_t)ll.bricks[(size_t)i].field].is2d ? ll.slot_order : ll.split_order).push_back(i);
      ll.split = !ll.split_order.empty() && split_wanted(tune_) && split_clusters() > 0;
      const int n3 = (int)ll.split_order.size(), nc = split_clusters();
      ll.split_grid = 2 * (n3 < nc ? n3 : nc);
      if (ll.split && !ll.slot_order.empty())
      {
        char on[96];
        snprintf(on, sizeof on, "enc.%s.L%d.order3", tag_.c_str(), l);
        ll.d_split_order = (int*)ctx_->ws(on, ll.split_order.size() * 4);
        snprintf(on, sizeof on, "enc.%s.L%d.order2", tag_.c_str(), l);
        ll.d_slot_order = (int*)ctx_->ws(on, ll.slot_order.size() * 4);
        if (!ll.d_split_order || !ll.d_slot_order)
          return OutOfMemory;
        cudaMemcpyAsync(ll.d_split_order, ll.split_order.data(), ll.split_order.size() * 4, cudaMemcpyHostToDevice,
                        st);
        cudaMemcpyAsync(ll.d_slot_order, ll.slot_order.data(), ll.slot_order.size() * 4, cudaMemcpyHostToDevice, st);
      }
    }
    max_grid = (size_t)ll.grid > max_grid ? (size_t)ll.grid : max_grid;
    char name[96];
    snprintf(name, sizeof name, "enc.%s.L%d.stream", tag_.c_str(), l);
    ll.sname = name;
    ll.cap = cap > ctx_->ws_size(name) ? cap : ctx_->ws_size(name);
    auto wsn = [&](const char* what, size_t bytes) -> void* {
      char n2[96];
      snprintf(n2, sizeof n2, "enc.%s.L%d.%s", tag_.c_str(), l, what);
      return ctx_->ws(n2, bytes);
    };
    ll.d_bricks = (enc_brick*)wsn("bricks", sizeof(enc_brick) * (size_t)(nbr > 0 ? nbr : 1));
    ll.d_fields = (enc_field*)wsn("fields", sizeof(enc_field) * (ll.fields.size() + 1));
    ll.d_geom = (uint64_t*)wsn("geom", (ll.geom.size() + 1) * 8);
    ll.d_nblocks = (int*)wsn("nblocks", (ll.nblocks.size() + 1) * 4);
    ll.d_off = (unsigned long long*)wsn("off", (size_t)(nbr > 0 ? nbr : 1) * 8 * 8);
    ll.d_misc = (unsigned long long*)wsn("misc", 64);
    if (l == 0)
    {
      ll.d_bmin = (double*)wsn("bmin", (size_t)(nbr > 0 ? nbr : 1) * 8);
      ll.d_bmax = (double*)wsn("bmax", (size_t)(nbr > 0 ? nbr : 1) * 8);
    }
    if (ll.nparents > 0)
      ll.d_parents = (double*)wsn("parents", (size_t)ll.nparents * (size_t)kNB3 * 8);
    uint32_t* d_stream = (uint32_t*)ctx_->ws(ll.sname, (size_t)ll.cap);
    if (!ll.d_bricks || !ll.d_fields || !ll.d_geom || !ll.d_nblocks || !ll.d_off || !ll.d_misc ||
        (l == 0 && (!ll.d_bmin || !ll.d_bmax)) || (ll.nparents > 0 && !ll.d_parents) || !d_stream)
      return OutOfMemory;
    ll.cap = ctx_->ws_size(ll.sname);
    for (size_t fi = 0; fi < ll.fields.size(); ++fi)
    {
      ll.fields[fi].geom = ll.d_geom + (size_t)field_layout[fi] * 8 * kMaxBlocksPerSubband;
      ll.fields[fi].nblocks = ll.d_nblocks + (size_t)field_layout[fi] * 8;
    }
    if (l == 0)
    {
      // level 0 reads each field through a tensor map where the field's layout allows TMA
      std::vector<CUtensorMap> maps(ll.fields.size());
      std::vector<char> has(ll.fields.size(), 0);
      size_t nmaps = 0;
      for (size_t fi = 0; fi < ll.fields.size(); ++fi)
        if (field_tensor_map(ll.fields[fi], &maps[fi]))
        {
          has[fi] = 1;
          ++nmaps;
        }
      if (nmaps)
      {
        CUtensorMap* d_maps = (CUtensorMap*)wsn("tmaps", sizeof(CUtensorMap) * ll.fields.size());
        CUtensorMap* h_maps = (CUtensorMap*)ctx_->pinned("enc." + tag_ + ".tmaps", sizeof(CUtensorMap) * ll.fields.size());
        if (!d_maps || !h_maps)
          return OutOfMemory;
        memcpy(h_maps, maps.data(), sizeof(CUtensorMap) * ll.fields.size());
        cudaMemcpyAsync(d_maps, h_maps, sizeof(CUtensorMap) * ll.fields.size(), cudaMemcpyHostToDevice, st);
        for (size_t fi = 0; fi < ll.fields.size(); ++fi)
          ll.fields[fi].tmap = has[fi] ? d_maps + fi : nullptr;
      }
    }
    if (nbr > 0)
      cudaMemcpyAsync(ll.d_bricks, ll.bricks.data(), sizeof(enc_brick) * (size_t)nbr, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ll.d_fields, ll.fields.data(), sizeof(enc_field) * ll.fields.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ll.d_geom, ll.geom.data(), ll.geom.size() * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ll.d_nblocks, ll.nblocks.data(), ll.nblocks.size() * 4, cudaMemcpyHostToDevice, st);
    enc_args& a = ll.args;
    memset(&a, 0, sizeof a);
    a.level = l;
    a.nbricks = nbr;
    a.first = 0;
    a.last = nbr;
    a.order = nullptr;
    a.planes = ll.planes;
    a.fields = ll.d_fields;
    a.bricks = ll.d_bricks;
    a.in_bricks = l > 0 ? levels_[(size_t)l - 1]->d_parents : nullptr;
    a.parent_bricks = ll.d_parents;
    a.offset = ll.d_off;
    a.stream = d_stream;
    a.cap_bytes = ll.cap;
    a.cursor = ll.d_misc;
    a.error = (int*)(ll.d_misc + 1);
    a.bmin = ll.d_bmin;
    a.bmax = ll.d_bmax;
    ll.smem = enc_smem_bytes(ll.planes);
  }
  double* d_slots = (double*)ctx_->ws("enc.slots", max_grid * (size_t)kNB3 * 8);
  if (!d_slots)
    return OutOfMemory;
  size_t max_smem = 0;
  for (auto& ll : levels_)
  {
    ll->args.slots = d_slots;
    max_smem = ll->smem > max_smem ? ll->smem : max_smem;
  }
  cudaFuncSetAttribute(enc_kernel(false), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
  cudaFuncSetAttribute(enc_kernel(true), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
  return cudaGetLastError() == cudaSuccess ? NoError : CudaError;
}

int batch_encoder::enqueue_level(int l)
{
  level_launch& ll = *levels_[(size_t)l];
  cudaStream_t st = ctx_->stream;
  cudaMemsetAsync(ll.d_misc, 0, 64, st);
  if (ll.nparents > 0)
    cudaMemsetAsync(ll.d_parents, 0, (size_t)ll.nparents * (size_t)kNB3 * 8, st);
  if (ll.args.nbricks > 0)
  {
    if (ll.split && !ll.slot_order.empty())
    {
      // 3D bricks by the split kernel, 2D bricks by the slot kernel, one after the other
      enc_args a3 = ll.args;
      a3.order = ll.d_split_order;
      a3.last = (int)ll.split_order.size();
      k_encode_split<<<ll.split_grid, kSplitThreads, split_smem_bytes(), st>>>(a3);
      enc_args a2 = ll.args;
      a2.order = ll.d_slot_order;
      a2.last = (int)ll.slot_order.size();
      enc_kernel(ll.three)<<<a2.last < ll.grid ? a2.last : ll.grid, kThreads, ll.smem, st>>>(a2);
      launches_ += 2;
      ctx_->launches += 2;
    }
    else
    {
      if (ll.split)
        k_encode_split<<<ll.split_grid, kSplitThreads, split_smem_bytes(), st>>>(ll.args);
      else
        enc_kernel(ll.three)<<<ll.grid, kThreads, ll.smem, st>>>(ll.args);
      ++launches_;
      ++ctx_->launches;
    }
  }
  return cudaGetLastError() == cudaSuccess ? NoError : CudaError;
}

int batch_encoder::enqueue_level0_streamed(const void* host, void* staged, int* nbands)
{
  *nbands = 0;
  level_launch& ll = *levels_[0];
  cudaStream_t st = ctx_->stream, cs = ctx_->copies();
  const int nbr = ll.args.nbricks;
  if (!cs || ll.fields.size() != 1 || ll.fields[0].is2d || nbr <= 0)
    return InvalidArgument;
  const enc_field& ef = ll.fields[0];
  const size_t plane = (size_t)ef.fdims[0] * (size_t)ef.fdims[1] * (ef.field_f32 ? 4 : 8);
  const long long nz = ef.fdims[2];
  // entries by brick row (z); bands of whole rows, about kBands of them
  std::vector<int> order((size_t)nbr);
  for (int i = 0; i < nbr; ++i)
    order[(size_t)i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return ll.bricks[(size_t)x].b3[2] < ll.bricks[(size_t)y].b3[2]; });
  constexpr int kBands = 16;
  std::vector<int> cuts(1, 0);
  auto row = [&](int i) { return ll.bricks[(size_t)order[(size_t)i]].b3[2]; };
  for (int g = 1; g < kBands; ++g)
  {
    int c = (int)((long long)nbr * g / kBands);
    while (c > 0 && c < nbr && row(c) == row(c - 1))
      ++c;
    if (c > cuts.back() && c < nbr)
      cuts.push_back(c);
  }
  cuts.push_back(nbr);
  const int nb = (int)cuts.size() - 1;
  int* d_order = (int*)ctx_->ws("enc.order", (size_t)nbr * 4);
  int* h_order = (int*)ctx_->pinned("enc.order", (size_t)nbr * 4);
  if (!d_order || !h_order)
    return OutOfMemory;
  memcpy(h_order, order.data(), (size_t)nbr * 4);
  cudaMemcpyAsync(d_order, h_order, (size_t)nbr * 4, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(ll.d_misc, 0, 64, st);
  if (ll.nparents > 0)
    cudaMemsetAsync(ll.d_parents, 0, (size_t)ll.nparents * (size_t)kNB3 * 8, st);
  // the coarser levels by bands of level 0: a brick's band is the latest band among its
  // children (the bricks that hand it their low bands), its bricks ordered by band
  follow_events_.assign(levels_.size(), {});
  std::vector<std::vector<int>> up_cuts(levels_.size());
  std::vector<int*> up_order(levels_.size(), nullptr);
  {
    std::vector<int> prev_band((size_t)nbr, 0);
    for (int g = 0; g < nb; ++g)
      for (int i = cuts[(size_t)g]; i < cuts[(size_t)g + 1]; ++i)
        prev_band[(size_t)order[(size_t)i]] = g;
    for (size_t l = 1; l < levels_.size(); ++l)
    {
      const level_launch& pl = *levels_[l - 1];
      level_launch& ul = *levels_[l];
      const int n = ul.args.nbricks;
      if (ul.split || ul.fields.size() != 1 || ul.fields[0].is2d || n <= 0)
        break;
      std::vector<int> parent_of(pl.bricks.size());
      for (size_t j = 0; j < pl.bricks.size(); ++j)
        parent_of[j] = pl.bricks[j].parent;
      level_bands lb = follow_bands(prev_band, parent_of, n, nb);
      const std::vector<int>& uo = lb.order;
      up_cuts[l] = lb.cuts;
      char nm[32];
      snprintf(nm, sizeof nm, "enc.order%zu", l);
      int* d_uo = (int*)ctx_->ws(nm, (size_t)n * 4);
      int* h_uo = (int*)ctx_->pinned(nm, (size_t)n * 4);
      if (!d_uo || !h_uo)
        return OutOfMemory;
      memcpy(h_uo, uo.data(), (size_t)n * 4);
      cudaMemcpyAsync(d_uo, h_uo, (size_t)n * 4, cudaMemcpyHostToDevice, st);
      up_order[l] = d_uo;
      cudaMemsetAsync(ul.d_misc, 0, 64, st);
      if (ul.nparents > 0)
        cudaMemsetAsync(ul.d_parents, 0, (size_t)ul.nparents * (size_t)kNB3 * 8, st);
      prev_band.swap(lb.band);
    }
  }
  // the copy stream starts after the work already on the stream (the staging buffer may
  // still be read by it)
  cudaEvent_t start = ctx_->ev(127);
  if (!start)
    return CudaError;
  cudaEventRecord(start, st);
  cudaStreamWaitEvent(cs, start, 0);
  // every band's planes on the copy stream, then each band's launch after its copy
  for (int g = 0; g < nb; ++g)
  {
    const long long z0 = (long long)row(cuts[(size_t)g]) * 32;
    long long z1 = ((long long)row(cuts[(size_t)g + 1] - 1) + 1) * 32;
    z1 = z1 < nz ? z1 : nz;
    if (g + 1 == nb)
      z1 = nz;
    cudaEvent_t ce = ctx_->ev(128 + (size_t)g);
    if (!ce)
      return CudaError;
    if (z1 > z0)
      cudaMemcpyAsync((uint8_t*)staged + (size_t)z0 * plane, (const uint8_t*)host + (size_t)z0 * plane,
                      (size_t)(z1 - z0) * plane, cudaMemcpyHostToDevice, cs);
    cudaEventRecord(ce, cs);
  }
  unsigned long long* h_cur = (unsigned long long*)ctx_->pinned("enc.cursor", (size_t)nb * 8);
  if (!h_cur)
    return OutOfMemory;
  for (int g = 0; g < nb; ++g)
  {
    cudaEvent_t t0 = ctx_->ev(2 * (size_t)g), t1 = ctx_->ev(2 * (size_t)g + 1);
    cudaEvent_t tc = ctx_->ev(160 + (size_t)g);
    if (!t0 || !t1 || !tc)
      return CudaError;
    cudaStreamWaitEvent(st, ctx_->ev(128 + (size_t)g), 0);
    cudaEventRecord(t0, st);
    enc_args a = ll.args;
    a.first = cuts[(size_t)g];
    a.last = cuts[(size_t)g + 1];
    a.order = d_order;
    const int n = a.last - a.first;
    if (ll.split)
      k_encode_split<<<2 * (n < ll.split_grid / 2 ? n : ll.split_grid / 2), kSplitThreads, split_smem_bytes(), st>>>(a);
    else
      enc_kernel(ll.three)<<<n < ll.grid ? n : ll.grid, kThreads, ll.smem, st>>>(a);
    cudaEventRecord(t1, st);
    // the region cursor after the band: its regions end there
    cudaMemcpyAsync(h_cur + g, ll.d_misc, 8, cudaMemcpyDeviceToHost, st);
    cudaEventRecord(tc, st);
    ++launches_;
    ++ctx_->launches;
    // the coarser levels' bricks whose children have all run
    for (size_t l = 1; l < levels_.size() && up_order[l]; ++l)
    {
      const int u0 = up_cuts[l][(size_t)g], u1 = up_cuts[l][(size_t)g + 1];
      if (u1 <= u0)
        continue;
      level_launch& ul = *levels_[l];
      const int evi = 256 + 2 * (int)(l - 1) * 32 + 2 * g;  // (an event pair per level and band)
      cudaEvent_t u_t0 = ctx_->ev((size_t)evi), u_t1 = ctx_->ev((size_t)evi + 1);
      if (!u_t0 || !u_t1)
        return CudaError;
      cudaEventRecord(u_t0, st);
      enc_args ua = ul.args;
      ua.first = u0;
      ua.last = u1;
      ua.order = up_order[l];
      enc_kernel(ul.three)<<<u1 - u0 < ul.grid ? u1 - u0 : ul.grid, kThreads, ul.smem, st>>>(ua);
      cudaEventRecord(u_t1, st);
      follow_events_[l].push_back(evi);
      ++launches_;
      ++ctx_->launches;
    }
  }
  *nbands = nb;
  return cudaGetLastError() == cudaSuccess ? NoError : CudaError;
}

float batch_encoder::followed_ms(int l) const
{
  float total = 0;
  if (l <= 0 || (size_t)l >= follow_events_.size())
    return 0;
  for (int ev : follow_events_[(size_t)l])
  {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx_->ev((size_t)ev), ctx_->ev((size_t)ev + 1));
    total += ms;
  }
  return total;
}

void batch_encoder::stream_out_level0(int nbands)
{
  level_launch& ll = *levels_[0];
  ll.prefetched = 0;
  char name[96];
  snprintf(name, sizeof name, "enc.pin.%s.%d", tag_.c_str(), 0);
  const size_t room = ctx_->pinned_size(name);
  cudaStream_t os = ctx_->copies_out();
  const unsigned long long* h_cur = (const unsigned long long*)ctx_->pinned("enc.cursor", (size_t)nbands * 8);
  if (!room || !os || !h_cur)
    return;
  uint8_t* pin = (uint8_t*)ctx_->pinned(name, room);
  unsigned long long done = 0;
  for (int g = 0; g < nbands; ++g)
  {
    if (cudaEventSynchronize(ctx_->ev(160 + (size_t)g)) != cudaSuccess)
      break;
    const unsigned long long end = h_cur[g];
    if (end > ll.cap || end > room)
      break;  // the regions overflowed (the level runs again) or the buffer is short
    if (end > done)
      cudaMemcpyAsync(pin + done, (const uint8_t*)ll.args.stream + done, (size_t)(end - done),
                      cudaMemcpyDeviceToHost, os);
    done = end;
  }
  ll.prefetched = done;
}

int batch_encoder::collect_level(int l, bool keep_device)
{
  level_launch& ll = *levels_[(size_t)l];
  cudaStream_t st = ctx_->stream;
  // copies of this level's streams still in flight end before the buffer is looked at
  const unsigned long long prefetched = ll.prefetched;
  ll.prefetched = 0;
  if (prefetched && cudaStreamSynchronize(ctx_->copies_out()) != cudaSuccess)
    return CudaError;
  std::vector<batch_field>& J = *fields_;
  const int nbr = ll.args.nbricks;
  unsigned long long misc[2] = { 0, 0 };
  for (int attempt = 0;; ++attempt)
  {
    cudaMemcpyAsync(misc, ll.d_misc, 16, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    const int err = (int)(misc[1] & 0xffffffffu);
    if (err == 4)
      return CudaError;  // a bulk copy of the gather did not complete
    if (err == 1)
      return DeviceStreamOverflow;  // more than kKeyWindow channels in one subband
    if (err != 2 && err != 8)
      break;
    if (attempt >= 3)
      return DeviceStreamOverflow;
    if (err == 8)
    {
      // a block of the split kernel needed more than its 32-plane tables: the level again with
      // the global-slot kernel (tables of ll.planes planes)
      ll.split = false;
      cudaEventRecord(ctx_->ev0, st);
      int e = enqueue_level(l);
      cudaEventRecord(ctx_->ev1, st);
      if (e)
        return e;
      if (cudaStreamSynchronize(st) != cudaSuccess)
        return CudaError;
      float ms = 0;
      cudaEventElapsedTime(&ms, ctx_->ev0, ctx_->ev1);
      kernel_ms_ += ms;
      continue;
    }
    // the regions did not fit: the level again with room for all of them (its outputs for
    // the next level are recomputed identically)
    uint32_t* d_stream = (uint32_t*)ctx_->ws(ll.sname, (size_t)(misc[0] + (1ull << 20)));
    if (!d_stream)
      return OutOfMemory;
    ll.cap = ctx_->ws_size(ll.sname);
    ll.args.stream = d_stream;
    ll.args.cap_bytes = ll.cap;
    cudaEventRecord(ctx_->ev0, st);
    int e = enqueue_level(l);
    cudaEventRecord(ctx_->ev1, st);
    if (e)
      return e;
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx_->ev0, ctx_->ev1);
    kernel_ms_ += ms;
  }
  ctx_->ws_mark_dirty(ll.sname, (size_t)(misc[0] < ll.cap ? misc[0] : ll.cap));
  const unsigned long long used = misc[0];
  // per field: exponent bytes, level output, value range
  std::vector<unsigned long long> off;
  const uint8_t* pin = nullptr;
  if (!keep_device && nbr > 0)
  {
    off.resize((size_t)nbr * 8);
    cudaMemcpyAsync(off.data(), ll.d_off, off.size() * 8, cudaMemcpyDeviceToHost, st);
    if (used)
    {
      char name[96];
      snprintf(name, sizeof name, "enc.pin.%s.%d", tag_.c_str(), l);
      const bool have = prefetched == used && ctx_->pinned_size(name) >= (size_t)used;
      pin = (const uint8_t*)ctx_->pinned(name, (size_t)used);
      if (!pin)
        return OutOfMemory;
      if (!have)
        cudaMemcpyAsync((void*)pin, ll.args.stream, (size_t)used, cudaMemcpyDeviceToHost, st);
    }
  }
  std::vector<double> mn, mx;
  if (l == 0 && nbr > 0)
  {
    mn.resize((size_t)nbr);
    mx.resize((size_t)nbr);
    cudaMemcpyAsync(mn.data(), ll.d_bmin, (size_t)nbr * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(mx.data(), ll.d_bmax, (size_t)nbr * 8, cudaMemcpyDeviceToHost, st);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return CudaError;
  for (size_t fi = 0; fi < ll.fields.size(); ++fi)
  {
    batch_field& bf = J[(size_t)ll.field_job[fi]];
    const dataset_format& f = *bf.f;
    const int j0 = ll.job_first[(size_t)ll.field_job[fi]];
    const int jn = (int)bf.plan->levels[(size_t)l].size();
    const int nsb = f.nsubbands();
    level_output& o = (*bf.outs)[(size_t)l];
    o.nbricks = jn;
    o.nsb = nsb;
    o.nexps.assign((size_t)nsb, 0);
    long long eb = 0;
    for (int sb = 0; sb < nsb; ++sb)
    {
      o.nexps[(size_t)sb] = ll.nblocks[(size_t)ll.layout[fi] * 8 + (size_t)sb];
      eb += (long long)jn * o.nexps[(size_t)sb] * (f.type == dtype::float32 ? 1 : 2);
    }
    bf.exp_bytes += eb;
    if (!keep_device)
    {
      o.offset.resize((size_t)jn * (size_t)nsb);
      for (int b = 0; b < jn; ++b)
        for (int sb = 0; sb < nsb; ++sb)
          o.offset[(size_t)b * (size_t)nsb + (size_t)sb] = off[(size_t)(j0 + b) * 8 + (size_t)sb];
      o.ext_stream = pin;
    }
    if (ll.fields.size() == 1)
    {
      bf.stream_bytes += (long long)used;
      bf.level_bytes[(size_t)l] = (long long)used + eb;
    }
    if (l == 0)
      for (int b = 0; b < jn; ++b)
      {
        const double a0 = mn[(size_t)(j0 + b)], a1 = mx[(size_t)(j0 + b)];
        bf.vmin = a0 < bf.vmin ? a0 : bf.vmin;
        bf.vmax = bf.vmax < a1 ? a1 : bf.vmax;
      }
  }
  return NoError;
}

void batch_encoder::device_level(int l, const uint8_t** stream, const unsigned long long** offset) const
{
  const level_launch& ll = *levels_[(size_t)l];
  *stream = reinterpret_cast<const uint8_t*>(ll.args.stream);
  *offset = ll.d_off;
}

int batch_encoder::copy_level_out(int l, level_output* o)
{
  level_launch& ll = *levels_[(size_t)l];
  cudaStream_t st = ctx_->stream;
  const int nbr = (int)ll.bricks.size();
  unsigned long long used = 0;
  cudaMemcpyAsync(&used, ll.d_misc, 8, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return CudaError;
  std::vector<unsigned long long> off((size_t)nbr * 8);
  const uint8_t* pin = nullptr;
  if (nbr > 0)
    cudaMemcpyAsync(off.data(), ll.d_off, off.size() * 8, cudaMemcpyDeviceToHost, st);
  if (used)
  {
    char name[96];
    snprintf(name, sizeof name, "enc.pin.%s.%d", tag_.c_str(), l);
    pin = (const uint8_t*)ctx_->pinned(name, (size_t)used);
    if (!pin)
      return OutOfMemory;
    cudaMemcpyAsync((void*)pin, ll.args.stream, (size_t)used, cudaMemcpyDeviceToHost, st);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return CudaError;
  const int nsb = o->nsb;
  o->offset.resize((size_t)nbr * (size_t)nsb);
  for (int b = 0; b < nbr; ++b)
    for (int sb = 0; sb < nsb; ++sb)
      o->offset[(size_t)b * (size_t)nsb + (size_t)sb] = off[(size_t)b * 8 + (size_t)sb];
  o->ext_stream = pin;
  return NoError;
}

int batch_encoder::run_all(bool use_graph, bool keep_device)
{
  cudaStream_t st = ctx_->stream;
  const int L = nlevels();
  if (use_graph)
  {
    // the level launches as one graph, kept on the context for the next batch of the same
    // launches: a byte image of every launch's parameters says whether the cached graph
    // (captured with the same workspace buffers, grids and arguments) still applies
    std::string sig;
    for (int l = 0; l < L; ++l)
    {
      const level_launch& ll = *levels_[(size_t)l];
      const int nsplit = (int)ll.split_order.size(), nslot = (int)ll.slot_order.size();
      const void* ptrs[5] = { ll.d_misc, ll.d_parents, ll.d_split_order, ll.d_slot_order, nullptr };
      const long long v[8] = { ll.grid, ll.split_grid, (long long)ll.split, (long long)ll.smem, ll.nparents,
                               nsplit, nslot, 0 };
      sig.append(reinterpret_cast<const char*>(&ll.args), sizeof ll.args);
      sig.append(reinterpret_cast<const char*>(ptrs), sizeof ptrs);
      sig.append(reinterpret_cast<const char*>(v), sizeof v);
    }
    device_ctx::cached_graph& cg_ = ctx_->graphs[tag_];
    if (!cg_.exec || cg_.launches != sig)
    {
      if (cg_.exec)
        cudaGraphExecDestroy(cg_.exec);
      cg_.exec = nullptr;
      cg_.launches.clear();
      cudaGraph_t g = nullptr;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return CudaError;
      int e = NoError;
      const long long before = launches_;
      for (int l = 0; l < L && !e; ++l)
        e = enqueue_level(l);
      const cudaError_t ce = cudaStreamEndCapture(st, &g);
      cudaGraphExec_t ge = nullptr;
      if (e || ce != cudaSuccess || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
      {
        if (g)
          cudaGraphDestroy(g);
        return e ? e : CudaError;
      }
      cudaGraphDestroy(g);
      cg_.exec = ge;
      cg_.launches = sig;
      cg_.kernels = launches_ - before;
      launches_ = before;
      ctx_->launches -= cg_.kernels;
    }
    graph_launches_ = cg_.kernels;
    stage_timer tt;
    cudaEventRecord(ctx_->ev0, st);
    cudaGraphLaunch(cg_.exec, st);
    cudaEventRecord(ctx_->ev1, st);
    launches_ += graph_launches_;
    ctx_->launches += graph_launches_;
    const cudaError_t se = cudaStreamSynchronize(st);
    tt.lap("batch.graph_run");
    if (se != cudaSuccess)
      return CudaError;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx_->ev0, ctx_->ev1);
    kernel_ms_ += ms;
    for (int l = 0; l < L; ++l)
    {
      const int e = collect_level(l, keep_device);
      if (e)
        return e;
    }
    tt.lap("batch.collect");
    return NoError;
  }
  for (int l = 0; l < L; ++l)
  {
    cudaEventRecord(ctx_->ev0, st);
    int e = enqueue_level(l);
    cudaEventRecord(ctx_->ev1, st);
    if (e)
      return e;
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx_->ev0, ctx_->ev1);
    kernel_ms_ += ms;
    for (batch_field& bf : *fields_)
      if (l < (int)bf.level_ms.size())
        bf.level_ms[(size_t)l] += ms;
    e = collect_level(l, keep_device);
    if (e)
      return e;
  }
  return NoError;
}

gpu_coder::gpu_coder(device_ctx* ctx, const dataset_format& f, const void* d_field, bool field_f32)
  : ctx_(ctx), f_(f)
{
  fields_.resize(1);
  fields_[0].f = &f_;
  fields_[0].d_field = d_field;
  fields_[0].f32 = field_f32;
  fields_[0].outs = &outs_;
}

gpu_coder::~gpu_coder() {}

int gpu_coder::run_level(int level, const encode_plan& plan, level_output* out)
{
  cudaStream_t st = ctx_->stream;
  if (level == 0 || !enc_)
  {
    fields_[0].plan = &plan;
    enc_.reset(new batch_encoder(ctx_, &fields_, "s"));
    int e = enc_->prepare(batch_tuning());
    if (e)
      return e;
  }
  if (level >= enc_->nlevels())
    return UnknownError;
  const double before = enc_->kernel_ms();
  stage_timer tt;
  float ms = 0;
  stream_fence host_copies{ level == 0 && host_field_ ? ctx_->copies() : nullptr };
  if (level == 0 && host_field_)
  {
    // the field is still in pinned host memory: its copy overlaps the level's launches
    int nb = 0;
    int e = enc_->enqueue_level0_streamed(host_field_, (void*)fields_[0].d_field, &nb);
    if (e)
      return e;
    if (!keep_device_)
      enc_->stream_out_level0(nb);
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    for (int g = 0; g < nb; ++g)
    {
      float m = 0;
      cudaEventElapsedTime(&m, ctx_->ev(2 * (size_t)g), ctx_->ev(2 * (size_t)g + 1));
      ms += m;
    }
  }
  else if (enc_->followed(level))
  {
    // launched with level 0's bands
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    ms = enc_->followed_ms(level);
  }
  else
  {
    cudaEventRecord(ctx_->ev0, st);
    int e = enc_->enqueue_level(level);
    cudaEventRecord(ctx_->ev1, st);
    if (e)
      return e;
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    cudaEventElapsedTime(&ms, ctx_->ev0, ctx_->ev1);
  }
  tt.lap(level == 0 ? "encode.level0" : level == 1 ? "encode.level1" : "encode.level2+");
  int e = NoError;
  e = enc_->collect_level(level, keep_device_);
  if (e)
    return e;
  tt.lap(level == 0 ? "encode.collect0" : level == 1 ? "encode.collect1" : "encode.collect2+");
  fields_[0].level_ms[(size_t)level] = ms + (float)(enc_->kernel_ms() - before);
  enc_->add_kernel_ms(ms);
  *out = std::move(outs_[(size_t)level]);
  return NoError;
}

#ifdef IDX2G_PHASE_TIMING
// Profiling builds: read and clear the per-phase cycle counters of the encode kernel.
extern "C" __attribute__((visibility("default"))) void idx2g_debug_phase_cycles(unsigned long long* out)
{
  cudaMemcpyFromSymbol(out, g_phase_cycles, sizeof(g_phase_cycles));
  unsigned long long z[16] = {};
  cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z));
}
#endif

void gpu_coder::value_range(double* vmin, double* vmax)
{
  *vmin = fields_[0].vmin;
  *vmax = fields_[0].vmax;
}

} // namespace idx2g
