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
#include "encoder.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace idx2g
{

namespace
{

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxPlanes = 64;
constexpr unsigned kStageBytes = 8192;

struct enc_brick
{
  int b3[3];      // brick coordinates (level 0: field origin = b3 * 32)
  int valid[3];   // valid dims
  int parent;     // parent index in the next level, -1 if none
  int pos[3];     // position inside the parent (0/1 per axis)
};

struct enc_args
{
  int level, nlevels, is2d, f32_exp, etol, end_bp, nsb, nbricks;
  uint64_t order;
  const void* field;
  int field_f32;
  long long fdims[3];
  const enc_brick* bricks;
  const double* in_bricks;   // level > 0: [nbricks][NB] assembled parents
  double* slots;             // [gridDim][NB]
  double* parent_bricks;     // [nparents][NB] (zeroed), null on the coarsest level
  const uint64_t* geom;      // [nsb][kMaxBlocksPerSubband]
  const int* nblocks;        // [nsb]
  double weight[8];
  int norm_mask;
  unsigned long long* offset;
  uint32_t* stream;
  unsigned long long cap_bytes;
  unsigned long long* cursor;
  int* error;
  double* bmin;
  double* bmax;
};

// shared memory layout (dynamic)
struct enc_smem
{
  unsigned long long X[kMaxBlocksPerSubband][kMaxPlanes];  // plane bit masks
  uint16_t off[kMaxBlocksPerSubband][kMaxPlanes];          // bit offset inside the channel
  uint8_t nin[kMaxBlocksPerSubband][kMaxPlanes];           // significant coefficients before plane
  long long q[kWarps][64];                                 // per-warp block scratch
  int16_t emax[kMaxBlocksPerSubband];
  int16_t ktop[kMaxBlocksPerSubband];
  uint8_t np[kMaxBlocksPerSubband];
  uint8_t nvals_log[kMaxBlocksPerSubband];
  uint32_t key_bits[kKeyWindow];
  uint32_t key_base[kKeyWindow];
  uint32_t stage[kStageBytes / 4];  // one (brick, subband) region being assembled
  unsigned alloc, hdr;
  dev::lift_stack stack;
  double red[2][kWarps];
  int kmin, kmax;
  unsigned long long region;
  int ok;
};

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

__global__ void __launch_bounds__(kThreads, 2) k_encode_level(const enc_args a)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  enc_smem& sm = *reinterpret_cast<enc_smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N[3] = { 33, 33, a.is2d ? 1 : 33 };
  const int NB = N[0] * N[1] * N[2];
  double* F = a.slots + (size_t)blockIdx.x * (size_t)NB;

  for (int bi = blockIdx.x; bi < a.nbricks; bi += gridDim.x)
  {
    const enc_brick br = a.bricks[bi];
    // ---------------- A: gather ----------------
    if (a.level == 0)
    {
      for (int i = tid; i < NB; i += kThreads)
        F[i] = 0.0;
      __syncthreads();
      double mn = 1.7976931348623157e308, mx = -1.7976931348623157e308;
      const int vx = br.valid[0], vy = br.valid[1], vz = br.valid[2];
      const int nvalid = vx * vy * vz;
      for (int i = tid; i < nvalid; i += kThreads)
      {
        int x = i % vx, y = (i / vx) % vy, z = i / (vx * vy);
        long long gx = (long long)br.b3[0] * 32 + x, gy = (long long)br.b3[1] * 32 + y,
                  gz = (long long)br.b3[2] * (a.is2d ? 1 : 32) + z;
        long long src = (gz * a.fdims[1] + gy) * a.fdims[0] + gx;
        double v = a.field_f32 ? (double)((const float*)a.field)[src] : ((const double*)a.field)[src];
        F[(z * 33 + y) * 33 + x] = v;
        mn = v < mn ? v : mn;
        mx = mx < v ? v : mx;
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
      const double* src = a.in_bricks + (size_t)bi * (size_t)NB;
      for (int i = tid; i < NB; i += kThreads)
        F[i] = src[i];
    }
    __syncthreads();

    // ---------------- B: transform ----------------
    {
      // extrapolation round trip (Core/Wavelet.cpp:68): forward on the valid dims, then the
      // inverse on the 33^3 grid except its last sweep (X at full resolution), which is fused
      // with the first sweep of the real transform below
      if (tid == 0)
        dev::build_stack(br.valid, 5, a.order, &sm.stack);
      __syncthreads();
      const int nf = sm.stack.n;
      for (int i = 0; i < nf; ++i)
      {
        dev::lift_sweep_regs<true>(F, N, sm.stack.g[i], sm.stack.axis[i]);
        __syncthreads();
      }
      if (tid == 0)
        dev::build_stack(N, 5, a.order, &sm.stack);
      __syncthreads();
      const int ni = sm.stack.n;
      for (int i = ni - 1; i >= 1; --i)
      {
        dev::lift_sweep_regs<false>(F, N, sm.stack.g[i], sm.stack.axis[i]);
        __syncthreads();
      }
      // inverse X (D = 33) then forward X of the one-level transform (Core/Wavelet.cpp:81)
      for (int li = tid; li < 33 * N[2]; li += kThreads)
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
      // forward Y, and forward Z; subband normalisation applied as the last sweep stores
      // (Core/Wavelet.cpp:111-137)
      for (int li = tid; li < 33 * N[2]; li += kThreads)
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
          if (a.is2d)
          {
            const int s = ((x & 1) << 1) | (k & 1);
            f = ((a.norm_mask >> s) & 1) ? __dmul_rn(f, a.weight[s]) : f;
          }
          col[k * 33] = f;
        }
      }
      __syncthreads();
      if (!a.is2d)
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
            col[k * 33 * 33] = ((a.norm_mask >> s) & 1) ? __dmul_rn(v[k], a.weight[s]) : v[k];
          }
        }
        __syncthreads();
      }
    }

    // ---------------- C: low band to the parent ----------------
    if (a.parent_bricks && br.parent >= 0)
    {
      double* P = a.parent_bricks + (size_t)br.parent * (size_t)NB;
      const int nz = a.is2d ? 1 : 16;
      for (int i = tid; i < 16 * 16 * nz; i += kThreads)
      {
        int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        int cz = a.is2d ? 0 : 2 * z;
        P[((br.pos[2] * nz + z) * 33 + (br.pos[1] * 16 + y)) * 33 + (br.pos[0] * 16 + x)] =
          F[(cz * 33 + 2 * y) * 33 + 2 * x];
      }
    }

    // ---------------- D: block coding per subband ----------------
    for (int s = 0; s < a.nsb; ++s)
    {
      int from[3], dims[3], strd[3];
      subband_grid(a.is2d, s, from, dims, strd);
      const int nb = a.nblocks[s];
      const uint64_t* geom = a.geom + (size_t)s * kMaxBlocksPerSubband;
      const size_t bs = (size_t)bi * (size_t)a.nsb + (size_t)s;

      // D1: warp per block
      for (int b = warp; b < nb; b += kWarps)
      {
        int d3[3], bd[3];
        unpack_geom(geom[b], d3, bd);
        const int nd = (bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1);
        const int nv = 1 << (2 * nd);
        const int prec = 63 - nd;
        long long* q = sm.q[warp];
        double v0 = 0, v1 = 0;
        int j0 = lane, j1 = lane + 32;
        if (j0 < nv)
        {
          int x = j0 % bd[0], y = (j0 / bd[0]) % bd[1], z = j0 / (bd[0] * bd[1]);
          v0 = F[((from[2] + (d3[2] + z) * strd[2]) * 33 + (from[1] + (d3[1] + y) * strd[1])) * 33 +
                 (from[0] + (d3[0] + x) * strd[0])];
        }
        if (j1 < nv)
        {
          int x = j1 % bd[0], y = (j1 / bd[0]) % bd[1], z = j1 / (bd[0] * bd[1]);
          v1 = F[((from[2] + (d3[2] + z) * strd[2]) * 33 + (from[1] + (d3[1] + y) * strd[1])) * 33 +
                 (from[0] + (d3[0] + x) * strd[0])];
        }
        double m = fabs(v0);
        double m1 = fabs(v1);
        m = m < m1 ? m1 : m;
        m = warp_max(m);
        const int emax = a.f32_exp ? dev::exponent_f32(__double2float_rn(m)) : dev::exponent_f64(m);
        const double scale = dev::pow2(prec - 1 - emax);
        if (j0 < nv)
          q[j0] = dev::trunc_i64(__dmul_rn(scale, v0));
        if (j1 < nv)
          q[j1] = dev::trunc_i64(__dmul_rn(scale, v1));
        __syncwarp();
        dev::warp_fwd_zfp(q, nd, lane);
        unsigned long long u0 = 0, u1 = 0;
        if (j0 < nv)
          u0 = ((unsigned long long)q[dev::perm(nd, j0)] + dev::kNegaMask) ^ dev::kNegaMask;
        if (j1 < nv)
          u1 = ((unsigned long long)q[dev::perm(nd, j1)] + dev::kNegaMask) ^ dev::kNegaMask;
        __syncwarp();
        const int np = dev::coded_planes(emax, a.etol, a.end_bp);
        for (int k = 0; k < np; ++k)
        {
          const int bit = 63 - k;
          unsigned lo = __ballot_sync(0xffffffffu, (u0 >> bit) & 1ull);
          unsigned hi = __ballot_sync(0xffffffffu, (u1 >> bit) & 1ull);
          if (lane == 0)
            sm.X[b][k] = (unsigned long long)lo | ((unsigned long long)hi << 32);
        }
        if (lane == 0)
        {
          sm.emax[b] = (int16_t)emax;
          sm.ktop[b] = (int16_t)(emax + 63 + 1024);
          sm.np[b] = (uint8_t)np;
          sm.nvals_log[b] = (uint8_t)(2 * nd);
        }
      }
      __syncthreads();

      // D2: significance chain per block
      for (int b = tid; b < nb; b += kThreads)
      {
        int n = 0;
        const int np = sm.np[b];
        for (int k = 0; k < np; ++k)
        {
          sm.nin[b][k] = (uint8_t)n;
          n = dev::plane_nout(sm.X[b][k], n);
        }
      }
      if (tid == 0)
      {
        int kmin = 1 << 30, kmax = -(1 << 30);
        for (int b = 0; b < nb; ++b)
        {
          if (!sm.np[b])
            continue;
          int lo = sm.ktop[b] - sm.np[b] + 1, hi = sm.ktop[b];
          kmin = lo < kmin ? lo : kmin;
          kmax = hi > kmax ? hi : kmax;
        }
        if (kmax < kmin)
        {
          kmin = 1;
          kmax = 0;
        }
        sm.kmin = kmin;
        sm.kmax = kmax;
        sm.ok = (kmax - kmin + 1) <= kKeyWindow;
        if (!sm.ok)
          atomicExch(a.error, 1);
      }
      __syncthreads();
      const int kmin = sm.kmin, kmax = sm.kmax;
      const int nkeys = sm.ok ? kmax - kmin + 1 : 0;

      // D3: per channel key, bit offsets of the blocks in Morton order
      for (int t = tid; t < nkeys; t += kThreads)
      {
        const int key = kmin + t;
        unsigned acc = 0;
        for (int b = 0; b < nb; ++b)
        {
          const int kk = sm.ktop[b] - key;
          if (kk < 0 || kk >= sm.np[b])
            continue;
          sm.off[b][kk] = (uint16_t)acc;
          acc += (unsigned)dev::plane_bits(sm.X[b][kk], sm.nin[b][kk], 1 << sm.nvals_log[b]);
        }
        sm.key_bits[t] = acc;
      }
      __syncthreads();

      // D4: channel byte bases and the region of this (brick, subband)
      // (regions are whole 32-bit words so every CTA owns the words it writes)
      if (tid == 0)
      {
        unsigned base = 0;
        for (int t = 0; t < nkeys; ++t)
        {
          sm.key_base[t] = base;
          base += (sm.key_bits[t] + 7) / 8;
        }
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
      __syncthreads();
      const unsigned long long region = sm.region;
      const unsigned alloc = sm.alloc;
      const unsigned hdr = sm.hdr;
      const bool fits = region + alloc <= a.cap_bytes;

      // D5: scatter the plane bits, into shared memory when the region is small enough, else
      // straight into the (zeroed) global region; then the region is stored with plain writes
      if (fits && alloc)
      {
        const bool staged = alloc <= kStageBytes;
        uint32_t* words = staged ? sm.stage : a.stream + region / 4;
        for (unsigned i = tid; i < alloc / 4; i += kThreads)
          words[i] = 0u;
        __syncthreads();
        if (tid == 0)
        {
          words[0] = (uint32_t)(nkeys ? kmin : 1);
          words[1] = (uint32_t)nkeys;
        }
        uint16_t* ew = reinterpret_cast<uint16_t*>(words + 2);
        for (int b = tid; b < nb; b += kThreads)
          ew[b] = (uint16_t)sm.emax[b];
        uint32_t* sw = words + 2 + ((2u * (unsigned)nb + 3u) >> 2);
        for (int t = tid; t < nkeys; t += kThreads)
          sw[t] = (sm.key_bits[t] + 7) / 8;
        for (int idx = tid; idx < nb * kMaxPlanes; idx += kThreads)
        {
          const int b = idx >> 6, kk = idx & 63;
          if (kk >= sm.np[b])
            continue;
          const int t = sm.ktop[b] - kk - kmin;
          const unsigned long long pos =
            ((unsigned long long)hdr + sm.key_base[t]) * 8ull + (unsigned long long)sm.off[b][kk];
          dev::write_plane(words, pos, sm.X[b][kk], sm.nin[b][kk], 1 << sm.nvals_log[b]);
        }
        __syncthreads();
        if (staged)
        {
          uint32_t* dst = a.stream + region / 4;
          for (unsigned i = tid; i < alloc / 4; i += kThreads)
            dst[i] = sm.stage[i];
        }
      }
      __syncthreads();
    }
  }
}

// Host-side weights of one level (Core/Wavelet.cpp:111-137, Core/Wavelet.h:19).
void level_weights(const dataset_format& f, int level, double w[8], int* mask)
{
  double scal[16], wave[16];
  double n1 = 3, n2 = 23;
  for (int i = 0; i < 16; ++i)
  {
    scal[i] = sqrt(n1 / (1 << (i + 1)));
    n1 = n1 * 4 - 1;
    wave[i] = sqrt(n2 / (1 << (i + 5)));
    n2 = n2 * 4 - 33;
  }
  const bool coarsest = level + 1 == f.nlevels;
  *mask = 0;
  for (int s = 0; s < f.nsubbands(); ++s)
  {
    const subband& sb = f.subbands[(size_t)s];
    double wx = f.brick_dims_ext.x == 1 ? 1
                : (sb.low_high.x == 0 ? scal[level + sb.level_rev.x - 1] : wave[level + sb.level_rev.x]);
    double wy = f.brick_dims_ext.y == 1 ? 1
                : (sb.low_high.y == 0 ? scal[level + sb.level_rev.y - 1] : wave[level + sb.level_rev.y]);
    double wz = f.brick_dims_ext.z == 1 ? 1
                : (sb.low_high.z == 0 ? scal[level + sb.level_rev.z - 1] : wave[level + sb.level_rev.z]);
    w[s] = wx * wy * wz;
    if (s == 0 && !coarsest)
      continue;
    *mask |= 1 << s;
  }
}

} // namespace

// ---------------------------------------------------------------------------
// device stage
// ---------------------------------------------------------------------------

gpu_coder::gpu_coder(device_ctx* ctx, const dataset_format& f, const void* d_field, bool field_f32)
  : ctx_(ctx), f_(f), d_field_(d_field), field_f32_(field_f32)
{
}

gpu_coder::~gpu_coder() {}

int gpu_coder::run_level(int level, const encode_plan& plan, level_output* out)
{
  if (f_.bit_planes_per_chunk != 1)
    return OptionNotSupported;
  if (f_.brick_dims.x != 32 || f_.brick_dims.y != 32 || (f_.brick_dims.z != 32 && f_.brick_dims.z != 1))
    return OptionNotSupported;
  cudaStream_t st = ctx_->stream;
  const bool is2d = f_.is2d();
  const int NB = 33 * 33 * (is2d ? 1 : 33);
  const std::vector<brick_entry>& bricks = plan.levels[(size_t)level];
  const int nbr = (int)bricks.size();
  const int nsb = f_.nsubbands();
  const bool has_parent = level + 1 < f_.nlevels;
  const int npar = has_parent ? (int)plan.levels[(size_t)level + 1].size() : 0;

  std::vector<enc_brick> hb((size_t)nbr);
  for (int i = 0; i < nbr; ++i)
  {
    const brick_entry& e = bricks[(size_t)i];
    hb[(size_t)i] = enc_brick{ { e.brick3.x, e.brick3.y, e.brick3.z },
                               { e.valid.x, e.valid.y, e.valid.z },
                               e.parent,
                               { e.pos_in_parent.x, e.pos_in_parent.y, e.pos_in_parent.z } };
  }
  std::vector<uint64_t> geom((size_t)nsb * kMaxBlocksPerSubband, 0);
  std::vector<int> nblocks((size_t)nsb, 0);
  for (int s = 0; s < nsb; ++s)
  {
    std::vector<block_geom> g;
    subband_blocks(f_, level, s, &g);
    nblocks[(size_t)s] = (int)g.size();
    for (size_t b = 0; b < g.size(); ++b)
      geom[(size_t)s * kMaxBlocksPerSubband + b] =
        (uint64_t)g[b].dx | ((uint64_t)g[b].dy << 8) | ((uint64_t)g[b].dz << 16) |
        ((uint64_t)g[b].bx << 24) | ((uint64_t)g[b].by << 32) | ((uint64_t)g[b].bz << 40);
  }

  enc_args a;
  memset(&a, 0, sizeof a);
  a.level = level;
  a.nlevels = f_.nlevels;
  a.is2d = is2d;
  a.f32_exp = f_.type == dtype::float32;
  a.etol = exponent_f64(f_.tolerance);
  a.end_bp = f_.type == dtype::float32 ? 32 : 64;
  a.nsb = nsb;
  a.nbricks = nbr;
  a.order = f_.transform_order;
  a.field = d_field_;
  a.field_f32 = field_f32_;
  a.fdims[0] = f_.dims.x;
  a.fdims[1] = f_.dims.y;
  a.fdims[2] = f_.dims.z;
  level_weights(f_, level, a.weight, &a.norm_mask);

  // workspace buffers, kept by the context across calls (grow-only)
  int nsm = ctx_->num_sms;
  int grid = nbr < 2 * nsm ? nbr : 2 * nsm;
  if (grid < 1)
    grid = 1;
  const size_t nbs = (size_t)nbr * (size_t)nsb;
  auto* d_bricks = (enc_brick*)ctx_->ws("enc.bricks", sizeof(enc_brick) * (size_t)nbr);
  auto* d_geom = (uint64_t*)ctx_->ws("enc.geom", geom.size() * 8);
  auto* d_nblocks = (int*)ctx_->ws("enc.nblocks", (size_t)nsb * sizeof(int));
  double* d_slots = (double*)ctx_->ws("enc.slots", (size_t)grid * (size_t)NB * sizeof(double));
  double* d_parents = has_parent ? (double*)ctx_->ws(level % 2 ? "enc.parA" : "enc.parB",
                                                     (size_t)npar * (size_t)NB * sizeof(double))
                                 : nullptr;
  auto* d_off = (unsigned long long*)ctx_->ws(level % 2 ? "enc.offA" : "enc.offB", nbs * 8);
  auto* d_misc = (unsigned long long*)ctx_->ws("enc.misc", 64);
  double* d_bmin = (double*)ctx_->ws("enc.bmin", (size_t)nbr * 8);
  double* d_bmax = (double*)ctx_->ws("enc.bmax", (size_t)nbr * 8);
  if (!d_bricks || !d_geom || !d_nblocks || !d_slots || (has_parent && !d_parents) || !d_off || !d_misc ||
      !d_bmin || !d_bmax)
    return OutOfMemory;
  cudaMemcpyAsync(d_bricks, hb.data(), sizeof(enc_brick) * (size_t)nbr, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_geom, geom.data(), geom.size() * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_nblocks, nblocks.data(), (size_t)nsb * sizeof(int), cudaMemcpyHostToDevice, st);

  const char* sname = level % 2 ? "enc.streamA" : "enc.streamB";
  unsigned long long cap = (unsigned long long)nbr * (unsigned long long)NB * 2ull + (16ull << 20);
  if (ctx_->ws_size(sname) > cap)
    cap = ctx_->ws_size(sname);
  for (int attempt = 0; attempt < 4; ++attempt)
  {
    uint32_t* d_stream = (uint32_t*)ctx_->ws(sname, (size_t)cap);
    if (!d_stream)
      return OutOfMemory;
    cap = ctx_->ws_size(sname);
    cudaMemsetAsync(d_misc, 0, 64, st);
    if (has_parent)
      cudaMemsetAsync(d_parents, 0, (size_t)npar * (size_t)NB * sizeof(double), st);
    a.bricks = d_bricks;
    a.in_bricks = level > 0 ? in_bricks_ : nullptr;
    a.slots = d_slots;
    a.parent_bricks = d_parents;
    a.geom = d_geom;
    a.nblocks = d_nblocks;
    a.offset = d_off;
    a.stream = d_stream;
    a.cap_bytes = cap;
    a.cursor = d_misc;
    a.error = (int*)(d_misc + 1);
    a.bmin = d_bmin;
    a.bmax = d_bmax;
    const size_t smem = sizeof(enc_smem);
    cudaFuncSetAttribute(k_encode_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaEventRecord(ctx_->ev0, st);
    k_encode_level<<<grid, kThreads, smem, st>>>(a);
    cudaEventRecord(ctx_->ev1, st);
    if (cudaGetLastError() != cudaSuccess)
      return CudaError;
    ++launches_;
    unsigned long long misc[2];
    cudaMemcpyAsync(misc, d_misc, 16, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx_->ev0, ctx_->ev1);
    ctx_->ws_mark_dirty(sname, (size_t)(misc[0] < cap ? misc[0] : cap));
    int err = (int)(misc[1] & 0xffffffffu);
    if (err == 1)
      return DeviceStreamOverflow;  // more than kKeyWindow channels in one subband
    if (err == 2)
    {
      cap = misc[0] + (1ull << 20);
      continue;
    }
    kernel_ms_ += ms;
    level_ms_.push_back(ms);
    stream_bytes_ += (long long)misc[0];
    long long eb = 0;
    for (int s = 0; s < nsb; ++s)
      eb += (long long)nbr * nblocks[(size_t)s] * (f_.type == dtype::float32 ? 1 : 2);
    exp_bytes_ += eb;
    level_bytes_.push_back((long long)misc[0] + eb);
    out->nbricks = nbr;
    out->nsb = nsb;
    out->nexps = nblocks;
    if (level == 0)
    {
      std::vector<double> mn((size_t)nbr), mx((size_t)nbr);
      cudaMemcpyAsync(mn.data(), d_bmin, (size_t)nbr * 8, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(mx.data(), d_bmax, (size_t)nbr * 8, cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess)
        return CudaError;
      for (int i = 0; i < nbr; ++i)
      {
        vmin_ = mn[(size_t)i] < vmin_ ? mn[(size_t)i] : vmin_;
        vmax_ = vmax_ < mx[(size_t)i] ? mx[(size_t)i] : vmax_;
      }
    }
    if (!keep_device_)
    {
      // results to the host for the packer: region offsets and the regions
      out->offset.resize(nbs);
      cudaMemcpyAsync(out->offset.data(), d_off, nbs * 8, cudaMemcpyDeviceToHost, st);
      if (misc[0])
      {
        // into pinned host memory kept by the context (one buffer per level)
        char name[32];
        snprintf(name, sizeof name, "enc.pin%d", level);
        uint8_t* pin = (uint8_t*)ctx_->pinned(name, (size_t)misc[0]);
        if (!pin)
          return OutOfMemory;
        cudaMemcpyAsync(pin, d_stream, (size_t)misc[0], cudaMemcpyDeviceToHost, st);
        out->ext_stream = pin;
      }
      if (cudaStreamSynchronize(st) != cudaSuccess)
        return CudaError;
    }
    in_bricks_ = d_parents;
    return NoError;
  }
  return DeviceStreamOverflow;
}

void gpu_coder::value_range(double* vmin, double* vmax)
{
  *vmin = vmin_;
  *vmax = vmax_;
}

} // namespace idx2g
