// Differentiable decode: the real-valued decode operator D and its adjoint D^T on sm_100a.
//
// D maps the dequantised zfp-domain coefficients of every brick to the decoded grid, the
// reference decode (Core/idx2Decode.cpp:141-320) with the integer inverse zfp replaced by its
// real counterpart (Core/Zfp.h:181 ILift with exact halvings in place of the arithmetic shifts;
// the bit-exact decode differs from D only by those floors, about 2^(EMax-59) per block):
//   per level, coarsest first, per brick: the parent's values on the low band
//   (Core/idx2Decode.cpp:285-293), the inverse zfp of every coded block written over them (in
//   3D the full low-band blocks are not coded below the coarsest level and the rest lie outside
//   the parent's 16^3 part; in 2D every low-band block is coded on every level,
//   Core/idx2Decode.cpp:126-130, so the parent's values are all overwritten), de-normalisation
//   and the one-level inverse CDF5/3 Z, Y, X (Core/Wavelet.cpp:144-203), then the brick goes to
//   its children or, on the finest level, to the grid.
// D is linear; D^T applies the transposed steps in the reverse order, finest level first, the
// low-band gradient of every child flowing into its parent's gradient brick (children cover
// disjoint 16^3 parts of the parent).
//
// Coefficient tensor of one field: levels 0 (finest) .. L-1; on each level the bricks in
// row-major order of their coordinates (x fastest); each brick 33^3 values (33^2 for 2D)
// indexed (z * 33 + y) * 33 + x, the coefficient of a block at the position of the sample it
// transforms (natural order inside the block). Positions of blocks that are not coded on a
// level (3D: the full low-band blocks below the coarsest level) are unused; their gradient is 0.
// The bit-exact decode leaves a block that had no bit plane above the tolerance unwritten; D
// writes every coded block, so in 2D, where such a block would keep the parent's values, D
// and the decode agree only where every low-band block below the coarsest level is decoded.
#include "codec_device.cuh"
#include "device.h"
#include "encoder.h"
#include "format.h"

#include <cstring>
#include <vector>

namespace idx2g
{

namespace
{

constexpr int kSynThreads = 256;
constexpr int kSynWarps = kSynThreads / 32;

struct syn_brick
{
  int b3[3];
  int valid[3];   // samples of the grid in the brick (finest level)
  int parent;     // index of the parent brick on the coarser level (all fields), -1 if none
  int pos[3];     // position inside the parent (0/1 per axis)
  int field;
  long long coff; // offset of the brick in its field's coefficient tensor (elements)
};

template <typename T>
struct syn_args
{
  int nbricks, is2d, nsb, coarsest, finest, norm_mask;
  int nblocks[8];
  double inv_weight[8];
  const uint64_t* geom;  // [8][kMaxBlocksPerSubband]
  const syn_brick* bricks;
  long long cstride;     // elements of one field's coefficient tensor
  long long gstride;     // elements of one field's grid
  long long gdims[3];
  // forward: in = coefficients, out = grid (finest level) or kept bricks, parents = kept bricks
  // of the coarser level. adjoint: in = gradient of the grid (finest level) or this level's
  // gradient bricks, out = gradient of the coefficients, pgrad = the coarser level's gradient
  // bricks (or null).
  const T* in;
  T* out;
  const T* parents;
  T* pgrad;
  T* bricks_out;         // forward: kept bricks of this level (non-finest)
  T* slots;
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

__device__ __forceinline__ void subband_parity(int s, int is2d, int& hx, int& hy, int& hz)
{
  if (is2d)
  {
    hx = (s >> 1) & 1;
    hy = s & 1;
    hz = 0;
  }
  else
  {
    hx = (s >> 2) & 1;
    hy = (s >> 1) & 1;
    hz = s & 1;
  }
}

// Brick position of sample j of a block (block dims 4 or 1 per axis).
__device__ __forceinline__ int block_pos(int j, const int d3[3], const int bd[3], int hx, int hy, int hz)
{
  const int x = bd[0] > 1 ? (j & 3) : 0;
  const int r = bd[0] > 1 ? j >> 2 : j;
  const int y = bd[1] > 1 ? (r & 3) : 0;
  const int z = bd[1] > 1 ? r >> 2 : r;
  return ((hz + 2 * (d3[2] + z)) * 33 + (hy + 2 * (d3[1] + y))) * 33 + (hx + 2 * (d3[0] + x));
}

// Real inverse zfp lifting of one 4-point line (Core/Zfp.h:181 ILift, halvings exact).
template <typename T>
__device__ __forceinline__ void rilift4(T* q, int i, int s)
{
  T x = q[i], y = q[i + s], z = q[i + 2 * s], w = q[i + 3 * s];
  y += w * T(0.5);
  w -= y * T(0.5);
  y += w;
  w *= T(2);
  w -= y;
  z += x;
  x *= T(2);
  x -= z;
  y += z;
  z *= T(2);
  z -= y;
  w += x;
  x *= T(2);
  x -= w;
  q[i] = x;
  q[i + s] = y;
  q[i + 2 * s] = z;
  q[i + 3 * s] = w;
}

// Its transpose: the elementary steps of rilift4 transposed, in reverse order.
template <typename T>
__device__ __forceinline__ void rilift4_adj(T* q, int i, int s)
{
  T x = q[i], y = q[i + s], z = q[i + 2 * s], w = q[i + 3 * s];
  w -= x;
  x *= T(2);
  x += w;
  y -= z;
  z *= T(2);
  z += y;
  z -= x;
  x *= T(2);
  x += z;
  y -= w;
  w *= T(2);
  w += y;
  y -= w * T(0.5);
  w += y * T(0.5);
  q[i] = x;
  q[i + s] = y;
  q[i + 2 * s] = z;
  q[i + 3 * s] = w;
}

// Inverse zfp of a block held by a warp in shared memory (z, y, x lines) and its transpose.
template <typename T>
__device__ __forceinline__ void warp_rinv_zfp(T* q, int nd, int lane)
{
  if (nd == 3)
  {
    if (lane < 16)
      rilift4(q, (lane & 3) + 4 * (lane >> 2), 16);
    __syncwarp();
    if (lane < 16)
      rilift4(q, 16 * (lane & 3) + (lane >> 2), 4);
    __syncwarp();
    if (lane < 16)
      rilift4(q, 4 * (lane & 3) + 16 * (lane >> 2), 1);
  }
  else if (nd == 2)
  {
    if (lane < 4)
      rilift4(q, lane, 4);
    __syncwarp();
    if (lane < 4)
      rilift4(q, 4 * lane, 1);
  }
  else if (nd == 1)
  {
    if (lane == 0)
      rilift4(q, 0, 1);
  }
  __syncwarp();
}

template <typename T>
__device__ __forceinline__ void warp_rinv_zfp_adj(T* q, int nd, int lane)
{
  if (nd == 3)
  {
    if (lane < 16)
      rilift4_adj(q, 4 * (lane & 3) + 16 * (lane >> 2), 1);
    __syncwarp();
    if (lane < 16)
      rilift4_adj(q, 16 * (lane & 3) + (lane >> 2), 4);
    __syncwarp();
    if (lane < 16)
      rilift4_adj(q, (lane & 3) + 4 * (lane >> 2), 16);
  }
  else if (nd == 2)
  {
    if (lane < 4)
      rilift4_adj(q, 4 * lane, 1);
    __syncwarp();
    if (lane < 4)
      rilift4_adj(q, lane, 4);
  }
  else if (nd == 1)
  {
    if (lane == 0)
      rilift4_adj(q, 0, 1);
  }
  __syncwarp();
}

// One-level inverse CDF5/3 of a 33-sample line (Core/Wavelet.h:250 ILiftCdf53, D = 33) and
// its transpose.
template <typename T>
__device__ __forceinline__ void rilift33(T (&v)[33])
{
#pragma unroll
  for (int x = 1; x < 31; x += 2)
  {
    const T V = v[x] * T(0.25);
    v[x - 1] -= V;
    v[x + 1] -= V;
  }
  {
    const T V = v[31] * T(0.25);
    v[30] -= V;
    v[32] -= V;
  }
#pragma unroll
  for (int x = 1; x < 31; x += 2)
    v[x] += (v[x - 1] + v[x + 1]) * T(0.5);
  v[31] += (v[32] + v[30]) * T(0.5);
}

template <typename T>
__device__ __forceinline__ void rilift33_adj(T (&g)[33])
{
  g[32] += g[31] * T(0.5);
  g[30] += g[31] * T(0.5);
#pragma unroll
  for (int x = 1; x < 31; x += 2)
  {
    g[x - 1] += g[x] * T(0.5);
    g[x + 1] += g[x] * T(0.5);
  }
  g[31] -= (g[30] + g[32]) * T(0.25);
#pragma unroll
  for (int x = 1; x < 31; x += 2)
    g[x] -= (g[x - 1] + g[x + 1]) * T(0.25);
}

template <typename T>
__device__ __forceinline__ T denorm(const syn_args<T>& a, int s, T v)
{
  return ((a.norm_mask >> s) & 1) ? v * (T)a.inv_weight[s] : v;
}

template <typename T>
__global__ void __launch_bounds__(kSynThreads, 2) k_synth(const syn_args<T> a)
{
  __shared__ T q[kSynWarps][64];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NZ = a.is2d ? 1 : 33;
  const int NB = 33 * 33 * NZ;
  T* F = a.slots + (size_t)blockIdx.x * (size_t)NB;
  for (int bi = blockIdx.x; bi < a.nbricks; bi += gridDim.x)
  {
    const syn_brick& br = a.bricks[bi];
    const T* C = a.in + (size_t)br.field * (size_t)a.cstride + (size_t)br.coff;
    for (int i = tid; i < NB; i += kSynThreads)
      F[i] = T(0);
    __syncthreads();
    // the parent's values on the low band first (Core/idx2Decode.cpp:285-293); coded blocks
    // overwrite them (in 2D every low-band block is coded on every level)
    if (!a.coarsest && br.parent >= 0)
    {
      const T* P = a.parents + (size_t)br.parent * (size_t)NB;
      const int nz = a.is2d ? 1 : 16;
      for (int i = tid; i < 16 * 16 * nz; i += kSynThreads)
      {
        const int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        F[(2 * z * 33 + 2 * y) * 33 + 2 * x] =
          P[((br.pos[2] * nz + z) * 33 + (br.pos[1] * 16 + y)) * 33 + (br.pos[0] * 16 + x)];
      }
    }
    __syncthreads();
    // coded blocks: inverse zfp of their coefficients
    for (int s = 0; s < a.nsb; ++s)
    {
      int hx, hy, hz;
      subband_parity(s, a.is2d, hx, hy, hz);
      const uint64_t* geom = a.geom + (size_t)s * kMaxBlocksPerSubband;
      for (int b = warp; b < a.nblocks[s]; b += kSynWarps)
      {
        int d3[3], bd[3];
        unpack_geom(geom[b], d3, bd);
        const int nd = (bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1);
        const int nv = 1 << (2 * nd);
        for (int j = lane; j < nv; j += 32)
          q[warp][j] = C[block_pos(j, d3, bd, hx, hy, hz)];
        __syncwarp();
        warp_rinv_zfp(q[warp], nd, lane);
        for (int j = lane; j < nv; j += 32)
          F[block_pos(j, d3, bd, hx, hy, hz)] = q[warp][j];
        __syncwarp();
      }
    }
    __syncthreads();
    // de-normalisation and inverse CDF5/3: Z, Y, X
    if (!a.is2d)
    {
      for (int li = tid; li < 33 * 33; li += kSynThreads)
      {
        const int x = li % 33, y = li / 33;
        T v[33];
#pragma unroll
        for (int z = 0; z < 33; ++z)
          v[z] = denorm(a, ((x & 1) << 2) | ((y & 1) << 1) | (z & 1), F[(z * 33 + y) * 33 + x]);
        rilift33(v);
#pragma unroll
        for (int z = 0; z < 33; ++z)
          F[(z * 33 + y) * 33 + x] = v[z];
      }
      __syncthreads();
    }
    for (int li = tid; li < 33 * NZ; li += kSynThreads)
    {
      const int x = li % 33, z = li / 33;
      T v[33];
#pragma unroll
      for (int y = 0; y < 33; ++y)
      {
        const T f = F[(z * 33 + y) * 33 + x];
        v[y] = a.is2d ? denorm(a, ((x & 1) << 1) | (y & 1), f) : f;
      }
      rilift33(v);
#pragma unroll
      for (int y = 0; y < 33; ++y)
        F[(z * 33 + y) * 33 + x] = v[y];
    }
    __syncthreads();
    for (int li = tid; li < 33 * NZ; li += kSynThreads)
    {
      const int y = li % 33, z = li / 33;
      T v[33];
      T* row = F + (z * 33 + y) * 33;
#pragma unroll
      for (int x = 0; x < 33; ++x)
        v[x] = row[x];
      rilift33(v);
      if (a.finest)
      {
        if (y < br.valid[1] && z < br.valid[2])
        {
          T* g = a.out + (size_t)br.field * (size_t)a.gstride +
                 (size_t)(((long long)br.b3[2] * (a.is2d ? 1 : 32) + z) * a.gdims[1] + (long long)br.b3[1] * 32 + y) *
                   (size_t)a.gdims[0] +
                 (size_t)br.b3[0] * 32;
#pragma unroll
          for (int x = 0; x < 32; ++x)
            if (x < br.valid[0])
              g[x] = v[x];
        }
      }
      else
      {
        T* dst = a.bricks_out + (size_t)bi * (size_t)NB + (size_t)(z * 33 + y) * 33;
#pragma unroll
        for (int x = 0; x < 33; ++x)
          dst[x] = v[x];
      }
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(kSynThreads, 2) k_synth_adj(const syn_args<T> a)
{
  __shared__ T q[kSynWarps][64];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NZ = a.is2d ? 1 : 33;
  const int NB = 33 * 33 * NZ;
  for (int bi = blockIdx.x; bi < a.nbricks; bi += gridDim.x)
  {
    const syn_brick& br = a.bricks[bi];
    T* G = a.finest ? a.slots + (size_t)blockIdx.x * (size_t)NB : const_cast<T*>(a.in) + (size_t)bi * (size_t)NB;
    if (a.finest)
    {
      // the grid's gradient on the brick (0 outside the grid and on the extension samples)
      const T* g0 = a.in + (size_t)br.field * (size_t)a.gstride;
      for (int i = tid; i < NB; i += kSynThreads)
      {
        const int x = i % 33, y = (i / 33) % 33, z = i / (33 * 33);
        T v = T(0);
        if (x < br.valid[0] && y < br.valid[1] && z < br.valid[2])
          v = g0[(size_t)(((long long)br.b3[2] * (a.is2d ? 1 : 32) + z) * a.gdims[1] + (long long)br.b3[1] * 32 + y) *
                   (size_t)a.gdims[0] +
                 (size_t)br.b3[0] * 32 + x];
        G[i] = v;
      }
      __syncthreads();
    }
    // transposed inverse CDF5/3: X, Y, Z, then the de-normalisation
    for (int li = tid; li < 33 * NZ; li += kSynThreads)
    {
      const int y = li % 33, z = li / 33;
      T v[33];
      T* row = G + (z * 33 + y) * 33;
#pragma unroll
      for (int x = 0; x < 33; ++x)
        v[x] = row[x];
      rilift33_adj(v);
#pragma unroll
      for (int x = 0; x < 33; ++x)
        row[x] = v[x];
    }
    __syncthreads();
    for (int li = tid; li < 33 * NZ; li += kSynThreads)
    {
      const int x = li % 33, z = li / 33;
      T v[33];
#pragma unroll
      for (int y = 0; y < 33; ++y)
        v[y] = G[(z * 33 + y) * 33 + x];
      rilift33_adj(v);
#pragma unroll
      for (int y = 0; y < 33; ++y)
        G[(z * 33 + y) * 33 + x] = a.is2d ? denorm(a, ((x & 1) << 1) | (y & 1), v[y]) : v[y];
    }
    __syncthreads();
    if (!a.is2d)
    {
      for (int li = tid; li < 33 * 33; li += kSynThreads)
      {
        const int x = li % 33, y = li / 33;
        T v[33];
#pragma unroll
        for (int z = 0; z < 33; ++z)
          v[z] = G[(z * 33 + y) * 33 + x];
        rilift33_adj(v);
#pragma unroll
        for (int z = 0; z < 33; ++z)
          G[(z * 33 + y) * 33 + x] = denorm(a, ((x & 1) << 2) | ((y & 1) << 1) | (z & 1), v[z]);
      }
      __syncthreads();
    }
    // the coded blocks' coefficients first (0 where nothing is coded), then what is left of
    // the low band to the parent
    T* Gc = a.out + (size_t)br.field * (size_t)a.cstride + (size_t)br.coff;
    for (int i = tid; i < NB; i += kSynThreads)
      Gc[i] = T(0);
    __syncthreads();
    for (int s = 0; s < a.nsb; ++s)
    {
      int hx, hy, hz;
      subband_parity(s, a.is2d, hx, hy, hz);
      const uint64_t* geom = a.geom + (size_t)s * kMaxBlocksPerSubband;
      for (int b = warp; b < a.nblocks[s]; b += kSynWarps)
      {
        int d3[3], bd[3];
        unpack_geom(geom[b], d3, bd);
        const int nd = (bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1);
        const int nv = 1 << (2 * nd);
        for (int j = lane; j < nv; j += 32)
        {
          const int p = block_pos(j, d3, bd, hx, hy, hz);
          q[warp][j] = G[p];
          G[p] = T(0);  // overwritten in the forward pass: nothing reaches the parent
        }
        __syncwarp();
        warp_rinv_zfp_adj(q[warp], nd, lane);
        for (int j = lane; j < nv; j += 32)
          Gc[block_pos(j, d3, bd, hx, hy, hz)] = q[warp][j];
        __syncwarp();
      }
    }
    __syncthreads();
    // the low band's gradient to the parent
    if (!a.coarsest && br.parent >= 0 && a.pgrad)
    {
      T* P = a.pgrad + (size_t)br.parent * (size_t)NB;
      const int nz = a.is2d ? 1 : 16;
      for (int i = tid; i < 16 * 16 * nz; i += kSynThreads)
      {
        const int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        P[((br.pos[2] * nz + z) * 33 + (br.pos[1] * 16 + y)) * 33 + (br.pos[0] * 16 + x)] =
          G[(2 * z * 33 + 2 * y) * 33 + 2 * x];
      }
    }
    __syncthreads();
  }
}

// Bricks, geometry and weights of every level of a format (levels finest first).
struct syn_level
{
  std::vector<syn_brick> bricks;  // one field
  std::vector<uint64_t> geom;     // [8][kMaxBlocksPerSubband]
  int nblocks[8] = {};
  double inv_weight[8] = {};
  int norm_mask = 0;
};

long long build_levels(const dataset_format& f, std::vector<syn_level>* out)
{
  const int L = f.nlevels;
  const int NB = f.is2d() ? 33 * 33 : 33 * 33 * 33;
  out->assign((size_t)L, syn_level());
  long long base = 0;
  for (int l = 0; l < L; ++l)
  {
    syn_level& sl = (*out)[(size_t)l];
    const v3 n3 = f.nbricks3[(size_t)l];
    const v3 np3 = l + 1 < L ? f.nbricks3[(size_t)l + 1] : v3(1);
    for (int bz = 0; bz < n3.z; ++bz)
      for (int by = 0; by < n3.y; ++by)
        for (int bx = 0; bx < n3.x; ++bx)
        {
          syn_brick b;
          memset(&b, 0, sizeof b);
          b.b3[0] = bx;
          b.b3[1] = by;
          b.b3[2] = bz;
          const v3 b3(bx, by, bz);
          const v3 v = vmin(f.brick_dims, f.dims - b3 * f.brick_dims);
          b.valid[0] = v.x;
          b.valid[1] = v.y;
          b.valid[2] = v.z;
          if (l + 1 < L)
          {
            const v3 p3 = b3 / f.group_brick3, pos = b3 % f.group_brick3;
            b.parent = (p3.z * np3.y + p3.y) * np3.x + p3.x;
            b.pos[0] = pos.x;
            b.pos[1] = pos.y;
            b.pos[2] = pos.z;
          }
          else
            b.parent = -1;
          b.coff = base;
          base += NB;
          sl.bricks.push_back(b);
        }
    sl.geom.assign((size_t)8 * kMaxBlocksPerSubband, 0);
    for (int s = 0; s < f.nsubbands(); ++s)
    {
      std::vector<block_geom> g;
      subband_blocks(f, l, s, &g);
      sl.nblocks[s] = (int)g.size();
      for (size_t k = 0; k < g.size(); ++k)
        sl.geom[(size_t)s * kMaxBlocksPerSubband + k] =
          (uint64_t)g[k].dx | ((uint64_t)g[k].dy << 8) | ((uint64_t)g[k].dz << 16) | ((uint64_t)g[k].bx << 24) |
          ((uint64_t)g[k].by << 32) | ((uint64_t)g[k].bz << 40);
    }
    double w[8];
    level_weights(f, l, w, &sl.norm_mask);
    for (int s = 0; s < 8; ++s)
      sl.inv_weight[s] = s < f.nsubbands() ? 1.0 / w[s] : 1.0;
  }
  return base;
}

template <typename T>
int run_synth(device_ctx* ctx, const dataset_format& f, int nbatch, const void* in, void* out, bool adjoint,
              double* kernel_ms)
{
  std::vector<syn_level> lv;
  const long long count = build_levels(f, &lv);
  const int L = f.nlevels;
  const int NB = f.is2d() ? 33 * 33 : 33 * 33 * 33;
  cudaStream_t st = ctx->stream;
  const long long gcount = (long long)f.dims.x * f.dims.y * f.dims.z;
  float total = 0;
  int grid_max = 1;
  for (int l = 0; l < L; ++l)
  {
    const int nbr = (int)lv[(size_t)l].bricks.size() * nbatch;
    const int g = nbr < 2 * ctx->num_sms ? nbr : 2 * ctx->num_sms;
    grid_max = g > grid_max ? g : grid_max;
  }
  T* slots = (T*)ctx->ws("syn.slots", (size_t)grid_max * (size_t)NB * sizeof(T));
  uint64_t* d_geom = (uint64_t*)ctx->ws("syn.geom", (size_t)8 * kMaxBlocksPerSubband * 8);
  if (!slots || !d_geom)
    return OutOfMemory;
  T* prev = nullptr;  // forward: kept bricks of the coarser level; adjoint: this level's gradient bricks
  for (int step = 0; step < L; ++step)
  {
    const int l = adjoint ? step : L - 1 - step;
    const syn_level& sl = lv[(size_t)l];
    const int per = (int)sl.bricks.size();
    const int nbr = per * nbatch;
    std::vector<syn_brick> hb((size_t)nbr);
    for (int fi = 0; fi < nbatch; ++fi)
      for (int i = 0; i < per; ++i)
      {
        syn_brick b = sl.bricks[(size_t)i];
        b.field = fi;
        if (b.parent >= 0)
          b.parent += fi * (int)lv[(size_t)l + 1].bricks.size();
        hb[(size_t)fi * (size_t)per + (size_t)i] = b;
      }
    char nm[32];
    snprintf(nm, sizeof nm, "syn.bricks%d", step & 1);
    syn_brick* d_bricks = (syn_brick*)ctx->ws(nm, sizeof(syn_brick) * (size_t)nbr);
    if (!d_bricks)
      return OutOfMemory;
    cudaMemcpyAsync(d_bricks, hb.data(), sizeof(syn_brick) * (size_t)nbr, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_geom, sl.geom.data(), sl.geom.size() * 8, cudaMemcpyHostToDevice, st);
    syn_args<T> a;
    memset(&a, 0, sizeof a);
    a.nbricks = nbr;
    a.is2d = f.is2d();
    a.nsb = f.nsubbands();
    a.coarsest = l + 1 == L;
    a.finest = l == 0;
    a.norm_mask = sl.norm_mask;
    memcpy(a.nblocks, sl.nblocks, sizeof a.nblocks);
    memcpy(a.inv_weight, sl.inv_weight, sizeof a.inv_weight);
    a.geom = d_geom;
    a.bricks = d_bricks;
    a.cstride = count;
    a.gstride = gcount;
    a.gdims[0] = f.dims.x;
    a.gdims[1] = f.dims.y;
    a.gdims[2] = f.dims.z;
    a.slots = slots;
    const int grid = nbr < 2 * ctx->num_sms ? nbr : 2 * ctx->num_sms;
    snprintf(nm, sizeof nm, "syn.lev%d", step & 1);
    if (!adjoint)
    {
      a.in = (const T*)in;
      a.parents = prev;
      if (l == 0)
        a.out = (T*)out;
      else
      {
        a.bricks_out = (T*)ctx->ws(nm, (size_t)nbr * (size_t)NB * sizeof(T));
        if (!a.bricks_out)
          return OutOfMemory;
      }
      cudaEventRecord(ctx->ev0, st);
      k_synth<T><<<grid, kSynThreads, 0, st>>>(a);
      cudaEventRecord(ctx->ev1, st);
      prev = a.bricks_out;
    }
    else
    {
      a.in = l == 0 ? (const T*)in : prev;
      a.out = (T*)out;
      if (l + 1 < L)
      {
        const size_t pn = (size_t)lv[(size_t)l + 1].bricks.size() * (size_t)nbatch * (size_t)NB;
        a.pgrad = (T*)ctx->ws(nm, pn * sizeof(T));
        if (!a.pgrad)
          return OutOfMemory;
        cudaMemsetAsync(a.pgrad, 0, pn * sizeof(T), st);
      }
      cudaEventRecord(ctx->ev0, st);
      k_synth_adj<T><<<grid, kSynThreads, 0, st>>>(a);
      cudaEventRecord(ctx->ev1, st);
      prev = a.pgrad;
    }
    ++ctx->launches;
    if (cudaGetLastError() != cudaSuccess)
      return CudaError;
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    total += ms;
  }
  if (kernel_ms)
    *kernel_ms = total;
  return NoError;
}

} // namespace

long long synth_coeff_count(const dataset_format& f)
{
  std::vector<syn_level> lv;
  return build_levels(f, &lv);
}

int synth(device_ctx* ctx, const dataset_format& f, int nbatch, const void* d_in, void* d_out, bool adjoint,
          double* kernel_ms)
{
  if (f.brick_dims.x != 32 || f.brick_dims.y != 32 || (f.brick_dims.z != 32 && f.brick_dims.z != 1))
    return OptionNotSupported;
  cudaSetDevice(ctx->device);
  return f.type == dtype::float32 ? run_synth<float>(ctx, f, nbatch, d_in, d_out, adjoint, kernel_ms)
                                  : run_synth<double>(ctx, f, nbatch, d_in, d_out, adjoint, kernel_ms);
}

} // namespace idx2g
