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
//   Core/idx2Decode.cpp:126-130 against BlockDims3 = 4^3, so the parent's values are all
//   overwritten), de-normalisation and the one-level inverse CDF5/3 along each axis
//   (Core/Wavelet.cpp:144-203), then the brick goes to its children or, on the finest level,
//   to the grid.
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
//
// Kernels. A 3D brick is worked on by a cluster of kCS CTAs, CTA r holding planes
// z in [8r, 8r + 8) of it in shared memory (the last CTA also plane 32): every zfp block spans
// 8 planes along z (4 samples at stride 2), so each block lies inside one CTA. The inverse zfp
// runs in place as 4-point lines along z, y and x over every block (a block of extent 1 along
// an axis has no line there); the forward pass then writes the parent's values over the
// uncoded blocks, the adjoint clears them before its transposed zfp. The one-level CDF5/3 runs
// along y and x inside each CTA and along z over the cluster's distributed shared memory; that
// Z pass writes the grid (finest level) or the kept brick straight from registers, and in the
// adjoint reads the grid's gradient the same way. A 2D brick is one CTA: X pass inside, Y pass
// as the column pass. The order of the three CDF passes differs from the decode's Z, Y, X:
// they act on different axes and commute, the results differ by rounding only.
#include "codec_device.cuh"
#include "device.h"
#include "encoder.h"
#include "format.h"

#include <cooperative_groups.h>

#include <cstring>
#include <set>
#include <tuple>
#include <vector>

namespace cg = cooperative_groups;

namespace idx2g
{

namespace
{

constexpr int kSynThreads = 320;
constexpr int kPlane = 33 * 33;
constexpr int kCS = 4;   // CTAs per 3D brick (a thread-block cluster)
constexpr int kPPC = 8;  // planes per CTA; the last CTA of the cluster also holds plane 32

template <typename T>
constexpr int syn_ctas_per_sm()
{
  return sizeof(T) == 4 ? 3 : 2;
}

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
  int nbricks, coarsest, finest, norm_mask;
  double inv_weight[8];
  const syn_brick* bricks;
  long long cstride;     // elements of one field's coefficient tensor
  long long gstride;     // elements of one field's grid
  long long gdims[3];
  // forward: in = coefficients, out = grid (finest level), bricks_out = kept bricks (other
  // levels), parents = kept bricks of the coarser level. adjoint: in = gradient of the grid
  // (finest level) or this level's gradient bricks, out = gradient of the coefficients,
  // pgrad = the coarser level's gradient bricks (or null).
  const T* in;
  T* out;
  const T* parents;
  T* pgrad;
  T* bricks_out;
};

// Real inverse zfp lifting of one 4-point line (Core/Zfp.h:181 ILift, halvings exact).
template <typename T>
__device__ __forceinline__ void rilift4(T* q, int s)
{
  T x = q[0], y = q[s], z = q[2 * s], w = q[3 * s];
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
  q[0] = x;
  q[s] = y;
  q[2 * s] = z;
  q[3 * s] = w;
}

// Its transpose: the elementary steps of rilift4 transposed, in reverse order.
template <typename T>
__device__ __forceinline__ void rilift4_adj(T* q, int s)
{
  T x = q[0], y = q[s], z = q[2 * s], w = q[3 * s];
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
  q[0] = x;
  q[s] = y;
  q[2 * s] = z;
  q[3 * s] = w;
}

template <typename T, bool ADJ>
__device__ __forceinline__ void lift4(T* q, int s)
{
  if constexpr (ADJ)
    rilift4_adj(q, s);
  else
    rilift4(q, s);
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

template <typename T, bool ADJ>
__device__ __forceinline__ void lift33(T (&v)[33])
{
  if constexpr (ADJ)
    rilift33_adj(v);
  else
    rilift33(v);
}

// Subband of a sample from its parities (the subband order of the format: 3D hx hy hz, 2D hx hy).
template <bool IS2D>
__device__ __forceinline__ int parity_index(int x, int y, int z)
{
  if constexpr (IS2D)
    return ((x & 1) << 1) | (y & 1);
  else
    return ((x & 1) << 2) | ((y & 1) << 1) | (z & 1);
}

// De-normalisation factors per subband in shared memory (1 where the subband is not weighted:
// a multiplication by 1 is exact), staged once per CTA.
template <typename T>
__device__ __forceinline__ void stage_weights(const syn_args<T>& a, T* sw, int tid)
{
  if (tid < 8)
    sw[tid] = ((a.norm_mask >> tid) & 1) ? (T)a.inv_weight[tid] : T(1);
  __syncthreads();
}

template <int CS>
__device__ __forceinline__ void cluster_sync()
{
  if constexpr (CS > 1)
    cg::this_cluster().sync();
  else
    __syncthreads();
}

// n contiguous values from global memory into shared memory (asynchronous copies, then a
// barrier).
template <typename T>
__device__ __forceinline__ void load_planes(T* S, const T* src, int n, int tid)
{
  const unsigned s0 = (unsigned)__cvta_generic_to_shared(S);
  for (int i = tid; i < n; i += kSynThreads)
  {
    if constexpr (sizeof(T) == 4)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s0 + 4u * (unsigned)i), "l"(src + i)
                   : "memory");
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s0 + 8u * (unsigned)i), "l"(src + i)
                   : "memory");
  }
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
}

// Lines of the in-place inverse zfp (or its transpose) over the CTA's planes. Along z (3D):
// the CTA's 8 planes are one block row per parity, planes hz + 2j. Along y and x: per plane
// and parity h, blocks k = 0..3 at h + 8k + 2j; the fifth block of the 17-sample low half has
// extent 1 and no line.
template <typename T, bool ADJ>
__device__ __forceinline__ void zfp_z(T* S, int tid)
{
  for (int L = tid; L < 2 * kPlane; L += kSynThreads)
  {
    const int xy = L % kPlane, hz = L / kPlane;
    lift4<T, ADJ>(S + hz * kPlane + xy, 2 * kPlane);
  }
}

template <typename T, bool ADJ>
__device__ __forceinline__ void zfp_y(T* S, int np, int tid)
{
  const int n = 33 * np;
  for (int L = tid; L < 8 * n; L += kSynThreads)
  {
    const int xp = L % n, g = L / n;
    const int x = xp % 33, p = xp / 33;
    lift4<T, ADJ>(S + (p * 33 + (g & 1) + 8 * (g >> 1)) * 33 + x, 66);
  }
}

template <typename T, bool ADJ>
__device__ __forceinline__ void zfp_x(T* S, int np, int tid)
{
  const int n = 33 * np;
  for (int L = tid; L < 8 * n; L += kSynThreads)
  {
    const int row = L % n, g = L / n;
    lift4<T, ADJ>(S + row * 33 + (g & 1) + 8 * (g >> 1), 2);
  }
}

// CDF5/3 lines along y (per x and plane) and along x (per row) inside the CTA; DN applies the
// de-normalisation before the lift (forward) or after the transposed lift (adjoint).
template <typename T, bool IS2D, bool ADJ, bool DN>
__device__ __forceinline__ void cdf_y(const T* sw, T* S, int np, int z0, int tid)
{
  for (int L = tid; L < 33 * np; L += kSynThreads)
  {
    const int x = L % 33, p = L / 33, z = z0 + p;
    T* col = S + p * kPlane + x;
    T v[33];
#pragma unroll
    for (int y = 0; y < 33; ++y)
      v[y] = (DN && !ADJ) ? col[y * 33] * sw[parity_index<IS2D>(x, y, z)] : col[y * 33];
    lift33<T, ADJ>(v);
#pragma unroll
    for (int y = 0; y < 33; ++y)
      col[y * 33] = (DN && ADJ) ? v[y] * sw[parity_index<IS2D>(x, y, z)] : v[y];
  }
}

template <typename T, bool IS2D, bool ADJ, bool DN>
__device__ __forceinline__ void cdf_x(const T* sw, T* S, int np, int z0, int tid)
{
  for (int L = tid; L < 33 * np; L += kSynThreads)
  {
    const int y = L % 33, z = z0 + L / 33;
    T* row = S + L * 33;
    T v[33];
#pragma unroll
    for (int x = 0; x < 33; ++x)
      v[x] = (DN && !ADJ) ? row[x] * sw[parity_index<IS2D>(x, y, z)] : row[x];
    lift33<T, ADJ>(v);
#pragma unroll
    for (int x = 0; x < 33; ++x)
      row[x] = (DN && ADJ) ? v[x] * sw[parity_index<IS2D>(x, y, z)] : v[x];
  }
}

// The cluster CTA holding plane z of the brick.
__device__ __forceinline__ int plane_rank(int z)
{
  return z < kPPC * (kCS - 1) ? z / kPPC : kCS - 1;
}

// Offset of the brick's first sample in a batch of grids.
template <typename T>
__device__ __forceinline__ size_t grid_offset(const syn_args<T>& a, const syn_brick& br, bool is2d)
{
  return (size_t)br.field * (size_t)a.gstride +
         (size_t)(((long long)br.b3[2] * (is2d ? 1 : 32)) * a.gdims[1] + (long long)br.b3[1] * 32) *
           (size_t)a.gdims[0] +
         (size_t)br.b3[0] * 32;
}

template <typename T, bool IS2D>
__global__ void __launch_bounds__(kSynThreads, syn_ctas_per_sm<T>()) k_synth(const syn_args<T> a)
{
  extern __shared__ __align__(16) unsigned char syn_smem[];
  __shared__ T sw[8];
  T* S = reinterpret_cast<T*>(syn_smem);
  constexpr int CS = IS2D ? 1 : kCS;
  const int tid = threadIdx.x;
  stage_weights(a, sw, tid);
  int rank = 0;
  unsigned base[CS];  // the cluster's brick planes, as shared::cluster addresses
  if constexpr (CS > 1)
  {
    rank = (int)cg::this_cluster().block_rank();
#pragma unroll
    for (int r = 0; r < CS; ++r)
      base[r] = dev::cluster_addr(S, r);
    cluster_sync<CS>();  // every CTA of the cluster has started before any remote access
  }
  const int z0 = IS2D ? 0 : rank * kPPC;
  const int np = IS2D ? 1 : (rank == CS - 1 ? 33 - z0 : kPPC);
  const size_t NB = IS2D ? kPlane : 33 * kPlane;
  const int nclusters = gridDim.x / CS;
  for (int bi = blockIdx.x / CS; bi < a.nbricks; bi += nclusters)
  {
    const syn_brick& br = a.bricks[bi];
    load_planes(S, a.in + (size_t)br.field * (size_t)a.cstride + (size_t)br.coff + (size_t)z0 * kPlane,
                np * kPlane, tid);
    // inverse zfp of every block, in place: z, y, x
    if constexpr (!IS2D)
    {
      zfp_z<T, false>(S, tid);
      __syncthreads();
    }
    zfp_y<T, false>(S, np, tid);
    __syncthreads();
    zfp_x<T, false>(S, np, tid);
    __syncthreads();
    if constexpr (!IS2D)
    {
      // the parent's values over the uncoded full low-band blocks (even samples below 32 of
      // this CTA's planes)
      if (!a.coarsest)
      {
        const T* P = a.parents + (size_t)br.parent * NB;
        for (int i = tid; i < 4 * 256; i += kSynThreads)
        {
          const int x = i & 15, y = (i >> 4) & 15, k = i >> 8;
          const int zz = (z0 >> 1) + k;
          S[((2 * k) * 33 + 2 * y) * 33 + 2 * x] =
            P[((br.pos[2] * 16 + zz) * 33 + (br.pos[1] * 16 + y)) * 33 + (br.pos[0] * 16 + x)];
        }
        __syncthreads();
      }
      cdf_y<T, false, false, true>(sw, S, np, z0, tid);
      __syncthreads();
      cdf_x<T, false, false, false>(sw, S, np, z0, tid);
      cluster_sync<CS>();
      // Z pass over the cluster: this CTA's share of the 33 x 33 columns
      constexpr int cpc = (kPlane + CS - 1) / CS;
      for (int cl = tid; cl < cpc; cl += kSynThreads)
      {
        const int c = rank * cpc + cl;
        if (c >= kPlane)
          break;
        const int x = c % 33, y = c / 33;
        T v[33];
#pragma unroll
        for (int z = 0; z < 33; ++z)
          v[z] = dev::ld_cluster<T>(base[plane_rank(z)] + (unsigned)(((z - plane_rank(z) * kPPC) * kPlane + c) * sizeof(T)));
        rilift33(v);
        if (a.finest)
        {
          if (x < br.valid[0] && y < br.valid[1])
          {
            T* g = a.out + grid_offset(a, br, false) + (size_t)y * (size_t)a.gdims[0] + x;
            const size_t zs = (size_t)a.gdims[1] * (size_t)a.gdims[0];
#pragma unroll
            for (int z = 0; z < 32; ++z)
              if (z < br.valid[2])
                g[(size_t)z * zs] = v[z];
          }
        }
        else
        {
          T* o = a.bricks_out + (size_t)bi * NB + c;
#pragma unroll
          for (int z = 0; z < 33; ++z)
            o[z * kPlane] = v[z];
        }
      }
      cluster_sync<CS>();
    }
    else
    {
      cdf_x<T, true, false, true>(sw, S, 1, 0, tid);
      __syncthreads();
      // Y pass: one column per x
      if (tid < 33)
      {
        const int x = tid;
        T v[33];
#pragma unroll
        for (int y = 0; y < 33; ++y)
          v[y] = S[y * 33 + x];
        rilift33(v);
        if (a.finest)
        {
          if (x < br.valid[0])
          {
            T* g = a.out + grid_offset(a, br, true) + x;
#pragma unroll
            for (int y = 0; y < 32; ++y)
              if (y < br.valid[1])
                g[(size_t)y * (size_t)a.gdims[0]] = v[y];
          }
        }
        else
        {
          T* o = a.bricks_out + (size_t)bi * NB + x;
#pragma unroll
          for (int y = 0; y < 33; ++y)
            o[y * 33] = v[y];
        }
      }
      __syncthreads();
    }
  }
}

template <typename T, bool IS2D>
__global__ void __launch_bounds__(kSynThreads, syn_ctas_per_sm<T>()) k_synth_adj(const syn_args<T> a)
{
  extern __shared__ __align__(16) unsigned char syn_smem[];
  __shared__ T sw[8];
  T* S = reinterpret_cast<T*>(syn_smem);
  constexpr int CS = IS2D ? 1 : kCS;
  const int tid = threadIdx.x;
  stage_weights(a, sw, tid);
  int rank = 0;
  unsigned base[CS];  // the cluster's brick planes, as shared::cluster addresses
  if constexpr (CS > 1)
  {
    rank = (int)cg::this_cluster().block_rank();
#pragma unroll
    for (int r = 0; r < CS; ++r)
      base[r] = dev::cluster_addr(S, r);
    cluster_sync<CS>();  // every CTA of the cluster has started before any remote access
  }
  const int z0 = IS2D ? 0 : rank * kPPC;
  const int np = IS2D ? 1 : (rank == CS - 1 ? 33 - z0 : kPPC);
  const size_t NB = IS2D ? kPlane : 33 * kPlane;
  const int nclusters = gridDim.x / CS;
  for (int bi = blockIdx.x / CS; bi < a.nbricks; bi += nclusters)
  {
    const syn_brick& br = a.bricks[bi];
    if constexpr (!IS2D)
    {
      // transposed Z pass: this CTA's columns of the incoming gradient, into the cluster
      constexpr int cpc = (kPlane + CS - 1) / CS;
      for (int cl = tid; cl < cpc; cl += kSynThreads)
      {
        const int c = rank * cpc + cl;
        if (c >= kPlane)
          break;
        const int x = c % 33, y = c / 33;
        T v[33];
        if (a.finest)
        {
          const int nz = x < br.valid[0] && y < br.valid[1] ? br.valid[2] : 0;  // valid[2] <= 32
          const T* g = a.in + grid_offset(a, br, false) + (size_t)y * (size_t)a.gdims[0] + x;
          const size_t zs = (size_t)a.gdims[1] * (size_t)a.gdims[0];
#pragma unroll
          for (int z = 0; z < 33; ++z)
          {
            v[z] = z < nz ? *g : T(0);
            g += zs;
          }
        }
        else
        {
          const T* gi = a.in + (size_t)bi * NB + c;
#pragma unroll
          for (int z = 0; z < 33; ++z)
            v[z] = gi[z * kPlane];
        }
        rilift33_adj(v);
#pragma unroll
        for (int z = 0; z < 33; ++z)
          dev::st_cluster<T>(base[plane_rank(z)] + (unsigned)(((z - plane_rank(z) * kPPC) * kPlane + c) * sizeof(T)), v[z]);
      }
      cluster_sync<CS>();
      cdf_x<T, false, true, false>(sw, S, np, z0, tid);
      __syncthreads();
      cdf_y<T, false, true, true>(sw, S, np, z0, tid);
      __syncthreads();
      // the low band over the uncoded blocks goes to the parent (and nowhere else)
      if (!a.coarsest)
      {
        T* P = a.pgrad + (size_t)br.parent * NB;
        for (int i = tid; i < 4 * 256; i += kSynThreads)
        {
          const int x = i & 15, y = (i >> 4) & 15, k = i >> 8;
          const int zz = (z0 >> 1) + k;
          T* s = S + ((2 * k) * 33 + 2 * y) * 33 + 2 * x;
          P[((br.pos[2] * 16 + zz) * 33 + (br.pos[1] * 16 + y)) * 33 + (br.pos[0] * 16 + x)] = *s;
          *s = T(0);
        }
        __syncthreads();
      }
    }
    else
    {
      // transposed Y pass: one column per x of the incoming gradient
      if (tid < 33)
      {
        const int x = tid;
        T v[33];
        if (a.finest)
        {
          const T* g = a.in + grid_offset(a, br, true) + x;
#pragma unroll
          for (int y = 0; y < 33; ++y)
            v[y] = (x < br.valid[0] && y < 32 && y < br.valid[1]) ? g[(size_t)y * (size_t)a.gdims[0]] : T(0);
        }
        else
        {
          const T* gi = a.in + (size_t)bi * NB + x;
#pragma unroll
          for (int y = 0; y < 33; ++y)
            v[y] = gi[y * 33];
        }
        rilift33_adj(v);
#pragma unroll
        for (int y = 0; y < 33; ++y)
          S[y * 33 + x] = v[y];
      }
      __syncthreads();
      cdf_x<T, true, true, true>(sw, S, 1, 0, tid);
      __syncthreads();
    }
    // transposed zfp: x, y, z
    zfp_x<T, true>(S, np, tid);
    __syncthreads();
    zfp_y<T, true>(S, np, tid);
    __syncthreads();
    if constexpr (!IS2D)
    {
      zfp_z<T, true>(S, tid);
      __syncthreads();
    }
    T* Gc = a.out + (size_t)br.field * (size_t)a.cstride + (size_t)br.coff + (size_t)z0 * kPlane;
    for (int i = tid; i < np * kPlane; i += kSynThreads)
      Gc[i] = S[i];
    // the next brick's transposed Z pass writes into every CTA of the cluster
    cluster_sync<CS>();
  }
}

// Bricks and weights of every level of a format (levels finest first).
struct syn_level
{
  std::vector<syn_brick> bricks;  // one field
  double inv_weight[8] = {};
  int norm_mask = 0;
};

// The kernels assume the block layout of an extended brick: subband s at the parities of its
// index (3D hx hy hz, 2D hx hy), 17 samples on a low and 16 on a high axis, blocks of 4 (the
// fifth of a low axis of extent 1), every block coded except, below the coarsest level, the
// full 4^3 low-band blocks (Core/idx2Decode.cpp:126-130). Checked against the coder's own
// block walk of every level.
bool uniform_blocks(const dataset_format& f, int level)
{
  const bool is2d = f.is2d();
  for (int s = 0; s < f.nsubbands(); ++s)
  {
    const subband& sb = f.subbands[(size_t)s];
    const int h[3] = { is2d ? (s >> 1) & 1 : (s >> 2) & 1, is2d ? s & 1 : (s >> 1) & 1, is2d ? 0 : s & 1 };
    const v3 ha(h[0], h[1], h[2]);
    if (!(sb.low_high == ha) || !(sb.g.from == ha))
      return false;
    const v3 want(17 - h[0], 17 - h[1], is2d ? 1 : 17 - h[2]);
    if (!(sb.g.dims == want))
      return false;
    std::set<std::tuple<int, int, int, int, int, int>> expect, got;
    const int nk[3] = { h[0] ? 4 : 5, h[1] ? 4 : 5, is2d ? 1 : (h[2] ? 4 : 5) };
    for (int kz = 0; kz < nk[2]; ++kz)
      for (int ky = 0; ky < nk[1]; ++ky)
        for (int kx = 0; kx < nk[0]; ++kx)
        {
          const int bx = kx < 4 ? 4 : 1, by = ky < 4 ? 4 : 1, bz = is2d ? 1 : (kz < 4 ? 4 : 1);
          const bool full = bx == 4 && by == 4 && bz == 4;
          if (s == 0 && level + 1 < f.nlevels && full)
            continue;
          expect.insert(std::make_tuple(kx, ky, kz, bx, by, bz));
        }
    std::vector<block_geom> g;
    subband_blocks(f, level, s, &g);
    for (const block_geom& b : g)
      got.insert(std::make_tuple((int)b.dx, (int)b.dy, (int)b.dz, (int)b.bx, (int)b.by, (int)b.bz));
    if (got != expect || got.size() != g.size())
      return false;
  }
  return true;
}

long long build_levels(const dataset_format& f, std::vector<syn_level>* out)
{
  const int L = f.nlevels;
  const int NB = f.is2d() ? 33 * 33 : 33 * 33 * 33;
  out->assign((size_t)L, syn_level());
  long long base = 0;
  for (int l = 0; l < L; ++l)
  {
    if (!uniform_blocks(f, l))
      return -1;
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
    double w[8];
    level_weights(f, l, w, &sl.norm_mask);
    for (int s = 0; s < 8; ++s)
      sl.inv_weight[s] = s < f.nsubbands() ? 1.0 / w[s] : 1.0;
  }
  return base;
}

template <typename T, bool IS2D>
int launch_synth(device_ctx* ctx, const syn_args<T>& a, bool adjoint, cudaStream_t st)
{
  constexpr int CS = IS2D ? 1 : kCS;
  const size_t smem = (size_t)(IS2D ? 1 : kPPC + 1) * kPlane * sizeof(T);
  void (*kern)(const syn_args<T>) = adjoint ? k_synth_adj<T, IS2D> : k_synth<T, IS2D>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return CudaError;
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof cfg);
  cudaLaunchAttribute attr[1];
  cfg.blockDim = dim3(kSynThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  int nclusters = ctx->num_sms * syn_ctas_per_sm<T>() / CS;
  if (CS > 1)
  {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(CS * nclusters);
    int active = 0;
    if (cudaOccupancyMaxActiveClusters(&active, kern, &cfg) == cudaSuccess && active > 0)
      nclusters = active;
  }
  if (nclusters > a.nbricks)
    nclusters = a.nbricks;
  if (nclusters < 1)
    return NoError;
  cfg.gridDim = dim3(CS * nclusters);
  return cudaLaunchKernelEx(&cfg, kern, a) == cudaSuccess ? NoError : CudaError;
}

template <typename T>
int run_synth(device_ctx* ctx, const dataset_format& f, int nbatch, const void* in, void* out, bool adjoint,
              double* kernel_ms)
{
  std::vector<syn_level> lv;
  const long long count = build_levels(f, &lv);
  if (count < 0)
    return OptionNotSupported;
  const int L = f.nlevels;
  const int NB = f.is2d() ? 33 * 33 : 33 * 33 * 33;
  cudaStream_t st = ctx->stream;
  const long long gcount = (long long)f.dims.x * f.dims.y * f.dims.z;
  float total = 0;
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
    syn_args<T> a;
    memset(&a, 0, sizeof a);
    a.nbricks = nbr;
    a.coarsest = l + 1 == L;
    a.finest = l == 0;
    a.norm_mask = sl.norm_mask;
    memcpy(a.inv_weight, sl.inv_weight, sizeof a.inv_weight);
    a.bricks = d_bricks;
    a.cstride = count;
    a.gstride = gcount;
    a.gdims[0] = f.dims.x;
    a.gdims[1] = f.dims.y;
    a.gdims[2] = f.dims.z;
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
    }
    cudaEventRecord(ctx->ev0, st);
    const int e = f.is2d() ? launch_synth<T, true>(ctx, a, adjoint, st) : launch_synth<T, false>(ctx, a, adjoint, st);
    cudaEventRecord(ctx->ev1, st);
    if (e)
      return e;
    prev = adjoint ? a.pgrad : a.bricks_out;
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
