// k_encode_split: the encode of 3D bricks with each brick held in shared memory,
// split over the two CTAs of a cluster by z parity (included by encode.cu inside its
// anonymous namespace, after k_encode_level, whose helpers it uses).
//
// A brick's 33^3 FP64 samples (287 KB) do not fit in one CTA's shared memory; its 17 even
// z-planes (148 KB) live in CTA 0 of the pair and its 16 odd planes in CTA 1. Sweeps along X
// and Y stay inside a plane, so each CTA lifts the lines of its own planes. A sweep along Z
// reads and writes both halves: the columns are shared out between the two CTAs and each
// column is lifted in registers from the two slabs (the peer's through distributed shared
// memory). The subbands of the brick take their z samples from one parity (subband
// 4hx + 2hy + hz lies on planes of parity hz), so CTA r codes the four subbands of parity r
// from its own slab, with the same coder as k_encode_level (code_subband). The even lattice
// of the coarser extrapolation levels lies on even planes: CTA 0 lifts it in its table space.
// The lifting functions and their operation order are those of k_encode_level, so the
// coefficients, and with them the bit streams, are the same bit for bit. The coding tables
// hold 32 bit planes (all a float32 dataset codes); a float64 block that needs more raises
// the level's error word 8 and the host codes the level again with k_encode_level.

constexpr int kSplitThreads = 512;
// encodes without a tuned choice take this kernel for their 3D bricks; the batch tuner offers it
constexpr bool kSplitByDefault = false;
constexpr bool kSplitOffered = false;
using split_smem = enc_smem_t<kSplitThreads>;
constexpr int kPlaneStride = 33 * 33;
constexpr size_t kSlabBytes = (size_t)17 * kPlaneStride * sizeof(double);
// table space of a split CTA: the coding tables of 32 planes, which also hold the gather's two
// chunk buffers and, in CTA 0, the 17^3 even lattice of the coarse extrapolation levels
constexpr size_t kSplitTableBytes =
  ((size_t)32 * ((size_t)kRowX * 8 + (size_t)kRowOff * 2 + (size_t)kRowNin) + 127) & ~(size_t)127;
static_assert(kSplitTableBytes >= (size_t)17 * 17 * 17 * 8, "the lattice fits in the table space");
static_assert(kSplitTableBytes >= (size_t)2 * kGz * 32 * 32 * 4, "two float32 chunk buffers fit");

constexpr size_t kSplitSmemBytes = ((sizeof(split_smem) + 127) & ~(size_t)127) + kSplitTableBytes + kSlabBytes;
static_assert(kSplitSmemBytes <= (size_t)227 * 1024, "a split CTA's shared memory fits the sm_100 limit");
inline size_t split_smem_bytes() { return kSplitSmemBytes; }

// Sample plane z of the brick: even planes in E, odd planes in O, each slab plane-major.
__device__ __forceinline__ double* split_plane(double* E, double* O, int z)
{
  return ((z & 1) ? O : E) + (z >> 1) * kPlaneStride;
}

// One column (x, y) of a first-level Z sweep (from z = 0, stride 1, D samples), lifted in
// registers from the two slabs; the same operations as lift_line_fixed.
template <bool FWD>
__device__ __forceinline__ void split_column(double* E, double* O, int off, int D)
{
  const bool ext = (D % 2) == 0;
  const int nload = D + (ext && !FWD ? 1 : 0);
  const int nstore = D + (ext && FWD ? 1 : 0);
  double v[33];
#pragma unroll
  for (int k = 0; k < 33; ++k)
    v[k] = k < nload ? ((k & 1) ? O : E)[(k >> 1) * kPlaneStride + off] : 0.0;
  dev::lift_regs<FWD>(v, D);
#pragma unroll
  for (int k = 0; k < 33; ++k)
    if (k < nstore)
      ((k & 1) ? O : E)[(k >> 1) * kPlaneStride + off] = v[k];
}

// One first-level sweep (grid from 0, stride 1 on every axis) of the split brick. X and Y:
// CTA r lifts the lines of its planes; Z: CTA r lifts every second column. The caller
// synchronises the cluster around Z sweeps (they touch both halves).
template <bool FWD>
__device__ void split_sweep(double* E, double* O, int r, const dev::dgrid& G, int ax)
{
  const int D = G.dims[ax];
  if (D == 1)
    return;
  if (ax == 2)
  {
    const int nx = G.dims[0], ncol = G.dims[0] * G.dims[1];
    for (int li = 2 * (int)threadIdx.x + r; li < ncol; li += 2 * (int)blockDim.x)
      split_column<FWD>(E, O, (li / nx) * 33 + li % nx, D);
    return;
  }
  // my planes of the grid: z = r, r + 2, ... < G.dims[2]
  const int nz = G.dims[2] > r ? (G.dims[2] - r + 1) / 2 : 0;
  double* const mine = r ? O : E;
  const int nu = G.dims[1 - ax];
  const int nlines = nu * nz;
  for (int li = threadIdx.x; li < nlines; li += blockDim.x)
  {
    double* L = mine + (li / nu) * kPlaneStride + (ax == 0 ? (li % nu) * 33 : li % nu);
    if (D == 33)
      ax == 0 ? dev::lift_line_strided<33, FWD, 1>(L) : dev::lift_line_strided<33, FWD, 33>(L);
    else if (D == 32)
      ax == 0 ? dev::lift_line_strided<32, FWD, 1>(L) : dev::lift_line_strided<32, FWD, 33>(L);
    else
      dev::lift_line<FWD>(L, ax == 0 ? 1 : 33, D);
  }
}

__device__ __forceinline__ bool first_level_grid(const dev::dgrid& g)
{
  return g.from[0] == 0 && g.from[1] == 0 && g.from[2] == 0 && g.strd[0] == 1 && g.strd[1] == 1 && g.strd[2] == 1;
}

// Bounded wait for the completion of an mbarrier phase (true if it completed).
__device__ __forceinline__ bool wait_parity(unsigned bar, unsigned par)
{
  int ok = 0;
  for (int it = 0; it < (1 << 22) && !ok; ++it)
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(bar), "r"(par)
                 : "memory");
  return ok != 0;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kSplitThreads, 1) k_encode_split(const enc_args a)
{
  extern __shared__ __align__(128) unsigned char smem_raw[];
  split_smem& sm = *reinterpret_cast<split_smem*>(smem_raw);
  unsigned char* const space = smem_raw + ((sizeof(split_smem) + 127) & ~(size_t)127);
  unsigned long long* const Xp = reinterpret_cast<unsigned long long*>(space);
  uint16_t* const OFF = reinterpret_cast<uint16_t*>(Xp + (size_t)kRowX * 32);
  uint8_t* const NIN = reinterpret_cast<uint8_t*>(OFF + (size_t)kRowOff * 32);
  double* const slab = reinterpret_cast<double*>(space + kSplitTableBytes);
  cg::cluster_group cl = cg::this_cluster();
  const int r = (int)cl.block_rank();  // the z parity of this CTA's planes
  double* const peer = cl.map_shared_rank(slab, r ^ 1);
  double* const E = r == 0 ? slab : peer;
  double* const O = r == 0 ? peer : slab;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = kSplitThreads / 32;
  if (tid < 64)
    sm.perm3[tid] = dev::perm(3, tid);
  if (tid < 16)
    sm.perm2[tid] = dev::perm(2, tid);
  if (tid == 0)
  {
    const unsigned b0 = (unsigned)__cvta_generic_to_shared(&sm.tma_bar[0]);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b0 + 8u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  unsigned tma_parity = 0;  // bit b: phase parity of chunk buffer b's next completion
  ENC_PHASE_INIT
  const int ncl = (int)gridDim.x / 2, cid = (int)blockIdx.x / 2;
  const int N[3] = { 33, 33, 33 };

  for (int it = a.first + cid; it < a.last; it += ncl)
  {
    const int bi = a.order ? a.order[it] : it;
    const enc_brick& br = a.bricks[bi];
    {
      static_assert(sizeof(enc_field) % 4 == 0, "enc_field is copied as words");
      const uint32_t* src = reinterpret_cast<const uint32_t*>(a.fields + br.field);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sm.fp);
      for (int i = tid; i < (int)(sizeof(enc_field) / 4); i += kSplitThreads)
        dst[i] = src[i];
    }
    if (tid == 0)
      dev::build_stack(br.valid, 5, a.fields[br.field].order, &sm.stack);
    __syncthreads();
    const enc_field& fp = sm.fp;
    const int nf = sm.stack.n, cf = sm.stack.coarse;
    // the extrapolation's first X and Y sweeps run on each plane as it arrives
    const bool xy_in_gather = a.level == 0 && cf >= 2 && sm.stack.axis[0] + sm.stack.axis[1] == 1 &&
                              first_level_grid(sm.stack.g[0]) && first_level_grid(sm.stack.g[1]);
    ENC_PHASE_START
    // ---------------- A: gather my planes ----------------
    double* const mine = slab;
    const int my_planes = r ? 16 : 17;
    if (a.level == 0)
    {
      const int vx = br.valid[0], vy = br.valid[1], vz = br.valid[2];
      double mn = 1.7976931348623157e308, mx = -1.7976931348623157e308;
      const long long gx0 = (long long)br.b3[0] * 32, gy0 = (long long)br.b3[1] * 32, gz0 = (long long)br.b3[2] * 32;
      // the first-level X and Y sweeps of one of my planes, z, if they are taken here
      auto plane_xy = [&](int z) {
        for (int k = 0; k < 2; ++k)
        {
          const dev::dgrid& G = sm.stack.g[k];
          const int ax = sm.stack.axis[k];
          const int D = G.dims[ax];
          if (D == 1 || z >= G.dims[2])
            continue;
          const int nu = G.dims[1 - ax];
          for (int li = tid; li < nu; li += kSplitThreads)
          {
            double* L = mine + (z >> 1) * kPlaneStride + (ax == 0 ? li * 33 : li);
            if (D == 32)
              ax == 0 ? dev::lift_line_strided<32, true, 1>(L) : dev::lift_line_strided<32, true, 33>(L);
            else if (D == 33)
              ax == 0 ? dev::lift_line_strided<33, true, 1>(L) : dev::lift_line_strided<33, true, 33>(L);
            else
              dev::lift_line<true>(L, ax == 0 ? 1 : 33, D);
          }
          __syncthreads();
        }
      };
      if (fp.tmap != nullptr && fp.field_f32)
      {
        // chunks of kGz planes by TMA (the field's tensor map, boxes 32 x 32 x kGz), double
        // buffered in the table space; this CTA keeps the planes of its parity
        unsigned char* const stage = space;
        const unsigned stage_bytes = (unsigned)(kGz * 32 * 32 * 4);
        const int nch = (33 + kGz - 1) / kGz;
        auto issue = [&](int c) {
          if (tid == 0 && c < nch && c * kGz < vz)
          {
            const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.tma_bar[c & 1]);
            const unsigned s0 = (unsigned)__cvta_generic_to_shared(stage) + (unsigned)(c & 1) * stage_bytes;
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(stage_bytes)
                         : "memory");
            asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
                         " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(s0),
                         "l"(fp.tmap), "r"((int)gx0), "r"((int)gy0), "r"((int)(gz0 + c * kGz)), "r"(bar)
                         : "memory");
          }
        };
        issue(0);
        for (int c = 0; c < nch; ++c)
        {
          issue(c + 1);
          int ok = 1;
          if (c * kGz < vz)
          {
            const unsigned bar = (unsigned)__cvta_generic_to_shared(&sm.tma_bar[c & 1]);
            ok = wait_parity(bar, (tma_parity >> (c & 1)) & 1u) ? 1 : 0;
            tma_parity ^= 1u << (c & 1);
          }
          if (!__syncthreads_and(ok) && tid == 0)
            atomicExch(a.error, 4);  // a lost copy: reported, and this brick's data is void
          const float* buf = reinterpret_cast<const float*>(stage + (size_t)(c & 1) * stage_bytes);
          // my planes of this chunk: z0 + r and z0 + r + 2
          for (int i = tid; i < 2 * kPlaneStride; i += kSplitThreads)
          {
            const int q = i / kPlaneStride, j = i % kPlaneStride;
            const int zz = r + 2 * q, z = c * kGz + zz;
            if (z > 32)
              continue;
            const int x = j % 33, y = j / 33;
            const bool in = x < vx && y < vy && z < vz;
            const double v = in ? (double)buf[(zz * 32 + y) * 32 + x] : 0.0;
            mine[(z >> 1) * kPlaneStride + j] = v;
            if (in)
            {
              mn = v < mn ? v : mn;
              mx = mx < v ? v : mx;
            }
          }
          __syncthreads();
          if (xy_in_gather)
            for (int q = 0; q < 2; ++q)
            {
              const int z = c * kGz + r + 2 * q;
              if (z <= 32)
                plane_xy(z);
            }
        }
      }
      else
      {
        // float64 fields, and fields TMA cannot take (pitches that are not multiples of 16
        // bytes): plain loads
        for (int i = tid; i < my_planes * kPlaneStride; i += kSplitThreads)
        {
          const int pl = i / kPlaneStride, j = i % kPlaneStride, z = 2 * pl + r;
          const int x = j % 33, y = j / 33;
          const bool in = x < vx && y < vy && z < vz;
          double v = 0.0;
          if (in)
          {
            const long long src = ((gz0 + z) * fp.fdims[1] + gy0 + y) * fp.fdims[0] + gx0 + x;
            v = fp.field_f32 ? (double)__ldg((const float*)fp.field + src) : __ldg((const double*)fp.field + src);
            mn = v < mn ? v : mn;
            mx = mx < v ? v : mx;
          }
          mine[i] = v;
        }
        __syncthreads();
        if (xy_in_gather)
          for (int pl = 0; pl < my_planes; ++pl)
            plane_xy(2 * pl + r);
      }
      for (int o = 16; o > 0; o >>= 1)
      {
        const double w1 = __shfl_xor_sync(0xffffffffu, mn, o), w2 = __shfl_xor_sync(0xffffffffu, mx, o);
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
        for (int w = 1; w < NW; ++w)
        {
          mn = sm.red[0][w] < mn ? sm.red[0][w] : mn;
          mx = mx < sm.red[1][w] ? sm.red[1][w] : mx;
        }
        sm.red[0][0] = mn;
        sm.red[1][0] = mx;
      }
    }
    else
    {
      // level > 0: the parent brick the children assembled (33^3, global)
      const double* src = a.in_bricks + (size_t)bi * (size_t)kNB3;
      for (int i = tid; i < my_planes * kPlaneStride; i += kSplitThreads)
      {
        const int pl = i / kPlaneStride, j = i % kPlaneStride;
        mine[i] = __ldcs(src + (size_t)(2 * pl + r) * kPlaneStride + j);
      }
    }
    cl.sync();  // both halves of the brick in place
    if (a.level == 0 && tid == 0 && r == 0)
    {
      // the brick's value range from both halves
      const double* pr = cl.map_shared_rank(&sm.red[0][0], 1);
      const double* px = cl.map_shared_rank(&sm.red[1][0], 1);
      const double m0 = sm.red[0][0] < *pr ? sm.red[0][0] : *pr;
      const double m1 = sm.red[1][0] < *px ? *px : sm.red[1][0];
      a.bmin[bi] = m0;
      a.bmax[bi] = m1;
    }
    ENC_PHASE(0)

    // ---------------- B: transform ----------------
    // A sweep along Z reads and writes both halves: the cluster synchronises before it (the
    // other CTA's in-plane sweeps done) and after it (before in-plane sweeps touch its writes).
    auto sweep = [&](int i, bool fwd) {
      const int ax = sm.stack.axis[i];
      if (ax == 2)
        cl.sync();
      if (fwd)
        split_sweep<true>(E, O, r, sm.stack.g[i], ax);
      else
        split_sweep<false>(E, O, r, sm.stack.g[i], ax);
      if (ax == 2)
        cl.sync();
      else
        __syncthreads();
    };
    // extrapolation, first level (Core/Wavelet.cpp:68): forward on the valid dims
    for (int i = xy_in_gather ? 2 : 0; i < cf; ++i)
      sweep(i, true);
    cl.sync();  // the even lattice complete in CTA 0's slab
    ENC_PHASE(2)
    // coarser levels on the 17^3 even lattice (all on even planes: CTA 0, in its table space)
    double* const S = reinterpret_cast<double*>(space);
    const int NS[3] = { 17, 17, 17 };
    constexpr int nsub = 17 * 17 * 17;
    if (r == 0)
    {
      for (int i = tid; i < nsub; i += kSplitThreads)
      {
        const int x = i % 17, y = (i / 17) % 17, z = i / 289;
        S[i] = E[z * kPlaneStride + (2 * y) * 33 + 2 * x];
      }
      __syncthreads();
      for (int i = cf; i < nf; ++i)
      {
        dev::lift_sweep(S, NS, dev::half_grid(sm.stack.g[i]), NS, sm.stack.axis[i], true);
        __syncthreads();
      }
    }
    ENC_PHASE(3)
    if (tid == 0)
      dev::build_stack(N, 5, fp.order, &sm.stack);
    __syncthreads();
    const int ni = sm.stack.n, ci = sm.stack.coarse;
    if (r == 0)
    {
      for (int i = ni - 1; i >= ci; --i)
      {
        dev::lift_sweep(S, NS, dev::half_grid(sm.stack.g[i]), NS, sm.stack.axis[i], false);
        __syncthreads();
      }
      for (int i = tid; i < nsub; i += kSplitThreads)
      {
        const int x = i % 17, y = (i / 17) % 17, z = i / 289;
        E[z * kPlaneStride + (2 * y) * 33 + 2 * x] = S[i];
      }
    }
    cl.sync();
    ENC_PHASE(4)
    // inverse of the first level, then the one-level forward transform (Core/Wavelet.cpp:81):
    // the inverse X is fused with the forward X when they are adjacent (the usual order)
    const bool fuse_x = ci >= 1 && sm.stack.axis[0] == 0 && sm.stack.g[0].dims[0] == 33 &&
                        sm.stack.g[0].dims[1] == 33 && sm.stack.g[0].dims[2] == 33 && first_level_grid(sm.stack.g[0]);
    for (int i = ci - 1; i >= (fuse_x ? 1 : 0); --i)
      sweep(i, false);
    ENC_PHASE(5)
    {
      // inverse X (if fused) then forward X, rows of my planes
      const int nrows = 33 * my_planes;
      for (int li = tid; li < nrows; li += kSplitThreads)
      {
        double* row = mine + li * 33;
        double v[33];
#pragma unroll
        for (int k = 0; k < 33; ++k)
          v[k] = row[k];
        if (fuse_x)
          dev::lift_regs<false>(v, 33);
        dev::lift_regs<true>(v, 33);
#pragma unroll
        for (int k = 0; k < 33; ++k)
          row[k] = v[k];
      }
      __syncthreads();
      // forward Y, columns of my planes
      for (int li = tid; li < nrows; li += kSplitThreads)
      {
        double* col = mine + (li / 33) * kPlaneStride + li % 33;
        double v[33];
#pragma unroll
        for (int k = 0; k < 33; ++k)
          v[k] = col[k * 33];
        dev::lift_regs<true>(v, 33);
#pragma unroll
        for (int k = 0; k < 33; ++k)
          col[k * 33] = v[k];
      }
    }
    cl.sync();
    ENC_PHASE(6)
    // forward Z over both halves, subband normalisation applied as it stores
    for (int li = 2 * tid + r; li < 33 * 33; li += 2 * kSplitThreads)
    {
      const int x = li % 33, y = li / 33;
      double v[33];
#pragma unroll
      for (int k = 0; k < 33; ++k)
        v[k] = ((k & 1) ? O : E)[(k >> 1) * kPlaneStride + li];
      dev::lift_regs<true>(v, 33);
#pragma unroll
      for (int k = 0; k < 33; ++k)
      {
        const int s = ((x & 1) << 2) | ((y & 1) << 1) | (k & 1);
        ((k & 1) ? O : E)[(k >> 1) * kPlaneStride + li] =
          ((fp.norm_mask >> s) & 1) ? __dmul_rn(v[k], fp.weight[s]) : v[k];
      }
    }
    cl.sync();
    ENC_PHASE(8)

    // ---------------- C: low band to the parent (even planes: CTA 0) ----------------
    if (r == 0 && a.parent_bricks && br.parent >= 0)
    {
      double* Pb = a.parent_bricks + (size_t)br.parent * (size_t)kNB3;
      for (int i = tid; i < 16 * 16 * 16; i += kSplitThreads)
      {
        const int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        __stcs(Pb + ((br.pos[2] * 16 + z) * 33 + (br.pos[1] * 16 + y)) * 33 + (br.pos[0] * 16 + x),
               E[z * kPlaneStride + (2 * y) * 33 + 2 * x]);
      }
    }
    ENC_PHASE(9)

    // ---------------- D: the four subbands of my parity ----------------
    for (int s = r; s < 8; s += 2)
    {
      if (r == 0 && a.level == 0 && s == 4 && it + ncl < a.last)
      {
        const int nx = a.order ? a.order[it + ncl] : it + ncl;
        prefetch_rows(a.fields[a.bricks[nx].field], a.bricks[nx]);
      }
      code_subband<kSplitThreads>(a, sm, Xp, OFF, NIN, 32, mine, kPlaneStride, true, bi, s, pacc_);
    }
  }
  // neither CTA leaves while the other may still read its slab
  cl.sync();
  ENC_PHASE_FLUSH
}
