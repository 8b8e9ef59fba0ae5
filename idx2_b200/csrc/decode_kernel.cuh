// k_decode_level: the device decode of one level (included by decode.cu, inside an
// anonymous namespace). See decode.cu for the pipeline overview.
#pragma once

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRing = 32;  // steps a decoded plane stays in the per-warp ring (>= channels)

struct dec_args
{
  int level, nlevels, is2d, nsb, nbricks, etol, end_bp, mask, norm_mask, is_output, out_f32;
  int spacing[8][3];
  int nblocks[8];
  double inv_weight[8];
  const uint64_t* geom;               // [8][kMaxBlocksPerSubband]
  const decode_brick* bricks;
  const int16_t* exps;                // [flat][sb][kMaxBlocksPerSubband]
  const int32_t* ckmin;
  const int32_t* cn;
  const unsigned long long* cfirst;
  const unsigned long long* coff;
  const uint8_t* blob;
  unsigned long long blob_bytes;
  const double* parents;              // decoded bricks of the coarser level
  double* bricks_out;                 // decoded bricks of this level (non-output level)
  double* slots;                      // per-CTA slots (output level)
  void* out;
  int out_dims[3];
  int* error;
};

struct dec_smem
{
  union
  {
    unsigned long long coef[kMaxBlocksPerSubband][64];  // CTA-wide path: one subband
    unsigned long long ring[kWarps][kRing][32];         // warp path: decoded planes in flight
  } u;
  long long q[kWarps][64];
  int16_t emax[8][kMaxBlocksPerSubband];
  int16_t ktop[8][kMaxBlocksPerSubband];
  uint8_t np[8][kMaxBlocksPerSubband];
  uint8_t nbps[8][kMaxBlocksPerSubband];
  uint8_t nd[8][kMaxBlocksPerSubband];
  uint8_t bypass[8][kMaxBlocksPerSubband];
  uint8_t nst[2][kKeyWindow];
  uint8_t stop[2][kKeyWindow];
  int kmax[8], nkeys[8];
  int wide;
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

// LSB-first bit reader over the blob with a 128-bit register window (Core/BitStream.h
// semantics). Words past the end of the blob read as zero.
struct bit_reader
{
  const unsigned long long* w;
  unsigned long long nwords, idx, w0, w1;
  int bit;
  __device__ __forceinline__ void init(const uint8_t* blob, unsigned long long nbytes, unsigned long long pos)
  {
    w = reinterpret_cast<const unsigned long long*>(blob);
    nwords = (nbytes + 7) >> 3;
    idx = pos >> 6;
    bit = (int)(pos & 63);
    w0 = idx < nwords ? w[idx] : 0ull;
    w1 = idx + 1 < nwords ? w[idx + 1] : 0ull;
  }
  __device__ __forceinline__ unsigned long long peek() const
  {
    return bit ? (w0 >> bit) | (w1 << (64 - bit)) : w0;
  }
  __device__ __forceinline__ void skip(int n)  // n <= 64
  {
    bit += n;
    if (bit >= 64)
    {
      bit -= 64;
      w0 = w1;
      ++idx;
      w1 = idx + 1 < nwords ? w[idx + 1] : 0ull;
    }
  }
  __device__ __forceinline__ unsigned long long read(int n)  // n <= 64
  {
    if (n <= 0)
      return 0ull;
    unsigned long long v = peek();
    if (n < 64)
      v &= (1ull << n) - 1ull;
    skip(n);
    return v;
  }
};

// One bit plane of the group-test decoder (Core/Zfp.h:990 Decode<u64>): returns the plane
// bits and advances n (significant coefficients). Runs of zeros are consumed 64 at a time.
__device__ __forceinline__ unsigned long long decode_plane(bit_reader& rd, int& n, int nvals)
{
  unsigned long long X = n > 0 ? rd.read(n) : 0ull;
  while (n < nvals)
  {
    if (!rd.read(1))
      break;
    const int lim = nvals - 1 - n;  // explicit bits before the last coefficient
    unsigned long long pk = rd.peek();
    int t = pk ? __ffsll((long long)pk) - 1 : 64;
    if (t >= lim)
    {
      rd.skip(lim);
      n = nvals - 1;
    }
    else
    {
      rd.skip(t + 1);
      n += t;
    }
    X += 1ull << n;
    ++n;
  }
  return X;
}

// Inverse shuffle / inverse zfp / dequantise of one block and scatter into the brick
// (Core/idx2Decode.cpp:203-227), by one warp; u holds the negabinary coefficients.
__device__ __forceinline__ void reconstruct_block(double* F, long long* q, unsigned long long u0,
                                                  unsigned long long u1, int nd, int emax, uint64_t g,
                                                  const int from[3], const int strd[3], int lane)
{
  int d3[3], bd[3];
  unpack_geom(g, d3, bd);
  const int nv = 1 << (2 * nd);
  if (lane < nv)
    q[dev::perm(nd, lane)] = (long long)((u0 ^ dev::kNegaMask) - dev::kNegaMask);
  if (lane + 32 < nv)
    q[dev::perm(nd, lane + 32)] = (long long)((u1 ^ dev::kNegaMask) - dev::kNegaMask);
  __syncwarp();
  dev::warp_inv_zfp(q, nd, lane);
  const double scale = __ddiv_rn(1.0, dev::pow2(63 - nd - 1 - emax));
  for (int j = lane; j < nv; j += 32)
  {
    int x = j % bd[0], y = (j / bd[0]) % bd[1], z = j / (bd[0] * bd[1]);
    F[((from[2] + (d3[2] + z) * strd[2]) * 33 + (from[1] + (d3[1] + y) * strd[1])) * 33 +
      (from[0] + (d3[0] + x) * strd[0])] = __dmul_rn(scale, __ll2double_rn(q[j]));
  }
  __syncwarp();
}

// One-level inverse CDF5/3 of a 33-sample line held in registers (Core/Wavelet.h:250
// ILiftCdf53 with D = 33, S = 1, no extrapolation, lift_option Normal).
__device__ __forceinline__ void ilift33(double (&v)[33])
{
#pragma unroll
  for (int x = 1; x < 31; x += 2)
  {
    double V = __dmul_rn(v[x], 0.25);
    v[x - 1] = __dsub_rn(v[x - 1], V);
    v[x + 1] = __dsub_rn(v[x + 1], V);
  }
  {
    double V = __dmul_rn(v[31], 0.25);
    v[30] = __dsub_rn(v[30], V);
    v[32] = __dsub_rn(v[32], V);
  }
#pragma unroll
  for (int x = 1; x < 31; x += 2)
    v[x] = __dadd_rn(v[x], __dmul_rn(__dadd_rn(v[x - 1], v[x + 1]), 0.5));
  v[31] = __dadd_rn(v[31], __dmul_rn(__dadd_rn(v[32], v[30]), 0.5));
}

__global__ void __launch_bounds__(kThreads, 2) k_decode_level(const dec_args a)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  dec_smem& sm = *reinterpret_cast<dec_smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N[3] = { 33, 33, a.is2d ? 1 : 33 };
  const int NB = N[0] * N[1] * N[2];

  for (int bi = blockIdx.x; bi < a.nbricks; bi += gridDim.x)
  {
    const decode_brick br = a.bricks[bi];
    double* F = a.is_output ? a.slots + (size_t)blockIdx.x * (size_t)NB
                            : a.bricks_out + (size_t)bi * (size_t)NB;
    // 1: zero + parent low band (Core/idx2Decode.cpp:285-293)
    for (int i = tid; i < NB; i += kThreads)
      F[i] = 0.0;
    __syncthreads();
    if (br.parent >= 0 && a.parents && (a.mask & 1))
    {
      const double* P = a.parents + (size_t)br.parent * (size_t)NB;
      const int nz = a.is2d ? 1 : 16;
      for (int i = tid; i < 16 * 16 * nz; i += kThreads)
      {
        int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        int cz = a.is2d ? 0 : 2 * z;
        F[(cz * 33 + 2 * y) * 33 + 2 * x] =
          P[((br.pos[2] * nz + z) * 33 + (br.pos[1] * 16 + y)) * 33 + (br.pos[0] * 16 + x)];
      }
    }

    // 2: per-block state of every decoded subband
    for (int i = tid; i < a.nsb * kMaxBlocksPerSubband; i += kThreads)
    {
      const int s = i / kMaxBlocksPerSubband, b = i % kMaxBlocksPerSubband;
      if (!((a.mask >> s) & 1) || b >= a.nblocks[s])
        continue;
      int d3[3], bd[3];
      unpack_geom(a.geom[(size_t)s * kMaxBlocksPerSubband + b], d3, bd);
      const size_t fs = (size_t)br.flat * (size_t)a.nsb + (size_t)s;
      const int emax = a.exps[fs * kMaxBlocksPerSubband + (size_t)b];
      sm.emax[s][b] = (int16_t)emax;
      sm.ktop[s][b] = (int16_t)(emax + 63 + 1024);
      sm.np[s][b] = (uint8_t)dev::coded_planes(emax, a.etol, a.end_bp);
      sm.nbps[s][b] = 0;
      sm.nd[s][b] = (uint8_t)((bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1));
      sm.bypass[s][b] = (uint8_t)((d3[0] % a.spacing[s][0]) != 0 || (d3[1] % a.spacing[s][1]) != 0 ||
                                  (d3[2] % a.spacing[s][2]) != 0);
    }
    __syncthreads();
    if (tid < a.nsb)
    {
      const int s = tid;
      int kmax = -(1 << 30), kmin = 1 << 30;
      if ((a.mask >> s) & 1)
        for (int b = 0; b < a.nblocks[s]; ++b)
        {
          if (!sm.np[s][b])
            continue;
          kmax = sm.ktop[s][b] > kmax ? sm.ktop[s][b] : kmax;
          int lo = sm.ktop[s][b] - sm.np[s][b] + 1;
          kmin = lo < kmin ? lo : kmin;
        }
      int nk = kmax >= kmin ? kmax - kmin + 1 : 0;
      if (nk > kKeyWindow)
      {
        atomicExch(a.error, 1);
        nk = 0;
      }
      sm.kmax[s] = kmax;
      sm.nkeys[s] = nk;
    }
    __syncthreads();
    if (tid == 0)
    {
      int wide = 0;
      for (int s = 0; s < a.nsb; ++s)
        wide |= sm.nkeys[s] > 32;
      sm.wide = wide;
    }
    __syncthreads();

    if (!sm.wide)
    {
      // 3a: warp w decodes subband w. Lane j owns channel (kmax - j); at step t it decodes
      // that plane of block t - j, taking the block's significance count from lane j - 1 of
      // step t - 1. Block t - (nkeys - 1) is complete after step t and is rebuilt at once.
      const int s = warp;
      if (s < a.nsb && ((a.mask >> s) & 1) && sm.nkeys[s] > 0)
      {
        const int nb = a.nblocks[s];
        const int nkeys = sm.nkeys[s], kmax = sm.kmax[s];
        const size_t fs = (size_t)br.flat * (size_t)a.nsb + (size_t)s;
        const uint64_t* geom = a.geom + (size_t)s * kMaxBlocksPerSubband;
        int from[3], dims[3], strd[3];
        subband_grid(a.is2d, s, from, dims, strd);
        const int key = kmax - lane;
        bit_reader rd;
        bool has = false;
        if (lane < nkeys)
        {
          const int ck = a.ckmin[fs], cn = a.cn[fs];
          if (key >= ck && key < ck + cn)
          {
            unsigned long long o = a.coff[a.cfirst[fs] + (unsigned long long)(key - ck)];
            if (o != ~0ull)
            {
              rd.init(a.blob, a.blob_bytes, o * 8ull);
              has = true;
            }
          }
        }
        int n_out = 0, stop_out = 0;
        unsigned long long(*ring)[32] = sm.u.ring[warp];
        const int steps = nb + nkeys - 1;
        for (int t = 0; t < steps; ++t)
        {
          const int n_left = __shfl_up_sync(0xffffffffu, n_out, 1);
          const int stop_left = __shfl_up_sync(0xffffffffu, stop_out, 1);
          n_out = 0;
          stop_out = 0;
          unsigned long long X = 0;
          const int b = t - lane;
          if (lane < nkeys && b >= 0 && b < nb)
          {
            const int top = sm.ktop[s][b], np = sm.np[s][b];
            if (np > 0 && key <= top && key > top - np)
            {
              int n = key == top ? 0 : n_left;
              const int stopped = key == top ? 0 : stop_left;
              if (stopped || !has)
              {
                stop_out = 1;
                n_out = n;
              }
              else
              {
                X = decode_plane(rd, n, 1 << (2 * sm.nd[s][b]));
                sm.nbps[s][b] += 1;
                n_out = n;
              }
            }
          }
          ring[t % kRing][lane] = X;
          __syncwarp();
          const int bc = t - (nkeys - 1);
          if (bc >= 0 && bc < nb && sm.nbps[s][bc] > 0 && !sm.bypass[s][bc])
          {
            const int top = sm.ktop[s][bc];
            unsigned long long u0 = 0, u1 = 0;
            for (int j = kmax - top; j < nkeys; ++j)
            {
              const int bp = 63 - (top - (kmax - j));
              if (bp < 0)
                break;
              const unsigned long long P = ring[(bc + j) % kRing][j];
              u0 |= ((P >> lane) & 1ull) << bp;
              u1 |= ((P >> (lane + 32)) & 1ull) << bp;
            }
            reconstruct_block(F, sm.q[warp], u0, u1, sm.nd[s][bc], sm.emax[s][bc], geom[bc], from, strd, lane);
          }
          __syncwarp();
        }
      }
    }
    else
    {
      // 3b: subbands with more than 32 channels: CTA-wide wavefront, one subband at a time
      for (int s = 0; s < a.nsb; ++s)
      {
        if (!((a.mask >> s) & 1))
          continue;
        int from[3], dims[3], strd[3];
        subband_grid(a.is2d, s, from, dims, strd);
        const int nb = a.nblocks[s];
        const uint64_t* geom = a.geom + (size_t)s * kMaxBlocksPerSubband;
        const size_t fs = (size_t)br.flat * (size_t)a.nsb + (size_t)s;
        const int nkeys = sm.nkeys[s], kmax = sm.kmax[s];
        for (int i = tid; i < nb * 64; i += kThreads)
          sm.u.coef[i >> 6][i & 63] = 0ull;
        const int key = kmax - tid;
        bit_reader rd;
        bool has = false;
        if (tid < nkeys)
        {
          const int ck = a.ckmin[fs], cn = a.cn[fs];
          if (key >= ck && key < ck + cn)
          {
            unsigned long long o = a.coff[a.cfirst[fs] + (unsigned long long)(key - ck)];
            if (o != ~0ull)
            {
              rd.init(a.blob, a.blob_bytes, o * 8ull);
              has = true;
            }
          }
          sm.nst[0][tid] = 0;
          sm.stop[0][tid] = 0;
        }
        __syncthreads();
        const int steps = nkeys > 0 ? nb + nkeys - 1 : 0;
        for (int t = 0; t < steps; ++t)
        {
          const int rb = t & 1, wb = rb ^ 1;
          if (tid < nkeys)
          {
            const int b = t - tid;
            uint8_t out_n = 0, out_stop = 0;
            if (b >= 0 && b < nb)
            {
              const int top = sm.ktop[s][b], np = sm.np[s][b];
              if (np > 0 && key <= top && key > top - np)
              {
                int n = key == top ? 0 : sm.nst[rb][tid - 1];
                const int stopped = key == top ? 0 : sm.stop[rb][tid - 1];
                if (stopped || !has)
                {
                  out_stop = 1;
                  out_n = (uint8_t)n;
                }
                else
                {
                  unsigned long long X = decode_plane(rd, n, 1 << (2 * sm.nd[s][b]));
                  const int bp = 63 - (top - key);
                  if (!sm.bypass[s][b])
                    for (unsigned long long y = X; y; y &= y - 1)
                      sm.u.coef[b][__ffsll((long long)y) - 1] += 1ull << bp;
                  sm.nbps[s][b] += 1;
                  out_n = (uint8_t)n;
                }
              }
            }
            sm.nst[wb][tid] = out_n;
            sm.stop[wb][tid] = out_stop;
          }
          __syncthreads();
        }
        for (int b = warp; b < nb; b += kWarps)
        {
          if (sm.nbps[s][b] == 0 || sm.bypass[s][b])
            continue;
          reconstruct_block(F, sm.q[warp], sm.u.coef[b][lane], sm.u.coef[b][lane + 32], sm.nd[s][b], sm.emax[s][b],
                            geom[b], from, strd, lane);
        }
        __syncthreads();
      }
    }
    __syncthreads();

    // 4: de-normalise + inverse CDF5/3 Z, Y, X (Core/Wavelet.cpp:144-203); the
    // de-normalisation is applied as the Z lines are loaded, the output crop and cast as the
    // X lines are stored.
    if (!a.is2d)
    {
      for (int li = tid; li < 33 * 33; li += kThreads)
      {
        const int x = li % 33, y = li / 33;
        double v[33];
#pragma unroll
        for (int z = 0; z < 33; ++z)
        {
          const int s = ((x & 1) << 2) | ((y & 1) << 1) | (z & 1);
          double f = F[(z * 33 + y) * 33 + x];
          v[z] = ((a.norm_mask >> s) & 1) ? __dmul_rn(f, a.inv_weight[s]) : f;
        }
        ilift33(v);
#pragma unroll
        for (int z = 0; z < 33; ++z)
          F[(z * 33 + y) * 33 + x] = v[z];
      }
      __syncthreads();
    }
    for (int li = tid; li < 33 * N[2]; li += kThreads)
    {
      const int x = li % 33, z = li / 33;
      double v[33];
#pragma unroll
      for (int y = 0; y < 33; ++y)
      {
        double f = F[(z * 33 + y) * 33 + x];
        if (a.is2d)
        {
          const int s = ((x & 1) << 1) | (y & 1);
          f = ((a.norm_mask >> s) & 1) ? __dmul_rn(f, a.inv_weight[s]) : f;
        }
        v[y] = f;
      }
      ilift33(v);
#pragma unroll
      for (int y = 0; y < 33; ++y)
        F[(z * 33 + y) * 33 + x] = v[y];
    }
    __syncthreads();
    for (int li = tid; li < 33 * N[2]; li += kThreads)
    {
      const int y = li % 33, z = li / 33;
      double v[33];
      double* row = F + (z * 33 + y) * 33;
#pragma unroll
      for (int x = 0; x < 33; ++x)
        v[x] = row[x];
      ilift33(v);
      if (!a.is_output)
      {
#pragma unroll
        for (int x = 0; x < 33; ++x)
          row[x] = v[x];
      }
      else
      {
        // 5: output (Core/idx2Decode.cpp:431-442 CopyGridGrid) for the samples of this row
        const int ry = y - br.src_from[1], rz = z - br.src_from[2];
        if (ry >= 0 && rz >= 0 && ry % br.src_strd[1] == 0 && rz % br.src_strd[2] == 0 &&
            ry / br.src_strd[1] < br.dims[1] && rz / br.src_strd[2] < br.dims[2])
        {
          const long long oy = br.dst_from[1] + (long long)(ry / br.src_strd[1]) * br.dst_strd[1];
          const long long oz = br.dst_from[2] + (long long)(rz / br.src_strd[2]) * br.dst_strd[2];
          const long long obase = (oz * a.out_dims[1] + oy) * a.out_dims[0];
#pragma unroll
          for (int x = 0; x < 33; ++x)
          {
            const int rx = x - br.src_from[0];
            if (rx >= 0 && rx % br.src_strd[0] == 0 && rx / br.src_strd[0] < br.dims[0])
            {
              const long long di = obase + br.dst_from[0] + (long long)(rx / br.src_strd[0]) * br.dst_strd[0];
              if (a.out_f32)
                ((float*)a.out)[di] = __double2float_rn(v[x]);
              else
                ((double*)a.out)[di] = v[x];
            }
          }
        }
      }
    }
    __syncthreads();
  }
}
