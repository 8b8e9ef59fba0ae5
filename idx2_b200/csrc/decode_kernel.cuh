// k_decode_level: the device decode of one level (included by decode.cu, inside an
// anonymous namespace). See decode.cu for the pipeline overview.
#pragma once

// Per-phase cycle counters of thread 0 of every CTA, for profiling builds only
// (-DIDX2G_PHASE_TIMING); compiled out otherwise.
#ifdef IDX2G_PHASE_TIMING
__device__ unsigned long long g_dec_phase_cycles[16];
#define DEC_PHASE_INIT \
  long long ph_[8] = {};   \
  long long ph_t = 0;
#define DEC_PHASE_START \
  if (threadIdx.x == 0) \
    ph_t = clock64();
#define DEC_PHASE(k)                 \
  if (threadIdx.x == 0)              \
  {                                  \
    const long long t_ = clock64();  \
    ph_[k] += t_ - ph_t;             \
    ph_t = t_;                       \
  }
#define DEC_PHASE_FLUSH           \
  if (threadIdx.x == 0)           \
    for (int k = 0; k < 8; ++k)   \
      atomicAdd(&g_dec_phase_cycles[k], (unsigned long long)ph_[k]);
#else
#define DEC_PHASE_INIT
#define DEC_PHASE_START
#define DEC_PHASE(k)
#define DEC_PHASE_FLUSH
#endif

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRing = 32;  // steps a decoded plane stays in the per-warp ring (>= channels)

struct dec_args
{
  int level, nlevels, is2d, nsb, nbricks, end_bp, norm_mask, out_f32;
  int bpc;                            // BitPlanesPerChunk: bit planes per channel key
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
  const double* parents;              // kept bricks of the coarser launch
  double* bricks_out;                 // kept bricks of this launch (by store index)
  double* slots;                      // per-CTA slots (output bricks)
  const decode_target* reqs;          // request table of the launch
  int* error;
  int* sig;                           // brick-map mode: significance per stored brick (or null)
  // coefficient mode: the dequantised zfp-domain coefficients of every brick, at their sample
  // positions in a 33^3 (33^2) brick of the dataset's dtype (brick `store` of the tensor), in
  // place of the decoded grid
  void* coeff_out;
  // decoded bit planes from k_decode_planes (null: the kernel runs the wavefront itself)
  const unsigned long long* planes;
  const unsigned long long* unit_off;  // [brick][subband] byte offset of the unit's table, ~0: none
};

// Arguments of the bit-plane kernel (one warp per (brick, subband) unit).
struct dec1_args
{
  int bpc;                          // BitPlanesPerChunk: bit planes per channel key
  int nsb, nbricks, end_bp;
  int unit_first, unit_last;        // the first pass decodes units [unit_first, unit_last)
  const decode_target* reqs;
  int nblocks[8];
  const uint64_t* geom;  // [8][kMaxBlocksPerSubband]
  const decode_brick* bricks;
  const int16_t* exps;
  const int32_t* ckmin;
  const int32_t* cn;
  const unsigned long long* cfirst;
  const unsigned long long* coff;
  const uint8_t* blob;
  unsigned long long blob_bytes;
  unsigned long long* planes;       // tables, allocated with the cursor
  unsigned long long cap_bytes;
  unsigned long long* cursor;
  unsigned long long* unit_off;
  int* error;                       // bit flags: 1 too many channels, 2 table capacity exceeded
  int* wide_count;                  // units with more than 32 channels, deferred by the first pass
  int* wide_list;
};

// The union comes last: a launch of the plane-table path with a float32 output needs only its
// float staging rows, and passes a dynamic shared-memory size that ends there
// (dec_smem_bytes).
struct dec_smem
{
  long long out_base[kWarps][32];  // offsets in the output of the staged rows (-1: no output)
  long long q[kWarps][2][80];  // per-warp block scratch (two blocks, padded in the table path)
  int16_t emax[8][kMaxBlocksPerSubband];
  int16_t ktop[8][kMaxBlocksPerSubband];
  uint8_t np[8][kMaxBlocksPerSubband];
  uint8_t nuse[8][kMaxBlocksPerSubband];  // planes that enter the coefficients (0: block not rebuilt)
  uint8_t nbps[8][kMaxBlocksPerSubband];
  uint8_t nd[8][kMaxBlocksPerSubband];
  uint8_t bypass[8][kMaxBlocksPerSubband];
  uint8_t perm3[64];
  uint8_t perm2[16];
  uint8_t nst[2][kKeyWindow];
  uint8_t stop[2][kKeyWindow];
  int kmax[8], nkeys[8];
  int wide;
  int sig;           // a block of a subband > 0 (or of the coarsest level) was decoded
  decode_target rq;  // the current brick's request
  union
  {
    double v[kWarps][32][33];   // output rows of the X sweep, one per lane (float64 output)
    float v32[kWarps][32][33];  // the same cast to float (float32 output)
    unsigned long long coef[kMaxBlocksPerSubband][64];  // CTA-wide path: one subband
    unsigned long long ring[kWarps][kRing][32];         // warp path: decoded planes in flight
  } u;
};

// Dynamic shared memory of a launch: all of dec_smem, or, for the plane-table path with a
// float32 output, up to the end of the float staging rows.
inline size_t dec_smem_bytes(bool planes, bool out_f32)
{
  if (planes && out_f32)
    return offsetof(dec_smem, u) + sizeof(float) * kWarps * 32 * 33;
  return sizeof(dec_smem);
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

// Decoded bricks are stored subband-major: the 33^3 samples are the 8 subbands (index
// 4hx + 2hy + hz, of 17 - h samples per axis) one after the other, each dense and x-fastest.
// Blocks then land in contiguous rows, and a line of the inverse transform reads two dense
// streams (its even and odd samples).
__device__ __forceinline__ int sbm_base(int hx, int hy, int hz, int is2d)
{
  const int dx = 17 - hx, dy = 17 - hy;
  return is2d ? hx * 17 * 33 + hy * dx * 17 : hx * 17 * 33 * 33 + hy * dx * 17 * 33 + hz * dx * dy * 17;
}

// Position (x, y, z) of the brick in the subband-major layout.
__device__ __forceinline__ int sbm(int x, int y, int z, int is2d)
{
  const int hx = x & 1, hy = y & 1, hz = z & 1;
  const int dx = 17 - hx, dy = 17 - hy;
  return sbm_base(hx, hy, hz, is2d) + (((z >> 1) * dy + (y >> 1)) * dx + (x >> 1));
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
// (Core/idx2Decode.cpp:203-227), by one warp; u holds the negabinary coefficients, perm the
// coefficient order (Core/Zfp.h:419 Perm3, :498 Perm2) in shared memory.
__device__ __forceinline__ void reconstruct_block(double* F, long long* q, const uint8_t* perm3,
                                                  const uint8_t* perm2, unsigned long long u0,
                                                  unsigned long long u1, int nd, int emax, uint64_t g,
                                                  int s, int is2d, int lane)
{
  int d3[3], bd[3];
  unpack_geom(g, d3, bd);
  const int nv = 1 << (2 * nd);
  auto perm = [&](int j) -> int { return nd == 3 ? (int)perm3[j] : (nd == 2 ? (int)perm2[j & 15] : j); };
  if (lane < nv)
    q[perm(lane)] = (long long)((u0 ^ dev::kNegaMask) - dev::kNegaMask);
  if (lane + 32 < nv)
    q[perm(lane + 32)] = (long long)((u1 ^ dev::kNegaMask) - dev::kNegaMask);
  __syncwarp();
  dev::warp_inv_zfp(q, nd, lane);
  // 1 / 2^k, exactly as the division of 1 by pow2(k) rounds (0 once 2^k overflows)
  const int k = 63 - nd - 1 - emax;
  const double scale = k > 1023 ? 0.0 : dev::pow2(-k);
  int hx, hy, hz;
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
  const int dx = 17 - hx, dy = 17 - hy;
  double* base = F + sbm_base(hx, hy, hz, is2d);
  for (int j = lane; j < nv; j += 32)
  {
    // block dims are 4 or 1 per axis
    const int x = bd[0] > 1 ? (j & 3) : 0;
    const int r = bd[0] > 1 ? j >> 2 : j;
    const int y = bd[1] > 1 ? (r & 3) : 0;
    const int z = bd[1] > 1 ? r >> 2 : r;
    base[((d3[2] + z) * dy + (d3[1] + y)) * dx + (d3[0] + x)] = __dmul_rn(scale, __ll2double_rn(q[j]));
  }
  __syncwarp();
}

// Per-block zfp scratch with one padding word after every 4 (conflict-free 4-point passes).
__device__ __forceinline__ int qpad(int i) { return i + (i >> 2); }

// One inverse zfp 4-point line (Core/Zfp.h:181 ILift) on the padded scratch: elements
// i, i + s, i + 2s, i + 3s of the block.
__device__ __forceinline__ void ilift4_padded(long long* q, int i, int s)
{
  dev::inv_lift4_at(q + qpad(i), q + qpad(i + s), q + qpad(i + 2 * s), q + qpad(i + 3 * s));
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

// ---------------------------------------------------------------------------
// Bit planes of one (brick, subband): the wavefront of the group-test decoder alone
// (Core/idx2Decode.cpp:141-202). Channel c = kmax - key is owned by lane c % 32 (G groups of
// 32 channels); at step t it decodes its plane of block t - c, taking the block's significance
// count from channel c - 1 at step t - 1. The plane masks of step t are stored as row t of the
// unit's table (row length nkeys): block b's plane in channel c is row b + c, column c.
// ---------------------------------------------------------------------------
constexpr int kPlaneWarps = 8;

struct plane_smem
{
  int16_t ktop[kPlaneWarps][2][kMaxBlocksPerSubband];  // [warp][unit of the warp][block]
  uint8_t np[kPlaneWarps][2][kMaxBlocksPerSubband];
  uint8_t nvl[kPlaneWarps][2][kMaxBlocksPerSubband];
};

template <int G, bool MULTI>
__device__ __forceinline__ void plane_wavefront(const dec1_args& a, size_t fs, int nb, int nkeys, int kmax,
                                                const int16_t* ktop, const uint8_t* npl, const uint8_t* nvl,
                                                unsigned long long* T, int lane)
{
  bit_reader rd[G];
  bool has[G];
  int n_out[G], stop_out[G];
  const int ck = a.ckmin[fs], cn = a.cn[fs];
  const unsigned long long cf = a.cfirst[fs];
#pragma unroll
  for (int g = 0; g < G; ++g)
  {
    const int c = 32 * g + lane, key = kmax - c;
    has[g] = false;
    n_out[g] = 0;
    stop_out[g] = 0;
    if (c < nkeys && key >= ck && key < ck + cn)
    {
      const unsigned long long o = a.coff[cf + (unsigned long long)(key - ck)];
      if (o != ~0ull)
      {
        rd[g].init(a.blob, a.blob_bytes, o * 8ull);
        has[g] = true;
      }
    }
  }
  const int steps = nb + nkeys - 1;
  for (int t = 0; t < steps; ++t)
  {
    int nl[G], sl[G];
#pragma unroll
    for (int g = 0; g < G; ++g)
    {
      nl[g] = __shfl_up_sync(0xffffffffu, n_out[g], 1);
      sl[g] = __shfl_up_sync(0xffffffffu, stop_out[g], 1);
      if (g > 0)
      {
        const int x = __shfl_sync(0xffffffffu, n_out[g - 1], 31);
        const int y = __shfl_sync(0xffffffffu, stop_out[g - 1], 31);
        if (lane == 0)
        {
          nl[g] = x;
          sl[g] = y;
        }
      }
    }
#pragma unroll
    for (int g = 0; g < G; ++g)
    {
      const int c = 32 * g + lane, b = t - c;
      unsigned long long X = 0;
      n_out[g] = 0;
      stop_out[g] = 0;
      if constexpr (!MULTI)
      {
        if (c < nkeys && b >= 0 && b < nb)
        {
          const int top = ktop[b], np = npl[b], key = kmax - c;
          if (np > 0 && key <= top && key > top - np)
          {
            int n = key == top ? 0 : nl[g];
            const int stopped = key == top ? 0 : sl[g];
            if (stopped || !has[g])
            {
              stop_out[g] = 1;
              n_out[g] = n;
            }
            else
            {
              X = decode_plane(rd[g], n, 1 << nvl[b]);
              n_out[g] = n;
            }
          }
        }
        if (c < nkeys)
          T[(size_t)t * (size_t)nkeys + (size_t)c] = X;
      }
      else if (c < nkeys)
      {
        // several planes per key: the block's planes of this key, top-down, from the same
        // stream; slot j of the (step, channel) entry holds key value key * bpc + bpc - 1 - j
        unsigned long long* row = T + ((size_t)t * (size_t)nkeys + (size_t)c) * (size_t)a.bpc;
        for (int j = 0; j < a.bpc; ++j)
          row[j] = 0ull;
        if (b >= 0 && b < nb && npl[b] > 0)
        {
          const int top = ktop[b], key = kmax - c;
          int kk0, kk1;
          dev::key_planes(top, npl[b], key, a.bpc, kk0, kk1);
          if (kk0 <= kk1)
          {
            int n = kk0 == 0 ? 0 : nl[g];
            const int stopped = kk0 == 0 ? 0 : sl[g];
            if (stopped || !has[g])
              stop_out[g] = 1;
            else
              for (int kk = kk0; kk <= kk1; ++kk)
                row[key * a.bpc + a.bpc - 1 - (top - kk)] = decode_plane(rd[g], n, 1 << nvl[b]);
            n_out[g] = n;
          }
        }
      }
    }
  }
}

// WIDE = false: every unit, those of up to 32 channels decoded at once (few registers, many
// warps per SM), the others listed; WIDE = true: the listed units (up to kKeyWindow channels).
// A (brick, subband) unit of the plane kernel after its preparation: block tables filled,
// channel window known, table allocated. run = 0: nothing to decode here (skipped, empty,
// deferred to the second pass, or no room).
struct plane_unit
{
  int run, nb, nkeys, kmax;
  size_t fs;
  unsigned long long* T;
};

template <bool WIDE, bool MULTI>
__device__ __forceinline__ plane_unit prep_unit(const dec1_args& a, int unit, int16_t* ktop, uint8_t* npl,
                                                uint8_t* nvl, int lane)
{
  plane_unit u;
  u.run = 0;
  u.nb = u.nkeys = u.kmax = 0;
  u.fs = 0;
  u.T = nullptr;
  const int bi = unit / a.nsb, s = unit - bi * a.nsb;
  const decode_target& rq = a.reqs[a.bricks[bi].req];
  if (!((rq.mask >> s) & 1))
  {
    if (lane == 0)
      a.unit_off[unit] = ~0ull;
    return u;
  }
  const int nb = a.nblocks[s];
  const size_t fs = (size_t)a.bricks[bi].flat * (size_t)a.nsb + (size_t)s;
  int kmin = 1 << 30, kmax = -(1 << 30);
  for (int b = lane; b < nb; b += 32)
  {
    int d3[3], bd[3];
    unpack_geom(a.geom[(size_t)s * kMaxBlocksPerSubband + b], d3, bd);
    const int emax = a.exps[fs * kMaxBlocksPerSubband + (size_t)b];
    const int np = dev::coded_planes(emax, rq.etol, a.end_bp, a.bpc);
    const int top = emax + 63 + 1024;
    ktop[b] = (int16_t)top;
    npl[b] = (uint8_t)np;
    nvl[b] = (uint8_t)(2 * ((bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1)));
    if (np)
    {
      if (top - np + 1 < 0)
        atomicOr(a.error, 1);  // negative key value: a tolerance below 2^-1070 (unsupported)
      const int kh = dev::plane_key(top, 0, a.bpc), kl = dev::plane_key(top, np - 1, a.bpc);
      kmax = kh > kmax ? kh : kmax;
      kmin = kl < kmin ? kl : kmin;
    }
  }
  for (int o = 16; o > 0; o >>= 1)
  {
    const int x = __shfl_xor_sync(0xffffffffu, kmax, o), y = __shfl_xor_sync(0xffffffffu, kmin, o);
    kmax = x > kmax ? x : kmax;
    kmin = y < kmin ? y : kmin;
  }
  __syncwarp();
  int nkeys = kmax >= kmin ? kmax - kmin + 1 : 0;
  if (nkeys > (MULTI ? 64 : kKeyWindow))
  {
    if (lane == 0)
      atomicOr(a.error, 1);
    nkeys = 0;
  }
  if (nkeys == 0)
  {
    if (lane == 0)
      a.unit_off[unit] = ~0ull;
    return u;
  }
  if (!WIDE && nkeys > 32)
  {
    if (lane == 0)
      a.wide_list[atomicAdd(a.wide_count, 1)] = unit;
    return u;
  }
  const unsigned long long bytes =
    (unsigned long long)(nb + nkeys - 1) * (unsigned long long)nkeys * 8ull * (unsigned long long)a.bpc;
  unsigned long long base = 0;
  if (lane == 0)
    base = atomicAdd(a.cursor, bytes);
  base = __shfl_sync(0xffffffffu, base, 0);
  if (base + bytes > a.cap_bytes)
  {
    if (lane == 0)
    {
      atomicOr(a.error, 2);
      a.unit_off[unit] = ~0ull;
    }
    return u;
  }
  if (lane == 0)
    a.unit_off[unit] = base;
  u.run = 1;
  u.nb = nb;
  u.nkeys = nkeys;
  u.kmax = kmax;
  u.fs = fs;
  u.T = a.planes + base / 8;
  return u;
}

// Two units of at most 16 channels in one warp, lanes 0-15 the first, 16-31 the second: the
// wavefront of plane_wavefront<1, false> with each half on its own unit. A half's lane 0 owns
// its unit's top key, where every block starts with no significant coefficient, so the
// significance count shuffled across the halves is never used.
__device__ __forceinline__ void plane_wavefront_pair(const dec1_args& a, const plane_unit& A, const plane_unit& B,
                                                     const int16_t* ktopA, const uint8_t* nplA, const uint8_t* nvlA,
                                                     const int16_t* ktopB, const uint8_t* nplB, const uint8_t* nvlB,
                                                     int lane)
{
  const int h = lane >> 4, c = lane & 15;
  const plane_unit& U = h ? B : A;
  const int16_t* ktop = h ? ktopB : ktopA;
  const uint8_t* npl = h ? nplB : nplA;
  const uint8_t* nvl = h ? nvlB : nvlA;
  const int nkeys = U.nkeys, nb = U.nb, kmax = U.kmax, key = kmax - c;
  bit_reader rd;
  bool has = false;
  if (c < nkeys)
  {
    const int ck = a.ckmin[U.fs], cn = a.cn[U.fs];
    if (key >= ck && key < ck + cn)
    {
      const unsigned long long o = a.coff[a.cfirst[U.fs] + (unsigned long long)(key - ck)];
      if (o != ~0ull)
      {
        rd.init(a.blob, a.blob_bytes, o * 8ull);
        has = true;
      }
    }
  }
  const int my_steps = nb + nkeys - 1;
  const int sA = A.nb + A.nkeys - 1, sB = B.nb + B.nkeys - 1;
  const int steps = sA > sB ? sA : sB;
  int n_out = 0, stop_out = 0;
  for (int t = 0; t < steps; ++t)
  {
    int nl = __shfl_up_sync(0xffffffffu, n_out, 1);
    int sl = __shfl_up_sync(0xffffffffu, stop_out, 1);
    if (c == 0)
    {
      nl = 0;
      sl = 0;
    }
    const int b = t - c;
    unsigned long long X = 0;
    n_out = 0;
    stop_out = 0;
    if (c < nkeys && b >= 0 && b < nb)
    {
      const int top = ktop[b], np = npl[b];
      if (np > 0 && key <= top && key > top - np)
      {
        int n = key == top ? 0 : nl;
        const int stopped = key == top ? 0 : sl;
        if (stopped || !has)
        {
          stop_out = 1;
          n_out = n;
        }
        else
        {
          X = decode_plane(rd, n, 1 << nvl[b]);
          n_out = n;
        }
      }
    }
    if (c < nkeys && t < my_steps)
      U.T[(size_t)t * (size_t)nkeys + (size_t)c] = X;
  }
}

template <bool WIDE, bool MULTI = false>
__global__ void __launch_bounds__(kPlaneWarps * 32, WIDE ? 2 : (MULTI ? 6 : 4)) k_decode_planes(const dec1_args a)
{
  __shared__ plane_smem sm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ufirst = WIDE ? 0 : a.unit_first;
  const int nunits = WIDE ? *a.wide_count : a.unit_last;
  if constexpr (!WIDE && !MULTI)
  {
    // two consecutive units per warp; a pair of units of up to 16 channels shares the warp
    for (int i = ufirst + 2 * (blockIdx.x * kPlaneWarps + warp); i < nunits; i += 2 * gridDim.x * kPlaneWarps)
    {
      const plane_unit A = prep_unit<false, false>(a, i, sm.ktop[warp][0], sm.np[warp][0], sm.nvl[warp][0], lane);
      plane_unit B;
      B.run = 0;
      B.nb = B.nkeys = B.kmax = 0;
      B.fs = 0;
      B.T = nullptr;
      if (i + 1 < nunits)
        B = prep_unit<false, false>(a, i + 1, sm.ktop[warp][1], sm.np[warp][1], sm.nvl[warp][1], lane);
      __syncwarp();
      if (A.run && B.run && A.nkeys <= 16 && B.nkeys <= 16)
        plane_wavefront_pair(a, A, B, sm.ktop[warp][0], sm.np[warp][0], sm.nvl[warp][0], sm.ktop[warp][1],
                             sm.np[warp][1], sm.nvl[warp][1], lane);
      else
      {
        if (A.run)
          plane_wavefront<1, false>(a, A.fs, A.nb, A.nkeys, A.kmax, sm.ktop[warp][0], sm.np[warp][0],
                                    sm.nvl[warp][0], A.T, lane);
        if (B.run)
          plane_wavefront<1, false>(a, B.fs, B.nb, B.nkeys, B.kmax, sm.ktop[warp][1], sm.np[warp][1],
                                    sm.nvl[warp][1], B.T, lane);
      }
      __syncwarp();
    }
    return;
  }
  for (int i = ufirst + blockIdx.x * kPlaneWarps + warp; i < nunits; i += gridDim.x * kPlaneWarps)
  {
    const int unit = WIDE ? a.wide_list[i] : i;
    int16_t* ktop = sm.ktop[warp][0];
    uint8_t* npl = sm.np[warp][0];
    uint8_t* nvl = sm.nvl[warp][0];
    const plane_unit U = prep_unit<WIDE, MULTI>(a, unit, ktop, npl, nvl, lane);
    if (!U.run)
      continue;
    const size_t fs = U.fs;
    const int nb = U.nb, nkeys = U.nkeys, kmax = U.kmax;
    unsigned long long* T = U.T;
    if constexpr (MULTI)
    {
      // several planes per key: units of up to 32 keys here, up to 64 in the second pass
      if (!WIDE)
        plane_wavefront<1, true>(a, fs, nb, nkeys, kmax, ktop, npl, nvl, T, lane);
      else
        plane_wavefront<2, true>(a, fs, nb, nkeys, kmax, ktop, npl, nvl, T, lane);
    }
    else if (!WIDE)
      plane_wavefront<1, false>(a, fs, nb, nkeys, kmax, ktop, npl, nvl, T, lane);
    else if (nkeys <= 32)
      plane_wavefront<1, false>(a, fs, nb, nkeys, kmax, ktop, npl, nvl, T, lane);
    else if (nkeys <= 64)
      plane_wavefront<2, false>(a, fs, nb, nkeys, kmax, ktop, npl, nvl, T, lane);
    else if (nkeys <= 96)
      plane_wavefront<3, false>(a, fs, nb, nkeys, kmax, ktop, npl, nvl, T, lane);
    else
      plane_wavefront<4, false>(a, fs, nb, nkeys, kmax, ktop, npl, nvl, T, lane);
    __syncwarp();
  }
}

// One inverse line over two dense streams (even samples at c0, odd at c1, compile-time stride
// ST), with the de-normalisation weights of the two streams applied as they are loaded.
template <int ST>
__device__ __forceinline__ void ilift_streams(double* c0, double* c1, bool n0, double w0, bool n1, double w1)
{
  double v[33];
#pragma unroll
  for (int k = 0; k < 33; ++k)
  {
    const double f = (k & 1) ? c1[(k >> 1) * ST] : c0[(k >> 1) * ST];
    v[k] = (k & 1) ? (n1 ? __dmul_rn(f, w1) : f) : (n0 ? __dmul_rn(f, w0) : f);
  }
  ilift33(v);
#pragma unroll
  for (int k = 0; k < 33; ++k)
    ((k & 1) ? c1 : c0)[(k >> 1) * ST] = v[k];
}

template <int CPS>
__global__ void __launch_bounds__(kThreads, CPS) k_decode_level(const dec_args a)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  dec_smem& sm = *reinterpret_cast<dec_smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N[3] = { 33, 33, a.is2d ? 1 : 33 };
  const int NB = N[0] * N[1] * N[2];
  DEC_PHASE_INIT
  if (tid < 64)
    sm.perm3[tid] = dev::perm(3, tid);
  if (tid < 16)
    sm.perm2[tid] = dev::perm(2, tid);

  for (int bi = blockIdx.x; bi < a.nbricks; bi += gridDim.x)
  {
    const decode_brick& br = a.bricks[bi];
    DEC_PHASE_START
    {
      // the request's parameters to shared memory (read often, and across barriers)
      static_assert(sizeof(decode_target) % 4 == 0, "decode_target is copied as words");
      const uint32_t* src = reinterpret_cast<const uint32_t*>(a.reqs + br.req);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sm.rq);
      for (int i = tid; i < (int)(sizeof(decode_target) / 4); i += kThreads)
        dst[i] = src[i];
    }
    if (tid == 0)
      sm.sig = 0;
    __syncthreads();
    const decode_target& rq = sm.rq;
    double* F = rq.is_output ? a.slots + (size_t)blockIdx.x * (size_t)NB
                             : a.bricks_out + (size_t)br.store * (size_t)NB;
    // 1: zero + parent low band (Core/idx2Decode.cpp:285-293)
    if (!a.coeff_out)
      for (int i = tid; i < NB; i += kThreads)
        F[i] = 0.0;
    __syncthreads();
    if (!a.coeff_out && br.parent >= 0 && a.parents && (rq.mask & 1))
    {
      const double* P = a.parents + (size_t)br.parent * (size_t)NB;
      const int nz = a.is2d ? 1 : 16;
      for (int i = tid; i < 16 * 16 * nz; i += kThreads)
      {
        int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        // even positions of the child: its subband 0, dense
        F[(z * 17 + y) * 17 + x] =
          P[sbm(br.pos[0] * 16 + x, br.pos[1] * 16 + y, br.pos[2] * nz + z, a.is2d)];
      }
    }

    DEC_PHASE(0)
    // 2: per-block state of every decoded subband
    for (int i = tid; i < a.nsb * kMaxBlocksPerSubband; i += kThreads)
    {
      const int s = i / kMaxBlocksPerSubband, b = i % kMaxBlocksPerSubband;
      if (!((rq.mask >> s) & 1) || b >= a.nblocks[s])
        continue;
      int d3[3], bd[3];
      unpack_geom(a.geom[(size_t)s * kMaxBlocksPerSubband + b], d3, bd);
      const size_t fs = (size_t)br.flat * (size_t)a.nsb + (size_t)s;
      const int emax = a.exps[fs * kMaxBlocksPerSubband + (size_t)b];
      sm.emax[s][b] = (int16_t)emax;
      sm.ktop[s][b] = (int16_t)(emax + 63 + 1024);
      const int np = dev::coded_planes(emax, rq.etol, a.end_bp, a.bpc);
      sm.np[s][b] = (uint8_t)np;
      // Core/idx2Decode.cpp:161-206: NBps counts the decoded planes within the tolerance; a
      // block with none is not rebuilt, and when more than 8 planes are decoded
      // (Exponent(tol) - 6 - EMax + 1 > 8) the planes go through TransposeRecursive
      // (Core/Zfp.h:1140), which reads plane rows below NBps rounded up to even only. With one
      // plane per key every decoded plane is within the tolerance.
      int nuse = np;
      if (a.bpc > 1)
      {
        const int np1 = dev::coded_planes(emax, rq.etol, a.end_bp);
        const int nbps = np1 < np ? np1 : np;
        if (nbps == 0)
          nuse = 0;
        else if (rq.etol - 6 - emax + 1 > 8)
        {
          const int r = (nbps + 1) & ~1;
          nuse = r < np ? r : np;
        }
      }
      sm.nuse[s][b] = (uint8_t)nuse;
      sm.nbps[s][b] = 0;
      sm.nd[s][b] = (uint8_t)((bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1));
      sm.bypass[s][b] = (uint8_t)((d3[0] % rq.spacing[s][0]) != 0 || (d3[1] % rq.spacing[s][1]) != 0 ||
                                  (d3[2] % rq.spacing[s][2]) != 0);
    }
    __syncthreads();
    if (tid < a.nsb)
    {
      const int s = tid;
      int kmax = -(1 << 30), kmin = 1 << 30;
      if ((rq.mask >> s) & 1)
        for (int b = 0; b < a.nblocks[s]; ++b)
        {
          if (!sm.np[s][b])
            continue;
          const int hi = dev::plane_key(sm.ktop[s][b], 0, a.bpc);
          const int lo = dev::plane_key(sm.ktop[s][b], sm.np[s][b] - 1, a.bpc);
          kmax = hi > kmax ? hi : kmax;
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
    DEC_PHASE(1)

    if (a.planes)
    {
      // 3: blocks rebuilt from the decoded planes (k_decode_planes), a warp per block
      for (int s = 0; s < a.nsb; ++s)
      {
        if (!((rq.mask >> s) & 1) || sm.nkeys[s] == 0)
          continue;
        const unsigned long long uo = a.unit_off[(size_t)bi * (size_t)a.nsb + (size_t)s];
        if (uo == ~0ull)
          continue;
        const unsigned long long* T = a.planes + uo / 8;
        const int nb = a.nblocks[s], nkeys = sm.nkeys[s], kmax = sm.kmax[s];
        const uint64_t* geom = a.geom + (size_t)s * kMaxBlocksPerSubband;
        int hx, hy, hz;
        if (a.is2d)
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
        const int dx = 17 - hx, dy = 17 - hy;
        double* const sbase = F + sbm_base(hx, hy, hz, a.is2d);
        // plane k of block b (bit plane 63 - k) is in channel c0 + k, table row b + c0 + k;
        // blocks with nothing to decode (no planes, or not part of the request) stay zero
        auto load_planes = [&](int b, unsigned long long& x0, unsigned long long& x1) {
          x0 = 0;
          x1 = 0;
          if (b >= nb)
            return;
          const int np = sm.nuse[s][b];
          if (!np || sm.bypass[s][b])
            return;
          const int top = sm.ktop[s][b], bpc = a.bpc;
          if (bpc == 1)
          {
            // plane kk in channel c0 + kk, table row b + c0 + kk
            const int c0 = kmax - top;
            if (lane < np && c0 + lane < nkeys)
              x0 = T[(size_t)(b + c0 + lane) * (size_t)nkeys + (size_t)(c0 + lane)];
            if (lane + 32 < np && c0 + lane + 32 < nkeys)
              x1 = T[(size_t)(b + c0 + lane + 32) * (size_t)nkeys + (size_t)(c0 + lane + 32)];
            return;
          }
          // plane kk: channel c = kmax - key, step b + c, slot key * bpc + bpc - 1 - (top - kk)
          auto at = [&](int kk) -> unsigned long long {
            const int key = dev::plane_key(top, kk, bpc), c = kmax - key;
            if (c >= nkeys)
              return 0ull;
            return T[((size_t)(b + c) * (size_t)nkeys + (size_t)c) * (size_t)bpc +
                     (size_t)(key * bpc + bpc - 1 - (top - kk))];
          };
          if (lane < np)
            x0 = at(lane);
          if (lane + 32 < np)
            x1 = at(lane + 32);
        };
        // coefficient bit vectors from plane masks: lane l gets bit l (u0) and bit l + 32 (u1)
        // of every plane, plane k at bit 63 - k
        auto transpose = [&](unsigned long long x0, unsigned long long x1, bool two,
                             unsigned long long& u0, unsigned long long& u1) {
          u0 = (unsigned long long)__brev(dev::warp_transpose32((uint32_t)x0, lane)) << 32;
          u1 = (unsigned long long)__brev(dev::warp_transpose32((uint32_t)(x0 >> 32), lane)) << 32;
          if (two)
          {
            u0 |= __brev(dev::warp_transpose32((uint32_t)x1, lane));
            u1 |= __brev(dev::warp_transpose32((uint32_t)(x1 >> 32), lane));
          }
        };
        const int npairs = (nb + 1) >> 1;
        unsigned long long cA0 = 0, cA1 = 0, cB0 = 0, cB1 = 0;
        if (warp < npairs)
        {
          load_planes(2 * warp, cA0, cA1);
          load_planes(2 * warp + 1, cB0, cB1);
        }
        for (int pr = warp; pr < npairs; pr += kWarps)
        {
          // the next pair's plane masks are loaded while this pair is rebuilt
          unsigned long long nA0 = 0, nA1 = 0, nB0 = 0, nB1 = 0;
          if (pr + kWarps < npairs)
          {
            load_planes(2 * (pr + kWarps), nA0, nA1);
            load_planes(2 * (pr + kWarps) + 1, nB0, nB1);
          }
          const int bA = 2 * pr, bB = 2 * pr + 1;
          const bool hasB = bB < nb;
          const bool actA = sm.nuse[s][bA] > 0 && !sm.bypass[s][bA];
          const bool actB = hasB && sm.nuse[s][bB] > 0 && !sm.bypass[s][bB];
          const int npA = sm.nuse[s][bA], npB = hasB ? sm.nuse[s][bB] : 0;
          // Core/idx2Decode.cpp:209-211: a decoded block of a subband > 0, or of the coarsest
          // level, makes the brick significant
          if (a.sig && lane == 0 && (actA || actB) && (s > 0 || a.level + 1 == a.nlevels))
            sm.sig = 1;
          unsigned long long uA0, uA1, uB0, uB1;
          transpose(cA0, cA1, npA > 32, uA0, uA1);
          transpose(cB0, cB1, npB > 32, uB0, uB1);
          const int ndA = sm.nd[s][bA], ndB = hasB ? sm.nd[s][bB] : 0;
          const int nvA = actA ? 1 << (2 * ndA) : 0, nvB = actB ? 1 << (2 * ndB) : 0;
          long long* qA = sm.q[warp][0];
          long long* qB = sm.q[warp][1];
          auto permj = [&](int nd, int j) -> int {
            return nd == 3 ? (int)sm.perm3[j] : (nd == 2 ? (int)sm.perm2[j & 15] : j);
          };
          // inverse shuffle (Core/Zfp.h:520 InverseShuffle): negabinary to two's complement
          if (lane < nvA)
            qA[qpad(permj(ndA, lane))] = (long long)((uA0 ^ dev::kNegaMask) - dev::kNegaMask);
          if (lane + 32 < nvA)
            qA[qpad(permj(ndA, lane + 32))] = (long long)((uA1 ^ dev::kNegaMask) - dev::kNegaMask);
          if (lane < nvB)
            qB[qpad(permj(ndB, lane))] = (long long)((uB0 ^ dev::kNegaMask) - dev::kNegaMask);
          if (lane + 32 < nvB)
            qB[qpad(permj(ndB, lane + 32))] = (long long)((uB1 ^ dev::kNegaMask) - dev::kNegaMask);
          __syncwarp();
          if (a.coeff_out)
          {
            // coefficient mode: q * 2^(EMax - Prec + 1) at the samples' positions, no inverse zfp
            auto put = [&](int b, long long* q, int nd, int nv) {
              int d3[3], bd[3];
              unpack_geom(geom[b], d3, bd);
              const int kk = 63 - nd - 1 - sm.emax[s][b];
              const double scale = kk > 1023 ? 0.0 : dev::pow2(-kk);
              const size_t cb = (size_t)br.store * (size_t)NB;
              for (int j = lane; j < nv; j += 32)
              {
                const int x = bd[0] > 1 ? (j & 3) : 0;
                const int r = bd[0] > 1 ? j >> 2 : j;
                const int y = bd[1] > 1 ? (r & 3) : 0;
                const int z = bd[1] > 1 ? r >> 2 : r;
                const int px = hx + 2 * (d3[0] + x), py = hy + 2 * (d3[1] + y), pz = hz + 2 * (d3[2] + z);
                const size_t at = cb + (size_t)((pz * 33 + py) * 33 + px);
                const double v = __dmul_rn(scale, __ll2double_rn(q[qpad(j)]));
                if (a.out_f32)
                  ((float*)a.coeff_out)[at] = (float)v;
                else
                  ((double*)a.coeff_out)[at] = v;
              }
            };
            if (actA)
              put(bA, qA, ndA, nvA);
            if (actB)
              put(bB, qB, ndB, nvB);
            __syncwarp();
            cA0 = nA0;
            cA1 = nA1;
            cB0 = nB0;
            cB1 = nB1;
            continue;
          }
          // inverse zfp (Core/Zfp.h:287): block A on lanes 0-15, block B on lanes 16-31
          {
            const int h = lane >> 4, l = lane & 15;
            const unsigned hm = h ? 0xffff0000u : 0x0000ffffu;
            long long* q = h ? qB : qA;
            const int nd = h ? (actB ? ndB : 0) : (actA ? ndA : 0);
            if (nd == 3)
            {
              ilift4_padded(q, (l & 3) + 4 * (l >> 2), 16);
              __syncwarp(hm);
              ilift4_padded(q, 16 * (l & 3) + (l >> 2), 4);
              __syncwarp(hm);
              ilift4_padded(q, 4 * (l & 3) + 16 * (l >> 2), 1);
            }
            else if (nd == 2)
            {
              if (l < 4)
                ilift4_padded(q, l, 4);
              __syncwarp(hm);
              if (l < 4)
                ilift4_padded(q, 4 * l, 1);
            }
            else if (nd == 1)
            {
              if (l == 0)
                ilift4_padded(q, 0, 1);
            }
            __syncwarp();
          }
          // dequantise (Core/Zfp.h Dequantize) and store into the subband
          auto store_block = [&](int b, long long* q, int nd, int nv) {
            int d3[3], bd[3];
            unpack_geom(geom[b], d3, bd);
            const int k = 63 - nd - 1 - sm.emax[s][b];
            const double scale = k > 1023 ? 0.0 : dev::pow2(-k);
            for (int j = lane; j < nv; j += 32)
            {
              const int x = bd[0] > 1 ? (j & 3) : 0;
              const int r = bd[0] > 1 ? j >> 2 : j;
              const int y = bd[1] > 1 ? (r & 3) : 0;
              const int z = bd[1] > 1 ? r >> 2 : r;
              sbase[((d3[2] + z) * dy + (d3[1] + y)) * dx + (d3[0] + x)] =
                __dmul_rn(scale, __ll2double_rn(q[qpad(j)]));
            }
          };
          if (actA)
            store_block(bA, qA, ndA, nvA);
          if (actB)
            store_block(bB, qB, ndB, nvB);
          __syncwarp();
          cA0 = nA0;
          cA1 = nA1;
          cB0 = nB0;
          cB1 = nB1;
        }
      }
    }
    else if (!sm.wide)
    {
      // 3a: warp w decodes subband w. Lane j owns channel (kmax - j); at step t it decodes
      // that plane of block t - j, taking the block's significance count from lane j - 1 of
      // step t - 1. Block t - (nkeys - 1) is complete after step t and is rebuilt at once.
      const int s = warp;
      if (s < a.nsb && ((rq.mask >> s) & 1) && sm.nkeys[s] > 0)
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
            reconstruct_block(F, sm.q[warp][0], sm.perm3, sm.perm2, u0, u1, sm.nd[s][bc], sm.emax[s][bc],
                              geom[bc], s, a.is2d, lane);
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
        if (!((rq.mask >> s) & 1))
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
          reconstruct_block(F, sm.q[warp][0], sm.perm3, sm.perm2, sm.u.coef[b][lane], sm.u.coef[b][lane + 32],
                            sm.nd[s][b], sm.emax[s][b], geom[b], s, a.is2d, lane);
        }
        __syncthreads();
      }
    }
    __syncthreads();
    DEC_PHASE(2)
    if (a.sig && tid == 0 && br.store >= 0)
      a.sig[br.store] = sm.sig;

    if (a.coeff_out)
      continue;
    // 4: de-normalise + inverse CDF5/3 Z, Y, X (Core/Wavelet.cpp:144-203); the
    // de-normalisation is applied as the Z lines are loaded, the output crop and cast as the
    // X lines are stored.
    if (!a.is2d)
    {
      for (int li = tid; li < 33 * 33; li += kThreads)
      {
        const int x = li % 33, y = li / 33;
        // even and odd z samples of the column: two dense streams of stride dx * dy
        const int hx = x & 1, hy = y & 1, dx = 17 - hx, dy = 17 - hy;
        const int off = (y >> 1) * dx + (x >> 1), sz = dx * dy;
        double* c0 = F + sbm_base(hx, hy, 0, 0) + off;
        double* c1 = F + sbm_base(hx, hy, 1, 0) + off;
        const int s0 = (hx << 2) | (hy << 1), s1 = s0 | 1;
        const bool n0 = (a.norm_mask >> s0) & 1, n1 = (a.norm_mask >> s1) & 1;
        const double w0 = a.inv_weight[s0], w1 = a.inv_weight[s1];
        if (sz == 17 * 17)
          ilift_streams<17 * 17>(c0, c1, n0, w0, n1, w1);
        else if (sz == 16 * 17)
          ilift_streams<16 * 17>(c0, c1, n0, w0, n1, w1);
        else
          ilift_streams<16 * 16>(c0, c1, n0, w0, n1, w1);
      }
      __syncthreads();
      DEC_PHASE(3)
    }
    for (int li = tid; li < 33 * N[2]; li += kThreads)
    {
      const int x = li % 33, z = li / 33;
      // even and odd y samples of the line: two dense streams of stride dx
      const int hx = x & 1, hz = z & 1, dx = 17 - hx;
      double* c0 = F + sbm_base(hx, 0, hz, a.is2d) + (z >> 1) * dx * 17 + (x >> 1);
      double* c1 = F + sbm_base(hx, 1, hz, a.is2d) + (z >> 1) * dx * 16 + (x >> 1);
      const int s0 = a.is2d ? (hx << 1) : ((hx << 2) | hz), s1 = a.is2d ? (s0 | 1) : (s0 | 2);
      const bool n0 = a.is2d && ((a.norm_mask >> s0) & 1), n1 = a.is2d && ((a.norm_mask >> s1) & 1);
      const double w0 = a.inv_weight[s0], w1 = a.inv_weight[s1];
      if (dx == 17)
        ilift_streams<17>(c0, c1, n0, w0, n1, w1);
      else
        ilift_streams<16>(c0, c1, n0, w0, n1, w1);
    }
    __syncthreads();
    DEC_PHASE(4)
    // X, warp-uniform iterations (the output rows are staged per warp and written back
    // row by row, lanes along x)
    for (int li0 = warp * 32; li0 < 33 * N[2]; li0 += kThreads)
    {
      const int li = li0 + lane;
      const bool active = li < 33 * N[2];
      const int y = li % 33, z = li / 33;
      // 5: output (Core/idx2Decode.cpp:431-442 CopyGridGrid): where this row goes, decided
      // before the row is loaded (fewer live registers around the lift)
      long long obase = -1;
      if (rq.is_output && active)
      {
        const int ry = y - br.src_from[1], rz = z - br.src_from[2];
        if (ry >= 0 && rz >= 0 && ry % br.src_strd[1] == 0 && rz % br.src_strd[2] == 0 &&
            ry / br.src_strd[1] < br.dims[1] && rz / br.src_strd[2] < br.dims[2])
        {
          const long long oy = br.dst_from[1] + (long long)(ry / br.src_strd[1]) * br.dst_strd[1];
          const long long oz = br.dst_from[2] + (long long)(rz / br.src_strd[2]) * br.dst_strd[2];
          obase = (oz * rq.out_dims[1] + oy) * rq.out_dims[0] + br.dst_from[0];
        }
      }
      if (active && (!rq.is_output || obase >= 0))
      {
        // even and odd x samples of the row: two dense runs
        const int hy = y & 1, hz = z & 1, dy = 17 - hy;
        double* r0 = F + sbm_base(0, hy, hz, a.is2d) + ((z >> 1) * dy + (y >> 1)) * 17;
        double* r1 = F + sbm_base(1, hy, hz, a.is2d) + ((z >> 1) * dy + (y >> 1)) * 16;
        double v[33];
#pragma unroll
        for (int x = 0; x < 33; ++x)
          v[x] = (x & 1) ? r1[x >> 1] : r0[x >> 1];
        ilift33(v);
#pragma unroll
        for (int x = 0; x < 33; ++x)
        {
          if (!rq.is_output)
            ((x & 1) ? r1 : r0)[x >> 1] = v[x];
          else if (a.out_f32)
            sm.u.v32[warp][lane][x] = __double2float_rn(v[x]);
          else
            sm.u.v[warp][lane][x] = v[x];
        }
      }
      if (rq.is_output)
      {
        // the warp's rows, lanes along x
        sm.out_base[warp][lane] = obase;
        __syncwarp();
        const int n0 = br.dims[0];
        for (int r = 0; r < 32; ++r)
        {
          const long long ob = sm.out_base[warp][r];
          if (ob < 0 || lane >= n0)
            continue;
          const long long di = ob + (long long)lane * br.dst_strd[0];
          const int sx = br.src_from[0] + lane * br.src_strd[0];
          if (a.out_f32)
            ((float*)rq.out)[di] = sm.u.v32[warp][r][sx];
          else
            ((double*)rq.out)[di] = sm.u.v[warp][r][sx];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    DEC_PHASE(5)
  }
  DEC_PHASE_FLUSH
}
