// Decode kernels for sm_100a (Core/idx2Decode.cpp:86-320, :431-442).
//
// One persistent CTA per brick slot. For every brick of a level:
//   1  zero the FP64 brick, copy the parent's reconstructed low band into it,
//   2  per decoded subband: read the block exponents, then decode the bit planes as
//      a wavefront: thread j owns bit-plane channel (kmax - j) and its bit cursor;
//      at step t it decodes plane (kmax - j) of block t - j, receiving the block's
//      significance count from thread j - 1 of the previous step.  The channel
//      streams are consumed strictly in the reference's order (blocks in Morton
//      order within a channel, planes top-down within a block).
//   3  inverse shuffle / inverse zfp / dequantise per block (warp per block),
//   4  de-normalise and inverse CDF5/3 (Z, Y, X) in FP64,
//   5  keep the brick for the next level, or crop + cast it into the output grid.
#include "codec_device.cuh"
#include "decode_device.h"

#include <cstring>
#include <mutex>

namespace idx2g
{

namespace
{

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

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
  unsigned long long coef[kMaxBlocksPerSubband][64];
  long long q[kWarps][64];
  int16_t emax[kMaxBlocksPerSubband];
  int16_t ktop[kMaxBlocksPerSubband];
  uint8_t np[kMaxBlocksPerSubband];
  uint8_t nbps[kMaxBlocksPerSubband];
  uint8_t nd[kMaxBlocksPerSubband];
  uint8_t bypass[kMaxBlocksPerSubband];
  uint8_t nst[2][kKeyWindow];
  uint8_t stop[2][kKeyWindow];
  int kmax_w, nkeys;
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

// Read n <= 64 bits at bit position pos of the blob (LSB-first); bits past the end read 0.
__device__ __forceinline__ unsigned long long read_bits(const uint8_t* blob, unsigned long long nbytes,
                                                        unsigned long long pos, int n)
{
  if (n <= 0)
    return 0;
  unsigned long long v = 0;
  int got = 0;
  while (got < n)
  {
    unsigned long long byte = (pos + (unsigned long long)got) >> 3;
    int sh = (int)((pos + (unsigned long long)got) & 7);
    unsigned long long b = byte < nbytes ? (unsigned long long)(blob[byte] >> sh) : 0ull;
    int take = 8 - sh;
    if (take > n - got)
      take = n - got;
    b &= (1ull << take) - 1ull;
    v |= b << got;
    got += take;
  }
  return v;
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
    __syncthreads();

    // 2-3: subbands
    for (int s = 0; s < a.nsb; ++s)
    {
      if (!((a.mask >> s) & 1))
        continue;
      int from[3], dims[3], strd[3];
      subband_grid(a.is2d, s, from, dims, strd);
      const int nb = a.nblocks[s];
      const uint64_t* geom = a.geom + (size_t)s * kMaxBlocksPerSubband;
      const size_t fs = (size_t)br.flat * (size_t)a.nsb + (size_t)s;
      const int16_t* ex = a.exps + fs * kMaxBlocksPerSubband;
      for (int b = tid; b < nb; b += kThreads)
      {
        int d3[3], bd[3];
        unpack_geom(geom[b], d3, bd);
        const int emax = ex[b];
        sm.emax[b] = (int16_t)emax;
        sm.ktop[b] = (int16_t)(emax + 63 + 1024);
        sm.np[b] = (uint8_t)dev::coded_planes(emax, a.etol, a.end_bp);
        sm.nbps[b] = 0;
        sm.nd[b] = (uint8_t)((bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1));
        sm.bypass[b] = (uint8_t)((d3[0] % a.spacing[s][0]) != 0 || (d3[1] % a.spacing[s][1]) != 0 ||
                                 (d3[2] % a.spacing[s][2]) != 0);
      }
      for (int i = tid; i < nb * 64; i += kThreads)
        sm.coef[i >> 6][i & 63] = 0ull;
      __syncthreads();
      if (tid == 0)
      {
        int kmax = -(1 << 30), kmin = 1 << 30;
        for (int b = 0; b < nb; ++b)
        {
          if (!sm.np[b])
            continue;
          kmax = sm.ktop[b] > kmax ? sm.ktop[b] : kmax;
          int lo = sm.ktop[b] - sm.np[b] + 1;
          kmin = lo < kmin ? lo : kmin;
        }
        int nk = kmax >= kmin ? kmax - kmin + 1 : 0;
        if (nk > kKeyWindow)
        {
          atomicExch(a.error, 1);
          nk = 0;
        }
        sm.kmax_w = kmax;
        sm.nkeys = nk;
      }
      __syncthreads();
      const int nkeys = sm.nkeys, kmax = sm.kmax_w;
      // channel of thread j
      unsigned long long cur = ~0ull;
      int key = kmax - tid;
      if (tid < nkeys)
      {
        const int ck = a.ckmin[fs], cn = a.cn[fs];
        if (key >= ck && key < ck + cn)
        {
          unsigned long long o = a.coff[a.cfirst[fs] + (unsigned long long)(key - ck)];
          if (o != ~0ull)
            cur = o * 8ull;
        }
        sm.nst[0][tid] = 0;
        sm.stop[0][tid] = 0;
      }
      __syncthreads();
      // wavefront over (block, plane)
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
            const int top = sm.ktop[b], np = sm.np[b];
            if (np > 0 && key <= top && key > top - np)
            {
              int n = key == top ? 0 : sm.nst[rb][tid - 1];
              int stopped = key == top ? 0 : sm.stop[rb][tid - 1];
              if (stopped || cur == ~0ull)
              {
                out_stop = 1;
                out_n = (uint8_t)n;
              }
              else
              {
                // Core/Zfp.h:990 Decode<u64>
                const int nvals = 1 << (2 * sm.nd[b]);
                unsigned long long X = n > 0 ? read_bits(a.blob, a.blob_bytes, cur, n) : 0ull;
                cur += (unsigned long long)n;
                while (n < nvals)
                {
                  unsigned long long g = read_bits(a.blob, a.blob_bytes, cur, 1);
                  cur += 1;
                  if (!g)
                    break;
                  while (n + 1 < nvals)
                  {
                    unsigned long long bit = read_bits(a.blob, a.blob_bytes, cur, 1);
                    cur += 1;
                    if (bit)
                      break;
                    ++n;
                  }
                  X += 1ull << n;
                  ++n;
                }
                const int bp = 63 - (top - key);
                if (!sm.bypass[b])
                  for (unsigned long long y = X; y; y &= y - 1)
                  {
                    int i = __ffsll((long long)y) - 1;
                    sm.coef[b][i] += 1ull << bp;
                  }
                sm.nbps[b] += 1;
                out_n = (uint8_t)n;
              }
            }
          }
          sm.nst[wb][tid] = out_n;
          sm.stop[wb][tid] = out_stop;
        }
        __syncthreads();
      }
      // 3: reconstruct blocks (warp per block)
      for (int b = warp; b < nb; b += kWarps)
      {
        if (sm.nbps[b] == 0 || sm.bypass[b])
          continue;
        int d3[3], bd[3];
        unpack_geom(geom[b], d3, bd);
        const int nd = sm.nd[b];
        const int nv = 1 << (2 * nd);
        long long* q = sm.q[warp];
        for (int i = lane; i < nv; i += 32)
          q[dev::perm(nd, i)] = (long long)((sm.coef[b][i] ^ dev::kNegaMask) - dev::kNegaMask);
        __syncwarp();
        dev::warp_inv_zfp(q, nd, lane);
        const int prec = 63 - nd;
        const double scale = __ddiv_rn(1.0, dev::pow2(prec - 1 - sm.emax[b]));
        for (int j = lane; j < nv; j += 32)
        {
          int x = j % bd[0], y = (j / bd[0]) % bd[1], z = j / (bd[0] * bd[1]);
          F[((from[2] + (d3[2] + z) * strd[2]) * 33 + (from[1] + (d3[1] + y) * strd[1])) * 33 +
            (from[0] + (d3[0] + x) * strd[0])] = __dmul_rn(scale, __ll2double_rn(q[j]));
        }
        __syncwarp();
      }
      __syncthreads();
    }

    // 4: de-normalise + inverse CDF5/3 (Core/Wavelet.cpp:144-203)
    for (int s = 0; s < a.nsb; ++s)
    {
      if (!((a.norm_mask >> s) & 1))
        continue;
      int from[3], dims[3], strd[3];
      subband_grid(a.is2d, s, from, dims, strd);
      const double W = a.inv_weight[s];
      const int n = dims[0] * dims[1] * dims[2];
      for (int i = tid; i < n; i += kThreads)
      {
        int x = i % dims[0], y = (i / dims[0]) % dims[1], z = i / (dims[0] * dims[1]);
        int idx = ((from[2] + z * strd[2]) * 33 + (from[1] + y * strd[1])) * 33 + (from[0] + x * strd[0]);
        F[idx] = __dmul_rn(F[idx], W);
      }
    }
    __syncthreads();
    {
      dev::dgrid G;
      for (int k = 0; k < 3; ++k)
      {
        G.from[k] = 0;
        G.dims[k] = N[k];
        G.strd[k] = 1;
      }
      for (int ax = a.is2d ? 1 : 2; ax >= 0; --ax)
      {
        dev::lift_sweep(F, N, G, N, ax, false);
        __syncthreads();
      }
    }

    // 5: output (Core/idx2Decode.cpp:431-442 CopyGridGrid)
    if (a.is_output)
    {
      const int n = br.dims[0] * br.dims[1] * br.dims[2];
      for (int i = tid; i < n; i += kThreads)
      {
        int x = i % br.dims[0], y = (i / br.dims[0]) % br.dims[1], z = i / (br.dims[0] * br.dims[1]);
        int sx = br.src_from[0] + x * br.src_strd[0], sy = br.src_from[1] + y * br.src_strd[1],
            sz = br.src_from[2] + z * br.src_strd[2];
        long long dx = br.dst_from[0] + (long long)x * br.dst_strd[0],
                  dy = br.dst_from[1] + (long long)y * br.dst_strd[1],
                  dz = br.dst_from[2] + (long long)z * br.dst_strd[2];
        long long di = (dz * a.out_dims[1] + dy) * a.out_dims[0] + dx;
        double v = F[(sz * 33 + sy) * 33 + sx];
        if (a.out_f32)
          ((float*)a.out)[di] = __double2float_rn(v);
        else
          ((double*)a.out)[di] = v;
      }
    }
    __syncthreads();
  }
}

} // namespace

decode_device::~decode_device()
{
  cudaFree(exps_);
  cudaFree(kmin_);
  cudaFree(n_);
  cudaFree(first_);
  cudaFree(off_);
  cudaFree(blob_);
}

template <typename T>
static int up(T** dst, const std::vector<T>& v, cudaStream_t st, size_t pad = 0)
{
  size_t bytes = v.size() * sizeof(T);
  if (cudaMalloc((void**)dst, bytes + pad + 16) != cudaSuccess)
    return OutOfMemory;
  if (bytes)
    cudaMemcpyAsync(*dst, v.data(), bytes, cudaMemcpyHostToDevice, st);
  if (pad)
    cudaMemsetAsync((char*)*dst + bytes, 0, pad + 16, st);
  return NoError;
}

int decode_device::upload(device_ctx* ctx, const std::vector<int16_t>& exps, const std::vector<int32_t>& kmin,
                          const std::vector<int32_t>& n, const std::vector<uint64_t>& first,
                          const std::vector<uint64_t>& off, const std::vector<uint8_t>& blob)
{
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  int e = up(&exps_, exps, st);
  if (!e)
    e = up(&kmin_, kmin, st);
  if (!e)
    e = up(&n_, n, st);
  if (!e)
    e = up((uint64_t**)&first_, first, st);
  if (!e)
    e = up((uint64_t**)&off_, off, st);
  if (!e)
    e = up((uint8_t**)&blob_, blob, st, 16);
  if (e)
    return e;
  resident_ = exps.size() * 2 + kmin.size() * 4 + n.size() * 4 + first.size() * 8 + off.size() * 8 + blob.size();
  blob_bytes_ = blob.size();
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return CudaError;
  return NoError;
}

int decode_device::decode(device_ctx* ctx, const decode_request& rq, void* out, size_t out_bytes,
                          bool out_on_device, double* kernel_ms)
{
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int NB = 33 * 33 * (rq.is2d ? 1 : 33);
  auto cleanup = []() {};
  void* d_out = out;
  if (!out_on_device)
  {
    d_out = ctx->ws("dec.out", out_bytes);
    if (!d_out)
      return OutOfMemory;
  }
  cudaMemsetAsync(d_out, 0, out_bytes, st);
  int* d_err = (int*)ctx->ws("dec.err", 16);
  uint64_t* d_geom = (uint64_t*)ctx->ws("dec.geom", sizeof(uint64_t) * 8 * kMaxBlocksPerSubband);
  if (!d_err || !d_geom)
  {
    cleanup();
    return OutOfMemory;
  }
  cudaMemsetAsync(d_err, 0, 16, st);
  const size_t smem = sizeof(dec_smem);
  cudaFuncSetAttribute(k_decode_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaEvent_t e0 = ctx->ev0, e1 = ctx->ev1;
  float total_ms = 0;
  double* prev = nullptr;
  int li = 0;
  for (const decode_level& lv : rq.levels)
  {
    ++li;
    const int nbr = (int)lv.bricks.size();
    if (nbr == 0)
      continue;
    decode_brick* d_bricks = (decode_brick*)ctx->ws("dec.bricks", sizeof(decode_brick) * (size_t)nbr);
    double* d_level =
      lv.is_output ? nullptr : (double*)ctx->ws(li % 2 ? "dec.levA" : "dec.levB", (size_t)nbr * (size_t)NB * 8);
    int grid = nbr < 2 * ctx->num_sms ? nbr : 2 * ctx->num_sms;
    double* d_slots = lv.is_output ? (double*)ctx->ws("dec.slots", (size_t)grid * (size_t)NB * 8) : nullptr;
    if (!d_bricks || (!lv.is_output && !d_level) || (lv.is_output && !d_slots))
    {
      cleanup();
      return OutOfMemory;
    }
    cudaMemcpyAsync(d_bricks, lv.bricks.data(), sizeof(decode_brick) * (size_t)nbr, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_geom, lv.geom, sizeof(uint64_t) * 8 * kMaxBlocksPerSubband, cudaMemcpyHostToDevice, st);
    dec_args a;
    memset(&a, 0, sizeof a);
    a.level = lv.level;
    a.nlevels = rq.nlevels;
    a.is2d = rq.is2d;
    a.nsb = rq.nsb;
    a.nbricks = nbr;
    a.etol = rq.etol;
    a.end_bp = rq.f32 ? 32 : 64;
    a.mask = lv.mask;
    a.norm_mask = lv.norm_mask;
    a.is_output = lv.is_output;
    a.out_f32 = rq.f32;
    memcpy(a.spacing, lv.spacing, sizeof a.spacing);
    memcpy(a.nblocks, lv.nblocks, sizeof a.nblocks);
    memcpy(a.inv_weight, lv.inv_weight, sizeof a.inv_weight);
    a.geom = d_geom;
    a.bricks = d_bricks;
    a.exps = exps_;
    a.ckmin = kmin_;
    a.cn = n_;
    a.cfirst = first_;
    a.coff = off_;
    a.blob = blob_;
    a.blob_bytes = blob_bytes_;
    a.parents = prev;
    a.bricks_out = d_level;
    a.slots = d_slots;
    a.out = d_out;
    a.out_dims[0] = rq.out_dims.x;
    a.out_dims[1] = rq.out_dims.y;
    a.out_dims[2] = rq.out_dims.z;
    a.error = d_err;
    cudaEventRecord(e0, st);
    k_decode_level<<<grid, kThreads, smem, st>>>(a);
    cudaEventRecord(e1, st);
    if (cudaGetLastError() != cudaSuccess)
    {
      cleanup();
      return CudaError;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess)
    {
      cleanup();
      return CudaError;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    total_ms += ms;
    prev = d_level;
    if (lv.is_output)
      break;
  }
  int herr = 0;
  cudaMemcpyAsync(&herr, d_err, 4, cudaMemcpyDeviceToHost, st);
  if (!out_on_device)
    cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, st);
  cudaError_t ce = cudaStreamSynchronize(st);
  cleanup();
  if (ce != cudaSuccess)
    return CudaError;
  if (herr)
    return DeviceStreamOverflow;
  if (kernel_ms)
    *kernel_ms = total_ms;
  return NoError;
}


// ---------------------------------------------------------------------------
// Allocation-free decode (idx2g_decode_noalloc)
//
// For callers that cannot allocate device memory at decode time: applications whose device
// memory is owned by another allocator (a framework's caching allocator or a pool sized to
// the whole GPU) and latency-bound serving loops, where a cudaMalloc either fails or
// synchronises the device. Such a caller opens the dataset once beforehand (that step
// allocates the resident dataset) and then decodes into its own device buffer; every
// temporary of the decode lives in the fixed array below.
//
// The array is a file-scope __device__ variable: every GPU that loads this library holds its
// kNoAllocScratchBytes (about 7.3 MB) until the process exits. Limits: at most
// kNoAllocMaxBricks bricks on the output level and at most kNoAllocLevelBricks bricks on each
// coarser level a request decodes; larger requests are rejected with ScratchTooSmall.
// All calls share the array and it keeps the last call's contents: the error word is cleared
// at the start of every call, and calls that overlap on the GPU (on different streams or
// different contexts of the same device) race on it.
// ---------------------------------------------------------------------------

namespace
{

constexpr int kNoAllocSlots = 8;          // output-level brick slots (= CTAs of that launch)
constexpr int kNoAllocLevelBricks = 8;    // bricks of each coarser (non-output) level
constexpr int kNoAllocMaxBricks = 4096;   // bricks of the output level
constexpr size_t kBrickBytes = (size_t)33 * 33 * 33 * sizeof(double);
constexpr size_t kOffSlots = 0;
constexpr size_t kOffLevA = kOffSlots + (size_t)kNoAllocSlots * kBrickBytes;
constexpr size_t kOffLevB = kOffLevA + (size_t)kNoAllocLevelBricks * kBrickBytes;
constexpr size_t kOffBricks = kOffLevB + (size_t)kNoAllocLevelBricks * kBrickBytes;
constexpr size_t kOffGeom = kOffBricks + (((size_t)kNoAllocMaxBricks * sizeof(decode_brick) + 255) & ~(size_t)255);
constexpr size_t kOffErr = kOffGeom + sizeof(uint64_t) * 8 * kMaxBlocksPerSubband;
constexpr size_t kNoAllocScratchBytes = kOffErr + 256;

static __device__ __align__(256) unsigned char g_decode_scratch[kNoAllocScratchBytes];

// Device address of g_decode_scratch per device, resolved once per device by the first call
// on that device (with that device current). In host code the symbol is only a stand-in.
std::mutex g_scratch_mu;
void* g_scratch_addr[64] = {};

int scratch_address(int device, unsigned char** out)
{
  if (device < 0 || device >= 64)
    return InvalidArgument;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[device])
  {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_decode_scratch) != cudaSuccess || !p)
      return CudaError;
    g_scratch_addr[device] = p;
  }
  *out = (unsigned char*)g_scratch_addr[device];
  return NoError;
}

} // namespace

int decode_device::decode_noalloc(device_ctx* ctx, const decode_request& rq, void* d_out, size_t out_bytes,
                                  double* kernel_ms)
{
  // limits of the fixed scratch
  bool seen_output = false;
  for (const decode_level& lv : rq.levels)
  {
    if (seen_output)
      break;
    const size_t nbr = lv.bricks.size();
    if (lv.is_output)
    {
      seen_output = true;
      if (nbr > (size_t)kNoAllocMaxBricks)
        return ScratchTooSmall;
    }
    else if (nbr > (size_t)kNoAllocLevelBricks)
      return ScratchTooSmall;
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess)
    return CudaError;
  unsigned char* base = nullptr;
  int e = scratch_address(ctx->device, &base);
  if (e)
    return e;
  cudaStream_t st = ctx->stream;
  const int NB = 33 * 33 * (rq.is2d ? 1 : 33);
  double* slots = (double*)(base + kOffSlots);
  double* lev[2] = { (double*)(base + kOffLevA), (double*)(base + kOffLevB) };
  decode_brick* d_bricks = (decode_brick*)(base + kOffBricks);
  uint64_t* d_geom = (uint64_t*)(base + kOffGeom);
  int* d_err = (int*)(base + kOffErr);
  cudaMemsetAsync(d_out, 0, out_bytes, st);
  cudaMemsetAsync(d_err, 0, 16, st);
  const size_t smem = sizeof(dec_smem);
  cudaFuncSetAttribute(k_decode_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  float total_ms = 0;
  double* prev = nullptr;
  int li = 0;
  for (const decode_level& lv : rq.levels)
  {
    const int nbr = (int)lv.bricks.size();
    if (nbr == 0)
      continue;
    double* d_level = lv.is_output ? nullptr : lev[li % 2];
    ++li;
    int grid = lv.is_output ? (nbr < kNoAllocSlots ? nbr : kNoAllocSlots) : nbr;
    cudaMemcpyAsync(d_bricks, lv.bricks.data(), sizeof(decode_brick) * (size_t)nbr, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_geom, lv.geom, sizeof(uint64_t) * 8 * kMaxBlocksPerSubband, cudaMemcpyHostToDevice, st);
    dec_args a;
    memset(&a, 0, sizeof a);
    a.level = lv.level;
    a.nlevels = rq.nlevels;
    a.is2d = rq.is2d;
    a.nsb = rq.nsb;
    a.nbricks = nbr;
    a.etol = rq.etol;
    a.end_bp = rq.f32 ? 32 : 64;
    a.mask = lv.mask;
    a.norm_mask = lv.norm_mask;
    a.is_output = lv.is_output;
    a.out_f32 = rq.f32;
    memcpy(a.spacing, lv.spacing, sizeof a.spacing);
    memcpy(a.nblocks, lv.nblocks, sizeof a.nblocks);
    memcpy(a.inv_weight, lv.inv_weight, sizeof a.inv_weight);
    a.geom = d_geom;
    a.bricks = d_bricks;
    a.exps = exps_;
    a.ckmin = kmin_;
    a.cn = n_;
    a.cfirst = first_;
    a.coff = off_;
    a.blob = blob_;
    a.blob_bytes = blob_bytes_;
    a.parents = prev;
    a.bricks_out = d_level;
    a.slots = slots;
    a.out = d_out;
    a.out_dims[0] = rq.out_dims.x;
    a.out_dims[1] = rq.out_dims.y;
    a.out_dims[2] = rq.out_dims.z;
    a.error = d_err;
    (void)NB;
    cudaEventRecord(ctx->ev0, st);
    k_decode_level<<<grid, kThreads, smem, st>>>(a);
    cudaEventRecord(ctx->ev1, st);
    if (cudaGetLastError() != cudaSuccess)
      return CudaError;
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return CudaError;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    total_ms += ms;
    prev = d_level;
    if (lv.is_output)
      break;
  }
  int herr = 0;
  cudaMemcpyAsync(&herr, d_err, 4, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return CudaError;
  if (herr)
    return DeviceStreamOverflow;
  if (kernel_ms)
    *kernel_ms = total_ms;
  return NoError;
}

} // namespace idx2g
