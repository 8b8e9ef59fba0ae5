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
#include "trace.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

namespace idx2g
{

namespace
{

#include "decode_kernel.cuh"

} // namespace

#ifdef IDX2G_PHASE_TIMING
// Profiling builds: read and clear the per-phase cycle counters of the decode kernel.
extern "C" __attribute__((visibility("default"))) void idx2g_debug_dec_phase_cycles(unsigned long long* out)
{
  cudaMemcpyFromSymbol(out, g_dec_phase_cycles, sizeof(g_dec_phase_cycles));
  unsigned long long z[16] = {};
  cudaMemcpyToSymbol(g_dec_phase_cycles, z, sizeof(z));
}
#endif

namespace
{

// Device memory of open datasets comes from one stream-ordered pool per device that keeps the
// memory of closed datasets for the next one: on a busy node a cudaMalloc or cudaFree of a
// dataset's gigabyte-sized blob took from milliseconds to over a second, where the pool's
// reuse takes microseconds. idx2g_ctx_destroy trims the memory no dataset holds.
struct dataset_pool
{
  cudaMemPool_t pool = nullptr;
  cudaStream_t stream = nullptr;  // orders the frees
};

dataset_pool* pool_for(int device)
{
  static std::mutex m;
  static std::map<int, dataset_pool> pools;
  std::lock_guard<std::mutex> lk(m);
  auto it = pools.find(device);
  if (it != pools.end())
    return it->second.pool ? &it->second : nullptr;
  dataset_pool& p = pools[device];
  cudaMemPoolProps props;
  memset(&props, 0, sizeof props);
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  if (cudaMemPoolCreate(&p.pool, &props) != cudaSuccess)
  {
    cudaGetLastError();
    p.pool = nullptr;
    return nullptr;
  }
  uint64_t keep = ~0ull;
  cudaMemPoolSetAttribute(p.pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if (cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking) != cudaSuccess)
  {
    cudaMemPoolDestroy(p.pool);
    p.pool = nullptr;
    return nullptr;
  }
  return &p;
}

// `bytes` of the pool on `stream` (plain cudaMalloc where no pool could be made)
cudaError_t pool_alloc(int device, void** p, size_t bytes, cudaStream_t stream)
{
  dataset_pool* dp = pool_for(device);
  if (!dp)
    return cudaMalloc(p, bytes);
  return cudaMallocFromPoolAsync(p, bytes, dp->pool, stream);
}

} // namespace

void trim_dataset_pool(int device)
{
  dataset_pool* dp = pool_for(device);
  if (dp)
  {
    cudaStreamSynchronize(dp->stream);
    cudaMemPoolTrimTo(dp->pool, 0);
  }
}

decode_device::~decode_device()
{
  void* ps[6] = { exps_, kmin_, n_, first_, off_, blob_ };
  dataset_pool* dp = pool_for(device_);
  if (!dp)
  {
    for (void* p : ps)
      cudaFree(p);
    return;
  }
  // kernels of any stream may still read the dataset (as with cudaFree, which waits for the
  // device): its memory returns to the pool once the device is idle
  cudaSetDevice(device_);
  cudaDeviceSynchronize();
  for (void* p : ps)
    if (p)
      cudaFreeAsync(p, dp->stream);
}

int decode_device::alloc(device_ctx* ctx, size_t nslots, size_t blob_bytes)
{
  cudaSetDevice(ctx->device);
  device_ = ctx->device;
  cudaStream_t st = ctx->stream;
  // the blob is padded with zero bytes for the bit readers' look-ahead
  if (pool_alloc(device_, (void**)&exps_, nslots * kMaxBlocksPerSubband * sizeof(int16_t) + 16, st) != cudaSuccess ||
      pool_alloc(device_, (void**)&kmin_, nslots * sizeof(int32_t) + 16, st) != cudaSuccess ||
      pool_alloc(device_, (void**)&n_, nslots * sizeof(int32_t) + 16, st) != cudaSuccess ||
      pool_alloc(device_, (void**)&first_, nslots * sizeof(uint64_t) + 16, st) != cudaSuccess ||
      pool_alloc(device_, (void**)&blob_, blob_bytes + 32, st) != cudaSuccess)
  {
    cudaGetLastError();
    return OutOfMemory;
  }
  cudaMemsetAsync(blob_ + blob_bytes, 0, 32, ctx->stream);
  nslots_ = nslots;
  blob_bytes_ = blob_bytes;
  return NoError;
}

void decode_device::upload_blob(device_ctx* ctx, const uint8_t* src, size_t offset, size_t bytes)
{
  cudaSetDevice(ctx->device);
  if (bytes && offset + bytes <= blob_bytes_)
    cudaMemcpyAsync(blob_ + offset, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
}

namespace
{

// ---------------------------------------------------------------------------
// device index: channel tables from the chunk headers in the blob
// ---------------------------------------------------------------------------
struct index_args
{
  const index_chunk* chunks;
  int nchunks, nsb;
  const uint8_t* blob;
  const int* bmap;  // per level: flat brick of each linear brick, or -1
  long long bmap_base[16];
  int bmap_size[16];
  int* kmin;
  int* kmax;
  int* n;
  unsigned long long* first;
  unsigned long long* off;
  unsigned long long* block_sums;
  unsigned long long* nchan;
  size_t nslots;
  int* error;
};

// Bits of one chunk of the blob, LSB-first, read through the blob's aligned 32-bit words (the
// blob's 32 bytes of zero padding cover the look-ahead); bits at or past the chunk's end read
// as zero, as the host index reader's bytes past a chunk do. Positions are absolute bit
// positions in the blob. varbyte and unary follow Core/VarInt.h:30 ReadVarByte, :90 ReadUnary.
struct chunk_bits
{
  const uint32_t* w;
  unsigned long long hi;  // the chunk's end
  __device__ __forceinline__ unsigned long long peek(unsigned long long pos) const
  {
    if (pos >= hi)
      return 0ull;
    const unsigned long long k = pos >> 5;
    const int sh = (int)(pos & 31);
    const unsigned long long x = (unsigned long long)__ldg(w + k) | ((unsigned long long)__ldg(w + k + 1) << 32);
    unsigned long long v = x >> sh;
    if (sh)
      v |= (unsigned long long)__ldg(w + k + 2) << (64 - sh);
    const unsigned long long left = hi - pos;
    if (left < 64)
      v &= (1ull << left) - 1ull;
    return v;
  }
  __device__ __forceinline__ unsigned long long varbyte(unsigned long long& pos) const
  {
    unsigned long long v = 0;
    int sh = 0;
    for (;;)
    {
      const unsigned long long b = peek(pos) & 0xFFull;
      pos += 8;
      v = ((b & 0x7Full) << ((7 * sh++) & 63)) + v;
      if (!(b >> 7) || sh > 10)
        break;
    }
    return v;
  }
  __device__ __forceinline__ unsigned long long unary(unsigned long long& pos) const
  {
    unsigned long long v = 0;
    for (;;)
    {
      const unsigned long long x = peek(pos) & ((1ull << 57) - 1);
      if (x)
      {
        const int z = __ffsll((long long)x) - 1;
        pos += (unsigned long long)z + 1;
        return v + (unsigned long long)z;
      }
      v += 57;
      pos += 57;
      if (pos >= hi + 8)
        return v;
    }
  }
};

// The position just after the need-th set bit (need >= 1) of the bit string from pos (test
// with flags() on each lane's 32 bits at pos + 32 lane), by the whole warp; or an end past
// `limit` when the string ends first.
template <typename Flags>
__device__ __forceinline__ unsigned long long warp_find_nth(const chunk_bits& bb, unsigned long long pos,
                                                            long long need, unsigned long long limit, int lane,
                                                            Flags flags, int unit)
{
  while (need > 0)
  {
    const uint32_t f = flags((uint32_t)bb.peek(pos + 32ull * (unsigned long long)lane));
    const int cnt = __popc(f);
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1)
    {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o)
        incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (total < need)
    {
      need -= total;
      pos += 1024;
      if (pos >= limit)
        return pos;
      continue;
    }
    const int L = __ffs(__ballot_sync(0xffffffffu, incl >= need)) - 1;
    int j = 0;
    if (lane == L)
    {
      uint32_t x = f;
      for (long long r = need - (incl - cnt); r > 1; --r)
        x &= x - 1;
      j = __ffs(x) - 1;
    }
    j = __shfl_sync(0xffffffffu, j, L);
    return pos + 32ull * (unsigned long long)L + (unsigned long long)(j + unit);
  }
  return pos;
}

// Position of the r-th set bit (1 <= r <= popc(x)) of x, by halving.
__device__ __forceinline__ int nth_set_bit(uint32_t x, int r)
{
  int pos = 0;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1)
  {
    const int c = __popc(x & ((1u << s) - 1u));
    if (c < r)
    {
      r -= c;
      x >>= s;
      pos += s;
    }
  }
  return pos;
}

// For each lane, the position just after the rr-th set bit (rr >= 1; rr = 0 gives cur) of the
// bit string from cur (flags() on each lane's 32 bits of a 1024-bit window); ~0 where the
// string reaches `limit` first. Every lane of the warp takes part.
template <typename Flags>
__device__ __forceinline__ unsigned long long warp_nth_each(const chunk_bits& bb, unsigned long long cur, int rr,
                                                            unsigned long long limit, int lane, Flags flags)
{
  constexpr unsigned long long kNone = ~0ull;
  unsigned long long res = rr == 0 ? cur : kNone;
  int need = rr;
  for (unsigned long long base = cur; __any_sync(0xffffffffu, res == kNone) && base < limit; base += 1024)
  {
    const uint32_t f = flags((uint32_t)bb.peek(base + 32ull * (unsigned long long)lane));
    const int cnt = __popc(f);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o)
        incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const bool here = res == kNone && need <= total;
    const int r = here ? need : 1;
    // the first lane whose inclusive count reaches r
    int lo = 0;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1)
      if (__shfl_sync(0xffffffffu, incl, lo + st - 1) < r)
        lo += st;
    lo = lo < 31 ? lo : 31;
    const uint32_t fw = __shfl_sync(0xffffffffu, f, lo);
    const int before = __shfl_sync(0xffffffffu, incl - cnt, lo);
    if (here)
      res = base + 32ull * (unsigned long long)lo + (unsigned long long)nth_set_bit(fw, r - before) + 1ull;
    else if (res == kNone)
      need -= total;
  }
  return res;
}

// Every brick of every chunk, a warp per chunk and a lane per brick, 32 bricks at a time: the
// bricks from the unary gaps (brick i > 0 is the first brick plus the bits up to the end of
// the i-th gap), the sizes from the varbyte final bytes (each lane decodes its own) and their
// exclusive sums for the data offsets (Core/idx2Decode.cpp:507-540 DecompressChunk).
// PASS 0 records the key range of each brick's slot, PASS 1 its data offset into the slot's
// row of the offset table.
template <int PASS>
__global__ void __launch_bounds__(128) k_index_chunks(const index_args a)
{
  constexpr unsigned long long kNone = ~0ull;
  const int lane = threadIdx.x & 31;
  for (int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); c < a.nchunks;
       c += (int)((gridDim.x * blockDim.x) >> 5))
  {
    const index_chunk C = a.chunks[c];
    const chunk_bits bb{ reinterpret_cast<const uint32_t*>(a.blob), (C.off + C.size) * 8ull };
    unsigned long long pos = C.off * 8ull;
    const unsigned long long nbr64 = bb.varbyte(pos);
    if (nbr64 > C.size * 8 + 1)
    {
      if (lane == 0)
        atomicOr(a.error, 1);
      continue;
    }
    const long long nbr = (long long)nbr64;
    if (nbr == 0)
      continue;
    unsigned long long gpos = pos;
    const unsigned long long first = bb.varbyte(gpos);  // then the unary gaps from gpos
    const unsigned long long gstart = gpos;
    const unsigned long long limit = bb.hi + 8;
    unsigned long long spos = 0, data = 0;
    if (PASS == 1)
    {
      // past the nbr - 1 gaps, then to the next byte: the sizes; past those: the data
      const unsigned long long p = warp_find_nth(bb, gstart, nbr - 1, limit, lane, [](uint32_t x) { return x; }, 1);
      spos = (p + 7) & ~7ull;
      data = warp_find_nth(bb, spos, nbr, limit, lane, [](uint32_t x) { return ~x & 0x80808080u; }, 1) >> 3;
    }
    const long long base = a.bmap_base[C.level & 15];
    const int msize = a.bmap_size[C.level & 15];
    unsigned long long gcur = gstart, scur = spos, acc = 0;
    bool bad = false;
    for (long long g0 = 0; g0 < nbr && !bad; g0 += 32)
    {
      const long long i = g0 + lane;
      const bool live = i < nbr;
      // gap ends: brick i > 0 needs the i-th one bit from gstart (the group's from gcur)
      const int rr = !live || i == 0 ? 0 : (g0 == 0 ? lane : lane + 1);
      const unsigned long long ge = warp_nth_each(bb, gcur, rr, limit, lane, [](uint32_t x) { return x; });
      unsigned long long send = 0, size = 0;
      if (PASS == 1)
      {
        // size ends: the (i + 1)-th varbyte final byte from spos (the group's from scur)
        send = warp_nth_each(bb, scur, live ? lane + 1 : 0, limit, lane,
                             [](uint32_t x) { return ~x & 0x80808080u; });
        unsigned long long sbeg = __shfl_up_sync(0xffffffffu, send, 1);
        sbeg = lane == 0 ? scur : sbeg;
        if (live && send != kNone && sbeg != kNone)
          size = bb.varbyte(sbeg);
      }
      if (__any_sync(0xffffffffu, live && (ge == kNone || (PASS == 1 && send == kNone))))
      {
        bad = true;
        if (lane == 0)
          atomicOr(a.error, 1);
        break;
      }
      // exclusive sums of the sizes
      unsigned long long incl = size;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1)
      {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o)
          incl += y;
      }
      const unsigned long long o = acc + incl - size;
      acc += __shfl_sync(0xffffffffu, incl, 31);
      gcur = __shfl_sync(0xffffffffu, ge, 31);
      if (PASS == 1)
        scur = __shfl_sync(0xffffffffu, send, 31);
      if (!live)
        continue;
      const unsigned long long b = i == 0 ? first : first + (ge - gstart);
      if (b >= (unsigned long long)msize)
        continue;
      const int flat = a.bmap[base + (long long)b];
      if (flat < 0)
        continue;
      const size_t slot = (size_t)flat * (size_t)a.nsb + (size_t)C.subband;
      if (PASS == 0)
      {
        atomicMin(&a.kmin[slot], C.bpkey);
        atomicMax(&a.kmax[slot], C.bpkey);
      }
      else
      {
        const int d = C.bpkey - a.kmin[slot];
        if (d >= 0 && d < a.n[slot])
          a.off[a.first[slot] + (unsigned long long)d] = data + o;
      }
    }
  }
}

constexpr int kScanBlock = 1024;  // slots per CTA of the key-count scan (256 threads x 4)

__global__ void __launch_bounds__(256) k_index_init(const index_args a)
{
  for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < a.nslots; i += (size_t)gridDim.x * 256)
  {
    a.kmin[i] = 1 << 30;
    a.kmax[i] = -1;
  }
}

// key counts per slot and their exclusive prefix within each block of kScanBlock slots
__global__ void __launch_bounds__(256) k_index_scan_blocks(const index_args a)
{
  __shared__ unsigned long long s_part[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t b0 = (size_t)blockIdx.x * kScanBlock;
  unsigned long long v[4], t = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
  {
    const size_t i = b0 + (size_t)tid * 4 + (size_t)k;
    unsigned long long c = 0;
    if (i < a.nslots)
    {
      if (a.kmax[i] < 0)
      {
        a.kmin[i] = 1;
        a.n[i] = 0;
      }
      else
      {
        a.n[i] = a.kmax[i] - a.kmin[i] + 1;
        c = (unsigned long long)a.n[i];
      }
    }
    v[k] = c;
    t += c;
  }
  unsigned long long inc = t;
  for (int o = 1; o < 32; o <<= 1)
  {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o)
      inc += y;
  }
  if (lane == 31)
    s_part[warp] = inc;
  __syncthreads();
  unsigned long long wbase = 0;
  for (int w = 0; w < warp; ++w)
    wbase += s_part[w];
  unsigned long long run = wbase + inc - t;
#pragma unroll
  for (int k = 0; k < 4; ++k)
  {
    const size_t i = b0 + (size_t)tid * 4 + (size_t)k;
    if (i < a.nslots)
      a.first[i] = run;
    run += v[k];
  }
  if (tid == 255)
    a.block_sums[blockIdx.x] = wbase + inc;
}

// the blocks' totals to exclusive prefixes (one CTA), and the table's size
__global__ void __launch_bounds__(1024) k_index_scan_sums(const index_args a, int nblocks)
{
  __shared__ unsigned long long s_part[32];
  __shared__ unsigned long long s_carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0)
    s_carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nblocks; b0 += 1024)
  {
    const int i = b0 + tid;
    const unsigned long long c = i < nblocks ? a.block_sums[i] : 0ull;
    unsigned long long inc = c;
    for (int o = 1; o < 32; o <<= 1)
    {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o)
        inc += y;
    }
    if (lane == 31)
      s_part[warp] = inc;
    __syncthreads();
    unsigned long long wbase = 0;
    for (int w = 0; w < warp; ++w)
      wbase += s_part[w];
    const unsigned long long carry = s_carry;
    if (i < nblocks)
      a.block_sums[i] = carry + wbase + inc - c;
    __syncthreads();
    if (tid == 1023)
      s_carry = carry + wbase + inc;
    __syncthreads();
  }
  if (tid == 0)
    *a.nchan = s_carry;
}

__global__ void __launch_bounds__(256) k_index_scan_add(const index_args a)
{
  const size_t b0 = (size_t)blockIdx.x * kScanBlock;
  const unsigned long long add = a.block_sums[blockIdx.x];
  for (int k = threadIdx.x; k < kScanBlock; k += 256)
    if (b0 + (size_t)k < a.nslots)
      a.first[b0 + (size_t)k] += add;
}

} // namespace

int decode_device::build_index(device_ctx* ctx, const std::vector<index_chunk>& chunks, const std::vector<int>& brick_map,
                               const std::vector<long long>& level_base, const std::vector<int>& level_size, int nsb,
                               const int16_t* exps, size_t* nchan_out)
{
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  stage_timer tt;
  if (level_base.size() > 16 || level_size.size() != level_base.size())
    return InvalidArgument;
  const size_t ns = nslots_;
  const int nblocks = (int)((ns + kScanBlock - 1) / kScanBlock);
  index_chunk* d_chunks = (index_chunk*)ctx->ws("dec.ix.chunks", sizeof(index_chunk) * (chunks.size() + 1));
  int* d_bmap = (int*)ctx->ws("dec.ix.bmap", sizeof(int) * (brick_map.size() + 1));
  int* d_kmax = (int*)ctx->ws("dec.ix.kmax", sizeof(int) * (ns + 1));
  unsigned long long* d_sums = (unsigned long long*)ctx->ws("dec.ix.sums", 8 * ((size_t)nblocks + 2));
  int* d_err = (int*)ctx->ws("dec.ix.err", 16);
  if (!d_chunks || !d_bmap || !d_kmax || !d_sums || !d_err)
    return OutOfMemory;
  if (!chunks.empty())
    cudaMemcpyAsync(d_chunks, chunks.data(), sizeof(index_chunk) * chunks.size(), cudaMemcpyHostToDevice, st);
  if (!brick_map.empty())
    cudaMemcpyAsync(d_bmap, brick_map.data(), sizeof(int) * brick_map.size(), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d_err, 0, 16, st);
  index_args a;
  memset(&a, 0, sizeof a);
  a.chunks = d_chunks;
  a.nchunks = (int)chunks.size();
  a.nsb = nsb;
  a.blob = blob_;
  a.bmap = d_bmap;
  for (size_t l = 0; l < level_base.size(); ++l)
  {
    a.bmap_base[l] = level_base[l];
    a.bmap_size[l] = level_size[l];
  }
  a.kmin = kmin_;
  a.kmax = d_kmax;
  a.n = n_;
  a.first = first_;
  a.block_sums = d_sums;
  a.nchan = d_sums + nblocks + 1;
  a.nslots = ns;
  a.error = d_err;
  const int cgrid = (int)((chunks.size() + 3) / 4);  // a warp per chunk
  if (ns)
  {
    k_index_init<<<ns / 256 + 1 < 4096 ? (unsigned)(ns / 256 + 1) : 4096u, 256, 0, st>>>(a);
    if (cgrid)
      k_index_chunks<0><<<cgrid, 128, 0, st>>>(a);
    k_index_scan_blocks<<<nblocks, 256, 0, st>>>(a);
    k_index_scan_sums<<<1, 1024, 0, st>>>(a, nblocks);
    k_index_scan_add<<<nblocks, 256, 0, st>>>(a);
    ctx->launches += 5;
  }
  else
    cudaMemsetAsync(a.nchan, 0, 8, st);
  unsigned long long nchan = 0;
  int err = 0;
  cudaMemcpyAsync(&nchan, a.nchan, 8, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, st);
  if (ns)
    cudaMemcpyAsync(exps_, exps, ns * kMaxBlocksPerSubband * sizeof(int16_t), cudaMemcpyHostToDevice, st);
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return CudaError;
  if (err)
    return CorruptStream;
  tt.lap("open.index.keys");
  if (pool_alloc(device_, (void**)&off_, nchan * sizeof(uint64_t) + 16, st) != cudaSuccess)
  {
    cudaGetLastError();
    return OutOfMemory;
  }
  if (nchan)
    cudaMemsetAsync(off_, 0xFF, nchan * sizeof(uint64_t), st);
  a.off = off_;
  if (ns && cgrid)
  {
    k_index_chunks<1><<<cgrid, 128, 0, st>>>(a);
    ctx->launches += 1;
  }
  resident_ = ns * (kMaxBlocksPerSubband * sizeof(int16_t) + 2 * sizeof(int32_t) + sizeof(uint64_t)) +
              nchan * sizeof(uint64_t) + blob_bytes_;
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return CudaError;
  tt.lap("open.index.offsets");
  *nchan_out = (size_t)nchan;
  return NoError;
}


int decode_device::decode(device_ctx* ctx, const decode_request& rq, void* out, size_t out_bytes,
                          bool out_on_device, double* kernel_ms)
{
  std::vector<const decode_request*> rqs(1, &rq);
  return decode_batch(ctx, rqs, &out, &out_bytes, out_on_device, kernel_ms);
}

int decode_device::decode_batch(device_ctx* ctx, const std::vector<const decode_request*>& rqs,
                                void* const* outs, const size_t* out_bytes, bool out_on_device, double* kernel_ms,
                                void* coeff_out, decode_keep* keep)
{
  const size_t n = rqs.size();
  if (n == 0)
    return NoError;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const decode_request& r0 = *rqs[0];  // the dataset-wide fields are common to all requests
  const int NB = 33 * 33 * (r0.is2d ? 1 : 33);
  const int L = r0.nlevels;
  // output grids on the device
  std::vector<void*> d_out(n);
  if (!out_on_device)
  {
    size_t total = 0;
    for (size_t i = 0; i < n; ++i)
      total += (out_bytes[i] + 255) & ~(size_t)255;
    uint8_t* stage = (uint8_t*)ctx->ws("dec.out", total);
    if (!stage)
      return OutOfMemory;
    size_t at = 0;
    for (size_t i = 0; i < n; ++i)
    {
      d_out[i] = stage + at;
      at += (out_bytes[i] + 255) & ~(size_t)255;
    }
  }
  else
    for (size_t i = 0; i < n; ++i)
      d_out[i] = outs[i];
  // coefficient mode: brick base of every level in the tensor (finest level first)
  std::vector<long long> coeff_base((size_t)L + 1, 0);
  if (coeff_out)
    for (int l = 0; l < L; ++l)
    {
      const size_t k = (size_t)(L - 1 - l);
      coeff_base[(size_t)l + 1] =
        coeff_base[(size_t)l] + (k < r0.levels.size() ? (long long)r0.levels[k].bricks.size() : 0);
    }
  // One request into pinned host memory: the output level runs as several launches over rows
  // of bricks (ordered by output z), and each band of output planes that the launches so far
  // have finished goes to the host on the copy stream while the next launches run.
  bool split_out = false;
  const size_t out_elem = r0.f32 ? 4 : 8;
  if (!out_on_device && n == 1 && !keep && !coeff_out && out_bytes[0] >= ((size_t)8 << 20))
  {
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, outs[0]) == cudaSuccess && pa.type == cudaMemoryTypeHost && ctx->copies() &&
        (size_t)r0.out_dims.x * (size_t)r0.out_dims.y * (size_t)r0.out_dims.z * out_elem <= out_bytes[0])
      split_out = true;
    cudaGetLastError();
  }
  cudaStream_t cs = split_out ? ctx->copies() : nullptr;
  stream_fence out_copies{ cs };  // band copies into the caller's buffer end before any return
  int* d_err = (int*)ctx->ws("dec.err", 16);  // [0] brick kernel, [1] plane kernels (bit flags)
  uint64_t* d_geom = (uint64_t*)ctx->ws("dec.geom", sizeof(uint64_t) * 8 * kMaxBlocksPerSubband);
  if (!d_err || !d_geom)
    return OutOfMemory;
  // the plane-table path's shared memory (float staging rows for a float32 output), and the
  // three-CTA build for an output level of many bricks with a float32 output
  const size_t smem = dec_smem_bytes(true, r0.f32);
  cudaFuncSetAttribute(k_decode_level<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(dec_smem));
  cudaFuncSetAttribute(k_decode_level<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(dec_smem));
  int occ3 = 0;
  if (r0.f32 && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3, k_decode_level<3>, kThreads, smem) != cudaSuccess)
  {
    cudaGetLastError();
    occ3 = 0;
  }
  // The levels run back to back without the host waiting in between: the host prepares a
  // level's tables while the previous level runs (stream order protects the device tables
  // that every level reuses), the plane kernels' error flags are read once at the end, and a
  // plane table that overflowed (rare) makes the whole call run again with a larger one.
  unsigned long long min_cap = 0;
  for (int attempt = 0; attempt < 4; ++attempt)
  {
    for (size_t i = 0; i < n; ++i)
      if (out_bytes[i])
        cudaMemsetAsync(d_out[i], 0, out_bytes[i], st);
    if (coeff_out)
      cudaMemsetAsync(coeff_out, 0, (size_t)coeff_base[(size_t)L] * (size_t)NB * (r0.f32 ? 4 : 8), st);
    cudaMemsetAsync(d_err, 0, 16, st);
    if (keep)
    {
      keep->bricks.assign((size_t)L, nullptr);
      keep->sig.assign((size_t)L, std::vector<int>());
    }
    size_t nev = 0;  // levels timed (event pairs of the pool)
    bool out_copied = false;  // the output went to the host band by band
    double* prev = nullptr;
    std::vector<int> prev_base(n, -1), cur_base(n, -1);
    std::vector<decode_brick> hb;
    std::vector<decode_target> targets;
    int li = 0;
    for (int l = L - 1; l >= 0; --l)
    {
      const size_t k = (size_t)(L - 1 - l);  // entry of level l in a request's level list
      hb.clear();
      targets.clear();
      const decode_level* lw = nullptr;  // level-wide tables (common to all requests)
      int nstore = 0;
      for (size_t i = 0; i < n; ++i)
      {
        cur_base[i] = -1;
        const decode_request& rq = *rqs[i];
        if (k >= rq.levels.size())
          continue;
        const decode_level& lv = rq.levels[k];
        if (lv.bricks.empty())
          continue;
        lw = &lv;
        decode_target t;
        memset(&t, 0, sizeof t);
        t.mask = lv.mask;
        t.is_output = keep ? 0 : lv.is_output;  // brick-map mode keeps the output level's bricks too
        t.etol = rq.etol;
        memcpy(t.spacing, lv.spacing, sizeof t.spacing);
        t.out = d_out[i];
        t.out_dims[0] = rq.out_dims.x;
        t.out_dims[1] = rq.out_dims.y;
        t.out_dims[2] = rq.out_dims.z;
        const int ti = (int)targets.size();
        targets.push_back(t);
        cur_base[i] = (lv.is_output && !keep) || coeff_out ? -1 : nstore;
        int li_in_level = 0;
        for (const decode_brick& b : lv.bricks)
        {
          decode_brick db = b;
          db.req = ti;
          db.parent = b.parent >= 0 && prev_base[i] >= 0 ? prev_base[i] + b.parent : -1;
          if (coeff_out)
            db.store = (int)(coeff_base[(size_t)l] + li_in_level++);
          else
            db.store = lv.is_output && !keep ? -1 : nstore++;
          hb.push_back(db);
        }
      }
      prev_base = cur_base;
      const int nbr = (int)hb.size();
      if (nbr == 0)
      {
        prev = nullptr;
        continue;
      }
      // output level of a split call: bricks by output z (output bricks are independent)
      const bool split_level = split_out && targets.size() == 1 && targets[0].is_output;
      if (split_level)
        std::stable_sort(hb.begin(), hb.end(),
                         [](const decode_brick& x, const decode_brick& y) { return x.dst_from[2] < y.dst_from[2]; });
      ++li;
      decode_brick* d_bricks = (decode_brick*)ctx->ws("dec.bricks", sizeof(decode_brick) * (size_t)nbr);
      decode_target* d_reqs = (decode_target*)ctx->ws("dec.reqs", sizeof(decode_target) * targets.size());
      char kn[32];
      snprintf(kn, sizeof kn, "dec.keep%d", l);
      double* d_level = nstore ? (double*)ctx->ws(keep ? kn : (li % 2 ? "dec.levA" : "dec.levB"),
                                                  (size_t)nstore * (size_t)NB * 8)
                               : nullptr;
      int* d_sig = nullptr;
      if (keep)
      {
        snprintf(kn, sizeof kn, "dec.sig%d", l);
        d_sig = (int*)ctx->ws(kn, (size_t)nstore * 4 + 4);
        if (!d_sig)
          return OutOfMemory;
        cudaMemsetAsync(d_sig, 0, (size_t)nstore * 4, st);
        keep->bricks[(size_t)l] = d_level;
        keep->sig[(size_t)l].assign((size_t)nstore, 0);
      }
      bool three = false;
      for (const decode_target& t : targets)
        three = three || t.is_output;
      three = three && occ3 >= 3 && nbr >= 6 * ctx->num_sms;
      const int cps = three ? 3 : 2;
      int grid = nbr < cps * ctx->num_sms ? nbr : cps * ctx->num_sms;
      double* d_slots = (double*)ctx->ws("dec.slots", (size_t)grid * (size_t)NB * 8);
      if (!d_bricks || !d_reqs || (nstore && !d_level) || !d_slots)
        return OutOfMemory;
      // the level's tables through pinned staging of its own (copies stay asynchronous; the
      // call's final synchronisation comes before any reuse)
      const size_t hb_bytes = sizeof(decode_brick) * (size_t)nbr;
      const size_t tg_bytes = sizeof(decode_target) * targets.size();
      const size_t gm_bytes = sizeof(uint64_t) * 8 * kMaxBlocksPerSubband;
      char pn[32];
      snprintf(pn, sizeof pn, "dec.hstage%d", l);
      uint8_t* hs = (uint8_t*)ctx->pinned(pn, hb_bytes + tg_bytes + gm_bytes);
      if (!hs)
        return OutOfMemory;
      memcpy(hs, hb.data(), hb_bytes);
      memcpy(hs + hb_bytes, targets.data(), tg_bytes);
      memcpy(hs + hb_bytes + tg_bytes, lw->geom, gm_bytes);
      cudaMemcpyAsync(d_bricks, hs, hb_bytes, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_reqs, hs + hb_bytes, tg_bytes, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_geom, hs + hb_bytes + tg_bytes, gm_bytes, cudaMemcpyHostToDevice, st);
      dec_args a;
      memset(&a, 0, sizeof a);
      a.level = l;
      a.nlevels = L;
      a.is2d = r0.is2d;
      a.nsb = r0.nsb;
      a.nbricks = nbr;
      a.end_bp = r0.f32 ? 32 : 64;
      a.norm_mask = lw->norm_mask;
      a.out_f32 = r0.f32;
      a.bpc = r0.bpc;
      memcpy(a.nblocks, lw->nblocks, sizeof a.nblocks);
      memcpy(a.inv_weight, lw->inv_weight, sizeof a.inv_weight);
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
      a.reqs = d_reqs;
      a.error = d_err;
      a.sig = d_sig;
      a.coeff_out = coeff_out;

      // bit planes of every (brick, subband) of the level: one warp each, tables allocated
      // with a cursor in a grow-only workspace; units of more than 32 channels go to a second
      // pass, whose count the kernel reads on the device
      const size_t nunits = (size_t)nbr * (size_t)r0.nsb;
      unsigned long long* d_uoff = (unsigned long long*)ctx->ws("dec.unitoff", nunits * 8);
      unsigned long long* d_pcur = (unsigned long long*)ctx->ws("dec.pcursor", 16);
      int* d_wide = (int*)ctx->ws("dec.widelist", nunits * 4);
      if (!d_uoff || !d_pcur || !d_wide)
        return OutOfMemory;
      unsigned long long cap = (unsigned long long)nunits * 16384ull + (16ull << 20);
      if (cap < min_cap)
        cap = min_cap;
      if (ctx->ws_size("dec.planes") > cap)
        cap = ctx->ws_size("dec.planes");
      unsigned long long* d_planes = (unsigned long long*)ctx->ws("dec.planes", (size_t)cap);
      if (!d_planes)
        return OutOfMemory;
      cap = ctx->ws_size("dec.planes");
      dec1_args pa;
      memset(&pa, 0, sizeof pa);
      pa.nsb = r0.nsb;
      pa.nbricks = nbr;
      pa.unit_first = 0;
      pa.unit_last = (int)nunits;
      pa.end_bp = a.end_bp;
      pa.bpc = r0.bpc;
      pa.reqs = d_reqs;
      memcpy(pa.nblocks, lw->nblocks, sizeof pa.nblocks);
      pa.geom = d_geom;
      pa.bricks = d_bricks;
      pa.exps = exps_;
      pa.ckmin = kmin_;
      pa.cn = n_;
      pa.cfirst = first_;
      pa.coff = off_;
      pa.blob = blob_;
      pa.blob_bytes = blob_bytes_;
      pa.cursor = d_pcur;
      pa.unit_off = d_uoff;
      pa.error = d_err + 1;
      pa.wide_count = (int*)(d_pcur + 1);
      pa.wide_list = d_wide;
      pa.planes = d_planes;
      pa.cap_bytes = cap;
      a.planes = d_planes;
      a.unit_off = d_uoff;
      cudaMemsetAsync(d_pcur, 0, 16, st);
      cudaEvent_t t0 = ctx->ev(2 * nev), t1 = ctx->ev(2 * nev + 1);
      if (!t0 || !t1)
        return CudaError;
      ++nev;
      cudaEventRecord(t0, st);
      // the plane kernels over units [p.unit_first, p.unit_last): the first pass, then the
      // units it deferred (more than 32 channels)
      auto launch_planes = [&](const dec1_args& p) {
        const int g1 = (p.unit_last - p.unit_first + kPlaneWarps - 1) / kPlaneWarps;
        if (r0.bpc == 1)
        {
          k_decode_planes<false><<<(g1 + 1) / 2, kPlaneWarps * 32, 0, st>>>(p);  // two units per warp
          k_decode_planes<true><<<2 * ctx->num_sms, kPlaneWarps * 32, 0, st>>>(p);
        }
        else
        {
          k_decode_planes<false, true><<<g1, kPlaneWarps * 32, 0, st>>>(p);
          k_decode_planes<true, true><<<2 * ctx->num_sms, kPlaneWarps * 32, 0, st>>>(p);
        }
      };
      if (!split_level)
        launch_planes(pa);
      if (split_level)
      {
        // about 9 launches, each of whole rows of bricks; after launch g every output plane
        // below the first plane of the bricks still to come is final. The first band is a
        // quarter of the others, so that the copies (which take longer than the kernels)
        // start early.
        constexpr int kBands = 8;
        std::vector<int> cuts(1, 0);
        for (int g = 0; g < kBands; ++g)
        {
          if (g == 0 && nbr < 32)
            continue;
          int c = (int)(g == 0 ? (long long)nbr / 32 : (long long)nbr * g / kBands);
          while (c > 0 && c < nbr && hb[(size_t)c].dst_from[2] == hb[(size_t)c - 1].dst_from[2])
            ++c;
          if (c > cuts.back() && c < nbr)
            cuts.push_back(c);
        }
        cuts.push_back(nbr);
        const size_t plane = (size_t)r0.out_dims.x * (size_t)r0.out_dims.y * out_elem;
        size_t z_done = 0;
        for (size_t g = 0; g + 1 < cuts.size(); ++g)
        {
          // the band's plane tables (the deferred-unit list starts empty for each band)
          dec1_args pg = pa;
          pg.unit_first = cuts[g] * r0.nsb;
          pg.unit_last = cuts[g + 1] * r0.nsb;
          if (g > 0)
            cudaMemsetAsync((int*)(d_pcur + 1), 0, sizeof(int), st);
          launch_planes(pg);
          ctx->launches += 2;
          dec_args ag = a;
          ag.bricks = d_bricks + cuts[g];
          ag.nbricks = cuts[g + 1] - cuts[g];
          ag.unit_off = d_uoff + (size_t)cuts[g] * (size_t)r0.nsb;
          const int gg = ag.nbricks < grid ? ag.nbricks : grid;
          (three ? k_decode_level<3> : k_decode_level<2>)<<<gg, kThreads, smem, st>>>(ag);
          ++ctx->launches;
          const size_t z_next =
            g + 2 < cuts.size() ? (size_t)hb[(size_t)cuts[g + 1]].dst_from[2] : (size_t)r0.out_dims.z;
          if (z_next > z_done)
          {
            cudaEvent_t ge = ctx->ev(64 + g);
            if (!ge)
              return CudaError;
            cudaEventRecord(ge, st);
            cudaStreamWaitEvent(cs, ge, 0);
            cudaMemcpyAsync((uint8_t*)outs[0] + z_done * plane, (const uint8_t*)d_out[0] + z_done * plane,
                            (z_next - z_done) * plane, cudaMemcpyDeviceToHost, cs);
            z_done = z_next;
          }
        }
        out_copied = true;
      }
      else
      {
        (three ? k_decode_level<3> : k_decode_level<2>)<<<grid, kThreads, smem, st>>>(a);
        ctx->launches += 3;
      }
      cudaEventRecord(t1, st);
      if (cudaGetLastError() != cudaSuccess)
        return CudaError;
      prev = d_level;
    }
    int herr[2] = { 0, 0 };
    cudaMemcpyAsync(herr, d_err, 8, cudaMemcpyDeviceToHost, st);
    if (keep)
      for (int l = 0; l < L; ++l)
        if (!keep->sig[(size_t)l].empty())
        {
          char kn[32];
          snprintf(kn, sizeof kn, "dec.sig%d", l);
          cudaMemcpyAsync(keep->sig[(size_t)l].data(), ctx->ws(kn, keep->sig[(size_t)l].size() * 4 + 4),
                          keep->sig[(size_t)l].size() * 4, cudaMemcpyDeviceToHost, st);
        }
    if (cudaStreamSynchronize(st) != cudaSuccess || (cs && cudaStreamSynchronize(cs) != cudaSuccess))
      return CudaError;
    if (herr[1] & 2)
    {
      min_cap = 2ull * (unsigned long long)ctx->ws_size("dec.planes");
      continue;
    }
    if ((herr[1] & 1) || herr[0])
      return DeviceStreamOverflow;  // more than kKeyWindow channels in one subband, or stream error
    float total_ms = 0;
    for (size_t e = 0; e < nev; ++e)
    {
      float ms = 0;
      cudaEventElapsedTime(&ms, ctx->ev(2 * e), ctx->ev(2 * e + 1));
      total_ms += ms;
    }
    if (!out_on_device && !out_copied)
    {
      for (size_t i = 0; i < n; ++i)
        if (out_bytes[i])
          cudaMemcpyAsync(outs[i], d_out[i], out_bytes[i], cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess)
        return CudaError;
    }
    if (kernel_ms)
      *kernel_ms = total_ms;
    return NoError;
  }
  return DeviceStreamOverflow;
}


namespace
{

// Pieces of kept bricks (subband-major) to a dense buffer, x fastest: a CTA per piece.
__global__ void k_gather_pieces(const brick_piece* pieces, int n, int is2d, double* out)
{
  for (int pi = blockIdx.x; pi < n; pi += gridDim.x)
  {
    const brick_piece p = pieces[pi];
    const int nxy = p.dims[0] * p.dims[1];
    const int cnt = nxy * p.dims[2];
    for (int i = threadIdx.x; i < cnt; i += blockDim.x)
    {
      const int x = i % p.dims[0], y = (i / p.dims[0]) % p.dims[1], z = i / nxy;
      out[p.out + i] = p.src[sbm(p.from[0] + x, p.from[1] + y, p.from[2] + z, is2d)];
    }
  }
}

} // namespace

int decode_device::gather_bricks(device_ctx* ctx, const std::vector<brick_piece>& pieces, bool is2d, size_t total,
                                 double* host_out)
{
  if (pieces.empty() || total == 0)
    return NoError;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  brick_piece* d_p = (brick_piece*)ctx->ws("dec.pieces", sizeof(brick_piece) * pieces.size());
  double* d_out = (double*)ctx->ws("dec.piecesout", total * 8);
  if (!d_p || !d_out)
    return OutOfMemory;
  cudaMemcpyAsync(d_p, pieces.data(), sizeof(brick_piece) * pieces.size(), cudaMemcpyHostToDevice, st);
  const int n = (int)pieces.size();
  k_gather_pieces<<<n < 8 * ctx->num_sms ? n : 8 * ctx->num_sms, 256, 0, st>>>(d_p, n, is2d ? 1 : 0, d_out);
  ++ctx->launches;
  if (cudaGetLastError() != cudaSuccess)
    return CudaError;
  cudaMemcpyAsync(host_out, d_out, total * 8, cudaMemcpyDeviceToHost, st);
  return cudaStreamSynchronize(st) == cudaSuccess ? NoError : CudaError;
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
// The array is a file-scope __device__ variable: a device holds its kNoAllocScratchBytes
// (about 7.3 MB) from the creation of the first context on it (noalloc_prepare loads this
// file's module there) until the process exits. Limits: at most
// kNoAllocMaxBricks bricks on the output level and at most kNoAllocLevelBricks bricks on each
// coarser level a request decodes; larger requests are rejected with ScratchTooSmall.
// All calls share the array and it keeps the last call's contents: the error word is cleared
// at the start of every call, and calls that overlap on the GPU (on different streams or
// different contexts of the same device) race on it.
// ---------------------------------------------------------------------------

namespace
{

constexpr int kNoAllocSlots = 8;          // output-level brick slots (= CTAs of that launch)
constexpr int kNoAllocLevelBricks = 8;    // 3D bricks of each coarser (non-output) level
constexpr int kNoAllocMaxBricks = 4096;   // bricks of the output level
constexpr size_t kBrickBytes = (size_t)33 * 33 * 33 * sizeof(double);
constexpr size_t kOffSlots = 0;
constexpr size_t kOffLevA = kOffSlots + (size_t)kNoAllocSlots * kBrickBytes;
constexpr size_t kOffLevB = kOffLevA + (size_t)kNoAllocLevelBricks * kBrickBytes;
constexpr size_t kOffBricks = kOffLevB + (size_t)kNoAllocLevelBricks * kBrickBytes;
constexpr size_t kOffGeom = kOffBricks + (((size_t)kNoAllocMaxBricks * sizeof(decode_brick) + 255) & ~(size_t)255);
constexpr size_t kOffErr = kOffGeom + sizeof(uint64_t) * 8 * kMaxBlocksPerSubband;
constexpr size_t kOffReq = kOffErr + 256;
constexpr size_t kNoAllocScratchBytes = kOffReq + ((sizeof(decode_target) + 255) & ~(size_t)255);

static __device__ __align__(256) unsigned char g_decode_scratch[kNoAllocScratchBytes];

// Device address of g_decode_scratch, resolved with the device current and cached per
// (device, CUDA context): a process that resets a device or makes a non-primary context current
// gets the address of the array in that context. In host code the symbol is only a stand-in.
std::mutex g_scratch_mu;
struct scratch_entry
{
  void* cu_ctx;
  void* addr;
};
scratch_entry g_scratch_addr[64] = {};

// cuCtxGetCurrent through the runtime's driver entry point (no link against libcuda)
void* current_cu_context()
{
  using get_fn = int (*)(void**);
  static get_fn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (get_fn) nullptr;
    return (get_fn)p;
  }();
  void* c = nullptr;
  if (!fn || fn(&c) != 0)
    return nullptr;
  return c;
}

int scratch_address(int device, unsigned char** out)
{
  if (device < 0 || device >= 64)
    return InvalidArgument;
  void* cu = current_cu_context();
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  scratch_entry& e = g_scratch_addr[device];
  if (!e.addr || e.cu_ctx != cu)
  {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_decode_scratch) != cudaSuccess || !p)
      return CudaError;
    e.addr = p;
    e.cu_ctx = cu;
  }
  *out = (unsigned char*)e.addr;
  return NoError;
}

} // namespace

// Loads this file's kernels into the current context and resolves the scratch array's
// address. With lazy module loading (the CUDA default since 12.2) the module, and with it the
// array's device memory, would otherwise come into being at the first launch from this file;
// the context set-up calls this so that the memory is taken there, before any
// allocation-free decode.
int noalloc_prepare(int device)
{
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, k_decode_level<2>) != cudaSuccess)
    return CudaError;
  unsigned char* base = nullptr;
  return scratch_address(device, &base);
}

int decode_device::decode_noalloc(device_ctx* ctx, const decode_request& rq, void* d_out, size_t out_bytes,
                                  double* kernel_ms)
{
  if (rq.bpc != 1)
    return OptionNotSupported;  // the single-kernel wavefront decodes one plane per channel
  // limits of the fixed scratch: bricks of the output level; bytes of each kept coarser level
  // (a 2D brick takes 33 x 33 of the 33^3 samples of a 3D one)
  const size_t brick_bytes = (size_t)33 * 33 * (rq.is2d ? 1 : 33) * sizeof(double);
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
    else if (nbr > (size_t)kNoAllocMaxBricks || nbr * brick_bytes > (size_t)kNoAllocLevelBricks * kBrickBytes)
      return ScratchTooSmall;
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess)
    return CudaError;
  // the call waits for its stream after every level, which a stream under capture does not allow
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
    return InvalidArgument;
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
  decode_target* d_req = (decode_target*)(base + kOffReq);
  cudaMemsetAsync(d_out, 0, out_bytes, st);
  cudaMemsetAsync(d_err, 0, 16, st);
  const size_t smem = sizeof(dec_smem);
  cudaFuncSetAttribute(k_decode_level<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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
    decode_target t;
    memset(&t, 0, sizeof t);
    t.mask = lv.mask;
    t.is_output = lv.is_output;
    t.etol = rq.etol;
    memcpy(t.spacing, lv.spacing, sizeof t.spacing);
    t.out = d_out;
    t.out_dims[0] = rq.out_dims.x;
    t.out_dims[1] = rq.out_dims.y;
    t.out_dims[2] = rq.out_dims.z;
    cudaMemcpyAsync(d_req, &t, sizeof t, cudaMemcpyHostToDevice, st);
    dec_args a;
    memset(&a, 0, sizeof a);
    a.level = lv.level;
    a.nlevels = rq.nlevels;
    a.is2d = rq.is2d;
    a.nsb = rq.nsb;
    a.nbricks = nbr;
    a.end_bp = rq.f32 ? 32 : 64;
    a.norm_mask = lv.norm_mask;
    a.out_f32 = rq.f32;
    a.bpc = 1;
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
    a.reqs = d_req;
    a.error = d_err;
    (void)NB;
    cudaEventRecord(ctx->ev0, st);
    k_decode_level<2><<<grid, kThreads, smem, st>>>(a);
    ++ctx->launches;
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
