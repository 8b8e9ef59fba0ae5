// Kernels of the device packer (dpack.h).
#include "codec_device.cuh"
#include "dpack_device.h"

namespace idx2g
{
namespace
{

constexpr int kPackThreads = 256;
constexpr int kPackWarps = kPackThreads / 32;
constexpr int kNoEvent = 0x7fffffff;

// The region of one event: its key window, exponents, per-key byte counts, channel streams
// (layout in encoder.h, region_view).
struct region_dev
{
  int kmin, nkeys;
  const int16_t* exps;
  const uint32_t* sizes;
  const uint8_t* bytes;
};

__device__ __forceinline__ region_dev region_of(const dpack_args& a, const dpack_segment& s, const dpack_event& e)
{
  const uint8_t* r = a.streams[s.level] + a.offsets[s.level][(size_t)e.brick * 8 + (size_t)s.subband];
  region_dev v;
  const int32_t* w = reinterpret_cast<const int32_t*>(r);
  v.nkeys = w[1] > 0 ? w[1] : 0;
  v.kmin = w[0];
  v.exps = reinterpret_cast<const int16_t*>(r + 8);
  const size_t eb = ((size_t)s.nexps * 2 + 3) & ~(size_t)3;
  v.sizes = reinterpret_cast<const uint32_t*>(r + 8 + eb);
  v.bytes = r + 8 + eb + (size_t)v.nkeys * 4;
  return v;
}

// bytes of the varbyte code of v (Core/VarInt.h:14)
__device__ __forceinline__ int vb_len(unsigned long long v)
{
  int n = 1;
  while (v >>= 7)
    ++n;
  return n;
}

// OR one byte into the zeroed image at byte position p. Every byte outside the interior
// words of a pair's data goes through here: each is written once, so the order of the ORs of
// different threads into one word does not matter.
__device__ __forceinline__ void or_byte(uint32_t* img, unsigned long long p, uint32_t b)
{
  if (b)
    atomicOr(img + (p >> 2), b << (8 * (unsigned)(p & 3)));
}

__device__ __forceinline__ void put_varbyte(uint32_t* img, unsigned long long p, unsigned long long v)
{
  for (;;)
  {
    const unsigned long long more = (v >> 7) != 0;
    or_byte(img, p++, (uint32_t)((v & 0x7F) | (more << 7)));
    v >>= 7;
    if (!more)
      break;
  }
}

// ---------------------------------------------------------------------------
// key totals, over every event at once (a warp per event), then per segment the entry ranks
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPackThreads) k_pack_init(const dpack_args a)
{
  const size_t n = (size_t)a.nseg * kSegKeys;
  for (size_t i = (size_t)blockIdx.x * kPackThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kPackThreads)
  {
    dpack_acc z;
    z.n = 0;
    z.szb = 0;
    z.first = kNoEvent;
    z.last = -1;
    z.db = 0;
    a.acc[i] = z;
    if (i < (size_t)a.nseg)
    {
      a.seg_kmin[i] = 0x7fffffff;
      a.seg_kmax[i] = -0x7fffffff;
    }
  }
}

// Per event: its region's key window, the byte offsets of its key streams (an exclusive scan
// of the per-key sizes into kb), and its segment's key range.
__global__ void __launch_bounds__(kPackThreads) k_pack_events(const dpack_args a)
{
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * kPackThreads + (int)threadIdx.x) >> 5; i < a.nev; i += (gridDim.x * kPackThreads) >> 5)
  {
    const dpack_event& e = a.evs[i];
    const dpack_segment& S = a.segs[e.seg];
    const region_dev r = region_of(a, S, e);
    unsigned long long base = 0;
    if (lane == 0)
    {
      a.ev_region[i] = (unsigned long long)(size_t)(r.exps) - 8ull;
      a.ev_kmin[i] = r.kmin;
      a.ev_nkeys[i] = r.nkeys;
      if (r.nkeys > 0)
      {
        atomicMin(&a.seg_kmin[e.seg], r.kmin);
        atomicMax(&a.seg_kmax[e.seg], r.kmin + r.nkeys - 1);
        base = atomicAdd(a.cursor, (unsigned long long)r.nkeys);
        if (base + (unsigned long long)r.nkeys > a.kb_cap)
        {
          atomicOr(a.error, 2);
          base = ~0ull;
        }
      }
      a.ev_kb[i] = base;
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    if (r.nkeys == 0 || base == ~0ull)
      continue;
    unsigned long long carry = 0;
    for (int j0 = 0; j0 < r.nkeys; j0 += 32)
    {
      const int j = j0 + lane;
      const uint32_t sz = j < r.nkeys ? r.sizes[j] : 0u;
      unsigned long long inc = sz;
      for (int o = 1; o < 32; o <<= 1)
      {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
          inc += y;
      }
      if (j < r.nkeys)
        a.kb[base + (unsigned long long)j] = (uint32_t)(carry + inc - sz);
      carry += __shfl_sync(0xffffffffu, inc, 31);
    }
  }
}

// Per sub-range of a segment (a CTA each): the keys' totals over its events in shared memory
// (order-free), written per sub-range and added to the segment's totals.
__global__ void __launch_bounds__(kPackThreads) k_pack_totals(const dpack_args a)
{
  __shared__ unsigned s_n[kSegKeys], s_szb[kSegKeys];
  __shared__ int s_first[kSegKeys], s_last[kSegKeys];
  __shared__ unsigned long long s_db[kSegKeys];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int ci = blockIdx.x; ci < a.nsub; ci += gridDim.x)
  {
    const int4 sr = a.subs[ci];
    const int seg = sr.x;
    const dpack_segment& S = a.segs[seg];
    const int K0 = a.seg_kmin[seg];
    if (a.seg_kmax[seg] < K0)
      continue;  // no keys in the segment
    if (a.seg_kmax[seg] - K0 + 1 > kSegKeys)
    {
      if (tid == 0)
        atomicOr(a.error, 1);
      continue;
    }
    for (int k = tid; k < kSegKeys; k += kPackThreads)
    {
      s_n[k] = 0;
      s_szb[k] = 0;
      s_db[k] = 0;
      s_first[k] = kNoEvent;
      s_last[k] = -1;
    }
    __syncthreads();
    const size_t eb = ((size_t)S.nexps * 2 + 3) & ~(size_t)3;
    for (int i = sr.y + warp; i < sr.z; i += kPackWarps)
    {
      const int nkeys = a.ev_nkeys[i];
      if (nkeys <= 0)
        continue;
      const int kmin = a.ev_kmin[i];
      const uint32_t* sizes = reinterpret_cast<const uint32_t*>((size_t)a.ev_region[i] + 8 + eb);
      const int li = i - S.ev0;
      for (int j = lane; j < nkeys; j += 32)
      {
        const uint32_t sz = sizes[j];
        if (!sz)
          continue;
        const int k = kmin + j - K0;
        atomicAdd(&s_n[k], 1u);
        atomicAdd(&s_szb[k], (unsigned)vb_len(sz));
        atomicAdd(&s_db[k], (unsigned long long)sz);
        atomicMin(&s_first[k], li);
        atomicMax(&s_last[k], li);
      }
    }
    __syncthreads();
    const int nk = a.seg_kmax[seg] - K0 + 1;
    dpack_acc* acc = a.acc + (size_t)seg * kSegKeys;
    dpack_sub* sub = a.sub_acc + ((size_t)a.seg_sub0[seg] + (size_t)sr.w) * kSegKeys;
    for (int k = tid; k < nk; k += kPackThreads)
    {
      sub[k].vb = s_szb[k];
      sub[k].data = s_db[k];
      if (!s_n[k])
        continue;
      atomicAdd(&acc[k].n, s_n[k]);
      atomicAdd(&acc[k].szb, s_szb[k]);
      atomicAdd(&acc[k].db, s_db[k]);
      atomicMin(&acc[k].first, s_first[k]);
      atomicMax(&acc[k].last, s_last[k]);
    }
    __syncthreads();
  }
}

// Per segment: the entry rank of each key (its place in the first-touch order of keys of its
// entry event: blocks in Morton order, each block's coded planes top-down, i.e. keys by first
// covering block, then descending), and the key records.
__global__ void __launch_bounds__(kPackThreads) k_pack_ranks(const dpack_args a)
{
  __shared__ int s_ev;
  __shared__ unsigned s_rank[kSegKeys];
  __shared__ int s_first[kSegKeys];
  __shared__ uint8_t s_done[kSegKeys];
  __shared__ int s_fb[kKeyWindow];  // first block covering each key of the entry event
  const int tid = threadIdx.x;
  for (int si = blockIdx.x; si < a.nseg; si += gridDim.x)
  {
    const dpack_segment& S = a.segs[si];
    const int K0 = a.seg_kmin[si];
    const bool any = a.seg_kmax[si] >= K0;
    if (any && a.seg_kmax[si] - K0 + 1 > kSegKeys)
    {
      if (tid == 0)
        a.seg_kmin[si] = 0x7fffffff;  // (the error flag is set: the host packs)
      continue;
    }
    const int nk = any ? a.seg_kmax[si] - K0 + 1 : 0;
    const dpack_acc* acc = a.acc + (size_t)si * kSegKeys;
    for (int k = tid; k < kSegKeys; k += kPackThreads)
    {
      s_rank[k] = 0;
      s_first[k] = k < nk && acc[k].n ? acc[k].first : kNoEvent;
      s_done[k] = 0;
    }
    __syncthreads();
    for (;;)
    {
      if (tid == 0)
        s_ev = kNoEvent;
      __syncthreads();
      for (int k = tid; k < nk; k += kPackThreads)
        if (s_first[k] != kNoEvent && !s_done[k])
          atomicMin(&s_ev, s_first[k]);
      __syncthreads();
      const int ev = s_ev;
      if (ev == kNoEvent)
        break;
      const region_dev r = region_of(a, S, a.evs[S.ev0 + ev]);
      for (int j = tid; j < kKeyWindow; j += kPackThreads)
        s_fb[j] = 0x7fffffff;
      __syncthreads();
      for (int b = tid; b < S.nexps; b += kPackThreads)
      {
        const int emax = r.exps[b];
        const int np = dev::coded_planes(emax, a.etol, a.end_bp, a.bpc);
        if (!np)
          continue;
        const int top = emax + 63 + 1024;
        const int hi = dev::plane_key(top, 0, a.bpc), lo = dev::plane_key(top, np - 1, a.bpc);
        for (int key = lo; key <= hi; ++key)
        {
          const int j = key - r.kmin;
          if (j >= 0 && j < r.nkeys && j < kKeyWindow)
            atomicMin(&s_fb[j], b);
        }
      }
      __syncthreads();
      for (int k = tid; k < nk; k += kPackThreads)
      {
        if (s_first[k] != ev || s_done[k])
          continue;
        const int jk = K0 + k - r.kmin;  // the key's index in the event's window
        const int fk = jk >= 0 && jk < kKeyWindow ? s_fb[jk] : 0x7fffffff;
        unsigned cnt = 0;
        const int nj = r.nkeys < kKeyWindow ? r.nkeys : kKeyWindow;
        for (int j = 0; j < nj; ++j)
        {
          const int fj = s_fb[j];
          cnt += fj != 0x7fffffff && (fj < fk || (fj == fk && j > jk));
        }
        s_rank[k] = cnt;
        s_done[k] = 1;
      }
      __syncthreads();
    }
    for (int k = tid; k < kSegKeys; k += kPackThreads)
    {
      dpack_key out;
      const dpack_acc t = acc[k];
      out.n = k < nk ? t.n : 0;
      out.sizes_bytes = t.szb;
      out.data_bytes = t.db;
      out.enter_rank = s_rank[k];
      if (out.n)
      {
        const dpack_event& e0 = a.evs[S.ev0 + t.first];
        out.enter_event = e0.gevent;
        out.first_brick = e0.linear;
        out.last_brick = a.evs[S.ev0 + t.last].linear;
      }
      else
      {
        out.enter_event = 0;
        out.first_brick = out.last_brick = 0;
      }
      a.keys[(size_t)si * kSegKeys + k] = out;
      // the key's offsets at the start of each sub-range: exclusive prefixes over them
      if (out.n)
      {
        const int ns = (S.ev1 - S.ev0 + kPackSub - 1) / kPackSub;
        dpack_sub* sub = a.sub_acc + (size_t)a.seg_sub0[si] * kSegKeys + k;
        unsigned long long vb = 0, data = 0;
        for (int q = 0; q < ns; ++q)
        {
          const dpack_sub t = sub[(size_t)q * kSegKeys];
          sub[(size_t)q * kSegKeys].vb = vb;
          sub[(size_t)q * kSegKeys].data = data;
          vb += t.vb;
          data += t.data;
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// per segment: raw exponents, and a warp per chunk writing its header and data
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPackThreads) k_pack_write(const dpack_args a)
{
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // a CTA per sub-range of a segment, a warp per key
  for (int ci = blockIdx.x; ci < a.nsub; ci += gridDim.x)
  {
    const int4 sr = a.subs[ci];
    const int si = sr.x;
    const dpack_segment& S = a.segs[si];
    // raw exponents (Core/idx2Encode.cpp:41 EncodeBrickSubbandExponents): EMax + 127 as a
    // byte (float32) or EMax + 1023 as a little-endian 16-bit word (float64), events in order
    for (int i = sr.y + warp; i < sr.z; i += kPackWarps)
    {
      const region_dev r = region_of(a, S, a.evs[i]);
      uint8_t* dst = a.exps + S.exp_off + (size_t)(i - S.ev0) * (size_t)S.nexps * (size_t)a.exp_bytes;
      for (int b = lane; b < S.nexps; b += 32)
      {
        const int v = r.exps[b];
        if (a.exp_bytes == 1)
          dst[b] = (uint8_t)(v + 127);
        else
        {
          const uint16_t u = (uint16_t)(v + 1023);
          dst[2 * b] = (uint8_t)(u & 0xFF);
          dst[2 * b + 1] = (uint8_t)(u >> 8);
        }
      }
    }
    const int K0 = a.seg_kmin[si];
    if (K0 == 0x7fffffff)
      continue;
    for (int k = warp; k < kSegKeys; k += kPackWarps)
    {
      const dpack_key rec = a.keys[(size_t)si * kSegKeys + k];
      if (!rec.n)
        continue;
      const int key = K0 + k;
      const unsigned long long base = a.chunk_off[(size_t)si * kSegKeys + k];
      // Core/idx2Write.cpp:221 WriteChunk: varbyte NBricks | brick deltas | brick sizes | data;
      // deltas: the first brick as a varbyte, then per brick (gap - 1) zeros and a one
      const unsigned long long d0 = base + (unsigned long long)vb_len(rec.n);
      const int vbf = vb_len(rec.first_brick);
      const unsigned long long dbits = 8ull * (unsigned long long)vbf + (rec.last_brick - rec.first_brick);
      const unsigned long long s0 = d0 + (dbits + 7) / 8;
      const unsigned long long x0 = s0 + rec.sizes_bytes;
      if (lane == 0 && sr.w == 0)
      {
        put_varbyte(a.image, base, rec.n);
        put_varbyte(a.image, d0, rec.first_brick);
      }
      // the key's varbyte-size and data offsets at the start of the sub-range
      const dpack_sub c0 = a.sub_acc[((size_t)a.seg_sub0[si] + (size_t)sr.w) * kSegKeys + k];
      unsigned long long vb_carry = c0.vb, data_carry = c0.data;
      for (int i0 = sr.y; i0 < sr.z; i0 += 32)
      {
        const int i = i0 + lane;
        uint32_t sz = 0;
        const uint8_t* src = nullptr;
        unsigned long long linear = 0;
        if (i < sr.z)
        {
          const int kmin = a.ev_kmin[i], nkeys = a.ev_nkeys[i];
          const int j = key - kmin;
          if (j >= 0 && j < nkeys)
          {
            const uint8_t* reg = reinterpret_cast<const uint8_t*>((size_t)a.ev_region[i]);
            const size_t eb = ((size_t)S.nexps * 2 + 3) & ~(size_t)3;
            sz = reinterpret_cast<const uint32_t*>(reg + 8 + eb)[j];
            if (sz)
            {
              // the key's stream after the lower keys' streams
              src = reg + 8 + eb + (size_t)nkeys * 4 + a.kb[a.ev_kb[i] + (unsigned long long)j];
              linear = a.evs[i].linear;
            }
          }
        }
        const unsigned vbs = sz ? (unsigned)vb_len(sz) : 0u;
        unsigned long long ivb = vbs, isz = sz;
        for (int o = 1; o < 32; o <<= 1)
        {
          const unsigned long long y1 = __shfl_up_sync(0xffffffffu, ivb, o);
          const unsigned long long y2 = __shfl_up_sync(0xffffffffu, isz, o);
          if (lane >= o)
          {
            ivb += y1;
            isz += y2;
          }
        }
        const unsigned long long my_vb = vb_carry + ivb - vbs, my_data = data_carry + isz - sz;
        if (sz)
        {
          put_varbyte(a.image, s0 + my_vb, sz);
          if (linear != rec.first_brick)
          {
            const unsigned long long bit = d0 * 8ull + 8ull * (unsigned long long)vbf + (linear - rec.first_brick) - 1ull;
            atomicOr(a.image + (bit >> 5), 1u << (unsigned)(bit & 31));
          }
        }
        // the pairs' bytes, a pair at a time, lanes over destination words: whole words inside
        // the pair's range are stored, the (shared) words at its two ends ORed byte by byte
        unsigned m = __ballot_sync(0xffffffffu, sz != 0);
        while (m)
        {
          const int l = __ffs(m) - 1;
          m &= m - 1;
          const uint8_t* ps = (const uint8_t*)__shfl_sync(0xffffffffu, (unsigned long long)src, l);
          const unsigned long long pd = x0 + __shfl_sync(0xffffffffu, my_data, l);
          const unsigned n = __shfl_sync(0xffffffffu, sz, l);
          const unsigned long long w0 = pd >> 2, w1 = (pd + n - 1) >> 2;
          for (unsigned long long w = w0 + lane; w <= w1; w += 32)
          {
            const unsigned long long p = w << 2;
            if (p >= pd && p + 4 <= pd + n)
            {
              const uint8_t* q = ps + (p - pd);
              a.image[w] = (uint32_t)q[0] | ((uint32_t)q[1] << 8) | ((uint32_t)q[2] << 16) | ((uint32_t)q[3] << 24);
            }
            else
            {
              for (int t = 0; t < 4; ++t)
                if (p + t >= pd && p + t < pd + n)
                  or_byte(a.image, p + t, ps[p + t - pd]);
            }
          }
        }
        vb_carry += __shfl_sync(0xffffffffu, ivb, 31);
        data_carry += __shfl_sync(0xffffffffu, isz, 31);
      }
    }
  }
}

} // namespace

void dpack_launch_keys(const dpack_args& a, int grid, cudaStream_t st)
{
  // a warp per event for the per-event passes
  const int eg = (int)((a.nev + kPackWarps - 1) / kPackWarps);
  const int egrid = eg < 65535 ? (eg > 0 ? eg : 1) : 65535;
  const int igrid = (int)(((size_t)a.nseg * kSegKeys + kPackThreads - 1) / kPackThreads);
  k_pack_init<<<igrid < 4096 ? igrid : 4096, kPackThreads, 0, st>>>(a);
  k_pack_events<<<egrid, kPackThreads, 0, st>>>(a);
  const int sgrid = a.nsub < 65535 ? a.nsub : 65535;
  k_pack_totals<<<sgrid > 0 ? sgrid : 1, kPackThreads, 0, st>>>(a);
  k_pack_ranks<<<grid, kPackThreads, 0, st>>>(a);
}

void dpack_launch_write(const dpack_args& a, int grid, cudaStream_t st)
{
  (void)grid;
  const int sgrid = a.nsub < 65535 ? a.nsub : 65535;
  k_pack_write<<<sgrid > 0 ? sgrid : 1, kPackThreads, 0, st>>>(a);
}

} // namespace idx2g
