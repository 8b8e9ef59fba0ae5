// Test infrastructure: the device packer's two kernels (idx2_b200/csrc/dpack.cu k_pack_keys,
// k_pack_write) restated on the host over host copies of the regions, so that the packer's
// host stages (dpack_plan.cpp) and the kernels' per-segment rules can be checked against the
// host packer's files on a machine without a GPU. Each loop follows the kernel's: the same
// key totals, the same entry-rank formula (first covering block, then descending key), the
// same scans and byte placement.
#pragma once

#include "dpack.h"
#include "encoder.h"

#include <climits>
#include <cstring>
#include <vector>

namespace idx2g
{
namespace emul
{

inline int vb_len(unsigned long long v)
{
  int n = 1;
  while (v >>= 7)
    ++n;
  return n;
}

inline int coded_planes(int emax, int etol, int end_bp, int bpc)
{
  if (bpc == 1)
  {
    int low = 57 + etol - emax;
    const int lim = 64 - end_bp;
    low = low > lim ? low : lim;
    return low <= 63 ? 64 - low : 0;
  }
  int np = 0;
  for (int bp = 63; bp >= 64 - end_bp; --bp)
  {
    const int realbp = bp + emax;
    if (58 > realbp - etol + 1 && ((realbp + 1024) % bpc) == 0)
      break;
    ++np;
  }
  return np;
}

inline int plane_key(int top, int kk, int bpc) { return bpc == 1 ? top - kk : (top - kk) / bpc; }

struct region
{
  int kmin, nkeys;
  const int16_t* exps;
  const uint32_t* sizes;
  const uint8_t* bytes;
};

inline region region_of(const std::vector<level_output>& outs, const dpack_segment& s, const dpack_event& e)
{
  const level_output& o = outs[(size_t)s.level];
  const uint8_t* r = o.bytes() + o.offset[(size_t)e.brick * (size_t)o.nsb + (size_t)s.subband];
  region v;
  int32_t w[2];
  memcpy(w, r, 8);
  v.nkeys = w[1] > 0 ? w[1] : 0;
  v.kmin = w[0];
  v.exps = reinterpret_cast<const int16_t*>(r + 8);
  const size_t eb = ((size_t)s.nexps * 2 + 3) & ~(size_t)3;
  v.sizes = reinterpret_cast<const uint32_t*>(r + 8 + eb);
  v.bytes = r + 8 + eb + (size_t)v.nkeys * 4;
  return v;
}

// k_pack_keys; returns 1 when a segment spans more than kSegKeys keys
inline int pack_keys(const dataset_format& f, const dpack_plan& P, const std::vector<level_output>& outs,
                     std::vector<dpack_key>* keys, std::vector<int>* kmin)
{
  const int etol = exponent_f64(f.tolerance), end_bp = f.type == dtype::float32 ? 32 : 64;
  const int bpc = f.bit_planes_per_chunk;
  keys->assign(P.segs.size() * kSegKeys, dpack_key{});
  kmin->assign(P.segs.size(), INT_MAX);
  int err = 0;
  for (size_t si = 0; si < P.segs.size(); ++si)
  {
    const dpack_segment& S = P.segs[si];
    int lo = INT_MAX, hi = -INT_MAX;
    for (int i = S.ev0; i < S.ev1; ++i)
    {
      const region r = region_of(outs, S, P.evs[(size_t)i]);
      if (r.nkeys > 0)
      {
        lo = r.kmin < lo ? r.kmin : lo;
        hi = r.kmin + r.nkeys - 1 > hi ? r.kmin + r.nkeys - 1 : hi;
      }
    }
    if (hi < lo)
      continue;
    if (hi - lo + 1 > kSegKeys)
    {
      err = 1;
      continue;
    }
    (*kmin)[si] = lo;
    std::vector<unsigned> n(kSegKeys, 0), szb(kSegKeys, 0), rank(kSegKeys, 0);
    std::vector<int> first(kSegKeys, INT_MAX), last(kSegKeys, -1);
    std::vector<unsigned long long> db(kSegKeys, 0);
    for (int i = S.ev0; i < S.ev1; ++i)
    {
      const region r = region_of(outs, S, P.evs[(size_t)i]);
      for (int j = 0; j < r.nkeys; ++j)
      {
        const uint32_t sz = r.sizes[j];
        if (!sz)
          continue;
        const int k = r.kmin + j - lo;
        ++n[(size_t)k];
        szb[(size_t)k] += (unsigned)vb_len(sz);
        db[(size_t)k] += sz;
        first[(size_t)k] = std::min(first[(size_t)k], i - S.ev0);
        last[(size_t)k] = std::max(last[(size_t)k], i - S.ev0);
      }
    }
    const int nk = hi - lo + 1;
    for (int k = 0; k < nk; ++k)
    {
      if (!n[(size_t)k])
        continue;
      const region r = region_of(outs, S, P.evs[(size_t)(S.ev0 + first[(size_t)k])]);
      std::vector<int> fb((size_t)kKeyWindow, INT_MAX);
      for (int b = 0; b < S.nexps; ++b)
      {
        const int emax = r.exps[b];
        const int np = coded_planes(emax, etol, end_bp, bpc);
        if (!np)
          continue;
        const int top = emax + 63 + 1024;
        for (int key = plane_key(top, np - 1, bpc); key <= plane_key(top, 0, bpc); ++key)
        {
          const int j = key - r.kmin;
          if (j >= 0 && j < r.nkeys && j < kKeyWindow)
            fb[(size_t)j] = std::min(fb[(size_t)j], b);
        }
      }
      const int jk = lo + k - r.kmin;
      const int fk = jk >= 0 && jk < kKeyWindow ? fb[(size_t)jk] : INT_MAX;
      unsigned cnt = 0;
      for (int j = 0; j < r.nkeys && j < kKeyWindow; ++j)
        cnt += fb[(size_t)j] != INT_MAX && (fb[(size_t)j] < fk || (fb[(size_t)j] == fk && j > jk));
      rank[(size_t)k] = cnt;
    }
    for (int k = 0; k < nk; ++k)
    {
      dpack_key& o = (*keys)[si * kSegKeys + (size_t)k];
      o.n = n[(size_t)k];
      o.sizes_bytes = szb[(size_t)k];
      o.data_bytes = db[(size_t)k];
      o.enter_rank = rank[(size_t)k];
      if (o.n)
      {
        const dpack_event& e0 = P.evs[(size_t)(S.ev0 + first[(size_t)k])];
        o.enter_event = e0.gevent;
        o.first_brick = e0.linear;
        o.last_brick = P.evs[(size_t)(S.ev0 + last[(size_t)k])].linear;
      }
    }
  }
  return err;
}

inline void put_varbyte(std::vector<uint8_t>& img, unsigned long long p, unsigned long long v)
{
  for (;;)
  {
    const unsigned long long more = (v >> 7) != 0;
    img[(size_t)p++] |= (uint8_t)((v & 0x7F) | (more << 7));
    v >>= 7;
    if (!more)
      break;
  }
}

// k_pack_write
inline void pack_write(const dpack_plan& P, const std::vector<level_output>& outs, const std::vector<dpack_key>& keys,
                       const std::vector<int>& kmin, const dpack_layout& L, std::vector<uint8_t>* image,
                       std::vector<uint8_t>* exps)
{
  image->assign((size_t)L.total + 8, 0);
  exps->assign((size_t)P.exp_total + 8, 0);
  for (size_t si = 0; si < P.segs.size(); ++si)
  {
    const dpack_segment& S = P.segs[si];
    for (int i = S.ev0; i < S.ev1; ++i)
    {
      const region r = region_of(outs, S, P.evs[(size_t)i]);
      uint8_t* dst = exps->data() + S.exp_off + (size_t)(i - S.ev0) * (size_t)S.nexps * (size_t)P.exp_bytes;
      for (int b = 0; b < S.nexps; ++b)
      {
        const int v = r.exps[b];
        if (P.exp_bytes == 1)
          dst[b] = (uint8_t)(v + 127);
        else
        {
          const uint16_t u = (uint16_t)(v + 1023);
          dst[2 * b] = (uint8_t)(u & 0xFF);
          dst[2 * b + 1] = (uint8_t)(u >> 8);
        }
      }
    }
    if (kmin[si] == INT_MAX)
      continue;
    for (int k = 0; k < kSegKeys; ++k)
    {
      const dpack_key& rec = keys[si * kSegKeys + (size_t)k];
      if (!rec.n)
        continue;
      const int key = kmin[si] + k;
      const unsigned long long base = L.chunk_off[si * kSegKeys + (size_t)k];
      const unsigned long long d0 = base + (unsigned long long)vb_len(rec.n);
      const int vbf = vb_len(rec.first_brick);
      const unsigned long long dbits = 8ull * (unsigned long long)vbf + (rec.last_brick - rec.first_brick);
      const unsigned long long s0 = d0 + (dbits + 7) / 8;
      const unsigned long long x0 = s0 + rec.sizes_bytes;
      put_varbyte(*image, base, rec.n);
      put_varbyte(*image, d0, rec.first_brick);
      unsigned long long vb_acc = 0, data_acc = 0;
      for (int i = S.ev0; i < S.ev1; ++i)
      {
        const dpack_event& e = P.evs[(size_t)i];
        const region r = region_of(outs, S, e);
        const int j = key - r.kmin;
        if (j < 0 || j >= r.nkeys || !r.sizes[j])
          continue;
        const uint32_t sz = r.sizes[j];
        unsigned long long kb = 0;
        for (int t = 0; t < j; ++t)
          kb += r.sizes[t];
        put_varbyte(*image, s0 + vb_acc, sz);
        if (e.linear != rec.first_brick)
        {
          const unsigned long long bit = d0 * 8ull + 8ull * (unsigned long long)vbf + (e.linear - rec.first_brick) - 1ull;
          (*image)[(size_t)(bit >> 3)] |= (uint8_t)(1u << (unsigned)(bit & 7));
        }
        for (uint32_t t = 0; t < sz; ++t)
          (*image)[(size_t)(x0 + data_acc + t)] |= r.bytes[kb + t];
        vb_acc += (unsigned long long)vb_len(sz);
        data_acc += sz;
      }
    }
  }
}

} // namespace emul
} // namespace idx2g
