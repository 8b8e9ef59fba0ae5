// Device packer, the host stages around the kernels (dpack.h): segments, flush stamps, file
// layout, exponent chunks, tails, statistics.
#include "dpack.h"

#include "parallel.h"
#include "trace.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <tuple>

namespace idx2g
{

namespace
{

constexpr uint64_t kFinal = ~0ull;  // stamp of the writes of the final flushes

int vb_len(unsigned long long v)
{
  int n = 1;
  while (v >>= 7)
    ++n;
  return n;
}

void put_i32(std::vector<uint8_t>* v, int32_t x)
{
  uint8_t b[4];
  memcpy(b, &x, 4);
  v->insert(v->end(), b, b + 4);
}

struct group_events
{
  int level, subband;
  std::vector<uint32_t> events;  // global event indices, in order
};

// The (level, subband) groups of the plan in order of first appearance.
std::vector<group_events> plan_groups(const encode_plan& plan)
{
  std::vector<group_events> gs;
  std::vector<int> gi(16 * 64, -1);  // (level, subband) -> group
  for (size_t e = 0; e < plan.events.size(); ++e)
  {
    const encode_event& ev = plan.events[e];
    const size_t k = (size_t)(ev.level & 15) * 64 + (size_t)(ev.subband & 63);
    if (gi[k] < 0)
    {
      gi[k] = (int)gs.size();
      gs.push_back(group_events{ ev.level, ev.subband, {} });
    }
    gs[(size_t)gi[k]].events.push_back((uint32_t)e);
  }
  return gs;
}

struct stamp
{
  uint64_t event;
  uint32_t rank;
  bool operator<(const stamp& o) const { return event != o.event ? event < o.event : rank < o.rank; }
};

struct chunk_rec
{
  stamp st;
  int level, subband, key;
  int seg, slot;
  unsigned long long n, first_brick, last_brick, data_bytes, sizes_bytes, deltas_bytes, bytes;
  unsigned long long offset = 0;  // in the image
};

struct exp_rec
{
  stamp st;
  int level, subband;
  int seg;  // segment whose exponents it holds, -1: none (empty)
  u64 last_brick;
};

} // namespace

bool device_pack_applies(const dataset_format& f, const encode_plan& plan)
{
  if (f.nlevels > 16 || (int)plan.levels.size() < f.nlevels)
    return false;
  for (const group_events& g : plan_groups(plan))
  {
    const int shift = log2_ceil(f.bricks_per_chunk[(size_t)g.level]);
    u64 prev = 0;
    bool first = true;
    for (uint32_t e : g.events)
    {
      const encode_event& ev = plan.events[e];
      const u64 lin = plan.levels[(size_t)ev.level][(size_t)ev.brick].linear;
      if (!first && (lin >> shift) < (prev >> shift))
        return false;  // bricks not in chunk order
      if (!first && (lin >> shift) == (prev >> shift) && lin <= prev)
        return false;  // bricks of a chunk not increasing
      prev = lin;
      first = false;
    }
  }
  return true;
}

int dpack_make_plan(const dataset_format& f, const encode_plan& plan, const std::vector<std::vector<int>>& nexps,
                    dpack_plan* P)
{
  const int exp_bytes = f.type == dtype::float32 ? 1 : 2;
  *P = dpack_plan();
  P->exp_bytes = exp_bytes;
  const std::vector<group_events> groups = plan_groups(plan);
  std::vector<dpack_segment>& segs = P->segs;
  std::vector<dpack_event>& evs = P->evs;
  std::vector<u64>& seg_chunk = P->seg_chunk;
  P->group_segs.resize(groups.size());
  unsigned long long exp_total = 0;
  auto close_seg = [&]() {
    exp_total += (unsigned long long)(segs.back().ev1 - segs.back().ev0) * (unsigned long long)segs.back().nexps *
                 (unsigned long long)exp_bytes;
  };
  for (size_t gi = 0; gi < groups.size(); ++gi)
  {
    const group_events& g = groups[gi];
    P->groups.push_back({ g.level, g.subband });
    if ((size_t)g.level >= nexps.size() || (size_t)g.subband >= nexps[(size_t)g.level].size())
      return InvalidArgument;
    const int shift = log2_ceil(f.bricks_per_chunk[(size_t)g.level]);
    const int ne = nexps[(size_t)g.level][(size_t)g.subband];
    P->group_segs[gi].first = segs.size();
    for (uint32_t e : g.events)
    {
      const encode_event& ev = plan.events[e];
      const u64 lin = plan.levels[(size_t)ev.level][(size_t)ev.brick].linear;
      const u64 c = lin >> shift;
      if (segs.size() == P->group_segs[gi].first || seg_chunk.back() != c)
      {
        if (segs.size() > P->group_segs[gi].first)
          close_seg();
        dpack_segment s;
        s.level = g.level;
        s.subband = g.subband;
        s.nexps = ne;
        s.ev0 = s.ev1 = (int)evs.size();
        s.pad_ = 0;
        s.exp_off = exp_total;
        segs.push_back(s);
        seg_chunk.push_back(c);
      }
      evs.push_back(dpack_event{ lin, e, ev.brick, (int)segs.size() - 1, 0 });
      segs.back().ev1 = (int)evs.size();
    }
    if (segs.size() > P->group_segs[gi].first)
      close_seg();
    P->group_segs[gi].second = segs.size();
  }
  P->exp_total = exp_total;
  return segs.empty() ? InvalidArgument : NoError;
}

int dpack_make_layout(const dataset_format& f, const dpack_plan& P, const std::vector<dpack_key>& keys,
                      const std::vector<int>& kmin, dpack_layout* L, packed_dataset* out)
{
  const std::vector<dpack_segment>& segs = P.segs;
  if (keys.size() < segs.size() * kSegKeys || kmin.size() < segs.size())
    return InvalidArgument;
  // bit-plane chunks and their flush stamps: a channel's chunk is written when the channel
  // enters its next chunk with bytes, else by FlushChunks in channel-key order
  std::vector<chunk_rec> chunks;
  std::map<std::tuple<int, int, int>, std::vector<size_t>> chans;  // (level, subband, key) -> chunks
  for (size_t gi = 0; gi < P.groups.size(); ++gi)
    for (size_t si = P.group_segs[gi].first; si < P.group_segs[gi].second; ++si)
    {
      if (kmin[si] == 0x7fffffff)
        continue;
      for (int k = 0; k < kSegKeys; ++k)
      {
        const dpack_key& r = keys[si * kSegKeys + (size_t)k];
        if (!r.n)
          continue;
        chunk_rec c;
        c.level = segs[si].level;
        c.subband = segs[si].subband;
        c.key = kmin[si] + k;
        c.seg = (int)si;
        c.slot = k;
        c.n = r.n;
        c.first_brick = r.first_brick;
        c.last_brick = r.last_brick;
        c.data_bytes = r.data_bytes;
        c.sizes_bytes = r.sizes_bytes;
        c.deltas_bytes = (8ull * (unsigned long long)vb_len(r.first_brick) + (r.last_brick - r.first_brick) + 7) / 8;
        c.bytes = (unsigned long long)vb_len(r.n) + c.deltas_bytes + c.sizes_bytes + c.data_bytes;
        c.st = stamp{ r.enter_event, r.enter_rank };  // its entry, until replaced by its flush
        chans[std::make_tuple(c.level, c.subband, c.key)].push_back(chunks.size());
        chunks.push_back(c);
      }
    }
  {
    std::vector<std::pair<uint32_t, std::vector<size_t>*>> order;
    for (auto& kv : chans)
      order.push_back({ channel_key(std::get<2>(kv.first), std::get<0>(kv.first), std::get<1>(kv.first)), &kv.second });
    std::sort(order.begin(), order.end(),
              [](const std::pair<uint32_t, std::vector<size_t>*>& x, const std::pair<uint32_t, std::vector<size_t>*>& y) {
                return x.first < y.first;
              });
    for (size_t i = 0; i < order.size(); ++i)
    {
      std::vector<size_t>& v = *order[i].second;
      for (size_t j = 0; j + 1 < v.size(); ++j)
        chunks[v[j]].st = chunks[v[j + 1]].st;
      chunks[v.back()].st = stamp{ kFinal, (uint32_t)i };
    }
  }
  std::vector<size_t> corder(chunks.size());
  for (size_t i = 0; i < corder.size(); ++i)
    corder[i] = i;
  std::sort(corder.begin(), corder.end(), [&](size_t x, size_t y) { return chunks[x].st < chunks[y].st; });
  std::map<std::string, file_buffer>& files = out->files;
  files.clear();
  out->stats = pack_stats();
  pack_stats& stats = out->stats;
  std::map<std::string, std::vector<size_t>> file_chunks;
  for (size_t ci : corder)
  {
    const chunk_rec& c = chunks[ci];
    stats.brick_deltas.add((double)c.deltas_bytes);
    stats.brick_sizes.add((double)c.sizes_bytes);
    stats.bit_plane_chunks.add((double)c.bytes);
    const std::string path = file_path(f, c.last_brick, c.level);
    file_buffer& fb = files[path];
    fb.has_chunks = true;
    fb.chunk_sizes.put_varbyte(c.bytes);
    fb.chunk_addrs.push_back(chunk_address(f, c.last_brick, c.level, c.subband, c.key));
    file_chunks[path].push_back(ci);
  }
  // the image: every file's chunks back to back, files one after the other
  std::vector<unsigned long long>& coff = L->chunk_off;
  coff.assign(P.segs.size() * kSegKeys, ~0ull);
  std::map<std::string, std::pair<unsigned long long, unsigned long long>>& file_span = L->file_span;
  file_span.clear();
  unsigned long long total = 0;
  for (auto& kv : file_chunks)
  {
    const unsigned long long b0 = total;
    for (size_t ci : kv.second)
    {
      chunks[ci].offset = total;
      coff[(size_t)chunks[ci].seg * kSegKeys + (size_t)chunks[ci].slot] = total;
      total += chunks[ci].bytes;
    }
    file_span[kv.first] = { b0, total - b0 };
  }
  L->total = total;
  return NoError;
}

int dpack_finish(const dataset_format& f, const dpack_plan& P, const dpack_layout& L, const uint8_t* image,
                 const uint8_t* exps, packed_dataset* out)
{
  stage_timer tt;
  std::map<std::string, file_buffer>& files = out->files;
  pack_stats& stats = out->stats;
  const uint8_t* h_img = image;
  const uint8_t* h_exps = exps;
  // exponent chunks and their stamps, while the kernel runs: a group writes the exponents
  // it holds at the first brick of each later chunk, and what it holds at the end in the
  // order of FlushChunkExponents (levels descending, then subbands)
  std::vector<exp_rec> erecs;
  std::vector<size_t> gord(P.groups.size());
  for (size_t i = 0; i < gord.size(); ++i)
    gord[i] = i;
  std::stable_sort(gord.begin(), gord.end(), [&](size_t x, size_t y) {
    if (P.groups[x].first == P.groups[y].first)
      return P.groups[x].second < P.groups[y].second;
    return P.groups[x].first > P.groups[y].first;
  });
  std::vector<uint32_t> final_rank(P.groups.size());
  for (size_t i = 0; i < gord.size(); ++i)
    final_rank[gord[i]] = (uint32_t)i;
  for (size_t gi = 0; gi < P.groups.size(); ++gi)
  {
    const size_t s0 = P.group_segs[gi].first, s1 = P.group_segs[gi].second;
    for (size_t si = s0; si < s1; ++si)
    {
      if (P.seg_chunk[si] >= 1)
      {
        exp_rec r;
        r.st = stamp{ P.evs[(size_t)P.segs[si].ev0].gevent, 0 };
        r.level = P.groups[gi].first;
        r.subband = P.groups[gi].second;
        r.seg = si > s0 ? (int)si - 1 : -1;
        r.last_brick = si > s0 ? P.evs[(size_t)P.segs[si - 1].ev1 - 1].linear : 0;
        erecs.push_back(r);
      }
    }
    exp_rec r;
    r.st = stamp{ kFinal, final_rank[gi] };
    r.level = P.groups[gi].first;
    r.subband = P.groups[gi].second;
    r.seg = (int)s1 - 1;
    r.last_brick = P.evs[(size_t)P.segs[s1 - 1].ev1 - 1].linear;
    erecs.push_back(r);
  }
  std::sort(erecs.begin(), erecs.end(), [](const exp_rec& x, const exp_rec& y) { return x.st < y.st; });
  auto raw_of = [&](const exp_rec& r, const uint8_t** p, size_t* n) {
    if (r.seg < 0)
    {
      *p = h_exps;
      *n = 0;
      return;
    }
    const dpack_segment& s = P.segs[(size_t)r.seg];
    *p = h_exps + s.exp_off;
    *n = (size_t)(s.ev1 - s.ev0) * (size_t)s.nexps * (size_t)P.exp_bytes;
  };
  out->image = h_img;
  out->exps_z.assign(erecs.size(), std::vector<uint8_t>());
  std::atomic<int> zerr{ 0 };
  parallel_for(erecs.size(), [&](size_t i) {
    const uint8_t* p;
    size_t n;
    raw_of(erecs[i], &p, &n);
    if (zstd_compress(p, n, &out->exps_z[i]))
      zerr = UnknownError;
  });
  if (zerr)
    return zerr;
  tt.lap("dpack.finish.exps");
  for (size_t i = 0; i < erecs.size(); ++i)
  {
    const uint8_t* p;
    size_t n;
    raw_of(erecs[i], &p, &n);
    stats.exp_chunks_raw.add((double)n);
  }
  for (size_t i = 0; i < erecs.size(); ++i)
  {
    const exp_rec& r = erecs[i];
    stats.exp_chunks_z.add((double)out->exps_z[i].size());
    file_buffer& fb = files[file_path(f, r.last_brick, r.level)];
    fb.has_exps = true;
    fb.exp_parts.push_back({ out->exps_z[i].data(), out->exps_z[i].size() });
    fb.exp_addrs.push_back(chunk_address(f, r.last_brick, r.level, r.subband, 0));
  }
  // file contents: the chunk section, then the tails (as packer::finish)
  for (auto& kv : files)
  {
    auto sp = L.file_span.find(kv.first);
    if (sp == L.file_span.end())
      continue;
    // in pieces of at most 16 MB, so that the writer's threads share a large file
    constexpr unsigned long long kPiece = 16ull << 20;
    for (unsigned long long o = 0; o < sp->second.second; o += kPiece)
    {
      const unsigned long long n = sp->second.second - o < kPiece ? sp->second.second - o : kPiece;
      kv.second.append_ref(h_img + sp->second.first + o, (size_t)n);
    }
  }
  for (auto& kv : files)
  {
    file_buffer& fb = kv.second;
    if (!fb.has_chunks)
      continue;
    const size_t n = fb.chunk_sizes.size();
    stats.chunk_sizes.add((double)n);
    std::vector<uint8_t> tail(fb.chunk_sizes.bytes.begin(), fb.chunk_sizes.bytes.begin() + (long)n);
    put_i32(&tail, (int32_t)n);
    std::vector<uint8_t> z;
    int e = zstd_compress((const uint8_t*)fb.chunk_addrs.data(), fb.chunk_addrs.size() * 8, &z);
    if (e)
      return e;
    tail.insert(tail.end(), z.begin(), z.end());
    put_i32(&tail, (int32_t)z.size());
    put_i32(&tail, (int32_t)fb.chunk_addrs.size());
    stats.chunk_addrs_raw.add((double)fb.chunk_addrs.size() * 8);
    stats.chunk_addrs_z.add((double)z.size());
    fb.append_owned(std::move(tail));
  }
  for (auto& kv : files)
  {
    file_buffer& fb = kv.second;
    if (!fb.has_exps)
      continue;
    int tot = 0;
    bit_writer sizes;
    for (const segment& sg : fb.exp_parts)
    {
      fb.append_ref(sg.p, sg.n);
      tot += (int)sg.n;
      sizes.put_varbyte(sg.n);
    }
    const size_t n = sizes.size();
    stats.exp_chunk_sizes.add((double)n);
    std::vector<uint8_t> tail(sizes.bytes.begin(), sizes.bytes.begin() + (long)n);
    put_i32(&tail, (int32_t)n);
    tot += (int)n + 4;
    std::vector<uint8_t> z;
    int e = zstd_compress((const uint8_t*)fb.exp_addrs.data(), fb.exp_addrs.size() * 8, &z);
    if (e)
      return e;
    stats.exp_addrs_raw.add((double)fb.exp_addrs.size() * 8);
    stats.exp_addrs_z.add((double)z.size());
    tail.insert(tail.end(), z.begin(), z.end());
    put_i32(&tail, (int32_t)z.size());
    tot += (int)z.size() + 4;
    put_i32(&tail, (int32_t)fb.exp_addrs.size());
    tot += 4;
    tot += 4;
    put_i32(&tail, (int32_t)tot);
    fb.append_owned(std::move(tail));
  }
  tt.lap("dpack.finish.tails");
  return NoError;
}

} // namespace idx2g
