// Sharded encode: shard plans, the header exchange payload, and each shard's share of the
// packing and file writes (shard.h).
#include "shard.h"
#include "parallel.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <fcntl.h>
#include <unistd.h>

namespace idx2g
{

int make_shard_plan(const dataset_format& f, const encode_plan& plan, int nshards, int shard, shard_plan* sp)
{
  const int L = (int)plan.levels.size();
  if (nshards < 1 || shard < 0 || shard >= nshards || L < 1)
    return InvalidArgument;
  const size_t ncoarse = plan.levels[(size_t)L - 1].size();
  if (ncoarse < (size_t)nshards)
    return InvalidArgument;  // fewer coarsest bricks than shards
  sp->nshards = nshards;
  sp->shard = shard;
  sp->owner.assign((size_t)L, {});
  sp->local_index.assign((size_t)L, {});
  // the coarsest level in nshards contiguous runs, then every brick takes its parent's shard
  sp->owner[(size_t)L - 1].resize(ncoarse);
  for (size_t i = 0; i < ncoarse; ++i)
    sp->owner[(size_t)L - 1][i] = (int)(i * (size_t)nshards / ncoarse);
  for (int l = L - 2; l >= 0; --l)
  {
    const std::vector<brick_entry>& bl = plan.levels[(size_t)l];
    std::vector<int>& own = sp->owner[(size_t)l];
    own.resize(bl.size());
    for (size_t i = 0; i < bl.size(); ++i)
    {
      const int par = bl[i].parent;
      if (par < 0 || (size_t)par >= sp->owner[(size_t)l + 1].size())
        return UnknownError;
      own[i] = sp->owner[(size_t)l + 1][(size_t)par];
    }
  }
  // this shard's bricks, in encode order, parents re-indexed
  sp->local.levels.assign((size_t)L, {});
  for (int l = L - 1; l >= 0; --l)
  {
    const std::vector<brick_entry>& bl = plan.levels[(size_t)l];
    std::vector<int>& li = sp->local_index[(size_t)l];
    li.assign(bl.size(), -1);
    for (size_t i = 0; i < bl.size(); ++i)
      if (sp->owner[(size_t)l][i] == shard)
      {
        li[i] = (int)sp->local.levels[(size_t)l].size();
        brick_entry e = bl[i];
        if (l + 1 < L)
          e.parent = sp->local_index[(size_t)l + 1][(size_t)e.parent];
        sp->local.levels[(size_t)l].push_back(e);
      }
  }
  sp->local.events.clear();
  for (const encode_event& ev : plan.events)
    if (sp->owner[(size_t)ev.level][(size_t)ev.brick] == shard)
      sp->local.events.push_back({ ev.level, sp->local_index[(size_t)ev.level][(size_t)ev.brick], ev.subband });
  // the samples the shard's level-0 bricks cover
  v3 lo(1 << 30), hi(0);
  for (const brick_entry& e : sp->local.levels[0])
  {
    const v3 from = e.brick3 * f.brick_dims;
    lo = vmin(lo, from);
    hi = v3(std::max(hi.x, from.x + e.valid.x), std::max(hi.y, from.y + e.valid.y), std::max(hi.z, from.z + e.valid.z));
  }
  sp->region = sp->local.levels[0].empty() ? extent{ v3(0), v3(0) } : extent{ lo, hi - lo };
  return NoError;
}

namespace
{

std::vector<std::vector<int>> blocks_per_subband(const dataset_format& f)
{
  std::vector<std::vector<int>> nb((size_t)f.nlevels, std::vector<int>((size_t)f.nsubbands(), 0));
  std::vector<block_geom> g;
  for (int l = 0; l < f.nlevels; ++l)
    for (int s = 0; s < f.nsubbands(); ++s)
    {
      subband_blocks(f, l, s, &g);
      nb[(size_t)l][(size_t)s] = (int)g.size();
    }
  return nb;
}

} // namespace

int shard_headers(const dataset_format& f, const encode_plan& plan, const shard_plan& sp,
                  const std::vector<level_output>& outs, std::vector<uint8_t>* blob)
{
  blob->clear();
  const std::vector<std::vector<int>> nb = blocks_per_subband(f);
  const int nsb = f.nsubbands();
  for (const encode_event& ev : plan.events)
  {
    if (sp.owner[(size_t)ev.level][(size_t)ev.brick] != sp.shard)
      continue;
    const level_output& o = outs[(size_t)ev.level];
    const int li = sp.local_index[(size_t)ev.level][(size_t)ev.brick];
    const uint8_t* r = o.bytes() + o.offset[(size_t)li * (size_t)nsb + (size_t)ev.subband];
    int32_t nkeys;
    memcpy(&nkeys, r + 4, 4);
    const size_t hb = region_header_bytes(nb[(size_t)ev.level][(size_t)ev.subband], nkeys > 0 ? nkeys : 0);
    blob->insert(blob->end(), r, r + hb);
  }
  return NoError;
}

namespace
{

// Positional writes of the parts of one file this shard owns: its stream bytes (within
// `mine`), and, for shard 0, every byte the packer made. Neighbouring kept segments are
// written together.
int write_file_part(const std::string& path, const file_buffer& fb, bool made_bytes,
                    const std::vector<std::pair<const uint8_t*, const uint8_t*>>& mine)
{
  if (make_dirs_for(path) != NoError)
    return CannotCreateDirectory;
  const int fd = open(path.c_str(), O_RDWR | O_CREAT, 0644);
  if (fd < 0)
    return FileCreateFailed;
  int err = NoError;
  if (made_bytes && ftruncate(fd, (off_t)fb.nbytes) != 0)
    err = FileWriteFailed;
  auto is_mine = [&](const uint8_t* p) {
    for (const auto& r : mine)
      if (p >= r.first && p < r.second)
        return true;
    return false;
  };
  std::vector<uint8_t> buf;
  size_t buf_off = 0, off = 0;
  auto flush = [&]() {
    size_t done = 0;
    while (done < buf.size() && !err)
    {
      const ssize_t w = pwrite(fd, buf.data() + done, buf.size() - done, (off_t)(buf_off + done));
      if (w <= 0)
        err = FileWriteFailed;
      else
        done += (size_t)w;
    }
    buf.clear();
  };
  constexpr size_t kFlush = (size_t)16 << 20;
  fb.for_each_segment([&](const segment& s) {
    const bool keep = s.p && s.n && (is_mine(s.p) ? true : made_bytes);
    if (keep)
    {
      if (buf.empty())
        buf_off = off;
      buf.insert(buf.end(), s.p, s.p + s.n);
      if (buf.size() >= kFlush)
        flush();
    }
    else if (!buf.empty())
      flush();
    off += s.n;
  });
  if (!buf.empty())
    flush();
  if (close(fd) != 0 && !err)
    err = FileWriteFailed;
  return err;
}

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

} // namespace

int pack_shard(const dataset_format* f, const params* p, const encode_plan& plan, const shard_plan& sp,
               const std::vector<level_output>& outs, const std::vector<const uint8_t*>& blobs,
               const std::vector<size_t>& sizes, encode_timing* timing)
{
  const double t0 = now_s();
  if ((int)blobs.size() != sp.nshards || (int)sizes.size() != sp.nshards)
    return InvalidArgument;
  const std::vector<std::vector<int>> nb = blocks_per_subband(*f);
  const int nsb = f->nsubbands();
  std::vector<size_t> cur((size_t)sp.nshards, 0);
  std::vector<subband_result> rs(plan.events.size());
  // this shard's stream bytes, per level
  std::vector<std::pair<const uint8_t*, const uint8_t*>> mine;
  std::vector<size_t> level_end(outs.size(), 0);
  for (size_t i = 0; i < plan.events.size(); ++i)
  {
    const encode_event& ev = plan.events[i];
    subband_result& r = rs[i];
    r.level = ev.level;
    r.brick = plan.levels[(size_t)ev.level][(size_t)ev.brick].linear;
    r.subband = ev.subband;
    r.nexps = nb[(size_t)ev.level][(size_t)ev.subband];
    const int s = sp.owner[(size_t)ev.level][(size_t)ev.brick];
    if (s == sp.shard)
    {
      const level_output& o = outs[(size_t)ev.level];
      const int li = sp.local_index[(size_t)ev.level][(size_t)ev.brick];
      const uint64_t at = o.offset[(size_t)li * (size_t)nsb + (size_t)ev.subband];
      const region_view v = view_region(o.bytes() + at, r.nexps);
      r.exps = v.exps;
      r.kmin = v.kmin;
      r.kmax = v.kmax;
      r.sizes = v.sizes;
      r.bytes = v.bytes;
      size_t data = 0;
      for (int k = v.kmin; k <= v.kmax; ++k)
        data += v.sizes[k - v.kmin];
      level_end[(size_t)ev.level] = std::max(level_end[(size_t)ev.level], (size_t)(v.bytes - o.bytes()) + data);
      continue;
    }
    // another shard's region: its header from that shard's payload, no stream bytes
    const uint8_t* h = blobs[(size_t)s] + cur[(size_t)s];
    if (cur[(size_t)s] + 8 > sizes[(size_t)s])
      return CorruptStream;
    int32_t kmin, nkeys;
    memcpy(&kmin, h, 4);
    memcpy(&nkeys, h + 4, 4);
    if (nkeys < 0 || nkeys > kKeyWindow)
      return CorruptStream;
    const size_t hb = region_header_bytes(r.nexps, nkeys);
    if (cur[(size_t)s] + hb > sizes[(size_t)s])
      return CorruptStream;
    const region_view v = view_region(h, r.nexps);
    r.exps = v.exps;
    r.kmin = v.kmin;
    r.kmax = v.kmax;
    r.sizes = v.sizes;
    r.bytes = nullptr;
    cur[(size_t)s] += hb;
  }
  for (int s = 0; s < sp.nshards; ++s)
    if (s != sp.shard && cur[(size_t)s] != sizes[(size_t)s])
      return CorruptStream;  // a payload that does not match the plan
  for (size_t l = 0; l < outs.size(); ++l)
    if (level_end[l])
      mine.push_back({ outs[l].bytes(), outs[l].bytes() + level_end[l] });
  packer pk(*f, f->tolerance);
  int e = pk.add_all(std::move(rs));
  if (!e)
    e = pk.finish();
  if (e)
    return e;
  const double t1 = now_s();
  std::vector<std::pair<std::string, const file_buffer*>> list;
  for (auto& kv : pk.files())
    list.push_back({ kv.first, &kv.second });
  std::atomic<int> werr{ 0 };
  parallel_for(list.size(), [&](size_t i) {
    const int we = write_file_part(list[i].first, *list[i].second, sp.shard == 0, mine);
    if (we)
      werr = we;
  });
  if (werr)
    return werr;
  unsigned long long total = 0;
  for (auto& kv : list)
    total += kv.second->nbytes;
  if (sp.shard == 0)
  {
    const std::string meta = meta_text(*f, *p) + pk.stats_text();
    total += meta.size();
    e = write_file(p->out_dir + "/" + p->name + "/" + p->field + ".idx2", std::vector<uint8_t>(meta.begin(), meta.end()));
    if (e)
      return e;
  }
  if (timing)
  {
    timing->pack_s = t1 - t0;
    timing->write_s = now_s() - t1;
    timing->file_bytes = total;
    timing->nfiles = (int)list.size() + (sp.shard == 0);
  }
  return NoError;
}

} // namespace idx2g
