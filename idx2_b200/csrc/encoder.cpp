// Encode driver (Core/idx2Encode.cpp:276-444).
#include "encoder.h"
#include "parallel.h"
#include "trace.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <errno.h>
#include <fcntl.h>
#include <functional>
#include <sys/stat.h>
#include <unistd.h>
#include <thread>
#include <unordered_map>

namespace idx2g
{

static uint32_t spread3(uint32_t x)
{
  uint32_t r = 0;
  for (int i = 0; i < 10; ++i)
    r |= ((x >> i) & 1u) << (3 * i);
  return r;
}
static uint32_t compact3(uint32_t c)
{
  uint32_t r = 0;
  for (int i = 0; i < 10; ++i)
    r |= ((c >> (3 * i)) & 1u) << i;
  return r;
}

void subband_blocks(const dataset_format& f, int level, int sb, std::vector<block_geom>* out)
{
  out->clear();
  const subband& s = f.subbands[(size_t)sb];
  v3 nb = (s.g.dims + f.block_dims - v3(1)) / f.block_dims;
  uint32_t last = spread3((uint32_t)nb.x - 1) | (spread3((uint32_t)nb.y - 1) << 1) |
                  (spread3((uint32_t)nb.z - 1) << 2);
  for (uint32_t b = 0; b <= last; ++b)
  {
    v3 z3((int)compact3(b), (int)compact3(b >> 1), (int)compact3(b >> 2));
    if (!all_lt(z3, nb))
    {
      // Core/idx2Common.h:23 idx2_NextMorton
      int lsb = __builtin_ctz(b);
      b = (((b >> (lsb + 1)) + 1) << (lsb + 1)) - 1;
      continue;
    }
    v3 d3 = z3 * f.block_dims;
    v3 bd = vmin(f.block_dims, s.g.dims - d3);
    bool coded_next = sb == 0 && level + 1 < f.nlevels && bd == f.block_dims;
    if (coded_next)
      continue;
    block_geom g;
    g.dx = (uint8_t)z3.x;
    g.dy = (uint8_t)z3.y;
    g.dz = (uint8_t)z3.z;
    g.bx = (uint8_t)bd.x;
    g.by = (uint8_t)bd.y;
    g.bz = (uint8_t)bd.z;
    g.code = (uint16_t)b;
    out->push_back(g);
  }
}

int make_encode_plan(const dataset_format& f, encode_plan* plan)
{
  const int L = f.nlevels;
  plan->levels.assign((size_t)L, {});
  plan->events.clear();
  // parents under construction: key (level, linear) -> entry + children waiting
  struct pending
  {
    brick_entry e;
    int ndone = 0;
    std::vector<std::pair<int, int>> children;  // (level, index)
  };
  std::vector<std::unordered_map<u64, pending>> pool((size_t)L);
  const v3 sb_nonext = v3(f.subbands[0].g.dims.x - (f.subbands[0].g.dims.x > 1),
                          f.subbands[0].g.dims.y - (f.subbands[0].g.dims.y > 1),
                          f.subbands[0].g.dims.z - (f.subbands[0].g.dims.z > 1));

  std::function<void(int, int)> encode_brick = [&](int level, int idx) {
    for (int sb = 0; sb < f.nsubbands(); ++sb)
    {
      if (sb == 0 && level + 1 < L)
      {
        brick_entry& me = plan->levels[(size_t)level][(size_t)idx];
        v3 pb3 = me.brick3 / f.group_brick3;
        u64 plin = linear_brick(f, level + 1, pb3);
        auto& pm = pool[(size_t)level + 1];
        auto it = pm.find(plin);
        if (it == pm.end())
        {
          pending p;
          p.e.brick3 = pb3;
          p.e.linear = plin;
          v3 from3 = pb3 * f.group_brick3;
          extent c = crop(extent{ from3, f.group_brick3 }, extent{ v3(0), f.nbricks3[(size_t)level] });
          p.e.nchildren = (int)prod(c.dims);
          p.e.valid = c.dims * sb_nonext;
          it = pm.emplace(plin, p).first;
        }
        me.pos_in_parent = me.brick3 % f.group_brick3;
        it->second.children.push_back({ level, idx });
        if (++it->second.ndone == it->second.e.nchildren)
        {
          int pidx = (int)plan->levels[(size_t)level + 1].size();
          plan->levels[(size_t)level + 1].push_back(it->second.e);
          for (auto& ch : it->second.children)
            plan->levels[(size_t)ch.first][(size_t)ch.second].parent = pidx;
          pm.erase(it);
          encode_brick(level + 1, pidx);
        }
      }
      plan->events.push_back({ level, idx, sb });
    }
  };

  const v3 nb0 = f.nbricks3[0];
  extent all{ v3(0), nb0 };
  traverse(f.bricks_order[0], v3(0), nb0, all, all, [&](const traverse_item& t) {
    brick_entry e;
    e.brick3 = t.from3;
    e.linear = linear_brick(f, 0, t.from3);
    extent be{ t.from3 * f.brick_dims, f.brick_dims };
    extent c = crop(be, extent{ v3(0), f.dims });
    e.valid = c.dims;
    int idx = (int)plan->levels[0].size();
    plan->levels[0].push_back(e);
    encode_brick(0, idx);
  });
  for (int l = 1; l < L; ++l)
    if (!pool[(size_t)l].empty())
      return UnknownError;
  return NoError;
}

int make_dirs_for(const std::string& path)
{
  size_t pos = 0;
  while ((pos = path.find('/', pos + 1)) != std::string::npos)
  {
    std::string d = path.substr(0, pos);
    if (d.empty())
      continue;
    if (mkdir(d.c_str(), 0755) != 0 && errno != EEXIST)
      return CannotCreateDirectory;
  }
  return NoError;
}

int write_file(const std::string& path, const std::vector<uint8_t>& data)
{
  if (make_dirs_for(path) != NoError)
    return CannotCreateDirectory;
  FILE* fp = fopen(path.c_str(), "wb");
  if (!fp)
    return FileCreateFailed;
  size_t n = data.empty() ? 0 : fwrite(data.data(), 1, data.size(), fp);
  fclose(fp);
  return n == data.size() ? NoError : FileWriteFailed;
}

static double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int encode_levels(dataset_format* f, brick_coder* coder, std::vector<level_output>* outs, const encode_plan& plan)
{
  int e = NoError;
  outs->assign((size_t)f->nlevels, level_output());
  for (int l = 0; l < f->nlevels; ++l)
  {
    e = coder->run_level(l, plan, &(*outs)[(size_t)l]);
    if (e)
      return e;
  }
  coder->value_range(&f->value_min, &f->value_max);
  return NoError;
}

std::thread preallocate_files(const dataset_format& f, const encode_plan& plan,
                              const std::vector<unsigned long long>& sizes)
{
  constexpr unsigned long long kMin = 64ull << 20;
  std::vector<std::pair<std::string, unsigned long long>> todo;
  for (int l = 0; l < f.nlevels && l < (int)sizes.size() && l < (int)plan.levels.size(); ++l)
    if (sizes[(size_t)l] >= kMin && !plan.levels[(size_t)l].empty())
      todo.push_back({ file_path(f, plan.levels[(size_t)l][0].linear, l), sizes[(size_t)l] });
  if (todo.empty())
    return std::thread();
  return std::thread([todo]() {
    stage_timer tt;
    // the writer sets each file's size and writes every byte, so pages of an older file of
    // the same name are as good as new ones
    for (const auto& t : todo)
    {
      if (make_dirs_for(t.first) != NoError)
        continue;
      const int fd = open(t.first.c_str(), O_RDWR | O_CREAT, 0644);
      if (fd < 0)
        continue;
      if (fallocate(fd, FALLOC_FL_KEEP_SIZE, 0, (off_t)t.second) != 0)
        errno = 0;
      close(fd);
    }
    tt.lap("write.prealloc (thread)");
  });
}

int encode_dataset(dataset_format* f, params* p, brick_coder* coder,
                   std::map<std::string, std::vector<uint8_t>>* files, bool write_files,
                   encode_timing* timing, const encode_plan* plan,
                   const std::vector<unsigned long long>* prealloc)
{
  double t0 = now_s();
  encode_plan local;
  if (!plan)
  {
    int e = make_encode_plan(*f, &local);
    if (e)
      return e;
    plan = &local;
  }
  std::thread pre;
  if (write_files && prealloc)
    pre = preallocate_files(*f, *plan, *prealloc);
  struct joiner
  {
    std::thread& t;
    ~joiner()
    {
      if (t.joinable())
        t.join();
    }
  } join_pre{ pre };
  std::vector<level_output> outs;
  int e = encode_levels(f, coder, &outs, *plan);
  if (e)
    return e;
  double t1 = now_s();
  e = pack_dataset(f, p, *plan, outs, files, write_files, timing, &pre);
  if (timing)
    timing->device_s = t1 - t0;
  return e;
}

// Bytes of every level's data file when each level has exactly one.
void note_level_files(const dataset_format& f, const encode_plan& plan, const std::map<std::string, file_buffer>& data,
                      encode_timing* timing)
{
  timing->level_file_bytes.clear();
  if ((int)data.size() != f.nlevels || (int)plan.levels.size() < f.nlevels)
    return;
  std::vector<unsigned long long> v((size_t)f.nlevels, 0);
  for (int l = 0; l < f.nlevels; ++l)
  {
    if (plan.levels[(size_t)l].empty())
      return;
    auto it = data.find(file_path(f, plan.levels[(size_t)l][0].linear, l));
    if (it == data.end())
      return;
    v[(size_t)l] = it->second.nbytes;
  }
  timing->level_file_bytes = v;
}

int pack_dataset(const dataset_format* f, const params* p, const encode_plan& plan,
                 const std::vector<level_output>& outs, std::map<std::string, std::vector<uint8_t>>* files,
                 bool write_files, encode_timing* timing, std::thread* before_write)
{
  double t1 = now_s();
  stage_timer tt;
  int e = NoError;
  packer pk(*f, f->tolerance);
  // the coder's regions, parsed in parallel, recorded in the plan's event order
  std::vector<subband_result> rs(plan.events.size());
  parallel_ranges(rs.size(), [&](size_t i0, size_t i1) {
    for (size_t i = i0; i < i1; ++i)
    {
      const encode_event& ev = plan.events[i];
      const level_output& o = outs[(size_t)ev.level];
      size_t bs = (size_t)ev.brick * (size_t)o.nsb + (size_t)ev.subband;
      subband_result& r = rs[i];
      r.level = ev.level;
      r.brick = plan.levels[(size_t)ev.level][(size_t)ev.brick].linear;
      r.subband = ev.subband;
      r.nexps = o.nexps[(size_t)ev.subband];
      region_view v = view_region(o.bytes() + o.offset[bs], r.nexps);
      r.exps = v.exps;
      r.kmin = v.kmin;
      r.kmax = v.kmax;
      r.sizes = v.sizes;
      r.bytes = v.bytes;
    }
  });
  e = pk.add_all(std::move(rs));
  if (e)
    return e;
  tt.lap("pack.events");
  e = pk.finish();
  if (e)
    return e;
  if (timing)
    note_level_files(*f, plan, pk.files(), timing);
  double t2 = now_s();
  return write_dataset(f, p, pk.files(), pk.stats_text(), files, write_files, timing, before_write, t2 - t1);
}

int write_dataset(const dataset_format* f, const params* p, std::map<std::string, file_buffer>& data,
                  const std::string& stats, std::map<std::string, std::vector<uint8_t>>* files, bool write_files,
                  encode_timing* timing, std::thread* before_write, double pack_s,
                  const std::function<void(const uint8_t*, size_t)>* ready)
{
  stage_timer tt;
  const double t2 = now_s();
  int e = NoError;
  std::string meta = meta_text(*f, *p) + stats;
  std::string meta_path = p->out_dir + "/" + p->name + "/" + p->field + ".idx2";
  std::vector<const std::pair<const std::string, file_buffer>*> list;
  unsigned long long total = meta.size();
  for (auto& kv : data)
  {
    list.push_back(&kv);
    total += kv.second.nbytes;
  }
  if (files)
  {
    files->clear();
    for (auto* kv : list)
    {
      std::vector<uint8_t>& d = (*files)[kv->first];
      d.reserve(kv->second.nbytes);
      kv->second.for_each_segment([&](const segment& s) {
        if (ready && *ready)
          (*ready)(s.p, s.n);
        d.insert(d.end(), s.p, s.p + s.n);
      });
    }
    (*files)[meta_path] = std::vector<uint8_t>(meta.begin(), meta.end());
  }
  if (write_files)
  {
    if (before_write && before_write->joinable())
      before_write->join();
    e = write_file(meta_path, std::vector<uint8_t>(meta.begin(), meta.end()));
    if (e)
      return e;
    std::vector<std::pair<std::string, const file_buffer*>> wl;
    wl.reserve(list.size());
    for (auto* kv : list)
      wl.push_back({ kv->first, &kv->second });
    tt.lap("write.meta");
    e = idx2g::write_files(wl, ready);
    if (e)
      return e;
    tt.lap("write.files");
  }
  double t3 = now_s();
  if (timing)
  {
    timing->pack_s = pack_s;
    timing->write_s = t3 - t2;
    timing->file_bytes = total;
    timing->nfiles = (int)list.size() + 1;
  }
  return NoError;
}

} // namespace idx2g
