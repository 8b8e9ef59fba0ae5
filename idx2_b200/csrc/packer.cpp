// Chunk/file packer (Core/idx2Write.cpp, Core/idx2Encode.cpp:41-137,233-249).
#include "packer.h"
#include "zstd_frame.h"

#include "encoder.h"
#include "parallel.h"
#include "trace.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <mutex>
#include <thread>
#include <unistd.h>

namespace idx2g
{

// ----------------------------------------------------------------------------
// bit writer
// ----------------------------------------------------------------------------

void bit_writer::put(uint64_t v, int n)
{
  if (n <= 0)
    return;
  if (n < 64)
    v &= ((uint64_t)1 << n) - 1;
  const size_t byte = (size_t)(nbits >> 3);
  const int off = (int)(nbits & 7);
  if (bytes.size() < byte + 16)
    bytes.resize(std::max(byte + 16, bytes.size() * 2), 0);
  // n <= 57 and off <= 7: the bits fit one little-endian 64-bit word at `byte`
  uint64_t w;
  memcpy(&w, bytes.data() + byte, 8);
  w |= v << off;
  memcpy(bytes.data() + byte, &w, 8);
  nbits += (uint64_t)n;
}

void bit_writer::put_varbyte(uint64_t v)
{
  if ((nbits & 7) == 0)
  {
    // byte-aligned (every size stream): the bytes go in whole
    const size_t byte = (size_t)(nbits >> 3);
    if (bytes.size() < byte + 16)
      bytes.resize(std::max(byte + 16, bytes.size() * 2), 0);
    uint8_t* d = bytes.data() + byte;
    size_t n = 0;
    do
    {
      const uint64_t more = (v >> 7) != 0;
      d[n++] = (uint8_t)((v & 0x7F) | (more << 7));
      v >>= 7;
    } while (v && n < 10);
    nbits += 8 * (uint64_t)n;
    return;
  }
  for (;;)
  {
    uint64_t more = (v >> 7) != 0;
    put((v & 0x7F) | (more << 7), 8);
    v >>= 7;
    if (!more)
      break;
  }
}

void bit_writer::put_unary(uint64_t v)
{
  // v zero bits (the buffer is zero-filled ahead of nbits), then a one bit
  nbits += v;
  put(1, 1);
}

double pack_stats::acc::sd() const
{
  double a = avg();
  return sqrt(ssq / (double)n - a * a);
}

// ----------------------------------------------------------------------------
// zstd: frames written by zstd_frame.cpp, read through the system library
// ----------------------------------------------------------------------------

namespace
{
struct zstd_api
{
  size_t (*compress)(void*, size_t, const void*, size_t, int) = nullptr;
  size_t (*bound)(size_t) = nullptr;
  size_t (*decompress)(void*, size_t, const void*, size_t) = nullptr;
  unsigned long long (*content_size)(const void*, size_t) = nullptr;
  unsigned (*is_error)(size_t) = nullptr;
  const char* (*version)() = nullptr;
  bool ok = false;
  zstd_api()
  {
    void* h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!h)
      h = dlopen("libzstd.so", RTLD_NOW | RTLD_LOCAL);
    if (!h)
      return;
    compress = (decltype(compress))dlsym(h, "ZSTD_compress");
    bound = (decltype(bound))dlsym(h, "ZSTD_compressBound");
    decompress = (decltype(decompress))dlsym(h, "ZSTD_decompress");
    content_size = (decltype(content_size))dlsym(h, "ZSTD_getFrameContentSize");
    is_error = (decltype(is_error))dlsym(h, "ZSTD_isError");
    version = (decltype(version))dlsym(h, "ZSTD_versionString");
    ok = compress && bound && decompress && content_size && is_error;
  }
};
zstd_api& zapi()
{
  static zstd_api a;
  return a;
}
} // namespace

const char* zstd_version()
{
  return zapi().version ? zapi().version() : "unavailable";
}

int zstd_compress(const uint8_t* src, size_t n, std::vector<uint8_t>* out)
{
  // Core/idx2Encode.cpp:23 CompressBufZstd: empty input gives an empty output; otherwise one
  // level-1 frame, byte-identical to the reference's vendored zstd 1.4.5 (zstd_frame.cpp)
  out->clear();
  if (n == 0)
    return NoError;
  zstd145::compress(src, n, out);
  return NoError;
}

int zstd_decompress(const uint8_t* src, size_t n, std::vector<uint8_t>* out)
{
  out->clear();
  if (n == 0)
    return NoError;
  if (!zapi().ok)
    return UnknownError;
  unsigned long long sz = zapi().content_size(src, n);
  if (sz == ~0ull || sz == ~0ull - 1)
    return CorruptStream;
  out->resize((size_t)sz);
  size_t r = zapi().decompress(out->data(), (size_t)sz, src, n);
  if (zapi().is_error(r) || r != sz)
    return CorruptStream;
  return NoError;
}

int exponent_f64(double v)
{
  if (v != 0)
  {
    int e;
    frexp(v, &e);
    return e > -1022 ? e : -1022;
  }
  return -1023;
}

// ----------------------------------------------------------------------------
// files
// ----------------------------------------------------------------------------

void file_buffer::append_owned(std::vector<uint8_t>&& v)
{
  if (v.empty())
    return;
  owned.push_back(std::move(v));
  append_ref(owned.back().data(), owned.back().size());
}

void file_buffer::append_ref(const uint8_t* p, size_t n)
{
  if (!n)
    return;
  singles.push_back({ p, n });
  append_run(&singles.back(), 1, n);
}

void file_buffer::append_run(const segment* s, size_t n, size_t bytes)
{
  if (!bytes)
    return;
  parts.push_back({ s, n, bytes });
  nbytes += bytes;
}

namespace
{

// Unmaps a written file's mapping on a thread of its own (tearing down the page tables of a
// 1 GB mapping takes some 15 ms); one at a time, the last one joined at exit.
struct unmapper
{
  std::mutex m;
  std::thread t;
  void later(uint8_t* p, size_t n)
  {
    std::lock_guard<std::mutex> g(m);
    if (t.joinable())
      t.join();
    t = std::thread([p, n]() { munmap(p, n); });
  }
  ~unmapper()
  {
    if (t.joinable())
      t.join();
  }
};

unmapper& unmap_queue()
{
  static unmapper u;
  return u;
}

} // namespace

int write_files(const std::vector<std::pair<std::string, const file_buffer*>>& files, const ready_fn* ready)
{
  // Every file is cut into ranges of whole runs of about kRange bytes, copied by a pool of
  // threads. Large files are written through a shared mapping (writes to one file through
  // write(2) are serialised by the kernel), their pages allocated up front in one call where
  // the file system allows it (page faults of the copies then find the pages in place);
  // small files, and any file that cannot be mapped, with pwrite from a staging buffer.
  constexpr size_t kRange = (size_t)16 << 20;
  constexpr size_t kMapMin = (size_t)64 << 20;
  struct range
  {
    int file;
    size_t p0, p1, offset, bytes;
  };
  std::vector<int> fds(files.size(), -1);
  std::vector<uint8_t*> maps(files.size(), nullptr);
  std::vector<size_t> map_len(files.size(), 0);
  std::vector<range> ranges;
  int err = NoError;
  // opens file i (its size set and pages allocated when it is mapped); 0 or an error code
  auto open_file = [&](size_t i, size_t total) -> int {
    if (make_dirs_for(files[i].first) != NoError)
      return CannotCreateDirectory;
    // a large file keeps the pages it has (every byte is written, the size set first)
    fds[i] = open(files[i].first.c_str(), O_RDWR | O_CREAT | (total >= kMapMin ? 0 : O_TRUNC), 0644);
    if (fds[i] < 0)
      return FileCreateFailed;
    if (total < kMapMin)
      return NoError;
    if (ftruncate(fds[i], (off_t)total) != 0)
      return FileWriteFailed;
    // pages for the whole file in one call, unless it has them already (allocated ahead, or
    // an older file's): a second allocation over allocated pages costs more than it saves
    struct stat sb;
    if ((fstat(fds[i], &sb) != 0 || (size_t)sb.st_blocks * 512 < total) && fallocate(fds[i], 0, 0, (off_t)total) != 0)
      errno = 0;  // pages come with the copies' page faults instead
    void* m = mmap(nullptr, total, PROT_WRITE, MAP_SHARED, fds[i], 0);
    if (m != MAP_FAILED)
    {
      maps[i] = (uint8_t*)m;
      map_len[i] = total;
    }
    else if (ftruncate(fds[i], 0) != 0)
      return FileWriteFailed;
    return NoError;
  };
  for (size_t i = 0; i < files.size() && !err; ++i)
  {
    if ((err = open_file(i, files[i].second->nbytes)) != NoError)
      break;
    const std::vector<segment_run>& parts = files[i].second->parts;
    size_t off = 0, start = 0, acc = 0;
    for (size_t k = 0; k < parts.size(); ++k)
    {
      acc += parts[k].bytes;
      if (acc >= kRange || k + 1 == parts.size())
      {
        ranges.push_back({ (int)i, start, k + 1, off, acc });
        off += acc;
        start = k + 1;
        acc = 0;
      }
    }
  }
  if (!err)
  {
    std::atomic<size_t> next{ 0 };
    std::atomic<int> werr{ 0 };
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt ? (nt > 16 ? 16 : nt) : 4;
    if (nt > ranges.size())
      nt = ranges.empty() ? 1 : (unsigned)ranges.size();
    auto work = [&]() {
      std::vector<uint8_t> stage;
      for (size_t i; (i = next.fetch_add(1)) < ranges.size();)
      {
        const range& r = ranges[i];
        const std::vector<segment_run>& parts = files[(size_t)r.file].second->parts;
        auto gather = [&](uint8_t* dst) {
          for (size_t k = r.p0; k < r.p1; ++k)
            for (size_t j = 0; j < parts[k].nseg; ++j)
            {
              if (ready && *ready)
                (*ready)(parts[k].seg[j].p, parts[k].seg[j].n);
              memcpy(dst, parts[k].seg[j].p, parts[k].seg[j].n);
              dst += parts[k].seg[j].n;
            }
        };
        if (maps[(size_t)r.file])
        {
          gather(maps[(size_t)r.file] + r.offset);
          continue;
        }
        const uint8_t* src;
        if (r.p1 - r.p0 == 1 && parts[r.p0].nseg == 1)
        {
          src = parts[r.p0].seg[0].p;
          if (ready && *ready)
            (*ready)(src, parts[r.p0].seg[0].n);
        }
        else
        {
          stage.resize(r.bytes);
          gather(stage.data());
          src = stage.data();
        }
        size_t done = 0;
        while (done < r.bytes)
        {
          ssize_t w = pwrite(fds[(size_t)r.file], src + done, r.bytes - done, (off_t)(r.offset + done));
          if (w <= 0)
          {
            werr = FileWriteFailed;
            break;
          }
          done += (size_t)w;
        }
      }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t)
      th.emplace_back(work);
    work();
    for (auto& t : th)
      t.join();
    err = werr;
  }
  for (size_t i = 0; i < files.size(); ++i)
    if (maps[i])
      unmap_queue().later(maps[i], map_len[i]);
  for (int fd : fds)
    if (fd >= 0 && close(fd) != 0 && !err)
      err = FileWriteFailed;
  return err;
}

// ----------------------------------------------------------------------------
// packer
// ----------------------------------------------------------------------------

namespace
{

constexpr uint64_t kFinalFlush = ~0ull;  // stamp of the writes of the final flushes

struct channel
{
  bit_writer deltas, sizes;
  std::vector<segment> bricks;
  size_t brick_bytes = 0;
  u64 last_chunk = 0, last_brick = 0;
  int nbricks = 0;
  int bpkey = 0;
};

struct chunk_rec
{
  uint64_t event;
  uint32_t rank;
  int bpkey;
  u64 last_brick;
  std::vector<segment> parts;  // header (owned by the group), then brick data
  size_t bytes;
  double deltas_bytes, sizes_bytes;
};

struct exp_rec
{
  uint64_t event;
  uint32_t rank;
  u64 last_brick;
  std::vector<uint8_t> raw, z;
};

template <typename T>
bool stamp_less(const T* a, const T* b)
{
  return a->event != b->event ? a->event < b->event : a->rank < b->rank;
}

} // namespace

struct packer::group
{
  int level = 0, subband = 0;
  std::vector<uint32_t> events;  // indices into packer::events_, in order
  std::vector<int32_t> index;    // bpkey -> channel, -1
  std::deque<channel> chans;
  std::vector<uint8_t> brick_exps;
  u64 exp_last_chunk = 0, exp_last_brick = 0;
  std::deque<std::vector<uint8_t>> owned;
  std::vector<chunk_rec> chunks;
  std::vector<exp_rec> exps;

  channel& chan(int bpkey)
  {
    int32_t& i = index[(size_t)bpkey];
    if (i < 0)
    {
      i = (int32_t)chans.size();
      chans.emplace_back();
      chans.back().bpkey = bpkey;
    }
    return chans[(size_t)i];
  }

  // Core/idx2Write.cpp:221 WriteChunk: varbyte NBricks | deltas | sizes | brick data
  void write_chunk(channel& c, uint64_t event, uint32_t rank)
  {
    bit_writer head;
    head.put_varbyte((uint64_t)c.nbricks);
    owned.emplace_back();
    std::vector<uint8_t>& meta = owned.back();
    meta.reserve(head.size() + c.deltas.size() + c.sizes.size());
    meta.insert(meta.end(), head.bytes.begin(), head.bytes.begin() + (long)head.size());
    meta.insert(meta.end(), c.deltas.bytes.begin(), c.deltas.bytes.begin() + (long)c.deltas.size());
    meta.insert(meta.end(), c.sizes.bytes.begin(), c.sizes.bytes.begin() + (long)c.sizes.size());
    chunk_rec r;
    r.event = event;
    r.rank = rank;
    r.bpkey = c.bpkey;
    r.last_brick = c.last_brick;
    r.bytes = meta.size() + c.brick_bytes;
    r.deltas_bytes = (double)c.deltas.size();
    r.sizes_bytes = (double)c.sizes.size();
    r.parts.reserve(c.bricks.size() + 1);
    if (!meta.empty())
      r.parts.push_back({ meta.data(), meta.size() });
    for (const segment& sg : c.bricks)
      r.parts.push_back(sg);
    chunks.push_back(std::move(r));
    c.deltas.clear();
    c.sizes.clear();
    c.bricks.clear();
    c.brick_bytes = 0;
  }

  // Core/idx2Write.cpp:38 WriteChunkExponents (compression deferred)
  void write_exps(uint64_t event, uint32_t rank)
  {
    exp_rec r;
    r.event = event;
    r.rank = rank;
    r.last_brick = exp_last_brick;
    r.raw.swap(brick_exps);
    brick_exps.clear();
    exps.push_back(std::move(r));
  }
};

packer::packer(const dataset_format& f, double tolerance) : f_(f), tol_(tolerance)
{
  etol_ = exponent_f64(tolerance);
}

packer::~packer() = default;

int packer::add(const subband_result& r)
{
  if (r.level < 0 || r.level >= 16 || r.subband < 0 || r.subband >= 64)
    return InvalidArgument;
  events_.push_back(r);
  return NoError;
}

int packer::add_all(std::vector<subband_result>&& rs)
{
  for (const subband_result& r : rs)
    if (r.level < 0 || r.level >= 16 || r.subband < 0 || r.subband >= 64)
      return InvalidArgument;
  if (events_.empty())
    events_ = std::move(rs);
  else
    events_.insert(events_.end(), rs.begin(), rs.end());
  return NoError;
}

static void put_i32(std::vector<uint8_t>* v, int32_t x)
{
  uint8_t b[4];
  memcpy(b, &x, 4);
  v->insert(v->end(), b, b + 4);
}

// ----------------------------------------------------------------------------
// channel state machine
// ----------------------------------------------------------------------------

namespace
{

bool pack_sequential()
{
  static const bool on = std::getenv("IDX2G_PACK_SEQUENTIAL") != nullptr;
  return on;
}

constexpr int kKeySpace = 4096;  // bit-plane keys are 12-bit (Core/idx2Lookup.h:21)

struct machine
{
  const std::vector<subband_result>& events;
  const dataset_format& f;
  int etol, end_bp, bpc;

  // keys of r's coded planes in first-touch order: blocks in Morton order, planes top-down
  void touch_order(const subband_result& r, std::vector<int>* order, std::vector<char>* seen) const
  {
    order->clear();
    if (r.kmin > r.kmax)
      return;
    seen->assign((size_t)(r.kmax - r.kmin + 1), 0);
    for (int b = 0; b < r.nexps; ++b)
    {
      const int emax = r.exps[b];
      for (int bp = 63; bp >= 64 - end_bp; --bp)
      {
        if (!plane_coded(bp, emax, etol, bpc))
          break;
        const int key = (bp + emax + 1024) / bpc;
        if (key < r.kmin || key > r.kmax)
          continue;
        char& sn = (*seen)[(size_t)(key - r.kmin)];
        if (!sn)
        {
          sn = 1;
          order->push_back(key);
        }
      }
    }
  }

  // exponents of one brick (Core/idx2Encode.cpp:41 EncodeBrickSubbandExponents)
  void append_exps(const subband_result& r, std::vector<uint8_t>* out) const
  {
    const size_t at = out->size();
    if (f.type == dtype::float64)
    {
      out->resize(at + 2 * (size_t)r.nexps);
      for (int i = 0; i < r.nexps; ++i)
      {
        const uint16_t v = (uint16_t)(r.exps[i] + 1023);
        (*out)[at + 2 * (size_t)i] = (uint8_t)(v & 0xFF);
        (*out)[at + 2 * (size_t)i + 1] = (uint8_t)(v >> 8);
      }
    }
    else
    {
      out->resize(at + (size_t)r.nexps);
      for (int i = 0; i < r.nexps; ++i)
        (*out)[at + (size_t)i] = (uint8_t)(r.exps[i] + 127);
    }
  }
};

// brick metadata and data of one channel (Core/idx2Encode.cpp:84)
inline void append_brick(channel& c, u64 brick, const uint8_t* p, uint32_t nb)
{
  if (c.nbricks == 0)
    c.deltas.put_varbyte(brick);
  else
    c.deltas.put_unary(brick - c.last_brick - 1);
  c.sizes.put_varbyte(nb);
  c.bricks.push_back({ p, nb });
  c.brick_bytes += nb;
  ++c.nbricks;
  c.last_brick = brick;
}

inline bool bad_keys(const subband_result& r)
{
  return r.kmin <= r.kmax && (r.kmin < 0 || r.kmax >= kKeySpace);
}

// The state machine of one group, event by event.
int run_group(packer::group& g, const machine& m)
{
  const int L = g.level;
  const u64 bpc_bricks = (u64)m.f.bricks_per_chunk[(size_t)L];
  const int shift = log2_ceil(m.f.bricks_per_chunk[(size_t)L]);
  std::vector<int> order;
  std::vector<char> seen;
  for (uint32_t ei : g.events)
  {
    const subband_result& r = m.events[ei];
    const u64 brick = r.brick;
    if (bad_keys(r))
      return InvalidArgument;
    // pass 1: channels in first-touch order; a channel entering a new chunk flushes the
    // previous one
    bool any_new = false;
    for (int k = r.kmin; k <= r.kmax && !any_new; ++k)
    {
      if (!r.sizes[k - r.kmin])
        continue;
      const int32_t ci = g.index[(size_t)k];
      const u64 last_chunk = ci >= 0 ? g.chans[(size_t)ci].last_chunk : 0;
      any_new = brick >= (last_chunk + 1) * bpc_bricks;
    }
    if (any_new)
    {
      m.touch_order(r, &order, &seen);
      uint32_t rank = 0;
      for (int k : order)
      {
        channel& c = g.chan(k);
        if (brick >= (c.last_chunk + 1) * bpc_bricks)
        {
          if (c.brick_bytes)
            g.write_chunk(c, ei, rank++);
          c.nbricks = 0;
          c.last_chunk = brick >> shift;
        }
      }
    }
    // exponents: a brick in a new chunk flushes the previous exponent chunk
    if (brick >= (g.exp_last_chunk + 1) * bpc_bricks)
    {
      g.write_exps(ei, 0);
      g.exp_last_chunk = brick >> shift;
    }
    m.append_exps(r, &g.brick_exps);
    g.exp_last_brick = brick;
    // pass 2: brick metadata and data per channel
    size_t off = 0;
    for (int k = r.kmin; k <= r.kmax; ++k)
    {
      const uint32_t nb = r.sizes[k - r.kmin];
      if (!nb)
        continue;
      append_brick(g.chan(k), brick, r.bytes ? r.bytes + off : nullptr, nb);
      off += nb;
    }
  }
  return NoError;
}

// The events of one group that fall in one chunk, run on their own. With bricks in chunk order,
// every channel's state at the range's start is the same for the sequential machine: a channel
// not yet seen in the range enters it at its first touch (flushing what it holds, with the
// stamp of that event and its place in the touch order), and its data in the range is a
// chunk of its own; the exponents of the range are one exponent chunk. merge_segments applies
// the ranges to the group in order.
struct seg_key
{
  channel ch;  // the range's data (after the channel entered)
  bool entered = false;
  uint64_t event = 0;
  uint32_t rank = 0;
};

struct segment_run
{
  packer::group* g = nullptr;
  size_t e0 = 0, e1 = 0;  // entries of g->events
  u64 chunk = 0;
  std::vector<seg_key> keys;  // references into it live within one event
  std::vector<uint8_t> exps;
  u64 exp_last_brick = 0;
  int status = NoError;  // NoError, InvalidArgument, or -1: the range needs the sequential machine
};

void run_segment(segment_run& s, const machine& m)
{
  thread_local std::vector<int32_t> index;
  if (index.empty())
    index.assign(kKeySpace, -1);
  s.keys.reserve(64);
  s.exps.reserve((size_t)(s.e1 - s.e0) * 128);
  auto key = [&](int k) -> seg_key& {
    int32_t& i = index[(size_t)k];
    if (i < 0)
    {
      i = (int32_t)s.keys.size();
      s.keys.emplace_back();
      s.keys.back().ch.bpkey = k;
    }
    return s.keys[(size_t)i];
  };
  std::vector<int> order;
  std::vector<char> seen;
  for (size_t i = s.e0; i < s.e1 && s.status == NoError; ++i)
  {
    const uint32_t ei = s.g->events[i];
    const subband_result& r = m.events[ei];
    const u64 brick = r.brick;
    if (bad_keys(r))
    {
      s.status = InvalidArgument;
      break;
    }
    if (s.chunk >= 1)
    {
      bool any_new = false;
      for (int k = r.kmin; k <= r.kmax && !any_new; ++k)
        any_new = r.sizes[k - r.kmin] && (index[(size_t)k] < 0 || !s.keys[(size_t)index[(size_t)k]].entered);
      if (any_new)
      {
        m.touch_order(r, &order, &seen);
        for (size_t pos = 0; pos < order.size(); ++pos)
        {
          seg_key& st = key(order[pos]);
          if (!st.entered)
          {
            st.entered = true;
            st.event = ei;
            st.rank = (uint32_t)pos;
          }
        }
      }
    }
    m.append_exps(r, &s.exps);
    s.exp_last_brick = brick;
    size_t off = 0;
    for (int k = r.kmin; k <= r.kmax; ++k)
    {
      const uint32_t nb = r.sizes[k - r.kmin];
      if (!nb)
        continue;
      seg_key& st = key(k);
      if (s.chunk >= 1 && !st.entered)
      {
        s.status = -1;  // data of a channel that did not enter: not separable
        break;
      }
      append_brick(st.ch, brick, r.bytes ? r.bytes + off : nullptr, nb);
      off += nb;
    }
  }
  for (const seg_key& st : s.keys)
    index[(size_t)st.ch.bpkey] = -1;
}

void merge_segments(packer::group& g, std::vector<segment_run>& segs)
{
  for (segment_run& s : segs)
  {
    if (s.chunk >= 1)
      g.write_exps(g.events[s.e0], 0);
    for (seg_key& st : s.keys)
    {
      channel& c = g.chan(st.ch.bpkey);
      if (st.entered)
      {
        if (c.brick_bytes)
          g.write_chunk(c, st.event, st.rank);
        c.nbricks = 0;
      }
      if (st.ch.nbricks)
      {
        c.deltas = std::move(st.ch.deltas);
        c.sizes = std::move(st.ch.sizes);
        c.bricks = std::move(st.ch.bricks);
        c.brick_bytes = st.ch.brick_bytes;
        c.nbricks = st.ch.nbricks;
        c.last_brick = st.ch.last_brick;
      }
    }
    g.brick_exps = std::move(s.exps);
    g.exp_last_brick = s.exp_last_brick;
  }
}

int run_machines(std::vector<std::unique_ptr<packer::group>>& groups, const machine& m, bool by_chunk)
{
  // chunk ranges of every group whose bricks come in chunk order
  std::vector<std::vector<segment_run>> segs(groups.size());
  std::vector<std::pair<size_t, size_t>> tasks;
  if (by_chunk)
    for (size_t gi = 0; gi < groups.size(); ++gi)
    {
      packer::group& g = *groups[gi];
      const int shift = log2_ceil(m.f.bricks_per_chunk[(size_t)g.level]);
      std::vector<segment_run>& v = segs[gi];
      bool ordered = true;
      for (size_t i = 0; i < g.events.size() && ordered; ++i)
      {
        const u64 c = m.events[g.events[i]].brick >> shift;
        if (v.empty() || c != v.back().chunk)
        {
          ordered = v.empty() || c > v.back().chunk;
          v.emplace_back();
          v.back().g = &g;
          v.back().e0 = i;
          v.back().chunk = c;
        }
        v.back().e1 = i + 1;
      }
      if (!ordered)
        v.clear();
      for (size_t k = 0; k < v.size(); ++k)
        tasks.push_back({ gi, k });
    }
  parallel_for(tasks.size(), [&](size_t t) { run_segment(segs[tasks[t].first][tasks[t].second], m); });
  std::atomic<int> err{ 0 };
  std::atomic<int> merged{ 0 };
  parallel_for(groups.size(), [&](size_t gi) {
    bool separable = !segs[gi].empty();
    for (const segment_run& s : segs[gi])
    {
      if (s.status > 0)
        err = s.status;
      separable = separable && s.status == NoError;
    }
    if (separable)
    {
      merge_segments(*groups[gi], segs[gi]);
      ++merged;
    }
    else if (int e = run_group(*groups[gi], m))
      err = e;
  });
  if (trace_on())
    fprintf(stderr, "idx2g pack.groups_by_chunk %d of %zu (%zu ranges)\n", merged.load(), groups.size(), tasks.size());
  return err;
}

} // namespace

int packer::finish()
{
  stage_timer tt;
  // events by (level, subband), in order
  {
    std::map<std::pair<int, int>, size_t> gi;
    for (size_t e = 0; e < events_.size(); ++e)
    {
      const subband_result& r = events_[e];
      auto it = gi.find({ r.level, r.subband });
      if (it == gi.end())
      {
        it = gi.emplace(std::make_pair(r.level, r.subband), groups_.size()).first;
        groups_.emplace_back(new group());
        groups_.back()->level = r.level;
        groups_.back()->subband = r.subband;
        groups_.back()->index.assign(kKeySpace, -1);
      }
      groups_[it->second]->events.push_back((uint32_t)e);
    }
  }
  const int end_bp = f_.type == dtype::float32 ? 32 : 64;
  const int bpc = f_.bit_planes_per_chunk;
  std::atomic<int> err{ 0 };
  tt.lap("pack.groups");

  // the state machine of every (level, subband) (Core/idx2Encode.cpp:41-137, :157-249): over
  // the group's chunk ranges in parallel where the group allows it, else in event order
  const machine m{ events_, f_, etol_, end_bp, bpc };
  int e = run_machines(groups_, m, !pack_sequential());
  if (e)
    return e;
  tt.lap("pack.channels");

  // FlushChunks (Core/idx2Write.cpp:317): every channel in channel-key order
  {
    struct ref
    {
      uint32_t key;
      group* g;
      channel* c;
    };
    std::vector<ref> all;
    for (auto& g : groups_)
      for (channel& c : g->chans)
        all.push_back({ channel_key(c.bpkey, g->level, g->subband), g.get(), &c });
    std::sort(all.begin(), all.end(), [](const ref& a, const ref& b) { return a.key < b.key; });
    for (size_t i = 0; i < all.size(); ++i)
      all[i].g->write_chunk(*all[i].c, kFinalFlush, (uint32_t)i);
  }
  // FlushChunkExponents (:121): sub-channels by level descending, then subband
  {
    std::vector<group*> gs;
    for (auto& g : groups_)
      gs.push_back(g.get());
    std::stable_sort(gs.begin(), gs.end(), [](const group* a, const group* b) {
      if (a->level == b->level)
        return a->subband < b->subband;
      return a->level > b->level;
    });
    for (size_t i = 0; i < gs.size(); ++i)
      gs[i]->write_exps(kFinalFlush, (uint32_t)i);
  }

  tt.lap("pack.flush");
  // bit-plane chunks in the sequential order: statistics and files
  struct chunk_ref
  {
    const chunk_rec* c;
    int level, subband;
  };
  std::vector<chunk_ref> chunks;
  for (auto& g : groups_)
    for (const chunk_rec& c : g->chunks)
      chunks.push_back({ &c, g->level, g->subband });
  std::sort(chunks.begin(), chunks.end(),
            [](const chunk_ref& a, const chunk_ref& b) { return stamp_less(a.c, b.c); });
  for (const chunk_ref& cr : chunks)
  {
    const chunk_rec& c = *cr.c;
    stats_.brick_deltas.add(c.deltas_bytes);
    stats_.brick_sizes.add(c.sizes_bytes);
    stats_.bit_plane_chunks.add((double)c.bytes);
    file_buffer& fb = files_[file_path(f_, c.last_brick, cr.level)];
    fb.append_run(c.parts.data(), c.parts.size(), c.bytes);
    fb.has_chunks = true;
    fb.chunk_sizes.put_varbyte(c.bytes);
    fb.chunk_addrs.push_back(chunk_address(f_, c.last_brick, cr.level, cr.subband, c.bpkey));
  }
  tt.lap("pack.chunk_files");
  // exponent chunks in the sequential order, compressed in parallel
  struct exp_ref
  {
    exp_rec* e;
    int level, subband;
  };
  std::vector<exp_ref> exps;
  for (auto& g : groups_)
    for (exp_rec& e : g->exps)
      exps.push_back({ &e, g->level, g->subband });
  std::sort(exps.begin(), exps.end(), [](const exp_ref& a, const exp_ref& b) { return stamp_less(a.e, b.e); });
  for (const exp_ref& er : exps)
    stats_.exp_chunks_raw.add((double)er.e->raw.size());
  parallel_for(exps.size(), [&](size_t i) {
    if (zstd_compress(exps[i].e->raw.data(), exps[i].e->raw.size(), &exps[i].e->z))
      err = UnknownError;
  });
  if (err)
    return err;
  for (const exp_ref& er : exps)
  {
    stats_.exp_chunks_z.add((double)er.e->z.size());
    file_buffer& fb = files_[file_path(f_, er.e->last_brick, er.level)];
    fb.has_exps = true;
    fb.exp_parts.push_back({ er.e->z.data(), er.e->z.size() });
    fb.exp_addrs.push_back(chunk_address(f_, er.e->last_brick, er.level, er.subband, 0));
  }

  tt.lap("pack.exponents");
  // file tails
  for (auto& kv : files_)
  {
    file_buffer& fb = kv.second;
    if (!fb.has_chunks)
      continue;
    const size_t n = fb.chunk_sizes.size();
    stats_.chunk_sizes.add((double)n);
    std::vector<uint8_t> tail(fb.chunk_sizes.bytes.begin(), fb.chunk_sizes.bytes.begin() + (long)n);
    put_i32(&tail, (int32_t)n);
    std::vector<uint8_t> z;
    int e = zstd_compress((const uint8_t*)fb.chunk_addrs.data(), fb.chunk_addrs.size() * 8, &z);
    if (e)
      return e;
    tail.insert(tail.end(), z.begin(), z.end());
    put_i32(&tail, (int32_t)z.size());
    put_i32(&tail, (int32_t)fb.chunk_addrs.size());
    stats_.chunk_addrs_raw.add((double)fb.chunk_addrs.size() * 8);
    stats_.chunk_addrs_z.add((double)z.size());
    fb.append_owned(std::move(tail));
  }
  for (auto& kv : files_)
  {
    file_buffer& fb = kv.second;
    if (!fb.has_exps)
      continue;
    int total = 0;
    bit_writer sizes;
    for (const segment& sg : fb.exp_parts)
    {
      fb.append_ref(sg.p, sg.n);
      total += (int)sg.n;
      sizes.put_varbyte(sg.n);
    }
    const size_t n = sizes.size();
    stats_.exp_chunk_sizes.add((double)n);
    std::vector<uint8_t> tail(sizes.bytes.begin(), sizes.bytes.begin() + (long)n);
    put_i32(&tail, (int32_t)n);
    total += (int)n + 4;
    std::vector<uint8_t> z;
    int e = zstd_compress((const uint8_t*)fb.exp_addrs.data(), fb.exp_addrs.size() * 8, &z);
    if (e)
      return e;
    stats_.exp_addrs_raw.add((double)fb.exp_addrs.size() * 8);
    stats_.exp_addrs_z.add((double)z.size());
    tail.insert(tail.end(), z.begin(), z.end());
    put_i32(&tail, (int32_t)z.size());
    total += (int)z.size() + 4;
    put_i32(&tail, (int32_t)fb.exp_addrs.size());
    total += 4;
    total += 4;
    put_i32(&tail, (int32_t)total);
    fb.append_owned(std::move(tail));
  }
  tt.lap("pack.tails");
  return NoError;
}

std::string pack_stats_text(const pack_stats& st)
{
  // Core/idx2Write.cpp:389 PrintStats
  char buf[1024];
  std::string o;
  o += "\n\n---------------- Statistics ----------------\n\n";
  snprintf(buf, sizeof buf, "num chunks = %lld (bit plane) and %lld (exponent) \n", st.bit_plane_chunks.n,
           st.exp_chunks_z.n);
  o += buf;
  snprintf(buf, sizeof buf, "bit plane chunk: total = %d avg = %d stddev = %d bytes\n", (int)st.bit_plane_chunks.s,
           (int)st.bit_plane_chunks.avg(), (int)st.bit_plane_chunks.sd());
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) brick deltas = %d bytes\n", (int)st.brick_deltas.s);
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) brick sizes = %d bytes\n", (int)st.brick_sizes.s);
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) chunk sizes = %d bytes\n", (int)st.chunk_sizes.s);
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) chunk addresses: uncompressed = %d, compressed = %d bytes\n",
           (int)st.chunk_addrs_raw.s, (int)st.chunk_addrs_z.s);
  o += buf;
  o += "exponent chunk:\n";
  snprintf(buf, sizeof buf, "  uncompressed: total = %d bytes\n", (int)st.exp_chunks_raw.s);
  o += buf;
  snprintf(buf, sizeof buf, "  compressed: total = %d avg = %d stddev = %d bytes\n", (int)st.exp_chunks_z.s,
           (int)st.exp_chunks_z.avg(), (int)st.exp_chunks_z.sd());
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) chunk sizes = %d bytes\n", (int)st.exp_chunk_sizes.s);
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) chunk addresses: uncompressed = %d, compressed = %d bytes\n",
           (int)st.exp_addrs_raw.s, (int)st.exp_addrs_z.s);
  o += buf;
  return o;
}

std::string packer::stats_text() const
{
  return pack_stats_text(stats_);
}

} // namespace idx2g
