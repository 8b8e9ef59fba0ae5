// Chunk/file packer (Core/idx2Write.cpp, Core/idx2Encode.cpp:41-137,233-249).
#include "packer.h"

#include "encoder.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <dlfcn.h>
#include <fcntl.h>
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
// zstd through the system library
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
  // Core/idx2Encode.cpp:23 CompressBufZstd: empty input gives an empty output
  out->clear();
  if (n == 0)
    return NoError;
  if (!zapi().ok)
    return UnknownError;
  out->resize(zapi().bound(n));
  size_t r = zapi().compress(out->data(), out->size(), src, n, 1);
  if (zapi().is_error(r))
    return UnknownError;
  out->resize(r);
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
  parts.push_back({ owned.back().data(), owned.back().size() });
  nbytes += owned.back().size();
}

void file_buffer::append_ref(const uint8_t* p, size_t n)
{
  if (!n)
    return;
  parts.push_back({ p, n });
  nbytes += n;
}

int write_files(const std::vector<std::pair<std::string, const file_buffer*>>& files)
{
  // Every file is cut into ranges of whole parts of about kRange bytes; a pool of
  // threads gathers each range into a staging buffer and writes it at its offset.
  constexpr size_t kRange = (size_t)16 << 20;
  struct range
  {
    int file;
    size_t p0, p1, offset;
  };
  std::vector<int> fds(files.size(), -1);
  std::vector<range> ranges;
  int err = NoError;
  for (size_t i = 0; i < files.size() && !err; ++i)
  {
    if (make_dirs_for(files[i].first) != NoError)
    {
      err = CannotCreateDirectory;
      break;
    }
    fds[i] = open(files[i].first.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fds[i] < 0)
    {
      err = FileCreateFailed;
      break;
    }
    const std::vector<segment>& parts = files[i].second->parts;
    size_t off = 0, start = 0, acc = 0;
    for (size_t k = 0; k < parts.size(); ++k)
    {
      acc += parts[k].n;
      if (acc >= kRange || k + 1 == parts.size())
      {
        ranges.push_back({ (int)i, start, k + 1, off });
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
        const std::vector<segment>& parts = files[(size_t)r.file].second->parts;
        size_t n = 0;
        for (size_t k = r.p0; k < r.p1; ++k)
          n += parts[k].n;
        const uint8_t* src;
        if (r.p1 - r.p0 == 1)
          src = parts[r.p0].p;
        else
        {
          stage.resize(n);
          size_t at = 0;
          for (size_t k = r.p0; k < r.p1; ++k)
          {
            memcpy(stage.data() + at, parts[k].p, parts[k].n);
            at += parts[k].n;
          }
          src = stage.data();
        }
        size_t done = 0;
        while (done < n)
        {
          ssize_t w = pwrite(fds[(size_t)r.file], src + done, n - done, (off_t)(r.offset + done));
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
constexpr int kKeySpace = 4096;  // bit-plane keys are 12-bit (Core/idx2Lookup.h:21)
inline size_t chan_slot(int level, int subband, int bpkey)
{
  return ((size_t)(level & 15) * 64 + (size_t)(subband & 63)) * kKeySpace + (size_t)(bpkey & (kKeySpace - 1));
}
} // namespace

packer::packer(const dataset_format& f, double tolerance) : f_(f), tol_(tolerance)
{
  etol_ = exponent_f64(tolerance);
  chan_index_.assign((size_t)16 * 64 * kKeySpace, -1);
}

packer::~packer() = default;

packer::channel* packer::find_chan(int level, int subband, int bpkey)
{
  int32_t i = chan_index_[chan_slot(level, subband, bpkey)];
  return i < 0 ? nullptr : &channels_[(size_t)i];
}

packer::channel& packer::chan(int level, int subband, int bpkey)
{
  int32_t& i = chan_index_[chan_slot(level, subband, bpkey)];
  if (i < 0)
  {
    i = (int32_t)channels_.size();
    channels_.emplace_back();
    channels_.back().key = channel_key(bpkey, level, subband);
  }
  return channels_[(size_t)i];
}

void packer::first_touch_order(const subband_result& r, std::vector<int>* keys) const
{
  // order in which EncodeSubbandBlocks first meets each channel: blocks in Morton order,
  // planes from the top down (Core/idx2Encode.cpp:157-249)
  keys->clear();
  if (r.kmin > r.kmax)
    return;
  std::vector<char> seen((size_t)(r.kmax - r.kmin + 1), 0);
  const int end_bp = f_.type == dtype::float32 ? 32 : 64;
  const int bpc = f_.bit_planes_per_chunk;
  for (int b = 0; b < r.nexps; ++b)
  {
    int emax = r.exps[b];
    for (int bp = 63; bp >= 64 - end_bp; --bp)
    {
      if (!plane_coded(bp, emax, etol_, bpc))
        break;
      int key = (bp + emax + 1024) / bpc;
      if (key < r.kmin || key > r.kmax)
        continue;
      char& s = seen[(size_t)(key - r.kmin)];
      if (!s)
      {
        s = 1;
        keys->push_back(key);
      }
    }
  }
}

void packer::write_chunk(channel& c, int level, int subband, int bpkey)
{
  // Core/idx2Write.cpp:221 WriteChunk: varbyte NBricks | deltas | sizes | brick data
  stats_.brick_deltas.add((double)c.deltas.size());
  stats_.brick_sizes.add((double)c.sizes.size());
  bit_writer head;
  head.put_varbyte((uint64_t)c.nbricks);
  std::vector<uint8_t> meta;
  meta.reserve(head.size() + c.deltas.size() + c.sizes.size());
  meta.insert(meta.end(), head.bytes.begin(), head.bytes.begin() + (long)head.size());
  meta.insert(meta.end(), c.deltas.bytes.begin(), c.deltas.bytes.begin() + (long)c.deltas.size());
  meta.insert(meta.end(), c.sizes.bytes.begin(), c.sizes.bytes.begin() + (long)c.sizes.size());
  const size_t chunk_bytes = meta.size() + c.brick_bytes;
  file_buffer& fb = files_[file_path(f_, c.last_brick, level)];
  fb.append_owned(std::move(meta));
  for (const segment& s : c.bricks)
    fb.append_ref(s.p, s.n);
  stats_.bit_plane_chunks.add((double)chunk_bytes);
  fb.has_chunks = true;
  fb.chunk_sizes.put_varbyte(chunk_bytes);
  fb.chunk_addrs.push_back(chunk_address(f_, c.last_brick, level, subband, bpkey));
  c.deltas.clear();
  c.sizes.clear();
  c.bricks.clear();
  c.brick_bytes = 0;
}

void packer::write_chunk_exps(sub_channel& s, int level, int subband)
{
  // Core/idx2Write.cpp:38 WriteChunkExponents (compression deferred to finish)
  stats_.exp_chunks_raw.add((double)s.brick_exps.size());
  exp_chunks_.emplace_back();
  exp_chunks_.back().raw.swap(s.brick_exps);
  s.brick_exps.clear();
  file_buffer& fb = files_[file_path(f_, s.last_brick, level)];
  fb.has_exps = true;
  fb.exp_chunks.push_back((int)exp_chunks_.size() - 1);
  fb.exp_addrs.push_back(chunk_address(f_, s.last_brick, level, subband, 0));
}

int packer::add(const subband_result& r)
{
  const int L = r.level, S = r.subband;
  const u64 brick = r.brick;
  const u64 bpc_bricks = (u64)f_.bricks_per_chunk[L];
  const int shift = log2_ceil(f_.bricks_per_chunk[L]);

  // pass 1: channels in first-touch order; a channel entering a new chunk flushes the
  // previous one (Core/idx2Encode.cpp:233-249)
  bool any_new = false;
  for (int k = r.kmin; k <= r.kmax && !any_new; ++k)
  {
    if (!r.sizes[k - r.kmin])
      continue;
    channel* c = find_chan(L, S, k);
    u64 last_chunk = c ? c->last_chunk : 0;
    any_new = brick >= (last_chunk + 1) * bpc_bricks;
  }
  if (any_new)
  {
    std::vector<int> order;
    first_touch_order(r, &order);
    for (int k : order)
    {
      channel& c = chan(L, S, k);
      if (brick >= (c.last_chunk + 1) * bpc_bricks)
      {
        if (c.brick_bytes)
          write_chunk(c, L, S, k);
        c.nbricks = 0;
        c.last_chunk = brick >> shift;
      }
    }
  }

  // exponents (Core/idx2Encode.cpp:41 EncodeBrickSubbandExponents)
  {
    sub_channel& sc = subs_[{ L, S }];
    if (brick >= (sc.last_chunk + 1) * bpc_bricks)
    {
      write_chunk_exps(sc, L, S);
      sc.last_chunk = brick >> shift;
    }
    const size_t at = sc.brick_exps.size();
    if (f_.type == dtype::float64)
    {
      sc.brick_exps.resize(at + 2 * (size_t)r.nexps);
      for (int i = 0; i < r.nexps; ++i)
      {
        uint16_t v = (uint16_t)(r.exps[i] + 1023);
        sc.brick_exps[at + 2 * (size_t)i] = (uint8_t)(v & 0xFF);
        sc.brick_exps[at + 2 * (size_t)i + 1] = (uint8_t)(v >> 8);
      }
    }
    else
    {
      sc.brick_exps.resize(at + (size_t)r.nexps);
      for (int i = 0; i < r.nexps; ++i)
        sc.brick_exps[at + (size_t)i] = (uint8_t)(r.exps[i] + 127);
    }
    sc.last_brick = brick;
  }

  // pass 2: brick metadata and data per channel (Core/idx2Encode.cpp:84)
  size_t off = 0;
  for (int k = r.kmin; k <= r.kmax; ++k)
  {
    const uint32_t nb = r.sizes[k - r.kmin];
    if (!nb)
      continue;
    channel& c = chan(L, S, k);
    if (c.nbricks == 0)
      c.deltas.put_varbyte(brick);
    else
      c.deltas.put_unary(brick - c.last_brick - 1);
    c.sizes.put_varbyte(nb);
    c.bricks.push_back({ r.bytes + off, nb });
    c.brick_bytes += nb;
    off += nb;
    ++c.nbricks;
    c.last_brick = brick;
  }
  return NoError;
}

static void put_i32(std::vector<uint8_t>* v, int32_t x)
{
  uint8_t b[4];
  memcpy(b, &x, 4);
  v->insert(v->end(), b, b + 4);
}

int packer::finish()
{
  // FlushChunks (Core/idx2Write.cpp:317): every channel in key order
  std::vector<channel*> order;
  order.reserve(channels_.size());
  for (channel& c : channels_)
    order.push_back(&c);
  std::sort(order.begin(), order.end(), [](const channel* a, const channel* b) { return a->key < b->key; });
  for (channel* c : order)
  {
    const int level = (int)(c->key & 0xF);
    const int subband = (int)((c->key >> 4) & 0xFFF);
    const int bpkey = (int)(c->key >> 16);
    write_chunk(*c, level, subband, bpkey);
  }
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
  // FlushChunkExponents (:121): sub-channels by level descending, then subband
  std::vector<std::pair<std::pair<int, int>, sub_channel*>> subs;
  for (auto& kv : subs_)
    subs.push_back({ kv.first, &kv.second });
  std::stable_sort(subs.begin(), subs.end(), [](const auto& a, const auto& b) {
    if (a.first.first == b.first.first)
      return a.first.second < b.first.second;
    return a.first.first > b.first.first;
  });
  for (auto& s : subs)
    write_chunk_exps(*s.second, s.first.first, s.first.second);
  // compress the exponent chunks in parallel (each is an independent zstd frame)
  {
    std::atomic<size_t> next{ 0 };
    std::atomic<int> err{ 0 };
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt ? (nt > 32 ? 32 : nt) : 4;
    auto work = [&]() {
      for (size_t i; (i = next.fetch_add(1)) < exp_chunks_.size();)
        if (zstd_compress(exp_chunks_[i].raw.data(), exp_chunks_[i].raw.size(), &exp_chunks_[i].z))
          err = UnknownError;
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t)
      th.emplace_back(work);
    work();
    for (auto& t : th)
      t.join();
    if (err)
      return err;
    for (auto& c : exp_chunks_)
      stats_.exp_chunks_z.add((double)c.z.size());
  }
  for (auto& kv : files_)
  {
    file_buffer& fb = kv.second;
    if (!fb.has_exps)
      continue;
    int total = 0;
    bit_writer sizes;
    for (int ci : fb.exp_chunks)
    {
      exp_chunk& c = exp_chunks_[(size_t)ci];
      fb.append_ref(c.z.data(), c.z.size());
      total += (int)c.z.size();
      sizes.put_varbyte(c.z.size());
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
  return NoError;
}

std::string packer::stats_text() const
{
  // Core/idx2Write.cpp:389 PrintStats
  char buf[1024];
  std::string o;
  o += "\n\n---------------- Statistics ----------------\n\n";
  snprintf(buf, sizeof buf, "num chunks = %lld (bit plane) and %lld (exponent) \n",
           stats_.bit_plane_chunks.n, stats_.exp_chunks_z.n);
  o += buf;
  snprintf(buf, sizeof buf, "bit plane chunk: total = %d avg = %d stddev = %d bytes\n",
           (int)stats_.bit_plane_chunks.s, (int)stats_.bit_plane_chunks.avg(),
           (int)stats_.bit_plane_chunks.sd());
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) brick deltas = %d bytes\n", (int)stats_.brick_deltas.s);
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) brick sizes = %d bytes\n", (int)stats_.brick_sizes.s);
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) chunk sizes = %d bytes\n", (int)stats_.chunk_sizes.s);
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) chunk addresses: uncompressed = %d, compressed = %d bytes\n",
           (int)stats_.chunk_addrs_raw.s, (int)stats_.chunk_addrs_z.s);
  o += buf;
  o += "exponent chunk:\n";
  snprintf(buf, sizeof buf, "  uncompressed: total = %d bytes\n", (int)stats_.exp_chunks_raw.s);
  o += buf;
  snprintf(buf, sizeof buf, "  compressed: total = %d avg = %d stddev = %d bytes\n",
           (int)stats_.exp_chunks_z.s, (int)stats_.exp_chunks_z.avg(), (int)stats_.exp_chunks_z.sd());
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) chunk sizes = %d bytes\n", (int)stats_.exp_chunk_sizes.s);
  o += buf;
  snprintf(buf, sizeof buf, "  (metadata) chunk addresses: uncompressed = %d, compressed = %d bytes\n",
           (int)stats_.exp_addrs_raw.s, (int)stats_.exp_addrs_z.s);
  o += buf;
  return o;
}

} // namespace idx2g
