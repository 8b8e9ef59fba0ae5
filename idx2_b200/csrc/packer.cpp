// Chunk/file packer (Core/idx2Write.cpp, Core/idx2Encode.cpp:41-137,233-249).
#include "packer.h"

#include <cmath>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <dlfcn.h>

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
  size_t need = (size_t)((nbits + (uint64_t)n + 7) / 8) + 8;
  if (bytes.size() < need)
    bytes.resize(need > bytes.size() * 2 ? need : bytes.size() * 2, 0);
  uint64_t pos = nbits;
  int left = n;
  while (left > 0)
  {
    size_t byte = (size_t)(pos >> 3);
    int off = (int)(pos & 7);
    int take = 8 - off < left ? 8 - off : left;
    bytes[byte] |= (uint8_t)((v & ((1u << take) - 1)) << off);
    v >>= take;
    pos += (uint64_t)take;
    left -= take;
  }
  nbits += (uint64_t)n;
}

void bit_writer::put_varbyte(uint64_t v)
{
  for (;;)
  {
    put(v & 0x7F, 7);
    v >>= 7;
    put(v != 0, 1);
    if (v == 0)
      break;
  }
}

void bit_writer::put_unary(uint64_t v)
{
  while (v >= 32)
  {
    put(0, 32);
    v -= 32;
  }
  put(0, (int)v);
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
// packer
// ----------------------------------------------------------------------------

packer::packer(const dataset_format& f, double tolerance) : f_(f), tol_(tolerance)
{
  etol_ = exponent_f64(tolerance);
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
  // Core/idx2Write.cpp:221 WriteChunk
  stats_.brick_deltas.add((double)c.deltas.size());
  stats_.brick_sizes.add((double)c.sizes.size());
  bit_writer head;
  head.put_varbyte((uint64_t)c.nbricks);
  std::string path = file_path(f_, c.last_brick, level);
  file_buffer& fb = files_[path];
  size_t before = fb.data.size();
  fb.data.insert(fb.data.end(), head.bytes.begin(), head.bytes.begin() + (long)head.size());
  fb.data.insert(fb.data.end(), c.deltas.bytes.begin(), c.deltas.bytes.begin() + (long)c.deltas.size());
  fb.data.insert(fb.data.end(), c.sizes.bytes.begin(), c.sizes.bytes.begin() + (long)c.sizes.size());
  fb.data.insert(fb.data.end(), c.bricks.begin(), c.bricks.end());
  size_t chunk_bytes = fb.data.size() - before;
  stats_.bit_plane_chunks.add((double)chunk_bytes);
  fb.has_chunks = true;
  fb.chunk_sizes.put_varbyte(chunk_bytes);
  fb.chunk_addrs.push_back(chunk_address(f_, c.last_brick, level, subband, bpkey));
  c.deltas.clear();
  c.sizes.clear();
  c.bricks.clear();
}

void packer::write_chunk_exps(sub_channel& s, int level, int subband)
{
  // Core/idx2Write.cpp:38 WriteChunkExponents
  stats_.exp_chunks_raw.add((double)s.brick_exps.size());
  std::vector<uint8_t> z;
  zstd_compress(s.brick_exps.data(), s.brick_exps.size(), &z);
  stats_.exp_chunks_z.add((double)z.size());
  s.brick_exps.clear();
  std::string path = file_path(f_, s.last_brick, level);
  file_buffer& fb = files_[path];
  fb.has_exps = true;
  fb.exp_sizes.put_varbyte(z.size());
  fb.exp_data.insert(fb.exp_data.end(), z.begin(), z.end());
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
  if (r.kmin <= r.kmax)
  {
    for (int k = r.kmin; k <= r.kmax; ++k)
    {
      if (!r.sizes[k - r.kmin])
        continue;
      auto it = channels_.find(channel_key(k, L, S));
      u64 last_chunk = it == channels_.end() ? 0 : it->second.last_chunk;
      if (brick >= (last_chunk + 1) * bpc_bricks)
      {
        any_new = true;
        break;
      }
    }
  }
  if (any_new)
  {
    std::vector<int> order;
    first_touch_order(r, &order);
    for (int k : order)
    {
      channel& c = channels_[channel_key(k, L, S)];
      if (brick >= (c.last_chunk + 1) * bpc_bricks)
      {
        if (!c.bricks.empty())
          write_chunk(c, L, S, k);
        c.nbricks = 0;
        c.last_chunk = brick >> shift;
      }
    }
  }
  else if (r.kmin <= r.kmax)
  {
    for (int k = r.kmin; k <= r.kmax; ++k)
      if (r.sizes[k - r.kmin])
        channels_[channel_key(k, L, S)];
  }

  // exponents (Core/idx2Encode.cpp:41 EncodeBrickSubbandExponents)
  {
    sub_channel& sc = subs_[{ L, S }];
    if (brick >= (sc.last_chunk + 1) * bpc_bricks)
    {
      write_chunk_exps(sc, L, S);
      sc.last_chunk = brick >> shift;
    }
    if (f_.type == dtype::float64)
    {
      for (int i = 0; i < r.nexps; ++i)
      {
        uint16_t v = (uint16_t)(r.exps[i] + 1023);
        sc.brick_exps.push_back((uint8_t)(v & 0xFF));
        sc.brick_exps.push_back((uint8_t)(v >> 8));
      }
    }
    else
    {
      for (int i = 0; i < r.nexps; ++i)
        sc.brick_exps.push_back((uint8_t)(r.exps[i] + 127));
    }
    sc.last_brick = brick;
  }

  // pass 2: brick metadata and data per channel (Core/idx2Encode.cpp:84)
  if (r.kmin <= r.kmax)
  {
    size_t off = 0;
    for (int k = r.kmin; k <= r.kmax; ++k)
    {
      uint32_t nb = r.sizes[k - r.kmin];
      if (!nb)
        continue;
      channel& c = channels_[channel_key(k, L, S)];
      if (c.nbricks == 0)
        c.deltas.put_varbyte(brick);
      else
        c.deltas.put_unary(brick - c.last_brick - 1);
      c.sizes.put_varbyte(nb);
      c.bricks.insert(c.bricks.end(), r.bytes + off, r.bytes + off + nb);
      off += nb;
      ++c.nbricks;
      c.last_brick = brick;
    }
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
  for (auto& kv : channels_)
  {
    uint32_t key = kv.first;
    int level = (int)(key & 0xF);
    int subband = (int)((key >> 4) & 0xFFF);
    int bpkey = (int)(key >> 16);
    write_chunk(kv.second, level, subband, bpkey);
  }
  for (auto& kv : files_)
  {
    file_buffer& fb = kv.second;
    if (!fb.has_chunks)
      continue;
    size_t n = fb.chunk_sizes.size();
    stats_.chunk_sizes.add((double)n);
    fb.data.insert(fb.data.end(), fb.chunk_sizes.bytes.begin(), fb.chunk_sizes.bytes.begin() + (long)n);
    put_i32(&fb.data, (int32_t)n);
    std::vector<uint8_t> z;
    int e = zstd_compress((const uint8_t*)fb.chunk_addrs.data(), fb.chunk_addrs.size() * 8, &z);
    if (e)
      return e;
    fb.data.insert(fb.data.end(), z.begin(), z.end());
    put_i32(&fb.data, (int32_t)z.size());
    put_i32(&fb.data, (int32_t)fb.chunk_addrs.size());
    stats_.chunk_addrs_raw.add((double)fb.chunk_addrs.size() * 8);
    stats_.chunk_addrs_z.add((double)z.size());
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
  for (auto& kv : files_)
  {
    file_buffer& fb = kv.second;
    if (!fb.has_exps)
      continue;
    int total = 0;
    fb.data.insert(fb.data.end(), fb.exp_data.begin(), fb.exp_data.end());
    total += (int)fb.exp_data.size();
    size_t n = fb.exp_sizes.size();
    stats_.exp_chunk_sizes.add((double)n);
    fb.data.insert(fb.data.end(), fb.exp_sizes.bytes.begin(), fb.exp_sizes.bytes.begin() + (long)n);
    put_i32(&fb.data, (int32_t)n);
    total += (int)n + 4;
    std::vector<uint8_t> z;
    int e = zstd_compress((const uint8_t*)fb.exp_addrs.data(), fb.exp_addrs.size() * 8, &z);
    if (e)
      return e;
    stats_.exp_addrs_raw.add((double)fb.exp_addrs.size() * 8);
    stats_.exp_addrs_z.add((double)z.size());
    fb.data.insert(fb.data.end(), z.begin(), z.end());
    put_i32(&fb.data, (int32_t)z.size());
    total += (int)z.size() + 4;
    put_i32(&fb.data, (int32_t)fb.exp_addrs.size());
    total += 4;
    total += 4;
    put_i32(&fb.data, (int32_t)total);
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
