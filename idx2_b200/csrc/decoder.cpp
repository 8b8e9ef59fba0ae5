// Decode side, host part (Core/idx2Decode.cpp:326-540, Core/idx2Read.cpp).
//
// dataset_open reads the metadata file and every data file of the dataset once,
// parses the chunk tables (file tails, chunk headers), decompresses the exponent
// chunks and builds a device-resident index:
//   blob      all bit-plane chunk bytes, as stored in the files
//   exps      per (level, brick, subband): the block exponents (coded blocks, Morton order)
//   chan      per (level, brick, subband): the byte offset in blob of the brick's data in
//             the chunk of each bit-plane channel present
// dataset_decode then plans the request (ROI, downsampling, tolerance) on the host and runs
// one device launch per decoded level, coarsest first.
#include "decoder.h"
#include "decode_device.h"
#include "packer.h"
#include "parallel.h"
#include "trace.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <fcntl.h>
#include <map>
#include <memory>
#include <set>
#include <tuple>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>
#include <unordered_map>
#include <unordered_set>

namespace idx2g
{

namespace
{

// LSB-first bit reader over a byte range (Core/BitStream.h); reads past the end give zeros.
struct bit_reader
{
  const uint8_t* p;
  size_t n;
  uint64_t pos = 0;
  // at least 57 valid bits starting at pos
  uint64_t peek() const
  {
    const size_t b = (size_t)(pos >> 3);
    uint64_t w = 0;
    if (b + 8 <= n)
      memcpy(&w, p + b, 8);
    else if (b < n)
      memcpy(&w, p + b, n - b);
    return w >> (pos & 7);
  }
  uint64_t get(int bits)  // bits <= 57
  {
    uint64_t v = peek() & ((1ull << bits) - 1);
    pos += (uint64_t)bits;
    return v;
  }
  uint64_t varbyte()
  {
    // Core/VarInt.h:30 ReadVarByte: 7 value bits then a continuation bit
    uint64_t v = 0;
    int sh = 0;
    while (true)
    {
      uint64_t b = get(8);
      v = ((b & 0x7F) << (7 * sh++)) + v;
      if (!(b >> 7))
        break;
      if (sh > 10)
        break;
    }
    return v;
  }
  uint64_t unary()
  {
    // Core/VarInt.h:90 ReadUnary: zero bits up to the next one bit
    uint64_t v = 0;
    while (true)
    {
      uint64_t w = peek() & ((1ull << 57) - 1);
      if (w)
      {
        int z = __builtin_ctzll(w);
        pos += (uint64_t)z + 1;
        return v + (uint64_t)z;
      }
      v += 57;
      pos += 57;
      if ((pos >> 3) > n)
        return v;
    }
  }
  void next_byte() { pos = (pos + 7) & ~7ull; }
};

inline int32_t rd_i32(const uint8_t* d, size_t off)
{
  int32_t v;
  memcpy(&v, d + off, 4);
  return v;
}

bool read_whole(const std::string& path, std::vector<uint8_t>* out)
{
  FILE* fp = fopen(path.c_str(), "rb");
  if (!fp)
    return false;
  fseek(fp, 0, SEEK_END);
  long sz = ftell(fp);
  fseek(fp, 0, SEEK_SET);
  out->resize((size_t)(sz > 0 ? sz : 0));
  size_t r = sz > 0 ? fread(out->data(), 1, (size_t)sz, fp) : 0;
  fclose(fp);
  return r == out->size();
}

} // namespace

struct dataset_handle
{
  dataset_format f;
  params p0;
  // per level: dense map from linear brick id to brick index (-1 if none)
  std::vector<std::vector<int>> brick_index;
  std::vector<std::vector<v3>> brick3;           // per level, per brick index
  std::vector<std::vector<int>> brick_in_chunk;  // per level, per brick index
  std::vector<std::vector<int>> blocks_per_sb;   // per level, per subband (coded blocks)
  std::vector<size_t> level_brick_base;          // brick index base of each level in flat tables
  // host index, built while the dataset opens in pinned staging buffers of the context
  size_t nslots = 0, nchan = 0;
  int16_t* exps = nullptr;                       // [level offset + brick][sb][kMaxBlocksPerSubband]
  // the bit-plane chunks and the linear -> flat brick maps, from which the device builds the
  // channel tables (per (brick, subband): key range, first entry; per entry: byte offset in
  // the blob, ~0 = absent)
  std::vector<index_chunk> ix_chunks;
  std::vector<int> ix_bmap;
  std::vector<long long> ix_base;
  std::vector<int> ix_size;
  const uint8_t* blob = nullptr;                 // every data file back to back (pinned host memory)
  size_t blob_bytes = 0;
  // device copies
  decode_device dev;
  // plans of the last few single-request decodes, by request (a request repeated on the
  // dataset, such as every time step's full read, plans once)
  struct cached_plan
  {
    std::string key;
    decode_request rq;
    size_t need = 0;
  };
  std::vector<std::unique_ptr<cached_plan>> plans;
  // what the files lack, for the reference's decode-time errors: the data files that were not
  // found (per level, the bits of the linear brick index that select the file) and the
  // exponent chunks present (their chunk addresses)
  std::vector<std::map<u64, int>> bad_files;  // per level: file bits -> FileNotFound / SizeMismatched
  std::vector<int> file_shift;
  std::unordered_set<u64> exp_chunk_addrs;
};

namespace
{

struct data_file
{
  std::string path;
  int level;
  u64 bits = 0;  // the bits of the linear brick index that select this file
  size_t base = 0, size = 0;
};

// a chunk located in the blob
struct chunk_ref
{
  size_t off, size;
  u64 addr;
  int level;
};

// one brick's data inside a bit-plane chunk

} // namespace

static int load_index(device_ctx* ctx, dataset_handle* h)
{
  dataset_format& f = h->f;
  const int L = f.nlevels;
  const int nsb = f.nsubbands();
  stage_timer tt;
  h->brick_index.assign((size_t)L, {});
  h->brick3.assign((size_t)L, {});
  h->brick_in_chunk.assign((size_t)L, {});
  h->blocks_per_sb.assign((size_t)L, std::vector<int>((size_t)nsb, 0));
  h->level_brick_base.assign((size_t)L + 1, 0);

  // enumerate bricks of every level with their index in the chunk, using the decoder's
  // file -> chunk -> brick traversal over the whole volume (Core/idx2Decode.cpp:403-470)
  for (int l = 0; l < L; ++l)
  {
    size_t nlin = (size_t)1 << f.bricks_order_str[(size_t)l].size();
    h->brick_index[(size_t)l].assign(nlin, -1);
    v3 b3 = f.brick_dims;
    for (int k = 0; k < l; ++k)
      b3 = b3 * f.group_brick3;
    v3 c3 = f.bricks_per_chunk3[(size_t)l] * b3;
    v3 fl3 = c3 * f.chunks_per_file3[(size_t)l];
    extent vol{ v3(0), f.dims };
    extent eb{ vol.from / b3, vol.last() / b3 - vol.from / b3 + v3(1) };
    extent ec{ vol.from / c3, vol.last() / c3 - vol.from / c3 + v3(1) };
    extent ef{ vol.from / fl3, vol.last() / fl3 - vol.from / fl3 + v3(1) };
    const brick_linearizer lin_of(f, l, f.nbricks3[(size_t)l]);
    traverse(f.files_order[(size_t)l], v3(0), f.nfiles3[(size_t)l], ef, ef, [&](const traverse_item& fi) {
      traverse(f.chunks_order_in_file[(size_t)l], fi.from3 * f.chunks_per_file3[(size_t)l],
               f.chunks_per_file3[(size_t)l], ec, ec, [&](const traverse_item& ci) {
                 traverse(f.bricks_order_in_chunk[(size_t)l], ci.from3 * f.bricks_per_chunk3[(size_t)l],
                          f.bricks_per_chunk3[(size_t)l], eb, eb, [&](const traverse_item& bi) {
                            u64 lin = lin_of(bi.from3);
                            if (lin >= nlin || h->brick_index[(size_t)l][lin] >= 0)
                              return;
                            h->brick_index[(size_t)l][lin] = (int)h->brick3[(size_t)l].size();
                            h->brick3[(size_t)l].push_back(bi.from3);
                            h->brick_in_chunk[(size_t)l].push_back(bi.item_in_parent);
                          });
               });
    });
    h->level_brick_base[(size_t)l + 1] = h->level_brick_base[(size_t)l] + h->brick3[(size_t)l].size();
    for (int s = 0; s < nsb; ++s)
    {
      std::vector<block_geom> g;
      subband_blocks(f, l, s, &g);
      h->blocks_per_sb[(size_t)l][(size_t)s] = (int)g.size();
    }
  }
  const size_t nflat = h->level_brick_base[(size_t)L];
  const size_t nslots = nflat * (size_t)nsb;
  if (nslots >= 0xFFFFFFFFull)
    return OptionNotSupported;
  h->nslots = nslots;
  h->exps = (int16_t*)ctx->pinned("dec.exps", nslots * kMaxBlocksPerSubband * sizeof(int16_t));
  if (!h->exps)
    return OutOfMemory;
  parallel_ranges(nslots, [&](size_t i0, size_t i1) {
    memset(h->exps + i0 * kMaxBlocksPerSubband, 0, (i1 - i0) * kMaxBlocksPerSubband * sizeof(int16_t));
  });

  tt.lap("open.bricks");
  // the set of data files: one per (level, brick >> log2(bricks per file)); a missing file
  // leaves its bricks undecoded (Core/idx2Decode.cpp:166-168). A file's path depends on the
  // bits of the linear brick index above `shift` only, so it is built once per run of bricks
  // that share them.
  std::map<std::string, std::pair<int, u64>> names;  // path -> (level, file bits of the brick index)
  h->bad_files.assign((size_t)L, {});
  h->file_shift.assign((size_t)L, 0);
  for (int l = 0; l < L; ++l)
  {
    const std::vector<int>& dd = f.files_dirs_depth[(size_t)l];
    int shift = (int)f.bricks_order_str[(size_t)l].size();
    for (size_t d = 0; d + 1 < dd.size(); ++d)
      shift -= dd[d];
    shift = shift < 0 ? 0 : shift > 63 ? 63 : shift;
    h->file_shift[(size_t)l] = shift;
    u64 prev = ~0ull;
    const brick_linearizer lin_of(f, l, f.nbricks3[(size_t)l]);
    for (size_t i = 0; i < h->brick3[(size_t)l].size(); ++i)
    {
      const u64 lin = lin_of(h->brick3[(size_t)l][i]);
      if ((lin >> shift) == prev)
        continue;
      prev = lin >> shift;
      names[file_path(f, lin, l)] = { l, lin >> shift };
    }
  }
  std::vector<data_file> files;
  size_t total = 0;
  for (auto& kv : names)
  {
    struct stat st;
    if (stat(kv.first.c_str(), &st) != 0 || !S_ISREG(st.st_mode))
    {
      // decoding a brick of this file fails with FileNotFound (Core/idx2Read.cpp:270,380)
      h->bad_files[(size_t)kv.second.first][kv.second.second] = FileNotFound;
      continue;
    }
    data_file df;
    df.path = kv.first;
    df.level = kv.second.first;
    df.bits = kv.second.second;
    df.base = total;
    df.size = (size_t)st.st_size;
    total += (df.size + 15) & ~(size_t)15;
    files.push_back(df);
  }

  tt.lap("open.files");
  // every file into one pinned buffer, in ranges of 4 MB read by a pool of threads; each
  // range goes on to the device as soon as it is read, while the other threads read on and
  // the index below is built (small ranges, so that the first copy starts after a few MB
  // rather than after a whole round of the threads' reads)
  uint8_t* blob = (uint8_t*)ctx->pinned("dec.files", total + 16);
  if (!blob)
    return OutOfMemory;
  if (int ae = h->dev.alloc(ctx, nslots, total))
    return ae;
  tt.lap("open.alloc");
  {
    struct range
    {
      int file;
      size_t off, n;
    };
    std::vector<range> rs;
    const size_t R = (size_t)4 << 20;
    for (size_t i = 0; i < files.size(); ++i)
      for (size_t o = 0; o < files[i].size; o += R)
        rs.push_back({ (int)i, o, std::min(R, files[i].size - o) });
    std::vector<int> fds(files.size(), -1);
    for (size_t i = 0; i < files.size(); ++i)
      fds[i] = open(files[i].path.c_str(), O_RDONLY);
    std::atomic<int> bad{ 0 };
    parallel_for(rs.size(), [&](size_t k) {
      const range& r = rs[k];
      size_t done = 0;
      while (done < r.n)
      {
        ssize_t got = fds[(size_t)r.file] < 0 ? -1
                      : pread(fds[(size_t)r.file], blob + files[(size_t)r.file].base + r.off + done,
                              r.n - done, (off_t)(r.off + done));
        if (got <= 0)
        {
          bad = 1;
          return;
        }
        done += (size_t)got;
      }
      h->dev.upload_blob(ctx, blob + files[(size_t)r.file].base + r.off, files[(size_t)r.file].base + r.off, r.n);
    });
    for (int fd : fds)
      if (fd >= 0)
        close(fd);
    if (bad)
      return FileReadFailed;
  }
  h->blob = blob;
  h->blob_bytes = total;
  tt.lap("open.read");

  // file tails: exponent chunks and bit-plane chunks
  std::vector<chunk_ref> exp_chunks, bp_chunks;
  for (const data_file& df : files)
  {
    const uint8_t* d = blob + df.base;
    const int level = df.level;
    if (df.size < 16)
      return CorruptStream;
    // exponent section (Core/idx2Read.cpp:252 ReadFileExponents)
    const size_t E = df.size;
    int32_t total_e = rd_i32(d, E - 4);
    int32_t nexp = rd_i32(d, E - 8);
    int32_t asz = rd_i32(d, E - 12);
    if (total_e < 16 || (size_t)total_e > E || asz < 0 || (size_t)asz + 16 > (size_t)total_e || nexp < 0)
      return CorruptStream;
    std::vector<uint8_t> addrs_raw;
    if (zstd_decompress(d + E - 12 - (size_t)asz, (size_t)asz, &addrs_raw))
      return CorruptStream;
    int32_t ssz = rd_i32(d, E - 16 - (size_t)asz);
    if (ssz < 0 || (size_t)ssz + (size_t)asz + 16 > (size_t)total_e)
      return CorruptStream;
    bit_reader sr{ d + E - 16 - (size_t)asz - (size_t)ssz, (size_t)ssz };
    {
      // the reference counts the size varbytes (to the end of their section) against the
      // chunk count, and wants whole sets of subbands; otherwise decoding any brick of the
      // file fails with SizeMismatched (Core/idx2Read.cpp:304-323)
      bit_reader cnt{ sr.p, sr.n };
      long long n2 = 0;
      while ((cnt.pos >> 3) < (uint64_t)ssz)
      {
        cnt.varbyte();
        ++n2;
      }
      if (n2 != nexp || nexp % nsb != 0)
      {
        h->bad_files[(size_t)level][df.bits] = SizeMismatched;
        continue;
      }
    }
    const size_t exp_beg = E - (size_t)total_e;
    size_t off = exp_beg;
    for (int c = 0; c < nexp; ++c)
    {
      uint64_t csz = sr.varbyte();
      if ((size_t)c * 8 + 8 > addrs_raw.size() || off + csz > E)
        return CorruptStream;
      u64 addr;
      memcpy(&addr, addrs_raw.data() + (size_t)c * 8, 8);
      exp_chunks.push_back({ df.base + off, (size_t)csz, addr, level });
      off += csz;
    }
    if (exp_beg == 0)
      continue;
    // bit-plane section (Core/idx2Read.cpp:82 ReadFile)
    const size_t E2 = exp_beg;
    if (E2 < 12)
      return CorruptStream;
    int32_t nch = rd_i32(d, E2 - 4);
    int32_t asz2 = rd_i32(d, E2 - 8);
    if (asz2 < 0 || (size_t)asz2 + 12 > E2 || nch < 0)
      return CorruptStream;
    std::vector<uint8_t> caddrs;
    if (zstd_decompress(d + E2 - 8 - (size_t)asz2, (size_t)asz2, &caddrs))
      return CorruptStream;
    int32_t ssz2 = rd_i32(d, E2 - 12 - (size_t)asz2);
    if (ssz2 < 0 || (size_t)ssz2 + (size_t)asz2 + 12 > E2)
      return CorruptStream;
    bit_reader csr{ d + E2 - 12 - (size_t)asz2 - (size_t)ssz2, (size_t)ssz2 };
    const size_t body_end = E2 - 12 - (size_t)asz2 - (size_t)ssz2;
    size_t coff = 0;
    for (int c = 0; c < nch; ++c)
    {
      uint64_t csz = csr.varbyte();
      if ((size_t)c * 8 + 8 > caddrs.size() || coff + csz > body_end)
        return CorruptStream;
      u64 addr;
      memcpy(&addr, caddrs.data() + (size_t)c * 8, 8);
      bp_chunks.push_back({ df.base + coff, (size_t)csz, addr, level });
      coff += csz;
    }
  }

  for (const chunk_ref& c : exp_chunks)
    h->exp_chunk_addrs.insert(c.addr);
  tt.lap("open.tails");
  // exponent chunks: decompress and spread over their bricks (chunks own disjoint rows)
  const int esz = f.type == dtype::float32 ? 1 : 2;
  std::atomic<int> err{ 0 };
  parallel_for(exp_chunks.size(), [&](size_t k) {
    const chunk_ref& c = exp_chunks[k];
    int sb = (int)((c.addr >> 12) & 0x3F);
    int lv = (int)((c.addr >> 60) & 0xF);
    u64 chunk = (c.addr >> 18) & 0x3FFFFFFFFFFull;
    if (lv != c.level || sb >= nsb)
      return;
    std::vector<uint8_t> ex;
    if (zstd_decompress(blob + c.off, c.size, &ex))
    {
      err = CorruptStream;
      return;
    }
    // every brick of this chunk: exps at BrickInChunk * BlockCount * esz
    int shift = log2_ceil(f.bricks_per_chunk[(size_t)lv]);
    u64 first = chunk << shift, last = (chunk + 1) << shift;
    const int bc = h->blocks_per_sb[(size_t)lv][(size_t)sb];
    for (u64 lin = first; lin < last && lin < h->brick_index[(size_t)lv].size(); ++lin)
    {
      int bi = h->brick_index[(size_t)lv][lin];
      if (bi < 0)
        continue;
      size_t pos = (size_t)h->brick_in_chunk[(size_t)lv][(size_t)bi] * (size_t)bc * (size_t)esz;
      size_t flat = h->level_brick_base[(size_t)lv] + (size_t)bi;
      int16_t* dst = h->exps + (flat * (size_t)nsb + (size_t)sb) * kMaxBlocksPerSubband;
      for (int b = 0; b < bc; ++b)
      {
        size_t q = pos + (size_t)b * (size_t)esz;
        int v = 0;
        if (q + (size_t)esz <= ex.size())
          v = esz == 2 ? (int)ex[q] | ((int)ex[q + 1] << 8) : (int)ex[q];
        dst[b] = (int16_t)(esz == 2 ? v - 1023 : v - 127);
      }
    }
  });
  if (err)
    return err;

  tt.lap("open.exponents");
  // bit-plane chunks for the device index (decode_device::build_index parses their headers,
  // Core/idx2Decode.cpp:507 DecompressChunk)
  h->ix_chunks.clear();
  h->ix_chunks.reserve(bp_chunks.size());
  for (const chunk_ref& c : bp_chunks)
  {
    const int sb = (int)((c.addr >> 12) & 0x3F), lv = (int)((c.addr >> 60) & 0xF);
    if (lv != c.level || lv >= L || sb >= nsb)
      continue;
    h->ix_chunks.push_back(index_chunk{ (unsigned long long)c.off, (unsigned long long)c.size, lv, sb,
                                        (int)(c.addr & 0xFFF), 0 });
  }
  h->ix_base.assign((size_t)L, 0);
  h->ix_size.assign((size_t)L, 0);
  size_t nmap = 0;
  for (int l = 0; l < L; ++l)
  {
    h->ix_base[(size_t)l] = (long long)nmap;
    h->ix_size[(size_t)l] = (int)h->brick_index[(size_t)l].size();
    nmap += h->brick_index[(size_t)l].size();
  }
  h->ix_bmap.resize(nmap);
  for (int l = 0; l < L; ++l)
  {
    const std::vector<int>& index = h->brick_index[(size_t)l];
    int* dst = h->ix_bmap.data() + h->ix_base[(size_t)l];
    for (size_t lin = 0; lin < index.size(); ++lin)
      dst[lin] = index[lin] < 0 ? -1 : (int)(h->level_brick_base[(size_t)l] + (size_t)index[lin]);
  }
  tt.lap("open.chunks");
  return NoError;
}

int dataset_open(device_ctx* ctx, const params& pin, dataset_handle** out)
{
  *out = nullptr;
  std::vector<uint8_t> meta;
  if (!read_whole(pin.input_file, &meta))
    return FileNotFound;
  dataset_handle* h = new dataset_handle;
  h->p0 = pin;
  int e = parse_meta(std::string(meta.begin(), meta.end()), &h->f);
  if (!e)
  {
    params p = pin;
    p.downsampling = v3(0);
    e = finalize_read(&h->f, &p);
  }
  if (!e)
    e = load_index(ctx, h);
  stage_timer tt;
  if (!e)
    e = h->dev.build_index(ctx, h->ix_chunks, h->ix_bmap, h->ix_base, h->ix_size, h->f.nsubbands(), h->exps,
                           &h->nchan);
  tt.lap("open.index");
  // the pinned staging buffers stay with the context
  h->blob = nullptr;
  h->exps = nullptr;
  h->ix_chunks.clear();
  h->ix_chunks.shrink_to_fit();
  h->ix_bmap.clear();
  h->ix_bmap.shrink_to_fit();
  if (e)
  {
    delete h;
    return e;
  }
  *out = h;
  return NoError;
}

// Decode masks and spacings of a request (Core/idx2Common.cpp:403-461).
static void request_format(const dataset_handle* h, const params& p, dataset_format* f)
{
  *f = h->f;
  f->downsampling = p.downsampling;
  params q = p;
  q.in_dir = h->f.dir;
  finalize_read(f, &q);
}

int dataset_output_grid(const dataset_handle* h, const params& p, grid* g)
{
  dataset_format f;
  request_format(h, p, &f);
  extent ext = p.has_extent ? p.decode_extent : extent{ v3(0), f.dims };
  *g = output_grid(f, ext);
  return NoError;
}

// The plan of a request from the dataset's cache (planned and kept on a miss).
static int cached_plan_decode(dataset_handle* h, const params& p, const decode_request** rq, size_t* need)
{
  char key[256];
  snprintf(key, sizeof key, "%d|%d %d %d|%d %d %d|%d %d %d|%.17g", p.has_extent ? 1 : 0, p.decode_extent.from.x,
           p.decode_extent.from.y, p.decode_extent.from.z, p.decode_extent.dims.x, p.decode_extent.dims.y,
           p.decode_extent.dims.z, p.downsampling.x, p.downsampling.y, p.downsampling.z, p.decode_tolerance);
  for (auto& c : h->plans)
    if (c->key == key)
    {
      *rq = &c->rq;
      *need = c->need;
      return NoError;
    }
  std::unique_ptr<dataset_handle::cached_plan> c(new dataset_handle::cached_plan());
  c->key = key;
  int e = plan_decode(h, p, &c->rq, &c->need);
  if (e)
    return e;
  if (h->plans.size() >= 4)
    h->plans.erase(h->plans.begin());
  h->plans.push_back(std::move(c));
  *rq = &h->plans.back()->rq;
  *need = h->plans.back()->need;
  return NoError;
}

int dataset_decode(device_ctx* ctx, dataset_handle* h, const params& p, void* out, size_t out_bytes,
                   bool out_on_device, double* kernel_ms)
{
  const decode_request* rq = nullptr;
  size_t need = 0;
  stage_timer tt;
  int e = cached_plan_decode(h, p, &rq, &need);
  if (e)
    return e;
  if (out_bytes < need)
    return SizeTooSmall;
  tt.lap("decode.plan");
  e = h->dev.decode(ctx, *rq, out, need, out_on_device, kernel_ms);
  tt.lap("decode.device");
  return e;
}

int plan_decode(const dataset_handle* h, const params& p, decode_request* rq_out, size_t* need_out)
{
  dataset_format f;
  request_format(h, p, &f);
  extent ext = p.has_extent ? p.decode_extent : extent{ v3(0), f.dims };
  grid og = output_grid(f, ext);
  const size_t esz = f.type == dtype::float32 ? 4 : 8;
  const size_t need = (size_t)prod(og.dims) * esz;
  *need_out = need;
  const double tol = std::max(f.tolerance, p.decode_tolerance);  // Core/idx2Decode.cpp:364
  const int L = f.nlevels;
  const int nsb = f.nsubbands();

  decode_request rq;
  rq.nlevels = L;
  rq.nsb = nsb;
  rq.is2d = f.is2d();
  rq.f32 = f.type == dtype::float32;
  rq.etol = exponent_f64(tol);
  rq.bpc = f.bit_planes_per_chunk;
  if (rq.bpc < 1 || rq.bpc > 8)
    return OptionNotSupported;  // keys of coded planes stay non-negative up to 8 planes per key
  rq.out_from = og.from;
  rq.out_dims = og.dims;
  rq.out_strd = og.strd;
  // decoded levels: from the coarsest down while the mask is not empty
  int lmin = L;
  for (int l = L - 1; l >= 0; --l)
  {
    if (f.decode_masks[(size_t)l] == 0)
      break;
    lmin = l;
  }
  // per level and brick index: the brick's entry in the level's list (-1: not decoded)
  std::vector<std::vector<int>> pos_of((size_t)L);
  for (int l = L - 1; l >= lmin; --l)
  {
    v3 b3 = f.brick_dims;
    for (int k = 0; k < l; ++k)
      b3 = b3 * f.group_brick3;
    v3 bf = ext.from / b3, bl = ext.last() / b3;
    bl = vmin(bl, f.nbricks3[(size_t)l] - v3(1));
    pos_of[(size_t)l].assign(h->brick3[(size_t)l].size(), -1);
    decode_level lv;
    lv.level = l;
    lv.mask = f.decode_masks[(size_t)l];
    lv.is_output = (l == 0 || f.decode_masks[(size_t)l - 1] == 0);
    for (int s = 0; s < nsb; ++s)
      for (int d = 0; d < 3; ++d)
        lv.spacing[s][d] = f.decode_spacings[(size_t)l][(size_t)s][d];
    // the exponent chunk of each subband that was found last (bricks of a chunk come in runs)
    std::vector<u64> chunk_seen((size_t)nsb, ~0ull);
    const brick_linearizer lin_of(f, l, f.nbricks3[(size_t)l]);
    const brick_linearizer plin_of(f, l + 1 < L ? l + 1 : l, l + 1 < L ? f.nbricks3[(size_t)l + 1] : v3(0));
    if (bl.x >= bf.x && bl.y >= bf.y && bl.z >= bf.z)
    {
      const size_t nbox = (size_t)(bl.x - bf.x + 1) * (size_t)(bl.y - bf.y + 1) * (size_t)(bl.z - bf.z + 1);
      lv.bricks.reserve(nbox);
      lv.b3.reserve(nbox);
    }
    for (int bz = bf.z; bz <= bl.z; ++bz)
      for (int by = bf.y; by <= bl.y; ++by)
        for (int bx = bf.x; bx <= bl.x; ++bx)
        {
          v3 b(bx, by, bz);
          u64 lin = lin_of(b);
          if (lin >= h->brick_index[(size_t)l].size())
            continue;
          int bi = h->brick_index[(size_t)l][lin];
          if (bi < 0)
            continue;
          // the reference reads the brick's exponents for every decoded subband first and
          // fails with FileNotFound / ChunkNotFound when its file or exponent chunk is absent
          // (Core/idx2Decode.cpp:104-106, Core/idx2Read.cpp:378-388)
          if (!h->bad_files[(size_t)l].empty())
          {
            auto bf = h->bad_files[(size_t)l].find(lin >> h->file_shift[(size_t)l]);
            if (bf != h->bad_files[(size_t)l].end())
              return bf->second;
          }
          for (int s = 0; s < nsb; ++s)
          {
            if (!((lv.mask >> s) & 1))
              continue;
            const u64 ca = chunk_address(f, lin, l, s, 0);
            if (ca == chunk_seen[(size_t)s])
              continue;
            if (!h->exp_chunk_addrs.count(ca))
              return ChunkNotFound;
            chunk_seen[(size_t)s] = ca;
          }
          decode_brick db;
          db.flat = (long long)(h->level_brick_base[(size_t)l] + (size_t)bi);
          db.parent = -1;
          db.pos[0] = db.pos[1] = db.pos[2] = 0;
          if (l + 1 < L)
          {
            v3 pb = b / f.group_brick3;
            u64 plin = plin_of(pb);
            int pbi = plin < h->brick_index[(size_t)l + 1].size() ? h->brick_index[(size_t)l + 1][plin] : -1;
            db.parent = pbi >= 0 && (size_t)pbi < pos_of[(size_t)l + 1].size() ? pos_of[(size_t)l + 1][(size_t)pbi] : -1;
            v3 lp = b % f.group_brick3;
            db.pos[0] = lp.x;
            db.pos[1] = lp.y;
            db.pos[2] = lp.z;
          }
          if (lv.is_output)
          {
            // Core/idx2Decode.cpp:431-442
            grid bg;
            bg.from = b * b3;
            bg.dims = f.brick_dims;
            bg.strd = v3(1 << l);
            grid ob = crop(og, bg);
            if (prod(ob.dims) <= 0)
              continue;
            grid local = relative(ob, bg);
            grid dst = relative(ob, og);
            for (int d = 0; d < 3; ++d)
            {
              db.src_from[d] = local.from[d];
              db.src_strd[d] = local.strd[d];
              db.dims[d] = ob.dims[d];
              db.dst_from[d] = dst.from[d];
              db.dst_strd[d] = dst.strd[d];
            }
          }
          db.req = 0;
          db.store = lv.is_output ? -1 : (int)lv.bricks.size();
          pos_of[(size_t)l][bi] = (int)lv.bricks.size();
          lv.bricks.push_back(db);
          lv.b3.push_back(b);
        }
    for (int s = 0; s < nsb; ++s)
    {
      std::vector<block_geom> g;
      subband_blocks(f, l, s, &g);
      lv.nblocks[s] = (int)g.size();
      for (size_t b = 0; b < g.size(); ++b)
        lv.geom[s][b] = (uint64_t)g[b].dx | ((uint64_t)g[b].dy << 8) | ((uint64_t)g[b].dz << 16) |
                        ((uint64_t)g[b].bx << 24) | ((uint64_t)g[b].by << 32) | ((uint64_t)g[b].bz << 40);
    }
    // de-normalisation weights (Core/Wavelet.cpp:151-177)
    double scal[16], wave[16];
    double n1 = 3, n2 = 23;
    for (int i = 0; i < 16; ++i)
    {
      scal[i] = sqrt(n1 / (1 << (i + 1)));
      n1 = n1 * 4 - 1;
      wave[i] = sqrt(n2 / (1 << (i + 5)));
      n2 = n2 * 4 - 33;
    }
    lv.norm_mask = 0;
    for (int s = 0; s < nsb; ++s)
    {
      const subband& sb = f.subbands[(size_t)s];
      double wx = f.brick_dims_ext.x == 1 ? 1
                  : (sb.low_high.x == 0 ? scal[l + sb.level_rev.x - 1] : wave[l + sb.level_rev.x]);
      double wy = f.brick_dims_ext.y == 1 ? 1
                  : (sb.low_high.y == 0 ? scal[l + sb.level_rev.y - 1] : wave[l + sb.level_rev.y]);
      double wz = f.brick_dims_ext.z == 1 ? 1
                  : (sb.low_high.z == 0 ? scal[l + sb.level_rev.z - 1] : wave[l + sb.level_rev.z]);
      lv.inv_weight[s] = 1.0 / (wx * wy * wz);
      if (!(s == 0 && l + 1 != L))
        lv.norm_mask |= 1 << s;
    }
    rq.levels.push_back(std::move(lv));
  }
  *rq_out = std::move(rq);
  return NoError;
}

int dataset_decode_batch(device_ctx* ctx, dataset_handle* h, const params* ps, int n, void* const* outs,
                         const size_t* out_bytes, bool out_on_device, double* kernel_ms)
{
  std::vector<decode_request> rqs((size_t)n);
  std::vector<const decode_request*> ptrs((size_t)n);
  std::vector<size_t> need((size_t)n);
  for (int i = 0; i < n; ++i)
  {
    int e = plan_decode(h, ps[i], &rqs[(size_t)i], &need[(size_t)i]);
    if (e)
      return e;
    if (out_bytes[i] < need[(size_t)i])
      return SizeTooSmall;
    ptrs[(size_t)i] = &rqs[(size_t)i];
  }
  return h->dev.decode_batch(ctx, ptrs, outs, need.data(), out_on_device, kernel_ms);
}

int dataset_coeffs(device_ctx* ctx, dataset_handle* h, const params& p, void* d_coeffs, size_t bytes,
                   double* kernel_ms)
{
  params q = p;
  q.has_extent = false;
  q.downsampling = v3(0);
  decode_request rq;
  size_t need = 0;
  int e = plan_decode(h, q, &rq, &need);
  if (e)
    return e;
  const size_t nb = (size_t)(h->f.is2d() ? 33 * 33 : 33 * 33 * 33);
  size_t count = 0;
  for (const decode_level& lv : rq.levels)
    count += lv.bricks.size() * nb;
  if (bytes < count * (h->f.type == dtype::float32 ? 4 : 8))
    return SizeTooSmall;
  std::vector<const decode_request*> rqs(1, &rq);
  void* none = nullptr;
  size_t zero = 0;
  return h->dev.decode_batch(ctx, rqs, &none, &zero, true, kernel_ms, d_coeffs);
}

// The reference's HashMap output (--brick_map; Core/idx2Decode.cpp:446-477 and
// Core/idx2SparseBricks.cpp:69-230): decode the whole field keeping every significant brick,
// give every finest brick the finest level at which its ancestor (or itself) is significant
// (ComputeBrickResolution), and write, for the finest bricks in row-major order, that
// brick's samples over the finest brick's part of it (GetBrickVolume, WriteBricks).
int dataset_decode_brick_map(device_ctx* ctx, dataset_handle* h, const params& p, const char* path,
                             double* kernel_ms)
{
  params q = p;
  q.has_extent = false;
  decode_request rq;
  size_t need = 0;
  int e = plan_decode(h, q, &rq, &need);
  if (e)
    return e;
  decode_keep keep;
  std::vector<const decode_request*> rqs(1, &rq);
  void* none = nullptr;
  size_t zero = 0;
  e = h->dev.decode_batch(ctx, rqs, &none, &zero, true, kernel_ms, nullptr, &keep);
  if (e)
    return e;
  const dataset_format& f = h->f;
  const int L = f.nlevels;
  const bool is2d = f.is2d();
  const size_t NB = is2d ? 33 * 33 : 33 * 33 * 33;
  // level, brick coordinates -> plan index
  std::vector<std::unordered_map<long long, int>> at((size_t)L);
  auto key = [&](int l, const v3& b) {
    const v3 n = f.nbricks3[(size_t)l];
    return ((long long)b.z * n.y + b.y) * n.x + b.x;
  };
  for (const decode_level& lv : rq.levels)
    for (size_t i = 0; i < lv.b3.size(); ++i)
      at[(size_t)lv.level][key(lv.level, lv.b3[i])] = (int)i;
  auto find = [&](int l, const v3& b) -> int {
    auto it = at[(size_t)l].find(key(l, b));
    return it == at[(size_t)l].end() ? -1 : it->second;
  };
  auto group_pow = [&](int r) {
    v3 g(1);
    for (int k = 0; k < r; ++k)
      g = g * f.group_brick3;
    return g;
  };
  const v3 n0 = f.nbricks3[0];
  std::vector<brick_piece> pieces;
  std::vector<v3> dims_of;
  pieces.reserve((size_t)prod(n0));
  long long total = 0;
  for (int bz = 0; bz < n0.z; ++bz)
    for (int by = 0; by < n0.y; ++by)
      for (int bx = 0; bx < n0.x; ++bx)
      {
        const v3 b3(bx, by, bz);
        // ComputeBrickResolution: the finest significant level along the chain, else the
        // coarsest level
        int r = L - 1;
        for (int l = L - 1; l >= 0; --l)
        {
          const int i = find(l, b3 / group_pow(l));
          if (i >= 0 && keep.sig[(size_t)l][(size_t)i])
            r = l;
        }
        const v3 a3 = b3 / group_pow(r);
        const int i = find(r, a3);
        if (i < 0 || !keep.bricks[(size_t)r])
          return BrickNotFound;
        brick_piece pc;
        memset(&pc, 0, sizeof pc);
        pc.src = keep.bricks[(size_t)r] + (size_t)i * NB;
        v3 from(0), dims = f.brick_dims_ext;
        if (r > 0)
        {
          const v3 bd(f.brick_dims.x >> r, f.brick_dims.y >> r, f.brick_dims.z >> r);
          dims = v3(bd.x + (bd.x > 1), bd.y + (bd.y > 1), bd.z + (bd.z > 1));  // idx2_ExtDims
          from = (b3 % group_pow(r)) * bd;
        }
        pc.from[0] = from.x;
        pc.from[1] = from.y;
        pc.from[2] = from.z;
        pc.dims[0] = dims.x;
        pc.dims[1] = dims.y;
        pc.dims[2] = dims.z;
        pc.out = total;
        total += (long long)dims.x * dims.y * dims.z;
        pieces.push_back(pc);
        dims_of.push_back(dims);
      }
  std::vector<double> samples((size_t)total);
  e = decode_device::gather_bricks(ctx, pieces, is2d, (size_t)total, samples.data());
  if (e)
    return e;
  FILE* fp = fopen(path, "wb");
  if (!fp)
    return FileCreateFailed;
  bool ok = true;
  auto put3 = [&](const v3& v) {
    const int32_t w[3] = { (int32_t)v.x, (int32_t)v.y, (int32_t)v.z };
    ok = ok && fwrite(w, sizeof w, 1, fp) == 1;
  };
  put3(f.dims);
  put3(f.brick_dims);
  put3(n0);
  size_t k = 0;
  for (int bz = 0; bz < n0.z; ++bz)
    for (int by = 0; by < n0.y; ++by)
      for (int bx = 0; bx < n0.x; ++bx, ++k)
      {
        put3(v3(bx, by, bz));
        put3(dims_of[k]);
        const size_t cnt = (size_t)prod(dims_of[k]);
        if (cnt)
          ok = ok && fwrite(samples.data() + pieces[k].out, 8, cnt, fp) == cnt;
      }
  ok = fclose(fp) == 0 && ok;
  return ok ? NoError : FileWriteFailed;
}

void dataset_close(dataset_handle* h)
{
  stage_timer tt;
  delete h;
  tt.lap("close");
}

int dataset_decode_noalloc(device_ctx* ctx, dataset_handle* h, const params& p, void* d_out, size_t out_bytes,
                           double* kernel_ms)
{
  decode_request rq;
  size_t need = 0;
  int e = plan_decode(h, p, &rq, &need);
  if (e)
    return e;
  if (out_bytes < need)
    return SizeTooSmall;
  return h->dev.decode_noalloc(ctx, rq, d_out, need, kernel_ms);
}

const dataset_format& dataset_fmt(const dataset_handle* h) { return h->f; }

size_t dataset_resident_bytes(const dataset_handle* h) { return h->dev.resident_bytes(); }

} // namespace idx2g
