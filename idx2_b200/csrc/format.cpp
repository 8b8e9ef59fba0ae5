// Dataset description and Finalize (Core/idx2Common.cpp:358-785, Core/Wavelet.cpp:407-568,
// Core/idx2Lookup.cpp). The derivations follow the reference step by step because the
// brick/chunk/file orders and the file names they produce are part of the on-disk format.
#include "format.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>

namespace idx2g
{

int log2_floor(i64 v)
{
  int r = -1;
  while (v)
  {
    v >>= 1;
    ++r;
  }
  return r;
}

int log2_ceil(i64 v)
{
  int m = log2_floor(v);
  return m + (v != ((i64)1 << m));
}

bool is_pow2(i64 v) { return v > 0 && (v & (v - 1)) == 0; }

extent crop(const extent& a, const extent& b)
{
  v3 f = vmax(a.from, b.from), l = vmin(a.last(), b.last());
  extent r;
  r.from = f;
  r.dims = all_le(f, l) ? l - f + v3(1) : v3(0);
  return r;
}

grid crop(const grid& a, const grid& b)
{
  // Core/Volume.h:1359 Crop: the result keeps a's stride and lattice
  v3 s = a.strd;
  v3 f = vmax(a.from, b.from);
  v3 al = a.from + (a.dims - v3(1)) * a.strd;
  v3 bl = b.from + (b.dims - v3(1)) * b.strd;
  v3 l = vmin(al, bl);
  f = ((f - a.from + s - v3(1)) / s) * s + a.from;
  l = ((l - a.from) / s) * s + a.from;
  grid r = a;
  r.from = f;
  r.dims = all_le(f, l) ? (l - f) / s + v3(1) : v3(0);
  return r;
}

grid relative(const grid& a, const grid& b)
{
  // Core/Volume.h:1349 Relative
  grid r;
  r.from = (a.from - b.from) / b.strd;
  r.dims = a.dims;
  r.strd = a.strd / b.strd;
  return r;
}

u64 encode_order(const std::string& s)
{
  u64 r = 0;
  for (int i = (int)s.size() - 1; i >= 0; --i)
  {
    char c = s[(size_t)i];
    int t = c == '+' ? 3 : c - 'X';
    r = (r << 2) + (u64)t;
  }
  return r;
}

std::string decode_order(u64 order)
{
  std::string s;
  while (order != 0)
  {
    int t = (int)(order & 3);
    s.push_back(t == 3 ? '+' : char('X' + t));
    order >>= 2;
  }
  return s;
}

static int next_pow2(int v)
{
  int r = 1;
  while (r < v)
    r <<= 1;
  return r;
}

std::string decode_order_for_dims(u64 input, v3 n3)
{
  // Core/Wavelet.cpp:436
  n3 = v3(next_pow2(n3.x), next_pow2(n3.y), next_pow2(n3.z));
  std::string out;
  u64 saved = input;
  while ((u64)n3.x * (u64)n3.y * (u64)n3.z > 1)
  {
    int t = (int)(input & 3);
    input >>= 2;
    if (t == 3)
    {
      if (input == 3)
        input = saved;
      else
        saved = input;
    }
    else
    {
      out.push_back(char('X' + t));
      n3[t] >>= 1;
    }
  }
  return out;
}

int decode_order_passes(u64 input, int passes, std::string* out)
{
  // Core/Wavelet.cpp:464
  out->clear();
  u64 saved = input;
  v3 p3(passes);
  while (true)
  {
    int t = (int)(input & 3);
    input >>= 2;
    if (t == 3)
    {
      if (input == 3)
        input = saved;
      else
        saved = input;
    }
    else
    {
      --p3[t];
      if (p3[t] < 0)
        break;
      out->push_back(char('X' + t));
    }
  }
  return (int)out->size();
}

// Core/Wavelet.cpp:503 BuildSubbands
static void build_subbands(v3 n3, int nlevels, u64 order, std::vector<subband>* out)
{
  struct sb
  {
    grid g;
    v3 level3, level3rev, low_high;
    int level;
  };
  std::deque<sb> q;
  std::vector<sb> res;
  sb first;
  first.g.from = v3(0);
  first.g.dims = n3;
  first.g.strd = v3(1);
  first.level3 = first.level3rev = first.low_high = v3(0);
  first.level = 0;
  q.push_back(first);
  int level = 0;
  u64 prev = order;
  while (level < nlevels)
  {
    int d = (int)(order & 3);
    order >>= 2;
    if (d == 3)
    {
      if (order == 3)
        order = prev;
      else
        prev = order;
      int sz = (int)q.size();
      for (int i = sz - 1; i >= 1; --i)
      {
        res.push_back(q[(size_t)i]);
        q.pop_back();
      }
      ++level;
    }
    else
    {
      int sz = (int)q.size();
      for (int i = 0; i < sz; ++i)
      {
        sb cur = q.front();
        // Core/Volume.cpp:175 SplitAlternate
        grid lo = cur.g, hi = cur.g;
        lo.dims[d] = (cur.g.dims[d] + 1) >> 1;
        lo.strd[d] = cur.g.strd[d] << 1;
        hi.dims[d] = cur.g.dims[d] - lo.dims[d];
        hi.strd[d] = cur.g.strd[d] << 1;
        hi.from[d] = cur.g.from[d] + cur.g.strd[d];
        sb a = cur, b = cur;
        a.g = lo;
        a.level3[d] += 1;
        a.level3rev = a.level3;
        a.low_high = cur.low_high;
        a.level = level;
        b.g = hi;
        b.level3 = cur.level3;
        b.level3rev = cur.level3;
        b.low_high = cur.low_high;
        b.low_high[d] = 1;
        b.level = level;
        q.push_back(a);
        q.push_back(b);
        q.pop_front();
      }
    }
  }
  if (!q.empty())
    res.push_back(q.front());
  out->clear();
  for (int i = (int)res.size() - 1; i >= 0; --i)
  {
    subband s;
    s.g = res[(size_t)i].g;
    s.low_high = res[(size_t)i].low_high;
    s.level_rev = res[(size_t)i].level3rev;
    out->push_back(s);
  }
}

static int set_from_params(dataset_format* f, const params& p)
{
  f->name = p.name;
  f->field = p.field;
  f->version[0] = p.version[0];
  f->version[1] = p.version[1];
  f->dims = p.dims;
  f->type = p.type;
  f->brick_dims = p.brick_dims;
  f->bricks_per_chunk_in = p.bricks_per_chunk;
  f->chunks_per_file_in = p.chunks_per_file;
  f->bit_planes_per_chunk = p.bit_planes_per_chunk;
  f->nlevels = (int)(int8_t)p.num_levels;
  f->tolerance = p.tolerance;
  f->files_per_dir = p.files_per_dir;
  f->dir = p.out_dir;
  return NoError;
}

static int finalize_common(dataset_format* f, params* p)
{
  // CheckBrickSize (Core/idx2Common.cpp:359)
  if (!(is_pow2(f->brick_dims.x) && is_pow2(f->brick_dims.y) && is_pow2(f->brick_dims.z)))
    return BrickSizeNotPowerOfTwo;
  if (!all_le(f->brick_dims, f->dims))
    return BrickSizeTooBig;
  p->tolerance = std::fmax(std::fabs(p->tolerance), f->tolerance);
  // GuessNumLevelsIfNeeded (:666)
  if (f->nlevels == 0)
  {
    v3 b = f->brick_dims;
    while (all_le(b, f->dims))
    {
      b.x = b.x == 1 ? b.x : b.x * 2;
      b.y = b.y == 1 ? b.y : b.y * 2;
      b.z = b.z == 1 ? b.z : b.z * 2;
      if (all_le(b, f->dims))
        ++f->nlevels;
    }
  }
  if (!(f->nlevels <= 16))
    return TooManyLevels;
  if (f->bit_planes_per_chunk > f->bit_planes_per_file ||
      (f->bit_planes_per_file % f->bit_planes_per_chunk) != 0)
    return SizeMismatched;
  if (f->nlevels <= 0)
    return TooManyLevels;

  // ComputeTransformOrder (:374)
  std::string tform;
  for (int d = 0; d < 3; ++d)
    if (f->brick_dims[d] > 1)
      tform.push_back(char('X' + d));
  tform += "++";
  f->transform_order = encode_order(tform);
  decode_order_passes(f->transform_order, 1, &f->transform_order_full);

  // BuildSubbands (:403)
  f->brick_dims_ext = v3(f->brick_dims.x + (f->brick_dims.x > 1), f->brick_dims.y + (f->brick_dims.y > 1),
                         f->brick_dims.z + (f->brick_dims.z > 1));
  build_subbands(f->brick_dims_ext, 1, f->transform_order, &f->subbands);
  build_subbands(f->brick_dims, 1, f->transform_order, &f->subbands_nonext);
  {
    v3 spacing3(1 << f->downsampling.x, 1 << f->downsampling.y, 1 << f->downsampling.z);
    int nsb = (int)f->subbands.size();
    std::vector<std::vector<v3>> sp(f->nlevels, std::vector<v3>(nsb));
    f->decode_masks.assign(f->nlevels, 0);
    f->decode_spacings.assign(f->nlevels, std::vector<v3>(nsb, v3(1)));
    for (int i = 0; i < f->nlevels; ++i)
    {
      int mask = 0xFF;
      for (int s = 0; s < nsb; ++s)
      {
        v3 mul = i > 0 ? sp[i - 1][0] : v3(1);
        v3 f3 = f->subbands[s].g.from * mul;
        v3 s3 = f->subbands[s].g.strd * mul;
        sp[i][s] = s3;
        f->decode_spacings[i][s] = v3(1);
        for (int d = 0; d < 3; ++d)
        {
          if (f3[d] % spacing3[d] == 0)
          {
            if (s3[d] % spacing3[d] != 0)
              f->decode_spacings[i][s][d] = spacing3[d] / s3[d];
          }
          else
            mask &= ~(1 << s);
        }
      }
      if (i + 1 < f->nlevels && mask == 1)
        mask = 0;
      f->decode_masks[i] = (uint8_t)mask;
    }
  }

  // ComputeNumBricksPerLevel (:464)
  f->group_brick3 = f->brick_dims / f->subbands_nonext[0].g.dims;
  {
    v3 nb = (f->dims + f->brick_dims - v3(1)) / f->brick_dims;
    f->nbricks3.assign(f->nlevels, v3(0));
    for (int i = 0; i < f->nlevels; ++i)
    {
      f->nbricks3[i] = nb;
      nb = (nb + f->group_brick3 - v3(1)) / f->group_brick3;
    }
  }

  // ComputeGlobalBricksOrder (:479)
  f->bricks_order.assign(f->nlevels, 0);
  f->bricks_order_str.assign(f->nlevels, "");
  for (int i = 0; i < f->nlevels; ++i)
  {
    v3 n3 = f->nbricks3[i];
    v3 logn(log2_ceil(n3.x), log2_ceil(n3.y), log2_ceil(n3.z));
    int minlog = std::min(logn.x, std::min(logn.y, logn.z));
    v3 left = logn - v3(f->brick_dims.x > 1, f->brick_dims.y > 1, f->brick_dims.z > 1) * v3(minlog);
    std::string bo;
    for (int d = 0; d < 3; ++d)
      if (f->brick_dims[d] == 1)
        while (left[d]-- > 0)
          bo.push_back(char('X' + d));
    while (!all_le(left, v3(0)))
      for (int d = 0; d < 3; ++d)
        if (left[d]-- > 0)
          bo.push_back(char('X' + d));
    if (!bo.empty())
      bo.push_back('+');
    bo += tform;
    f->bricks_order[i] = encode_order(bo);
    f->bricks_order_str[i] = decode_order_for_dims(f->bricks_order[i], n3);
    if (f->bricks_order_str[i].size() < f->transform_order_full.size())
      return TooManyLevels;
  }

  // ComputeLocalBricksChunksFilesOrders (:525)
  if (!(f->bricks_per_chunk_in <= 32768))
    return TooManyBricksPerChunk;
  if (!is_pow2(f->bricks_per_chunk_in))
    return BricksPerChunkNotPowerOf2;
  if (!(f->chunks_per_file_in <= 4906))
    return TooManyChunksPerFile;
  if (!is_pow2(f->chunks_per_file_in))
    return ChunksPerFileNotPowerOf2;
  int L = f->nlevels;
  f->bricks_per_chunk.assign(L, 0);
  f->chunks_per_file.assign(L, 0);
  f->bricks_per_file.assign(L, 0);
  f->bricks_per_chunk3.assign(L, v3(1));
  f->chunks_per_file3.assign(L, v3(1));
  f->nchunks3.assign(L, v3(0));
  f->nfiles3.assign(L, v3(0));
  f->bricks_order_in_chunk.assign(L, 0);
  f->chunks_order_in_file.assign(L, 0);
  f->chunks_order.assign(L, 0);
  f->files_order.assign(L, 0);
  f->chunks_order_str.assign(L, "");
  f->files_order_str.assign(L, "");
  f->files_dirs_depth.assign(L, {});
  for (int i = 0; i < L; ++i)
  {
    const std::string& bos = f->bricks_order_str[i];
    int len = (int)bos.size();
    f->bricks_per_chunk[i] = 1 << std::min(log2_ceil(f->bricks_per_chunk_in), len);
    int boic_len = log2_ceil(f->bricks_per_chunk[i]);
    std::string boic((size_t)boic_len, ' ');
    f->bricks_per_chunk3[i] = v3(1);
    for (int j = 0; j < boic_len; ++j)
    {
      char c = bos[(size_t)(len - j - 1)];
      f->bricks_per_chunk3[i][c - 'X'] *= 2;
      boic[(size_t)(boic_len - j - 1)] = c;
    }
    f->bricks_order_in_chunk[i] = encode_order(boic);

    f->nchunks3[i] =
      (f->nbricks3[i] + f->bricks_per_chunk3[i] - v3(1)) / f->bricks_per_chunk3[i];
    f->chunks_per_file[i] = 1 << std::min(log2_ceil(f->chunks_per_file_in), len - boic_len);
    int coif_len = log2_ceil(f->chunks_per_file[i]);
    std::string coif((size_t)coif_len, ' ');
    f->chunks_per_file3[i] = v3(1);
    for (int j = 0; j < coif_len; ++j)
    {
      char c = bos[(size_t)(len - boic_len - j - 1)];
      f->chunks_per_file3[i][c - 'X'] *= 2;
      coif[(size_t)(coif_len - j - 1)] = c;
    }
    f->chunks_order_in_file[i] = encode_order(coif);
    f->nfiles3[i] =
      (f->nchunks3[i] + f->chunks_per_file3[i] - v3(1)) / f->chunks_per_file3[i];

    {
      int chunks_per_vol = 1 << (len - boic_len);
      int co_len = log2_ceil(chunks_per_vol);
      std::string co((size_t)co_len, ' ');
      for (int j = 0; j < co_len; ++j)
        co[(size_t)(co_len - j - 1)] = bos[(size_t)(len - boic_len - j - 1)];
      f->chunks_order[i] = encode_order(co);
      f->chunks_order_str[i] = decode_order_for_dims(f->chunks_order[i], f->nchunks3[i]);
    }
    {
      int files_per_vol = 1 << (len - boic_len - coif_len);
      int fo_len = log2_ceil(files_per_vol);
      std::string fo((size_t)fo_len, ' ');
      for (int j = 0; j < fo_len; ++j)
        fo[(size_t)(fo_len - j - 1)] = bos[(size_t)(len - boic_len - coif_len - j - 1)];
      f->files_order[i] = encode_order(fo);
      f->files_order_str[i] = decode_order_for_dims(f->files_order[i], f->nfiles3[i]);
    }
  }

  // ComputeFileDirDepths (:627)
  if (!(f->files_per_dir <= 4096))
    return TooManyFilesPerDir;
  for (int i = 0; i < L; ++i)
  {
    f->bricks_per_file[i] = f->bricks_per_chunk[i] * f->chunks_per_file[i];
    std::vector<int>& dd = f->files_dirs_depth[i];
    dd.clear();
    int acc = log2_ceil(f->bricks_per_file[i]);
    dd.push_back(acc);
    int len = (int)f->bricks_order_str[i].size();
    while (acc < len)
    {
      int inc = std::min(len - acc, log2_ceil(f->files_per_dir));
      dd.push_back(inc);
      acc += inc;
      // the depth is limited to 4 (idx2_file::MaxSpatialDepth); with one file per directory
      // (inc = 0) the reference's loop never ends, here it is the same error
      if (dd.size() > 4)
        return TooManyFilesPerDir;
    }
    if (dd.size() > 4)
      return TooManyFilesPerDir;
    std::vector<int> r(dd.rbegin(), dd.rend());
    dd = r;
  }
  return NoError;
}

int finalize(dataset_format* f, params* p)
{
  set_from_params(f, *p);
  return finalize_common(f, p);
}

int finalize_read(dataset_format* f, params* p)
{
  f->dir = p->in_dir;
  f->downsampling = p->downsampling;
  int e = finalize_common(f, p);
  if (e != NoError)
    return e;
  if (!p->has_extent)
  {
    p->decode_extent.from = v3(0);
    p->decode_extent.dims = f->dims;
  }
  return NoError;
}

u64 linear_brick(const dataset_format& f, int level, v3 b3)
{
  const std::string& s = f.bricks_order_str[level];
  int n = (int)s.size();
  u64 r = 0;
  for (int i = n - 1; i >= 0; --i)
  {
    int d = s[(size_t)i] - 'X';
    r |= ((u64)b3[d] & 1u) << (n - i - 1);
    b3[d] >>= 1;
  }
  return r;
}

brick_linearizer::brick_linearizer(const dataset_format& fmt, int l, v3 n) : f(&fmt), level(l)
{
  for (int d = 0; d < 3; ++d)
  {
    const int m = n[d] > 0 ? n[d] : 0;
    t[d].resize((size_t)m);
    for (int c = 0; c < m; ++c)
    {
      v3 b(0);
      b[d] = c;
      t[d][(size_t)c] = linear_brick(fmt, l, b);
    }
  }
}

v3 spatial_brick(const dataset_format& f, int level, u64 lin)
{
  const std::string& s = f.bricks_order_str[level];
  int n = (int)s.size();
  v3 b(0);
  for (int i = 0; i < n; ++i)
  {
    int d = s[(size_t)i] - 'X';
    int j = n - i - 1;
    b[d] |= (int)((lin >> j) & 1u);
    b[d] <<= 1;
  }
  return v3(b.x >> 1, b.y >> 1, b.z >> 1);
}

u64 chunk_address(const dataset_format& f, u64 brick, int level, int subband, int bpkey)
{
  return get_address(brick, log2_ceil(f.bricks_per_chunk[level]), level, subband, bpkey);
}

u64 file_address(const dataset_format& f, u64 brick, int level)
{
  return get_address(brick, log2_ceil(f.bricks_per_file[level]), level, 0, 0);
}

std::string file_path(const dataset_format& f, u64 brick, int level)
{
  // Core/idx2Lookup.cpp:78 ConstructFilePath
  char buf[512];
  std::string out = f.dir + "/" + f.name + "/" + f.field + "/";
  snprintf(buf, sizeof buf, "L%02x", level);
  out += buf;
  const std::vector<int>& dd = f.files_dirs_depth[level];
  int len = (int)f.bricks_order_str[level].size();
  for (size_t depth = 0; depth + 1 < dd.size(); ++depth)
  {
    int bitlen = 64 - len + dd[depth];
    u64 top = bitlen >= 64 ? brick : (brick >> (64 - bitlen));
    snprintf(buf, sizeof buf, "/B%llx", (unsigned long long)top);
    out += buf;
    brick <<= dd[depth];
  }
  out += ".bin";
  return out;
}

grid output_grid(const dataset_format& f, const extent& ext)
{
  extent c = crop(ext, extent{ v3(0), f.dims });
  v3 s(1 << f.downsampling.x, 1 << f.downsampling.y, 1 << f.downsampling.z);
  v3 first = c.from, last = c.last();
  last = ((last + s - v3(1)) / s) * s;
  first = (first / s) * s;
  grid g;
  g.from = first;
  g.dims = (last - first) / s + v3(1);
  g.strd = s;
  return g;
}

std::string meta_text(const dataset_format& f, const params& p)
{
  // Core/idx2Common.cpp:150 WriteMetaFile
  std::string o;
  char buf[512];
  o += "(\n";
  o += "  (common\n";
  o += "    (type \"Simulation\")\n";
  snprintf(buf, sizeof buf, "    (name \"%s\")\n", p.name.c_str());
  o += buf;
  snprintf(buf, sizeof buf, "    (field \"%s\")\n", p.field.c_str());
  o += buf;
  snprintf(buf, sizeof buf, "    (dimensions %d %d %d)\n", f.dims.x, f.dims.y, f.dims.z);
  o += buf;
  snprintf(buf, sizeof buf, "    (data-type \"%s\")\n",
           f.type == dtype::float32 ? "float32" : "float64");
  o += buf;
  snprintf(buf, sizeof buf, "    (min-max %.20f %.20f)\n", f.value_min, f.value_max);
  o += buf;
  snprintf(buf, sizeof buf, "    (accuracy %.20f)\n", f.tolerance);
  o += buf;
  o += "  )\n";
  o += "  (format\n";
  snprintf(buf, sizeof buf, "    (version %d %d)\n", f.version[0], f.version[1]);
  o += buf;
  snprintf(buf, sizeof buf, "    (brick-size %d %d %d)\n", f.brick_dims.x, f.brick_dims.y,
           f.brick_dims.z);
  o += buf;
  snprintf(buf, sizeof buf, "    (transform-order \"%s\")\n", decode_order(f.transform_order).c_str());
  o += buf;
  snprintf(buf, sizeof buf, "    (num-levels %d)\n", f.nlevels);
  o += buf;
  snprintf(buf, sizeof buf, "    (transform-passes-per-levels %d)\n", 1);
  o += buf;
  snprintf(buf, sizeof buf, "    (bricks-per-chunk %d)\n", f.bricks_per_chunk_in);
  o += buf;
  snprintf(buf, sizeof buf, "    (chunks-per-file %d)\n", f.chunks_per_file_in);
  o += buf;
  snprintf(buf, sizeof buf, "    (files-per-directory %d)\n", f.files_per_dir);
  o += buf;
  snprintf(buf, sizeof buf, "    (bit-planes-per-chunk %d)\n", f.bit_planes_per_chunk);
  o += buf;
  o += "  )\n";
  o += ")\n";
  return o;
}

// A minimal s-expression reader for the metadata file: lists of an identifier
// followed by strings / numbers (the grammar WriteMetaFile produces).
namespace
{
struct tok
{
  int kind; // 0 '(' 1 ')' 2 id 3 string 4 number
  std::string s;
};

bool tokenize(const std::string& t, std::vector<tok>* out)
{
  size_t i = 0, n = t.size();
  while (i < n)
  {
    char c = t[i];
    if (c == ';')
    {
      while (i < n && t[i] != '\n')
        ++i;
    }
    else if (c == '(' || c == ')')
    {
      out->push_back({ c == '(' ? 0 : 1, "" });
      ++i;
    }
    else if (c == '"')
    {
      size_t j = i + 1;
      while (j < n && t[j] != '"')
        ++j;
      if (j >= n)
        return false;
      out->push_back({ 3, t.substr(i + 1, j - i - 1) });
      i = j + 1;
    }
    else if (isspace((unsigned char)c))
      ++i;
    else
    {
      size_t j = i;
      while (j < n && !isspace((unsigned char)t[j]) && t[j] != '(' && t[j] != ')' && t[j] != '"')
        ++j;
      std::string w = t.substr(i, j - i);
      bool num = !w.empty() && (isdigit((unsigned char)w[0]) || w[0] == '-' || w[0] == '+' || w[0] == '.');
      out->push_back({ num ? 4 : 2, w });
      i = j;
    }
  }
  return true;
}
} // namespace

int parse_meta(const std::string& text, dataset_format* f)
{
  // Only the leading s-expression is read; the statistics appended after it are text.
  std::vector<tok> tk;
  size_t end = text.size();
  {
    int depth = 0;
    bool started = false;
    bool in_str = false;
    for (size_t i = 0; i < text.size(); ++i)
    {
      char c = text[i];
      if (c == '"')
        in_str = !in_str;
      if (in_str)
        continue;
      if (c == '(')
      {
        ++depth;
        started = true;
      }
      else if (c == ')')
      {
        --depth;
        if (started && depth == 0)
        {
          end = i + 1;
          break;
        }
      }
    }
  }
  if (!tokenize(text.substr(0, end), &tk))
    return SyntaxError;
  int depth = 0;
  for (size_t i = 0; i < tk.size(); ++i)
  {
    if (tk[i].kind == 0)
    {
      ++depth;
      continue;
    }
    if (tk[i].kind == 1)
    {
      --depth;
      if (depth < 0)
        return SyntaxError;
      continue;
    }
    if (tk[i].kind != 2 || i == 0 || tk[i - 1].kind != 0)
      continue;
    const std::string& id = tk[i].s;
    std::vector<std::string> args;
    for (size_t j = i + 1; j < tk.size() && (tk[j].kind == 3 || tk[j].kind == 4); ++j)
      args.push_back(tk[j].s);
    auto ai = [&](size_t k) { return k < args.size() ? atoi(args[k].c_str()) : 0; };
    if (id == "version" && args.size() >= 2)
    {
      f->version[0] = ai(0);
      f->version[1] = ai(1);
    }
    else if (id == "name" && !args.empty())
      f->name = args[0];
    else if (id == "field" && !args.empty())
      f->field = args[0];
    else if (id == "dimensions" && args.size() >= 3)
      f->dims = v3(ai(0), ai(1), ai(2));
    else if (id == "accuracy" && !args.empty())
      f->tolerance = strtod(args[0].c_str(), nullptr);
    else if (id == "data-type" && !args.empty())
    {
      if (args[0] == "float32")
        f->type = dtype::float32;
      else if (args[0] == "float64")
        f->type = dtype::float64;
      else
        return TypeNotSupported;
    }
    else if (id == "min-max" && args.size() >= 2)
    {
      f->value_min = strtod(args[0].c_str(), nullptr);
      f->value_max = strtod(args[1].c_str(), nullptr);
    }
    else if (id == "brick-size" && args.size() >= 3)
      f->brick_dims = v3(ai(0), ai(1), ai(2));
    else if (id == "transform-order" && !args.empty())
      f->transform_order = encode_order(args[0]);
    else if (id == "num-levels" && !args.empty())
      f->nlevels = (int)(int8_t)ai(0);
    else if (id == "bricks-per-chunk" && !args.empty())
      f->bricks_per_chunk_in = ai(0);
    else if (id == "chunks-per-file" && !args.empty())
      f->chunks_per_file_in = ai(0);
    else if (id == "files-per-directory" && !args.empty())
      f->files_per_dir = ai(0);
    else if (id == "bit-planes-per-chunk" && !args.empty())
      f->bit_planes_per_chunk = ai(0);
  }
  if (depth != 0)
    return SyntaxError;
  return NoError;
}

// Subband normalisation weights of one level (Core/Wavelet.cpp:111-137, Core/Wavelet.h:19).
void level_weights(const dataset_format& f, int level, double w[8], int* mask)
{
  double scal[16], wave[16];
  double n1 = 3, n2 = 23;
  for (int i = 0; i < 16; ++i)
  {
    scal[i] = sqrt(n1 / (1 << (i + 1)));
    n1 = n1 * 4 - 1;
    wave[i] = sqrt(n2 / (1 << (i + 5)));
    n2 = n2 * 4 - 33;
  }
  const bool coarsest = level + 1 == f.nlevels;
  *mask = 0;
  for (int s = 0; s < f.nsubbands(); ++s)
  {
    const subband& sb = f.subbands[(size_t)s];
    double wx = f.brick_dims_ext.x == 1 ? 1
                : (sb.low_high.x == 0 ? scal[level + sb.level_rev.x - 1] : wave[level + sb.level_rev.x]);
    double wy = f.brick_dims_ext.y == 1 ? 1
                : (sb.low_high.y == 0 ? scal[level + sb.level_rev.y - 1] : wave[level + sb.level_rev.y]);
    double wz = f.brick_dims_ext.z == 1 ? 1
                : (sb.low_high.z == 0 ? scal[level + sb.level_rev.z - 1] : wave[level + sb.level_rev.z]);
    w[s] = wx * wy * wz;
    if (s == 0 && !coarsest)
      continue;
    *mask |= 1 << s;
  }
}


} // namespace idx2g
