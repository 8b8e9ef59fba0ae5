// Level-1 zstd frame compressor, byte-identical to zstd 1.4.5 (see zstd_frame.h).
//
// The steps restate the published zstd 1.4.5 compressor as the reference vendors it
// (Core/zstd/zstd.c; section names below are that release's): frame and block headers
// (RFC 8878), parameter selection (ZSTD_getCParams + ZSTD_adjustCParams at level 1), the fast
// match finder (zstd_fast.c, ZSTD_compressBlock_fast_generic), literal compression
// (zstd_compress_literals.c, huf_compress.c), sequence encoding (zstd_compress_sequences.c,
// fse_compress.c, entropy_common.c) and the block decisions of zstd_compress.c. Every
// numeric rule that decides an output byte is kept; the code structure is this file's own.
#include "zstd_frame.h"

#include <algorithm>
#include <cstring>

namespace idx2g
{
namespace zstd145
{

namespace
{

using u8 = uint8_t;
using u16 = uint16_t;
using u32 = uint32_t;
using u64 = uint64_t;
using i16 = int16_t;

inline u32 highbit32(u32 v) { return 31u - (u32)__builtin_clz(v); }  // v > 0
inline u32 rd32(const u8* p)
{
  u32 v;
  memcpy(&v, p, 4);
  return v;
}
inline u64 rd64(const u8* p)
{
  u64 v;
  memcpy(&v, p, 8);
  return v;
}

// ---------------------------------------------------------------------------------------------
// format constants (RFC 8878 section 3.1.1.3.2)

constexpr int kMaxLL = 35, kMaxML = 52, kMaxOff = 31, kDefaultMaxOff = 28;
constexpr u32 kLLFSELog = 9, kMLFSELog = 9, kOffFSELog = 8;
constexpr u32 kLLBits[kMaxLL + 1] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  1,  1,
                                      1, 1, 2, 2, 3, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16 };
constexpr u32 kMLBits[kMaxML + 1] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                      0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1,
                                      2, 2, 3, 3, 4, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16 };
constexpr i16 kLLDefaultNorm[kMaxLL + 1] = { 4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2,
                                             2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1 };
constexpr i16 kMLDefaultNorm[kMaxML + 1] = { 1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                             1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                             1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1 };
constexpr i16 kOFDefaultNorm[kDefaultMaxOff + 1] = { 1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1,
                                                     1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1 };
constexpr u32 kLLDefaultLog = 6, kMLDefaultLog = 6, kOFDefaultLog = 5;

u32 ll_code(u32 ll)
{
  static const u8 t[64] = { 0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15,
                            16, 16, 17, 17, 18, 18, 19, 19, 20, 20, 20, 20, 21, 21, 21, 21,
                            22, 22, 22, 22, 22, 22, 22, 22, 23, 23, 23, 23, 23, 23, 23, 23,
                            24, 24, 24, 24, 24, 24, 24, 24, 24, 24, 24, 24, 24, 24, 24, 24 };
  return ll > 63 ? highbit32(ll) + 19 : t[ll];
}

u32 ml_code(u32 mlb)
{
  if (mlb > 127)
    return highbit32(mlb) + 36;
  if (mlb < 32)
    return mlb;
  // 32..127: codes 32..42, each code doubling its range after 35
  static const u8 t[96] = { 32, 32, 33, 33, 34, 34, 35, 35, 36, 36, 36, 36, 37, 37, 37, 37, 38, 38, 38, 38,
                            38, 38, 38, 38, 39, 39, 39, 39, 39, 39, 39, 39, 40, 40, 40, 40, 40, 40, 40, 40,
                            40, 40, 40, 40, 40, 40, 40, 40, 41, 41, 41, 41, 41, 41, 41, 41, 41, 41, 41, 41,
                            41, 41, 41, 41, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42,
                            42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42, 42 };
  return t[mlb - 32];
}

// ---------------------------------------------------------------------------------------------
// LSB-first bit stream (the format's forward bit streams: FSE, Huffman and sequence streams)

struct bit_writer
{
  // The stream goes to out[start, pos); out is grown ahead in steps (its tail past pos is
  // scratch until close() cuts it), so that the accumulator's whole bytes are stored with one
  // 8-byte store.
  std::vector<u8>* out;
  size_t start, pos;
  u64 acc = 0;
  unsigned n = 0;  // bits held in acc
  explicit bit_writer(std::vector<u8>* o) : out(o), start(o->size()), pos(o->size()) { grow(); }
  void grow()
  {
    constexpr size_t kStep = 4096;
    out->resize(pos + kStep);
  }
  // nb bits of v, not stored yet (n + nb <= 64)
  void put(u64 v, unsigned nb)
  {
    acc |= (v & ((1ull << nb) - 1)) << n;
    n += nb;
  }
  // stores the whole bytes held; fewer than 8 bits stay
  void flush()
  {
    if (pos + 8 > out->size())
      grow();
    memcpy(out->data() + pos, &acc, 8);
    const unsigned nbytes = n >> 3;
    pos += nbytes;
    acc = nbytes == 8 ? 0 : acc >> (8 * nbytes);
    n &= 7;
  }
  void add(u64 v, unsigned nb)  // nb <= 32
  {
    put(v, nb);
    if (n >= 32)
      flush();
  }
  // the end mark (one 1 bit) and the last partial byte; returns the stream's size
  size_t close()
  {
    put(1, 1);
    flush();
    if (n)
      (*out)[pos++] = (u8)acc;
    acc = 0;
    n = 0;
    out->resize(pos);
    return pos - start;
  }
};

// ---------------------------------------------------------------------------------------------
// histograms

// counts of src's symbols; *max_sym becomes the largest symbol present; returns the largest count
u32 histogram(const u8* src, size_t n, u32* count, u32* max_sym)
{
  std::fill(count, count + *max_sym + 1, 0u);
  if (n == 0)
  {
    *max_sym = 0;
    return 0;
  }
  for (size_t i = 0; i < n; ++i)
    count[src[i]]++;
  u32 m = *max_sym;
  while (!count[m])
    m--;
  *max_sym = m;
  u32 largest = 0;
  for (u32 s = 0; s <= m; ++s)
    largest = std::max(largest, count[s]);
  return largest;
}

// ---------------------------------------------------------------------------------------------
// FSE (finite state entropy) tables

constexpr u32 kFSEMinLog = 5, kFSEMaxLog = 12, kFSEDefaultLog = 11;

u32 fse_min_log(size_t total, u32 max_sym)
{
  const u32 a = highbit32((u32)total) + 1;
  const u32 b = highbit32(max_sym) + 2;
  return a < b ? a : b;
}

u32 fse_optimal_log(u32 max_log, size_t total, u32 max_sym, u32 minus)
{
  u32 src_bits = highbit32((u32)(total - 1)) - minus;
  u32 log = max_log ? max_log : kFSEDefaultLog;
  const u32 min_bits = fse_min_log(total, max_sym);
  if (src_bits < log)
    log = src_bits;
  if (min_bits > log)
    log = min_bits;
  log = std::max(log, kFSEMinLog);
  log = std::min(log, kFSEMaxLog);
  return log;
}

// Secondary normalisation, for distributions the first method cannot round well.
bool fse_normalize_fallback(i16* norm, u32 log, const u32* count, size_t total, u32 max_sym)
{
  const i16 kUnset = -2;
  u32 distributed = 0;
  const u32 low_threshold = (u32)(total >> log);
  u32 low_one = (u32)((total * 3) >> (log + 1));
  for (u32 s = 0; s <= max_sym; ++s)
  {
    if (count[s] == 0)
    {
      norm[s] = 0;
      continue;
    }
    if (count[s] <= low_threshold)
    {
      norm[s] = -1;
      distributed++;
      total -= count[s];
      continue;
    }
    if (count[s] <= low_one)
    {
      norm[s] = 1;
      distributed++;
      total -= count[s];
      continue;
    }
    norm[s] = kUnset;
  }
  u32 to_distribute = (1u << log) - distributed;
  if (to_distribute == 0)
    return true;
  if ((total / to_distribute) > low_one)
  {
    low_one = (u32)((total * 3) / (to_distribute * 2));
    for (u32 s = 0; s <= max_sym; ++s)
      if (norm[s] == kUnset && count[s] <= low_one)
      {
        norm[s] = 1;
        distributed++;
        total -= count[s];
      }
    to_distribute = (1u << log) - distributed;
  }
  if (distributed == max_sym + 1)
  {
    u32 max_v = 0, max_c = 0;
    for (u32 s = 0; s <= max_sym; ++s)
      if (count[s] > max_c)
      {
        max_v = s;
        max_c = count[s];
      }
    norm[max_v] = (i16)(norm[max_v] + (i16)to_distribute);
    return true;
  }
  if (total == 0)
  {
    for (u32 s = 0; to_distribute > 0; s = (s + 1) % (max_sym + 1))
      if (norm[s] > 0)
      {
        to_distribute--;
        norm[s]++;
      }
    return true;
  }
  const u64 vstep_log = 62 - log;
  const u64 mid = (1ull << (vstep_log - 1)) - 1;
  const u64 rstep = (((1ull << vstep_log) * to_distribute) + mid) / total;
  u64 tmp = mid;
  for (u32 s = 0; s <= max_sym; ++s)
    if (norm[s] == kUnset)
    {
      const u64 end = tmp + (count[s] * rstep);
      const u32 w = (u32)(end >> vstep_log) - (u32)(tmp >> vstep_log);
      if (w < 1)
        return false;
      norm[s] = (i16)w;
      tmp = end;
    }
  return true;
}

// Normalised counts summing to 1 << log (-1 marks a low-probability symbol).
bool fse_normalize(i16* norm, u32 log, const u32* count, size_t total, u32 max_sym)
{
  static const u32 rtb[] = { 0, 473195, 504333, 520860, 550000, 700000, 750000, 830000 };
  const u64 scale = 62 - log;
  const u64 step = (1ull << 62) / total;
  const u64 vstep = 1ull << (scale - 20);
  int still = 1 << log;
  u32 largest = 0;
  i16 largest_p = 0;
  const u32 low_threshold = (u32)(total >> log);
  for (u32 s = 0; s <= max_sym; ++s)
  {
    if (count[s] == total)
      return true;  // a single symbol (the callers do not reach this)
    if (count[s] == 0)
    {
      norm[s] = 0;
      continue;
    }
    if (count[s] <= low_threshold)
    {
      norm[s] = -1;
      still--;
    }
    else
    {
      i16 p = (i16)((count[s] * step) >> scale);
      if (p < 8)
      {
        const u64 rest = vstep * rtb[p];
        p = (i16)(p + (((count[s] * step) - ((u64)p << scale)) > rest));
      }
      if (p > largest_p)
      {
        largest_p = p;
        largest = s;
      }
      norm[s] = p;
      still -= p;
    }
  }
  if (-still >= (norm[largest] >> 1))
    return fse_normalize_fallback(norm, log, count, total, max_sym);
  norm[largest] = (i16)(norm[largest] + still);
  return true;
}

// The normalised counts' header (the format's FSE table description).
void fse_write_header(std::vector<u8>* out, const i16* norm, u32 max_sym, u32 log)
{
  const int table = 1 << log;
  u32 bits = 0;
  int nbits = 0;
  auto flush16 = [&]() {
    out->push_back((u8)bits);
    out->push_back((u8)(bits >> 8));
    bits >>= 16;
  };
  bits += (log - kFSEMinLog) << nbits;
  nbits += 4;
  int remaining = table + 1;
  int threshold = table;
  int nb = (int)log + 1;
  u32 sym = 0;
  const u32 alphabet = max_sym + 1;
  bool prev0 = false;
  while (sym < alphabet && remaining > 1)
  {
    if (prev0)
    {
      u32 start = sym;
      while (sym < alphabet && !norm[sym])
        sym++;
      if (sym == alphabet)
        break;
      while (sym >= start + 24)
      {
        start += 24;
        bits += 0xFFFFu << nbits;
        flush16();
      }
      while (sym >= start + 3)
      {
        start += 3;
        bits += 3u << nbits;
        nbits += 2;
      }
      bits += (sym - start) << nbits;
      nbits += 2;
      if (nbits > 16)
      {
        flush16();
        nbits -= 16;
      }
    }
    {
      int c = norm[sym++];
      const int max = (2 * threshold - 1) - remaining;
      remaining -= c < 0 ? -c : c;
      c++;
      if (c >= threshold)
        c += max;
      bits += (u32)c << nbits;
      nbits += nb;
      nbits -= (c < max);
      prev0 = (c == 1);
      while (remaining < threshold)
      {
        nb--;
        threshold >>= 1;
      }
    }
    if (nbits > 16)
    {
      flush16();
      nbits -= 16;
    }
  }
  out->push_back((u8)bits);
  out->push_back((u8)(bits >> 8));
  // only (nbits + 7) / 8 of the last two bytes belong to the header
  out->resize(out->size() - 2 + (size_t)((nbits + 7) / 8));
}

struct fse_table
{
  u32 log = 0;
  std::vector<u16> next;     // state transitions, sorted by symbol
  std::vector<int> find;     // per symbol: offset of its first transition
  std::vector<u32> nbdelta;  // per symbol: bit-count threshold term
};

void fse_build(fse_table* t, const i16* norm, u32 max_sym, u32 log)
{
  const u32 size = 1u << log, mask = size - 1;
  const u32 step = (size >> 1) + (size >> 3) + 3;
  std::vector<u8> sym_at(size);
  std::vector<u32> cumul(max_sym + 2);
  u32 high = size - 1;
  cumul[0] = 0;
  for (u32 u = 1; u <= max_sym + 1; ++u)
  {
    if (norm[u - 1] == -1)
    {
      cumul[u] = cumul[u - 1] + 1;
      sym_at[high--] = (u8)(u - 1);
    }
    else
      cumul[u] = cumul[u - 1] + (u32)norm[u - 1];
  }
  cumul[max_sym + 1] = size + 1;
  u32 pos = 0;
  for (u32 s = 0; s <= max_sym; ++s)
    for (int k = 0; k < norm[s]; ++k)
    {
      sym_at[pos] = (u8)s;
      pos = (pos + step) & mask;
      while (pos > high)
        pos = (pos + step) & mask;
    }
  t->log = log;
  t->next.assign(size, 0);
  for (u32 u = 0; u < size; ++u)
    t->next[cumul[sym_at[u]]++] = (u16)(size + u);
  t->find.assign(max_sym + 1, 0);
  t->nbdelta.assign(max_sym + 1, 0);
  u32 total = 0;
  for (u32 s = 0; s <= max_sym; ++s)
  {
    switch (norm[s])
    {
      case 0:
        t->nbdelta[s] = ((log + 1) << 16) - (1u << log);
        break;
      case -1:
      case 1:
        t->nbdelta[s] = (log << 16) - (1u << log);
        t->find[s] = (int)total - 1;
        total++;
        break;
      default:
      {
        const u32 max_out = log - highbit32((u32)norm[s] - 1);
        const u32 min_plus = (u32)norm[s] << max_out;
        t->nbdelta[s] = (max_out << 16) - min_plus;
        t->find[s] = (int)total - norm[s];
        total += (u32)norm[s];
      }
    }
  }
}

// a table of one symbol: every code takes no bit
void fse_build_rle(fse_table* t, u32 sym)
{
  t->log = 0;
  t->next.assign(2, 0);
  t->find.assign(sym + 1, 0);
  t->nbdelta.assign(sym + 1, 0);
}

struct fse_state
{
  long long value;
  const u16* next;
  const int* find;
  const u32* nbdelta;
  u32 log;
};

fse_state fse_start(const fse_table& t, u32 sym)
{
  fse_state st{ (long long)1 << t.log, t.next.data(), t.find.data(), t.nbdelta.data(), t.log };
  const u32 nb = (t.nbdelta[sym] + (1u << 15)) >> 16;
  const u32 v = (nb << 16) - t.nbdelta[sym];
  st.value = t.next[(size_t)((long long)(v >> nb) + t.find[sym])];
  return st;
}

inline void fse_encode(bit_writer& bw, fse_state& st, u32 sym)
{
  const u32 nb = (u32)((st.value + (long long)st.nbdelta[sym]) >> 16);
  bw.add((u64)st.value, nb);
  st.value = st.next[(size_t)((st.value >> nb) + st.find[sym])];
}

// as fse_encode, the bits left in the accumulator (room for them is the caller's)
inline void fse_put(bit_writer& bw, fse_state& st, u32 sym)
{
  const u32 nb = (u32)((st.value + (long long)st.nbdelta[sym]) >> 16);
  bw.put((u64)st.value, nb);
  st.value = st.next[(size_t)((st.value >> nb) + st.find[sym])];
}

void fse_finish(bit_writer& bw, const fse_state& st) { bw.add((u64)st.value, st.log); }

// FSE compression of a small byte array with two interleaved states (Huffman weights).
// Returns the stream size, or 0 when the input is too short.
size_t fse_compress_bytes(std::vector<u8>* out, const u8* src, size_t n, const fse_table& t)
{
  if (n <= 2)
    return 0;
  bit_writer bw(out);
  const u8* ip = src + n;
  fse_state s1, s2;
  if (n & 1)
  {
    s1 = fse_start(t, *--ip);
    s2 = fse_start(t, *--ip);
    fse_encode(bw, s1, *--ip);
  }
  else
  {
    s2 = fse_start(t, *--ip);
    s1 = fse_start(t, *--ip);
  }
  n -= 2;
  if (n & 2)
  {
    fse_encode(bw, s2, *--ip);
    fse_encode(bw, s1, *--ip);
  }
  while (ip > src)
  {
    fse_encode(bw, s2, *--ip);
    fse_encode(bw, s1, *--ip);
    fse_encode(bw, s2, *--ip);
    fse_encode(bw, s1, *--ip);
  }
  fse_finish(bw, s2);
  fse_finish(bw, s1);
  return bw.close();
}

// ---------------------------------------------------------------------------------------------
// Huffman literals

constexpr u32 kHufMaxLog = 12, kHufDefaultLog = 11;

struct huf_code
{
  u16 val = 0;
  u8 nbits = 0;
};

struct huf_table
{
  huf_code e[256];
};

struct huf_node
{
  u32 count = 0;
  u16 parent = 0;
  u8 byte = 0;
  u8 nbits = 0;
};

// symbols by decreasing count (stable within a count), into node[0..max_sym]
void huf_sort(huf_node* node, const u32* count, u32 max_sym)
{
  struct rank_pos
  {
    u32 base = 0, current = 0;
  } rank[32];
  for (u32 n = 0; n <= max_sym; ++n)
    rank[highbit32(count[n] + 1)].base++;
  for (u32 n = 30; n > 0; --n)
    rank[n - 1].base += rank[n].base;
  for (u32 n = 0; n < 32; ++n)
    rank[n].current = rank[n].base;
  for (u32 n = 0; n <= max_sym; ++n)
  {
    const u32 c = count[n];
    const u32 r = highbit32(c + 1) + 1;
    u32 pos = rank[r].current++;
    while (pos > rank[r].base && c > node[pos - 1].count)
    {
      node[pos] = node[pos - 1];
      pos--;
    }
    node[pos].count = c;
    node[pos].byte = (u8)n;
  }
}

// Limits code lengths to max_bits, repaying the cost on the shortest codes that can absorb it.
u32 huf_limit_height(huf_node* node, u32 last, u32 max_bits)
{
  const u32 largest = node[last].nbits;
  if (largest <= max_bits)
    return largest;
  int cost = 0;
  const u32 base_cost = 1u << (largest - max_bits);
  u32 n = last;
  while (node[n].nbits > max_bits)
  {
    cost += (int)(base_cost - (1u << (largest - node[n].nbits)));
    node[n].nbits = (u8)max_bits;
    n--;
  }
  while (node[n].nbits == max_bits)
    n--;
  cost >>= (largest - max_bits);
  const u32 none = 0xF0F0F0F0u;
  u32 rank_last[kHufMaxLog + 2];
  for (u32& r : rank_last)
    r = none;
  {
    u32 cur = max_bits;
    for (int pos = (int)n; pos >= 0; --pos)
    {
      if (node[pos].nbits >= cur)
        continue;
      cur = node[pos].nbits;
      rank_last[max_bits - cur] = (u32)pos;
    }
  }
  while (cost > 0)
  {
    u32 dec = highbit32((u32)cost) + 1;
    for (; dec > 1; --dec)
    {
      const u32 hi = rank_last[dec], lo = rank_last[dec - 1];
      if (hi == none)
        continue;
      if (lo == none)
        break;
      if (node[hi].count <= 2 * node[lo].count)
        break;
    }
    while (dec <= kHufMaxLog && rank_last[dec] == none)
      dec++;
    cost -= 1 << (dec - 1);
    if (rank_last[dec - 1] == none)
      rank_last[dec - 1] = rank_last[dec];
    node[rank_last[dec]].nbits++;
    if (rank_last[dec] == 0)
      rank_last[dec] = none;
    else
    {
      rank_last[dec]--;
      if (node[rank_last[dec]].nbits != max_bits - dec)
        rank_last[dec] = none;
    }
  }
  while (cost < 0)
  {
    if (rank_last[1] == none)
    {
      while (node[n].nbits == max_bits)
        n--;
      node[n + 1].nbits--;
      rank_last[1] = n + 1;
      cost++;
      continue;
    }
    node[rank_last[1] + 1].nbits--;
    rank_last[1]++;
    cost++;
  }
  return max_bits;
}

// Huffman code of the counts (symbols 0..max_sym) with lengths up to max_bits; returns the
// longest length used.
u32 huf_build(huf_table* t, const u32* count, u32 max_sym, u32 max_bits)
{
  std::vector<huf_node> nodes(2 * 256 + 2);
  huf_node* const node0 = nodes.data();
  huf_node* const node = node0 + 1;
  const u32 start = 256;
  u16 next = (u16)start;
  huf_sort(node, count, max_sym);
  u32 nonnull = max_sym;
  while (node[nonnull].count == 0)
    nonnull--;
  int lows = (int)nonnull;
  const u32 root = next + (u32)lows - 1;
  int lown = next;
  node[next].count = node[lows].count + node[lows - 1].count;
  node[lows].parent = node[lows - 1].parent = next;
  next++;
  lows -= 2;
  for (u32 n = next; n <= root; ++n)
    node[n].count = 1u << 30;
  node0[0].count = 1u << 31;
  while (next <= root)
  {
    const int n1 = (node[lows].count < node[lown].count) ? lows-- : lown++;
    const int n2 = (node[lows].count < node[lown].count) ? lows-- : lown++;
    node[next].count = node[n1].count + node[n2].count;
    node[n1].parent = node[n2].parent = next;
    next++;
  }
  node[root].nbits = 0;
  for (u32 n = root - 1; n >= start; --n)
    node[n].nbits = (u8)(node[node[n].parent].nbits + 1);
  for (u32 n = 0; n <= nonnull; ++n)
    node[n].nbits = (u8)(node[node[n].parent].nbits + 1);
  max_bits = huf_limit_height(node, nonnull, max_bits);
  u16 per_rank[kHufMaxLog + 1] = {};
  u16 val_rank[kHufMaxLog + 1] = {};
  for (u32 n = 0; n <= nonnull; ++n)
    per_rank[node[n].nbits]++;
  {
    u16 min = 0;
    for (u32 n = max_bits; n > 0; --n)
    {
      val_rank[n] = min;
      min = (u16)(min + per_rank[n]);
      min >>= 1;
    }
  }
  for (u32 n = 0; n <= max_sym; ++n)
    t->e[node[n].byte].nbits = node[n].nbits;
  for (u32 n = 0; n <= max_sym; ++n)
    t->e[n].val = val_rank[t->e[n].nbits]++;
  for (u32 n = max_sym + 1; n < 256; ++n)
    t->e[n] = huf_code();
  return max_bits;
}

// The table's header: weights FSE-compressed when that is shorter, else 4 bits each.
// Returns false when neither form applies.
bool huf_write_table(std::vector<u8>* out, const huf_table& t, u32 max_sym, u32 log)
{
  u8 weight[256];
  for (u32 n = 0; n < max_sym; ++n)
    weight[n] = t.e[n].nbits ? (u8)(log + 1 - t.e[n].nbits) : 0;
  // FSE-compressed weights
  {
    std::vector<u8> z;
    size_t hs = 0;
    const size_t wn = max_sym;
    if (wn > 1)
    {
      u32 count[kHufMaxLog + 1];
      u32 wmax = kHufMaxLog;
      const u32 top = histogram(weight, wn, count, &wmax);
      if (top == wn)
        hs = 1;
      else if (top != 1)
      {
        const u32 wlog = fse_optimal_log(6, wn, wmax, 2);
        i16 norm[kHufMaxLog + 1];
        if (fse_normalize(norm, wlog, count, wn, wmax))
        {
          fse_write_header(&z, norm, wmax, wlog);
          fse_table ft;
          fse_build(&ft, norm, wmax, wlog);
          const size_t cs = fse_compress_bytes(&z, weight, wn, ft);
          hs = cs ? z.size() : 0;
        }
      }
    }
    if (hs > 1 && hs < max_sym / 2)
    {
      out->push_back((u8)hs);
      out->insert(out->end(), z.begin(), z.end());
      return true;
    }
  }
  if (max_sym > 128)
    return false;
  out->push_back((u8)(128 + (max_sym - 1)));
  weight[max_sym] = 0;
  for (u32 n = 0; n < max_sym; n += 2)
    out->push_back((u8)((weight[n] << 4) + weight[n + 1]));
  return true;
}

// One Huffman stream of src (symbols coded last to first).
size_t huf_stream(std::vector<u8>* out, const u8* src, size_t n, const huf_table& t)
{
  bit_writer bw(out);
  for (size_t i = n; i-- > 0;)
    bw.add(t.e[src[i]].val, t.e[src[i]].nbits);
  return bw.close();
}

// Huffman-coded literals in one or four streams (the four behind a 6-byte jump table).
// Returns the size, 0 when the input cannot gain.
size_t huf_streams(std::vector<u8>* out, const u8* src, size_t n, bool four, const huf_table& t)
{
  const size_t base = out->size();
  if (!four)
    huf_stream(out, src, n, t);
  else
  {
    if (n < 12)
      return 0;
    const size_t seg = (n + 3) / 4;
    out->resize(base + 6);
    size_t sizes[3];
    for (int k = 0; k < 3; ++k)
      sizes[k] = huf_stream(out, src + (size_t)k * seg, seg, t);
    huf_stream(out, src + 3 * seg, n - 3 * seg, t);
    for (int k = 0; k < 3; ++k)
    {
      (*out)[base + 2 * (size_t)k] = (u8)sizes[k];
      (*out)[base + 2 * (size_t)k + 1] = (u8)(sizes[k] >> 8);
    }
  }
  return out->size() - base;
}

enum class huf_repeat
{
  none,
  check
};

struct huf_state
{
  huf_table t;
  huf_repeat repeat = huf_repeat::none;
};

size_t huf_cost(const huf_table& t, const u32* count, u32 max_sym)
{
  size_t bits = 0;
  for (u32 s = 0; s <= max_sym; ++s)
    bits += (size_t)t.e[s].nbits * count[s];
  return bits >> 3;
}

bool huf_covers(const huf_table& t, const u32* count, u32 max_sym)
{
  for (u32 s = 0; s <= max_sym; ++s)
    if (count[s] != 0 && t.e[s].nbits == 0)
      return false;
  return true;
}

// Huffman literal coding with table reuse. Appends the (table +) streams to out; returns the
// size, 0 = store raw, 1 = one repeated byte (the first byte of out then holds it). *repeat
// becomes none when a new table was written (saved into *table), stays otherwise.
size_t huf_compress(std::vector<u8>* out, const u8* src, size_t n, bool four, huf_table* table, huf_repeat* repeat,
                    bool prefer_repeat)
{
  const size_t base = out->size();
  u32 count[256];
  u32 max_sym = 255;
  const u32 largest = histogram(src, n, count, &max_sym);
  if (largest == n)
  {
    out->push_back(src[0]);
    return 1;
  }
  if (largest <= (n >> 7) + 4)
    return 0;
  if (*repeat == huf_repeat::check && !huf_covers(*table, count, max_sym))
    *repeat = huf_repeat::none;
  auto with_table = [&](const huf_table& t) -> size_t {
    out->resize(base);
    const size_t cs = huf_streams(out, src, n, four, t);
    if (cs == 0 || cs >= n - 1)
    {
      out->resize(base);
      return 0;
    }
    return cs;
  };
  if (prefer_repeat && *repeat != huf_repeat::none)
    return with_table(*table);
  u32 log = fse_optimal_log(kHufDefaultLog, n, max_sym, 1);
  huf_table fresh;
  log = huf_build(&fresh, count, max_sym, log);
  std::vector<u8> hdr;
  if (!huf_write_table(&hdr, fresh, max_sym, log))
    return 0;
  const size_t hs = hdr.size();
  if (*repeat != huf_repeat::none)
  {
    const size_t old_size = huf_cost(*table, count, max_sym);
    const size_t new_size = huf_cost(fresh, count, max_sym);
    if (old_size <= hs + new_size || hs + 12 >= n)
      return with_table(*table);
  }
  if (hs + 12 >= n)
    return 0;
  *repeat = huf_repeat::none;
  *table = fresh;
  out->insert(out->end(), hdr.begin(), hdr.end());
  const size_t cs = huf_streams(out, src, n, four, fresh);
  if (cs == 0 || hs + cs >= n - 1)
  {
    out->resize(base);
    return 0;
  }
  return hs + cs;
}

// ---------------------------------------------------------------------------------------------
// block contents

struct sequence
{
  u32 ll;   // literal length
  u32 mlb;  // match length - 3
  u32 off;  // offset value: 1 for the repeat offset, else offset + 3
};

struct entropy_state
{
  huf_state huf;
  u32 rep[3] = { 1, 4, 8 };
};

constexpr size_t kBlockMax = 128 * 1024;

size_t min_gain(size_t n) { return (n >> 6) + 2; }

void write_le(std::vector<u8>* out, u64 v, int bytes)
{
  for (int k = 0; k < bytes; ++k)
    out->push_back((u8)(v >> (8 * k)));
}

void literals_raw(std::vector<u8>* out, const u8* src, size_t n)
{
  const int fl = 1 + (n > 31) + (n > 4095);
  if (fl == 1)
    out->push_back((u8)(n << 3));
  else if (fl == 2)
    write_le(out, (u32)((1u << 2) + (n << 4)), 2);
  else
    write_le(out, (u32)((3u << 2) + (n << 4)), 3);
  out->insert(out->end(), src, src + n);
}

void literals_rle(std::vector<u8>* out, u8 b, size_t n)
{
  const int fl = 1 + (n > 31) + (n > 4095);
  if (fl == 1)
    out->push_back((u8)(1 + (n << 3)));
  else if (fl == 2)
    write_le(out, (u32)(1 + (1u << 2) + (n << 4)), 2);
  else
    write_le(out, (u32)(1 + (3u << 2) + (n << 4)), 3);
  out->push_back(b);
}

// The literals section; next gets the Huffman state the block leaves behind.
void literals_section(std::vector<u8>* out, const u8* src, size_t n, const huf_state& prev, huf_state* next)
{
  *next = prev;
  if (n <= 63)
  {
    literals_raw(out, src, n);
    return;
  }
  const size_t lh = 3 + (n >= 1024) + (n >= 16 * 1024);
  const bool single = n < 256;
  const size_t at = out->size();
  out->resize(at + lh);
  huf_repeat rep = prev.repeat;
  huf_table table = prev.t;
  const size_t cs = huf_compress(out, src, n, !single, &table, &rep, n <= 1024);
  const bool reused = rep != huf_repeat::none;
  if (cs == 0 || cs >= n - min_gain(n))
  {
    out->resize(at);
    *next = prev;
    literals_raw(out, src, n);
    return;
  }
  if (cs == 1)
  {
    const u8 b = (*out)[at + lh];
    out->resize(at);
    *next = prev;
    literals_rle(out, b, n);
    return;
  }
  const u32 type = reused ? 3u : 2u;  // set_repeat : set_compressed
  next->t = table;
  if (!reused)
    next->repeat = huf_repeat::check;
  u8* h = out->data() + at;
  if (lh == 3)
  {
    const u32 v = type + ((u32)(!single) << 2) + ((u32)n << 4) + ((u32)cs << 14);
    h[0] = (u8)v;
    h[1] = (u8)(v >> 8);
    h[2] = (u8)(v >> 16);
  }
  else if (lh == 4)
  {
    const u32 v = type + (2u << 2) + ((u32)n << 4) + ((u32)cs << 18);
    memcpy(h, &v, 4);
  }
  else
  {
    const u32 v = type + (3u << 2) + ((u32)n << 4) + ((u32)cs << 22);
    memcpy(h, &v, 4);
    h[4] = (u8)(cs >> 10);
  }
}

enum set_type : u32
{
  set_basic = 0,
  set_rle = 1,
  set_compressed = 2,
};

// Encoding type of one symbol stream under the fast strategy's rules.
u32 select_type(const u32* count, u32 max, u32 most, size_t nseq, u32 default_log, bool default_ok)
{
  (void)count;
  (void)max;
  if (most == nseq)
    return (default_ok && nseq <= 2) ? set_basic : set_rle;
  if (default_ok)
  {
    const size_t mult = 10 - 1;  // 10 - strategy (fast = 1)
    const size_t dyn_min = (((size_t)1 << default_log) * mult) >> 3;
    if (nseq < dyn_min || most < (nseq >> (default_log - 1)))
      return set_basic;
  }
  return set_compressed;
}

// Builds the stream's table (writing its header when compressed); returns the header size.
size_t build_table(std::vector<u8>* out, fse_table* t, u32 type, u32* count, u32 max, const u8* codes, size_t nseq,
                   const i16* default_norm, u32 default_log, u32 default_max, u32 max_log)
{
  switch (type)
  {
    case set_rle:
      fse_build_rle(t, max);
      out->push_back(codes[0]);
      return 1;
    case set_basic:
      fse_build(t, default_norm, default_max, default_log);
      return 0;
    default:
    {
      i16 norm[kMaxML + 1];
      size_t n1 = nseq;
      const u32 log = fse_optimal_log(max_log, nseq, max, 2);
      if (count[codes[nseq - 1]] > 1)
      {
        count[codes[nseq - 1]]--;
        n1--;
      }
      fse_normalize(norm, log, count, n1, max);
      const size_t before = out->size();
      fse_write_header(out, norm, max, log);
      fse_build(t, norm, max, log);
      return out->size() - before;
    }
  }
}

// The compressed block body (literals + sequences); 0 when it must be stored raw.
size_t block_body(std::vector<u8>* out, const std::vector<sequence>& seqs, const std::vector<u8>& lits,
                  const entropy_state& prev, entropy_state* next, size_t src_size)
{
  const size_t base = out->size();
  literals_section(out, lits.data(), lits.size(), prev.huf, &next->huf);
  const size_t nseq = seqs.size();
  if (nseq < 128)
    out->push_back((u8)nseq);
  else if (nseq < 0x7F00)
  {
    out->push_back((u8)((nseq >> 8) + 0x80));
    out->push_back((u8)nseq);
  }
  else
  {
    out->push_back(0xFF);
    write_le(out, nseq - 0x7F00, 2);
  }
  if (nseq > 0)
  {
    std::vector<u8> llc(nseq), ofc(nseq), mlc(nseq);
    for (size_t i = 0; i < nseq; ++i)
    {
      llc[i] = (u8)ll_code(seqs[i].ll);
      ofc[i] = (u8)highbit32(seqs[i].off);
      mlc[i] = (u8)ml_code(seqs[i].mlb);
    }
    const size_t head = out->size();
    out->push_back(0);
    size_t last_ncount = 0;  // position of the last compressed table's header + 1, 0 = none
    fse_table tll, tof, tml;
    u32 types[3];
    {
      u32 count[kMaxML + 1];
      u32 max = kMaxLL;
      const u32 most = histogram(llc.data(), nseq, count, &max);
      types[0] = select_type(count, max, most, nseq, kLLDefaultLog, true);
      const size_t at = out->size();
      build_table(out, &tll, types[0], count, max, llc.data(), nseq, kLLDefaultNorm, kLLDefaultLog, kMaxLL, kLLFSELog);
      if (types[0] == set_compressed)
        last_ncount = at + 1;
    }
    {
      u32 count[kMaxML + 1];
      u32 max = kMaxOff;
      const u32 most = histogram(ofc.data(), nseq, count, &max);
      const bool dflt = max <= (u32)kDefaultMaxOff;
      types[1] = select_type(count, max, most, nseq, kOFDefaultLog, dflt);
      const size_t at = out->size();
      build_table(out, &tof, types[1], count, max, ofc.data(), nseq, kOFDefaultNorm, kOFDefaultLog, kDefaultMaxOff,
                  kOffFSELog);
      if (types[1] == set_compressed)
        last_ncount = at + 1;
    }
    {
      u32 count[kMaxML + 1];
      u32 max = kMaxML;
      const u32 most = histogram(mlc.data(), nseq, count, &max);
      types[2] = select_type(count, max, most, nseq, kMLDefaultLog, true);
      const size_t at = out->size();
      build_table(out, &tml, types[2], count, max, mlc.data(), nseq, kMLDefaultNorm, kMLDefaultLog, kMaxML, kMLFSELog);
      if (types[2] == set_compressed)
        last_ncount = at + 1;
    }
    (*out)[head] = (u8)((types[0] << 6) + (types[1] << 4) + (types[2] << 2));
    // the sequences, last to first, three interleaved states
    {
      bit_writer bw(out);
      const size_t l = nseq - 1;
      fse_state sml = fse_start(tml, mlc[l]);
      fse_state sof = fse_start(tof, ofc[l]);
      fse_state sll = fse_start(tll, llc[l]);
      // (bit budget between flushes, at most 7 bits held after one: the three states take
      // at most 8 + 9 + 9 bits, the literal and match length bits at most 16 each, the
      // offset bits at most 31)
      bw.put(seqs[l].ll, kLLBits[llc[l]]);
      bw.put(seqs[l].mlb, kMLBits[mlc[l]]);
      bw.flush();
      bw.put(seqs[l].off, ofc[l]);
      bw.flush();
      for (size_t n = nseq - 1; n-- > 0;)
      {
        // (at most 7 + 26 bits held after the states; the length and offset bits flushed
        // ahead only when they would not fit, as they mostly do)
        fse_put(bw, sof, ofc[n]);
        fse_put(bw, sml, mlc[n]);
        fse_put(bw, sll, llc[n]);
        const unsigned llb = kLLBits[llc[n]], mlb = kMLBits[mlc[n]], ofb = ofc[n];
        if (bw.n + llb + mlb >= 64)
          bw.flush();
        bw.put(seqs[n].ll, llb);
        bw.put(seqs[n].mlb, mlb);
        if (bw.n + ofb >= 64)
          bw.flush();
        bw.put(seqs[n].off, ofb);
        bw.flush();
      }
      fse_finish(bw, sml);
      fse_finish(bw, sof);
      fse_finish(bw, sll);
      bw.close();
    }
    // a compressed table header directly followed by a bit stream of one byte is stored raw
    // (old decoders misread it)
    if (last_ncount && out->size() - (last_ncount - 1) < 4)
    {
      out->resize(base);
      return 0;
    }
  }
  const size_t cs = out->size() - base;
  if (cs >= src_size - min_gain(src_size))
  {
    out->resize(base);
    return 0;
  }
  return cs;
}

// ---------------------------------------------------------------------------------------------
// the fast match finder

struct matcher
{
  std::vector<u32> hash;
  u32 hlog, mls, wlog;
  const u8* data;  // the frame's input; byte p has index p + 1
  size_t size = 0;  // its bytes
  template <u32 MLS>
  size_t hpos(size_t p) const
  {
    const u8* q = data + p;
    switch (MLS)
    {
      case 5:
        return (size_t)(((rd64(q) << (64 - 40)) * 889523592379ull) >> (64 - hlog));
      case 6:
        return (size_t)(((rd64(q) << (64 - 48)) * 227718039650203ull) >> (64 - hlog));
      case 7:
        return (size_t)(((rd64(q) << (64 - 56)) * 58295818150454627ull) >> (64 - hlog));
      case 8:
        return (size_t)((rd64(q) * 0xCF1BBCDCB7A56463ull) >> (64 - hlog));
      default:
        return (size_t)((rd32(q) * 2654435761u) >> (32 - hlog));
    }
  }
  // length of the common run of positions a and b (b < a), up to limit; 8 bytes at a time
  size_t count(size_t a, size_t b, size_t limit) const
  {
    size_t n = 0;
    while (a + n + 8 <= limit)
    {
      const u64 x = rd64(data + a + n) ^ rd64(data + b + n);
      if (x)
        return n + ((size_t)__builtin_ctzll(x) >> 3);
      n += 8;
    }
    while (a + n < limit && data[a + n] == data[b + n])
      n++;
    return n;
  }

  // Sequences of block [bs, be); the trailing literals are lits' tail. rep: the two repeat
  // offsets in and out.
  void block(size_t bs, size_t be, u32 rep[2], std::vector<sequence>* seqs, std::vector<u8>* lits)
  {
    // room for the worst case (a sequence per 4 bytes, every byte a literal), cut after
    seqs->resize((be - bs) / 3 + 2);
    lits->resize(be - bs + 16);  // (+16: literal runs are copied 16 bytes at a time)
    size_t ns = 0, nl = 0;
    switch (mls)
    {
      case 5:
        run<5>(bs, be, rep, seqs->data(), &ns, lits->data(), &nl);
        break;
      case 6:
        run<6>(bs, be, rep, seqs->data(), &ns, lits->data(), &nl);
        break;
      case 7:
        run<7>(bs, be, rep, seqs->data(), &ns, lits->data(), &nl);
        break;
      case 8:
        run<8>(bs, be, rep, seqs->data(), &ns, lits->data(), &nl);
        break;
      default:
        run<4>(bs, be, rep, seqs->data(), &ns, lits->data(), &nl);
    }
    seqs->resize(ns);
    lits->resize(nl);
  }

  template <u32 MLS>
  void run(size_t bs, size_t be, u32 rep[2], sequence* seq_out, size_t* nseq, u8* lit_out, size_t* nlit)
  {
    const long long end_index = (long long)be + 1;
    const long long max_dist = 1ll << wlog;
    const long long prefix_index = (end_index - 1 > max_dist) ? end_index - max_dist : 1;
    const long long prefix = prefix_index - 1;  // position
    long long ip0 = (long long)bs;
    ip0 += (ip0 == prefix);
    long long ip1 = ip0 + 1;
    long long anchor = (long long)bs;
    const long long iend = (long long)be;
    const long long ilimit = iend - 8;
    u32 off1 = rep[0], off2 = rep[1], saved = 0;
    {
      const u32 max_rep = (u32)(ip0 - prefix);
      if (off2 > max_rep)
      {
        saved = off2;
        off2 = 0;
      }
      if (off1 > max_rep)
      {
        saved = off1;
        off1 = 0;
      }
    }
    size_t ns = 0, nl = 0;
    auto store = [&](long long ll, long long from, u32 off_value, long long mlb) {
      // short runs as one 16-byte copy where the input has those bytes (the bytes past the run
      // land in the literal buffer's slack and are overwritten or cut)
      if (ll <= 16 && (size_t)from + 16 <= size)
        memcpy(lit_out + nl, data + from, 16);
      else
        memcpy(lit_out + nl, data + from, (size_t)ll);
      nl += (size_t)ll;
      seq_out[ns++] = sequence{ (u32)ll, (u32)mlb, off_value };
    };
    while (ip1 < ilimit)
    {
      const long long ip2 = ip0 + 2;
      const size_t h0 = hpos<MLS>((size_t)ip0), h1 = hpos<MLS>((size_t)ip1);
      const u32 val0 = rd32(data + ip0), val1 = rd32(data + ip1);
      const u32 cur0 = (u32)(ip0 + 1), cur1 = (u32)(ip1 + 1);
      const u32 mi0 = hash[h0], mi1 = hash[h1];
      const long long rep_at = ip2 - (long long)off1;
      long long m0 = (long long)mi0 - 1;
      const long long m1 = (long long)mi1 - 1;
      hash[h0] = cur0;
      hash[h1] = cur1;
      long long mlen;
      u32 offcode;
      bool matched = false, rep_match = false;
      if (off1 > 0 && rd32(data + rep_at) == rd32(data + ip2))
      {
        mlen = data[ip2 - 1] == data[rep_at - 1] ? 1 : 0;
        ip0 = ip2 - mlen;
        m0 = rep_at - mlen;
        offcode = 0;
        rep_match = true;
      }
      else if (mi0 > (u32)prefix_index && rd32(data + m0) == val0)
        matched = true;
      else if (mi1 > (u32)prefix_index && rd32(data + m1) == val1)
      {
        ip0 = ip1;
        m0 = m1;
        matched = true;
      }
      else
      {
        const long long step = ((ip0 - anchor) >> 7) + 2;
        ip0 += step;
        ip1 += step;
        continue;
      }
      if (matched)
      {
        off2 = off1;
        off1 = (u32)(ip0 - m0);
        offcode = off1 + 2;
        mlen = 0;
        while (ip0 > anchor && m0 > prefix && data[ip0 - 1] == data[m0 - 1])
        {
          ip0--;
          m0--;
          mlen++;
        }
      }
      (void)rep_match;
      mlen += (long long)count((size_t)(ip0 + mlen + 4), (size_t)(m0 + mlen + 4), (size_t)iend) + 4;
      store(ip0 - anchor, anchor, offcode + 1, mlen - 3);
      ip0 += mlen;
      anchor = ip0;
      ip1 = ip0 + 1;
      if (ip0 <= ilimit)
      {
        hash[hpos<MLS>((size_t)cur0 + 1)] = cur0 + 2;
        hash[hpos<MLS>((size_t)(ip0 - 2))] = (u32)(ip0 - 1);
        while (ip0 <= ilimit && off2 > 0 && rd32(data + ip0) == rd32(data + ip0 - off2))
        {
          const long long rlen = (long long)count((size_t)(ip0 + 4), (size_t)(ip0 + 4 - off2), (size_t)iend) + 4;
          std::swap(off1, off2);
          hash[hpos<MLS>((size_t)ip0)] = (u32)(ip0 + 1);
          ip0 += rlen;
          ip1 = ip0 + 1;
          store(0, anchor, 1, rlen - 3);
          anchor = ip0;
        }
      }
    }
    rep[0] = off1 ? off1 : saved;
    rep[1] = off2 ? off2 : saved;
    memcpy(lit_out + nl, data + anchor, (size_t)(iend - anchor));
    nl += (size_t)(iend - anchor);
    *nseq = ns;
    *nlit = nl;
  }
};

struct level1_params
{
  u32 wlog, hlog, mls;
};

// Level 1's row of the parameter tables for n input bytes, then the size adjustment.
level1_params params_for(size_t n)
{
  level1_params p;
  if (n <= 16 * 1024)
    p = { 14, 15, 5 };
  else if (n <= 128 * 1024)
    p = { 17, 13, 6 };
  else if (n <= 256 * 1024)
    p = { 18, 14, 6 };
  else
    p = { 19, 14, 7 };
  if (n < (1ull << 30))
  {
    const u32 src_log = n < 64 ? 6 : highbit32((u32)(n - 1)) + 1;
    if (p.wlog > src_log)
      p.wlog = src_log;
  }
  if (p.hlog > p.wlog + 1)
    p.hlog = p.wlog + 1;
  if (p.wlog < 10)
    p.wlog = 10;
  return p;
}

} // namespace

size_t compress_bound(size_t n)
{
  return n + (n >> 8) + (n < (128u << 10) ? (((128u << 10) - n) >> 11) : 0);
}

void compress(const uint8_t* src, size_t n, std::vector<uint8_t>* out)
{
  out->clear();
  out->reserve(compress_bound(n) + 32);
  const level1_params p = params_for(n);
  // frame header: magic, descriptor, window (unless one segment), content size
  write_le(out, 0xFD2FB528u, 4);
  {
    const u64 window = 1ull << p.wlog;
    const bool single = window >= n;
    const u32 fcs = (n >= 256) + (n >= 65536 + 256) + (n >= 0xFFFFFFFFull);
    out->push_back((u8)((single ? 1u << 5 : 0u) + (fcs << 6)));
    if (!single)
      out->push_back((u8)((p.wlog - 10) << 3));
    switch (fcs)
    {
      case 0:
        if (single)
          out->push_back((u8)n);
        break;
      case 1:
        write_le(out, n - 256, 2);
        break;
      case 2:
        write_le(out, n, 4);
        break;
      default:
        write_le(out, n, 8);
    }
  }
  if (n == 0)
  {
    write_le(out, 1u, 3);  // one empty raw block, the last
    return;
  }
  matcher m;
  m.hlog = p.hlog;
  m.mls = p.mls;
  m.wlog = p.wlog;
  m.data = src;
  m.size = n;
  m.hash.assign((size_t)1 << p.hlog, 0);
  const size_t block_size = std::min(kBlockMax, (size_t)1 << p.wlog);
  entropy_state prev;
  bool first = true;
  std::vector<sequence> seqs;
  std::vector<u8> lits;
  for (size_t bs = 0; bs < n; bs += block_size)
  {
    const size_t be = std::min(n, bs + block_size);
    const size_t sz = be - bs;
    const u32 last = be == n ? 1u : 0u;
    const size_t hdr = out->size();
    write_le(out, 0, 3);
    size_t cs = 0;
    entropy_state next = prev;
    bool tried = false;
    if (sz >= 7)
    {
      tried = true;
      seqs.clear();
      lits.clear();
      u32 rep2[2] = { prev.rep[0], prev.rep[1] };
      m.block(bs, be, rep2, &seqs, &lits);
      next.rep[0] = rep2[0];
      next.rep[1] = rep2[1];
      cs = block_body(out, seqs, lits, prev, &next, sz);
    }
    if (tried && !first && cs < 25)
    {
      bool same = true;
      for (size_t i = 1; i < sz && same; ++i)
        same = src[bs + i] == src[bs];
      if (same)
      {
        out->resize(hdr + 3);
        out->push_back(src[bs]);
        cs = 1;
      }
    }
    if (cs > 1)
      prev = next;
    u32 h;
    if (cs == 0)
    {
      out->resize(hdr + 3);
      out->insert(out->end(), src + bs, src + be);
      h = last + (0u << 1) + (u32)(sz << 3);
    }
    else if (cs == 1)
      h = last + (1u << 1) + (u32)(sz << 3);
    else
      h = last + (2u << 1) + (u32)(cs << 3);
    (*out)[hdr] = (u8)h;
    (*out)[hdr + 1] = (u8)(h >> 8);
    (*out)[hdr + 2] = (u8)(h >> 16);
    first = false;
  }
}

} // namespace zstd145
} // namespace idx2g
