/* CPU restatement of the idx2 brick codec (TEST INFRASTRUCTURE ONLY).
 * See idx2_oracle.h. Reference paths are relative to the reference's Source/. */
#include "idx2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int imin(int a, int b) { return a < b ? a : b; }

/* ------------------------------------------------------------------ */
/* geometry                                                            */
/* ------------------------------------------------------------------ */

typedef struct
{
  int from[3], dims[3], strd[3];
} ogrid;

/* transform orders "XYZ++" / "XY++" in the reference's base-4 encoding
   (Core/Wavelet.cpp:407 EncodeTransformOrder: first character in the lowest bits) */
static uint64_t order_code(int is2d)
{
  const char* s = is2d ? "XY++" : "XYZ++";
  int n = (int)strlen(s);
  uint64_t r = 0;
  for (int i = n - 1; i >= 0; --i)
    r = (r << 2) + (uint64_t)(s[i] == '+' ? 3 : s[i] - 'X');
  return r;
}

static void brick_dims(int is2d, int N[3])
{
  N[0] = ORACLE_BRICK_EXT;
  N[1] = ORACLE_BRICK_EXT;
  N[2] = is2d ? 1 : ORACLE_BRICK_EXT;
}

/* ------------------------------------------------------------------ */
/* CDF5/3 lifting (Core/Wavelet.h:178-310)                             */
/* ------------------------------------------------------------------ */

/* One lifting sweep along axis a over every line of grid G, forward or inverse,
   option Normal. The X/Y/Z macro instantiations of the reference differ only in
   which two axes index the lines; lines are independent. */
static void lift(double* F, const int N[3], const ogrid* G, const int M[3], int a, int forward)
{
  const int P = G->from[a], D = G->dims[a], S = G->strd[a];
  if (D == 1)
    return;
  const int b = a == 0 ? 1 : 0;
  const int c = a == 2 ? 1 : 2;
  const long st[3] = { 1, N[0], (long)N[0] * N[1] };
  const int x0 = imin(P + S * D, M[a]);       /* extrapolated position */
  const int x1 = imin(P + S * (D - 1), M[a]); /* last position */
  const int x2 = P + S * (D - 2);             /* second last */
  const int x3 = P + S * (D - 3);             /* third last */
  const int ext = (D % 2) == 0;
  const long s = st[a];
  for (int v = G->from[c]; v < G->from[c] + G->strd[c] * G->dims[c]; v += G->strd[c])
  {
    const int vv = imin(v, M[c]);
    for (int u = G->from[b]; u < G->from[b] + G->strd[b] * G->dims[b]; u += G->strd[b])
    {
      const int uu = imin(u, M[b]);
      double* L = F + (long)uu * st[b] + (long)vv * st[c];
#define AT(t) L[(long)(t) * s]
      if (forward)
      {
        if (ext)
        {
          double A = AT(x2), B = AT(x1);
          AT(x0) = 2 * B - A;
        }
        for (int x = P + S; x < P + S * (D - 2); x += 2 * S)
          AT(x) -= (AT(x - S) + AT(x + S)) / 2;
        if (!ext)
          AT(x2) -= (AT(x1) + AT(x3)) / 2;
        else if (x1 < M[a])
          AT(x1) = 0;
        for (int x = P + S; x < P + S * (D - 2); x += 2 * S)
        {
          double V = AT(x);
          AT(x - S) += V / 4;
          AT(x + S) += V / 4;
        }
        if (!ext)
        {
          double V = AT(x2);
          AT(x3) += V / 4;
          AT(x1) += V / 4;
        }
      }
      else
      {
        for (int x = P + S; x < P + S * (D - 2); x += 2 * S)
        {
          double V = AT(x);
          AT(x - S) -= V / 4;
          AT(x + S) -= V / 4;
        }
        if (!ext)
        {
          double V = AT(x2);
          AT(x3) -= V / 4;
          AT(x1) -= V / 4;
        }
        else
        {
          double A = AT(x0), B = AT(x2);
          AT(x1) = (A + B) / 2;
        }
        for (int x = P + S; x < P + S * (D - 2); x += 2 * S)
          AT(x) += (AT(x - S) + AT(x + S)) / 2;
        if (!ext)
          AT(x2) += (AT(x1) + AT(x3)) / 2;
      }
#undef AT
    }
  }
}

/* Multi-level transform on the first Dims3 samples (Core/Wavelet.cpp:210 ForwardCdf53 and
   :304 InverseCdf53, no normalisation). The grid sequence is shared by both. */
typedef struct
{
  ogrid g[32];
  int axis[32];
  int n;
} lift_stack;

static void build_stack(const int Dims3[3], int nlevels, uint64_t order, lift_stack* st)
{
  int level = 0;
  uint64_t prev = order;
  int D3[3] = { Dims3[0], Dims3[1], Dims3[2] };
  int R3[3] = { Dims3[0], Dims3[1], Dims3[2] };
  int S3[3] = { 1, 1, 1 };
  ogrid G = { { 0, 0, 0 }, { Dims3[0], Dims3[1], Dims3[2] }, { 1, 1, 1 } };
  st->n = 0;
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
      for (int k = 0; k < 3; ++k)
      {
        G.strd[k] = S3[k];
        G.dims[k] = D3[k];
        R3[k] = D3[k];
      }
      ++level;
    }
    else
    {
      st->g[st->n] = G;
      st->axis[st->n++] = d;
      R3[d] = D3[d] + (D3[d] % 2 == 0);
      for (int k = 0; k < 3; ++k)
        G.dims[k] = R3[k];
      D3[d] = (R3[d] + 1) >> 1;
      S3[d] <<= 1;
    }
  }
}

void oracle_brick_extrapolate(double* brick, int is2d, const int valid3[3])
{
  /* Core/Wavelet.cpp:68 ExtrapolateCdf53 */
  int N[3];
  brick_dims(is2d, N);
  int M[3] = { N[0] == 1 ? 1 : N[0] - 1, N[1] == 1 ? 1 : N[1] - 1, N[2] == 1 ? 1 : N[2] - 1 };
  const int nlevels = 5; /* Log2Floor(33) */
  const uint64_t order = order_code(is2d);
  lift_stack fw, iv;
  build_stack(valid3, nlevels, order, &fw);
  for (int i = 0; i < fw.n; ++i)
    lift(brick, N, &fw.g[i], M, fw.axis[i], 1);
  build_stack(N, nlevels, order, &iv);
  for (int i = iv.n - 1; i >= 0; --i)
    lift(brick, N, &iv.g[i], M, iv.axis[i], 0);
}

/* CDF5/3 basis norms (Core/Wavelet.h:19 GetCdf53NormsFast<16>). */
static void cdf53_norms(double scal[16], double wave[16])
{
  double n1 = 3, n2 = 23;
  for (int i = 0; i < 16; ++i)
  {
    scal[i] = sqrt(n1 / (1 << (i + 1)));
    n1 = n1 * 4 - 1;
    wave[i] = sqrt(n2 / (1 << (i + 5)));
    n2 = n2 * 4 - 33;
  }
}

/* Subband s of a one-level transform of the extended brick (Core/Wavelet.cpp:503
   BuildSubbands with "XYZ++"/"XY++", one pass): the bits of s are the high/low
   flags of the transformed axes, first axis most significant. */
static int nsubbands(int is2d) { return is2d ? 4 : 8; }

static void subband_grid(int is2d, int s, ogrid* g, int hi3[3])
{
  int N[3];
  brick_dims(is2d, N);
  int h[3] = { 0, 0, 0 };
  if (is2d)
  {
    h[0] = (s >> 1) & 1;
    h[1] = s & 1;
  }
  else
  {
    h[0] = (s >> 2) & 1;
    h[1] = (s >> 1) & 1;
    h[2] = s & 1;
  }
  for (int k = 0; k < 3; ++k)
  {
    hi3[k] = h[k];
    if (N[k] == 1)
    {
      g->from[k] = 0;
      g->dims[k] = 1;
      g->strd[k] = 1;
    }
    else
    {
      int low = (N[k] + 1) >> 1;
      g->from[k] = h[k];
      g->dims[k] = h[k] ? N[k] - low : low;
      g->strd[k] = 2;
    }
  }
}

static double subband_weight(int is2d, int s, int level)
{
  double scal[16], wave[16];
  cdf53_norms(scal, wave);
  int N[3];
  brick_dims(is2d, N);
  ogrid g;
  int h[3];
  subband_grid(is2d, s, &g, h);
  double w[3];
  for (int k = 0; k < 3; ++k)
    w[k] = N[k] == 1 ? 1 : (h[k] == 0 ? scal[level] : wave[level]);
  return w[0] * w[1] * w[2];
}

static void scale_grid(double* F, const int N[3], const ogrid* g, double W)
{
  for (int z = 0; z < g->dims[2]; ++z)
    for (int y = 0; y < g->dims[1]; ++y)
      for (int x = 0; x < g->dims[0]; ++x)
      {
        long i = ((long)(g->from[2] + z * g->strd[2]) * N[1] + (g->from[1] + y * g->strd[1])) * N[0] +
                 (g->from[0] + x * g->strd[0]);
        F[i] = F[i] * W;
      }
}

void oracle_brick_forward(double* brick, int is2d, const int valid3[3], int level, int coarsest)
{
  oracle_brick_extrapolate(brick, is2d, valid3);
  /* Core/Wavelet.cpp:81 ForwardCdf53(M3 = 33^3, ...): X, Y, Z sweeps on the whole brick. */
  int N[3];
  brick_dims(is2d, N);
  ogrid G = { { 0, 0, 0 }, { N[0], N[1], N[2] }, { 1, 1, 1 } };
  for (int a = 0; a < (is2d ? 2 : 3); ++a)
    lift(brick, N, &G, N, a, 1);
  for (int s = 0; s < nsubbands(is2d); ++s)
  {
    if (s == 0 && !coarsest)
      continue;
    ogrid g;
    int h[3];
    subband_grid(is2d, s, &g, h);
    scale_grid(brick, N, &g, subband_weight(is2d, s, level));
  }
}

void oracle_brick_inverse(double* brick, int is2d, int level, int coarsest)
{
  /* Core/Wavelet.cpp:144 InverseCdf53 */
  int N[3];
  brick_dims(is2d, N);
  for (int s = 0; s < nsubbands(is2d); ++s)
  {
    if (s == 0 && !coarsest)
      continue;
    ogrid g;
    int h[3];
    subband_grid(is2d, s, &g, h);
    scale_grid(brick, N, &g, 1.0 / subband_weight(is2d, s, level));
  }
  ogrid G = { { 0, 0, 0 }, { N[0], N[1], N[2] }, { 1, 1, 1 } };
  for (int a = (is2d ? 1 : 2); a >= 0; --a)
    lift(brick, N, &G, N, a, 0);
}

void oracle_copy_to_parent(const double* child, double* parent, int is2d, const int pos3[3])
{
  /* Core/idx2Encode.cpp:324-328: CopyGridExtent of subband 0 with non-extrapolated dims */
  int N[3];
  brick_dims(is2d, N);
  int nd[3] = { 16, 16, is2d ? 1 : 16 };
  for (int z = 0; z < nd[2]; ++z)
    for (int y = 0; y < nd[1]; ++y)
      for (int x = 0; x < nd[0]; ++x)
      {
        int cz = is2d ? 0 : 2 * z;
        long src = ((long)cz * N[1] + 2 * y) * N[0] + 2 * x;
        long dst = ((long)(pos3[2] * nd[2] + z) * N[1] + (pos3[1] * nd[1] + y)) * N[0] +
                   (pos3[0] * nd[0] + x);
        parent[dst] = child[src];
      }
}

void oracle_copy_from_parent(const double* parent, double* child, int is2d, const int pos3[3])
{
  /* Core/idx2Decode.cpp:285-293: CopyExtentGrid */
  int N[3];
  brick_dims(is2d, N);
  int nd[3] = { 16, 16, is2d ? 1 : 16 };
  for (int z = 0; z < nd[2]; ++z)
    for (int y = 0; y < nd[1]; ++y)
      for (int x = 0; x < nd[0]; ++x)
      {
        int cz = is2d ? 0 : 2 * z;
        long dst = ((long)cz * N[1] + 2 * y) * N[0] + 2 * x;
        long src = ((long)(pos3[2] * nd[2] + z) * N[1] + (pos3[1] * nd[1] + y)) * N[0] +
                   (pos3[0] * nd[0] + x);
        child[dst] = parent[src];
      }
}

/* ------------------------------------------------------------------ */
/* bit streams: LSB-first, bytes little-endian (Core/BitStream.h)      */
/* ------------------------------------------------------------------ */

typedef struct
{
  uint8_t* buf;
  long cap;  /* bytes */
  long bits; /* bits written */
} bitw;

static void bw_put(bitw* w, uint64_t v, int n)
{
  for (int i = 0; i < n; ++i)
  {
    long p = w->bits + i;
    if ((p >> 3) < w->cap)
    {
      if ((v >> i) & 1u)
        w->buf[p >> 3] |= (uint8_t)(1u << (p & 7));
    }
  }
  w->bits += n;
}

typedef struct
{
  const uint8_t* buf;
  long bytes;
  long pos; /* bit position */
} bitr;

static uint64_t br_get(bitr* r, int n)
{
  uint64_t v = 0;
  for (int i = 0; i < n; ++i)
  {
    long p = r->pos + i;
    uint64_t b = (p >> 3) < r->bytes ? (r->buf[p >> 3] >> (p & 7)) & 1u : 0;
    v |= b << i;
  }
  r->pos += n;
  return v;
}

long long oracle_varint_stream(const uint64_t* vals, int n_var, int n_total, uint8_t* out,
                               long long cap)
{
  /* Core/VarInt.h:14 WriteVarByte (7 data bits, then a continue bit) and :82 WriteUnary
     (Val zero bits, then a one bit) */
  memset(out, 0, (size_t)cap);
  bitw w = { out, (long)cap, 0 };
  for (int i = 0; i < n_total; ++i)
  {
    uint64_t v = vals[i];
    if (i < n_var)
    {
      for (;;)
      {
        bw_put(&w, v & 0x7f, 7);
        v >>= 7;
        bw_put(&w, v != 0, 1);
        if (v == 0)
          break;
      }
    }
    else
    {
      for (uint64_t k = 0; k < v; ++k)
        bw_put(&w, 0, 1);
      bw_put(&w, 1, 1);
    }
  }
  return w.bits;
}

/* ------------------------------------------------------------------ */
/* Morton order (Core/BitOps.h:249,282)                                */
/* ------------------------------------------------------------------ */

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

uint32_t oracle_encode_morton3(uint32_t x, uint32_t y, uint32_t z)
{
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

/* ------------------------------------------------------------------ */
/* block transform (Core/Zfp.h, Core/Function.h, Core/Math.h)          */
/* ------------------------------------------------------------------ */

int oracle_exponent_f64(double v)
{
  /* Core/Math.h:524 Exponent<f64>: frexp exponent, clamped to 1-1023; zero -> -1023 */
  if (v != 0)
  {
    int e;
    frexp(v, &e);
    return e > -1022 ? e : -1022;
  }
  return -1023;
}

int oracle_exponent_f32(float v)
{
  if (v != 0)
  {
    int e;
    frexpf(v, &e);
    return e > -126 ? e : -126;
  }
  return -127;
}

/* zfp 4-point lifting (Core/Zfp.h:145 FLift, :181 ILift) */
static void fwd_lift4(int64_t* p, int s)
{
  int64_t x = p[0], y = p[s], z = p[2 * s], w = p[3 * s];
  x += w;
  x >>= 1;
  w -= x;
  z += y;
  z >>= 1;
  y -= z;
  x += z;
  x >>= 1;
  z -= x;
  w += y;
  w >>= 1;
  y -= w;
  w += y >> 1;
  y -= w >> 1;
  p[0] = x;
  p[s] = y;
  p[2 * s] = z;
  p[3 * s] = w;
}

static void inv_lift4(int64_t* p, int s)
{
  int64_t x = p[0], y = p[s], z = p[2 * s], w = p[3 * s];
  y += w >> 1;
  w -= y >> 1;
  y += w;
  w = (int64_t)((uint64_t)w << 1);
  w -= y;
  z += x;
  x = (int64_t)((uint64_t)x << 1);
  x -= z;
  y += z;
  z = (int64_t)((uint64_t)z << 1);
  z -= y;
  w += x;
  x = (int64_t)((uint64_t)x << 1);
  x -= w;
  p[0] = x;
  p[s] = y;
  p[2 * s] = z;
  p[3 * s] = w;
}

static void fwd_zfp(int64_t* p, int d)
{
  /* Core/Zfp.h:262 ForwardZfp(P, D): x, then y, then z */
  if (d == 3)
  {
    for (int z = 0; z < 4; ++z)
      for (int y = 0; y < 4; ++y)
        fwd_lift4(p + 4 * y + 16 * z, 1);
    for (int x = 0; x < 4; ++x)
      for (int z = 0; z < 4; ++z)
        fwd_lift4(p + 16 * z + x, 4);
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x)
        fwd_lift4(p + x + 4 * y, 16);
  }
  else if (d == 2)
  {
    for (int y = 0; y < 4; ++y)
      fwd_lift4(p + 4 * y, 1);
    for (int x = 0; x < 4; ++x)
      fwd_lift4(p + x, 4);
  }
  else if (d == 1)
    fwd_lift4(p, 1);
}

static void inv_zfp(int64_t* p, int d)
{
  /* Core/Zfp.h:312 InverseZfp(P, D): z, then y, then x */
  if (d == 3)
  {
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x)
        inv_lift4(p + x + 4 * y, 16);
    for (int x = 0; x < 4; ++x)
      for (int z = 0; z < 4; ++z)
        inv_lift4(p + 16 * z + x, 4);
    for (int z = 0; z < 4; ++z)
      for (int y = 0; y < 4; ++y)
        inv_lift4(p + 4 * y + 16 * z, 1);
  }
  else if (d == 2)
  {
    for (int x = 0; x < 4; ++x)
      inv_lift4(p + x, 4);
    for (int y = 0; y < 4; ++y)
      inv_lift4(p + 4 * y, 1);
  }
  else if (d == 1)
    inv_lift4(p, 1);
}

/* Coefficient order by total sequency (Core/Zfp.h:419 Perm3, :498 Perm2): the zfp
   ordering, written here as (i, j, k) triples. */
static const unsigned char kPerm3[64][3] = {
  { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 }, { 0, 1, 1 }, { 1, 0, 1 }, { 1, 1, 0 },
  { 2, 0, 0 }, { 0, 2, 0 }, { 0, 0, 2 }, { 1, 1, 1 }, { 2, 1, 0 }, { 2, 0, 1 }, { 0, 2, 1 },
  { 1, 2, 0 }, { 1, 0, 2 }, { 0, 1, 2 }, { 3, 0, 0 }, { 0, 3, 0 }, { 0, 0, 3 }, { 2, 1, 1 },
  { 1, 2, 1 }, { 1, 1, 2 }, { 0, 2, 2 }, { 2, 0, 2 }, { 2, 2, 0 }, { 3, 1, 0 }, { 3, 0, 1 },
  { 0, 3, 1 }, { 1, 3, 0 }, { 1, 0, 3 }, { 0, 1, 3 }, { 1, 2, 2 }, { 2, 1, 2 }, { 2, 2, 1 },
  { 3, 1, 1 }, { 1, 3, 1 }, { 1, 1, 3 }, { 3, 2, 0 }, { 3, 0, 2 }, { 0, 3, 2 }, { 2, 3, 0 },
  { 2, 0, 3 }, { 0, 2, 3 }, { 2, 2, 2 }, { 3, 2, 1 }, { 3, 1, 2 }, { 1, 3, 2 }, { 2, 3, 1 },
  { 2, 1, 3 }, { 1, 2, 3 }, { 0, 3, 3 }, { 3, 0, 3 }, { 3, 3, 0 }, { 3, 2, 2 }, { 2, 3, 2 },
  { 2, 2, 3 }, { 1, 3, 3 }, { 3, 1, 3 }, { 3, 3, 1 }, { 2, 3, 3 }, { 3, 2, 3 }, { 3, 3, 2 },
  { 3, 3, 3 }
};
static const unsigned char kPerm2[16][2] = { { 0, 0 }, { 1, 0 }, { 0, 1 }, { 1, 1 },
                                             { 2, 0 }, { 0, 2 }, { 2, 1 }, { 1, 2 },
                                             { 3, 0 }, { 0, 3 }, { 2, 2 }, { 3, 1 },
                                             { 1, 3 }, { 3, 2 }, { 2, 3 }, { 3, 3 } };

static int perm_index(int d, int i)
{
  if (d == 3)
    return kPerm3[i][0] + 4 * kPerm3[i][1] + 16 * kPerm3[i][2];
  if (d == 2)
    return kPerm2[i][0] + 4 * kPerm2[i][1];
  return i;
}

static const uint64_t kNegaMask = 0xaaaaaaaaaaaaaaaaull;

static int quantize(const double* vals, int nvals, int prec, int is_f32, int64_t* q)
{
  /* Core/Function.h:98 QuantizeF32 / :115 QuantizeF64 */
  double maxabs = 0;
  for (int i = 0; i < nvals; ++i)
  {
    double a = fabs(vals[i]);
    maxabs = maxabs > a ? maxabs : a;
  }
  int emax = is_f32 ? oracle_exponent_f32((float)maxabs) : oracle_exponent_f64(maxabs);
  double scale = ldexp(1, prec - 1 - emax);
  for (int i = 0; i < nvals; ++i)
  {
    double v = scale * vals[i];
    /* truncating conversion; the reference relies on x86 cvttsd2si, which yields
       INT64_MIN for NaN or out-of-range values (only reachable for blocks whose planes
       are never coded) */
    if (v != v || v >= 9223372036854775808.0 || v < -9223372036854775808.0)
      q[i] = INT64_MIN;
    else
      q[i] = (int64_t)v;
  }
  return emax;
}

/* One bit plane of the group-test coder (Core/Zfp.h:771 Encode<u64>). */
static void encode_plane(const uint64_t* u, int nvals, int bp, int* N, bitw* w)
{
  uint64_t X = 0;
  for (int i = 0; i < nvals; ++i)
    X += ((u[i] >> bp) & 1u) << i;
  int n = *N;
  if (n > 0)
  {
    bw_put(w, X, n);
    X = n < 64 ? X >> n : X;
  }
  while (n < nvals)
  {
    int g = X != 0;
    bw_put(w, (uint64_t)g, 1);
    if (!g)
      break;
    while (n + 1 < nvals)
    {
      int b = (int)(X & 1u);
      bw_put(w, (uint64_t)b, 1);
      if (b)
        break;
      X >>= 1;
      ++n;
    }
    X >>= 1;
    ++n;
  }
  *N = n;
}

/* One bit plane of the decoder (Core/Zfp.h:990 Decode<u64>). */
static void decode_plane(uint64_t* u, int nvals, int bp, int* N, bitr* r, int deposit)
{
  int n = *N;
  uint64_t X = n > 0 ? br_get(r, n) : 0;
  while (n < nvals)
  {
    if (br_get(r, 1))
    {
      while (n + 1 < nvals)
      {
        if (br_get(r, 1))
          break;
        ++n;
      }
      X += 1ull << n;
      ++n;
    }
    else
      break;
  }
  if (deposit)
    for (int i = 0; X; ++i, X >>= 1)
      u[i] += (uint64_t)(X & 1u) << bp;
  *N = n;
}

/* plane-loop bounds (Core/idx2Encode.cpp:195-206, Core/idx2Decode.cpp:145-159):
   returns 1 when plane bp is coded for a block with exponent emax. Planes are
   visited from 63 down and the loop stops at the first plane that is not. */
static int plane_coded(int bp, int emax, int etol, int bpc)
{
  int realbp = bp + emax;
  int too_high = 64 - 6 > realbp - etol + 1;
  return !(too_high && ((realbp + 1024) % bpc) == 0);
}

static int block_ndims(const int bd[3])
{
  return (bd[0] > 1) + (bd[1] > 1) + (bd[2] > 1);
}

int oracle_block_encode(const double* vals, int ndims, int is_f32, double tol, int bpc,
                        int* emax_out, uint64_t* ucoeffs, int* plane_bp, int* plane_nin,
                        int* plane_bits, uint64_t* plane_words)
{
  const int nvals = 1 << (2 * ndims);
  const int prec = 63 - ndims;
  int64_t q[64];
  int emax = quantize(vals, nvals, prec, is_f32, q);
  fwd_zfp(q, ndims);
  for (int i = 0; i < nvals; ++i)
    ucoeffs[i] = ((uint64_t)q[perm_index(ndims, i)] + kNegaMask) ^ kNegaMask;
  *emax_out = emax;
  const int etol = oracle_exponent_f64(tol);
  const int end_bp = is_f32 ? 32 : 64;
  int N = 0, k = 0;
  for (int bp = 63; bp >= 64 - end_bp; --bp)
  {
    if (!plane_coded(bp, emax, etol, bpc))
      break;
    uint8_t buf[32];
    memset(buf, 0, sizeof buf);
    bitw w = { buf, 32, 0 };
    plane_bp[k] = bp;
    plane_nin[k] = N;
    encode_plane(ucoeffs, nvals, bp, &N, &w);
    plane_bits[k] = (int)w.bits;
    memcpy(plane_words + 4 * k, buf, 32);
    ++k;
  }
  return k;
}

static void dequantize_block(uint64_t* u, int ndims, int emax, double* out)
{
  const int nvals = 1 << (2 * ndims);
  const int prec = 63 - ndims;
  int64_t q[64];
  for (int i = 0; i < nvals; ++i)
    q[perm_index(ndims, i)] = (int64_t)((u[i] ^ kNegaMask) - kNegaMask);
  inv_zfp(q, ndims);
  /* Core/Function.h:140 Dequantize */
  double scale = 1.0 / ldexp(1, prec - 1 - emax);
  for (int i = 0; i < nvals; ++i)
    out[i] = scale * (double)q[i];
}

int oracle_block_decode(int ndims, int emax, int nplanes, const int* plane_bp,
                        const uint64_t* plane_words, double* out_vals)
{
  const int nvals = 1 << (2 * ndims);
  uint64_t u[64];
  memset(u, 0, sizeof u);
  int N = 0;
  for (int k = 0; k < nplanes; ++k)
  {
    bitr r = { (const uint8_t*)(plane_words + 4 * k), 32, 0 };
    decode_plane(u, nvals, plane_bp[k], &N, &r, 1);
  }
  dequantize_block(u, ndims, emax, out_vals);
  return 0;
}

/* ------------------------------------------------------------------ */
/* subband block loop (Core/idx2Encode.cpp:141-256)                    */
/* ------------------------------------------------------------------ */

/* Visit the blocks of a subband in the reference's Morton walk
   (Core/idx2Common.h:23 idx2_NextMorton). Returns the number of valid codes written to
   codes[] (at most 512). */
static int morton_walk(const int nb[3], uint32_t* codes)
{
  uint32_t last = oracle_encode_morton3((uint32_t)nb[0] - 1, (uint32_t)nb[1] - 1,
                                        (uint32_t)nb[2] - 1);
  int n = 0;
  for (uint32_t b = 0; b <= last; ++b)
  {
    uint32_t z[3] = { compact3(b), compact3(b >> 1), compact3(b >> 2) };
    if (!((int)z[0] < nb[0] && (int)z[1] < nb[1] && (int)z[2] < nb[2]))
    {
      int lsb = __builtin_ctz(b);
      b = (((b >> (lsb + 1)) + 1) << (lsb + 1)) - 1;
      continue;
    }
    codes[n++] = b;
  }
  return n;
}

typedef struct
{
  int bpkey, first_block, last_block;
  long bits;
  uint8_t* buf;
  long cap;
  int order; /* first-touch rank */
} ochan;

static void put_i32(uint8_t** p, int32_t v)
{
  memcpy(*p, &v, 4);
  *p += 4;
}

long oracle_encode_brick(const double* brick, int is2d, int level, int nlevels, int is_f32,
                         double tol, int bpc, uint8_t* out, long cap)
{
  int N[3];
  brick_dims(is2d, N);
  const int etol = oracle_exponent_f64(tol);
  const int end_bp = is_f32 ? 32 : 64;
  long need = 0;
  /* first pass computes into heap buffers, second serialises */
  uint8_t* tmp = (uint8_t*)malloc((size_t)(1 << 22));
  uint8_t* tp = tmp;
  for (int s = 0; s < nsubbands(is2d); ++s)
  {
    ogrid g;
    int h[3];
    subband_grid(is2d, s, &g, h);
    int nb[3] = { (g.dims[0] + 3) / 4, (g.dims[1] + 3) / 4, (g.dims[2] + 3) / 4 };
    uint32_t codes[512];
    int ncodes = morton_walk(nb, codes);
    int16_t exps[512];
    int nexps = 0;
    ochan ch[4096];
    int nch = 0;
    int key_to_ch[4096];
    for (int i = 0; i < 4096; ++i)
      key_to_ch[i] = -1;
    for (int bi = 0; bi < ncodes; ++bi)
    {
      uint32_t b = codes[bi];
      int z3[3] = { (int)compact3(b), (int)compact3(b >> 1), (int)compact3(b >> 2) };
      int d3[3], bd[3];
      for (int k = 0; k < 3; ++k)
      {
        d3[k] = z3[k] * 4;
        bd[k] = imin(4, g.dims[k] - d3[k]);
      }
      int coded_next = s == 0 && level + 1 < nlevels && bd[0] == 4 && bd[1] == 4 && bd[2] == 4;
      if (coded_next)
        continue;
      int nd = block_ndims(bd);
      int nvals = 1 << (2 * nd);
      int prec = 63 - nd;
      double vals[64];
      int j = 0;
      for (int z = 0; z < bd[2]; ++z)
        for (int y = 0; y < bd[1]; ++y)
          for (int x = 0; x < bd[0]; ++x)
          {
            long idx = ((long)(g.from[2] + (d3[2] + z) * g.strd[2]) * N[1] +
                        (g.from[1] + (d3[1] + y) * g.strd[1])) *
                         N[0] +
                       (g.from[0] + (d3[0] + x) * g.strd[0]);
            vals[j++] = brick[idx];
          }
      int64_t q[64];
      int emax = quantize(vals, nvals, prec, is_f32, q);
      exps[nexps++] = (int16_t)emax;
      fwd_zfp(q, nd);
      uint64_t u[64];
      for (int i = 0; i < nvals; ++i)
        u[i] = ((uint64_t)q[perm_index(nd, i)] + kNegaMask) ^ kNegaMask;
      int n = 0;
      for (int bp = 63; bp >= 64 - end_bp; --bp)
      {
        if (!plane_coded(bp, emax, etol, bpc))
          break;
        int bpkey = (bp + emax + 1024) / bpc;
        int c = key_to_ch[bpkey];
        if (c < 0)
        {
          c = nch++;
          key_to_ch[bpkey] = c;
          ch[c].bpkey = bpkey;
          ch[c].first_block = (int)b;
          ch[c].bits = 0;
          ch[c].cap = 1 << 16;
          ch[c].buf = (uint8_t*)calloc((size_t)ch[c].cap, 1);
          ch[c].order = c;
        }
        ch[c].last_block = (int)b;
        bitw w = { ch[c].buf, ch[c].cap, ch[c].bits };
        encode_plane(u, nvals, bp, &n, &w);
        ch[c].bits = w.bits;
      }
    }
    put_i32(&tp, nexps);
    memcpy(tp, exps, sizeof(int16_t) * (size_t)nexps);
    tp += sizeof(int16_t) * (size_t)nexps;
    put_i32(&tp, nch);
    for (int c = 0; c < nch; ++c)
    {
      int nbytes = (int)((ch[c].bits + 7) / 8);
      put_i32(&tp, ch[c].bpkey);
      put_i32(&tp, ch[c].first_block);
      put_i32(&tp, ch[c].last_block);
      put_i32(&tp, nbytes);
      memcpy(tp, ch[c].buf, (size_t)nbytes);
      tp += nbytes;
      free(ch[c].buf);
    }
  }
  need = (long)(tp - tmp);
  if (need <= cap)
    memcpy(out, tmp, (size_t)need);
  free(tmp);
  return need <= cap ? need : -need;
}

int oracle_decode_brick(double* brick, int is2d, int level, int nlevels, int is_f32,
                        double tol, int bpc, int mask, const int* spacing,
                        const uint8_t* rec, long rec_bytes)
{
  int N[3];
  brick_dims(is2d, N);
  const int etol = oracle_exponent_f64(tol);
  const int end_bp = is_f32 ? 32 : 64;
  const uint8_t* rp = rec;
  const uint8_t* rend = rec + rec_bytes;
  for (int s = 0; s < nsubbands(is2d); ++s)
  {
    if (rp + 4 > rend)
      return 1;
    int32_t nexps;
    memcpy(&nexps, rp, 4);
    rp += 4;
    const uint8_t* exps_p = rp;
    rp += 2 * (long)nexps;
    int32_t nch;
    memcpy(&nch, rp, 4);
    rp += 4;
    const uint8_t* chan_p[4096];
    bitr rd[4096];
    for (int i = 0; i < 4096; ++i)
      chan_p[i] = NULL;
    for (int c = 0; c < nch; ++c)
    {
      int32_t key, fb, lb, nbytes;
      memcpy(&key, rp, 4);
      memcpy(&fb, rp + 4, 4);
      memcpy(&lb, rp + 8, 4);
      memcpy(&nbytes, rp + 12, 4);
      rp += 16;
      chan_p[key] = rp;
      rd[key].buf = rp;
      rd[key].bytes = nbytes;
      rd[key].pos = 0;
      rp += nbytes;
    }
    if (!((mask >> s) & 1))
      continue;
    ogrid g;
    int h[3];
    subband_grid(is2d, s, &g, h);
    int nb[3] = { (g.dims[0] + 3) / 4, (g.dims[1] + 3) / 4, (g.dims[2] + 3) / 4 };
    uint32_t codes[512];
    int ncodes = morton_walk(nb, codes);
    int ei = 0;
    const int* sp = spacing + 3 * s;
    for (int bi = 0; bi < ncodes; ++bi)
    {
      uint32_t b = codes[bi];
      int z3[3] = { (int)compact3(b), (int)compact3(b >> 1), (int)compact3(b >> 2) };
      int d3[3], bd[3];
      for (int k = 0; k < 3; ++k)
      {
        d3[k] = z3[k] * 4;
        bd[k] = imin(4, g.dims[k] - d3[k]);
      }
      int bypass = (d3[0] % sp[0]) != 0 || (d3[1] % sp[1]) != 0 || (d3[2] % sp[2]) != 0;
      int coded_next = s == 0 && level + 1 < nlevels && bd[0] == 4 && bd[1] == 4 && bd[2] == 4;
      if (coded_next)
        continue;
      int nd = block_ndims(bd);
      int nvals = 1 << (2 * nd);
      int16_t e16;
      memcpy(&e16, exps_p + 2 * ei, 2);
      ++ei;
      int emax = e16;
      uint64_t u[64];
      memset(u, 0, sizeof u);
      int n = 0, nbps = 0;
      for (int bp = 63; bp >= 64 - end_bp; --bp)
      {
        if (!plane_coded(bp, emax, etol, bpc))
          break;
        int bpkey = (bp + emax + 1024) / bpc;
        if (!chan_p[bpkey])
          break; /* a missing chunk ends the block's planes (Core/idx2Decode.cpp:166-168) */
        ++nbps;
        decode_plane(u, nvals, bp, &n, &rd[bpkey], !bypass);
      }
      if (nbps > 0 && !bypass)
      {
        double vals[64];
        dequantize_block(u, nd, emax, vals);
        int j = 0;
        for (int z = 0; z < bd[2]; ++z)
          for (int y = 0; y < bd[1]; ++y)
            for (int x = 0; x < bd[0]; ++x)
            {
              long idx = ((long)(g.from[2] + (d3[2] + z) * g.strd[2]) * N[1] +
                          (g.from[1] + (d3[1] + y) * g.strd[1])) *
                           N[0] +
                         (g.from[0] + (d3[0] + x) * g.strd[0]);
              brick[idx] = vals[j++];
            }
      }
    }
  }
  return 0;
}
