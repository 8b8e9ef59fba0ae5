// The oracle's CPU brick coder behind the library's brick_coder interface (test
// infrastructure): transforms and codes each brick of a plan level with oracle/idx2_oracle.c,
// so the library's host plan, packer and shard logic run on a machine without a GPU.
#pragma once

#include "encoder.h"
#include "format.h"

extern "C"
{
#include "idx2_oracle.h"
}

#include <algorithm>
#include <cstring>
#include <vector>

namespace idx2g
{

class oracle_coder : public brick_coder
{
public:
  oracle_coder(const dataset_format& f, const void* field) : f_(f), field_(field) {}

  int run_level(int level, const encode_plan& plan, level_output* out) override
  {
    const bool is2d = f_.is2d();
    const int NB = 33 * 33 * (is2d ? 1 : 33);
    const std::vector<brick_entry>& bricks = plan.levels[(size_t)level];
    const int nsb = f_.nsubbands();
    const int L = f_.nlevels;
    if (level + 1 < L)
      next_.assign(plan.levels[(size_t)level + 1].size() * (size_t)NB, 0.0);
    out->nbricks = (int)bricks.size();
    out->nsb = nsb;
    out->nexps.assign((size_t)nsb, 0);
    out->offset.assign(bricks.size() * (size_t)nsb, 0);
    out->stream.clear();
    std::vector<double> buf((size_t)NB);
    std::vector<uint8_t> rec(1 << 24);
    for (size_t bi = 0; bi < bricks.size(); ++bi)
    {
      const brick_entry& b = bricks[bi];
      if (level == 0)
      {
        std::fill(buf.begin(), buf.end(), 0.0);
        v3 from = b.brick3 * f_.brick_dims;
        for (int z = 0; z < b.valid.z; ++z)
          for (int y = 0; y < b.valid.y; ++y)
            for (int x = 0; x < b.valid.x; ++x)
            {
              size_t src = ((size_t)(from.z + z) * (size_t)f_.dims.y + (size_t)(from.y + y)) *
                             (size_t)f_.dims.x +
                           (size_t)(from.x + x);
              double v = f_.type == dtype::float32 ? (double)((const float*)field_)[src]
                                                   : ((const double*)field_)[src];
              buf[((size_t)z * 33 + (size_t)y) * 33 + (size_t)x] = v;
              vmin_ = v < vmin_ ? v : vmin_;
              vmax_ = vmax_ < v ? v : vmax_;
            }
      }
      else
      {
        std::copy(cur_.begin() + (long)(bi * (size_t)NB), cur_.begin() + (long)((bi + 1) * (size_t)NB),
                  buf.begin());
      }
      int valid[3] = { b.valid.x, b.valid.y, b.valid.z };
      oracle_brick_forward(buf.data(), is2d, valid, level, level + 1 == L);
      if (level + 1 < L)
      {
        int pos[3] = { b.pos_in_parent.x, b.pos_in_parent.y, b.pos_in_parent.z };
        oracle_copy_to_parent(buf.data(), next_.data() + (size_t)b.parent * (size_t)NB, is2d, pos);
      }
      long n = oracle_encode_brick(buf.data(), is2d, level, L, f_.type == dtype::float32, f_.tolerance,
                                   f_.bit_planes_per_chunk, rec.data(), (long)rec.size());
      if (n < 0)
        return UnknownError;
      const uint8_t* p = rec.data();
      for (int s = 0; s < nsb; ++s)
      {
        size_t bs = bi * (size_t)nsb + (size_t)s;
        int32_t ne;
        memcpy(&ne, p, 4);
        p += 4;
        out->nexps[(size_t)s] = ne;
        const uint8_t* exps = p;
        p += 2 * (size_t)ne;
        int32_t nch;
        memcpy(&nch, p, 4);
        p += 4;
        struct ch
        {
          int key, nbytes;
          const uint8_t* data;
        };
        std::vector<ch> chs;
        for (int c = 0; c < nch; ++c)
        {
          int32_t key, fb, lb, nbytes;
          memcpy(&key, p, 4);
          memcpy(&fb, p + 4, 4);
          memcpy(&lb, p + 8, 4);
          memcpy(&nbytes, p + 12, 4);
          p += 16;
          chs.push_back({ key, nbytes, p });
          p += nbytes;
        }
        // region in the layout of encoder.h: header, exponents, sizes, channel streams
        int kmin = 1 << 30, kmax = -1;
        for (auto& c : chs)
        {
          kmin = c.key < kmin ? c.key : kmin;
          kmax = c.key > kmax ? c.key : kmax;
        }
        const int nkeys = chs.empty() ? 0 : kmax - kmin + 1;
        if (nkeys > kKeyWindow)
          return DeviceStreamOverflow;
        std::vector<uint8_t>& st = out->stream;
        out->offset[bs] = st.size();
        size_t base = st.size();
        st.resize(base + region_header_bytes(ne, nkeys), 0);
        int32_t h[2] = { nkeys ? kmin : 1, nkeys };
        memcpy(st.data() + base, h, 8);
        memcpy(st.data() + base + 8, exps, 2 * (size_t)ne);
        uint32_t* sizes = (uint32_t*)(st.data() + base + 8 + ((2 * (size_t)ne + 3) & ~(size_t)3));
        std::sort(chs.begin(), chs.end(), [](const ch& a, const ch& b) { return a.key < b.key; });
        for (auto& c : chs)
          sizes[c.key - kmin] = (uint32_t)c.nbytes;
        for (auto& c : chs)
          st.insert(st.end(), c.data, c.data + c.nbytes);
        while (st.size() % 4)
          st.push_back(0);
      }
    }
    cur_.swap(next_);
    return NoError;
  }

  void value_range(double* vmin, double* vmax) override
  {
    *vmin = vmin_;
    *vmax = vmax_;
  }

private:
  const dataset_format& f_;
  const void* field_;
  std::vector<double> cur_, next_;
  double vmin_ = 1.7976931348623157e308, vmax_ = -1.7976931348623157e308;
};

} // namespace idx2g
