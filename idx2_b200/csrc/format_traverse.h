// Hierarchical traversal used for bricks, chunks and files (Core/idx2Common.h:318-462).
// The reference expands the same loop three times as macros; here it is one
// template.  The visiting order, the running counters and the cropping tests are
// the reference's, so that brick addresses and "brick in chunk" indices agree.
#pragma once

#include <cstdint>

namespace idx2g
{

namespace detail
{
inline int next_pow2(int v)
{
  int r = 1;
  while (r < v)
    r <<= 1;
  return r;
}
inline i64 crop_prod(v3 from, v3 to, const extent& e)
{
  v3 f = vmax(from, e.from), l = vmin(to - v3(1), e.last());
  if (!all_le(f, l))
    return 0;
  return prod(l - f + v3(1));
}
} // namespace detail

template <typename F>
void traverse(u64 order, v3 from3, v3 dims3, const extent& ext, const extent& ext2, F&& body)
{
  struct item
  {
    u64 order, prev;
    v3 from, to;
    i64 before;
    int in_parent;
    u64 address;
  };
  item stack[128];
  int top = 0;
  v3 ext3(detail::next_pow2(dims3.x), detail::next_pow2(dims3.y), detail::next_pow2(dims3.z));
  stack[0] = item{ order, order, from3, from3 + ext3, 0, 0, 0 };
  while (top >= 0)
  {
    item& t = stack[top];
    int d = (int)(t.order & 3);
    t.order >>= 2;
    if (d == 3)
    {
      if (t.order == 3)
        t.order = t.prev;
      else
        t.prev = t.order;
      continue;
    }
    item cur = t;
    --top;
    if (cur.to - cur.from == v3(1))
    {
      traverse_item ti;
      ti.from3 = cur.from;
      ti.address = cur.address;
      ti.item_in_parent = cur.in_parent;
      ti.items_before = cur.before;
      body(ti);
      continue;
    }
    item first = cur, second = cur;
    int half = cur.from[d] + (cur.to[d] - cur.from[d]) / 2;
    first.to[d] = half;
    second.from[d] = half;
    second.before = first.before + detail::crop_prod(first.from, first.to, ext);
    second.in_parent = first.in_parent + (int)detail::crop_prod(first.from, first.to, ext2);
    first.address = cur.address;
    second.address = cur.address + (u64)prod(first.to - first.from);
    if (all_lt(second.from, ext.to()) && all_lt(ext.from, second.to))
      stack[++top] = second;
    if (all_lt(first.from, ext.to()) && all_lt(ext.from, first.to))
      stack[++top] = first;
  }
}

} // namespace idx2g
