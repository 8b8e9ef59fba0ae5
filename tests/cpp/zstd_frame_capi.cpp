// C entry point around the library's zstd-1.4.5-compatible frame compressor, for the parity
// tests (tests/test_zstd_frames.py builds it with idx2_b200/csrc/zstd_frame.cpp).
#include "zstd_frame.h"

#include <cstring>
#include <vector>

extern "C" size_t idx2g_test_zstd_compress(const void* src, size_t n, void* dst, size_t cap)
{
  std::vector<uint8_t> out;
  idx2g::zstd145::compress((const uint8_t*)src, n, &out);
  if (out.size() > cap)
    return 0;
  memcpy(dst, out.data(), out.size());
  return out.size();
}
