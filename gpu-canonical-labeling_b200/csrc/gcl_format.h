// gcl_format.h -- the reference's canonical adjacency list, one row at a
// time, from a bit-packed canonical row (host and device).
//
// print_canonical_adjacency_list (main.cpp:33-70) writes, for canonical
// vertex i, the prefix "%3u : ", then " j" for every neighbour j in
// ascending order, starting a new line "\n    " (width 4) before a token when
// the line is not empty of tokens and width + token + 1 would exceed 80, and
// ends the row with ";\n".  format_row produces those bytes from the packed
// row (bit j % 64 of word j / 64 set for an edge to canonical vertex j), so
// the text can be written where the rows are, without the n x n byte matrix.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define GCL_HD __host__ __device__
#else
#define GCL_HD
#endif

namespace gcl {

GCL_HD inline uint32_t dec_len(uint32_t v) {
  uint32_t k = 1;
  while (v >= 10) {
    v /= 10;
    ++k;
  }
  return k;
}

GCL_HD inline void put_dec(char* p, uint32_t v, uint32_t len) {
  for (uint32_t k = len; k-- > 0;) {
    p[k] = (char)('0' + v % 10);
    v /= 10;
  }
}

GCL_HD inline uint32_t lowest_bit(uint64_t x) {
#if defined(__CUDA_ARCH__)
  return (uint32_t)(__ffsll((long long)x) - 1);
#else
  return (uint32_t)__builtin_ctzll(x);
#endif
}

constexpr int kListWidth = 80;  // max_width of print_canonical_adjacency_list

// Bytes of row i of an n-vertex graph's adjacency list; the bytes are written
// to out unless it is null.
GCL_HD inline uint64_t format_row(const uint64_t* row, uint32_t n, uint32_t i, char* out) {
  const uint32_t il = dec_len(i);
  const uint32_t pad = il < 3 ? 3 - il : 0;
  uint64_t len = 0;
  if (out) {
    for (uint32_t k = 0; k < pad; ++k) out[k] = ' ';
    put_dec(out + pad, i, il);
    out[pad + il] = ' ';
    out[pad + il + 1] = ':';
    out[pad + il + 2] = ' ';
  }
  len = pad + il + 3;
  int width = (int)len;
  bool first = true;
  const uint32_t words = (n + 63) / 64;
  for (uint32_t w = 0; w < words; ++w) {
    uint64_t bits = row[w];
    if (w + 1 == words && (n & 63)) bits &= (1ull << (n & 63)) - 1;  // only j < n
    while (bits) {
      const uint32_t j = w * 64 + lowest_bit(bits);
      bits &= bits - 1;
      const uint32_t tl = 1 + dec_len(j);
      if (!first && width + (int)tl + 1 > kListWidth) {
        if (out) {
          out[len] = '\n';
          for (int k = 1; k <= 4; ++k) out[len + k] = ' ';
        }
        len += 5;
        width = 4;
      }
      if (out) {
        out[len] = ' ';
        put_dec(out + len + 1, j, tl - 1);
      }
      len += tl;
      width += (int)tl;
      first = false;
    }
  }
  if (out) {
    out[len] = ';';
    out[len + 1] = '\n';
  }
  return len + 2;
}

}  // namespace gcl
