#include "encoder.h"

#include <algorithm>
#include <cstring>
#include <thread>

namespace syn {

namespace {

// True when layers >= 4 each hold exactly one parity edge outside the first four
// parity blocks, on their own column kb + layer with shift 0, and layers 0..3 hold
// none: the 5G NR core/extension structure.
bool has_nr_extension(const Graph& g) {
  if (g.mb < 5) return false;
  for (int l = 0; l < g.mb; ++l) {
    int ext = 0;
    for (int e = g.layer_off[l]; e < g.layer_off[l + 1]; ++e) {
      if (g.cols[e] >= g.kb + 4) {
        if (l < 4 || g.cols[e] != g.kb + l || g.shifts[e] != 0) return false;
        ++ext;
      }
    }
    if (l >= 4 && ext != 1) return false;
  }
  return true;
}

}  // namespace

bool Encoder::init(const Graph& g) {
  g_ = g;
  const int z = g.z;
  core_blocks_ = has_nr_extension(g) ? 4 : g.mb;
  core_bits_ = core_blocks_ * z;
  // Augmented [H_core | I] and Gauss-Jordan elimination over GF(2).
  const int w2 = (2 * core_bits_ + 63) / 64;
  std::vector<uint64_t> a((size_t)core_bits_ * w2, 0);
  auto row = [&](int r) { return &a[(size_t)r * w2]; };
  for (int l = 0; l < core_blocks_; ++l)
    for (int e = g.layer_off[l]; e < g.layer_off[l + 1]; ++e) {
      int c = g.cols[e];
      if (c < g.kb || c >= g.kb + core_blocks_) continue;
      for (int zi = 0; zi < z; ++zi) {
        int s = zi + g.shifts[e];
        int col = (c - g.kb) * z + (s >= z ? s - z : s);
        row(l * z + zi)[col >> 6] ^= 1ull << (col & 63);
      }
    }
  for (int r = 0; r < core_bits_; ++r) {
    int col = core_bits_ + r;
    row(r)[col >> 6] |= 1ull << (col & 63);
  }
  for (int col = 0; col < core_bits_; ++col) {
    int piv = -1;
    for (int r = col; r < core_bits_; ++r)
      if ((row(r)[col >> 6] >> (col & 63)) & 1) {
        piv = r;
        break;
      }
    if (piv < 0) return false;
    if (piv != col) std::swap_ranges(row(piv), row(piv) + w2, row(col));
    const uint64_t* pr = row(col);
    for (int r = 0; r < core_bits_; ++r) {
      if (r == col || !((row(r)[col >> 6] >> (col & 63)) & 1)) continue;
      uint64_t* rr = row(r);
      for (int w = 0; w < w2; ++w) rr[w] ^= pr[w];
    }
  }
  words_ = (core_bits_ + 63) / 64;
  inv_.assign((size_t)core_bits_ * words_, 0);
  for (int r = 0; r < core_bits_; ++r)
    for (int c = 0; c < core_bits_; ++c) {
      int col = core_bits_ + c;
      if ((row(r)[col >> 6] >> (col & 63)) & 1) inv_[(size_t)r * words_ + (c >> 6)] |= 1ull << (c & 63);
    }
  return true;
}

void Encoder::encode(const uint8_t* info, uint8_t* cw) const {
  const Graph& g = g_;
  const int z = g.z;
  const long long k = g.k();
  for (long long i = 0; i < k; ++i) cw[i] = info[i] & 1;
  // Core syndrome of the systematic part, packed.
  std::vector<uint64_t> syn(words_, 0);
  for (int l = 0; l < core_blocks_; ++l)
    for (int e = g.layer_off[l]; e < g.layer_off[l + 1]; ++e) {
      int c = g.cols[e];
      if (c >= g.kb) continue;
      const uint8_t* src = cw + (long long)c * z;
      const int sh = g.shifts[e];
      for (int zi = 0; zi < z; ++zi) {
        int s = zi + sh;
        if (src[s >= z ? s - z : s]) {
          int b = l * z + zi;
          syn[b >> 6] ^= 1ull << (b & 63);
        }
      }
    }
  uint8_t* par = cw + k;
  for (int r = 0; r < core_bits_; ++r) {
    const uint64_t* ir = &inv_[(size_t)r * words_];
    uint64_t acc = 0;
    for (int w = 0; w < words_; ++w) acc ^= ir[w] & syn[w];
    par[r] = (uint8_t)(__builtin_popcountll(acc) & 1);
  }
  // Extension layers: each fixes its own unshifted parity block.
  for (int l = core_blocks_; l < g.mb; ++l) {
    uint8_t* dst = cw + (long long)(g.kb + l) * z;
    std::memset(dst, 0, z);
    for (int e = g.layer_off[l]; e < g.layer_off[l + 1]; ++e) {
      int c = g.cols[e];
      if (c == g.kb + l) continue;
      const uint8_t* src = cw + (long long)c * z;
      const int sh = g.shifts[e];
      for (int zi = 0; zi < z; ++zi) {
        int s = zi + sh;
        dst[zi] ^= src[s >= z ? s - z : s];
      }
    }
  }
}

void Encoder::encode_batch(const uint8_t* info, long long info_stride, uint8_t* codewords,
                           long long cw_stride, long long count, int threads) const {
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  threads = (int)std::min<long long>(threads, std::max<long long>(count, 1));
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([=]() {
      for (long long i = t; i < count; i += threads)
        encode(info + i * info_stride, codewords + i * cw_stride);
    });
  for (auto& th : pool) th.join();
}

}  // namespace syn
