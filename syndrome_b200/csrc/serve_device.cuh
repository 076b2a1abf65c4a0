// Device helpers of the serving path shared by the step kernels (serve_kernels.cu) and
// the persistent serving kernel (nr_pair_kernels.cu): CRC-24 arithmetic and the HARQ
// combine of one circular-buffer position.
//
// CRC-24A / CRC-24B (crc.rs:65-350): MSB-first register, zero initial value, no final
// XOR, so the register of a message M is M(x) * x^24 mod P and CRCs compose linearly:
// CRC(A|B) = CRC(A) * x^|B| + CRC(B) (mod P).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "serve_kernels.h"

namespace syn {
namespace srv {

constexpr uint32_t kPolyA = 0x864CFBu, kPolyB = 0x800063u;
constexpr int kCombMaxAdds = 16;  // contributions per position: E <= 8 * ncb and M >= ncb / 2

// a * b mod P (24-bit polynomials).
__host__ __device__ inline uint32_t crc_mulmod(uint32_t a, uint32_t b, uint32_t poly) {
  uint32_t r = 0;
  for (int i = 23; i >= 0; --i) {
    r <<= 1;
    if (r & 0x1000000u) r ^= 0x1000000u | poly;
    if ((b >> i) & 1u) r ^= a;
  }
  return r;
}

// x^n mod P.
__host__ __device__ inline uint32_t crc_xpow(long long n, uint32_t poly) {
  uint32_t result = 1u, base = 2u;  // x^0, x^1
  while (n > 0) {
    if (n & 1) result = crc_mulmod(result, base, poly);
    base = crc_mulmod(base, base, poly);
    n >>= 1;
  }
  return result;
}

__device__ inline uint32_t crc_bit(uint32_t reg, uint32_t bit, uint32_t poly) {
  const uint32_t fb = ((reg >> 23) ^ bit) & 1u;
  reg = (reg << 1) & 0xFFFFFFu;
  return fb ? reg ^ poly : reg;
}

// Slice-by-4 register step of one 32-bit word w (first stream bit in the MSB) from
// register reg: ((reg << 8) ^ w) * x^24 mod P, with t[k][v] = v * x^(8k + 24) mod P.
__device__ __forceinline__ uint32_t crc_step4(uint32_t reg, uint32_t w, const uint32_t (*t)[256]) {
  const uint32_t x = (reg << 8) ^ w;
  return t[3][x >> 24] ^ t[2][(x >> 16) & 0xFFu] ^ t[1][(x >> 8) & 0xFFu] ^ t[0][x & 0xFFu];
}

// CRC register of bits [0, nbits) of LSB-first packed words (stream bit i is bit i % 32
// of word i / 32), one thread.
__device__ inline uint32_t thread_crc(const uint32_t* words, int nbits, const uint32_t (*t)[256], uint32_t poly) {
  const int full = nbits >> 5, rem = nbits & 31;
  uint32_t reg = 0;
  for (int w = 0; w < full; ++w) reg = crc_step4(reg, __brev(words[w]), t);
  if (rem) {
    const uint32_t w = words[full];
    for (int i = 0; i < rem; ++i) reg = crc_bit(reg, (w >> i) & 1u, poly);
  }
  return reg;
}

// x * y mod P for a fixed y, from the tables m[k][v] = (v << 8k) * y mod P.
__device__ __forceinline__ uint32_t mul_fixed(uint32_t x, const uint32_t (*m)[256]) {
  return m[0][x & 0xFFu] ^ m[1][(x >> 8) & 0xFFu] ^ m[2][(x >> 16) & 0xFFu];
}

// The rate-matching walk of one code block and transmission (tb.h RmWalk) with the
// fields the combine needs.
struct CombineWalk {
  int ncb, fs, fe, m, c0, e_len, qm, first;
};

// HARQ combine of circular-buffer position p (harq.rs:142-161 with
// rate_matching.rs:675-700): acc[p] (+)= the received LLRs that rate matching put at p,
// added in received order, exactly the order of the reference's scatter loop, so the
// f32 sums are bit-identical; then llr[p] = quantize(acc[p] * scale) (quantize.rs:331-343)
// unless llr is null.  c0 is already reduced mod m.  Accumulators and received values
// are read through L2 (ld.cg): a persistent kernel reuses their memory while it runs.
__device__ __forceinline__ void combine_position(int p, const CombineWalk& w, float* __restrict__ acc,
                                                 const float* __restrict__ e, int8_t* __restrict__ llr, float scale) {
  if (p >= w.fs && p < w.fe) {  // filler positions: never transmitted, the decoder pins them
    if (w.first) acc[p] = 0.0f;
    if (llr) llr[p] = 0;
    return;
  }
  const int c = p < w.fs ? p : p - (w.fe - w.fs);
  int k = c - w.c0;
  if (k < 0) k += w.m;
  float a = w.first ? 0.0f : __ldcg(acc + p);
  if (w.qm == 1) {
    for (int kk = k; kk < w.e_len; kk += w.m) a = __fadd_rn(a, __ldcg(e + kk));
  } else {
    // received index of selection kk: q = (kk % qm) * rows + kk / qm; add in q order
    const int rows = w.e_len / w.qm;
    int q[kCombMaxAdds];
    int n = 0;
    for (int kk = k; kk < w.e_len && n < kCombMaxAdds; kk += w.m) {
      const int d = kk / w.qm;
      const int v = (kk - d * w.qm) * rows + d;
      int j = n++;
      while (j > 0 && q[j - 1] > v) {
        q[j] = q[j - 1];
        --j;
      }
      q[j] = v;
    }
    for (int j = 0; j < n; ++j) a = __fadd_rn(a, __ldcg(e + q[j]));
  }
  acc[p] = a;
  if (!llr) return;  // f32 decode: the accumulator is the decoder input
  const float v = __fmul_rn(a, scale);
  int qv = 0;
  if (!isnan(v)) qv = (int)fminf(fmaxf(roundf(v), -127.0f), 127.0f);
  llr[p] = (int8_t)qv;
}

// The combine of one code block's positions by `threads` threads of a CTA (thread t:
// positions t, t + threads, ...).  BPSK (qm = 1) takes kCombU positions per thread at a
// time, their loads issued together (each position's contributions still added in
// received order); other qm go position by position.
constexpr int kCombU = 8;
__device__ __forceinline__ void combine_cb(const CombineWalk& w, float* __restrict__ acc,
                                           const float* __restrict__ e, int8_t* __restrict__ llr, float scale,
                                           int t, int threads) {
  if (w.qm != 1) {
    for (int p = t; p < w.ncb; p += threads) combine_position(p, w, acc, e, llr, scale);
    return;
  }
  for (int base = t; base < w.ncb; base += kCombU * threads) {
    float a[kCombU];
    int kk[kCombU];
    bool live[kCombU];
#pragma unroll
    for (int u = 0; u < kCombU; ++u) {
      const int p = base + u * threads;
      live[u] = p < w.ncb && (p < w.fs || p >= w.fe);
      const int c = p < w.fs ? p : p - (w.fe - w.fs);
      int k = c - w.c0;
      if (k < 0) k += w.m;
      kk[u] = live[u] ? k : w.e_len;
      a[u] = (live[u] && !w.first) ? __ldcg(acc + p) : 0.0f;
    }
    for (;;) {
      bool more = false;
#pragma unroll
      for (int u = 0; u < kCombU; ++u) {
        if (kk[u] < w.e_len) {
          a[u] = __fadd_rn(a[u], __ldcg(e + kk[u]));
          kk[u] += w.m;
          more = true;
        }
      }
      if (!more) break;
    }
#pragma unroll
    for (int u = 0; u < kCombU; ++u) {
      const int p = base + u * threads;
      if (p >= w.ncb) continue;
      if (!live[u]) {  // filler positions: never transmitted, the decoder pins them
        if (w.first) acc[p] = 0.0f;
        if (llr) llr[p] = 0;
        continue;
      }
      acc[p] = a[u];
      if (!llr) continue;
      const float v = __fmul_rn(a[u], scale);
      int qv = 0;
      if (!isnan(v)) qv = (int)fminf(fmaxf(roundf(v), -127.0f), 127.0f);
      llr[p] = (int8_t)qv;
    }
  }
}

}  // namespace srv
}  // namespace syn
