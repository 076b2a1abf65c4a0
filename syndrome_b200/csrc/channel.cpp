#include "channel.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace syn {

namespace {

inline float uniform01(uint64_t* st) {
  uint64_t x = *st;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  *st = x;
  uint32_t bits = 0x3F800000u | (uint32_t)(x >> 41);
  float f;
  std::memcpy(&f, &bits, 4);
  return f - 1.0f;
}

inline float gaussian(uint64_t* st) {
  const float u1 = std::max(uniform01(st), 1e-38f);
  const float u2 = uniform01(st);
  const float two_pi = 2.0f * 3.14159265358979323846f;
  return std::sqrt(-2.0f * std::log(u1)) * std::cos(two_pi * u2);
}

}  // namespace

uint64_t splitmix64(uint64_t seed) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return z == 0 ? 1 : z;
}

float awgn_sigma(float ebno_db, float rate) {
  const float lin = std::pow(10.0f, ebno_db / 10.0f);
  return std::sqrt(1.0f / (2.0f * rate * lin));
}

void awgn_llr(float ebno_db, float rate, uint64_t seed, const uint8_t* bits, long long n,
              float* out) {
  uint64_t st = splitmix64(seed);
  const float sigma = awgn_sigma(ebno_db, rate);
  const float scale = 2.0f / (sigma * sigma);
  for (long long i = 0; i < n; ++i) {
    const float x = bits[i] == 0 ? 1.0f : -1.0f;
    const float g = gaussian(&st);
    const float y = x + g * sigma;
    out[i] = y * scale;
  }
}

int16_t quantize_llr_i16(float llr, float scale) {
  const float v = llr * scale;
  if (std::isnan(v)) return 0;
  const float r = std::round(v);
  if (r >= 127.0f) return 127;
  if (r <= -127.0f) return -127;
  return (int16_t)r;
}

int8_t quantize_llr_i8(float llr, float scale) { return (int8_t)quantize_llr_i16(llr, scale); }

int beta_q(float beta, float scale) {
  const float s = beta * scale;
  if (!std::isfinite(s)) return 127;
  return (int)std::min(std::max(std::round(s), 0.0f), 127.0f);
}

void awgn_quantized_batch(const uint8_t* bits, long long n, long long bits_stride,
                          long long tx_begin, const float* ebno, float rate,
                          const uint64_t* seeds, float scale, int8_t* out,
                          long long out_stride, long long count, int threads) {
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  threads = (int)std::min<long long>(threads, std::max<long long>(count, 1));
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([=]() {
      std::vector<float> llr((size_t)n);
      for (long long b = t; b < count; b += threads) {
        awgn_llr(ebno[b], rate, seeds[b], bits + b * bits_stride, n, llr.data());
        int8_t* o = out + b * out_stride;
        for (long long i = tx_begin; i < n; ++i) o[i - tx_begin] = quantize_llr_i8(llr[i], scale);
      }
    });
  for (auto& th : pool) th.join();
}

}  // namespace syn
