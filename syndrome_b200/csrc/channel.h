// Synthetic channel data for tests and benchmarks: BPSK over AWGN and the
// fixed-point LLR format.
//
// AwgnChannel follows syndrome src/channel_sim.rs:61-241: the state is seeded
// with splitmix64, uniforms come from xorshift64 (top 23 bits as an f32 mantissa
// in [1,2) minus 1), Gaussians from the Box-Muller cosine branch, and the channel
// LLR is 2 y / sigma^2 with sigma^2 = 1 / (2 R 10^(Eb/N0 / 10)).
//
// The fixed-point format follows src/quantize.rs: llr_q = clamp(round_half_away(
// llr * scale), -127, 127), NaN -> 0; beta_q = clamp(round(beta * scale), 0, 127),
// non-finite -> 127.
#pragma once

#include <cstdint>

namespace syn {

uint64_t splitmix64(uint64_t seed);
float awgn_sigma(float ebno_db, float rate);

// LLRs of `n` BPSK symbols (bit 0 -> +1) with the reference channel's stream.
void awgn_llr(float ebno_db, float rate, uint64_t seed, const uint8_t* bits, long long n,
              float* llr_out);

int8_t quantize_llr_i8(float llr, float scale);
int16_t quantize_llr_i16(float llr, float scale);
int beta_q(float beta, float scale);

// Batch helper: for each codeword b, runs the reference channel with seed
// seeds[b] (Eb/N0 ebno[b]) over bits [tx_begin, n) and writes the quantized LLRs
// (scale) to out + b * out_stride.  Uses `threads` host threads (0 = all).
void awgn_quantized_batch(const uint8_t* bits, long long n, long long bits_stride,
                          long long tx_begin, const float* ebno, float rate,
                          const uint64_t* seeds, float scale, int8_t* out,
                          long long out_stride, long long count, int threads);

}  // namespace syn
