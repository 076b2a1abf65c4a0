// Device kernels around the decoder for transport-block serving (serve_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace syn {

// One code block of one transmission in a serving step.
struct ServeCb {
  float* acc;            // HARQ accumulator, ncb floats (circular buffer, variables 2Z..N)
  const float* e;        // received LLRs of this code block (e_len floats, interleaved order)
  int8_t* llr;           // decoder input: ncb int8 values (variables 2Z..N); null = f32 (acc only)
  const uint32_t* hard;  // decoder output: K' hard decisions, LSB-first words
  int ncb, fs, fe, m, c0;  // rate-matching walk (see tb.h RmWalk)
  int e_len, qm;
  int first;             // first transmission of the TB: the accumulator starts at +0
  int k_prime;           // bits covered by the code-block CRC-24B (CRC included)
  int crc_len;           // leading bits of this block inside the TB CRC-24A range
  int tb;                // index of the block's transport block in the step
  int hard_words;        // words of `hard` (K' bits)
};

// One transport block (one transmission) in a serving step.
struct ServeTb {
  int first_cb, n_cb;
  int payload;           // TB bits per code block
  int has_cb_crc;
  long long tb_size;     // A
  uint32_t x_payload;    // x^payload mod P_A
  uint32_t x_last;       // x^(CRC-24A bits of the last code block) mod P_A
  uint32_t* tb_bits;     // output: tb_size bits, LSB-first words
  int32_t* result;       // [0] crc_ok, [1] max iterations, [2 + i/32] bit i%32 = code block i CRC ok
};

// Per code block results of the CRC kernel.
struct ServeCbCrc {
  uint32_t crc_a;        // CRC-24A register of the block's first crc_len bits
  int ok_b;              // CRC-24B over K' bits is zero (or the TB has no CB CRC)
};

// x^n mod P for the 24-bit generator poly (MSB-first register convention).
uint32_t crc24_xpow_host(long long n, uint32_t poly);

// HARQ soft combining + quantization: acc[p] (+)= the received LLRs rate-matched to
// position p, in received order; llr[p] = quantize(acc[p] * scale).
cudaError_t serve_combine_launch(const ServeCb* d_cbs, int n_cbs, int max_ncb, float scale, cudaStream_t stream);
// Code-block CRCs (CRC-24B check, CRC-24A register of the TB part).
cudaError_t serve_cb_crc_launch(const ServeCb* d_cbs, int n_cbs, ServeCbCrc* d_out, cudaStream_t stream);
// Transport-block CRC fold, results and desegmented TB bits; iters[i] = iterations
// of code block i of the step.
cudaError_t serve_tb_finish_launch(const ServeTb* d_tbs, int n_tbs, const ServeCb* d_cbs, const ServeCbCrc* d_crc,
                                   const int32_t* d_iters, cudaStream_t stream);

}  // namespace syn
