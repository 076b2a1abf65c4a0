// Host interface of the 5G NR specialised int8 kernel (nr_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace syn {

// Launch description shared by BG1/BG2.  See BatchRequest (decoder.h) for the
// meaning of the fields; app_clamp must be >= 255 and the input int8.
struct NrCommon {
  int z;
  int beta_q;
  int app_clamp;
  int prologue;
  int k;
  long long k_prime;
  const int8_t* llr;
  long long llr_stride;
  int llr_offset;
  long long batch;
  int cpb;
  int iterations;
  uint32_t* hard_packed;
  int hard_bits;
  long long hard_words_stride;
  int32_t* iters;
  int16_t* app_out;
  long long app_stride;
  int8_t* edge_r_out;
  long long edge_r_stride;
  uint8_t* hard_out;
  long long hard_stride;
  // Run-time constants (set by the launcher) that keep multiplies on the FMA pipe.
  int k32;
  int two;
};

// True if the layer-ordered column list equals the compiled BG tables.
bool nr_layout_matches(int bg, const int* cols, int n_edges);
// Codewords per CTA used by the kernel for lifting size z.
int nr_cpb(int bg, int z);
// shifts: per edge in layer order, already reduced mod z.
cudaError_t nr_decode_i8(int bg, const NrCommon& c, const int* shifts, int sms, cudaStream_t stream);

}  // namespace syn
