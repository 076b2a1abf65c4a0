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

// ---- mixed batches (one persistent launch over any BG / Z mix) ----
constexpr int kMixLiftSizes = 51;   // lifting sizes of TS 38.212 Table 5.3.2-1 (all <= 384)
constexpr int kMixEdges = 316;      // table row length (BG1 edge count; BG2 uses the first 197)

struct MixItem {
  int bg;     // 0 = BG1, 1 = BG2
  int z;      // lifting size
  int zi;     // index of z in the lifting-size list
  int count;  // codewords in this item
  int first;  // first entry of the item in MixArgs::cws
};

struct MixCodeword {
  long long llr_off;  // byte offset of the codeword's N - 2Z int8 LLRs in MixArgs::llr
  long long out_off;  // word offset of its packed hard decisions in MixArgs::out
  int n_filler;
  int hard_bits;
  int index;          // position of the codeword in the caller's list (iteration output)
  int pad;
};

struct MixArgs {
  const MixItem* items;
  int n_items;
  const MixCodeword* cws;
  const int8_t* llr;
  uint32_t* out;
  int32_t* iters;
  const short* shift_tab;  // [2][kMixLiftSizes][kMixEdges] shifts in layer order
  const int* colz_tab;     // [2][kMixLiftSizes][kMixEdges] column * z
  unsigned* queue;         // work counter, zeroed before each launch
  int beta_q;
  int app_clamp;
  int iterations;
  int k32;
  int two;
};

// Codewords one work item of shape (bg, z) can hold in the mixed kernel.
int mixed_slot_capacity(int bg, int z);
// Column bases (column * z) of the compiled BG tables in layer order.
void mixed_column_bases(int bg, int z, int* colz_out);
// Raises the kernel's dynamic shared-memory limit (once per device, outside capture).
cudaError_t mixed_kernel_prepare();
// Zeroes the queue and launches the persistent kernel on `sms` CTAs.
cudaError_t mixed_decode_launch(const MixArgs& m, int sms, cudaStream_t stream);

// True if the layer-ordered column list equals the compiled BG tables.
bool nr_layout_matches(int bg, const int* cols, int n_edges);
// Codewords per CTA used by the kernel for lifting size z.
int nr_cpb(int bg, int z);
// shifts: per edge in layer order, already reduced mod z.
cudaError_t nr_decode_i8(int bg, const NrCommon& c, const int* shifts, int sms, cudaStream_t stream);

// Paired kernel (nr_pair_kernels.cu, two codewords per 32-bit word): applies when
// app_clamp >= 3938 (>= 7874 with filler bits), where no posterior of a non-filler
// variable can reach the clamp.  c.cpb is chosen by the launcher.
bool nr_pair_applies(const NrCommon& c);

// f32 5G NR decode with compressed messages (nr_f32_kernels.cu), any lifting size: the
// same results as the generic f32 kernel.  ext_ws: nr_f32_workspace_bytes(bg, z, batch,
// sms) bytes; shifts: per edge in layer order, reduced mod z.
struct NrF32Common {
  const float* llr = nullptr;
  long long llr_stride = 0;
  int llr_offset = 0;
  long long batch = 0;
  int iterations = 0;
  float beta = 0.0f;
  int prologue = 0;
  long long k_prime = 0;
  uint32_t* hard_packed = nullptr;
  int hard_bits = 0;
  long long hard_words_stride = 0;
  int32_t* iters = nullptr;
  float* app_out = nullptr;
  long long app_stride = 0;
  float* edge_r_out = nullptr;
  long long edge_r_stride = 0;
  uint8_t* hard_out = nullptr;
  long long hard_stride = 0;
  float* ext_ws = nullptr;
};
bool nr_f32_applies(int bg, int z);
size_t nr_f32_workspace_bytes(int bg, int z, long long batch, int sms);
cudaError_t nr_f32_decode(int bg, const NrF32Common& c, int z, const int* shifts, int sms, cudaStream_t stream);
// Paired mixed-shape kernel (same MixArgs as mixed_decode_launch; needs app_clamp >=
// 7874).  Work items hold up to pair_mixed_capacity codewords of one shape.
int pair_mixed_capacity(int bg, int z);
cudaError_t pair_mixed_prepare();
cudaError_t pair_mixed_launch(const MixArgs& m, int sms, cudaStream_t stream);
// The same decode with the check-row state mostly in tensor memory, two CTAs per SM
// (same items and results); for batches whose codewords report hard decisions of at
// most their pair_mixed_core_columns(bg) * z core variables.
cudaError_t pair_tm_mixed_prepare();
cudaError_t pair_tm_mixed_launch(const MixArgs& m, int sms, cudaStream_t stream);
int pair_mixed_core_columns(int bg);
// tmem: at Z = 384, the variant that keeps most check-row state in tensor memory (two
// codeword pairs per SM) instead of the one that keeps it all in shared memory.
cudaError_t nr_pair_decode_i8(int bg, const NrCommon& c, const int* shifts, int sms, cudaStream_t stream,
                              bool tmem = true);

}  // namespace syn
