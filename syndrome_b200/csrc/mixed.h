// Host plan of a mixed-shape 5G NR int8 batch (see mixed.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "nr_kernels.h"

namespace syn {

struct MixedCodeword {
  int bg;               // 0 = BG1, 1 = BG2
  int z;                // lifting size
  int n_filler;         // K - K'
  int hard_bits;        // leading variables whose hard decisions are reported
  long long llr_offset; // byte offset of its N - 2Z int8 LLRs (variables 2Z..N)
  long long out_offset; // word offset of its packed hard decisions
};

// Codewords per work item for one shape (from the tuner).
struct TileHint {
  int bg, z, tile;
};

class MixedPlan {
 public:
  ~MixedPlan();
  bool init(const std::vector<MixedCodeword>& cws, int beta_q, int app_clamp, int iterations,
            const std::vector<TileHint>& hints, std::string* err);
  // Decodes the batch whose LLRs start at d_llr; d_iters (nullable) gets one entry
  // per codeword in the caller's order.
  cudaError_t decode(const int8_t* d_llr, uint32_t* d_out, int32_t* d_iters, bool use_graph, cudaStream_t stream);
  // Smallest buffers the batch reads and writes.
  long long llr_bytes_needed() const { return need_llr_; }
  long long out_words_needed() const { return need_out_; }
  int items() const { return n_items_; }
  // 0: automatic (the tensor-memory paired kernel when every codeword reports at most
  // its core columns' hard decisions), 5: the shared-memory paired kernel.  Returns
  // false for other values.
  bool set_kernel(int kernel);
  bool tmem() const { return tmem_; }
  int codewords() const { return n_codewords_; }
  const std::vector<MixItem>& item_list() const { return items_; }

 private:
  void release();
  MixArgs args(const int8_t* d_llr, uint32_t* d_out, int32_t* d_iters) const;
  int device_ = -1, sms_ = 0, n_items_ = 0, n_codewords_ = 0;
  bool paired_ = false;  // paired kernel (app_clamp >= 7874) or one codeword per thread
  bool tmem_ = false;    // paired, and no codeword reports hard decisions past its core columns
  int kernel_ = 0;
  int beta_q_ = 0, app_clamp_ = 32767, iterations_ = 0;
  long long need_llr_ = 0, need_out_ = 0;
  MixItem* d_items_ = nullptr;
  MixCodeword* d_cws_ = nullptr;
  unsigned* d_queue_ = nullptr;
  short* d_shift_ = nullptr;
  int* d_colz_ = nullptr;
  std::vector<MixItem> items_;
  cudaGraphExec_t exec_ = nullptr;
  const int8_t* g_llr_ = nullptr;
  uint32_t* g_out_ = nullptr;
  int32_t* g_iters_ = nullptr;
};

}  // namespace syn
