// Mixed batches of the twelve IEEE 802.11 LDPC matrices, f32 layered offset min-sum,
// one persistent launch (kernel in ldpc_kernels.cu, host plan in wifi_mixed.cpp).
//
// No counterpart in the reference, which decodes one codeword per call; the
// per-codeword arithmetic is its f32 decode_layered_offset_min_sum
// (src/qc_ldpc.rs:962-1221) on the matrices of src/wifi_ldpc_tables.rs:339-453.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace syn {

// One matrix as the kernel sees it.
struct WmShape {
  int z, n, mb, n_edges;
  int cpb;          // codeword slots per CTA: floor(384 / z)
  int st_words;     // compressed-message state words per thread
  int maxdeg_tmpl;  // row-update instantiation (8, 12, 16 or 24)
  int edge_off;     // first edge word in WmArgs::edges: (col * z) << 16 | shift
  int loff_off;     // first layer offset in WmArgs::loffs (mb + 1 entries)
  int pad;
};

struct WmCodeword {
  long long llr_off;  // offset (elements) of its N f32 channel LLRs in WmArgs::llr
  long long out_off;  // word offset of its packed hard decisions in WmArgs::out
  int hard_bits;      // leading variables reported
  int index;          // position in the caller's list (iteration output)
};

// A run of consecutive codeword records of one matrix, taken from the device queue
// by a CTA as a unit; its slots refill from the run as codewords finish.
struct WmChunk {
  int shape;
  int first;
  int count;
  int pad;
};

struct WmArgs {
  const WmShape* shapes;
  const uint32_t* edges;
  const int32_t* loffs;
  const WmCodeword* cws;
  const WmChunk* chunks;
  int n_chunks;
  const float* llr;
  uint32_t* out;
  int32_t* iters;
  unsigned* queue;  // chunk counter, zeroed before each launch
  int iterations;
  float beta;
};

constexpr int kWmThreads = 384;
constexpr int kWmMaxEdges = 96;
constexpr int kWmMaxLayers = 16;
constexpr int kWmMaxSlots = 16;

// Shared-memory bytes of a CTA holding `shape` (header, tables, posteriors, state).
int wifi_mixed_smem_bytes(const WmShape& s);
// Raises the kernel's shared-memory limit; CTAs per SM the kernel gets with `smem`.
cudaError_t wifi_mixed_prepare(int smem, int* ctas_per_sm);
cudaError_t wifi_mixed_launch(const WmArgs& a, int ctas, int smem, cudaStream_t stream);

struct WifiMixedCodeword {
  int z, rate_num, rate_den;
  int hard_bits;
  long long llr_offset;  // elements (f32) into the batch's LLR buffer
  long long out_offset;  // words into the output
};

class WifiMixedPlan {
 public:
  ~WifiMixedPlan();
  // chunk: codewords per queue entry of a matrix (0: about four chunks per CTA over the
  // whole batch, at least four codewords or a CTA's slots if fewer).
  bool init(const std::vector<WifiMixedCodeword>& cws, float beta, int iterations, int chunk, std::string* err);
  cudaError_t decode(const float* d_llr, uint32_t* d_out, int32_t* d_iters, bool use_graph, cudaStream_t stream);
  long long llr_needed() const { return need_llr_; }
  long long out_words_needed() const { return need_out_; }
  int codewords() const { return n_codewords_; }
  int chunks() const { return n_chunks_; }
  int ctas() const { return ctas_; }

 private:
  void release();
  WmArgs args(const float* d_llr, uint32_t* d_out, int32_t* d_iters) const;
  int device_ = -1, ctas_ = 0, smem_ = 0, n_chunks_ = 0, n_codewords_ = 0, iterations_ = 0;
  float beta_ = 0.0f;
  long long need_llr_ = 0, need_out_ = 0;
  WmShape* d_shapes_ = nullptr;
  uint32_t* d_edges_ = nullptr;
  int32_t* d_loffs_ = nullptr;
  WmCodeword* d_cws_ = nullptr;
  WmChunk* d_chunks_ = nullptr;
  unsigned* d_queue_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  const float* g_llr_ = nullptr;
  uint32_t* g_out_ = nullptr;
  int32_t* g_iters_ = nullptr;
};

}  // namespace syn
