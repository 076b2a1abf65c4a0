// Batched GPU layered offset min-sum decoder (host-side interface).
//
// The decoder owns a copy of the code's layer tables on the device and launches
// the sm_100a kernels in ldpc_kernels.cu.  All data buffers are device pointers
// supplied by the caller; nothing on the decode path allocates.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "graph.h"

namespace syn {

// One batched decode request.  Codeword b's channel LLRs are
// llr[b * llr_stride + j] for variables llr_offset + j, j in [0, n - llr_offset);
// variables [0, llr_offset) start as erasures (0).  With prologue_5g the 5G NR
// initialisation is applied on top: filler positions [K - n_filler, K) are pinned
// (f32: 1e6, int8: app_clamp) and [0, 2Z) are erased (src/qc_ldpc.rs:711-732,
// 1496-1513).
struct BatchRequest {
  const void* llr = nullptr;      // int8 or int16 (int8 path, see llr_i16) or float (f32 path)
  int llr_i16 = 0;                // int8 path: input elements are int16 instead of int8
  long long llr_stride = 0;       // elements between codewords
  int llr_offset = 0;
  long long batch = 0;
  int iterations = 0;
  int prologue_5g = 0;
  long long n_filler = 0;
  // f32 path, Wi-Fi shortening and puncturing (src/wifi_rate_matching.rs:267-302): with
  // shorten set, row b holds the shorten_tx transmitted LLRs of codeword b, the
  // shorten_payload real information bits then the parity bits that were sent; the
  // decode starts from variables [0, P) = the payload, [P, K) = 1e6 (shortened,
  // known zero), [K, K + T - P) = the sent parity and the rest = 0 (punctured).
  // llr_offset must be 0 and prologue_5g off.
  int shorten = 0;
  long long shorten_payload = 0;
  long long shorten_tx = 0;
  // int8 path numerics (src/quantize.rs): beta_q = round(beta * scale) clamped, app clamp.
  int beta_q = 0;
  int app_clamp = 32767;
  // f32 path numerics.
  float beta = 0.0f;
  // Outputs (each nullable except where noted).
  uint32_t* hard_packed = nullptr;   // [batch][hard_words_stride] LSB-first bits of variables [0, hard_bits)
  int hard_bits = 0;
  long long hard_words_stride = 0;
  int32_t* iters = nullptr;          // [batch] iterations used
  void* app = nullptr;               // [batch][app_stride] final posterior (int16 or float)
  long long app_stride = 0;
  uint8_t* hard = nullptr;           // [batch][hard_stride] one byte per variable
  long long hard_stride = 0;
  void* edge_r = nullptr;            // [batch][edge_r_stride] final C->V messages, reference layout
  long long edge_r_stride = 0;
  // Kernel selection: 0 = automatic, 1 = generic layered kernel, 2 = 5G NR kernel,
  // 3 = paired 5G NR kernel (two codewords per 32-bit word), 4 = generic layered
  // kernel with its messages in global memory (1 compresses them into shared memory
  // where they fit).
  int kernel = 0;
  // Scratch for C->V messages when edge_r is null.
  void* workspace = nullptr;
  size_t workspace_bytes = 0;
};

enum class Precision { kInt8, kF32 };

class Decoder {
 public:
  ~Decoder();
  // Copies the layer tables to the current device.  Returns false with err set.
  bool init(const Graph& g, float offset_beta, std::string* err);
  const Graph& graph() const { return g_; }
  float offset_beta() const { return beta_; }

  // Scratch bytes the kernel needs for `batch` codewords when edge_r is not given.
  size_t workspace_bytes(Precision p, long long batch) const;

  // Launches the decode on `stream`.  Returns cudaSuccess or the launch error;
  // argument errors are reported as cudaErrorInvalidValue with err set.
  cudaError_t decode(Precision p, const BatchRequest& req, cudaStream_t stream,
                     std::string* err) const;

  // Generic int8 decode with its message scratch in a static device array instead
  // of a caller workspace: allocates nothing.  See ldpc_kernels.cu for the limits.
  cudaError_t decode_i8_noalloc(const BatchRequest& req, cudaStream_t stream, std::string* err) const;
  // Size of that static array (the public header's SYNDROME_NOALLOC_SCRATCH_BYTES,
  // checked equal at compile time in capi.cpp).
  static constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
  static constexpr size_t noalloc_scratch_bytes() { return kNoAllocScratchBytes; }

  // Kernel launch geometry chosen for this code (exposed for the tuner and tests).
  struct Geometry {
    int cpb;          // codewords per CTA
    int threads;      // threads per CTA
    int smem;         // dynamic shared memory bytes
    int max_ctas;     // resident CTAs on the device
    int maxdeg_tmpl;  // kernel instantiation
    int st_words;     // f32: compressed-message state words per thread (0: messages in global memory)
    int st_off;       // byte offset of that state in shared memory
  };
  // compress: messages compressed in shared memory where they fit (else in global memory)
  Geometry geometry(Precision p, long long batch, bool compress = true) const;

 private:
  Graph g_;
  float beta_ = 0.0f;
  int device_ = -1;
  int sms_ = 0;
  int nr_bg_ = -1;               // 0/1 when the 5G NR kernel applies to this code
  uint32_t* d_edge_ = nullptr;   // [E] (col * z) << 16 | shift
  int32_t* d_loff_ = nullptr;    // [mb + 1]
};

}  // namespace syn
