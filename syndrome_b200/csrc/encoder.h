// Systematic QC-LDPC encoder (host side).
//
// Produces the unique codeword c = [info | parity] with H c = 0 for the codes the
// decoder supports (5G NR BG1/BG2 at every lifting size, the twelve 802.11
// matrices, any raw graph whose parity part is invertible).  Same results as
// syndrome's QcLdpcEncoder::encode (src/qc_ldpc.rs:2592-2618): the parity part of
// H is invertible, so the codeword is unique.
//
// Method (this library's own): the parity columns split into a "core" that must
// be solved jointly and an "extension" whose blocks are each fixed by one layer.
// For 5G NR the core is the 4 double-diagonal parity blocks and every layer >= 4
// carries an unshifted identity on its own extension column; for 802.11 the whole
// parity part is the core.  The core's GF(2) inverse is computed once per code;
// each codeword then costs one core syndrome, one bit-matrix/vector product and
// one pass over the extension layers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

#include "graph.h"

namespace syn {

class Encoder {
 public:
  // Returns false if the parity part of the graph is singular.
  bool init(const Graph& g);
  const Graph& graph() const { return g_; }

  // info: k() bits (one per byte, LSB used); codeword: n() bytes.
  void encode(const uint8_t* info, uint8_t* codeword) const;

  // Encodes `count` codewords with `threads` host threads (0 = hardware concurrency).
  void encode_batch(const uint8_t* info, long long info_stride, uint8_t* codewords,
                    long long cw_stride, long long count, int threads) const;

  // The same codewords computed on the GPU (encoder_kernels.cu): info and codewords are
  // device arrays (one bit per byte), enqueued on `stream`.  The device copy of the
  // tables is made on the first call, on the current device.
  cudaError_t encode_batch_device(const uint8_t* d_info, long long info_stride, uint8_t* d_codewords,
                                  long long cw_stride, long long count, cudaStream_t stream) const;

 private:
  Graph g_;
  int core_blocks_ = 0;                 // parity blocks solved jointly
  int core_bits_ = 0;                   // core_blocks_ * z
  int words_ = 0;                       // 64-bit words per inverse row
  std::vector<uint64_t> inv_;           // core_bits_ x words_ bit matrix (row-major)
  // Device tables (encoder_kernels.cu), made on first use and shared by copies.
  struct Dev {
    std::mutex mu;
    int device = -1;
    uint32_t* inv_t = nullptr;  // [words32][core_bits] transposed inverse
    int32_t* loff = nullptr;    // [mb + 1]
    uint32_t* edge = nullptr;   // [E] col << 16 | shift
    ~Dev();
  };
  std::shared_ptr<Dev> dev_ = std::make_shared<Dev>();
};

}  // namespace syn
