// The reference's per-transport-block f32 decoder and its frame pipeline, on the GPU
// (frames.cpp):
//   DlSchF32  transport_block.rs:405-1060 DlSchDecoder (f32 code-block decode)
//   FramePipe ldpc_pipeline.rs:288-598 LdpcPipeline (acquire / submit / try_recv /
//             release of N-length f32 frames)
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "decoder.h"
#include "serve_kernels.h"
#include "tb.h"

namespace syn {

// DlSchDecoder::decode with the f32 code-block decode: HARQ f32 soft combining
// (device accumulators, the serving engine's combine kernel in f32 mode), the 5G
// prologue on the N-length code-block LLRs and decode_layered_offset_min_sum for all
// C code blocks in one batched launch, then the CB CRC-24B and TB CRC-24A checks and
// the HARQ flush on success, as transport_block.rs:829-1053.
class DlSchF32 {
 public:
  ~DlSchF32();
  bool init(long long tb_size, float rate, int qm, long long g, int iterations, float beta, std::string* err);
  const TbParams& params() const { return p_; }
  long long e_per_cb() const { return e_; }
  long long output_bits() const { return e_ * p_.c; }
  // rx: C * E host f32 LLRs.  report = {crc_ok, max_iters_used, harq_tx_count};
  // cb_crc[C]; tb_out[tb_size] is written only when the CRCs pass.  Returns a
  // SyndromeStatus code.
  int decode(const float* rx, long long rx_len, int rv, uint8_t* tb_out, long long tb_len, int* report,
             uint8_t* cb_crc, std::string* err);
  void flush() { tx_ = 0; }

 private:
  TbParams p_;
  long long tb_size_ = 0, e_ = 0;
  int qm_ = 1, iterations_ = 0, tx_ = 0, words_ = 0;
  Graph g_;
  Decoder dec_;
  cudaStream_t stream_ = nullptr;
  float* d_acc_ = nullptr;     // [C][ncb] HARQ accumulators
  float* d_rx_ = nullptr;      // [C * E]
  ServeCb* d_cbs_ = nullptr;   // [C]
  uint32_t* d_hard_ = nullptr; // [C][words] K' decoded bits per block
  int32_t* d_iters_ = nullptr; // [C]
  void* d_ws_ = nullptr;
  size_t ws_bytes_ = 0;
  std::vector<ServeCb> h_cbs_;
  std::vector<uint32_t> h_hard_;
  std::vector<int32_t> h_iters_;
};

// LdpcPipeline on the GPU: a pool of pinned N-length f32 frames; submitted frames are
// decoded (decode_layered_offset_min_sum, the frame's LLRs become its posterior) in
// batches by `workers` host threads, each with its own stream and device buffers,
// and come back through try_recv in completion order.
class FramePipe {
 public:
  static constexpr int kPool = 256;       // frames (the reference's pool holds 16)
  static constexpr int kMaxBatch = 64;    // frames per decode launch
  ~FramePipe();
  bool init(const Graph& g, const Decoder* dec, int iterations, int workers, std::string* err);
  int workers() const { return (int)threads_.size(); }
  int acquire();                     // frame index, or -1 when every frame is taken
  bool submit(int f);                // false if f is not an acquired frame
  int try_recv();                    // a decoded frame, or -1
  bool release(int f);               // false if f is not a received frame
  float* llr(int f) { return h_llr_ + (size_t)f * n_; }
  const uint8_t* hard(int f) const { return h_hard_ + (size_t)f * n_; }
  int iterations_used(int f) const { return iters_[f]; }
  size_t& tag(int f) { return tags_[f]; }
  bool valid(int f) const { return f >= 0 && f < kPool; }
  const std::string& fatal() const { return fatal_; }

 private:
  enum State : uint8_t { kFree, kHeld, kQueued, kDecoding, kDone, kReceived };
  void run(int w);

  int n_ = 0, edge_ = 0, iterations_ = 0, device_ = 0;
  const Decoder* dec_ = nullptr;
  float* h_llr_ = nullptr;     // pinned [kPool][N]
  uint8_t* h_hard_ = nullptr;  // pinned [kPool][N]
  int32_t* h_iters_ = nullptr; // pinned [kPool]
  std::vector<int> iters_;
  std::vector<size_t> tags_;
  std::vector<State> state_;
  std::vector<int> free_;
  std::deque<int> queued_, done_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool stop_ = false;
  std::string fatal_;
  struct Worker {
    cudaStream_t stream = nullptr;
    float* d_llr = nullptr;   // [kMaxBatch][N] in, posterior out
    float* d_app = nullptr;
    uint8_t* d_hard = nullptr;
    int32_t* d_iters = nullptr;
    void* d_ws = nullptr;
    size_t ws_bytes = 0;
  };
  std::vector<Worker> ws_;
  std::vector<std::thread> threads_;
};

}  // namespace syn
