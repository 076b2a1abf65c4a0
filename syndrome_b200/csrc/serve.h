// Transport-block serving engine: continuous batching of 5G NR DL-SCH
// transmissions on one GPU (serve.cpp).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/syndrome_ldpc.h"
#include "nr_kernels.h"
#include "serve_kernels.h"
#include "tb.h"

namespace syn {

struct ServeConfig {
  int max_step_cbs = 2048;               // code blocks per GPU step (at least one whole TB)
  // Steps in flight (concurrent on free SMs).  6: the same saturated throughput as 8
  // and more, with a shorter tail near saturation (concurrent steps share the SMs, so
  // each waits for its slowest work item longer).
  int slots = 6;
  // Steps beyond latency_slots go in flight only while at least backlog_cbs code blocks
  // wait: a light load keeps few steps sharing the SMs (each finishes sooner), a backlog
  // gets the concurrency that fills the SMs.  3 and 128: the same saturated throughput
  // as 6 steps always, p99 per transmission 0.81 instead of 1.10 ms at half of capacity.
  int latency_slots = 3;
  int backlog_cbs = 128;
  long long harq_bytes = 8LL << 30;      // device memory for HARQ accumulators
  long long staging_bytes = 256LL << 20; // device staging of host-memory LLRs, per step
  int iterations = 8;
  float beta = 0.5f;
  float scale = 8.0f;
  int app_clamp = 32767;
  // Code-block decode: 0 = the paired kernel in its tensor-memory form (two CTAs per SM),
  // 5 = the paired kernel with all state in shared memory (one CTA per SM).
  int decode_kernel = 0;
  // 0 = continuous: one persistent kernel takes each transmission's code blocks as soon
  // as they are published (serve_cont.cpp; with the tensor-memory decode, else steps);
  // 1 = steps of up to max_step_cbs code blocks, up to `slots` in flight.
  int mode = 0;
  // Continuous mode: the kernel exits once no CTA has found work for this long (it is
  // relaunched with the next transmission).
  long long idle_us = 2000;
};

// Best-fit allocator of [0, size) in units: free ranges by offset (merged on release)
// and by length, so that both take O(log n).
struct RangeAlloc {
  std::map<long long, long long> free_;  // offset -> length
  std::multimap<long long, long long> by_len_;  // length -> offset
  std::unordered_map<long long, long long> used_;
  long long used = 0;
  void reset(long long size) {
    free_.clear();
    by_len_.clear();
    used_.clear();
    used = 0;
    if (size > 0) add(0, size);
  }
  long long alloc(long long n);  // offset, or -1
  void release(long long off);

 private:
  void add(long long off, long long len) {
    free_[off] = len;
    by_len_.emplace(len, off);
  }
  void drop(std::map<long long, long long>::iterator it) {
    auto r = by_len_.equal_range(it->second);
    for (auto j = r.first; j != r.second; ++j)
      if (j->second == it->first) {
        by_len_.erase(j);
        break;
      }
    free_.erase(it);
  }
};

struct ServeResult {
  uint64_t id = 0;
  int crc_ok = 0;
  int max_iters = 0;
  int harq_tx = 0;
  int n_cb = 0;
  uint32_t cb_crc[5] = {0, 0, 0, 0, 0};
  double latency_us = 0.0;  // submit to completion
  double queue_us = 0.0;    // submit to the launch of its step
  double step_us = 0.0;     // GPU time of its step (first copy to last)
};

struct ServeStats {
  long long steps = 0, code_blocks = 0, transmissions = 0, harq_bytes_used = 0, pending = 0, in_flight = 0;
  long long tbs_held = 0, max_pending = 0;
  long long items = 0, item_threads = 0;  // work items launched and threads they occupy (of 384 each)
  double decode_ms = 0.0;                 // GPU time of the decode launches (CUDA events)
  double step_ms = 0.0;                   // GPU time from a step's first copy to its last
  double host_launch_ms = 0.0, host_finish_ms = 0.0;  // worker time building and finishing steps
};

// Continuous engine: what the persistent kernel and the worker spent their time on.
struct ServeCoreStats {
  long long items = 0;  // work items the kernel finished
  double busy_us = 0, combine_us = 0, decode_us = 0, crc_us = 0, finish_us = 0;  // summed over CTAs
  long long loops = 0;  // worker iterations
  double admit_us = 0, publish_us = 0, complete_us = 0;
};

class ServeEngine {
 public:
  ~ServeEngine();
  bool init(const ServeConfig& cfg, std::string* err);
  // Queues one transmission (redundancy version rv) of transport block id.  llr holds
  // C * E f32 channel LLRs (host memory unless on_device); it must stay valid until
  // the transmission's result has been polled.  Returns a SyndromeStatus code.
  int submit(uint64_t id, long long tb_size, float rate, int qm, long long g, int rv, const float* llr,
             long long llr_len, bool on_device, std::string* err);
  // Completed transmissions in completion order; waits up to timeout_us for the first.
  int poll(ServeResult* out, int cap, long long timeout_us);
  // Payload bits of the last decode of id (valid when its result had crc_ok).
  int fetch(uint64_t id, uint8_t* bits, long long len, std::string* err);
  // Drops the state of id (HARQ accumulators included).  Not while a transmission is in flight.
  int release(uint64_t id, std::string* err);
  ServeStats stats();
  // Zeros in the step engine.
  ServeCoreStats core_stats();
  // Codewords per work item for one shape (0 = as many as a CTA holds); takes effect
  // from the next step.
  void set_tile(int bg, int z, int tile);

 private:
  struct Tb {
    TbParams p;
    long long tb_size = 0, g = 0, e = 0;
    float rate = 0.0f;
    int qm = 1;
    long long harq_off = -1;  // bytes into the HARQ arena, -1 = none
    int tx_count = 0;
    bool busy = false;
    std::vector<uint32_t> bits;  // last decode's payload, LSB-first words
  };
  struct Pending {
    uint64_t id;
    int rv;
    const float* llr;
    bool on_device;
    std::chrono::steady_clock::time_point t0;
  };
  struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;  // around the decode launch
    cudaEvent_t ts = nullptr;                // step start
    bool busy = false;
    // device
    int8_t* d_llr = nullptr;
    uint32_t* d_hard = nullptr;
    int32_t* d_iters = nullptr;
    ServeCb* d_cbs = nullptr;
    ServeCbCrc* d_crc = nullptr;
    ServeTb* d_tbs = nullptr;
    int32_t* d_res = nullptr;
    uint32_t* d_bits = nullptr;
    MixItem* d_items = nullptr;
    MixCodeword* d_cws = nullptr;
    unsigned* d_queue = nullptr;
    float* d_stage = nullptr;
    // pinned host
    ServeCb* h_cbs = nullptr;
    ServeTb* h_tbs = nullptr;
    MixItem* h_items = nullptr;
    MixCodeword* h_cws = nullptr;
    int32_t* h_res = nullptr;
    uint32_t* h_bits = nullptr;
    // step contents
    std::vector<Pending> txs;
    std::vector<long long> bits_off;
    int n_cbs = 0;
    std::chrono::steady_clock::time_point launched;
  };

  // A transmission of the continuous mode from admission to its result.
  struct Flight {
    Pending pd;
    int tx = -1;              // transmission slot (record, code-block slots, report)
    int n_cb = 0;
    long long bits_off = -1;  // words into the host-mapped bits arena
    long long stage_off = -1; // floats into the device staging arena (host LLRs)
    cudaEvent_t staged = nullptr;
    uint32_t seq = 0;
    bool published = false;
    std::chrono::steady_clock::time_point t_pub;
  };

  void worker();
  bool launch_step(Slot& s);
  void finish_step(Slot& s);
  long long harq_alloc(long long bytes);
  void harq_free(long long off);
  bool init_cont(std::string* err);
  void release_cont();
  void worker_cont();
  bool admit_cont();
  bool publish_cont();
  bool complete_cont();
  void fail_all_cont();

  ServeConfig cfg_;
  int device_ = 0, sms_ = 0, max_words_ = 0, max_tb_words_ = 0, beta_q_ = 0;
  bool paired_ = false;  // paired mixed-shape decode (app_clamp >= 7874)
  bool tmem_ = false;    // ... in its tensor-memory form
  char* d_harq_ = nullptr;
  short* d_shift_ = nullptr;
  int* d_colz_ = nullptr;
  RangeAlloc harq_;  // HARQ arena, bytes (256-byte units are rounded up by harq_alloc)
  std::vector<Slot> slots_;
  std::deque<int> order_;                    // busy slots (worker thread only)
  int inflight_ = 0;                         // order_.size(), readable under mu_
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::unordered_map<uint64_t, Tb> tbs_;
  std::deque<Pending> pending_retx_;  // transmissions of blocks that hold accumulators
  std::deque<Pending> pending_new_;   // first transmissions (need accumulators)
  long long pending_cbs_ = 0;         // code blocks of the two queues
  std::deque<ServeResult> done_;
  std::atomic<long long> done_n_{0};  // done_.size(), readable without mu_
  static constexpr long long kPollSpinUs = 200;
  void push_done(const ServeResult& r);
  ServeStats stats_;
  bool stop_ = false;
  std::thread thread_;
  std::string fatal_;
  std::atomic<int> tiles_[2][385] = {};

  // ---- continuous mode ----
  bool cont_ = false;
  cudaStream_t c_stream_ = nullptr, c_copy_ = nullptr;
  cudaEvent_t c_kernel_done_ = nullptr;
  bool c_running_ = false;
  ServeContArgs c_args_{};
  ServeJob* h_ring_ = nullptr;       // host-mapped
  ServeTxRec* h_recs_ = nullptr;
  ServeTxOut* h_outs_ = nullptr;
  unsigned long long* h_tail_ = nullptr;
  unsigned* h_stop_ = nullptr;
  uint32_t* h_bits_ = nullptr;
  uint32_t* d_bits_map_ = nullptr;   // device address of h_bits_
  unsigned long long c_tail_ = 0;    // items published
  int c_txs_ = 0;
  long long c_cbs_ = 0, c_bits_words_ = 0, c_stage_floats_ = 0;
  int8_t* d_c_llr_ = nullptr;
  uint32_t* d_c_hard_ = nullptr;
  int32_t* d_c_iters_ = nullptr;
  ServeCbCrc* d_c_crc_ = nullptr;
  int* d_c_done_ = nullptr;
  int* d_c_smbusy_ = nullptr;
  ServeCtl* d_c_ctl_ = nullptr;
  uint32_t* d_c_tabs_ = nullptr;     // CRC slice tables, then x^n tables
  float* d_c_stage_ = nullptr;
  std::vector<int> c_free_tx_;
  std::vector<int> c_free_cb_;  // free code-block slots
  int* h_slots_ = nullptr;       // host-mapped [c_txs_][kServeMaxCbs] code-block slots per transmission
  RangeAlloc c_bits_alloc_, c_stage_alloc_;
  // flights by transmission slot (worker thread only): admitted and not yet published
  // (admission order), published (any order, c_pub_pos_ = index in c_pub_ or -1)
  std::vector<Flight> c_fl_;
  std::vector<int> c_unpub_, c_pub_, c_pub_pos_, c_done_scratch_;
  std::vector<cudaEvent_t> c_events_;  // free staging events
  uint32_t c_seq_ = 0;
  unsigned c_epoch_ = 0;  // launches of the persistent kernel
  std::atomic<long long> c_loops_{0}, c_admit_ns_{0}, c_publish_ns_{0}, c_complete_ns_{0};
};

// Open-loop Poisson load against an engine (serve_load.cpp, syndrome_serve_run_load).
int run_load(ServeEngine& eng, const SyndromeLoadTb* pool, size_t pool_n, const SyndromeLoadSpec& spec,
             SyndromeLoadReport* rep, double* lat_out, size_t lat_cap, std::string* err);

}  // namespace syn
