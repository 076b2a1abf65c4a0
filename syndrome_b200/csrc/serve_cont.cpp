// Continuous mode of the serving engine (serve.h, ServeConfig::mode = 0).
//
// No steps: one persistent kernel (serve_cont_kernel, nr_pair_kernels.cu) serves the
// whole stream.  The worker thread admits transmissions in the step engine's order
// (retransmissions first, then new blocks while their HARQ accumulators fit the HBM
// budget), gives each a transmission slot, a code-block slot per code block (decoder
// input, hard decisions, CRC record; any free ones, listed in host-mapped memory, so
// that no fragmentation holds up a large block) and a range of the host-mapped bits
// arena, writes its record and work items (code blocks of the transmission, up to a
// CTA's worth each) into host-mapped memory and publishes them by advancing the ring's
// tail.  The kernel's CTAs claim items as they come; a transmission's result is
// complete when its completion flag (host-mapped) carries the record's sequence
// number.  Host-memory LLRs are copied into a device staging arena first and published
// when the copy has finished.  The kernel winds down as a whole once no CTA has claimed
// work for idle_us; the worker relaunches it when it publishes into a ring no kernel
// serves.
//
// Results per transmission are those of the step engine (the same combine, decode,
// CRC and desegmentation, now in one kernel): identical whatever else is in flight.
#include <algorithm>
#include <atomic>
#include <cstring>

#include "serve.h"

namespace syn {

namespace {

constexpr int kLiftingSizes[kMixLiftSizes] = {2,  3,  4,  5,  6,  7,   8,   9,   10,  11,  12,  13,  14,
                                              15, 16, 18, 20, 22, 24,  26,  28,  30,  32,  36,  40,  44,
                                              48, 52, 56, 60, 64, 72,  80,  88,  96,  104, 112, 120, 128,
                                              144, 160, 176, 192, 208, 224, 240, 256, 288, 320, 352, 384};

int lift_index_of(int z) {
  for (int i = 0; i < kMixLiftSizes; ++i)
    if (kLiftingSizes[i] == z) return i;
  return -1;
}

template <class T>
bool host_mapped(T** p, size_t count) {
  void* v = nullptr;
  if (cudaHostAlloc(&v, sizeof(T) * std::max<size_t>(count, 1), cudaHostAllocMapped | cudaHostAllocPortable) !=
      cudaSuccess)
    return false;
  std::memset(v, 0, sizeof(T) * std::max<size_t>(count, 1));
  *p = static_cast<T*>(v);
  return true;
}

template <class T>
T* device_view(T* host) {
  void* d = nullptr;
  return cudaHostGetDevicePointer(&d, host, 0) == cudaSuccess ? static_cast<T*>(d) : nullptr;
}

}  // namespace

bool ServeEngine::init_cont(std::string* err) {
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return false;
  };
  c_cbs_ = std::max<long long>(2LL * 160, (long long)cfg_.max_step_cbs * cfg_.slots);
  c_txs_ = (int)std::min<long long>(c_cbs_, 8192);
  c_bits_words_ = 48LL << 20;  // 192 MiB of decoded payload in flight
  c_stage_floats_ = cfg_.staging_bytes / 4;
  bool ok = host_mapped(&h_ring_, (size_t)c_cbs_) && host_mapped(&h_recs_, (size_t)c_txs_) &&
            host_mapped(&h_outs_, (size_t)c_txs_) && host_mapped(&h_tail_, 1) && host_mapped(&h_stop_, 1) &&
            host_mapped(&h_slots_, (size_t)c_txs_ * kServeMaxCbs) &&
            host_mapped(&h_bits_, (size_t)c_bits_words_);
  if (!ok) return fail("allocating host-mapped serving memory failed");
  ok = cudaMalloc(&d_c_llr_, (size_t)c_cbs_ * kServeLlrStride) == cudaSuccess &&
       cudaMalloc(&d_c_hard_, sizeof(uint32_t) * (size_t)c_cbs_ * kServeHardWords) == cudaSuccess &&
       cudaMalloc(&d_c_iters_, sizeof(int32_t) * (size_t)c_cbs_) == cudaSuccess &&
       cudaMalloc(&d_c_crc_, sizeof(ServeCbCrc) * (size_t)c_cbs_) == cudaSuccess &&
       cudaMalloc(&d_c_done_, sizeof(int) * (size_t)c_txs_) == cudaSuccess &&
       cudaMalloc(&d_c_smbusy_, sizeof(int) * 1024) == cudaSuccess &&
       cudaMalloc(&d_c_ctl_, sizeof(ServeCtl)) == cudaSuccess &&
       cudaMalloc(&d_c_tabs_, sizeof(uint32_t) * (2 * 1024 + 2 * kServeXpow)) == cudaSuccess &&
       (c_stage_floats_ == 0 || cudaMalloc(&d_c_stage_, sizeof(float) * (size_t)c_stage_floats_) == cudaSuccess);
  if (!ok) return fail("allocating the serving buffers failed (HBM budget too large?)");
  // CRC tables: T_k[v] = v * x^(8k + 24) mod P, then x^n mod P for n <= 8448
  std::vector<uint32_t> tabs(2 * 1024 + 2 * kServeXpow);
  const uint32_t polys[2] = {kCrc24A, kCrc24B};
  for (int pi = 0; pi < 2; ++pi) {
    for (int k = 0; k < 4; ++k) {
      const uint32_t xk = crc24_xpow_host(8 * k + 24, polys[pi]);
      for (int v = 0; v < 256; ++v) tabs[pi * 1024 + k * 256 + v] = crc24_mulmod_host((uint32_t)v, xk, polys[pi]);
    }
    uint32_t x = 1u;
    for (int n = 0; n < kServeXpow; ++n) {
      tabs[2 * 1024 + pi * kServeXpow + n] = x;
      x = crc24_mulmod_host(x, 2u, polys[pi]);
    }
  }
  ok = cudaMemcpy(d_c_tabs_, tabs.data(), sizeof(uint32_t) * tabs.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemset(d_c_done_, 0, sizeof(int) * (size_t)c_txs_) == cudaSuccess &&
       cudaMemset(d_c_smbusy_, 0, sizeof(int) * 1024) == cudaSuccess &&
       cudaMemset(d_c_ctl_, 0, sizeof(ServeCtl)) == cudaSuccess &&
       cudaStreamCreateWithFlags(&c_stream_, cudaStreamNonBlocking) == cudaSuccess &&
       cudaStreamCreateWithFlags(&c_copy_, cudaStreamNonBlocking) == cudaSuccess &&
       cudaEventCreateWithFlags(&c_kernel_done_, cudaEventDisableTiming) == cudaSuccess &&
       serve_cont_prepare() == cudaSuccess;
  if (!ok) return fail("configuring the persistent serving kernel failed");
  d_bits_map_ = device_view(h_bits_);
  ServeContArgs& a = c_args_;
  a.ring = device_view(h_ring_);
  a.ring_cap = (unsigned long long)c_cbs_;  // items in flight <= code blocks in flight
  a.recs = device_view(h_recs_);
  a.slots = device_view(h_slots_);
  a.outs = device_view(h_outs_);
  a.host_tail = device_view(h_tail_);
  a.host_stop = device_view(h_stop_);
  if (!d_bits_map_ || !a.ring || !a.recs || !a.slots || !a.outs || !a.host_tail || !a.host_stop)
    return fail("no device address for host-mapped memory");
  a.ctl = d_c_ctl_;
  a.tx_done = d_c_done_;
  a.sm_busy = d_c_smbusy_;
  a.llr = d_c_llr_;
  a.hard = d_c_hard_;
  a.iters = d_c_iters_;
  a.crc = d_c_crc_;
  a.crc_tab = d_c_tabs_;
  a.xpow = d_c_tabs_ + 2 * 1024;
  a.shift_tab = d_shift_;
  a.colz_tab = d_colz_;
  a.beta_q = beta_q_;
  a.app_clamp = cfg_.app_clamp;
  a.iterations = cfg_.iterations;
  a.scale = cfg_.scale;
  a.idle_ns = (unsigned long long)cfg_.idle_us * 1000ULL;
  c_free_tx_.clear();
  for (int i = c_txs_ - 1; i >= 0; --i) c_free_tx_.push_back(i);
  c_fl_.assign(c_txs_, Flight());
  c_pub_pos_.assign(c_txs_, -1);
  c_unpub_.clear();
  c_pub_.clear();
  c_unpub_.reserve(c_txs_);
  c_pub_.reserve(c_txs_);
  c_free_cb_.clear();
  for (long long i = c_cbs_ - 1; i >= 0; --i) c_free_cb_.push_back((int)i);
  c_bits_alloc_.reset(c_bits_words_);
  c_stage_alloc_.reset(c_stage_floats_);
  return true;
}

void ServeEngine::release_cont() {
  if (h_stop_) {
    reinterpret_cast<std::atomic<unsigned>*>(h_stop_)->store(1u, std::memory_order_release);
    if (c_stream_) cudaStreamSynchronize(c_stream_);  // CTAs exit once the ring is drained
  }
  if (c_copy_) cudaStreamSynchronize(c_copy_);
  for (int tx : c_unpub_)
    if (c_fl_[tx].staged) c_events_.push_back(c_fl_[tx].staged);
  c_unpub_.clear();
  c_pub_.clear();
  for (cudaEvent_t e : c_events_) cudaEventDestroy(e);
  c_events_.clear();
  if (c_kernel_done_) cudaEventDestroy(c_kernel_done_);
  if (c_stream_) cudaStreamDestroy(c_stream_);
  if (c_copy_) cudaStreamDestroy(c_copy_);
  c_kernel_done_ = nullptr;
  c_stream_ = c_copy_ = nullptr;
  cudaFree(d_c_llr_);
  cudaFree(d_c_hard_);
  cudaFree(d_c_iters_);
  cudaFree(d_c_crc_);
  cudaFree(d_c_done_);
  cudaFree(d_c_smbusy_);
  cudaFree(d_c_ctl_);
  cudaFree(d_c_tabs_);
  cudaFree(d_c_stage_);
  d_c_llr_ = nullptr;
  d_c_hard_ = nullptr;
  d_c_iters_ = nullptr;
  d_c_crc_ = nullptr;
  d_c_done_ = nullptr;
  d_c_smbusy_ = nullptr;
  d_c_ctl_ = nullptr;
  d_c_tabs_ = nullptr;
  d_c_stage_ = nullptr;
  for (void* p : {(void*)h_ring_, (void*)h_recs_, (void*)h_outs_, (void*)h_tail_, (void*)h_stop_, (void*)h_bits_,
                  (void*)h_slots_})
    if (p) cudaFreeHost(p);
  h_ring_ = nullptr;
  h_recs_ = nullptr;
  h_outs_ = nullptr;
  h_tail_ = nullptr;
  h_stop_ = nullptr;
  h_bits_ = nullptr;
  h_slots_ = nullptr;
}

// Moves queued transmissions into flights while every resource they need is free:
// retransmissions first, then new transport blocks while their accumulators fit.
bool ServeEngine::admit_cont() {
  std::vector<int> stage;  // flights that copy host LLRs
  const size_t before = c_unpub_.size();
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (!fatal_.empty()) return false;
    auto admit = [&](std::deque<Pending>& q, bool need_harq) {
      while (!q.empty()) {
        const Pending pd = q.front();
        Tb& t = tbs_[pd.id];
        const TbParams& p = t.p;
        if (c_free_tx_.empty()) return;
        const long long stage_n = pd.on_device ? 0 : (long long)p.c * t.e;
        if ((long long)c_free_cb_.size() < p.c) return;
        const long long bits = c_bits_alloc_.alloc((t.tb_size + 31) / 32);
        if (bits < 0) return;
        long long st = -1;
        if (stage_n > 0 && (st = c_stage_alloc_.alloc(stage_n)) < 0) {
          c_bits_alloc_.release(bits);
          return;
        }
        if (need_harq && t.harq_off < 0) {
          t.harq_off = harq_alloc((long long)p.c * p.ncb * 4);
          if (t.harq_off < 0) {  // HBM budget full: wait for accumulators to free
            c_bits_alloc_.release(bits);
            if (st >= 0) c_stage_alloc_.release(st);
            return;
          }
          t.tx_count = 0;
        }
        const int tx = c_free_tx_.back();
        c_free_tx_.pop_back();
        Flight& f = c_fl_[tx];
        f = Flight();
        f.pd = pd;
        f.tx = tx;
        int* slots = h_slots_ + (long long)f.tx * kServeMaxCbs;
        for (int i = 0; i < p.c; ++i) {
          slots[i] = c_free_cb_.back();
          c_free_cb_.pop_back();
        }
        f.n_cb = p.c;
        f.bits_off = bits;
        f.stage_off = st;
        f.seq = ++c_seq_ == 0 ? ++c_seq_ : c_seq_;
        // the record (the slot is free: its previous result has been taken)
        const RmWalk w = rm_walk(p.bg, p.z, pd.rv, p.n_filler);
        ServeTxRec& r = h_recs_[f.tx];
        r.acc = reinterpret_cast<float*>(d_harq_ + t.harq_off);
        r.e = st >= 0 ? d_c_stage_ + st : pd.llr;
        r.bits = d_bits_map_ + bits;
        r.tb_size = t.tb_size;
        r.b = p.b;
        r.ncb = w.ncb;
        r.fs = w.fs;
        r.fe = w.fe;
        r.m = w.m;
        r.c0 = w.c0 % w.m;
        r.e_len = (int)t.e;
        r.qm = t.qm;
        r.first = t.tx_count == 0 ? 1 : 0;
        r.bg = p.bg;
        r.z = p.z;
        r.zi = lift_index_of(p.z);
        r.n_filler = p.n_filler;
        r.k_prime = p.k_prime;
        r.has_cb_crc = p.has_cb_crc ? 1 : 0;
        r.n_cb = p.c;
        r.payload = p.payload;
        r.pad = 0;
        r.x_payload = crc24_xpow_host(p.payload, kCrc24A);
        r.x_last = crc24_xpow_host(
            std::max<long long>(0, std::min<long long>(p.payload, p.b - (long long)(p.c - 1) * p.payload)), kCrc24A);
        r.seq = f.seq;
        pending_cbs_ -= p.c;
        stats_.code_blocks += p.c;
        stats_.transmissions += 1;
        q.pop_front();
        if (stage_n > 0) stage.push_back(tx);
        c_unpub_.push_back(tx);
      }
    };
    admit(pending_retx_, false);
    admit(pending_new_, true);
    inflight_ = (int)(c_unpub_.size() + c_pub_.size());
  }
  for (int tx : stage) {  // host LLRs: copy, published once the copy has finished
    Flight& f = c_fl_[tx];
    if (c_events_.empty()) {
      cudaEvent_t e = nullptr;
      cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      c_events_.push_back(e);
    }
    f.staged = c_events_.back();
    c_events_.pop_back();
    const Tb* t;
    {
      std::lock_guard<std::mutex> lk(mu_);
      t = &tbs_[f.pd.id];
    }
    cudaMemcpyAsync(d_c_stage_ + f.stage_off, f.pd.llr, sizeof(float) * (size_t)t->p.c * t->e, cudaMemcpyHostToDevice,
                    c_copy_);
    cudaEventRecord(f.staged, c_copy_);
  }
  return c_unpub_.size() > before;
}

// Writes the work items of admitted flights whose inputs are on the device into the
// ring and advances the tail.
bool ServeEngine::publish_cont() {
  unsigned long long tail = c_tail_;
  long long items = 0, threads = 0;
  const auto now = std::chrono::steady_clock::now();
  size_t kept = 0;  // flights still waiting for their staged LLRs stay, in order
  for (size_t i = 0; i < c_unpub_.size(); ++i) {
    Flight& f = c_fl_[c_unpub_[i]];
    if (f.staged) {
      const cudaError_t q = cudaEventQuery(f.staged);
      if (q == cudaErrorNotReady) {
        c_unpub_[kept++] = f.tx;
        continue;
      }
      c_events_.push_back(f.staged);
      f.staged = nullptr;
    }
    const ServeTxRec& r = h_recs_[f.tx];
    int cap = std::min(kServeMaxItemCbs, pair_mixed_capacity(r.bg, r.z));
    const int hint = tiles_[r.bg][r.z].load(std::memory_order_relaxed);
    if (hint > 0) cap = std::min(cap, hint);
    for (int c = 0; c < f.n_cb; c += cap) {
      ServeJob& j = h_ring_[tail % (unsigned long long)c_cbs_];
      j.tx = f.tx;
      j.first_cb = c;
      j.count = std::min(cap, f.n_cb - c);
      j.pad = 0;
      ++tail;
      items += 1;
      threads += (long long)((j.count + 1) / 2) * r.z;
    }
    f.published = true;
    f.t_pub = now;
    c_pub_pos_[f.tx] = (int)c_pub_.size();
    c_pub_.push_back(f.tx);
  }
  c_unpub_.resize(kept);
  if (tail == c_tail_) return false;
  {
    std::lock_guard<std::mutex> lk(mu_);
    stats_.items += items;
    stats_.item_threads += threads;
  }
  c_tail_ = tail;
  std::atomic_thread_fence(std::memory_order_release);
  reinterpret_cast<std::atomic<unsigned long long>*>(h_tail_)->store(tail, std::memory_order_release);
  return true;
}

// Takes the results of flights whose completion flag is set.
bool ServeEngine::complete_cont() {
  std::vector<int>& done = c_done_scratch_;
  done.clear();
  for (int tx : c_pub_)
    if (reinterpret_cast<std::atomic<uint32_t>*>(&h_outs_[tx].flag)->load(std::memory_order_acquire) == c_fl_[tx].seq)
      done.push_back(tx);
  if (done.empty()) return false;
  const auto now = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lk(mu_);
    for (int tx : done) {
      Flight& f = c_fl_[tx];
      const int32_t* r = h_outs_[tx].result;
      Tb& t = tbs_[f.pd.id];
      t.tx_count += 1;
      ServeResult res;
      res.id = f.pd.id;
      res.crc_ok = r[0];
      res.max_iters = r[1];
      res.harq_tx = t.tx_count;
      res.n_cb = t.p.c;
      for (int w = 0; w < 5; ++w) res.cb_crc[w] = (uint32_t)r[2 + w];
      res.latency_us = std::chrono::duration<double, std::micro>(now - f.pd.t0).count();
      res.queue_us = std::chrono::duration<double, std::micro>(f.t_pub - f.pd.t0).count();
      res.step_us = std::chrono::duration<double, std::micro>(now - f.t_pub).count();
      const long long nw = (t.tb_size + 31) / 32;
      t.bits.assign(h_bits_ + f.bits_off, h_bits_ + f.bits_off + nw);
      if (res.crc_ok) {  // DlSchDecoder flushes the HARQ buffers on success
        harq_free(t.harq_off);
        t.harq_off = -1;
        t.tx_count = 0;
      }
      t.busy = false;
      push_done(res);
      stats_.step_ms += res.step_us * 1e-3;
      const int* slots = h_slots_ + (long long)tx * kServeMaxCbs;
      for (int i = 0; i < f.n_cb; ++i) c_free_cb_.push_back(slots[i]);
      c_bits_alloc_.release(f.bits_off);
      if (f.stage_off >= 0) c_stage_alloc_.release(f.stage_off);
      c_free_tx_.push_back(tx);
      // out of the published list: the last entry takes its place
      const int pos = c_pub_pos_[tx], back = c_pub_.back();
      c_pub_[pos] = back;
      c_pub_pos_[back] = pos;
      c_pub_.pop_back();
      c_pub_pos_[tx] = -1;
    }
    inflight_ = (int)(c_unpub_.size() + c_pub_.size());
  }
  cv_done_.notify_all();
  return true;
}

// After a kernel failure: every flight and queued transmission ends with crc_ok = 0.
void ServeEngine::fail_all_cont() {
  std::lock_guard<std::mutex> lk(mu_);
  for (const std::vector<int>* list : {&c_unpub_, &c_pub_})
    for (int tx : *list) {
      Flight& f = c_fl_[tx];
      ServeResult res;
      res.id = f.pd.id;
      tbs_[res.id].busy = false;
      push_done(res);
      if (f.staged) c_events_.push_back(f.staged);
      f.staged = nullptr;
      c_pub_pos_[tx] = -1;
    }
  c_unpub_.clear();
  c_pub_.clear();
  for (std::deque<Pending>* q : {&pending_retx_, &pending_new_})
    while (!q->empty()) {
      ServeResult res;
      res.id = q->front().id;
      tbs_[res.id].busy = false;
      q->pop_front();
      push_done(res);
    }
  pending_cbs_ = 0;
  inflight_ = 0;
  cv_done_.notify_all();
}

void ServeEngine::worker_cont() {
  cudaSetDevice(device_);
  using clk = std::chrono::steady_clock;
  auto ns = [](clk::time_point a, clk::time_point b) {
    return (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(b - a).count();
  };
  auto last_busy = clk::now();
  for (;;) {
    const auto t0 = clk::now();
    bool progressed = complete_cont();
    const auto t1 = clk::now();
    progressed |= admit_cont();
    const auto t2 = clk::now();
    progressed |= publish_cont();
    const auto t3 = clk::now();
    c_loops_.fetch_add(1, std::memory_order_relaxed);
    c_complete_ns_.fetch_add(ns(t0, t1), std::memory_order_relaxed);
    c_admit_ns_.fetch_add(ns(t1, t2), std::memory_order_relaxed);
    c_publish_ns_.fetch_add(ns(t2, t3), std::memory_order_relaxed);
    const bool waiting = !c_pub_.empty();  // published items whose results are outstanding
    if (c_running_) {
      const cudaError_t q = cudaEventQuery(c_kernel_done_);
      if (q == cudaSuccess) {
        c_running_ = false;
      } else if (q != cudaErrorNotReady) {
        std::lock_guard<std::mutex> lk(mu_);
        fatal_ = std::string("serving kernel failed: ") + cudaGetErrorString(q);
      }
    }
    if (waiting && !c_running_ && fatal_.empty()) {
      const auto h0 = std::chrono::steady_clock::now();
      c_args_.epoch = ++c_epoch_ == 0 ? ++c_epoch_ : c_epoch_;
      cudaError_t e = serve_cont_launch(c_args_, sms_, c_stream_);
      if (e == cudaSuccess) e = cudaEventRecord(c_kernel_done_, c_stream_);
      std::lock_guard<std::mutex> lk(mu_);
      if (e != cudaSuccess)
        fatal_ = std::string("serving kernel launch failed: ") + cudaGetErrorString(e);
      else
        c_running_ = true;
      stats_.steps += 1;
      stats_.host_launch_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
    }
    {
      std::unique_lock<std::mutex> lk(mu_);
      if (stop_) break;
      if (!fatal_.empty()) {
        lk.unlock();
        fail_all_cont();
        lk.lock();
        if (stop_) break;
      }
      if (c_unpub_.empty() && c_pub_.empty() && pending_retx_.empty() && pending_new_.empty()) {
        // idle: watch the queues for a while before sleeping (a woken thread takes tens
        // of microseconds; the next transmission, often a retransmission, is near)
        if (clk::now() - last_busy < std::chrono::microseconds(kPollSpinUs)) {
          lk.unlock();
          std::this_thread::yield();
          continue;
        }
        cv_work_.wait_for(lk, std::chrono::milliseconds(5));
        continue;
      }
      last_busy = clk::now();
    }
    if (!progressed) std::this_thread::yield();
  }
}

ServeCoreStats ServeEngine::core_stats() {
  ServeCoreStats r;
  if (!cont_ || !d_c_ctl_) return r;
  ServeCtl c{};
  cudaSetDevice(device_);
  if (cudaMemcpyAsync(&c, d_c_ctl_, sizeof(c), cudaMemcpyDeviceToHost, c_copy_) != cudaSuccess ||
      cudaStreamSynchronize(c_copy_) != cudaSuccess)
    return r;
  r.items = (long long)c.items;
  r.busy_us = c.busy_ns * 1e-3;
  r.combine_us = c.combine_ns * 1e-3;
  r.decode_us = c.decode_ns * 1e-3;
  r.crc_us = c.crc_ns * 1e-3;
  r.finish_us = c.finish_ns * 1e-3;
  r.loops = c_loops_.load();
  r.admit_us = c_admit_ns_.load() * 1e-3;
  r.publish_us = c_publish_ns_.load() * 1e-3;
  r.complete_us = c_complete_ns_.load() * 1e-3;
  return r;
}

}  // namespace syn
