// Transport-block serving engine (see serve.h).
//
// Continuous batching: a worker thread turns the queue of submitted transmissions
// into GPU steps while earlier steps are still running (up to cfg.slots in flight,
// each with its own stream and buffers).  A step admits transmissions in arrival
// order while they fit its code-block budget and, for a transport block seen for the
// first time, while its HARQ accumulators fit the HBM budget; a new block that does
// not fit waits, and so do the new blocks behind it, while retransmissions of blocks
// that already hold accumulators (kept in their own queue) go first.  A step runs, on
// its stream:
//   1. serve_combine_kernel: HARQ soft combining into the device-resident
//      accumulators and quantization to int8 decoder input,
//   2. the persistent mixed-shape 5G NR decode (one work queue over every code block
//      of every transport block in the step),
//   3. code-block CRCs and 4. transport-block CRC, report and desegmented bits,
//   5. one copy of the reports and bits to pinned host memory.
// When the step's event completes, each transport block whose CRCs pass frees its
// accumulators (transport_block.rs:1041-1047 flushes them); a failed one keeps them
// for its retransmission.  Semantics per transmission are those of
// DlSchDecoder::decode (transport_block.rs:829-1053) with the int8 code-block decode.
#include "serve.h"

#include <algorithm>
#include <cstring>

#include "../../include/syndrome_ldpc.h"
#include "channel.h"
#include "graph.h"

namespace syn {

namespace {

constexpr int kResWords = 7;  // crc_ok, max_iters, 5 words of per-block CRC bits
constexpr int kMaxCbPerTb = 160;

const int kLiftingSizes[kMixLiftSizes] = {2,  3,  4,  5,  6,  7,   8,   9,   10,  11,  12,  13,  14,
                                          15, 16, 18, 20, 22, 24,  26,  28,  30,  32,  36,  40,  44,
                                          48, 52, 56, 60, 64, 72,  80,  88,  96,  104, 112, 120, 128,
                                          144, 160, 176, 192, 208, 224, 240, 256, 288, 320, 352, 384};

int lift_index(int z) {
  for (int i = 0; i < kMixLiftSizes; ++i)
    if (kLiftingSizes[i] == z) return i;
  return -1;
}

long long al256(long long x) { return (x + 255) & ~255LL; }

}  // namespace

ServeEngine::~ServeEngine() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_work_.notify_all();
  if (thread_.joinable()) thread_.join();
  cudaSetDevice(device_);
  release_cont();
  for (Slot& s : slots_) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    cudaFree(s.d_llr);
    cudaFree(s.d_hard);
    cudaFree(s.d_iters);
    cudaFree(s.d_cbs);
    cudaFree(s.d_crc);
    cudaFree(s.d_tbs);
    cudaFree(s.d_res);
    cudaFree(s.d_bits);
    cudaFree(s.d_items);
    cudaFree(s.d_cws);
    cudaFree(s.d_queue);
    cudaFree(s.d_stage);
    cudaFreeHost(s.h_cbs);
    cudaFreeHost(s.h_tbs);
    cudaFreeHost(s.h_items);
    cudaFreeHost(s.h_cws);
    cudaFreeHost(s.h_res);
    cudaFreeHost(s.h_bits);
    if (s.done) cudaEventDestroy(s.done);
    if (s.t0) cudaEventDestroy(s.t0);
    if (s.ts) cudaEventDestroy(s.ts);
    if (s.t1) cudaEventDestroy(s.t1);
    if (s.stream) cudaStreamDestroy(s.stream);
  }
  cudaFree(d_harq_);
  cudaFree(d_shift_);
  cudaFree(d_colz_);
}

bool ServeEngine::init(const ServeConfig& cfg, std::string* err) {
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return false;
  };
  cfg_ = cfg;
  if (cfg_.max_step_cbs < kMaxCbPerTb) cfg_.max_step_cbs = kMaxCbPerTb;
  if (cfg_.max_step_cbs > 65535) return fail("max_step_cbs above 65535");
  cfg_.slots = std::max(1, std::min(cfg_.slots, 16));
  cfg_.latency_slots = std::max(1, std::min(cfg_.latency_slots, cfg_.slots));
  if (cfg_.backlog_cbs <= 0) cfg_.backlog_cbs = 128;
  if (cfg_.harq_bytes <= 0 || cfg_.staging_bytes < 0) return fail("negative memory budget");
  if (cfg_.mode != 0 && cfg_.mode != 1) return fail("mode must be 0 (continuous) or 1 (steps)");
  if (cfg_.idle_us < 10 || cfg_.idle_us > 1000000) return fail("idle_us must be in [10, 1e6]");
  if (cfg_.iterations < 0) return fail("iterations must be non-negative");
  if (cfg_.app_clamp < 255) return fail("app_clamp below 255 is not supported by the serving decoder");
  beta_q_ = syn::beta_q(cfg_.beta, cfg_.scale);
  if (cudaGetDevice(&device_) != cudaSuccess) return fail("no CUDA device");
  cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_);
  paired_ = cfg_.app_clamp >= 7874;
  tmem_ = paired_ && cfg_.decode_kernel != 5;  // code blocks report their K' <= K bits
  if ((paired_ ? pair_mixed_prepare() : mixed_kernel_prepare()) != cudaSuccess ||
      (tmem_ && pair_tm_mixed_prepare() != cudaSuccess))
    return fail("cannot configure the decode kernel");
  // shift and column-base tables of every 5G NR shape
  std::vector<short> shift((size_t)2 * kMixLiftSizes * kMixEdges, 0);
  std::vector<int> colz((size_t)2 * kMixLiftSizes * kMixEdges, 0);
  for (int bg = 0; bg < 2; ++bg)
    for (int zi = 0; zi < kMixLiftSizes; ++zi) {
      Graph g;
      if (!build_nr_graph(bg, kLiftingSizes[zi], &g) || !nr_layout_matches(bg, g.cols.data(), g.edges()))
        return fail("internal: base graph layout mismatch");
      short* sh = &shift[((size_t)bg * kMixLiftSizes + zi) * kMixEdges];
      for (int e = 0; e < g.edges(); ++e) sh[e] = (short)g.shifts[e];
      mixed_column_bases(bg, kLiftingSizes[zi], &colz[((size_t)bg * kMixLiftSizes + zi) * kMixEdges]);
    }
  const int M = cfg_.max_step_cbs;
  max_words_ = (8448 + 31) / 32;
  max_tb_words_ = M * max_words_ + M;
  bool ok = cudaMalloc(&d_shift_, sizeof(short) * shift.size()) == cudaSuccess &&
            cudaMalloc(&d_colz_, sizeof(int) * colz.size()) == cudaSuccess &&
            cudaMalloc(&d_harq_, (size_t)cfg_.harq_bytes) == cudaSuccess;
  if (ok) {
    ok = cudaMemcpy(d_shift_, shift.data(), sizeof(short) * shift.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(d_colz_, colz.data(), sizeof(int) * colz.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  harq_.reset(cfg_.harq_bytes & ~255LL);
  cont_ = tmem_ && cfg_.mode == 0;
  if (cont_) {
    if (!ok || !init_cont(err)) {
      cudaGetLastError();
      if (!ok) return fail("allocating the serving buffers failed (HBM budget too large?)");
      return false;
    }
    thread_ = std::thread([this] { worker_cont(); });
    return true;
  }
  slots_.resize(cfg_.slots);
  for (Slot& s : slots_) {
    if (!ok) break;
    ok = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreate(&s.done) == cudaSuccess && cudaEventCreate(&s.ts) == cudaSuccess &&
         cudaEventCreate(&s.t0) == cudaSuccess && cudaEventCreate(&s.t1) == cudaSuccess &&
         cudaMalloc(&s.d_llr, (size_t)M * 25344) == cudaSuccess &&
         cudaMalloc(&s.d_hard, sizeof(uint32_t) * (size_t)M * max_words_) == cudaSuccess &&
         cudaMalloc(&s.d_iters, sizeof(int32_t) * M) == cudaSuccess &&
         cudaMalloc(&s.d_cbs, sizeof(ServeCb) * M) == cudaSuccess &&
         cudaMalloc(&s.d_crc, sizeof(ServeCbCrc) * M) == cudaSuccess &&
         cudaMalloc(&s.d_tbs, sizeof(ServeTb) * M) == cudaSuccess &&
         cudaMalloc(&s.d_res, sizeof(int32_t) * kResWords * M) == cudaSuccess &&
         cudaMalloc(&s.d_bits, sizeof(uint32_t) * (size_t)max_tb_words_) == cudaSuccess &&
         cudaMalloc(&s.d_items, sizeof(MixItem) * M) == cudaSuccess &&
         cudaMalloc(&s.d_cws, sizeof(MixCodeword) * M) == cudaSuccess &&
         cudaMalloc(&s.d_queue, sizeof(unsigned)) == cudaSuccess &&
         (cfg_.staging_bytes == 0 || cudaMalloc(&s.d_stage, (size_t)cfg_.staging_bytes) == cudaSuccess) &&
         cudaMallocHost(&s.h_cbs, sizeof(ServeCb) * M) == cudaSuccess &&
         cudaMallocHost(&s.h_tbs, sizeof(ServeTb) * M) == cudaSuccess &&
         cudaMallocHost(&s.h_items, sizeof(MixItem) * M) == cudaSuccess &&
         cudaMallocHost(&s.h_cws, sizeof(MixCodeword) * M) == cudaSuccess &&
         cudaMallocHost(&s.h_res, sizeof(int32_t) * kResWords * M) == cudaSuccess &&
         cudaMallocHost(&s.h_bits, sizeof(uint32_t) * (size_t)max_tb_words_) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    return fail("allocating the serving buffers failed (HBM budget too large?)");
  }
  thread_ = std::thread([this] { worker(); });
  return true;
}

long long RangeAlloc::alloc(long long n) {
  if (n <= 0) return -1;
  auto b = by_len_.lower_bound(n);  // the shortest free range that holds n
  if (b == by_len_.end()) return -1;
  const long long off = b->second, len = b->first;
  by_len_.erase(b);
  free_.erase(off);
  if (len > n) add(off + n, len - n);
  used_[off] = n;
  used += n;
  return off;
}

void RangeAlloc::release(long long off) {
  auto u = used_.find(off);
  if (u == used_.end()) return;
  long long size = u->second;
  used_.erase(u);
  used -= size;
  auto next = free_.lower_bound(off);
  if (next != free_.end() && off + size == next->first) {
    size += next->second;
    drop(next);
  }
  auto it = free_.lower_bound(off);
  if (it != free_.begin()) {
    auto prev = std::prev(it);
    if (prev->first + prev->second == off) {
      const long long start = prev->first;
      size += prev->second;
      drop(prev);
      add(start, size);
      return;
    }
  }
  add(off, size);
}

long long ServeEngine::harq_alloc(long long bytes) { return harq_.alloc(al256(bytes)); }

void ServeEngine::harq_free(long long off) { harq_.release(off); }

int ServeEngine::submit(uint64_t id, long long tb_size, float rate, int qm, long long g, int rv, const float* llr,
                        long long llr_len, bool on_device, std::string* err) {
  auto fail = [&](int code, const std::string& m) {
    if (err) *err = m;
    return code;
  };
  if (!llr) return fail(SYNDROME_NULL_POINTER, "llr is null");
  if (rv < 0 || rv > 3) return fail(SYNDROME_INVALID_PARAM, "RV must be 0..=3");
  if (tb_size <= 0 || qm <= 0 || qm > 16 || g <= 0 || g % qm)
    return fail(SYNDROME_INVALID_PARAM, "Qm and G must be positive; G % Qm must be 0");
  std::unique_lock<std::mutex> lk(mu_);
  if (!fatal_.empty()) return fail(SYNDROME_CUDA_ERROR, fatal_);
  auto it = tbs_.find(id);
  if (it == tbs_.end()) {
    Tb t;
    std::string e2;
    if (!compute_segmentation(tb_size, rate, &t.p, &e2)) return fail(SYNDROME_INVALID_PARAM, e2);
    t.e = (g / t.p.c / qm) * qm;
    if (t.e <= 0) return fail(SYNDROME_INVALID_PARAM, "G too small: no bits per code block");
    for (int r = 0; r < 4; ++r)
      if (!rm_walk_covers(rm_walk(t.p.bg, t.p.z, r, t.p.n_filler), t.e) || t.e > 8LL * t.p.ncb)
        return fail(SYNDROME_INVALID_PARAM, "E per code block exceeds the rate-matching walk");
    if (t.p.c > kMaxCbPerTb) return fail(SYNDROME_INVALID_PARAM, "too many code blocks");
    if (!on_device && (long long)t.p.c * t.e * 4 > cfg_.staging_bytes)
      return fail(SYNDROME_INVALID_PARAM, "host LLRs larger than the staging buffer");
    if (al256((long long)t.p.c * t.p.ncb * 4) > cfg_.harq_bytes)
      return fail(SYNDROME_INVALID_PARAM, "HARQ accumulators larger than the HBM budget");
    t.tb_size = tb_size;
    t.g = g;
    t.rate = rate;
    t.qm = qm;
    it = tbs_.emplace(id, std::move(t)).first;
  } else {
    const Tb& t = it->second;
    if (t.tb_size != tb_size || t.g != g || t.qm != qm || t.rate != rate)
      return fail(SYNDROME_INVALID_PARAM, "transport block id reused with different parameters");
    if (t.busy) return fail(SYNDROME_INVALID_PARAM, "a transmission of this transport block is still in flight");
  }
  Tb& t = it->second;
  if (llr_len < (long long)t.p.c * t.e) return fail(SYNDROME_BUFFER_TOO_SMALL, "llr shorter than C * E");
  t.busy = true;
  const Pending pd{id, rv, llr, on_device, std::chrono::steady_clock::now()};
  if (t.harq_off >= 0)
    pending_retx_.push_back(pd);
  else
    pending_new_.push_back(pd);
  pending_cbs_ += t.p.c;
  stats_.max_pending =
      std::max<long long>(stats_.max_pending, (long long)(pending_retx_.size() + pending_new_.size()));
  lk.unlock();
  cv_work_.notify_one();
  return SYNDROME_OK;
}

bool ServeEngine::launch_step(Slot& s) {
  const auto h0 = std::chrono::steady_clock::now();
  // --- admission (under the lock) and step layout
  s.txs.clear();
  s.bits_off.clear();
  std::vector<const Tb*> tbv;
  std::vector<int> first_tx;
  long long stage_used = 0;
  int n_cbs = 0;
  {
    // Retransmissions first (their blocks hold accumulators, and a new block may be
    // waiting for exactly those to be freed), then new blocks in arrival order while
    // their accumulators fit the HBM budget.
    std::lock_guard<std::mutex> lk(mu_);
    auto admit = [&](std::deque<Pending>& q, bool need_harq) {
      while (!q.empty()) {
        const Pending pd = q.front();
        Tb& t = tbs_[pd.id];
        if (n_cbs > 0 && n_cbs + t.p.c > cfg_.max_step_cbs) return;
        const long long need_stage = pd.on_device ? 0 : (long long)t.p.c * t.e * 4;
        if (need_stage && stage_used + need_stage > cfg_.staging_bytes) return;
        if (need_harq && t.harq_off < 0) {
          t.harq_off = harq_alloc((long long)t.p.c * t.p.ncb * 4);
          if (t.harq_off < 0) return;  // HBM budget full: wait for accumulators to free
          t.tx_count = 0;
        }
        stage_used += need_stage;
        n_cbs += t.p.c;
        s.txs.push_back(pd);
        tbv.push_back(&t);
        first_tx.push_back(t.tx_count == 0 ? 1 : 0);
        pending_cbs_ -= t.p.c;
        q.pop_front();
      }
    };
    admit(pending_retx_, false);
    admit(pending_new_, true);
  }
  if (s.txs.empty()) return false;
  s.launched = std::chrono::steady_clock::now();
  cudaEventRecord(s.ts, s.stream);
  // --- descriptors (Tb records are stable while busy)
  std::map<std::pair<int, int>, std::vector<int>> shapes;
  long long llr_off = 0, hard_off = 0, bits_off = 0, stage_off = 0;
  int c_idx = 0;
  for (size_t j = 0; j < s.txs.size(); ++j) {
    const Tb& t = *tbv[j];
    const TbParams& p = t.p;
    const float* e_src = s.txs[j].llr;
    if (!s.txs[j].on_device) {
      cudaMemcpyAsync(s.d_stage + stage_off / 4, e_src, (size_t)p.c * t.e * 4, cudaMemcpyHostToDevice, s.stream);
      e_src = s.d_stage + stage_off / 4;
      stage_off += (long long)p.c * t.e * 4;
    }
    const RmWalk w = rm_walk(p.bg, p.z, s.txs[j].rv, p.n_filler);
    ServeTb& tb = s.h_tbs[j];
    tb.first_cb = c_idx;
    tb.n_cb = p.c;
    tb.payload = p.payload;
    tb.has_cb_crc = p.has_cb_crc ? 1 : 0;
    tb.tb_size = t.tb_size;
    tb.x_payload = crc24_xpow_host(p.payload, kCrc24A);
    tb.x_last = crc24_xpow_host(std::max<long long>(0, std::min<long long>(p.payload, p.b - (long long)(p.c - 1) * p.payload)),
                                kCrc24A);
    tb.tb_bits = s.d_bits + bits_off;
    tb.result = s.d_res + kResWords * j;
    s.bits_off.push_back(bits_off);
    bits_off += (t.tb_size + 31) / 32;
    const int words = (p.k_prime + 31) / 32;
    for (int ci = 0; ci < p.c; ++ci, ++c_idx) {
      ServeCb& cb = s.h_cbs[c_idx];
      cb.acc = reinterpret_cast<float*>(d_harq_ + t.harq_off) + (long long)ci * p.ncb;
      cb.e = e_src + (long long)ci * t.e;
      cb.llr = s.d_llr + llr_off;
      cb.hard = s.d_hard + hard_off;
      cb.hard_words = words;
      cb.ncb = w.ncb;
      cb.fs = w.fs;
      cb.fe = w.fe;
      cb.m = w.m;
      cb.c0 = w.c0;
      cb.e_len = (int)t.e;
      cb.qm = t.qm;
      cb.first = first_tx[j];
      cb.k_prime = p.has_cb_crc ? p.k_prime : 0;
      cb.crc_len = (int)std::max<long long>(0, std::min<long long>(p.payload, p.b - (long long)ci * p.payload));
      cb.tb = (int)j;
      MixCodeword& mc = s.h_cws[c_idx];
      mc.llr_off = llr_off;
      mc.out_off = hard_off;
      mc.n_filler = p.n_filler;
      mc.hard_bits = p.k_prime;
      mc.index = c_idx;
      mc.pad = 0;
      shapes[{p.bg, p.z}].push_back(c_idx);
      llr_off += p.ncb;
      hard_off += words;
    }
  }
  s.n_cbs = n_cbs;
  // work items: same-shape tiles, longest first
  std::vector<MixItem> items;
  std::vector<MixCodeword> ordered;
  ordered.reserve(n_cbs);
  for (auto& kv : shapes) {
    const int bg = kv.first.first, z = kv.first.second;
    int cap = paired_ ? pair_mixed_capacity(bg, z) : mixed_slot_capacity(bg, z);
    const int hint = (bg == 0 || bg == 1) && z >= 1 && z <= 384 ? tiles_[bg][z].load(std::memory_order_relaxed) : 0;
    if (hint > 0) cap = std::min(cap, hint);  // tuned item size (autotune.py)
    const std::vector<int>& idx = kv.second;
    for (size_t a = 0; a < idx.size(); a += cap) {
      MixItem m{};
      m.bg = bg;
      m.z = z;
      m.zi = lift_index(z);
      m.count = (int)std::min<size_t>(cap, idx.size() - a);
      m.first = (int)ordered.size();
      for (int q = 0; q < m.count; ++q) ordered.push_back(s.h_cws[idx[a + q]]);
      items.push_back(m);
    }
  }
  auto cost = [](const MixItem& m) { return (long long)(m.bg == 0 ? 316 : 197) * m.z * m.count; };
  std::stable_sort(items.begin(), items.end(), [&](const MixItem& a, const MixItem& b) { return cost(a) > cost(b); });
  std::copy(ordered.begin(), ordered.end(), s.h_cws);
  std::copy(items.begin(), items.end(), s.h_items);
  cudaStream_t st = s.stream;
  const int n_tb = (int)s.txs.size();
  cudaMemcpyAsync(s.d_cbs, s.h_cbs, sizeof(ServeCb) * n_cbs, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.d_tbs, s.h_tbs, sizeof(ServeTb) * n_tb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.d_cws, s.h_cws, sizeof(MixCodeword) * n_cbs, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.d_items, s.h_items, sizeof(MixItem) * items.size(), cudaMemcpyHostToDevice, st);
  int max_ncb = 0;
  for (int i = 0; i < n_cbs; ++i) max_ncb = std::max(max_ncb, s.h_cbs[i].ncb);
  cudaError_t e = serve_combine_launch(s.d_cbs, n_cbs, max_ncb, cfg_.scale, st);
  MixArgs m{};
  m.items = s.d_items;
  m.n_items = (int)items.size();
  m.cws = s.d_cws;
  m.llr = s.d_llr;
  m.out = s.d_hard;
  m.iters = s.d_iters;
  m.shift_tab = d_shift_;
  m.colz_tab = d_colz_;
  m.queue = s.d_queue;
  m.beta_q = beta_q_;
  m.app_clamp = cfg_.app_clamp;
  m.iterations = cfg_.iterations;
  m.k32 = 32;
  m.two = 2;
  if (e == cudaSuccess) e = cudaEventRecord(s.t0, st);
  if (e == cudaSuccess)
    e = tmem_ ? pair_tm_mixed_launch(m, sms_, st)
              : (paired_ ? pair_mixed_launch(m, sms_, st) : mixed_decode_launch(m, sms_, st));
  if (e == cudaSuccess) e = cudaEventRecord(s.t1, st);
  if (e == cudaSuccess) e = serve_cb_crc_launch(s.d_cbs, n_cbs, s.d_crc, st);
  if (e == cudaSuccess) e = serve_tb_finish_launch(s.d_tbs, n_tb, s.d_cbs, s.d_crc, s.d_iters, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.h_res, s.d_res, sizeof(int32_t) * kResWords * n_tb, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.h_bits, s.d_bits, sizeof(uint32_t) * bits_off, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaEventRecord(s.done, st);
  if (e != cudaSuccess) {
    std::lock_guard<std::mutex> lk(mu_);
    fatal_ = std::string("serving step launch failed: ") + cudaGetErrorString(e);
  }
  long long threads = 0;
  for (const MixItem& it : items) threads += (long long)(paired_ ? (it.count + 1) / 2 : it.count) * it.z;
  std::lock_guard<std::mutex> lk(mu_);
  stats_.steps += 1;
  stats_.code_blocks += n_cbs;
  stats_.transmissions += n_tb;
  stats_.items += (long long)items.size();
  stats_.item_threads += threads;
  stats_.host_launch_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
  return true;
}

void ServeEngine::finish_step(Slot& s) {
  const auto now = std::chrono::steady_clock::now();
  float ms = 0.0f, span = 0.0f;
  cudaEventElapsedTime(&ms, s.t0, s.t1);
  cudaEventElapsedTime(&span, s.ts, s.done);
  std::lock_guard<std::mutex> lk(mu_);
  stats_.decode_ms += ms;
  stats_.step_ms += span;
  for (size_t j = 0; j < s.txs.size(); ++j) {
    Tb& t = tbs_[s.txs[j].id];
    const int32_t* r = s.h_res + kResWords * j;
    t.tx_count += 1;
    ServeResult res;
    res.id = s.txs[j].id;
    res.crc_ok = fatal_.empty() ? r[0] : 0;
    res.max_iters = r[1];
    res.harq_tx = t.tx_count;
    res.n_cb = t.p.c;
    for (int w = 0; w < 5; ++w) res.cb_crc[w] = (uint32_t)r[2 + w];
    res.latency_us = std::chrono::duration<double, std::micro>(now - s.txs[j].t0).count();
    res.queue_us = std::chrono::duration<double, std::micro>(s.launched - s.txs[j].t0).count();
    res.step_us = 1000.0 * span;
    const long long nw = (t.tb_size + 31) / 32;
    t.bits.assign(s.h_bits + s.bits_off[j], s.h_bits + s.bits_off[j] + nw);
    if (res.crc_ok) {  // DlSchDecoder flushes the HARQ buffers on success
      harq_free(t.harq_off);
      t.harq_off = -1;
      t.tx_count = 0;
    }
    t.busy = false;
    push_done(res);
  }
  s.txs.clear();
  s.busy = false;
  stats_.host_finish_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - now).count();
  cv_done_.notify_all();
}

void ServeEngine::worker() {
  cudaSetDevice(device_);
  for (;;) {
    bool progressed = false;
    // completed steps, whichever finished (a long step does not hold back short ones)
    for (auto it = order_.begin(); it != order_.end();) {
      Slot& s = slots_[*it];
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) {
        ++it;
        continue;
      }
      if (q != cudaSuccess) {
        std::lock_guard<std::mutex> lk(mu_);
        fatal_ = std::string("serving step failed: ") + cudaGetErrorString(q);
      }
      finish_step(s);
      it = order_.erase(it);
      {
        std::lock_guard<std::mutex> lk(mu_);
        inflight_ = (int)order_.size();
      }
      progressed = true;
    }
    {
      std::unique_lock<std::mutex> lk(mu_);
      if (stop_) break;
      if (!fatal_.empty()) {
        // fail every queued transmission
        for (std::deque<Pending>* q : {&pending_retx_, &pending_new_})
          while (!q->empty()) {
            ServeResult res;
            res.id = q->front().id;
            tbs_[res.id].busy = false;
            q->pop_front();
            push_done(res);
          }
        pending_cbs_ = 0;
        cv_done_.notify_all();
      }
      if (order_.empty() && pending_retx_.empty() && pending_new_.empty()) {
        cv_work_.wait_for(lk, std::chrono::milliseconds(5));
        continue;
      }
    }
    // launch into a free slot
    int free_slot = -1;
    for (int i = 0; i < (int)slots_.size(); ++i)
      if (!slots_[i].busy) {
        free_slot = i;
        break;
      }
    if (free_slot >= 0) {
      bool have;
      {
        std::lock_guard<std::mutex> lk(mu_);
        have = (!pending_retx_.empty() || !pending_new_.empty()) && fatal_.empty() &&
               ((int)order_.size() < cfg_.latency_slots || pending_cbs_ >= cfg_.backlog_cbs);
      }
      if (have && launch_step(slots_[free_slot])) {
        slots_[free_slot].busy = true;
        order_.push_back(free_slot);
        std::lock_guard<std::mutex> lk(mu_);
        inflight_ = (int)order_.size();
        progressed = true;
      }
    }
    if (!progressed) std::this_thread::yield();
  }
}

void ServeEngine::push_done(const ServeResult& r) {  // under mu_
  done_.push_back(r);
  done_n_.store((long long)done_.size(), std::memory_order_release);
}

int ServeEngine::poll(ServeResult* out, int cap, long long timeout_us) {
  if (timeout_us > 0 && done_n_.load(std::memory_order_acquire) == 0) {
    // A result is usually a few hundred microseconds away: watch for it for up to
    // kPollSpinUs before sleeping (a thread woken from a condition variable takes tens
    // of microseconds, once per HARQ round trip).
    const auto t0 = std::chrono::steady_clock::now();
    const long long spin = std::min<long long>(timeout_us, kPollSpinUs);
    while (done_n_.load(std::memory_order_acquire) == 0 &&
           std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count() < spin)
      std::this_thread::yield();
    timeout_us -= (long long)std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
  }
  std::unique_lock<std::mutex> lk(mu_);
  if (done_.empty() && timeout_us > 0)
    cv_done_.wait_for(lk, std::chrono::microseconds(timeout_us), [&] { return !done_.empty(); });
  int n = 0;
  while (n < cap && !done_.empty()) {
    out[n++] = done_.front();
    done_.pop_front();
  }
  done_n_.store((long long)done_.size(), std::memory_order_release);
  return n;
}

int ServeEngine::fetch(uint64_t id, uint8_t* bits, long long len, std::string* err) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = tbs_.find(id);
  if (it == tbs_.end()) {
    if (err) *err = "unknown transport block id";
    return SYNDROME_INVALID_PARAM;
  }
  const Tb& t = it->second;
  if (len < t.tb_size) {
    if (err) *err = "output shorter than tb_size";
    return SYNDROME_BUFFER_TOO_SMALL;
  }
  if (t.bits.empty()) {
    if (err) *err = "no completed decode for this transport block";
    return SYNDROME_INVALID_PARAM;
  }
  for (long long i = 0; i < t.tb_size; ++i) bits[i] = (t.bits[i >> 5] >> (i & 31)) & 1u;
  return SYNDROME_OK;
}

int ServeEngine::release(uint64_t id, std::string* err) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = tbs_.find(id);
  if (it == tbs_.end()) return SYNDROME_OK;
  if (it->second.busy) {
    if (err) *err = "a transmission of this transport block is still in flight";
    return SYNDROME_INVALID_PARAM;
  }
  if (it->second.harq_off >= 0) harq_free(it->second.harq_off);
  tbs_.erase(it);
  return SYNDROME_OK;
}

void ServeEngine::set_tile(int bg, int z, int tile) {
  if ((bg == 0 || bg == 1) && z >= 1 && z <= 384) tiles_[bg][z].store(std::max(tile, 0), std::memory_order_relaxed);
}

ServeStats ServeEngine::stats() {
  std::lock_guard<std::mutex> lk(mu_);
  ServeStats s = stats_;
  s.harq_bytes_used = harq_.used;
  s.pending = (long long)(pending_retx_.size() + pending_new_.size());
  s.in_flight = inflight_;
  s.tbs_held = (long long)tbs_.size();
  return s;
}

}  // namespace syn
