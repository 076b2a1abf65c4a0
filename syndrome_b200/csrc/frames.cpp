// DlSchF32 and FramePipe (frames.h).
#include "frames.h"

#include <algorithm>

#include "../../include/syndrome_ldpc.h"
#include "graph.h"

namespace syn {

namespace {

bool cuda_ok(cudaError_t e, const char* what, std::string* err) {
  if (e == cudaSuccess) return true;
  if (err) *err = std::string("CUDA ") + what + ": " + cudaGetErrorString(e);
  return false;
}

uint32_t msb_fold(const uint8_t* bits) {
  uint32_t r = 0;
  for (int i = 0; i < 24; ++i) r = (r << 1) | (bits[i] & 1u);
  return r;
}

}  // namespace

// ------------------------------------------------------------------ DlSchF32 --

DlSchF32::~DlSchF32() {
  if (stream_) cudaStreamSynchronize(stream_);
  cudaFree(d_acc_);
  cudaFree(d_rx_);
  cudaFree(d_cbs_);
  cudaFree(d_hard_);
  cudaFree(d_iters_);
  cudaFree(d_ws_);
  if (stream_) cudaStreamDestroy(stream_);
}

bool DlSchF32::init(long long tb_size, float rate, int qm, long long g, int iterations, float beta,
                    std::string* err) {
  // transport_block.rs:612-627
  if (tb_size <= 0) return (*err = "tb_size must be > 0", false);
  if (qm <= 0 || g <= 0 || g % qm) return (*err = "Qm and G must be positive; G % Qm must be 0", false);
  if (iterations < 0) return (*err = "iterations must be non-negative", false);
  if (!compute_segmentation(tb_size, rate, &p_, err)) return false;
  tb_size_ = tb_size;
  qm_ = qm;
  iterations_ = iterations;
  e_ = (g / p_.c / qm) * qm;  // transport_block.rs:640
  if (!build_nr_graph(p_.bg, p_.z, &g_)) return (*err = "no base graph for this segmentation", false);
  if (!dec_.init(g_, beta, err)) return (*err = "CUDA decoder set-up: " + *err, false);
  const int c = p_.c;
  words_ = (p_.k_prime + 31) / 32;
  ws_bytes_ = dec_.workspace_bytes(Precision::kF32, c);
  if (!cuda_ok(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream", err) ||
      !cuda_ok(cudaMalloc(&d_acc_, sizeof(float) * (size_t)c * p_.ncb), "HARQ buffers", err) ||
      !cuda_ok(cudaMalloc(&d_rx_, sizeof(float) * std::max<size_t>((size_t)(c * e_), 1)), "LLR staging", err) ||
      !cuda_ok(cudaMalloc(&d_cbs_, sizeof(ServeCb) * c), "descriptors", err) ||
      !cuda_ok(cudaMalloc(&d_hard_, sizeof(uint32_t) * (size_t)c * words_), "hard bits", err) ||
      !cuda_ok(cudaMalloc(&d_iters_, sizeof(int32_t) * c), "iterations", err) ||
      !cuda_ok(cudaMalloc(&d_ws_, std::max<size_t>(ws_bytes_, 1)), "workspace", err))
    return false;
  h_cbs_.resize(c);
  h_hard_.resize((size_t)c * words_);
  h_iters_.resize(c);
  return true;
}

int DlSchF32::decode(const float* rx, long long rx_len, int rv, uint8_t* tb_out, long long tb_len, int* report,
                     uint8_t* cb_crc, std::string* err) {
  const int c = p_.c;
  if (rx_len < e_ * c) return (*err = "rx_llr shorter than C * E", SYNDROME_BUFFER_TOO_SMALL);
  if (tb_len < tb_size_) return (*err = "tb_out shorter than tb_size", SYNDROME_BUFFER_TOO_SMALL);
  if (rv < 0 || rv > 3) return (*err = "rv must be 0..3", SYNDROME_INVALID_PARAM);
  const RmWalk w = rm_walk(p_.bg, p_.z, rv, p_.n_filler);
  if (!rm_walk_covers(w, e_) || e_ > 8LL * p_.ncb)
    return (*err = "E too large for the circular buffer of this code block", SYNDROME_INVALID_PARAM);
  const int harq_tx = tx_ + 1;
  for (int ci = 0; ci < c; ++ci) {
    ServeCb& cb = h_cbs_[ci];
    cb = ServeCb{};
    cb.acc = d_acc_ + (long long)ci * p_.ncb;
    cb.e = d_rx_ + (long long)ci * e_;
    cb.llr = nullptr;  // f32: the accumulators are the decoder input
    cb.hard = d_hard_ + (long long)ci * words_;
    cb.hard_words = words_;
    cb.ncb = w.ncb;
    cb.fs = w.fs;
    cb.fe = w.fe;
    cb.m = w.m;
    cb.c0 = w.c0;
    cb.e_len = (int)e_;
    cb.qm = qm_;
    cb.first = tx_ == 0;
  }
  cudaError_t e;
  if ((e_ * c > 0 && (e = cudaMemcpyAsync(d_rx_, rx, sizeof(float) * e_ * c, cudaMemcpyHostToDevice, stream_)) !=
                         cudaSuccess) ||
      (e = cudaMemcpyAsync(d_cbs_, h_cbs_.data(), sizeof(ServeCb) * c, cudaMemcpyHostToDevice, stream_)) !=
          cudaSuccess ||
      (e = serve_combine_launch(d_cbs_, c, p_.ncb, 1.0f, stream_)) != cudaSuccess)
    return (*err = std::string("HARQ combine: ") + cudaGetErrorString(e), SYNDROME_CUDA_ERROR);
  // prepare_cb_llr (transport_block.rs:473-496): [0] * 2Z ++ accumulator, init_5g_llr,
  // then decode_layered_offset_min_sum, all code blocks in one launch.
  BatchRequest r;
  r.llr = d_acc_;
  r.llr_stride = p_.ncb;
  r.llr_offset = 2 * p_.z;
  r.batch = c;
  r.iterations = iterations_;
  r.prologue_5g = 1;
  r.n_filler = p_.n_filler;
  r.beta = dec_.offset_beta();
  r.hard_packed = d_hard_;
  r.hard_bits = p_.k_prime;
  r.hard_words_stride = words_;
  r.iters = d_iters_;
  r.workspace = d_ws_;
  r.workspace_bytes = ws_bytes_;
  std::string msg;
  if ((e = dec_.decode(Precision::kF32, r, stream_, &msg)) != cudaSuccess)
    return (*err = "decode: " + msg, SYNDROME_CUDA_ERROR);
  if ((e = cudaMemcpyAsync(h_hard_.data(), d_hard_, sizeof(uint32_t) * h_hard_.size(), cudaMemcpyDeviceToHost,
                           stream_)) != cudaSuccess ||
      (e = cudaMemcpyAsync(h_iters_.data(), d_iters_, sizeof(int32_t) * c, cudaMemcpyDeviceToHost, stream_)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(stream_)) != cudaSuccess)
    return (*err = std::string("copy out: ") + cudaGetErrorString(e), SYNDROME_CUDA_ERROR);
  tx_ += 1;
  // CB CRC-24B, desegmentation and TB CRC-24A (transport_block.rs:960-1053).
  const int kp = p_.k_prime, pay = p_.payload;
  std::vector<uint8_t> bits((size_t)kp), all((size_t)c * pay);
  int max_iters = 0;
  bool all_cb = true;
  for (int ci = 0; ci < c; ++ci) {
    const uint32_t* hw = h_hard_.data() + (size_t)ci * words_;
    for (int i = 0; i < kp; ++i) bits[i] = (uint8_t)((hw[i >> 5] >> (i & 31)) & 1u);
    bool ok = true;
    if (p_.has_cb_crc) ok = crc24_bits(bits.data(), kp - 24, kCrc24B) == msb_fold(bits.data() + kp - 24);
    cb_crc[ci] = ok ? 1 : 0;
    all_cb = all_cb && ok;
    std::copy(bits.begin(), bits.begin() + pay, all.begin() + (size_t)ci * pay);
    max_iters = std::max(max_iters, (int)h_iters_[ci]);
  }
  bool tb_ok = false;
  if ((long long)all.size() >= tb_size_ + 24)
    tb_ok = crc24_bits(all.data(), tb_size_, kCrc24A) == msb_fold(all.data() + tb_size_);
  if (all_cb && tb_ok) {
    std::copy(all.begin(), all.begin() + tb_size_, tb_out);
    tx_ = 0;  // HARQ flush: the next transmission starts the accumulators at zero
  }
  report[0] = all_cb && tb_ok;
  report[1] = max_iters;
  report[2] = harq_tx;
  return SYNDROME_OK;
}

// ----------------------------------------------------------------- FramePipe --

FramePipe::~FramePipe() {
  {
    std::lock_guard<std::mutex> l(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  for (auto& t : threads_) t.join();
  for (auto& w : ws_) {
    if (w.stream) cudaStreamSynchronize(w.stream);
    cudaFree(w.d_llr);
    cudaFree(w.d_app);
    cudaFree(w.d_hard);
    cudaFree(w.d_iters);
    cudaFree(w.d_ws);
    if (w.stream) cudaStreamDestroy(w.stream);
  }
  cudaFreeHost(h_llr_);
  cudaFreeHost(h_hard_);
  cudaFreeHost(h_iters_);
}

bool FramePipe::init(const Graph& g, const Decoder* dec, int iterations, int workers, std::string* err) {
  if (iterations < 0) return (*err = "iterations must be non-negative", false);
  n_ = (int)g.n();
  edge_ = (int)g.edge_buffer();
  iterations_ = iterations;
  dec_ = dec;
  workers = std::max(1, std::min(workers, 8));  // ldpc_pipeline.rs:375 clamps to 1..=8
  if (!cuda_ok(cudaGetDevice(&device_), "device", err) ||
      !cuda_ok(cudaHostAlloc((void**)&h_llr_, sizeof(float) * (size_t)kPool * n_, cudaHostAllocDefault),
               "pinned frames", err) ||
      !cuda_ok(cudaHostAlloc((void**)&h_hard_, (size_t)kPool * n_, cudaHostAllocDefault), "pinned frames", err) ||
      !cuda_ok(cudaHostAlloc((void**)&h_iters_, sizeof(int32_t) * kPool, cudaHostAllocDefault), "pinned frames",
               err))
    return false;
  std::fill(h_llr_, h_llr_ + (size_t)kPool * n_, 0.0f);
  std::fill(h_hard_, h_hard_ + (size_t)kPool * n_, (uint8_t)0);
  iters_.assign(kPool, 0);
  tags_.assign(kPool, 0);
  state_.assign(kPool, kFree);
  for (int f = kPool - 1; f >= 0; --f) free_.push_back(f);
  ws_.resize(workers);
  for (auto& w : ws_) {
    w.ws_bytes = dec->workspace_bytes(Precision::kF32, kMaxBatch);
    if (!cuda_ok(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking), "stream", err) ||
        !cuda_ok(cudaMalloc(&w.d_llr, sizeof(float) * (size_t)kMaxBatch * n_), "device frames", err) ||
        !cuda_ok(cudaMalloc(&w.d_app, sizeof(float) * (size_t)kMaxBatch * n_), "device frames", err) ||
        !cuda_ok(cudaMalloc(&w.d_hard, (size_t)kMaxBatch * n_), "device frames", err) ||
        !cuda_ok(cudaMalloc(&w.d_iters, sizeof(int32_t) * kMaxBatch), "device frames", err) ||
        !cuda_ok(cudaMalloc(&w.d_ws, std::max<size_t>(w.ws_bytes, 1)), "workspace", err))
      return false;
  }
  for (int i = 0; i < workers; ++i) threads_.emplace_back([this, i] { run(i); });
  return true;
}

int FramePipe::acquire() {
  std::lock_guard<std::mutex> l(mu_);
  if (free_.empty()) return -1;
  const int f = free_.back();
  free_.pop_back();
  state_[f] = kHeld;
  return f;
}

bool FramePipe::submit(int f) {
  {
    std::lock_guard<std::mutex> l(mu_);
    if (!valid(f) || state_[f] != kHeld) return false;
    state_[f] = kQueued;
    queued_.push_back(f);
  }
  cv_.notify_one();
  return true;
}

int FramePipe::try_recv() {
  std::lock_guard<std::mutex> l(mu_);
  if (done_.empty()) return -1;
  const int f = done_.front();
  done_.pop_front();
  state_[f] = kReceived;
  return f;
}

bool FramePipe::release(int f) {
  std::lock_guard<std::mutex> l(mu_);
  if (!valid(f) || (state_[f] != kReceived && state_[f] != kHeld)) return false;
  state_[f] = kFree;
  free_.push_back(f);
  return true;
}

void FramePipe::run(int wi) {
  Worker& w = ws_[wi];
  cudaSetDevice(device_);
  std::vector<int> batch;
  for (;;) {
    {
      std::unique_lock<std::mutex> l(mu_);
      cv_.wait(l, [&] { return stop_ || !queued_.empty(); });
      if (stop_) return;
      batch.clear();
      while (!queued_.empty() && (int)batch.size() < kMaxBatch) {
        batch.push_back(queued_.front());
        queued_.pop_front();
        state_[batch.back()] = kDecoding;
      }
    }
    const int nb = (int)batch.size();
    const size_t fb = sizeof(float) * (size_t)n_;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < nb && e == cudaSuccess; ++i)
      e = cudaMemcpyAsync(w.d_llr + (size_t)i * n_, llr(batch[i]), fb, cudaMemcpyHostToDevice, w.stream);
    if (e == cudaSuccess) {
      BatchRequest r;
      r.llr = w.d_llr;
      r.llr_stride = n_;
      r.batch = nb;
      r.iterations = iterations_;
      r.beta = dec_->offset_beta();
      r.app = w.d_app;
      r.app_stride = n_;
      r.hard = w.d_hard;
      r.hard_stride = n_;
      r.iters = w.d_iters;
      r.workspace = w.d_ws;
      r.workspace_bytes = w.ws_bytes;
      std::string msg;
      e = dec_->decode(Precision::kF32, r, w.stream, &msg);
    }
    for (int i = 0; i < nb && e == cudaSuccess; ++i) {
      const int f = batch[i];
      if ((e = cudaMemcpyAsync(llr(f), w.d_app + (size_t)i * n_, fb, cudaMemcpyDeviceToHost, w.stream)) !=
              cudaSuccess ||
          (e = cudaMemcpyAsync(h_hard_ + (size_t)f * n_, w.d_hard + (size_t)i * n_, n_, cudaMemcpyDeviceToHost,
                               w.stream)) != cudaSuccess)
        break;
      e = cudaMemcpyAsync(h_iters_ + f, w.d_iters + i, sizeof(int32_t), cudaMemcpyDeviceToHost, w.stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(w.stream);
    std::lock_guard<std::mutex> l(mu_);
    for (int f : batch) {
      // a failed decode reports 0 iterations, as the reference's unwrap_or(0)
      iters_[f] = e == cudaSuccess ? h_iters_[f] : 0;
      state_[f] = kDone;
      done_.push_back(f);
    }
    if (e != cudaSuccess && fatal_.empty()) fatal_ = cudaGetErrorString(e);
  }
}

}  // namespace syn
