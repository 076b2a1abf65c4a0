// extern "C" boundary of libsyndrome_b200.so (declarations: include/syndrome_ldpc.h).
//
// Group 1 mirrors syndrome capi/src/lib.rs function by function: same null checks
// first, then the same validation order as the Rust entry points it wraps, the same
// status codes, and a catch-all guard that reports an internal exception as
// SYNDROME_PANIC (the reference's catch_unwind guard, capi/src/lib.rs:113-115).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/syndrome_ldpc.h"
#include "channel.h"
#include "decoder.h"
#include "encoder.h"
#include "frames.h"
#include "graph.h"
#include "mixed.h"
#include "wifi_mixed.h"
#include "serve.h"
#include "tb.h"

struct SyndromeLdpcDecoder {
  syn::Graph graph;
  syn::Decoder dec;
  int kernel = 0;
  std::mutex mu;  // serialises the host-buffer wrappers that share the staging buffers
  void* staging = nullptr;
  size_t staging_bytes = 0;
  ~SyndromeLdpcDecoder() {
    if (staging) cudaFree(staging);
  }
};

struct SyndromeLdpcEncoder {
  syn::Encoder enc;
};

struct SyndromeMixedPlan {
  syn::MixedPlan plan;
};

struct SyndromeWifiMixedPlan {
  syn::WifiMixedPlan plan;
};

struct SyndromeServer {
  syn::ServeEngine engine;
};

struct SyndromeDlSchEncoder {
  syn::TbEncoder enc;
  size_t tb_size = 0;
};

namespace {

thread_local std::string g_last_error;

template <class F>
int32_t guard(F&& body) {
  try {
    return body();
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return SYNDROME_PANIC;
  } catch (...) {
    g_last_error = "unknown exception";
    return SYNDROME_PANIC;
  }
}

int32_t fail(int32_t code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int32_t from_cuda(cudaError_t e, const std::string& msg) {
  if (e == cudaSuccess) return SYNDROME_OK;
  if (e == cudaErrorInvalidValue && !msg.empty()) {
    const bool small = msg.find("workspace") != std::string::npos;
    return fail(small ? SYNDROME_BUFFER_TOO_SMALL : SYNDROME_INVALID_PARAM, msg);
  }
  return fail(SYNDROME_CUDA_ERROR, std::string(cudaGetErrorString(e)) + (msg.empty() ? "" : ": " + msg));
}

int32_t make_decoder(const syn::Graph& g, float beta, SyndromeLdpcDecoder** out) {
  auto* d = new SyndromeLdpcDecoder();
  d->graph = g;
  std::string err;
  if (!d->dec.init(g, beta, &err)) {
    delete d;
    cudaGetLastError();
    const bool cuda = err.find("CUDA") != std::string::npos || err.find("cuda") != std::string::npos;
    return fail(cuda ? SYNDROME_CUDA_ERROR : SYNDROME_INVALID_PARAM, err);
  }
  *out = d;
  return SYNDROME_OK;
}

// Grows the handle's device staging buffer; caller holds d->mu.
bool ensure_staging(SyndromeLdpcDecoder* d, size_t bytes) {
  if (d->staging_bytes >= bytes) return true;
  if (d->staging) cudaFree(d->staging);
  d->staging = nullptr;
  d->staging_bytes = 0;
  if (cudaMalloc(&d->staging, bytes) != cudaSuccess) return false;
  d->staging_bytes = bytes;
  return true;
}

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Shared host-buffer path: one codeword, device staging, synchronous.
// elem: 4 (f32) or 2 (int16 posterior + int8 messages).
int32_t host_decode(SyndromeLdpcDecoder* d, bool f32, void* app, void* edge_r, uint8_t* hard,
                    size_t iterations, float scale, int16_t app_clamp, size_t* out_iters) {
  const syn::Graph& g = d->graph;
  const size_t n = (size_t)g.n(), ez = (size_t)g.edge_buffer();
  const size_t app_b = n * (f32 ? 4 : 2), edge_b = ez * (f32 ? 4 : 1);
  const size_t off_app = 0, off_out = al256(app_b), off_edge = off_out + al256(app_b);
  const size_t off_hard = off_edge + al256(edge_b), off_it = off_hard + al256(n);
  const size_t total = off_it + 256;
  std::lock_guard<std::mutex> lock(d->mu);
  if (!ensure_staging(d, total)) {
    cudaGetLastError();
    return fail(SYNDROME_CUDA_ERROR, "cudaMalloc of the staging buffer failed");
  }
  char* base = static_cast<char*>(d->staging);
  cudaError_t e = cudaMemcpy(base + off_app, app, app_b, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return from_cuda(e, "copy in");
  syn::BatchRequest r;
  r.llr = base + off_app;
  r.llr_i16 = f32 ? 0 : 1;
  r.llr_stride = (long long)n;
  r.batch = 1;
  r.iterations = (int)std::min<size_t>(iterations, INT_MAX);
  r.beta = d->dec.offset_beta();
  r.beta_q = syn::beta_q(d->dec.offset_beta(), scale);
  r.app_clamp = std::max<int>(app_clamp, 0);
  r.app = base + off_out;
  r.app_stride = (long long)n;
  r.edge_r = base + off_edge;
  r.edge_r_stride = (long long)ez;
  r.hard = reinterpret_cast<uint8_t*>(base + off_hard);
  r.hard_stride = (long long)n;
  r.iters = reinterpret_cast<int32_t*>(base + off_it);
  r.kernel = d->kernel;
  std::string msg;
  e = d->dec.decode(f32 ? syn::Precision::kF32 : syn::Precision::kInt8, r, 0, &msg);
  if (e != cudaSuccess) return from_cuda(e, msg);
  int32_t used = 0;
  if ((e = cudaMemcpy(app, base + off_out, app_b, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(edge_r, base + off_edge, edge_b, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(hard, base + off_hard, n, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(&used, base + off_it, 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return from_cuda(e, "copy out");
  if (out_iters) *out_iters = (size_t)used;
  return SYNDROME_OK;
}

// Validation shared by the f32/int8 host wrappers, in the reference's order
// (src/qc_ldpc.rs:980-1004 and :1544-1568).
int32_t validate_buffers(const syn::Graph& g, size_t app_len, size_t hard_len, size_t edge_len,
                         size_t scratch_len) {
  if (app_len != (size_t)g.n()) return fail(SYNDROME_INVALID_PARAM, "llr length must equal variable_node_count()");
  if (hard_len != (size_t)g.n())
    return fail(SYNDROME_INVALID_PARAM, "hard_output length must equal variable_node_count()");
  if (edge_len < (size_t)g.edge_buffer()) return fail(SYNDROME_BUFFER_TOO_SMALL, "edge_r too small");
  if (scratch_len < (size_t)g.layer_buffer())
    return fail(SYNDROME_BUFFER_TOO_SMALL, "layer_scratch too small");
  return SYNDROME_OK;
}

void nr_prologue_f32(const syn::Graph& g, float* llr, size_t n_filler) {
  const size_t k = (size_t)g.k(), kp = n_filler > k ? 0 : k - n_filler;
  for (size_t i = kp; i < k; ++i) llr[i] = 1000000.0f;
  for (size_t i = 0; i < (size_t)(2 * g.z); ++i) llr[i] = 0.0f;
}

void nr_prologue_i16(const syn::Graph& g, int16_t* app, size_t n_filler, int16_t app_clamp) {
  const size_t k = (size_t)g.k(), kp = n_filler > k ? 0 : k - n_filler;
  const int16_t fill = std::max<int16_t>(app_clamp, 0);
  for (size_t i = kp; i < k; ++i) app[i] = fill;
  for (size_t i = 0; i < (size_t)(2 * g.z); ++i) app[i] = 0;
}

}  // namespace

extern "C" {

const char* syndrome_last_error(void) { return g_last_error.c_str(); }

int32_t syndrome_ldpc_decoder_set_kernel(SyndromeLdpcDecoder* decoder, int32_t kernel) {
  if (!decoder) return SYNDROME_NULL_POINTER;
  if (kernel < 0 || kernel > 5) return fail(SYNDROME_INVALID_PARAM, "kernel must be 0 to 5");
  decoder->kernel = kernel;
  return SYNDROME_OK;
}

// ------------------------------------------------------------- group 1 ------

int32_t syndrome_ldpc_decoder_create(int32_t base_graph, size_t z, float offset_beta,
                                     SyndromeLdpcDecoder** out_decoder) {
  return guard([&]() -> int32_t {
    if (!out_decoder) return SYNDROME_NULL_POINTER;
    *out_decoder = nullptr;
    if (base_graph != 0 && base_graph != 1) return fail(SYNDROME_INVALID_PARAM, "base_graph must be 0 (BG1) or 1 (BG2)");
    syn::Graph g;
    if (z > 384 || !syn::build_nr_graph(base_graph, (int)z, &g))
      return fail(SYNDROME_INVALID_PARAM, "z is not a valid 3GPP lifting size");
    return make_decoder(g, offset_beta, out_decoder);
  });
}

void syndrome_ldpc_decoder_destroy(SyndromeLdpcDecoder* decoder) { delete decoder; }

size_t syndrome_ldpc_decoder_variable_node_count(const SyndromeLdpcDecoder* d) {
  return (size_t)d->graph.n();
}
size_t syndrome_ldpc_decoder_info_bit_count(const SyndromeLdpcDecoder* d) { return (size_t)d->graph.k(); }
size_t syndrome_ldpc_decoder_required_edge_buffer(const SyndromeLdpcDecoder* d) {
  return (size_t)d->graph.edge_buffer();
}
size_t syndrome_ldpc_decoder_required_layer_buffer(const SyndromeLdpcDecoder* d) {
  return (size_t)d->graph.layer_buffer();
}

int32_t syndrome_ldpc_decode_5g(SyndromeLdpcDecoder* decoder, float* llr, size_t llr_len,
                                size_t n_filler, float* edge_r, size_t edge_r_len,
                                float* layer_scratch, size_t layer_scratch_len,
                                uint8_t* hard_output, size_t hard_output_len, size_t iterations,
                                size_t* out_iterations_used) {
  return guard([&]() -> int32_t {
    if (!decoder || !llr || !edge_r || !layer_scratch || !hard_output) return SYNDROME_NULL_POINTER;
    const syn::Graph& g = decoder->graph;
    if (llr_len != (size_t)g.n()) return fail(SYNDROME_INVALID_PARAM, "llr length must equal variable_node_count()");
    nr_prologue_f32(g, llr, n_filler);  // init_5g_llr runs before the decode validates
    int32_t st = validate_buffers(g, llr_len, hard_output_len, edge_r_len, layer_scratch_len);
    if (st != SYNDROME_OK) return st;
    return host_decode(decoder, true, llr, edge_r, hard_output, iterations, 8.0f, 0, out_iterations_used);
  });
}

int32_t syndrome_ldpc_encoder_create(int32_t base_graph, size_t z, SyndromeLdpcEncoder** out) {
  return guard([&]() -> int32_t {
    if (!out) return SYNDROME_NULL_POINTER;
    *out = nullptr;
    if (base_graph != 0 && base_graph != 1) return fail(SYNDROME_INVALID_PARAM, "base_graph must be 0 (BG1) or 1 (BG2)");
    syn::Graph g;
    if (z > 384 || !syn::build_nr_graph(base_graph, (int)z, &g))
      return fail(SYNDROME_INVALID_PARAM, "z is not a valid 3GPP lifting size");
    auto* e = new SyndromeLdpcEncoder();
    if (!e->enc.init(g)) {
      delete e;
      return fail(SYNDROME_INVALID_PARAM, "parity matrix is singular - cannot encode");
    }
    *out = e;
    return SYNDROME_OK;
  });
}

void syndrome_ldpc_encoder_destroy(SyndromeLdpcEncoder* encoder) { delete encoder; }

size_t syndrome_ldpc_encoder_info_bit_count(const SyndromeLdpcEncoder* e) {
  return (size_t)e->enc.graph().k();
}
size_t syndrome_ldpc_encoder_codeword_bit_count(const SyndromeLdpcEncoder* e) {
  return (size_t)e->enc.graph().n();
}

int32_t syndrome_ldpc_encode_5g(const SyndromeLdpcEncoder* encoder, const uint8_t* info_bits,
                                size_t info_len, size_t n_filler, uint8_t* codeword,
                                size_t codeword_len) {
  return guard([&]() -> int32_t {
    if (!encoder || !info_bits || !codeword) return SYNDROME_NULL_POINTER;
    const syn::Graph& g = encoder->enc.graph();
    const size_t k = (size_t)g.k();
    if (n_filler > k) return fail(SYNDROME_INVALID_PARAM, "n_filler exceeds k_bits");
    if (info_len != k - n_filler) return fail(SYNDROME_BUFFER_TOO_SMALL, "info length must equal K - n_filler");
    if (codeword_len != (size_t)g.n()) return fail(SYNDROME_BUFFER_TOO_SMALL, "codeword length must equal N");
    std::vector<uint8_t> full(k, 0);
    std::memcpy(full.data(), info_bits, info_len);
    encoder->enc.encode(full.data(), codeword);
    return SYNDROME_OK;
  });
}

// ------------------------------------------------------------- group 2 ------

int32_t syndrome_ldpc_decoder_create_wifi(size_t z, size_t rate_num, size_t rate_den,
                                          float offset_beta, SyndromeLdpcDecoder** out_decoder) {
  return guard([&]() -> int32_t {
    if (!out_decoder) return SYNDROME_NULL_POINTER;
    *out_decoder = nullptr;
    syn::Graph g;
    if (z > 384 || rate_num > 16 || rate_den > 16 || !syn::build_wifi_graph((int)z, (int)rate_num, (int)rate_den, &g))
      return fail(SYNDROME_INVALID_PARAM, "z/rate is not one of the 12 supported 802.11 LDPC (Z, R) combinations");
    return make_decoder(g, offset_beta, out_decoder);
  });
}

int32_t syndrome_ldpc_decoder_create_raw(const uint8_t* rows, const uint8_t* cols,
                                         const int16_t* shifts, size_t n_edges,
                                         size_t num_row_blocks, size_t num_col_blocks, size_t z,
                                         float offset_beta, SyndromeLdpcDecoder** out_decoder) {
  return guard([&]() -> int32_t {
    if (!out_decoder) return SYNDROME_NULL_POINTER;
    *out_decoder = nullptr;
    if (n_edges > 0 && (!rows || !cols || !shifts)) return SYNDROME_NULL_POINTER;
    if (n_edges > 65536 || num_row_blocks > 255 || num_col_blocks > 255 || z > 384)
      return fail(SYNDROME_INVALID_PARAM, "dimensions out of range");
    std::vector<int> r(n_edges), c(n_edges), s(n_edges);
    for (size_t i = 0; i < n_edges; ++i) {
      r[i] = rows[i];
      c[i] = cols[i];
      s[i] = shifts[i];
    }
    syn::Graph g;
    std::string err;
    if (!syn::build_raw_graph(r.data(), c.data(), s.data(), (int)n_edges, (int)num_row_blocks,
                              (int)num_col_blocks, (int)z, &g, &err))
      return fail(SYNDROME_INVALID_PARAM, err);
    return make_decoder(g, offset_beta, out_decoder);
  });
}

size_t syndrome_ldpc_decoder_check_node_count(const SyndromeLdpcDecoder* d) { return (size_t)d->graph.m(); }

int32_t syndrome_ldpc_decoder_dims(const SyndromeLdpcDecoder* d, size_t* out5) {
  if (!d || !out5) return SYNDROME_NULL_POINTER;
  out5[0] = (size_t)d->graph.z;
  out5[1] = (size_t)d->graph.mb;
  out5[2] = (size_t)d->graph.nb;
  out5[3] = (size_t)d->graph.edges();
  out5[4] = (size_t)d->graph.maxdeg;
  return SYNDROME_OK;
}

int32_t syndrome_ldpc_init_5g_llr(const SyndromeLdpcDecoder* decoder, float* llr, size_t llr_len,
                                  size_t n_filler) {
  return guard([&]() -> int32_t {
    if (!decoder || !llr) return SYNDROME_NULL_POINTER;
    if (llr_len != (size_t)decoder->graph.n())
      return fail(SYNDROME_INVALID_PARAM, "llr length must equal variable_node_count()");
    nr_prologue_f32(decoder->graph, llr, n_filler);
    return SYNDROME_OK;
  });
}

int32_t syndrome_ldpc_decode(SyndromeLdpcDecoder* decoder, float* llr, size_t llr_len,
                             float* edge_r, size_t edge_r_len, float* layer_scratch,
                             size_t layer_scratch_len, uint8_t* hard_output,
                             size_t hard_output_len, size_t iterations,
                             size_t* out_iterations_used) {
  return guard([&]() -> int32_t {
    if (!decoder || !llr || !edge_r || !layer_scratch || !hard_output) return SYNDROME_NULL_POINTER;
    int32_t st = validate_buffers(decoder->graph, llr_len, hard_output_len, edge_r_len, layer_scratch_len);
    if (st != SYNDROME_OK) return st;
    return host_decode(decoder, true, llr, edge_r, hard_output, iterations, 8.0f, 0, out_iterations_used);
  });
}

int32_t syndrome_ldpc_decode_i8(SyndromeLdpcDecoder* decoder, int16_t* app, size_t app_len,
                                int8_t* edge_r, size_t edge_r_len, int8_t* layer_scratch,
                                size_t layer_scratch_len, uint8_t* hard_output,
                                size_t hard_output_len, size_t iterations, float scale,
                                int16_t app_clamp, size_t* out_iterations_used) {
  return guard([&]() -> int32_t {
    if (!decoder || !app || !edge_r || !layer_scratch || !hard_output) return SYNDROME_NULL_POINTER;
    int32_t st = validate_buffers(decoder->graph, app_len, hard_output_len, edge_r_len, layer_scratch_len);
    if (st != SYNDROME_OK) return st;
    return host_decode(decoder, false, app, edge_r, hard_output, iterations, scale, app_clamp,
                       out_iterations_used);
  });
}

int32_t syndrome_ldpc_decode_5g_i8(SyndromeLdpcDecoder* decoder, int16_t* app, size_t app_len,
                                   size_t n_filler, int8_t* edge_r, size_t edge_r_len,
                                   int8_t* layer_scratch, size_t layer_scratch_len,
                                   uint8_t* hard_output, size_t hard_output_len,
                                   size_t iterations, float scale, int16_t app_clamp,
                                   size_t* out_iterations_used) {
  return guard([&]() -> int32_t {
    if (!decoder || !app || !edge_r || !layer_scratch || !hard_output) return SYNDROME_NULL_POINTER;
    if (app_len != (size_t)decoder->graph.n())
      return fail(SYNDROME_INVALID_PARAM, "app length must equal variable_node_count()");
    nr_prologue_i16(decoder->graph, app, n_filler, app_clamp);
    int32_t st = validate_buffers(decoder->graph, app_len, hard_output_len, edge_r_len, layer_scratch_len);
    if (st != SYNDROME_OK) return st;
    return host_decode(decoder, false, app, edge_r, hard_output, iterations, scale, app_clamp,
                       out_iterations_used);
  });
}

int32_t syndrome_ldpc_encoder_create_wifi(size_t z, size_t rate_num, size_t rate_den,
                                          SyndromeLdpcEncoder** out) {
  return guard([&]() -> int32_t {
    if (!out) return SYNDROME_NULL_POINTER;
    *out = nullptr;
    syn::Graph g;
    if (z > 384 || rate_num > 16 || rate_den > 16 || !syn::build_wifi_graph((int)z, (int)rate_num, (int)rate_den, &g))
      return fail(SYNDROME_INVALID_PARAM, "z/rate is not one of the 12 supported 802.11 LDPC (Z, R) combinations");
    auto* e = new SyndromeLdpcEncoder();
    if (!e->enc.init(g)) {
      delete e;
      return fail(SYNDROME_INVALID_PARAM, "parity matrix is singular - cannot encode");
    }
    *out = e;
    return SYNDROME_OK;
  });
}

int32_t syndrome_ldpc_encode(const SyndromeLdpcEncoder* encoder, const uint8_t* info_bits,
                             size_t info_len, uint8_t* codeword, size_t codeword_len) {
  return guard([&]() -> int32_t {
    if (!encoder || !info_bits || !codeword) return SYNDROME_NULL_POINTER;
    const syn::Graph& g = encoder->enc.graph();
    if (info_len != (size_t)g.k()) return fail(SYNDROME_BUFFER_TOO_SMALL, "info length must equal K");
    if (codeword_len != (size_t)g.n()) return fail(SYNDROME_BUFFER_TOO_SMALL, "codeword length must equal N");
    encoder->enc.encode(info_bits, codeword);
    return SYNDROME_OK;
  });
}

int32_t syndrome_ldpc_encode_batch_device(const SyndromeLdpcEncoder* encoder, const uint8_t* d_info,
                                          size_t info_stride, uint8_t* d_codewords, size_t codeword_stride,
                                          size_t count, void* stream) {
  return guard([&]() -> int32_t {
    if (!encoder || ((!d_info || !d_codewords) && count)) return SYNDROME_NULL_POINTER;
    const syn::Graph& g = encoder->enc.graph();
    if (info_stride < (size_t)g.k() || codeword_stride < (size_t)g.n())
      return fail(SYNDROME_BUFFER_TOO_SMALL, "row stride smaller than K or N");
    if (count > (size_t)LLONG_MAX / 2) return fail(SYNDROME_INVALID_PARAM, "count out of range");
    const cudaError_t e = encoder->enc.encode_batch_device(d_info, (long long)info_stride, d_codewords,
                                                           (long long)codeword_stride, (long long)count,
                                                           static_cast<cudaStream_t>(stream));
    return from_cuda(e, "device encode");
  });
}

int32_t syndrome_ldpc_encode_batch(const SyndromeLdpcEncoder* encoder, const uint8_t* info_bits,
                                   size_t info_stride, uint8_t* codewords, size_t codeword_stride,
                                   size_t count, int32_t threads) {
  return guard([&]() -> int32_t {
    if (!encoder || ((!info_bits || !codewords) && count)) return SYNDROME_NULL_POINTER;
    const syn::Graph& g = encoder->enc.graph();
    if (info_stride < (size_t)g.k() || codeword_stride < (size_t)g.n())
      return fail(SYNDROME_BUFFER_TOO_SMALL, "row stride smaller than K or N");
    encoder->enc.encode_batch(info_bits, (long long)info_stride, codewords, (long long)codeword_stride,
                              (long long)count, threads);
    return SYNDROME_OK;
  });
}

void syndrome_quantize_llr_i16(const float* llr, int16_t* out, size_t n, float scale) {
  for (size_t i = 0; i < n; ++i) out[i] = syn::quantize_llr_i16(llr[i], scale);
}

int32_t syndrome_beta_q(float offset_beta, float scale) { return syn::beta_q(offset_beta, scale); }

void syndrome_awgn_llr(float ebno_db, float code_rate, uint64_t seed, const uint8_t* bits, size_t n,
                       float* llr_out) {
  syn::awgn_llr(ebno_db, code_rate, seed, bits, (long long)n, llr_out);
}

void syndrome_awgn_quantized_batch(const uint8_t* bits, size_t n, size_t bits_stride,
                                   size_t tx_begin, const float* ebno_db, float code_rate,
                                   const uint64_t* seeds, float scale, int8_t* out,
                                   size_t out_stride, size_t count, int32_t threads) {
  syn::awgn_quantized_batch(bits, (long long)n, (long long)bits_stride, (long long)tx_begin, ebno_db,
                            code_rate, seeds, scale, out, (long long)out_stride, (long long)count,
                            threads);
}

// ------------------------------------------------------------- group 3 ------

size_t syndrome_ldpc_batch_workspace_size(const SyndromeLdpcDecoder* decoder, int32_t precision,
                                          size_t batch) {
  if (!decoder) return 0;
  return decoder->dec.workspace_bytes(
      precision == SYNDROME_PRECISION_F32 ? syn::Precision::kF32 : syn::Precision::kInt8, (long long)batch);
}

static int32_t batch_common(const SyndromeLdpcDecoder* decoder, syn::Precision p, const void* d_llr,
                            size_t llr_stride, size_t llr_offset, size_t batch, int32_t nr_prologue,
                            size_t n_filler, size_t iterations, float scale, int16_t app_clamp,
                            uint32_t* d_hard_packed, size_t hard_bits, size_t hard_words_stride,
                            int32_t* d_iters, void* d_app, size_t app_stride, void* d_edge_r,
                            size_t edge_r_stride, uint8_t* d_hard, size_t hard_stride,
                            void* d_workspace, size_t workspace_bytes, void* stream,
                            const long long* shorten = nullptr) {
  if (!decoder || (!d_llr && batch)) return SYNDROME_NULL_POINTER;
  const syn::Graph& g = decoder->graph;
  const size_t n = (size_t)g.n();
  if (llr_offset > n) return fail(SYNDROME_INVALID_PARAM, "llr_offset exceeds N");
  if (!shorten && llr_stride < n - llr_offset) return fail(SYNDROME_INVALID_PARAM, "llr_stride smaller than N - llr_offset");
  if (d_app && app_stride < n) return fail(SYNDROME_INVALID_PARAM, "app_stride smaller than N");
  if (d_hard && hard_stride < n) return fail(SYNDROME_INVALID_PARAM, "hard_stride smaller than N");
  if (d_edge_r && edge_r_stride < (size_t)g.edge_buffer())
    return fail(SYNDROME_INVALID_PARAM, "edge_r_stride smaller than the edge buffer");
  if (d_hard_packed && (hard_bits > n || hard_words_stride < (hard_bits + 31) / 32))
    return fail(SYNDROME_INVALID_PARAM, "hard_bits / hard_words_stride out of range");
  if (iterations > (size_t)INT_MAX || batch > (size_t)LLONG_MAX / 2) return fail(SYNDROME_INVALID_PARAM, "size out of range");
  syn::BatchRequest r;
  r.llr = d_llr;
  r.llr_stride = (long long)llr_stride;
  r.llr_offset = (int)llr_offset;
  r.batch = (long long)batch;
  r.iterations = (int)iterations;
  r.prologue_5g = nr_prologue ? 1 : 0;
  r.n_filler = (long long)std::min<size_t>(n_filler, (size_t)1 << 40);
  r.beta = decoder->dec.offset_beta();
  r.beta_q = syn::beta_q(decoder->dec.offset_beta(), scale);
  r.app_clamp = std::max<int>(app_clamp, 0);
  r.hard_packed = d_hard_packed;
  r.hard_bits = (int)hard_bits;
  r.hard_words_stride = (long long)hard_words_stride;
  r.iters = d_iters;
  r.app = d_app;
  r.app_stride = (long long)app_stride;
  r.edge_r = d_edge_r;
  r.edge_r_stride = (long long)edge_r_stride;
  r.hard = d_hard;
  r.hard_stride = (long long)hard_stride;
  r.workspace = d_workspace;
  r.workspace_bytes = workspace_bytes;
  r.kernel = decoder->kernel;
  if (shorten) {
    r.shorten = 1;
    r.shorten_payload = shorten[0];
    r.shorten_tx = shorten[1];
  }
  std::string msg;
  cudaError_t e = decoder->dec.decode(p, r, static_cast<cudaStream_t>(stream), &msg);
  return from_cuda(e, msg);
}

int32_t syndrome_ldpc_decode_batch_i8(const SyndromeLdpcDecoder* decoder, const int8_t* d_llr,
                                      size_t llr_stride, size_t llr_offset, size_t batch,
                                      int32_t nr_prologue, size_t n_filler, size_t iterations,
                                      float scale, int16_t app_clamp, uint32_t* d_hard_packed,
                                      size_t hard_bits, size_t hard_words_stride, int32_t* d_iters,
                                      int16_t* d_app, size_t app_stride, int8_t* d_edge_r,
                                      size_t edge_r_stride, uint8_t* d_hard, size_t hard_stride,
                                      void* d_workspace, size_t workspace_bytes, void* stream) {
  return guard([&]() -> int32_t {
    return batch_common(decoder, syn::Precision::kInt8, d_llr, llr_stride, llr_offset, batch,
                        nr_prologue, n_filler, iterations, scale, app_clamp, d_hard_packed, hard_bits,
                        hard_words_stride, d_iters, d_app, app_stride, d_edge_r, edge_r_stride, d_hard,
                        hard_stride, d_workspace, workspace_bytes, stream);
  });
}

static_assert(SYNDROME_NOALLOC_SCRATCH_BYTES == syn::Decoder::kNoAllocScratchBytes,
              "the header's allocation-free scratch size must be the kernel's");

int32_t syndrome_ldpc_decode_batch_i8_noalloc(const SyndromeLdpcDecoder* decoder, const int8_t* d_llr,
                                              size_t llr_stride, size_t llr_offset, size_t batch,
                                              int32_t nr_prologue, size_t n_filler, size_t iterations,
                                              float scale, int16_t app_clamp, uint32_t* d_hard_packed,
                                              size_t hard_bits, size_t hard_words_stride, int32_t* d_iters,
                                              int16_t* d_app, size_t app_stride, int8_t* d_edge_r,
                                              size_t edge_r_stride, uint8_t* d_hard, size_t hard_stride,
                                              void* stream) {
  return guard([&]() -> int32_t {
    if (!decoder || (!d_llr && batch)) return SYNDROME_NULL_POINTER;
    const syn::Graph& g = decoder->graph;
    const size_t n = (size_t)g.n();
    if (llr_offset > n) return fail(SYNDROME_INVALID_PARAM, "llr_offset exceeds N");
    if (llr_stride < n - llr_offset) return fail(SYNDROME_INVALID_PARAM, "llr_stride smaller than N - llr_offset");
    if (d_app && app_stride < n) return fail(SYNDROME_INVALID_PARAM, "app_stride smaller than N");
    if (d_hard && hard_stride < n) return fail(SYNDROME_INVALID_PARAM, "hard_stride smaller than N");
    if (d_edge_r && edge_r_stride < (size_t)g.edge_buffer())
      return fail(SYNDROME_INVALID_PARAM, "edge_r_stride smaller than the edge buffer");
    if (d_hard_packed && (hard_bits > n || hard_words_stride < (hard_bits + 31) / 32))
      return fail(SYNDROME_INVALID_PARAM, "hard_bits / hard_words_stride out of range");
    if (iterations > (size_t)INT_MAX || batch > (size_t)LLONG_MAX / 2)
      return fail(SYNDROME_INVALID_PARAM, "size out of range");
    syn::BatchRequest r;
    r.llr = d_llr;
    r.llr_stride = (long long)llr_stride;
    r.llr_offset = (int)llr_offset;
    r.batch = (long long)batch;
    r.iterations = (int)iterations;
    r.prologue_5g = nr_prologue ? 1 : 0;
    r.n_filler = (long long)std::min<size_t>(n_filler, (size_t)1 << 40);
    r.beta_q = syn::beta_q(decoder->dec.offset_beta(), scale);
    r.app_clamp = std::max<int>(app_clamp, 0);
    r.hard_packed = d_hard_packed;
    r.hard_bits = (int)hard_bits;
    r.hard_words_stride = (long long)hard_words_stride;
    r.iters = d_iters;
    r.app = d_app;
    r.app_stride = (long long)app_stride;
    r.edge_r = d_edge_r;
    r.edge_r_stride = (long long)edge_r_stride;
    r.hard = d_hard;
    r.hard_stride = (long long)hard_stride;
    r.kernel = decoder->kernel;
    std::string msg;
    cudaError_t e = decoder->dec.decode_i8_noalloc(r, static_cast<cudaStream_t>(stream), &msg);
    return from_cuda(e, msg);
  });
}

int32_t syndrome_ldpc_decode_batch_f32(const SyndromeLdpcDecoder* decoder, const float* d_llr,
                                       size_t llr_stride, size_t llr_offset, size_t batch,
                                       int32_t nr_prologue, size_t n_filler, size_t iterations,
                                       uint32_t* d_hard_packed, size_t hard_bits,
                                       size_t hard_words_stride, int32_t* d_iters, float* d_app,
                                       size_t app_stride, float* d_edge_r, size_t edge_r_stride,
                                       uint8_t* d_hard, size_t hard_stride, void* d_workspace,
                                       size_t workspace_bytes, void* stream) {
  return guard([&]() -> int32_t {
    return batch_common(decoder, syn::Precision::kF32, d_llr, llr_stride, llr_offset, batch,
                        nr_prologue, n_filler, iterations, 8.0f, 0, d_hard_packed, hard_bits,
                        hard_words_stride, d_iters, d_app, app_stride, d_edge_r, edge_r_stride, d_hard,
                        hard_stride, d_workspace, workspace_bytes, stream);
  });
}

// ------------------------------------------- Wi-Fi shortening / puncturing ---
// src/wifi_rate_matching.rs:88-132 (counts), :163-192 (encode), :267-302 (decode).

static int32_t wifi_counts(size_t k, size_t n, size_t payload, size_t target, size_t* n_shrt, size_t* n_punc) {
  if (n < k) return fail(SYNDROME_INVALID_PARAM, "codeword length N must be at least the information length K");
  if (payload > k)
    return fail(SYNDROME_INVALID_PARAM,
                "payload_bits exceeds this codeword's K; multi-codeword segmentation is not implemented");
  if (target < payload)
    return fail(SYNDROME_INVALID_PARAM, "target_coded_bits must be at least payload_bits");
  const size_t shrt = k - payload, max_coded = n - shrt;
  if (target > max_coded) return fail(SYNDROME_INVALID_PARAM, "target_coded_bits exceeds N - n_shrt");
  *n_shrt = shrt;
  *n_punc = max_coded - target;
  return SYNDROME_OK;
}

int32_t syndrome_wifi_shortening_counts(size_t k, size_t n, size_t payload_bits, size_t target_coded_bits,
                                        size_t* out_n_shrt, size_t* out_n_punc) {
  return guard([&]() -> int32_t {
    if (!out_n_shrt || !out_n_punc) return SYNDROME_NULL_POINTER;
    return wifi_counts(k, n, payload_bits, target_coded_bits, out_n_shrt, out_n_punc);
  });
}

int32_t syndrome_wifi_encode_shortened(const SyndromeLdpcEncoder* encoder, const uint8_t* payload,
                                       size_t payload_bits, size_t target_coded_bits, uint8_t* out,
                                       size_t out_len) {
  return guard([&]() -> int32_t {
    if (!encoder || (!payload && payload_bits) || !out) return SYNDROME_NULL_POINTER;
    const syn::Graph& g = encoder->enc.graph();
    const size_t k = (size_t)g.k(), n = (size_t)g.n();
    size_t shrt = 0, punc = 0;
    int32_t st = wifi_counts(k, n, payload_bits, target_coded_bits, &shrt, &punc);
    if (st != SYNDROME_OK) return st;
    if (out_len != target_coded_bits) return fail(SYNDROME_BUFFER_TOO_SMALL, "out length must equal target_coded_bits");
    std::vector<uint8_t> info(k, 0), cw(n);
    std::copy(payload, payload + payload_bits, info.begin());
    encoder->enc.encode(info.data(), cw.data());
    const size_t par = (n - k) - punc;
    std::copy(payload, payload + payload_bits, out);
    std::copy(cw.begin() + k, cw.begin() + k + par, out + payload_bits);
    return SYNDROME_OK;
  });
}

int32_t syndrome_wifi_decode_shortened(SyndromeLdpcDecoder* decoder, size_t payload_bits, const float* rx_llr,
                                       size_t rx_len, float* codeword_llr, size_t codeword_len,
                                       float* edge_r, size_t edge_r_len, float* layer_scratch,
                                       size_t layer_scratch_len, uint8_t* hard_output, size_t hard_output_len,
                                       size_t iterations, size_t* out_iterations_used) {
  return guard([&]() -> int32_t {
    if (!decoder || (!rx_llr && rx_len) || !codeword_llr || !edge_r || !layer_scratch || !hard_output)
      return SYNDROME_NULL_POINTER;
    const syn::Graph& g = decoder->graph;
    const size_t n = (size_t)g.n(), k = n - (size_t)g.m();
    size_t shrt = 0, punc = 0;
    int32_t st = wifi_counts(k, n, payload_bits, rx_len, &shrt, &punc);
    if (st != SYNDROME_OK) return st;
    if (codeword_len != n) return fail(SYNDROME_BUFFER_TOO_SMALL, "codeword_llr length must equal N");
    const size_t par = (n - k) - punc;
    std::copy(rx_llr, rx_llr + payload_bits, codeword_llr);
    std::fill(codeword_llr + payload_bits, codeword_llr + k, 1000000.0f);
    std::copy(rx_llr + payload_bits, rx_llr + payload_bits + par, codeword_llr + k);
    std::fill(codeword_llr + k + par, codeword_llr + n, 0.0f);
    st = validate_buffers(g, codeword_len, hard_output_len, edge_r_len, layer_scratch_len);
    if (st != SYNDROME_OK) return st;
    return host_decode(decoder, true, codeword_llr, edge_r, hard_output, iterations, 8.0f, 0, out_iterations_used);
  });
}

int32_t syndrome_wifi_decode_shortened_batch_f32(const SyndromeLdpcDecoder* decoder, const float* d_rx,
                                                 size_t rx_stride, size_t payload_bits, size_t target_coded_bits,
                                                 size_t batch, size_t iterations, uint32_t* d_hard_packed,
                                                 size_t hard_bits, size_t hard_words_stride, int32_t* d_iters,
                                                 float* d_app, size_t app_stride, float* d_edge_r,
                                                 size_t edge_r_stride, uint8_t* d_hard, size_t hard_stride,
                                                 void* d_workspace, size_t workspace_bytes, void* stream) {
  return guard([&]() -> int32_t {
    if (!decoder) return SYNDROME_NULL_POINTER;
    const syn::Graph& g = decoder->graph;
    const size_t n = (size_t)g.n(), k = n - (size_t)g.m();
    size_t shrt = 0, punc = 0;
    int32_t st = wifi_counts(k, n, payload_bits, target_coded_bits, &shrt, &punc);
    if (st != SYNDROME_OK) return st;
    if (rx_stride < target_coded_bits) return fail(SYNDROME_INVALID_PARAM, "rx_stride smaller than target_coded_bits");
    const long long sh[2] = {(long long)payload_bits, (long long)target_coded_bits};
    return batch_common(decoder, syn::Precision::kF32, d_rx, rx_stride, 0, batch, 0, 0, iterations, 8.0f, 0,
                        d_hard_packed, hard_bits, hard_words_stride, d_iters, d_app, app_stride, d_edge_r,
                        edge_r_stride, d_hard, hard_stride, d_workspace, workspace_bytes, stream, sh);
  });
}

// ------------------------------------------------------- mixed batches ------

int32_t syndrome_mixed_plan_create(const SyndromeMixedCodeword* codewords, size_t count, float offset_beta,
                                   float scale, int16_t app_clamp, size_t iterations,
                                   const int32_t* tile_hints, size_t n_hints, SyndromeMixedPlan** out_plan) {
  return guard([&]() -> int32_t {
    if (!out_plan || (!codewords && count) || (!tile_hints && n_hints)) return SYNDROME_NULL_POINTER;
    *out_plan = nullptr;
    if (iterations > (size_t)INT_MAX || count > (size_t)INT_MAX / 2) return fail(SYNDROME_INVALID_PARAM, "size out of range");
    std::vector<syn::MixedCodeword> cws(count);
    for (size_t i = 0; i < count; ++i) {
      const SyndromeMixedCodeword& c = codewords[i];
      cws[i] = syn::MixedCodeword{c.base_graph, c.z, c.n_filler, c.hard_bits, (long long)c.llr_offset,
                                  (long long)c.out_offset};
    }
    std::vector<syn::TileHint> hints(n_hints);
    for (size_t i = 0; i < n_hints; ++i) hints[i] = syn::TileHint{tile_hints[3 * i], tile_hints[3 * i + 1], tile_hints[3 * i + 2]};
    auto* p = new SyndromeMixedPlan();
    std::string err;
    if (!p->plan.init(cws, syn::beta_q(offset_beta, scale), std::max<int>(app_clamp, 0), (int)iterations, hints, &err)) {
      delete p;
      cudaGetLastError();
      return fail(err.find("CUDA") != std::string::npos || err.find("cuda") != std::string::npos
                      ? SYNDROME_CUDA_ERROR
                      : SYNDROME_INVALID_PARAM,
                  err);
    }
    *out_plan = p;
    return SYNDROME_OK;
  });
}

void syndrome_mixed_plan_destroy(SyndromeMixedPlan* plan) { delete plan; }

int32_t syndrome_mixed_plan_items(const SyndromeMixedPlan* plan, int32_t* out_items, size_t cap, size_t* n_items) {
  if (!plan || !n_items) return SYNDROME_NULL_POINTER;
  const auto& items = plan->plan.item_list();
  *n_items = items.size();
  if (out_items)
    for (size_t i = 0; i < items.size() && i < cap; ++i) {
      out_items[3 * i] = items[i].bg;
      out_items[3 * i + 1] = items[i].z;
      out_items[3 * i + 2] = items[i].count;
    }
  return SYNDROME_OK;
}

int32_t syndrome_mixed_plan_set_kernel(SyndromeMixedPlan* plan, int32_t kernel, int32_t* is_tmem) {
  if (!plan) return SYNDROME_NULL_POINTER;
  if (!plan->plan.set_kernel(kernel)) return fail(SYNDROME_INVALID_PARAM, "mixed-plan kernel must be 0 or 5");
  if (is_tmem) *is_tmem = plan->plan.tmem() && kernel != 5;
  return SYNDROME_OK;
}

int32_t syndrome_mixed_tile_capacity(int32_t base_graph, int32_t z) {
  if ((base_graph != 0 && base_graph != 1) || syn::lifting_set_index(z) < 0) return 0;
  return syn::pair_mixed_capacity(base_graph, z);
}

int32_t syndrome_mixed_decode(SyndromeMixedPlan* plan, const int8_t* d_llr, size_t llr_bytes,
                              uint32_t* d_hard_packed, size_t out_words, int32_t* d_iters, size_t iters_len,
                              int32_t use_graph, void* stream) {
  return guard([&]() -> int32_t {
    if (!plan || !d_llr || !d_hard_packed) return SYNDROME_NULL_POINTER;
    if ((long long)llr_bytes < plan->plan.llr_bytes_needed())
      return fail(SYNDROME_BUFFER_TOO_SMALL, "LLR buffer shorter than the planned offsets");
    if ((long long)out_words < plan->plan.out_words_needed())
      return fail(SYNDROME_BUFFER_TOO_SMALL, "output buffer shorter than the planned offsets");
    if (d_iters && iters_len < (size_t)plan->plan.codewords())
      return fail(SYNDROME_BUFFER_TOO_SMALL, "iteration buffer shorter than the codeword count");
    return from_cuda(plan->plan.decode(d_llr, d_hard_packed, d_iters, use_graph != 0,
                                       static_cast<cudaStream_t>(stream)),
                     "");
  });
}

int32_t syndrome_wifi_mixed_plan_create(const SyndromeWifiMixedCodeword* codewords, size_t count, float offset_beta,
                                        size_t iterations, size_t chunk, SyndromeWifiMixedPlan** out_plan) {
  return guard([&]() -> int32_t {
    if (!out_plan || (!codewords && count)) return SYNDROME_NULL_POINTER;
    *out_plan = nullptr;
    if (iterations > (size_t)INT_MAX || chunk > (size_t)INT_MAX || count > (size_t)INT_MAX / 2)
      return fail(SYNDROME_INVALID_PARAM, "size out of range");
    std::vector<syn::WifiMixedCodeword> cws(count);
    for (size_t i = 0; i < count; ++i) {
      const SyndromeWifiMixedCodeword& c = codewords[i];
      cws[i] = syn::WifiMixedCodeword{c.z, c.rate_num, c.rate_den, c.hard_bits, (long long)c.llr_offset,
                                      (long long)c.out_offset};
    }
    auto* p = new SyndromeWifiMixedPlan();
    std::string err;
    if (!p->plan.init(cws, offset_beta, (int)iterations, (int)chunk, &err)) {
      delete p;
      cudaGetLastError();
      return fail(err.find("CUDA") != std::string::npos || err.find("cuda") != std::string::npos
                      ? SYNDROME_CUDA_ERROR
                      : SYNDROME_INVALID_PARAM,
                  err);
    }
    *out_plan = p;
    return SYNDROME_OK;
  });
}

void syndrome_wifi_mixed_plan_destroy(SyndromeWifiMixedPlan* plan) { delete plan; }

int32_t syndrome_wifi_mixed_plan_chunks(const SyndromeWifiMixedPlan* plan, size_t* n_chunks, size_t* ctas) {
  if (!plan || !n_chunks) return SYNDROME_NULL_POINTER;
  *n_chunks = (size_t)plan->plan.chunks();
  if (ctas) *ctas = (size_t)plan->plan.ctas();
  return SYNDROME_OK;
}

int32_t syndrome_wifi_mixed_decode(SyndromeWifiMixedPlan* plan, const float* d_llr, size_t llr_len,
                                   uint32_t* d_hard_packed, size_t out_words, int32_t* d_iters, size_t iters_len,
                                   int32_t use_graph, void* stream) {
  return guard([&]() -> int32_t {
    if (!plan || !d_llr || !d_hard_packed) return SYNDROME_NULL_POINTER;
    if ((long long)llr_len < plan->plan.llr_needed())
      return fail(SYNDROME_BUFFER_TOO_SMALL, "LLR buffer shorter than the planned offsets");
    if ((long long)out_words < plan->plan.out_words_needed())
      return fail(SYNDROME_BUFFER_TOO_SMALL, "output buffer shorter than the planned offsets");
    if (d_iters && iters_len < (size_t)plan->plan.codewords())
      return fail(SYNDROME_BUFFER_TOO_SMALL, "iteration buffer shorter than the codeword count");
    return from_cuda(plan->plan.decode(d_llr, d_hard_packed, d_iters, use_graph != 0,
                                       static_cast<cudaStream_t>(stream)),
                     "");
  });
}

// ------------------------------------------------------- transport blocks ---

int32_t syndrome_tb_segmentation(size_t tb_size, float target_rate, int64_t* out10) {
  return guard([&]() -> int32_t {
    if (!out10) return SYNDROME_NULL_POINTER;
    syn::TbParams p;
    std::string err;
    if (!syn::compute_segmentation((long long)std::min<size_t>(tb_size, (size_t)LLONG_MAX), target_rate, &p, &err))
      return fail(SYNDROME_INVALID_PARAM, err);
    const int64_t v[10] = {p.bg, p.z, p.c, p.b, p.k_prime, p.k, p.ncb, p.n_filler, p.has_cb_crc ? 1 : 0, p.payload};
    for (int i = 0; i < 10; ++i) out10[i] = v[i];
    return SYNDROME_OK;
  });
}

uint32_t syndrome_crc24(const uint8_t* bits, size_t n, int32_t kind) {
  if (!bits && n) return 0;
  return syn::crc24_bits(bits, (long long)n, kind == 0 ? syn::kCrc24A : syn::kCrc24B);
}

int32_t syndrome_dlsch_encoder_create(size_t tb_size, float target_rate, size_t qm, size_t g,
                                      SyndromeDlSchEncoder** out) {
  return guard([&]() -> int32_t {
    if (!out) return SYNDROME_NULL_POINTER;
    *out = nullptr;
    if (tb_size > (size_t)syn::kMaxTbBits * 2 || qm > 64 || g > ((size_t)1 << 40))
      return fail(SYNDROME_INVALID_PARAM, "argument out of range");
    auto* e = new SyndromeDlSchEncoder();
    std::string err;
    if (!e->enc.init((long long)tb_size, target_rate, (int)qm, (long long)g, &err)) {
      delete e;
      return fail(SYNDROME_INVALID_PARAM, err);
    }
    e->tb_size = tb_size;
    *out = e;
    return SYNDROME_OK;
  });
}

void syndrome_dlsch_encoder_destroy(SyndromeDlSchEncoder* encoder) { delete encoder; }

size_t syndrome_dlsch_encoder_output_bits(const SyndromeDlSchEncoder* e) {
  return e ? (size_t)e->enc.output_bits() : 0;
}

size_t syndrome_dlsch_encoder_num_code_blocks(const SyndromeDlSchEncoder* e) {
  return e ? (size_t)e->enc.params().c : 0;
}

int32_t syndrome_dlsch_encode(const SyndromeDlSchEncoder* e, const uint8_t* tb, size_t tb_len, size_t rv, uint8_t* out,
                              size_t out_len) {
  return guard([&]() -> int32_t {
    if (!e || !tb || !out) return SYNDROME_NULL_POINTER;
    if (tb_len != e->tb_size) return fail(SYNDROME_BUFFER_TOO_SMALL, "tb length must equal tb_size");
    if (out_len < (size_t)e->enc.output_bits()) return fail(SYNDROME_BUFFER_TOO_SMALL, "output shorter than output_bits");
    if (rv > 3) return fail(SYNDROME_INVALID_PARAM, "RV must be 0..=3");
    e->enc.encode(tb, (int)rv, out);
    return SYNDROME_OK;
  });
}

// ------------------------------------------------ DL-SCH decoder (f32) -----

struct SyndromeDlSchDecoder {
  syn::DlSchF32 d;
  size_t workers = 0;
};

int32_t syndrome_dlsch_decoder_create(size_t tb_size, float target_rate, size_t qm, size_t g, size_t iterations,
                                      float offset_beta, SyndromeDlSchDecoder** out) {
  return guard([&]() -> int32_t {
    if (!out) return SYNDROME_NULL_POINTER;
    *out = nullptr;
    if (tb_size > (size_t)syn::kMaxTbBits * 2 || qm > 64 || g > ((size_t)1 << 40) || iterations > (size_t)INT_MAX)
      return fail(SYNDROME_INVALID_PARAM, "size out of range");
    auto* d = new SyndromeDlSchDecoder();
    std::string err;
    if (!d->d.init((long long)tb_size, target_rate, (int)qm, (long long)g, (int)iterations, offset_beta, &err)) {
      delete d;
      cudaGetLastError();
      return fail(err.rfind("CUDA ", 0) == 0 ? SYNDROME_CUDA_ERROR : SYNDROME_INVALID_PARAM, err);
    }
    *out = d;
    return SYNDROME_OK;
  });
}

void syndrome_dlsch_decoder_destroy(SyndromeDlSchDecoder* d) { delete d; }
size_t syndrome_dlsch_decoder_num_code_blocks(const SyndromeDlSchDecoder* d) { return d ? (size_t)d->d.params().c : 0; }
size_t syndrome_dlsch_decoder_output_bits(const SyndromeDlSchDecoder* d) { return d ? (size_t)d->d.output_bits() : 0; }

int32_t syndrome_dlsch_decoder_with_pipeline(SyndromeDlSchDecoder* d, size_t n_workers) {
  return guard([&]() -> int32_t {
    if (!d) return SYNDROME_NULL_POINTER;
    if (n_workers == 0) return fail(SYNDROME_INVALID_PARAM, "n_workers must be > 0");
    d->workers = std::min<size_t>(n_workers, 8);
    return SYNDROME_OK;
  });
}

size_t syndrome_dlsch_decoder_worker_count(const SyndromeDlSchDecoder* d) { return d ? d->workers : 0; }

int32_t syndrome_dlsch_decode(SyndromeDlSchDecoder* d, const float* rx, size_t rx_len, size_t rv, uint8_t* tb_out,
                              size_t tb_len, SyndromeDecodeReport* report, uint8_t* cb_crc, size_t cb_crc_len) {
  return guard([&]() -> int32_t {
    if (!d || (!rx && rx_len) || !tb_out || !report) return SYNDROME_NULL_POINTER;
    const int c = d->d.params().c;
    if (cb_crc && cb_crc_len < (size_t)c) return fail(SYNDROME_BUFFER_TOO_SMALL, "cb_crc shorter than C");
    if (rv > 3) return fail(SYNDROME_INVALID_PARAM, "rv must be 0..3");
    std::vector<uint8_t> cbs((size_t)c);
    int rep[3] = {0, 0, 0};
    std::string err;
    const int st = d->d.decode(rx, (long long)std::min<size_t>(rx_len, (size_t)LLONG_MAX), (int)rv, tb_out,
                               (long long)std::min<size_t>(tb_len, (size_t)LLONG_MAX), rep, cbs.data(), &err);
    if (st != SYNDROME_OK) return fail(st, err);
    report->crc_ok = rep[0];
    report->max_iters_used = rep[1];
    report->harq_tx_count = rep[2];
    report->num_code_blocks = c;
    if (cb_crc) std::copy(cbs.begin(), cbs.end(), cb_crc);
    return SYNDROME_OK;
  });
}

void syndrome_dlsch_decoder_flush_harq(SyndromeDlSchDecoder* d) {
  if (d) d->d.flush();
}

// ------------------------------------------------------- frame pipeline -----

struct SyndromeLdpcPipeline {
  syn::FramePipe p;
};

int32_t syndrome_ldpc_pipeline_create(const SyndromeLdpcDecoder* decoder, size_t iterations, size_t n_workers,
                                      SyndromeLdpcPipeline** out) {
  return guard([&]() -> int32_t {
    if (!decoder || !out) return SYNDROME_NULL_POINTER;
    *out = nullptr;
    if (iterations > (size_t)INT_MAX) return fail(SYNDROME_INVALID_PARAM, "iterations out of range");
    int w = (int)std::min<size_t>(n_workers, 8);
    if (w == 0) w = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    auto* p = new SyndromeLdpcPipeline();
    std::string err;
    if (!p->p.init(decoder->graph, &decoder->dec, (int)iterations, w, &err)) {
      delete p;
      cudaGetLastError();
      return fail(SYNDROME_CUDA_ERROR, err);
    }
    *out = p;
    return SYNDROME_OK;
  });
}

void syndrome_ldpc_pipeline_destroy(SyndromeLdpcPipeline* p) { delete p; }
size_t syndrome_ldpc_pipeline_worker_count(const SyndromeLdpcPipeline* p) { return p ? (size_t)p->p.workers() : 0; }
size_t syndrome_ldpc_pipeline_pool_size(const SyndromeLdpcPipeline*) { return (size_t)syn::FramePipe::kPool; }
int64_t syndrome_ldpc_pipeline_acquire(SyndromeLdpcPipeline* p) { return p ? p->p.acquire() : -1; }
int64_t syndrome_ldpc_pipeline_try_recv(SyndromeLdpcPipeline* p) { return p ? p->p.try_recv() : -1; }

int32_t syndrome_ldpc_pipeline_submit(SyndromeLdpcPipeline* p, int64_t f) {
  if (!p) return SYNDROME_NULL_POINTER;
  if (f < 0 || f >= syn::FramePipe::kPool || !p->p.submit((int)f))
    return fail(SYNDROME_INVALID_PARAM, "not an acquired frame");
  return SYNDROME_OK;
}

int32_t syndrome_ldpc_pipeline_release(SyndromeLdpcPipeline* p, int64_t f) {
  if (!p) return SYNDROME_NULL_POINTER;
  if (f < 0 || f >= syn::FramePipe::kPool || !p->p.release((int)f))
    return fail(SYNDROME_INVALID_PARAM, "not a received or acquired frame");
  return SYNDROME_OK;
}

float* syndrome_ldpc_pipeline_frame_llr(SyndromeLdpcPipeline* p, int64_t f) {
  return p && p->p.valid((int)f) && f == (int)f ? p->p.llr((int)f) : nullptr;
}
const uint8_t* syndrome_ldpc_pipeline_frame_hard(const SyndromeLdpcPipeline* p, int64_t f) {
  return p && p->p.valid((int)f) && f == (int)f ? p->p.hard((int)f) : nullptr;
}
size_t syndrome_ldpc_pipeline_frame_iterations(const SyndromeLdpcPipeline* p, int64_t f) {
  return p && p->p.valid((int)f) && f == (int)f ? (size_t)p->p.iterations_used((int)f) : 0;
}
void syndrome_ldpc_pipeline_frame_set_tag(SyndromeLdpcPipeline* p, int64_t f, size_t tag) {
  if (p && p->p.valid((int)f) && f == (int)f) p->p.tag((int)f) = tag;
}
size_t syndrome_ldpc_pipeline_frame_tag(const SyndromeLdpcPipeline* p, int64_t f) {
  return p && p->p.valid((int)f) && f == (int)f ? const_cast<syn::FramePipe&>(p->p).tag((int)f) : 0;
}

// ----------------------------------------------------------------- serving ---

int32_t syndrome_serve_create(const SyndromeServeConfig* config, SyndromeServer** out) {
  return guard([&]() -> int32_t {
    if (!out) return SYNDROME_NULL_POINTER;
    *out = nullptr;
    syn::ServeConfig c;
    if (config) {
      if (config->max_step_code_blocks) c.max_step_cbs = (int)std::min<uint32_t>(config->max_step_code_blocks, 65535);
      if (config->steps_in_flight) c.slots = (int)std::min<uint32_t>(config->steps_in_flight, 16);
      if (config->harq_bytes) c.harq_bytes = (long long)config->harq_bytes;
      if (config->staging_bytes) c.staging_bytes = (long long)config->staging_bytes;
      c.iterations = config->iterations;
      c.beta = config->offset_beta;
      c.scale = config->scale;
      c.app_clamp = config->app_clamp;
      if (config->latency_steps) c.latency_slots = (int)std::min<uint32_t>(config->latency_steps, 16);
      if (config->backlog_code_blocks)
        c.backlog_cbs = (int)std::min<uint32_t>(config->backlog_code_blocks, 1u << 30);
      if (config->decode_kernel != 0 && config->decode_kernel != 5)
        return fail(SYNDROME_INVALID_PARAM, "decode_kernel must be 0 or 5");
      c.decode_kernel = config->decode_kernel;
      if (config->engine != 0 && config->engine != 1) return fail(SYNDROME_INVALID_PARAM, "engine must be 0 or 1");
      c.mode = config->engine;
      if (config->idle_us) c.idle_us = (long long)std::min<uint32_t>(config->idle_us, 1000000u);
    }
    auto* s = new SyndromeServer();
    std::string err;
    if (!s->engine.init(c, &err)) {
      delete s;
      cudaGetLastError();
      return fail(err.find("alloc") != std::string::npos || err.find("CUDA") != std::string::npos
                      ? SYNDROME_CUDA_ERROR
                      : SYNDROME_INVALID_PARAM,
                  err);
    }
    *out = s;
    return SYNDROME_OK;
  });
}

void syndrome_serve_destroy(SyndromeServer* server) { delete server; }

int32_t syndrome_serve_submit(SyndromeServer* server, uint64_t tb_id, size_t tb_size, float target_rate, size_t qm,
                              size_t g, size_t rv, const float* llr, size_t llr_len, int32_t llr_on_device) {
  return guard([&]() -> int32_t {
    if (!server || !llr) return SYNDROME_NULL_POINTER;
    if (tb_size > (size_t)syn::kMaxTbBits * 2 || qm > 64 || g > ((size_t)1 << 40) || rv > 3 ||
        llr_len > ((size_t)1 << 40))
      return fail(SYNDROME_INVALID_PARAM, "argument out of range");
    std::string err;
    const int r = server->engine.submit(tb_id, (long long)tb_size, target_rate, (int)qm, (long long)g, (int)rv, llr,
                                        (long long)llr_len, llr_on_device != 0, &err);
    return r == SYNDROME_OK ? SYNDROME_OK : fail(r, err);
  });
}

int32_t syndrome_serve_poll(SyndromeServer* server, SyndromeServeResult* out, size_t cap, size_t* n_out,
                            int64_t timeout_us) {
  return guard([&]() -> int32_t {
    if (!server || !n_out || (!out && cap)) return SYNDROME_NULL_POINTER;
    std::vector<syn::ServeResult> buf(std::min<size_t>(cap, 4096));
    const int n = server->engine.poll(buf.data(), (int)buf.size(), timeout_us);
    for (int i = 0; i < n; ++i) {
      SyndromeServeResult& r = out[i];
      std::memset(&r, 0, sizeof(r));
      r.tb_id = buf[i].id;
      r.crc_ok = buf[i].crc_ok;
      r.max_iters_used = buf[i].max_iters;
      r.harq_tx_count = buf[i].harq_tx;
      r.num_code_blocks = buf[i].n_cb;
      for (int w = 0; w < 5; ++w) r.cb_crc[w] = buf[i].cb_crc[w];
      r.latency_us = buf[i].latency_us;
    }
    *n_out = (size_t)n;
    return SYNDROME_OK;
  });
}

int32_t syndrome_serve_fetch(SyndromeServer* server, uint64_t tb_id, uint8_t* tb_bits, size_t tb_len) {
  return guard([&]() -> int32_t {
    if (!server || !tb_bits) return SYNDROME_NULL_POINTER;
    std::string err;
    const int r = server->engine.fetch(tb_id, tb_bits, (long long)std::min<size_t>(tb_len, (size_t)1 << 40), &err);
    return r == SYNDROME_OK ? SYNDROME_OK : fail(r, err);
  });
}

int32_t syndrome_serve_release(SyndromeServer* server, uint64_t tb_id) {
  return guard([&]() -> int32_t {
    if (!server) return SYNDROME_NULL_POINTER;
    std::string err;
    const int r = server->engine.release(tb_id, &err);
    return r == SYNDROME_OK ? SYNDROME_OK : fail(r, err);
  });
}

int32_t syndrome_serve_set_tiles(SyndromeServer* server, const int32_t* triples, size_t n) {
  return guard([&]() -> int32_t {
    if (!server || (!triples && n)) return SYNDROME_NULL_POINTER;
    for (size_t i = 0; i < n; ++i) {
      const int bg = triples[3 * i], z = triples[3 * i + 1];
      if ((bg != 0 && bg != 1) || z < 1 || z > 384) return fail(SYNDROME_INVALID_PARAM, "base graph or z out of range");
    }
    for (size_t i = 0; i < n; ++i) server->engine.set_tile(triples[3 * i], triples[3 * i + 1], triples[3 * i + 2]);
    return SYNDROME_OK;
  });
}

int32_t syndrome_serve_stats(SyndromeServer* server, int64_t* out14) {
  return guard([&]() -> int32_t {
    if (!server || !out14) return SYNDROME_NULL_POINTER;
    const syn::ServeStats s = server->engine.stats();
    const int64_t v[14] = {s.steps, s.code_blocks, s.transmissions, s.harq_bytes_used, s.pending, s.in_flight,
                           s.tbs_held, s.max_pending, s.items, s.item_threads, (int64_t)(s.decode_ms * 1000.0),
                           (int64_t)(s.step_ms * 1000.0), (int64_t)(s.host_launch_ms * 1000.0),
                           (int64_t)(s.host_finish_ms * 1000.0)};
    for (int i = 0; i < 14; ++i) out14[i] = v[i];
    return SYNDROME_OK;
  });
}

int32_t syndrome_serve_core_stats(SyndromeServer* server, double* out10) {
  return guard([&]() -> int32_t {
    if (!server || !out10) return SYNDROME_NULL_POINTER;
    const syn::ServeCoreStats s = server->engine.core_stats();
    const double v[10] = {(double)s.items, s.busy_us,  s.combine_us, s.decode_us,  s.crc_us,
                          s.finish_us,     (double)s.loops, s.admit_us, s.publish_us, s.complete_us};
    for (int i = 0; i < 10; ++i) out10[i] = v[i];
    return SYNDROME_OK;
  });
}

int32_t syndrome_serve_run_load(SyndromeServer* server, const SyndromeLoadTb* pool, size_t pool_n,
                                const SyndromeLoadSpec* spec, SyndromeLoadReport* report, double* latencies_us,
                                size_t latencies_cap) {
  return guard([&]() -> int32_t {
    if (!server || !pool || !spec || !report) return SYNDROME_NULL_POINTER;
    if (pool_n == 0 || !(spec->offered_tb_per_s > 0.0) || !(spec->duration_s >= 0.0) || spec->duration_s > 3600.0)
      return fail(SYNDROME_INVALID_PARAM, "empty pool or bad rate / duration");
    for (size_t i = 0; i < pool_n; ++i)
      for (int k = 0; k < 4; ++k)
        if (!pool[i].llr[k]) return fail(SYNDROME_NULL_POINTER, "pool LLR pointer is null");
    std::string err;
    const int r = syn::run_load(server->engine, pool, pool_n, *spec, report, latencies_us, latencies_cap, &err);
    return r == SYNDROME_OK ? SYNDROME_OK : fail(r, err);
  });
}

}  // extern "C"
