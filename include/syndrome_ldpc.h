/*
 * syndrome_ldpc.h - C ABI of the B200 QC-LDPC layered offset min-sum decoder.
 *
 * Three groups of entry points:
 *
 *  1. The drop-in set.  Same symbol names, argument order, argument meaning,
 *     buffer ownership and status codes as the reference's C ABI crate
 *     (syndrome capi/src/lib.rs); each declaration cites the function it
 *     replaces.  Buffers are host memory owned by the caller; the decode runs
 *     on the current CUDA device and returns when the results are in the
 *     caller's buffers.
 *  2. The rest of the reference's Rust decoder API (src/qc_ldpc.rs,
 *     src/wifi_ldpc_tables.rs, src/quantize.rs, src/channel_sim.rs) as C
 *     functions, so a Rust shim can keep QcLdpcDecoder's method set.
 *  3. The batched device API: device pointers, a caller-supplied CUDA stream,
 *     many codewords per call, packed hard decisions.  This is the GPU-native
 *     path the drop-in set is built on; it has no counterpart in the reference
 *     (which decodes one codeword per call on one CPU thread).
 *
 * Status codes are the reference's SyndromeStatus (capi/src/lib.rs:73-94) plus
 * SYNDROME_CUDA_ERROR.  No function allocates on the decode path except the
 * host-buffer wrappers of group 1/2, which keep per-handle device staging
 * buffers (allocated on first use, reused, freed by *_destroy).
 */
#ifndef SYNDROME_LDPC_H
#define SYNDROME_LDPC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* SyndromeStatus, capi/src/lib.rs:73-94. */
#define SYNDROME_OK 0
#define SYNDROME_INVALID_PARAM (-1)
#define SYNDROME_CRC_MISMATCH (-2)
#define SYNDROME_DECODER_NOT_CONVERGED (-3) /* reserved, never returned (as in the reference) */
#define SYNDROME_BUFFER_TOO_SMALL (-4)
#define SYNDROME_NULL_POINTER (-5)
#define SYNDROME_PANIC (-6)                 /* an internal C++ exception was caught */
#define SYNDROME_CUDA_ERROR (-7)            /* no counterpart in the reference: a CUDA call failed */

/* Precision selector of the batched API. */
#define SYNDROME_PRECISION_INT8 0
#define SYNDROME_PRECISION_F32 1

typedef struct SyndromeLdpcDecoder SyndromeLdpcDecoder;
typedef struct SyndromeLdpcEncoder SyndromeLdpcEncoder;

/* ===================================================== 1. drop-in set ===== */

/* capi/src/lib.rs:148 syndrome_ldpc_decoder_create.  base_graph 0 = BG1, 1 = BG2;
 * z must be a 3GPP lifting size.  *out_decoder is set to NULL on failure. */
int32_t syndrome_ldpc_decoder_create(int32_t base_graph, size_t z, float offset_beta,
                                     SyndromeLdpcDecoder** out_decoder);
/* capi/src/lib.rs:187.  NULL is a no-op. */
void syndrome_ldpc_decoder_destroy(SyndromeLdpcDecoder* decoder);
/* capi/src/lib.rs:202 (N = n_b * Z). */
size_t syndrome_ldpc_decoder_variable_node_count(const SyndromeLdpcDecoder* decoder);
/* capi/src/lib.rs:216 (K = k_b * Z, filler bits included). */
size_t syndrome_ldpc_decoder_info_bit_count(const SyndromeLdpcDecoder* decoder);
/* capi/src/lib.rs:230 (edges * Z). */
size_t syndrome_ldpc_decoder_required_edge_buffer(const SyndromeLdpcDecoder* decoder);
/* capi/src/lib.rs:245 (max layer degree * Z). */
size_t syndrome_ldpc_decoder_required_layer_buffer(const SyndromeLdpcDecoder* decoder);
/* capi/src/lib.rs:290 syndrome_ldpc_decode_5g -> QcLdpcDecoder::decode_5g
 * (src/qc_ldpc.rs:644): 5G prologue on llr (filler = 1e6, [0,2Z) = 0), then f32
 * LOMS.  llr becomes the posterior, edge_r the final C->V messages, hard the hard
 * decisions.  llr_len and hard_output_len must equal N (INVALID_PARAM); edge_r and
 * layer_scratch must hold at least the required sizes (BUFFER_TOO_SMALL).
 * layer_scratch is validated but not written. */
int32_t syndrome_ldpc_decode_5g(SyndromeLdpcDecoder* decoder, float* llr, size_t llr_len,
                                size_t n_filler, float* edge_r, size_t edge_r_len,
                                float* layer_scratch, size_t layer_scratch_len,
                                uint8_t* hard_output, size_t hard_output_len, size_t iterations,
                                size_t* out_iterations_used);
/* capi/src/lib.rs:369. */
int32_t syndrome_ldpc_encoder_create(int32_t base_graph, size_t z,
                                     SyndromeLdpcEncoder** out_encoder);
/* capi/src/lib.rs:407.  NULL is a no-op. */
void syndrome_ldpc_encoder_destroy(SyndromeLdpcEncoder* encoder);
/* capi/src/lib.rs:422. */
size_t syndrome_ldpc_encoder_info_bit_count(const SyndromeLdpcEncoder* encoder);
/* capi/src/lib.rs:436. */
size_t syndrome_ldpc_encoder_codeword_bit_count(const SyndromeLdpcEncoder* encoder);
/* capi/src/lib.rs:461 -> QcLdpcEncoder::encode_5g (src/qc_ldpc.rs:2547): info_len
 * must equal K - n_filler, codeword_len must equal N (BUFFER_TOO_SMALL). */
int32_t syndrome_ldpc_encode_5g(const SyndromeLdpcEncoder* encoder, const uint8_t* info_bits,
                                size_t info_len, size_t n_filler, uint8_t* codeword,
                                size_t codeword_len);

/* ====================================== 2. rest of the reference API ===== */

/* src/wifi_ldpc_tables.rs:521 wifi_ldpc_decoder (802.11, Z in {27,54,81}). */
int32_t syndrome_ldpc_decoder_create_wifi(size_t z, size_t rate_num, size_t rate_den,
                                          float offset_beta, SyndromeLdpcDecoder** out_decoder);
/* src/qc_ldpc.rs:566 QcLdpcDecoder::from_raw_edges.  Literal (row, col, shift)
 * triples, shift < z <= 384.  Additionally rejects a column that appears twice in
 * one layer (INVALID_PARAM): the GPU kernels update a layer's variables in
 * parallel. */
int32_t syndrome_ldpc_decoder_create_raw(const uint8_t* rows, const uint8_t* cols,
                                         const int16_t* shifts, size_t n_edges,
                                         size_t num_row_blocks, size_t num_col_blocks, size_t z,
                                         float offset_beta, SyndromeLdpcDecoder** out_decoder);
/* src/qc_ldpc.rs:588 (M = m_b * Z). */
size_t syndrome_ldpc_decoder_check_node_count(const SyndromeLdpcDecoder* decoder);
/* Lifting size and block dimensions: out[0..4] = {z, m_b, n_b, edges, max layer degree}. */
int32_t syndrome_ldpc_decoder_dims(const SyndromeLdpcDecoder* decoder, size_t* out5);
/* src/qc_ldpc.rs:711 init_5g_llr (host buffer, no GPU work). */
int32_t syndrome_ldpc_init_5g_llr(const SyndromeLdpcDecoder* decoder, float* llr, size_t llr_len,
                                  size_t n_filler);
/* src/qc_ldpc.rs:794 decode_layered_offset_min_sum (f32, no prologue).  Same
 * buffers and errors as syndrome_ldpc_decode_5g. */
int32_t syndrome_ldpc_decode(SyndromeLdpcDecoder* decoder, float* llr, size_t llr_len,
                             float* edge_r, size_t edge_r_len, float* layer_scratch,
                             size_t layer_scratch_len, uint8_t* hard_output,
                             size_t hard_output_len, size_t iterations,
                             size_t* out_iterations_used);
/* src/qc_ldpc.rs:1345 decode_layered_offset_min_sum_i8: int8 messages, int16
 * posterior.  QuantParams is passed as (scale, app_clamp) (src/quantize.rs:217);
 * beta_q = round(offset_beta * scale) clamped to [0,127].  app is clamped to
 * +-max(app_clamp, 0) on entry and becomes the posterior. */
int32_t syndrome_ldpc_decode_i8(SyndromeLdpcDecoder* decoder, int16_t* app, size_t app_len,
                                int8_t* edge_r, size_t edge_r_len, int8_t* layer_scratch,
                                size_t layer_scratch_len, uint8_t* hard_output,
                                size_t hard_output_len, size_t iterations, float scale,
                                int16_t app_clamp, size_t* out_iterations_used);
/* src/qc_ldpc.rs:1486 decode_5g_i8: filler = max(app_clamp, 0), [0,2Z) = 0, then
 * the int8 decode. */
int32_t syndrome_ldpc_decode_5g_i8(SyndromeLdpcDecoder* decoder, int16_t* app, size_t app_len,
                                   size_t n_filler, int8_t* edge_r, size_t edge_r_len,
                                   int8_t* layer_scratch, size_t layer_scratch_len,
                                   uint8_t* hard_output, size_t hard_output_len,
                                   size_t iterations, float scale, int16_t app_clamp,
                                   size_t* out_iterations_used);
/* src/wifi_ldpc_tables.rs:490 wifi_ldpc_encoder. */
int32_t syndrome_ldpc_encoder_create_wifi(size_t z, size_t rate_num, size_t rate_den,
                                          SyndromeLdpcEncoder** out_encoder);
/* src/qc_ldpc.rs:2592 QcLdpcEncoder::encode (info_len == K, codeword_len == N). */
int32_t syndrome_ldpc_encode(const SyndromeLdpcEncoder* encoder, const uint8_t* info_bits,
                             size_t info_len, uint8_t* codeword, size_t codeword_len);
/* Many codewords at once on `threads` host threads (0 = all cores); row strides in bytes. */
int32_t syndrome_ldpc_encode_batch(const SyndromeLdpcEncoder* encoder, const uint8_t* info_bits,
                                   size_t info_stride, uint8_t* codewords, size_t codeword_stride,
                                   size_t count, int32_t threads);
/* ------------------------------------ Wi-Fi shortening and puncturing ---- */
/* src/wifi_rate_matching.rs:88 shortening_and_puncture_counts: n_shrt = k - payload_bits,
 * n_punc = (n - n_shrt) - target_coded_bits.  INVALID_PARAM when n < k,
 * payload_bits > k, target_coded_bits < payload_bits or target_coded_bits > n - n_shrt. */
int32_t syndrome_wifi_shortening_counts(size_t k, size_t n, size_t payload_bits, size_t target_coded_bits,
                                        size_t* out_n_shrt, size_t* out_n_punc);
/* src/wifi_rate_matching.rs:163 encode_shortened: payload padded with zeros to K,
 * encoded, then the payload and the first (N - K) - n_punc parity bits are sent
 * (out_len == target_coded_bits, else BUFFER_TOO_SMALL). */
int32_t syndrome_wifi_encode_shortened(const SyndromeLdpcEncoder* encoder, const uint8_t* payload,
                                       size_t payload_bits, size_t target_coded_bits, uint8_t* out,
                                       size_t out_len);
/* src/wifi_rate_matching.rs:267 decode_shortened: codeword_llr (length N, else
 * BUFFER_TOO_SMALL) is rebuilt from rx_llr (rx_len = target_coded_bits) -- payload,
 * 1e6 for the shortened bits, the sent parity, 0 for the punctured bits -- and decoded
 * in place as syndrome_ldpc_decode does (it ends as the posterior).  The payload is
 * hard_output[0 .. payload_bits). */
int32_t syndrome_wifi_decode_shortened(SyndromeLdpcDecoder* decoder, size_t payload_bits, const float* rx_llr,
                                       size_t rx_len, float* codeword_llr, size_t codeword_len,
                                       float* edge_r, size_t edge_r_len, float* layer_scratch,
                                       size_t layer_scratch_len, uint8_t* hard_output, size_t hard_output_len,
                                       size_t iterations, size_t* out_iterations_used);
/* Batched form on the device: row b of d_rx (d_rx[b * rx_stride + t], t <
 * target_coded_bits) is one received shortened / punctured codeword; the f32 kernel
 * rebuilds the full codeword while loading it (no N-length staging buffer).  Outputs
 * as syndrome_ldpc_decode_batch_f32; the payload is the first payload_bits hard
 * decisions. */
int32_t syndrome_wifi_decode_shortened_batch_f32(const SyndromeLdpcDecoder* decoder, const float* d_rx,
                                                 size_t rx_stride, size_t payload_bits, size_t target_coded_bits,
                                                 size_t batch, size_t iterations, uint32_t* d_hard_packed,
                                                 size_t hard_bits, size_t hard_words_stride, int32_t* d_iters,
                                                 float* d_app, size_t app_stride, float* d_edge_r,
                                                 size_t edge_r_stride, uint8_t* d_hard, size_t hard_stride,
                                                 void* d_workspace, size_t workspace_bytes, void* stream);
/* The same batch encoded on the GPU (src/qc_ldpc.rs:2592-2727 codewords, which are
 * unique): d_info [count][info_stride] and d_codewords [count][codeword_stride] are
 * device arrays, one bit per byte; enqueued on `stream` (cudaStream_t, NULL = legacy
 * default stream).  The encoder's tables are copied to the current device on the
 * first call; later calls must use the same device (else CUDA_ERROR). */
int32_t syndrome_ldpc_encode_batch_device(const SyndromeLdpcEncoder* encoder, const uint8_t* d_info,
                                          size_t info_stride, uint8_t* d_codewords, size_t codeword_stride,
                                          size_t count, void* stream);
/* src/quantize.rs:331 quantize_llr_i16. */
void syndrome_quantize_llr_i16(const float* llr, int16_t* out, size_t n, float scale);
/* src/quantize.rs:298 QuantParams::beta_q. */
int32_t syndrome_beta_q(float offset_beta, float scale);
/* src/channel_sim.rs:139 AwgnChannel::new(ebno_db, rate, seed).transmit(bits). */
void syndrome_awgn_llr(float ebno_db, float code_rate, uint64_t seed, const uint8_t* bits,
                       size_t n, float* llr_out);
/* Batch of AwgnChannel::transmit + quantize to int8: codeword b uses seeds[b] and
 * ebno_db[b]; bits [tx_begin, n) of row b are written to out + b * out_stride. */
void syndrome_awgn_quantized_batch(const uint8_t* bits, size_t n, size_t bits_stride,
                                   size_t tx_begin, const float* ebno_db, float code_rate,
                                   const uint64_t* seeds, float scale, int8_t* out,
                                   size_t out_stride, size_t count, int32_t threads);

/* ------------------------------------------------------ frame pipeline ---- */
/* src/ldpc_pipeline.rs:288-598 LdpcPipeline.  A pool of N-length f32 frames in pinned
 * host memory: acquire a frame (its index; -1 when every frame is in use), fill its
 * LLRs, submit it; host worker threads (n_workers, clamped to 1..8; 0 = one per core
 * as LdpcPipeline::new, clamped the same way) decode submitted frames in batches on
 * their own CUDA streams (decode_layered_offset_min_sum: the frame's LLRs become the
 * posterior, hard decisions and iterations used are filled in); try_recv returns
 * decoded frames in completion order (-1 when none is ready), release returns a
 * frame to the pool.  The pool holds 256 frames (the reference's 16 is too few to
 * keep a GPU busy).  The decoder must outlive the pipeline. */
typedef struct SyndromeLdpcPipeline SyndromeLdpcPipeline;
int32_t syndrome_ldpc_pipeline_create(const SyndromeLdpcDecoder* decoder, size_t iterations, size_t n_workers,
                                      SyndromeLdpcPipeline** out_pipeline);
void syndrome_ldpc_pipeline_destroy(SyndromeLdpcPipeline* pipeline);
size_t syndrome_ldpc_pipeline_worker_count(const SyndromeLdpcPipeline* pipeline);
size_t syndrome_ldpc_pipeline_pool_size(const SyndromeLdpcPipeline* pipeline);
int64_t syndrome_ldpc_pipeline_acquire(SyndromeLdpcPipeline* pipeline);
/* INVALID_PARAM unless the frame was acquired and not yet submitted. */
int32_t syndrome_ldpc_pipeline_submit(SyndromeLdpcPipeline* pipeline, int64_t frame);
int64_t syndrome_ldpc_pipeline_try_recv(SyndromeLdpcPipeline* pipeline);
/* INVALID_PARAM unless the frame was received (or acquired and not submitted). */
int32_t syndrome_ldpc_pipeline_release(SyndromeLdpcPipeline* pipeline, int64_t frame);
/* LdpcFrame accessors: N f32 LLRs (the posterior after decoding), N hard decisions,
 * iterations used, the caller's tag.  NULL / 0 for an invalid frame index. */
float* syndrome_ldpc_pipeline_frame_llr(SyndromeLdpcPipeline* pipeline, int64_t frame);
const uint8_t* syndrome_ldpc_pipeline_frame_hard(const SyndromeLdpcPipeline* pipeline, int64_t frame);
size_t syndrome_ldpc_pipeline_frame_iterations(const SyndromeLdpcPipeline* pipeline, int64_t frame);
void syndrome_ldpc_pipeline_frame_set_tag(SyndromeLdpcPipeline* pipeline, int64_t frame, size_t tag);
size_t syndrome_ldpc_pipeline_frame_tag(const SyndromeLdpcPipeline* pipeline, int64_t frame);

/* ================================================= 3. batched device API == */

/* Device scratch bytes that syndrome_ldpc_decode_batch_* needs for `batch`
 * codewords when d_edge_r is NULL. */
size_t syndrome_ldpc_batch_workspace_size(const SyndromeLdpcDecoder* decoder, int32_t precision,
                                          size_t batch);
/* Batched int8 decode.  Codeword b's int8 channel LLRs are
 * d_llr[b * llr_stride + j] for variables llr_offset + j (j < N - llr_offset);
 * variables [0, llr_offset) start at 0.  nr_prologue != 0 applies decode_5g_i8's
 * initialisation.  Outputs (all device memory, each optional):
 *   d_hard_packed[b * hard_words_stride + w]: bit t of word w = hard decision of
 *     variable 32w + t, for the first hard_bits variables;
 *   d_iters[b]: iterations used (early stop on a zero syndrome);
 *   d_app[b * app_stride + i]: final int16 posterior;
 *   d_edge_r[b * edge_r_stride + e]: final C->V messages (reference layout);
 *   d_hard[b * hard_stride + i]: hard decisions, one byte per variable.
 * Enqueued on `stream` (a cudaStream_t; NULL = legacy default stream). */
int32_t syndrome_ldpc_decode_batch_i8(const SyndromeLdpcDecoder* decoder, const int8_t* d_llr,
                                      size_t llr_stride, size_t llr_offset, size_t batch,
                                      int32_t nr_prologue, size_t n_filler, size_t iterations,
                                      float scale, int16_t app_clamp, uint32_t* d_hard_packed,
                                      size_t hard_bits, size_t hard_words_stride, int32_t* d_iters,
                                      int16_t* d_app, size_t app_stride, int8_t* d_edge_r,
                                      size_t edge_r_stride, uint8_t* d_hard, size_t hard_stride,
                                      void* d_workspace, size_t workspace_bytes, void* stream);
/* Batched f32 decode (decode_layered_offset_min_sum / decode_5g semantics). */
int32_t syndrome_ldpc_decode_batch_f32(const SyndromeLdpcDecoder* decoder, const float* d_llr,
                                       size_t llr_stride, size_t llr_offset, size_t batch,
                                       int32_t nr_prologue, size_t n_filler, size_t iterations,
                                       uint32_t* d_hard_packed, size_t hard_bits,
                                       size_t hard_words_stride, int32_t* d_iters, float* d_app,
                                       size_t app_stride, float* d_edge_r, size_t edge_r_stride,
                                       uint8_t* d_hard, size_t hard_stride, void* d_workspace,
                                       size_t workspace_bytes, void* stream);
/* Allocation-free batched int8 decode.  No counterpart in the reference.
 * For callers that cannot allocate device memory while decoding: a baseband thread
 * working to a per-slot deadline must not call cudaMalloc (it can synchronise the
 * device and take milliseconds), and a plug-in inside an application that owns all
 * device allocations has no allocator to call.  Same arguments and results as
 * syndrome_ldpc_decode_batch_i8 without the workspace.  On 5G NR graphs it runs the
 * kernel syndrome_ldpc_decoder_set_kernel chose (the NR kernels keep their state on
 * chip and need no device memory) unless that is 1 or 4; otherwise the generic int8
 * kernel keeps its messages in a static device array of SYNDROME_NOALLOC_SCRATCH_BYTES
 * that every GPU loading this library holds until exit.  A launch runs at most
 * SYNDROME_NOALLOC_SCRATCH_BYTES / (codewords per CTA * edges * Z) CTAs; a code whose
 * per-CTA messages exceed the array is rejected with SYNDROME_INVALID_PARAM.  The
 * first call on a device looks up the array's address (cudaGetSymbolAddress), so make
 * that first call before any stream capture; the address is kept for the process, so
 * calls must not cross a cudaDeviceReset.  Nothing in the array must start at zero
 * and it keeps the last call's contents; calls that overlap on the GPU share the
 * array and race.  The current device must be the decoder's.  The array is used when
 * d_edge_r is NULL (with d_edge_r the messages go there instead).  The generic path
 * runs at the throughput of kernel 4 (messages in global memory) and every call
 * queries that kernel's occupancy on the host. */
#define SYNDROME_NOALLOC_SCRATCH_BYTES (32u << 20)
int32_t syndrome_ldpc_decode_batch_i8_noalloc(const SyndromeLdpcDecoder* decoder,
                                              const int8_t* d_llr, size_t llr_stride,
                                              size_t llr_offset, size_t batch, int32_t nr_prologue,
                                              size_t n_filler, size_t iterations, float scale,
                                              int16_t app_clamp, uint32_t* d_hard_packed,
                                              size_t hard_bits, size_t hard_words_stride,
                                              int32_t* d_iters, int16_t* d_app, size_t app_stride,
                                              int8_t* d_edge_r, size_t edge_r_stride,
                                              uint8_t* d_hard, size_t hard_stride, void* stream);
/* Kernel selection for this decoder's batched int8 decodes: 0 = automatic (the
 * paired 5G NR kernel when it applies, else the 5G NR kernel, else the generic
 * layered kernel), 1 = always the generic kernel, 2 = require the 5G NR kernel,
 * 3 = require the paired 5G NR kernel (two codewords per 32-bit word; needs
 * app_clamp >= 3938, or >= 7874 with filler bits), 4 = the generic kernel with its
 * check-to-variable messages in global memory (1 keeps them compressed in shared
 * memory where they fit), 5 = the paired kernel with all its check-row state in
 * shared memory, one codeword pair per SM (at Z = 384, 0 and 3 run the variant that
 * keeps most of that state in tensor memory, two pairs per SM).  2, 3 and 5 return
 * INVALID_PARAM on a request they cannot serve.  All kernels produce identical
 * results. */
int32_t syndrome_ldpc_decoder_set_kernel(SyndromeLdpcDecoder* decoder, int32_t kernel);
/* ----------------------------------------------- mixed-shape batches ---- */
/* One codeword of a mixed 5G NR int8 batch.  No counterpart in the reference
 * (it decodes one code block per call).  Its int8 LLRs cover variables 2Z..N (the
 * circular buffer of rate matching; the first 2Z columns are punctured) and start
 * llr_offset bytes into the batch's LLR buffer; its hard decisions of variables
 * 0..hard_bits-1 are written LSB-first from word out_offset of the output. */
typedef struct {
  int32_t base_graph; /* 0 = BG1, 1 = BG2 */
  int32_t z;          /* lifting size */
  int32_t n_filler;   /* filler bits K - K' (decode_5g_i8 prologue) */
  int32_t hard_bits;  /* leading variables reported, e.g. K' information bits */
  int64_t llr_offset;
  int64_t out_offset;
} SyndromeMixedCodeword;

typedef struct SyndromeMixedPlan SyndromeMixedPlan;

/* Plans a batch of codewords of any BG / Z mix for one persistent launch: groups
 * equal shapes into work items of at most a tile of codewords (tile_hints: n_hints
 * triples (base_graph, z, tile), nullable; default = what one CTA holds), orders the
 * items by decreasing work and uploads the tables.  int8 LOMS with beta_q =
 * round(offset_beta * scale), app_clamp >= 255, at most `iterations` iterations with
 * early stop. */
int32_t syndrome_mixed_plan_create(const SyndromeMixedCodeword* codewords, size_t count, float offset_beta,
                                   float scale, int16_t app_clamp, size_t iterations,
                                   const int32_t* tile_hints, size_t n_hints, SyndromeMixedPlan** out_plan);
void syndrome_mixed_plan_destroy(SyndromeMixedPlan* plan);
/* Number of work items; out_items (nullable, room for `cap` items) receives
 * (base_graph, z, codewords) per item in launch order. */
int32_t syndrome_mixed_plan_items(const SyndromeMixedPlan* plan, int32_t* out_items, size_t cap, size_t* n_items);
/* Kernel of the plan's decode: 0 = automatic (the default; the paired kernel keeps
 * most of its check-row state in tensor memory, two CTAs per SM, when app_clamp >=
 * 7874 and no codeword reports hard decisions past its core columns, 26Z for BG1 and
 * 14Z for BG2), 5 = the paired kernel with all check-row state in shared memory, one
 * CTA per SM.  Other values give SYNDROME_INVALID_PARAM.  Both produce identical
 * results.  *is_tmem (nullable) receives 1 when decode runs the tensor-memory form. */
int32_t syndrome_mixed_plan_set_kernel(SyndromeMixedPlan* plan, int32_t kernel, int32_t* is_tmem);
/* Most codewords one work item of this shape can hold with the default app_clamp
 * (paired kernel; plans with app_clamp below 7874 use smaller items). */
int32_t syndrome_mixed_tile_capacity(int32_t base_graph, int32_t z);
/* Decodes the planned batch from device LLRs (llr_bytes long) into d_hard_packed
 * (out_words long); d_iters (nullable, iters_len entries) receives the iterations of
 * codeword i at index i.  Buffers shorter than the plan's offsets need give
 * SYNDROME_BUFFER_TOO_SMALL.  use_graph != 0 captures the launch into a CUDA graph on
 * first use (per buffer set) and replays it afterwards. */
int32_t syndrome_mixed_decode(SyndromeMixedPlan* plan, const int8_t* d_llr, size_t llr_bytes,
                              uint32_t* d_hard_packed, size_t out_words, int32_t* d_iters, size_t iters_len,
                              int32_t use_graph, void* stream);

/* One codeword of a mixed batch of 802.11 codewords (f32).  No counterpart in the
 * reference, which decodes one codeword per call (decode_layered_offset_min_sum,
 * src/qc_ldpc.rs:962, on the matrices of src/wifi_ldpc_tables.rs:339-453).  Its N f32
 * channel LLRs start llr_offset elements into the batch's LLR buffer; its hard
 * decisions of variables 0..hard_bits-1 are written LSB-first from word out_offset. */
typedef struct {
  int32_t z;         /* 27, 54 or 81 (n = 648, 1296, 1944) */
  int32_t rate_num;  /* rate 1/2, 2/3, 3/4 or 5/6 */
  int32_t rate_den;
  int32_t hard_bits; /* leading variables reported, e.g. the K information bits */
  int64_t llr_offset;
  int64_t out_offset;
} SyndromeWifiMixedCodeword;

typedef struct SyndromeWifiMixedPlan SyndromeWifiMixedPlan;

/* Plans a batch of codewords of any mix of the twelve 802.11 matrices for one
 * persistent f32 launch: codewords grouped by matrix into chunks of `chunk` codewords
 * (0: about four chunks per CTA over the batch, at least four codewords) on a
 * device queue, the costliest matrices
 * first; every codeword slot of a CTA takes the next codeword as soon as its own
 * stops (zero syndrome or `iterations`), so skewed iteration counts keep the slots
 * busy.  f32 layered offset min-sum with offset_beta. */
int32_t syndrome_wifi_mixed_plan_create(const SyndromeWifiMixedCodeword* codewords, size_t count, float offset_beta,
                                        size_t iterations, size_t chunk, SyndromeWifiMixedPlan** out_plan);
void syndrome_wifi_mixed_plan_destroy(SyndromeWifiMixedPlan* plan);
/* Chunks on the plan's queue and CTAs of its launch (ctas nullable). */
int32_t syndrome_wifi_mixed_plan_chunks(const SyndromeWifiMixedPlan* plan, size_t* n_chunks, size_t* ctas);
/* Decodes the planned batch from device LLRs (llr_len floats) into d_hard_packed
 * (out_words long); d_iters (nullable, iters_len entries) receives the iterations of
 * codeword i at index i.  Buffers shorter than the plan's offsets need give
 * SYNDROME_BUFFER_TOO_SMALL.  use_graph != 0 captures the launch into a CUDA graph on
 * first use (per buffer set) and replays it afterwards. */
int32_t syndrome_wifi_mixed_decode(SyndromeWifiMixedPlan* plan, const float* d_llr, size_t llr_len,
                                   uint32_t* d_hard_packed, size_t out_words, int32_t* d_iters, size_t iters_len,
                                   int32_t use_graph, void* stream);

/* ===================================== 4. transport blocks (DL-SCH) ===== */

/* src/segmentation.rs:265 compute_segmentation.  out10 = {base graph (0 = BG1),
 * Z, C code blocks, B = A + 24, K', K, Ncb = N - 2Z, filler bits, has CB CRC,
 * TB bits per code block}. */
int32_t syndrome_tb_segmentation(size_t tb_size, float target_rate, int64_t* out10);
/* src/crc.rs:153 Crc24::compute over n bits (one per byte, LSB used): kind 0 =
 * CRC-24A (0x864CFB), 1 = CRC-24B (0x800063).  MSB-first, zero initial value. */
uint32_t syndrome_crc24(const uint8_t* bits, size_t n, int32_t kind);

typedef struct SyndromeDlSchEncoder SyndromeDlSchEncoder;
/* src/transport_block.rs:221 DlSchEncoder::new(tb_size, target_rate, qm, g).
 * Additionally rejects an E per code block that the reference's rate-matching walk
 * would not fill (code rates far below 1/5). */
int32_t syndrome_dlsch_encoder_create(size_t tb_size, float target_rate, size_t qm, size_t g,
                                      SyndromeDlSchEncoder** out_encoder);
void syndrome_dlsch_encoder_destroy(SyndromeDlSchEncoder* encoder);
/* src/transport_block.rs:275 output_bits (C * E). */
size_t syndrome_dlsch_encoder_output_bits(const SyndromeDlSchEncoder* encoder);
/* src/transport_block.rs:280 num_code_blocks. */
size_t syndrome_dlsch_encoder_num_code_blocks(const SyndromeDlSchEncoder* encoder);
/* src/transport_block.rs:303 encode: TB CRC-24A, segmentation with CRC-24B, LDPC
 * encoding, rate matching for redundancy version rv.  tb_len must equal tb_size and
 * out_len be at least output_bits (BUFFER_TOO_SMALL); rv > 3 is INVALID_PARAM. */
int32_t syndrome_dlsch_encode(const SyndromeDlSchEncoder* encoder, const uint8_t* tb, size_t tb_len,
                              size_t rv, uint8_t* out, size_t out_len);
/* src/transport_block.rs:405-1060 DlSchDecoder with the f32 code-block decode: HARQ
 * f32 soft combining into device accumulators, the 5G prologue, all C code blocks
 * decoded in one batched f32 launch (decode_layered_offset_min_sum), CB CRC-24B, TB
 * CRC-24A, HARQ flush on success.  create: INVALID_PARAM for tb_size 0, Qm or G 0 or
 * G % Qm != 0, or a TB size segmentation rejects (transport_block.rs:612-627). */
typedef struct SyndromeDlSchDecoder SyndromeDlSchDecoder;
typedef struct {
  int32_t crc_ok;          /* TB CRC-24A and every CB CRC-24B passed */
  int32_t max_iters_used;  /* largest iteration count over the code blocks */
  int32_t harq_tx_count;   /* transmissions combined, this one included */
  int32_t num_code_blocks;
} SyndromeDecodeReport;
int32_t syndrome_dlsch_decoder_create(size_t tb_size, float target_rate, size_t qm, size_t g, size_t iterations,
                                      float offset_beta, SyndromeDlSchDecoder** out_decoder);
void syndrome_dlsch_decoder_destroy(SyndromeDlSchDecoder* decoder);
size_t syndrome_dlsch_decoder_num_code_blocks(const SyndromeDlSchDecoder* decoder);
size_t syndrome_dlsch_decoder_output_bits(const SyndromeDlSchDecoder* decoder);
/* :729 with_pipeline.  Accepted for API parity (INVALID_PARAM for 0): every decode
 * already runs its code blocks concurrently in one batched GPU launch; the count is
 * what worker_count reports (0 before any with_pipeline call). */
int32_t syndrome_dlsch_decoder_with_pipeline(SyndromeDlSchDecoder* decoder, size_t n_workers);
size_t syndrome_dlsch_decoder_worker_count(const SyndromeDlSchDecoder* decoder);
/* :829 decode.  rx_llr holds C * E f32 LLRs (else BUFFER_TOO_SMALL), tb_len >= tb_size
 * (else BUFFER_TOO_SMALL), rv 0..3.  tb_out is written only when crc_ok.  cb_crc
 * (nullable, cb_crc_len >= C) receives each code block's CRC-24B result. */
int32_t syndrome_dlsch_decode(SyndromeDlSchDecoder* decoder, const float* rx_llr, size_t rx_len, size_t rv,
                              uint8_t* tb_out, size_t tb_len, SyndromeDecodeReport* report, uint8_t* cb_crc,
                              size_t cb_crc_len);
/* :1055 flush_harq. */
void syndrome_dlsch_decoder_flush_harq(SyndromeDlSchDecoder* decoder);

/* ============================================ 5. transport-block serving ===== */
/* A device-resident serving engine for DL-SCH transmissions.  No single counterpart
 * in the reference: it replaces DlSchDecoder::decode (src/transport_block.rs:829)
 * driven by LdpcPipeline (src/ldpc_pipeline.rs) with continuous batching on one GPU.
 * Per transmission the results are those of DlSchDecoder::decode with the int8
 * code-block decode: HARQ soft combining (src/harq.rs:142) in f32 accumulators that
 * stay in device memory across retransmissions, quantize_llr_i16, decode_5g_i8,
 * CRC-24B per code block, CRC-24A per transport block, accumulators flushed when
 * both pass.  A worker thread forms GPU steps from the submission queue in arrival
 * order while earlier steps run; a new transport block is admitted when its HARQ
 * accumulators fit the HBM budget (otherwise it and the new blocks behind it wait;
 * retransmissions of blocks that hold accumulators go ahead). */
typedef struct SyndromeServer SyndromeServer;
typedef struct {
  uint32_t max_step_code_blocks; /* code blocks per GPU step, >= 160 (0 = 2048); the
                                    continuous engine holds max_step_code_blocks *
                                    steps_in_flight code blocks in flight */
  uint32_t steps_in_flight;      /* 1..16 (0 = 6): steps run concurrently on free SMs */
  uint64_t harq_bytes;           /* device memory for HARQ accumulators (0 = 8 GiB) */
  uint64_t staging_bytes;        /* device staging for host-memory LLRs, per step (the
                                    continuous engine: in all) (0 = 256 MiB) */
  int32_t iterations;            /* maximum LOMS iterations (early stop on a zero syndrome) */
  float offset_beta;             /* beta_q = round(offset_beta * scale) clamped to [0, 127] */
  float scale;                   /* LLR quantizer scale (src/quantize.rs DEFAULT_SCALE = 8) */
  int32_t app_clamp;             /* posterior clamp, >= 255 */
  uint32_t latency_steps;        /* steps in flight while few code blocks wait (0 = 3, at most
                                    steps_in_flight): fewer steps share the SMs, each ends sooner */
  uint32_t backlog_code_blocks;  /* waiting code blocks from which up to steps_in_flight steps
                                    run (0 = 128) */
  int32_t decode_kernel;         /* 0 = the paired kernel with its check-row state mostly in
                                    tensor memory (two CTAs per SM), 5 = all of it in shared
                                    memory (one CTA per SM); identical results */
  int32_t engine;                /* 0 = continuous: one persistent kernel takes each
                                    transmission's code blocks as they arrive (with
                                    decode_kernel 0 and app_clamp >= 7874; otherwise steps),
                                    1 = steps of up to max_step_code_blocks, up to
                                    steps_in_flight at once; identical results */
  uint32_t idle_us;              /* continuous engine: the kernel exits after this long
                                    without work and is relaunched with the next
                                    transmission (0 = 2000) */
} SyndromeServeConfig;
typedef struct {
  uint64_t tb_id;
  int32_t crc_ok;                /* DecodeReport::crc_ok */
  int32_t max_iters_used;        /* DecodeReport::max_iters_used */
  int32_t harq_tx_count;         /* DecodeReport::harq_tx_count */
  int32_t num_code_blocks;
  uint32_t cb_crc[5];            /* DecodeReport::cb_crc: bit i = code block i passed */
  uint32_t reserved;
  double latency_us;             /* submit to completion */
} SyndromeServeResult;
int32_t syndrome_serve_create(const SyndromeServeConfig* config, SyndromeServer** out_server);
void syndrome_serve_destroy(SyndromeServer* server);
/* Queues one transmission of transport block tb_id (DlSchDecoder::new parameters
 * tb_size, target_rate, qm, g plus the redundancy version rv): llr holds C * E f32
 * channel LLRs (E = floor(g / C / qm) * qm), in device memory when llr_on_device,
 * else host memory.  The buffer must stay valid until this transmission's result
 * has been polled.  A new tb_id starts with empty accumulators; a tb_id whose last
 * transmission failed keeps them (retransmission).  Reusing a tb_id with other
 * parameters, or while one of its transmissions is in flight, is INVALID_PARAM. */
int32_t syndrome_serve_submit(SyndromeServer* server, uint64_t tb_id, size_t tb_size, float target_rate,
                              size_t qm, size_t g, size_t rv, const float* llr, size_t llr_len,
                              int32_t llr_on_device);
/* Up to cap completed transmissions, waiting up to timeout_us for the first. */
int32_t syndrome_serve_poll(SyndromeServer* server, SyndromeServeResult* out, size_t cap, size_t* n_out,
                            int64_t timeout_us);
/* Payload of tb_id's last decode, one bit per byte (the tb_out of a passing decode). */
int32_t syndrome_serve_fetch(SyndromeServer* server, uint64_t tb_id, uint8_t* tb_bits, size_t tb_len);
/* Forgets tb_id and frees its accumulators (after success, or when giving up). */
int32_t syndrome_serve_release(SyndromeServer* server, uint64_t tb_id);
/* out14 = {steps, code blocks, transmissions, HARQ bytes in use, queued, steps in flight,
 * transport blocks held, largest queue seen, decode work items, threads those items
 * occupy (of 384 per item), GPU microseconds in the decode launches, GPU microseconds
 * from each step's first copy to its last, worker microseconds building steps,
 * worker microseconds finishing steps}. */
int32_t syndrome_serve_stats(SyndromeServer* server, int64_t* out14);
/* Continuous engine (zeros for the step engine): out10 = {work items the persistent
 * kernel finished, then microseconds summed over its CTAs: busy, HARQ combine, decode,
 * code-block CRCs, transport-block finish; then the worker's iterations and its
 * microseconds admitting, publishing and taking results}. */
int32_t syndrome_serve_core_stats(SyndromeServer* server, double* out10);
/* Work-item sizes per shape: n triples (base_graph, z, codewords per item; 0 = as many
 * as one CTA holds), as chosen by the autotuner (syndrome_b200/autotune.py).  Takes
 * effect from the next step; results do not depend on it.  INVALID_PARAM for a base
 * graph other than 0/1 or z outside 1..384. */
int32_t syndrome_serve_set_tiles(SyndromeServer* server, const int32_t* triples, size_t n);

/* Open-loop load test of a server (the serving benchmark; no counterpart in the
 * reference).  Transport blocks arrive as a Poisson process of offered_tb_per_s for
 * duration_s; arrival i is pool entry i % pool_n, whose llr[rv index] are device
 * pointers to the C * E LLRs of its transmissions with redundancy versions 0, 2, 3, 1.
 * A failed transmission is retransmitted at once with the next version, up to
 * max_transmissions.  A block's latency runs from its scheduled arrival to the result
 * of its last transmission; latencies_us (nullable) receives them in arrival order. */
typedef struct {
  size_t tb_size;
  float target_rate;
  size_t qm;
  size_t g;
  const float* llr[4];
  size_t llr_len;
} SyndromeLoadTb;
typedef struct {
  double offered_tb_per_s;
  double duration_s;
  uint32_t max_transmissions;
  uint64_t seed;
} SyndromeLoadSpec;
typedef struct {
  uint64_t tbs, tbs_ok, transmissions;
  double wall_s;
  double info_bits_ok;       /* payload bits of the blocks whose CRCs passed */
  double info_bits_decoded;  /* payload bits over all transmissions (decode work done) */
  double p50_us, p99_us, mean_us, max_us;  /* per transport block, arrival to last result */
  double tx_p50_us, tx_p99_us;             /* per transmission, submit to result */
  double tx_mean_queue_us;                 /* mean wait from submit to the launch of its step */
  double tx_mean_step_us;                  /* mean GPU time of the step that decoded it */
} SyndromeLoadReport;
int32_t syndrome_serve_run_load(SyndromeServer* server, const SyndromeLoadTb* pool, size_t pool_n,
                                const SyndromeLoadSpec* spec, SyndromeLoadReport* report,
                                double* latencies_us, size_t latencies_cap);

/* Text of the last error on this thread (empty if none). */
const char* syndrome_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SYNDROME_LDPC_H */
