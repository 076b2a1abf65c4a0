// Device kernels around the decoder for transport-block serving (serve_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace syn {

// One code block of one transmission in a serving step.
struct ServeCb {
  float* acc;            // HARQ accumulator, ncb floats (circular buffer, variables 2Z..N)
  const float* e;        // received LLRs of this code block (e_len floats, interleaved order)
  int8_t* llr;           // decoder input: ncb int8 values (variables 2Z..N); null = f32 (acc only)
  const uint32_t* hard;  // decoder output: K' hard decisions, LSB-first words
  int ncb, fs, fe, m, c0;  // rate-matching walk (see tb.h RmWalk)
  int e_len, qm;
  int first;             // first transmission of the TB: the accumulator starts at +0
  int k_prime;           // bits covered by the code-block CRC-24B (CRC included)
  int crc_len;           // leading bits of this block inside the TB CRC-24A range
  int tb;                // index of the block's transport block in the step
  int hard_words;        // words of `hard` (K' bits)
};

// One transport block (one transmission) in a serving step.
struct ServeTb {
  int first_cb, n_cb;
  int payload;           // TB bits per code block
  int has_cb_crc;
  long long tb_size;     // A
  uint32_t x_payload;    // x^payload mod P_A
  uint32_t x_last;       // x^(CRC-24A bits of the last code block) mod P_A
  uint32_t* tb_bits;     // output: tb_size bits, LSB-first words
  int32_t* result;       // [0] crc_ok, [1] max iterations, [2 + i/32] bit i%32 = code block i CRC ok
};

// Per code block results of the CRC kernel.
struct ServeCbCrc {
  uint32_t crc_a;        // CRC-24A register of the block's first crc_len bits
  int ok_b;              // CRC-24B over K' bits is zero (or the TB has no CB CRC)
};

// x^n mod P for the 24-bit generator poly (MSB-first register convention).
uint32_t crc24_xpow_host(long long n, uint32_t poly);
// a * b mod P.
uint32_t crc24_mulmod_host(uint32_t a, uint32_t b, uint32_t poly);

// ---- continuous serving: one persistent kernel over a ring of work items ----
//
// The host writes one record per transmission (ServeTxRec), the slots of its code blocks
// and its work items (ServeJob: up to a CTA's worth of its code blocks) into host-mapped memory and
// publishes them by advancing a 64-bit tail.  The kernel's CTAs claim items in ring
// order; per item a CTA combines the code blocks' HARQ buffers into int8 decoder input,
// decodes them, checks their CRCs and counts them done; the CTA that completes a
// transmission's last code block folds the TB CRC, writes the report and the
// desegmented bits to host-mapped memory and then the completion flag.
constexpr int kServeLlrStride = 25344;   // int8 LLR bytes per code-block slot (N - 2Z, BG1 Z=384)
constexpr int kServeHardWords = 264;     // packed hard-decision words per code-block slot (K' <= 8448)
constexpr int kServeMaxItemCbs = 32;     // code blocks per work item
constexpr int kServeXpow = 8449;         // entries of each x^n mod P table (n = 0 .. 8448)
constexpr int kServeMaxCbs = 160;        // code blocks per transport block (code-block slot list length)

struct ServeTxRec {
  float* acc;          // HARQ accumulators of code block 0 (block i at acc + i * ncb)
  const float* e;      // received LLRs of code block 0 (block i at e + i * e_len)
  uint32_t* bits;      // host-mapped output: tb_size bits, LSB-first words
  long long tb_size;   // A
  long long b;         // A + 24
  int ncb, fs, fe, m, c0, e_len, qm, first;  // rate-matching walk, c0 reduced mod m
  int bg, z, zi, n_filler, k_prime, has_cb_crc;
  int n_cb, payload, pad;
  uint32_t x_payload;  // x^payload mod P_A
  uint32_t x_last;     // x^(CRC-24A bits of the last code block) mod P_A
  uint32_t seq;        // value of the completion flag
};

struct ServeTxOut {
  int32_t result[8];   // [0] crc_ok, [1] max iterations, [2 + i/32] bit i%32 = code block i CRC ok
  uint32_t flag;       // seq of the record once result and bits are written
  uint32_t pad[7];
};

struct ServeJob {
  int tx;              // transmission slot
  int first_cb;        // first code block of the item within the transmission
  int count;           // code blocks in the item
  int pad;
};

struct ServeCtl {      // device memory
  unsigned long long head;     // next item to claim
  unsigned long long tail;     // items published (mirror of the host tail)
  unsigned long long last_ns;  // global timer of the last claim or newly seen item
  unsigned watch;              // 1 while a CTA reads the host tail
  unsigned closing;            // = the launch's epoch once that launch is winding down
  // telemetry: items done and global-timer nanoseconds per phase, summed over CTAs
  unsigned long long items, busy_ns, combine_ns, decode_ns, crc_ns, finish_ns;
  unsigned pad[12];
};

struct ServeContArgs {
  const ServeJob* ring;            // host-mapped, ring_cap entries
  unsigned long long ring_cap;
  const ServeTxRec* recs;          // host-mapped, per transmission slot
  const int* slots;                // host-mapped, per transmission slot: its code blocks' slots [kServeMaxCbs]
  ServeTxOut* outs;                // host-mapped, per transmission slot
  const unsigned long long* host_tail;  // host-mapped
  const unsigned* host_stop;       // host-mapped: 1 = exit once no item is left
  ServeCtl* ctl;
  int* sm_busy;                    // [1024] items in progress per SM id (0 between launches)
  int* tx_done;                    // per transmission slot: code blocks finished (0 between uses)
  int8_t* llr;                     // per code-block slot kServeLlrStride bytes
  uint32_t* hard;                  // per code-block slot kServeHardWords words
  int32_t* iters;                  // per code-block slot
  ServeCbCrc* crc;                 // per code-block slot
  const uint32_t* crc_tab;         // [2][4][256] slice tables, P_A then P_B
  const uint32_t* xpow;            // [2][kServeXpow] x^n mod P, P_A then P_B
  const short* shift_tab;          // as MixArgs
  const int* colz_tab;
  int beta_q, app_clamp, iterations;
  float scale;
  unsigned long long idle_ns;      // the kernel exits once no CTA has claimed an item for this long
  unsigned epoch;                  // launch number (never 0)
};

// Raises the persistent kernel's shared-memory limit (once per device).
cudaError_t serve_cont_prepare();
// Launches the persistent kernel: two CTAs per SM, each holding 256 TMEM columns until
// the kernel winds down as a whole (no claim for idle_ns, or host_stop with the ring
// drained): the CTA that sees it marks the launch closing and every CTA leaves at its
// next claim, so a kernel never runs on with a fraction of its CTAs.
cudaError_t serve_cont_launch(const ServeContArgs& a, int sms, cudaStream_t stream);

// HARQ soft combining + quantization: acc[p] (+)= the received LLRs rate-matched to
// position p, in received order; llr[p] = quantize(acc[p] * scale).
cudaError_t serve_combine_launch(const ServeCb* d_cbs, int n_cbs, int max_ncb, float scale, cudaStream_t stream);
// Code-block CRCs (CRC-24B check, CRC-24A register of the TB part).
cudaError_t serve_cb_crc_launch(const ServeCb* d_cbs, int n_cbs, ServeCbCrc* d_out, cudaStream_t stream);
// Transport-block CRC fold, results and desegmented TB bits; iters[i] = iterations
// of code block i of the step.
cudaError_t serve_tb_finish_launch(const ServeTb* d_tbs, int n_tbs, const ServeCb* d_cbs, const ServeCbCrc* d_crc,
                                   const int32_t* d_iters, cudaStream_t stream);

}  // namespace syn
