// Device work around the decoder for transport-block serving, sm_100a.
//
// serve_combine_kernel  HARQ soft combining and quantization (harq.rs:142-161 with
//     rate_matching.rs:675-700, then quantize.rs:331-343), as a gather: the thread of
//     circular-buffer position p finds the received bits that rate matching put there
//     (selection k with (c0 + k) mod M = compressed(p), every M selections) and adds
//     them in received order, exactly the order of the reference's scatter loop, so the
//     f32 sums are bit-identical.  No atomics: each position has one owner.
// serve_cb_crc_kernel   one thread per code block: the CRC-24B check over its K' decoded
//     bits and the CRC-24A register of the bits it carries for the TB CRC, 32 bits per
//     step with slice-by-4 tables in shared memory (register' = sum over the four
//     bytes b_k of ((R << 8) ^ word) of T_k[b_k], T_k[v] = v * x^(8k + 24) mod P).
// serve_tb_finish_kernel one CTA per transport block: the TB CRC-24A from the blocks'
//     registers, CRC(A|B) = CRC(A) * x^|B| + CRC(B) (mod P), the multiplication by the
//     fixed x^payload done with three 256-entry tables built by the CTA (crc.rs check:
//     the register over payload + received CRC is zero iff they match); the report
//     (crc_ok, max iterations, per-block CRC); the desegmented TB bits
//     (transport_block.rs:1014-1050), one thread per output word, each a funnel shift of
//     the packed bits of at most two code blocks.
#include "serve_kernels.h"

#include <algorithm>

#include "serve_device.cuh"

namespace syn {

namespace {

using srv::crc_mulmod;
using srv::crc_xpow;
using srv::kPolyA;
using srv::kPolyB;
using srv::mul_fixed;
using srv::thread_crc;

constexpr int kCombThreads = 256, kCombPer = 4;  // positions per thread (block-strided)

__global__ void __launch_bounds__(kCombThreads) serve_combine_kernel(const ServeCb* __restrict__ cbs, float scale) {
  // Only the fields used, once per thread, and 32-bit index arithmetic throughout (the
  // kernel is otherwise bound by its integer instructions, not by memory).
  const ServeCb* cbp = cbs + blockIdx.y;
  srv::CombineWalk w;
  w.ncb = cbp->ncb;
  w.fs = cbp->fs;
  w.fe = cbp->fe;
  w.m = cbp->m;
  w.c0 = cbp->c0 % w.m;
  w.e_len = cbp->e_len;
  w.qm = cbp->qm;
  w.first = cbp->first;
  float* acc = cbp->acc;
  const float* e = cbp->e;
  int8_t* llr = cbp->llr;
#pragma unroll
  for (int i = 0; i < kCombPer; ++i) {
    const int p = (blockIdx.x * kCombPer + i) * kCombThreads + threadIdx.x;
    if (p >= w.ncb) break;
    srv::combine_position(p, w, acc, e, llr, scale);
  }
}

constexpr int kCrcWarps = 4;
constexpr int kCrcMaxWords = (8448 + 31) / 32;  // K' of the largest code block

__global__ void serve_cb_crc_kernel(const ServeCb* __restrict__ cbs, int n_cbs, ServeCbCrc* __restrict__ out) {
  __shared__ uint32_t tab[2][4][256];
  __shared__ uint32_t bits[kCrcWarps][kCrcMaxWords];
  for (int i = threadIdx.x; i < 2048; i += blockDim.x) {
    const uint32_t poly = i < 1024 ? kPolyA : kPolyB;
    const int k = (i >> 8) & 3;
    uint32_t reg = (uint32_t)(i & 255) << 16;
    for (int b = 0; b < 8 * (k + 1); ++b) reg = (reg & 0x800000u) ? ((reg << 1) ^ poly) & 0xFFFFFFu : (reg << 1) & 0xFFFFFFu;
    tab[i >> 10][k][i & 255] = reg;
  }
  __syncthreads();
  // one warp per code block: its packed bits to shared memory (coalesced), then lane 0
  // the CRC-24A register and lane 1 the CRC-24B check, side by side
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int i = blockIdx.x * kCrcWarps + wi;
  if (i >= n_cbs) return;
  const ServeCb cb = cbs[i];
  const int nw = min(cb.hard_words, kCrcMaxWords);
  for (int w = lane; w < nw; w += 32) bits[wi][w] = cb.hard[w];
  __syncwarp();
  if (lane == 0) out[i].crc_a = thread_crc(bits[wi], min(cb.crc_len, 32 * nw), tab[0], kPolyA);
  if (lane == 1) out[i].ok_b = cb.k_prime > 0 ? thread_crc(bits[wi], min(cb.k_prime, 32 * nw), tab[1], kPolyB) == 0u : 1;
}

__global__ void serve_tb_finish_kernel(const ServeTb* __restrict__ tbs, const ServeCb* __restrict__ cbs,
                                       const ServeCbCrc* __restrict__ crc, const int32_t* __restrict__ iters) {
  __shared__ uint32_t my[3][256];  // (v << 8k) * x^payload mod P_A
  const ServeTb tb = tbs[blockIdx.x];
  for (int i = threadIdx.x; i < 768; i += blockDim.x)
    my[i >> 8][i & 255] = crc_mulmod((uint32_t)(i & 255) << (8 * (i >> 8)), tb.x_payload, kPolyA);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t total = 0;
    int all_cb = 1, max_it = 0;
    for (int i = 0; i < tb.n_cb; ++i) {
      const int c = tb.first_cb + i;
      const int len = cbs[c].crc_len;
      if (len == tb.payload)
        total = mul_fixed(total, my) ^ crc[c].crc_a;
      else if (len > 0)
        total = crc_mulmod(total, i == tb.n_cb - 1 ? tb.x_last : crc_xpow(len, kPolyA), kPolyA) ^ crc[c].crc_a;
      all_cb &= crc[c].ok_b;
      max_it = max(max_it, iters[c]);
    }
    tb.result[0] = (all_cb && total == 0u) ? 1 : 0;
    tb.result[1] = max_it;
  }
  for (int w = threadIdx.x; w < (tb.n_cb + 31) / 32; w += blockDim.x) {
    uint32_t bits = 0;
    for (int t = 0; t < 32 && 32 * w + t < tb.n_cb; ++t) bits |= (uint32_t)crc[tb.first_cb + 32 * w + t].ok_b << t;
    tb.result[2 + w] = (int32_t)bits;
  }
  // desegmentation: TB bit i is bit i % payload of code block i / payload; a word spans
  // at most two code blocks (with more than one block, payload > 32)
  auto bits_at = [&](int c, int j) -> uint32_t {  // 32 bits of block c from bit j on (0 past its words)
    const ServeCb& cb = cbs[tb.first_cb + c];
    const int w = j >> 5;
    const uint32_t lo = w < cb.hard_words ? cb.hard[w] : 0u, hi = w + 1 < cb.hard_words ? cb.hard[w + 1] : 0u;
    return __funnelshift_r(lo, hi, (unsigned)(j & 31));
  };
  const int nwords = (int)((tb.tb_size + 31) >> 5);
  for (int w = threadIdx.x; w < nwords; w += blockDim.x) {
    const int i0 = 32 * w;
    const int c = i0 / tb.payload, j = i0 - c * tb.payload;
    uint32_t v = bits_at(c, j);
    const int avail = tb.payload - j;
    if (avail < 32) {
      v &= (1u << avail) - 1u;
      if (c + 1 < tb.n_cb) v |= bits_at(c + 1, 0) << avail;
    }
    const long long left = tb.tb_size - i0;
    if (left < 32) v &= (1u << left) - 1u;
    tb.tb_bits[w] = v;
  }
}

}  // namespace

uint32_t crc24_xpow_host(long long n, uint32_t poly) { return crc_xpow(n, poly); }
uint32_t crc24_mulmod_host(uint32_t a, uint32_t b, uint32_t poly) { return crc_mulmod(a, b, poly); }

cudaError_t serve_combine_launch(const ServeCb* d_cbs, int n_cbs, int max_ncb, float scale, cudaStream_t stream) {
  if (n_cbs <= 0) return cudaSuccess;
  const int per_block = kCombThreads * kCombPer;
  const dim3 grid((unsigned)((max_ncb + per_block - 1) / per_block), (unsigned)n_cbs);
  serve_combine_kernel<<<grid, kCombThreads, 0, stream>>>(d_cbs, scale);
  return cudaGetLastError();
}

cudaError_t serve_cb_crc_launch(const ServeCb* d_cbs, int n_cbs, ServeCbCrc* d_out, cudaStream_t stream) {
  if (n_cbs <= 0) return cudaSuccess;
  serve_cb_crc_kernel<<<(n_cbs + kCrcWarps - 1) / kCrcWarps, 32 * kCrcWarps, 0, stream>>>(d_cbs, n_cbs, d_out);
  return cudaGetLastError();
}

cudaError_t serve_tb_finish_launch(const ServeTb* d_tbs, int n_tbs, const ServeCb* d_cbs, const ServeCbCrc* d_crc,
                                   const int32_t* d_iters, cudaStream_t stream) {
  if (n_tbs <= 0) return cudaSuccess;
  serve_tb_finish_kernel<<<n_tbs, 256, 0, stream>>>(d_tbs, d_cbs, d_crc, d_iters);
  return cudaGetLastError();
}

}  // namespace syn
