// Device work around the decoder for transport-block serving, sm_100a.
//
// serve_combine_kernel  HARQ soft combining and quantization (harq.rs:142-161 with
//     rate_matching.rs:675-700, then quantize.rs:331-343), as a gather: the thread of
//     circular-buffer position p finds the received bits that rate matching put there
//     (selection k with (c0 + k) mod M = compressed(p), every M selections) and adds
//     them in received order, exactly the order of the reference's scatter loop, so the
//     f32 sums are bit-identical.  No atomics: each position has one owner.
// serve_cb_crc_kernel   one warp per code block: the CRC-24B check over its K' decoded
//     bits and the CRC-24A register of the bits it carries for the TB CRC.  Lanes take
//     contiguous word chunks (byte-table CRC, tables in shared memory) and the chunk
//     registers are joined with CRC(A|B) = CRC(A) * x^|B| + CRC(B) (mod P).
// serve_tb_finish_kernel one CTA per transport block: the TB CRC-24A from the blocks'
//     registers (crc.rs check: the register over payload + received CRC is zero iff
//     they match), the report (crc_ok, max iterations, per-block CRC) and the
//     desegmented TB bits (transport_block.rs:1014-1050).
#include "serve_kernels.h"

#include <algorithm>

namespace syn {

namespace {

constexpr uint32_t kPolyA = 0x864CFBu, kPolyB = 0x800063u;

__host__ __device__ inline uint32_t crc_mulmod(uint32_t a, uint32_t b, uint32_t poly) {
  uint32_t r = 0;
  for (int i = 23; i >= 0; --i) {
    r <<= 1;
    if (r & 0x1000000u) r ^= 0x1000000u | poly;
    if ((b >> i) & 1u) r ^= a;
  }
  return r;
}

__host__ __device__ inline uint32_t crc_xpow(long long n, uint32_t poly) {
  uint32_t result = 1u, base = 2u;  // x^0, x^1
  while (n > 0) {
    if (n & 1) result = crc_mulmod(result, base, poly);
    base = crc_mulmod(base, base, poly);
    n >>= 1;
  }
  return result;
}

__device__ inline uint32_t crc_byte(uint32_t reg, uint32_t byte, const uint32_t* table) {
  return ((reg << 8) & 0xFFFFFFu) ^ table[((reg >> 16) ^ byte) & 0xFFu];
}

__device__ inline uint32_t crc_bit(uint32_t reg, uint32_t bit, uint32_t poly) {
  const uint32_t fb = ((reg >> 23) ^ bit) & 1u;
  reg = (reg << 1) & 0xFFFFFFu;
  return fb ? reg ^ poly : reg;
}

// CRC register of bits [0, nbits) of LSB-first packed words, computed by one warp.
__device__ uint32_t warp_crc(const uint32_t* __restrict__ words, int nbits, const uint32_t* table, uint32_t poly,
                             int lane) {
  const int full = nbits >> 5, rem = nbits & 31;
  const int chunk = (full + 31) >> 5;
  const int lo = lane * chunk, hi = min(lo + chunk, full);
  uint32_t reg = 0;
  for (int w = lo; w < hi; ++w) {
    const uint32_t r = __brev(words[w]);  // bit 0 (first in order) becomes the MSB
    reg = crc_byte(reg, r >> 24, table);
    reg = crc_byte(reg, (r >> 16) & 0xFFu, table);
    reg = crc_byte(reg, (r >> 8) & 0xFFu, table);
    reg = crc_byte(reg, r & 0xFFu, table);
  }
  const uint32_t xchunk = chunk > 0 ? crc_xpow(32LL * chunk, poly) : 1u;
  uint32_t total = 0;
  for (int l = 0; l < 32; ++l) {
    const uint32_t cl = __shfl_sync(0xFFFFFFFFu, reg, l);
    const int nw = max(0, min(chunk, full - l * chunk));
    if (nw == chunk && nw > 0)
      total = crc_mulmod(total, xchunk, poly) ^ cl;
    else if (nw > 0)
      total = crc_mulmod(total, crc_xpow(32LL * nw, poly), poly) ^ cl;
  }
  if (rem) {
    const uint32_t w = words[full];
    for (int i = 0; i < rem; ++i) total = crc_bit(total, (w >> i) & 1u, poly);
  }
  return total;
}

__global__ void serve_combine_kernel(const ServeCb* __restrict__ cbs, float scale) {
  const ServeCb cb = cbs[blockIdx.y];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= cb.ncb) return;
  if (p >= cb.fs && p < cb.fe) {  // filler positions: never transmitted, decoder pins them
    if (cb.first) cb.acc[p] = 0.0f;
    if (cb.llr) cb.llr[p] = 0;
    return;
  }
  const int c = p < cb.fs ? p : p - (cb.fe - cb.fs);
  int k = c - cb.c0 % cb.m;
  if (k < 0) k += cb.m;
  float a = cb.first ? 0.0f : cb.acc[p];
  if (cb.qm == 1) {
    for (long long kk = k; kk < cb.e_len; kk += cb.m) a = __fadd_rn(a, cb.e[kk]);
  } else {
    // received index of selection kk: q = (kk % qm) * rows + kk / qm; add in q order
    const long long rows = cb.e_len / cb.qm;
    long long q[8];
    int n = 0;
    for (long long kk = k; kk < cb.e_len && n < 8; kk += cb.m) {
      const long long v = (kk % cb.qm) * rows + kk / cb.qm;
      int i = n++;
      while (i > 0 && q[i - 1] > v) {
        q[i] = q[i - 1];
        --i;
      }
      q[i] = v;
    }
    for (int i = 0; i < n; ++i) a = __fadd_rn(a, cb.e[q[i]]);
  }
  cb.acc[p] = a;
  if (!cb.llr) return;  // f32 decode: the accumulator is the decoder input
  const float v = __fmul_rn(a, scale);
  int qv = 0;
  if (!isnan(v)) qv = (int)fminf(fmaxf(roundf(v), -127.0f), 127.0f);
  cb.llr[p] = (int8_t)qv;
}

__global__ void serve_cb_crc_kernel(const ServeCb* __restrict__ cbs, int n_cbs, ServeCbCrc* __restrict__ out) {
  __shared__ uint32_t tab[2][256];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) {
    const uint32_t poly = i < 256 ? kPolyA : kPolyB;
    uint32_t reg = (uint32_t)(i & 255) << 16;
    for (int b = 0; b < 8; ++b) reg = (reg & 0x800000u) ? ((reg << 1) ^ poly) & 0xFFFFFFu : (reg << 1) & 0xFFFFFFu;
    tab[i >> 8][i & 255] = reg;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= n_cbs) return;
  const ServeCb cb = cbs[i];
  const uint32_t ra = warp_crc(cb.hard, cb.crc_len, tab[0], kPolyA, lane);
  int ok = 1;
  if (cb.k_prime > 0) ok = warp_crc(cb.hard, cb.k_prime, tab[1], kPolyB, lane) == 0u;
  if (lane == 0) {
    out[i].crc_a = ra;
    out[i].ok_b = ok;
  }
}

__global__ void serve_tb_finish_kernel(const ServeTb* __restrict__ tbs, const ServeCb* __restrict__ cbs,
                                       const ServeCbCrc* __restrict__ crc, const int32_t* __restrict__ iters) {
  const ServeTb tb = tbs[blockIdx.x];
  if (threadIdx.x == 0) {
    uint32_t total = 0;
    int all_cb = 1, max_it = 0;
    for (int i = 0; i < tb.n_cb; ++i) {
      const int c = tb.first_cb + i;
      const int len = cbs[c].crc_len;
      if (len > 0) {
        const uint32_t xl = len == tb.payload ? tb.x_payload : crc_xpow(len, kPolyA);
        total = crc_mulmod(total, xl, kPolyA) ^ crc[c].crc_a;
      }
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
  // desegmentation: TB bit i is bit i % payload of code block i / payload
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const long long nwords = (tb.tb_size + 31) >> 5;
  for (long long w = warp; w < nwords; w += nwarps) {
    const long long i = (w << 5) + lane;
    bool bit = false;
    if (i < tb.tb_size) {
      const long long c = i / tb.payload, j = i - c * tb.payload;
      bit = (cbs[tb.first_cb + c].hard[j >> 5] >> (j & 31)) & 1u;
    }
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
    if (lane == 0) tb.tb_bits[w] = m;
  }
}

}  // namespace

uint32_t crc24_xpow_host(long long n, uint32_t poly) { return crc_xpow(n, poly); }

cudaError_t serve_combine_launch(const ServeCb* d_cbs, int n_cbs, int max_ncb, float scale, cudaStream_t stream) {
  if (n_cbs <= 0) return cudaSuccess;
  const dim3 grid((unsigned)((max_ncb + 255) / 256), (unsigned)n_cbs);
  serve_combine_kernel<<<grid, 256, 0, stream>>>(d_cbs, scale);
  return cudaGetLastError();
}

cudaError_t serve_cb_crc_launch(const ServeCb* d_cbs, int n_cbs, ServeCbCrc* d_out, cudaStream_t stream) {
  if (n_cbs <= 0) return cudaSuccess;
  serve_cb_crc_kernel<<<(n_cbs + 3) / 4, 128, 0, stream>>>(d_cbs, n_cbs, d_out);
  return cudaGetLastError();
}

cudaError_t serve_tb_finish_launch(const ServeTb* d_tbs, int n_tbs, const ServeCb* d_cbs, const ServeCbCrc* d_crc,
                                   const int32_t* d_iters, cudaStream_t stream) {
  if (n_tbs <= 0) return cudaSuccess;
  serve_tb_finish_kernel<<<n_tbs, 256, 0, stream>>>(d_tbs, d_cbs, d_crc, d_iters);
  return cudaGetLastError();
}

}  // namespace syn
