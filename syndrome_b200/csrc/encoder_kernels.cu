// Batched systematic encoding on the GPU (Encoder::encode_batch_device), for
// generating large test batches on the device.  Same method and results as the host
// Encoder (encoder.cpp): the core syndrome of the information bits, the core parity
// as the GF(2) product with the precomputed inverse of the core, then each extension
// layer's parity block from the bits it touches.  Same codewords as syndrome's
// QcLdpcEncoder::encode (src/qc_ldpc.rs:2592-2727), which are unique.
//
// One CTA per codeword (persistent over the batch).  The codeword's bits sit in
// shared memory one per byte; the core syndrome is packed into 32-bit words with a
// warp ballot per 32 consecutive check rows; the inverse is stored column-major
// (word w of every row contiguous), so the threads of a warp, one core row each,
// read it coalesced from L2.
#include <algorithm>
#include <string>

#include "encoder.h"
#include "smem_limit.h"

namespace syn {

namespace {

constexpr int kEncThreads = 384;

struct EncArgs {
  int z, mb, kb, core_blocks, core_bits, words32;
  const int32_t* loff;
  const uint32_t* edge;   // col << 16 | shift
  const uint32_t* inv_t;  // [words32][core_bits]
  const uint8_t* info;
  long long info_stride;
  uint8_t* out;
  long long out_stride;
  long long count;
};

__global__ void __launch_bounds__(kEncThreads) encode_kernel(const __grid_constant__ EncArgs a) {
  extern __shared__ __align__(16) unsigned char enc_smem[];
  const int z = a.z, k = a.kb * z, n = (a.kb + a.mb) * z;
  uint32_t* syn = reinterpret_cast<uint32_t*>(enc_smem);
  uint8_t* cw = enc_smem + 4 * a.words32;
  const int tid = threadIdx.x, lane = tid & 31;
  for (long long b = blockIdx.x; b < a.count; b += gridDim.x) {
    const uint8_t* in = a.info + b * a.info_stride;
    for (int i = tid; i < k; i += blockDim.x) cw[i] = in[i] & 1u;
    __syncthreads();
    // core syndrome, 32 check rows per warp step (every lane takes part in the ballot)
    const int rows32 = a.words32 * 32;
    for (int r0 = tid - lane; r0 < rows32; r0 += blockDim.x) {
      const int r = r0 + lane;
      uint32_t bit = 0;
      if (r < a.core_bits) {
        const int l = r / z, zi = r - l * z;
        for (int e = a.loff[l]; e < a.loff[l + 1]; ++e) {
          const uint32_t ed = a.edge[e];
          const int c = (int)(ed >> 16), sh = (int)(ed & 0xFFFFu);
          if (c >= a.kb) continue;
          const int s = zi + sh;
          bit ^= cw[c * z + (s >= z ? s - z : s)];
        }
      }
      const uint32_t word = __ballot_sync(0xFFFFFFFFu, bit != 0);
      if (lane == 0) syn[r0 >> 5] = word;
    }
    __syncthreads();
    // core parity = inverse x syndrome over GF(2)
    for (int r = tid; r < a.core_bits; r += blockDim.x) {
      uint32_t acc = 0;
      for (int w = 0; w < a.words32; ++w) acc ^= a.inv_t[(long long)w * a.core_bits + r] & syn[w];
      cw[k + r] = (uint8_t)(__popc(acc) & 1);
    }
    __syncthreads();
    // extension layers: each fixes its own unshifted parity block
    const int ext = (a.mb - a.core_blocks) * z;
    for (int i = tid; i < ext; i += blockDim.x) {
      const int l = a.core_blocks + i / z, zi = i % z;
      uint32_t bit = 0;
      for (int e = a.loff[l]; e < a.loff[l + 1]; ++e) {
        const uint32_t ed = a.edge[e];
        const int c = (int)(ed >> 16), sh = (int)(ed & 0xFFFFu);
        if (c == a.kb + l) continue;
        const int s = zi + sh;
        bit ^= cw[c * z + (s >= z ? s - z : s)];
      }
      cw[(a.kb + l) * z + zi] = (uint8_t)bit;
    }
    __syncthreads();
    uint8_t* o = a.out + b * a.out_stride;
    for (int i = tid; i < n; i += blockDim.x) o[i] = cw[i];
    __syncthreads();
  }
}

}  // namespace

Encoder::Dev::~Dev() {
  cudaFree(inv_t);
  cudaFree(loff);
  cudaFree(edge);
}

cudaError_t Encoder::encode_batch_device(const uint8_t* d_info, long long info_stride, uint8_t* d_codewords,
                                         long long cw_stride, long long count, cudaStream_t stream) const {
  if (count <= 0) return cudaSuccess;
  const Graph& g = g_;
  const int words32 = (core_bits_ + 31) / 32;
  int cur = 0;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lock(dev_->mu);
    if (dev_->device != cur) {
      if (dev_->device >= 0) return cudaErrorInvalidDevice;  // tables live on another device
      std::vector<uint32_t> inv_t((size_t)words32 * core_bits_, 0u);
      for (int r = 0; r < core_bits_; ++r)
        for (int w = 0; w < words32; ++w)
          inv_t[(size_t)w * core_bits_ + r] = (uint32_t)(inv_[(size_t)r * words_ + (w >> 1)] >> (32 * (w & 1)));
      std::vector<uint32_t> edge(g.cols.size());
      for (size_t i = 0; i < edge.size(); ++i) edge[i] = ((uint32_t)g.cols[i] << 16) | (uint32_t)g.shifts[i];
      std::vector<int32_t> loff(g.layer_off.begin(), g.layer_off.end());
      if ((e = cudaMalloc(&dev_->inv_t, sizeof(uint32_t) * std::max<size_t>(inv_t.size(), 1))) != cudaSuccess ||
          (e = cudaMalloc(&dev_->edge, sizeof(uint32_t) * edge.size())) != cudaSuccess ||
          (e = cudaMalloc(&dev_->loff, sizeof(int32_t) * loff.size())) != cudaSuccess ||
          (e = cudaMemcpy(dev_->inv_t, inv_t.data(), sizeof(uint32_t) * inv_t.size(), cudaMemcpyHostToDevice)) !=
              cudaSuccess ||
          (e = cudaMemcpy(dev_->edge, edge.data(), sizeof(uint32_t) * edge.size(), cudaMemcpyHostToDevice)) !=
              cudaSuccess ||
          (e = cudaMemcpy(dev_->loff, loff.data(), sizeof(int32_t) * loff.size(), cudaMemcpyHostToDevice)) !=
              cudaSuccess)
        return e;
      dev_->device = cur;
    }
  }
  EncArgs a;
  a.z = g.z;
  a.mb = g.mb;
  a.kb = g.kb;
  a.core_blocks = core_blocks_;
  a.core_bits = core_bits_;
  a.words32 = words32;
  a.loff = dev_->loff;
  a.edge = dev_->edge;
  a.inv_t = dev_->inv_t;
  a.info = d_info;
  a.info_stride = info_stride;
  a.out = d_codewords;
  a.out_stride = cw_stride;
  a.count = count;
  const int smem = 4 * words32 + (int)g.n();
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  if ((e = allow_max_dynamic_smem((const void*)encode_kernel)) != cudaSuccess) return e;
  int sms = 0, per_sm = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cur)) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, encode_kernel, kEncThreads, smem)) != cudaSuccess)
    return e;
  const long long ctas = std::min<long long>(count, (long long)sms * std::max(per_sm, 1));
  encode_kernel<<<(unsigned)ctas, kEncThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace syn
