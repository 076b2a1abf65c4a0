// Batched layered offset min-sum (LOMS) decoder kernels for sm_100a.
//
// Algorithm: syndrome src/qc_ldpc.rs:962-1221 (f32) and :1530-1758 (int8 messages,
// int16 posterior), restated for the GPU with the reference's exact arithmetic:
//   Q     = APP - R_old                         (int8 path: clamped to +-127)
//   pass1 min1 / min2 / XOR of signs over the layer's edges
//   R_new = sign * max(min_excl - beta, 0)      (min_excl = min2 on the min1 edge)
//   APP  += R_new - R_old                       (int8 path: clamped to +-app_clamp)
// followed by the syndrome check after every iteration (early stop), and hard
// decisions APP < 0.
//
// Mapping: one CTA owns `cpb` codewords of one code; thread (slot, z) owns lifting
// index z of codeword slot, i.e. check row (layer, z) of every layer.  The
// posteriors of the CTA's codewords live in shared memory for the whole decode;
// the cyclic shift of each block is index arithmetic on the shared-memory
// address.  Layers run in order with a CTA barrier between them (the layered
// schedule's dependency).  Check-to-variable messages live in global memory in
// the reference's edge_r layout (edge-major, z fastest), so consecutive threads
// touch consecutive bytes; the per-CTA scratch is small enough to stay in L2.
//
// The kernel is persistent over codeword groups: grid = resident CTAs, each CTA
// walks groups blockIdx.x, blockIdx.x + gridDim.x, ...  Codewords that pass the
// syndrome check stop updating while the other slots of their CTA continue.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <mutex>
#include <string>

#include "decoder.h"
#include "smem_limit.h"
#include "nr_kernels.h"
#include "wifi_mixed.h"

namespace syn {

namespace {

constexpr int kMaxThreads = 384;
constexpr int kCompressedSmem = 113 * 1024;  // f32 compressed-message CTA: two per SM

struct KArgs {
  int z, mb, n_edges, n, k;
  const uint32_t* edge;   // [E] (col * z) << 16 | shift
  const int32_t* loff;    // [mb + 1]
  const void* llr;
  long long llr_stride;
  int llr_offset;
  int llr_i16;
  long long batch;
  int cpb;
  int iterations;
  int beta_q;
  int app_clamp;
  float beta;
  int prologue;
  long long k_prime;      // filler positions are [k_prime, k)
  int shorten;            // f32: Wi-Fi shortened / punctured rows (BatchRequest::shorten)
  long long sh_pay;       // payload bits P
  long long sh_par_end;   // K + transmitted parity bits
  void* r_out;            // C->V messages of codeword b at r_out + b * r_out_stride
  long long r_out_stride;
  void* r_ws;             // else per (CTA, slot) scratch
  uint32_t* hard_packed;
  int hard_bits;
  long long hard_words_stride;
  int32_t* iters;
  void* app_out;
  long long app_stride;
  uint8_t* hard_out;
  long long hard_stride;
  int st_words;           // f32 compressed messages: state words per thread (0: messages in r_ws / r_out)
  int st_off;             // byte offset of the state words in shared memory
};

__host__ __device__ constexpr int align16(int x) { return (x + 15) & ~15; }

__host__ __device__ inline int table_bytes(int n_edges, int mb, int cpb) {
  return align16(n_edges * 4) + align16((mb + 1) * 4) + align16(cpb * 4);
}

template <typename App>
struct Smem {
  uint32_t* edge;
  int32_t* loff;
  int32_t* fail;
  App* app;
};

template <typename App>
__device__ inline Smem<App> carve(unsigned char* base, const KArgs& a) {
  Smem<App> s;
  s.edge = reinterpret_cast<uint32_t*>(base);
  s.loff = reinterpret_cast<int32_t*>(base + align16(a.n_edges * 4));
  s.fail = reinterpret_cast<int32_t*>(base + align16(a.n_edges * 4) + align16((a.mb + 1) * 4));
  s.app = reinterpret_cast<App*>(base + table_bytes(a.n_edges, a.mb, a.cpb));
  return s;
}

// Variable index of edge word w for check row zi: col*z + (zi + shift) mod z.
__device__ __forceinline__ int var_index(uint32_t w, int zi, int Z) {
  int r = zi + (int)(w & 0xFFFFu);
  r = (r >= Z) ? r - Z : r;
  return (int)(w >> 16) + r;
}

// The two smallest of v[0..D) (min1, then the second smallest counting ties: the
// reference's sequential rule "|Q| <= min1: min2 = min1, min1 = |Q|; else |Q| < min2:
// min2 = |Q|" started at FLT_MAX, whose result does not depend on the order) as a
// pairwise min/max tree: depth log2(D) instead of a D-long dependent chain.  The
// caller clamps each |Q| to FLT_MAX first (fminf drops NaN), which is what the
// sequential rule does with +inf and NaN (never taken), so the pair is bit-identical.
template <int N>
__device__ __forceinline__ void merge_min2(float* lo, float* hi) {
  if constexpr (N > 1) {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const float l1 = lo[2 * i], l2 = lo[2 * i + 1], h = fminf(hi[2 * i], hi[2 * i + 1]);
      lo[i] = fminf(l1, l2);
      hi[i] = fminf(fmaxf(l1, l2), h);
    }
    if constexpr ((N & 1) != 0) {
      lo[N / 2] = lo[N - 1];
      hi[N / 2] = hi[N - 1];
    }
    merge_min2<(N + 1) / 2>(lo, hi);
  }
}
template <int D>
__device__ __forceinline__ void min2_tree(const float* v, float& m1, float& m2) {
  constexpr int P = (D + 1) / 2;
  float lo[P], hi[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    if (2 * i + 1 < D) {
      lo[i] = fminf(v[2 * i], v[2 * i + 1]);
      hi[i] = fmaxf(v[2 * i], v[2 * i + 1]);
    } else {
      lo[i] = v[2 * i];
      hi[i] = FLT_MAX;
    }
  }
  merge_min2<P>(lo, hi);
  m1 = lo[0];
  m2 = hi[0];
}

// Integer form of min2_tree (int8 path: |Q| <= 127, padding 127, the start of both
// minima in qc_ldpc.rs's int8 pass).
template <int N>
__device__ __forceinline__ void merge_min2_i(int* lo, int* hi) {
  if constexpr (N > 1) {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const int l1 = lo[2 * i], l2 = lo[2 * i + 1], h = min(hi[2 * i], hi[2 * i + 1]);
      lo[i] = min(l1, l2);
      hi[i] = min(max(l1, l2), h);
    }
    if constexpr ((N & 1) != 0) {
      lo[N / 2] = lo[N - 1];
      hi[N / 2] = hi[N - 1];
    }
    merge_min2_i<(N + 1) / 2>(lo, hi);
  }
}
template <int D>
__device__ __forceinline__ void min2_tree_i(const int* v, int& m1, int& m2) {
  constexpr int P = (D + 1) / 2;
  int lo[P], hi[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    if (2 * i + 1 < D) {
      lo[i] = min(v[2 * i], v[2 * i + 1]);
      hi[i] = max(v[2 * i], v[2 * i + 1]);
    } else {
      lo[i] = v[2 * i];
      hi[i] = 127;
    }
  }
  merge_min2_i<P>(lo, hi);
  m1 = lo[0];
  m2 = hi[0];
}

// ---------------------------------------------------------------- int8 path --

template <int MAXDEG>
__device__ __forceinline__ void layer_i8(const uint32_t* __restrict__ s_edge, int lb, int deg, int Z,
                                         int zi, int16_t* __restrict__ A, int8_t* __restrict__ R,
                                         bool first, int beta_q, int C) {
  int vidx[MAXDEG], av[MAXDEG], qv[MAXDEG], ro[MAXDEG];
  int m1 = 127, m2 = 127;
  unsigned sx = 0;
  int8_t* Rl = R + (long long)lb * Z + zi;
#pragma unroll
  for (int e = 0; e < MAXDEG; ++e) {
    if (e < deg) {
      vidx[e] = var_index(s_edge[lb + e], zi, Z);
      av[e] = A[vidx[e]];
      ro[e] = first ? 0 : (int)Rl[e * Z];
      const int q = min(max(av[e] - ro[e], -127), 127);
      qv[e] = q;
      const int aq = abs(q);
      sx ^= (unsigned)q;
      const int om1 = m1;
      m1 = min(om1, aq);
      m2 = min(m2, max(om1, aq));
    }
  }
  if (deg < 2) {
    if (deg == 0) m1 = 0;
    m2 = m1;
  }
#pragma unroll
  for (int e = 0; e < MAXDEG; ++e) {
    if (e < deg) {
      const int q = qv[e];
      const int aq = abs(q);
      const int mex = (aq == m1) ? m2 : m1;
      const int mag = max(mex - beta_q, 0);
      const int nr = ((sx ^ (unsigned)q) >> 31) ? -mag : mag;
      Rl[e * Z] = (int8_t)nr;
      A[vidx[e]] = (int16_t)min(max(av[e] + nr - ro[e], -C), C);
    }
  }
}

template <typename App>
__device__ bool syndrome_fails(const uint32_t* __restrict__ s_edge, const int32_t* __restrict__ s_loff,
                               int mb, int Z, int zi, const App* __restrict__ A) {
  for (int l = 0; l < mb; ++l) {
    const int lb = s_loff[l], le = s_loff[l + 1];
    unsigned par = 0;
    for (int e = lb; e < le; ++e) par ^= (A[var_index(s_edge[e], zi, Z)] < (App)0) ? 1u : 0u;
    if (par) return true;
  }
  return false;
}

template <typename App>
__device__ void write_outputs(const KArgs& a, const Smem<App>& s, long long grp) {
  const int N = a.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int sl = 0; sl < a.cpb; ++sl) {
    const long long cw = grp * a.cpb + sl;
    if (cw >= a.batch) break;
    const App* As = s.app + (long long)sl * N;
    if (a.app_out) {
      App* dst = reinterpret_cast<App*>(a.app_out) + cw * a.app_stride;
      for (int j = threadIdx.x; j < N; j += blockDim.x) dst[j] = As[j];
    }
    if (a.hard_out) {
      uint8_t* dst = a.hard_out + cw * a.hard_stride;
      for (int j = threadIdx.x; j < N; j += blockDim.x) dst[j] = As[j] < (App)0 ? 1 : 0;
    }
    if (a.hard_packed) {
      const int nwords = (a.hard_bits + 31) >> 5;
      uint32_t* dst = a.hard_packed + cw * a.hard_words_stride;
      for (int w = warp; w < nwords; w += nwarps) {
        const int j = (w << 5) + lane;
        const bool bit = j < a.hard_bits && As[j] < (App)0;
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
        if (lane == 0) dst[w] = m;
      }
    }
  }
}

// The codewords of group grp into shared memory (the int8 kernels' load: int8 or int16
// input, [0, llr_offset) erased, the 5G prologue, the posterior clamp).
__device__ void load_i8_group(const KArgs& a, int16_t* app, long long grp) {
  const int Z = a.z, N = a.n, C = a.app_clamp;
  for (int sl = 0; sl < a.cpb; ++sl) {
    const long long cw = grp * a.cpb + sl;
    if (cw >= a.batch) break;
    const int8_t* src8 = reinterpret_cast<const int8_t*>(a.llr) + cw * a.llr_stride;
    const int16_t* src16 = reinterpret_cast<const int16_t*>(a.llr) + cw * a.llr_stride;
    int16_t* dst = app + (long long)sl * N;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
      int v = 0;
      if (j >= a.llr_offset) v = a.llr_i16 ? (int)src16[j - a.llr_offset] : (int)src8[j - a.llr_offset];
      if (a.prologue) {
        if (j < 2 * Z)
          v = 0;
        else if (j >= a.k_prime && j < a.k)
          v = C;
      }
      dst[j] = (int16_t)min(max(v, -C), C);
    }
  }
}

template <int MAXDEG>
__global__ void __launch_bounds__(kMaxThreads) loms_i8_kernel(const KArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Smem<int16_t> s = carve<int16_t>(smem_raw, a);
  for (int i = threadIdx.x; i < a.n_edges; i += blockDim.x) s.edge[i] = a.edge[i];
  for (int i = threadIdx.x; i <= a.mb; i += blockDim.x) s.loff[i] = a.loff[i];

  const int Z = a.z, N = a.n, C = a.app_clamp;
  const int slot = threadIdx.x / Z;
  const int zi = threadIdx.x - slot * Z;
  const bool lane_ok = slot < a.cpb;
  const long long ngroups = (a.batch + a.cpb - 1) / a.cpb;
  const long long ez = (long long)a.n_edges * Z;

  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    __syncthreads();
    load_i8_group(a, s.app, grp);
    __syncthreads();

    const long long cw = grp * a.cpb + slot;
    bool active = lane_ok && cw < a.batch;
    int8_t* R = nullptr;
    if (active)
      R = a.r_out ? reinterpret_cast<int8_t*>(a.r_out) + cw * a.r_out_stride
                  : reinterpret_cast<int8_t*>(a.r_ws) + ((long long)blockIdx.x * a.cpb + slot) * ez;
    int16_t* A = s.app + (long long)(lane_ok ? slot : 0) * N;
    int used = 0;
    for (int it = 0; it < a.iterations; ++it) {
      if (!__syncthreads_or(active)) break;
      if (active) ++used;
      for (int l = 0; l < a.mb; ++l) {
        if (active) {
          const int lb = s.loff[l];
          layer_i8<MAXDEG>(s.edge, lb, s.loff[l + 1] - lb, Z, zi, A, R, it == 0, a.beta_q, C);
        }
        __syncthreads();
      }
      if (lane_ok && zi == 0) s.fail[slot] = 0;
      __syncthreads();
      if (active && syndrome_fails(s.edge, s.loff, a.mb, Z, zi, A)) s.fail[slot] = 1;
      __syncthreads();
      if (active && s.fail[slot] == 0) active = false;
    }
    if (lane_ok && cw < a.batch) {
      if (zi == 0 && a.iters) a.iters[cw] = used;
      if (used == 0 && a.r_out) {
        int8_t* Rz = reinterpret_cast<int8_t*>(a.r_out) + cw * a.r_out_stride;
        for (long long j = zi; j < ez; j += Z) Rz[j] = 0;
      }
    }
    __syncthreads();
    write_outputs<int16_t>(a, s, grp);
  }
}

// ------------------------------------------------ int8, compressed messages --
//
// The int8 messages of a check row are +-max(m1 - beta_q, 0) on the edges whose |Q| is
// not the row minimum and +-max(m2 - beta_q, 0) on those that are (qc_ldpc.rs:1700-1718),
// so a row is one word (both magnitudes, 0..127, in bytes 0 and 1) plus two bits per edge
// (|Q| == m1, R negative).  loms_i8c_kernel keeps that in shared memory: per thread and
// layer one magnitude word and max(1, ceil(deg / 16)) code words, word w of thread t
// at st[w * threads + t].  Same arithmetic and results as loms_i8_kernel.

__device__ __forceinline__ int i8c_message(uint32_t mags, unsigned bb) {
  const int mag = (int)((mags >> ((bb & 1u) << 3)) & 0xFFu);
  return (bb & 2u) ? -mag : mag;
}

template <int MAXDEG>
__device__ __forceinline__ void layer_i8c(const uint32_t* __restrict__ s_edge, int lb, int deg, int Z, int zi,
                                          int16_t* __restrict__ A, uint32_t* __restrict__ st, int ns, int mw,
                                          int cwo, int beta_q, int C) {
  int vidx[MAXDEG], av[MAXDEG], qv[MAXDEG], ro[MAXDEG];
  const uint32_t mags = st[mw * ns];
  const uint32_t lo = st[cwo * ns];
  const uint32_t hi = deg > 16 ? st[(cwo + 1) * ns] : 0u;
  const unsigned long long bits = ((unsigned long long)hi << 32) | lo;
  constexpr bool kTree = MAXDEG >= 16;  // as in layer_f32c
  int m1 = 127, m2 = 127, ak[MAXDEG];
  unsigned sx = 0;
#pragma unroll
  for (int e = 0; e < MAXDEG; ++e) {
    ak[e] = 127;  // edges past deg: 127, the starting value of both minima
    if (e < deg) {
      vidx[e] = var_index(s_edge[lb + e], zi, Z);
      av[e] = A[vidx[e]];
      ro[e] = i8c_message(mags, (unsigned)(bits >> (2 * e)) & 3u);
      const int q = min(max(av[e] - ro[e], -127), 127);
      qv[e] = q;
      const int aq = abs(q);
      sx ^= (unsigned)q;
      if constexpr (kTree) {
        ak[e] = aq;
      } else {
        const int om1 = m1;
        m1 = min(om1, aq);
        m2 = min(m2, max(om1, aq));
      }
    }
  }
  if constexpr (kTree) min2_tree_i<MAXDEG>(ak, m1, m2);
  if (deg < 2) {
    if (deg == 0) m1 = 0;
    m2 = m1;
  }
  const int nA = max(m1 - beta_q, 0), nB = max(m2 - beta_q, 0);
  unsigned long long nbits = 0ull;
#pragma unroll
  for (int e = 0; e < MAXDEG; ++e) {
    if (e < deg) {
      const int q = qv[e];
      const int aq = abs(q);
      const bool is_min = aq == m1;
      const int mag = is_min ? nB : nA;
      const bool neg = ((sx ^ (unsigned)q) >> 31) != 0u;
      const int nr = neg ? -mag : mag;
      A[vidx[e]] = (int16_t)min(max(av[e] + nr - ro[e], -C), C);
      nbits |= (unsigned long long)((is_min ? 1u : 0u) | (neg ? 2u : 0u)) << (2 * e);
    }
  }
  st[mw * ns] = (uint32_t)nA | ((uint32_t)nB << 8);
  st[cwo * ns] = (uint32_t)nbits;
  if (deg > 16) st[(cwo + 1) * ns] = (uint32_t)(nbits >> 32);
}

template <int MAXDEG>
__global__ void __launch_bounds__(kMaxThreads) loms_i8c_kernel(const KArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Smem<int16_t> s = carve<int16_t>(smem_raw, a);
  for (int i = threadIdx.x; i < a.n_edges; i += blockDim.x) s.edge[i] = a.edge[i];
  for (int i = threadIdx.x; i <= a.mb; i += blockDim.x) s.loff[i] = a.loff[i];

  const int Z = a.z, C = a.app_clamp, ns = (int)blockDim.x;
  const int slot = threadIdx.x / Z;
  const int zi = threadIdx.x - slot * Z;
  const bool lane_ok = slot < a.cpb;
  const long long ngroups = (a.batch + a.cpb - 1) / a.cpb;
  uint32_t* st = reinterpret_cast<uint32_t*>(smem_raw + a.st_off) + threadIdx.x;

  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    __syncthreads();
    load_i8_group(a, s.app, grp);
    for (int w = 0; w < a.st_words; ++w) st[w * ns] = 0u;  // R = 0 before the first iteration
    __syncthreads();

    const long long cw = grp * a.cpb + slot;
    bool active = lane_ok && cw < a.batch;
    int16_t* A = s.app + (long long)(lane_ok ? slot : 0) * a.n;
    int used = 0;
    for (int it = 0; it < a.iterations; ++it) {
      if (!__syncthreads_or(active)) break;
      if (active) ++used;
      int cwo = a.mb;  // code words follow the mb magnitude words
      for (int l = 0; l < a.mb; ++l) {
        const int lb = s.loff[l], deg = s.loff[l + 1] - lb;
        if (active) layer_i8c<MAXDEG>(s.edge, lb, deg, Z, zi, A, st, ns, l, cwo, a.beta_q, C);
        cwo += max(1, (deg + 15) >> 4);
        __syncthreads();
      }
      if (lane_ok && zi == 0) s.fail[slot] = 0;
      __syncthreads();
      if (active && syndrome_fails(s.edge, s.loff, a.mb, Z, zi, A)) s.fail[slot] = 1;
      __syncthreads();
      if (active && s.fail[slot] == 0) active = false;
    }
    if (lane_ok && cw < a.batch) {
      if (zi == 0 && a.iters) a.iters[cw] = used;
      if (a.r_out) {  // the messages in the reference's edge_r layout, rebuilt from the state
        int8_t* Rz = reinterpret_cast<int8_t*>(a.r_out) + cw * a.r_out_stride + zi;
        int cwo = a.mb;
        for (int l = 0; l < a.mb; ++l) {
          const int lb = s.loff[l], deg = s.loff[l + 1] - lb;
          const uint32_t mags = st[l * ns];
          const unsigned long long bits =
              ((unsigned long long)(deg > 16 ? st[(cwo + 1) * ns] : 0u) << 32) | st[cwo * ns];
          for (int e = 0; e < deg; ++e)
            Rz[(long long)(lb + e) * Z] = (int8_t)i8c_message(mags, (unsigned)(bits >> (2 * e)) & 3u);
          cwo += max(1, (deg + 15) >> 4);
        }
      }
    }
    __syncthreads();
    write_outputs<int16_t>(a, s, grp);
  }
}

// ----------------------------------------------------------------- f32 path --

template <int MAXDEG>
__device__ __forceinline__ void layer_f32(const uint32_t* __restrict__ s_edge, int lb, int deg, int Z,
                                          int zi, float* __restrict__ A, float* __restrict__ R,
                                          bool first, float beta) {
  int vidx[MAXDEG];
  float av[MAXDEG], qv[MAXDEG], ro[MAXDEG];
  float m1 = FLT_MAX, m2 = FLT_MAX;
  unsigned sx = 0;
  float* Rl = R + (long long)lb * Z + zi;
#pragma unroll
  for (int e = 0; e < MAXDEG; ++e) {
    if (e < deg) {
      vidx[e] = var_index(s_edge[lb + e], zi, Z);
      av[e] = A[vidx[e]];
      ro[e] = first ? 0.0f : Rl[e * Z];
      const float q = __fsub_rn(av[e], ro[e]);
      qv[e] = q;
      const unsigned b = __float_as_uint(q);
      const float aq = __uint_as_float(b & 0x7FFFFFFFu);
      sx ^= b & 0x80000000u;
      if (aq <= m1) {
        m2 = m1;
        m1 = aq;
      } else if (aq < m2) {
        m2 = aq;
      }
    }
  }
  if (m1 == FLT_MAX) m1 = 0.0f;
  if (m2 == FLT_MAX) m2 = m1;
#pragma unroll
  for (int e = 0; e < MAXDEG; ++e) {
    if (e < deg) {
      const unsigned b = __float_as_uint(qv[e]);
      const float aq = __uint_as_float(b & 0x7FFFFFFFu);
      const unsigned sgn = sx ^ (b & 0x80000000u);
      const float mex = (aq == m1) ? m2 : m1;
      float mag = __fsub_rn(mex, beta);
      if (mag < 0.0f) mag = 0.0f;
      const float nr = __uint_as_float(__float_as_uint(mag) | sgn);
      Rl[e * Z] = nr;
      A[vidx[e]] = __fadd_rn(av[e], __fsub_rn(nr, ro[e]));
    }
  }
}

// The codewords of group grp into shared memory (the f32 kernels' load: [0, llr_offset)
// erased, the 5G prologue or the Wi-Fi shortened-row rebuild on top).
__device__ void load_f32_group(const KArgs& a, float* app, long long grp) {
  const int Z = a.z, N = a.n;
  for (int sl = 0; sl < a.cpb; ++sl) {
    const long long cw = grp * a.cpb + sl;
    if (cw >= a.batch) break;
    const float* src = reinterpret_cast<const float*>(a.llr) + cw * a.llr_stride;
    float* dst = app + (long long)sl * N;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
      float v = j >= a.llr_offset ? src[j - a.llr_offset] : 0.0f;
      if (a.prologue) {
        if (j < 2 * Z)
          v = 0.0f;
        else if (j >= a.k_prime && j < a.k)
          v = 1000000.0f;
      }
      if (a.shorten) {
        // the row holds the sent bits only: payload, then the parity that was not punctured
        if (j < a.sh_pay)
          v = src[j];
        else if (j < a.k)
          v = 1000000.0f;  // shortened: known zero (LLR_KNOWN_ZERO, wifi_rate_matching.rs:58)
        else if (j < a.sh_par_end)
          v = src[j - (a.k - a.sh_pay)];
        else
          v = 0.0f;  // punctured: erasure
      }
      dst[j] = v;
    }
  }
}

template <int MAXDEG>
__global__ void __launch_bounds__(kMaxThreads) loms_f32_kernel(const KArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Smem<float> s = carve<float>(smem_raw, a);
  for (int i = threadIdx.x; i < a.n_edges; i += blockDim.x) s.edge[i] = a.edge[i];
  for (int i = threadIdx.x; i <= a.mb; i += blockDim.x) s.loff[i] = a.loff[i];

  const int Z = a.z, N = a.n;
  const int slot = threadIdx.x / Z;
  const int zi = threadIdx.x - slot * Z;
  const bool lane_ok = slot < a.cpb;
  const long long ngroups = (a.batch + a.cpb - 1) / a.cpb;
  const long long ez = (long long)a.n_edges * Z;

  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    __syncthreads();
    load_f32_group(a, s.app, grp);
    __syncthreads();

    const long long cw = grp * a.cpb + slot;
    bool active = lane_ok && cw < a.batch;
    float* R = nullptr;
    if (active)
      R = a.r_out ? reinterpret_cast<float*>(a.r_out) + cw * a.r_out_stride
                  : reinterpret_cast<float*>(a.r_ws) + ((long long)blockIdx.x * a.cpb + slot) * ez;
    float* A = s.app + (long long)(lane_ok ? slot : 0) * N;
    int used = 0;
    for (int it = 0; it < a.iterations; ++it) {
      if (!__syncthreads_or(active)) break;
      if (active) ++used;
      for (int l = 0; l < a.mb; ++l) {
        if (active) {
          const int lb = s.loff[l];
          layer_f32<MAXDEG>(s.edge, lb, s.loff[l + 1] - lb, Z, zi, A, R, it == 0, a.beta);
        }
        __syncthreads();
      }
      if (lane_ok && zi == 0) s.fail[slot] = 0;
      __syncthreads();
      if (active && syndrome_fails(s.edge, s.loff, a.mb, Z, zi, A)) s.fail[slot] = 1;
      __syncthreads();
      if (active && s.fail[slot] == 0) active = false;
    }
    if (lane_ok && cw < a.batch) {
      if (zi == 0 && a.iters) a.iters[cw] = used;
      if (used == 0 && a.r_out) {
        float* Rz = reinterpret_cast<float*>(a.r_out) + cw * a.r_out_stride;
        for (long long j = zi; j < ez; j += Z) Rz[j] = 0.0f;
      }
    }
    __syncthreads();
    write_outputs<float>(a, s, grp);
  }
}

// ------------------------------------------------- f32, compressed messages --
//
// The reference's f32 messages of a check row are a function of two magnitudes,
// max(min1 - beta, 0) and max(min2 - beta, 0), and two bits per edge (|Q| was the row
// minimum, R's sign), from which R_old is rebuilt bit for bit (signed zeros included).
// loms_f32c_kernel keeps them in shared memory next to the posteriors: per thread and
// layer two magnitude words and max(1, ceil(deg / 16)) code words, word w of thread t at
// st[w * threads + t].  Same arithmetic, order and results as loms_f32_kernel.

__device__ __forceinline__ float f32c_message(float magA, float magB, unsigned bb) {
  return __uint_as_float(__float_as_uint((bb & 1u) ? magB : magA) | ((bb & 2u) << 30));
}

template <int MAXDEG>
__device__ __forceinline__ void layer_f32c(const uint32_t* __restrict__ s_edge, int lb, int deg, int Z, int zi,
                                           float* __restrict__ A, uint32_t* __restrict__ st, int ns, int mw,
                                           int cwo, float beta) {
  int vidx[MAXDEG];
  float av[MAXDEG], qv[MAXDEG], ro[MAXDEG];
  const float magA = __uint_as_float(st[mw * ns]), magB = __uint_as_float(st[(mw + 1) * ns]);
  const uint32_t lo = st[cwo * ns];
  const uint32_t hi = deg > 16 ? st[(cwo + 1) * ns] : 0u;
  const unsigned long long bits = ((unsigned long long)hi << 32) | lo;
  // rows of up to 12 edges: the sequential rule (the tree's extra registers would cost
  // a resident CTA); longer rows: the tree
  constexpr bool kTree = MAXDEG >= 16;
  float m1 = FLT_MAX, m2 = FLT_MAX, ak[MAXDEG];
  unsigned sx = 0;
#pragma unroll
  for (int e = 0; e < MAXDEG; ++e) {
    ak[e] = FLT_MAX;  // edges past deg: FLT_MAX, which the two smallest never need
    if (e < deg) {
      vidx[e] = var_index(s_edge[lb + e], zi, Z);
      av[e] = A[vidx[e]];
      ro[e] = f32c_message(magA, magB, (unsigned)(bits >> (2 * e)) & 3u);
      const float q = __fsub_rn(av[e], ro[e]);
      qv[e] = q;
      const unsigned b = __float_as_uint(q);
      const float aq = __uint_as_float(b & 0x7FFFFFFFu);
      sx ^= b & 0x80000000u;
      if constexpr (kTree) {
        ak[e] = fminf(aq, FLT_MAX);
      } else if (aq <= m1) {
        m2 = m1;
        m1 = aq;
      } else if (aq < m2) {
        m2 = aq;
      }
    }
  }
  if constexpr (kTree) min2_tree<MAXDEG>(ak, m1, m2);
  if (m1 == FLT_MAX) m1 = 0.0f;
  if (m2 == FLT_MAX) m2 = m1;
  float nA = __fsub_rn(m1, beta), nB = __fsub_rn(m2, beta);  // messages of the non-minimum / minimum edges
  if (nA < 0.0f) nA = 0.0f;
  if (nB < 0.0f) nB = 0.0f;
  unsigned long long nbits = 0ull;
#pragma unroll
  for (int e = 0; e < MAXDEG; ++e) {
    if (e < deg) {
      const unsigned b = __float_as_uint(qv[e]);
      const float aq = __uint_as_float(b & 0x7FFFFFFFu);
      const unsigned sgn = sx ^ (b & 0x80000000u);
      const bool is_min = aq == m1;
      const float nr = __uint_as_float(__float_as_uint(is_min ? nB : nA) | sgn);
      A[vidx[e]] = __fadd_rn(av[e], __fsub_rn(nr, ro[e]));
      nbits |= (unsigned long long)((is_min ? 1u : 0u) | (sgn >> 30)) << (2 * e);
    }
  }
  st[mw * ns] = __float_as_uint(nA);
  st[(mw + 1) * ns] = __float_as_uint(nB);
  st[cwo * ns] = (uint32_t)nbits;
  if (deg > 16) st[(cwo + 1) * ns] = (uint32_t)(nbits >> 32);
}

template <int MAXDEG>
__global__ void __launch_bounds__(kMaxThreads) loms_f32c_kernel(const KArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Smem<float> s = carve<float>(smem_raw, a);
  for (int i = threadIdx.x; i < a.n_edges; i += blockDim.x) s.edge[i] = a.edge[i];
  for (int i = threadIdx.x; i <= a.mb; i += blockDim.x) s.loff[i] = a.loff[i];

  const int Z = a.z, ns = (int)blockDim.x;
  const int slot = threadIdx.x / Z;
  const int zi = threadIdx.x - slot * Z;
  const bool lane_ok = slot < a.cpb;
  const long long ngroups = (a.batch + a.cpb - 1) / a.cpb;
  uint32_t* st = reinterpret_cast<uint32_t*>(smem_raw + a.st_off) + threadIdx.x;

  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    __syncthreads();
    load_f32_group(a, s.app, grp);
    for (int w = 0; w < a.st_words; ++w) st[w * ns] = 0u;  // R = +0 before the first iteration
    __syncthreads();

    const long long cw = grp * a.cpb + slot;
    bool active = lane_ok && cw < a.batch;
    float* A = s.app + (long long)(lane_ok ? slot : 0) * a.n;
    int used = 0;
    for (int it = 0; it < a.iterations; ++it) {
      if (!__syncthreads_or(active)) break;
      if (active) ++used;
      int cwo = 2 * a.mb;  // code words follow the 2 * mb magnitude words
      for (int l = 0; l < a.mb; ++l) {
        const int lb = s.loff[l], deg = s.loff[l + 1] - lb;
        if (active) layer_f32c<MAXDEG>(s.edge, lb, deg, Z, zi, A, st, ns, 2 * l, cwo, a.beta);
        cwo += max(1, (deg + 15) >> 4);
        __syncthreads();
      }
      if (lane_ok && zi == 0) s.fail[slot] = 0;
      __syncthreads();
      if (active && syndrome_fails(s.edge, s.loff, a.mb, Z, zi, A)) s.fail[slot] = 1;
      __syncthreads();
      if (active && s.fail[slot] == 0) active = false;
    }
    if (lane_ok && cw < a.batch) {
      if (zi == 0 && a.iters) a.iters[cw] = used;
      if (a.r_out) {  // the messages in the reference's edge_r layout, rebuilt from the state
        float* Rz = reinterpret_cast<float*>(a.r_out) + cw * a.r_out_stride + zi;
        int cwo = 2 * a.mb;
        for (int l = 0; l < a.mb; ++l) {
          const int lb = s.loff[l], deg = s.loff[l + 1] - lb;
          const float magA = __uint_as_float(st[2 * l * ns]), magB = __uint_as_float(st[(2 * l + 1) * ns]);
          const unsigned long long bits =
              ((unsigned long long)(deg > 16 ? st[(cwo + 1) * ns] : 0u) << 32) | st[cwo * ns];
          for (int e = 0; e < deg; ++e)
            Rz[(long long)(lb + e) * Z] = f32c_message(magA, magB, (unsigned)(bits >> (2 * e)) & 3u);
          cwo += max(1, (deg + 15) >> 4);
        }
      }
    }
    __syncthreads();
    write_outputs<float>(a, s, grp);
  }
}

typedef void (*KernelFn)(const KArgs);

int pick_maxdeg(int maxdeg) {
  if (maxdeg <= 8) return 8;
  if (maxdeg <= 12) return 12;
  if (maxdeg <= 16) return 16;
  if (maxdeg <= 20) return 20;
  if (maxdeg <= 24) return 24;
  return -1;
}

KernelFn kernel_for(Precision p, int tmpl, bool compressed = false) {
  if (p == Precision::kInt8 && compressed) {
    switch (tmpl) {
      case 8: return loms_i8c_kernel<8>;
      case 12: return loms_i8c_kernel<12>;
      case 16: return loms_i8c_kernel<16>;
      case 20: return loms_i8c_kernel<20>;
      case 24: return loms_i8c_kernel<24>;
    }
    return nullptr;
  }
  if (p == Precision::kF32 && compressed) {
    switch (tmpl) {
      case 8: return loms_f32c_kernel<8>;
      case 12: return loms_f32c_kernel<12>;
      case 16: return loms_f32c_kernel<16>;
      case 20: return loms_f32c_kernel<20>;
      case 24: return loms_f32c_kernel<24>;
    }
    return nullptr;
  }
  if (p == Precision::kInt8) {
    switch (tmpl) {
      case 8: return loms_i8_kernel<8>;
      case 12: return loms_i8_kernel<12>;
      case 16: return loms_i8_kernel<16>;
      case 20: return loms_i8_kernel<20>;
      case 24: return loms_i8_kernel<24>;
    }
  } else {
    switch (tmpl) {
      case 8: return loms_f32_kernel<8>;
      case 12: return loms_f32_kernel<12>;
      case 16: return loms_f32_kernel<16>;
      case 20: return loms_f32_kernel<20>;
      case 24: return loms_f32_kernel<24>;
    }
  }
  return nullptr;
}

// ------------------------------------------- 802.11 mixed batches (f32) --
//
// One persistent launch over codewords of all twelve 802.11 matrices
// (wifi_mixed.h).  A CTA takes a chunk (a run of codewords of one matrix) from the
// device queue and runs a session of that matrix: the matrix's tables go to shared
// memory, and each of its floor(384 / Z) codeword slots (Z threads each) decodes one
// codeword at a time with the compressed-message row update of loms_f32c_kernel.  All
// slots take the layers together (a barrier per layer), each on its own iteration:
// after every iteration a slot whose codeword reached a zero syndrome or the iteration
// limit writes its results and takes the next codeword of the chunk, and when the chunk
// runs out the CTA takes the next chunk from the queue.  If that chunk is of another
// matrix, the slots drain and the session ends; the CTA then starts a session of the
// new matrix.  Codewords that converge in one iteration and codewords that run all of
// them thus keep every slot busy (the batch's iteration counts are heavily skewed).

extern __shared__ __align__(16) unsigned char wm_smem[];

// The row update of layer_f32c with nothing per edge kept between its two passes:
// the second pass reads each posterior again (still the old value: a row touches each
// of its variables once, and only the second pass writes them) and rebuilds the old
// message from the stored bits, so the subtraction, the sign and the minimum test see
// exactly the values of the first pass.  Row minima by the reference's sequential
// rule (qc_ldpc.rs:1100-1113).  Same results as layer_f32c in a fraction of its
// registers, for a kernel that runs every matrix under one register budget.
__device__ __forceinline__ void layer_f32c_lean(const uint32_t* __restrict__ s_edge, int lb, int deg, int Z, int zi,
                                                float* __restrict__ A, uint32_t* __restrict__ st, int ns, int mw,
                                                int cwo, float beta) {
  const float magA = __uint_as_float(st[mw * ns]), magB = __uint_as_float(st[(mw + 1) * ns]);
  const uint32_t lo = st[cwo * ns];
  const uint32_t hi = deg > 16 ? st[(cwo + 1) * ns] : 0u;
  const unsigned long long bits = ((unsigned long long)hi << 32) | lo;
  float m1 = FLT_MAX, m2 = FLT_MAX;
  unsigned sx = 0;
#pragma unroll 4
  for (int e = 0; e < deg; ++e) {
    const float av = A[var_index(s_edge[lb + e], zi, Z)];
    const float ro = f32c_message(magA, magB, (unsigned)(bits >> (2 * e)) & 3u);
    const unsigned b = __float_as_uint(__fsub_rn(av, ro));
    const float aq = __uint_as_float(b & 0x7FFFFFFFu);
    sx ^= b & 0x80000000u;
    if (aq <= m1) {
      m2 = m1;
      m1 = aq;
    } else if (aq < m2) {
      m2 = aq;
    }
  }
  if (m1 == FLT_MAX) m1 = 0.0f;
  if (m2 == FLT_MAX) m2 = m1;
  float nA = __fsub_rn(m1, beta), nB = __fsub_rn(m2, beta);
  if (nA < 0.0f) nA = 0.0f;
  if (nB < 0.0f) nB = 0.0f;
  unsigned long long nbits = 0ull;
#pragma unroll 4
  for (int e = 0; e < deg; ++e) {
    const int v = var_index(s_edge[lb + e], zi, Z);
    const float av = A[v];
    const float ro = f32c_message(magA, magB, (unsigned)(bits >> (2 * e)) & 3u);
    const unsigned b = __float_as_uint(__fsub_rn(av, ro));
    const float aq = __uint_as_float(b & 0x7FFFFFFFu);
    const unsigned sgn = sx ^ (b & 0x80000000u);
    const bool is_min = aq == m1;
    const float nr = __uint_as_float(__float_as_uint(is_min ? nB : nA) | sgn);
    A[v] = __fadd_rn(av, __fsub_rn(nr, ro));
    nbits |= (unsigned long long)((is_min ? 1u : 0u) | (sgn >> 30)) << (2 * e);
  }
  st[mw * ns] = __float_as_uint(nA);
  st[(mw + 1) * ns] = __float_as_uint(nB);
  st[cwo * ns] = (uint32_t)nbits;
  if (deg > 16) st[(cwo + 1) * ns] = (uint32_t)(nbits >> 32);
}

struct WmHdr {
  int chunk, pending, cur, end, shape, pad[3];
  int slot_cw[kWmMaxSlots], slot_used[kWmMaxSlots], slot_fail[kWmMaxSlots], slot_new[kWmMaxSlots];
};
constexpr int kWmHdr = (int)((sizeof(WmHdr) + 15) / 16 * 16);
constexpr int kWmTab = kWmMaxEdges * 4 + align16((kWmMaxLayers + 1) * 4);

__device__ __forceinline__ void wm_session(const WmArgs& a, const WmShape& sh) {
  WmHdr* h = reinterpret_cast<WmHdr*>(wm_smem);
  uint32_t* s_edge = reinterpret_cast<uint32_t*>(wm_smem + kWmHdr);
  int32_t* s_loff = reinterpret_cast<int32_t*>(wm_smem + kWmHdr + kWmMaxEdges * 4);
  float* app = reinterpret_cast<float*>(wm_smem + kWmHdr + kWmTab);
  const int Z = sh.z, N = sh.n, cpb = sh.cpb, ns = (int)blockDim.x, tid = (int)threadIdx.x;
  uint32_t* st = reinterpret_cast<uint32_t*>(wm_smem + kWmHdr + kWmTab + align16(cpb * N * 4)) + tid;
  const int slot = tid / Z, zi = tid - slot * Z;
  const bool lane_ok = slot < cpb;
  for (int i = tid; i < sh.n_edges; i += ns) s_edge[i] = a.edges[sh.edge_off + i];
  for (int i = tid; i <= sh.mb; i += ns) s_loff[i] = a.loffs[sh.loff_off + i];
  if (tid < kWmMaxSlots) {
    h->slot_cw[tid] = -1;
    h->slot_used[tid] = 0;
    h->slot_fail[tid] = 0;
    h->slot_new[tid] = 0;
  }
  if (tid == 0) {
    const WmChunk ch = a.chunks[h->chunk];
    h->cur = ch.first;
    h->end = ch.first + ch.count;
    h->shape = ch.shape;
    h->pending = -1;
  }
  __syncthreads();
  for (;;) {
    // every idle slot takes the next codeword of this matrix (thread 0 hands them out)
    if (tid == 0) {
      for (int s = 0; s < cpb; ++s) {
        if (h->slot_cw[s] >= 0) continue;
        while (h->cur >= h->end && h->pending < 0) {
          const int nc = (int)atomicAdd(a.queue, 1u);
          if (nc < a.n_chunks && a.chunks[nc].shape == h->shape) {
            h->cur = a.chunks[nc].first;
            h->end = h->cur + a.chunks[nc].count;
          } else {
            h->pending = nc;  // another matrix, or the end of the queue: after this session
          }
        }
        if (h->cur >= h->end) break;
        h->slot_cw[s] = h->cur++;
        h->slot_used[s] = 0;
        h->slot_new[s] = 1;
      }
    }
    __syncthreads();
    const int my = lane_ok ? h->slot_cw[slot] : -1;
    if (my >= 0 && h->slot_new[slot]) {  // a new codeword: channel LLRs in, messages R = +0
      const float* src = a.llr + a.cws[my].llr_off;
      float* A = app + slot * N;
      for (int j = zi; j < N; j += Z) A[j] = src[j];
      for (int w = 0; w < sh.st_words; ++w) st[w * ns] = 0u;
    }
    int n_act = 0;
    for (int s = 0; s < cpb; ++s) n_act += h->slot_cw[s] >= 0 ? 1 : 0;
    __syncthreads();
    if (tid < cpb) h->slot_new[tid] = 0;
    if (n_act == 0) break;  // the same for the whole CTA: the chunk is drained
    const bool active = my >= 0;
    float* A = app + (lane_ok ? slot : 0) * N;
    if (a.iterations > 0) {
      int cwo = 2 * sh.mb;
      for (int l = 0; l < sh.mb; ++l) {
        const int lb = s_loff[l], deg = s_loff[l + 1] - lb;
        if (active) layer_f32c_lean(s_edge, lb, deg, Z, zi, A, st, ns, 2 * l, cwo, a.beta);
        cwo += max(1, (deg + 15) >> 4);
        __syncthreads();
      }
      if (lane_ok && zi == 0) h->slot_fail[slot] = 0;
      __syncthreads();
      if (active && syndrome_fails(s_edge, s_loff, sh.mb, Z, zi, A)) h->slot_fail[slot] = 1;
      __syncthreads();
      if (tid < cpb && h->slot_cw[tid] >= 0) ++h->slot_used[tid];
      __syncthreads();
    }
    // results of the codewords that stop here: zero syndrome, or the iteration limit
    const bool fin = active && (a.iterations == 0 || h->slot_fail[slot] == 0 || h->slot_used[slot] >= a.iterations);
    if (fin) {
      const WmCodeword rec = a.cws[my];
      if (zi == 0 && a.iters) a.iters[rec.index] = h->slot_used[slot];
      const int nwords = (rec.hard_bits + 31) >> 5;
      for (int w = zi; w < nwords; w += Z) {
        uint32_t m = 0u;
        for (int b = 0; b < 32; ++b) {
          const int j = 32 * w + b;
          if (j < rec.hard_bits && A[j] < 0.0f) m |= 1u << b;
        }
        a.out[rec.out_off + w] = m;
      }
    }
    __syncthreads();
    if (fin && zi == 0) h->slot_cw[slot] = -1;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kWmThreads, 2) wifi_mixed_f32_kernel(const __grid_constant__ WmArgs a) {
  WmHdr* h = reinterpret_cast<WmHdr*>(wm_smem);
  if (threadIdx.x == 0) h->pending = -1;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      int c = h->pending;  // the chunk that ended the previous session, if any
      if (c < 0) c = (int)atomicAdd(a.queue, 1u);
      h->chunk = c;
    }
    __syncthreads();
    const int c = h->chunk;
    if (c >= a.n_chunks) break;
    wm_session(a, a.shapes[a.chunks[c].shape]);
  }
}

}  // namespace

Decoder::~Decoder() {
  if (device_ >= 0) {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device_);
    cudaFree(d_edge_);
    cudaFree(d_loff_);
    if (prev >= 0) cudaSetDevice(prev);
  }
}

bool Decoder::init(const Graph& g, float offset_beta, std::string* err) {
  if (pick_maxdeg(g.maxdeg) < 0) {
    if (err) *err = "layer degree above 24 is not supported by the GPU kernels";
    return false;
  }
  if (g.n() > 65535 * 4) {
    if (err) *err = "code too long";
    return false;
  }
  // The shared-memory address arithmetic needs each column to appear at most once per layer.
  for (int l = 0; l < g.mb; ++l)
    for (int e = g.layer_off[l]; e < g.layer_off[l + 1]; ++e)
      for (int f = g.layer_off[l]; f < e; ++f)
        if (g.cols[f] == g.cols[e]) {
          if (err) *err = "a column appears twice in one layer";
          return false;
        }
  g_ = g;
  beta_ = offset_beta;
  if (cudaGetDevice(&device_) != cudaSuccess) {
    if (err) *err = "no CUDA device";
    device_ = -1;
    return false;
  }
  std::vector<uint32_t> ew(g.edges());
  for (int e = 0; e < g.edges(); ++e) ew[e] = ((uint32_t)(g.cols[e] * g.z) << 16) | (uint32_t)g.shifts[e];
  if (cudaMalloc(&d_edge_, sizeof(uint32_t) * std::max(1, g.edges())) != cudaSuccess ||
      cudaMalloc(&d_loff_, sizeof(int32_t) * (g.mb + 1)) != cudaSuccess) {
    if (err) *err = "cudaMalloc failed for the layer tables";
    return false;
  }
  cudaMemcpy(d_edge_, ew.data(), sizeof(uint32_t) * g.edges(), cudaMemcpyHostToDevice);
  cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_);
  nr_bg_ = -1;
  if ((g.kind == GraphKind::kNrBg1 || g.kind == GraphKind::kNrBg2) && g.maxdeg <= 31) {
    const int bg = g.kind == GraphKind::kNrBg1 ? 0 : 1;
    bool ok = nr_layout_matches(bg, g.cols.data(), g.edges());
    for (int l = 4; ok && l < g.mb; ++l)
      for (int e = g.layer_off[l]; e < g.layer_off[l + 1]; ++e)
        if (g.cols[e] == g.kb + l && g.shifts[e] != 0) ok = false;
    if (ok) nr_bg_ = bg;
  }
  cudaMemcpy(d_loff_, g.layer_off.data(), sizeof(int32_t) * (g.mb + 1), cudaMemcpyHostToDevice);
  return cudaGetLastError() == cudaSuccess;
}

Decoder::Geometry Decoder::geometry(Precision p, long long batch, bool compress) const {
  Geometry geo{};
  const int elem = p == Precision::kInt8 ? 2 : 4;
  const int Z = g_.z;
  const long long N = g_.n();
  int cpb = std::max(1, std::min(64, kMaxThreads / Z));
  while (cpb > 1 && table_bytes(g_.edges(), g_.mb, cpb) + (long long)cpb * N * elem > 100 * 1024) --cpb;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_ < 0 ? 0 : device_);
  // a batch too small to give every SM a full group spreads over the SMs in smaller
  // groups (the kernels are latency-bound: fewer codewords per CTA finish sooner)
  if (batch > 0) cpb = (int)std::min<long long>(cpb, std::max<long long>(1, (batch + sms - 1) / std::max(sms, 1)));
  geo.cpb = cpb;
  geo.threads = ((cpb * Z + 31) / 32) * 32;
  geo.smem = table_bytes(g_.edges(), g_.mb, cpb) + (int)(cpb * N * elem);
  geo.maxdeg_tmpl = pick_maxdeg(g_.maxdeg);
  geo.st_words = 0;
  geo.st_off = 0;
  if (compress) {
    // compressed messages in shared memory when two CTAs still fit an SM: per layer
    // two magnitude words (f32) or one (int8, both magnitudes in bytes), then code words
    int words = (p == Precision::kF32 ? 2 : 1) * g_.mb;
    for (int l = 0; l < g_.mb; ++l) words += std::max(1, (g_.layer_off[l + 1] - g_.layer_off[l] + 15) / 16);
    const long long off = align16(geo.smem);
    const long long total = off + (long long)geo.threads * words * 4;
    if (total <= kCompressedSmem) {
      geo.st_words = words;
      geo.st_off = (int)off;
      geo.smem = (int)total;
    }
  }
  KernelFn fn = kernel_for(p, geo.maxdeg_tmpl, geo.st_words > 0);
  allow_max_dynamic_smem((const void*)fn);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, geo.threads, geo.smem);
  geo.max_ctas = std::max(1, per_sm) * std::max(1, sms);
  return geo;
}

size_t Decoder::workspace_bytes(Precision p, long long batch) const {
  // the messages of the global-memory kernel (kernel 4, or where the compressed state
  // does not fit shared memory); the compressed kernels need none
  const Geometry geo = geometry(p, batch, false);
  const long long groups = (batch + geo.cpb - 1) / geo.cpb;
  const long long ctas = std::min<long long>(groups, geo.max_ctas);
  const long long elem = p == Precision::kInt8 ? 1 : 4;
  size_t bytes = (size_t)(ctas * geo.cpb * g_.edge_buffer() * elem);
  if (p == Precision::kF32 && nr_bg_ >= 0 && nr_f32_applies(nr_bg_, g_.z))
    bytes = std::max(bytes, nr_f32_workspace_bytes(nr_bg_, g_.z, batch, sms_));
  return bytes;
}

cudaError_t Decoder::decode(Precision p, const BatchRequest& req, cudaStream_t stream,
                            std::string* err) const {
  auto bad = [&](const char* m) {
    if (err) *err = m;
    return cudaErrorInvalidValue;
  };
  if (req.batch < 0) return bad("batch must be non-negative");
  if (req.batch == 0) return cudaSuccess;
  if (!req.llr) return bad("llr is null");
  if (req.iterations < 0) return bad("iterations must be non-negative");
  if (req.llr_offset < 0 || req.llr_offset > g_.n()) return bad("llr_offset out of range");
  if (req.hard_packed && (req.hard_bits < 0 || req.hard_bits > g_.n() ||
                          req.hard_words_stride < (req.hard_bits + 31) / 32))
    return bad("hard_bits / hard_words_stride out of range");
  if (req.app_clamp < 0 && p == Precision::kInt8) return bad("app_clamp must be non-negative");
  if (req.shorten) {
    if (p != Precision::kF32) return bad("shortened / punctured decodes are f32");
    if (req.llr_offset != 0 || req.prologue_5g) return bad("a shortened decode takes no llr_offset or 5G prologue");
    if (req.shorten_payload < 0 || req.shorten_payload > g_.k() || req.shorten_tx < req.shorten_payload ||
        req.shorten_tx > g_.n() - (g_.k() - req.shorten_payload))
      return bad("payload / transmitted bit counts out of range");
    if (req.llr_stride < req.shorten_tx) return bad("llr_stride smaller than the transmitted bits");
  }
  const bool nr_ok = p == Precision::kInt8 && nr_bg_ >= 0 && !req.llr_i16 && req.app_clamp >= 255;
  if ((req.kernel == 2 || req.kernel == 3 || req.kernel == 5) && !nr_ok)
    return bad("the 5G NR kernel does not apply to this request");
  const bool generic_only = req.kernel == 1 || req.kernel == 4;
  if (nr_ok && !generic_only) {
    NrCommon c{};
    c.z = g_.z;
    c.beta_q = req.beta_q;
    c.app_clamp = req.app_clamp;
    c.prologue = req.prologue_5g;
    c.k = (int)g_.k();
    c.k_prime = req.n_filler > g_.k() ? 0 : g_.k() - req.n_filler;
    c.llr = static_cast<const int8_t*>(req.llr);
    c.llr_stride = req.llr_stride;
    c.llr_offset = req.llr_offset;
    c.batch = req.batch;
    c.cpb = std::min<long long>(nr_cpb(nr_bg_, g_.z), req.batch);
    c.iterations = req.iterations;
    c.hard_packed = req.hard_packed;
    c.hard_bits = req.hard_bits;
    c.hard_words_stride = req.hard_words_stride;
    c.iters = req.iters;
    c.app_out = static_cast<int16_t*>(req.app);
    c.app_stride = req.app_stride;
    c.edge_r_out = static_cast<int8_t*>(req.edge_r);
    c.edge_r_stride = req.edge_r_stride;
    c.hard_out = req.hard;
    c.hard_stride = req.hard_stride;
    const bool pair_ok = nr_pair_applies(c);
    if ((req.kernel == 3 || req.kernel == 5) && !pair_ok)
      return bad("the paired 5G NR kernel needs app_clamp >= 3938 (7874 with filler)");
    if (pair_ok && req.kernel != 2)
      return nr_pair_decode_i8(nr_bg_, c, g_.shifts.data(), sms_, stream, req.kernel != 5);
    return nr_decode_i8(nr_bg_, c, g_.shifts.data(), sms_, stream);
  }
  // f32 5G NR: the compressed-message kernel, when the caller's workspace holds its
  // extension posteriors (else the generic kernel below).
  if (p == Precision::kF32 && nr_bg_ >= 0 && nr_f32_applies(nr_bg_, g_.z) && !req.shorten && !generic_only &&
      req.workspace && req.workspace_bytes >= nr_f32_workspace_bytes(nr_bg_, g_.z, req.batch, sms_)) {
    NrF32Common c;
    c.llr = static_cast<const float*>(req.llr);
    c.llr_stride = req.llr_stride;
    c.llr_offset = req.llr_offset;
    c.batch = req.batch;
    c.iterations = req.iterations;
    c.beta = req.beta;
    c.prologue = req.prologue_5g;
    c.k_prime = req.n_filler > g_.k() ? 0 : g_.k() - req.n_filler;
    c.hard_packed = req.hard_packed;
    c.hard_bits = req.hard_bits;
    c.hard_words_stride = req.hard_words_stride;
    c.iters = req.iters;
    c.app_out = static_cast<float*>(req.app);
    c.app_stride = req.app_stride;
    c.edge_r_out = static_cast<float*>(req.edge_r);
    c.edge_r_stride = req.edge_r_stride;
    c.hard_out = req.hard;
    c.hard_stride = req.hard_stride;
    c.ext_ws = static_cast<float*>(req.workspace);
    return nr_f32_decode(nr_bg_, c, g_.z, g_.shifts.data(), sms_, stream);
  }
  const Geometry geo = geometry(p, req.batch, req.kernel != 4);
  const long long groups = (req.batch + geo.cpb - 1) / geo.cpb;
  const long long ctas = std::min<long long>(groups, geo.max_ctas);
  if (!req.edge_r && geo.st_words == 0) {
    const long long elem = p == Precision::kInt8 ? 1 : 4;
    const long long need = ctas * geo.cpb * g_.edge_buffer() * elem;
    if (!req.workspace || (long long)req.workspace_bytes < need) return bad("workspace too small");
  }
  KArgs a{};
  a.z = g_.z;
  a.mb = g_.mb;
  a.n_edges = g_.edges();
  a.n = (int)g_.n();
  a.k = (int)g_.k();
  a.edge = d_edge_;
  a.loff = d_loff_;
  a.llr = req.llr;
  a.llr_stride = req.llr_stride;
  a.llr_offset = req.llr_offset;
  a.llr_i16 = req.llr_i16;
  a.batch = req.batch;
  a.cpb = geo.cpb;
  a.iterations = req.iterations;
  a.beta_q = req.beta_q;
  a.app_clamp = req.app_clamp;
  a.beta = req.beta;
  a.prologue = req.prologue_5g;
  a.k_prime = req.n_filler > g_.k() ? 0 : g_.k() - req.n_filler;
  a.shorten = req.shorten;
  a.sh_pay = req.shorten_payload;
  a.sh_par_end = g_.k() + (req.shorten_tx - req.shorten_payload);
  a.r_out = req.edge_r;
  a.r_out_stride = req.edge_r_stride;
  a.r_ws = req.workspace;
  a.hard_packed = req.hard_packed;
  a.hard_bits = req.hard_bits;
  a.hard_words_stride = req.hard_words_stride;
  a.iters = req.iters;
  a.app_out = req.app;
  a.app_stride = req.app_stride;
  a.hard_out = req.hard;
  a.hard_stride = req.hard_stride;
  a.st_words = geo.st_words;
  a.st_off = geo.st_off;
  KernelFn fn = kernel_for(p, geo.maxdeg_tmpl, geo.st_words > 0);
  fn<<<(unsigned)ctas, geo.threads, geo.smem, stream>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free entry (syndrome_ldpc_decode_batch_i8_noalloc).
//
// Some callers cannot allocate device memory at decode time: a baseband thread
// working to a per-slot deadline must not call cudaMalloc, which can synchronise
// the device and take milliseconds, and a plug-in hosted by an application that
// owns every device allocation has no allocator to call.  This entry runs the
// generic int8 kernel above with its message scratch in the static array below,
// which every GPU that loads this library holds until the process exits.
//
// The scratch holds the check-to-variable messages of the CTAs resident at once.
// A launch uses at most kNoAllocScratchBytes / (codewords per CTA x edges x Z)
// CTAs (the persistent kernel walks the batch with however many it gets); a code
// whose messages for one CTA exceed the array is rejected.  The kernel writes
// every message before it reads it within a decode, so nothing in the array has
// to start at zero, and the array keeps the last call's contents.  Calls that
// overlap on the GPU (different streams, or different host threads without
// ordering) share the array and race.

namespace {
constexpr size_t kNoAllocScratchBytes = Decoder::kNoAllocScratchBytes;
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};
}  // namespace

static __device__ __align__(256) int8_t g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the static scratch on the current device, looked up once per
// device (the first call on a device does the lookup) and kept for the life of the
// process: a cudaDeviceReset, or anything else that tears down and recreates the
// device's primary context, leaves the kept address stale, so calls must not cross
// one.
static cudaError_t noalloc_scratch(int device, void** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[device] = p;
  }
  *out = g_noalloc_addr[device];
  return cudaSuccess;
}

cudaError_t Decoder::decode_i8_noalloc(const BatchRequest& req, cudaStream_t stream, std::string* err) const {
  auto bad = [&](const std::string& m) {
    if (err) *err = m;
    return cudaErrorInvalidValue;
  };
  if (req.batch < 0) return bad("batch must be non-negative");
  if (req.batch == 0) return cudaSuccess;
  if (!req.llr) return bad("llr is null");
  if (req.iterations < 0) return bad("iterations must be non-negative");
  if (req.llr_offset < 0 || req.llr_offset > g_.n()) return bad("llr_offset out of range");
  if (req.hard_packed && (req.hard_bits < 0 || req.hard_bits > g_.n() ||
                          req.hard_words_stride < (req.hard_bits + 31) / 32))
    return bad("hard_bits / hard_words_stride out of range");
  if (req.app_clamp < 0) return bad("app_clamp must be non-negative");
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  if (cur != device_) return bad("the current device is not the decoder's device");
  // 5G NR graphs: the NR kernels keep their check-row state on chip and need no device
  // memory beyond the caller's outputs, so the decoder's own choice runs unchanged
  if (nr_bg_ >= 0 && !req.llr_i16 && req.app_clamp >= 255 && req.kernel != 1 && req.kernel != 4)
    return decode(Precision::kInt8, req, stream, err);
  void* scratch = nullptr;
  e = noalloc_scratch(cur, &scratch);
  if (e != cudaSuccess) return e;
  const Geometry geo = geometry(Precision::kInt8, req.batch, false);
  const long long per_cta = (long long)geo.cpb * g_.edge_buffer();
  if (per_cta > (long long)kNoAllocScratchBytes)
    return bad("the messages of one CTA (" + std::to_string(per_cta) + " bytes) exceed the " +
               std::to_string(kNoAllocScratchBytes) + "-byte static scratch of the allocation-free entry");
  const long long groups = (req.batch + geo.cpb - 1) / geo.cpb;
  const long long fit = (long long)kNoAllocScratchBytes / per_cta;
  const long long ctas = std::min<long long>(std::min<long long>(groups, geo.max_ctas), fit);
  KArgs a{};
  a.z = g_.z;
  a.mb = g_.mb;
  a.n_edges = g_.edges();
  a.n = (int)g_.n();
  a.k = (int)g_.k();
  a.edge = d_edge_;
  a.loff = d_loff_;
  a.llr = req.llr;
  a.llr_stride = req.llr_stride;
  a.llr_offset = req.llr_offset;
  a.llr_i16 = req.llr_i16;
  a.batch = req.batch;
  a.cpb = geo.cpb;
  a.iterations = req.iterations;
  a.beta_q = req.beta_q;
  a.app_clamp = req.app_clamp;
  a.beta = req.beta;
  a.prologue = req.prologue_5g;
  a.k_prime = req.n_filler > g_.k() ? 0 : g_.k() - req.n_filler;
  a.r_out = req.edge_r;
  a.r_out_stride = req.edge_r_stride;
  a.r_ws = scratch;
  a.hard_packed = req.hard_packed;
  a.hard_bits = req.hard_bits;
  a.hard_words_stride = req.hard_words_stride;
  a.iters = req.iters;
  a.app_out = req.app;
  a.app_stride = req.app_stride;
  a.hard_out = req.hard;
  a.hard_stride = req.hard_stride;
  KernelFn fn = kernel_for(Precision::kInt8, geo.maxdeg_tmpl);
  fn<<<(unsigned)ctas, geo.threads, geo.smem, stream>>>(a);
  return cudaGetLastError();
}

int wifi_mixed_smem_bytes(const WmShape& s) {
  return kWmHdr + kWmTab + align16(s.cpb * s.n * 4) + s.st_words * kWmThreads * 4;
}

cudaError_t wifi_mixed_prepare(int smem, int* ctas_per_sm) {
  cudaError_t e = allow_max_dynamic_smem((const void*)wifi_mixed_f32_kernel);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wifi_mixed_f32_kernel, kWmThreads, smem);
  if (e != cudaSuccess) return e;
  *ctas_per_sm = std::max(per_sm, 1);
  return cudaSuccess;
}

cudaError_t wifi_mixed_launch(const WmArgs& a, int ctas, int smem, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  if (a.n_chunks <= 0) return cudaSuccess;
  wifi_mixed_f32_kernel<<<std::max(1, std::min(ctas, a.n_chunks)), kWmThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace syn
