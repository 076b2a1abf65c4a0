// f32 layered offset min-sum for the 5G NR base graphs at Z = 384 on sm_100a, with the
// check-to-variable messages compressed in shared memory.
//
// Arithmetic of syndrome src/qc_ldpc.rs:1146-1205 (the scalar f32 pass): Q = app - R_old,
// min1/min2 of |Q| (a tie moves min1 to min2), R_new = sign * max(mex - beta, 0) with
// mex = min2 where |Q| == min1 and min1 elsewhere, sign = the row's sign parity times
// Q's sign, app += R_new - R_old; all in round-to-nearest f32 in the reference's order.
// The messages of a row are therefore a function of two magnitudes,
// max(min1 - beta, 0) and max(min2 - beta, 0), and two bits per edge (|Q| == min1,
// R's sign bit), from which R_old is rebuilt bit for bit (signed zeros included):
// 8 bytes per row plus 2 bits per edge instead of 4 bytes per edge.
//
// One codeword per CTA of 384 threads (thread z owns row z of every layer and the
// variables (column, z)).  Shared memory: the f32 posteriors of the KB + 4 core columns
// and the compressed state (magnitudes and code bits word-major per thread).  The
// extension columns' posteriors (one per layer >= 4, touched only by that layer's row
// z) cannot be recomputed from channel value + message (f32 rounding makes the running
// sum path-dependent), so each thread keeps its own in a per-CTA global buffer: a
// coalesced load per row, issued early (global and shared accesses never alias).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "nr_graph.cuh"
#include "nr_kernels.h"
#include "smem_limit.h"

namespace syn {
namespace nrf {

using nr::barrier_after;
using nr::deg_of;
using nr::ext_pos;
using nr::static_for;
using nr::Tab;

constexpr int kZ = 384;        // the compile-time lifting size
constexpr int kThreads = 384;  // most threads (codeword rows) per CTA

extern __shared__ __align__(16) unsigned char f32_smem[];

template <int BG>
struct Layout {
  static constexpr int CORE = Tab<BG>::KB + 4, NEXT = Tab<BG>::MB - 4;
  static constexpr int NMAG = 2 * Tab<BG>::MB;                // two magnitudes per row
  static constexpr int NCODE = (2 * Tab<BG>::E + 31) / 32;    // 2 bits per edge, packed across rows
  static constexpr int APP = 16;                              // byte offset of the core posteriors
  static constexpr int MAG = APP + CORE * kZ * 4;             // state words: [word][thread]
  static constexpr int CODE = MAG + NMAG * kThreads * 4;
  static constexpr int BYTES = CODE + NCODE * kThreads * 4;
};

// Any lifting size (ZT = 0): cpb = min(384 / Z, batch) codewords per CTA, thread t
// owning row t % Z of codeword slot t / Z.  Shared memory: a flag word per slot and
// stage, the state words laid out as at Z = 384 (compile-time offsets), then the slots'
// core posteriors.
template <int BG>
struct RtLayout {
  static constexpr int FLAGS = 0;
  static constexpr int MAG = 2 * kThreads * 4;
  static constexpr int CODE = MAG + Layout<BG>::NMAG * kThreads * 4;
  static constexpr int APP = CODE + Layout<BG>::NCODE * kThreads * 4;
  __host__ __device__ static constexpr int bytes(int z, int cpb) { return APP + cpb * Layout<BG>::CORE * z * 4; }
};

template <int BG>
struct F32Args {
  NrF32Common c;
  int z, cpb;
  int sh4[Tab<BG>::E];  // 4 * shift of each edge, reduced mod z (ZT = 0)
  int cz4[Tab<BG>::E];  // 4 * col * z
};

// ZT = 384: shifts, column bases and the shared-memory layout are compile-time
// constants.  ZT = 0: any Z, shifts and column bases from the kernel parameters.
template <int BG, int ZT>
struct Ctx {
  static constexpr int MAGB = ZT > 0 ? Layout<BG>::MAG : RtLayout<BG>::MAG;
  static constexpr int CODEB = ZT > 0 ? Layout<BG>::CODE : RtLayout<BG>::CODE;
  int tid;
  int z4;
  int Z4;   // 4 * Z (ZT = 0)
  int ap;   // byte offset of this slot's core posteriors (ZT = 0)
  float* ext;  // this thread's extension posteriors: ext[(layer - 4) * 384]
  const F32Args<BG>* a;
  template <int GE>
  __device__ __forceinline__ int vb() const {
    int zl = z4;
    asm volatile("" : "+r"(zl));  // keeps the unrolled graph's addresses from being hoisted
    if constexpr (ZT > 0) {
      const unsigned r = (unsigned)(zl + Tab<BG>::z384_shift(GE) * 4);
      const unsigned rr = min(r, r - (unsigned)(kZ * 4));
      return (int)rr + Tab<BG>::col(GE) * kZ * 4;
    } else {
      const unsigned r = (unsigned)(zl + a->sh4[GE]);
      const unsigned rr = min(r, r - (unsigned)Z4);
      return (int)rr + a->cz4[GE];
    }
  }
  __device__ __forceinline__ int apb() const { return ZT > 0 ? Layout<BG>::APP : ap; }
  __device__ __forceinline__ float ld_ap(int b) const {
    return *reinterpret_cast<const float*>(f32_smem + apb() + b);
  }
  __device__ __forceinline__ void st_ap(int b, float v) const {
    *reinterpret_cast<float*>(f32_smem + apb() + b) = v;
  }
  __device__ __forceinline__ float ld_mag(int w) const {
    return *reinterpret_cast<const float*>(f32_smem + MAGB + 4 * (w * kThreads + tid));
  }
  __device__ __forceinline__ void st_mag(int w, float v) const {
    *reinterpret_cast<float*>(f32_smem + MAGB + 4 * (w * kThreads + tid)) = v;
  }
  __device__ __forceinline__ uint32_t ld_code(int w) const {
    return *reinterpret_cast<const uint32_t*>(f32_smem + CODEB + 4 * (w * kThreads + tid));
  }
  __device__ __forceinline__ void st_code(int w, uint32_t v) const {
    *reinterpret_cast<uint32_t*>(f32_smem + CODEB + 4 * (w * kThreads + tid)) = v;
  }
  __device__ __forceinline__ float ld_ext(int i) const { return ext[i * kThreads]; }
  __device__ __forceinline__ void st_ext(int i, float v) const { ext[i * kThreads] = v; }
};

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

// R_old of edge e from the row's magnitudes and the edge's two code bits
// (bit 0: |Q| was the row minimum, bit 1: R's sign).
__device__ __forceinline__ float message(float magA, float magB, unsigned bb) {
  return __uint_as_float(__float_as_uint((bb & 1u) ? magB : magA) | ((bb & 2u) << 30));
}

template <int BG, int ZT, int L>
__device__ __forceinline__ void row(const Ctx<BG, ZT>& c, float beta) {
  constexpr int lb = Tab<BG>::loff(L), deg = deg_of<BG>(L);
  constexpr int ep = L >= 4 ? ext_pos<BG>(L) : -1;
  constexpr int b0 = 2 * lb, w0 = b0 >> 5, w1 = (b0 + 2 * deg - 1) >> 5, sh = b0 & 31;
  float av[deg], qv[deg];
  int vb[deg];
  // the extension posterior first: a global load, the longest latency of the row
  if constexpr (ep >= 0) av[ep] = c.ld_ext(L - 4);
  const float magA = c.ld_mag(2 * L), magB = c.ld_mag(2 * L + 1);
  const uint32_t lo = c.ld_code(w0);
  const uint32_t hi = w1 != w0 ? c.ld_code(w1) : 0u;
  const unsigned long long word = ((unsigned long long)hi << 32) | lo;
  const unsigned long long bits = word >> sh;
  float m1, m2, ak[deg];
  unsigned sx = 0u;
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    if constexpr (e != ep) {
      vb[e] = c.template vb<lb + e>();
      av[e] = c.ld_ap(vb[e]);
    }
    const float ro = message(magA, magB, (unsigned)(bits >> (2 * e)) & 3u);
    const float q = __fsub_rn(av[e], ro);
    qv[e] = q;
    const unsigned b = __float_as_uint(q);
    ak[e] = fminf(__uint_as_float(b & 0x7FFFFFFFu), FLT_MAX);
    sx ^= b & 0x80000000u;
  });
  min2_tree<deg>(ak, m1, m2);
  if (m1 == FLT_MAX) m1 = 0.0f;
  if (m2 == FLT_MAX) m2 = m1;
  float nA = __fsub_rn(m1, beta), nB = __fsub_rn(m2, beta);  // messages of the non-minimum / minimum edges
  if (nA < 0.0f) nA = 0.0f;
  if (nB < 0.0f) nB = 0.0f;
  unsigned long long nbits = 0ull;
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    const unsigned b = __float_as_uint(qv[e]);
    const float aq = __uint_as_float(b & 0x7FFFFFFFu);
    const unsigned sgn = sx ^ (b & 0x80000000u);
    const bool is_min = aq == m1;
    const float nr = __uint_as_float(__float_as_uint(is_min ? nB : nA) | sgn);
    const float ro = message(magA, magB, (unsigned)(bits >> (2 * e)) & 3u);
    const float nv = __fadd_rn(av[e], __fsub_rn(nr, ro));
    if constexpr (e == ep)
      c.st_ext(L - 4, nv);
    else
      c.st_ap(vb[e], nv);
    nbits |= (unsigned long long)((is_min ? 1u : 0u) | (sgn >> 30)) << (2 * e);
  });
  c.st_mag(2 * L, nA);
  c.st_mag(2 * L + 1, nB);
  constexpr unsigned long long mask = ((deg >= 32 ? 0ull : (1ull << (2 * deg))) - 1ull) << sh;
  const unsigned long long nw = (word & ~mask) | ((nbits << sh) & mask);
  c.st_code(w0, (uint32_t)nw);
  if constexpr (w1 != w0) c.st_code(w1, (uint32_t)(nw >> 32));
}

// Odd parity of check row (L, z) (qc_ldpc.rs:1231-1252: negative = app < 0).
template <int BG, int ZT, int L>
__device__ __forceinline__ bool row_odd(const Ctx<BG, ZT>& c) {
  constexpr int lb = Tab<BG>::loff(L), deg = deg_of<BG>(L);
  constexpr int ep = L >= 4 ? ext_pos<BG>(L) : -1;
  unsigned par = 0u;
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    const float v = e == ep ? c.ld_ext(L - 4) : c.ld_ap(c.template vb<lb + e>());
    par ^= v < 0.0f ? 1u : 0u;
  });
  return par != 0u;
}

// The syndrome check in two stages: the few smallest layers for every iteration, the
// others only when those pass (nr::is_quick); the second stage out of line.
template <int BG, int ZT>
__device__ __forceinline__ bool quick_odd(const Ctx<BG, ZT>& c) {
  bool odd = false;
  static_for<0, Tab<BG>::MB>([&](auto li) {
    constexpr int L = decltype(li)::value;
    if constexpr (nr::is_quick<BG>(L)) odd = odd || row_odd<BG, ZT, L>(c);
  });
  return odd;
}
template <int BG, int ZT>
__device__ __noinline__ bool rest_odd(const Ctx<BG, ZT> c) {
  bool odd = false;
  static_for<0, Tab<BG>::MB>([&](auto li) {
    constexpr int L = decltype(li)::value;
    if constexpr (!nr::is_quick<BG>(L)) odd = odd || row_odd<BG, ZT, L>(c);
  });
  return odd;
}

// Bytes [0, bytes) of a codeword's row into L2, one 128-byte line per thread and step;
// every address lies inside the row.
__device__ __noinline__ void prefetch_row_l2(const char* row, long long bytes, int z, int Z) {
  for (long long i = 128LL * z; i < bytes; i += 128LL * Z)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(row + i)));
}

// Results of the codewords of group g (out of line: keeps the iteration loop's registers
// free).  on: this thread's row z of slot `slot` holds codeword g * cpb + slot.
template <int BG, int ZT>
__device__ __noinline__ void write_out(const F32Args<BG>* pa, const Ctx<BG, ZT> c, long long g, int slot, int z,
                                       bool on, int used) {
  using T = Tab<BG>;
  constexpr int CORE = Layout<BG>::CORE;
  const NrF32Common* a = &pa->c;
  const int Z = ZT > 0 ? kZ : pa->z, cpb = ZT > 0 ? 1 : pa->cpb;
  const int lane = c.tid & 31, warp = c.tid >> 5;
  const long long cw = g * cpb + slot;
  if (on) {
    const float* A = reinterpret_cast<const float*>(f32_smem + c.apb());
    if (z == 0 && a->iters) a->iters[cw] = used;
    if (a->app_out) {
      float* dst = a->app_out + cw * a->app_stride;
      for (int col = 0; col < T::NB; ++col) dst[col * Z + z] = col < CORE ? A[col * Z + z] : c.ld_ext(col - CORE);
    }
    if (a->hard_out) {
      uint8_t* dst = a->hard_out + cw * a->hard_stride;
      for (int col = 0; col < T::NB; ++col)
        dst[col * Z + z] = (col < CORE ? A[col * Z + z] : c.ld_ext(col - CORE)) < 0.0f ? 1 : 0;
    }
    if (a->edge_r_out) {
      float* er = a->edge_r_out + cw * a->edge_r_stride;
      static_for<0, T::MB>([&](auto li) {
        constexpr int L = decltype(li)::value;
        constexpr int lb = T::loff(L), deg = deg_of<BG>(L);
        constexpr int b0 = 2 * lb, w0 = b0 >> 5, w1 = (b0 + 2 * deg - 1) >> 5, sh = b0 & 31;
        const float magA = c.ld_mag(2 * L), magB = c.ld_mag(2 * L + 1);
        const unsigned long long word =
            ((unsigned long long)(w1 != w0 ? c.ld_code(w1) : 0u) << 32) | c.ld_code(w0);
        static_for<0, deg>([&](auto ei) {
          constexpr int e = decltype(ei)::value;
          er[(long long)(lb + e) * Z + z] = message(magA, magB, (unsigned)((word >> sh) >> (2 * e)) & 3u);
        });
      });
    }
  }
  if (a->hard_packed) {
    // the extension posteriors are in global memory, written by their own threads
    __syncthreads();
    const int nwords = (a->hard_bits + 31) >> 5;
    const int nwarps = (int)(blockDim.x >> 5);
    const float* X = a->ext_ws + (long long)blockIdx.x * Layout<BG>::NEXT * kThreads;
    for (int t = warp; t < cpb * nwords; t += nwarps) {
      const int s = ZT > 0 ? 0 : t / nwords, w = t - s * nwords;
      if (g * cpb + s >= a->batch) continue;  // warp-uniform
      const float* A = reinterpret_cast<const float*>(
          f32_smem + (ZT > 0 ? Layout<BG>::APP : RtLayout<BG>::APP + s * CORE * Z * 4));
      const int j = (w << 5) + lane;
      bool bit = false;
      if (j < a->hard_bits) {
        float v;
        if (j < CORE * Z) {
          v = A[j];
        } else {
          const int i = (j - CORE * Z) / Z, zz = j - CORE * Z - i * Z;
          v = X[i * kThreads + s * Z + zz];
        }
        bit = v < 0.0f;
      }
      const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
      if (lane == 0) a->hard_packed[(g * cpb + s) * a->hard_words_stride + w] = m;
    }
  }
}

template <int BG, int ZT>
__global__ void __launch_bounds__(kThreads, 1) nr_f32_kernel(const __grid_constant__ F32Args<BG> pa) {
  using T = Tab<BG>;
  using LY = Layout<BG>;
  constexpr int CORE = LY::CORE, NEXT = LY::NEXT;
  const NrF32Common& a = pa.c;
  const int tid = threadIdx.x;
  const int Z = ZT > 0 ? kZ : pa.z, cpb = ZT > 0 ? 1 : pa.cpb, K = T::KB * Z;
  const int slot0 = ZT > 0 ? 0 : tid / Z;
  const bool live = slot0 < cpb;  // threads past cpb * Z only join the barriers
  const int slot = min(slot0, cpb - 1);
  const int z = ZT > 0 ? tid : (live ? tid - slot0 * Z : 0);
  Ctx<BG, ZT> c;
  c.tid = tid;
  c.z4 = z * 4;
  c.Z4 = Z * 4;
  c.ap = RtLayout<BG>::APP + slot * CORE * Z * 4;
  c.a = &pa;
  // [layer - 4][row of the CTA], the row of thread t being t (slot * Z + z)
  c.ext = a.ext_ws + (long long)blockIdx.x * NEXT * kThreads + tid;
  int* flag = reinterpret_cast<int*>(f32_smem + RtLayout<BG>::FLAGS);  // ZT = 0: [stage][slot]
  float* A = reinterpret_cast<float*>(f32_smem + c.apb());
  for (long long g = blockIdx.x; g * cpb < a.batch; g += gridDim.x) {
    const long long cw = g * cpb + slot;
    const bool on = live && cw < a.batch;
    __syncthreads();
    // ---- load (the f32 kernels' prologue: [0, llr_offset) erased, 5G init on top)
    if (on) {
      const float* src = a.llr + cw * a.llr_stride;
      auto value = [&](int j) -> float {
        float v = j >= a.llr_offset ? src[j - a.llr_offset] : 0.0f;
        if (a.prologue) {
          if (j < 2 * Z)
            v = 0.0f;
          else if (j >= a.k_prime && j < K)
            v = 1000000.0f;
        }
        return v;
      };
      for (int col = 0; col < CORE; ++col) A[col * Z + z] = value(col * Z + z);
#pragma unroll 1
      for (int i = 0; i < NEXT; ++i) c.st_ext(i, value((CORE + i) * Z + z));
    }
    // this slot's next codeword into L2 while this one decodes (its load then reads L2)
    if (live && (g + gridDim.x) * cpb + slot < a.batch)
      prefetch_row_l2(reinterpret_cast<const char*>(a.llr + ((g + gridDim.x) * cpb + slot) * a.llr_stride),
                      4LL * (T::NB * Z - a.llr_offset), z, Z);
#pragma unroll 1
    for (int w = 0; w < LY::NMAG; ++w) c.st_mag(w, 0.0f);
#pragma unroll 1
    for (int w = 0; w < LY::NCODE; ++w) c.st_code(w, 0u);
    __syncthreads();
    // ---- iterations with early stop on a zero syndrome (qc_ldpc.rs:1146-1221), per codeword
    int used = 0;
    bool active = on;
    for (int it = 0; it < a.iterations; ++it) {
      if (!__syncthreads_or(active)) break;
      if constexpr (ZT == 0) {
        if (tid < 2 * cpb) flag[tid] = 0;  // read back only after the layers' barriers
      }
      used += active ? 1 : 0;
      static_for<0, T::MB>([&](auto li) {
        constexpr int L = decltype(li)::value;
        if (ZT > 0 || active) row<BG, ZT, L>(c, a.beta);
        if constexpr (barrier_after<BG>(L)) __syncthreads();
      });
      if constexpr (ZT > 0) {
        bool odd = __syncthreads_or(quick_odd<BG, ZT>(c)) != 0;
        if (!odd) odd = __syncthreads_or(rest_odd<BG, ZT>(c)) != 0;
        active = odd;
      } else {
        if (active && quick_odd<BG, ZT>(c)) flag[slot] = 1;
        __syncthreads();
        bool odd = active && flag[slot] != 0;
        const bool rest = active && !odd;
        if (__syncthreads_or(rest)) {
          if (rest && rest_odd<BG, ZT>(c)) flag[cpb + slot] = 1;
          __syncthreads();
          odd = odd || (rest && flag[cpb + slot] != 0);
        }
        active = odd;
      }
    }
    write_out<BG, ZT>(&pa, c, g, slot, z, on, used);
  }
}

// Launch shape of the any-Z kernel: codewords per CTA, threads, shared memory, CTAs.
struct Plan {
  int cpb = 1, threads = kThreads, smem = 0;
  long long ctas = 0;
};

template <int BG>
Plan plan(int z, long long batch, int sms) {
  Plan p;
  if (batch <= 0) return p;
  if (z == kZ) {
    p.smem = Layout<BG>::BYTES;
    p.ctas = std::min<long long>(batch, std::max(sms, 1));
    return p;
  }
  p.cpb = (int)std::max<long long>(1, std::min<long long>(kThreads / z, batch));
  p.threads = ((p.cpb * z + 31) / 32) * 32;
  p.smem = RtLayout<BG>::bytes(z, p.cpb);
  int per_sm = 0;
  const void* fn = (const void*)nr_f32_kernel<BG, 0>;
  if (allow_max_dynamic_smem(fn) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, nr_f32_kernel<BG, 0>, p.threads, p.smem) !=
          cudaSuccess)
    per_sm = 1;
  const long long groups = (batch + p.cpb - 1) / p.cpb;
  p.ctas = std::min<long long>(groups, (long long)std::max(per_sm, 1) * std::max(sms, 1));
  return p;
}

template <int BG>
size_t workspace(int z, long long batch, int sms) {
  const Plan p = plan<BG>(z, batch, sms);
  return (size_t)p.ctas * Layout<BG>::NEXT * kThreads * sizeof(float);
}

template <int BG>
cudaError_t launch(const NrF32Common& c, int z, const int* shifts, int sms, cudaStream_t stream) {
  const Plan p = plan<BG>(z, c.batch, sms);
  if (p.ctas <= 0) return cudaSuccess;
  F32Args<BG> a;
  a.c = c;
  a.z = z;
  a.cpb = p.cpb;
  for (int e = 0; e < Tab<BG>::E; ++e) {
    a.sh4[e] = shifts ? shifts[e] * 4 : 0;
    a.cz4[e] = Tab<BG>::col(e) * z * 4;
  }
  if (z == kZ) {
    cudaError_t e = allow_max_dynamic_smem((const void*)nr_f32_kernel<BG, kZ>);
    if (e != cudaSuccess) return e;
    nr_f32_kernel<BG, kZ><<<(unsigned)p.ctas, kThreads, p.smem, stream>>>(a);
  } else {
    if (!shifts) return cudaErrorInvalidValue;
    cudaError_t e = allow_max_dynamic_smem((const void*)nr_f32_kernel<BG, 0>);
    if (e != cudaSuccess) return e;
    nr_f32_kernel<BG, 0><<<(unsigned)p.ctas, p.threads, p.smem, stream>>>(a);
  }
  return cudaGetLastError();
}

}  // namespace nrf

bool nr_f32_applies(int bg, int z) { return (bg == 0 || bg == 1) && z >= 2 && z <= nrf::kZ; }

size_t nr_f32_workspace_bytes(int bg, int z, long long batch, int sms) {
  return bg == 0 ? nrf::workspace<0>(z, batch, sms) : nrf::workspace<1>(z, batch, sms);
}

cudaError_t nr_f32_decode(int bg, const NrF32Common& c, int z, const int* shifts, int sms, cudaStream_t stream) {
  if (c.batch <= 0) return cudaSuccess;
  return bg == 0 ? nrf::launch<0>(c, z, shifts, sms, stream) : nrf::launch<1>(c, z, shifts, sms, stream);
}

}  // namespace syn
