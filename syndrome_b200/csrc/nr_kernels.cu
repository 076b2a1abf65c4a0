// int8 LOMS decode specialised for the 5G NR base graphs (BG1, BG2), sm_100a.
//
// Same arithmetic as the generic kernel (syndrome src/qc_ldpc.rs:1530-1758, int8
// messages, int16 posterior), restructured around three facts of the 5G graphs:
//
//  1. Layers >= 4 each own one extension parity column (column kb + layer, an
//     unshifted identity) that no other layer touches.  Its posterior is
//     channel + (that edge's message), so its variable-to-check message is the
//     channel value clamped to +-127 in every iteration, and it needs no shared
//     memory: the kernel keeps the int8 channel values of these columns and
//     rebuilds their posteriors at the end.  Valid when app_clamp >= 255 (the
//     posterior of such a column never reaches the clamp).
//  2. The base graph is fixed at compile time, so the layer loop and each layer's
//     edges are fully unrolled; each thread keeps the check-to-variable messages of
//     its check rows compressed in registers: per row min1', min2' (offset
//     magnitudes), the argmin edge and one sign bit per edge (the reference's
//     messages are exactly this function, ties included).  The per-Z cyclic
//     shifts arrive as kernel parameters (constant bank) and become index
//     arithmetic on the shared-memory posterior.
//  3. New magnitudes need no per-edge select: with S' = min1 + min2 - beta,
//     |R_new| = max(min1', S' - |Q|): the argmin edge (|Q| = min1) gets min2',
//     every other edge has |Q| >= min2 and gets min1' (ties give min2' = min1').
//     min1 / min2 / argmin come from one min-pair over keys |Q| * 32 + edge.
//
// One thread per lifting index z of each codeword slot; a CTA holds `cpb`
// codewords.  The syndrome check after each iteration tests the smallest layer
// first (it almost always fails before convergence) and the remaining layers only
// when that one passes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <type_traits>

#include "nr_graph.cuh"
#include "smem_limit.h"
#include "nr_kernels.h"

namespace syn {
namespace nr {

// Compressed state words of a layer: one when signs (deg bits) fit below bit 13.
template <int BG>
__host__ __device__ constexpr int words_of(int l) {
  return deg_of<BG>(l) <= 13 ? 1 : 2;
}
template <int BG>
__host__ __device__ constexpr int word_off(int l) {
  int w = 0;
  for (int i = 0; i < l; ++i) w += words_of<BG>(i);
  return w;
}

template <int BG>
struct Args {
  NrCommon c;
  int sh[Tab<BG>::E];  // shift of each edge (reduced mod z)
  int cz[Tab<BG>::E];  // col * z: first shared-memory posterior of the edge's column
};

// Where a layer reads its edges' cyclic shift and column base from.  The
// single-shape kernel passes them as kernel parameters (constant bank, indexed by
// compile-time edge numbers); the mixed-shape kernel stages them per work item in
// shared memory.
template <int BG>
struct ParamEdges {
  const Args<BG>& a;
  __device__ __forceinline__ int sh(int e) const { return a.sh[e]; }
  __device__ __forceinline__ int cz(int e) const { return a.cz[e]; }
};

struct SmemEdges {
  const int* __restrict__ s_sh;
  const int* __restrict__ s_cz;
  __device__ __forceinline__ int sh(int e) const { return s_sh[e]; }
  __device__ __forceinline__ int cz(int e) const { return s_cz[e]; }
};

// Per-launch scalars of a decode.
struct RunConsts {
  int z, beta_q, app_clamp, k32;
  unsigned two;
};

// Meta bits of a compressed row: argmin [13,18), min1' [18,25), min2' [25,32).
__device__ __forceinline__ uint32_t pack_meta(int idx, int m1p, int m2p) {
  return ((uint32_t)idx << 13) | ((uint32_t)m1p << 18) | ((uint32_t)m2p << 25);
}

// Message of edge e from a compressed row (sign word, meta word).
__device__ __forceinline__ int row_message(uint32_t signs, uint32_t meta, int e) {
  const int idx = (meta >> 13) & 31, m1p = (meta >> 18) & 127, m2p = meta >> 25;
  const int mag = idx == e ? m2p : m1p;
  return ((signs >> e) & 1u) ? -mag : mag;
}

// Top bit of x as 0 or 1, computed as the high word of x * two (two == 2 at run time),
// i.e. an IMAD.HI on the FMA pipe instead of a shift on the ALU pipe.
__device__ __forceinline__ int top_bit(int x, unsigned two) { return (int)__umulhi((unsigned)x, two); }

// Compressed rows live in shared memory, word-major: word w of thread t at st[w * ns + t].
//
// Instruction budget: on sm_100 every integer logic, shift, select, compare and
// min/max instruction issues to the ALU pipe (two warp instructions per clock per
// SM), as do plain integer adds, while IMAD issues to the FMA pipe at the same rate.
// The sign algebra below therefore uses multiplications by +-1: with
// sigma = (-1)^(sign bit of the row's XOR), R_new = sigma * (1 - 2*bit(u_e)) * mag_e,
// and the sign bits of the new messages are accumulated as acc -= sgn_e * 2^e
// (acc starting at 2^deg - 1 gives acc = 2 * sum(bit_e * 2^e)).
template <int BG, bool CLAMP, int L, class EDGES>
__device__ __forceinline__ void layer(const EDGES ed, const RunConsts rc, int z, int16_t* __restrict__ A,
                                      const int8_t* __restrict__ X, uint32_t* __restrict__ st, int ns) {
  using T = Tab<BG>;
  const int beta_q = rc.beta_q, C = rc.app_clamp;
  constexpr int lb = T::loff(L), deg = deg_of<BG>(L), W = word_off<BG>(L);
  constexpr bool two_words = words_of<BG>(L) == 2;
  const uint32_t w_signs = st[W * ns];
  const uint32_t w_meta = two_words ? st[(W + 1) * ns] : w_signs;
  const int idxo = (w_meta >> 13) & 31, m1o = (w_meta >> 18) & 127, m2o = w_meta >> 25;
  const int Z = rc.z;
  const int k32 = rc.k32;
  const unsigned two = rc.two;
  int vidx[deg], u[deg], ab[deg];
  int m1k = 4095, m2k = 4095;  // (127 << 5) | 31: the message ceiling, no edge
  int sx = 0;
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    if constexpr (is_ext<BG>(L, e)) {
      const int q = max((int)X[(L - 4) * Z + z], -127);
      u[e] = q;
      ab[e] = abs(q);
    } else {
      // (z + shift) mod Z as an unsigned min: below Z the second candidate wraps high.
      const unsigned r = (unsigned)(z + ed.sh(lb + e));
      const unsigned rr = min(r, r - (unsigned)Z);
      const int vi = (int)rr + ed.cz(lb + e);
      vidx[e] = vi;
      const int app = A[vi];
      const int mag = idxo == e ? m2o : m1o;
      u[e] = ((w_signs >> e) & 1u) ? app + mag : app - mag;  // app - R_old
      ab[e] = abs(u[e]);
    }
    sx ^= u[e];
    const int key = ab[e] * k32 + e;
    m2k = min(m2k, max(m1k, key));
    m1k = min(m1k, key);
  });
  const int m1 = m1k >> 5, m2 = m2k >> 5, idx = m1k & 31;
  const int m1p = max(m1 - beta_q, 0), m2p = max(m2 - beta_q, 0), sp = m1 + m2 - beta_q;
  const int sigma = 1 - 2 * top_bit(sx, two);
  const int m2sigma = -2 * sigma;
  int acc = (1 << deg) - 1;
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    const int sgn = top_bit(u[e], two) * m2sigma + sigma;  // sign of R_new
    acc -= sgn * (1 << e);
    if constexpr (!is_ext<BG>(L, e)) {
      const int mag = max(m1p, sp - ab[e]);
      int v = mag * sgn + u[e];
      if (CLAMP) v = min(max(v, -C), C);
      A[vidx[e]] = (int16_t)v;
    }
  });
  const uint32_t signs = (uint32_t)acc >> 1;
  const uint32_t meta = pack_meta(idx, m1p, m2p);
  if constexpr (two_words) {
    st[W * ns] = signs;
    st[(W + 1) * ns] = meta;
  } else {
    st[W * ns] = signs | meta;
  }
}

// Parity of check row (L, z) under the current posteriors: true if odd.
template <int BG, int L, class EDGES>
__device__ __forceinline__ bool row_parity(const EDGES ed, int Z, int z, const int16_t* __restrict__ A,
                                           const int8_t* __restrict__ X, const uint32_t* __restrict__ st,
                                           int ns) {
  using T = Tab<BG>;
  constexpr int lb = T::loff(L), deg = deg_of<BG>(L), W = word_off<BG>(L);
  constexpr bool two = words_of<BG>(L) == 2;
  unsigned par = 0;
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    if constexpr (is_ext<BG>(L, e)) {
      const uint32_t w0 = st[W * ns];
      const int r = row_message(w0, two ? st[(W + 1) * ns] : w0, e);
      par ^= ((int)X[(L - 4) * Z + z] + r) < 0 ? 1u : 0u;
    } else {
      const unsigned r = (unsigned)(z + ed.sh(lb + e));
      const int vi = (int)min(r, r - (unsigned)Z) + ed.cz(lb + e);
      par ^= A[vi] < 0 ? 1u : 0u;
    }
  });
  return par != 0;
}

// Runs up to `iterations` layered iterations with early stop on the CTA's codeword
// slots and returns the iterations this thread's slot used.  All threads of the CTA
// call it (it contains barriers); `active` says whether this thread owns a live
// check row.  Compressed rows are cleared first (messages start at zero).
template <int BG, bool CLAMP, class EDGES>
__device__ __forceinline__ int iterate(const EDGES ed, const RunConsts rc, bool active, bool lane_ok, int slot,
                                       int z, int16_t* __restrict__ A, const int8_t* __restrict__ X,
                                       uint32_t* __restrict__ st, int ns, int* s_flag, int iterations) {
  using T = Tab<BG>;
  constexpr int NWT = word_off<BG>(T::MB);
#pragma unroll 1
  for (int i = 0; i < NWT; ++i) st[i * ns] = 0;
  int used = 0;
  for (int it = 0; it < iterations; ++it) {
    if (!__syncthreads_or(active)) break;
    if (active) ++used;
    static_for<0, T::MB>([&](auto li) {
      constexpr int L = decltype(li)::value;
      if (active) layer<BG, CLAMP, L>(ed, rc, z, A, X, st, ns);
      __syncthreads();
    });
    if (lane_ok && z == 0) s_flag[slot] = 0;
    __syncthreads();
    if (active) {
      bool odd = false;
      static_for<0, T::MB>([&](auto li) {
        constexpr int L = decltype(li)::value;
        if constexpr (is_quick<BG>(L)) odd |= row_parity<BG, L>(ed, rc.z, z, A, X, st, ns);
      });
      if (odd) s_flag[slot] = 1;
    }
    __syncthreads();
    if (active && s_flag[slot] == 0) {
      bool odd = false;
      static_for<0, T::MB>([&](auto li) {
        constexpr int L = decltype(li)::value;
        if constexpr (!is_quick<BG>(L)) odd |= row_parity<BG, L>(ed, rc.z, z, A, X, st, ns);
      });
      if (odd) s_flag[slot] = 1;
    }
    __syncthreads();
    if (active && s_flag[slot] == 0) active = false;
  }
  return used;
}

// Posteriors of the extension columns (channel + the column's one message), written
// to app_out when given, and their hard decisions left in X for the output pass.
template <int BG>
__device__ __forceinline__ void finish_extension(int Z, int z, int8_t* __restrict__ X, const uint32_t* __restrict__ st,
                                                 int ns, int16_t* app_out_core_end) {
  using T = Tab<BG>;
  static_for<4, T::MB>([&](auto li) {
    constexpr int L = decltype(li)::value;
    constexpr int W = word_off<BG>(L);
    constexpr bool two = words_of<BG>(L) == 2;
    constexpr int e_ext = ext_pos<BG>(L);
    static_assert(e_ext >= 0, "every layer >= 4 has an extension column");
    const uint32_t w0 = st[W * ns];
    const int app = (int)X[(L - 4) * Z + z] + row_message(w0, two ? st[(W + 1) * ns] : w0, e_ext);
    if (app_out_core_end) app_out_core_end[(L - 4) * Z + z] = (int16_t)app;
    X[(L - 4) * Z + z] = app < 0 ? 1 : 0;
  });
}

// Messages of every edge in the reference's edge_r layout (edge-major, z fastest).
template <int BG>
__device__ __forceinline__ void write_messages(int Z, int z, const uint32_t* __restrict__ st, int ns,
                                               int8_t* __restrict__ R) {
  using T = Tab<BG>;
  static_for<0, T::MB>([&](auto li) {
    constexpr int L = decltype(li)::value;
    constexpr int W = word_off<BG>(L), lb = T::loff(L);
    constexpr bool two = words_of<BG>(L) == 2;
    static_for<0, deg_of<BG>(L)>([&](auto ei) {
      constexpr int e = decltype(ei)::value;
      const uint32_t w0 = st[W * ns];
      R[(long long)(lb + e) * Z + z] = (int8_t)row_message(w0, two ? st[(W + 1) * ns] : w0, e);
    });
  });
}

// Packed hard decisions of one codeword slot (core posteriors' signs, extension
// hard decisions from finish_extension), LSB-first words, cooperative over the CTA.
__device__ __forceinline__ void write_packed(const int16_t* __restrict__ As, const int8_t* __restrict__ Hs, int core_n,
                                             int hard_bits, uint32_t* __restrict__ dst) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int nwords = (hard_bits + 31) >> 5;
  for (int w = warp; w < nwords; w += nwarps) {
    const int j = (w << 5) + lane;
    bool bit = false;
    if (j < hard_bits) bit = j < core_n ? As[j] < 0 : Hs[j - core_n] != 0;
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
    if (lane == 0) dst[w] = m;
  }
}

__host__ __device__ inline int al16(int x) { return (x + 15) & ~15; }

template <int BG>
__host__ __device__ inline int slot_bytes(int z) {
  using T = Tab<BG>;
  return al16((T::KB + 4) * z * 2) + al16((T::MB - 4) * z);
}

// Compressed-row state: word_off(MB) words per thread.
template <int BG>
__host__ __device__ inline int state_bytes(int threads) {
  return word_off<BG>(Tab<BG>::MB) * threads * 4;
}

template <int BG, bool CLAMP>
__global__ void __launch_bounds__(768, 1) nr_i8_kernel(const __grid_constant__ Args<BG> a) {
  using T = Tab<BG>;
  extern __shared__ __align__(16) unsigned char smem[];
  const NrCommon& c = a.c;
  const int Z = c.z, N = T::NB * Z;
  const int core_n = (T::KB + 4) * Z;
  int* s_flag = reinterpret_cast<int*>(smem);
  uint32_t* st = reinterpret_cast<uint32_t*>(smem + al16(c.cpb * 4)) + threadIdx.x;
  const int ns = blockDim.x;
  unsigned char* slots = smem + al16(c.cpb * 4) + state_bytes<BG>(blockDim.x);
  const int sb = slot_bytes<BG>(Z);
  const int slot = threadIdx.x / Z;
  const int z = threadIdx.x - slot * Z;
  const bool lane_ok = slot < c.cpb;
  int16_t* A = reinterpret_cast<int16_t*>(slots + (lane_ok ? slot : 0) * sb);
  int8_t* X = reinterpret_cast<int8_t*>(slots + (lane_ok ? slot : 0) * sb + al16(core_n * 2));
  const int C = c.app_clamp;
  const RunConsts rc{Z, c.beta_q, c.app_clamp, c.k32, (unsigned)c.two};
  const long long ngroups = (c.batch + c.cpb - 1) / c.cpb;
  const bool vec_ok = (c.llr_stride % 16 == 0) && (c.llr_offset % 16 == 0) &&
                      ((reinterpret_cast<uintptr_t>(c.llr) & 15) == 0);

  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    __syncthreads();
    // ---- load: channel LLRs -> int16 core posteriors / int8 extension channel values
    for (int sl = 0; sl < c.cpb; ++sl) {
      const long long cw = grp * c.cpb + sl;
      if (cw >= c.batch) break;
      const int8_t* src = c.llr + cw * c.llr_stride;
      int16_t* As = reinterpret_cast<int16_t*>(slots + sl * sb);
      int8_t* Xs = reinterpret_cast<int8_t*>(slots + sl * sb + al16(core_n * 2));
      auto put = [&](int j, int v) {
        if (c.prologue) {
          if (j < 2 * Z)
            v = 0;
          else if (j >= c.k_prime && j < c.k)
            v = C;
        }
        if (j < core_n)
          As[j] = (int16_t)min(max(v, -C), C);
        else
          Xs[j - core_n] = (int8_t)v;
      };
      for (int j = threadIdx.x; j < c.llr_offset; j += blockDim.x) put(j, 0);
      const int n_in = N - c.llr_offset;
      if (vec_ok) {
        const int nvec = n_in >> 4;
        const uint4* s4 = reinterpret_cast<const uint4*>(src);
        for (int q = threadIdx.x; q < nvec; q += blockDim.x) {
          const uint4 w = s4[q];
          const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int i = 0; i < 16; ++i)
            put(c.llr_offset + (q << 4) + i, (int)(int8_t)(ws[i >> 2] >> ((i & 3) * 8)));
        }
        for (int j = (nvec << 4) + threadIdx.x; j < n_in; j += blockDim.x) put(c.llr_offset + j, src[j]);
      } else {
        for (int j = threadIdx.x; j < n_in; j += blockDim.x) put(c.llr_offset + j, src[j]);
      }
    }
    __syncthreads();

    const long long cw = grp * c.cpb + slot;
    const int used = iterate<BG, CLAMP>(ParamEdges<BG>{a}, rc, lane_ok && cw < c.batch, lane_ok, slot, z, A,
                                        X, st, ns, s_flag, c.iterations);

    // ---- outputs
    __syncthreads();
    if (lane_ok && cw < c.batch) {
      if (z == 0 && c.iters) c.iters[cw] = used;
      finish_extension<BG>(Z, z, X, st, ns, c.app_out ? c.app_out + cw * c.app_stride + core_n : nullptr);
      if (c.edge_r_out) write_messages<BG>(Z, z, st, ns, c.edge_r_out + cw * c.edge_r_stride);
    }
    __syncthreads();
    for (int sl = 0; sl < c.cpb; ++sl) {
      const long long cwo = grp * c.cpb + sl;
      if (cwo >= c.batch) break;
      const int16_t* As = reinterpret_cast<const int16_t*>(slots + sl * sb);
      const int8_t* Hs = reinterpret_cast<const int8_t*>(slots + sl * sb + al16(core_n * 2));
      if (c.app_out)
        for (int j = threadIdx.x; j < core_n; j += blockDim.x) c.app_out[cwo * c.app_stride + j] = As[j];
      if (c.hard_out)
        for (int j = threadIdx.x; j < N; j += blockDim.x)
          c.hard_out[cwo * c.hard_stride + j] = j < core_n ? (As[j] < 0 ? 1 : 0) : (uint8_t)Hs[j - core_n];
      if (c.hard_packed) write_packed(As, Hs, core_n, c.hard_bits, c.hard_packed + cwo * c.hard_words_stride);
    }
  }
}

template <int BG>
cudaError_t launch_bg(const NrCommon& c, const int* shifts, bool clamp, int sms, cudaStream_t stream,
                      int* ctas_out) {
  using T = Tab<BG>;
  Args<BG> a;
  a.c = c;
  a.c.k32 = 32;
  a.c.two = 2;
  for (int e = 0; e < T::E; ++e) {
    a.sh[e] = shifts[e];
    a.cz[e] = T::col(e) * c.z;
  }
  const int threads = ((c.cpb * c.z + 31) / 32) * 32;
  const int smem = al16(c.cpb * 4) + state_bytes<BG>(threads) + c.cpb * slot_bytes<BG>(c.z);
  auto fn = clamp ? nr_i8_kernel<BG, true> : nr_i8_kernel<BG, false>;
  cudaError_t e = allow_max_dynamic_smem((const void*)fn);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  if (e != cudaSuccess) return e;
  const long long groups = (c.batch + c.cpb - 1) / c.cpb;
  const long long ctas = std::min<long long>(groups, (long long)std::max(per_sm, 1) * sms);
  if (ctas_out) *ctas_out = (int)ctas;
  if (ctas <= 0) return cudaSuccess;
  fn<<<(unsigned)ctas, threads, smem, stream>>>(a);
  return cudaGetLastError();
}

// ------------------------------------------------------------ mixed batches --
//
// One persistent launch decodes codewords of any 5G NR base graph and lifting size.
// The host groups codewords of equal (BG, Z) into work items of up to `count`
// codewords (the tile size, chosen per shape by the tuner) and orders items by
// decreasing work.  Each CTA (768 threads, one per SM) takes the next item from a
// device counter, stages that shape's shifts and column bases in shared memory and
// runs the same layered iteration as the single-shape kernel.  Codewords carry
// their own filler count; the posterior clamp is always applied (filler bits are
// the common case in rate-matched code blocks).

constexpr int kMixStateBytes = 50 * 768 * 4;                     // BG1 compressed rows, 768 threads
constexpr int kMixTableInts = 320 + 320 + 64;                     // shifts, column bases, slot flags
constexpr int kMixSmem = 232448 - 1024;                           // 227 KB per CTA less static smem
constexpr int kMixSlotBytes = kMixSmem - kMixStateBytes - kMixTableInts * 4;

static_assert(word_off<0>(Tab<0>::MB) == 50, "BG1 state words");
static_assert(word_off<1>(Tab<1>::MB) <= 50, "BG2 state words");

template <int BG>
__device__ __forceinline__ void mixed_item(const MixArgs& m, const MixItem& it, int* s_sh, int* s_cz, int* s_flag,
                                           uint32_t* st, unsigned char* slots) {
  using T = Tab<BG>;
  const int Z = it.z, N = T::NB * Z, K = T::KB * Z;
  const int core_n = (T::KB + 4) * Z;
  const int ns = blockDim.x;
  const short* sh_src = m.shift_tab + (long long)(BG * kMixLiftSizes + it.zi) * kMixEdges;
  const int* cz_src = m.colz_tab + (long long)(BG * kMixLiftSizes + it.zi) * kMixEdges;
  for (int e = threadIdx.x; e < T::E; e += blockDim.x) {
    s_sh[e] = sh_src[e];
    s_cz[e] = cz_src[e];
  }
  const int sb = slot_bytes<BG>(Z);
  const int C = m.app_clamp;
  // channel LLRs of the item's codewords: variables 2Z..N (the punctured 2Z are erasures)
  for (int sl = 0; sl < it.count; ++sl) {
    const MixCodeword cw = m.cws[it.first + sl];
    const int8_t* src = m.llr + cw.llr_off;
    int16_t* As = reinterpret_cast<int16_t*>(slots + sl * sb);
    int8_t* Xs = reinterpret_cast<int8_t*>(slots + sl * sb + al16(core_n * 2));
    const int kp = cw.n_filler > K ? 0 : K - cw.n_filler;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
      int v = j < 2 * Z ? 0 : (int)src[j - 2 * Z];
      if (j >= kp && j < K && j >= 2 * Z) v = C;
      if (j < core_n)
        As[j] = (int16_t)min(max(v, -C), C);
      else
        Xs[j - core_n] = (int8_t)v;
    }
  }
  __syncthreads();
  const int slot = threadIdx.x / Z;
  const int z = threadIdx.x - slot * Z;
  const bool lane_ok = slot < it.count;
  int16_t* A = reinterpret_cast<int16_t*>(slots + (lane_ok ? slot : 0) * sb);
  int8_t* X = reinterpret_cast<int8_t*>(slots + (lane_ok ? slot : 0) * sb + al16(core_n * 2));
  const RunConsts rc{Z, m.beta_q, C, m.k32, (unsigned)m.two};
  const int used = iterate<BG, true>(SmemEdges{s_sh, s_cz}, rc, lane_ok, lane_ok, slot, z, A, X, st, ns, s_flag,
                                     m.iterations);
  __syncthreads();
  if (lane_ok) {
    if (z == 0 && m.iters) m.iters[m.cws[it.first + slot].index] = used;
    finish_extension<BG>(Z, z, X, st, ns, nullptr);
  }
  __syncthreads();
  for (int sl = 0; sl < it.count; ++sl) {
    const MixCodeword cw = m.cws[it.first + sl];
    write_packed(reinterpret_cast<const int16_t*>(slots + sl * sb),
                 reinterpret_cast<const int8_t*>(slots + sl * sb + al16(core_n * 2)), core_n, cw.hard_bits,
                 m.out + cw.out_off);
  }
}

__global__ void __launch_bounds__(768, 1) nr_mixed_i8_kernel(const __grid_constant__ MixArgs m) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item;
  int* s_sh = reinterpret_cast<int*>(smem);
  int* s_cz = s_sh + 320;
  int* s_flag = s_cz + 320;
  uint32_t* st = reinterpret_cast<uint32_t*>(smem + kMixTableInts * 4) + threadIdx.x;
  unsigned char* slots = smem + kMixTableInts * 4 + kMixStateBytes;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = (int)atomicAdd(m.queue, 1u);
    __syncthreads();
    const int item = s_item;
    if (item >= m.n_items) break;
    const MixItem it = m.items[item];
    if (it.bg == 0)
      mixed_item<0>(m, it, s_sh, s_cz, s_flag, st, slots);
    else
      mixed_item<1>(m, it, s_sh, s_cz, s_flag, st, slots);
  }
}

}  // namespace nr

int mixed_slot_capacity(int bg, int z) {
  const int sb = bg == 0 ? nr::slot_bytes<0>(z) : nr::slot_bytes<1>(z);
  return std::max(1, std::min(std::min(64, 768 / z), nr::kMixSlotBytes / sb));
}

void mixed_column_bases(int bg, int z, int* colz_out) {
  const int E = bg == 0 ? nr::Tab<0>::E : nr::Tab<1>::E;
  for (int e = 0; e < E; ++e) colz_out[e] = (bg == 0 ? nr::Tab<0>::col(e) : nr::Tab<1>::col(e)) * z;
}

cudaError_t mixed_kernel_prepare() {
  return cudaFuncSetAttribute(nr::nr_mixed_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, nr::kMixSmem);
}

cudaError_t mixed_decode_launch(const MixArgs& m, int sms, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(m.queue, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  const int ctas = std::max(1, std::min(sms, m.n_items));
  nr::nr_mixed_i8_kernel<<<ctas, 768, nr::kMixSmem, stream>>>(m);
  return cudaGetLastError();
}

bool nr_layout_matches(int bg, const int* cols, int n_edges) {
  if (bg == 0) {
    if (n_edges != nr::Tab<0>::E) return false;
    for (int e = 0; e < n_edges; ++e)
      if (cols[e] != nr::Tab<0>::col(e)) return false;
    return true;
  }
  if (bg == 1) {
    if (n_edges != nr::Tab<1>::E) return false;
    for (int e = 0; e < n_edges; ++e)
      if (cols[e] != nr::Tab<1>::col(e)) return false;
    return true;
  }
  return false;
}

// One 768-thread CTA per SM: every warp of the SM runs the same layer's code between
// barriers, which keeps the unrolled base graph's instruction working set small.
int nr_cpb(int bg, int z) {
  (void)bg;
  return std::max(1, std::min(64, 768 / z));
}

cudaError_t nr_decode_i8(int bg, const NrCommon& c, const int* shifts, int sms, cudaStream_t stream) {
  // Posteriors stay inside +-3938 (|channel| <= 128, <= 30 messages of <= 127 per
  // column) unless filler bits pin some at app_clamp or the clamp is below that.
  const bool clamp = (c.prologue && c.k_prime < c.k) || c.app_clamp < 3938;
  if (bg == 0) return nr::launch_bg<0>(c, shifts, clamp, sms, stream, nullptr);
  return nr::launch_bg<1>(c, shifts, clamp, sms, stream, nullptr);
}

}  // namespace syn
