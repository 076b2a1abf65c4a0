// Paired int8 LOMS decode for the 5G NR base graphs on sm_100a: two codewords per
// 32-bit word (nr_pair.cuh), one thread per (codeword pair, lifting index z).
//
// Per CTA, for each of its codeword pairs, shared memory holds
//   * the packed posteriors of the KB + 4 core columns (4 bytes per variable pair),
//   * the compressed check-row state of every row (meta + code words, word-major
//     per thread so that a warp's accesses are conflict-free),
//   * a byte per extension variable for the hard decisions written on output;
// the int8 channel values of the degree-1 extension columns stay in registers of
// the thread that owns their row (a layer's extension column is only touched by
// that layer, and the row of (layer, z) is the one at variable z).
//
// The graph is unrolled at compile time; the per-Z cyclic shifts are kernel
// parameters (constant bank).  With ZT = 384 the column bases are immediates.
// Each lane stops on its own zero syndrome: its outputs are written after the
// iteration that finished it while the other lane of the pair keeps decoding.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "nr_kernels.h"
#include "smem_limit.h"
#include "nr_pair.cuh"
#include "serve_device.cuh"

namespace syn {
namespace nrp {

constexpr int kPairThreads = 384;

// The kernel's dynamic shared memory.  The context below addresses it by byte offsets
// from this symbol (not by pointers), so that every access compiles to a shared-memory
// instruction also inside the non-inlined helpers.
extern __shared__ __align__(16) unsigned char pair_smem[];

template <int BG>
struct PairArgs {
  NrCommon c;               // c.cpb = codeword pairs per CTA
  int sh4[Tab<BG>::E];      // 4 * shift of each edge (reduced mod z)
  int cz4[Tab<BG>::E];      // 4 * col * z
};

// ZT = 384: lifting size, shifts, column bases and the CTA width (one pair of 384
// threads) are compile-time constants, so every shared-memory address is a register
// plus an immediate.  ZT = 0: any Z, shifts and column bases from the kernel parameters.
// ZT = -1 (mixed-shape kernel): any Z, shifts and column bases from per-item tables in
// shared memory.  APC: byte offset of the posteriors in pair_smem when ZT > 0 (the
// CTA then holds one codeword pair at a fixed place).
template <int BG, int ZT, int APC = 16>
struct DevCtx : WordRows<BG, DevCtx<BG, ZT, APC>> {
  static_assert(ZT == 0 || ZT == 384 || ZT == -1, "compile-time lifting size must be 384");
  static constexpr int NX = ext_regs<BG>();
  static constexpr int NS = ZT > 0 ? kPairThreads : 0;
  int tab;  // ZT = -1: byte offset in pair_smem of the 4 * shift table (4 * col * z follows)
  int ap;   // byte offset of this pair's posteriors in pair_smem
  int st;   // byte offset of this thread's first state word in pair_smem
  int ns;
  int z4;
  int Z4;
  const PairArgs<BG>* a;
  uint32_t x[NX];
  // Constants the row update takes from registers (a LOP3 or IMAD addend): set once
  // and made opaque to the compiler, which would otherwise fold them into immediates
  // and split the instruction in two.
  uint32_t sc;   // 0xC480, the byte-permute selector's fixed bits
  uint32_t k7f;  // 0x7F7F7F7F, the message tables' bias

  __device__ __forceinline__ uint32_t selc() const { return sc; }
  __device__ __forceinline__ uint32_t c7f() const { return k7f; }
  template <int GE>
  __device__ __forceinline__ int vb() const {
    // (z + shift) mod Z in bytes, as an unsigned min: below Z the second candidate wraps high.
    // An opaque copy of z4 per edge keeps the compiler from hoisting all the loop-invariant
    // addresses of the unrolled graph out of the iteration loop (hundreds of registers).
    int zl = z4;
    asm volatile("" : "+r"(zl));
    if constexpr (ZT > 0) {
      const unsigned r = (unsigned)(zl + Tab<BG>::z384_shift(GE) * 4);
      const unsigned rr = min(r, r - (unsigned)(ZT * 4));
      return (int)rr + Tab<BG>::col(GE) * ZT * 4;
    } else if constexpr (ZT < 0) {
      const int* t = reinterpret_cast<const int*>(pair_smem + tab);
      const unsigned r = (unsigned)(zl + t[GE]);
      const unsigned rr = min(r, r - (unsigned)Z4);
      return (int)rr + t[Tab<BG>::E + GE];
    } else {
      const unsigned r = (unsigned)(zl + a->sh4[GE]);
      const unsigned rr = min(r, r - (unsigned)Z4);
      return (int)rr + a->cz4[GE];
    }
  }
  __device__ __forceinline__ int stride() const { return NS > 0 ? NS : ns; }
  __device__ __forceinline__ int apb() const { return ZT > 0 ? APC : ap; }
  __device__ __forceinline__ uint32_t ld_ap(int b) const {
    return *reinterpret_cast<const uint32_t*>(pair_smem + apb() + b);
  }
  __device__ __forceinline__ void st_ap(int b, uint32_t v) { *reinterpret_cast<uint32_t*>(pair_smem + apb() + b) = v; }
  __device__ __forceinline__ uint32_t ld_st(int w) const {
    return *reinterpret_cast<const uint32_t*>(pair_smem + st + 4 * w * stride());
  }
  __device__ __forceinline__ void st_st(int w, uint32_t v) {
    *reinterpret_cast<uint32_t*>(pair_smem + st + 4 * w * stride()) = v;
  }
  __device__ __forceinline__ uint32_t xr(int i) const { return x[i]; }
};

__host__ __device__ inline int al16(int x) { return (x + 15) & ~15; }

// Layers 0-3 of BG1 all have 19 edges and no extension column: at Z = 384 they share
// one code body, a runtime loop over the layer whose shifts and column bases come from
// constant memory (4 * col * 384 << 16 | 4 * shift per edge).  That keeps about 1500
// instructions of unrolled code out of the iteration loop, which otherwise outgrows
// the instruction cache (measured: 1.4 % faster, bit-identical).
struct HeadTab {
  uint32_t v[76];
};
__host__ __device__ constexpr HeadTab make_head_tab() {
  HeadTab t{};
  for (int e = 0; e < 76; ++e)
    t.v[e] = ((uint32_t)(Tab<0>::col(e) * 384 * 4) << 16) | (uint32_t)(Tab<0>::z384_shift(e) * 4);
  return t;
}
static __constant__ HeadTab kHeadTab = make_head_tab();

// Row context of head layer l (0..3) over a DevCtx<0, 384, APC>: layer 0's compile-time
// structure with layer l's addresses and state words.
template <class Base>
struct HeadCtx : WordRows<0, HeadCtx<Base>> {
  __device__ HeadCtx(Base& base, int layer) : b(base), l(layer) {}
  Base& b;
  int l;
  __device__ __forceinline__ uint32_t selc() const { return b.selc(); }
  __device__ __forceinline__ uint32_t c7f() const { return b.c7f(); }
  template <int GE>
  __device__ __forceinline__ int vb() const {
    const uint32_t t = kHeadTab.v[l * 19 + GE];
    int zl = b.z4;
    asm volatile("" : "+r"(zl));
    const unsigned r = (unsigned)zl + (t & 0xFFFFu);
    const unsigned rr = min(r, r - 384u * 4u);
    return (int)rr + (int)(t >> 16);
  }
  __device__ __forceinline__ uint32_t ld_ap(int o) const { return b.ld_ap(o); }
  __device__ __forceinline__ void st_ap(int o, uint32_t v) { b.st_ap(o, v); }
  __device__ __forceinline__ uint32_t ld_st(int w) const { return b.ld_st(4 * l + w); }
  __device__ __forceinline__ void st_st(int w, uint32_t v) { b.st_st(4 * l + w, v); }
  __device__ __forceinline__ uint32_t xr(int i) const { return b.xr(i); }
};
static_assert(deg_of<0>(0) == 19 && deg_of<0>(1) == 19 && deg_of<0>(2) == 19 && deg_of<0>(3) == 19 &&
                  state_off<0>(1) == 4 && state_off<0>(3) == 12,
              "BG1 head layers");

template <int BG>
__host__ __device__ inline int pair_smem_bytes(int pairs, int z, int threads) {
  using T = Tab<BG>;
  return al16(8 * pairs) + pairs * (T::KB + 4) * z * 4 + state_words<BG>() * threads * 4 +
         al16(pairs * (T::MB - 4) * z);
}

// Signed value of one lane of a biased word: bias kPB (computed posteriors) or kAB (stored).
__device__ __forceinline__ int lane_of(uint32_t w, int lane, uint32_t bias = kPB) {
  return (int)((w >> (16 * lane)) & 0xFFFFu) - (int)bias;
}

// Cold paths as separate functions (own register allocation; the caller passes a copy
// of its context so that the hot loop's registers stay where they are).

// Parity of every check row outside the quick-stage layers (bit 0 lane A odd, bit 1 lane B).
template <int BG, class Ctx>
__device__ __noinline__ uint32_t full_parity(const Ctx* cx) {
  uint32_t odd = 0u;
  static_for<0, Tab<BG>::MB>([&](auto li) {
    constexpr int L = decltype(li)::value;
    if constexpr (!is_quick<BG>(L)) odd |= pair_parity<BG, L>(*cx);
  });
  return odd;
}

// This thread's share of lane X's results: its extension posteriors / hard decisions
// (also into the shared-memory byte array eh for the packed output, unless eh_off < 0)
// and the messages of its check rows in the reference's edge_r layout.
template <int BG, class Ctx>
__device__ __noinline__ void write_rows(const Ctx* cx, const NrCommon* c, int X, long long cw, int Z, int z,
                                        int eh_off) {
  using T = Tab<BG>;
  static_for<4, T::MB>([&](auto li) {
    constexpr int L = decltype(li)::value;
    const int v = lane_of(pair_ext_app<BG, L>(*cx), X);
    const int j = (T::KB + L) * Z + z;
    if (eh_off >= 0) pair_smem[eh_off + (L - 4) * Z + z] = v < 0 ? 1 : 0;
    if (c->app_out) c->app_out[cw * c->app_stride + j] = (int16_t)v;
    if (c->hard_out) c->hard_out[cw * c->hard_stride + j] = v < 0 ? 1 : 0;
  });
  if (c->edge_r_out) {
    int8_t* er = c->edge_r_out + cw * c->edge_r_stride;
    static_for<0, T::MB>([&](auto li) {
      constexpr int L = decltype(li)::value;
      static_for<0, deg_of<BG>(L)>([&](auto ei) {
        constexpr int e = decltype(ei)::value;
        const uint32_t m = pair_message<BG, L, e>(*cx);
        er[(long long)(T::loff(L) + e) * Z + z] = (int8_t)((int)((m >> (16 * X)) & 0xFFu) - 127);
      });
    });
  }
}

// A codeword's stored channel LLRs (bytes [0, bytes) of its row) into L2, one 128-byte
// line per thread and step: issued for the CTA's next group while this one decodes, so
// that the next load phase reads L2 instead of waiting on HBM.  Every address lies
// inside the row.
__device__ __noinline__ void prefetch_row_l2(const int8_t* row, long long bytes, int z, int Z) {
  for (long long i = 128LL * z; i < bytes; i += 128LL * Z)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(row + i)));
}

template <int BG, int ZT, bool FILL>
__global__ void __launch_bounds__(kPairThreads, 1) nr_pair_kernel(const __grid_constant__ PairArgs<BG> a) {
  using T = Tab<BG>;
  constexpr int NW = state_words<BG>(), CORE = T::KB + 4, NEXT = T::MB - 4;
  unsigned char* smem = pair_smem;
  const NrCommon& c = a.c;
  const int Z = ZT > 0 ? ZT : c.z;
  const int P = ZT > 0 ? 1 : c.cpb;
  const int ns = ZT > 0 ? kPairThreads : (int)blockDim.x;
  int* s_fail = reinterpret_cast<int*>(smem);
  int* s_done = s_fail + P;
  unsigned char* ap_base = smem + al16(8 * P);
  const int ap_pair = CORE * Z * 4;
  uint32_t* st_base = reinterpret_cast<uint32_t*>(ap_base + P * ap_pair);
  uint8_t* eh_base = reinterpret_cast<uint8_t*>(st_base + NW * ns);
  const int tid = threadIdx.x;
  const int p = tid / Z, z = tid - p * Z;
  const bool lane_ok = p < P;
  const int pq = lane_ok ? p : 0;
  DevCtx<BG, ZT> cx;
  cx.ap = (int)(ap_base - smem) + pq * ap_pair;
  cx.st = (int)(reinterpret_cast<unsigned char*>(st_base) - smem) + 4 * tid;
  cx.ns = ns;
  cx.z4 = z * 4;
  cx.Z4 = Z * 4;
  cx.sc = 0xC480u;
  cx.k7f = 0x7F7F7F7Fu;
  asm volatile("" : "+r"(cx.sc), "+r"(cx.k7f));
  cx.a = &a;
  uint8_t* eh = eh_base + pq * NEXT * Z;
  const uint32_t bq2 = pair_beta(c.beta_q);
  const int core_n = CORE * Z, K = T::KB * Z;
  const long long npairs = (c.batch + 1) / 2;
  const long long ngroups = (npairs + P - 1) / P;
  const int lane = tid & 31, warp = tid >> 5, nwarps = ns >> 5;

  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const long long g = grp * P + p;
    const bool va = lane_ok && 2 * g < c.batch, vbv = lane_ok && 2 * g + 1 < c.batch;
    __syncthreads();
    // ---- load: this thread's variables (col, z) of both codewords
    if (lane_ok) {
      const int8_t* sa = va ? c.llr + 2 * g * c.llr_stride - c.llr_offset : nullptr;
      const int8_t* sb = vbv ? c.llr + (2 * g + 1) * c.llr_stride - c.llr_offset : nullptr;
      auto fetch = [&](const int8_t* s, int j) -> int { return (s && j >= c.llr_offset) ? (int)s[j] : 0; };
      uint32_t* apw = reinterpret_cast<uint32_t*>(smem + cx.ap);
      for (int col = 0; col < CORE; ++col) {
        const int j = col * Z + z;
        uint32_t l0 = kAB + (uint32_t)fetch(sa, j), l1 = kAB + (uint32_t)fetch(sb, j);
        if (c.prologue) {
          if (j < 2 * Z) {
            l0 = l1 = kAB;
          } else if (FILL && j >= c.k_prime && j < K) {
            l0 = l1 = kAB + kCapV;
          }
        }
        apw[j] = (l0 & 0xFFFFu) | (l1 << 16);
      }
      static_for<0, DevCtx<BG, ZT>::NX>([&](auto ri) {
        constexpr int r = decltype(ri)::value;
        uint32_t w = 0u;
        static_for<0, 2>([&](auto hi) {
          constexpr int h = decltype(hi)::value;
          constexpr int xi = 2 * r + h;
          if constexpr (xi < NEXT) {
            const int j = (CORE + xi) * Z + z;
            const uint32_t b0 = (uint32_t)(fetch(sa, j) + 128) & 0xFFu, b1 = (uint32_t)(fetch(sb, j) + 128) & 0xFFu;
            w |= (b0 | (b1 << 8)) << (16 * h);
          }
        });
        cx.x[r] = w;
      });
#pragma unroll 1
      for (int w = 0; w < NW; ++w) st_base[w * ns + tid] = 0u;
      const long long gn = (grp + gridDim.x) * P + p;  // this slot's next codeword pair
      const long long row_bytes = (long long)T::NB * Z - c.llr_offset;
      if (2 * gn < c.batch) prefetch_row_l2(c.llr + 2 * gn * c.llr_stride, row_bytes, z, Z);
      if (2 * gn + 1 < c.batch) prefetch_row_l2(c.llr + (2 * gn + 1) * c.llr_stride, row_bytes, z, Z);
    }
    __syncthreads();

    // ---- layered iterations with per-lane early stop.  A lane's results are written
    // at the top of the loop after the iteration that finished it (zero syndrome or
    // the iteration limit); the other lane of its pair keeps decoding.
    uint32_t act = (va ? 1u : 0u) | (vbv ? 2u : 0u);
    uint32_t done = c.iterations <= 0 ? act : 0u;
    int it = 0;
    for (;;) {
#pragma unroll 1
      for (int X = 0; X < 2; ++X) {
        const bool mine = ((done >> X) & 1u) != 0u;
        if (!__syncthreads_or(mine)) continue;
        if (lane_ok && z == 0) s_done[p] = mine ? 1 : 0;
        if (mine) {
          const long long cw = 2 * g + X;
          if (z == 0 && c.iters) c.iters[cw] = it;
          const DevCtx<BG, ZT> copy = cx;
          write_rows<BG>(&copy, &c, X, cw, Z, z, (int)(eh - smem));
        }
        __syncthreads();
        for (int q = 0; q < P; ++q) {
          if (!s_done[q]) continue;
          const long long cwo = 2 * (grp * P + q) + X;
          const uint32_t* apq = reinterpret_cast<const uint32_t*>(ap_base + q * ap_pair);
          const uint8_t* ehq = eh_base + q * NEXT * Z;
          if (c.app_out || c.hard_out) {
            for (int j = tid; j < core_n; j += ns) {
              int v = lane_of(apq[j], X, kAB);
              if (FILL && j >= c.k_prime && j < K) v += c.app_clamp - kCapV;
              if (c.app_out) c.app_out[cwo * c.app_stride + j] = (int16_t)v;
              if (c.hard_out) c.hard_out[cwo * c.hard_stride + j] = v < 0 ? 1 : 0;
            }
          }
          if (c.hard_packed) {
            uint32_t* dst = c.hard_packed + cwo * c.hard_words_stride;
            const int nwords = (c.hard_bits + 31) >> 5;
            for (int w = warp; w < nwords; w += nwarps) {
              const int j = (w << 5) + lane;
              bool bit = false;
              if (j < c.hard_bits) bit = j < core_n ? lane_of(apq[j], X, kAB) < 0 : ehq[j - core_n] != 0;
              const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
              if (lane == 0) dst[w] = m;
            }
          }
        }
        __syncthreads();
      }
      act &= ~done;
      if (!__syncthreads_or(act != 0u)) break;
      ++it;
      constexpr bool head_loop = BG == 0 && ZT == 384;
      if constexpr (head_loop) {
#pragma unroll 1
        for (int l = 0; l < 4; ++l) {
          if (lane_ok) {
            HeadCtx<DevCtx<BG, ZT>> h(cx, l);
            pair_row<BG, 0, FILL>(h, bq2);
          }
          __syncthreads();
        }
      }
      static_for<head_loop ? 4 : 0, T::MB>([&](auto li) {
        constexpr int L = decltype(li)::value;
        if (lane_ok) pair_row<BG, L, FILL>(cx, bq2);
        if constexpr (nr::barrier_after<BG>(L)) __syncthreads();
      });
      // syndrome: the smallest layer first, the others only for lanes that pass it
      if (lane_ok && z == 0) s_fail[p] = 0;
      __syncthreads();
      if (act) {
        const uint32_t odd = quick_parity<BG>(cx) & act;
        if (odd) atomicOr(&s_fail[p], (int)odd);
      }
      __syncthreads();
      const uint32_t pass = act & ~(uint32_t)(lane_ok ? s_fail[p] : 0);
      if (pass) {
        const DevCtx<BG, ZT> copy = cx;
        const uint32_t odd = full_parity<BG>(&copy) & pass;
        if (odd) atomicOr(&s_fail[p], (int)odd);
      }
      __syncthreads();
      done = it >= c.iterations ? act : act & ~(uint32_t)(lane_ok ? s_fail[p] : 0);
    }
  }
}

template <int BG, int ZT, bool FILL>
cudaError_t launch(const NrCommon& c0, const int* shifts, int sms, cudaStream_t stream) {
  using T = Tab<BG>;
  PairArgs<BG> a;
  a.c = c0;
  for (int e = 0; e < T::E; ++e) {
    a.sh4[e] = shifts[e] * 4;
    a.cz4[e] = T::col(e) * c0.z * 4;
  }
  const long long npairs = (c0.batch + 1) / 2;
  a.c.cpb = (int)std::max<long long>(1, std::min<long long>(kPairThreads / c0.z, npairs));
  const int threads = ((a.c.cpb * c0.z + 31) / 32) * 32;
  const int smem = pair_smem_bytes<BG>(a.c.cpb, c0.z, threads);
  auto fn = nr_pair_kernel<BG, ZT, FILL>;
  cudaError_t e = allow_max_dynamic_smem((const void*)fn);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  if (e != cudaSuccess) return e;
  const long long groups = (npairs + a.c.cpb - 1) / a.c.cpb;
  const long long ctas = std::min<long long>(groups, (long long)std::max(per_sm, 1) * sms);
  if (ctas <= 0) return cudaSuccess;
  fn<<<(unsigned)ctas, threads, smem, stream>>>(a);
  return cudaGetLastError();
}

template <int BG>
cudaError_t launch_bg(const NrCommon& c, const int* shifts, bool fill, int sms, cudaStream_t stream) {
  if (c.z == 384)
    return fill ? launch<BG, 384, true>(c, shifts, sms, stream) : launch<BG, 384, false>(c, shifts, sms, stream);
  return fill ? launch<BG, 0, true>(c, shifts, sms, stream) : launch<BG, 0, false>(c, shifts, sms, stream);
}

// ------------------------------------------------------- TMEM-backed variant --
//
// Z = 384, one codeword pair per CTA and two CTAs per SM.  The kernel above holds a
// pair's whole check-row state (158 KB at BG1) and posteriors in shared memory, one
// pair per SM: three warps per scheduler, all reaching the layer barriers together,
// so the row updates between barriers are latency-bound.  Here most of each thread's
// check-row state lives in tensor memory (TMEM, 256 KB per SM, used purely as
// per-thread storage: tcgen05.ld / tcgen05.st of the thread's own lane), which lets
// two CTAs of independent codeword pairs share an SM; their barriers do not line up,
// so one CTA's row updates fill the other's waits.
//
// Per CTA: 256 TMEM columns (half of the SM's 512).  Lane quarter q of TMEM (lanes
// 32q .. 32q + 31) is reachable from warps q, q + 4 and q + 8 of the CTA, so each
// thread owns an 85-column slot: columns 85 * (warp / 4) .. + 84 of lane
// 32 * (warp % 4) + lane (at most column 254).  The rows of the compressed state go
// to the slot in layer order, each padded to 2 or 4 words so that one tcgen05.ld.x2 /
// .x4 moves it; the quick-stage syndrome layers and the rows that do not fit stay in
// shared memory, as do the extension columns' channel values (a word per two layers)
// and the posteriors.  While a row is updated, the next TMEM row is already being
// loaded (row_next); the wait for it comes at that row's start.  Every TMEM access is
// warp-uniform: one CTA holds one pair, so every branch around an access (iteration
// control, done lanes, syndrome stages) is the same for all threads of the CTA.
namespace tm {

constexpr int kCols = 256;  // TMEM columns per CTA
constexpr int kSlot = 85;   // columns per thread: three warps share each lane quarter

__host__ __device__ constexpr int pow2ceil(int x) {
  int p = 1;
  while (p < x) p *= 2;
  return p;
}
template <int BG>
__host__ __device__ constexpr int row_len(int L) {
  return 1 + ncw(deg_of<BG>(L));
}
template <int BG>
__host__ __device__ constexpr int row_pad(int L) {
  return pow2ceil(row_len<BG>(L));
}
// Storage plan of a base graph's rows: in TMEM greedily in layer order, skipping the
// quick-stage layers (read every iteration by the syndrome check); the TMEM column or
// shared state word of each row.  Computed once per base graph.
struct Plan {
  bool in[48];
  int col[49];
  int smw[49];
};
template <int BG>
__host__ __device__ constexpr Plan make_plan() {
  Plan p{};
  constexpr int MB = Tab<BG>::MB;
  int deg[48] = {};
  for (int l = 0; l < MB; ++l) deg[l] = deg_of<BG>(l);
  int used = 0, w = 0;
  for (int l = 0; l < MB; ++l) {
    int rank = 0;  // nr::is_quick
    for (int m = 0; m < MB; ++m)
      if (deg[m] < deg[l] || (deg[m] == deg[l] && m < l)) ++rank;
    const int len = 1 + ncw(deg[l]), pad = pow2ceil(len);
    p.col[l] = used;
    p.smw[l] = w;
    p.in[l] = rank >= nr::kQuick && used + pad <= kSlot;
    if (p.in[l])
      used += pad;
    else
      w += len;
  }
  p.col[MB] = used;
  p.smw[MB] = w;
  return p;
}
template <int BG>
struct PlanOf {
  static constexpr Plan v = make_plan<BG>();
};
template <int BG>
__host__ __device__ constexpr bool in_tm(int L) {
  return PlanOf<BG>::v.in[L];
}
template <int BG>
__host__ __device__ constexpr int tm_col(int L) {
  return PlanOf<BG>::v.col[L];
}
template <int BG>
__host__ __device__ constexpr int sm_word(int L) {
  return PlanOf<BG>::v.smw[L];
}
template <int BG>
__host__ __device__ constexpr int sm_words() {
  return sm_word<BG>(Tab<BG>::MB);
}
template <int BG>
__host__ __device__ constexpr int tm_words() {
  return tm_col<BG>(Tab<BG>::MB);
}
static_assert(tm_words<0>() <= kSlot && tm_words<1>() <= kSlot, "TMEM slot overflow");
static_assert(in_tm<0>(0) && in_tm<0>(1) && in_tm<0>(2) && in_tm<0>(3) && tm_col<0>(1) == 4 && tm_col<0>(3) == 12,
              "BG1 head layers take TMEM columns 0-15");

// Shared memory: [0, 16) s_fail, s_done, TMEM base; posteriors at kAp; then the shared
// state words [sm_words][384]; then the extension channel words [ext_regs][384].
constexpr int kAp = 16;
template <int BG>
__host__ __device__ constexpr int smem_bytes() {
  return kAp + (Tab<BG>::KB + 4) * 384 * 4 + (sm_words<BG>() + ext_regs<BG>()) * 384 * 4;
}
// Dynamic shared memory a TMEM-kernel CTA is launched with: at least a third of the
// SM's 228 KB, so that no SM ever holds three CTAs of the TMEM kernels (each takes 256
// of the SM's 512 TMEM columns; a third would wait in tcgen05.alloc), whatever the
// register count.
constexpr int kTwoPerSm = 233472 / 3 + 16;
template <int BG>
__host__ __device__ constexpr int launch_smem() {
  return smem_bytes<BG>() > kTwoPerSm ? smem_bytes<BG>() : kTwoPerSm;
}

// ---- tcgen05 storage primitives (sm_100a) ----
__device__ __forceinline__ void ld2(uint32_t t, uint32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(v[0]), "=r"(v[1]) : "r"(t));
}
__device__ __forceinline__ void ld4(uint32_t t, uint32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(t));
}
// Waits for this thread's TMEM loads; v passes through, so no use of the loaded
// registers can move above the wait.
__device__ __forceinline__ void wait_ld(uint32_t (&v)[4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3])::"memory");
}
__device__ __forceinline__ uint32_t ld1_now(uint32_t t) {
  uint32_t v;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(v) : "r"(t));
  asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(v)::"memory");
  return v;
}
__device__ __forceinline__ void st2(uint32_t t, uint32_t a, uint32_t b) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(t), "r"(a), "r"(b) : "memory");
}
__device__ __forceinline__ void st4(uint32_t t, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(t), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
}
__device__ __forceinline__ void st1(uint32_t t, uint32_t a) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(t), "r"(a) : "memory");
}
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Row context of the TMEM variant.  pf holds the next TMEM row while its load is in
// flight; the cold paths (syndrome stages, outputs) run only while no load is in
// flight, which is what lets them work on a copy of the context.  State and extension
// words are laid out for 384 threads.  ZT = 384: one codeword pair at Z = 384, its
// posteriors at byte APC of pair_smem, compile-time shifts.  ZT = -1 (mixed-shape
// kernel): any Z, the thread's pair's posteriors at byte `ap`, shifts and column bases
// from the item's table at byte `tab` (4 * shift [E], then 4 * col * Z [E]); a thread
// past the item's pairs runs the row updates on pair 0's posteriors without storing
// them (`live` false), so that every TMEM access stays warp-wide.
template <int BG, int ZT = 384, int APC = kAp>
struct TmCtx {
  static_assert(ZT == 384 || ZT == -1, "TMEM context: Z = 384 or run-time Z");
  uint32_t tmb;  // TMEM address of this thread's slot: lane (32 * (warp % 4)) << 16 | column
  int st;        // byte offset in pair_smem of this thread's first shared state word
  int xo;        // byte offset in pair_smem of this thread's first extension channel word
  int z4;
  uint32_t sc, k7f;
  int ap, tab, Z4;  // ZT = -1 only
  bool live;        // ZT = -1 only
  uint32_t pf[4];

  __device__ __forceinline__ uint32_t selc() const { return sc; }
  __device__ __forceinline__ uint32_t c7f() const { return k7f; }
  template <int GE>
  __device__ __forceinline__ int vb() const {
    // (z + shift) mod Z in bytes, the wrap as an unsigned min (below Z the second
    // candidate wraps high; add and min fuse); at Z = 384 the column base folds into
    // the shared-memory instruction's immediate
    int zl = z4;
    asm volatile("" : "+r"(zl));
    if constexpr (ZT > 0) {
      const unsigned r = (unsigned)(zl + Tab<BG>::z384_shift(GE) * 4);
      const unsigned rr = min(r, r - 384u * 4u);
      return (int)rr + Tab<BG>::col(GE) * 384 * 4;
    } else {
      const int* t = reinterpret_cast<const int*>(pair_smem + tab);
      const unsigned r = (unsigned)(zl + t[GE]);
      const unsigned rr = min(r, r - (unsigned)Z4);
      return (int)rr + t[Tab<BG>::E + GE];
    }
  }
  __device__ __forceinline__ int apb() const { return ZT > 0 ? APC : ap; }
  __device__ __forceinline__ uint32_t ld_ap(int b) const {
    return *reinterpret_cast<const uint32_t*>(pair_smem + apb() + b);
  }
  __device__ __forceinline__ void st_ap(int b, uint32_t v) {
    if (ZT > 0 || live) *reinterpret_cast<uint32_t*>(pair_smem + apb() + b) = v;
  }
  __device__ __forceinline__ uint32_t xr(int i) const {
    return *reinterpret_cast<const uint32_t*>(pair_smem + xo + 4 * 384 * i);
  }
  __device__ __forceinline__ uint32_t sm_ld(int w) const {
    return *reinterpret_cast<const uint32_t*>(pair_smem + st + 4 * 384 * w);
  }
  __device__ __forceinline__ void sm_st(int w, uint32_t v) {
    *reinterpret_cast<uint32_t*>(pair_smem + st + 4 * 384 * w) = v;
  }
  // Issues the load of the TMEM row at column col (row_pad words) into pf.
  template <int PAD>
  __device__ __forceinline__ void fetch(int col) {
    if constexpr (PAD == 4)
      ld4(tmb + (uint32_t)col, pf);
    else
      ld2(tmb + (uint32_t)col, pf);
  }
  template <int N>
  __device__ __forceinline__ void take(uint32_t (&w)[N]) {
    wait_ld(pf);
    static_for<0, N>([&](auto ii) { w[decltype(ii)::value] = pf[decltype(ii)::value]; });
  }
  template <int N>
  __device__ __forceinline__ void put(int col, const uint32_t (&w)[N]) {
    static_assert(N >= 2 && N <= 4, "row length");
    if constexpr (N == 2)
      st2(tmb + (uint32_t)col, w[0], w[1]);
    else if constexpr (N == 3)
      st4(tmb + (uint32_t)col, w[0], w[1], w[2], w[2]);  // the padding word takes a copy
    else
      st4(tmb + (uint32_t)col, w[0], w[1], w[2], w[3]);
  }

  template <int L, int N>
  __device__ __forceinline__ void row_load(uint32_t (&w)[N]) {
    if constexpr (in_tm<BG>(L)) {
      take(w);
    } else {
      static_for<0, N>([&](auto ii) { w[decltype(ii)::value] = sm_ld(sm_word<BG>(L) + decltype(ii)::value); });
    }
  }
  template <int L>
  __device__ __forceinline__ void row_next() {
    if constexpr (L + 1 < Tab<BG>::MB) {
      if constexpr (in_tm<BG>(L + 1)) fetch<row_pad<BG>(L + 1)>(tm_col<BG>(L + 1));
    }
  }
  template <int L, int N>
  __device__ __forceinline__ void row_store(const uint32_t (&w)[N]) {
    if constexpr (in_tm<BG>(L)) {
      put(tm_col<BG>(L), w);
    } else {
      static_for<0, N>([&](auto ii) { sm_st(sm_word<BG>(L) + decltype(ii)::value, w[decltype(ii)::value]); });
    }
  }
  template <int L>
  __device__ __forceinline__ uint32_t row_word(int i) const {
    if constexpr (in_tm<BG>(L))
      return ld1_now(tmb + (uint32_t)(tm_col<BG>(L) + i));
    else
      return sm_ld(sm_word<BG>(L) + i);
  }
  // Starts the load of the first row of an iteration.
  __device__ __forceinline__ void first_row() {
    if constexpr (in_tm<BG>(0)) fetch<row_pad<BG>(0)>(tm_col<BG>(0));
  }
};

// BG1 head layer l (0..3) over a TmCtx<0, 384, APC>: layer 0's compile-time structure
// with layer l's addresses and TMEM row (columns 4l .. 4l + 3).
template <int APC>
struct TmHeadCtxT {
  TmCtx<0, 384, APC>& b;
  int l;
  __device__ TmHeadCtxT(TmCtx<0, 384, APC>& base, int layer) : b(base), l(layer) {}
  __device__ __forceinline__ uint32_t selc() const { return b.selc(); }
  __device__ __forceinline__ uint32_t c7f() const { return b.c7f(); }
  template <int GE>
  __device__ __forceinline__ int vb() const {
    const uint32_t t = kHeadTab.v[l * 19 + GE];
    int zl = b.z4;
    asm volatile("" : "+r"(zl));
    const unsigned r = (unsigned)zl + (t & 0xFFFFu);
    const unsigned rr = min(r, r - 384u * 4u);
    return (int)rr + (int)(t >> 16);
  }
  __device__ __forceinline__ uint32_t ld_ap(int o) const { return b.ld_ap(o); }
  __device__ __forceinline__ void st_ap(int o, uint32_t v) { b.st_ap(o, v); }
  __device__ __forceinline__ uint32_t xr(int i) const { return b.xr(i); }
  template <int L, int N>
  __device__ __forceinline__ void row_load(uint32_t (&w)[N]) {
    static_assert(L == 0 && N == 4, "head rows");
    b.take(w);
  }
  template <int L>
  __device__ __forceinline__ void row_next() {
    if (l < 3)
      b.fetch<4>(4 * (l + 1));
    else if constexpr (in_tm<0>(4))
      b.fetch<row_pad<0>(4)>(tm_col<0>(4));
  }
  template <int L, int N>
  __device__ __forceinline__ void row_store(const uint32_t (&w)[N]) {
    b.put(4 * l, w);
  }
};

template <int BG, bool FILL>
__global__ void __launch_bounds__(kPairThreads, 2) nr_pair_tm_kernel(const __grid_constant__ PairArgs<BG> a) {
  using T = Tab<BG>;
  constexpr int Z = 384, CORE = T::KB + 4, NEXT = T::MB - 4, NX = ext_regs<BG>(), NSW = sm_words<BG>();
  unsigned char* smem = pair_smem;
  const NrCommon& c = a.c;
  int* s_fail = reinterpret_cast<int*>(smem);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + 8);
  const int tid = threadIdx.x, z = tid, lane = tid & 31, warp = tid >> 5;
  const int sw_off = kAp + CORE * Z * 4, x_off = sw_off + NSW * Z * 4;

  // TMEM: warp 0 allocates the CTA's columns and hands the address over shared memory.
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(s_tmem)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  TmCtx<BG> cx;
  cx.tmb = *s_tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(kSlot * (warp >> 2));
  cx.st = sw_off + 4 * tid;
  cx.xo = x_off + 4 * tid;
  cx.z4 = z * 4;
  cx.sc = 0xC480u;
  cx.k7f = 0x7F7F7F7Fu;
  asm volatile("" : "+r"(cx.sc), "+r"(cx.k7f));
  const uint32_t bq2 = pair_beta(c.beta_q);
  const int core_n = CORE * Z, K = T::KB * Z;
  const long long npairs = (c.batch + 1) / 2;
  // 128-bit loads when every codeword row starts on a 16-byte boundary
  const bool vec = ((reinterpret_cast<uintptr_t>(c.llr) | (uintptr_t)c.llr_stride | (uintptr_t)c.llr_offset) & 15u) == 0;

  for (long long g = blockIdx.x; g < npairs; g += gridDim.x) {
    const bool va = 2 * g < c.batch, vbv = 2 * g + 1 < c.batch;
    __syncthreads();
    // ---- load: both codewords' channel LLRs into the posteriors and extension words
    {
      const int8_t* sa = va ? c.llr + 2 * g * c.llr_stride - c.llr_offset : nullptr;
      const int8_t* sb = vbv ? c.llr + (2 * g + 1) * c.llr_stride - c.llr_offset : nullptr;
      auto fetch = [&](const int8_t* src, int j) -> int { return (src && j >= c.llr_offset) ? (int)src[j] : 0; };
      uint32_t* apw = reinterpret_cast<uint32_t*>(smem + kAp);
      if (vec) {
        // 128-bit loads: chunk q holds variables 16q .. 16q + 15 of one column (Z and
        // llr_offset are multiples of 16, so a chunk never straddles a column or the
        // transmitted boundary), turned into 16 posterior words of the pair and
        // stored as four 128-bit words at the same place in the variable-indexed array
        for (int q = tid; q < core_n / 16; q += Z) {
          const int j0 = 16 * q;
          uint4 ra = make_uint4(0u, 0u, 0u, 0u), rb = ra;
          if (j0 >= c.llr_offset) {
            if (sa) ra = *reinterpret_cast<const uint4*>(sa + j0);
            if (sb) rb = *reinterpret_cast<const uint4*>(sb + j0);
          }
          const uint32_t av[4] = {ra.x ^ 0x80808080u, ra.y ^ 0x80808080u, ra.z ^ 0x80808080u, ra.w ^ 0x80808080u};
          const uint32_t bv[4] = {rb.x ^ 0x80808080u, rb.y ^ 0x80808080u, rb.z ^ 0x80808080u, rb.w ^ 0x80808080u};
          uint32_t wv[16];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            // offset-binary bytes a + 128, b + 128 interleaved, then spread to 16-bit
            // lanes: (a + 128) + (PB + 127 - 128) = PB + 127 + a, no carry between lanes
            const uint32_t lo = prmt(av[k], bv[k], 0x5140u), hi = prmt(av[k], bv[k], 0x7362u);
            wv[4 * k] = prmt(lo, 0u, 0x4140u) + (kAB2 - 0x00800080u);
            wv[4 * k + 1] = prmt(lo, 0u, 0x4342u) + (kAB2 - 0x00800080u);
            wv[4 * k + 2] = prmt(hi, 0u, 0x4140u) + (kAB2 - 0x00800080u);
            wv[4 * k + 3] = prmt(hi, 0u, 0x4342u) + (kAB2 - 0x00800080u);
          }
          if (c.prologue) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int j = j0 + i;
              if (j < 2 * Z)
                wv[i] = kAB2;
              else if (FILL && j >= c.k_prime && j < K)
                wv[i] = kCapS2;
            }
          }
          uint4* dst = reinterpret_cast<uint4*>(apw + j0);
#pragma unroll
          for (int k = 0; k < 4; ++k) dst[k] = make_uint4(wv[4 * k], wv[4 * k + 1], wv[4 * k + 2], wv[4 * k + 3]);
        }
      } else {
        for (int col = 0; col < CORE; ++col) {
          const int j = col * Z + z;
          uint32_t l0 = kAB + (uint32_t)fetch(sa, j), l1 = kAB + (uint32_t)fetch(sb, j);
          if (c.prologue) {
            if (j < 2 * Z) {
              l0 = l1 = kAB;
            } else if (FILL && j >= c.k_prime && j < K) {
              l0 = l1 = kAB + kCapV;
            }
          }
          apw[j] = (l0 & 0xFFFFu) | (l1 << 16);
        }
      }
      uint32_t* xw = reinterpret_cast<uint32_t*>(smem + x_off);
      // BG1's shared state area holds both codewords' extension bytes (2 x 42 x 384 B):
      // with 128-bit rows they are staged there in memory order, then each thread
      // gathers its own (layer, z) bytes; the area is cleared afterwards
      constexpr bool kStage = NSW * 4 >= 2 * NEXT;
      if (kStage && vec) {
        unsigned char* stage = smem + sw_off;
        constexpr int QC = NEXT * 384 / 16;  // chunks per codeword
        for (int q = tid; q < 2 * QC; q += Z) {
          const int8_t* src = q < QC ? sa : sb;
          const int qq = q < QC ? q : q - QC;
          uint4 v = make_uint4(0u, 0u, 0u, 0u);  // absent codeword or erased variables: LLR 0
          if (src && core_n + 16 * qq >= c.llr_offset) v = *reinterpret_cast<const uint4*>(src + core_n + 16 * qq);
          *reinterpret_cast<uint4*>(stage + 16 * q) = v;
        }
        __syncthreads();
#pragma unroll 1
        for (int r = 0; r < NX; ++r) {
          uint32_t w = 0u;
          for (int h = 0; h < 2; ++h) {
            const int xi = 2 * r + h;
            if (xi < NEXT) {
              const uint32_t b0 = (uint32_t)(stage[xi * 384 + z] ^ 0x80u), b1 = (uint32_t)(stage[(NEXT + xi) * 384 + z] ^ 0x80u);
              w |= (b0 | (b1 << 8)) << (16 * h);
            }
          }
          xw[r * Z + tid] = w;
        }
        __syncthreads();
      } else {
#pragma unroll 1
        for (int r = 0; r < NX; ++r) {
          uint32_t w = 0u;
          for (int h = 0; h < 2; ++h) {
            const int xi = 2 * r + h;
            if (xi < NEXT) {
              const int j = (CORE + xi) * Z + z;
              const uint32_t b0 = (uint32_t)(fetch(sa, j) + 128) & 0xFFu, b1 = (uint32_t)(fetch(sb, j) + 128) & 0xFFu;
              w |= (b0 | (b1 << 8)) << (16 * h);
            }
          }
          xw[r * Z + tid] = w;
        }
      }
      uint32_t* sw = reinterpret_cast<uint32_t*>(smem + sw_off);
#pragma unroll 1
      for (int w = 0; w < NSW; ++w) sw[w * Z + tid] = 0u;
#pragma unroll 1
      for (int col = 0; col + 4 <= kSlot; col += 4) st4(cx.tmb + (uint32_t)col, 0u, 0u, 0u, 0u);
      st1(cx.tmb + (uint32_t)(kSlot - 1), 0u);
      wait_st();
      const long long gn = g + gridDim.x;  // this CTA's next codeword pair
      const long long row_bytes = (long long)T::NB * Z - c.llr_offset;
      if (2 * gn < c.batch) prefetch_row_l2(c.llr + 2 * gn * c.llr_stride, row_bytes, z, Z);
      if (2 * gn + 1 < c.batch) prefetch_row_l2(c.llr + (2 * gn + 1) * c.llr_stride, row_bytes, z, Z);
    }
    __syncthreads();

    // ---- layered iterations with per-lane early stop (as the kernel above)
    uint32_t act = (va ? 1u : 0u) | (vbv ? 2u : 0u);
    uint32_t done = c.iterations <= 0 ? act : 0u;
    int it = 0;
    for (;;) {
#pragma unroll 1
      for (int X = 0; X < 2; ++X) {
        if (!((done >> X) & 1u)) continue;  // the same for the whole CTA
        const long long cw = 2 * g + X;
        if (z == 0 && c.iters) c.iters[cw] = it;
        {
          const TmCtx<BG> copy = cx;
          write_rows<BG>(&copy, &c, X, cw, Z, z, -1);
        }
        const uint32_t* apq = reinterpret_cast<const uint32_t*>(smem + kAp);
        if (c.app_out || c.hard_out) {
          for (int j = tid; j < core_n; j += Z) {
            int v = lane_of(apq[j], X, kAB);
            if (FILL && j >= c.k_prime && j < K) v += c.app_clamp - kCapV;
            if (c.app_out) c.app_out[cw * c.app_stride + j] = (int16_t)v;
            if (c.hard_out) c.hard_out[cw * c.hard_stride + j] = v < 0 ? 1 : 0;
          }
        }
        if (c.hard_packed) {
          uint32_t* dst = c.hard_packed + cw * c.hard_words_stride;
          const int nwords = (c.hard_bits + 31) >> 5, ncore = core_n >> 5;
          for (int w = warp; w < min(nwords, ncore); w += Z / 32) {
            const int j = (w << 5) + lane;
            const bool bit = j < c.hard_bits && lane_of(apq[j], X, kAB) < 0;
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
            if (lane == 0) dst[w] = m;
          }
          if (nwords > ncore) {  // extension columns: word ncore + 12 (L - 4) + warp holds (L, 32 warp ..)
            const TmCtx<BG> copy = cx;
            static_for<4, T::MB>([&](auto li) {
              constexpr int L = decltype(li)::value;
              const int w = ncore + (Z / 32) * (L - 4) + warp;
              const int j = (w << 5) + lane;
              const bool bit = j < c.hard_bits && lane_of(pair_ext_app<BG, L>(copy), X) < 0;
              const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
              if (lane == 0 && w < nwords) dst[w] = m;
            });
          }
        }
      }
      act &= ~done;
      if (!act) break;  // the same for the whole CTA
      ++it;
      __syncthreads();
      cx.first_row();
      if constexpr (BG == 0) {
#pragma unroll 1
        for (int l = 0; l < 4; ++l) {
          TmHeadCtxT<kAp> h(cx, l);
          pair_row<0, 0, FILL>(h, bq2);
          __syncthreads();
        }
      }
      static_for<BG == 0 ? 4 : 0, T::MB>([&](auto li) {
        constexpr int L = decltype(li)::value;
        pair_row<BG, L, FILL>(cx, bq2);
        if constexpr (nr::barrier_after<BG>(L)) __syncthreads();
      });
      wait_st();  // this iteration's TMEM rows before the syndrome stages read them
      // syndrome: the quick-stage layers first, the others only for lanes that pass them
      if (z == 0) *s_fail = 0;
      __syncthreads();
      {
        const uint32_t odd = quick_parity<BG>(cx) & act;
        if (odd) atomicOr(s_fail, (int)odd);
      }
      __syncthreads();
      const uint32_t pass = act & ~(uint32_t)*s_fail;
      if (pass) {  // the same for the whole CTA
        const TmCtx<BG> copy = cx;
        const uint32_t odd = full_parity<BG>(&copy) & pass;
        if (odd) atomicOr(s_fail, (int)odd);
      }
      __syncthreads();
      done = it >= c.iterations ? act : act & ~(uint32_t)*s_fail;
    }
  }
  // Every TMEM access of this CTA completes before warp 0 frees the columns.
  wait_st();
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*s_tmem), "r"(kCols) : "memory");
  }
}

template <int BG, bool FILL>
cudaError_t launch_tm(const NrCommon& c0, int sms, cudaStream_t stream) {
  PairArgs<BG> a;
  a.c = c0;
  for (int e = 0; e < Tab<BG>::E; ++e) {
    a.sh4[e] = 0;
    a.cz4[e] = 0;
  }
  a.c.cpb = 1;
  const long long npairs = (c0.batch + 1) / 2;
  auto fn = nr_pair_tm_kernel<BG, FILL>;
  constexpr int smem = launch_smem<BG>();
  cudaError_t e = allow_max_dynamic_smem((const void*)fn);
  if (e != cudaSuccess) return e;
  // The whole unified L1 / shared array as shared memory, so that two CTAs (2 x 107 KB
  // with the per-CTA reserve) fit an SM.
  e = cudaFuncSetAttribute((const void*)fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                           cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  // The grid is sized for two CTAs per SM, the kernel's design point (80 registers x 384
  // threads: at most two are ever resident on an SM, so their 2 x 256 TMEM columns
  // never exceed the SM's 512 and no tcgen05.alloc waits on a CTA that is not running).
  // The occupancy calculator reported one CTA per SM here while the launch itself runs
  // two (ncu: register and shared-memory limits of two blocks each).
  const long long ctas = std::min<long long>(npairs, 2LL * sms);
  if (ctas <= 0) return cudaSuccess;
  fn<<<(unsigned)ctas, kPairThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace tm

// ------------------------------------------------------------ mixed shapes --
//
// Persistent paired decode of a mixed batch (the work items and per-codeword records
// of nr_kernels.h MixArgs): each CTA takes the next item from the device counter, an
// item being up to 2 * floor(384 / Z) codewords of one (BG, Z), decoded as consecutive
// pairs (codeword 2q in lane A, 2q + 1 in lane B).  The item's shifts and column bases
// are staged in shared memory (DevCtx<BG, -1>).  Every codeword gets the 5G prologue
// with its own filler count (the filler proxy is always on; it never touches a variable
// that is not filler) and writes its iterations and packed hard decisions.

constexpr int kPairMixTab = 2 * 316 * 4;  // 4 * shift and 4 * col * z of the largest graph
constexpr int kPairMixSmem = 232448 - 1024;

// ZT = 384: an item of Z = 384 (one codeword pair, CTA width 384), decoded with the
// compile-time shifts of the batch kernel; its posteriors sit at the fixed offset
// kPairMixAp384.  ZT = -1: any Z, shifts and column bases staged in shared memory.
// Out of line: each instantiation gets its own register allocation, which keeps the
// Z = 384 path free of the spills that the generic path's allocation has (measured:
// Z = 384 items as fast as the batch kernel, serving capacity +6 %).
constexpr int kPairMixAp384 = kPairMixTab + 16;

template <int BG, int ZT>
__device__ __noinline__ void pair_mixed_item(const MixArgs& m, const MixItem& it, int tab_off) {
  using T = Tab<BG>;
  using Ctx = DevCtx<BG, ZT, kPairMixAp384>;
  constexpr int NW = state_words<BG>(), CORE = T::KB + 4, NEXT = T::MB - 4;
  unsigned char* smem = pair_smem;
  const int Z = ZT > 0 ? ZT : it.z, ns = ZT > 0 ? kPairThreads : (int)blockDim.x, tid = (int)threadIdx.x;
  const int P = ZT > 0 ? 1 : (it.count + 1) / 2;
  if (ZT < 0) {
    int* t = reinterpret_cast<int*>(smem + tab_off);
    const short* sh = m.shift_tab + (long long)(BG * kMixLiftSizes + it.zi) * kMixEdges;
    const int* cz = m.colz_tab + (long long)(BG * kMixLiftSizes + it.zi) * kMixEdges;
    for (int e = tid; e < T::E; e += ns) {
      t[e] = 4 * (int)sh[e];
      t[T::E + e] = 4 * cz[e];
    }
  }
  const int base = tab_off + kPairMixTab;
  int* s_fail = reinterpret_cast<int*>(smem + base);
  int* s_done = s_fail + P;
  const int ap_base = base + al16(8 * P);
  const int ap_pair = CORE * Z * 4;
  const int st_base = ap_base + P * ap_pair;
  const int eh_base = st_base + NW * ns * 4;
  const int p = tid / Z, z = tid - p * Z;
  const bool lane_ok = p < P;
  const int pq = lane_ok ? p : 0;
  Ctx cx;
  cx.tab = tab_off;
  cx.ap = ap_base + pq * ap_pair;
  cx.st = st_base + 4 * tid;
  cx.ns = ns;
  cx.z4 = z * 4;
  cx.Z4 = Z * 4;
  cx.sc = 0xC480u;
  cx.k7f = 0x7F7F7F7Fu;
  asm volatile("" : "+r"(cx.sc), "+r"(cx.k7f));
  cx.a = nullptr;
  const int eh_off = eh_base + pq * NEXT * Z;
  const uint32_t bq2 = pair_beta(m.beta_q);
  const int core_n = CORE * Z, K = T::KB * Z;
  const int lane = tid & 31, warp = tid >> 5, nwarps = ns >> 5;
  const bool va = lane_ok && 2 * p < it.count, vbv = lane_ok && 2 * p + 1 < it.count;
  // ---- load: channel LLRs of variables 2Z..N; the punctured 2Z are erasures
  if (lane_ok) {
    const MixCodeword ca = m.cws[it.first + 2 * p];
    const MixCodeword cb = vbv ? m.cws[it.first + 2 * p + 1] : ca;
    const int8_t* sa = va ? m.llr + ca.llr_off - 2 * Z : nullptr;
    const int8_t* sb = vbv ? m.llr + cb.llr_off - 2 * Z : nullptr;
    const int kpa = ca.n_filler > K ? 0 : K - ca.n_filler, kpb = cb.n_filler > K ? 0 : K - cb.n_filler;
    auto fetch = [&](const int8_t* s, int j) -> int { return (s && j >= 2 * Z) ? (int)s[j] : 0; };
    uint32_t* apw = reinterpret_cast<uint32_t*>(smem + cx.ap);
    for (int col = 0; col < CORE; ++col) {
      const int j = col * Z + z;
      uint32_t l0 = kAB + (uint32_t)fetch(sa, j), l1 = kAB + (uint32_t)fetch(sb, j);
      if (j >= kpa && j < K) l0 = kAB + kCapV;
      if (j >= kpb && j < K) l1 = kAB + kCapV;
      apw[j] = (l0 & 0xFFFFu) | (l1 << 16);
    }
    static_for<0, Ctx::NX>([&](auto ri) {
      constexpr int r = decltype(ri)::value;
      uint32_t w = 0u;
      static_for<0, 2>([&](auto hi) {
        constexpr int h = decltype(hi)::value;
        constexpr int xi = 2 * r + h;
        if constexpr (xi < NEXT) {
          const int j = (CORE + xi) * Z + z;
          const uint32_t b0 = (uint32_t)(fetch(sa, j) + 128) & 0xFFu, b1 = (uint32_t)(fetch(sb, j) + 128) & 0xFFu;
          w |= (b0 | (b1 << 8)) << (16 * h);
        }
      });
      cx.x[r] = w;
    });
#pragma unroll 1
    for (int w = 0; w < NW; ++w) *reinterpret_cast<uint32_t*>(smem + st_base + 4 * (w * ns + tid)) = 0u;
  }
  __syncthreads();
  NrCommon none{};  // the mixed outputs are the packed hard decisions and iterations only
  uint32_t act = (va ? 1u : 0u) | (vbv ? 2u : 0u);
  uint32_t done = m.iterations <= 0 ? act : 0u;
  int itn = 0;
  for (;;) {
#pragma unroll 1
    for (int X = 0; X < 2; ++X) {
      const bool mine = ((done >> X) & 1u) != 0u;
      if (!__syncthreads_or(mine)) continue;
      if (lane_ok && z == 0) s_done[p] = mine ? 1 : 0;
      if (mine) {
        if (z == 0 && m.iters) m.iters[m.cws[it.first + 2 * p + X].index] = itn;
        const Ctx copy = cx;
        write_rows<BG>(&copy, &none, X, 0, Z, z, eh_off);
      }
      __syncthreads();
      for (int q = 0; q < P; ++q) {
        if (!s_done[q]) continue;
        const MixCodeword cw = m.cws[it.first + 2 * q + X];
        const uint32_t* apq = reinterpret_cast<const uint32_t*>(smem + ap_base + q * ap_pair);
        const uint8_t* ehq = smem + eh_base + q * NEXT * Z;
        uint32_t* dst = m.out + cw.out_off;
        const int nwords = (cw.hard_bits + 31) >> 5;
        for (int w = warp; w < nwords; w += nwarps) {
          const int j = (w << 5) + lane;
          bool bit = false;
          if (j < cw.hard_bits) bit = j < core_n ? lane_of(apq[j], X, kAB) < 0 : ehq[j - core_n] != 0;
          const uint32_t mm = __ballot_sync(0xFFFFFFFFu, bit);
          if (lane == 0) dst[w] = mm;
        }
      }
      __syncthreads();
    }
    act &= ~done;
    if (!__syncthreads_or(act != 0u)) break;
    ++itn;
    static_for<0, T::MB>([&](auto li) {
      constexpr int L = decltype(li)::value;
      if (lane_ok) pair_row<BG, L, true>(cx, bq2);
      if constexpr (nr::barrier_after<BG>(L)) __syncthreads();
    });
    if (lane_ok && z == 0) s_fail[p] = 0;
    __syncthreads();
    if (act) {
      const uint32_t odd = quick_parity<BG>(cx) & act;
      if (odd) atomicOr(&s_fail[p], (int)odd);
    }
    __syncthreads();
    const uint32_t pass = act & ~(uint32_t)(lane_ok ? s_fail[p] : 0);
    if (pass) {
      const Ctx copy = cx;
      const uint32_t odd = full_parity<BG>(&copy) & pass;
      if (odd) atomicOr(&s_fail[p], (int)odd);
    }
    __syncthreads();
    done = itn >= m.iterations ? act : act & ~(uint32_t)(lane_ok ? s_fail[p] : 0);
  }
}

__global__ void __launch_bounds__(kPairThreads, 1) nr_pair_mixed_kernel(const __grid_constant__ MixArgs m) {
  __shared__ int s_item;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = (int)atomicAdd(m.queue, 1u);
    __syncthreads();
    const int item = s_item;
    if (item >= m.n_items) break;
    const MixItem it = m.items[item];
    if (it.bg == 0) {
      if (it.z == 384)
        pair_mixed_item<0, 384>(m, it, 0);
      else
        pair_mixed_item<0, -1>(m, it, 0);
    } else {
      if (it.z == 384)
        pair_mixed_item<1, 384>(m, it, 0);
      else
        pair_mixed_item<1, -1>(m, it, 0);
    }
  }
}

// ------------------------------------------------- mixed shapes, TMEM state --
//
// The mixed-shape decode with the state layout of nr_pair_tm_kernel: two CTAs per SM,
// each with 256 TMEM columns for the CTA's life, taking work items from the device
// queue (an item: up to 2 * floor(384 / Z) codewords of one (BG, Z) as consecutive
// pairs).  Every thread runs every row update, syndrome stage and TMEM access of an
// item -- threads past the item's pairs on pair 0's posteriors without storing them,
// and the full syndrome stage for all threads whenever any pair passed the quick one --
// so that the warp-wide tcgen05 instructions never diverge (a warp can hold the rows
// of two pairs, which stop at different iterations).  The only per-pair work is the
// output: iterations and the packed hard decisions of the core columns, read from
// shared memory; a batch in which some codeword reports hard decisions beyond its
// core columns (the extension columns' decisions live in TMEM rows) goes to
// nr_pair_mixed_kernel instead.

constexpr int kTmMixTab = 16;                                    // 4 * shift [316], 4 * col * z [316]
constexpr int kTmMixFlags = kTmMixTab + 2 * 316 * 4;             // s_fail [192], s_done [192]
constexpr int kTmMixAp = kTmMixFlags + 2 * 192 * 4;              // posteriors, <= 26 * 384 words
constexpr int kTmMixSt = kTmMixAp + 26 * 384 * 4;                // shared state words [sm_words][384]
constexpr int kTmMixX = kTmMixSt + tm::sm_words<0>() * 384 * 4;  // extension words [ext_regs][384]
constexpr int kTmMixSmem = kTmMixX + ext_regs<0>() * 384 * 4;
static_assert(kTmMixAp % 16 == 0 && kTmMixSt % 16 == 0 && kTmMixX % 16 == 0, "alignment");
static_assert(tm::sm_words<1>() <= tm::sm_words<0>() && ext_regs<1>() <= ext_regs<0>() && 14 <= 26, "BG2 fits BG1's layout");
static_assert(kTmMixSmem + 1024 <= 233472 / 2, "two CTAs per SM");
// ... and never three of the two TMEM kernels on one SM (each holds 256 of the SM's
// 512 TMEM columns, so a third would wait in tcgen05.alloc)
static_assert(kTmMixSmem >= tm::kTwoPerSm, "at most two TMEM CTAs per SM");

template <int BG, int ZT>
__device__ __noinline__ void tm_mixed_item(const MixArgs& m, const MixItem& it, uint32_t tmb) {
  using T = Tab<BG>;
  using Ctx = tm::TmCtx<BG, ZT, kTmMixAp>;
  constexpr int CORE = T::KB + 4, NEXT = T::MB - 4, NX = ext_regs<BG>(), NSW = tm::sm_words<BG>();
  constexpr int NS = kPairThreads;
  unsigned char* smem = pair_smem;
  const int tid = (int)threadIdx.x;
  const int Z = ZT > 0 ? ZT : it.z;
  const int P = ZT > 0 ? 1 : (it.count + 1) / 2;
  if (ZT < 0) {
    int* t = reinterpret_cast<int*>(smem + kTmMixTab);
    const short* sh = m.shift_tab + (long long)(BG * kMixLiftSizes + it.zi) * kMixEdges;
    const int* cz = m.colz_tab + (long long)(BG * kMixLiftSizes + it.zi) * kMixEdges;
    for (int e = tid; e < T::E; e += NS) {
      t[e] = 4 * (int)sh[e];
      t[T::E + e] = 4 * cz[e];
    }
  }
  int* s_fail = reinterpret_cast<int*>(smem + kTmMixFlags);
  int* s_done = s_fail + 192;
  const int ap_pair = CORE * Z * 4;
  const int p = tid / Z, z = tid - p * Z;
  const bool lane_ok = p < P;
  const int pq = lane_ok ? p : 0, zq = lane_ok ? z : 0;
  Ctx cx;
  cx.tmb = tmb;
  cx.st = kTmMixSt + 4 * tid;
  cx.xo = kTmMixX + 4 * tid;
  cx.z4 = zq * 4;
  cx.sc = 0xC480u;
  cx.k7f = 0x7F7F7F7Fu;
  asm volatile("" : "+r"(cx.sc), "+r"(cx.k7f));
  cx.ap = kTmMixAp + pq * ap_pair;
  cx.tab = kTmMixTab;
  cx.Z4 = Z * 4;
  cx.live = lane_ok;
  const uint32_t bq2 = pair_beta(m.beta_q);
  const int K = T::KB * Z;
  const int lane = tid & 31, warp = tid >> 5, nwarps = NS >> 5;
  const bool va = lane_ok && 2 * p < it.count, vbv = lane_ok && 2 * p + 1 < it.count;
  // ---- load: channel LLRs of variables 2Z..N (the punctured 2Z are erasures), the
  // filler proxy for every codeword's filler bits, cleared state
  {
    const MixCodeword ca = m.cws[it.first + 2 * pq];
    const MixCodeword cb = vbv ? m.cws[it.first + 2 * p + 1] : ca;
    const int8_t* sa = va ? m.llr + ca.llr_off - 2 * Z : nullptr;
    const int8_t* sb = vbv ? m.llr + cb.llr_off - 2 * Z : nullptr;
    // through L2: the persistent serving kernel rewrites these bytes while it runs
    auto fetch = [&](const int8_t* src, int j) -> int { return (src && j >= 2 * Z) ? (int)__ldcg(src + j) : 0; };
    if (lane_ok) {
      const int kpa = ca.n_filler > K ? 0 : K - ca.n_filler, kpb = cb.n_filler > K ? 0 : K - cb.n_filler;
      uint32_t* apw = reinterpret_cast<uint32_t*>(smem + cx.ap);
      for (int col = 0; col < CORE; ++col) {
        const int j = col * Z + z;
        uint32_t l0 = kAB + (uint32_t)fetch(sa, j), l1 = kAB + (uint32_t)fetch(sb, j);
        if (j >= kpa && j < K) l0 = kAB + kCapV;
        if (j >= kpb && j < K) l1 = kAB + kCapV;
        apw[j] = (l0 & 0xFFFFu) | (l1 << 16);
      }
    }
    uint32_t* xw = reinterpret_cast<uint32_t*>(smem + kTmMixX);
#pragma unroll 1
    for (int r = 0; r < NX; ++r) {
      uint32_t w = 0u;
      for (int h = 0; h < 2; ++h) {
        const int xi = 2 * r + h;
        if (xi < NEXT) {
          const int j = (CORE + xi) * Z + z;
          const uint32_t b0 = (uint32_t)(fetch(sa, j) + 128) & 0xFFu, b1 = (uint32_t)(fetch(sb, j) + 128) & 0xFFu;
          w |= (b0 | (b1 << 8)) << (16 * h);
        }
      }
      xw[r * NS + tid] = w;
    }
    uint32_t* sw = reinterpret_cast<uint32_t*>(smem + kTmMixSt);
#pragma unroll 1
    for (int w = 0; w < NSW; ++w) sw[w * NS + tid] = 0u;
#pragma unroll 1
    for (int col = 0; col + 4 <= tm::kSlot; col += 4) tm::st4(tmb + (uint32_t)col, 0u, 0u, 0u, 0u);
    tm::st1(tmb + (uint32_t)(tm::kSlot - 1), 0u);
    tm::wait_st();
  }
  __syncthreads();
  const int core_n = CORE * Z;
  uint32_t act = (va ? 1u : 0u) | (vbv ? 2u : 0u);
  uint32_t done = m.iterations <= 0 ? act : 0u;
  int itn = 0;
  for (;;) {
#pragma unroll 1
    for (int X = 0; X < 2; ++X) {
      const bool mine = ((done >> X) & 1u) != 0u;
      if (!__syncthreads_or(mine)) continue;
      if (lane_ok && z == 0) s_done[p] = mine ? 1 : 0;
      if (mine && z == 0 && m.iters) m.iters[m.cws[it.first + 2 * p + X].index] = itn;
      __syncthreads();
      for (int q = 0; q < P; ++q) {
        if (!s_done[q]) continue;
        const MixCodeword cw = m.cws[it.first + 2 * q + X];
        const uint32_t* apq = reinterpret_cast<const uint32_t*>(smem + kTmMixAp + q * ap_pair);
        uint32_t* dst = m.out + cw.out_off;
        const int nwords = (cw.hard_bits + 31) >> 5;  // hard_bits <= core_n: the plan checks
        for (int w = warp; w < nwords; w += nwarps) {
          const int j = (w << 5) + lane;
          const bool bit = j < cw.hard_bits && j < core_n && lane_of(apq[j], X, kAB) < 0;
          const uint32_t mm = __ballot_sync(0xFFFFFFFFu, bit);
          if (lane == 0) dst[w] = mm;
        }
      }
      __syncthreads();
    }
    act &= ~done;
    if (!__syncthreads_or(act != 0u)) break;
    ++itn;
    cx.first_row();
    constexpr bool head_loop = BG == 0 && ZT > 0;
    if constexpr (head_loop) {
#pragma unroll 1
      for (int l = 0; l < 4; ++l) {
        tm::TmHeadCtxT<kTmMixAp> h(cx, l);
        pair_row<0, 0, true>(h, bq2);
        __syncthreads();
      }
    }
    static_for<head_loop ? 4 : 0, T::MB>([&](auto li) {
      constexpr int L = decltype(li)::value;
      pair_row<BG, L, true>(cx, bq2);
      if constexpr (nr::barrier_after<BG>(L)) __syncthreads();
    });
    tm::wait_st();  // this iteration's TMEM rows before the syndrome stages read them
    if (lane_ok && z == 0) s_fail[p] = 0;
    __syncthreads();
    {
      const uint32_t odd = quick_parity<BG>(cx) & act;
      if (odd) atomicOr(&s_fail[pq], (int)odd);
    }
    __syncthreads();
    const uint32_t pass = act & ~(uint32_t)(lane_ok ? s_fail[p] : 0);
    if (__syncthreads_or(pass != 0u)) {  // every thread, so that the TMEM reads stay warp-wide
      const Ctx copy = cx;
      const uint32_t odd = full_parity<BG>(&copy) & pass;
      if (odd) atomicOr(&s_fail[pq], (int)odd);
    }
    __syncthreads();
    done = itn >= m.iterations ? act : act & ~(uint32_t)(lane_ok ? s_fail[p] : 0);
  }
}

__global__ void __launch_bounds__(kPairThreads, 2) nr_pair_tm_mixed_kernel(const __grid_constant__ MixArgs m) {
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(pair_smem);
  int* s_item = reinterpret_cast<int*>(pair_smem + 4);
  const int warp = (int)threadIdx.x >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(s_tmem)),
                 "r"(tm::kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tm::fence_before();
  __syncthreads();
  tm::fence_after();
  const uint32_t tmb = *s_tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(tm::kSlot * (warp >> 2));
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) *s_item = (int)atomicAdd(m.queue, 1u);
    __syncthreads();
    const int item = *s_item;
    if (item >= m.n_items) break;
    const MixItem it = m.items[item];
    if (it.bg == 0) {
      if (it.z == 384)
        tm_mixed_item<0, 384>(m, it, tmb);
      else
        tm_mixed_item<0, -1>(m, it, tmb);
    } else {
      if (it.z == 384)
        tm_mixed_item<1, 384>(m, it, tmb);
      else
        tm_mixed_item<1, -1>(m, it, tmb);
    }
  }
  tm::wait_st();
  tm::fence_before();
  __syncthreads();
  if (warp == 0) {
    tm::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*s_tmem), "r"(tm::kCols) : "memory");
  }
}

// ------------------------------------------------- persistent serving kernel --
//
// One kernel for the whole serving stream (serve_kernels.h, ServeContArgs): CTAs claim
// work items from a ring the host publishes into host-mapped memory; per item a CTA
// runs the HARQ combine of its code blocks into int8 decoder input, the decode of
// tm_mixed_item, the code blocks' CRCs, and counts them done; the CTA that completes a
// transmission's last code block folds the TB CRC, writes the report and the
// desegmented bits to host-mapped memory and then the completion flag.
//
// Memory written while the kernel runs (decoder input, accumulators, staged LLRs, hard
// decisions, CRC records) is read through L2 (ld.cg); host-mapped records through
// ld.cv.  The only wait is the claim loop: bounded by idle_ns of the global timer and
// by an iteration limit, after which the CTA exits (the host relaunches the kernel when
// it publishes into a ring no kernel serves).

constexpr int kSrvHdr = kTmMixSmem;  // SrvHdr
constexpr int kSrvCws = kSrvHdr + 512;  // MixCodeword[kServeMaxItemCbs]
constexpr int kSrvSmem = kSrvCws + kServeMaxItemCbs * (int)sizeof(MixCodeword);
static_assert(kSrvSmem + 1024 <= 233472 / 2, "two CTAs per SM");

struct SrvHdr {
  long long item;  // claimed ring index, -1 = exit
  int last;        // this CTA completed the transmission
  int pad;
  ServeJob job;
  ServeTxRec rec;
  uint32_t red[2 * 12];
};
static_assert(sizeof(SrvHdr) <= 512 && sizeof(ServeTxRec) % 4 == 0 && sizeof(ServeJob) == 16, "serving header");

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_sys64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_acquire_sys32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_sys32(unsigned* p, unsigned v) {
  asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0: the next ring index, or -1 once this launch is closing.  The launch closes
// when no CTA has claimed an item (or seen a new one) for idle_ns, counted from the
// later of the last claim and this CTA's start, on the host's stop with the ring
// drained, or at the iteration limit.  One CTA at a time reads the host tail and
// mirrors it into device memory; the others poll the mirror.
//
// Placement: the two CTAs of an SM slow each other down (a lone BG1 Z=384 pair decodes
// in ~180 us, two side by side in ~320 us), so a CTA whose SM sibling is busy leaves a
// shallow queue (at most kShallow items) for up to kGraceNs to the CTAs of idle SMs.
constexpr unsigned long long kShallow = 2, kGraceNs = 20000;
__device__ __forceinline__ unsigned sm_id() {
  unsigned v;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(v));
  return v & 1023u;
}
__device__ long long srv_claim(const ServeContArgs& a, unsigned long long t_start) {
  ServeCtl* ctl = a.ctl;
  const unsigned sm = sm_id();
  unsigned nap = 256;  // backoff of an idle CTA, up to 8 us, so pollers leave the claim line to the claimers
  unsigned long long seen = 0;  // when this CTA first saw a claimable item it left to others
  for (int spins = 0; spins < (1 << 22); ++spins) {
    if (*reinterpret_cast<volatile unsigned*>(&ctl->closing) == a.epoch) return -1;
    const unsigned long long h = ld_acquire_gpu(&ctl->head), t = ld_acquire_gpu(&ctl->tail);
    if (h < t) {
      if (t - h <= kShallow && *reinterpret_cast<volatile int*>(a.sm_busy + sm) > 0) {
        const unsigned long long now = global_ns();
        if (seen == 0) seen = now;
        if (now - seen < kGraceNs) {
          __nanosleep(1000);
          continue;
        }
      }
      if (atomicCAS(&ctl->head, h, h + 1) == h) {
        atomicAdd(a.sm_busy + sm, 1);
        atomicMax(&ctl->last_ns, global_ns());
        __threadfence_system();  // the item's host-written records after the tail that covers it
        return (long long)h;
      }
      continue;
    }
    if (atomicCAS(&ctl->watch, 0u, 1u) == 0u) {
      const unsigned long long ht = ld_acquire_sys64(a.host_tail);
      const unsigned stop = ld_acquire_sys32(a.host_stop);
      if (ht > t) {
        __threadfence();
        atomicMax(&ctl->tail, ht);
        atomicMax(&ctl->last_ns, global_ns());
      }
      atomicExch(&ctl->watch, 0u);
      if (ht > h) continue;
      if (stop) break;
    }
    // (another CTA may stamp last_ns after this CTA read the timer: no unsigned wrap)
    const unsigned long long now = global_ns(), last = ld_acquire_gpu(&ctl->last_ns);
    const unsigned long long ref = last > t_start ? last : t_start;
    if (now > ref && now - ref > a.idle_ns) break;
    __nanosleep(nap);
    if (nap < 8192) nap *= 2;
  }
  atomicExch(&ctl->closing, a.epoch);
  return -1;
}

// CRC-24A register of the code block's first crc_len bits and the CRC-24B check over
// its K' bits, by the whole CTA: word w contributes (its bits * x^24 mod P) * x^(bits
// after it) mod P, and the contributions add (XOR).
__device__ void srv_cb_crc(const ServeContArgs& a, SrvHdr* hdr, const uint32_t* hard, int kp, int len, bool check_b,
                           ServeCbCrc* out) {
  const int tid = (int)threadIdx.x;
  const uint32_t(*ta)[256] = reinterpret_cast<const uint32_t(*)[256]>(a.crc_tab);
  const uint32_t(*tb)[256] = reinterpret_cast<const uint32_t(*)[256]>(a.crc_tab + 1024);
  const uint32_t* xa = a.xpow;
  const uint32_t* xb = a.xpow + kServeXpow;
  uint32_t ra = 0u, rb = 0u;
  for (int w = tid; 32 * w < kp; w += kPairThreads) {
    const uint32_t v = __brev(__ldcg(hard + w));  // first stream bit in the MSB
    const int nb = min(32, kp - 32 * w);
    const uint32_t vb = nb < 32 ? v >> (32 - nb) : v;
    rb ^= srv::crc_mulmod(srv::crc_step4(0u, vb, tb), __ldg(xb + (kp - 32 * w - nb)), srv::kPolyB);
    if (32 * w < len) {
      const int na = min(32, len - 32 * w);
      const uint32_t va = na < 32 ? v >> (32 - na) : v;
      ra ^= srv::crc_mulmod(srv::crc_step4(0u, va, ta), __ldg(xa + (len - 32 * w - na)), srv::kPolyA);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ra ^= __shfl_xor_sync(0xFFFFFFFFu, ra, o);
    rb ^= __shfl_xor_sync(0xFFFFFFFFu, rb, o);
  }
  const int lane = tid & 31, warp = tid >> 5;
  if (lane == 0) {
    hdr->red[2 * warp] = ra;
    hdr->red[2 * warp + 1] = rb;
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t sa = 0u, sb = 0u;
    for (int i = 0; i < kPairThreads / 32; ++i) {
      sa ^= hdr->red[2 * i];
      sb ^= hdr->red[2 * i + 1];
    }
    out->crc_a = sa;
    out->ok_b = check_b ? (sb == 0u ? 1 : 0) : 1;
  }
  __syncthreads();
}

// The transmission's report and desegmented bits (transport_block.rs:1014-1050), by the
// CTA that finished its last code block; then the completion flag.
__device__ void srv_finish(const ServeContArgs& a, const ServeTxRec& rec, int tx) {
  const int tid = (int)threadIdx.x;
  unsigned char* sm = pair_smem + kTmMixAp;  // the decode's areas are free here
  uint32_t(*my)[256] = reinterpret_cast<uint32_t(*)[256]>(sm);  // (v << 8k) * x^payload mod P_A
  uint32_t* s_crc = reinterpret_cast<uint32_t*>(sm + 3 * 1024);
  int* s_ok = reinterpret_cast<int*>(s_crc + 160);
  int* s_it = s_ok + 160;
  int* s_slot = s_it + 160;
  const int C = rec.n_cb;
  for (int i = tid; i < 768; i += kPairThreads)
    my[i >> 8][i & 255] = srv::crc_mulmod((uint32_t)(i & 255) << (8 * (i >> 8)), rec.x_payload, srv::kPolyA);
  for (int i = tid; i < C; i += kPairThreads) {
    const int slot = __ldcv(a.slots + (long long)tx * kServeMaxCbs + i);
    s_slot[i] = slot;
    s_crc[i] = __ldcg(&a.crc[slot].crc_a);
    s_ok[i] = __ldcg(&a.crc[slot].ok_b);
    s_it[i] = __ldcg(a.iters + slot);
  }
  __syncthreads();
  ServeTxOut* out = a.outs + tx;
  if (tid == 0) {
    uint32_t total = 0;
    int all_cb = 1, max_it = 0;
    for (int i = 0; i < C; ++i) {
      const long long rest = rec.b - (long long)i * rec.payload;
      const int len = (int)(rest < 0 ? 0 : (rest < rec.payload ? rest : rec.payload));
      if (len == rec.payload)
        total = srv::mul_fixed(total, my) ^ s_crc[i];
      else if (len > 0)
        total = srv::crc_mulmod(total, i == C - 1 ? rec.x_last : srv::crc_xpow(len, srv::kPolyA), srv::kPolyA) ^
                s_crc[i];
      all_cb &= s_ok[i];
      max_it = max(max_it, s_it[i]);
    }
    out->result[0] = (all_cb && total == 0u) ? 1 : 0;
    out->result[1] = max_it;
  }
  if (tid < 6) {
    uint32_t bits = 0;
    for (int t = 0; t < 32 && 32 * tid + t < C; ++t) bits |= (uint32_t)s_ok[32 * tid + t] << t;
    out->result[2 + tid] = (int32_t)bits;
  }
  // TB bit i is bit i % payload of code block i / payload; a word spans at most two
  // code blocks (with more than one block, payload > 32)
  const int hw = (rec.k_prime + 31) >> 5;
  auto bits_at = [&](int c, int j) -> uint32_t {  // 32 bits of block c from bit j on (0 past its words)
    const uint32_t* h = a.hard + (long long)s_slot[c] * kServeHardWords;
    const int w = j >> 5;
    const uint32_t lo = w < hw ? __ldcg(h + w) : 0u, hi = w + 1 < hw ? __ldcg(h + w + 1) : 0u;
    return __funnelshift_r(lo, hi, (unsigned)(j & 31));
  };
  const int nwords = (int)((rec.tb_size + 31) >> 5);
  for (int w = tid; w < nwords; w += kPairThreads) {
    const int i0 = 32 * w;
    const int c = i0 / rec.payload, j = i0 - c * rec.payload;
    uint32_t v = bits_at(c, j);
    const int avail = rec.payload - j;
    if (avail < 32) {
      v &= (1u << avail) - 1u;
      if (c + 1 < C) v |= bits_at(c + 1, 0) << avail;
    }
    const long long left = rec.tb_size - i0;
    if (left < 32) v &= (1u << left) - 1u;
    rec.bits[w] = v;
  }
  __threadfence_system();
  __syncthreads();
  if (tid == 0) {
    a.tx_done[tx] = 0;  // ready for the slot's next transmission
    __threadfence_system();
    st_release_sys32(&out->flag, rec.seq);
  }
}

__global__ void __launch_bounds__(kPairThreads, 2) serve_cont_kernel(const __grid_constant__ ServeContArgs a) {
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(pair_smem);
  SrvHdr* hdr = reinterpret_cast<SrvHdr*>(pair_smem + kSrvHdr);
  MixCodeword* cws = reinterpret_cast<MixCodeword*>(pair_smem + kSrvCws);
  const int tid = (int)threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(s_tmem)),
                 "r"(tm::kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tm::fence_before();
  __syncthreads();
  tm::fence_after();
  const uint32_t tmb = *s_tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(tm::kSlot * (warp >> 2));
  const unsigned long long t_start = global_ns();
  MixArgs m{};
  m.cws = cws;
  m.llr = a.llr;
  m.out = a.hard;
  m.iters = a.iters;
  m.shift_tab = a.shift_tab;
  m.colz_tab = a.colz_tab;
  m.beta_q = a.beta_q;
  m.app_clamp = a.app_clamp;
  m.iterations = a.iterations;
  m.k32 = 32;
  m.two = 2;
  for (;;) {
    __syncthreads();
    if (tid == 0) hdr->item = srv_claim(a, t_start);
    __syncthreads();
    const long long item = hdr->item;
    if (item < 0) break;
    unsigned long long tp[5];  // phase boundaries (thread 0)
    if (tid == 0) tp[0] = global_ns();
    // the job and its transmission's record, host-mapped
    if (tid < 4)
      reinterpret_cast<int*>(&hdr->job)[tid] =
          __ldcv(reinterpret_cast<const int*>(a.ring + (unsigned long long)item % a.ring_cap) + tid);
    __syncthreads();
    const int tx = hdr->job.tx;
    if (tid < (int)(sizeof(ServeTxRec) / 4))
      reinterpret_cast<int*>(&hdr->rec)[tid] = __ldcv(reinterpret_cast<const int*>(a.recs + tx) + tid);
    __syncthreads();
    const ServeTxRec& rec = hdr->rec;
    const int first_cb = hdr->job.first_cb, count = hdr->job.count;
    if (tid < count) {
      const int slot = __ldcv(a.slots + (long long)tx * kServeMaxCbs + first_cb + tid);
      MixCodeword c{};
      c.llr_off = (long long)slot * kServeLlrStride;
      c.out_off = (long long)slot * kServeHardWords;
      c.n_filler = rec.n_filler;
      c.hard_bits = rec.k_prime;
      c.index = slot;
      cws[tid] = c;
    }
    __syncthreads();
    // HARQ combine of the item's code blocks into their decoder input
    {
      srv::CombineWalk w;
      w.ncb = rec.ncb;
      w.fs = rec.fs;
      w.fe = rec.fe;
      w.m = rec.m;
      w.c0 = rec.c0;
      w.e_len = rec.e_len;
      w.qm = rec.qm;
      w.first = rec.first;
      for (int j = 0; j < count; ++j) {
        const int ci = first_cb + j;
        float* acc = rec.acc + (long long)ci * rec.ncb;
        const float* e = rec.e + (long long)ci * rec.e_len;
        int8_t* llr = a.llr + cws[j].llr_off;
        srv::combine_cb(w, acc, e, llr, a.scale, tid, kPairThreads);
      }
    }
    __syncthreads();
    if (tid == 0) tp[1] = global_ns();
    MixItem it{};
    it.bg = rec.bg;
    it.z = rec.z;
    it.zi = rec.zi;
    it.count = count;
    it.first = 0;
    if (it.bg == 0) {
      if (it.z == 384)
        tm_mixed_item<0, 384>(m, it, tmb);
      else
        tm_mixed_item<0, -1>(m, it, tmb);
    } else {
      if (it.z == 384)
        tm_mixed_item<1, 384>(m, it, tmb);
      else
        tm_mixed_item<1, -1>(m, it, tmb);
    }
    __syncthreads();
    if (tid == 0) tp[2] = global_ns();
    for (int j = 0; j < count; ++j) {
      const int ci = first_cb + j, slot = cws[j].index;
      const long long rest = rec.b - (long long)ci * rec.payload;
      const int len = (int)(rest < 0 ? 0 : (rest < rec.payload ? rest : rec.payload));
      srv_cb_crc(a, hdr, a.hard + (long long)slot * kServeHardWords, rec.k_prime, len, rec.has_cb_crc != 0,
                 a.crc + slot);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      tp[3] = global_ns();
      hdr->last = atomicAdd(a.tx_done + tx, count) + count == rec.n_cb ? 1 : 0;
    }
    __syncthreads();
    if (hdr->last) {
      __threadfence();
      srv_finish(a, rec, tx);
    }
    if (tid == 0) {
      tp[4] = global_ns();
      atomicSub(a.sm_busy + sm_id(), 1);
      ServeCtl* c = a.ctl;
      atomicAdd(&c->items, 1ull);
      atomicAdd(&c->busy_ns, tp[4] - tp[0]);
      atomicAdd(&c->combine_ns, tp[1] - tp[0]);
      atomicAdd(&c->decode_ns, tp[2] - tp[1]);
      atomicAdd(&c->crc_ns, tp[3] - tp[2]);
      atomicAdd(&c->finish_ns, tp[4] - tp[3]);
    }
  }
  tm::wait_st();
  tm::fence_before();
  __syncthreads();
  if (warp == 0) {
    tm::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*s_tmem), "r"(tm::kCols) : "memory");
  }
}

}  // namespace nrp

cudaError_t serve_cont_prepare() {
  cudaError_t e = cudaFuncSetAttribute(nrp::serve_cont_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       nrp::kSrvSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(nrp::serve_cont_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                              cudaSharedmemCarveoutMaxShared);
}

// Two CTAs per SM (see pair_tm_mixed_launch); every CTA stays until it finds no item.
cudaError_t serve_cont_launch(const ServeContArgs& a, int sms, cudaStream_t stream) {
  nrp::serve_cont_kernel<<<2 * std::max(sms, 1), nrp::kPairThreads, nrp::kSrvSmem, stream>>>(a);
  return cudaGetLastError();
}

bool nr_pair_applies(const NrCommon& c) {
  const bool fill = c.prologue && c.k_prime < c.k;
  return c.app_clamp >= (fill ? nrp::kMinFillerClamp : nrp::kMaxReach) && c.z >= 1 && c.z <= 384;
}

cudaError_t nr_pair_decode_i8(int bg, const NrCommon& c, const int* shifts, int sms, cudaStream_t stream,
                              bool tmem) {
  const bool fill = c.prologue && c.k_prime < c.k;
  if (tmem && c.z == 384) {
    if (bg == 0) return fill ? nrp::tm::launch_tm<0, true>(c, sms, stream) : nrp::tm::launch_tm<0, false>(c, sms, stream);
    return fill ? nrp::tm::launch_tm<1, true>(c, sms, stream) : nrp::tm::launch_tm<1, false>(c, sms, stream);
  }
  if (bg == 0) return nrp::launch_bg<0>(c, shifts, fill, sms, stream);
  return nrp::launch_bg<1>(c, shifts, fill, sms, stream);
}

int pair_mixed_capacity(int bg, int z) {
  (void)bg;
  return 2 * std::max(1, nrp::kPairThreads / std::max(z, 1));
}

cudaError_t pair_mixed_prepare() {
  return cudaFuncSetAttribute(nrp::nr_pair_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              nrp::kPairMixSmem);
}

cudaError_t pair_tm_mixed_prepare() {
  cudaError_t e = cudaFuncSetAttribute(nrp::nr_pair_tm_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       nrp::kTmMixSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(nrp::nr_pair_tm_mixed_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                              cudaSharedmemCarveoutMaxShared);
}

// Two CTAs per SM (80 registers x 384 threads: never more on one SM, so their 2 x 256
// TMEM columns never exceed the SM's 512).
cudaError_t pair_tm_mixed_launch(const MixArgs& m, int sms, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(m.queue, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  const int ctas = std::max(1, std::min(2 * sms, m.n_items));
  nrp::nr_pair_tm_mixed_kernel<<<ctas, nrp::kPairThreads, nrp::kTmMixSmem, stream>>>(m);
  return cudaGetLastError();
}

int pair_mixed_core_columns(int bg) { return bg == 0 ? 26 : 14; }

cudaError_t pair_mixed_launch(const MixArgs& m, int sms, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(m.queue, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  const int ctas = std::max(1, std::min(sms, m.n_items));
  nrp::nr_pair_mixed_kernel<<<ctas, nrp::kPairThreads, nrp::kPairMixSmem, stream>>>(m);
  return cudaGetLastError();
}

}  // namespace syn

