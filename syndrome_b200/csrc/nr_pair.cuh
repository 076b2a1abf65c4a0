// Two-codeword (paired) int8 layered offset min-sum row update for the 5G NR base
// graphs, shared by the sm_100a kernel (nr_pair_kernels.cu) and the host
// emulation the tests run against the oracle.
//
// Arithmetic of syndrome src/qc_ldpc.rs:1530-1758 (int8 messages, int16
// posterior, Q clamped to +-127, R = sign-excluded product * max(min_excl - beta_q, 0),
// posterior += R_new - R_old), computed for two codewords at once: every 32-bit
// word holds codeword A in its low 16-bit lane and codeword B in its high lane.
//
// Lane encodings (per 16-bit lane, all values non-negative so that one 32-bit add
// or subtract never carries across lanes, and unsigned 16x2 min/max order them):
//   posterior / Q      PB + v with PB = 0x8000 (|v| <= 3938 + 127, or the filler
//                      proxy below); the lane's top bit is 1 iff v >= 0
//   message table out  127 + R (R in [-127, 127]), zero-extended
//   min-sum key        |Q| * 256 + tag(edge)
//
// Per check row the compressed C->V state is one meta word, bytes
// [min1'A, min2'A, min1'B, min2'B] (offset magnitudes), and ceil(deg / 8) code
// words with two bits per lane and edge: bit 0 = "this edge takes min2'" (the
// argmin), bit 1 = "R >= 0".  For edge j of a code word (j < 8) lane A's code sits
// at bit s_j = 2 * (j & 3) + 16 * (j >> 2) and lane B's at s_j + 8, so that
// ((code >> s_j) & 0x0303) | 0xC480 is a byte-permute selector that picks both
// lanes' messages out of the row's 8-byte table
//   [127 - m1'A, 127 - m2'A, 127 + m1'A, 127 + m2'A, same for B]
// (nibbles 1 and 3 replicate the sign of table bytes 0 and 4, which are < 128,
// giving zero high bytes).  The reference's messages are exactly this function of
// the row state: every edge gets min1' except the argmin, which gets min2', and
// ties give min2' = min1' (qc_ldpc.rs:1700-1718).
//
// Filler proxy: a filler variable starts at app_clamp C and, while C >= 7874, its
// Q is always clamped to +127 and its posterior only ever meets the upper clamp;
// the posterior equals C - d with d the same non-negative deficit that CAPV - d
// follows under min(., CAPV).  The kernel stores min(posterior, CAPV) (exact for
// every non-filler variable, which never exceeds 3938) and adds C - CAPV back to
// filler posteriors on output.
#pragma once

#include <cstdint>

#include "nr_graph.cuh"

namespace syn {
namespace nrp {

using nr::deg_of;
using nr::ext_pos;
using nr::is_ext;
using nr::is_quick;
using nr::static_for;
using nr::Tab;

constexpr uint32_t kPB = 0x8000u;            // lane bias of computed values (Q, app)
constexpr uint32_t kPB2 = 0x80008000u;
// Stored posterior lanes carry kAB = PB + 127, the message table's bias, so that
// Q = stored - message and stored' = Q + message need no constant.
constexpr uint32_t kAB = kPB + 127u;
constexpr uint32_t kAB2 = kAB * 0x10001u;
constexpr int kCapV = 8192;                  // filler proxy ceiling (>= 7874)
constexpr uint32_t kCapS2 = (kAB + kCapV) * 0x10001u;  // filler proxy ceiling, stored form
constexpr int kMinFillerClamp = 7874;        // 30 * 254 + 2 * 127: deficit bound plus Q clamp
constexpr int kMaxReach = 3938;              // 128 + 30 * 127: largest reachable |posterior|

// Multipliers read from the constant bank: the compiler cannot see their values, so
// the multiply-adds below stay multiply-adds on the FMA pipe instead of becoming
// shifts, adds or LEAs on the integer ALU pipe, which is the kernel's binding pipe.
// [0] 1, [1] -1, [2] 256, [3] 0xFFFF, [4..6] 2^30, 2^28, 2^26, [7] 2^16,
// [8..11] 2^16, 2^14, 2^12, 2^10.
#define SYN_PAIR_K \
  { 1u, 0xFFFFFFFFu, 256u, 0xFFFFu, 1u << 30, 1u << 28, 1u << 26, 1u << 16, 1u << 16, 1u << 14, 1u << 12, 1u << 10 }
#ifdef __CUDACC__
static __constant__ uint32_t kPairK[12] = SYN_PAIR_K;
#endif

// ------------------------------------------------------------------ SWAR ops --

__host__ __device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t s) {
#ifdef __CUDA_ARCH__
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(s));
  return d;
#else
  const uint64_t src = (uint64_t)a | ((uint64_t)b << 32);
  uint32_t d = 0;
  for (int i = 0; i < 4; ++i) {
    const uint32_t n = (s >> (4 * i)) & 15u;
    uint32_t byte = (uint32_t)(src >> (8 * (n & 7))) & 0xFFu;
    if (n & 8) byte = (byte & 0x80u) ? 0xFFu : 0u;
    d |= byte << (8 * i);
  }
  return d;
#endif
}

__host__ __device__ __forceinline__ uint32_t vmaxu2(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  uint32_t d;
  asm("max.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
#else
  const uint32_t lo = (a & 0xFFFFu) > (b & 0xFFFFu) ? (a & 0xFFFFu) : (b & 0xFFFFu);
  const uint32_t hi = (a >> 16) > (b >> 16) ? (a >> 16) : (b >> 16);
  return lo | (hi << 16);
#endif
}

__host__ __device__ __forceinline__ uint32_t vminu2(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  uint32_t d;
  asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
#else
  const uint32_t lo = (a & 0xFFFFu) < (b & 0xFFFFu) ? (a & 0xFFFFu) : (b & 0xFFFFu);
  const uint32_t hi = (a >> 16) < (b >> 16) ? (a >> 16) : (b >> 16);
  return lo | (hi << 16);
#endif
}

// High word of a * b: a >> (32 - log2 b) for a power-of-two b, as a multiply (FMA pipe)
// instead of a shift (ALU pipe).
__host__ __device__ __forceinline__ uint32_t mulhi(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// x << n with n >= 32 (including "negative" n wrapped to large unsigned) giving 0.
__host__ __device__ __forceinline__ uint32_t shl_sat(uint32_t x, uint32_t n) {
#ifdef __CUDA_ARCH__
  uint32_t d;
  asm("shl.b32 %0, %1, %2;" : "=r"(d) : "r"(x), "r"(n));
  return d;
#else
  return n >= 32 ? 0u : x << n;
#endif
}

// ------------------------------------------------------------ row geometry --

__host__ __device__ constexpr int ncw(int deg) { return (deg + 7) / 8; }

// Bit offset of edge e's lane-A code inside its code word.
__host__ __device__ constexpr int code_shift(int e) { return 2 * ((e & 7) & 3) + 16 * ((e & 7) >> 2); }
// Min-sum key tag of edge e: code word index * 32 + code_shift.
__host__ __device__ constexpr int key_tag(int e) { return 32 * (e >> 3) + code_shift(e); }

// First state word (the meta word) of layer l; code words follow it.
template <int BG>
__host__ __device__ constexpr int state_off(int l) {
  int w = 0;
  for (int i = 0; i < l; ++i) w += 1 + ncw(deg_of<BG>(i));
  return w;
}
template <int BG>
__host__ __device__ constexpr int state_words() {
  return state_off<BG>(Tab<BG>::MB);
}
// Extension-column channel registers: two layers (4 bytes: A, B, A, B) per word.
template <int BG>
__host__ __device__ constexpr int ext_regs() {
  return (Tab<BG>::MB - 4 + 1) / 2;
}

// a * K[ki] + b and hi(a * K[ki]), with K the multiplier table above (IMADs on the device).
__host__ __device__ __forceinline__ uint32_t mad_k(uint32_t a, int ki, uint32_t b) {
#ifdef __CUDA_ARCH__
  return a * kPairK[ki] + b;
#else
  constexpr uint32_t K[12] = SYN_PAIR_K;
  return a * K[ki] + b;
#endif
}
__host__ __device__ __forceinline__ uint32_t mulhi_k(uint32_t a, int ki) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, kPairK[ki]);
#else
  constexpr uint32_t K[12] = SYN_PAIR_K;
  return (uint32_t)(((uint64_t)a * K[ki]) >> 32);
#endif
}

// Byte-permute selector of an edge from its code word: ((code >> shift) & 0x0303) | selc
// with selc = 0xC480, the shift as a multiply-high and the mask-and-or as one LOP3
// (written out: the compiler splits it in two otherwise).
__host__ __device__ __forceinline__ uint32_t code_sel(uint32_t code_word, int shift, uint32_t selc) {
  const uint32_t w = shift ? mulhi_k(code_word, shift < 16 ? 3 + (shift >> 1) : 8 + ((shift - 16) >> 1)) : code_word;
#ifdef __CUDA_ARCH__
  uint32_t d;
  asm("lop3.b32 %0, %1, 0x0303, %2, 0xEA;" : "=r"(d) : "r"(w), "r"(selc));
  return d;
#else
  return (w & 0x0303u) | selc;
#endif
}

// Message tables of a meta word [m1'A, m2'A, m1'B, m2'B]: lo = lane A's bytes
// [127 - m1', 127 - m2', 127 + m1', 127 + m2'], hi = lane B's; c7f = 0x7F7F7F7F.
// With mB = meta >> 16: hi = mB * 0xFFFF + c7f and lo = (meta & 0xFFFF) * 0xFFFF + c7f
// = meta * 0xFFFF + mB * 2^16 + c7f (mod 2^32), all multiply-adds.
__host__ __device__ __forceinline__ void tables(uint32_t meta, uint32_t c7f, uint32_t& lo, uint32_t& hi) {
  const uint32_t mB = mulhi_k(meta, 7);
  hi = mad_k(mB, 3, c7f);
  lo = mad_k(mB, 7, mad_k(meta, 3, c7f));
}

// Biased channel value lanes (PB + x) of extension layer index xi (= layer - 4).
__host__ __device__ __forceinline__ uint32_t ext_lanes(uint32_t xreg, int xi) {
  return prmt(xreg, 0u, (xi & 1) ? 0x4342u : 0x4140u) + 0x7F807F80u;
}

// ------------------------------------------------------------- row update ---
//
// Ctx provides, for one (codeword pair, lifting index z):
//   template <int GE> int vb() const     byte offset in the pair's posterior array
//                                        of edge GE's variable (column, (z + shift) mod Z)
//   uint32_t ld_ap(int) / void st_ap(int, uint32_t)
//   template <int L, int N> void row_load(uint32_t (&w)[N])    the N = 1 + ncw(deg) state
//   template <int L, int N> void row_store(const uint32_t (&w)[N])  words of layer L's row
//                                        (meta word, then the code words)
//   template <int L> void row_next()     called once per row after row_load: the context
//                                        may start fetching the state of the row after L
//   template <int L> uint32_t row_word(int i) const   state word i of layer L's row (cold
//                                        paths: syndrome, outputs)
//   uint32_t xr(int i) const             extension channel register i
//   uint32_t selc() const, c7f() const   the constants 0xC480 and 0x7F7F7F7F (registers)

// Offset beta_q in the key domain (beta_q * 256 in both lanes; the pair_row argument).
__host__ __device__ constexpr uint32_t pair_beta(int beta_q) { return (uint32_t)beta_q * 0x01000100u; }

template <int BG, int L, bool FILL, class C>
__host__ __device__ __forceinline__ void pair_row(C& c, uint32_t bq2) {
  constexpr int lb = Tab<BG>::loff(L), deg = deg_of<BG>(L), NC = ncw(deg);
  constexpr int ep = L >= 4 ? ext_pos<BG>(L) : -1;
  const uint32_t selc = c.selc(), c7f = c.c7f();
  uint32_t rw[1 + NC];
  c.template row_load<L, 1 + NC>(rw);
  c.template row_next<L>();
  const uint32_t meta = rw[0];
  uint32_t code[NC];
  static_for<0, NC>([&](auto ki) {
    constexpr int k = decltype(ki)::value;
    code[k] = rw[1 + k];
  });
  uint32_t tlo, thi;
  tables(meta, c7f, tlo, thi);
  uint32_t qu[deg];
  int vb[deg];
  // The two smallest keys (distinct: the tags differ), with the keys taken in pairs:
  // sort the pair, then merge it into the running (min1, min2).  That is fewer
  // operations than one key at a time and halves the dependency chain through min1.
  uint32_t m1k = 0u, m2k = 0u, held = 0u;
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    if constexpr (e == ep) {
      qu[e] = ext_lanes(c.xr((L - 4) >> 1), L - 4);  // Q of the extension edge is its channel value
      vb[e] = 0;
    } else {
      vb[e] = c.template vb<lb + e>();
      // PB + app - R_old = stored - (127 + R_old)
      qu[e] = mad_k(prmt(tlo, thi, code_sel(code[e >> 3], code_shift(e), selc)), 1, c.ld_ap(vb[e]));
    }
    // PB + min(|Q|, 127) (0x10000 - Q32 is PB - Q in both lanes), then
    // key = |Q| * 256 + tag (the 256 * PB terms cancel mod 2^32)
    const uint32_t aq = vminu2(vmaxu2(qu[e], mad_k(qu[e], 1, 0x00010000u)), 0x807F807Fu);
    const uint32_t key = mad_k(aq, 2, (uint32_t)key_tag(e) * 0x10001u - 0x00800000u);
    if constexpr (e % 2 == 0 && e + 1 < deg) {
      held = key;
    } else if constexpr (e % 2 == 1) {
      const uint32_t lo = vminu2(held, key), hi = vmaxu2(held, key);
      if constexpr (e == 1) {
        m1k = lo, m2k = hi;
      } else {
        m2k = vminu2(vminu2(m2k, hi), vmaxu2(m1k, lo));
        m1k = vminu2(m1k, lo);
      }
    } else {  // odd degree: the last key alone
      m2k = vminu2(m2k, vmaxu2(m1k, key));
      m1k = vminu2(m1k, key);
    }
  });
  // Row results.  In the key domain, max(key, 256 beta) - 256 beta has byte 1 of each
  // lane = max(min - beta, 0), the offset magnitude; one byte permute gathers
  // [min1'A, min2'A, min1'B, min2'B] into the new meta word.
  const uint32_t m1x = vmaxu2(m1k, bq2) - bq2, m2x = vmaxu2(m2k, bq2) - bq2;
  const uint32_t nmeta = prmt(m1x, m2x, 0x7351u);
  uint32_t nlo, nhi;
  tables(nmeta, c7f, nlo, nhi);
  // Code words: the Q >= 0 bits (top bits of the lanes) of edges j and j + 4 spread to
  // whole bytes by one sign-replicating byte-permute, then masked into each edge's
  // sign slot ...
  uint32_t nc[NC];
  uint32_t sacc = 0u;
  static_for<0, NC>([&](auto ki) {
    constexpr int k = decltype(ki)::value;
    nc[k] = 0u;
    static_for<0, 4>([&](auto ji) {
      constexpr int j = decltype(ji)::value;
      constexpr int e0 = 8 * k + j, e1 = 8 * k + j + 4;
      if constexpr (e0 < deg) {
        uint32_t hi = 0u;
        if constexpr (e1 < deg) hi = qu[e1];
        const uint32_t t = prmt(qu[e0], hi, 0xFDB9u);  // bytes: A_j, B_j, A_j+4, B_j+4 as 0x00 / 0xFF
        nc[k] |= t & (0x02020202u << (2 * j));
        sacc ^= t;
      }
    });
  });
  // ... turned into R's sign (Q >= 0 xor an odd count of negative Q in the row):
  // bytes [A, B, A, B] of par are each lane's parity of Q >= 0 as 0x00 / 0xFF ...
  const uint32_t par = sacc ^ prmt(sacc, sacc, 0x1032u);
  const uint32_t smask = ((deg & 1) ? ~par : par) & 0xAAAAAAAAu;
  // ... plus the argmin flag from the winning key's tag.
  const uint32_t tA = m1k & 255u, tB = prmt(m1k, 0u, 0x4442u);
  static_for<0, NC>([&](auto ki) {
    constexpr int k = decltype(ki)::value;
    nc[k] = (nc[k] ^ smask) | shl_sat(1u, tA - 32u * k) | shl_sat(256u, tB - 32u * k);
  });
  // Posterior update: stored = Q + 127 + R_new.
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    if constexpr (e != ep) {
      uint32_t v = mad_k(prmt(nlo, nhi, code_sel(nc[e >> 3], code_shift(e), selc)), 0, qu[e]);
      if constexpr (FILL) v = vminu2(v, kCapS2);
      c.st_ap(vb[e], v);
    }
  });
  uint32_t nw[1 + NC];
  nw[0] = nmeta;
  static_for<0, NC>([&](auto ki) {
    constexpr int k = decltype(ki)::value;
    nw[1 + k] = nc[k];
  });
  c.template row_store<L, 1 + NC>(nw);
}

// Message lanes (127 + R) of edge e of layer L from the stored state.
template <int BG, int L, int E, class C>
__host__ __device__ __forceinline__ uint32_t pair_message(const C& c) {
  uint32_t lo, hi;
  tables(c.template row_word<L>(0), 0x7F7F7F7Fu, lo, hi);
  return prmt(lo, hi, code_sel(c.template row_word<L>(1 + (E >> 3)), code_shift(E), 0xC480u));
}

// Row-level state access over word accessors ld_st(w) / st_st(w, v) (w = state word
// index, state_off<BG>(L) + i for word i of layer L's row): the storage of the
// one-pair-per-SM kernel and of the host emulation.  B is the base graph, D the
// context deriving from this.
template <int BG, class D>
struct WordRows {
  template <int L, int N>
  __host__ __device__ __forceinline__ void row_load(uint32_t (&w)[N]) const {
    static_for<0, N>([&](auto ii) { w[decltype(ii)::value] = self().ld_st(state_off<BG>(L) + decltype(ii)::value); });
  }
  template <int L, int N>
  __host__ __device__ __forceinline__ void row_store(const uint32_t (&w)[N]) {
    static_for<0, N>([&](auto ii) { self().st_st(state_off<BG>(L) + decltype(ii)::value, w[decltype(ii)::value]); });
  }
  template <int L>
  __host__ __device__ __forceinline__ void row_next() {}
  template <int L>
  __host__ __device__ __forceinline__ uint32_t row_word(int i) const {
    return self().ld_st(state_off<BG>(L) + i);
  }

 private:
  __host__ __device__ __forceinline__ const D& self() const { return static_cast<const D&>(*this); }
  __host__ __device__ __forceinline__ D& self() { return static_cast<D&>(*this); }
};

// Posterior lanes (PB + app) of the extension column of layer L >= 4.
template <int BG, int L, class C>
__host__ __device__ __forceinline__ uint32_t pair_ext_app(const C& c) {
  constexpr int ep = ext_pos<BG>(L);
  return ext_lanes(c.xr((L - 4) >> 1), L - 4) + pair_message<BG, L, ep>(c) - 0x007F007Fu;
}

// Parity of check row (L, z) under the current posteriors: bit 0 = lane A has an
// odd number of negative posteriors, bit 1 = lane B.
template <int BG, int L, class C>
__host__ __device__ __forceinline__ uint32_t pair_parity(const C& c) {
  constexpr int lb = Tab<BG>::loff(L), deg = deg_of<BG>(L);
  constexpr int ep = L >= 4 ? ext_pos<BG>(L) : -1;
  uint32_t x = 0u;
  static_for<0, deg>([&](auto ei) {
    constexpr int e = decltype(ei)::value;
    if constexpr (e == ep) {
      x ^= pair_ext_app<BG, L>(c);
    } else {
      x ^= c.ld_ap(c.template vb<lb + e>()) - (kAB2 - kPB2);  // stored lanes to PB + app
    }
  });
  const uint32_t nn = ((x >> 15) & 1u) | ((x >> 30) & 2u);
  return nn ^ ((deg & 1) ? 3u : 0u);
}

// Parity of the quick-stage layers (same bits as pair_parity).
template <int BG, class C>
__host__ __device__ __forceinline__ uint32_t quick_parity(const C& c) {
  uint32_t odd = 0u;
  static_for<0, Tab<BG>::MB>([&](auto li) {
    constexpr int L = decltype(li)::value;
    if constexpr (is_quick<BG>(L)) odd |= pair_parity<BG, L>(c);
  });
  return odd;
}

}  // namespace nrp
}  // namespace syn
