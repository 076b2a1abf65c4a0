// Compile-time view of the 5G NR base graphs (BG1, BG2) in layered order, shared
// by the 5G NR int8 kernels (nr_kernels.cu, nr_pair_kernels.cu) and the host
// emulation of the paired kernel used by the tests.
//
// Layer l's edges are loff(l)..loff(l+1)-1 with column col(e), in the order of
// the reference's build_layout (src/qc_ldpc.rs:281-319).  Layers >= 4 each own
// one degree-1 extension column, column KB + l.  z384_shift(e) is edge e's cyclic
// shift at lifting size 384.
#pragma once

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline __attribute__((always_inline))
#endif
#endif

#include <type_traits>

#include "nr_layered_tables.h"

namespace syn {
namespace nr {

template <int BG>
struct Tab;

template <>
struct Tab<0> {
  static constexpr int MB = 46, NB = 68, KB = 22, E = 316;
  __host__ __device__ static constexpr int loff(int i) { return syn_bg1_loff(i); }
  __host__ __device__ static constexpr int col(int e) { return syn_bg1_lcol(e); }
  __host__ __device__ static constexpr int z384_shift(int e) { return syn_bg1_lz384(e); }
};

template <>
struct Tab<1> {
  static constexpr int MB = 42, NB = 52, KB = 10, E = 197;
  __host__ __device__ static constexpr int loff(int i) { return syn_bg2_loff(i); }
  __host__ __device__ static constexpr int col(int e) { return syn_bg2_lcol(e); }
  __host__ __device__ static constexpr int z384_shift(int e) { return syn_bg2_lz384(e); }
};

template <int BG>
__host__ __device__ constexpr int deg_of(int l) {
  return Tab<BG>::loff(l + 1) - Tab<BG>::loff(l);
}

template <int BG>
__host__ __device__ constexpr bool is_ext(int l, int e) {
  return l >= 4 && Tab<BG>::col(Tab<BG>::loff(l) + e) == Tab<BG>::KB + l;
}

template <int BG>
__host__ __device__ constexpr int ext_pos(int l) {
  for (int e = 0; e < deg_of<BG>(l); ++e)
    if (is_ext<BG>(l, e)) return e;
  return -1;
}

// True if layers a and b share a core column (a variable kept in shared memory).
template <int BG>
__host__ __device__ constexpr bool share_core(int a, int b) {
  for (int i = 0; i < deg_of<BG>(a); ++i) {
    const int ca = Tab<BG>::col(Tab<BG>::loff(a) + i);
    if (ca >= Tab<BG>::KB + 4) continue;
    for (int j = 0; j < deg_of<BG>(b); ++j)
      if (Tab<BG>::col(Tab<BG>::loff(b) + j) == ca) return true;
  }
  return false;
}

// Layers run in order, and a block barrier separates two of them only where the later
// one reads a core column that a layer since the previous barrier wrote: runs of
// consecutive layers with pairwise disjoint columns (most of the degree-5 tail of both
// base graphs) touch disjoint variables, so their rows may interleave freely and the
// result is the same as strictly in order.
template <int BG>
__host__ __device__ constexpr int group_start(int l) {
  int s = 0;
  for (int m = 1; m <= l; ++m)
    for (int k = s; k < m; ++k)
      if (share_core<BG>(k, m)) {
        s = m;
        break;
      }
  return s;
}
template <int BG>
__host__ __device__ constexpr bool barrier_after(int l) {
  return l + 1 >= Tab<BG>::MB || group_start<BG>(l + 1) == l + 1;
}

// Syndrome check after every iteration, in two stages: the kQuick layers with the
// fewest edges (lower index first among equal degrees) for every codeword, the other
// layers only for codewords that satisfy those.  One layer alone passes too often on
// codewords still far from converged (BG1's 3-edge layer 4 is satisfied in about a
// third of the iterations at 1 dB, the other layers in 10-20 %), and every pass costs
// a check of all the other rows.
constexpr int kQuick = 3;
template <int BG>
__host__ __device__ constexpr bool is_quick(int l) {
  int rank = 0;
  for (int m = 0; m < Tab<BG>::MB; ++m)
    if (deg_of<BG>(m) < deg_of<BG>(l) || (deg_of<BG>(m) == deg_of<BG>(l) && m < l)) ++rank;
  return rank < kQuick;
}

template <int I, int N, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, N>(f);
  }
}

}  // namespace nr
}  // namespace syn
