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

// Layer with the fewest edges: checked first after every iteration.
template <int BG>
__host__ __device__ constexpr int quick_layer() {
  int best = 0;
  for (int l = 1; l < Tab<BG>::MB; ++l)
    if (deg_of<BG>(l) < deg_of<BG>(best)) best = l;
  return best;
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
