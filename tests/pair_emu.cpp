// Host emulation of the paired 5G NR int8 kernel's arithmetic (test infrastructure).
//
// Runs the row update and parity check of syndrome_b200/csrc/nr_pair.cuh, the same
// code the sm_100a kernel inlines, on the CPU: rows of one layer one after another
// (they touch disjoint variables), layers in order, two codewords per 32-bit word.
// The tests compare its results with the oracle to check the packed-lane
// arithmetic on the CPU; the GPU parity tests check the kernel itself.
#include <cstdint>
#include <cstring>
#include <vector>

#include "nr_pair.cuh"

using namespace syn::nrp;

namespace {

template <int BG>
struct EmuCtx : WordRows<BG, EmuCtx<BG>> {
  EmuCtx(uint32_t* ap_, uint32_t* st_, const uint32_t* x_, int z_, int Z_, const int* sh_)
      : ap(ap_), st(st_), x(x_), z(z_), Z(Z_), sh(sh_) {}
  uint32_t* ap;
  uint32_t* st;
  const uint32_t* x;
  int z, Z;
  const int* sh;
  template <int GE>
  int vb() const {
    // at Z = 384 the compile-time shift table, as in the kernel's Z = 384 instantiation
    const int s = Z == 384 ? Tab<BG>::z384_shift(GE) : sh[GE];
    return (Tab<BG>::col(GE) * Z + (z + s) % Z) * 4;
  }
  uint32_t ld_ap(int b) const { return ap[b / 4]; }
  void st_ap(int b, uint32_t v) { ap[b / 4] = v; }
  uint32_t ld_st(int w) const { return st[w]; }
  void st_st(int w, uint32_t v) { st[w] = v; }
  uint32_t xr(int i) const { return x[i]; }
  uint32_t selc() const { return 0xC480u; }
  uint32_t c7f() const { return 0x7F7F7F7Fu; }
};

template <int BG, bool FILL>
int run(int Z, const int* shifts, int beta_q, int app_clamp, int prologue, int n_filler, const int8_t* llr_a,
        const int8_t* llr_b, int iterations, int16_t* app_out, int8_t* edge_r_out, int32_t* iters_out) {
  using T = Tab<BG>;
  const int N = T::NB * Z, core = (T::KB + 4) * Z, K = T::KB * Z;
  const int kp = n_filler > K ? 0 : K - n_filler;
  constexpr int NW = state_words<BG>(), NX = ext_regs<BG>();
  std::vector<uint32_t> ap(core), st((size_t)NW * Z, 0u), xr((size_t)NX * Z, 0u);
  const int8_t* src[2] = {llr_a, llr_b};
  for (int j = 0; j < N; ++j) {
    uint32_t lanes[2];
    for (int l = 0; l < 2; ++l) {
      int v = src[l][j];
      if (prologue && j < 2 * Z) v = 0;
      const bool filler = prologue && j >= kp && j < K;
      if (j < core)
        lanes[l] = filler ? kAB + kCapV : kAB + v;
      else
        lanes[l] = (uint32_t)(v + 128) & 0xFFu;
    }
    if (j < core) {
      ap[j] = lanes[0] | (lanes[1] << 16);
    } else {
      const int xi = j / Z - T::KB - 4, z = j % Z;
      xr[(size_t)z * NX + (xi >> 1)] |= (lanes[0] | (lanes[1] << 8)) << (16 * (xi & 1));
    }
  }
  const uint32_t bq2 = pair_beta(beta_q);
  auto ctx = [&](int z) {
    return EmuCtx<BG>(ap.data(), st.data() + (size_t)z * NW, xr.data() + (size_t)z * NX, z, Z, shifts);
  };
  auto snapshot = [&](int lane, int used) {
    iters_out[lane] = used;
    int16_t* app = app_out + (size_t)lane * N;
    int8_t* er = edge_r_out + (size_t)lane * T::E * Z;
    for (int j = 0; j < core; ++j) {
      int v = (int)((ap[j] >> (16 * lane)) & 0xFFFFu) - (int)kAB;
      if (FILL && j >= kp && j < K) v += app_clamp - kCapV;
      app[j] = (int16_t)v;
    }
    for (int z = 0; z < Z; ++z) {
      auto c = ctx(z);
      static_for<0, T::MB>([&](auto li) {
        constexpr int L = decltype(li)::value;
        if constexpr (L >= 4) {
          const uint32_t a = pair_ext_app<BG, L>(c);
          app[(T::KB + L) * Z + z] = (int16_t)((int)((a >> (16 * lane)) & 0xFFFFu) - (int)kPB);
        }
        static_for<0, deg_of<BG>(L)>([&](auto ei) {
          constexpr int e = decltype(ei)::value;
          const uint32_t m = pair_message<BG, L, e>(c);
          er[(size_t)(T::loff(L) + e) * Z + z] = (int8_t)((int)((m >> (16 * lane)) & 0xFFu) - 127);
        });
      });
    }
  };
  uint32_t act = 3u;
  for (int it = 1; it <= iterations && act; ++it) {
    static_for<0, T::MB>([&](auto li) {
      constexpr int L = decltype(li)::value;
      for (int z = 0; z < Z; ++z) {
        auto c = ctx(z);
        pair_row<BG, L, FILL>(c, bq2);
      }
    });
    uint32_t odd = 0u;
    for (int z = 0; z < Z; ++z) {
      auto c = ctx(z);
      static_for<0, T::MB>([&](auto li) {
        constexpr int L = decltype(li)::value;
        odd |= pair_parity<BG, L>(c);
      });
    }
    const uint32_t done = act & ~odd;
    for (int lane = 0; lane < 2; ++lane)
      if (done >> lane & 1u) snapshot(lane, it);
    act &= ~done;
  }
  for (int lane = 0; lane < 2; ++lane)
    if (act >> lane & 1u) snapshot(lane, iterations);
  return 0;
}

}  // namespace

extern "C" {

// Decodes codewords A and B (int8 channel values of all N variables) of 5G NR base
// graph bg (0 = BG1) at lifting size Z with the paired arithmetic.  shifts: per edge
// in layer order, reduced mod Z.  Outputs per lane: app_out[2][N], edge_r_out[2][E*Z],
// iters_out[2].  Returns -1 if the paired arithmetic does not apply (app_clamp too small).
int pair_emu_decode(int bg, int Z, const int* shifts, int beta_q, int app_clamp, int prologue, int n_filler,
                    const int8_t* llr_a, const int8_t* llr_b, int iterations, int16_t* app_out,
                    int8_t* edge_r_out, int32_t* iters_out) {
  const bool fill = prologue && n_filler > 0;
  if (app_clamp < (fill ? kMinFillerClamp : kMaxReach)) return -1;
  if (bg == 0)
    return fill ? run<0, true>(Z, shifts, beta_q, app_clamp, prologue, n_filler, llr_a, llr_b, iterations, app_out,
                               edge_r_out, iters_out)
                : run<0, false>(Z, shifts, beta_q, app_clamp, prologue, n_filler, llr_a, llr_b, iterations,
                                app_out, edge_r_out, iters_out);
  return fill ? run<1, true>(Z, shifts, beta_q, app_clamp, prologue, n_filler, llr_a, llr_b, iterations, app_out,
                             edge_r_out, iters_out)
              : run<1, false>(Z, shifts, beta_q, app_clamp, prologue, n_filler, llr_a, llr_b, iterations,
                              app_out, edge_r_out, iters_out);
}

}  // extern "C"
