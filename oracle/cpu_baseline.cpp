// CPU baseline: the reference's own CPU decode path, restated in C++ so it can be
// timed on the GPU host (the Rust original cannot be built there).  Test and
// benchmark infrastructure only; the decoder library never links it.
//
//   * AVX2 int8 kernels   syndrome src/simd_avx2.rs:546-847 (q_build_edge_i8_avx2,
//                         decode_layer_passes_i8_avx2, apply_delta16_i8_avx2)
//   * int8 driver loop    src/qc_ldpc.rs:1530-1758 (deg < 2 layers on the scalar path)
//   * 5G int8 prologue    src/qc_ldpc.rs:1486-1523
//   * LdpcPipeline        src/ldpc_pipeline.rs:267-575: a pool of 16 frame slots,
//                         one SPSC work ring and one done ring per worker,
//                         fewest-outstanding dispatch with a rotating cursor, workers
//                         pinned to cores and spinning on their ring.
// Compiled with -mavx2 and without AVX-512, like the reference's kernels.  The
// reference clamps the pipeline to POOL_SIZE/2 = 8 workers
// (src/ldpc_pipeline.rs:375); `max_workers` lifts that clamp so every host core
// can be used.
#include <immintrin.h>
#include <pthread.h>
#include <sched.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../syndrome_b200/csrc/graph_tables.h"
#include "../syndrome_b200/csrc/base_graph_tables.inc"

namespace {

struct Layout {
  int z = 0, mb = 0, nb = 0, maxdeg = 0;
  std::vector<int> lo, cols, shifts;
  long long n() const { return (long long)nb * z; }
  long long k() const { return (long long)(nb - mb) * z; }
  int edges() const { return (int)cols.size(); }
};

const int kSets[8][8] = {{2, 4, 8, 16, 32, 64, 128, 256},   {3, 6, 12, 24, 48, 96, 192, 384},
                         {5, 10, 20, 40, 80, 160, 320, -1}, {7, 14, 28, 56, 112, 224, -1, -1},
                         {9, 18, 36, 72, 144, 288, -1, -1}, {11, 22, 44, 88, 176, 352, -1, -1},
                         {13, 26, 52, 104, 208, -1, -1, -1}, {15, 30, 60, 120, 240, -1, -1, -1}};

bool make_layout(int bg, int z, Layout* L) {
  int ils = -1;
  for (int s = 0; s < 8 && ils < 0; ++s)
    for (int j = 0; j < 8; ++j)
      if (kSets[s][j] == z) ils = s;
  if (ils < 0 || (bg != 0 && bg != 1)) return false;
  const syn_bg_entry_t* ents = bg == 0 ? syn_bg1_entries : syn_bg2_entries;
  const int n = bg == 0 ? SYN_BG1_EDGES : SYN_BG2_EDGES;
  L->z = z;
  L->mb = bg == 0 ? SYN_BG1_ROWS : SYN_BG2_ROWS;
  L->nb = bg == 0 ? SYN_BG1_COLS : SYN_BG2_COLS;
  std::vector<int> deg(L->mb, 0);
  for (int i = 0; i < n; ++i) ++deg[ents[i].r];
  L->lo.assign(L->mb + 1, 0);
  for (int i = 0; i < L->mb; ++i) L->lo[i + 1] = L->lo[i] + deg[i];
  L->cols.assign(n, 0);
  L->shifts.assign(n, 0);
  std::vector<int> fill(L->lo.begin(), L->lo.end() - 1);
  for (int i = 0; i < n; ++i) {
    int p = fill[ents[i].r]++;
    L->cols[p] = ents[i].c;
    L->shifts[p] = ents[i].v[ils] % z;
  }
  L->maxdeg = *std::max_element(deg.begin(), deg.end());
  return true;
}

inline int wrap(int s, int z) { return s >= z ? s - z : s; }

// simd_avx2.rs:591-669.
void q_build_i8(int z, int shift, int var_base, int q_base, int base_edge, const int16_t* app,
                const int8_t* er, int8_t* q) {
  const __m256i hi = _mm256_set1_epi16(127), lo = _mm256_set1_epi16(-127);
  const int full = z & ~15;
  int i = 0;
  for (; i < full; i += 16) {
    const int start = wrap(i + shift, z);
    __m256i a;
    if (start + 16 <= z) {
      a = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(app + var_base + start));
    } else {
      alignas(32) int16_t tmp[16];
      for (int j = 0; j < 16; ++j) tmp[j] = app[var_base + wrap(start + j, z)];
      a = _mm256_load_si256(reinterpret_cast<const __m256i*>(tmp));
    }
    const __m256i r = _mm256_cvtepi8_epi16(_mm_loadu_si128(reinterpret_cast<const __m128i*>(er + base_edge + i)));
    __m256i d = _mm256_subs_epi16(a, r);
    d = _mm256_min_epi16(_mm256_max_epi16(d, lo), hi);
    const __m256i p = _mm256_packs_epi16(d, d);
    _mm_storel_epi64(reinterpret_cast<__m128i*>(q + q_base + i), _mm256_castsi256_si128(p));
    _mm_storel_epi64(reinterpret_cast<__m128i*>(q + q_base + i + 8), _mm256_extracti128_si256(p, 1));
  }
  for (; i < z; ++i) {
    int d = (int)app[var_base + wrap(i + shift, z)] - (int)er[base_edge + i];
    q[q_base + i] = (int8_t)std::min(std::max(d, -127), 127);
  }
}

// simd_avx2.rs:546-576.
inline void apply_delta16(int16_t* app, int var_base, int shift, int z, int zi, __m256i delta, __m256i clo,
                          __m256i chi, int C) {
  const int start = wrap(zi + shift, z);
  if (start + 16 <= z) {
    __m256i* p = reinterpret_cast<__m256i*>(app + var_base + start);
    const __m256i v = _mm256_adds_epi16(_mm256_loadu_si256(p), delta);
    _mm256_storeu_si256(p, _mm256_min_epi16(_mm256_max_epi16(v, clo), chi));
  } else {
    alignas(32) int16_t tmp[16];
    _mm256_store_si256(reinterpret_cast<__m256i*>(tmp), delta);
    for (int j = 0; j < 16; ++j) {
      int16_t* slot = &app[var_base + wrap(start + j, z)];
      int v = std::min(std::max((int)*slot + tmp[j], -32768), 32767);
      *slot = (int16_t)std::min(std::max(v, -C), C);
    }
  }
}

// simd_avx2.rs:683-847.
void layer_passes_i8(int z, int deg, int beta_q, int C, const int8_t* q, int8_t* er, int lb,
                     const int* cols, const int* shifts, int16_t* app, int8_t* m1, int8_t* m2,
                     uint8_t* sx) {
  const __m256i sign_mask = _mm256_set1_epi8((char)0x80), msg_max = _mm256_set1_epi8(127);
  const __m256i ones = _mm256_set1_epi8(1), beta = _mm256_set1_epi8((char)beta_q);
  const __m256i zero = _mm256_setzero_si256();
  const __m256i chi = _mm256_set1_epi16((short)C), clo = _mm256_set1_epi16((short)-C);
  const int full = z & ~31;
  for (int i = 0; i < full; i += 32) {
    _mm256_storeu_si256(reinterpret_cast<__m256i*>(m1 + i), msg_max);
    _mm256_storeu_si256(reinterpret_cast<__m256i*>(m2 + i), msg_max);
    _mm256_storeu_si256(reinterpret_cast<__m256i*>(sx + i), zero);
  }
  for (int i = full; i < z; ++i) {
    m1[i] = 127;
    m2[i] = 127;
    sx[i] = 0;
  }
  for (int e = 0; e < deg; ++e) {
    const int8_t* qp = q + e * z;
    for (int c = 0; c < full; c += 32) {
      const __m256i qq = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(qp + c));
      const __m256i a = _mm256_abs_epi8(qq);
      __m256i* sp = reinterpret_cast<__m256i*>(sx + c);
      _mm256_storeu_si256(sp, _mm256_xor_si256(_mm256_loadu_si256(sp), _mm256_and_si256(qq, sign_mask)));
      __m256i* p1 = reinterpret_cast<__m256i*>(m1 + c);
      __m256i* p2 = reinterpret_cast<__m256i*>(m2 + c);
      const __m256i v1 = _mm256_loadu_si256(p1), v2 = _mm256_loadu_si256(p2);
      _mm256_storeu_si256(p1, _mm256_min_epi8(v1, a));
      _mm256_storeu_si256(p2, _mm256_min_epi8(v2, _mm256_max_epi8(v1, a)));
    }
    for (int i = full; i < z; ++i) {
      const int8_t qq = qp[i];
      const int8_t a = (int8_t)(qq < 0 ? -qq : qq);
      sx[i] ^= (uint8_t)qq & 0x80;
      const int8_t o1 = m1[i];
      m1[i] = std::min(o1, a);
      m2[i] = std::min(m2[i], std::max(o1, a));
    }
  }
  for (int e = 0; e < deg; ++e) {
    const int var_base = cols[lb + e] * z, shift = shifts[lb + e];
    const int8_t* qp = q + e * z;
    int8_t* rp = er + (long long)(lb + e) * z;
    for (int c = 0; c < full; c += 32) {
      const __m256i qq = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(qp + c));
      const __m256i a = _mm256_abs_epi8(qq);
      const __m256i v1 = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(m1 + c));
      const __m256i v2 = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(m2 + c));
      const __m256i s = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(sx + c));
      const __m256i eq = _mm256_cmpeq_epi8(a, v1);
      const __m256i mex = _mm256_blendv_epi8(v1, v2, eq);
      const __m256i mag = _mm256_max_epi8(_mm256_sub_epi8(mex, beta), zero);
      const __m256i sgn = _mm256_xor_si256(s, _mm256_and_si256(qq, sign_mask));
      const __m256i nr = _mm256_sign_epi8(mag, _mm256_or_si256(sgn, ones));
      const __m256i orr = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(rp + c));
      _mm256_storeu_si256(reinterpret_cast<__m256i*>(rp + c), nr);
      const __m256i dlo = _mm256_sub_epi16(_mm256_cvtepi8_epi16(_mm256_castsi256_si128(nr)),
                                           _mm256_cvtepi8_epi16(_mm256_castsi256_si128(orr)));
      const __m256i dhi = _mm256_sub_epi16(_mm256_cvtepi8_epi16(_mm256_extracti128_si256(nr, 1)),
                                           _mm256_cvtepi8_epi16(_mm256_extracti128_si256(orr, 1)));
      apply_delta16(app, var_base, shift, z, c, dlo, clo, chi, C);
      apply_delta16(app, var_base, shift, z, c + 16, dhi, clo, chi, C);
    }
    for (int i = full; i < z; ++i) {
      const int8_t qq = qp[i];
      const int8_t a = (int8_t)(qq < 0 ? -qq : qq);
      const uint8_t sg = sx[i] ^ ((uint8_t)qq & 0x80);
      const int8_t mex = a == m1[i] ? m2[i] : m1[i];
      const int8_t mag = (int8_t)std::max(mex - beta_q, 0);
      const int8_t neg = (int8_t)((int8_t)sg >> 7);
      const int8_t nr = (int8_t)((int8_t)(mag ^ neg) - neg);
      const int8_t orr = rp[i];
      rp[i] = nr;
      int16_t* slot = &app[var_base + wrap(i + shift, z)];
      int v = std::min(std::max((int)*slot + (int)nr - (int)orr, -32768), 32767);
      *slot = (int16_t)std::min(std::max(v, -C), C);
    }
  }
}

// Scalar passes for degenerate layers (src/qc_ldpc.rs:1670-1745).
void layer_passes_scalar(int z, int deg, int beta_q, int C, const int8_t* q, int8_t* er, int lb,
                         const int* cols, const int* shifts, int16_t* app, int8_t* m1, int8_t* m2,
                         uint8_t* sx) {
  for (int i = 0; i < z; ++i) {
    m1[i] = 127;
    m2[i] = 127;
    sx[i] = 0;
  }
  for (int e = 0; e < deg; ++e)
    for (int i = 0; i < z; ++i) {
      const int8_t qq = q[e * z + i];
      const int8_t a = (int8_t)(qq < 0 ? -qq : qq);
      sx[i] ^= (uint8_t)qq & 0x80;
      const int8_t o1 = m1[i];
      m1[i] = std::min(o1, a);
      m2[i] = std::min(m2[i], std::max(o1, a));
    }
  if (deg < 2)
    for (int i = 0; i < z; ++i) {
      if (deg == 0) m1[i] = 0;
      m2[i] = m1[i];
    }
  for (int e = 0; e < deg; ++e) {
    const int var_base = cols[lb + e] * z, shift = shifts[lb + e];
    int8_t* rp = er + (long long)(lb + e) * z;
    for (int i = 0; i < z; ++i) {
      const int8_t qq = q[e * z + i];
      const int8_t a = (int8_t)(qq < 0 ? -qq : qq);
      const uint8_t sg = sx[i] ^ ((uint8_t)qq & 0x80);
      const int8_t mex = a == m1[i] ? m2[i] : m1[i];
      const int8_t mag = (int8_t)std::max(mex - beta_q, 0);
      const int8_t neg = (int8_t)((int8_t)sg >> 7);
      const int8_t nr = (int8_t)((int8_t)(mag ^ neg) - neg);
      const int8_t orr = rp[i];
      rp[i] = nr;
      int16_t* slot = &app[var_base + wrap(i + shift, z)];
      int v = std::min(std::max((int)*slot + (int)nr - (int)orr, -32768), 32767);
      *slot = (int16_t)std::min(std::max(v, -C), C);
    }
  }
}

bool syndrome_ok(const Layout& L, const int16_t* app) {
  const int z = L.z;
  for (int l = 0; l < L.mb; ++l)
    for (int zi = 0; zi < z; ++zi) {
      unsigned par = 0;
      for (int e = L.lo[l]; e < L.lo[l + 1]; ++e) par ^= app[L.cols[e] * z + wrap(zi + L.shifts[e], z)] < 0;
      if (par) return false;
    }
  return true;
}

struct Frame {
  std::vector<int16_t> app;
  std::vector<int8_t> er, q, m1, m2;
  std::vector<uint8_t> sx, hard;
  int iters = 0;
  long long tag = 0;
};

// src/qc_ldpc.rs:1530-1758 with the AVX2 passes.
int decode_i8_avx2(const Layout& L, int beta_q, int C, Frame& f, int iterations) {
  const int z = L.z;
  const long long n = L.n();
  std::fill(f.er.begin(), f.er.end(), 0);
  for (long long i = 0; i < n; ++i) f.app[i] = (int16_t)std::min(std::max((int)f.app[i], -C), C);
  int used = 0;
  for (int it = 0; it < iterations; ++it) {
    ++used;
    for (int l = 0; l < L.mb; ++l) {
      const int lb = L.lo[l], deg = L.lo[l + 1] - lb;
      for (int e = 0; e < deg; ++e)
        q_build_i8(z, L.shifts[lb + e], L.cols[lb + e] * z, e * z, (lb + e) * z, f.app.data(), f.er.data(),
                   f.q.data());
      if (deg >= 2)
        layer_passes_i8(z, deg, beta_q, C, f.q.data(), f.er.data(), lb, L.cols.data(), L.shifts.data(),
                        f.app.data(), f.m1.data(), f.m2.data(), f.sx.data());
      else
        layer_passes_scalar(z, deg, beta_q, C, f.q.data(), f.er.data(), lb, L.cols.data(), L.shifts.data(),
                            f.app.data(), f.m1.data(), f.m2.data(), f.sx.data());
    }
    if (syndrome_ok(L, f.app.data())) break;
  }
  for (long long i = 0; i < n; ++i) f.hard[i] = f.app[i] < 0;
  return used;
}

void init_frame(const Layout& L, Frame& f) {
  f.app.assign(L.n(), 0);
  f.er.assign((size_t)L.edges() * L.z + 32, 0);
  f.q.assign((size_t)L.maxdeg * L.z + 32, 0);
  f.m1.assign(L.z + 32, 0);
  f.m2.assign(L.z + 32, 0);
  f.sx.assign(L.z + 32, 0);
  f.hard.assign(L.n(), 0);
}

// Fills a frame the way decode_5g_i8 sees it: int8 channel values of variables
// [llr_offset, n), then the filler and puncture prologue (src/qc_ldpc.rs:1506-1513).
void load_frame(const Layout& L, Frame& f, const int8_t* llr, int llr_offset, long long n_filler, int C) {
  const long long n = L.n(), k = L.k();
  for (long long i = 0; i < llr_offset; ++i) f.app[i] = 0;
  for (long long i = llr_offset; i < n; ++i) f.app[i] = llr[i - llr_offset];
  const long long kp = n_filler > k ? 0 : k - n_filler;
  for (long long i = kp; i < k; ++i) f.app[i] = (int16_t)std::max(C, 0);
  for (long long i = 0; i < 2LL * L.z; ++i) f.app[i] = 0;
}

// Lock-free single-producer single-consumer ring of slot indices (src/spsc_queue.rs:171-260).
struct Spsc {
  alignas(64) std::atomic<size_t> head{0};
  alignas(64) std::atomic<size_t> tail{0};
  int buf[16];
  bool push(int v) {
    const size_t t = tail.load(std::memory_order_relaxed);
    if (t - head.load(std::memory_order_acquire) == 16) return false;
    buf[t & 15] = v;
    tail.store(t + 1, std::memory_order_release);
    return true;
  }
  bool pop(int* v) {
    const size_t h = head.load(std::memory_order_relaxed);
    if (h == tail.load(std::memory_order_acquire)) return false;
    *v = buf[h & 15];
    head.store(h + 1, std::memory_order_release);
    return true;
  }
};

// src/ldpc_pipeline.rs:267-286.
int pick_worker(const std::vector<int>& outstanding, size_t cursor) {
  const int n = (int)outstanding.size();
  int best = (int)(cursor % n);
  int load = outstanding[best];
  for (int step = 1; step < n; ++step) {
    const int wi = (int)((cursor + step) % n);
    if (outstanding[wi] < load) {
      best = wi;
      load = outstanding[wi];
    }
  }
  return best;
}

void pin(int core) {
  cpu_set_t set;
  CPU_ZERO(&set);
  CPU_SET(core % CPU_SETSIZE, &set);
  pthread_setaffinity_np(pthread_self(), sizeof(set), &set);
}

}  // namespace

extern "C" {

// Single-threaded AVX2 int8 decode of one codeword (decode_5g_i8 when nr_prologue).
// app/edge_r/hard are in/out like the reference's buffers.  Returns iterations used,
// -1 for an invalid code.
int cpb_decode_i8(int bg, int z, int beta_q, int app_clamp, int16_t* app, int8_t* edge_r, uint8_t* hard,
                  int iterations) {
  Layout L;
  if (!make_layout(bg, z, &L)) return -1;
  Frame f;
  init_frame(L, f);
  std::copy(app, app + L.n(), f.app.begin());
  const int used = decode_i8_avx2(L, beta_q, std::max(app_clamp, 0), f, iterations);
  std::copy(f.app.begin(), f.app.end(), app);
  std::copy(f.er.begin(), f.er.begin() + (size_t)L.edges() * z, edge_r);
  std::copy(f.hard.begin(), f.hard.end(), hard);
  return used;
}

// Median single-threaded decode time (ns) of the reference's own int8 benchmark shape
// (src/bin/ldpc_bench_export.rs:111-215: every variable's LLR +0.5 / -0.5 alternating,
// quantized at the default scale, no 5G prologue, a fixed iteration count that never
// converges), over `reps` decodes of one preallocated frame on the calling thread.
double cpb_bench_shape_ns(int bg, int z, int beta_q, int app_clamp, const int16_t* app0, int iterations,
                         int reps, int* iters_used) {
  Layout L;
  if (!make_layout(bg, z, &L) || reps < 1) return -1.0;
  Frame f;
  init_frame(L, f);
  std::vector<double> ns;
  int used = 0;
  for (int r = 0; r < reps; ++r) {
    std::copy(app0, app0 + L.n(), f.app.begin());
    const auto t0 = std::chrono::steady_clock::now();
    used = decode_i8_avx2(L, beta_q, std::max(app_clamp, 0), f, iterations);
    const auto t1 = std::chrono::steady_clock::now();
    ns.push_back(std::chrono::duration<double, std::nano>(t1 - t0).count());
  }
  if (iters_used) *iters_used = used;
  std::sort(ns.begin(), ns.end());
  return ns[ns.size() / 2];
}

// Decodes `count` codewords (int8 channel rows, variables [llr_offset, n)) through
// the restated LdpcPipeline with `workers` spinning worker threads.  Writes the
// iterations used per codeword and the packed hard bits of the first `hard_bits`
// variables (LSB-first words).  Returns the wall seconds from the first submit to
// the last receive, or -1 on invalid arguments.
double cpb_pipeline_i8(int bg, int z, int beta_q, int app_clamp, const int8_t* llr, long long stride,
                       int llr_offset, long long n_filler, long long count, int iterations, int workers,
                       int32_t* iters_out, uint32_t* hard_packed, int hard_bits, long long words_stride) {
  Layout L;
  if (!make_layout(bg, z, &L) || workers < 1 || workers > 256) return -1.0;
  const int C = std::max(app_clamp, 0);
  const int kPool = std::max(16, 2 * workers);
  std::vector<Frame> pool(kPool);
  for (auto& f : pool) init_frame(L, f);
  std::vector<Spsc> work(workers), done(workers);
  std::atomic<bool> stop{false};
  std::vector<std::thread> th;
  for (int w = 0; w < workers; ++w)
    th.emplace_back([&, w]() {
      pin(w);
      int idx;
      for (;;) {
        if (work[w].pop(&idx)) {
          Frame& f = pool[idx];
          f.iters = decode_i8_avx2(L, beta_q, C, f, iterations);
          while (!done[w].push(idx)) std::this_thread::yield();
        } else if (stop.load(std::memory_order_acquire)) {
          break;
        } else {
          _mm_pause();
        }
      }
    });
  std::vector<int> free_list;
  for (int i = kPool - 1; i >= 0; --i) free_list.push_back(i);
  std::vector<int> outstanding(workers, 0);
  size_t cursor = 0;
  long long next = 0, received = 0;
  const auto t0 = std::chrono::steady_clock::now();
  while (received < count) {
    while (next < count && !free_list.empty()) {
      const int w = pick_worker(outstanding, cursor);
      if (outstanding[w] >= 16) break;
      const int idx = free_list.back();
      free_list.pop_back();
      Frame& f = pool[idx];
      f.tag = next;
      load_frame(L, f, llr + next * stride, llr_offset, n_filler, C);
      while (!work[w].push(idx)) _mm_pause();
      ++outstanding[w];
      ++cursor;
      ++next;
    }
    for (int w = 0; w < workers; ++w) {
      int idx;
      while (done[w].pop(&idx)) {
        Frame& f = pool[idx];
        if (iters_out) iters_out[f.tag] = f.iters;
        if (hard_packed) {
          uint32_t* dst = hard_packed + f.tag * words_stride;
          for (int wd = 0; wd < (hard_bits + 31) / 32; ++wd) {
            uint32_t m = 0;
            for (int b = 0; b < 32 && wd * 32 + b < hard_bits; ++b) m |= (uint32_t)f.hard[wd * 32 + b] << b;
            dst[wd] = m;
          }
        }
        --outstanding[w];
        free_list.push_back(idx);
        ++received;
      }
    }
  }
  const auto t1 = std::chrono::steady_clock::now();
  stop.store(true, std::memory_order_release);
  for (auto& t : th) t.join();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
