// Oracle: a CPU restatement of syndrome's QC-LDPC path, used ONLY as a checker.
//
// This file is test infrastructure.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load the library built from it; the decoder
// library (syndrome_b200/) never links or calls it.
//
// Every function restates the reference's algorithm with the reference's own
// operation order so that results are bit-identical:
//   * layered CSR layout        syndrome src/qc_ldpc.rs:116-140, 281-319, 339-455
//   * f32 LOMS decode           src/qc_ldpc.rs:962-1221 (scalar branch :1146-1205)
//   * f32 syndrome check        src/qc_ldpc.rs:1231-1252
//   * 5G f32 prologue           src/qc_ldpc.rs:711-732
//   * int8/int16 LOMS decode    src/qc_ldpc.rs:1530-1758 (scalar branch :1670-1745)
//   * int16 syndrome check      src/qc_ldpc.rs:1766-1787
//   * 5G int8 prologue          src/qc_ldpc.rs:1486-1523
//   * quantizer / beta_q        src/quantize.rs:148-155, 298-305, 331-343 (+float_ext.rs round)
//   * Wi-Fi shortening          src/wifi_rate_matching.rs:88-132, 163-192, 267-302
//   * encoder                   src/qc_ldpc.rs:2166-2727 (sparse core solve) and :1996-2125 (dense)
//   * AWGN channel              src/channel_sim.rs:61-241
//   * DL-SCH transport blocks   segmentation.rs:75-400, crc.rs:65-350, rate_matching.rs:72-700,
//                               harq.rs:77-195, transport_block.rs:203-1053 (the decoder chain
//                               with the int8 decode: HARQ f32 sum -> quantize -> decode_5g_i8)
// Built with -ffp-contract=off and without -ffast-math so IEEE f32 operations
// happen exactly as written.
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>
#include <algorithm>

#include "../syndrome_b200/csrc/graph_tables.h"
#include "../syndrome_b200/csrc/base_graph_tables.inc"

namespace {

struct Params {
  int bg;  // 0 = BG1, 1 = BG2, -1 = raw edge list
  int z;
  int mb;
  int nb;
  std::vector<int> layer_off;
  std::vector<int> cols;
  std::vector<int> shifts;
  int maxdeg;
  // encoder state
  int enc_kind;  // 0 unbuilt, 1 sparse, 2 dense, -1 singular
  int sp[9];     // sparse core layout (see derive_core)
  std::vector<std::vector<uint64_t>> gen;  // dense generator rows (m rows of k bits)
};

// syndrome src/qc_ldpc.rs:93-122 (Table 5.3.2-1 lifting sets).
const int kLiftingSets[8][8] = {
    {2, 4, 8, 16, 32, 64, 128, 256}, {3, 6, 12, 24, 48, 96, 192, 384},
    {5, 10, 20, 40, 80, 160, 320, 0}, {7, 14, 28, 56, 112, 224, 0, 0},
    {9, 18, 36, 72, 144, 288, 0, 0},  {11, 22, 44, 88, 176, 352, 0, 0},
    {13, 26, 52, 104, 208, 0, 0, 0},  {15, 30, 60, 120, 240, 0, 0, 0}};

int ils_for_z(int z) {
  for (int s = 0; s < 8; ++s)
    for (int j = 0; j < 8; ++j)
      if (kLiftingSets[s][j] == z && z != 0) return s;
  return -1;
}

// syndrome src/qc_ldpc.rs:281-319: group edges by row, keeping entry order inside a row.
void build_layout(Params* p, const std::vector<int>& r, const std::vector<int>& c,
                  const std::vector<int>& s) {
  std::vector<int> deg(p->mb, 0);
  for (int x : r) deg[x]++;
  p->layer_off.assign(p->mb + 1, 0);
  for (int i = 0; i < p->mb; ++i) p->layer_off[i + 1] = p->layer_off[i] + deg[i];
  int total = p->layer_off[p->mb];
  p->cols.assign(total, 0);
  p->shifts.assign(total, 0);
  std::vector<int> fill(p->mb, 0);
  for (size_t i = 0; i < r.size(); ++i) {
    int pos = p->layer_off[r[i]] + fill[r[i]]++;
    p->cols[pos] = c[i];
    p->shifts[pos] = s[i];
  }
  p->maxdeg = 0;
  for (int d : deg) p->maxdeg = std::max(p->maxdeg, d);
}

inline int rot(int zi, int shift, int z) {
  int s = zi + shift;
  return s >= z ? s - z : s;
}

bool syndrome_ok_f32(const Params* p, const float* llr) {
  const int z = p->z;
  for (int l = 0; l < p->mb; ++l) {
    for (int zi = 0; zi < z; ++zi) {
      unsigned par = 0;
      for (int e = p->layer_off[l]; e < p->layer_off[l + 1]; ++e)
        par ^= (llr[p->cols[e] * z + rot(zi, p->shifts[e], z)] < 0.0f) ? 1u : 0u;
      if (par) return false;
    }
  }
  return true;
}

bool syndrome_ok_i16(const Params* p, const int16_t* app) {
  const int z = p->z;
  for (int l = 0; l < p->mb; ++l) {
    for (int zi = 0; zi < z; ++zi) {
      unsigned par = 0;
      for (int e = p->layer_off[l]; e < p->layer_off[l + 1]; ++e)
        par ^= (app[p->cols[e] * z + rot(zi, p->shifts[e], z)] < 0) ? 1u : 0u;
      if (par) return false;
    }
  }
  return true;
}

inline uint32_t f2u(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}
inline float u2f(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}

// ---------------------------------------------------------------- encoder --
// syndrome src/qc_ldpc.rs:2129-2141 (rotl_xor_into): dst[i] ^= src[(i + shift) mod z].
void rotl_xor(uint8_t* dst, const uint8_t* src, int shift, int z) {
  for (int i = 0; i < z; ++i) dst[i] ^= src[rot(i, shift, z)];
}
void rotl_set(uint8_t* dst, const uint8_t* src, int shift, int z) {
  for (int i = 0; i < z; ++i) dst[i] = src[rot(i, shift, z)];
}

// Core parity entries (offset, shift) of a row: syndrome src/qc_ldpc.rs:2190-2205.
int core_entries(const Params* p, int row, int kb, int out[4][2]) {
  int n = 0;
  for (int e = p->layer_off[row]; e < p->layer_off[row + 1]; ++e) {
    int c = p->cols[e];
    if (c >= kb && c < kb + 4 && n < 4) {
      out[n][0] = c - kb;
      out[n][1] = p->shifts[e];
      ++n;
    }
  }
  return n;
}
int shift_for(int ent[4][2], int n, int off) {
  for (int i = 0; i < n; ++i)
    if (ent[i][0] == off) return ent[i][1];
  return -1;
}

// syndrome src/qc_ldpc.rs:2238-2318 (CoreLayout::derive).  sp[] = {p1_edge, p1_x,
// row_x_is_1, s0p2, s1p2, s1p3, s2p3, s2p4, s3p4}.
bool derive_core(const Params* p, int kb, int sp[9]) {
  if (p->mb < 4 || p->nb < kb + 4) return false;
  int r0[4][2], r1[4][2], r2[4][2], r3[4][2];
  int n0 = core_entries(p, 0, kb, r0), n1 = core_entries(p, 1, kb, r1);
  int n2 = core_entries(p, 2, kb, r2), n3 = core_entries(p, 3, kb, r3);
  if (n0 != 2 || n3 != 2) return false;
  int s0p1 = shift_for(r0, n0, 0), s0p2 = shift_for(r0, n0, 1);
  int s3p1 = shift_for(r3, n3, 0), s3p4 = shift_for(r3, n3, 3);
  if (s0p1 < 0 || s0p2 < 0 || s3p1 < 0 || s3p4 < 0 || s0p1 != s3p1) return false;
  int r1p1 = shift_for(r1, n1, 0), r2p1 = shift_for(r2, n2, 0);
  int row_x_is_1, px;
  if (r1p1 >= 0 && r2p1 < 0) {
    row_x_is_1 = 1;
    px = r1p1;
  } else if (r1p1 < 0 && r2p1 >= 0) {
    row_x_is_1 = 0;
    px = r2p1;
  } else {
    return false;
  }
  int s1p2 = shift_for(r1, n1, 1), s1p3 = shift_for(r1, n1, 2);
  int s2p3 = shift_for(r2, n2, 2), s2p4 = shift_for(r2, n2, 3);
  if (s1p2 < 0 || s1p3 < 0 || s2p3 < 0 || s2p4 < 0) return false;
  if (n1 != (row_x_is_1 ? 3 : 2) || n2 != (row_x_is_1 ? 2 : 3)) return false;
  for (int row = 4; row < p->mb; ++row) {
    int hits = 0;
    for (int e = p->layer_off[row]; e < p->layer_off[row + 1]; ++e) {
      int c = p->cols[e];
      if (c >= kb + 4) {
        ++hits;
        if (c != kb + row || p->shifts[e] != 0) return false;
      }
    }
    if (hits != 1) return false;
  }
  int v[9] = {s0p1, px, row_x_is_1, s0p2, s1p2, s1p3, s2p3, s2p4, s3p4};
  memcpy(sp, v, sizeof(v));
  return true;
}

// syndrome src/qc_ldpc.rs:2006-2085 (ParityGenerator::build): Gauss-Jordan over
// the augmented [H_p | H_s] system, parity bit i = variable k + i.
bool build_dense(Params* p) {
  const int z = p->z, mb = p->mb, nb = p->nb, kb = nb - mb;
  const int m = mb * z, k = kb * z;
  const int aug_words = (m + k + 63) / 64;
  std::vector<std::vector<uint64_t>> aug(m, std::vector<uint64_t>(aug_words, 0));
  for (int l = 0; l < mb; ++l)
    for (int e = p->layer_off[l]; e < p->layer_off[l + 1]; ++e)
      for (int zi = 0; zi < z; ++zi) {
        int row = l * z + zi;
        int var = p->cols[e] * z + (zi + p->shifts[e]) % z;
        int bit = var < k ? m + var : var - k;
        aug[row][bit >> 6] ^= 1ull << (bit & 63);
      }
  for (int col = 0; col < m; ++col) {
    int piv = -1;
    for (int r = col; r < m; ++r)
      if ((aug[r][col >> 6] >> (col & 63)) & 1) {
        piv = r;
        break;
      }
    if (piv < 0) return false;
    if (piv != col) std::swap(aug[piv], aug[col]);
    const std::vector<uint64_t> pr = aug[col];
    for (int r = 0; r < m; ++r)
      if (r != col && ((aug[r][col >> 6] >> (col & 63)) & 1))
        for (int w = 0; w < aug_words; ++w) aug[r][w] ^= pr[w];
  }
  const int gw = (k + 63) / 64;
  p->gen.assign(m, std::vector<uint64_t>(gw, 0));
  for (int i = 0; i < m; ++i)
    for (int b = 0; b < k; ++b)
      if ((aug[i][(m + b) >> 6] >> ((m + b) & 63)) & 1) p->gen[i][b >> 6] |= 1ull << (b & 63);
  return true;
}

void ensure_encoder(Params* p) {
  if (p->enc_kind != 0) return;
  const int kb = p->nb - p->mb;
  if (derive_core(p, kb, p->sp))
    p->enc_kind = 1;
  else
    p->enc_kind = build_dense(p) ? 2 : -1;
}

void lambda_row(const Params* p, int row, int kb, const uint8_t* cw, uint8_t* lam) {
  const int z = p->z;
  memset(lam, 0, z);
  for (int e = p->layer_off[row]; e < p->layer_off[row + 1]; ++e)
    if (p->cols[e] < kb) rotl_xor(lam, cw + p->cols[e] * z, p->shifts[e], z);
}

// syndrome src/qc_ldpc.rs:2620-2727 (encode_sparse).
void encode_sparse(const Params* p, uint8_t* cw) {
  const int z = p->z, kb = p->nb - p->mb, k = kb * z;
  const int* sp = p->sp;
  std::vector<uint8_t> l0(z), l1(z), l2(z), l3(z), p1(z), p2(z), p3(z), p4(z), t(z);
  lambda_row(p, 0, kb, cw, l0.data());
  lambda_row(p, 1, kb, cw, l1.data());
  lambda_row(p, 2, kb, cw, l2.data());
  lambda_row(p, 3, kb, cw, l3.data());
  auto inv = [z](int s) { return (z - s) % z; };
  for (int i = 0; i < z; ++i) t[i] = l0[i] ^ l1[i] ^ l2[i] ^ l3[i];
  rotl_set(p1.data(), t.data(), inv(sp[1]), z);
  t = l0;
  rotl_xor(t.data(), p1.data(), sp[0], z);
  rotl_set(p2.data(), t.data(), inv(sp[3]), z);
  t = l1;
  rotl_xor(t.data(), p2.data(), sp[4], z);
  if (sp[2]) rotl_xor(t.data(), p1.data(), sp[1], z);
  rotl_set(p3.data(), t.data(), inv(sp[5]), z);
  t = l2;
  rotl_xor(t.data(), p3.data(), sp[6], z);
  if (!sp[2]) rotl_xor(t.data(), p1.data(), sp[1], z);
  rotl_set(p4.data(), t.data(), inv(sp[7]), z);
  memcpy(cw + k, p1.data(), z);
  memcpy(cw + k + z, p2.data(), z);
  memcpy(cw + k + 2 * z, p3.data(), z);
  memcpy(cw + k + 3 * z, p4.data(), z);
  const uint8_t* core[4] = {p1.data(), p2.data(), p3.data(), p4.data()};
  for (int row = 4; row < p->mb; ++row) {
    std::fill(t.begin(), t.end(), 0);
    for (int e = p->layer_off[row]; e < p->layer_off[row + 1]; ++e) {
      int c = p->cols[e];
      if (c < kb)
        rotl_xor(t.data(), cw + c * z, p->shifts[e], z);
      else if (c < kb + 4)
        rotl_xor(t.data(), core[c - kb], p->shifts[e], z);
    }
    memcpy(cw + k + row * z, t.data(), z);
  }
}

// syndrome src/channel_sim.rs:61-67.
uint64_t splitmix64(uint64_t seed) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return z == 0 ? 1 : z;
}
// syndrome src/channel_sim.rs:77-89.
float next_uniform(uint64_t* st) {
  uint64_t x = *st;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  *st = x;
  uint32_t mant = (uint32_t)(x >> 41);
  return u2f(0x3F800000u | mant) - 1.0f;
}
// syndrome src/channel_sim.rs:96-103 (Box-Muller, cosine branch).
float next_gaussian(uint64_t* st) {
  float u1 = std::max(next_uniform(st), 1e-38f);
  float u2 = next_uniform(st);
  const float two_pi = 2.0f * 3.14159265358979323846f;
  return sqrtf(-2.0f * logf(u1)) * cosf(two_pi * u2);
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------ layout --
void* orc_params_5g(int bg, int z) {
  int ils = ils_for_z(z);
  if (ils < 0 || (bg != 0 && bg != 1)) return nullptr;
  const syn_bg_entry_t* ents = bg == 0 ? syn_bg1_entries : syn_bg2_entries;
  int n = bg == 0 ? SYN_BG1_EDGES : SYN_BG2_EDGES;
  Params* p = new Params();
  p->bg = bg;
  p->z = z;
  p->mb = bg == 0 ? SYN_BG1_ROWS : SYN_BG2_ROWS;
  p->nb = bg == 0 ? SYN_BG1_COLS : SYN_BG2_COLS;
  p->enc_kind = 0;
  std::vector<int> r(n), c(n), s(n);
  for (int i = 0; i < n; ++i) {
    r[i] = ents[i].r;
    c[i] = ents[i].c;
    s[i] = (int)((unsigned)ents[i].v[ils] % (unsigned)z);  // syndrome qc_ldpc.rs:135-140
  }
  build_layout(p, r, c, s);
  return p;
}

void* orc_params_raw(const int* rows, const int* cols, const int* shifts, int n, int mb, int nb,
                     int z) {
  if (z <= 0 || z > 384) return nullptr;  // syndrome qc_ldpc.rs:418-423
  for (int i = 0; i < n; ++i)
    if (rows[i] < 0 || rows[i] >= mb || cols[i] < 0 || cols[i] >= nb || shifts[i] < 0 ||
        shifts[i] >= z)
      return nullptr;
  Params* p = new Params();
  p->bg = -1;
  p->z = z;
  p->mb = mb;
  p->nb = nb;
  p->enc_kind = 0;
  build_layout(p, std::vector<int>(rows, rows + n), std::vector<int>(cols, cols + n),
               std::vector<int>(shifts, shifts + n));
  return p;
}

void* orc_params_wifi(int z, int rate_num, int rate_den) {
  for (int i = 0; i < SYN_WIFI_MATRIX_COUNT; ++i) {
    const syn_wifi_matrix_t& m = syn_wifi_matrices[i];
    if (m.z == z && m.rate_num == rate_num && m.rate_den == rate_den) {
      std::vector<int> r(m.edge_count), c(m.edge_count), s(m.edge_count);
      for (int j = 0; j < m.edge_count; ++j) {
        r[j] = m.edges[j].r;
        c[j] = m.edges[j].c;
        s[j] = m.edges[j].s;
      }
      return orc_params_raw(r.data(), c.data(), s.data(), m.edge_count, m.row_blocks,
                            m.col_blocks, m.z);
    }
  }
  return nullptr;
}

void orc_params_free(void* h) { delete static_cast<Params*>(h); }

// info[0..7] = {mb, nb, z, edges, maxdeg, N, K, M}
void orc_params_info(const void* h, int* info) {
  const Params* p = static_cast<const Params*>(h);
  info[0] = p->mb;
  info[1] = p->nb;
  info[2] = p->z;
  info[3] = (int)p->cols.size();
  info[4] = p->maxdeg;
  info[5] = p->nb * p->z;
  info[6] = (p->nb - p->mb) * p->z;
  info[7] = p->mb * p->z;
}

void orc_params_layout(const void* h, int* layer_off, int* cols, int* shifts) {
  const Params* p = static_cast<const Params*>(h);
  std::copy(p->layer_off.begin(), p->layer_off.end(), layer_off);
  std::copy(p->cols.begin(), p->cols.end(), cols);
  std::copy(p->shifts.begin(), p->shifts.end(), shifts);
}

// ------------------------------------------------------------- f32 decode --
// Returns iterations used.  trace (nullable) receives the N hard bits after every
// completed iteration, before the syndrome check (qc_ldpc.rs:1208).
long orc_decode_f32(const void* h, float beta, float* llr, float* edge_r, uint8_t* hard,
                    long iterations, uint8_t* trace) {
  const Params* p = static_cast<const Params*>(h);
  const int z = p->z;
  const long n = (long)p->nb * z;
  const long ecount = (long)p->cols.size() * z;
  for (long i = 0; i < ecount; ++i) edge_r[i] = 0.0f;
  std::vector<float> q((size_t)std::max(p->maxdeg, 1) * z), m1(z), m2(z);
  std::vector<uint32_t> sx(z);
  long used = 0;
  for (long it = 0; it < iterations; ++it) {
    ++used;
    for (int l = 0; l < p->mb; ++l) {
      const int lb = p->layer_off[l], deg = p->layer_off[l + 1] - lb;
      for (int e = 0; e < deg; ++e) {
        const int vb = p->cols[lb + e] * z, sh = p->shifts[lb + e];
        const float* r = edge_r + (long)(lb + e) * z;
        for (int zi = 0; zi < z; ++zi) q[e * z + zi] = llr[vb + rot(zi, sh, z)] - r[zi];
      }
      for (int zi = 0; zi < z; ++zi) {
        m1[zi] = FLT_MAX;
        m2[zi] = FLT_MAX;
        sx[zi] = 0;
      }
      for (int e = 0; e < deg; ++e)
        for (int zi = 0; zi < z; ++zi) {
          uint32_t b = f2u(q[e * z + zi]);
          float a = u2f(b & 0x7FFFFFFFu);
          sx[zi] ^= b & 0x80000000u;
          float mm1 = m1[zi];
          if (a <= mm1) {
            m2[zi] = mm1;
            m1[zi] = a;
          } else if (a < m2[zi]) {
            m2[zi] = a;
          }
        }
      for (int zi = 0; zi < z; ++zi) {
        if (m1[zi] == FLT_MAX) m1[zi] = 0.0f;
        if (m2[zi] == FLT_MAX) m2[zi] = m1[zi];
      }
      for (int e = 0; e < deg; ++e) {
        const int vb = p->cols[lb + e] * z, sh = p->shifts[lb + e];
        float* r = edge_r + (long)(lb + e) * z;
        for (int zi = 0; zi < z; ++zi) {
          uint32_t qb = f2u(q[e * z + zi]);
          float a = u2f(qb & 0x7FFFFFFFu);
          uint32_t sgn = sx[zi] ^ (qb & 0x80000000u);
          float mex = (a == m1[zi]) ? m2[zi] : m1[zi];
          float mag = mex - beta;
          if (mag < 0.0f) mag = 0.0f;
          float nr = u2f(f2u(mag) | sgn);
          float orr = r[zi];
          r[zi] = nr;
          float* dst = &llr[vb + rot(zi, sh, z)];
          *dst = *dst + (nr - orr);
        }
      }
    }
    if (trace)
      for (long i = 0; i < n; ++i) trace[(it)*n + i] = llr[i] < 0.0f ? 1 : 0;
    if (syndrome_ok_f32(p, llr)) break;
  }
  for (long i = 0; i < n; ++i) hard[i] = llr[i] < 0.0f ? 1 : 0;
  return used;
}

// syndrome src/qc_ldpc.rs:711-732.
void orc_init_5g_f32(const void* h, float* llr, long n_filler) {
  const Params* p = static_cast<const Params*>(h);
  const long z = p->z, k = (long)(p->nb - p->mb) * z;
  const long kp = n_filler > k ? 0 : k - n_filler;
  for (long i = kp; i < k; ++i) llr[i] = 1000000.0f;
  for (long i = 0; i < 2 * z; ++i) llr[i] = 0.0f;
}

// ------------------------------------------------------------ int8 decode --
long orc_decode_i8(const void* h, int beta_q, int app_clamp, int16_t* app, int8_t* edge_r,
                   uint8_t* hard, long iterations) {
  const Params* p = static_cast<const Params*>(h);
  const int z = p->z;
  const long n = (long)p->nb * z;
  const long ecount = (long)p->cols.size() * z;
  const int C = std::max(app_clamp, 0);
  for (long i = 0; i < ecount; ++i) edge_r[i] = 0;
  for (long i = 0; i < n; ++i) app[i] = (int16_t)std::min(std::max((int)app[i], -C), C);
  std::vector<int8_t> q((size_t)std::max(p->maxdeg, 1) * z), m1(z), m2(z);
  std::vector<uint8_t> sx(z);
  long used = 0;
  for (long it = 0; it < iterations; ++it) {
    ++used;
    for (int l = 0; l < p->mb; ++l) {
      const int lb = p->layer_off[l], deg = p->layer_off[l + 1] - lb;
      for (int e = 0; e < deg; ++e) {
        const int vb = p->cols[lb + e] * z, sh = p->shifts[lb + e];
        const int8_t* r = edge_r + (long)(lb + e) * z;
        for (int zi = 0; zi < z; ++zi) {
          int d = (int)app[vb + rot(zi, sh, z)] - (int)r[zi];
          q[e * z + zi] = (int8_t)std::min(std::max(d, -127), 127);
        }
      }
      for (int zi = 0; zi < z; ++zi) {
        m1[zi] = 127;
        m2[zi] = 127;
        sx[zi] = 0;
      }
      for (int e = 0; e < deg; ++e)
        for (int zi = 0; zi < z; ++zi) {
          int8_t qq = q[e * z + zi];
          int8_t a = (int8_t)(qq < 0 ? -qq : qq);
          sx[zi] ^= (uint8_t)qq & 0x80u;
          int8_t mm1 = m1[zi];
          m1[zi] = std::min(mm1, a);
          m2[zi] = std::min(m2[zi], std::max(mm1, a));
        }
      if (deg < 2)
        for (int zi = 0; zi < z; ++zi) {
          if (deg == 0) m1[zi] = 0;
          m2[zi] = m1[zi];
        }
      for (int e = 0; e < deg; ++e) {
        const int vb = p->cols[lb + e] * z, sh = p->shifts[lb + e];
        int8_t* r = edge_r + (long)(lb + e) * z;
        for (int zi = 0; zi < z; ++zi) {
          int8_t qq = q[e * z + zi];
          int8_t a = (int8_t)(qq < 0 ? -qq : qq);
          uint8_t sgn = sx[zi] ^ ((uint8_t)qq & 0x80u);
          int8_t mex = (a == m1[zi]) ? m2[zi] : m1[zi];
          int8_t mag = (int8_t)std::max(mex - beta_q, 0);
          int8_t neg = (int8_t)((int8_t)sgn >> 7);
          int8_t nr = (int8_t)((int8_t)(mag ^ neg) - neg);
          int8_t orr = r[zi];
          r[zi] = nr;
          int delta = (int)nr - (int)orr;
          int16_t* dst = &app[vb + rot(zi, sh, z)];
          int v = (int)*dst + delta;
          v = std::min(std::max(v, -32768), 32767);  // i16 saturating add
          *dst = (int16_t)std::min(std::max(v, -C), C);
        }
      }
    }
    if (syndrome_ok_i16(p, app)) break;
  }
  for (long i = 0; i < n; ++i) hard[i] = app[i] < 0 ? 1 : 0;
  return used;
}

// syndrome src/qc_ldpc.rs:1496-1513.
void orc_prologue_5g_i8(const void* h, int16_t* app, long n_filler, int app_clamp) {
  const Params* p = static_cast<const Params*>(h);
  const long z = p->z, k = (long)(p->nb - p->mb) * z;
  const long kp = n_filler > k ? 0 : k - n_filler;
  const int16_t fill = (int16_t)std::max(app_clamp, 0);
  for (long i = kp; i < k; ++i) app[i] = fill;
  for (long i = 0; i < 2 * z; ++i) app[i] = 0;
}

// syndrome src/quantize.rs:298-305.
int orc_beta_q(float beta, float scale) {
  float s = beta * scale;
  if (!std::isfinite(s)) return 127;
  float r = roundf(s);
  r = std::min(std::max(r, 0.0f), 127.0f);
  return (int)r;
}

// syndrome src/quantize.rs:331-343.
void orc_quantize_i16(const float* llr, int16_t* out, long n, float scale) {
  for (long i = 0; i < n; ++i) {
    float v = llr[i] * scale;
    if (std::isnan(v)) {
      out[i] = 0;
      continue;
    }
    float r = roundf(v);
    out[i] = (int16_t)(r >= 127.0f ? 127 : (r <= -127.0f ? -127 : (int)r));
  }
}

// ------------------------------------------------------------------ encode --
// Returns 0 on success, -1 if the parity part is singular.
int orc_encode(void* h, const uint8_t* info, uint8_t* cw) {
  Params* p = static_cast<Params*>(h);
  ensure_encoder(p);
  const int z = p->z, kb = p->nb - p->mb, k = kb * z, m = p->mb * z;
  for (int i = 0; i < k; ++i) cw[i] = info[i] & 1;
  if (p->enc_kind == 1) {
    encode_sparse(p, cw);
    return 0;
  }
  if (p->enc_kind != 2) return -1;
  const int gw = (k + 63) / 64;
  std::vector<uint64_t> sys(gw, 0);
  for (int j = 0; j < k; ++j)
    if (cw[j]) sys[j >> 6] |= 1ull << (j & 63);
  for (int i = 0; i < m; ++i) {
    uint64_t acc = 0;
    for (int w = 0; w < gw; ++w) acc ^= (uint64_t)__builtin_popcountll(p->gen[i][w] & sys[w]);
    cw[k + i] = (uint8_t)(acc & 1);
  }
  return 0;
}

int orc_encoder_is_sparse(void* h) {
  Params* p = static_cast<Params*>(h);
  ensure_encoder(p);
  return p->enc_kind == 1;
}

// Parity check of a hard-decision vector: 1 if H*c = 0.
int orc_check_codeword(const void* h, const uint8_t* bits) {
  const Params* p = static_cast<const Params*>(h);
  const int z = p->z;
  for (int l = 0; l < p->mb; ++l)
    for (int zi = 0; zi < z; ++zi) {
      unsigned par = 0;
      for (int e = p->layer_off[l]; e < p->layer_off[l + 1]; ++e)
        par ^= bits[p->cols[e] * z + rot(zi, p->shifts[e], z)] & 1u;
      if (par) return 0;
    }
  return 1;
}

// ----------------------------------------------------------------- channel --
// syndrome src/channel_sim.rs:139-150 and :204-221.
float orc_awgn_sigma(float ebno_db, float rate) {
  float lin = powf(10.0f, ebno_db / 10.0f);
  return sqrtf(1.0f / (2.0f * rate * lin));
}

void orc_awgn_transmit(float ebno_db, float rate, uint64_t seed, const uint8_t* bits, long n,
                       float* out) {
  uint64_t st = splitmix64(seed);
  float sigma = orc_awgn_sigma(ebno_db, rate);
  float scale = 2.0f / (sigma * sigma);
  for (long i = 0; i < n; ++i) {
    float x = bits[i] == 0 ? 1.0f : -1.0f;
    float g = next_gaussian(&st);
    float r = x + g * sigma;
    out[i] = r * scale;
  }
}

// FNV-1a over hard decisions (syndrome src/bin/ldpc_bench_export.rs:44-51).
uint64_t orc_fnv1a_hard(const uint8_t* hard, long n) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (long i = 0; i < n; ++i) {
    h ^= (uint64_t)(hard[i] & 1);
    h *= 0x00000100000001b3ull;
  }
  return h;
}

}  // extern "C"

// ------------------------------------------------------------------ DL-SCH --
// Transport-block chain, restated from syndrome segmentation.rs, crc.rs,
// rate_matching.rs (the step-by-step selection walk), harq.rs and
// transport_block.rs (DlSchEncoder::encode, DlSchDecoder::decode with its
// sequential per-code-block loop).  The code-block decode is the int8 one:
// HARQ-combined f32 LLRs quantized by quantize_llr_i16, then decode_5g_i8.

struct OrcSeg {
  int bg, z, c;
  long b;
  int kp, k, n, nf, has_crc, payload;
};

static int orc_seg(long a, float r, OrcSeg* s) {
  static const int vz[] = {2,  3,  4,  5,  6,  7,  8,  9,   10,  11,  12,  13,  14,  15,  16,  18,  20,
                           22, 24, 26, 28, 30, 32, 36, 40,  44,  48,  52,  56,  60,  64,  72,  80,  88,
                           96, 104, 112, 120, 128, 144, 160, 176, 192, 208, 224, 240, 256, 288, 320, 352, 384};
  if (a == 0 || a > 1277992) return -1;
  const int bg2 = a <= 292 || (a <= 3824 && r <= 0.67f) || r <= 0.25f;
  const long k_cb = bg2 ? 3840 : 8448;
  const int n_b = bg2 ? 50 : 66;
  const long b = a + 24;
  long c = 1, l = 0;
  if (b > k_cb) {
    c = (b + (k_cb - 24) - 1) / (k_cb - 24);
    l = 24;
  }
  const long bp = b + c * l;
  const long kp = (bp + c - 1) / c;
  int kb = 22;
  if (bg2) kb = b > 640 ? 10 : (b > 560 ? 9 : (b > 192 ? 8 : 6));
  int z = 0;
  for (int v : vz)
    if ((long)kb * v >= kp) {
      z = v;
      break;
    }
  if (!z) return -1;
  s->bg = bg2 ? 1 : 0;
  s->z = z;
  s->c = (int)c;
  s->b = b;
  s->kp = (int)kp;
  s->k = (bg2 ? 10 : 22) * z;
  s->n = n_b * z;
  s->nf = s->k - s->kp;
  s->has_crc = l > 0;
  s->payload = l > 0 ? s->kp - 24 : s->kp;
  return 0;
}

// crc.rs bit_serial_step over the whole message.
static uint32_t orc_crc_bits(const uint8_t* bits, long n, uint32_t poly) {
  uint32_t reg = 0;
  for (long i = 0; i < n; ++i) {
    const uint32_t fb = ((reg >> 23) ^ (bits[i] & 1u)) & 1u;
    const uint32_t sh = (reg << 1) & 0xFFFFFFu;
    reg = fb ? sh ^ poly : sh;
  }
  return reg;
}

// rate_matching.rs selection_walk: positions of the e selected bits (0 where the
// walk's 2 * ncb guard stopped it).
static std::vector<long> orc_sel_walk(int bg, int z, int rv, int nf, long e) {
  static const int k0s[2][4] = {{0, 17, 33, 56}, {0, 13, 25, 43}};
  const long ncb = (bg == 0 ? 66L : 50L) * z, k = (bg == 0 ? 22L : 10L) * z;
  const long kp = k > nf ? k - nf : 0, tz = 2L * z;
  const long fs = kp > tz ? kp - tz : 0, fe = k > tz ? k - tz : 0;
  const long k0 = (long)k0s[bg][rv] * z;
  std::vector<long> sel(e, 0);
  long ks = 0, j = 0;
  while (ks < e) {
    const long pos = (k0 + j) % ncb;
    if (pos >= fs && pos < fe) {
      ++j;
      continue;
    }
    sel[ks] = pos;
    ++ks;
    ++j;
    if (j > 2 * ncb) break;
  }
  return sel;
}

struct OrcDlsch {
  OrcSeg s;
  long tb_size, e;
  int qm, iterations, beta_q, app_clamp;
  float scale;
  void* params;
  std::vector<std::vector<float>> acc;
  std::vector<int> tx;
  int f32 = 0;        // the reference's own f32 code-block decode (orc_dlsch_set_f32)
  float beta = 0.0f;
};

extern "C" {

// compute_segmentation: out10 = {bg, z, c, b, K', K, ncb, n_filler, has_cb_crc, payload}.
int orc_segmentation(long a, float rate, long* out10) {
  OrcSeg s;
  if (orc_seg(a, rate, &s)) return -1;
  const long v[10] = {s.bg, s.z, s.c, s.b, s.kp, s.k, s.n, s.nf, s.has_crc, s.payload};
  for (int i = 0; i < 10; ++i) out10[i] = v[i];
  return 0;
}

// kind 0 = CRC-24A (0x864CFB), 1 = CRC-24B (0x800063).
unsigned orc_crc24(const uint8_t* bits, long n, int kind) {
  return orc_crc_bits(bits, n, kind == 0 ? 0x864CFBu : 0x800063u);
}

// DlSchEncoder::new + encode: out receives C * E bits.  Returns the bit count or -1.
long orc_dlsch_encode(long tb_size, float rate, int qm, long g, int rv, const uint8_t* tb, uint8_t* out) {
  OrcSeg s;
  if (tb_size <= 0 || qm <= 0 || g <= 0 || g % qm || rv < 0 || rv > 3 || orc_seg(tb_size, rate, &s)) return -1;
  const long e = (g / s.c / qm) * qm;
  std::vector<uint8_t> tbc(tb, tb + tb_size);
  const uint32_t crc = orc_crc_bits(tbc.data(), tb_size, 0x864CFBu);
  for (int i = 23; i >= 0; --i) tbc.push_back((crc >> i) & 1u);
  void* p = orc_params_5g(s.bg, s.z);
  const long n = (long)s.n + 2L * s.z;
  std::vector<uint8_t> info(s.k), cw(n), ebuf(e), tmp(e);
  const std::vector<long> sel = orc_sel_walk(s.bg, s.z, rv, s.nf, e);
  for (int ci = 0; ci < s.c; ++ci) {
    std::vector<uint8_t> cb;
    const long start = (long)ci * s.payload, end = std::min(start + s.payload, s.b);
    for (long i = start; i < end; ++i) cb.push_back(tbc[i]);
    cb.resize(s.payload, 0);
    if (s.has_crc) {
      const uint32_t cc = orc_crc_bits(cb.data(), (long)cb.size(), 0x800063u);
      for (int i = 23; i >= 0; --i) cb.push_back((cc >> i) & 1u);
    }
    std::fill(info.begin(), info.end(), 0);
    std::copy(cb.begin(), cb.end(), info.begin());
    orc_encode(p, info.data(), cw.data());
    for (long ks = 0; ks < e; ++ks) {
      const long idx = sel[ks] + 2L * s.z;
      ebuf[ks] = idx < n ? cw[idx] : 0;
    }
    // rate_matching.rs interleave: out[col * rows + row] = e[row * qm + col]
    const long rows = e / qm;
    for (int col = 0; col < qm; ++col)
      for (long row = 0; row < rows; ++row) tmp[col * rows + row] = ebuf[row * qm + col];
    std::copy(tmp.begin(), tmp.end(), out + (long)ci * e);
  }
  orc_params_free(p);
  return (long)s.c * e;
}

void* orc_dlsch_decoder_new(long tb_size, float rate, int qm, long g, int iterations, int beta_q, float scale,
                            int app_clamp) {
  OrcSeg s;
  if (tb_size <= 0 || qm <= 0 || g <= 0 || g % qm || orc_seg(tb_size, rate, &s)) return nullptr;
  OrcDlsch* d = new OrcDlsch();
  d->s = s;
  d->tb_size = tb_size;
  d->e = (g / s.c / qm) * qm;
  d->qm = qm;
  d->iterations = iterations;
  d->beta_q = beta_q;
  d->scale = scale;
  d->app_clamp = app_clamp;
  d->params = orc_params_5g(s.bg, s.z);
  d->acc.assign(s.c, std::vector<float>(s.n, 0.0f));
  d->tx.assign(s.c, 0);
  return d;
}

void orc_dlsch_decoder_free(void* h) {
  OrcDlsch* d = static_cast<OrcDlsch*>(h);
  if (!d) return;
  orc_params_free(d->params);
  delete d;
}

// DlSchDecoder::decode.  report4 = {crc_ok, max_iters_used, harq_tx_count, C};
// cb_crc[C]; tb_out[tb_size] is written only when the CRCs pass; llr_out (nullable)
// receives the quantized int8 decoder input of each code block (C x ncb, variables
// 2Z..N); iters_out (nullable) the iterations of each code block.
int orc_dlsch_decode(void* h, const float* rx, int rv, uint8_t* tb_out, int* report4, uint8_t* cb_crc,
                     int8_t* llr_out, int* iters_out) {
  OrcDlsch* d = static_cast<OrcDlsch*>(h);
  const OrcSeg& s = d->s;
  const long e = d->e, z = s.z, n = (long)s.n + 2 * z;
  const int harq_tx = d->tx[0] + 1;
  // RateMatchCache::dec_idx: received bit q -> selection index (q % rows) * qm + q / rows
  const std::vector<long> sel = orc_sel_walk(s.bg, s.z, rv, s.nf, e);
  const long rows = e / d->qm;
  std::vector<uint8_t> all_info((size_t)s.c * s.payload, 0), hard(n);
  std::vector<int16_t> app(n);
  std::vector<float> llr(n);
  int max_iters = 0;
  bool all_cb = true;
  for (int ci = 0; ci < s.c; ++ci) {
    std::vector<float>& acc = d->acc[ci];
    const float* x = rx + (long)ci * e;
    for (long q = 0; q < e; ++q) {
      const long idx = sel[(q % rows) * d->qm + q / rows];
      if (idx < (long)acc.size()) acc[idx] += x[q];
    }
    d->tx[ci] += 1;
    std::fill(llr.begin(), llr.end(), 0.0f);
    std::copy(acc.begin(), acc.end(), llr.begin() + 2 * z);
    if (d->f32) {  // prepare_cb_llr + decode_layered_offset_min_sum (transport_block.rs:473-496, 555)
      orc_init_5g_f32(d->params, llr.data(), s.nf);
      std::vector<float> er((size_t)(static_cast<Params*>(d->params)->cols.size() * z));
      const long it = orc_decode_f32(d->params, d->beta, llr.data(), er.data(), hard.data(), d->iterations, nullptr);
      if (iters_out) iters_out[ci] = (int)it;
      max_iters = std::max(max_iters, (int)it);
    } else {
    orc_quantize_i16(llr.data(), app.data(), n, d->scale);
    if (llr_out)
      for (long j = 0; j < s.n; ++j) llr_out[(long)ci * s.n + j] = (int8_t)app[2 * z + j];
    orc_prologue_5g_i8(d->params, app.data(), s.nf, d->app_clamp);
    std::vector<int8_t> edge_r((size_t)(static_cast<Params*>(d->params)->cols.size() * z));
    const long it = orc_decode_i8(d->params, d->beta_q, d->app_clamp, app.data(), edge_r.data(), hard.data(),
                                  d->iterations);
    if (iters_out) iters_out[ci] = (int)it;
    max_iters = std::max(max_iters, (int)it);
    }
    bool ok = true;
    if (s.has_crc) {  // crc.rs check: payload CRC against the trailing 24 bits
      uint32_t rec = 0;
      for (int i = 0; i < 24; ++i) rec = (rec << 1) | (hard[s.kp - 24 + i] & 1u);
      ok = orc_crc_bits(hard.data(), s.kp - 24, 0x800063u) == rec;
    }
    cb_crc[ci] = ok ? 1 : 0;
    all_cb = all_cb && ok;
    std::copy(hard.begin(), hard.begin() + s.payload, all_info.begin() + (long)ci * s.payload);
  }
  const long ts = d->tb_size;
  bool tb_ok = false;
  if ((long)all_info.size() >= ts + 24) {
    uint32_t rec = 0;
    for (int i = 0; i < 24; ++i) rec = (rec << 1) | (all_info[ts + i] & 1u);
    tb_ok = orc_crc_bits(all_info.data(), ts, 0x864CFBu) == rec;
  }
  if (all_cb && tb_ok) {
    std::copy(all_info.begin(), all_info.begin() + ts, tb_out);
    for (auto& a : d->acc) std::fill(a.begin(), a.end(), 0.0f);
    std::fill(d->tx.begin(), d->tx.end(), 0);
  }
  report4[0] = all_cb && tb_ok;
  report4[1] = max_iters;
  report4[2] = harq_tx;
  report4[3] = s.c;
  return 0;
}

// Switches the decoder to the f32 code-block decode with offset beta (the reference's
// DlSchDecoder, transport_block.rs:829-1053); llr_out is not written then.
void orc_dlsch_set_f32(void* h, float beta) {
  OrcDlsch* d = static_cast<OrcDlsch*>(h);
  d->f32 = 1;
  d->beta = beta;
}

void orc_dlsch_flush(void* h) {
  OrcDlsch* d = static_cast<OrcDlsch*>(h);
  for (auto& a : d->acc) std::fill(a.begin(), a.end(), 0.0f);
  std::fill(d->tx.begin(), d->tx.end(), 0);
}

}  // extern "C"

// ----------------------------------------------- Wi-Fi shortening / puncturing --
// src/wifi_rate_matching.rs: shortening_and_puncture_counts :88-132, encode_shortened
// :163-192, decode_shortened :267-302 (known-zero LLR 1e6 :58).
extern "C" {

// out2 = {n_shrt, n_punc}; returns 0, or -1 for the reference's InvalidParam cases.
int orc_wifi_counts(long k, long n, long payload, long target, long* out2) {
  if (n < k || payload > k || target < payload) return -1;
  const long shrt = k - payload, max_coded = n - shrt;
  if (target > max_coded) return -1;
  out2[0] = shrt;
  out2[1] = max_coded - target;
  return 0;
}

int orc_wifi_encode_shortened(void* h, const uint8_t* payload, long payload_bits, long target, uint8_t* out) {
  Params* p = static_cast<Params*>(h);
  const long z = p->z, n = (long)p->nb * z, k = (long)(p->nb - p->mb) * z;
  long c[2];
  if (orc_wifi_counts(k, n, payload_bits, target, c) != 0) return -1;
  std::vector<uint8_t> info((size_t)k, 0), cw((size_t)n, 0);
  for (long i = 0; i < payload_bits; ++i) info[(size_t)i] = payload[i];
  if (orc_encode(h, info.data(), cw.data()) != 0) return -1;
  const long par = (n - k) - c[1];
  for (long i = 0; i < payload_bits; ++i) out[i] = payload[i];
  for (long i = 0; i < par; ++i) out[payload_bits + i] = cw[(size_t)(k + i)];
  return 0;
}

// Rebuilds codeword_llr[N] from rx[target] and decodes it (f32 LOMS, in place).
// Returns the iterations used, or -1 for invalid counts.
long orc_wifi_decode_shortened(const void* h, float beta, long payload_bits, const float* rx, long target,
                               float* codeword_llr, float* edge_r, uint8_t* hard, long iterations) {
  const Params* p = static_cast<const Params*>(h);
  const long z = p->z, n = (long)p->nb * z, k = n - (long)p->mb * z;
  long c[2];
  if (orc_wifi_counts(k, n, payload_bits, target, c) != 0) return -1;
  const long par = (n - k) - c[1];
  for (long i = 0; i < payload_bits; ++i) codeword_llr[i] = rx[i];
  for (long i = payload_bits; i < k; ++i) codeword_llr[i] = 1000000.0f;
  for (long i = 0; i < par; ++i) codeword_llr[k + i] = rx[payload_bits + i];
  for (long i = k + par; i < n; ++i) codeword_llr[i] = 0.0f;
  return orc_decode_f32(h, beta, codeword_llr, edge_r, hard, iterations, nullptr);
}

}  // extern "C"

// ------------------------------------------------------------ batch helpers --
// Threaded loops over the single-codeword functions above, so that the checker and
// the CPU reference arm can cover the benchmark's batch sizes without loading the
// decoder library.  Every codeword runs the same single-threaded code as the
// per-codeword entries; threads only split the batch.

namespace {

template <class F>
void orc_parallel(long count, int threads, F&& f) {
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  threads = (int)std::min<long>(threads, std::max<long>(count, 1));
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([=, &f]() {
      for (long b = t; b < count; b += threads) f(b);
    });
  for (auto& th : pool) th.join();
}

void orc_pack(const uint8_t* hard, long bits, uint32_t* dst) {
  for (long w = 0; w < (bits + 31) / 32; ++w) {
    uint32_t m = 0;
    for (long b = 0; b < 32 && w * 32 + b < bits; ++b) m |= (uint32_t)(hard[w * 32 + b] & 1u) << b;
    dst[w] = m;
  }
}

}  // namespace

extern "C" {

// Info bits [count][K] -> codewords (orc_encode) -> BPSK/AWGN over all N bits with
// seed seeds[b] (orc_awgn_transmit) -> int8 LLRs of bits [tx_begin, N) at `scale`
// (orc_quantize_i16, which saturates at +-127) into out[b * out_stride ...].
// Returns 0, or -1 if a codeword could not be encoded.
int orc_batch_channel_i8(void* h, const uint8_t* info, long count, const float* ebno, float rate,
                         const uint64_t* seeds, float scale, long tx_begin, int8_t* out, long out_stride,
                         int threads) {
  Params* p = static_cast<Params*>(h);
  ensure_encoder(p);  // built once here, read-only in the threads
  const long n = (long)p->nb * p->z, k = (long)(p->nb - p->mb) * p->z;
  std::vector<int> rc((size_t)std::max<long>(count, 1), 0);
  orc_parallel(count, threads, [&](long b) {
    std::vector<uint8_t> cw((size_t)n);
    std::vector<float> llr((size_t)n);
    std::vector<int16_t> q((size_t)n);
    rc[(size_t)b] = orc_encode(p, info + b * k, cw.data());
    orc_awgn_transmit(ebno[b], rate, seeds[b], cw.data(), n, llr.data());
    orc_quantize_i16(llr.data(), q.data(), n, scale);
    for (long i = tx_begin; i < n; ++i) out[b * out_stride + (i - tx_begin)] = (int8_t)q[(size_t)i];
  });
  for (long b = 0; b < count; ++b)
    if (rc[(size_t)b] != 0) return -1;
  return 0;
}

// int8 decode of a batch the way the batched device API sees it: row b holds the
// int8 channel values of variables [llr_offset, N); the punctured [0, llr_offset)
// are zero; with nr_prologue the 5G prologue (orc_prologue_5g_i8: filler to
// app_clamp, the first 2Z to 0) follows.  Writes iterations, the packed hard
// decisions of the first hard_bits variables, and for the first `detail` codewords
// the final posteriors [N] and messages [E*Z].
void orc_decode_i8_batch(const void* h, int beta_q, int app_clamp, const int8_t* llr, long llr_stride,
                         long llr_offset, int nr_prologue, long n_filler, long count, long iterations,
                         int threads, int32_t* iters, uint32_t* packed, long hard_bits, long words_stride,
                         int16_t* app_out, int8_t* edge_r_out, long detail) {
  const Params* p = static_cast<const Params*>(h);
  const long n = (long)p->nb * p->z, ez = (long)p->cols.size() * p->z;
  orc_parallel(count, threads, [&](long b) {
    std::vector<int16_t> app((size_t)n, 0);
    std::vector<int8_t> er((size_t)ez);
    std::vector<uint8_t> hard((size_t)n);
    for (long i = llr_offset; i < n; ++i) app[(size_t)i] = llr[b * llr_stride + (i - llr_offset)];
    if (nr_prologue) orc_prologue_5g_i8(p, app.data(), n_filler, app_clamp);
    iters[b] = (int32_t)orc_decode_i8(p, beta_q, app_clamp, app.data(), er.data(), hard.data(), iterations);
    if (packed) orc_pack(hard.data(), hard_bits, packed + b * words_stride);
    if (b < detail) {
      if (app_out) std::copy(app.begin(), app.end(), app_out + b * n);
      if (edge_r_out) std::copy(er.begin(), er.end(), edge_r_out + b * ez);
    }
  });
}

// f32 counterpart: row b holds the f32 channel LLRs of variables [llr_offset, N);
// with nr_prologue orc_init_5g_f32 runs first.  Final posteriors of the first
// `detail` codewords go to app_out.
void orc_decode_f32_batch(const void* h, float beta, const float* llr, long llr_stride, long llr_offset,
                          int nr_prologue, long n_filler, long count, long iterations, int threads,
                          int32_t* iters, uint32_t* packed, long hard_bits, long words_stride, float* app_out,
                          long detail) {
  const Params* p = static_cast<const Params*>(h);
  const long n = (long)p->nb * p->z, ez = (long)p->cols.size() * p->z;
  orc_parallel(count, threads, [&](long b) {
    std::vector<float> app((size_t)n, 0.0f), er((size_t)ez);
    std::vector<uint8_t> hard((size_t)n);
    for (long i = llr_offset; i < n; ++i) app[(size_t)i] = llr[b * llr_stride + (i - llr_offset)];
    if (nr_prologue) orc_init_5g_f32(p, app.data(), n_filler);
    iters[b] = (int32_t)orc_decode_f32(p, beta, app.data(), er.data(), hard.data(), iterations, nullptr);
    if (packed) orc_pack(hard.data(), hard_bits, packed + b * words_stride);
    if (b < detail && app_out) std::copy(app.begin(), app.end(), app_out + b * n);
  });
}

}  // extern "C"

extern "C" {

// f32 counterpart of orc_batch_channel_i8: the channel LLRs of bits [tx_begin, N).
int orc_batch_channel_f32(void* h, const uint8_t* info, long count, const float* ebno, float rate,
                          const uint64_t* seeds, long tx_begin, float* out, long out_stride, int threads) {
  Params* p = static_cast<Params*>(h);
  ensure_encoder(p);
  const long n = (long)p->nb * p->z, k = (long)(p->nb - p->mb) * p->z;
  std::vector<int> rc((size_t)std::max<long>(count, 1), 0);
  orc_parallel(count, threads, [&](long b) {
    std::vector<uint8_t> cw((size_t)n);
    std::vector<float> llr((size_t)n);
    rc[(size_t)b] = orc_encode(p, info + b * k, cw.data());
    orc_awgn_transmit(ebno[b], rate, seeds[b], cw.data(), n, llr.data());
    for (long i = tx_begin; i < n; ++i) out[b * out_stride + (i - tx_begin)] = llr[(size_t)i];
  });
  for (long b = 0; b < count; ++b)
    if (rc[(size_t)b] != 0) return -1;
  return 0;
}

}  // extern "C"
