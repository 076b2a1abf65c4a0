// Transport-block host logic (see tb.h).
#include "tb.h"

#include <algorithm>
#include <array>

#include "graph.h"

namespace syn {

namespace {

const int kValidZ[] = {2,  3,  4,  5,  6,  7,  8,  9,   10,  11,  12,  13,  14,  15,  16,  18,  20,
                       22, 24, 26, 28, 30, 32, 36, 40,  44,  48,  52,  56,  60,  64,  72,  80,  88,
                       96, 104, 112, 120, 128, 144, 160, 176, 192, 208, 224, 240, 256, 288, 320, 352, 384};

const int kRvK0[2][4] = {{0, 17, 33, 56}, {0, 13, 25, 43}};

// Byte-at-a-time CRC table of a 24-bit polynomial (MSB-first register).
struct CrcTable {
  std::array<uint32_t, 256> t{};
  explicit CrcTable(uint32_t poly) {
    for (int i = 0; i < 256; ++i) {
      uint32_t reg = (uint32_t)i << 16;
      for (int b = 0; b < 8; ++b) reg = (reg & 0x800000u) ? ((reg << 1) ^ poly) & 0xFFFFFFu : (reg << 1) & 0xFFFFFFu;
      t[i] = reg;
    }
  }
};

const CrcTable& table_for(uint32_t poly) {
  static const CrcTable a(kCrc24A), b(kCrc24B);
  return poly == kCrc24A ? a : b;
}

}  // namespace

int select_base_graph(long long a, float rate) {
  return (a <= 292 || (a <= 3824 && rate <= 0.67f) || rate <= 0.25f) ? 1 : 0;
}

bool compute_segmentation(long long a, float rate, TbParams* p, std::string* err) {
  auto fail = [&](const char* m) {
    if (err) *err = m;
    return false;
  };
  if (a <= 0) return fail("transport block size must be > 0");
  if (a > kMaxTbBits) return fail("transport block size exceeds the 3GPP maximum (1,277,992 bits)");
  TbParams q;
  q.bg = select_base_graph(a, rate);
  const long long k_cb = q.bg == 0 ? 8448 : 3840;
  const int n_b = q.bg == 0 ? 66 : 50;
  q.b = a + 24;
  long long c = 1, l = 0;
  if (q.b > k_cb) {
    c = (q.b + (k_cb - 24) - 1) / (k_cb - 24);
    l = 24;
  }
  const long long b_prime = q.b + c * l;
  const long long k_prime = (b_prime + c - 1) / c;
  int k_b = 22;
  if (q.bg == 1) k_b = q.b > 640 ? 10 : q.b > 560 ? 9 : q.b > 192 ? 8 : 6;
  int z = 0;
  for (int v : kValidZ)
    if ((long long)k_b * v >= k_prime) {
      z = v;
      break;
    }
  if (z == 0) return fail("K' too large: no valid 3GPP lifting size exists");
  q.z = z;
  q.c = (int)c;
  q.k_prime = (int)k_prime;
  q.k = (q.bg == 0 ? 22 : 10) * z;
  q.ncb = n_b * z;
  q.n_filler = q.k - q.k_prime;
  q.has_cb_crc = l > 0;
  q.payload = q.has_cb_crc ? q.k_prime - 24 : q.k_prime;
  *p = q;
  return true;
}

uint32_t crc24_bits(const uint8_t* bits, long long n, uint32_t poly) {
  const CrcTable& t = table_for(poly);
  uint32_t reg = 0;
  long long i = 0;
  for (; i + 8 <= n; i += 8) {
    uint32_t byte = 0;
    for (int k = 0; k < 8; ++k) byte = (byte << 1) | (bits[i + k] & 1u);
    reg = ((reg << 8) & 0xFFFFFFu) ^ t.t[((reg >> 16) ^ byte) & 0xFFu];
  }
  for (; i < n; ++i) {
    const uint32_t fb = ((reg >> 23) ^ bits[i]) & 1u;
    reg = (reg << 1) & 0xFFFFFFu;
    if (fb) reg ^= poly;
  }
  return reg;
}

RmWalk rm_walk(int bg, int z, int rv, int n_filler) {
  RmWalk w;
  const int n_b = bg == 0 ? 66 : 50, k_b = bg == 0 ? 22 : 10;
  w.ncb = n_b * z;
  const int k = k_b * z, kp = std::max(k - n_filler, 0);
  w.fs = std::max(kp - 2 * z, 0);
  w.fe = std::max(k - 2 * z, 0);
  if (w.fe < w.fs) w.fe = w.fs;
  w.m = w.ncb - (w.fe - w.fs);
  w.k0 = kRvK0[bg][rv & 3] * z;
  // first non-filler position at or after k0, in compressed coordinates (left
  // unreduced: a window reaching the end of the buffer makes the walk wrap first)
  if (w.k0 < w.fs)
    w.c0 = w.k0;
  else if (w.k0 < w.fe)
    w.c0 = w.fs;
  else
    w.c0 = w.k0 - (w.fe - w.fs);
  return w;
}

bool rm_walk_covers(const RmWalk& w, long long e) {
  if (e <= 1) return true;
  // step index of selection e - 2 (the reference stops once a selection lands past 2 * ncb - 1)
  const long long t = w.c0 + e - 2;
  const long long lap = t / w.m;
  const long long j = lap * w.ncb + rm_position(w, e - 2) - w.k0;
  return j < 2LL * w.ncb;
}

bool TbEncoder::init(long long tb_size, float rate, int qm, long long g, std::string* err) {
  auto fail = [&](const char* m) {
    if (err) *err = m;
    return false;
  };
  if (tb_size <= 0) return fail("tb_size must be > 0");
  if (qm <= 0) return fail("qm must be >= 1");
  if (g <= 0 || g % qm != 0) return fail("G must be > 0 and divisible by Qm");
  TbParams p;
  if (!compute_segmentation(tb_size, rate, &p, err)) return false;
  const long long e = (g / p.c / qm) * qm;
  if (e <= 0) return fail("G too small: no bits per code block");
  Graph gr;
  if (!build_nr_graph(p.bg, p.z, &gr) || !enc_.init(gr)) return fail("internal: cannot build the 5G NR encoder");
  for (int rv = 0; rv < 4; ++rv)
    if (!rm_walk_covers(rm_walk(p.bg, p.z, rv, p.n_filler), e))
      return fail("E per code block exceeds the rate-matching walk (code rate below the supported range)");
  p_ = p;
  tb_size_ = tb_size;
  e_ = e;
  qm_ = qm;
  return true;
}

bool TbEncoder::encode(const uint8_t* tb, int rv, uint8_t* out) const {
  if (rv < 0 || rv > 3) return false;
  const TbParams& p = p_;
  std::vector<uint8_t> tbc(tb, tb + tb_size_);
  const uint32_t crc = crc24_bits(tbc.data(), tb_size_, kCrc24A);
  for (int s = 23; s >= 0; --s) tbc.push_back((crc >> s) & 1u);
  const int n = p.ncb + 2 * p.z;
  std::vector<uint8_t> info(p.k), cw(n);
  const RmWalk w = rm_walk(p.bg, p.z, rv, p.n_filler);
  const long long rows = e_ / qm_;
  for (int ci = 0; ci < p.c; ++ci) {
    std::fill(info.begin(), info.end(), 0);
    const long long start = (long long)ci * p.payload;
    const long long end = std::min<long long>(start + p.payload, p.b);
    for (long long i = start; i < end; ++i) info[i - start] = tbc[i] & 1u;
    if (p.has_cb_crc) {
      const uint32_t cc = crc24_bits(info.data(), p.payload, kCrc24B);
      for (int s = 0; s < 24; ++s) info[p.payload + s] = (cc >> (23 - s)) & 1u;
    }
    enc_.encode(info.data(), cw.data());
    uint8_t* o = out + (long long)ci * e_;
    for (long long q = 0; q < e_; ++q) o[q] = cw[2 * p.z + rm_position(w, rm_selection(q, qm_, rows))];
  }
  return true;
}

}  // namespace syn
