// 5G NR transport-block (DL-SCH) host logic: segmentation, CRC, the rate-matching
// walk and the transport-block encoder.
//
// Follows syndrome's segmentation.rs:75-400 (compute_segmentation, segment),
// crc.rs:65-350 (CRC-24A / CRC-24B: MSB-first register, zero initial value, no final
// XOR), rate_matching.rs:72-700 (circular buffer of N - 2Z bits, k0 = j * Z per RV,
// filler positions skipped, Qm-row interleaving) and transport_block.rs:203-340
// (DlSchEncoder: TB CRC, segmentation, LDPC encoding, rate matching, E per code block
// = floor(G / C / Qm) * Qm).
//
// The rate-matching positions come from a closed form instead of the reference's
// step-by-step walk: the non-filler positions of the circular buffer, taken in
// buffer order, form a cycle of M = Ncb - (filler window) positions, and the walk
// visits them in order starting at the first one at or after k0.  Selection k is
// compressed position (c0 + k) mod M.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "encoder.h"

namespace syn {

constexpr long long kMaxTbBits = 1277992;  // segmentation.rs MAX_TB_SIZE_BITS
constexpr uint32_t kCrc24A = 0x864CFBu;
constexpr uint32_t kCrc24B = 0x800063u;

struct TbParams {
  int bg = 0;            // 0 = BG1, 1 = BG2
  int z = 0;             // lifting size
  int c = 0;             // code blocks
  long long b = 0;       // A + 24 (TB with its CRC)
  int k_prime = 0;       // bits per code block before filler (CB CRC included)
  int k = 0;             // systematic bits seen by the encoder (k_b * Z)
  int ncb = 0;           // circular buffer length n_b * Z = N - 2Z
  int n_filler = 0;      // K - K'
  bool has_cb_crc = false;
  int payload = 0;       // TB bits carried per code block (K' - 24 with CB CRC, else K')
};

// BG1 = 0, BG2 = 1 (segmentation.rs select_base_graph).
int select_base_graph(long long a, float rate);
// compute_segmentation; false with err for a = 0 or a above kMaxTbBits.
bool compute_segmentation(long long a, float rate, TbParams* p, std::string* err);

// CRC of n bits (one per byte, LSB used) with the 24-bit polynomial poly.
uint32_t crc24_bits(const uint8_t* bits, long long n, uint32_t poly);

// The rate-matching walk of one code block shape and RV.
struct RmWalk {
  int ncb = 0;   // circular buffer length
  int fs = 0;    // filler window [fs, fe) in buffer coordinates
  int fe = 0;
  int m = 0;     // non-filler positions (cycle length)
  int c0 = 0;    // compressed position of the first selection (may equal m: wraps first)
  int k0 = 0;    // RV start position
};
// k0 = {0, 17, 33, 56} * Z (BG1) / {0, 13, 25, 43} * Z (BG2) for rv 0..3.
RmWalk rm_walk(int bg, int z, int rv, int n_filler);
// Buffer position (0 .. ncb-1) of selection k.
inline int rm_position(const RmWalk& w, long long k) {
  const int c = (int)((w.c0 + k) % w.m);
  return c < w.fs ? c : c + (w.fe - w.fs);
}
// Selection index of received (interleaved) bit q for Qm with E / Qm rows.
inline long long rm_selection(long long q, int qm, long long rows) { return (q % rows) * qm + q / rows; }
// True when the reference's walk, which gives up after 2 * ncb steps, selects all
// e bits (this implementation rejects larger e instead of leaving bits unset).
bool rm_walk_covers(const RmWalk& w, long long e);

// DlSchEncoder: tb_size bits (one per byte) -> G' = C * E bits for redundancy version rv.
class TbEncoder {
 public:
  bool init(long long tb_size, float rate, int qm, long long g, std::string* err);
  const TbParams& params() const { return p_; }
  long long e_per_cb() const { return e_; }
  long long output_bits() const { return e_ * p_.c; }
  int qm() const { return qm_; }
  // tb: tb_size bits; out: output_bits() bits.  Returns false for rv > 3.
  bool encode(const uint8_t* tb, int rv, uint8_t* out) const;

 private:
  TbParams p_;
  long long tb_size_ = 0, e_ = 0;
  int qm_ = 1;
  Encoder enc_;
};

}  // namespace syn
