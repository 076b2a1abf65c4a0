// Layered description of an expanded QC-LDPC code (host side).
//
// Mirrors syndrome's QcLdpcParams (src/qc_ldpc.rs:233-260): a base graph with m_b
// block rows (layers) and n_b block columns, each non-null block an identity
// matrix cyclically shifted by `shift` at lifting size Z.  Edges are grouped by
// layer (CSR: layer_off[m_b + 1]) in the order the reference's build_layout
// (src/qc_ldpc.rs:281-319) produces; inside a layer the order does not change
// any decoder output because every column appears at most once per layer.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace syn {

enum class GraphKind : int { kNrBg1 = 0, kNrBg2 = 1, kRaw = 2 };

struct Graph {
  GraphKind kind = GraphKind::kRaw;
  int z = 0;        // lifting size
  int mb = 0;       // block rows (layers)
  int nb = 0;       // block columns
  int kb = 0;       // systematic block columns (nb - mb)
  int maxdeg = 0;   // largest layer degree
  std::vector<int> layer_off;  // [mb + 1]
  std::vector<int> cols;       // [E] column block per edge
  std::vector<int> shifts;     // [E] cyclic shift per edge, already < z

  int edges() const { return (int)cols.size(); }
  long long n() const { return (long long)nb * z; }   // variable nodes
  long long m() const { return (long long)mb * z; }   // check nodes
  long long k() const { return (long long)kb * z; }   // 5G information bits incl. filler
  long long edge_buffer() const { return (long long)edges() * z; }
  long long layer_buffer() const { return (long long)maxdeg * z; }
};

// 3GPP TS 38.212 Table 5.3.2-1: lifting-size set index of z, or -1.
int lifting_set_index(int z);

// Expands BG1 (bg = 0) or BG2 (bg = 1) at lifting size z (src/qc_ldpc.rs:339-366).
// Returns false (and leaves g untouched) when z is not a 3GPP lifting size.
bool build_nr_graph(int bg, int z, Graph* g);

// Builds a graph from literal (row, col, shift) triples (src/qc_ldpc.rs:412-455).
// Returns false with a message when z is outside 1..384 or a triple is out of range.
bool build_raw_graph(const int* rows, const int* cols, const int* shifts, int n_edges, int mb,
                     int nb, int z, Graph* g, std::string* err);

// One of the twelve IEEE 802.11 matrices (src/wifi_ldpc_tables.rs:339-453).
bool build_wifi_graph(int z, int rate_num, int rate_den, Graph* g);

}  // namespace syn
