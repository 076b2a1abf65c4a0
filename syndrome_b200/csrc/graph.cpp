#include "graph.h"

#include <algorithm>

#include "graph_tables.h"
#include "base_graph_tables.inc"

namespace syn {

namespace {

// 3GPP TS 38.212 Table 5.3.2-1 (syndrome src/qc_ldpc.rs:93-122).
const int kSets[8][8] = {{2, 4, 8, 16, 32, 64, 128, 256},   {3, 6, 12, 24, 48, 96, 192, 384},
                         {5, 10, 20, 40, 80, 160, 320, -1}, {7, 14, 28, 56, 112, 224, -1, -1},
                         {9, 18, 36, 72, 144, 288, -1, -1}, {11, 22, 44, 88, 176, 352, -1, -1},
                         {13, 26, 52, 104, 208, -1, -1, -1}, {15, 30, 60, 120, 240, -1, -1, -1}};

// CSR grouping by layer, keeping the input order within a layer.
void group_by_layer(const std::vector<int>& r, const std::vector<int>& c,
                    const std::vector<int>& s, Graph* g) {
  std::vector<int> deg(g->mb, 0);
  for (int x : r) ++deg[x];
  g->layer_off.assign(g->mb + 1, 0);
  for (int i = 0; i < g->mb; ++i) g->layer_off[i + 1] = g->layer_off[i] + deg[i];
  g->cols.assign(r.size(), 0);
  g->shifts.assign(r.size(), 0);
  std::vector<int> cursor(g->layer_off.begin(), g->layer_off.end() - 1);
  for (size_t i = 0; i < r.size(); ++i) {
    int pos = cursor[r[i]]++;
    g->cols[pos] = c[i];
    g->shifts[pos] = s[i];
  }
  g->maxdeg = deg.empty() ? 0 : *std::max_element(deg.begin(), deg.end());
  g->kb = g->nb - g->mb;
}

}  // namespace

int lifting_set_index(int z) {
  if (z <= 0) return -1;
  for (int s = 0; s < 8; ++s)
    for (int j = 0; j < 8; ++j)
      if (kSets[s][j] == z) return s;
  return -1;
}

bool build_nr_graph(int bg, int z, Graph* g) {
  int ils = lifting_set_index(z);
  if (ils < 0 || (bg != 0 && bg != 1)) return false;
  const syn_bg_entry_t* ents = bg == 0 ? syn_bg1_entries : syn_bg2_entries;
  const int n = bg == 0 ? SYN_BG1_EDGES : SYN_BG2_EDGES;
  Graph out;
  out.kind = bg == 0 ? GraphKind::kNrBg1 : GraphKind::kNrBg2;
  out.z = z;
  out.mb = bg == 0 ? SYN_BG1_ROWS : SYN_BG2_ROWS;
  out.nb = bg == 0 ? SYN_BG1_COLS : SYN_BG2_COLS;
  std::vector<int> r(n), c(n), s(n);
  for (int i = 0; i < n; ++i) {
    r[i] = ents[i].r;
    c[i] = ents[i].c;
    s[i] = ents[i].v[ils] % z;  // table values are non-negative
  }
  group_by_layer(r, c, s, &out);
  *g = std::move(out);
  return true;
}

bool build_raw_graph(const int* rows, const int* cols, const int* shifts, int n_edges, int mb,
                     int nb, int z, Graph* g, std::string* err) {
  if (z <= 0 || z > 384) {
    if (err) *err = "z must be in 1..=384";
    return false;
  }
  if (mb <= 0 || nb <= mb || mb > 255 || nb > 255 || n_edges < 0) {
    if (err) *err = "invalid block dimensions";
    return false;
  }
  for (int i = 0; i < n_edges; ++i) {
    if (rows[i] < 0 || rows[i] >= mb) {
      if (err) *err = "raw edge row_block is out of range for num_row_blocks";
      return false;
    }
    if (cols[i] < 0 || cols[i] >= nb) {
      if (err) *err = "raw edge col_block is out of range for num_col_blocks";
      return false;
    }
    if (shifts[i] < 0 || shifts[i] >= z) {
      if (err) *err = "raw edge shift must satisfy 0 <= shift < z";
      return false;
    }
  }
  Graph out;
  out.kind = GraphKind::kRaw;
  out.z = z;
  out.mb = mb;
  out.nb = nb;
  group_by_layer(std::vector<int>(rows, rows + n_edges), std::vector<int>(cols, cols + n_edges),
                 std::vector<int>(shifts, shifts + n_edges), &out);
  *g = std::move(out);
  return true;
}

bool build_wifi_graph(int z, int rate_num, int rate_den, Graph* g) {
  for (int i = 0; i < SYN_WIFI_MATRIX_COUNT; ++i) {
    const syn_wifi_matrix_t& m = syn_wifi_matrices[i];
    if (m.z != z || m.rate_num != rate_num || m.rate_den != rate_den) continue;
    std::vector<int> r(m.edge_count), c(m.edge_count), s(m.edge_count);
    for (int j = 0; j < m.edge_count; ++j) {
      r[j] = m.edges[j].r;
      c[j] = m.edges[j].c;
      s[j] = m.edges[j].s;
    }
    return build_raw_graph(r.data(), c.data(), s.data(), m.edge_count, m.row_blocks, m.col_blocks,
                           m.z, g, nullptr);
  }
  return false;
}

}  // namespace syn
