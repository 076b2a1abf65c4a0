/* Record layouts of the base-graph tables in base_graph_tables.inc.
 *
 * 5G NR base graphs (3GPP TS 38.212 Tables 5.3.2-2/5.3.2-3): one record per
 * non-null block (row, col) holding the raw shift value for each of the eight
 * lifting-size sets iLS = 0..7.  The cyclic shift used at lifting size Z is
 * v[iLS(Z)] mod Z (syndrome src/qc_ldpc.rs:135-140).
 *
 * IEEE 802.11 matrices: literal (row, col, shift) triples, shift already < Z
 * (syndrome src/wifi_ldpc_tables.rs:109-328).
 */
#ifndef SYNDROME_B200_GRAPH_TABLES_H
#define SYNDROME_B200_GRAPH_TABLES_H

typedef struct {
  unsigned char r;
  unsigned char c;
  short v[8];
} syn_bg_entry_t;

typedef struct {
  unsigned char r;
  unsigned char c;
  short s;
} syn_raw_edge_t;

typedef struct {
  int z;
  int rate_num;
  int rate_den;
  int row_blocks;
  int col_blocks;
  int edge_count;
  const syn_raw_edge_t* edges;
} syn_wifi_matrix_t;

#endif
