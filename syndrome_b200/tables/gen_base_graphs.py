"""Generate the base-graph table file used by the decoder library and by the oracle.

The tables are standard data, not an algorithm: the 5G NR BG1/BG2 shift tables of
3GPP TS 38.212 Tables 5.3.2-2/5.3.2-3 (one shift per lifting-size set iLS) and the
twelve IEEE 802.11 LDPC parity-check matrices (Z in {27, 54, 81} x R in {1/2, 2/3,
3/4, 5/6}, literal per-Z shifts). They must be identical to the ones the reference
compiles against, so this script reads them from the reference's own data files
(syndrome `data/bg_tables.json` and `src/wifi_ldpc_tables.rs`) and writes them in
this library's own C layout.  Entry order is preserved: it is the order in which
the reference's `build_layout` (src/qc_ldpc.rs:281-319) fills each layer.

Usage: python syndrome_b200/tables/gen_base_graphs.py <reference-root>
Writes syndrome_b200/csrc/base_graph_tables.inc next to the kernels.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "..", "csrc", "base_graph_tables.inc")
OUT_LAYERED = os.path.join(HERE, "..", "csrc", "nr_layered_tables.h")

WIFI_RE = re.compile(
    r"const WIFI_Z(\d+)_R(\d)_(\d)_ENTRIES: \[\(u8, u8, i16\); (\d+)\] = \[(.*?)\];", re.S)
TRIPLE_RE = re.compile(r"\(\s*(\d+)\s*,\s*(\d+)\s*,\s*(-?\d+)\s*\)")
WIFI_ROWS = {(1, 2): 12, (2, 3): 8, (3, 4): 6, (5, 6): 4}


def load_bg(ref_root):
    with open(os.path.join(ref_root, "data", "bg_tables.json")) as f:
        d = json.load(f)
    out = {}
    for name in ("bg1", "bg2"):
        g = d[name]
        ents = [(int(e["r"]), int(e["c"]), [int(v) for v in e["v"]]) for e in g["entries"]]
        assert all(len(v) == 8 for _, _, v in ents)
        out[name] = (int(g["rows"]), int(g["cols"]), ents)
    return out


def load_wifi(ref_root):
    with open(os.path.join(ref_root, "src", "wifi_ldpc_tables.rs")) as f:
        src = f.read()
    mats = []
    for m in WIFI_RE.finditer(src):
        z, rn, rd, n, body = int(m.group(1)), int(m.group(2)), int(m.group(3)), int(m.group(4)), m.group(5)
        edges = [(int(a), int(b), int(c)) for a, b, c in TRIPLE_RE.findall(body)]
        assert len(edges) == n, (z, rn, rd, len(edges), n)
        mats.append((z, rn, rd, WIFI_ROWS[(rn, rd)], 24, edges))
    assert len(mats) == 12, len(mats)
    return mats


def render(bgs, wifi):
    lines = [
        "/* Base-graph tables: 3GPP TS 38.212 BG1/BG2 (Tables 5.3.2-2/3) and the twelve",
        " * IEEE 802.11 LDPC matrices.  Generated by syndrome_b200/tables/gen_base_graphs.py;",
        " * do not edit.  Layout: see graph_tables.h. */",
        "",
    ]
    for name in ("bg1", "bg2"):
        rows, cols, ents = bgs[name]
        up = name.upper()
        lines.append(f"#define SYN_{up}_ROWS {rows}")
        lines.append(f"#define SYN_{up}_COLS {cols}")
        lines.append(f"#define SYN_{up}_EDGES {len(ents)}")
        lines.append(f"static const syn_bg_entry_t syn_{name}_entries[{len(ents)}] = {{")
        for r, c, v in ents:
            lines.append("  {%d, %d, {%s}}," % (r, c, ", ".join(str(x) for x in v)))
        lines.append("};")
        lines.append("")
    for z, rn, rd, rows, cols, edges in wifi:
        lines.append(f"static const syn_raw_edge_t syn_wifi_z{z}_r{rn}_{rd}[{len(edges)}] = {{")
        for i in range(0, len(edges), 6):
            chunk = edges[i:i + 6]
            lines.append("  " + " ".join("{%d, %d, %d}," % e for e in chunk))
        lines.append("};")
    lines.append("")
    lines.append(f"#define SYN_WIFI_MATRIX_COUNT {len(wifi)}")
    lines.append(f"static const syn_wifi_matrix_t syn_wifi_matrices[{len(wifi)}] = {{")
    for z, rn, rd, rows, cols, edges in wifi:
        lines.append(f"  {{{z}, {rn}, {rd}, {rows}, {cols}, {len(edges)}, syn_wifi_z{z}_r{rn}_{rd}}},")
    lines.append("};")
    return "\n".join(lines) + "\n"


def render_layered(bgs):
    """constexpr layered layout of BG1/BG2 (rows grouped, entry order kept), for the
    kernels that unroll the base graph at compile time."""
    lines = [
        "// Layered (row-grouped) layout of the 5G NR base graphs as constexpr tables.",
        "// Generated by syndrome_b200/tables/gen_base_graphs.py; do not edit.",
        "// For layer l, edges loff(l)..loff(l+1)-1 have column col(e) and take their",
        "// shift from base_graph_tables.inc entry ent(e) (the order of the reference's",
        "// build_layout, src/qc_ldpc.rs:281-319); lz384(e) is that edge's shift at",
        "// Z = 384 (lifting set 1, reduced mod 384).  Functions with local constexpr",
        "// tables so that device code can evaluate them at compile time.",
        "#pragma once",
        "",
    ]
    for name in ("bg1", "bg2"):
        rows, cols, ents = bgs[name]
        order = []
        for r in range(rows):
            order += [i for i, (rr, _, _) in enumerate(ents) if rr == r]
        off = [0]
        for r in range(rows):
            off.append(off[-1] + sum(1 for rr, _, _ in ents if rr == r))
        up = name.upper()
        # shifts at Z = 384 (lifting set index 1, a = 3), reduced mod 384 like build_nr_graph
        z384 = [ents[i][2][1] % 384 for i in order]
        for fn, vals in (("loff", off), ("lcol", [ents[i][1] for i in order]), ("lent", order), ("lz384", z384)):
            lines.append(f"__host__ __device__ constexpr int syn_{name}_{fn}(int i) {{")
            lines.append(f"  constexpr int t[{len(vals)}] = {{{', '.join(str(x) for x in vals)}}};")
            lines.append("  return t[i];")
            lines.append("}")
        lines.append("")
    return "\n".join(lines) + "\n"


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SYNDROME_REFERENCE_ROOT")
    if not ref_root:
        raise SystemExit("usage: gen_base_graphs.py <reference-root>")
    bgs = load_bg(ref_root)
    text = render(bgs, load_wifi(ref_root))
    with open(OUT, "w") as f:
        f.write(text)
    with open(OUT_LAYERED, "w") as f:
        f.write(render_layered(bgs))
    print("wrote", os.path.normpath(OUT), "and", os.path.normpath(OUT_LAYERED))


if __name__ == "__main__":
    main()
