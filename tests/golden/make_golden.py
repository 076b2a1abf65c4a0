"""Regenerate the golden fixtures in this folder from the reference's own
recorded outputs.  Run in a checkout that has the reference tree:

    python tests/golden/make_golden.py <reference-root>

Fixtures written (bits are packed LSB-first into bytes, then hex):
  ldpc_convergence_wifi27_r12.json  <- bench/results/ldpc_convergence.json
      802.11 Z=27 R=1/2, beta=0.25, AWGN Eb/N0=0 dB seed 139, 14 max iterations;
      the transmitted codeword and the hard decisions after every iteration.
  ldpc_checksums.json               <- bench/results/ldpc_{rust,cpp}.checksum
      FNV-1a of the hard decisions of BG1 Z=384, beta=0.25, llr=+0.5/-0.5
      alternating, 10 iterations (src/bin/ldpc_bench_export.rs).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def pack(bits):
    return np.packbits(np.asarray(bits, dtype=np.uint8), bitorder="little").tobytes().hex()


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SYNDROME_REFERENCE_ROOT")
    if not ref:
        raise SystemExit("usage: make_golden.py <reference-root>")
    res = os.path.join(ref, "bench", "results")
    with open(os.path.join(res, "ldpc_convergence.json")) as f:
        d = json.load(f)
    conv = {
        "source": "bench/results/ldpc_convergence.json",
        "code": d["code"],
        "channel": d["channel"],
        "info_bits_rule": "bit i = ((i * 2654435761) >> 31) & 1 (64-bit wrapping)",
        "max_iterations": d["max_iterations"],
        "iterations_used": d["iterations_used"],
        "converged": d["converged"],
        "n": len(d["transmitted_codeword"]),
        "transmitted_codeword": pack(d["transmitted_codeword"]),
        "frames": [
            {"iteration": fr["iteration"], "bit_errors": fr["bit_errors"], "hard_bits": pack(fr["hard_bits"])}
            for fr in d["frames"]
        ],
    }
    with open(os.path.join(HERE, "ldpc_convergence_wifi27_r12.json"), "w") as f:
        json.dump(conv, f, indent=1)
    sums = {}
    for name in ("ldpc_rust.checksum", "ldpc_cpp.checksum"):
        with open(os.path.join(res, name)) as f:
            sums[name] = f.read().strip()
    out = {
        "source": "bench/results/ldpc_rust.checksum, bench/results/ldpc_cpp.checksum",
        "config": {"bg": 1, "z": 384, "offset_beta": 0.25, "iterations": 10,
                   "llr": "+0.5 at even index, -0.5 at odd index", "path": "f32 LOMS, no 5G prologue"},
        "fnv1a_offset": "0xcbf29ce484222325", "fnv1a_prime": "0x100000001b3",
        "checksums": sums,
    }
    with open(os.path.join(HERE, "ldpc_checksums.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
