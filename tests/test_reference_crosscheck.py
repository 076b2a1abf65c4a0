"""Cross-checks that need the reference source tree (skipped where it is absent):
the committed base-graph tables equal the reference's data files, and the
reference's own C++ port (bench/cpp/loms_decode.cpp, compiled into oracle/_ref
by `make -C oracle ref`) reproduces the oracle's checksum."""
import os
import shutil
import subprocess

import pytest

from conftest import REFERENCE_ROOT, ROOT, needs_reference


@needs_reference
def test_tables_match_reference_sources(tmp_path):
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "gen", os.path.join(ROOT, "syndrome_b200", "tables", "gen_base_graphs.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    text = gen.render(gen.load_bg(REFERENCE_ROOT), gen.load_wifi(REFERENCE_ROOT))
    with open(os.path.join(ROOT, "syndrome_b200", "csrc", "base_graph_tables.inc")) as f:
        assert f.read() == text


@needs_reference
def test_reference_cpp_port_checksum(tmp_path):
    """The reference's C++ port writes <root>/bench/results; it is run against a
    scratch root under oracle/_ref so nothing is written into the reference."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref",
                           f"REF={REFERENCE_ROOT}"])
    run_root = os.path.join(ROOT, "oracle", "_ref", "run")
    os.makedirs(os.path.join(run_root, "data"), exist_ok=True)
    shutil.copyfile(os.path.join(REFERENCE_ROOT, "data", "bg_tables.json"),
                    os.path.join(run_root, "data", "bg_tables.json"))
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "loms_decode"), run_root],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    with open(os.path.join(run_root, "bench", "results", "ldpc_cpp.checksum")) as f:
        assert f.read().strip() == "a2448e8cf5272825"
