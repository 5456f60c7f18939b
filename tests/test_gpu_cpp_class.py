"""The C++ GIR class (include/gir_b200.hpp): a caller written like the reference's own drivers
compiles against the header and libgir_b200.so, and sees the reference's results on the example
graph (the known answers of runTargetedSplitTest, gir_test.cpp:704-753)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "graph-intermedia-representation_b200")


def test_cpp_caller_on_example_graph(golden, tmp_path):
    exe = str(tmp_path / "gir_drop_in")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "gir_drop_in.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-L", PKG, "-lgir_b200", f"-Wl,-rpath,{PKG}", "-o", exe],
                   check=True)
    d = str(tmp_path) + "/"
    for name, key in (("fw_begin", "in_fw_beg"), ("fw_adjacent", "in_fw_adj"), ("bw_begin", "in_bw_beg"),
                      ("bw_adjacent", "in_bw_adj")):
        golden[f"example/{key}"].astype(np.int32).tofile(d + name + ".bin")
    out = subprocess.run([exe, d], check=True, capture_output=True, text=True).stdout
    kv = {}
    for line in out.splitlines():
        parts = line.split()
        kv[parts[0]] = parts[1:]
    assert kv["V"] == ["18"]
    n_wcc = len(np.unique(golden["example/s0/wcc"]))
    n_scc = len(np.unique(golden["example/s0/scc"]))
    assert kv["wcc"] == [str(n_wcc), "scc", str(n_scc)]
    assert kv["case1"] == ["1"] and kv["case5c"] == ["1"] and kv["case5b"] == ["1"]
    assert kv["blocks_of_scc0"] == ["1"]  # {0,1,2} after the split: one block
    assert kv["bfs_0_9"][0] == str(golden["example/s3/bfs"][0][9])
    assert kv["bfs_0_9"][2] == str(golden["example/s3/sssp"][0][1])
    assert kv["has"] == ["1", "0", "1"]
    assert kv["reach_matches_bfs"] == ["1"]
    assert kv["inc_matches_scratch"] == ["1"]
    assert kv["error_missing"] == ["1"]
    assert kv["queryvec"] == ["1"] and kv["reach_noindex"] == ["1"]
    assert kv["forest_ok"] == ["1"] and kv["bicon_self"] == ["1"] and kv["bc_ok"] == ["1"]
    assert kv["ingest"] == ["1", "1", "1", "1"]  # pending, getters unchanged, BFS sees it, synced
    assert kv["from_graph"] == ["4", "2", "18"]
