"""The compiled C++ caller (tests/cpp/pimdal_host.cpp): a host program that
includes include/pimdal_gpu.h and links libpimdal_b200.so, as the reference's
host programs (pimdal/main/*/host) would after the drop-in.  It is built with
g++ here (no GPU needed) and, on a GPU, runs selection, sort, hash join and
group-by on the golden fixtures' inputs -- its outputs must equal the golden
outputs, which come from the reference's own CPU operators -- and the TPC-H
Q6 pipeline through the fused scan, checked against a numpy restatement."""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


def build_host(out_dir: Path) -> Path:
    exe = out_dir / "pimdal_host"
    lib_dir = ROOT / "pimdal_b200"
    assert (lib_dir / "libpimdal_b200.so").exists(), "build the library first"
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-Wall", "-Werror",
           str(ROOT / "tests" / "cpp" / "pimdal_host.cpp"),
           f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}",
           f"-L{lib_dir}", "-lpimdal_b200", f"-L{CUDA / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{CUDA / 'lib64'}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.fixture(scope="module")
def host_exe(tmp_path_factory):
    return build_host(tmp_path_factory.mktemp("cpp"))


def test_cpp_caller_builds_against_the_header_and_library(host_exe):
    r = subprocess.run([str(host_exe)], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr  # PIMDAL_ERR_ARG, no GPU touched


def run(exe, d, *args):
    r = subprocess.run([str(exe), str(d), *map(str, args)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_cpp_caller_select_matches_golden(host_exe, tmp_path):
    g = np.load(GOLDEN / "select.npz")
    for n in (1, 31, 7999, 8000, 8001, 100003):
        keys = g[f"own_keys_{n}"]
        keys.astype(np.int32).tofile(tmp_path / "sel_keys.i32")
        run(host_exe, tmp_path, "select", 10, 29)   # the reference's 10 <= v < 30
        vals = np.fromfile(tmp_path / "sel_vals.i32", np.int32)
        rows = np.fromfile(tmp_path / "sel_rows.u32", np.uint32)
        assert np.array_equal(vals, g[f"own_out_{n}"])
        assert np.array_equal(keys[rows], vals) and np.all(np.diff(rows.astype(np.int64)) > 0)


@pytest.mark.gpu
def test_cpp_caller_sort_matches_golden(host_exe, tmp_path):
    g = np.load(GOLDEN / "sort.npz")
    for n in (1, 2, 1000, 65537):
        for kind in ("u", "d"):
            g[f"{kind}_keys_{n}"].astype(np.uint32).tofile(tmp_path / "sort_keys.u32")
            run(host_exe, tmp_path, "sort")
            out = g[f"{kind}_out_{n}"]
            assert np.array_equal(np.fromfile(tmp_path / "sort_keys_out.u32", np.uint32), out[0])
            assert np.array_equal(np.fromfile(tmp_path / "sort_rows.u32", np.uint32), out[1])


@pytest.mark.gpu
def test_cpp_caller_hash_join_matches_golden(host_exe, tmp_path):
    g = np.load(GOLDEN / "hash_join.npz")
    for i in range(3):
        for name in ("bk", "bp", "pk"):
            g[f"{name}_{i}"].astype(np.int32).tofile(tmp_path / f"hj_{name}.i32")
        run(host_exe, tmp_path, "hash_join")
        pay = np.fromfile(tmp_path / "hj_pay.u32", np.uint32)
        row = np.fromfile(tmp_path / "hj_row.u32", np.uint32)
        epay, erow = g[f"pay_{i}"], g[f"row_{i}"]
        a, b = np.lexsort((pay, row)), np.lexsort((epay, erow))
        assert pay.size == epay.size
        assert np.array_equal(pay[a], epay[b]) and np.array_equal(row[a], erow[b])


@pytest.mark.gpu
def test_cpp_caller_group_by_matches_golden(host_exe, tmp_path):
    g = np.load(GOLDEN / "group_by.npz")
    for i in range(3):
        g[f"k_{i}"].astype(np.int32).tofile(tmp_path / "gb_k.i32")
        g[f"v_{i}"].astype(np.int64).tofile(tmp_path / "gb_v.i64")
        run(host_exe, tmp_path, "group_by")
        assert np.array_equal(np.fromfile(tmp_path / "gb_key.i32", np.int32), g[f"key_{i}"])
        for c in ("sum", "count", "min", "max"):
            assert np.array_equal(np.fromfile(tmp_path / f"gb_{c}.i64", np.int64), g[f"{c}_{i}"]), c


@pytest.mark.gpu
def test_cpp_caller_tpch_q6_matches_numpy(host_exe, tmp_path, ctx):
    """The Q6 pipeline of pimdal/main/tpc_h/query6 run by the C++ host through
    pimdal_select_aggregate, on the synthetic lineitem columns, against the
    numpy restatement of host_q6.cpp:70-100."""
    from pimdal_b200 import serve, tpch
    li = tpch.Lineitem(ctx, serve.Tables(ctx, orders=100_000, parts=5_000, supps=1_000, seed=17))
    h = {"date": li.shipdate.cpu().numpy(), "qty": li.quantity.cpu().numpy(),
         "disc": li.discount.cpu().numpy(), "price": li.price.cpu().numpy()}
    h["date"].astype(np.int32).tofile(tmp_path / "q6_date.i32")
    h["qty"].astype(np.int32).tofile(tmp_path / "q6_qty.i32")
    h["disc"].astype(np.int32).tofile(tmp_path / "q6_disc.i32")
    h["price"].astype(np.int64).tofile(tmp_path / "q6_price.i64")
    lo, hi = tpch.packed(tpch.Q6_DATE_LO), tpch.packed(tpch.Q6_DATE_HI)
    run(host_exe, tmp_path, "q6", lo, hi, tpch.Q6_QUANTITY, tpch.Q6_DISCOUNT)
    revenue, rows = np.fromfile(tmp_path / "q6_out.i64", np.int64)
    m = (h["date"] >= lo) & (h["date"] < hi) & (h["qty"] < tpch.Q6_QUANTITY)
    m &= (h["disc"] >= tpch.Q6_DISCOUNT - 1) & (h["disc"] <= tpch.Q6_DISCOUNT + 1)
    assert rows == m.sum() > 0
    assert revenue == int((h["disc"][m].astype(np.int64) * h["price"][m]).sum())
