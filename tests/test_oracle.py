"""Pins the CPU oracle: against the golden fixtures made by the reference's own
CPU operators (tests/golden/make_golden.py) and, where the reference harnesses
are built (oracle/_ref), against the reference directly on fresh inputs."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen

GOLD = Path(__file__).resolve().parent / "golden"


def _load(name):
    return np.load(GOLD / f"{name}.npz")


def test_select_matches_golden():
    g = _load("select")
    for n in [0, 1, 31, 7999, 8000, 8001, 100003]:
        v, p = oracle.select(g[f"cfg_keys_{n}"], -2**63, 214748364 - 1)
        assert np.array_equal(v, g[f"cfg_out_{n}"]), n
        assert np.array_equal(g[f"cfg_keys_{n}"][p], v)
        assert np.all(np.diff(p.astype(np.int64)) > 0)
        v2, _ = oracle.select(g[f"own_keys_{n}"], 10, 29)
        assert np.array_equal(v2, g[f"own_out_{n}"]), n


def test_sort_matches_golden():
    g = _load("sort")
    for n in [0, 1, 2, 1000, 65537]:
        for tag, signed in (("u", False), ("d", False), ("s", True)):
            k, p = oracle.sort_pairs(g[f"{tag}_keys_{n}"], is_signed=signed)
            assert np.array_equal(np.stack([k, p]), g[f"{tag}_out_{n}"]), (tag, n)


def test_hash_join_matches_golden_in_reference_order():
    g = _load("hash_join")
    for i in range(3):
        pay, row = oracle.hash_join(g[f"bk_{i}"], g[f"bp_{i}"], g[f"pk_{i}"])
        assert np.array_equal(pay, g[f"pay_{i}"].view(np.uint32)), i
        assert np.array_equal(row, g[f"row_{i}"]), i


def test_group_by_matches_golden():
    g = _load("group_by")
    for i in range(3):
        for fn in (oracle.group_by, oracle.sort_group_by):
            out = fn(g[f"k_{i}"], g[f"v_{i}"])
            for name, arr in zip(("key", "sum", "count", "min", "max"), out):
                assert np.array_equal(arr, g[f"{name}_{i}"]), (fn.__name__, name, i)


def test_smj_matches_golden():
    g = _load("smj")
    rk, sk = g["rk"], g["sk"]
    n = rk.size
    r_pay, s_pay = oracle.sort_merge_join(rk, np.arange(n, dtype=np.uint32), sk,
                                          np.arange(n, dtype=np.uint32), is_signed=False)
    assert np.array_equal(sk[s_pay], g["outer_res"])
    assert np.array_equal(rk[r_pay], g["inner_res"])


def test_smj_emits_every_duplicate_match():
    rk = np.array([1, 2, 2, 3], np.uint32)
    sk = np.array([2, 2, 4, 1], np.uint32)
    r_pay, s_pay = oracle.sort_merge_join(rk, np.arange(4, dtype=np.uint32), sk,
                                          np.arange(4, dtype=np.uint32))
    pairs = sorted(zip(r_pay.tolist(), s_pay.tolist()))
    assert pairs == [(0, 3), (1, 0), (1, 1), (2, 0), (2, 1)]


def test_part_hash0_is_a_stable_partition():
    k = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=1, lo=0, hi=2**32 - 1), 20000)
    ok, op, sizes = oracle.part_hash0(k, shift=27, part_n=32)
    assert sizes[0] == 0 and sizes[-1] == k.size
    assert np.array_equal(k[op], ok)
    for p in range(32):
        seg = op[sizes[p]:sizes[p + 1]]
        assert np.all(np.diff(seg.astype(np.int64)) > 0)


REF = pytest.mark.skipif(not oracle.Ref.available("select"), reason="oracle/_ref not built")


@REF
def test_oracle_vs_reference_fresh_inputs():
    ref = oracle.Ref()
    n = 300001
    k = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=11, lo=0, hi=2**31 - 1), n)
    ref.set_threads("select", 1)
    v, _ = oracle.select(k, -2**63, 214748364 - 1)
    assert np.array_equal(v, ref.select(k, -2**63, 214748364 - 1))
    ku = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=12, lo=0, hi=2**20), n)
    assert np.array_equal(np.stack(oracle.sort_pairs(ku)), np.stack(ref.sort_pairs(ku)))
    ck = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=13, lo=0, hi=999,
                                   perm_domain=0), n)
    cv = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I64, seed=13, stream_id=1, lo=100,
                                   hi=10**7), n)
    for a, b in zip(oracle.group_by(ck, cv), ref.group_by(ck, cv)):
        assert np.array_equal(a, b)
