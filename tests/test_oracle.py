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


def test_bloom_matches_golden():
    g = _load("bloom")
    for w in range(5):
        assert np.array_equal(oracle.hash_fn(w, g["h_keys"]), g[f"h{w}"]), w
    filt = oracle.bloom_build(g["bk"], g["bps"])
    assert np.array_equal(filt, g["filters"])
    mk, mp, ms = oracle.bloom_match(filt, g["pk"], g["pps"])
    assert np.array_equal(mk, g["match_key"]) and np.array_equal(mp, g["match_ptr"])
    assert np.array_equal(ms, g["match_sizes"])
    # every probe row whose key is in its partition's build keys is kept
    bps, pps = g["bps"].astype(int), g["pps"].astype(int)
    kept = set(mp.tolist())
    for p in range(bps.size - 1):
        bset = set(g["bk"][bps[p]:bps[p + 1]].tolist())
        for r in range(pps[p], pps[p + 1]):
            if int(g["pk"][r]) in bset:
                assert r in kept


def test_bloom_match_drops_rows_outside_every_partition():
    k = np.arange(100, dtype=np.uint32)
    ps = np.array([10, 40, 60], np.uint64)
    filt = oracle.bloom_build(k, ps)
    mk, mp, ms = oracle.bloom_match(filt, k, ps)
    assert np.array_equal(mp, np.arange(10, 60, dtype=np.uint32))
    assert ms.tolist() == [0, 30, 20]


@pytest.mark.skipif(not oracle.Ref.available("bloom"), reason="oracle/_ref not built")
def test_bloom_oracle_vs_reference_fresh_inputs():
    ref = oracle.Ref()
    k = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=21, lo=0, hi=2**32 - 1), 50000)
    for w in range(5):
        assert np.array_equal(oracle.hash_fn(w, k[:3000]), ref.hash_fn(w, k[:3000]))
    ps = np.array([0, 1, 1, 2500, 20000, 50000], np.uint64)
    filt = oracle.bloom_build(k, ps)
    assert np.array_equal(filt, ref.bloom_build(k, ps))
    q = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=22, lo=0, hi=2**32 - 1), 50000)
    q[::4] = k[::4]
    for a, b in zip(oracle.bloom_match(filt, q, ps), ref.bloom_match(filt, q, ps)):
        assert np.array_equal(a, b)


def test_parallel_group_by_equals_serial():
    """The key-partitioned, threaded group-by (used at full sizes) returns
    exactly the serial oracle's groups."""
    rng = np.random.default_rng(41)
    k = rng.integers(-5000, 5000, 300_000).astype(np.int32)
    k[::11] = -1
    v = rng.integers(-10**12, 10**12, k.size).astype(np.int64)
    exp = oracle.group_by(k, v)
    got = oracle.group_by_parallel(k, v, threads=4, parts_log2=3)
    for a, b in zip(got, exp):
        assert np.array_equal(a, b)
    got = oracle.group_by_parallel(k, None, threads=2, parts_log2=1)
    for a, b in zip(got, oracle.group_by(k, None)):
        assert np.array_equal(a, b)


def test_parallel_hash_join_equals_serial():
    """The key-partitioned, threaded hash join returns the serial oracle's
    multiset of (build payload, probe row id), duplicate build keys included."""
    rng = np.random.default_rng(42)
    bk = rng.integers(0, 20_000, 30_000).astype(np.uint32)
    bp = rng.integers(0, 2**32, bk.size, dtype=np.uint64).astype(np.uint32)
    pk = rng.integers(0, 40_000, 200_000).astype(np.uint32)
    ep, er = oracle.hash_join(bk, bp, pk)
    gp, gr = oracle.hash_join_parallel(bk, bp, pk, threads=4, parts_log2=4)
    a, b = np.lexsort((gp, gr)), np.lexsort((ep, er))
    assert gp.size == ep.size
    assert np.array_equal(gp[a], ep[b]) and np.array_equal(gr[a], er[b])
