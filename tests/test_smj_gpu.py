"""GPU parity of K-SMJ (pimdal_smj_merge / pimdal_sort_merge_join) against the
oracle: the same (inner payload, outer payload) rows in the same order."""
import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu


def cuda_i32(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def u32(t):
    return t.cpu().numpy().view(np.uint32)


def run_smj(ctx, rk, rp, sk, sp, key_dtype=L.I32, capacity=None):
    res, oi, oo = ops.sort_merge_join(ctx, cuda_i32(rk), None if rp is None else cuda_i32(rp),
                                      cuda_i32(sk), None if sp is None else cuda_i32(sp),
                                      key_dtype=key_dtype, capacity=capacity)
    ctx.sync()
    c = int(res.item())
    return c, u32(oi[:c]), u32(oo[:c])


def expected(rk, rp, sk, sp, signed=True):
    rp = np.arange(rk.size, dtype=np.uint32) if rp is None else rp
    sp = np.arange(sk.size, dtype=np.uint32) if sp is None else sp
    return oracle.sort_merge_join(rk, rp, sk, sp, is_signed=signed)


@pytest.mark.parametrize("nr,ns", [(1, 1), (7, 100), (1000, 4000), (5000, 2047), (65536, 262147)])
def test_smj_config_shape(ctx, nr, ns):
    # R = permutation of 0..nr-1 (unique), S drawn from R's keys
    rk = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.I32, seed=31, perm_domain=nr), nr)
    rp = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=31, stream_id=1, lo=-2**31, hi=2**31 - 1), nr)
    sk = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=31, stream_id=2, lo=0, hi=nr - 1,
                                   perm_domain=nr), ns)
    sp = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=31, stream_id=3, lo=-2**31, hi=2**31 - 1), ns)
    c, oi, oo = run_smj(ctx, rk, rp, sk, sp)
    ei, eo = expected(rk, rp, sk, sp)
    assert c == ns == ei.size
    assert np.array_equal(oi, ei.view(np.uint32)) and np.array_equal(oo, eo.view(np.uint32))


@pytest.mark.parametrize("dup", [2, 16, 300])
def test_smj_duplicates_both_sides(ctx, dup):
    # many-to-many: keys repeat on both sides; inner runs cross the tile size
    nr, ns = 20000, 30011
    rk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=32, lo=0, hi=nr // dup), nr)
    sk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=32, stream_id=1, lo=-5, hi=nr // dup + 5), ns)
    cap = int(expected(rk, None, sk, None)[0].size)
    c, oi, oo = run_smj(ctx, rk, None, sk, None, capacity=cap)
    ei, eo = expected(rk, None, sk, None)
    assert c == ei.size and np.array_equal(oi, ei) and np.array_equal(oo, eo)


def test_smj_sparse_outer_wide_inner_range(ctx):
    # a few outer rows spanning a huge inner range (HBM search path)
    nr = 200000
    rk = np.arange(nr, dtype=np.int32)
    sk = np.array([0, 5, 99999, 150000, 199999, 250000], np.int32)
    c, oi, oo = run_smj(ctx, rk, None, sk, None)
    ei, eo = expected(rk, None, sk, None)
    assert c == ei.size == 5 and np.array_equal(oi, ei) and np.array_equal(oo, eo)


def test_smj_unsigned_and_no_match(ctx):
    rk = np.array([0xFFFFFFFF, 1, 0x80000000], np.uint32)
    sk = np.array([0x80000000, 2, 0xFFFFFFFF, 0xFFFFFFFF], np.uint32)
    c, oi, oo = run_smj(ctx, rk, None, sk, None, key_dtype=L.U32)
    ei, eo = expected(rk, None, sk, None, signed=False)
    assert c == 3 and np.array_equal(oi, ei) and np.array_equal(oo, eo)
    c, _, _ = run_smj(ctx, np.array([1, 2], np.int32), None, np.array([3, 4], np.int32), None)
    assert c == 0


def test_smj_capacity_overflow_reports_error(ctx):
    rk = np.zeros(100, np.int32)
    sk = np.zeros(100, np.int32)
    res, _, _ = ops.sort_merge_join(ctx, cuda_i32(rk), None, cuda_i32(sk), None, capacity=50)
    with pytest.raises(L.PimdalError) as e:
        ctx.sync()
    assert e.value.status == 7
    assert int(res.item()) == 10000


def test_smj_merge_matches_reference_semantics(ctx):
    # merge of pre-sorted relations, reference-shaped: inner = shuffled 1..N sorted
    n = 64000
    g = np.load(__import__("pathlib").Path(__file__).parent / "golden" / "smj.npz")
    rk, sk = np.sort(g["rk"]), np.sort(g["sk"])
    res, oo, oi = ops.smj_merge(ctx, cuda_i32(rk), cuda_i32(np.arange(n, dtype=np.int32)),
                                cuda_i32(sk), cuda_i32(np.arange(n, dtype=np.int32)), key_dtype=L.U32)
    ctx.sync()
    c = int(res.item())
    assert c == n
    # inner key of each match, in outer order, equals the reference's inner_res
    assert np.array_equal(rk[u32(oi[:c])], g["inner_res"])
    assert np.array_equal(sk[u32(oo[:c])], g["outer_res"])


def test_smj_config2_full_size(ctx):
    nr, ns = 1 << 24, 1 << 26
    rk = ops.gen_column(ctx, gen.Spec(L.GEN_PERM, L.I32, seed=0xB200, perm_domain=nr), nr)
    sk = ops.gen_column(ctx, gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=0xB200, stream_id=12, lo=0,
                                      hi=nr - 1, perm_domain=nr), ns)
    res, oi, oo = ops.sort_merge_join(ctx, rk, None, sk, None)
    res2, oi2, oo2 = ops.sort_merge_join(ctx, rk, None, sk, None)
    ctx.sync()
    assert int(res.item()) == ns
    # size-independent checks with row ids as payloads: every S row exactly
    # once, in key order, stable; the R row of each pair carries the same key
    rk_h, sk_h = rk.cpu().numpy(), sk.cpu().numpy()
    oi_h, oo_h = oi.cpu().numpy().astype(np.int64), oo.cpu().numpy().astype(np.int64)
    assert np.array_equal(np.bincount(oo_h, minlength=ns), np.ones(ns, np.int64))
    assert np.array_equal(rk_h[oi_h], sk_h[oo_h])
    ks = sk_h[oo_h].astype(np.int64)
    assert np.all(np.diff(ks) >= 0)
    same = ks[1:] == ks[:-1]
    assert np.all(oo_h[1:][same] > oo_h[:-1][same])
    assert torch.equal(oi, oi2) and torch.equal(oo, oo2)
