"""The plain operators' autotuner (pimdal_hash_join_autotune,
pimdal_group_autotune): it times its candidates on the call's own inputs,
caches the fastest per shape in the context, and later calls of that shape
use it -- with results still equal to the oracle's."""
import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu


def i32(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def u32(t):
    return t.cpu().numpy().view(np.uint32)


def sorted_pairs(pay, row):
    o = np.lexsort((pay, row))
    return pay[o], row[o]


def test_hash_join_autotune_caches_and_is_used(ctx):
    nb, npr = 1 << 20, 1 << 22
    bk = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.I32, seed=91, perm_domain=2 * nb), nb)
    bp = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=91, stream_id=1, lo=-2**31,
                                   hi=2**31 - 1), nb)
    pk = gen.generate_cpu(gen.Spec(L.GEN_PROBE, L.I32, seed=91, stream_id=2, lo=nb,
                                   perm_domain=2 * nb, match_permille=500), npr)
    epay, erow = oracle.hash_join(bk, bp, pk)
    exp = sorted_pairs(epay, erow)
    budget = 2 << 20  # a small L2 budget makes the library partition (3 bits here)
    t, cached, res, pay, row = ops.hash_join_autotune(ctx, i32(bk), i32(bp), i32(pk),
                                                      l2_budget_bytes=budget)
    ctx.sync()
    assert not cached and t["candidates"] >= 6 and t["ms"] > 0
    assert t["load_factor_pct"] in (35, 50, 70)
    assert t["partition_bits"] == 0xFFFFFFFF or 1 <= t["partition_bits"] <= 8
    c = int(res.item())
    assert c == epay.size
    got = sorted_pairs(u32(pay[:c]), u32(row[:c]))
    assert np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1])
    # the same shape again: the cached choice, nothing run
    t2, cached2, *_ = ops.hash_join_autotune(ctx, i32(bk), i32(bp), i32(pk), l2_budget_bytes=budget)
    assert cached2 and t2["candidates"] == 0
    assert (t2["partition_bits"], t2["load_factor_pct"]) == (t["partition_bits"], t["load_factor_pct"])
    # a plain call of the shape (partition_bits = load_factor_pct = 0) uses it
    res, pay, row = ops.hash_join(ctx, i32(bk), i32(bp), i32(pk), l2_budget_bytes=budget)
    ctx.sync()
    c = int(res.item())
    got = sorted_pairs(u32(pay[:c]), u32(row[:c]))
    assert c == epay.size and np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1])


def group_inputs(n, card, seed):
    k = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=seed, lo=0, hi=card - 1,
                                  perm_domain=0), n)
    v = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I64, seed=seed, stream_id=1, lo=100,
                                  hi=10**7), n)
    return k, v


def group_outputs(res, outs):
    g = int(res.item())
    return tuple(outs[c][:g].cpu().numpy() for c in ("key", "sum", "count", "min", "max"))


def check(got, exp):
    for name, a, b in zip(("key", "sum", "count", "min", "max"), got, exp):
        assert np.array_equal(a, b), name


def test_group_autotune_high_cardinality(ctx):
    n, card = 1 << 21, 1 << 18
    k, v = group_inputs(n, card, 92)
    exp = oracle.group_by(k, v)
    t, cached, res, outs = ops.group_autotune(ctx, i32(k), torch.from_numpy(v).cuda(),
                                              expected_groups=card)
    ctx.sync()
    assert not cached and t["candidates"] >= 3 and t["group_mode"] in (1, 2)
    if t["group_mode"] == 1:
        assert 1 <= t["group_part_bits"] <= 12
    check(group_outputs(res, outs), exp)
    t2, cached2, *_ = ops.group_autotune(ctx, i32(k), torch.from_numpy(v).cuda(),
                                         expected_groups=card)
    assert cached2 and t2["candidates"] == 0 and t2["group_mode"] == t["group_mode"]
    res, outs = ops.group_kernel(ctx, i32(k), torch.from_numpy(v).cuda(), expected_groups=card)
    ctx.sync()
    check(group_outputs(res, outs), exp)


def test_group_autotune_nothing_to_choose(ctx):
    k, v = group_inputs(100_003, 16, 93)
    t, cached, res, outs = ops.group_autotune(ctx, i32(k), torch.from_numpy(v).cuda(),
                                              expected_groups=16)
    ctx.sync()
    assert not cached and t["candidates"] == 0 and t["group_mode"] == 0
    check(group_outputs(res, outs), oracle.group_by(k, v))
