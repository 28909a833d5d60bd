"""GPU parity of K-HGB / K-SGB (pimdal_group_kernel) against the oracle:
identical (key, SUM, COUNT, MIN, MAX) rows in key order, bit-exact int64."""
import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu

METHODS = [L.GROUP_HASH, L.GROUP_SORT]


def inputs(n, card, seed):
    k = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=seed, lo=0, hi=card - 1,
                                  perm_domain=0), n)
    v = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I64, seed=seed, stream_id=1, lo=100,
                                  hi=10**7), n)
    return k, v


def run(ctx, k, v, method, expected=0, key_dtype=L.I32):
    kt = torch.from_numpy(np.ascontiguousarray(k).view(np.int32)).cuda()
    vt = None if v is None else torch.from_numpy(np.ascontiguousarray(v)).cuda()
    res, outs = ops.group_kernel(ctx, kt, vt, method=method, expected_groups=expected,
                                 key_dtype=key_dtype)
    ctx.sync()
    g = int(res.item())
    return tuple(outs[c][:g].cpu().numpy() for c in ("key", "sum", "count", "min", "max"))


def check(got, exp):
    for name, a, b in zip(("key", "sum", "count", "min", "max"), got, exp):
        assert np.array_equal(a, b), name


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("n,card", [(1, 1), (31, 4), (4097, 16), (100003, 4096),
                                    (1 << 20, 16), (1 << 20, 1 << 16)])
def test_group_by_matches_oracle(ctx, method, n, card):
    k, v = inputs(n, card, 51)
    check(run(ctx, k, v, method, expected=card), oracle.group_by(k, v))


@pytest.mark.parametrize("method", METHODS)
def test_group_by_negative_keys_sentinel_and_count_only(ctx, method):
    k, v = inputs(50000, 300, 52)
    k[::13] = -1
    k[::17] = np.iinfo(np.int32).min
    k[::19] = np.iinfo(np.int32).max
    v[::7] = -5 * 10**12
    check(run(ctx, k, v, method, expected=512), oracle.group_by(k, v))
    check(run(ctx, k, None, method, expected=512), oracle.group_by(k, None))


@pytest.mark.parametrize("method", METHODS)
def test_group_by_overflowing_shared_tables(ctx, method):
    # far more groups than a CTA's shared-memory table holds
    k, v = inputs(1 << 21, 1 << 20, 53)
    check(run(ctx, k, v, method, expected=1 << 20), oracle.group_by(k, v))


def test_hash_and_sort_methods_agree_and_are_deterministic(ctx):
    k, v = inputs(1 << 22, 1 << 12, 54)
    a = run(ctx, k, v, L.GROUP_HASH, expected=1 << 12)
    b = run(ctx, k, v, L.GROUP_SORT)
    c = run(ctx, k, v, L.GROUP_HASH, expected=1 << 12)
    check(a, b)
    check(a, c)


@pytest.mark.parametrize("card", [16, 1 << 12, 1 << 22])
def test_group_by_config3_full_size(ctx, card):
    n = 1 << 28
    ks = gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=0xB203, stream_id=5, lo=0, hi=card - 1,
                  perm_domain=0)
    vs = gen.Spec(L.GEN_UNIFORM, L.I64, seed=0xB203, stream_id=6, lo=100, hi=10**7)
    kd = ops.gen_column(ctx, ks, n)
    vd = ops.gen_column(ctx, vs, n)
    r1, o1 = ops.group_kernel(ctx, kd, vd, method=L.GROUP_HASH, expected_groups=card)
    r2, o2 = ops.group_kernel(ctx, kd, vd, method=L.GROUP_SORT, capacity=2 * card)
    ctx.sync()
    g = int(r1.item())
    assert g == int(r2.item()) == card
    for c in ("key", "sum", "count", "min", "max"):
        assert torch.equal(o1[c][:g], o2[c][:g]), c
    # size-independent checks: counts add up, sums add up, keys ascending
    assert int(o1["count"][:g].sum().item()) == n
    assert int(o1["sum"][:g].sum().item()) == int(vd.sum().item())
    kk = o1["key"][:g].cpu().numpy()
    assert np.all(np.diff(kk.astype(np.int64)) > 0)
    assert int(o1["min"][:g].min().item()) >= 100 and int(o1["max"][:g].max().item()) <= 10**7


@pytest.mark.parametrize("expected", [4, 16, 32, 64, 1000])
def test_group_by_all_ones_key_in_every_table_mode(ctx, expected):
    # the all-ones key (-1) is the shared tables' empty marker: it must still aggregate
    k, v = inputs(20000, min(expected, 8), 55)
    k[::3] = -1
    check(run(ctx, k, v, L.GROUP_HASH, expected=expected), oracle.group_by(k, v))


@pytest.mark.parametrize("card,expected", [(1 << 13, 1 << 13), (1 << 15, 1 << 15),
                                           (1 << 18, 1 << 18), (1 << 18, 1 << 20)])
def test_partitioned_hash_group_by(ctx, card, expected):
    """Many groups: rows radix-partitioned by a key hash, chunks aggregated in
    shared memory.  Heavy hitters (a third of the rows on a few keys), the
    all-ones key, int32 extremes, unsigned order and count-only, against the
    oracle; partition counts from one pass (<= 6 bits) to two."""
    n = (1 << 21) + 77
    k, v = inputs(n, card, 54)
    k[::3] = np.array([7, -1, 123456789], np.int32)[np.arange(k[::3].size) % 3]
    k[::101] = np.iinfo(np.int32).min
    k[::103] = np.iinfo(np.int32).max
    v[::5] = -3 * 10**13
    exp = oracle.group_by(k, v)
    check(run(ctx, k, v, L.GROUP_HASH, expected=expected), exp)
    check(run(ctx, k, None, L.GROUP_HASH, expected=expected), oracle.group_by(k, None))
    got = run(ctx, k, v, L.GROUP_HASH, expected=expected, key_dtype=L.U32)
    o = np.argsort(exp[0].view(np.uint32), kind="stable")
    for name, a, b in zip(("key", "sum", "count", "min", "max"), got, exp):
        assert np.array_equal(a, b[o]), name


@pytest.mark.parametrize("span", [2**32 - 1, 2**32])
def test_sort_group_by_value_range_edges(ctx, span):
    """Sort method: values whose range is exactly 2^32 - 1 travel through the
    sort as 32-bit payloads; one more and the row-id path takes over -- the
    same groups either way, against the oracle."""
    k, v = inputs(200003, 1000, 55)
    base = -(2**40) + 12345
    v = (base + (v - 100) % 7).astype(np.int64)
    v[5], v[777] = base, base + span
    check(run(ctx, k, v, L.GROUP_SORT, expected=1000), oracle.group_by(k, v))
