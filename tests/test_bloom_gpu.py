"""GPU parity of the Bloom-filter prefilter (pimdal_filter_kernel /
pimdal_match_kernel) against the oracle and the golden fixture made from the
reference's hash functions: filter bytes identical, kept rows identical and
in input order, per-partition counts identical.  Covers empty partitions,
rows outside every partition, tiles spanning a few or many partitions,
large single-partition tiles, both layouts, filters exchanged with the
oracle, an empty input and an output capacity overflow."""
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"


def dev(a, dtype=np.int32):
    return torch.from_numpy(np.ascontiguousarray(a).view(dtype)).cuda()


def u32(t):
    return t.cpu().numpy().view(np.uint32)


def run_match(ctx, filters, keys, ps, ptr=None, pairs=False):
    if pairs:
        kp = np.stack([keys, np.arange(keys.size, dtype=np.uint32) if ptr is None else ptr], axis=1)
        res, out, _, sizes = ops.match_kernel(ctx, filters, dev(kp), dev(ps, np.int64), pairs=True)
        ctx.sync()
        c = int(res.item())
        o = u32(out[:c])
        return o[:, 0], o[:, 1], sizes.cpu().numpy().view(np.uint64)
    res, out, orow, sizes = ops.match_kernel(ctx, filters, dev(keys), dev(ps, np.int64),
                                             None if ptr is None else dev(ptr))
    ctx.sync()
    c = int(res.item())
    return u32(out[:c]), u32(orow[:c]), sizes.cpu().numpy().view(np.uint64)


def check(ctx, bk, bps, pk, pps, pairs=False, ptr=None):
    exp_f = oracle.bloom_build(bk, bps)
    if pairs:
        bkp = np.stack([bk, np.arange(bk.size, dtype=np.uint32)], axis=1)
        f = ops.filter_kernel(ctx, dev(bkp), dev(bps, np.int64), pairs=True)
    else:
        f = ops.filter_kernel(ctx, dev(bk), dev(bps, np.int64))
    ctx.sync()
    assert np.array_equal(f.cpu().numpy(), exp_f)
    ek, ep, es = oracle.bloom_match(exp_f, pk, pps, ptr)
    gk, gp, gs = run_match(ctx, f, pk, pps, ptr, pairs)
    assert np.array_equal(gk, ek) and np.array_equal(gp, ep)
    assert np.array_equal(gs, es)


def sizes_to_offsets(sz):
    return np.concatenate([[0], np.cumsum(sz)]).astype(np.uint64)


def test_bloom_matches_golden(ctx):
    g = np.load(GOLD / "bloom.npz")
    f = ops.filter_kernel(ctx, dev(g["bk"]), dev(g["bps"], np.int64))
    ctx.sync()
    assert np.array_equal(f.cpu().numpy(), g["filters"])
    k, p, s = run_match(ctx, f, g["pk"], g["pps"])
    assert np.array_equal(k, g["match_key"]) and np.array_equal(p, g["match_ptr"])
    assert np.array_equal(s, g["match_sizes"])


@pytest.mark.parametrize("pairs", [False, True])
@pytest.mark.parametrize("probe_rows", [120, 1500])
def test_bloom_small_partitions(ctx, pairs, probe_rows):
    # 16384 partitions of ~2000 build keys (the CPU join's partitioning).
    # Probe partitions of ~60 rows put dozens of partitions in one tile (the
    # global path); ~750 rows put a few in one tile (the shared-memory path).
    part_n = 16384
    rng = np.random.default_rng(3 + probe_rows)
    bsz = rng.integers(0, 4000, part_n)
    bsz[::97] = 0
    psz = rng.integers(0, probe_rows, part_n)
    psz[::89] = 0
    bps, pps = sizes_to_offsets(bsz), sizes_to_offsets(psz)
    bk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=31, lo=0, hi=2**32 - 1), int(bps[-1]))
    pk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=32, lo=0, hi=2**32 - 1), int(pps[-1]))
    for p in range(0, part_n, 7):  # some probe keys taken from their partition's build keys
        lo, hi = int(pps[p]), int(pps[p + 1])
        if bsz[p] and hi > lo:
            pk[lo:hi:2] = bk[int(bps[p]) + rng.integers(0, bsz[p], (hi - lo + 1) // 2)]
    check(ctx, bk, bps, pk, pps, pairs=pairs)


def test_bloom_large_partitions_and_rows_outside(ctx):
    # three large partitions (single-partition tiles), rows before the first
    # and after the last partition, explicit row ids
    n = 300001
    bk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=41, lo=0, hi=2**32 - 1), 9000)
    bps = np.array([0, 1000, 1000, 9000], np.uint64)
    pk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=42, lo=0, hi=2**32 - 1), n)
    pk[5000::3] = bk[np.arange(5000, n, 3) % 9000]
    pps = np.array([4097, 100000, 100000, 290000], np.uint64)
    ptr = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=43, lo=0, hi=2**32 - 1), n)
    check(ctx, bk, bps, pk, pps, ptr=ptr)


@pytest.mark.parametrize("pairs", [False, True])
def test_bloom_partitions_above_and_below_the_shared_memory_size(ctx, pairs):
    # build partitions of 20000 and 30000 rows (the tile path) between small
    # ones (stored whole by one CTA each), one empty
    bsz = np.array([100, 20000, 0, 50, 30000, 7, 16384, 16385, 3000], np.uint64)
    bps = np.concatenate([[0], np.cumsum(bsz)]).astype(np.uint64)
    bk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=44, lo=0, hi=2**32 - 1), int(bps[-1]))
    psz = np.array([500, 3000, 10, 700, 4000, 0, 2000, 2000, 900], np.uint64)
    pps = np.concatenate([[0], np.cumsum(psz)]).astype(np.uint64)
    n = int(pps[-1])
    pk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=45, lo=0, hi=2**32 - 1), n)
    pk[::4] = bk[np.arange(0, n, 4) % bk.size]
    check(ctx, bk, bps, pk, pps, pairs=pairs)


def test_bloom_every_build_key_passes(ctx):
    # partition both sides with part_kernel (hash0 bits), then the filter of a
    # build partition must keep every probe row whose key it holds
    nb, npr, part_n = 1 << 16, 1 << 18, 64
    bk = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.I32, seed=51, perm_domain=2 * nb), nb)
    pk = gen.generate_cpu(gen.Spec(L.GEN_PROBE, L.I32, seed=51, stream_id=2, lo=nb, perm_domain=2 * nb,
                                   match_permille=100), npr)
    obk, _, bps = ops.part_kernel(ctx, dev(bk), shift=32, part_n=part_n)
    opk, oprow, pps = ops.part_kernel(ctx, dev(pk), shift=32, part_n=part_n)
    ctx.sync()
    f = ops.filter_kernel(ctx, obk, bps)
    res, kk, kr, sizes = ops.match_kernel(ctx, f, opk, pps, oprow)
    ctx.sync()
    c = int(res.item())
    kept = set(u32(kr[:c]).tolist())
    bset = set(bk.view(np.uint32).tolist())
    must = {i for i, k in enumerate(pk.view(np.uint32).tolist()) if k in bset}
    assert must <= kept
    # and the same result as the oracle on the partitioned inputs
    ek, ep, es = oracle.bloom_match(oracle.bloom_build(u32(obk), bps.cpu().numpy()), u32(opk),
                                    pps.cpu().numpy(), u32(oprow))
    assert np.array_equal(u32(kk[:c]), ek) and np.array_equal(u32(kr[:c]), ep)
    assert np.array_equal(sizes.cpu().numpy().view(np.uint64), es)


def test_bloom_filters_exchange_with_the_oracle(ctx):
    # filters built on the CPU (reference layout) probe on the GPU
    bk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=61, lo=0, hi=2**32 - 1), 20000)
    bps = np.array([0, 5000, 12000, 20000], np.uint64)
    pk = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=62, lo=0, hi=2**32 - 1), 50000)
    pk[::2] = bk[np.arange(0, 50000, 2) % 20000]
    pps = np.array([0, 10000, 30000, 50000], np.uint64)
    cpu_f = oracle.bloom_build(bk, bps)
    gk, gp, gs = run_match(ctx, torch.from_numpy(cpu_f).cuda(), pk, pps)
    ek, ep, es = oracle.bloom_match(cpu_f, pk, pps)
    assert np.array_equal(gk, ek) and np.array_equal(gp, ep) and np.array_equal(gs, es)


def test_bloom_empty_input(ctx):
    f = ops.filter_kernel(ctx, dev(np.zeros(1, np.uint32)), dev(np.zeros(3, np.uint64), np.int64))
    res, _, _, sizes = ops.match_kernel(ctx, f, dev(np.zeros(0, np.uint32)),
                                        dev(np.zeros(3, np.uint64), np.int64))
    ctx.sync()
    assert int(res.item()) == 0 and not sizes.any()
    assert not f.any()


def test_bloom_capacity_overflow_reports_error(ctx):
    k = np.arange(10000, dtype=np.uint32)
    ps = np.array([0, 10000], np.uint64)
    f = ops.filter_kernel(ctx, dev(k), dev(ps, np.int64))
    res, _, _, _ = ops.match_kernel(ctx, f, dev(k), dev(ps, np.int64), capacity=100)
    with pytest.raises(L.PimdalError) as e:
        ctx.sync()
    assert e.value.status == 7
    assert int(res.item()) == 10000
