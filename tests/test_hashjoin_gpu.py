"""GPU parity of K-PART / K-BUILD / K-PROBE and the hash join against the
oracle (bit-exact as multisets; probe order within a partition)."""
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


def inputs(nb, npr, seed, zipf=None, match=500):
    bk = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.I32, seed=seed, perm_domain=2 * nb), nb)
    bp = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=seed, stream_id=1, lo=-2**31, hi=2**31 - 1), nb)
    cdf = None if zipf is None else gen.zipf_cdf(nb, zipf)
    pk = gen.generate_cpu(gen.Spec(L.GEN_PROBE, L.I32, seed=seed, stream_id=2, lo=nb,
                                   perm_domain=2 * nb, match_permille=match, cdf=cdf), npr)
    return bk, bp, pk


def as_sorted_pairs(pay, row):
    o = np.lexsort((pay, row))
    return pay[o], row[o]


def check_join(ctx, bk, bp, pk, **kw):
    res, pay, row = ops.hash_join(ctx, cuda_i32(bk), cuda_i32(bp), cuda_i32(pk), **kw)
    ctx.sync()
    c = int(res.item())
    epay, erow = oracle.hash_join(bk, bp, pk)
    assert c == epay.size
    gp, gr = u32(pay[:c]), u32(row[:c])
    a, b = as_sorted_pairs(gp, gr), as_sorted_pairs(epay, erow)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    return gp, gr


@pytest.mark.parametrize("nb,npr", [(1, 1), (1, 1000), (100, 4097), (5000, 40000), (1 << 16, 1 << 20)])
def test_hash_join_direct(ctx, nb, npr):
    bk, bp, pk = inputs(nb, npr, 41)
    gp, gr = check_join(ctx, bk, bp, pk)
    # not partitioned: output in probe order
    assert np.all(np.diff(gr.astype(np.int64)) > 0)


@pytest.mark.parametrize("bits", [1, 3, 8])
def test_hash_join_partitioned(ctx, bits):
    bk, bp, pk = inputs(1 << 16, (1 << 20) + 3, 42)
    check_join(ctx, bk, bp, pk, partition_bits=bits)


@pytest.mark.parametrize("bits,zipf", [(9, None), (10, 0.75), (16, None)])
def test_hash_join_shared_memory_partitions(ctx, bits, zipf):
    bk, bp, pk = inputs(1 << 16, (1 << 20) + 5, 47, zipf=zipf)
    gp, gr = check_join(ctx, bk, bp, pk, partition_bits=bits)
    # partitions in order, probe order within each
    h = pk[gr].astype(np.uint32).astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    part = (h >> np.uint64(64 - bits)).astype(np.int64)
    assert np.all(np.diff(part * 2**32 + gr.astype(np.int64)) > 0)


def test_hash_join_shared_memory_partition_in_chunks(ctx):
    # 20000 build rows of one key fill one partition past a table's capacity:
    # the partition is joined one chunk of build rows at a time
    bk = np.concatenate([np.full(20000, 77, np.int32), np.arange(1000, 3000, dtype=np.int32)])
    bp = np.arange(bk.size, dtype=np.int32)
    pk = np.array([77, 5, 1500, 77, -1, 2999, 77], np.int32)
    check_join(ctx, bk, bp, pk, partition_bits=9, capacity=70000)


def test_hash_join_auto_partition_small_budget(ctx):
    bk, bp, pk = inputs(1 << 17, 1 << 20, 43, zipf=0.75)
    check_join(ctx, bk, bp, pk, l2_budget_bytes=1 << 18)


def test_hash_join_duplicate_build_keys_and_sentinel(ctx):
    # duplicate build keys (every match emitted) and the all-ones key/payload row
    bk = np.array([5, 5, 7, -1, -1, 9, 5], np.int32)
    bp = np.array([1, 2, 3, -1, 4, 5, 6], np.int32)
    pk = np.array([5, -1, 8, 7, 5, 9, -1], np.int32)
    res, pay, row = ops.hash_join(ctx, cuda_i32(bk), cuda_i32(bp), cuda_i32(pk), capacity=64)
    ctx.sync()
    c = int(res.item())
    got = sorted(zip(u32(row[:c]).tolist(), u32(pay[:c]).tolist()))
    exp = sorted((i, int(np.uint32(bp[j]))) for i, k in enumerate(pk) for j, b in enumerate(bk) if b == k)
    assert got == exp


@pytest.mark.parametrize("partition_bits", [0xFFFFFFFF, 3, 9])
def test_hash_join_sentinel_row_alone(ctx, partition_bits):
    # the all-ones key/payload row is the only build match of an all-ones probe
    # key: one match, whose payload is all ones
    bk = np.array([5, -1, 7, 9], np.int32)
    bp = np.array([1, -1, 3, 5], np.int32)
    pk = np.array([5, -1, 8, 7, -1, 9], np.int32)
    res, pay, row = ops.hash_join(ctx, cuda_i32(bk), cuda_i32(bp), cuda_i32(pk), capacity=64,
                                  partition_bits=partition_bits)
    ctx.sync()
    c = int(res.item())
    got = sorted(zip(u32(row[:c]).tolist(), u32(pay[:c]).tolist()))
    exp = sorted((i, int(np.uint32(bp[j]))) for i, k in enumerate(pk) for j, b in enumerate(bk) if b == k)
    assert got == exp


def test_hash_join_zipf_probe_and_match_rates(ctx):
    for match in (0, 1000):
        bk, bp, pk = inputs(4096, 100000, 44, zipf=0.75, match=match)
        check_join(ctx, bk, bp, pk)


def test_hash_kernel_and_probe_building_blocks(ctx):
    bk, bp, pk = inputs(3000, 50000, 45)
    table = ops.hash_kernel(ctx, cuda_i32(bk), cuda_i32(bp), table_size=8192)
    res, oo, oi = ops.hj_probe(ctx, table, 8192, cuda_i32(pk))
    ctx.sync()
    c = int(res.item())
    epay, erow = oracle.hash_join(bk, bp, pk)
    assert c == epay.size
    assert np.array_equal(u32(oo[:c]), np.sort(erow))  # probe order
    a = as_sorted_pairs(u32(oi[:c]), u32(oo[:c]))
    b = as_sorted_pairs(epay, erow)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_hash_table_full_is_reported(ctx):
    keys = np.arange(100, dtype=np.int32)
    ops.hash_kernel(ctx, cuda_i32(keys), None, table_size=128)
    ctx.sync()
    with pytest.raises(L.PimdalError):
        ops.hash_kernel(ctx, cuda_i32(np.arange(300, dtype=np.int32)), None, table_size=256)
        ctx.sync()


@pytest.mark.parametrize("part_n,shift", [(1, 32), (16, 32), (32, 27), (256, 20), (8192, 32)])
def test_part_kernel_matches_reference_partition(ctx, part_n, shift):
    k = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=46, lo=0, hi=2**32 - 1), 300007)
    out, optr, sizes = ops.part_kernel(ctx, cuda_i32(k), shift=shift, part_n=part_n)
    ctx.sync()
    ok, op, es = oracle.part_hash0(k, shift=shift, part_n=part_n)
    assert np.array_equal(sizes.cpu().numpy().view(np.uint64), es)
    assert np.array_equal(u32(out), ok) and np.array_equal(u32(optr), op)


def test_hash_join_config3_full_size(ctx):
    nb, npr = 1 << 25, 1 << 28
    bk = ops.gen_column(ctx, gen.Spec(L.GEN_PERM, L.I32, seed=0xB203, perm_domain=2 * nb), nb)
    pk = ops.gen_column(ctx, gen.Spec(L.GEN_PROBE, L.I32, seed=0xB203, stream_id=2, lo=nb,
                                      perm_domain=2 * nb, match_permille=500), npr)
    res, pay, row = ops.hash_join(ctx, bk, None, pk, capacity=npr)
    ctx.sync()
    c = int(res.item())
    assert abs(c / npr - 0.5) < 0.001
    # size-independent checks: every match pairs equal keys; probe rows unique
    pay_h = pay[:c].cpu().numpy().astype(np.int64)
    row_h = row[:c].cpu().numpy().astype(np.int64)
    bk_h, pk_h = bk.cpu().numpy(), pk.cpu().numpy()
    assert np.array_equal(bk_h[pay_h], pk_h[row_h])
    assert np.unique(row_h).size == c
    # the non-matching probe keys are exactly the ones not in the build set
    matched = np.zeros(npr, bool)
    matched[row_h] = True
    assert not np.isin(pk_h[~matched][:1000000], bk_h).any()
    del pay_h, row_h
