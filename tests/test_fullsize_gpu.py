"""GPU parity at the configs' full sizes, against the oracle (not against the
library itself):

  * config 3 hash join: build 2^25 unique int32 keys + payloads, probe 2^28
    keys at a 50% match rate, uniform and Zipf(0.75) probes, and the
    uniform probe over 4096 shared-memory partitions -- the full
    multiset of (build payload, probe row id) equals the oracle's
    (reference/db_operators/hash_join.cpp:57-157 restated);
  * config 3 group-by: 2^28 rows at 16, 2^12 and 2^22 groups, hash and sort
    methods -- all five columns (key, SUM, COUNT, MIN, MAX) equal the
    oracle's (aggregate.cpp:40-83 restated, int64);
  * config 4 batched form: the 4096-instance batch (2048 group-bys, 2048
    hash joins, log-uniform sizes) -- every instance equals the oracle;
  * config 5 served form: 60 requests over the 6e7-row tables, fused and
    serial staged -- every request's groups equal a numpy restatement.

The oracle runs over disjoint key partitions in host threads
(oracle.group_by_parallel / hash_join_parallel, pinned to the serial oracle
in tests/test_oracle.py)."""
import os

import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops, serve

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, len(os.sched_getaffinity(0))))


def u32(t):
    return t.cpu().numpy().view(np.uint32)


def assert_join_equal(gpay, grow, epay, erow, n_probe):
    """(payload, probe row) multisets equal, probe rows unique on both sides
    (build keys are unique): compared through per-row arrays, O(n)."""
    assert gpay.size == epay.size
    seen_g = np.zeros(n_probe, bool)
    seen_g[grow] = True
    seen_e = np.zeros(n_probe, bool)
    seen_e[erow] = True
    assert np.count_nonzero(seen_g) == grow.size, "a probe row matched twice"
    assert np.array_equal(seen_g, seen_e)
    by_g = np.zeros(n_probe, np.uint32)
    by_g[grow] = gpay
    by_e = np.zeros(n_probe, np.uint32)
    by_e[erow] = epay
    assert np.array_equal(by_g, by_e)


@pytest.mark.parametrize("zipf,partition_bits", [(False, 0), (True, 0), (False, 12)],
                         ids=["uniform", "zipf0.75", "uniform-shared-memory-partitions"])
def test_hash_join_config3_matches_oracle(ctx, zipf, partition_bits):
    nb, npr = 1 << 25, 1 << 28
    s = 0xB200 + 2
    g = lambda spec, n: ops.gen_column(ctx, spec, n)
    bk = g(gen.Spec(L.GEN_PERM, L.I32, seed=s, perm_domain=2 * nb), nb)
    bp = g(gen.Spec(L.GEN_UNIFORM, L.I32, seed=s, stream_id=1, lo=-2**31, hi=2**31 - 1), nb)
    pk = g(gen.Spec(L.GEN_PROBE, L.I32, seed=s, stream_id=3 if zipf else 2, lo=nb,
                    perm_domain=2 * nb, match_permille=500,
                    cdf=gen.zipf_cdf(nb, 0.75) if zipf else None), npr)
    res, pay, row = ops.hash_join(ctx, bk, bp, pk, capacity=npr, partition_bits=partition_bits)
    ctx.sync()
    m = int(res.item())
    hb, hp, hk = u32(bk), u32(bp), u32(pk)
    gpay, grow = u32(pay[:m]), u32(row[:m])
    del bk, bp, pk, pay, row
    torch.cuda.empty_cache()
    epay, erow = oracle.hash_join_parallel(hb, hp, hk, threads=THREADS)
    assert 0.45 * npr < m < 0.55 * npr
    assert_join_equal(gpay, grow, epay, erow, npr)


@pytest.fixture(scope="module")
def group_values(ctx):
    n = 1 << 28
    v = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.I64, seed=0xB200 + 3, stream_id=1, lo=100,
                                     hi=10**7), n)
    yield v, v.cpu().numpy()
    del v
    torch.cuda.empty_cache()


@pytest.mark.parametrize("card_i,card", [(0, 16), (1, 1 << 12), (2, 1 << 22)])
def test_group_by_config3_matches_oracle(ctx, group_values, card_i, card):
    n = 1 << 28
    dv, hv = group_values
    keys = ops.gen_column(ctx, gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=0xB200 + 3,
                                        stream_id=10 + card_i, lo=0, hi=card - 1, perm_domain=0), n)
    hk = keys.cpu().numpy()
    exp = oracle.group_by_parallel(hk, hv, threads=THREADS)
    assert exp[0].size == card and int(exp[2].sum()) == n
    for method in (L.GROUP_HASH, L.GROUP_SORT):
        res, outs = ops.group_kernel(ctx, keys, dv, method=method, expected_groups=card,
                                     capacity=card + 8)
        ctx.sync()
        gcount = int(res.item())
        assert gcount == card, method
        for name, e in zip(("key", "sum", "count", "min", "max"), exp):
            assert np.array_equal(outs[name][:gcount].cpu().numpy(), e), (method, name)
        del outs
    del keys
    torch.cuda.empty_cache()


def batch_shapes():
    """The config-4 batch: 2048 group-by instances (rows log-U[2^10, 2^22],
    cardinality log-U[4, 2^16]) and 2048 hash joins (probe rows
    log-U[2^10, 2^22] over rows/4 unique build keys), seeded as the bench's."""
    rng = np.random.default_rng(0xB204)
    rows_g = np.rint(2.0 ** rng.uniform(10, 22, 2048)).astype(np.int64)
    card = np.rint(2.0 ** rng.uniform(2, 16, 2048)).astype(np.int64)
    rows_j = np.rint(2.0 ** rng.uniform(10, 22, 2048)).astype(np.int64)
    return rows_g, card, rows_j, np.maximum(rows_j // 4, 1)


def test_batch_config4_every_instance_matches_oracle(ctx):
    from concurrent.futures import ThreadPoolExecutor
    rows_g, card, rows_j, nbj = batch_shapes()
    s0 = 0xB200 + 4
    dev = "cuda"
    # group-by instances
    gin, gargs = [], []
    for i in range(rows_g.size):
        n, c = int(rows_g[i]), int(card[i])
        k = ops.gen_column(ctx, gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s0 + i, stream_id=1, lo=0,
                                         hi=c - 1, perm_domain=0), n)
        v = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.I64, seed=s0 + i, stream_id=2, lo=100,
                                         hi=10**7), n)
        outs = {w: torch.empty(c + 8, dtype=torch.int64, device=dev)
                for w in ("sum", "count", "min", "max")}
        outs["key"] = torch.empty(c + 8, dtype=torch.int32, device=dev)
        gin.append((k, v, outs))
        gargs.append(ops.group_args(k, v, outs, expected_groups=c))
    # hash-join instances
    jin, jargs = [], []
    for i in range(rows_j.size):
        nb, npr = int(nbj[i]), int(rows_j[i])
        sj = 1 << 20 | i
        bk = ops.gen_column(ctx, gen.Spec(L.GEN_PERM, L.I32, seed=s0 + sj, perm_domain=nb), nb)
        bp = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.I32, seed=s0 + sj, stream_id=1,
                                          lo=-2**31, hi=2**31 - 1), nb)
        pk = ops.gen_column(ctx, gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s0 + sj, stream_id=3,
                                          lo=0, hi=nb - 1, perm_domain=nb), npr)
        pay = torch.empty(npr, dtype=torch.int32, device=dev)
        row = torch.empty(npr, dtype=torch.int32, device=dev)
        jin.append((bk, bp, pk, pay, row))
        jargs.append(ops.hash_join_args(bk, bp, pk, None, pay, row))
    tg, _ = ops.Batch.autotune(ctx, L.BATCH_GROUP, gargs)
    tj, _ = ops.Batch.autotune(ctx, L.BATCH_HASH_JOIN, jargs)
    gb = ops.Batch(ctx, L.BATCH_GROUP, gargs, tuning=tg)
    jb = ops.Batch(ctx, L.BATCH_HASH_JOIN, jargs, tuning=tj)
    for _ in range(2):  # a second run: self-resetting queues, advanced epoch
        gb.run()
        jb.run()
    ctx.sync()
    rg, rj = gb.results.cpu().numpy(), jb.results.cpu().numpy()

    def check_group(i):
        k, v, outs = gin[i]
        exp = oracle.group_by(k.cpu().numpy(), v.cpu().numpy(), max_groups=int(card[i]))
        gcount = int(rg[i])
        if gcount != exp[0].size:
            return f"group {i}: {gcount} groups, oracle {exp[0].size}"
        for name, e in zip(("key", "sum", "count", "min", "max"), exp):
            if not np.array_equal(outs[name][:gcount].cpu().numpy(), e):
                return f"group {i}: column {name}"
        return None

    def check_join(i):
        bk, bp, pk, pay, row = jin[i]
        epay, erow = oracle.hash_join(u32(bk), u32(bp), u32(pk))
        m = int(rj[i])
        if m != epay.size:
            return f"join {i}: {m} matches, oracle {epay.size}"
        gp, gr = u32(pay[:m]), u32(row[:m])
        a, b = np.lexsort((gp, gr)), np.lexsort((epay, erow))
        if not (np.array_equal(gp[a], epay[b]) and np.array_equal(gr[a], erow[b])):
            return f"join {i}: pairs differ"
        return None

    with ThreadPoolExecutor(THREADS) as ex:
        bad = [e for e in ex.map(check_group, range(len(gin))) if e]
        bad += [e for e in ex.map(check_join, range(len(jin))) if e]
    gb.close()
    jb.close()
    assert not bad, bad[:5]


def test_served_config5_requests_match_numpy(ctx):
    t = serve.Tables(ctx)
    server = serve.Server(t, slots=8)
    server.warm()
    reqs = serve.make_requests(60, t.n, rate=None, seed=0xB209)
    served = server.run(reqs)                 # fused passes, 8 slots
    serial = server.run(reqs, serial=True)    # staged plain operators, one at a time
    assert served.max_inflight > 1
    assert serve.same_results(served, serial)
    h = {name: getattr(t, name).cpu().numpy() for name in
         ("l_date", "l_orderkey", "l_partkey", "l_price", "l_discount", "l_rflag", "l_lstatus",
          "o_key", "o_prio", "p_cat")}
    order = np.argsort(h["o_key"])
    okey_sorted, oprio_sorted = h["o_key"][order], h["o_prio"][order]
    for r in reqs:
        rows = np.arange(r.r0, r.r0 + r.n)
        rows = rows[(h["l_date"][rows] >= r.d0) & (h["l_date"][rows] <= r.d1)]
        if r.dim == 0:
            attr = oprio_sorted[np.searchsorted(okey_sorted, h["l_orderkey"][rows])]
            flag, nflag = h["l_rflag"][rows], serve.N_RFLAG
        else:
            attr = h["p_cat"][h["l_partkey"][rows] - 1]
            flag, nflag = h["l_lstatus"][rows], serve.N_LSTATUS
        key = attr.astype(np.int64) * (nflag if r.two_keys else 1) + (flag if r.two_keys else 0)
        val = h["l_price"][rows] * (100 - h["l_discount"][rows].astype(np.int64))
        uk, inv = np.unique(key, return_inverse=True)
        sums = np.zeros(uk.size, np.int64)
        np.add.at(sums, inv, val)
        cnt = np.bincount(inv, minlength=uk.size)
        got = served.results[r.rid]
        assert np.array_equal(got.keys, uk.astype(np.int32)), r.rid
        assert np.array_equal(got.sums, sums), r.rid
        assert np.array_equal(got.counts, cnt), r.rid
    server.close()
