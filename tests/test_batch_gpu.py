"""GPU parity of the batched form (pimdal_group_batch_create /
pimdal_hash_join_batch_create / pimdal_batch_run): every instance of a batch
returns exactly what the plain call returns for it (group-by rows identical,
bit-exact int64; hash-join pairs identical and in the same probe order), and
both match the oracle.  Covers ragged sizes, empty instances, signed and
unsigned keys, count-only group-bys, replays of a run and of a CUDA graph
that captured it, and the autotuner's cache."""
import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu


def cuda(a, dtype=np.int32):
    return torch.from_numpy(np.ascontiguousarray(a).view(dtype)).cuda()


def gb_instance(rng, i):
    n = int(rng.choice([0, 1, 7, 128, 1000, 4099, 20000, 65536, 100003, 300000]))
    card = int(rng.choice([1, 4, 16, 40, 300, 2000, 5000, 70000]))
    k = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=1000 + i, lo=0, hi=card - 1,
                                  perm_domain=0), n)
    v = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I64, seed=1000 + i, stream_id=1, lo=-10**12,
                                  hi=10**12), n)
    if i % 5 == 0 and n:
        k[::7] = -1  # the shared tables' empty marker
    dtype = L.U32 if i % 3 == 1 else L.I32
    with_vals = i % 4 != 3
    return k, (v if with_vals else None), card, dtype


def gb_outs(cap):
    outs = {w: torch.empty(cap, dtype=torch.int64, device="cuda") for w in ("sum", "count", "min", "max")}
    outs["key"] = torch.empty(cap, dtype=torch.int32, device="cuda")
    return outs


def gb_expected(k, v, dtype):
    exp = tuple(np.asarray(e) for e in oracle.group_by(k, v))  # ascending signed keys
    if dtype == L.U32:  # the same groups, ascending unsigned keys
        o = np.argsort(exp[0].view(np.uint32), kind="stable")
        exp = tuple(e[o] for e in exp)
        exp = (exp[0].view(np.uint32).astype(np.int64),) + exp[1:]
    return exp


def gb_got(outs, g, dtype):
    key = outs["key"][:g].cpu().numpy()
    if dtype == L.U32:
        key = key.view(np.uint32).astype(np.int64)
    return (key,) + tuple(outs[c][:g].cpu().numpy() for c in ("sum", "count", "min", "max"))


def build_group_batch(rng, count):
    inst, args = [], []
    for i in range(count):
        k, v, card, dtype = gb_instance(rng, i)
        kt = cuda(k)
        vt = None if v is None else cuda(v, np.int64)
        cap = max(1, min(len(k), card) + 8)
        outs = gb_outs(cap)
        inst.append((k, v, dtype, kt, vt, outs, card))
        args.append(ops.group_args(kt, vt, outs, expected_groups=card, key_dtype=dtype))
    return inst, args


def check_group_batch(ctx, inst, b):
    b.ctx.sync()
    res = b.results.cpu().numpy()
    for i, (k, v, dtype, kt, vt, outs, card) in enumerate(inst):
        g = int(res[i])
        got = gb_got(outs, g, dtype)
        exp = gb_expected(k, v, dtype)
        assert g == len(exp[0]), i
        for name, a, e in zip(("key", "sum", "count", "min", "max"), got, exp):
            assert np.array_equal(a, np.asarray(e)), (i, name)
        # and identical to the plain call
        r2, o2 = ops.group_kernel(ctx, kt, vt, method=L.GROUP_HASH, expected_groups=card,
                                  key_dtype=dtype, capacity=outs["key"].numel())
        ctx.sync()
        assert int(r2.item()) == g
        for c in ("key", "sum", "count", "min", "max"):
            assert torch.equal(o2[c][:g], outs[c][:g]), (i, c)


@pytest.mark.parametrize("rows_per_item", [128, 4096, 65536])
def test_group_batch_matches_plain_and_oracle(ctx, rows_per_item):
    rng = np.random.default_rng(7 + rows_per_item)
    inst, args = build_group_batch(rng, 24)
    t = L.BatchTuning(rows_per_item=rows_per_item, load_factor_pct=50)
    b = ops.Batch(ctx, L.BATCH_GROUP, args, tuning=t)
    b.run()
    check_group_batch(ctx, inst, b)
    b.close()


def hj_instance(i):
    nb = [0, 1, 100, 3000, 1 << 14, 50000][i % 6]
    npr = [0, 1, 5000, 4096, 40000, 200001][(i * 5 + 1) % 6]
    nb_eff = max(nb, 1)
    bk = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.I32, seed=2000 + i, perm_domain=2 * nb_eff), nb)
    bp = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=2000 + i, stream_id=1, lo=-2**31,
                                   hi=2**31 - 1), nb)
    pk = gen.generate_cpu(gen.Spec(L.GEN_PROBE, L.I32, seed=2000 + i, stream_id=2, lo=nb_eff,
                                   perm_domain=2 * nb_eff, match_permille=500), npr)
    if nb == 0:
        pk = pk[:npr]
    return bk, bp, pk


def build_join_batch(count):
    inst, args = [], []
    for i in range(count):
        bk, bp, pk = hj_instance(i)
        t = [cuda(bk), cuda(bp), cuda(pk)]
        cap = max(1, len(pk))
        pay = torch.empty(cap, dtype=torch.int32, device="cuda")
        row = torch.empty(cap, dtype=torch.int32, device="cuda")
        inst.append((bk, bp, pk, t, pay, row))
        args.append(ops.hash_join_args(t[0], t[1], t[2], None, pay, row))
    return inst, args


def check_join_batch(ctx, inst, b):
    b.ctx.sync()
    res = b.results.cpu().numpy()
    for i, (bk, bp, pk, t, pay, row) in enumerate(inst):
        c = int(res[i])
        epay, erow = oracle.hash_join(bk, bp, pk) if len(bk) and len(pk) else (np.zeros(0), np.zeros(0))
        assert c == len(epay), i
        gp = pay[:c].cpu().numpy().view(np.uint32)
        gr = row[:c].cpu().numpy().view(np.uint32)
        o1, o2 = np.lexsort((gp, gr)), np.lexsort((epay, erow))
        assert np.array_equal(gp[o1], np.asarray(epay)[o2]) and np.array_equal(gr[o1], np.asarray(erow)[o2])
        if len(bk) and len(pk):
            r2, p2, w2 = ops.hash_join(ctx, t[0], t[1], t[2], partition_bits=0xFFFFFFFF)
            ctx.sync()
            assert int(r2.item()) == c
            assert torch.equal(p2[:c], pay[:c]) and torch.equal(w2[:c], row[:c]), i


@pytest.mark.parametrize("rows_per_item,lf", [(128, 50), (65536, 70)])
def test_join_batch_matches_plain_and_oracle(ctx, rows_per_item, lf):
    inst, args = build_join_batch(18)
    for a in args:
        a.load_factor_pct = lf
    t = L.BatchTuning(rows_per_item=rows_per_item, load_factor_pct=lf)
    b = ops.Batch(ctx, L.BATCH_HASH_JOIN, args, tuning=t)
    b.run()
    check_join_batch(ctx, inst, b)
    b.close()


def test_batch_runs_replay_and_graph_capture(ctx):
    rng = np.random.default_rng(99)
    ginst, gargs = build_group_batch(rng, 10)
    jinst, jargs = build_join_batch(8)
    gb = ops.Batch(ctx, L.BATCH_GROUP, gargs)
    jb = ops.Batch(ctx, L.BATCH_HASH_JOIN, jargs)
    for _ in range(3):  # repeated runs: self-resetting queues, advancing epoch
        gb.run()
        jb.run()
    check_group_batch(ctx, ginst, gb)
    check_join_batch(ctx, jinst, jb)
    for _, _, _, _, _, outs, _ in ginst:
        for t in outs.values():
            t.zero_()
    for inst in jinst:
        inst[4].zero_()
        inst[5].zero_()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        gb.run(stream=s)
        jb.run(stream=s)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    check_group_batch(ctx, ginst, gb)
    check_join_batch(ctx, jinst, jb)
    del g
    gb.close()
    jb.close()


def test_autotune_caches_per_shape(ctx):
    rng = np.random.default_rng(5)
    inst, args = build_group_batch(rng, 6)
    best, cached = ops.Batch.autotune(ctx, L.BATCH_GROUP, args)
    assert not cached and best.rows_per_item in (16384, 65536, 262144)
    best2, cached2 = ops.Batch.autotune(ctx, L.BATCH_GROUP, args)
    assert cached2 and best2.rows_per_item == best.rows_per_item
    b = ops.Batch(ctx, L.BATCH_GROUP, args, tuning=best)
    b.run()
    check_group_batch(ctx, inst, b)
    b.close()
