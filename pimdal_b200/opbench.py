"""Runs one operator on seeded device-resident inputs and prints its timing.

    python -m pimdal_b200.opbench select    --rows 16777216 --iters 20
    python -m pimdal_b200.opbench sort      --rows 67108864 [--zipf]
    python -m pimdal_b200.opbench smj       --rows 67108864          (inner = rows / 4)
    python -m pimdal_b200.opbench hash_join --rows 268435456         (build = rows / 8)
    python -m pimdal_b200.opbench group     --rows 268435456 --card 4096 --method hash|sort
    python -m pimdal_b200.opbench bloom     --rows 268435456 --parts 16384 --match-permille 50
                                             (build = rows / 8; both sides partitioned first,
                                              untimed; times filter + match)
    python -m pimdal_b200.opbench served    [--orders 15000000]      (one fused request of the
                                             served form over the whole lineitem table: dates
                                             in a quarter of the range, joined to the part
                                             attribute, revenue summed per attribute)
    python -m pimdal_b200.opbench tpch      --query q6|q1|q4|q3|q5 [--orders 15000000]
                                             (q6, q1: the fused pass over the lineitem-shaped
                                              table of the served form, about 4 rows per order;
                                              q4, q3, q5: the multi-table pipelines over it)

The per-operator counterpart of the reference's benchmark programs
(reference/db_operators/*.cpp main: generate, run the kernel a fixed number of
times, print the mean).  It is also the program the committed ncu summaries
profile: small row counts give captures that end in seconds.  Each iteration
is timed with CUDA events on the launching stream, all of them enqueued
behind a GPU sleep so that host-side launch overhead is not timed; the inputs
are generated on the device by the seeded generator (include/pimdal_gpu.h
pimdal_gen_column).
"""
from __future__ import annotations

import argparse
import json
import statistics

import torch

from . import _lib as L
from . import gen, ops


def _inputs(ctx: ops.Context, a) -> tuple:
    g = lambda spec, n: ops.gen_column(ctx, spec, n)
    n = a.rows
    if a.op == "select":
        return (g(gen.Spec(L.GEN_UNIFORM, L.I32, seed=a.seed, lo=0, hi=2**31 - 1), n),)
    if a.op == "sort":
        if a.zipf:
            spec = gen.Spec(L.GEN_PERM_ZIPF, L.U32, seed=a.seed, stream_id=1, perm_domain=0,
                            cdf=gen.zipf_cdf(1 << 24, 1.0))
        else:
            spec = gen.Spec(L.GEN_UNIFORM, L.U32, seed=a.seed, lo=0, hi=2**32 - 1)
        return g(spec, n), torch.arange(n, dtype=torch.int32, device=f"cuda:{ctx.device}")
    if a.op == "smj":
        nr = max(n // 4, 1)
        rk = g(gen.Spec(L.GEN_PERM, L.I32, seed=a.seed, perm_domain=nr), nr)
        sk = g(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=a.seed, stream_id=3, lo=0, hi=nr - 1,
                        perm_domain=nr), n)
        return rk, sk
    if a.op == "hash_join":
        nb = max(n // 8, 1)
        spec_p = gen.Spec(L.GEN_PROBE, L.I32, seed=a.seed, stream_id=2, lo=nb, perm_domain=2 * nb,
                          match_permille=500,
                          cdf=gen.zipf_cdf(nb, 0.75) if a.zipf else None)
        return (g(gen.Spec(L.GEN_PERM, L.I32, seed=a.seed, perm_domain=2 * nb), nb),
                g(gen.Spec(L.GEN_UNIFORM, L.I32, seed=a.seed, stream_id=1, lo=-2**31, hi=2**31 - 1), nb),
                g(spec_p, n))
    if a.op == "bloom":
        nb = max(n // 8, 1)
        bk = g(gen.Spec(L.GEN_PERM, L.I32, seed=a.seed, perm_domain=2 * nb), nb)
        pk = g(gen.Spec(L.GEN_PROBE, L.I32, seed=a.seed, stream_id=2, lo=nb, perm_domain=2 * nb,
                        match_permille=a.match_permille), n)
        obk, _, bps = ops.part_kernel(ctx, bk, shift=32, part_n=a.parts, want_ptr=False)
        opk, oprow, pps = ops.part_kernel(ctx, pk, shift=32, part_n=a.parts)
        ctx.sync()
        return obk, bps, opk, oprow, pps
    if a.op == "tpch":
        from . import serve, tpch
        li = tpch.Lineitem(ctx, serve.Tables(ctx, orders=a.orders))
        return (li, tpch.Schema(ctx, li) if a.query in ("q3", "q4", "q5") else None)
    if a.op == "served":
        from . import serve
        return (serve.Tables(ctx, orders=a.orders),)
    if a.op == "group":
        keys = g(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=a.seed, stream_id=10, lo=0,
                          hi=a.card - 1, perm_domain=0), n)
        vals = g(gen.Spec(L.GEN_UNIFORM, L.I64, seed=a.seed, stream_id=1, lo=100, hi=10**7), n)
        return keys, vals
    raise SystemExit(f"unknown operator {a.op}")


def _runner(ctx: ops.Context, a, inp):
    n = a.rows
    dev = f"cuda:{ctx.device}"
    if a.op == "select":
        pred = ops.make_pred(L.PRED_LT, 214748364)
        out, ptr = torch.empty_like(inp[0]), torch.empty_like(inp[0])
        res = torch.empty(1, dtype=torch.int64, device=dev)
        return lambda: ops.sel_kernel(ctx, inp[0], pred, out=out, out_ptr=ptr, result=res)
    if a.op == "sort":
        out, ptr = torch.empty_like(inp[0]), torch.empty_like(inp[0])
        return lambda: ops.sort_kernel(ctx, inp[0], inp[1], out=out, out_ptr=ptr)
    if a.op == "smj":
        oi = torch.empty(n, dtype=torch.int32, device=dev)
        oo = torch.empty(n, dtype=torch.int32, device=dev)
        res = torch.empty(1, dtype=torch.int64, device=dev)
        return lambda: ops.sort_merge_join(ctx, inp[0], None, inp[1], None, out_inner=oi,
                                           out_outer=oo, result=res)
    if a.op == "hash_join":
        op = torch.empty(n, dtype=torch.int32, device=dev)
        orow = torch.empty(n, dtype=torch.int32, device=dev)
        res = torch.empty(1, dtype=torch.int64, device=dev)
        return lambda: ops.hash_join(ctx, inp[0], inp[1], inp[2], capacity=n, out_payload=op,
                                     out_row=orow, result=res, partition_bits=a.partition_bits,
                                     load_factor_pct=a.load_factor)
    if a.op == "bloom":
        obk, bps, opk, oprow, pps = inp
        filt = torch.empty(a.parts * L.FILTER_BYTES, dtype=torch.uint8, device=dev)
        ok = torch.empty(n, dtype=torch.int32, device=dev)
        orow = torch.empty(n, dtype=torch.int32, device=dev)
        res = torch.empty(1, dtype=torch.int64, device=dev)

        def bloom():
            ops.filter_kernel(ctx, obk, bps, filters=filt)
            ops.match_kernel(ctx, filt, opk, pps, oprow, out=ok, out_row=orow, result=res)
        bloom.result = res
        return bloom
    if a.op == "served":
        from . import serve
        t = inp[0]
        a.rows = t.l_date.numel()
        col, table, tsize, _, _ = t.dim(0)
        res = torch.empty(1, dtype=torch.int64, device=dev)
        d0 = serve.DAYS // 8
        return lambda: ops.select_join_aggregate(ctx, t.l_date, d0, d0 + serve.DAYS // 4, col, table,
                                                 tsize, t.l_price, t.l_discount,
                                                 key_space=t.n_attr(0), result=res)
    if a.op == "tpch":
        from . import tpch
        li, schema = inp
        a.rows = li.n
        res = torch.empty(1, dtype=torch.int64, device=dev)
        if schema is not None:  # the multi-table pipelines: chains of plain operators
            return lambda: getattr(tpch, a.query)(ctx, schema)
        if a.query == "q6":
            preds, exprs = tpch.q6_args(li)
            run = lambda: ops.select_aggregate(ctx, li.n, preds=preds, exprs=exprs, result=res)
        else:
            pred, group, exprs = tpch.q1_args(li)
            run = lambda: ops.select_aggregate(ctx, li.n, preds=[pred], group=group,
                                               key_space=tpch.N_RFLAG * tpch.N_LSTATUS,
                                               exprs=exprs, result=res)
        return run
    method = {"hash": L.GROUP_HASH, "sort": L.GROUP_SORT, "auto": L.GROUP_AUTO}[a.method]
    cap = 2 * a.card
    outs = {w: torch.empty(cap, dtype=torch.int64, device=dev) for w in ("sum", "count", "min", "max")}
    outs["key"] = torch.empty(cap, dtype=torch.int32, device=dev)
    res = torch.empty(1, dtype=torch.int64, device=dev)
    return lambda: ops.group_kernel(ctx, inp[0], inp[1], method=method, expected_groups=a.card,
                                    capacity=cap, outs=outs, result=res)


def main(argv=None) -> None:
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("op", choices=["select", "sort", "smj", "hash_join", "group", "bloom", "tpch",
                                  "served"])
    p.add_argument("--rows", type=int, default=1 << 24)
    p.add_argument("--iters", type=int, default=10)
    p.add_argument("--warmup", type=int, default=2)
    p.add_argument("--seed", type=int, default=0xB200)
    p.add_argument("--zipf", action="store_true", help="Zipf keys (sort: s=1.0, hash_join: s=0.75)")
    p.add_argument("--card", type=int, default=4096, help="group cardinality")
    p.add_argument("--method", default="hash", choices=["hash", "sort", "auto"])
    p.add_argument("--partition-bits", type=int, default=0,
                   help="hash join: 0 = auto, 4294967295 = never partition, else 1..8")
    p.add_argument("--load-factor", type=int, default=0, help="hash join table load factor, percent")
    p.add_argument("--parts", type=int, default=16384, help="bloom: partitions (power of 2)")
    p.add_argument("--match-permille", type=int, default=50, help="bloom: probe match rate")
    p.add_argument("--query", default="q6", choices=["q6", "q1", "q4", "q3", "q5"],
                   help="tpch: the query")
    p.add_argument("--orders", type=int, default=15_000_000, help="tpch, served: orders of the table")
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--kernels", action="store_true",
                   help="also print the mean time of each library kernel class")
    a = p.parse_args(argv)
    torch.cuda.set_device(a.device)
    ctx = ops.Context(a.device)
    inp = _inputs(ctx, a)
    run = _runner(ctx, a, inp)
    for _ in range(a.warmup):
        run()
    ctx.sync()
    stream = torch.cuda.current_stream()
    names = {getattr(L, k): k[len("KERNEL_"):].lower() for k in dir(L)
             if k.startswith("KERNEL_") and k != "KERNEL_COUNT"}
    if a.kernels:
        for k in names:
            ctx.kernel_time(k)  # reset
        ctx.set_profiling(True)
    # All iterations are enqueued behind a GPU sleep, so the host's launch
    # path (Python, ctypes) never leaves the GPU idle inside a timed region.
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(a.iters)]
    torch.cuda._sleep(int(2e8))
    for e0, e1 in evs:
        e0.record(stream)
        run()
        e1.record(stream)
    ctx.sync()
    times = [e0.elapsed_time(e1) for e0, e1 in evs]
    kernels = None
    if a.kernels:
        ctx.set_profiling(False)
        kernels = {}
        for k, nm in sorted(names.items()):
            n, ms = ctx.kernel_time(k)
            if n:
                kernels[nm] = {"launches_per_iter": n / max(a.iters, 1), "ms_per_iter": ms / max(a.iters, 1)}
    med = statistics.median(times) if times else float("nan")
    print(json.dumps({"op": a.op, "rows": a.rows, "iters": a.iters, "zipf": a.zipf,
                      "card": a.card if a.op == "group" else None,
                      "method": a.method if a.op == "group" else None,
                      "ms_median": med, "ms_min": min(times) if times else None,
                      "rows_per_s": a.rows / (med * 1e-3) if times else None,
                      "kept": int(run.result.item()) if hasattr(run, "result") else None,
                      "kernels": kernels}))


if __name__ == "__main__":
    main()
