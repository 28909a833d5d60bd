#!/usr/bin/env python3
"""Benchmark of the pimdal_b200 operators on one node (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sort_smj|select|...]

Prints ONE JSON line (rank 0).  A "step" is one pass of the workload's
operators over one batch of synthetic input already resident in HBM.  Every
rank runs the same workload on its own GPU (independent replicas: the
operators shard by rows with no data-path exchange), so `value` is the sum
of the ranks' rows over the max over ranks of the device time.

  value  = input rows / s over the timed steps (CUDA events per step on the
           launching stream; L2 flushed between steps by writing 256 MiB)
  e2e    = the same metric through the public API with host buffers: pinned
           host inputs copied in and outputs copied back inside the region
  roofline   = the dominant kernel's algorithmic bytes per launch / its mean
               launch duration (CUDA events recorded by the library on the
               launching stream), against MEASURED_PEAKS.json hbm_gbs
  cpu_baseline = the reference's own CPU operators (oracle/_ref, all host
               threads) on a bounded sample of the same workload, rank 0
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0

# DRAM traffic of a dominant kernel per unit it processes, from one committed
# ncu capture (dram__bytes_read.sum + dram__bytes_write.sum of the captured
# launch divided by its units).  A full-size launch's traffic is this figure
# times its units: each kernel streams its input once per unit, so traffic
# grows in proportion to the units processed.
NCU_TRAFFIC = {
    "k_sort_pass": ((268.9e6 + 217.8e6) / 2**25, "pair",
                    "profiles/k_sort_pass_2p25_pairs.md"),
    "k_select_coop": ((537.0e6 + 39.6e6) / 2**26, "row",
                      "profiles/k_select_coop_2p26.md (2^26 rows; at 2^24 the second read hits L2)"),
    "k_hj_probe": ((339.5e6 + 90.9e6) / 2**25, "partitioned probe row",
                   "profiles/k_hj_probe_2p25_probe.md"),
    "k_gb_aggregate_shared": ((403.1e6 + 5.9e6) / 2**25, "row",
                              "profiles/k_gb_aggregate_2p25_rows.md (4096 groups)"),
    "k_gb_aggregate_direct": ((3528.9e6 + 874.8e6) / 2**25, "row",
                              "profiles/k_gb_aggregate_2p25_rows.md (2^22 groups)"),
    "k_smj_merge": ((336.1e6 + 215.0e6) / 2**25, "outer row",
                    "profiles/k_smj_merge_2p25_outer.md"),
    "k_gb_chunks": ((424.5e6 + 7.8e6) / 2**25, "row",
                    "profiles/k_gb_chunks_2p25_rows.md (chunk aggregation after partitioning)"),
}


def ncu_traffic(kernel: str, units: float) -> dict | None:
    """Traffic of one launch over `units` units, scaled from the capture."""
    if kernel not in NCU_TRAFFIC:
        return None
    per, unit, src = NCU_TRAFFIC[kernel]
    return {"bytes": round(per * units), "per_unit": round(per, 3), "unit": unit, "source": src}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def hbm_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks / throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        self.file.flush()

    def summary(self) -> dict:
        rows = []
        try:
            for line in Path(self.file.name).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.file.name)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
class Workload:
    name = ""
    config = {}
    rows_per_step = 0
    dominant = None            # kernel id for the roofline
    dominant_name = ""
    traffic_per_launch = None  # bytes, from the committed ncu summary

    def setup(self, ctx, dev):  # device-resident inputs + pinned host copies
        raise NotImplementedError

    def step(self):             # inputs resident in HBM
        raise NotImplementedError

    def step_e2e(self, stream):  # host inputs -> device -> host outputs
        raise NotImplementedError

    def algorithmic_bytes_per_launch(self) -> float:
        raise NotImplementedError

    def cpu_sample(self, ref, threads, budget_s):  # -> (rows, seconds, description)
        raise NotImplementedError


class SelectWorkload(Workload):
    """Selection over 2^24 int32 values U[0, 2^31), predicate v < 214748364."""
    name = "select"
    N = 1 << 24

    def __init__(self):
        from pimdal_b200 import _lib as L
        from pimdal_b200 import gen
        self.spec = gen.Spec(L.GEN_UNIFORM, L.I32, seed=0xB200, lo=0, hi=2**31 - 1)
        self.config = {"workload": "selection 2^24 int32 U[0,2^31), v < 214748364 (~10%)",
                       "rows": self.N, "l2": "flushed between steps (input 64 MiB < L2)"}
        self.rows_per_step = self.N
        self.dominant = L.KERNEL_SELECT
        self.dominant_name = "k_select"

    def setup(self, ctx, dev):
        import torch
        from pimdal_b200 import _lib as L
        from pimdal_b200 import gen, ops
        self.ctx, self.ops, self.L = ctx, ops, L
        self.spec = gen.Spec(L.GEN_UNIFORM, L.I32, seed=0xB200, lo=0, hi=2**31 - 1)
        self.keys = ops.gen_column(ctx, self.spec, self.N)
        self.pred = ops.make_pred(L.PRED_LT, 214748364)
        self.out = torch.empty_like(self.keys)
        self.out_ptr = torch.empty_like(self.keys)
        self.res = torch.empty(1, dtype=torch.int64, device=dev)
        self.h_keys = torch.from_numpy(gen.generate_cpu(self.spec, self.N)).pin_memory()
        self.h_out = torch.empty(self.N, dtype=torch.int32).pin_memory()
        self.h_ptr = torch.empty(self.N, dtype=torch.int32).pin_memory()
        self.h_cnt = torch.empty(1, dtype=torch.int64).pin_memory()
        self.d_in2 = torch.empty_like(self.keys)
        ops.sel_kernel(ctx, self.keys, self.pred, out=self.out, out_ptr=self.out_ptr, result=self.res)
        ctx.sync()
        self.count = int(self.res.item())

    def step(self):
        self.ops.sel_kernel(self.ctx, self.keys, self.pred, out=self.out, out_ptr=self.out_ptr,
                            result=self.res)

    def step_e2e(self, stream):
        self.d_in2.copy_(self.h_keys, non_blocking=True)
        self.ops.sel_kernel(self.ctx, self.d_in2, self.pred, out=self.out, out_ptr=self.out_ptr,
                            result=self.res)
        self.h_cnt.copy_(self.res, non_blocking=True)
        k = self.count  # output size is known from setup (same input every step)
        self.h_out[:k].copy_(self.out[:k], non_blocking=True)
        self.h_ptr[:k].copy_(self.out_ptr[:k], non_blocking=True)
        return 4 * self.N, 8 + 8 * k

    def algorithmic_bytes_per_launch(self):
        return 4 * self.N + 8 * self.count

    def cpu_sample(self, ref, threads, budget_s):
        from pimdal_b200 import gen
        n = self.N
        if not hasattr(self, "_cpu_keys"):
            self._cpu_keys = gen.generate_cpu(self.spec, n)
            ref.set_threads("select", threads)
            ref.select(self._cpu_keys, -2**63, 214748364 - 1)
        reps = 0
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < budget_s or reps < 1:
            ref.select(self._cpu_keys, -2**63, 214748364 - 1)
            reps += 1
        dt = time.perf_counter() - t0
        return n * reps, dt, f"reference select() body (select.cpp:77-100) on the full 2^24 column x{reps}"


class SortSmjWorkload(Workload):
    """Stable radix sort of 2^26 (uint32 key, uint32 row id) pairs with uniform
    32-bit keys and with Zipf(1.0) keys over 2^24 distinct values, then the
    sort-merge join of R = 2^24 unique int32 keys (a permutation of
    0..2^24-1) with int32 payloads against S = 2^26 keys drawn uniformly from
    R's keys with int32 payloads.  One step runs all three.  The sorts' row
    ids are the row index, made on the device by the sort (in_ptr = NULL), as
    the reference's sort program makes them on the DPU from the uploaded keys
    (create_ptr, pimdal/main/sort/dpu/kernel_sort.c:32-36,73)."""
    name = "sort_smj"
    N = 1 << 26
    NR = 1 << 24
    NS = 1 << 26

    def __init__(self):
        from pimdal_b200 import _lib as L
        from pimdal_b200 import gen
        self.L = L
        s = 0xB200 + 1
        self.spec_u = gen.Spec(L.GEN_UNIFORM, L.U32, seed=s, lo=0, hi=2**32 - 1)
        self.spec_z = gen.Spec(L.GEN_PERM_ZIPF, L.U32, seed=s, stream_id=1, perm_domain=0,
                               cdf=None)
        self.spec_rk = gen.Spec(L.GEN_PERM, L.I32, seed=s, perm_domain=self.NR)
        self.spec_rp = gen.Spec(L.GEN_UNIFORM, L.I32, seed=s, stream_id=2, lo=-2**31, hi=2**31 - 1)
        self.spec_sk = gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s, stream_id=3, lo=0,
                                hi=self.NR - 1, perm_domain=self.NR)
        self.spec_sp = gen.Spec(L.GEN_UNIFORM, L.I32, seed=s, stream_id=4, lo=-2**31, hi=2**31 - 1)
        self.config = {
            "workload": "radix sort 2^26 (uint32 key, uint32 row id) pairs, uniform keys and "
                        "Zipf(1.0) over 2^24 keys; sort-merge join R=2^24 unique int32 keys + "
                        "int32 payload vs S=2^26 keys uniform over R + int32 payload; the sorts' "
                        "row ids are the row index, generated on the device",
            "sort_rows": self.N, "smj_inner_rows": self.NR, "smj_outer_rows": self.NS,
            "l2": "inputs larger than L2 (512 MiB per sorted array); L2 also flushed between steps"}
        self.rows_per_step = 2 * self.N + self.NR + self.NS
        self.dominant = L.KERNEL_SORT_PASS
        self.dominant_name = "k_sort_pass (onesweep digit pass)"

    def setup(self, ctx, dev):
        import torch
        from pimdal_b200 import gen, ops
        self.ctx, self.ops = ctx, ops
        self.spec_z.cdf = gen.zipf_cdf(1 << 24, 1.0)
        g = lambda spec, n: ops.gen_column(ctx, spec, n)
        self.ku, self.kz = g(self.spec_u, self.N), g(self.spec_z, self.N)
        self.rk, self.rp = g(self.spec_rk, self.NR), g(self.spec_rp, self.NR)
        self.sk, self.sp = g(self.spec_sk, self.NS), g(self.spec_sp, self.NS)
        e = lambda n: torch.empty(n, dtype=torch.int32, device=dev)
        self.ou, self.oup, self.oz, self.ozp = e(self.N), e(self.N), e(self.N), e(self.N)
        self.ji, self.jo = e(self.NS), e(self.NS)
        self.res = torch.empty(1, dtype=torch.int64, device=dev)
        self.step()
        ctx.sync()
        assert int(self.res.item()) == self.NS
        # pinned host copies for the end-to-end run
        pin = lambda t: t.cpu().pin_memory()
        self.h_in = [pin(t) for t in (self.ku, self.kz, self.rk, self.rp, self.sk, self.sp)]
        self.d_in2 = [torch.empty_like(t) for t in (self.ku, self.kz, self.rk, self.rp, self.sk,
                                                    self.sp)]
        self.h_out = [torch.empty(t.numel(), dtype=t.dtype).pin_memory()
                      for t in (self.ou, self.oup, self.oz, self.ozp, self.ji, self.jo)]
        # algorithmic bytes of the digit passes of one step: 16 B per pair per
        # active pass (uniform and Zipf keys: 4 passes; R and S keys < 2^24: 3),
        # less the row ids the first pass of each index-id sort does not read
        pairs = 4 * self.N + 4 * self.N + 3 * self.NR + 3 * self.NS
        self.pass_bytes = 16 * pairs - 4 * 2 * self.N
        self.active_passes = 4 + 4 + 3 + 3
        t = ncu_traffic("k_sort_pass", pairs / self.active_passes)
        self.traffic_per_launch = t["bytes"]
        self.traffic_source = t

    def release(self):
        """Drops the device and pinned buffers (the per-operator suite runs next)."""
        for name in ("ku", "kz", "rows", "rk", "rp", "sk", "sp", "ou", "oup", "oz", "ozp", "ji",
                     "jo", "h_in", "d_in2", "h_out", "_streams"):
            if hasattr(self, name):
                delattr(self, name)

    def _run(self, ku, kz, rk, rp, sk, sp):
        ops = self.ops
        ops.sort_kernel(self.ctx, ku, None, out=self.ou, out_ptr=self.oup)
        ops.sort_kernel(self.ctx, kz, None, out=self.oz, out_ptr=self.ozp)
        ops.sort_merge_join(self.ctx, rk, rp, sk, sp, out_inner=self.ji, out_outer=self.jo,
                            result=self.res)

    def step(self):
        self._run(self.ku, self.kz, self.rk, self.rp, self.sk, self.sp)

    def step_e2e(self, stream):
        """Pinned host inputs -> device -> pinned host outputs through the public
        API, pipelined over three streams ordered by events: the upload of an
        operator's inputs, the previous operator's compute and the download of
        an earlier operator's outputs overlap (PCIe is full duplex).  The sorts
        upload their keys only (the row ids are made on the device) and
        download sorted keys and row ids; the join uploads keys and payloads
        and downloads the (R payload, S payload) pairs."""
        import torch
        if not hasattr(self, "_streams"):
            self._streams = [torch.cuda.Stream() for _ in range(3)]
        up, comp, down = self._streams
        ops, ctx, d = self.ops, self.ctx, self.d_in2
        start = torch.cuda.Event()
        start.record(stream)
        for s in self._streams:
            s.wait_event(start)
        outs = (self.ou, self.oup, self.oz, self.ozp, self.ji, self.jo)
        plan = [((0,), (0, 1)), ((1,), (2, 3)), ((2, 3, 4, 5), (4, 5))]
        for g, (ins, outs_idx) in enumerate(plan):
            with torch.cuda.stream(up):
                for i in ins:
                    d[i].copy_(self.h_in[i], non_blocking=True)
            e_in = torch.cuda.Event()
            e_in.record(up)
            comp.wait_event(e_in)
            if g == 0:
                ops.sort_kernel(ctx, d[0], None, out=self.ou, out_ptr=self.oup, stream=comp)
            elif g == 1:
                ops.sort_kernel(ctx, d[1], None, out=self.oz, out_ptr=self.ozp, stream=comp)
            else:
                ops.sort_merge_join(ctx, d[2], d[3], d[4], d[5], out_inner=self.ji,
                                    out_outer=self.jo, result=self.res, stream=comp)
            e_c = torch.cuda.Event()
            e_c.record(comp)
            down.wait_event(e_c)
            with torch.cuda.stream(down):
                for o in outs_idx:
                    self.h_out[o].copy_(outs[o], non_blocking=True)
        end = torch.cuda.Event()
        end.record(down)
        stream.wait_event(end)
        h2d = sum(t.numel() * 4 for t in self.h_in)
        d2h = sum(t.numel() * 4 for t in self.h_out)
        return h2d, d2h

    def roofline_bytes(self, launches: int, steps: int) -> float:
        """Algorithmic bytes of all digit-pass launches of the timed region."""
        return self.pass_bytes * steps

    def algorithmic_bytes_per_launch(self):
        return self.pass_bytes / self.active_passes

    SMJ_BUFFER = 67112000  # the reference SMJ's BUFFER_SIZE: smallest multiple of 8000 >= 2^26

    def cpu_sample(self, ref, threads, budget_s):
        """The full workload on the host cores, one whole step per repetition
        (at least one; more while the budget lasts): the reference's
        sort_kernel (sort.cpp:30-40) on the 2^26 uniform and the 2^26 Zipf
        (key, row id) pairs -- packed into the harness's 64-bit pair words
        before the timed region, so the timed call is the reference kernel
        alone -- and the reference's sort_merge_join_kernel
        (sort_merge_join.cpp:48-103) on the 2^24 R keys and 2^26 S keys (key
        columns, as the reference joins; its merge cursor races with more
        than one thread, which is the code as shipped).  The same seeded
        inputs as the GPU arm."""
        from pimdal_b200 import gen
        if not hasattr(self, "_cpu"):
            self.spec_z.cdf = gen.zipf_cdf(1 << 24, 1.0)
            pu = ref.pack_pairs(gen.generate_cpu(self.spec_u, self.N))
            pz = ref.pack_pairs(gen.generate_cpu(self.spec_z, self.N))
            rk = gen.generate_cpu(self.spec_rk, self.NR).view(np.uint32)
            sk = gen.generate_cpu(self.spec_sk, self.NS).view(np.uint32)
            out = np.empty(self.N, np.uint64)
            self._cpu = (pu, pz, rk, sk, out, 2 * self.N + self.NR + self.NS)
            for lib in ("sort", f"smj_{self.SMJ_BUFFER}"):
                ref.set_threads(lib, threads)
        pu, pz, rk, sk, out, rows = self._cpu
        reps = 0
        dt = 0.0
        while reps < 1 or dt < budget_s:
            t0 = time.perf_counter()
            ref.sort_packed(pu, out)
            ref.sort_packed(pz, out)
            ref.smj(rk, sk, self.SMJ_BUFFER, threads=threads)
            dt += time.perf_counter() - t0
            reps += 1
        return rows * reps, dt, (
            "full config: reference sort_kernel (sort.cpp:30-40) on 2^26 uniform and 2^26 Zipf "
            "(key, row id) pairs packed before the timed region + sort_merge_join_kernel "
            f"(sort_merge_join.cpp:48-103) on 2^24 x 2^26 keys, x{reps}")


class HashJoinWorkload(Workload):
    """Hash join: build 2^25 unique int32 keys (a seeded sample of [0, 2^26))
    with int32 payloads, probe 2^28 int32 keys at a 50% match rate, uniform
    and Zipf(0.75) probe variants.  One step runs both joins."""
    name = "hash_join"
    NB = 1 << 25
    NP = 1 << 28

    def __init__(self):
        from pimdal_b200 import _lib as L
        from pimdal_b200 import gen
        self.L = L
        s = 0xB200 + 2
        self.spec_bk = gen.Spec(L.GEN_PERM, L.I32, seed=s, perm_domain=2 * self.NB)
        self.spec_bp = gen.Spec(L.GEN_UNIFORM, L.I32, seed=s, stream_id=1, lo=-2**31, hi=2**31 - 1)
        self.spec_pu = gen.Spec(L.GEN_PROBE, L.I32, seed=s, stream_id=2, lo=self.NB,
                                perm_domain=2 * self.NB, match_permille=500)
        self.spec_pz = gen.Spec(L.GEN_PROBE, L.I32, seed=s, stream_id=3, lo=self.NB,
                                perm_domain=2 * self.NB, match_permille=500)
        self.config = {"workload": "hash join build 2^25 unique int32 keys + int32 payload, "
                                   "probe 2^28 int32 keys at 50% match, uniform and Zipf(0.75)",
                       "build_rows": self.NB, "probe_rows": self.NP,
                       "l2": "inputs larger than L2; L2 also flushed between steps"}
        self.rows_per_step = 2 * (self.NB + self.NP)
        self.dominant = L.KERNEL_HJ_PROBE
        self.dominant_name = "k_hj_probe"

    def setup(self, ctx, dev):
        import torch
        from pimdal_b200 import gen, ops
        self.ctx, self.ops = ctx, ops
        self.spec_pz.cdf = gen.zipf_cdf(self.NB, 0.75)
        g = lambda spec, n: ops.gen_column(ctx, spec, n)
        self.bk, self.bp = g(self.spec_bk, self.NB), g(self.spec_bp, self.NB)
        self.pu, self.pz = g(self.spec_pu, self.NP), g(self.spec_pz, self.NP)
        e = lambda n: torch.empty(n, dtype=torch.int32, device=dev)
        self.op, self.orow = e(self.NP), e(self.NP)
        self.res = [torch.empty(1, dtype=torch.int64, device=dev) for _ in range(2)]
        self.step()
        ctx.sync()
        self.matches = [int(r.item()) for r in self.res]
        pin = lambda t: t.cpu().pin_memory()
        self.h_in = [pin(t) for t in (self.bk, self.bp, self.pu, self.pz)]
        self.d_in2 = [torch.empty_like(t) for t in (self.bk, self.bp, self.pu, self.pz)]
        self.h_out = [torch.empty(self.NP, dtype=torch.int32).pin_memory() for _ in range(2)]

    def _run(self, bk, bp, pu, pz):
        for i, pk in enumerate((pu, pz)):
            self.ops.hash_join(self.ctx, bk, bp, pk, capacity=self.NP, out_payload=self.op,
                               out_row=self.orow, result=self.res[i])

    def step(self):
        self._run(self.bk, self.bp, self.pu, self.pz)

    def step_e2e(self, stream):
        for d, h in zip(self.d_in2, self.h_in):
            d.copy_(h, non_blocking=True)
        self._run(*self.d_in2)
        k = self.matches[1]
        self.h_out[0][:k].copy_(self.op[:k], non_blocking=True)
        self.h_out[1][:k].copy_(self.orow[:k], non_blocking=True)
        return sum(t.numel() * 4 for t in self.h_in), 8 * k + 16

    def roofline_bytes(self, launches: int, steps: int) -> float:
        # all probe launches of a step: 4 B per probe row + 8 B per match
        return steps * sum(4 * self.NP + 8 * m for m in self.matches)

    def algorithmic_bytes_per_launch(self):
        return sum(4 * self.NP + 8 * m for m in self.matches)

    def cpu_sample(self, ref, threads, budget_s):
        from pimdal_b200 import gen
        if not hasattr(self, "_cpu"):
            nb, npr = self.NB // 16, self.NP // 16
            bk = gen.generate_cpu(gen.Spec(self.L.GEN_PERM, self.L.I32, seed=9, perm_domain=2 * nb), nb)
            bp = gen.generate_cpu(self.spec_bp, nb)
            pk = gen.generate_cpu(gen.Spec(self.L.GEN_PROBE, self.L.I32, seed=9, stream_id=2, lo=nb,
                                           perm_domain=2 * nb, match_permille=500), npr)
            self._cpu = (bk, bp, pk, nb + npr)
            ref.set_threads("hash_join", threads)
        bk, bp, pk, rows = self._cpu
        reps = 0
        t0 = time.perf_counter()
        while reps < 1 or time.perf_counter() - t0 < budget_s:
            ref.hash_join(bk, bp, pk)
            reps += 1
        return rows * reps, time.perf_counter() - t0, (
            f"reference partition + join_partitions (hash_join.cpp:57-157) on 2^21 build x "
            f"2^24 probe rows (1/16 sample), x{reps}")


class GroupByWorkload(Workload):
    """Group-by over 2^28 rows (int32 key, int64 value U[100, 1e7]) at group
    cardinality 16, 2^12 and 2^22, hash and sort methods: one step runs the
    six group-bys."""
    name = "group_by"
    N = 1 << 28
    CARDS = (16, 1 << 12, 1 << 22)

    def __init__(self):
        from pimdal_b200 import _lib as L
        from pimdal_b200 import gen
        self.L = L
        s = 0xB200 + 3
        self.spec_k = [gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s, stream_id=10 + i, lo=0, hi=c - 1,
                                perm_domain=0) for i, c in enumerate(self.CARDS)]
        self.spec_v = gen.Spec(L.GEN_UNIFORM, L.I64, seed=s, stream_id=1, lo=100, hi=10**7)
        self.config = {"workload": "group-by 2^28 rows int32 key + int64 value U[100,1e7], "
                                   "cardinality 16 / 2^12 / 2^22, hash and sort methods",
                       "rows": self.N, "cardinalities": list(self.CARDS),
                       "l2": "inputs larger than L2; L2 also flushed between steps"}
        self.rows_per_step = 6 * self.N
        self.dominant = L.KERNEL_GROUP
        self.dominant_name = "k_gb_aggregate (hash method)"

    def setup(self, ctx, dev):
        import torch
        from pimdal_b200 import gen, ops
        self.ctx, self.ops = ctx, ops
        self.keys = [ops.gen_column(ctx, sp, self.N) for sp in self.spec_k]
        self.vals = ops.gen_column(ctx, self.spec_v, self.N)
        cap = 2 * max(self.CARDS)
        self.outs = {w: torch.empty(cap, dtype=torch.int64, device=dev)
                     for w in ("sum", "count", "min", "max")}
        self.outs["key"] = torch.empty(cap, dtype=torch.int32, device=dev)
        self.res = torch.empty(1, dtype=torch.int64, device=dev)
        self.step()
        ctx.sync()
        pin = lambda t: t.cpu().pin_memory()
        self.h_in = [pin(t) for t in self.keys] + [pin(self.vals)]
        self.d_in2 = [torch.empty_like(t) for t in self.keys] + [torch.empty_like(self.vals)]
        self.h_cnt = torch.empty(1, dtype=torch.int64).pin_memory()
        self.h_sum = torch.empty(max(self.CARDS), dtype=torch.int64).pin_memory()

    def _run(self, keys, vals):
        for k, c in zip(keys, self.CARDS):
            for m in (self.L.GROUP_HASH, self.L.GROUP_SORT):
                self.ops.group_kernel(self.ctx, k, vals, method=m, expected_groups=c,
                                      capacity=2 * max(self.CARDS), outs=self.outs,
                                      result=self.res)

    def step(self):
        self._run(self.keys, self.vals)

    def step_e2e(self, stream):
        for d, h in zip(self.d_in2, self.h_in):
            d.copy_(h, non_blocking=True)
        self._run(self.d_in2[:3], self.d_in2[3])
        g = max(self.CARDS)
        self.h_cnt.copy_(self.res, non_blocking=True)
        self.h_sum[:g].copy_(self.outs["sum"][:g], non_blocking=True)
        return sum(t.numel() * t.element_size() for t in self.h_in), 8 + 8 * g

    def roofline_bytes(self, launches: int, steps: int) -> float:
        # hash-method aggregation launches: 12 B per row (key + value)
        return launches * 12 * self.N

    def algorithmic_bytes_per_launch(self):
        return 12 * self.N

    def cpu_sample(self, ref, threads, budget_s):
        from pimdal_b200 import gen
        if not hasattr(self, "_cpu"):
            n = self.N // 64
            ks = [gen.generate_cpu(sp, n) for sp in self.spec_k]
            v = gen.generate_cpu(self.spec_v, n)
            self._cpu = (ks, v, 3 * n)
            ref.set_threads("aggregate", threads)
        ks, v, rows = self._cpu
        reps = 0
        t0 = time.perf_counter()
        while reps < 1 or time.perf_counter() - t0 < budget_s:
            for k in ks:
                ref.group_by(k, v)
            reps += 1
        return rows * reps, time.perf_counter() - t0, (
            f"reference hash_table_aggregate (aggregate.cpp:40-83) with int64 SUM/COUNT/MIN/MAX "
            f"on 2^22 rows x 3 cardinalities (1/64 sample), x{reps}")


class BatchWorkload(Workload):
    """Batched form: 2048 group-by instances (int32 key, int64 value
    U[100, 1e7], rows log-uniform over 2^10..2^22, group cardinality
    log-uniform over 4..2^16) and 2048 hash-join instances (rows log-uniform
    over 2^10..2^22 probe keys drawn uniformly from the build relation of
    rows/4 unique int32 keys with int32 payloads).  Each operator kind is one
    autotuned plan; both runs are captured in one CUDA graph and a step is one
    replay.  The same 4096 instances as plain launches (one
    pimdal_group_kernel / pimdal_hash_join call each) are timed beside it and
    every instance's output is compared."""
    name = "batch"
    NG = 2048
    NJ = 2048

    def __init__(self):
        from pimdal_b200 import _lib as L
        self.L = L
        rng = np.random.default_rng(0xB204)
        self.rows_g = np.rint(2.0 ** rng.uniform(10, 22, self.NG)).astype(np.int64)
        self.card = np.rint(2.0 ** rng.uniform(2, 16, self.NG)).astype(np.int64)
        self.rows_j = np.rint(2.0 ** rng.uniform(10, 22, self.NJ)).astype(np.int64)
        self.nb = np.maximum(self.rows_j // 4, 1)
        self.config = {
            "workload": "batched: 2048 group-by instances (int32 key + int64 value U[100,1e7], "
                        "rows log-U[2^10,2^22], cardinality log-U[4,2^16]) + 2048 hash joins "
                        "(probe rows log-U[2^10,2^22] uniform over rows/4 unique build keys), "
                        "one autotuned plan per operator, CUDA-graph replay per step",
            "instances": self.NG + self.NJ, "group_rows": int(self.rows_g.sum()),
            "join_probe_rows": int(self.rows_j.sum()), "join_build_rows": int(self.nb.sum()),
            "l2": "inputs larger than L2 (GBs per step); L2 also flushed between steps"}
        self.rows_per_step = int(self.rows_g.sum() + self.rows_j.sum() + self.nb.sum())
        self.dominant = L.KERNEL_GROUP
        self.dominant_name = "k_gbb_aggregate (batched group-by aggregation)"

    @staticmethod
    def _slices(lengths, align=4):
        offs, o = [], 0
        for n in lengths:
            offs.append(o)
            o += (int(n) + align - 1) // align * align
        return offs, o

    def setup(self, ctx, dev):
        import torch
        from pimdal_b200 import gen, ops
        L = self.L
        self.ctx, self.ops = ctx, ops
        s0 = 0xB200 + 4
        og, tg = self._slices(self.rows_g)
        self.gk = torch.empty(tg, dtype=torch.int32, device=dev)
        self.gv = torch.empty(tg, dtype=torch.int64, device=dev)
        ocap, tcap = self._slices(self.card + 8)
        outs = lambda: {**{w: torch.empty(tcap, dtype=torch.int64, device=dev)
                           for w in ("sum", "count", "min", "max")},
                        "key": torch.empty(tcap, dtype=torch.int32, device=dev)}
        self.gouts, self.pgouts = outs(), outs()
        self.gin, gargs = [], []
        for i in range(self.NG):
            n, c, o = int(self.rows_g[i]), int(self.card[i]), og[i]
            k, v = self.gk[o:o + n], self.gv[o:o + n]
            ops.gen_column(ctx, gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s0 + i, stream_id=1,
                                         lo=0, hi=c - 1, perm_domain=0), n, out=k)
            ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.I64, seed=s0 + i, stream_id=2, lo=100,
                                         hi=10**7), n, out=v)
            sl = lambda d: {w: t[ocap[i]:ocap[i] + c + 8] for w, t in d.items()}
            self.gin.append((k, v, c, sl(self.gouts), sl(self.pgouts)))
            gargs.append(ops.group_args(k, v, self.gin[-1][3], expected_groups=c))
        ob, tb = self._slices(self.nb)
        op, tp = self._slices(self.rows_j)
        self.bk = torch.empty(tb, dtype=torch.int32, device=dev)
        self.bp = torch.empty(tb, dtype=torch.int32, device=dev)
        self.pk = torch.empty(tp, dtype=torch.int32, device=dev)
        self.jpay, self.jrow = [torch.empty(tp, dtype=torch.int32, device=dev) for _ in range(2)]
        self.pjpay, self.pjrow = [torch.empty(tp, dtype=torch.int32, device=dev) for _ in range(2)]
        self.jin, jargs = [], []
        for i in range(self.NJ):
            nb, npr = int(self.nb[i]), int(self.rows_j[i])
            b = slice(ob[i], ob[i] + nb)
            q = slice(op[i], op[i] + npr)
            sj = 1 << 20 | i
            ops.gen_column(ctx, gen.Spec(L.GEN_PERM, L.I32, seed=s0 + sj, perm_domain=nb), nb,
                           out=self.bk[b])
            ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.I32, seed=s0 + sj, stream_id=1,
                                         lo=-2**31, hi=2**31 - 1), nb, out=self.bp[b])
            ops.gen_column(ctx, gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s0 + sj, stream_id=3,
                                         lo=0, hi=nb - 1, perm_domain=nb), npr, out=self.pk[q])
            self.jin.append((self.bk[b], self.bp[b], self.pk[q], self.jpay[q], self.jrow[q],
                             self.pjpay[q], self.pjrow[q]))
            jargs.append(ops.hash_join_args(self.bk[b], self.bp[b], self.pk[q], None,
                                            self.jpay[q], self.jrow[q]))
        ctx.sync()
        # autotune each plan on these instances, then capture both runs
        self.tune_g, _ = ops.Batch.autotune(ctx, L.BATCH_GROUP, gargs)
        self.tune_j, _ = ops.Batch.autotune(ctx, L.BATCH_HASH_JOIN, jargs)
        self.gb = ops.Batch(ctx, L.BATCH_GROUP, gargs, tuning=self.tune_g)
        self.jb = ops.Batch(ctx, L.BATCH_HASH_JOIN, jargs, tuning=self.tune_j)
        l0 = ctx.launches
        self.gb.run()
        self.jb.run()
        ctx.sync()
        self.launches_per_step = ctx.launches - l0  # kernels in one replay of the graph
        self.capture_stream = torch.cuda.Stream()
        self.graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with torch.cuda.graph(self.graph, stream=self.capture_stream):
            self.gb.run(stream=self.capture_stream)
            self.jb.run(stream=self.capture_stream)
        torch.cuda.synchronize()
        self.step()
        ctx.sync()
        self._compare_plain(dev)

    def _plain(self, res_g, res_j):
        L, ops, ctx = self.L, self.ops, self.ctx
        for i, (k, v, c, _, po) in enumerate(self.gin):
            ops.group_kernel(ctx, k, v, method=L.GROUP_HASH, expected_groups=c, capacity=c + 8,
                             outs=po, result=res_g[i:i + 1])
        for i, (bk, bp, pk, _, _, ppay, prow) in enumerate(self.jin):
            ops.hash_join(ctx, bk, bp, pk, capacity=pk.numel(), partition_bits=0xFFFFFFFF,
                          out_payload=ppay, out_row=prow, result=res_j[i:i + 1])

    def _compare_plain(self, dev):
        """Times the 4096 plain launches (CUDA events on the launching stream,
        L2 flushed before) and compares every instance with the batched run."""
        import torch
        res_g = torch.zeros(self.NG, dtype=torch.int64, device=dev)
        res_j = torch.zeros(self.NJ, dtype=torch.int64, device=dev)
        self._plain(res_g, res_j)  # warm-up: workspace, first launches
        self.ctx.sync()
        flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
        times = []
        for _ in range(2):
            flush.fill_(3)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self._plain(res_g, res_j)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        self.ctx.sync()
        rg, rj = self.gb.results[:self.NG], self.jb.results[:self.NJ]
        same = 0
        for i, (_, _, c, bo, po) in enumerate(self.gin):
            g = int(res_g[i])
            ok = g == int(rg[i]) and all(torch.equal(bo[w][:g], po[w][:g]) for w in bo)
            same += ok
        for i, (_, _, _, pay, row, ppay, prow) in enumerate(self.jin):
            m = int(res_j[i])
            ok = m == int(rj[i]) and torch.equal(pay[:m], ppay[:m]) and torch.equal(row[:m], prow[:m])
            same += ok
        ms = min(times)
        # the plain calls' device-busy time: every library kernel's duration
        # (its CUDA events on the launching stream), summed -- what the 4096
        # calls cost without the host's launch gaps between them
        for k in range(self.L.KERNEL_COUNT):
            self.ctx.kernel_time(k)
        self.ctx.set_profiling(True)
        self._plain(res_g, res_j)
        self.ctx.sync()
        self.ctx.set_profiling(False)
        busy = sum(self.ctx.kernel_time(k)[1] for k in range(self.L.KERNEL_COUNT))
        self.plain = {"ms_per_step": round(ms, 3),
                      "value": round(self.rows_per_step / (ms / 1e3), 1), "unit": "rows/s",
                      "device_busy_ms": round(busy, 3),
                      "host_overhead_ms": round(max(0.0, ms - busy), 3),
                      "launches": "4096 plain operator calls (pimdal_group_kernel, "
                                  "pimdal_hash_join unpartitioned), eager from Python",
                      "bit_exact_instances": f"{same}/{self.NG + self.NJ}"}

    def close(self):
        del self.graph
        self.gb.close()
        self.jb.close()

    def step(self):
        self.graph.replay()

    def dominant_timing(self):
        """(launches, ms) of the batched aggregation kernel over one eager run."""
        self.ctx.kernel_time(self.L.KERNEL_GROUP)
        self.ctx.set_profiling(True)
        self.gb.run()
        self.ctx.sync()
        self.ctx.set_profiling(False)
        return self.ctx.kernel_time(self.L.KERNEL_GROUP)

    def roofline_bytes(self, launches: int, steps: int) -> float:
        return launches * 12 * float(self.rows_g.sum())

    def algorithmic_bytes_per_launch(self):
        return 12 * float(self.rows_g.sum())

    def extra(self) -> dict:
        t = lambda b: {"rows_per_item": b.rows_per_item, "load_factor_pct": b.load_factor_pct}
        return {"plain_launches": self.plain,
                "autotuned": {"group_by": t(self.tune_g), "hash_join": t(self.tune_j)}}

    def step_e2e(self, stream):
        """Pinned host inputs -> device, graph replay, outputs -> pinned host."""
        import torch
        if not hasattr(self, "_h_in"):
            pin = lambda t: torch.empty(t.numel(), dtype=t.dtype, pin_memory=True).copy_(t)
            self._d_in = [self.gk, self.gv, self.bk, self.bp, self.pk]
            self._h_in = [pin(t) for t in self._d_in]
            self._d_out = [self.gouts[w] for w in ("key", "sum", "count", "min", "max")] + \
                          [self.jpay, self.jrow, self.gb.results, self.jb.results]
            self._h_out = [torch.empty(t.numel(), dtype=t.dtype, pin_memory=True) for t in self._d_out]
        for d, h in zip(self._d_in, self._h_in):
            d.copy_(h, non_blocking=True)
        self.graph.replay()
        for d, h in zip(self._d_out, self._h_out):
            h.copy_(d, non_blocking=True)
        return (sum(t.numel() * t.element_size() for t in self._h_in),
                sum(t.numel() * t.element_size() for t in self._h_out))

    def cpu_sample(self, ref, threads, budget_s):
        """The reference CPU group-by and hash join over the first instances
        of the batch (as many as fit the budget, at least one of each)."""
        from pimdal_b200 import gen
        L = self.L
        s0 = 0xB200 + 4
        if not hasattr(self, "_cpu"):
            self._cpu = []
            for i in range(8):
                n, c = int(self.rows_g[i]), int(self.card[i])
                k = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s0 + i, stream_id=1,
                                              lo=0, hi=c - 1, perm_domain=0), n)
                v = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I64, seed=s0 + i, stream_id=2,
                                              lo=100, hi=10**7), n)
                nb, npr = int(self.nb[i]), int(self.rows_j[i])
                sj = 1 << 20 | i
                bk = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.I32, seed=s0 + sj, perm_domain=nb), nb)
                bp = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=s0 + sj, stream_id=1,
                                               lo=-2**31, hi=2**31 - 1), nb)
                pk = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s0 + sj, stream_id=3,
                                               lo=0, hi=nb - 1, perm_domain=nb), npr)
                self._cpu.append((k, v, bk, bp, pk))
            ref.set_threads("aggregate", threads)
            ref.set_threads("hash_join", threads)
        rows = reps = 0
        t0 = time.perf_counter()
        while reps < 1 or time.perf_counter() - t0 < budget_s:
            for k, v, bk, bp, pk in self._cpu:
                ref.group_by(k, v)
                ref.hash_join(bk, bp, pk)
                rows += k.size + bk.size + pk.size
            reps += 1
        return rows, time.perf_counter() - t0, (
            f"reference hash_table_aggregate (aggregate.cpp:40-83) and partition + join "
            f"(hash_join.cpp:57-157) over the batch's first 8 group-by and 8 join instances, x{reps}")


class ServeWorkload(Workload):
    """Served form: filter -> join -> group-by pipelines over a resident
    lineitem-shaped fact table (about 6e7 rows: orderkey with 1-7 rows per
    order over 1.5e7 orders, partkey U[1,2e6], suppkey U[1,1e5], quantity,
    price cents U[90000,10500000], discount U[0,10], date over 2557 days, two
    flags) and two dimensions (1.5e7 orders, 2e6 parts), request row ranges
    log-uniform in [1e5, 6e7], date selectivity 1-50%, 8 concurrency slots
    under a 150 GB HBM budget.  A step is one saturated stream of 200 requests
    (all arrived at the start), each run as one fused filter-join-group-by
    pass; the same stream run serially through the staged plain operators (one
    request at a time), the concurrent staged run, and a Poisson stream at 70%
    of the serial throughput are measured beside it."""
    name = "serve"
    R = 200
    SLOTS = 8
    metric_name = "queries/s"
    unit = "queries/s"

    def __init__(self, requests: int | None = None):
        from pimdal_b200 import _lib as L
        self.L = L
        if requests:
            self.R = requests
        self.config = {"workload": "served filter->join->group-by pipelines (SUM(price*(100-discount)), "
                                   "COUNT by 1-2 keys) over a 6e7-row fact table + 1.5e7 / 2e6-row "
                                   "dimensions, ranges log-U[1e5,6e7], selectivity U[1%,50%]",
                       "requests_per_step": self.R, "slots": self.SLOTS, "hbm_budget_gb": 150,
                       "l2": "inputs (resident tables, GBs) larger than L2"}
        self.units_per_step = self.R
        self.dominant = L.KERNEL_FUSED
        self.dominant_name = "k_sja_aggregate (fused filter-join-group-by pass)"

    def setup(self, ctx, dev):
        import torch
        from pimdal_b200 import serve
        self.serve = serve
        self.tables = serve.Tables(ctx)
        self.server = serve.Server(self.tables, device=ctx.device, slots=self.SLOTS)
        self.server.warm()
        self.reqs = serve.make_requests(self.R, self.tables.n, rate=None, seed=0xB206)
        self.rows_per_step = sum(r.n for r in self.reqs)
        self.config["fact_rows"] = self.tables.n
        self._runs = []

    def step(self):
        import torch
        l0 = sum(sl.ctx.launches for sl in self.server.slots)
        st = self.server.run(self.reqs)
        # kernels of this step (the slots launch through their own contexts)
        self.launches_per_step = sum(sl.ctx.launches for sl in self.server.slots) - l0
        cur = torch.cuda.current_stream()
        for sl in self.server.slots:
            cur.wait_stream(sl.stream)
        self._runs.append(st)

    def dominant_timing(self):
        """(launches, ms) of the fused pass over one served run (profiled)."""
        for sl in self.server.slots:
            sl.ctx.kernel_time(self.dominant)
            sl.ctx.set_profiling(True)
        st = self.server.run(self.reqs)
        n = ms = 0
        for sl in self.server.slots:
            sl.ctx.sync(sl.stream)
            sl.ctx.set_profiling(False)
            a, b = sl.ctx.kernel_time(self.dominant)
            n += a
            ms += b
        self._sel_rows = sum(r.n for r in self.reqs)
        return n, ms

    def roofline_bytes(self, launches: int, steps: int) -> float:
        # the date column of every request's range (4 B per row); outputs are small
        return 4.0 * self._sel_rows * steps

    def algorithmic_bytes_per_launch(self):
        return 4.0 * self.rows_per_step / self.R

    def extra(self) -> dict:
        serve = self.serve
        served = self._runs[-1]
        serial = self.server.run(self.reqs, serial=True)
        ser = serial.summary()
        rate = 0.7 * ser["queries_per_s"]
        pois = serve.make_requests(self.R, self.tables.n, rate=rate, seed=0xB207)
        p_served = self.server.run(pois).summary()
        p_serial = self.server.run(pois, serial=True).summary()
        staged = self.server.run(self.reqs, fused=False)
        same = serve.same_results(served, serial) and serve.same_results(staged, serial)
        stg = staged.summary()
        return {"requests_per_arm": self.R,
                "served_saturated": served.summary(), "serial_saturated": ser,
                "served_staged_saturated": stg,
                "poisson": {"rate_per_s": round(rate, 2), "served": p_served, "serial": p_serial,
                            "p99_served_over_serial": round(p_served["p99_ms"] / p_serial["p99_ms"], 3)},
                "served_equals_serial": same,
                "speedup_vs_serial": round(served.summary()["queries_per_s"] / ser["queries_per_s"], 3),
                "speedup_staged_concurrency_only": round(stg["queries_per_s"] / ser["queries_per_s"], 3)}

    def close(self):
        self.server.close()

    def step_e2e(self, stream):
        """A served run: request parameters in kernel arguments, each result
        (groups) copied to pinned host memory; the tables stay resident."""
        import torch
        st = self.server.run(self.reqs)
        for sl in self.server.slots:
            stream.wait_stream(sl.stream)
        d2h = sum(r.keys.nbytes + r.sums.nbytes + r.counts.nbytes + 24 for r in st.results.values())
        return 0, d2h

    def cpu_sample(self, ref, threads, budget_s):
        """The reference's CPU operators composed per request: select over the
        date range (select.cpp), hash join of the selected join keys against
        the dimension (hash_join.cpp), hash aggregation (aggregate.cpp); the
        gathers between them in numpy."""
        serve = self.serve if hasattr(self, "serve") else __import__("pimdal_b200.serve").serve
        if not hasattr(self, "_cpu"):
            import torch
            from pimdal_b200 import ops
            ctx = ops.Context(0) if torch.cuda.is_available() else None
            t = self.tables if hasattr(self, "tables") else serve.Tables(ctx)
            c = lambda x: x.cpu().numpy()
            self._cpu = dict(date=c(t.l_date), okey=c(t.l_orderkey), pkey=c(t.l_partkey),
                             price=c(t.l_price), disc=c(t.l_discount), rflag=c(t.l_rflag),
                             lstat=c(t.l_lstatus), o_key=c(t.o_key), o_prio=c(t.o_prio),
                             p_key=c(t.p_key), p_cat=c(t.p_cat), n=t.n)
            self._cpu_reqs = serve.make_requests(64, t.n, rate=None, seed=0xB208)
            for lib in ("select", "hash_join", "aggregate"):
                ref.set_threads(lib, threads)
        d = self._cpu
        done = rows = 0
        t0 = time.perf_counter()
        for r in self._cpu_reqs:
            if done and time.perf_counter() - t0 >= budget_s:
                break
            dates = d["date"][r.r0:r.r0 + r.n]
            ref.select(dates, r.d0, r.d1)  # the reference's filter (values only)
            rows_sel = r.r0 + np.flatnonzero((dates >= r.d0) & (dates <= r.d1))
            if r.dim == 0:
                jk, bk, bp, flag, nf = d["okey"][rows_sel], d["o_key"], d["o_prio"], d["rflag"], 3
            else:
                jk, bk, bp, flag, nf = d["pkey"][rows_sel], d["p_key"], d["p_cat"], d["lstat"], 2
            pay, prow = ref.hash_join(bk, bp, jk.astype(np.int32))
            sel = rows_sel[prow.astype(np.int64)]
            key = pay.astype(np.int64) * (nf if r.two_keys else 1) + (flag[sel] if r.two_keys else 0)
            val = d["price"][sel] * (100 - d["disc"][sel].astype(np.int64))
            ref.group_by(key.astype(np.int32), val)
            done += 1
            rows += r.n
        return done, time.perf_counter() - t0, (
            f"reference select (select.cpp:77-100), partition + join (hash_join.cpp:57-157) and "
            f"hash_table_aggregate (aggregate.cpp:40-83) composed per request, numpy gathers "
            f"between them, {done} requests of the served mix")


# ---------------------------------------------------------------------------
# per-operator records of the default run: every config beside the headline
# ---------------------------------------------------------------------------
def _timed(fn, iters, flush, stream) -> list[float]:
    """Device milliseconds of each of `iters` calls of fn, the L2 flushed
    (256 MiB written) before each call, outside its events.  All calls are
    enqueued behind a GPU sleep, so host-side launch gaps are not timed."""
    import torch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(iters)]
    torch.cuda._sleep(int(1e8))
    for i, (e0, e1) in enumerate(evs):
        flush.fill_(i)
        e0.record(stream)
        fn()
        e1.record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs]


def _kernel_split(ctx, fn, iters=3) -> dict:
    """Mean device milliseconds per call of each library kernel class (the
    library's own CUDA events on the launching stream)."""
    from pimdal_b200 import _lib as L
    names = {getattr(L, k): k[len("KERNEL_"):].lower() for k in dir(L)
             if k.startswith("KERNEL_") and k != "KERNEL_COUNT"}
    for k in names:
        ctx.kernel_time(k)
    ctx.set_profiling(True)
    for _ in range(iters):
        fn()
    ctx.sync()
    ctx.set_profiling(False)
    out = {}
    for k, nm in sorted(names.items()):
        n, ms = ctx.kernel_time(k)
        if n:
            out[nm] = {"launches": round(n / iters, 2), "ms": round(ms / iters, 4)}
    return out


def _op_record(rows, times, alg_bytes, peak, split=None, dominant=None, dom_bytes=None,
               traffic=None) -> dict:
    """rows/s, GB/s and roofline fraction of the whole operator (median of the
    timed calls), and of its dominant kernel where one is named."""
    med = statistics.median(times)
    gbs = alg_bytes / (med * 1e-3) / 1e9
    rec = {"rows": int(rows), "ms": round(med, 4), "ms_min": round(min(times), 4),
           "calls": len(times), "rows_per_s": round(rows / (med * 1e-3), 1),
           "algorithmic_bytes": int(alg_bytes), "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    if split is not None:
        rec["kernels_ms"] = split
    if dominant and split and dominant in split:
        kms = split[dominant]["ms"]
        k = {"kernel_class": dominant, "ms": kms, "share": round(kms / med, 3)}
        if dom_bytes:
            kg = dom_bytes / (kms * 1e-3) / 1e9
            k.update({"algorithmic_bytes": int(dom_bytes), "gbs": round(kg, 1),
                      "frac": round(kg / peak, 4)})
        if traffic:
            k["traffic"] = traffic
            if dom_bytes:
                k["traffic_over_algorithmic"] = round(traffic["bytes"] / dom_bytes, 3)
        rec["dominant"] = k
    return rec


def per_operator(ctx, dev, peak, iters=7) -> dict:
    """The operators of configs 1, 3, 4 and 5 (and config 2's parts), each on
    its config's full-size seeded inputs, measured in this run."""
    import torch
    from pimdal_b200 import _lib as L
    from pimdal_b200 import gen, ops
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    out = {}
    g = lambda spec, n: ops.gen_column(ctx, spec, n)
    e32 = lambda n: torch.empty(n, dtype=torch.int32, device=dev)
    res = torch.empty(1, dtype=torch.int64, device=dev)

    # ---- config 1: selection 2^24 int32 U[0, 2^31), v < 214748364 ----------
    n = 1 << 24
    keys = g(gen.Spec(L.GEN_UNIFORM, L.I32, seed=0xB200, lo=0, hi=2**31 - 1), n)
    pred = ops.make_pred(L.PRED_LT, 214748364)
    o1, o2 = e32(n), e32(n)
    run = lambda: ops.sel_kernel(ctx, keys, pred, out=o1, out_ptr=o2, result=res)
    run()
    ctx.sync()
    k = int(res.item())
    t = _timed(run, 20, flush, stream)
    alg = 4 * n + 8 * k
    out["select_cfg1"] = dict(_op_record(n, t, alg, peak, _kernel_split(ctx, run), "select", alg,
                                         ncu_traffic("k_select_coop", n)), selected=k)
    del keys, o1, o2

    # ---- config 2, by operator ----------------------------------------------
    n = 1 << 26
    for name, spec in (("sort_uniform_cfg2", gen.Spec(L.GEN_UNIFORM, L.U32, seed=0xB201, lo=0,
                                                      hi=2**32 - 1)),
                       ("sort_zipf_cfg2", gen.Spec(L.GEN_PERM_ZIPF, L.U32, seed=0xB201, stream_id=1,
                                                   perm_domain=0, cdf=gen.zipf_cdf(1 << 24, 1.0)))):
        keys = g(spec, n)
        rows = torch.arange(n, dtype=torch.int32, device=dev)
        ok, op = e32(n), e32(n)
        run = lambda: ops.sort_kernel(ctx, keys, rows, out=ok, out_ptr=op)
        run()
        t = _timed(run, iters, flush, stream)
        split = _kernel_split(ctx, run)
        passes = split.get("sort_pass", {}).get("launches", 4)
        out[name] = _op_record(n, t, 16 * n, peak, split, "sort_pass", 16 * n * passes,
                               ncu_traffic("k_sort_pass", n * passes))
        del keys, rows, ok, op

    # ---- config 3: hash join, build 2^25 / probe 2^28, uniform and Zipf(0.75)
    nb, npr = 1 << 25, 1 << 28
    s3 = 0xB200 + 2
    bk = g(gen.Spec(L.GEN_PERM, L.I32, seed=s3, perm_domain=2 * nb), nb)
    bp = g(gen.Spec(L.GEN_UNIFORM, L.I32, seed=s3, stream_id=1, lo=-2**31, hi=2**31 - 1), nb)
    opay, orow = e32(npr), e32(npr)
    for name, sid, cdf in (("hash_join_uniform_cfg3", 2, None),
                           ("hash_join_zipf_cfg3", 3, gen.zipf_cdf(nb, 0.75))):
        pk = g(gen.Spec(L.GEN_PROBE, L.I32, seed=s3, stream_id=sid, lo=nb, perm_domain=2 * nb,
                        match_permille=500, cdf=cdf), npr)
        # the autotuner picks the partition fan-out and load factor for this
        # shape (the Zipf probe has the uniform one's shape: the cached choice)
        tuning, _, _, _, _ = ops.hash_join_autotune(ctx, bk, bp, pk, capacity=npr,
                                                    out_payload=opay, out_row=orow, result=res)
        run = lambda: ops.hash_join(ctx, bk, bp, pk, capacity=npr, out_payload=opay,
                                    out_row=orow, result=res)
        run()
        ctx.sync()
        m = int(res.item())
        t = _timed(run, iters, flush, stream)
        split = _kernel_split(ctx, run)
        alg = 8 * nb + 4 * npr + 8 * m
        out[name] = dict(_op_record(nb + npr, t, alg, peak, split, "hj_probe",
                                    8 * npr + 8 * m, ncu_traffic("k_hj_probe", npr)),
                         matches=m, build_rows=nb, probe_rows=npr, tuning=tuning)
        del pk
    del bk, bp, opay, orow
    torch.cuda.empty_cache()

    # ---- config 3: group-by 2^28 rows, cardinality 16 / 2^12 / 2^22 ----------
    n = 1 << 28
    s3 = 0xB200 + 3
    vals = g(gen.Spec(L.GEN_UNIFORM, L.I64, seed=s3, stream_id=1, lo=100, hi=10**7), n)
    cap = 2 << 22
    outs = {w: torch.empty(cap, dtype=torch.int64, device=dev) for w in ("sum", "count", "min", "max")}
    outs["key"] = e32(cap)
    for i, c in enumerate((16, 1 << 12, 1 << 22)):
        keys = g(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=s3, stream_id=10 + i, lo=0, hi=c - 1,
                          perm_domain=0), n)
        for mname, method in (("hash", L.GROUP_HASH), ("sort", L.GROUP_SORT)):
            tuning = None
            if method == L.GROUP_HASH:  # the autotuner's mode for this shape (if any choice)
                tuning, _, _, _ = ops.group_autotune(ctx, keys, vals, method=method,
                                                     expected_groups=c, capacity=cap, outs=outs,
                                                     result=res)
            run = lambda: ops.group_kernel(ctx, keys, vals, method=method, expected_groups=c,
                                           capacity=cap, outs=outs, result=res)
            run()
            ctx.sync()
            groups = int(res.item())
            t = _timed(run, iters, flush, stream)
            split = _kernel_split(ctx, run)
            alg = 12 * n + 36 * groups
            dom = "group" if method == L.GROUP_HASH else "sort_pass"
            tr = None
            if method == L.GROUP_HASH:  # above 4608 groups the rows are partitioned first
                tr = ncu_traffic("k_gb_chunks" if c > 4608 else "k_gb_aggregate_shared", n)
            out[f"group_{mname}_{c}_cfg3"] = dict(
                _op_record(n, t, alg, peak, split, dom, 12 * n if method == L.GROUP_HASH else None, tr),
                groups=groups, **({"tuning": tuning} if tuning else {}))
        del keys
    del vals, outs
    torch.cuda.empty_cache()

    # ---- config 4: batched form vs plain launches ---------------------------
    bw = BatchWorkload()
    bw.setup(ctx, dev)
    t = _timed(bw.step, 5, flush, stream)
    med = statistics.median(t)
    plain = bw.plain
    out["batched_cfg4"] = {
        "instances": bw.NG + bw.NJ, "rows": bw.rows_per_step,
        "batched_ms": round(med, 3), "batched_rows_per_s": round(bw.rows_per_step / (med * 1e-3), 1),
        "plain": plain,
        "speedup_vs_plain_wall": round(plain["ms_per_step"] / med, 3),
        "speedup_vs_plain_device_busy": round(plain["device_busy_ms"] / med, 3),
        "autotuned": bw.extra()["autotuned"]}
    bw.close()
    del bw
    torch.cuda.empty_cache()

    # ---- config 5: served form ------------------------------------------------
    sw = ServeWorkload(requests=10_000)
    sw.setup(ctx, dev)
    sw.step()
    out["served_cfg5"] = sw.extra()
    sw.close()

    # ---- the reference's TPC-H Q6 and Q1 pipelines, on the same table --------
    from pimdal_b200 import tpch
    li = tpch.Lineitem(ctx, sw.tables)
    n = li.n
    s6 = tpch.q6(ctx, li, staged=True)
    preds, exprs = tpch.q6_args(li)
    run = lambda: ops.select_aggregate(ctx, n, preds=preds, exprs=exprs, result=res)
    run()
    t = _timed(run, 20, flush, stream)
    alg = tpch.algorithmic_bytes_q6(n, s6.stage_rows)
    out["tpch_q6_fused"] = dict(_op_record(n, t, alg, peak, _kernel_split(ctx, run), "scan_agg", alg),
                                stage_rows=list(s6.stage_rows), revenue=s6.revenue)
    t = _timed(lambda: tpch.q6(ctx, li, staged=True), 5, flush, stream)
    out["tpch_q6_staged"] = _op_record(n, t, alg, peak)
    pred, group, exprs = tpch.q1_args(li)
    sel = int(((li.shipdate < tpch.packed(tpch.Q1_DATE))).sum().item())
    run = lambda: ops.select_aggregate(ctx, n, preds=[pred], group=group, key_space=6,
                                       exprs=exprs, result=res)
    run()
    t = _timed(run, 20, flush, stream)
    alg = tpch.algorithmic_bytes_q1(n, sel)
    out["tpch_q1_fused"] = dict(_op_record(n, t, alg, peak, _kernel_split(ctx, run), "scan_agg", alg),
                                selected=sel)
    t = _timed(lambda: tpch.q1(ctx, li, staged=True), 5, flush, stream)
    out["tpch_q1_staged"] = _op_record(n, t, alg, peak)
    # the multi-table pipelines (Q4, Q3, Q5): chains of plain operators with
    # the counts read back between steps, as the reference reads its DPUs'
    # result sizes between launches
    schema = tpch.Schema(ctx, li)
    for q in ("q4", "q3", "q5"):
        fn = getattr(tpch, q)
        run = lambda fn=fn: fn(ctx, schema)
        run()
        t = _timed(run, 5, flush, stream)
        out[f"tpch_{q}"] = dict(_op_record(n, t, tpch.column_bytes(q, schema), peak,
                                           _kernel_split(ctx, run, iters=1)),
                                bytes="columns read once in full (tpch.column_bytes)")
    del li, sw, schema
    torch.cuda.empty_cache()
    return out


WORKLOADS = {"select": SelectWorkload, "sort_smj": SortSmjWorkload,
             "hash_join": HashJoinWorkload, "group_by": GroupByWorkload,
             "batch": BatchWorkload, "serve": ServeWorkload}
DEFAULT_WORKLOAD = "sort_smj"


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    return world, rank, local


def _rank_tensor(x: float):
    """x in a tensor on the device the process group reduces on (the GPU
    under NCCL, the host under gloo)."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    return torch.tensor([x], dtype=torch.float64, device=dev)


def reduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch.distributed as dist
    t = _rank_tensor(x)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch.distributed as dist
    t = _rank_tensor(x)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_ours(args) -> None:
    import torch
    from pimdal_b200 import ops

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    ctx = ops.Context(local)
    wl = WORKLOADS[args.workload]()
    wl.setup(ctx, dev)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    for _ in range(args.warmup):
        flush.fill_(1)
        wl.step()
    ctx.sync()

    # ---- device-resident timing ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ctx.kernel_time(wl.dominant)  # reset
    barrier(world)
    torch.cuda.synchronize()
    launches0 = ctx.launches
    with ClockSampler(local) as clk:
        ctx.set_profiling(True)
        for i in range(args.steps):
            flush.fill_(i)
            starts[i].record(stream)
            wl.step()
            stops[i].record(stream)
        torch.cuda.synchronize()
        ctx.set_profiling(False)
    barrier(world)
    launches = ctx.launches - launches0
    if hasattr(wl, "launches_per_step"):  # graph replays bypass the host-side counter
        launches = wl.launches_per_step * args.steps
    ctx.sync()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    total_ms = reduce_max(sum(step_ms), world)
    k_launches, k_ms = ctx.kernel_time(wl.dominant)
    clocks = clk.summary()
    if hasattr(wl, "dominant_timing"):  # graph replays carry no per-kernel events
        k_launches, k_ms = wl.dominant_timing()
        k_launches = k_launches * args.steps
        k_ms = k_ms * args.steps

    # ---- end-to-end timing (public API, host buffers) ----
    for _ in range(max(1, args.warmup // 2)):
        wl.step_e2e(stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h2d = d2h = 0
    for _ in range(args.steps):
        h2d, d2h = wl.step_e2e(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = reduce_max(e0.elapsed_time(e1), world)
    ctx.sync()

    units = getattr(wl, "units_per_step", wl.rows_per_step)
    rows_total = reduce_sum(float(units * args.steps), world)
    value = rows_total / (total_ms / 1e3)
    e2e_value = rows_total / (e2e_ms / 1e3)

    peak, peak_kind = hbm_peak()
    roof = None
    if k_launches:
        if hasattr(wl, "roofline_bytes"):
            total_b = wl.roofline_bytes(k_launches, args.steps)
        else:
            total_b = wl.algorithmic_bytes_per_launch() * k_launches
        ach = total_b / (k_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": wl.dominant_name, "achieved": round(ach, 1),
                "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
                "peak_source": peak_kind,
                "traffic": wl.traffic_per_launch,
                "traffic_source": getattr(wl, "traffic_source", None),
                "algorithmic_bytes_per_launch": wl.algorithmic_bytes_per_launch(),
                "mean_launch_ms": round(k_ms / k_launches, 5), "launches": k_launches}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl)

    per_op = None
    if world == 1 and args.workload == DEFAULT_WORKLOAD and not args.no_per_operator:
        if hasattr(wl, "release"):
            wl.release()
        del flush
        torch.cuda.empty_cache()
        per_op = per_operator(ctx, dev, peak)

    if rank == 0:
        line = {
            "metric": getattr(wl, "metric_name", "rows/s"), "value": round(value, 1),
            "unit": getattr(wl, "unit", "rows/s"), "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/uint32 keys, int64 sums",
            "data": "synthetic (seeded counter-based generator)",
            "config": dict(wl.config, parallelism=f"replicas x{world}"),
            "e2e": {"value": round(e2e_value, 1), "unit": getattr(wl, "unit", "rows/s"),
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": round(e2e_ms / args.steps, 4)},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": launches, "impl": "ours",
        }
        if per_op is not None:
            line["per_operator"] = per_op
        if hasattr(wl, "extra"):
            line.update(wl.extra())
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def host_cpu() -> dict:
    """The host's CPU as the reference's runs record it: nproc, the lscpu
    model name and socket count, and the threads the baseline uses."""
    info = {"nproc": os.cpu_count(), "threads_used": host_threads()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=20).stdout
        for line in out.splitlines():
            key, _, val = line.partition(":")
            key, val = key.strip(), val.strip()
            if key == "Model name":
                info["model"] = val
            elif key == "Socket(s)":
                info["sockets"] = int(val) if val.isdigit() else val
            elif key == "Thread(s) per core":
                info["threads_per_core"] = int(val) if val.isdigit() else val
    except Exception:
        pass
    return info


def cpu_baseline(wl) -> dict | None:
    import oracle
    if not oracle.Ref.available("select"):
        return {"value": None, "unavailable": "oracle/_ref not built"}
    threads = host_threads()
    rows, secs, desc = wl.cpu_sample(oracle.Ref(), threads, 12.0)
    return {"value": round(rows / secs, 1), "unit": getattr(wl, "unit", "rows/s"), "cores": threads,
            "kind": "reference", "sample": desc, "cpu": host_cpu()}


def run_reference(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    wl = WORKLOADS[args.workload]()
    if not oracle.Ref.available("select"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's CPU "
                          "operators) was not built on this machine"}))
        return
    threads = host_threads()
    ref = oracle.Ref()
    # one step = one repetition of the workload's sample (the default
    # workload's sample is the whole config); no extra budget per step
    budget = 0.0 if args.workload == DEFAULT_WORKLOAD else max(0.5, min(5.0, 150.0 / (args.steps + args.warmup)))
    for _ in range(args.warmup):
        wl.cpu_sample(ref, threads, 0.0)
    rows = secs = 0.0
    desc = ""
    for _ in range(args.steps):
        r, s, desc = wl.cpu_sample(ref, threads, budget)
        rows += r
        secs += s
    value = rows / secs
    unit = getattr(wl, "unit", "rows/s")
    per_step = getattr(wl, "units_per_step", wl.rows_per_step)
    print(json.dumps({
        "metric": getattr(wl, "metric_name", "rows/s"), "value": round(value, 1), "unit": unit,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(per_step / value * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/uint32 keys, int64 sums", "data": "synthetic (seeded counter-based generator)",
        "config": dict(wl.config, parallelism=f"replicas x{world}"), "impl": "reference",
        "execution": f"host CPU, {threads} threads (the reference's own CPU operators)",
        "cpu_baseline": {"value": round(value, 1), "unit": unit, "cores": threads,
                         "kind": "reference", "sample": desc, "cpu": host_cpu()},
        "e2e": {"value": round(value, 1), "unit": unit, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-operator", action="store_true",
                    help="skip the per-operator records of the default run (configs 1, 3, 4, 5)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
