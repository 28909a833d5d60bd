"""Served form: a request loop over filter -> join -> group-by pipelines.

A synthetic fact table (lineitem-shaped: orderkey with 1-7 rows per order,
partkey, suppkey, quantity, price cents, discount percent, date, two flag
columns) and two dimensions (orders: orderkey, date, priority; part: partkey,
category) are generated into HBM once.  The hash tables of both dimensions
are built once (pimdal_hash_kernel, the dimension attribute as the build
payload) and stay resident.  A request is

    SELECT attr [, flag], SUM(price * (100 - discount)), COUNT(*)
    FROM fact[r0 : r0 + n] JOIN dim USING (key)
    WHERE date BETWEEN d0 AND d1  GROUP BY attr [, flag]  ORDER BY attr [, flag]

run either fused -- one pass, pimdal_select_join_aggregate: date filter,
probe of the resident table, revenue, group-by into a table indexed by the
small group key -- or as the plain operators in stages: selection of the
date range (row ids), gather of the join keys, probe of the resident table,
fused key/revenue gather, hash group-by (groups come out ordered by key).
Both give identical groups.  The stages are a non-blocking state machine: a
stage is launched on the request's slot (one CUDA stream and one library
context each), the counts it produces are copied to pinned host memory, and
the next stage starts when they arrive.

Scheduling (continuous batching): requests arrive (Poisson); an arrived
request is admitted as soon as a slot is free and its working-set bytes fit
the HBM byte budget left after the resident tables and the slots' fixed
memory; admitted requests run concurrently, their stages interleaving on the
device.  The charge is what the request really holds on the device while it
runs: a staged request allocates its per-row buffers (selected row ids and
values, join keys, matches, group keys and values: 32 bytes per range row)
in one allocation when it starts and frees it when it ends; a fused request
allocates nothing per row and is charged its group table (16 bytes per key
of its key space) and its outputs.  Served runs use the fused pass by
default; serial plain execution is the same loop with one slot, one request
at a time, through the staged plain operators.  The reference runs one query
at a time on the DPUs (pimdal/main/tpc_h/*/host).
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import gen, ops

DAYS = 2557
N_PRIO = 5
N_RFLAG = 3
N_CAT = 25
N_LSTATUS = 2
STAGED_ROW_BYTES = 32   # staged buffers per range row: 6 x int32 + 1 x int64


@dataclass
class Request:
    rid: int
    arrival: float  # seconds from the start of the run
    r0: int         # first fact row of the range
    n: int          # rows in the range
    d0: int         # date range, inclusive
    d1: int
    dim: int        # 0: orders (group by priority), 1: part (group by category)
    two_keys: bool  # also group by the fact's flag column

    def key_space(self) -> int:
        """Group keys of the request: dimension attribute (x flag values)."""
        attrs = N_PRIO if self.dim == 0 else N_CAT
        return attrs * ((N_RFLAG if self.dim == 0 else N_LSTATUS) if self.two_keys else 1)

    def need_bytes(self, fused: bool) -> int:
        """Device bytes the request holds while it runs."""
        if fused:  # the fused pass's group table (16 B per key) and nothing per row
            return 16 * self.key_space()
        return STAGED_ROW_BYTES * self.n


@dataclass
class Result:
    keys: np.ndarray
    sums: np.ndarray
    counts: np.ndarray
    selected: int = 0
    joined: int = 0
    start: float = 0.0
    done: float = 0.0


class Tables:
    """The resident fact and dimension columns and the dimension hash tables."""

    def __init__(self, ctx: ops.Context, orders: int = 15_000_000, parts: int = 2_000_000,
                 supps: int = 100_000, seed: int = 0xB205):
        dev = f"cuda:{ctx.device}"
        g = lambda spec, n: ops.gen_column(ctx, spec, n)
        U = lambda sid, lo, hi, dt=L.I32: gen.Spec(L.GEN_UNIFORM, dt, seed=seed, stream_id=sid, lo=lo, hi=hi)
        self.n_orders, self.n_parts, self.n_supps = orders, parts, supps
        # orders dimension: distinct keys (a seeded sample of [0, 2^31)), date, priority
        self.o_key = g(gen.Spec(L.GEN_PERM, L.I32, seed=seed, perm_domain=1 << 31), orders)
        self.o_date = g(U(1, 0, DAYS - 1), orders)
        self.o_prio = g(U(2, 0, N_PRIO - 1), orders)
        per_order = g(U(3, 1, 7), orders).to(torch.int64)
        order_of_row = torch.repeat_interleave(torch.arange(orders, device=dev), per_order)
        n = int(order_of_row.numel())
        self.n = n
        self.l_orderkey = self.o_key[order_of_row].contiguous()
        del order_of_row, per_order
        self.l_partkey = g(U(4, 1, parts), n)
        self.l_suppkey = g(U(5, 1, supps), n)
        self.l_quantity = g(U(6, 1, 50), n)
        self.l_price = g(U(7, 90_000, 10_500_000, L.I64), n)
        self.l_discount = g(U(8, 0, 10), n)
        self.l_date = g(U(9, 0, DAYS - 1), n)
        self.l_rflag = g(U(10, 0, N_RFLAG - 1), n).to(torch.uint8)
        self.l_lstatus = g(U(11, 0, N_LSTATUS - 1), n).to(torch.uint8)
        # part dimension: partkey 1..parts, category
        self.p_key = torch.arange(1, parts + 1, dtype=torch.int32, device=dev)
        self.p_cat = g(U(12, 0, N_CAT - 1), parts)
        # resident hash tables: key -> attribute
        self.t_orders_size = 1 << math.ceil(math.log2(2 * orders))
        self.t_part_size = 1 << math.ceil(math.log2(2 * parts))
        self.t_orders = ops.hash_kernel(ctx, self.o_key, self.o_prio, table_size=self.t_orders_size)
        self.t_part = ops.hash_kernel(ctx, self.p_key, self.p_cat, table_size=self.t_part_size)
        ctx.sync()

    @property
    def resident_bytes(self) -> int:
        ts = [v for v in vars(self).values() if isinstance(v, torch.Tensor)]
        return sum(t.numel() * t.element_size() for t in ts)

    def n_attr(self, which: int) -> int:
        """Distinct values of the dimension attribute (the build payload)."""
        return N_PRIO if which == 0 else N_CAT

    def dim(self, which: int):
        """(join key column of the fact, table, table size, flag column, attribute count)."""
        if which == 0:
            return self.l_orderkey, self.t_orders, self.t_orders_size, self.l_rflag, N_RFLAG
        return self.l_partkey, self.t_part, self.t_part_size, self.l_lstatus, N_LSTATUS


def make_requests(count: int, fact_rows: int, rate: float | None, seed: int = 0xB206,
                  min_rows: int = 100_000, max_rows: int = 60_000_000) -> list[Request]:
    """Poisson arrivals (rate requests/s; None: all at time 0), row ranges
    log-uniform in [min_rows, max_rows], date selectivity uniform 1-50%."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    hi = min(max_rows, fact_rows)
    lo = min(min_rows, hi)
    for i in range(count):
        if rate:
            t += rng.exponential(1.0 / rate)
        n = int(round(10 ** rng.uniform(math.log10(lo), math.log10(hi))))
        n = max(1, min(n, fact_rows))
        r0 = int(rng.integers(0, fact_rows - n + 1))
        width = max(1, int(round(rng.uniform(0.01, 0.50) * DAYS)))
        d0 = int(rng.integers(0, DAYS - width + 1))
        out.append(Request(i, t if rate else 0.0, r0, n, d0, d0 + width - 1,
                           int(rng.integers(0, 2)), bool(rng.integers(0, 2))))
    return out


class Slot:
    """One concurrency slot: a CUDA stream, a library context, the outputs of
    one request, and (while a staged request runs) its per-row buffers."""

    MAX_GROUPS = N_CAT * N_LSTATUS + N_PRIO * N_RFLAG

    def __init__(self, device: int, max_rows: int):
        dev = f"cuda:{device}"
        self.dev = dev
        self.ctx = ops.Context(device)
        self.stream = torch.cuda.Stream(device=dev)
        self.buf = None
        e32 = lambda k: torch.empty(k, dtype=torch.int32, device=dev)
        g = self.MAX_GROUPS
        self.outs = {"key": e32(g), "sum": torch.empty(g, dtype=torch.int64, device=dev),
                     "count": torch.empty(g, dtype=torch.int64, device=dev)}
        self.res = torch.zeros(3, dtype=torch.int64, device=dev)
        self.h_cnt = torch.zeros(3, dtype=torch.int64, pin_memory=True)
        self.h_key = torch.zeros(g, dtype=torch.int32, pin_memory=True)
        self.h_sum = torch.zeros(g, dtype=torch.int64, pin_memory=True)
        self.h_count = torch.zeros(g, dtype=torch.int64, pin_memory=True)
        self.event = torch.cuda.Event()
        self.req: Request | None = None
        self.stage = 0
        self.result: Result | None = None
        self.fused = False  # run requests as one fused pass (else the staged operators)

    def close(self):
        self.ctx.close()

    # -- stages --------------------------------------------------------------
    def start(self, tables: Tables, req: Request, now: float) -> None:
        self.req, self.stage = req, 0
        self.result = Result(np.zeros(0, np.int32), np.zeros(0, np.int64), np.zeros(0, np.int64),
                             start=now)
        if not self.fused:
            # one allocation of exactly the charged bytes, on the slot's stream
            m = max(req.n, 1)
            with torch.cuda.stream(self.stream):
                self.buf = torch.empty(8 * m, dtype=torch.int32, device=self.dev)
            b = self.buf
            self.sel_val, self.sel_row, self.jkey = b[0:m], b[m:2 * m], b[2 * m:3 * m]
            self.mrow, self.mattr, self.gkey = b[3 * m:4 * m], b[4 * m:5 * m], b[5 * m:6 * m]
            self.gval = b[6 * m:8 * m].view(torch.int64)
        self._launch(tables)

    def _launch(self, t: Tables) -> None:
        r, s, ctx = self.req, self.stream, self.ctx
        with torch.cuda.stream(s):
            if self.fused:
                col, table, tsize, flag, nflag = t.dim(r.dim)
                mult = nflag if r.two_keys else 1
                rng = slice(r.r0, r.r0 + r.n)
                ops.select_join_aggregate(
                    ctx, t.l_date[rng], r.d0, r.d1, col[rng], table, tsize, t.l_price[rng],
                    t.l_discount[rng], flag=flag[rng] if r.two_keys else None, attr_mult=mult,
                    key_space=t.n_attr(r.dim) * mult, outs=self.outs, result=self.res[2:3], stream=s)
                self.h_cnt[2:3].copy_(self.res[2:3], non_blocking=True)
                self.h_key.copy_(self.outs["key"], non_blocking=True)
                self.h_sum.copy_(self.outs["sum"], non_blocking=True)
                self.h_count.copy_(self.outs["count"], non_blocking=True)
            elif self.stage == 0:
                pred = ops.make_pred(L.PRED_BETWEEN, r.d0, r.d1)
                ops.sel_kernel(ctx, t.l_date[r.r0:r.r0 + r.n], pred, ptr_base=r.r0,
                               out=self.sel_val, out_ptr=self.sel_row, result=self.res[0:1],
                               stream=s)
                self.h_cnt[0:1].copy_(self.res[0:1], non_blocking=True)
            elif self.stage == 1:
                k = int(self.h_cnt[0])
                col, table, tsize, _, _ = t.dim(r.dim)
                ops.gather_u32(ctx, col, self.sel_row, k, out=self.jkey, stream=s)
                ops.hj_probe(ctx, table, tsize, self.jkey[:k], capacity=k, out_outer=self.mrow,
                             out_inner=self.mattr, result=self.res[1:2], stream=s)
                self.h_cnt[1:2].copy_(self.res[1:2], non_blocking=True)
            else:
                m = int(self.h_cnt[1])
                _, _, _, flag, nflag = t.dim(r.dim)
                ops.revenue_keys(ctx, m, self.mrow, self.mattr, self.sel_row, t.l_price,
                                 t.l_discount, flag if r.two_keys else None,
                                 nflag if r.two_keys else 1, self.gkey, self.gval, stream=s)
                ops.group_kernel(ctx, self.gkey[:m], self.gval[:m], method=L.GROUP_HASH,
                                 expected_groups=self.MAX_GROUPS, capacity=self.MAX_GROUPS,
                                 outs=self.outs, result=self.res[2:3], stream=s)
                self.h_cnt[2:3].copy_(self.res[2:3], non_blocking=True)
                self.h_key.copy_(self.outs["key"], non_blocking=True)
                self.h_sum.copy_(self.outs["sum"], non_blocking=True)
                self.h_count.copy_(self.outs["count"], non_blocking=True)
            self.event.record(s)

    def poll(self, tables: Tables, now: float) -> bool:
        """Advances the request when its stage finished; True when it is done."""
        if not self.event.query():
            return False
        if self.fused:
            return self._finish(now, int(self.h_cnt[2]))
        if self.stage == 0:
            self.result.selected = int(self.h_cnt[0])
            if self.result.selected == 0:
                return self._finish(now, 0)
        elif self.stage == 1:
            self.result.joined = int(self.h_cnt[1])
            if self.result.joined == 0:
                return self._finish(now, 0)
        else:
            return self._finish(now, int(self.h_cnt[2]))
        self.stage += 1
        self._launch(tables)
        return False

    def _finish(self, now: float, groups: int) -> bool:
        self.ctx.sync(self.stream)  # raises on any device-side error of this request
        # the stream has passed every use of the staged buffers: release them
        self.buf = self.sel_val = self.sel_row = self.jkey = None
        self.mrow = self.mattr = self.gkey = self.gval = None
        r = self.result
        r.keys = self.h_key[:groups].numpy().copy()
        r.sums = self.h_sum[:groups].numpy().copy()
        r.counts = self.h_count[:groups].numpy().copy()
        r.done = now
        return True


@dataclass
class RunStats:
    results: dict = field(default_factory=dict)
    latencies: list = field(default_factory=list)
    makespan: float = 0.0
    rows: int = 0
    max_inflight: int = 0
    max_reserved: int = 0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies) * 1e3
        q = lambda p: float(np.percentile(lat, p)) if lat.size else None
        return {"queries": len(self.latencies),
                "queries_per_s": len(self.latencies) / self.makespan if self.makespan else None,
                "rows_per_s": self.rows / self.makespan if self.makespan else None,
                "p50_ms": q(50), "p99_ms": q(99), "p999_ms": q(99.9),
                "mean_ms": float(lat.mean()) if lat.size else None,
                "max_inflight": self.max_inflight, "max_reserved_bytes": self.max_reserved}


class Admission:
    """Byte-budget admission: a request may start when a slot is free and its
    working-set bytes fit in what the budget has left."""

    def __init__(self, budget_bytes: int):
        self.budget = budget_bytes
        self.reserved = 0

    def fits(self, need: int) -> bool:
        return self.reserved + need <= self.budget or self.reserved == 0

    def take(self, need: int) -> None:
        self.reserved += need

    def give(self, need: int) -> None:
        self.reserved -= need


class Server:
    def __init__(self, tables: Tables, device: int = 0, slots: int = 8,
                 hbm_budget_bytes: int = 150 * 10**9):
        self.tables = tables
        self.max_rows = min(tables.n, 60_000_000)
        self.slots = [Slot(device, self.max_rows) for _ in range(slots)]
        self.hbm_budget = hbm_budget_bytes
        self.budget = max(0, hbm_budget_bytes - tables.resident_bytes)

    def fixed_bytes(self) -> int:
        """Device bytes the slots hold between requests: their contexts'
        workspaces (grown by the first requests) and output buffers."""
        return sum(sl.ctx.workspace_bytes() + 1024 for sl in self.slots)

    def close(self):
        for s in self.slots:
            s.close()

    def warm(self) -> None:
        """A large request of each dimension through every slot, staged and
        fused: the contexts' workspaces reach their size; the budget left for
        requests is what the tables and the slots do not hold."""
        rs = [Request(0, 0.0, 0, self.max_rows, 0, DAYS - 1, d, True) for d in (0, 1)]
        for s in self.slots:
            for fused in (False, True):
                s.fused = fused
                for r in rs:
                    s.start(self.tables, r, 0.0)
                    while not s.poll(self.tables, 0.0):
                        pass
        self.budget = max(0, self.hbm_budget - self.tables.resident_bytes - self.fixed_bytes())

    def run(self, requests: list[Request], serial: bool = False,
            fused: bool | None = None) -> RunStats:
        """Plays the request stream (arrival times relative to the start).
        serial: one slot, one request at a time.  fused: one pass per request
        (default: fused when served, the staged plain operators when serial)."""
        slots = self.slots[:1] if serial else self.slots
        for s in slots:
            s.fused = (not serial) if fused is None else fused
        adm = Admission(self.budget)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue: deque[Request] = deque()
        free = list(slots)
        busy: list[Slot] = []
        charged: dict[int, int] = {}
        st = RunStats()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        first = pending[0].arrival if pending else 0.0
        while pending or queue or busy:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            while (queue and free and adm.fits(queue[0].need_bytes(free[-1].fused))
                   and not (serial and busy)):
                r = queue.popleft()
                s = free.pop()
                r_need = r.need_bytes(s.fused)
                charged[r.rid] = r_need
                adm.take(r_need)
                s.start(self.tables, r, now)
                busy.append(s)
                st.max_inflight = max(st.max_inflight, len(busy))
                st.max_reserved = max(st.max_reserved, adm.reserved)
            for s in list(busy):
                now = time.perf_counter() - t0
                if s.poll(self.tables, now):
                    r = s.req
                    st.results[r.rid] = s.result
                    st.latencies.append(now - r.arrival)
                    st.rows += r.n
                    adm.give(charged.pop(r.rid))
                    busy.remove(s)
                    free.append(s)
            if not busy and not queue and pending:
                # idle until the next arrival
                time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 1e-3)))
        st.makespan = time.perf_counter() - t0 - first
        return st


def same_results(a: RunStats, b: RunStats) -> bool:
    if a.results.keys() != b.results.keys():
        return False
    for k, x in a.results.items():
        y = b.results[k]
        if not (np.array_equal(x.keys, y.keys) and np.array_equal(x.sums, y.sums)
                and np.array_equal(x.counts, y.counts)):
            return False
    return True
