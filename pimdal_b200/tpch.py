"""The reference's TPC-H Q1 and Q6 pipelines on the C ABI.

The reference runs them as DPU programs over parquet-loaded lineitem columns
(pimdal/main/tpc_h/query6, pimdal/main/tpc_h/query1).  Here they run over a
lineitem-shaped table resident in HBM -- the served form's synthetic fact
table (pimdal_b200/serve.py: 6e7 rows of quantity, price cents, discount
percent, ship day over 2557 days, return-flag and line-status codes) plus a
packed ship date (the reference reader's date_to_int encoding) and a tax
percent column U[0, 8] -- because no TPC-H data or generator exists here.

Each query has two forms with the same result:

  * fused: one pimdal_select_aggregate pass (predicates, products and the
    group-by in one scan);
  * staged: the reference's own chain of plain operators -- pimdal_sel_kernel
    per predicate with a pimdal_gather_u32 of the next column in between (the
    DPU kernels' sel_kernel + load_next), then pimdal_select_aggregate over
    the surviving row ids in place of arithmetic_kernel + reduce_kernel /
    group_kernel.

Q6 follows pimdal/main/tpc_h/query6/dpu/kernel_q6.c:112-156 with the
parameters of host/host_q6.cpp:48-51 and the check plan of :70-100: ship date
in [date_to_int("1994-01-01"), date_to_int("1995-01-01")), quantity < 24,
discount within 6 +- 1; revenue = SUM(price * discount) (the reference prints
it divided by 10^4; here the exact int64 sum is returned).

Q1 follows pimdal/main/tpc_h/query1/dpu/kernel_q1_1.c:84-227 with the
parameter of host/host_q1.cpp:57 and the check plan of :263-322: ship date <
date_to_int("1998-09-02"); per (return flag, line status) group SUM(quantity),
SUM(price), SUM(price * (100 - discount)), SUM(price * (100 - discount) *
(100 + tax)), SUM(discount) and COUNT; the averages are the sums divided by
the count on the host, as aggr_host does (:236-261).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import pyarrow as pa
import torch

from . import _lib as L
from . import gen, ingest, ops, serve

FIRST_DAY = np.datetime64("1992-01-01")  # ship day 0 of the synthetic table


def packed(day: str) -> int:
    """The reference reader's packed date of "YYYY-MM-DD"."""
    return int(ingest.date_to_int(pa.array([day]))[0])


Q6_DATE_LO, Q6_DATE_HI = "1994-01-01", "1995-01-01"   # host_q6.cpp:48-49
Q6_DISCOUNT, Q6_QUANTITY = 6, 24                      # host_q6.cpp:50-51
Q1_DATE = "1998-09-02"                                # host_q1.cpp:57
N_RFLAG, N_LSTATUS = serve.N_RFLAG, serve.N_LSTATUS


class Lineitem:
    """Lineitem-shaped columns in HBM: the served fact table's columns plus a
    packed ship date and a tax column."""

    def __init__(self, ctx: ops.Context, tables: serve.Tables | None = None, seed: int = 0xB20A):
        t = tables if tables is not None else serve.Tables(ctx)
        dev = f"cuda:{ctx.device}"
        self.n = t.n
        days = (FIRST_DAY - np.datetime64("1970-01-01")).astype(np.int64) + np.arange(serve.DAYS)
        lut = ingest.date_to_int(pa.array(days.astype(np.int32), type=pa.date32()))
        self.shipdate = torch.from_numpy(np.ascontiguousarray(lut, np.int32)).to(dev)[
            t.l_date.long()].contiguous()
        self.tax = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.I32, seed=seed, stream_id=1, lo=0,
                                                hi=8), t.n)
        self.quantity, self.price, self.discount = t.l_quantity, t.l_price, t.l_discount
        self.returnflag, self.linestatus = t.l_rflag, t.l_lstatus
        self.tables = t


@dataclass
class Q6Result:
    revenue: int     # SUM(price * discount), exact
    rows: int        # qualifying rows
    stage_rows: tuple = ()  # staged form: rows after each selection


@dataclass
class Q1Result:
    returnflag: np.ndarray
    linestatus: np.ndarray
    sum_qty: np.ndarray
    sum_base_price: np.ndarray
    sum_disc_price: np.ndarray
    sum_charge: np.ndarray
    sum_disc: np.ndarray
    count_order: np.ndarray

    def averages(self) -> dict:
        """avg_qty, avg_price, avg_disc: the sums over the count, integer
        division as the reference's host plan divides int64 columns."""
        c = self.count_order
        return {"avg_qty": self.sum_qty // c, "avg_price": self.sum_base_price // c,
                "avg_disc": self.sum_disc // c}


def q6_args(li: Lineitem):
    preds = [(li.shipdate, ops.make_pred(L.PRED_RANGE, packed(Q6_DATE_LO), packed(Q6_DATE_HI))),
             (li.quantity, ops.make_pred(L.PRED_LT, Q6_QUANTITY)),
             (li.discount, ops.make_pred(L.PRED_BETWEEN, Q6_DISCOUNT - 1, Q6_DISCOUNT + 1))]
    return preds, [[li.price, li.discount]]


def q6(ctx: ops.Context, li: Lineitem, *, staged: bool = False, stream=None) -> Q6Result:
    """Q6 revenue, fused (one pass) or staged (the reference's operator chain)."""
    preds, exprs = q6_args(li)
    if not staged:
        res, outs = ops.select_aggregate(ctx, li.n, preds=preds, exprs=exprs, stream=stream)
        ctx.sync(stream)
        g = int(res.item())
        return Q6Result(int(outs["sum0"][0]) if g else 0, int(outs["count"][0]) if g else 0)
    # ship date -> (row ids); quantity of those rows -> select; discount -> select
    dev = li.shipdate.device
    rows, counts = None, []
    buf = torch.empty(li.n, dtype=torch.int32, device=dev)
    for (col, pred), nxt in zip(preds, [None, li.quantity, li.discount]):
        if rows is None:
            res, _, rows = ops.sel_kernel(ctx, col, pred, stream=stream)
        else:
            k = counts[-1]
            ops.gather_u32(ctx, col, rows, k, out=buf, stream=stream)
            res, _, rows = ops.sel_kernel(ctx, buf[:k], pred, in_ptr=rows[:k], stream=stream)
        ctx.sync(stream)
        counts.append(int(res.item()))
    k = counts[-1]
    res, outs = ops.select_aggregate(ctx, k, rows=rows[:k] if k else rows, exprs=exprs,
                                     stream=stream)
    ctx.sync(stream)
    g = int(res.item())
    return Q6Result(int(outs["sum0"][0]) if g else 0, k, tuple(counts))


def q1_args(li: Lineitem):
    pred = (li.shipdate, ops.make_pred(L.PRED_LT, packed(Q1_DATE)))
    group = [(li.returnflag, N_LSTATUS), (li.linestatus, 1)]
    disc_price = [li.price, (li.discount, 1, 100)]                       # price * (100 - disc)
    exprs = [[li.quantity], [li.price], disc_price,
             disc_price + [(li.tax, 0, 100)],                            # * (100 + tax)
             [li.discount]]
    return pred, group, exprs


def q1(ctx: ops.Context, li: Lineitem, *, staged: bool = False, stream=None) -> Q1Result:
    """Q1 groups, fused (one pass) or staged (selection, then the per-row
    sums and the group-by over the selected row ids)."""
    pred, group, exprs = q1_args(li)
    ks = N_RFLAG * N_LSTATUS
    if not staged:
        res, outs = ops.select_aggregate(ctx, li.n, preds=[pred], group=group, key_space=ks,
                                         exprs=exprs, stream=stream)
    else:
        r1, _, rows = ops.sel_kernel(ctx, pred[0], pred[1], stream=stream)
        ctx.sync(stream)
        k = int(r1.item())
        res, outs = ops.select_aggregate(ctx, k, rows=rows, group=group, key_space=ks,
                                         exprs=exprs, stream=stream)
    ctx.sync(stream)
    g = int(res.item())
    h = {name: t[:g].cpu().numpy() for name, t in outs.items()}
    key = h["key"].astype(np.int64)
    return Q1Result(key // N_LSTATUS, key % N_LSTATUS, h["sum0"], h["sum1"], h["sum2"], h["sum3"],
                    h["sum4"], h["count"])


def algorithmic_bytes_q6(n: int, stage_rows) -> int:
    """Bytes the Q6 plan must read at least: the ship date of every row, the
    quantity of the rows in the date range, the discount of those with
    quantity < 24, the price of the qualifying rows (the reference's
    load_next order, kernel_q6.c:120-145)."""
    k1, k2, k3 = stage_rows
    return 4 * n + 4 * k1 + 4 * k2 + 8 * k3


def algorithmic_bytes_q1(n: int, selected: int) -> int:
    """The ship date of every row; flag, status (1 B each), quantity,
    discount, tax (4 B) and price (8 B) of the selected rows."""
    return 4 * n + 22 * selected
