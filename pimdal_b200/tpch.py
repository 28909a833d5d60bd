"""The reference's TPC-H pipelines (Q1, Q3, Q4, Q5, Q6) on the C ABI.

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

Q4, Q3 and Q5 join several tables; they run over a Schema (lineitem plus
orders, customer, supplier, nation and region columns of own synthetic
distributions) as the reference's chains of plain operators: a selection per
filter, load_next gathers (pimdal_gather_u32, pimdal_project), a hash join
per join (pimdal_hash_join), per-row arithmetic (pimdal_project) and a
group-by (pimdal_group_kernel, pimdal_select_aggregate), with the counts read
back between steps as the reference's hosts read their DPUs' result sizes.
Market segments, regions and nations are dictionary codes.
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


# ---------------------------------------------------------------------------
# Q4, Q3 and Q5: the reference's multi-table pipelines
# ---------------------------------------------------------------------------
Q4_DATE_LO, Q4_DATE_HI = "1993-07-01", "1993-10-01"  # host_q4.cpp:47-48 (populate_mram_1)
Q3_DATE = "1995-03-15"                               # host_q3.cpp:72,98
Q5_DATE_LO, Q5_DATE_HI = "1994-01-01", "1995-01-01"  # host_q5.cpp:83-84
N_SEGMENT, N_NATION, N_REGION = 5, 25, 5
Q3_SEGMENT = 1  # the market-segment code the query selects (host_q3.cpp:46 names one segment)
Q5_REGION = 2   # the region code the query selects (host_q5.cpp:58 names one region)
DATE_SLACK = 31  # days before the first and after the last ship day the date columns reach


class Schema:
    """Lineitem plus the orders, customer, supplier, nation and region columns
    the multi-table pipelines read, all resident in HBM.

    Own synthetic distributions (seeded; no TPC-H data or generator exists
    here): orders keep the served table's keys, order day and priority code
    and add a customer key U[1, customers] and a ship-priority code U[0, 3];
    customers are keyed 1..customers with a market-segment code
    U[0, N_SEGMENT) and a nation U[0, N_NATION); suppliers are keyed
    1..suppliers (the lineitem's supplier keys) with a nation
    U[0, N_NATION); nation k lies in region k mod N_REGION; a lineitem's
    commit day is its ship day + U[-30, 30], its receipt day its ship day +
    U[1, 30].  Dates are packed as the reference's reader packs them
    (date_to_int)."""

    def __init__(self, ctx: ops.Context, li: Lineitem, customers: int | None = None,
                 seed: int = 0xB20B):
        t = li.tables
        dev = f"cuda:{ctx.device}"
        g = lambda spec, n: ops.gen_column(ctx, spec, n)
        U = lambda sid, lo, hi: gen.Spec(L.GEN_UNIFORM, L.I32, seed=seed, stream_id=sid, lo=lo, hi=hi)
        self.li = li
        self.n = li.n
        self.n_orders = t.n_orders
        self.n_cust = customers if customers is not None else max(t.n_orders // 10, 1)
        self.n_supp = t.n_supps
        first = (FIRST_DAY - np.datetime64("1970-01-01")).astype(np.int64) - DATE_SLACK
        days = first + np.arange(serve.DAYS + 2 * DATE_SLACK)
        lut = torch.from_numpy(np.ascontiguousarray(
            ingest.date_to_int(pa.array(days.astype(np.int32), type=pa.date32())), np.int32)).to(dev)
        # orders
        self.o_orderkey, self.o_orderpriority = t.o_key, t.o_prio
        self.o_orderdate = lut[t.o_date.long() + DATE_SLACK].contiguous()
        self.o_custkey = g(U(1, 1, self.n_cust), self.n_orders)
        self.o_shippriority = g(U(2, 0, 3), self.n_orders)
        # customers
        self.c_custkey = torch.arange(1, self.n_cust + 1, dtype=torch.int32, device=dev)
        self.c_mktsegment = g(U(3, 0, N_SEGMENT - 1), self.n_cust)
        self.c_nationkey = g(U(4, 0, N_NATION - 1), self.n_cust)
        # suppliers, nations, regions
        self.s_suppkey = torch.arange(1, self.n_supp + 1, dtype=torch.int32, device=dev)
        self.s_nationkey = g(U(5, 0, N_NATION - 1), self.n_supp)
        self.n_nationkey = torch.arange(N_NATION, dtype=torch.int32, device=dev)
        self.n_regionkey = (self.n_nationkey % N_REGION).contiguous()
        self.r_regionkey = torch.arange(N_REGION, dtype=torch.int32, device=dev)
        self.r_name = self.r_regionkey.clone()  # region name codes
        # lineitem commit and receipt dates around the ship day
        day = t.l_date.long() + DATE_SLACK
        self.l_commitdate = lut[day + g(U(6, -30, 30), self.n).long()].contiguous()
        self.l_receiptdate = lut[day + g(U(7, 1, 30), self.n).long()].contiguous()
        del day
        ctx.sync()


def _count(ctx, res, stream) -> int:
    ctx.sync(stream)
    return int(res.item())


@dataclass
class Q4Result:
    priority: np.ndarray    # order-priority codes present, ascending
    order_count: np.ndarray  # orders of the date range with a late lineitem, per priority


def q4(ctx: ops.Context, s: Schema, stream=None) -> Q4Result:
    """Q4 after pimdal/main/tpc_h/query4/dpu/kernel_q4_1.c..kernel_q4_4.c and
    host/host_q4.cpp:210-233: the orders whose order date lies in
    [Q4_DATE_LO, Q4_DATE_HI) (kernel_q4_1.c: pred_o) that have at least one
    lineitem with commit date < receipt date (kernel_q4_2.c: pred_l), joined
    on the order key and made distinct per order (kernel_q4_3.c: hash_kernel,
    merge_kernel, group_kernel with `unique`), counted per order priority
    (kernel_q4_4.c, aggr_host) and ordered by priority."""
    lo, hi = packed(Q4_DATE_LO), packed(Q4_DATE_HI)
    r_o, _, o_rows = ops.sel_kernel(ctx, s.o_orderdate, ops.make_pred(L.PRED_RANGE, lo, hi),
                                    stream=stream)
    late = ops.project(ctx, s.n, [s.l_commitdate], minus=[s.l_receiptdate], out_dtype=L.I32,
                       stream=stream)  # commit - receipt
    r_l, _, l_rows = ops.sel_kernel(ctx, late, ops.make_pred(L.PRED_LT, 0), stream=stream)
    k_o, k_l = _count(ctx, r_o, stream), _count(ctx, r_l, stream)
    del late
    if k_o == 0 or k_l == 0:
        return Q4Result(np.zeros(0, np.int64), np.zeros(0, np.int64))
    o_keys = ops.gather_u32(ctx, s.o_orderkey, o_rows, k_o, stream=stream)
    l_keys = ops.gather_u32(ctx, s.li.tables.l_orderkey, l_rows, k_l, stream=stream)
    r_j, o_match, _ = ops.hash_join(ctx, o_keys[:k_o], o_rows[:k_o], l_keys[:k_l], capacity=k_l,
                                    stream=stream)
    m = _count(ctx, r_j, stream)
    if m == 0:
        return Q4Result(np.zeros(0, np.int64), np.zeros(0, np.int64))
    r_g, outs = ops.group_kernel(ctx, o_match[:m], None, want=("count",), expected_groups=k_o,
                                 capacity=k_o, stream=stream)
    nd = _count(ctx, r_g, stream)
    r_p, po = ops.select_aggregate(ctx, nd, rows=outs["key"][:nd],
                                   group=[(s.o_orderpriority, 1)], key_space=serve.N_PRIO,
                                   stream=stream)
    gp = _count(ctx, r_p, stream)
    return Q4Result(po["key"][:gp].cpu().numpy().astype(np.int64),
                    po["count"][:gp].cpu().numpy())


@dataclass
class Q3Result:
    orderkey: np.ndarray      # the 10 orders of the largest revenue, descending
    revenue: np.ndarray       # SUM(price * (100 - discount)) over the order's lineitems
    orderdate: np.ndarray
    shippriority: np.ndarray
    groups: int               # orders with a qualifying lineitem


def q3(ctx: ops.Context, s: Schema, top: int = 10, stream=None) -> Q3Result:
    """Q3 after pimdal/main/tpc_h/query3/dpu/kernel_q3_1.c..kernel_q3_5.c and
    host/host_q3.cpp:46,72,98,279-315: customers of one market segment
    (kernel_q3_1.c: pred_c); their orders dated before Q3_DATE
    (kernel_q3_2.c: pred_o, kernel_q3_3.c: the join on the customer key);
    the lineitems shipped after Q3_DATE (kernel_q3_4.c: pred_l) of those
    orders (kernel_q3_5.c: the join on the order key) with revenue
    price * (100 - discount) (kernel_q3_5.c:107) summed per order
    (group_kernel with sum), then the `top` orders by revenue, descending
    (the per-DPU sort_kernel and the host's merge of the DPUs' lists).
    Equal revenues are ordered by ascending order row."""
    d = packed(Q3_DATE)
    li, t = s.li, s.li.tables
    r_c, _, c_rows = ops.sel_kernel(ctx, s.c_mktsegment, ops.make_pred(L.PRED_EQ, Q3_SEGMENT),
                                    stream=stream)
    r_o, _, o_rows = ops.sel_kernel(ctx, s.o_orderdate, ops.make_pred(L.PRED_LT, d), stream=stream)
    r_l, _, l_rows = ops.sel_kernel(ctx, li.shipdate, ops.make_pred(L.PRED_GT, d), stream=stream)
    k_c, k_o, k_l = _count(ctx, r_c, stream), _count(ctx, r_o, stream), _count(ctx, r_l, stream)
    empty = Q3Result(*(np.zeros(0, np.int64) for _ in range(4)), 0)
    if min(k_c, k_o, k_l) == 0:
        return empty
    c_keys = ops.gather_u32(ctx, s.c_custkey, c_rows, k_c, stream=stream)
    o_cust = ops.gather_u32(ctx, s.o_custkey, o_rows, k_o, stream=stream)
    # orders of those customers: build the customer keys, probe the orders' customer keys
    r1, _, o_idx = ops.hash_join(ctx, c_keys[:k_c], c_rows[:k_c], o_cust[:k_o], capacity=k_o,
                                 stream=stream)
    m1 = _count(ctx, r1, stream)
    if m1 == 0:
        return empty
    q_rows = ops.gather_u32(ctx, o_rows, o_idx, m1, stream=stream)
    q_keys = ops.gather_u32(ctx, s.o_orderkey, q_rows, m1, stream=stream)
    l_keys = ops.gather_u32(ctx, t.l_orderkey, l_rows, k_l, stream=stream)
    # lineitems of those orders: build the order keys (payload: order row)
    r2, o_of, l_idx = ops.hash_join(ctx, q_keys[:m1], q_rows[:m1], l_keys[:k_l], capacity=k_l,
                                    stream=stream)
    m2 = _count(ctx, r2, stream)
    if m2 == 0:
        return empty
    l_row = ops.gather_u32(ctx, l_rows, l_idx, m2, stream=stream)
    rev = ops.project(ctx, m2, [li.price, (li.discount, 1, 100)], rows=l_row, stream=stream)
    r3, outs = ops.group_kernel(ctx, o_of[:m2], rev[:m2], want=("sum",), expected_groups=m1,
                                capacity=m1, stream=stream)
    ng = _count(ctx, r3, stream)
    # descending revenue: two stable sorts of the 64-bit key ~revenue, by its
    # low word (unsigned) and then by its high word (signed)
    sums = outs["sum"][:ng]
    lo32 = ops.project(ctx, ng, [(sums, 1, -1)], out_dtype=L.I32, stream=stream)
    hi32 = ops.project(ctx, ng, [(sums, 1, -1)], out_dtype=L.I32, shift=32, stream=stream)
    _, perm1 = ops.sort_kernel(ctx, lo32[:ng], None, key_dtype=L.U32, stream=stream)
    hi_p = ops.gather_u32(ctx, hi32, perm1, ng, stream=stream)
    _, perm = ops.sort_kernel(ctx, hi_p[:ng], perm1, key_dtype=L.I32, stream=stream)
    k = min(top, ng)
    ctx.sync(stream)
    sel = perm[:k].long()
    rows = outs["key"][:ng][sel]
    c = lambda x: x.cpu().numpy().astype(np.int64)
    return Q3Result(c(s.o_orderkey[rows.long()]), c(sums[sel]), c(s.o_orderdate[rows.long()]),
                    c(s.o_shippriority[rows.long()]), ng)


@dataclass
class Q5Result:
    nation: np.ndarray   # nation codes, by revenue descending (ties: ascending code)
    revenue: np.ndarray  # SUM(price * (100 - discount))


def q5(ctx: ops.Context, s: Schema, stream=None) -> Q5Result:
    """Q5 after pimdal/main/tpc_h/query5/dpu/kernel_q5_1.c..kernel_q5_7.c and
    host/host_q5.cpp:58,83-84,440-500: the nations of one region
    (kernel_q5_1.c: pred_r, the joins region-nation and nation-customer),
    their customers' orders dated in [Q5_DATE_LO, Q5_DATE_HI), those orders'
    lineitems, and their suppliers, keeping the lineitems whose supplier
    lies in the customer's nation; revenue price * (100 - discount) summed
    per nation (hash_sum by n_nationkey) and ordered by revenue, descending."""
    lo, hi = packed(Q5_DATE_LO), packed(Q5_DATE_HI)
    li, t = s.li, s.li.tables
    empty = Q5Result(np.zeros(0, np.int64), np.zeros(0, np.int64))
    r_r, _, r_rows = ops.sel_kernel(ctx, s.r_name, ops.make_pred(L.PRED_EQ, Q5_REGION), stream=stream)
    k_r = _count(ctx, r_r, stream)
    if k_r == 0:
        return empty
    r_keys = ops.gather_u32(ctx, s.r_regionkey, r_rows, k_r, stream=stream)
    # nations of the region (payload: nation key), then their customers
    r1, _, n_idx = ops.hash_join(ctx, r_keys[:k_r], r_keys[:k_r], s.n_regionkey, stream=stream)
    k_n = _count(ctx, r1, stream)
    if k_n == 0:
        return empty
    n_keys = ops.gather_u32(ctx, s.n_nationkey, n_idx, k_n, stream=stream)
    r2, c_nat, c_rows = ops.hash_join(ctx, n_keys[:k_n], n_keys[:k_n], s.c_nationkey, stream=stream)
    k_c = _count(ctx, r2, stream)
    r_o, _, o_rows = ops.sel_kernel(ctx, s.o_orderdate, ops.make_pred(L.PRED_RANGE, lo, hi),
                                    stream=stream)
    k_o = _count(ctx, r_o, stream)
    if k_c == 0 or k_o == 0:
        return empty
    c_keys = ops.gather_u32(ctx, s.c_custkey, c_rows, k_c, stream=stream)
    o_cust = ops.gather_u32(ctx, s.o_custkey, o_rows, k_o, stream=stream)
    # orders of those customers (payload: the customer's nation)
    r3, o_nat, o_idx = ops.hash_join(ctx, c_keys[:k_c], c_nat[:k_c], o_cust[:k_o], capacity=k_o,
                                     stream=stream)
    m_o = _count(ctx, r3, stream)
    if m_o == 0:
        return empty
    q_rows = ops.gather_u32(ctx, o_rows, o_idx, m_o, stream=stream)
    q_keys = ops.gather_u32(ctx, s.o_orderkey, q_rows, m_o, stream=stream)
    # their lineitems (payload: the customer's nation)
    r4, l_nat, l_row = ops.hash_join(ctx, q_keys[:m_o], o_nat[:m_o], t.l_orderkey, stream=stream)
    m_l = _count(ctx, r4, stream)
    if m_l == 0:
        return empty
    # the lineitems' suppliers (payload: the supplier's nation)
    l_supp = ops.gather_u32(ctx, t.l_suppkey, l_row, m_l, stream=stream)
    r5, s_nat, s_idx = ops.hash_join(ctx, s.s_suppkey, s.s_nationkey, l_supp[:m_l], capacity=m_l,
                                     stream=stream)
    m_s = _count(ctx, r5, stream)
    c_nat2 = ops.gather_u32(ctx, l_nat, s_idx, m_s, stream=stream)
    row2 = ops.gather_u32(ctx, l_row, s_idx, m_s, stream=stream)
    same = ops.project(ctx, m_s, [s_nat], minus=[c_nat2], out_dtype=L.I32, stream=stream)
    r6, _, keep = ops.sel_kernel(ctx, same[:m_s], ops.make_pred(L.PRED_EQ, 0), stream=stream)
    k = _count(ctx, r6, stream)
    rev = ops.project(ctx, m_s, [li.price, (li.discount, 1, 100)], rows=row2, stream=stream)
    r7, outs = ops.select_aggregate(ctx, k, rows=keep[:k] if k else keep,
                                    group=[(c_nat2, 1)], key_space=N_NATION, exprs=[[rev]],
                                    stream=stream)
    g = _count(ctx, r7, stream)
    nation = outs["key"][:g].cpu().numpy().astype(np.int64)
    revenue = outs["sum0"][:g].cpu().numpy()
    order = np.lexsort((nation, -revenue))  # host_q5.cpp:493: order by revenue, descending
    return Q5Result(nation[order], revenue[order])


def column_bytes(query: str, s: Schema) -> int:
    """Bytes of the columns a multi-table query reads, each once in full (4 B
    per key, date, code or discount, 8 B per price): Q4 reads the orders'
    date, key and priority and the lineitems' commit date, receipt date and
    order key; Q3 the customers' segment and key, the orders' date, customer
    key, key and ship priority, and the lineitems' ship date, order key,
    price and discount; Q5 the customers' nation and key, the orders' date,
    customer key and key, the lineitems' order key, supplier key, price and
    discount, the suppliers' key and nation, and the nation and region
    columns."""
    o, n, c, sp = s.n_orders, s.n, s.n_cust, s.n_supp
    if query == "q4":
        return 12 * o + 12 * n
    if query == "q3":
        return 8 * c + 16 * o + 20 * n
    if query == "q5":
        return 8 * c + 12 * o + 20 * n + 8 * sp + 8 * N_NATION + 8 * N_REGION
    raise ValueError(query)
