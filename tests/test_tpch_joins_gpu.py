"""GPU parity of the TPC-H Q4, Q3 and Q5 pipelines (pimdal_b200/tpch.py) on
the synthetic multi-table schema: each query's chain of plain operators
through the C ABI equals a numpy restatement of the reference's pipeline
(pimdal/main/tpc_h/query4/dpu/kernel_q4_1.c..4, query3/dpu/kernel_q3_1.c..5,
query5/dpu/kernel_q5_1.c..7 with their hosts' parameters and final
orderings).  Also covers pimdal_project, the per-row arithmetic the
pipelines use."""
import numpy as np
import pytest
import torch

from pimdal_b200 import _lib as L
from pimdal_b200 import ops, serve, tpch

pytestmark = pytest.mark.gpu


def host(s: tpch.Schema) -> dict:
    t, li = s.li.tables, s.li
    c = lambda x: x.cpu().numpy().astype(np.int64)
    return dict(o_key=c(s.o_orderkey), o_date=c(s.o_orderdate), o_prio=c(s.o_orderpriority),
                o_cust=c(s.o_custkey), o_ship=c(s.o_shippriority), c_seg=c(s.c_mktsegment),
                c_nat=c(s.c_nationkey), s_nat=c(s.s_nationkey), n_reg=c(s.n_regionkey),
                l_okey=c(t.l_orderkey), l_supp=c(t.l_suppkey), l_ship=c(li.shipdate),
                l_commit=c(s.l_commitdate), l_receipt=c(s.l_receiptdate), price=c(li.price),
                disc=c(li.discount))


def order_row_of(h, keys):
    """Row of each order key in the orders table (keys must exist); the
    queries are searched in sorted order, which keeps large lookups fast."""
    srt = np.argsort(h["o_key"], kind="stable")
    qo = np.argsort(keys, kind="stable")
    pos = np.empty(keys.size, np.int64)
    pos[qo] = np.searchsorted(h["o_key"][srt], keys[qo])
    return srt[pos]


def numpy_q4(h):
    lo, hi = tpch.packed(tpch.Q4_DATE_LO), tpch.packed(tpch.Q4_DATE_HI)
    late_keys = np.unique(h["l_okey"][h["l_commit"] < h["l_receipt"]])
    ok = (h["o_date"] >= lo) & (h["o_date"] < hi) & np.isin(h["o_key"], late_keys)
    cnt = np.bincount(h["o_prio"][ok], minlength=serve.N_PRIO)
    pr = np.nonzero(cnt)[0]
    return pr, cnt[pr]


def group_sum(keys, vals):
    """(distinct keys ascending, exact int64 sums) by a stable sort."""
    o = np.argsort(keys, kind="stable")
    k, v = keys[o], vals[o]
    if k.size == 0:
        return k, v
    starts = np.concatenate(([0], np.nonzero(k[1:] != k[:-1])[0] + 1))
    return k[starts], np.add.reduceat(v, starts)


def numpy_q3(h, top=10):
    d = tpch.packed(tpch.Q3_DATE)
    custs = np.nonzero(h["c_seg"] == tpch.Q3_SEGMENT)[0] + 1          # customer keys
    o_ok = (h["o_date"] < d) & np.isin(h["o_cust"], custs)
    l_ok = (h["l_ship"] > d) & np.isin(h["l_okey"], h["o_key"][o_ok])
    orow = order_row_of(h, h["l_okey"][l_ok])
    rows, sums = group_sum(orow, h["price"][l_ok] * (100 - h["disc"][l_ok]))
    order = np.lexsort((rows, -sums))[:top]
    r = rows[order]
    return h["o_key"][r], sums[order], h["o_date"][r], h["o_ship"][r], rows.size


def numpy_q5(h):
    lo, hi = tpch.packed(tpch.Q5_DATE_LO), tpch.packed(tpch.Q5_DATE_HI)
    nations = np.nonzero(h["n_reg"] == tpch.Q5_REGION)[0]
    cust_nat = h["c_nat"][h["o_cust"] - 1]                             # per order
    o_ok = (h["o_date"] >= lo) & (h["o_date"] < hi) & np.isin(cust_nat, nations)
    orow = order_row_of(h, h["l_okey"])
    l_ok = o_ok[orow]
    cn = cust_nat[orow]
    sn = h["s_nat"][h["l_supp"] - 1]
    keep = l_ok & (cn == sn)
    nat, rev = group_sum(cn[keep], h["price"][keep] * (100 - h["disc"][keep]))
    order = np.lexsort((nat, -rev))
    return nat[order], rev[order]


@pytest.fixture(scope="module")
def schema(ctx):
    t = serve.Tables(ctx, orders=150_000, parts=5_000, supps=1_000, seed=13)
    li = tpch.Lineitem(ctx, t)
    s = tpch.Schema(ctx, li, customers=15_000)
    return s, host(s)


def test_q4_matches_numpy(ctx, schema):
    s, h = schema
    pr, cnt = numpy_q4(h)
    got = tpch.q4(ctx, s)
    assert cnt.sum() > 0
    assert np.array_equal(got.priority, pr) and np.array_equal(got.order_count, cnt)


def test_q3_matches_numpy(ctx, schema):
    s, h = schema
    okey, rev, odate, ship, ng = numpy_q3(h)
    got = tpch.q3(ctx, s)
    assert ng > 10 and got.groups == ng
    assert np.array_equal(got.orderkey, okey)
    assert np.array_equal(got.revenue, rev)
    assert np.array_equal(got.orderdate, odate) and np.array_equal(got.shippriority, ship)
    # a longer list exercises the 64-bit descending order through both sorts
    okey, rev, _, _, _ = numpy_q3(h, top=1000)
    got = tpch.q3(ctx, s, top=1000)
    assert np.array_equal(got.orderkey, okey) and np.array_equal(got.revenue, rev)


def test_q5_matches_numpy(ctx, schema):
    s, h = schema
    nat, rev = numpy_q5(h)
    got = tpch.q5(ctx, s)
    assert nat.size > 0
    assert np.array_equal(got.nation, nat) and np.array_equal(got.revenue, rev)


def test_q4_q3_q5_full_schema(ctx):
    """The 6e7-row lineitem table of the served form with 1.5e7 orders and
    1.5e6 customers: every query equals its numpy restatement."""
    s = tpch.Schema(ctx, tpch.Lineitem(ctx))
    h = host(s)
    pr, cnt = numpy_q4(h)
    got = tpch.q4(ctx, s)
    assert np.array_equal(got.priority, pr) and np.array_equal(got.order_count, cnt)
    okey, rev, odate, ship, ng = numpy_q3(h)
    got = tpch.q3(ctx, s)
    assert got.groups == ng and np.array_equal(got.orderkey, okey)
    assert np.array_equal(got.revenue, rev) and np.array_equal(got.orderdate, odate)
    assert np.array_equal(got.shippriority, ship)
    nat, rev = numpy_q5(h)
    got = tpch.q5(ctx, s)
    assert np.array_equal(got.nation, nat) and np.array_equal(got.revenue, rev)


def test_project_gather_products_and_high_words(ctx):
    rng = np.random.default_rng(5)
    n = 100_003
    a = rng.integers(-2**31, 2**31, n).astype(np.int32)
    b = rng.integers(-2**40, 2**40, n).astype(np.int64)
    u = rng.integers(0, 256, n).astype(np.uint8)
    rows = rng.permutation(n)[: n // 3].astype(np.int32)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    da, db, du, dr = d(a), d(b), d(u), d(rows)
    # gather of an int64 column by row ids
    got = ops.project(ctx, rows.size, [db], rows=dr)
    ctx.sync()
    assert np.array_equal(got.cpu().numpy(), b[rows])
    # (a) * (100 - u) * (-b + 7), wrapping int64, all rows
    got = ops.project(ctx, n, [da, (du, 1, 100), (db, 1, 7)])
    ctx.sync()
    with np.errstate(over="ignore"):
        exp = a.astype(np.int64) * (100 - u.astype(np.int64)) * (7 - b)
    assert np.array_equal(got.cpu().numpy(), exp)
    # low and high 32-bit words of ~b
    lo = ops.project(ctx, n, [(db, 1, -1)], out_dtype=L.I32)
    hi = ops.project(ctx, n, [(db, 1, -1)], out_dtype=L.I32, shift=32)
    ctx.sync()
    nb = ~b
    assert np.array_equal(lo.cpu().numpy(), (nb & 0xFFFFFFFF).astype(np.uint32).view(np.int32))
    assert np.array_equal(hi.cpu().numpy(), (nb >> 32).astype(np.int32))
    # a difference of two expressions, 32-bit output
    got = ops.project(ctx, n, [da], minus=[du, (da, 0, 1)], out_dtype=L.I32)
    ctx.sync()
    with np.errstate(over="ignore"):
        exp = a.astype(np.int64) - u.astype(np.int64) * (a.astype(np.int64) + 1)
    assert np.array_equal(got.cpu().numpy(), (exp & 0xFFFFFFFF).astype(np.uint32).view(np.int32))
    # a constant-only expression and an empty call
    got = ops.project(ctx, 10, [-3, 5])
    ctx.sync()
    assert np.array_equal(got[:10].cpu().numpy(), np.full(10, -15))
    ops.project(ctx, 0, [da])
    ctx.sync()
