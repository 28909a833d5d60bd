"""GPU parity of the TPC-H Q1 and Q6 pipelines (pimdal_b200/tpch.py) on the
lineitem-shaped synthetic table: the fused pass (pimdal_select_aggregate),
the staged chain of plain operators (pimdal_sel_kernel + pimdal_gather_u32 +
pimdal_select_aggregate over row ids) and a numpy restatement of the
reference's own check plans (pimdal/main/tpc_h/query6/host/host_q6.cpp:70-100,
pimdal/main/tpc_h/query1/host/host_q1.cpp:263-322) agree exactly (int64).
Also covers the fused scan's edge cases: an empty range, no qualifying row,
a key outside the key space and too small an output."""
import numpy as np
import pytest
import torch

from pimdal_b200 import _lib as L
from pimdal_b200 import ops, serve, tpch

pytestmark = pytest.mark.gpu


def host(li):
    c = lambda t: t.cpu().numpy()
    return dict(date=c(li.shipdate), qty=c(li.quantity), price=c(li.price), disc=c(li.discount),
                tax=c(li.tax), rflag=c(li.returnflag), lstat=c(li.linestatus))


def numpy_q6(h):
    """host_q6.cpp:70-100: three filters, project discount * price, sum."""
    m = (h["date"] >= tpch.packed(tpch.Q6_DATE_LO)) & (h["date"] < tpch.packed(tpch.Q6_DATE_HI))
    m &= h["qty"] < tpch.Q6_QUANTITY
    m &= (h["disc"] >= tpch.Q6_DISCOUNT - 1) & (h["disc"] <= tpch.Q6_DISCOUNT + 1)
    return int((h["disc"][m].astype(np.int64) * h["price"][m]).sum()), int(m.sum())


def numpy_q1(h):
    """host_q1.cpp:263-322: filter, project, hash_sum / hash_count by (flag, status)."""
    m = h["date"] < tpch.packed(tpch.Q1_DATE)
    key = h["rflag"][m].astype(np.int64) * tpch.N_LSTATUS + h["lstat"][m]
    price = h["price"][m]
    disc = h["disc"][m].astype(np.int64)
    disc_price = price * (100 - disc)
    charge = disc_price * (100 + h["tax"][m].astype(np.int64))
    uk = np.unique(key)
    cols = {"sum_qty": h["qty"][m].astype(np.int64), "sum_base_price": price,
            "sum_disc_price": disc_price, "sum_charge": charge, "sum_disc": disc}
    out = {"key": uk}
    for name, v in cols.items():
        out[name] = np.array([v[key == k].sum() for k in uk], np.int64)
    out["count_order"] = np.array([(key == k).sum() for k in uk], np.int64)
    return out


def check_q1(got, exp):
    key = got.returnflag * tpch.N_LSTATUS + got.linestatus
    assert np.array_equal(key, exp["key"])
    for name in ("sum_qty", "sum_base_price", "sum_disc_price", "sum_charge", "sum_disc",
                 "count_order"):
        assert np.array_equal(getattr(got, name), exp[name]), name


@pytest.fixture(scope="module")
def small(ctx):
    t = serve.Tables(ctx, orders=150_000, parts=5_000, supps=1_000, seed=13)
    li = tpch.Lineitem(ctx, t)
    return li, host(li)


def test_q6_fused_staged_numpy_agree(ctx, small):
    li, h = small
    exp_rev, exp_rows = numpy_q6(h)
    f = tpch.q6(ctx, li)
    s = tpch.q6(ctx, li, staged=True)
    assert exp_rows > 0
    assert f.revenue == s.revenue == exp_rev
    assert f.rows == s.rows == exp_rows
    k1, k2, k3 = s.stage_rows
    assert k1 >= k2 >= k3 == exp_rows


def test_q1_fused_staged_numpy_agree(ctx, small):
    li, h = small
    exp = numpy_q1(h)
    check_q1(tpch.q1(ctx, li), exp)
    check_q1(tpch.q1(ctx, li, staged=True), exp)


def test_q1_q6_full_table(ctx):
    """The 6e7-row table of the served form."""
    li = tpch.Lineitem(ctx)
    h = host(li)
    rev, rows = numpy_q6(h)
    f = tpch.q6(ctx, li)
    assert (f.revenue, f.rows) == (rev, rows)
    s = tpch.q6(ctx, li, staged=True)
    assert (s.revenue, s.rows) == (rev, rows)
    exp = numpy_q1(h)
    check_q1(tpch.q1(ctx, li), exp)
    check_q1(tpch.q1(ctx, li, staged=True), exp)


def test_select_aggregate_edges(ctx):
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    n = 5000
    rng = np.random.default_rng(3)
    a = rng.integers(-1000, 1000, n).astype(np.int32)
    b = rng.integers(-2**40, 2**40, n).astype(np.int64)
    g = rng.integers(0, 5, n).astype(np.uint8)
    # empty input: no group
    res, _ = ops.select_aggregate(ctx, 0, preds=[(d(a[:0]), ops.make_pred(L.PRED_LT, 0))],
                                  exprs=[[d(b[:0])]])
    ctx.sync()
    assert int(res.item()) == 0
    # no qualifying row
    res, _ = ops.select_aggregate(ctx, n, preds=[(d(a), ops.make_pred(L.PRED_GT, 5000))],
                                  exprs=[[d(b)]])
    ctx.sync()
    assert int(res.item()) == 0
    # signed predicate, NE, wrapping int64 products, groups from a uint8 column
    res, outs = ops.select_aggregate(ctx, n, preds=[(d(a), ops.make_pred(L.PRED_NE, 7)),
                                                    (d(a), ops.make_pred(L.PRED_GE, -500))],
                                     group=[(d(g), 1)], key_space=5,
                                     exprs=[[d(b), d(b), (d(a), 1, 3)], [-2], [d(a)]])
    ctx.sync()
    m = (a != 7) & (a >= -500)
    with np.errstate(over="ignore"):
        v0 = b * b * (3 - a.astype(np.int64))
    for k in range(5):
        sel = m & (g == k)
        assert int(outs["count"][k]) == sel.sum()
        assert int(outs["sum0"][k]) == int(np.sum(v0[sel], dtype=np.int64))
        assert int(outs["sum1"][k]) == -2 * sel.sum()
        assert int(outs["sum2"][k]) == int(a[sel].astype(np.int64).sum())
    assert int(res.item()) == 5
    # a key beyond the key space
    ops.select_aggregate(ctx, n, group=[(d(g), 1)], key_space=4, exprs=[[d(b)]])
    with pytest.raises(L.PimdalError) as e:
        ctx.sync()
    assert e.value.status == 1
    # too small an output
    small = {"key": torch.empty(2, dtype=torch.int32, device="cuda"),
             "count": torch.empty(2, dtype=torch.int64, device="cuda")}
    res, _ = ops.select_aggregate(ctx, n, group=[(d(g), 1)], key_space=5, outs=small)
    with pytest.raises(L.PimdalError) as e:
        ctx.sync()
    assert e.value.status == 7 and int(res.item()) == 5
