"""GPU parity of the served form: every request's groups (key, SUM of
price * (100 - discount), COUNT) equal a numpy restatement of the pipeline,
and are identical through the fused pass and the staged plain operators,
alone (serial plain execution), in the concurrent mix and under a byte
budget that admits one request at a time.  The fused operator
(pimdal_select_join_aggregate) is also checked on its own: duplicate build
keys, a second group column, empty ranges, no selected row, a key outside the
key space and a full output."""
import numpy as np
import pytest
import torch

from pimdal_b200 import _lib as L
from pimdal_b200 import ops, serve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def server(ctx):
    t = serve.Tables(ctx, orders=60_000, parts=5_000, supps=1_000, seed=11)
    s = serve.Server(t, slots=4)
    s.warm()
    yield s
    s.close()


def expected(t, r):
    date = t.l_date.cpu().numpy()
    rows = np.arange(r.r0, r.r0 + r.n)
    rows = rows[(date[rows] >= r.d0) & (date[rows] <= r.d1)]
    if r.dim == 0:
        okey, oprio = t.o_key.cpu().numpy(), t.o_prio.cpu().numpy()
        order = np.argsort(okey)
        pos = np.searchsorted(okey[order], t.l_orderkey.cpu().numpy()[rows])
        attr = oprio[order][pos]
        flag, nflag = t.l_rflag.cpu().numpy()[rows], serve.N_RFLAG
    else:
        attr = t.p_cat.cpu().numpy()[t.l_partkey.cpu().numpy()[rows] - 1]
        flag, nflag = t.l_lstatus.cpu().numpy()[rows], serve.N_LSTATUS
    key = attr.astype(np.int64) * (nflag if r.two_keys else 1) + (flag if r.two_keys else 0)
    val = t.l_price.cpu().numpy()[rows] * (100 - t.l_discount.cpu().numpy()[rows].astype(np.int64))
    uk, inv = np.unique(key, return_inverse=True)
    sums = np.zeros(uk.size, np.int64)
    np.add.at(sums, inv, val)
    return uk.astype(np.int32), sums, np.bincount(inv, minlength=uk.size).astype(np.int64)


def test_served_equals_serial_and_numpy(server):
    t = server.tables
    reqs = serve.make_requests(40, t.n, rate=2000.0, seed=21, min_rows=1_000, max_rows=t.n)
    served = server.run(reqs)                      # fused passes, concurrent
    staged = server.run(reqs, fused=False)         # staged operators, concurrent
    serial = server.run(reqs, serial=True)         # staged operators, one at a time
    assert len(served.results) == len(serial.results) == len(reqs)
    assert served.max_inflight > 1 and serial.max_inflight == 1
    assert serve.same_results(served, serial) and serve.same_results(staged, serial)
    for r in reqs:
        k, s, c = expected(t, r)
        got = served.results[r.rid]
        assert np.array_equal(got.keys, k) and np.array_equal(got.sums, s), r.rid
        assert np.array_equal(got.counts, c), r.rid


@pytest.mark.parametrize("fused", [True, False])
def test_budget_admits_one_request_at_a_time(server, fused):
    """A budget with room for the smallest request alone admits one request
    at a time; the charge is the request's real device bytes (the fused
    pass's group table, or the staged pass's per-row buffers)."""
    t = server.tables
    reqs = serve.make_requests(12, t.n, rate=None, seed=22, min_rows=50_000, max_rows=t.n)
    need = [r.need_bytes(fused) for r in reqs]
    if fused:
        assert max(need) <= 16 * serve.N_CAT * serve.N_LSTATUS
    else:
        assert need == [serve.STAGED_ROW_BYTES * r.n for r in reqs]
    free = server.budget
    server.budget = min(need)  # room for exactly one request
    try:
        tight = server.run(reqs, fused=fused)
    finally:
        server.budget = free
    assert tight.max_inflight == 1
    assert tight.max_reserved <= max(need)
    loose = server.run(reqs, fused=fused)
    assert loose.max_inflight > 1
    assert serve.same_results(tight, loose)


def fused_expected(date, lo, hi, jkey, bkey, battr, flag, mult, price, disc):
    """numpy: every selected row joined with every build row of its key."""
    sel = np.nonzero((date >= lo) & (date <= hi))[0]
    order = np.argsort(bkey, kind="stable")
    sk = bkey[order]
    keys, vals = [], []
    for r in sel:
        a, b = np.searchsorted(sk, jkey[r], "left"), np.searchsorted(sk, jkey[r], "right")
        for i in order[a:b]:
            keys.append(int(battr[i]) * mult + (int(flag[r]) if flag is not None else 0))
            vals.append(int(price[r]) * (100 - int(disc[r])))
    keys = np.asarray(keys, np.int64)
    vals = np.asarray(vals, np.int64)
    uk, inv = np.unique(keys, return_inverse=True)
    sums = np.zeros(uk.size, np.int64)
    np.add.at(sums, inv, vals)
    return uk, sums, np.bincount(inv, minlength=uk.size).astype(np.int64)


def test_fused_operator_matches_numpy_with_duplicate_build_keys(ctx):
    rng = np.random.default_rng(31)
    n, nb, attrs, nflag = 50_000, 3000, 12, 3
    bkey = rng.integers(0, 2000, nb).astype(np.uint32)   # many duplicate keys
    battr = rng.integers(0, attrs, nb).astype(np.uint32)
    jkey = rng.integers(0, 2600, n).astype(np.uint32)
    date = rng.integers(0, 2557, n).astype(np.int32)
    price = rng.integers(90_000, 10_500_000, n).astype(np.int64)
    disc = rng.integers(0, 11, n).astype(np.int32)
    flag = rng.integers(0, nflag, n).astype(np.uint8)
    d = lambda a: torch.from_numpy(a).cuda()
    table = ops.hash_kernel(ctx, d(bkey.view(np.int32)), d(battr.view(np.int32)), table_size=8192)
    for lo, hi, fl in ((300, 1500, flag), (0, 2556, None), (3000, 4000, None)):
        mult = nflag if fl is not None else 1
        res, outs = ops.select_join_aggregate(
            ctx, d(date), lo, hi, d(jkey.view(np.int32)), table, 8192, d(price), d(disc),
            flag=None if fl is None else d(fl), attr_mult=mult, key_space=attrs * mult)
        ctx.sync()
        g = int(res.item())
        k, s_, c = fused_expected(date, lo, hi, jkey, bkey, battr, fl, mult, price, disc)
        assert g == k.size
        assert np.array_equal(outs["key"][:g].cpu().numpy(), k)
        assert np.array_equal(outs["sum"][:g].cpu().numpy(), s_)
        assert np.array_equal(outs["count"][:g].cpu().numpy(), c)


def test_fused_operator_edges(ctx):
    d = lambda a: torch.from_numpy(a).cuda()
    bkey = np.arange(100, dtype=np.int32)
    table = ops.hash_kernel(ctx, d(bkey), d(bkey % 7), table_size=256)
    z32, z64 = np.zeros(0, np.int32), np.zeros(0, np.int64)
    res, _ = ops.select_join_aggregate(ctx, d(z32), 0, 10, d(z32), table, 256, d(z64), d(z32),
                                       key_space=7)
    ctx.sync()
    assert int(res.item()) == 0
    n = 1000
    date = np.full(n, 5, np.int32)
    jk = np.arange(n, dtype=np.int32) % 100
    price, disc = np.ones(n, np.int64), np.zeros(n, np.int32)
    res, _ = ops.select_join_aggregate(ctx, d(date), 6, 9, d(jk), table, 256, d(price), d(disc),
                                       key_space=7)
    ctx.sync()
    assert int(res.item()) == 0  # no row selected
    res, _ = ops.select_join_aggregate(ctx, d(date), 0, 9, d(jk), table, 256, d(price), d(disc),
                                       key_space=6)  # attribute 6 lies outside the key space
    with pytest.raises(L.PimdalError) as e:
        ctx.sync()
    assert e.value.status == 1
    small = {"key": torch.empty(3, dtype=torch.int32, device="cuda"),
             "sum": torch.empty(3, dtype=torch.int64, device="cuda"),
             "count": torch.empty(3, dtype=torch.int64, device="cuda")}
    res, _ = ops.select_join_aggregate(ctx, d(date), 0, 9, d(jk), table, 256, d(price), d(disc),
                                       key_space=7, outs=small)
    with pytest.raises(L.PimdalError) as e:
        ctx.sync()
    assert e.value.status == 7 and int(res.item()) == 7


def test_fused_and_staged_agree_on_the_all_ones_build_row(ctx):
    """A build row whose key and payload are both 0xFFFFFFFF is the one row
    the table counts on the side (its slot word would equal the empty word).
    The fused pass and the staged operators (probe, then pimdal_revenue_keys,
    then the group-by) compute the same 32-bit wrapping group key for it:
    with attr_mult 1 and flag 1 the attribute 0xFFFFFFFF wraps to key 0."""
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    bkey = np.array([0xFFFFFFFF, 0xFFFFFFFF, 7, 9], np.uint32)
    battr = np.array([0xFFFFFFFF, 2, 1, 0xFFFFFFFF], np.uint32)
    table = ops.hash_kernel(ctx, d(bkey.view(np.int32)), d(battr.view(np.int32)), table_size=64)
    n = 64
    jkey = np.array([0xFFFFFFFF, 7, 9, 3] * (n // 4), np.uint32)
    date = np.arange(n, dtype=np.int32)
    price = (np.arange(n, dtype=np.int64) + 1) * 1000
    disc = (np.arange(n) % 11).astype(np.int32)
    flag = np.ones(n, np.uint8)
    lo, hi = 3, 50
    res, outs = ops.select_join_aggregate(
        ctx, d(date), lo, hi, d(jkey.view(np.int32)), table, 64, d(price), d(disc),
        flag=d(flag), attr_mult=1, key_space=8)
    ctx.sync()
    g = int(res.item())
    fused = tuple(outs[c][:g].cpu().numpy() for c in ("key", "sum", "count"))
    # staged: selected rows -> join-key gather -> probe -> revenue keys -> group-by
    sel = np.flatnonzero((date >= lo) & (date <= hi)).astype(np.int32)
    jk_sel = d(jkey[sel].view(np.int32))
    pres, prow, pay = ops.hj_probe(ctx, table, 64, jk_sel)  # probe row = index into sel
    ctx.sync()
    m = int(pres.item())
    kt = torch.empty(m, dtype=torch.int32, device="cuda")
    vt = torch.empty(m, dtype=torch.int64, device="cuda")
    ops.revenue_keys(ctx, m, prow, pay, d(sel), d(price), d(disc), d(flag), 1, kt, vt)
    gres, gouts = ops.group_kernel(ctx, kt, vt, key_dtype=L.U32, method=L.GROUP_HASH,
                                   expected_groups=16)
    ctx.sync()
    gg = int(gres.item())
    staged = (gouts["key"][:gg].cpu().numpy(), gouts["sum"][:gg].cpu().numpy(),
              gouts["count"][:gg].cpu().numpy())
    # numpy restatement: every (selected row, matching build row) pair
    keys, vals = [], []
    for r in sel:
        for b in range(bkey.size):
            if bkey[b] == jkey[r]:
                keys.append((int(battr[b]) * 1 + 1) & 0xFFFFFFFF)
                vals.append(int(price[r]) * (100 - int(disc[r])))
    uk, inv = np.unique(np.asarray(keys, np.int64), return_inverse=True)
    sums = np.zeros(uk.size, np.int64)
    np.add.at(sums, inv, np.asarray(vals, np.int64))
    cnts = np.bincount(inv, minlength=uk.size)
    assert g == gg == uk.size
    assert np.array_equal(fused[0].view(np.uint32), uk) and np.array_equal(staged[0].view(np.uint32), uk)
    assert np.array_equal(fused[1], sums) and np.array_equal(staged[1], sums)
    assert np.array_equal(fused[2], cnts) and np.array_equal(staged[2], cnts)
