"""GPU parity of the served form: every request's groups (key, SUM of
price * (100 - discount), COUNT) equal a numpy restatement of the pipeline,
and are identical alone (serial plain execution), in the concurrent mix and
under a byte budget that admits one request at a time."""
import numpy as np
import pytest
import torch

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
    served = server.run(reqs)
    serial = server.run(reqs, serial=True)
    assert len(served.results) == len(serial.results) == len(reqs)
    assert served.max_inflight > 1 and serial.max_inflight == 1
    assert serve.same_results(served, serial)
    for r in reqs:
        k, s, c = expected(t, r)
        got = served.results[r.rid]
        assert np.array_equal(got.keys, k) and np.array_equal(got.sums, s), r.rid
        assert np.array_equal(got.counts, c), r.rid


def test_budget_admits_one_request_at_a_time(server):
    t = server.tables
    reqs = serve.make_requests(12, t.n, rate=None, seed=22, min_rows=50_000, max_rows=t.n)
    free = server.budget
    server.budget = min(r.need_bytes for r in reqs)  # room for exactly one request
    try:
        tight = server.run(reqs)
    finally:
        server.budget = free
    assert tight.max_inflight == 1
    assert tight.max_reserved <= max(r.need_bytes for r in reqs)
    loose = server.run(reqs)
    assert serve.same_results(tight, loose)
