"""Host logic of the served form that needs no GPU: the seeded request
stream and the byte-budget admission controller."""
import numpy as np

from pimdal_b200 import serve


def test_request_stream_is_seeded_and_in_bounds():
    a = serve.make_requests(200, 1_000_000, rate=500.0, seed=3)
    b = serve.make_requests(200, 1_000_000, rate=500.0, seed=3)
    assert [vars(x) for x in a] == [vars(y) for y in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) >= 0) and arr[0] > 0
    for r in a:
        assert 1 <= r.n <= 1_000_000 and 0 <= r.r0 and r.r0 + r.n <= 1_000_000
        assert 0 <= r.d0 <= r.d1 < serve.DAYS
        width = r.d1 - r.d0 + 1
        assert 0.009 * serve.DAYS <= width <= 0.501 * serve.DAYS
    assert all(r.arrival == 0.0 for r in serve.make_requests(10, 10_000, rate=None))
    # log-uniform sizes: most requests are small, some are near the top
    sizes = np.array([r.n for r in serve.make_requests(2000, 60_000_000, rate=None, seed=1)])
    assert np.median(sizes) < 5_000_000 and sizes.max() > 20_000_000


def test_admission_respects_the_byte_budget():
    adm = serve.Admission(100)
    assert adm.fits(60)
    adm.take(60)
    assert not adm.fits(50) and adm.fits(40)
    adm.take(40)
    assert not adm.fits(1)
    adm.give(60)
    assert adm.fits(50)
    adm.give(40)
    # a request larger than the whole budget still runs, alone
    assert adm.fits(1000)
