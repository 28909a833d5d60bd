"""CPU side of the seeded generator: determinism and distribution properties."""
import numpy as np

from pimdal_b200 import _lib as L
from pimdal_b200 import gen


def test_rows_are_independent_of_offset():
    s = gen.Spec(L.GEN_UNIFORM, L.I32, seed=7, stream_id=3, lo=0, hi=2**31 - 1)
    full = gen.generate_cpu(s, 10000)
    part = gen.generate_cpu(s, 1000, row_offset=4000)
    assert np.array_equal(full[4000:5000], part)


def test_uniform_range_and_streams_differ():
    s = gen.Spec(L.GEN_UNIFORM, L.I64, seed=1, lo=100, hi=10**7)
    v = gen.generate_cpu(s, 200000)
    assert v.min() >= 100 and v.max() <= 10**7
    assert abs(v.mean() - (100 + 10**7) / 2) < 0.01 * 10**7
    s2 = gen.Spec(L.GEN_UNIFORM, L.I64, seed=1, stream_id=1, lo=100, hi=10**7)
    assert not np.array_equal(v[:100], gen.generate_cpu(s2, 100))


def test_full_32bit_uniform():
    s = gen.Spec(L.GEN_UNIFORM, L.U32, seed=2, lo=0, hi=2**32 - 1)
    v = gen.generate_cpu(s, 100000)
    assert v.dtype == np.uint32 and v.max() > 2**31


def test_perm_is_a_bijection():
    for n in (1, 2, 3, 1000, 4096, 65537):
        p = gen.Perm(5, n)(np.arange(n, dtype=np.uint64))
        assert np.array_equal(np.sort(p), np.arange(n, dtype=np.uint64)), n


def test_perm_32bit_distinct():
    p = gen.Perm(9, 0)(np.arange(1 << 16, dtype=np.uint64))
    assert np.unique(p).size == 1 << 16 and p.max() < 2**32


def test_probe_match_rate():
    nb = 4096
    build = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.I32, seed=3, perm_domain=2 * nb), nb)
    probe = gen.generate_cpu(gen.Spec(L.GEN_PROBE, L.I32, seed=3, stream_id=1, lo=nb,
                                      perm_domain=2 * nb, match_permille=500), 100000)
    frac = np.isin(probe, build).mean()
    assert 0.48 < frac < 0.52


def test_zipf_skew():
    cdf = gen.zipf_cdf(1 << 16, 1.0)
    v = gen.generate_cpu(gen.Spec(L.GEN_PERM_ZIPF, L.U32, seed=4, perm_domain=0, cdf=cdf), 200000)
    _, counts = np.unique(v, return_counts=True)
    top = counts.max() / v.size
    expect = 1.0 / np.sum(1.0 / np.arange(1, (1 << 16) + 1))
    assert abs(top - expect) < 0.01
