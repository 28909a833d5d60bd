"""Seeded column generator: numpy mirror of pimdal_gen_column (csrc/gen.cu).

Row i's value is a pure function of (seed, stream_id, i), identical on CPU and
GPU for any launch shape.  It replaces the thread-count-dependent generators
of reference/db_operators/shared.cpp:10-60.  The CPU side is used to build
host-resident inputs (end-to-end runs) and test inputs; tests check that both
sides agree bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as L

M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15
_C1 = np.uint64(0xBF58476D1CE4E5B9)
_C2 = np.uint64(0x94D049BB133111EB)


def _mix64_int(z: int) -> int:
    z &= M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def mix64(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64, copy=False)
    z = (z ^ (z >> np.uint64(30))) * _C1
    z = (z ^ (z >> np.uint64(27))) * _C2
    return z ^ (z >> np.uint64(31))


def stream_key(seed: int, stream: int) -> int:
    return _mix64_int(((seed * GOLDEN) & M64) ^ _mix64_int(stream + 0x632BE59BD9B4E019))


def rand(key: int, rows: np.ndarray) -> np.ndarray:
    return mix64(np.uint64(key) + (rows.astype(np.uint64) + np.uint64(1)) * np.uint64(GOLDEN))


def rand2(r: np.ndarray) -> np.ndarray:
    return mix64(r ^ np.uint64(0xD1B54A32D192ED03))


def uniform(r: np.ndarray, lo: int, span: int) -> np.ndarray:
    """lo + floor(hi32(r) * span / 2^32) as int64 (span <= 2^32)."""
    v = ((r >> np.uint64(32)) * np.uint64(span)) >> np.uint64(32)
    return v.astype(np.int64) + np.int64(lo)


def unit(r: np.ndarray) -> np.ndarray:
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class Perm:
    """Bijection of [0, n) (n = 0 means 2^32), seeded; mirrors pd_perm."""

    def __init__(self, seed: int, n: int):
        self.n = n if n else 1 << 32
        b = 0
        while (1 << b) < self.n:
            b += 1
        self.bits = b
        self.mask = (1 << b) - 1
        self.shift = max(1, (b + 1) // 2)
        k = stream_key(seed, 0xFFFF0000)
        self.mul, self.add = [], []
        for r in range(4):
            c = _mix64_int(k + (r + 1) * GOLDEN)
            self.mul.append((c | 1) & self.mask)
            self.add.append((c >> 32) & self.mask)

    def _pow2(self, x: np.ndarray) -> np.ndarray:
        m = np.uint64(self.mask)
        s = np.uint64(self.shift)
        for r in range(4):
            x = (x * np.uint64(self.mul[r]) + np.uint64(self.add[r])) & m
            x = x ^ (x >> s)
        return x

    def __call__(self, x) -> np.ndarray:
        x = np.asarray(x, dtype=np.uint64)
        if self.bits == 0:
            return np.zeros_like(x)
        y = self._pow2(x)
        n = np.uint64(self.n)
        for _ in range(4096):
            bad = y >= n
            if not bad.any():
                break
            y[bad] = self._pow2(y[bad])
        return np.where(y < n, y, y % n)


def zipf_cdf(n: int, s: float) -> np.ndarray:
    """Normalised CDF of Zipf(s) over ranks 1..n (float64, ascending)."""
    w = np.arange(1, n + 1, dtype=np.float64) ** (-float(s))
    c = np.cumsum(w)
    c /= c[-1]
    return c


def zipf_index(cdf: np.ndarray, u: np.ndarray) -> np.ndarray:
    i = np.searchsorted(cdf, u, side="right").astype(np.uint64)
    return np.minimum(i, np.uint64(len(cdf) - 1))


@dataclass
class Spec:
    """Mirror of pimdal_gen_spec_t."""
    kind: int
    out_dtype: int = L.I32
    seed: int = 0
    stream_id: int = 0
    lo: int = 0
    hi: int = 0
    perm_domain: int = 0
    cdf: np.ndarray | None = None   # host copy of the CDF (uploaded for the GPU)
    match_permille: int = 0

    @property
    def np_dtype(self):
        return {L.U32: np.uint32, L.I32: np.int32, L.I64: np.int64}[self.out_dtype]


def generate_cpu(spec: Spec, n: int, row_offset: int = 0) -> np.ndarray:
    rows = np.arange(row_offset, row_offset + n, dtype=np.uint64)
    key = stream_key(spec.seed, spec.stream_id)
    r = rand(key, rows)
    span = spec.hi - spec.lo + 1
    k = spec.kind
    if k == L.GEN_UNIFORM:
        v = uniform(r, spec.lo, span)
    elif k == L.GEN_PERM:
        v = Perm(spec.seed, spec.perm_domain)(rows).astype(np.int64)
    elif k == L.GEN_PERM_UNIFORM:
        v = Perm(spec.seed, spec.perm_domain)(uniform(r, spec.lo, span).astype(np.uint64)).astype(np.int64)
    elif k == L.GEN_PERM_ZIPF:
        v = Perm(spec.seed, spec.perm_domain)(zipf_index(spec.cdf, unit(r))).astype(np.int64)
    elif k == L.GEN_PROBE:
        dom = spec.perm_domain if spec.perm_domain else 1 << 32
        nb = spec.lo
        match = uniform(rand2(r), 0, 1000) < spec.match_permille
        if spec.cdf is not None:
            idx_m = zipf_index(spec.cdf, unit(r))
        else:
            idx_m = uniform(r, 0, nb).astype(np.uint64)
        idx_n = np.uint64(nb) + uniform(r, 0, dom - nb).astype(np.uint64)
        v = Perm(spec.seed, spec.perm_domain)(np.where(match, idx_m, idx_n)).astype(np.int64)
    else:
        raise ValueError(f"unknown generator kind {k}")
    if spec.out_dtype == L.I64:
        return v.astype(np.int64)
    return (v.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32).view(spec.np_dtype)
