"""CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm may import this package, and only as the checker or the timed CPU
baseline.  The product (pimdal_b200) never imports it.

Two layers:
  * liboracle.so -- plain-C restatement of the reference algorithms
    (oracle.c, built by `make -C oracle`);
  * _ref/libref_*.so -- the reference's own CPU operators from
    reference/db_operators, compiled where they lie through oracle/ref/*.cpp
    (`make -C oracle ref`, needs the reference checkout at build time only).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_P = C.c_void_p
_U64 = C.c_uint64


def build(ref: bool = False) -> None:
    """Builds liboracle.so (and, with ref=True, the reference harnesses)."""
    targets = ["oracle"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True)


def _p(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        l = C.CDLL(str(path), mode=os.RTLD_LOCAL)
        l.oracle_select.restype = _U64
        l.oracle_select.argtypes = [_P, _U64, C.c_int, C.c_int64, C.c_int64, C.c_int, _P, _U64, _P, _P]
        l.oracle_sort_pairs.restype = None
        l.oracle_sort_pairs.argtypes = [_P, _P, _U64, C.c_int, _P, _P]
        l.oracle_smj_merge.restype = _U64
        l.oracle_smj_merge.argtypes = [_P, _P, _U64, _P, _P, _U64, C.c_int, _P, _P, _U64]
        l.oracle_hash_join.restype = _U64
        l.oracle_hash_join.argtypes = [_P, _P, _U64, _P, _P, _U64, C.c_uint32, _P, _P, _U64]
        l.oracle_part_hash0.restype = None
        l.oracle_part_hash0.argtypes = [_P, _P, _U64, C.c_uint32, C.c_uint32, _P, _P, _P]
        l.oracle_hash.restype = C.c_uint32
        l.oracle_hash.argtypes = [C.c_int, C.c_uint32]
        l.oracle_bloom_build.restype = None
        l.oracle_bloom_build.argtypes = [_P, _P, C.c_uint32, _P]
        l.oracle_bloom_match.restype = _U64
        l.oracle_bloom_match.argtypes = [_P, _P, _P, _U64, _P, C.c_uint32, _P, _P, _U64, _P]
        for f in (l.oracle_group_by, l.oracle_sort_group_by):
            f.restype = _U64
            f.argtypes = [_P, _P, _U64, _P, _P, _P, _P, _P]
        _lib = l
    return _lib


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a).view(np.uint32) if np.asarray(a).dtype.itemsize == 4
                                else np.asarray(a, dtype=np.uint32))


# ----------------------------------------------------------------- select
def select(keys: np.ndarray, lo: int, hi: int, invert: bool = False, is_signed: bool = True,
           in_ptr: np.ndarray | None = None, ptr_base: int = 0):
    """Returns (values, row ids) of the selected rows, ascending by row."""
    k = _u32(keys)
    n = k.size
    out_k = np.empty(max(n, 1), np.uint32)
    out_p = np.empty(max(n, 1), np.uint32)
    ip = None if in_ptr is None else _u32(in_ptr)
    c = lib().oracle_select(_p(k), n, int(is_signed), lo, hi, int(invert), _p(ip), ptr_base,
                            _p(out_k), _p(out_p))
    dt = np.int32 if is_signed else np.uint32
    return out_k[:c].view(dt), out_p[:c]


def sort_pairs(keys: np.ndarray, ptr: np.ndarray | None = None, is_signed: bool = False):
    k = _u32(keys)
    n = k.size
    ok = np.empty(max(n, 1), np.uint32)
    op = np.empty(max(n, 1), np.uint32)
    pp = None if ptr is None else _u32(ptr)
    lib().oracle_sort_pairs(_p(k), _p(pp), n, int(is_signed), _p(ok), _p(op))
    return ok[:n], op[:n]


def smj_merge(ikey, iptr, okey, optr, is_signed: bool = True):
    ik, ip, ok, op = map(_u32, (ikey, iptr, okey, optr))
    cnt = lib().oracle_smj_merge(_p(ik), _p(ip), ik.size, _p(ok), _p(op), ok.size, int(is_signed),
                                 None, None, 0)
    oo = np.empty(max(cnt, 1), np.uint32)
    oi = np.empty(max(cnt, 1), np.uint32)
    lib().oracle_smj_merge(_p(ik), _p(ip), ik.size, _p(ok), _p(op), ok.size, int(is_signed),
                           _p(oo), _p(oi), cnt)
    return oo[:cnt], oi[:cnt]


def sort_merge_join(rkey, rpay, skey, spay, is_signed: bool = True):
    """Sorts R and S stably by key and merges; returns (R payload, S payload)
    per match, S-major (outer = S, inner = R)."""
    rk, rp = sort_pairs(rkey, rpay, is_signed)
    sk, sp = sort_pairs(skey, spay, is_signed)
    s_pay, r_pay = smj_merge(rk, rp, sk, sp, is_signed)
    return r_pay, s_pay


def hash_join(bkey, bpay, pkey, prow=None, part_n: int = 16384):
    bk, bp, pk = map(_u32, (bkey, bpay, pkey))
    pr = None if prow is None else _u32(prow)
    cnt = lib().oracle_hash_join(_p(bk), _p(bp), bk.size, _p(pk), _p(pr), pk.size, part_n,
                                 None, None, 0)
    op = np.empty(max(cnt, 1), np.uint32)
    orow = np.empty(max(cnt, 1), np.uint32)
    lib().oracle_hash_join(_p(bk), _p(bp), bk.size, _p(pk), _p(pr), pk.size, part_n,
                           _p(op), _p(orow), cnt)
    return op[:cnt], orow[:cnt]


def part_hash0(keys, ptr=None, shift: int = 32, part_n: int = 32):
    k = _u32(keys)
    n = k.size
    ok = np.empty(max(n, 1), np.uint32)
    op = np.empty(max(n, 1), np.uint32)
    sizes = np.empty(part_n + 1, np.uint64)
    pp = None if ptr is None else _u32(ptr)
    lib().oracle_part_hash0(_p(k), _p(pp), n, shift, part_n, _p(ok), _p(op), _p(sizes))
    return ok[:n], op[:n], sizes


FILTER_BITS = 16384
FILTER_BYTES = FILTER_BITS // 8


def hash_fn(which: int, keys) -> np.ndarray:
    """hash0 (which = 0) or the filter hash hashK (which = K = 1..4)."""
    f = lib().oracle_hash
    return np.fromiter((f(which, int(x)) for x in _u32(keys)), np.uint32, count=np.size(keys))


def bloom_build(keys, part_sizes) -> np.ndarray:
    """One FILTER_BYTES filter per partition of the partitioned keys
    (part_sizes: part_n + 1 offsets), as a uint8 array."""
    k = _u32(keys)
    ps = np.ascontiguousarray(part_sizes, dtype=np.uint64)
    part_n = ps.size - 1
    out = np.zeros(max(part_n, 1) * FILTER_BYTES, np.uint8)
    lib().oracle_bloom_build(_p(k), _p(ps), part_n, _p(out))
    return out[:part_n * FILTER_BYTES]


def bloom_match(filters, keys, part_sizes, ptr=None):
    """Kept (keys, row ids) in input order and match_sizes (part_n + 1)."""
    f = np.ascontiguousarray(filters, dtype=np.uint8)
    k = _u32(keys)
    ps = np.ascontiguousarray(part_sizes, dtype=np.uint64)
    part_n = ps.size - 1
    pp = None if ptr is None else _u32(ptr)
    ok = np.empty(max(k.size, 1), np.uint32)
    op = np.empty(max(k.size, 1), np.uint32)
    ms = np.empty(part_n + 1, np.uint64)
    c = lib().oracle_bloom_match(_p(f), _p(k), _p(pp), k.size, _p(ps), part_n, _p(ok), _p(op),
                                 k.size, _p(ms))
    return ok[:c], op[:c], ms


def _group(fn, keys, vals, max_groups=None):
    k = np.ascontiguousarray(keys, dtype=np.int32)
    v = None if vals is None else np.ascontiguousarray(vals, dtype=np.int64)
    n = k.size
    cap = max(1, n if max_groups is None else min(n, max_groups))
    outs = [np.empty(cap, np.int32)] + [np.empty(cap, np.int64) for _ in range(4)]
    if max_groups is not None and n > cap:
        # the C function writes every group: bound the count first
        if np.unique(k).size > cap:
            raise ValueError("more groups than max_groups")
    g = fn(_p(k), _p(v), n, *map(_p, outs))
    return tuple(o[:g] for o in outs)


def group_by(keys, vals=None, max_groups=None):
    """(key, SUM, COUNT, MIN, MAX) per group, ascending by key.  max_groups
    (optional) bounds the output arrays' size."""
    return _group(lib().oracle_group_by, keys, vals, max_groups)


def sort_group_by(keys, vals=None):
    return _group(lib().oracle_sort_group_by, keys, vals)


def _key_parts(keys_u32: np.ndarray, parts_log2: int) -> np.ndarray:
    """Partition index of every key: the top bits of key * 2^64/phi."""
    h = keys_u32.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    return (h >> np.uint64(64 - parts_log2)).astype(np.uint16)


def _split_by_key(parts_log2: int, keys_u32: np.ndarray, *cols):
    """Rows regrouped by key partition (stable): (bounds, keys, cols...)."""
    part = _key_parts(keys_u32, parts_log2)
    order = np.argsort(part, kind="stable")
    bounds = np.concatenate([[0], np.cumsum(np.bincount(part, minlength=1 << parts_log2))])
    return (bounds, keys_u32[order]) + tuple(None if c is None else c[order] for c in cols)


def group_by_parallel(keys, vals=None, threads: int = 16, parts_log2: int = 6):
    """group_by over disjoint key partitions in host threads (the C oracle
    releases the GIL): every group lies in one partition, so the union of the
    partitions' groups, ordered by key, is exactly group_by(keys, vals)."""
    from concurrent.futures import ThreadPoolExecutor
    k = np.ascontiguousarray(keys, dtype=np.int32)
    v = None if vals is None else np.ascontiguousarray(vals, dtype=np.int64)
    bounds, ks, vs = _split_by_key(parts_log2, k.view(np.uint32), v)
    ks = ks.view(np.int32)

    def one(p):
        a, b = int(bounds[p]), int(bounds[p + 1])
        return group_by(ks[a:b], None if vs is None else vs[a:b])

    with ThreadPoolExecutor(threads) as ex:
        res = list(ex.map(one, range(1 << parts_log2)))
    cols = [np.concatenate([r[i] for r in res]) for i in range(5)]
    order = np.argsort(cols[0], kind="stable")
    return tuple(c[order] for c in cols)


def hash_join_parallel(bkey, bpay, pkey, threads: int = 16, parts_log2: int = 6):
    """hash_join over disjoint key partitions in host threads: a probe row
    can only match build rows of its own key partition, so the union of the
    partitions' matches is the multiset hash_join(bkey, bpay, pkey) returns
    (probe row ids are global)."""
    from concurrent.futures import ThreadPoolExecutor
    bk, bp, pk = map(_u32, (bkey, bpay, pkey))
    bb, bks, bps = _split_by_key(parts_log2, bk, bp)
    pb, pks, prow = _split_by_key(parts_log2, pk, np.arange(pk.size, dtype=np.uint32))

    def one(p):
        a, b = int(bb[p]), int(bb[p + 1])
        c, d = int(pb[p]), int(pb[p + 1])
        if a == b or c == d:
            return np.zeros(0, np.uint32), np.zeros(0, np.uint32)
        return hash_join(bks[a:b], bps[a:b], pks[c:d], prow[c:d])

    with ThreadPoolExecutor(threads) as ex:
        res = list(ex.map(one, range(1 << parts_log2)))
    return (np.concatenate([r[0] for r in res]), np.concatenate([r[1] for r in res]))


# ------------------------------------------------------------ reference libs
class Ref:
    """The reference's own CPU operators (oracle/_ref/libref_*.so)."""

    def __init__(self):
        self._libs: dict[str, C.CDLL] = {}

    @staticmethod
    def available(name: str = "select") -> bool:
        return (REF_DIR / f"libref_{name}.so").exists()

    def _get(self, name: str) -> C.CDLL:
        if name not in self._libs:
            path = REF_DIR / f"libref_{name}.so"
            if not path.exists():
                raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
            self._libs[name] = C.CDLL(str(path), mode=os.RTLD_LOCAL)
        return self._libs[name]

    def set_threads(self, name: str, t: int) -> None:
        f = self._get(name).pimdal_ref_set_threads
        f.argtypes = [C.c_int]
        f(t)

    def sel_count(self, keys: np.ndarray, lo: int, hi: int) -> int:
        f = self._get("select").pimdal_ref_sel_count
        f.restype = _U64
        f.argtypes = [_P, _U64, C.c_int64, C.c_int64]
        k = np.ascontiguousarray(keys, dtype=np.int32)
        return int(f(_p(k), k.size, lo, hi))

    def select(self, keys: np.ndarray, lo: int, hi: int) -> np.ndarray:
        f = self._get("select").pimdal_ref_select
        f.restype = _U64
        f.argtypes = [_P, _U64, C.c_int64, C.c_int64, _P]
        k = np.ascontiguousarray(keys, dtype=np.int32)
        out = np.empty(k.size + 1, np.int32)
        c = int(f(_p(k), k.size, lo, hi, _p(out)))
        return out[:c]

    def sort_pairs(self, keys, ptr=None, is_signed: bool = False):
        f = self._get("sort").pimdal_ref_sort_pairs
        f.restype = None
        f.argtypes = [_P, _P, _U64, C.c_int, _P, _P]
        k = _u32(keys)
        pp = None if ptr is None else _u32(ptr)
        ok = np.empty(max(k.size, 1), np.uint32)
        op = np.empty(max(k.size, 1), np.uint32)
        f(_p(k), _p(pp), k.size, int(is_signed), _p(ok), _p(op))
        return ok[:k.size], op[:k.size]

    def sort_packed(self, packed: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        """The reference's sort_kernel on pre-packed (key, index) pairs: uint64
        words with the key in the low 32 bits (pack with pack_pairs)."""
        f = self._get("sort").pimdal_ref_sort_packed
        f.restype = None
        f.argtypes = [_P, _P, _U64]
        src = np.ascontiguousarray(packed, dtype=np.uint64)
        if out is None:
            out = np.empty(max(src.size, 1), np.uint64)
        f(_p(src), _p(out), src.size)
        return out[:src.size]

    @staticmethod
    def pack_pairs(keys) -> np.ndarray:
        """(key, row index) pairs as the sort harness's 64-bit words."""
        k = _u32(keys).astype(np.uint64)
        return k | (np.arange(k.size, dtype=np.uint64) << np.uint64(32))

    def sort_keys(self, keys):
        f = self._get("sort").pimdal_ref_sort_keys
        f.restype = None
        f.argtypes = [_P, _P, _U64]
        k = _u32(keys)
        out = np.empty(max(k.size, 1), np.uint32)
        f(_p(k), _p(out), k.size)
        return out[:k.size]

    def hash_join(self, bkey, bpay, pkey, part_n: int = 16384):
        f = self._get("hash_join").pimdal_ref_hash_join
        f.restype = _U64
        f.argtypes = [_P, _P, _U64, _P, _U64, C.c_uint32, _P, _P]
        bk, bp, pk = map(_u32, (bkey, bpay, pkey))
        op = np.empty(max(pk.size, 1), np.uint32)
        orow = np.empty(max(pk.size, 1), np.uint32)
        c = int(f(_p(bk), _p(bp), bk.size, _p(pk), pk.size, part_n, _p(op), _p(orow)))
        return op[:c], orow[:c]

    def group_by(self, keys, vals):
        f = self._get("aggregate").pimdal_ref_group_by
        f.restype = _U64
        f.argtypes = [_P, _P, _U64, _P, _P, _P, _P, _P]
        k = np.ascontiguousarray(keys, dtype=np.int32)
        v = np.ascontiguousarray(vals, dtype=np.int64)
        n = k.size
        outs = [np.empty(max(n, 1), np.int32)] + [np.empty(max(n, 1), np.int64) for _ in range(4)]
        g = int(f(_p(k), _p(v), n, *map(_p, outs)))
        return tuple(o[:g] for o in outs)

    def hash_fn(self, which: int, keys) -> np.ndarray:
        f = self._get("bloom").pimdal_ref_hash
        f.restype = None
        f.argtypes = [C.c_int, _P, _U64, _P]
        k = _u32(keys)
        out = np.empty(max(k.size, 1), np.uint32)
        f(which, _p(k), k.size, _p(out))
        return out[:k.size]

    def bloom_build(self, keys, part_sizes) -> np.ndarray:
        f = self._get("bloom").pimdal_ref_bloom_build
        f.restype = None
        f.argtypes = [_P, _P, C.c_uint32, _P]
        k = _u32(keys)
        ps = np.ascontiguousarray(part_sizes, dtype=np.uint64)
        out = np.zeros(max(ps.size - 1, 1) * FILTER_BYTES, np.uint8)
        f(_p(k), _p(ps), ps.size - 1, _p(out))
        return out[:(ps.size - 1) * FILTER_BYTES]

    def bloom_match(self, filters, keys, part_sizes, ptr=None):
        f = self._get("bloom").pimdal_ref_bloom_match
        f.restype = _U64
        f.argtypes = [_P, _P, _P, _P, C.c_uint32, _P, _P, _P]
        fl = np.ascontiguousarray(filters, dtype=np.uint8)
        k = _u32(keys)
        ps = np.ascontiguousarray(part_sizes, dtype=np.uint64)
        pp = None if ptr is None else _u32(ptr)
        ok = np.empty(max(k.size, 1), np.uint32)
        op = np.empty(max(k.size, 1), np.uint32)
        ms = np.empty(ps.size, np.uint64)
        c = int(f(_p(fl), _p(k), _p(pp), _p(ps), ps.size - 1, _p(ok), _p(op), _p(ms)))
        return ok[:c], op[:c], ms

    def date_to_int(self, dates) -> np.ndarray:
        """The reference reader's packed dates of "YYYY-MM-DD" strings."""
        f = self._get("reader").pimdal_ref_date_to_int
        f.restype = None
        f.argtypes = [C.c_char_p, _U64, _P]
        buf = "".join(dates).encode()
        assert len(buf) == 10 * len(dates)
        out = np.empty(max(len(dates), 1), np.int32)
        f(buf, len(dates), _p(out))
        return out[:len(dates)]

    def smj(self, inner_keys, outer_keys, buffer_size: int, threads: int = 1):
        """Reference sort-merge join on key columns (the outer size must equal
        the library's BUFFER_SIZE).  With one thread the result is exact:
        (matched inner keys, sorted outer keys); with more threads the
        reference's shared merge cursor races (sort_merge_join.cpp:81-101),
        which is only used for timing."""
        lb = self._get(f"smj_{buffer_size}")
        lb.pimdal_ref_set_threads.argtypes = [C.c_int]
        lb.pimdal_ref_set_threads(threads)
        f = lb.pimdal_ref_smj
        f.restype = None
        f.argtypes = [_P, _U64, _P, _U64, _P, _P]
        ik, ok = _u32(inner_keys), _u32(outer_keys)
        assert ok.size <= buffer_size
        # the merge walks all BUFFER_SIZE/8000 blocks of 8000 rows (:83-101):
        # an outer size below BUFFER_SIZE needs that much slack in the buffers
        room = buffer_size + 1
        ires = np.zeros(room, np.uint32)
        ores = np.zeros(room, np.uint32)
        f(_p(ik), ik.size, _p(ok), ok.size, _p(ires), _p(ores))
        return ires[:ok.size], ores[:ok.size]
