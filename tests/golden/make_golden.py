"""Generates the golden fixtures in tests/golden/*.npz from the reference itself.

Inputs come from the seeded generator (pimdal_b200.gen, CPU side); outputs
come from the reference's own CPU operators (reference/db_operators, compiled
where they lie into oracle/_ref/ by `make -C oracle ref`).  The fixtures pin
the oracle (tests/test_oracle.py) on machines without the reference checkout.

    make -C oracle ref && python tests/golden/make_golden.py [fixture ...]

With names (select sort hash_join group_by smj bloom dates), only those fixtures
are rewritten.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from pimdal_b200 import _lib as L  # noqa: E402
from pimdal_b200 import gen  # noqa: E402

OUT = Path(__file__).resolve().parent
SEED = 0xB200


def uni(n, lo, hi, stream, dt=L.I32, seed=SEED):
    return gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, dt, seed=seed, stream_id=stream, lo=lo, hi=hi), n)


def bloom(ref) -> None:
    """Hash values of hash0..hash4 and per-partition Bloom filters / matches
    from the reference's hash functions (pimdal/hash/hash_func.h)."""
    b = {}
    hk = uni(4096, 0, 2**32 - 1, 100, L.U32)
    hk[:4] = [0, 1, 0xFFFFFFFF, 272333]
    b["h_keys"] = hk
    for w in range(5):
        b[f"h{w}"] = ref.hash_fn(w, hk)
    # build side: 8 partitions, two of them empty; probe side: half of each
    # partition's rows drawn from that partition's build keys
    bps = np.array([0, 0, 700, 700, 3000, 3001, 6000, 9000, 9000], np.uint64)
    pps = np.array([0, 10, 2000, 2000, 7000, 7001, 12000, 20000, 20000], np.uint64)
    bk = uni(int(bps[-1]), 0, 2**32 - 1, 101, L.U32)
    pk = uni(int(pps[-1]), 0, 2**32 - 1, 102, L.U32)
    pick = uni(int(pps[-1]), 0, 2**31 - 1, 103, L.U32)
    for p in range(8):
        lo, hi, blo, bhi = int(pps[p]), int(pps[p + 1]), int(bps[p]), int(bps[p + 1])
        if bhi > blo:
            rows = np.arange(lo, hi)[::2]
            pk[rows] = bk[blo + pick[rows] % (bhi - blo)]
    filt = ref.bloom_build(bk, bps)
    mk, mp, ms = ref.bloom_match(filt, pk, pps)
    b.update(bk=bk, bps=bps, pk=pk, pps=pps, filters=filt, match_key=mk, match_ptr=mp,
             match_sizes=ms)
    np.savez_compressed(OUT / "bloom.npz", **b)


def dates(ref) -> None:
    """Packed dates from the reference reader's date_to_int
    (pimdal/main/tpc_h/reader/read_table.cpp:8-16) over 1992-1998 and edges."""
    days = uni(5000, 0, 2556, 110)
    d = (np.datetime64("1992-01-01") + days.astype("timedelta64[D]")).astype(str).tolist()
    d += ["1970-01-01", "1900-01-01", "1999-12-31", "2000-02-29", "2024-02-29", "2099-12-31"]
    np.savez_compressed(OUT / "dates.npz", dates=np.array(d), packed=ref.date_to_int(d))


def main(only: list[str]) -> None:
    want = lambda name: not only or name in only
    ref = oracle.Ref()
    if want("bloom"):
        bloom(ref)
    if want("dates"):
        dates(ref)
    if only and set(only) <= {"bloom", "dates"}:
        print("golden fixtures written to", OUT)
        return
    for name in ("select", "sort", "hash_join", "aggregate", "smj_64000"):
        ref.set_threads(name, 1)

    # Selection: the config predicate (v < 214748364) on U[0, 2^31) and the
    # reference's own workload (10 <= v < 30 on U[1, 50], select.cpp:19,34-35)
    # at sizes around the reference's 8000-row block.
    sel = {}
    for i, n in enumerate([0, 1, 31, 7999, 8000, 8001, 100003]):
        k1 = uni(n, 0, 2**31 - 1, 10 + i)
        sel[f"cfg_keys_{n}"] = k1
        sel[f"cfg_out_{n}"] = ref.select(k1, -2**63, 214748364 - 1)
        k2 = uni(n, 1, 50, 20 + i)
        sel[f"own_keys_{n}"] = k2
        sel[f"own_out_{n}"] = ref.select(k2, 10, 29)
    np.savez_compressed(OUT / "select.npz", **sel)

    # Stable key/row-id sort: uniform 32-bit keys and heavy duplicates.
    srt = {}
    for i, n in enumerate([0, 1, 2, 1000, 65537]):
        ku = uni(n, 0, 2**32 - 1, 30 + i, L.U32)
        kd = uni(n, 0, 15, 40 + i, L.U32)
        ks = uni(n, -2**31, 2**31 - 1, 50 + i, L.I32)
        srt[f"u_keys_{n}"] = ku
        srt[f"u_out_{n}"] = np.stack(ref.sort_pairs(ku))
        srt[f"d_keys_{n}"] = kd
        srt[f"d_out_{n}"] = np.stack(ref.sort_pairs(kd))
        srt[f"s_keys_{n}"] = ks
        srt[f"s_out_{n}"] = np.stack(ref.sort_pairs(ks, is_signed=True))
    np.savez_compressed(OUT / "sort.npz", **srt)

    # Hash join: unique build keys (a seeded sample of [0, 2 nb)), probes at
    # 50% match rate; output in the reference's own order.
    hj = {}
    for i, (nb, npr) in enumerate([(1, 7), (100, 1000), (5000, 40000)]):
        bk = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.I32, seed=SEED + i, perm_domain=2 * nb), nb)
        bp = uni(nb, -2**31, 2**31 - 1, 60 + i)
        pk = gen.generate_cpu(gen.Spec(L.GEN_PROBE, L.I32, seed=SEED + i, stream_id=70 + i, lo=nb,
                                       perm_domain=2 * nb, match_permille=500), npr)
        pay, row = ref.hash_join(bk, bp, pk)
        hj.update({f"bk_{i}": bk, "bp_%d" % i: bp, f"pk_{i}": pk, f"pay_{i}": pay, f"row_{i}": row})
    np.savez_compressed(OUT / "hash_join.npz", **hj)

    # Group-by: cardinalities 1, 16, 4096 with keys that include negatives
    # and -1 (the reference's empty-slot sentinel as int32).
    gb = {}
    for i, (n, c) in enumerate([(1, 1), (1000, 16), (50000, 4096)]):
        k = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=SEED + i, stream_id=80 + i,
                                      lo=0, hi=c - 1, perm_domain=0), n)
        if n > 10:
            k[::97] = -1
        v = uni(n, 100, 10**7, 90 + i, L.I64)
        out = ref.group_by(k, v)
        gb[f"k_{i}"] = k
        gb[f"v_{i}"] = v
        for name, arr in zip(("key", "sum", "count", "min", "max"), out):
            gb[f"{name}_{i}"] = arr
    np.savez_compressed(OUT / "group_by.npz", **gb)

    # Sort-merge join on the reference's own workload shape (inner = shuffled
    # 1..N, outer drawn from the inner keys), N = 64000.
    n = 64000
    rk = gen.generate_cpu(gen.Spec(L.GEN_PERM, L.U32, seed=SEED, perm_domain=n), n) + np.uint32(1)
    sk = gen.generate_cpu(gen.Spec(L.GEN_PERM_UNIFORM, L.U32, seed=SEED, stream_id=99, lo=0,
                                   hi=n - 1, perm_domain=n), n) + np.uint32(1)
    ires, ores = ref.smj(rk, sk, 64000)
    np.savez_compressed(OUT / "smj.npz", rk=rk, sk=sk, inner_res=ires, outer_res=ores)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main(sys.argv[1:])
