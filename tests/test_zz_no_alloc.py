"""The allocation-free selection entry point (pimdal_sel_kernel_noalloc).

It exists for callers that cannot allocate device memory -- a host whose
memory manager (a buffer pool, a caching allocator) owns every device
allocation, or a latency-critical path where an allocation could block on a
device-wide synchronisation -- and so cannot create the context the regular
entry point needs.  Called here directly through the C ABI (ctypes), with
only caller-owned buffers, two calls in a row per case (the second reuses
the library's fixed scratch array as the first left it), and compared bit
for bit with the oracle and with the regular pimdal_sel_kernel.

Cases: both paths (the chunked one for 16-byte-aligned inputs of 2^20 rows
or more, the tile one otherwise), both layouts, signed and unsigned keys,
with and without a row-id column, a misaligned view of exactly 2^24 rows
(4096 tiles, the tile path's limit), a selection that keeps no row, a call
of 2^29 rows (4096 chunks, the chunked path's limit), and the rejection of
sizes beyond the scratch.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu


def call_noalloc(keys, pred, out, out_ptr, result, key_dtype=L.I32, layout=L.LAYOUT_COLUMNS,
                 in_ptr=None, ptr_base=0):
    a = L.SelArguments(size=keys.numel(), in_=keys.data_ptr(),
                       in_ptr=None if in_ptr is None else in_ptr.data_ptr(), ptr_base=ptr_base,
                       out=out.data_ptr(), out_ptr=None if out_ptr is None else out_ptr.data_ptr(),
                       pred=pred, key_dtype=key_dtype, layout=layout)
    return L.lib().pimdal_sel_kernel_noalloc(C.byref(a), result.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream)


def u32(t):
    return t.cpu().numpy().view(np.uint32)


def oracle_select(keys_u32, rows_u32, lo, hi, key_dtype):
    """(values, row ids) of lo <= key <= hi in input order; rows_u32 None means
    row id = index."""
    signed = key_dtype == L.I32
    k = keys_u32.view(np.int32) if signed else keys_u32
    v, r = oracle.select(k, lo, hi, is_signed=signed, in_ptr=rows_u32)
    return np.asarray(v).view(np.uint32), np.asarray(r)


def columns_case(ctx, n, key_dtype, with_rows, misalign=False, seed=77):
    """Seeded key column (and row-id column) of n rows; misalign views them
    4 bytes past a 16-byte boundary."""
    hi_gen = 2**31 - 1 if key_dtype == L.I32 else 2**32 - 1
    extra = 1 if misalign else 0
    buf = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, key_dtype, seed=seed, lo=0, hi=hi_gen),
                         n + extra)
    keys = buf[extra:]
    rows = None
    if with_rows:
        rbuf = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.U32, seed=seed, stream_id=5, lo=0,
                                            hi=2**32 - 1), n + extra)
        rows = rbuf[extra:]
    return keys, rows


def run_columns(ctx, keys, rows, key_dtype, lo, hi):
    n = keys.numel()
    pred = ops.make_pred(L.PRED_BETWEEN, lo, hi)
    ek, er = oracle_select(u32(keys), None if rows is None else u32(rows), lo, hi, key_dtype)
    rr, rk, rp = ops.sel_kernel(ctx, keys, pred, in_ptr=rows, key_dtype=key_dtype)
    ctx.sync()
    c = int(rr.item())
    assert c == ek.size
    assert np.array_equal(u32(rk[:c]), ek) and np.array_equal(u32(rp[:c]), er)
    for call in range(2):
        out = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        out_ptr = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        res = torch.full((1,), -5, dtype=torch.int64, device="cuda")
        assert call_noalloc(keys, pred, out, out_ptr, res, key_dtype=key_dtype, in_ptr=rows) == 0
        torch.cuda.synchronize()
        assert int(res.item()) == c, call
        assert np.array_equal(u32(out[:c]), ek), call
        assert np.array_equal(u32(out_ptr[:c]), er), call
        assert torch.equal(out[:c], rk[:c]) and torch.equal(out_ptr[:c], rp[:c]), call


@pytest.mark.parametrize("n,key_dtype,lo,hi,with_rows", [
    (1 << 22, L.I32, -2**31, 214748364 - 1, False),  # chunked path, config-1 predicate
    ((1 << 21) + 3, L.U32, 2**31, 2**31 + 2**29, True),  # chunked, ragged, unsigned, row ids
    (300007, L.U32, 10, 2**30, True),                  # tile path
    (300007, L.I32, 5, 4, False),                      # an empty interval: nothing kept
    ((1 << 20) + 5, L.I32, -2**31, -1, False),         # all keys >= 0: nothing kept (chunked)
])
def test_noalloc_columns_match_oracle_twice(ctx, n, key_dtype, lo, hi, with_rows):
    keys, rows = columns_case(ctx, n, key_dtype, with_rows)
    run_columns(ctx, keys, rows, key_dtype, lo, hi)


def test_noalloc_misaligned_view_at_its_tile_limit(ctx):
    # a misaligned view takes the tile path: 4096 rows per look-back word,
    # so 2^24 rows are exactly the 4096 words of the scratch
    keys, rows = columns_case(ctx, 1 << 24, L.I32, True, misalign=True, seed=78)
    assert keys.data_ptr() % 16 != 0
    run_columns(ctx, keys, rows, L.I32, -2**31, 214748364 - 1)


def test_noalloc_at_its_chunk_limit(ctx):
    # 2^29 aligned rows: 4096 chunks of 2^17 rows, the chunked path's limit
    keys, _ = columns_case(ctx, 1 << 29, L.I32, False, seed=79)
    run_columns(ctx, keys, None, L.I32, -2**31, (1 << 27) - 1)


@pytest.mark.parametrize("n,key_dtype", [((1 << 21) + 1, L.I32), (5000, L.U32)])
def test_noalloc_pairs_match_oracle_twice(ctx, n, key_dtype):
    hi_gen = 2**31 - 1 if key_dtype == L.I32 else 2**32 - 1
    k = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, key_dtype, seed=80, lo=0, hi=hi_gen), n)
    r = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.U32, seed=80, stream_id=1, lo=0,
                                     hi=2**32 - 1), n)
    pairs = torch.stack([k, r], dim=1).contiguous().view(torch.int64).view(-1)
    lo, hi = 1000, 2**30
    pred = ops.make_pred(L.PRED_BETWEEN, lo, hi)
    ek, er = oracle_select(u32(k), u32(r), lo, hi, key_dtype)
    for call in range(2):
        out = torch.full((n,), -7, dtype=torch.int64, device="cuda")
        res = torch.full((1,), -5, dtype=torch.int64, device="cuda")
        assert call_noalloc(pairs, pred, out, None, res, key_dtype=key_dtype,
                            layout=L.LAYOUT_PAIRS) == 0
        torch.cuda.synchronize()
        c = int(res.item())
        assert c == ek.size, call
        got = out[:c].cpu().numpy().view(np.uint32).reshape(-1, 2)
        assert np.array_equal(got[:, 0], ek) and np.array_equal(got[:, 1], er), call


def test_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    # a misaligned view uses one look-back word per 4096 rows: 2^24 rows max
    buf = torch.zeros((1 << 24) + 4096 + 1, dtype=torch.int32, device="cuda")
    keys = buf[1:]
    out = torch.empty(1, dtype=torch.int32, device="cuda")
    res = torch.empty(1, dtype=torch.int64, device="cuda")
    st = call_noalloc(keys, ops.make_pred(L.PRED_EQ, 0), out, out, res)
    assert st == 3  # PIMDAL_ERR_WORKSPACE, nothing launched
