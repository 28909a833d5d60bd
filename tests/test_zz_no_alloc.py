"""The allocation-free selection entry point (pimdal_sel_kernel_noalloc).

It exists for callers that cannot allocate device memory -- a host whose
memory manager owns every device allocation, code running while a CUDA graph
is captured, latency-critical paths -- and so cannot create the context the
regular entry point needs.  Called here directly through the C ABI (ctypes),
with only caller-owned buffers, and compared bit for bit with the regular
pimdal_sel_kernel on two calls in a row (the second call reuses the
library's fixed scratch array left over from the first).  This file is named
to be collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu


def call_noalloc(keys, pred, out, out_ptr, result, key_dtype=L.I32):
    a = L.SelArguments(size=keys.numel(), in_=keys.data_ptr(), in_ptr=None, ptr_base=0,
                       out=out.data_ptr(), out_ptr=out_ptr.data_ptr(), pred=pred,
                       key_dtype=key_dtype, layout=L.LAYOUT_COLUMNS)
    return L.lib().pimdal_sel_kernel_noalloc(C.byref(a), result.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("n,lo,hi", [
    (1 << 22, 0, 214748364 - 1),      # chunked path (aligned input >= 2^20 rows)
    (300007, 10, 20),                 # tile path
])
def test_noalloc_matches_regular_entry_point_twice(ctx, n, lo, hi):
    hi_gen = 2**31 - 1 if lo == 0 else 50
    keys = ops.gen_column(ctx, gen.Spec(L.GEN_UNIFORM, L.I32, seed=77, lo=0, hi=hi_gen), n)
    pred = ops.make_pred(L.PRED_BETWEEN, lo, hi)
    ref_res, ref_out, ref_ptr = ops.sel_kernel(ctx, keys, pred)
    ctx.sync()
    c = int(ref_res.item())
    for _ in range(2):
        out = torch.full_like(keys, -7)
        out_ptr = torch.full_like(keys, -7)
        res = torch.full((1,), -5, dtype=torch.int64, device="cuda")
        assert call_noalloc(keys, pred, out, out_ptr, res) == 0
        torch.cuda.synchronize()
        assert int(res.item()) == c
        assert torch.equal(out[:c], ref_out[:c])
        assert torch.equal(out_ptr[:c], ref_ptr[:c])


def test_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    # a misaligned view uses one look-back word per 4096 rows: 2^24 rows max
    buf = torch.zeros((1 << 24) + 4096 + 1, dtype=torch.int32, device="cuda")
    keys = buf[1:]
    out = torch.empty(1, dtype=torch.int32, device="cuda")
    res = torch.empty(1, dtype=torch.int64, device="cuda")
    st = call_noalloc(keys, ops.make_pred(L.PRED_EQ, 0), out, out, res)
    assert st == 3  # PIMDAL_ERR_WORKSPACE, nothing launched
