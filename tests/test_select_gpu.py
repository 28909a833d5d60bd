"""GPU parity of the generator and of K-SEL (pimdal_sel_kernel) against the oracle."""
import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu

CFG_HI = 214748364 - 1  # predicate v < 214748364


def to_np(t: torch.Tensor, dtype=None) -> np.ndarray:
    a = t.cpu().numpy()
    return a.view(dtype) if dtype is not None else a


@pytest.mark.parametrize("spec", [
    gen.Spec(L.GEN_UNIFORM, L.I32, seed=1, lo=0, hi=2**31 - 1),
    gen.Spec(L.GEN_UNIFORM, L.U32, seed=1, stream_id=4, lo=0, hi=2**32 - 1),
    gen.Spec(L.GEN_UNIFORM, L.I64, seed=2, lo=100, hi=10**7),
    gen.Spec(L.GEN_PERM, L.I32, seed=3, perm_domain=1 << 20),
    gen.Spec(L.GEN_PERM, L.U32, seed=3, perm_domain=1000003),
    gen.Spec(L.GEN_PERM_UNIFORM, L.I32, seed=4, lo=0, hi=4095, perm_domain=0),
    gen.Spec(L.GEN_PERM_ZIPF, L.U32, seed=5, perm_domain=0, cdf=gen.zipf_cdf(1 << 16, 1.0)),
    gen.Spec(L.GEN_PROBE, L.I32, seed=6, lo=1 << 15, perm_domain=1 << 16, match_permille=500),
    gen.Spec(L.GEN_PROBE, L.I32, seed=6, lo=1 << 15, perm_domain=1 << 16, match_permille=500,
             cdf=gen.zipf_cdf(1 << 15, 0.75)),
], ids=lambda s: f"kind{s.kind}_dt{s.out_dtype}")
def test_generator_gpu_equals_cpu(ctx, spec):
    n = 300007
    d = ops.gen_column(ctx, spec, n, row_offset=12345)
    torch.cuda.synchronize()
    c = gen.generate_cpu(spec, n, row_offset=12345)
    assert np.array_equal(to_np(d).view(c.dtype), c)


def run_sel(ctx, keys_np, pred, key_dtype=L.I32, in_ptr=None, ptr_base=0, offset=0):
    t = torch.from_numpy(np.ascontiguousarray(keys_np).view(np.int32)).cuda()
    if offset:  # misaligned view (scalar-load path)
        buf = torch.empty(t.numel() + offset, dtype=torch.int32, device="cuda")
        buf[offset:] = t
        t = buf[offset:]
    ip = None if in_ptr is None else torch.from_numpy(in_ptr.view(np.int32)).cuda()
    res, out, out_ptr = ops.sel_kernel(ctx, t, pred, in_ptr=ip, ptr_base=ptr_base,
                                       key_dtype=key_dtype)
    ctx.sync()
    c = int(res.item())
    return c, to_np(out[:c], np.uint32), to_np(out_ptr[:c], np.uint32)


SIZES = [0, 1, 31, 4095, 4096, 4097, 7999, 8001, 100003, (1 << 20) + 17]


@pytest.mark.parametrize("n", SIZES)
def test_select_config_predicate(ctx, n):
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=0xB200, lo=0, hi=2**31 - 1), n)
    c, v, p = run_sel(ctx, keys, ops.make_pred(L.PRED_LT, 214748364))
    ov, op = oracle.select(keys, -2**63, CFG_HI)
    assert c == ov.size
    assert np.array_equal(v, ov.view(np.uint32))
    assert np.array_equal(p, op)


PREDS = [
    (L.PRED_BETWEEN, 10, 20, 10, 20, False),
    (L.PRED_RANGE, 10, 30, 10, 29, False),
    (L.PRED_NE, 25, 0, 25, 25, True),
    (L.PRED_GE, 40, 0, 40, 2**63 - 1, False),
    (L.PRED_LE, 1, 0, -2**63, 1, False),
    (L.PRED_EQ, 7, 0, 7, 7, False),
    (L.PRED_GT, 50, 0, 51, 2**63 - 1, False),  # selects nothing
]


@pytest.mark.parametrize("op,a,b,lo,hi,inv", PREDS)
@pytest.mark.parametrize("n", [8001, 262147])
def test_select_predicates_small_domain(ctx, op, a, b, lo, hi, inv, n):
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=3, lo=1, hi=50), n)
    c, v, p = run_sel(ctx, keys, ops.make_pred(op, a, b))
    ov, opp = oracle.select(keys, lo, hi, inv)
    assert c == ov.size and np.array_equal(v.view(np.int32), ov) and np.array_equal(p, opp)


def test_select_unsigned_and_row_id_column(ctx):
    n = 500009
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=8, lo=0, hi=2**32 - 1), n)
    rows = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=8, stream_id=1, lo=0,
                                     hi=2**32 - 1), n)
    c, v, p = run_sel(ctx, keys, ops.make_pred(L.PRED_GE, 3 * 2**30), key_dtype=L.U32,
                      in_ptr=rows)
    ov, opp = oracle.select(keys, 3 * 2**30, 2**63 - 1, is_signed=False, in_ptr=rows)
    assert c == ov.size and np.array_equal(v, ov) and np.array_equal(p, opp)


def test_select_ptr_base_and_misaligned_input(ctx):
    n = 123457
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=9, lo=-1000, hi=1000), n)
    c, v, p = run_sel(ctx, keys, ops.make_pred(L.PRED_BETWEEN, -10, 10), ptr_base=1 << 31,
                      offset=1)
    ov, opp = oracle.select(keys, -10, 10, ptr_base=1 << 31)
    assert c == ov.size and np.array_equal(v.view(np.int32), ov) and np.array_equal(p, opp)


def test_select_pairs_layout(ctx):
    n = 200003
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=10, lo=1, hi=50), n)
    pairs = np.empty((n, 2), np.uint32)
    pairs[:, 0] = keys.view(np.uint32)
    pairs[:, 1] = np.arange(n, dtype=np.uint32) * 3
    t = torch.from_numpy(pairs.reshape(-1).view(np.int64)).cuda()
    res, out, _ = ops.sel_kernel(ctx, t, ops.make_pred(L.PRED_BETWEEN, 10, 20),
                                 layout=L.LAYOUT_PAIRS)
    ctx.sync()
    c = int(res.item())
    got = to_np(out, np.uint32).reshape(-1, 2)[:c]
    ov, opp = oracle.select(keys, 10, 20, in_ptr=pairs[:, 1].copy())
    assert c == ov.size
    assert np.array_equal(got[:, 0].view(np.int32), ov) and np.array_equal(got[:, 1], opp)


def test_select_config1_full_size_and_determinism(ctx):
    n = 1 << 24
    spec = gen.Spec(L.GEN_UNIFORM, L.I32, seed=0xB200, lo=0, hi=2**31 - 1)
    keys_d = ops.gen_column(ctx, spec, n)
    keys = gen.generate_cpu(spec, n)
    pred = ops.make_pred(L.PRED_LT, 214748364)
    r1, o1, p1 = ops.sel_kernel(ctx, keys_d, pred)
    r2, o2, p2 = ops.sel_kernel(ctx, keys_d, pred)
    ctx.sync()
    c = int(r1.item())
    ov, op = oracle.select(keys, -2**63, CFG_HI)
    assert c == ov.size == int(r2.item())
    assert np.array_equal(to_np(o1[:c]), ov) and np.array_equal(to_np(p1[:c], np.uint32), op)
    assert torch.equal(o1[:c], o2[:c]) and torch.equal(p1[:c], p2[:c])


def test_select_epoch_wraparound(ctx):
    # > 65535 lookback launches: the status words are cleared when the 16-bit
    # epoch wraps, and results stay exact across the wrap.
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=12, lo=1, hi=50), 3 * 4096 + 5)
    t = torch.from_numpy(keys).cuda()
    pred = ops.make_pred(L.PRED_BETWEEN, 10, 20)
    expect, _ = oracle.select(keys, 10, 20)
    res = torch.empty(1, dtype=torch.int64, device="cuda")
    out = torch.empty_like(t)
    optr = torch.empty_like(t)
    for i in range(66000):
        ops.sel_kernel(ctx, t, pred, out=out, out_ptr=optr, result=res)
        if i % 16500 == 0 or i > 65530:
            ctx.sync()
            assert int(res.item()) == expect.size
    ctx.sync()
    assert np.array_equal(to_np(out[:expect.size]), expect)
