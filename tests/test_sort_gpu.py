"""GPU parity of K-SORT (pimdal_sort_kernel) against the oracle: stable
ascending (key, row id) order, bit-exact."""
import numpy as np
import pytest
import torch

import oracle
from pimdal_b200 import _lib as L
from pimdal_b200 import gen, ops

pytestmark = pytest.mark.gpu


def cuda_i32(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def host_u32(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


def check_sort(ctx, keys, ptr=None, key_dtype=L.U32, **kw):
    out, out_ptr = ops.sort_kernel(ctx, cuda_i32(keys), None if ptr is None else cuda_i32(ptr),
                                   key_dtype=key_dtype, **kw)
    ctx.sync()
    ok, op = oracle.sort_pairs(keys, ptr, is_signed=(key_dtype == L.I32))
    assert np.array_equal(host_u32(out), ok)
    assert np.array_equal(host_u32(out_ptr), op)


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 100003, (1 << 20) + 5])
def test_sort_uniform_u32(ctx, n):
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=21, lo=0, hi=2**32 - 1), n)
    check_sort(ctx, keys)


@pytest.mark.parametrize("n", [1000, 65537, 1 << 20])
def test_sort_signed_and_row_ids(ctx, n):
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.I32, seed=22, lo=-2**31, hi=2**31 - 1), n)
    rows = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=22, stream_id=1, lo=0,
                                     hi=2**32 - 1), n)
    check_sort(ctx, keys, rows, key_dtype=L.I32)


@pytest.mark.parametrize("hi", [0, 1, 15, 255, 65535, (1 << 24) - 1])
def test_sort_duplicates_and_skipped_passes(ctx, hi):
    # small key ranges leave whole digits constant: those passes are skipped
    n = 300007
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=23, lo=0, hi=hi), n)
    check_sort(ctx, keys)


def test_sort_zipf_keys(ctx):
    n = 1 << 21
    cdf = gen.zipf_cdf(1 << 20, 1.0)
    keys = gen.generate_cpu(gen.Spec(L.GEN_PERM_ZIPF, L.U32, seed=24, perm_domain=0, cdf=cdf), n)
    check_sort(ctx, keys)


def test_sort_all_bits_set_and_extremes(ctx):
    n = 50001
    keys = np.full(n, 0xFFFFFFFF, np.uint32)
    keys[::7] = 0
    keys[::11] = 0x80000000
    check_sort(ctx, keys)
    check_sort(ctx, keys, key_dtype=L.I32)


def test_sort_pairs_layout(ctx):
    n = 200003
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=25, lo=0, hi=2**32 - 1), n)
    rows = np.arange(n, dtype=np.uint32) * 3 + 1
    pairs = np.stack([keys, rows], axis=1).reshape(-1)
    t = torch.from_numpy(pairs.view(np.int64)).cuda()
    out, _ = ops.sort_kernel(ctx, t, layout=L.LAYOUT_PAIRS)
    ctx.sync()
    got = out.cpu().numpy().view(np.uint32).reshape(-1, 2)
    ok, op = oracle.sort_pairs(keys, rows)
    assert np.array_equal(got[:, 0], ok) and np.array_equal(got[:, 1], op)


def test_sort_keys_only_and_bit_range(ctx):
    n = 123457
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=26, lo=0, hi=2**32 - 1), n)
    out, _ = ops.sort_kernel(ctx, cuda_i32(keys), want_ptr=False)
    ctx.sync()
    assert np.array_equal(host_u32(out), np.sort(keys))
    # sort on bits [8, 24) only: stable order by the middle 16 bits
    out, out_ptr = ops.sort_kernel(ctx, cuda_i32(keys), begin_bit=8, end_bit=24)
    ctx.sync()
    mid = (keys >> 8) & 0xFFFF
    order = np.argsort(mid, kind="stable")
    assert np.array_equal(host_u32(out_ptr), order.astype(np.uint32))


def test_sort_config2_full_size_uniform_and_zipf(ctx):
    n = 1 << 26
    for spec in (gen.Spec(L.GEN_UNIFORM, L.U32, seed=0xB200, lo=0, hi=2**32 - 1),
                 gen.Spec(L.GEN_PERM_ZIPF, L.U32, seed=0xB200, stream_id=1, perm_domain=0,
                          cdf=gen.zipf_cdf(1 << 24, 1.0))):
        keys_d = ops.gen_column(ctx, spec, n)
        out, out_ptr = ops.sort_kernel(ctx, keys_d)
        out2, out_ptr2 = ops.sort_kernel(ctx, keys_d)
        ctx.sync()
        # size-independent properties: sorted, a permutation, stable, deterministic
        k = out.cpu().numpy().view(np.uint32)
        r = out_ptr.cpu().numpy().view(np.uint32)
        src = keys_d.cpu().numpy().view(np.uint32)
        assert np.all(k[1:] >= k[:-1])
        assert np.array_equal(src[r], k)
        same = k[1:] == k[:-1]
        assert np.all(r[1:][same] > r[:-1][same])
        assert np.array_equal(np.bincount(r, minlength=n), np.ones(n, np.int64))
        assert torch.equal(out, out2) and torch.equal(out_ptr, out_ptr2)


@pytest.mark.parametrize("bits", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("n", [1, 5119, 5120, 5121, 300007])
def test_single_small_digit_is_a_stable_partition(ctx, bits, n):
    """A sort on one digit of <= 6 bits (the small-radix partition pass):
    the stable order of the digit, rows carried, for signed and unsigned
    keys, keys alone and with row ids, over ragged tile tails."""
    keys = gen.generate_cpu(gen.Spec(L.GEN_UNIFORM, L.U32, seed=60 + bits, lo=0, hi=2**32 - 1), n)
    lo = 32 - bits if bits % 2 else 11
    for dtype in (L.U32, L.I32):
        flip = np.uint32(0x80000000) if dtype == L.I32 else np.uint32(0)
        digit = ((keys ^ flip) >> np.uint32(lo)) & np.uint32((1 << bits) - 1)
        order = np.argsort(digit, kind="stable")
        out, out_ptr = ops.sort_kernel(ctx, cuda_i32(keys), key_dtype=dtype, begin_bit=lo,
                                       end_bit=lo + bits)
        ko, _ = ops.sort_kernel(ctx, cuda_i32(keys), key_dtype=dtype, begin_bit=lo,
                                end_bit=lo + bits, want_ptr=False)
        ctx.sync()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), keys[order])
        assert np.array_equal(out_ptr.cpu().numpy().view(np.uint32), order.astype(np.uint32))
        assert np.array_equal(ko.cpu().numpy().view(np.uint32), keys[order])
