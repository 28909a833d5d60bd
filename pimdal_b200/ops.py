"""Python host layer over the C ABI (include/pimdal_gpu.h).

Operator names and argument meaning follow the reference's DPU library
(pimdal/select/sel.h, pimdal/sort/sort.h, pimdal/join/*.h,
pimdal/aggregate/aggregate.h).  Columns are torch CUDA tensors resident in
HBM; torch is used only for device memory and streams.  Every call goes
through libpimdal_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .gen import Spec

_TORCH_DT = {L.U32: torch.int32, L.I32: torch.int32, L.I64: torch.int64}


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(stream) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


class Context:
    """A pimdal_ctx_t plus a torch-allocated workspace it grows on demand."""

    def __init__(self, device: int = 0):
        self.device = device
        self.lib = L.lib()
        h = C.c_void_p()
        L.check(self.lib.pimdal_ctx_create(C.byref(h), device), "pimdal_ctx_create")
        self.handle = h
        self._ws: torch.Tensor | None = None

    def close(self) -> None:
        if self.handle:
            torch.cuda.synchronize(self.device)
            self.lib.pimdal_ctx_destroy(self.handle)
            self.handle = None
            self._ws = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, nbytes: int) -> None:
        """Makes sure the caller-owned workspace holds at least nbytes."""
        if nbytes <= 0:
            return
        if self._ws is None or self._ws.numel() < nbytes:
            size = max(nbytes, 1 << 20)
            self._ws = torch.empty(size, dtype=torch.uint8, device=f"cuda:{self.device}")
            L.check(self.lib.pimdal_ctx_set_workspace(self.handle, self._ws.data_ptr(), size),
                    "pimdal_ctx_set_workspace")

    def workspace_bytes(self) -> int:
        """Bytes of the workspace this context holds."""
        return 0 if self._ws is None else self._ws.numel()

    def sync(self, stream=None) -> None:
        """Waits for the stream and raises if a kernel reported a device error."""
        L.check(self.lib.pimdal_ctx_sync_status(self.handle, _stream(stream)),
                "pimdal_ctx_sync_status")

    def set_profiling(self, enable: bool) -> None:
        L.check(self.lib.pimdal_ctx_set_profiling(self.handle, int(enable)),
                "pimdal_ctx_set_profiling")

    def kernel_time(self, kernel_id: int) -> tuple[int, float]:
        """(launches, summed milliseconds) of one kernel since the last read."""
        n = C.c_uint64()
        ms = C.c_double()
        L.check(self.lib.pimdal_ctx_kernel_time(self.handle, kernel_id, C.byref(n), C.byref(ms)),
                "pimdal_ctx_kernel_time")
        return int(n.value), float(ms.value)

    @property
    def launches(self) -> int:
        return int(self.lib.pimdal_ctx_launch_count(self.handle))


# ---------------------------------------------------------------------------
# Generator
# ---------------------------------------------------------------------------
def gen_column(ctx: Context, spec: Spec, n: int, row_offset: int = 0, out=None, stream=None):
    """Device twin of gen.generate_cpu: returns a CUDA tensor of n values."""
    dev = f"cuda:{ctx.device}"
    if out is None:
        out = torch.empty(n, dtype=_TORCH_DT[spec.out_dtype], device=dev)
    cdf_t = None
    if spec.cdf is not None:
        cdf_t = torch.from_numpy(np.ascontiguousarray(spec.cdf, dtype=np.float64)).to(dev)
    s = L.GenSpec(kind=spec.kind, out_dtype=spec.out_dtype, seed=spec.seed,
                  stream_id=spec.stream_id, lo=spec.lo, hi=spec.hi,
                  perm_domain=spec.perm_domain,
                  cdf=_ptr(cdf_t), cdf_n=0 if cdf_t is None else cdf_t.numel(),
                  match_permille=spec.match_permille)
    L.check(ctx.lib.pimdal_gen_column(ctx.handle, C.byref(s), _ptr(out), n, row_offset,
                                      _stream(stream)), "pimdal_gen_column")
    if cdf_t is not None:
        torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
    return out


# ---------------------------------------------------------------------------
# Selection (sel_kernel, pimdal/select/sel.h:21)
# ---------------------------------------------------------------------------
def make_pred(op: int, lo: int = 0, hi: int = 0) -> L.Pred:
    return L.Pred(op=op, pad=0, lo=lo, hi=hi)


def sel_kernel(ctx: Context, keys: torch.Tensor, pred: L.Pred, *, in_ptr=None, ptr_base: int = 0,
               key_dtype: int = L.I32, out=None, out_ptr=None, want_ptr: bool = True,
               layout: int = L.LAYOUT_COLUMNS, result=None, stream=None):
    """Stable selection.  keys: int32 column (or int64 view of key_ptr32 pairs
    for layout=PAIRS).  Returns (result uint64[1] device tensor, out, out_ptr)."""
    n = keys.numel()
    dev = keys.device
    if out is None:
        out = torch.empty_like(keys)
    if layout == L.LAYOUT_COLUMNS and want_ptr and out_ptr is None:
        out_ptr = torch.empty(n, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.SelArguments(size=n, in_=_ptr(keys), in_ptr=_ptr(in_ptr), ptr_base=ptr_base,
                       out=_ptr(out), out_ptr=_ptr(out_ptr), pred=pred, key_dtype=key_dtype,
                       layout=layout)
    L.check(ctx.lib.pimdal_sel_kernel(ctx.handle, C.byref(a), _ptr(result), _stream(stream)),
            "pimdal_sel_kernel")
    return result, out, out_ptr


# ---------------------------------------------------------------------------
# Sort (sort_kernel, pimdal/sort/sort.h:25)
# ---------------------------------------------------------------------------
def _workspace(ctx: Context, fn, args) -> None:
    sz = C.c_size_t()
    L.check(fn(C.byref(args), C.byref(sz)), fn.__name__)
    ctx.reserve(sz.value)


def sort_kernel(ctx: Context, keys: torch.Tensor, ptr: torch.Tensor | None = None, *,
                ptr_base: int = 0, key_dtype: int = L.U32, layout: int = L.LAYOUT_COLUMNS,
                out=None, out_ptr=None, want_ptr: bool = True, begin_bit: int = 0,
                end_bit: int = 32, stream=None):
    """Stable ascending sort of (key, row id).  keys: int32 tensor (or int64
    view of key_ptr32 pairs with layout=PAIRS).  Returns (out, out_ptr)."""
    n = keys.numel()
    if out is None:
        out = torch.empty_like(keys)
    if layout == L.LAYOUT_COLUMNS and want_ptr and out_ptr is None:
        out_ptr = torch.empty(n, dtype=torch.int32, device=keys.device)
    a = L.SortArguments(nr_elements=n, in_=_ptr(keys), in_ptr=_ptr(ptr), ptr_base=ptr_base,
                        out=_ptr(out), out_ptr=_ptr(out_ptr), key_dtype=key_dtype, layout=layout,
                        begin_bit=begin_bit, end_bit=end_bit)
    _workspace(ctx, ctx.lib.pimdal_sort_workspace_size, a)
    L.check(ctx.lib.pimdal_sort_kernel(ctx.handle, C.byref(a), _stream(stream)),
            "pimdal_sort_kernel")
    return out, out_ptr


# ---------------------------------------------------------------------------
# Sort-merge join (merge_kernel, pimdal/join/sort_merge.h:23)
# ---------------------------------------------------------------------------
def smj_merge(ctx: Context, inner, inner_ptr, outer, outer_ptr, *, key_dtype: int = L.I32,
              capacity: int | None = None, out_outer=None, out_inner=None, result=None,
              stream=None):
    """Merge of key-sorted relations.  Returns (result, out_outer, out_inner)."""
    dev = outer.device
    if capacity is None:
        capacity = max(outer.numel(), 1)
    if out_outer is None:
        out_outer = torch.empty(capacity, dtype=torch.int32, device=dev)
    if out_inner is None:
        out_inner = torch.empty(capacity, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.SmjMergeArguments(inner=_ptr(inner), inner_ptr=_ptr(inner_ptr), size_inner=inner.numel(),
                            outer=_ptr(outer), outer_ptr=_ptr(outer_ptr), size_outer=outer.numel(),
                            out_outer=_ptr(out_outer), out_inner=_ptr(out_inner),
                            out_capacity=capacity, key_dtype=key_dtype)
    _workspace(ctx, ctx.lib.pimdal_smj_merge_workspace_size, a)
    L.check(ctx.lib.pimdal_smj_merge(ctx.handle, C.byref(a), _ptr(result), _stream(stream)),
            "pimdal_smj_merge")
    return result, out_outer, out_inner


def sort_merge_join(ctx: Context, inner_key, inner_payload, outer_key, outer_payload, *,
                    key_dtype: int = L.I32, capacity: int | None = None, out_inner=None,
                    out_outer=None, result=None, stream=None):
    """Sorts both relations and merges them.  Returns (result, inner payloads,
    outer payloads) of the matches, outer-major."""
    dev = outer_key.device
    if capacity is None:
        capacity = max(outer_key.numel(), 1)
    if out_inner is None:
        out_inner = torch.empty(capacity, dtype=torch.int32, device=dev)
    if out_outer is None:
        out_outer = torch.empty(capacity, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.SmjArguments(inner_key=_ptr(inner_key), inner_payload=_ptr(inner_payload),
                       size_inner=inner_key.numel(), outer_key=_ptr(outer_key),
                       outer_payload=_ptr(outer_payload), size_outer=outer_key.numel(),
                       out_inner_payload=_ptr(out_inner), out_outer_payload=_ptr(out_outer),
                       out_capacity=capacity, key_dtype=key_dtype)
    _workspace(ctx, ctx.lib.pimdal_sort_merge_join_workspace_size, a)
    L.check(ctx.lib.pimdal_sort_merge_join(ctx.handle, C.byref(a), _ptr(result), _stream(stream)),
            "pimdal_sort_merge_join")
    return result, out_inner, out_outer


# ---------------------------------------------------------------------------
# Radix partition (part_kernel, pimdal/join/hash_join.h:72)
# ---------------------------------------------------------------------------
def part_kernel(ctx: Context, keys, ptr=None, *, shift: int = 32, part_n: int = 32,
                out=None, out_ptr=None, want_ptr: bool = True, stream=None):
    """Stable partition by bits [shift - log2(part_n), shift) of hash0(key).
    Returns (out keys, out row ids, part_sizes uint64[part_n + 1])."""
    n = keys.numel()
    dev = keys.device
    if out is None:
        out = torch.empty_like(keys)
    if want_ptr and out_ptr is None:
        out_ptr = torch.empty(n, dtype=torch.int32, device=dev)
    sizes = torch.empty(part_n + 1, dtype=torch.int64, device=dev)
    a = L.PartArguments(in_=_ptr(keys), in_ptr=_ptr(ptr), size=n, shift=shift, part_n=part_n,
                        part_out=_ptr(out), part_out_ptr=_ptr(out_ptr), part_sizes=_ptr(sizes),
                        layout=L.LAYOUT_COLUMNS)
    _workspace(ctx, ctx.lib.pimdal_part_workspace_size, a)
    L.check(ctx.lib.pimdal_part_kernel(ctx.handle, C.byref(a), _stream(stream)), "pimdal_part_kernel")
    return out, out_ptr, sizes


# ---------------------------------------------------------------------------
# Hash tables (hash_kernel / merge_kernel, pimdal/join/hash_join.h:62,82)
# ---------------------------------------------------------------------------
def hash_kernel(ctx: Context, keys, ptr=None, *, table_size: int, table=None, stream=None):
    """Builds a linear-probing table; returns the table (uint8 device tensor)."""
    if table is None:
        nbytes = int(ctx.lib.pimdal_hash_table_bytes(table_size))
        table = torch.empty(nbytes, dtype=torch.uint8, device=keys.device)
    a = L.HashArguments(in_key=_ptr(keys), in_ptr=_ptr(ptr), size=keys.numel(),
                        table_ptr=_ptr(table), table_size=table_size)
    L.check(ctx.lib.pimdal_hash_kernel(ctx.handle, C.byref(a), _stream(stream)), "pimdal_hash_kernel")
    return table


def hj_probe(ctx: Context, table, table_size: int, keys, ptr=None, *, capacity: int | None = None,
             out_outer=None, out_inner=None, result=None, stream=None):
    """Probes a table; returns (result, probe ptr per match, build payload per match)."""
    dev = keys.device
    if capacity is None:
        capacity = max(keys.numel(), 1)
    if out_outer is None:
        out_outer = torch.empty(capacity, dtype=torch.int32, device=dev)
    if out_inner is None:
        out_inner = torch.empty(capacity, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.ProbeArguments(table_ptr=_ptr(table), table_size=table_size, in_key=_ptr(keys),
                         in_ptr=_ptr(ptr), size=keys.numel(), out_outer=_ptr(out_outer),
                         out_inner=_ptr(out_inner), out_capacity=capacity)
    L.check(ctx.lib.pimdal_hj_probe(ctx.handle, C.byref(a), _ptr(result), _stream(stream)),
            "pimdal_hj_probe")
    return result, out_outer, out_inner


def select_join_aggregate(ctx: Context, date, lo: int, hi: int, jkey, table, table_size: int,
                          price, discount, *, flag=None, attr_mult: int = 1, key_space: int,
                          outs=None, result=None, stream=None):
    """One query's date filter -> join -> SUM(price*(100-discount)), COUNT
    group-by in one pass.  Returns (result, outs) with outs key/sum/count
    columns holding the groups in key order (result[0] of them)."""
    dev = date.device
    if outs is None:
        outs = {"key": torch.empty(key_space, dtype=torch.int32, device=dev),
                "sum": torch.empty(key_space, dtype=torch.int64, device=dev),
                "count": torch.empty(key_space, dtype=torch.int64, device=dev)}
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.SelectJoinAggregateArguments(
        size=date.numel(), date=_ptr(date), date_lo=lo, date_hi=hi, jkey=_ptr(jkey),
        table_ptr=_ptr(table), table_size=table_size, flag=_ptr(flag), price=_ptr(price),
        discount=_ptr(discount), attr_mult=attr_mult, key_space=key_space, out_key=_ptr(outs["key"]),
        out_sum=_ptr(outs["sum"]), out_count=_ptr(outs["count"]), out_capacity=outs["key"].numel())
    L.check(ctx.lib.pimdal_select_join_aggregate(ctx.handle, C.byref(a), _ptr(result),
                                                 _stream(stream)), "pimdal_select_join_aggregate")
    return result, outs


# ---------------------------------------------------------------------------
# Bloom-filter prefilter (filter_kernel / match_kernel, pimdal/join/hash_join.h:66,76)
# ---------------------------------------------------------------------------
def filter_kernel(ctx: Context, keys, part_sizes, *, filters=None, pairs: bool = False,
                  stream=None):
    """One PIMDAL_FILTER_BYTES Bloom filter per partition of partitioned keys
    (part_sizes: int64 device tensor of part_n + 1 row offsets).  keys is a
    uint32/int32 column, or an (n, 2) key_ptr32 pair tensor with pairs=True.
    Returns the filters (uint8 device tensor)."""
    part_n = part_sizes.numel() - 1
    if filters is None:
        filters = torch.empty(part_n * L.FILTER_BYTES, dtype=torch.uint8, device=keys.device)
    a = L.FilterArguments(in_=_ptr(keys), filter_ptr=_ptr(filters), part_sizes=_ptr(part_sizes),
                          part_n=part_n, layout=L.LAYOUT_PAIRS if pairs else L.LAYOUT_COLUMNS)
    L.check(ctx.lib.pimdal_filter_kernel(ctx.handle, C.byref(a), _stream(stream)),
            "pimdal_filter_kernel")
    return filters


def match_kernel(ctx: Context, filters, keys, part_sizes, ptr=None, *, pairs: bool = False,
                 capacity: int | None = None, out=None, out_row=None, want_row: bool = True,
                 result=None, stream=None):
    """Keeps the rows whose key hits its partition's filter, in input order.
    Returns (result, kept keys or pairs, kept row ids or None, match_sizes)."""
    dev = keys.device
    n = keys.shape[0]
    part_n = part_sizes.numel() - 1
    if capacity is None:
        capacity = max(n, 1)
    if out is None:
        out = torch.empty((capacity, 2) if pairs else capacity, dtype=torch.int32, device=dev)
    if not pairs and want_row and out_row is None:
        out_row = torch.empty(capacity, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    sizes = torch.empty(part_n + 1, dtype=torch.int64, device=dev)
    a = L.MatchArguments(filter_ptr=_ptr(filters), size=n, part_ptr=_ptr(keys), part_row=_ptr(ptr),
                         out_ptr=_ptr(out), out_row=_ptr(out_row), out_capacity=capacity,
                         match_sizes=_ptr(sizes), part_sizes=_ptr(part_sizes), part_n=part_n,
                         layout=L.LAYOUT_PAIRS if pairs else L.LAYOUT_COLUMNS)
    L.check(ctx.lib.pimdal_match_kernel(ctx.handle, C.byref(a), _ptr(result), _stream(stream)),
            "pimdal_match_kernel")
    return result, out, (None if pairs else out_row), sizes


def hash_join(ctx: Context, build_key, build_payload, probe_key, probe_ptr=None, *,
              capacity: int | None = None, partition_bits: int = 0, load_factor_pct: int = 0,
              l2_budget_bytes: int = 0, out_payload=None, out_row=None, result=None, stream=None):
    """Hash join; returns (result, build payload per match, probe row id per match)."""
    dev = probe_key.device
    if capacity is None:
        capacity = max(probe_key.numel(), 1)
    if out_payload is None:
        out_payload = torch.empty(capacity, dtype=torch.int32, device=dev)
    if out_row is None:
        out_row = torch.empty(capacity, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.HashJoinArguments(build_key=_ptr(build_key), build_payload=_ptr(build_payload),
                            size_build=build_key.numel(), probe_key=_ptr(probe_key),
                            probe_ptr=_ptr(probe_ptr), size_probe=probe_key.numel(),
                            out_build_payload=_ptr(out_payload), out_probe_ptr=_ptr(out_row),
                            out_capacity=capacity, partition_bits=partition_bits,
                            load_factor_pct=load_factor_pct, l2_budget_bytes=l2_budget_bytes)
    _workspace(ctx, ctx.lib.pimdal_hash_join_workspace_size, a)
    L.check(ctx.lib.pimdal_hash_join(ctx.handle, C.byref(a), _ptr(result), _stream(stream)),
            "pimdal_hash_join")
    return result, out_payload, out_row


def hash_join_autotune(ctx: Context, build_key, build_payload, probe_key, probe_ptr=None, *,
                       capacity: int | None = None, l2_budget_bytes: int = 0, out_payload=None,
                       out_row=None, result=None, stream=None):
    """pimdal_hash_join_autotune: times the candidate partition fan-outs and
    load factors on these inputs (writing the outputs) and caches the fastest
    for this shape; later hash_join calls of the shape with partition_bits=0
    and load_factor_pct=0 use it.  Returns (tuning dict, cached, result,
    out_payload, out_row)."""
    dev = probe_key.device
    if capacity is None:
        capacity = max(probe_key.numel(), 1)
    if out_payload is None:
        out_payload = torch.empty(capacity, dtype=torch.int32, device=dev)
    if out_row is None:
        out_row = torch.empty(capacity, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.HashJoinArguments(build_key=_ptr(build_key), build_payload=_ptr(build_payload),
                            size_build=build_key.numel(), probe_key=_ptr(probe_key),
                            probe_ptr=_ptr(probe_ptr), size_probe=probe_key.numel(),
                            out_build_payload=_ptr(out_payload), out_probe_ptr=_ptr(out_row),
                            out_capacity=capacity, partition_bits=0, load_factor_pct=0,
                            l2_budget_bytes=l2_budget_bytes)
    _workspace(ctx, ctx.lib.pimdal_hash_join_workspace_size, a)
    t, cached = L.Tuning(), C.c_int()
    L.check(ctx.lib.pimdal_hash_join_autotune(ctx.handle, C.byref(a), _ptr(result), C.byref(t),
                                              C.byref(cached), _stream(stream)),
            "pimdal_hash_join_autotune")
    return t.as_dict(), bool(cached.value), result, out_payload, out_row


# ---------------------------------------------------------------------------
# Group-by (group_kernel, pimdal/aggregate/aggregate.h:25)
# ---------------------------------------------------------------------------
def group_kernel(ctx: Context, keys, vals=None, *, method: int = L.GROUP_HASH,
                 key_dtype: int = L.I32, expected_groups: int = 0, capacity: int | None = None,
                 want=("sum", "count", "min", "max"), outs=None, result=None, stream=None):
    """Group-by with exact int64 aggregates, groups ascending by key.
    Returns (result, out_key, {name: column})."""
    dev = keys.device
    n = keys.numel()
    if capacity is None:
        capacity = max(1, min(n, expected_groups * 2 if expected_groups else n))
    if outs is None:
        outs = {w: torch.empty(capacity, dtype=torch.int64, device=dev) for w in want}
        outs["key"] = torch.empty(capacity, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.AggrArguments(size=n, in_=_ptr(keys), in_val=_ptr(vals), out=_ptr(outs.get("key")),
                        out_sum=_ptr(outs.get("sum")), out_count=_ptr(outs.get("count")),
                        out_min=_ptr(outs.get("min")), out_max=_ptr(outs.get("max")),
                        out_capacity=capacity, expected_groups=expected_groups,
                        key_dtype=key_dtype, method=method)
    _workspace(ctx, ctx.lib.pimdal_group_workspace_size, a)
    L.check(ctx.lib.pimdal_group_kernel(ctx.handle, C.byref(a), _ptr(result), _stream(stream)),
            "pimdal_group_kernel")
    return result, outs


def group_autotune(ctx: Context, keys, vals=None, *, method: int = L.GROUP_HASH,
                   key_dtype: int = L.I32, expected_groups: int = 0, capacity: int | None = None,
                   want=("sum", "count", "min", "max"), outs=None, result=None, stream=None):
    """pimdal_group_autotune: for a high-cardinality hash group-by, times the
    partitioned mode at a few partition counts and the direct global table on
    these inputs (writing the outputs) and caches the fastest for this shape;
    later group_kernel calls of the shape use it.  Returns (tuning dict,
    cached, result, outs)."""
    dev = keys.device
    n = keys.numel()
    if capacity is None:
        capacity = max(1, min(n, expected_groups * 2 if expected_groups else n))
    if outs is None:
        outs = {w: torch.empty(capacity, dtype=torch.int64, device=dev) for w in want}
        outs["key"] = torch.empty(capacity, dtype=torch.int32, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a = L.AggrArguments(size=n, in_=_ptr(keys), in_val=_ptr(vals), out=_ptr(outs.get("key")),
                        out_sum=_ptr(outs.get("sum")), out_count=_ptr(outs.get("count")),
                        out_min=_ptr(outs.get("min")), out_max=_ptr(outs.get("max")),
                        out_capacity=capacity, expected_groups=expected_groups,
                        key_dtype=key_dtype, method=method)
    _workspace(ctx, ctx.lib.pimdal_group_workspace_size, a)
    t, cached = L.Tuning(), C.c_int()
    L.check(ctx.lib.pimdal_group_autotune(ctx.handle, C.byref(a), _ptr(result), C.byref(t),
                                          C.byref(cached), _stream(stream)),
            "pimdal_group_autotune")
    return t.as_dict(), bool(cached.value), result, outs


# ---------------------------------------------------------------------------
# Pipeline glue (pimdal_gather_u32, pimdal_revenue_keys)
# ---------------------------------------------------------------------------
def gather_u32(ctx: Context, col, idx, n: int | None = None, out=None, stream=None):
    """out[i] = col[idx[i]] for the first n indices."""
    n = idx.numel() if n is None else n
    if out is None:
        out = torch.empty(max(n, 1), dtype=torch.int32, device=idx.device)
    L.check(ctx.lib.pimdal_gather_u32(ctx.handle, _ptr(col), _ptr(idx), n, _ptr(out), _stream(stream)),
            "pimdal_gather_u32")
    return out


_DTYPE_OF = {torch.int32: L.I32, torch.int64: L.I64, torch.uint8: L.U8}


def _col_dtype(t, dtype=None) -> int:
    return _DTYPE_OF[t.dtype] if dtype is None else dtype


def select_aggregate(ctx: Context, size: int, *, preds=(), group=(), key_space: int = 1,
                     exprs=(), rows=None, outs=None, result=None, stream=None):
    """Fused select -> arithmetic -> group-by scan (pimdal_select_aggregate).

    preds: (column, pred) or (column, pred, dtype); group: (column, mult) or
    (column, mult, dtype); exprs: lists of terms, a term being a column, an
    int constant, or (column | None, negate, add[, dtype]) for
    (negate ? -col : col) + add.  Column dtypes follow the tensors (int32 ->
    PIMDAL_I32, int64 -> I64, uint8 -> U8) unless given.  Returns
    (result, outs) with outs "key", "count" and "sum0".. "sum{n-1}" holding
    the groups in key order (result[0] of them)."""
    dev = f"cuda:{ctx.device}"
    a = L.SelectAggregateArguments()
    a.size = size
    a.rows = _ptr(rows)
    a.n_preds = len(preds)
    for q, pr in enumerate(preds):
        col, pred = pr[0], pr[1]
        a.pred[q] = L.ColumnPred(col=_ptr(col), dtype=_col_dtype(col, pr[2] if len(pr) > 2 else None),
                                 pad=0, pred=pred)
    a.n_group = len(group)
    for g, gr in enumerate(group):
        col, mult = gr[0], gr[1]
        a.group[g] = L.GroupCol(col=_ptr(col), dtype=_col_dtype(col, gr[2] if len(gr) > 2 else None),
                                mult=mult)
    a.key_space = key_space
    a.n_exprs = len(exprs)
    for e, terms in enumerate(exprs):
        a.expr[e] = _expr(terms)
    if outs is None:
        outs = {"key": torch.empty(key_space, dtype=torch.int32, device=dev),
                "count": torch.empty(key_space, dtype=torch.int64, device=dev)}
        for e in range(len(exprs)):
            outs[f"sum{e}"] = torch.empty(key_space, dtype=torch.int64, device=dev)
    if result is None:
        result = torch.empty(1, dtype=torch.int64, device=dev)
    a.out_key = _ptr(outs["key"])
    a.out_count = _ptr(outs["count"])
    for e in range(len(exprs)):
        a.out_sum[e] = _ptr(outs.get(f"sum{e}"))
    a.out_capacity = outs["key"].numel()
    _workspace(ctx, ctx.lib.pimdal_select_aggregate_workspace_size, a)
    L.check(ctx.lib.pimdal_select_aggregate(ctx.handle, C.byref(a), _ptr(result), _stream(stream)),
            "pimdal_select_aggregate")
    return result, outs


def _expr(terms) -> L.Expr:
    """Expression struct of a list of terms (as select_aggregate's exprs)."""
    x = L.Expr()
    x.n_terms = len(terms)
    for t, term in enumerate(terms):
        if isinstance(term, int):
            term = (None, 0, term)
        elif isinstance(term, torch.Tensor):
            term = (term, 0, 0)
        col, neg, add = term[0], term[1], term[2]
        dt = 0 if col is None else _col_dtype(col, term[3] if len(term) > 3 else None)
        x.term[t] = L.Term(col=_ptr(col), dtype=dt, negate=neg, add=add)
    return x


def project(ctx: Context, size: int, terms, *, minus=(), rows=None, out=None,
            out_dtype: int = L.I64, shift: int = 0, stream=None) -> torch.Tensor:
    """Per-row arithmetic (pimdal_project): out[i] = (the product of `terms`)
    - (the product of `minus`, 0 when empty) at row rows[i] (or i), shifted
    right by shift bits.  Terms as select_aggregate's expressions; a single
    column term makes it a gather of that column."""
    if out is None:
        dt = torch.int64 if out_dtype == L.I64 else torch.int32
        out = torch.empty(max(size, 1), dtype=dt, device=f"cuda:{ctx.device}")
    a = L.ProjectArguments(size=size, rows=_ptr(rows), expr=_expr(terms), minus=_expr(minus),
                           out=_ptr(out), out_dtype=out_dtype, shift=shift)
    L.check(ctx.lib.pimdal_project(ctx.handle, C.byref(a), _stream(stream)), "pimdal_project")
    return out


def revenue_keys(ctx: Context, n: int, match_row, match_attr, sel_rows, price, discount, flag,
                 attr_mult: int, out_key, out_val, stream=None) -> None:
    """key = attr * attr_mult + flag[row], value = price[row] * (100 - discount[row])
    for the first n joined rows (row = sel_rows[match_row[i]])."""
    a = L.RevenueArguments(size=n, match_row=_ptr(match_row), match_attr=_ptr(match_attr),
                           sel_rows=_ptr(sel_rows), price=_ptr(price), discount=_ptr(discount),
                           flag=_ptr(flag), attr_mult=attr_mult, out_key=_ptr(out_key),
                           out_val=_ptr(out_val))
    L.check(ctx.lib.pimdal_revenue_keys(ctx.handle, C.byref(a), _stream(stream)), "pimdal_revenue_keys")


# ---------------------------------------------------------------------------
# Batched form (pimdal_group_batch_create / pimdal_hash_join_batch_create)
# ---------------------------------------------------------------------------
def group_args(keys, vals, outs, *, expected_groups: int = 0, capacity: int | None = None,
               key_dtype: int = L.I32, method: int = L.GROUP_HASH) -> L.AggrArguments:
    """Argument struct of one group-by instance (outputs: dict as group_kernel)."""
    n = keys.numel()
    if capacity is None:
        capacity = outs["key"].numel() if "key" in outs else max(n, 1)
    return L.AggrArguments(size=n, in_=_ptr(keys), in_val=_ptr(vals), out=_ptr(outs.get("key")),
                           out_sum=_ptr(outs.get("sum")), out_count=_ptr(outs.get("count")),
                           out_min=_ptr(outs.get("min")), out_max=_ptr(outs.get("max")),
                           out_capacity=capacity, expected_groups=expected_groups,
                           key_dtype=key_dtype, method=method)


def hash_join_args(build_key, build_payload, probe_key, probe_ptr, out_payload, out_row, *,
                   capacity: int | None = None, load_factor_pct: int = 0) -> L.HashJoinArguments:
    """Argument struct of one (unpartitioned) hash-join instance."""
    if capacity is None:
        capacity = out_payload.numel()
    return L.HashJoinArguments(build_key=_ptr(build_key), build_payload=_ptr(build_payload),
                               size_build=build_key.numel(), probe_key=_ptr(probe_key),
                               probe_ptr=_ptr(probe_ptr), size_probe=probe_key.numel(),
                               out_build_payload=_ptr(out_payload), out_probe_ptr=_ptr(out_row),
                               out_capacity=capacity, partition_bits=0xFFFFFFFF,
                               load_factor_pct=load_factor_pct, l2_budget_bytes=0)


class Batch:
    """A plan of many instances of one operator, run by one persistent launch
    per phase.  results: int64 device tensor of the per-instance counts."""

    def __init__(self, ctx: Context, kind: int, args: list, *, tuning: L.BatchTuning | None = None):
        self.ctx = ctx
        self.kind = kind
        n = len(args)
        self.results = torch.zeros(max(n, 1), dtype=torch.int64, device=f"cuda:{ctx.device}")
        typ = L.AggrArguments if kind == L.BATCH_GROUP else L.HashJoinArguments
        self._args = (typ * max(n, 1))(*args)
        self.count = n
        h = C.c_void_p()
        fn = (ctx.lib.pimdal_group_batch_create if kind == L.BATCH_GROUP
              else ctx.lib.pimdal_hash_join_batch_create)
        L.check(fn(ctx.handle, self._args, n, C.byref(tuning) if tuning is not None else None,
                   self.results.data_ptr(), C.byref(h)), fn.__name__)
        self.handle = h

    @staticmethod
    def autotune(ctx: Context, kind: int, args: list, results=None, stream=None):
        """(best tuning, came from the cache).  Runs the instances while timing."""
        n = len(args)
        typ = L.AggrArguments if kind == L.BATCH_GROUP else L.HashJoinArguments
        arr = (typ * max(n, 1))(*args)
        if results is None:
            results = torch.zeros(max(n, 1), dtype=torch.int64, device=f"cuda:{ctx.device}")
        best = L.BatchTuning()
        cached = C.c_int()
        L.check(ctx.lib.pimdal_batch_autotune(ctx.handle, kind, C.cast(arr, C.c_void_p), n,
                                              results.data_ptr(), C.byref(best), C.byref(cached),
                                              _stream(stream)), "pimdal_batch_autotune")
        return best, bool(cached.value)

    def run(self, stream=None) -> None:
        L.check(self.ctx.lib.pimdal_batch_run(self.ctx.handle, self.handle, _stream(stream)),
                "pimdal_batch_run")

    @property
    def device_bytes(self) -> int:
        b = C.c_size_t()
        L.check(self.ctx.lib.pimdal_batch_device_bytes(self.handle, C.byref(b)),
                "pimdal_batch_device_bytes")
        return int(b.value)

    def close(self) -> None:
        if self.handle:
            self.ctx.lib.pimdal_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
