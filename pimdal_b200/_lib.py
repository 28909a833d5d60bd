"""ctypes binding of the C ABI in include/pimdal_gpu.h.

The shared library is loaded from the package directory only (built in-tree by
pimdal_b200/build.py).  There is no fallback: if the library is missing every
operator raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpimdal_b200.so"

# ---- enums (mirror include/pimdal_gpu.h) ----------------------------------
PIMDAL_OK = 0
STATUS_NAMES = {
    0: "PIMDAL_OK", 1: "PIMDAL_ERR_ARG", 2: "PIMDAL_ERR_OOM", 3: "PIMDAL_ERR_WORKSPACE",
    4: "PIMDAL_ERR_TABLE_FULL", 5: "PIMDAL_ERR_DEVICE_TIMEOUT", 6: "PIMDAL_ERR_CUDA",
    7: "PIMDAL_ERR_CAPACITY", 8: "PIMDAL_ERR_BUDGET", 9: "PIMDAL_ERR_NOT_SUPPORTED",
}
U32, I32, I64, U8 = 0, 1, 2, 3
LAYOUT_COLUMNS, LAYOUT_PAIRS = 0, 1
PRED_LT, PRED_LE, PRED_GT, PRED_GE, PRED_EQ, PRED_NE, PRED_BETWEEN, PRED_RANGE = range(8)
GEN_UNIFORM, GEN_PERM, GEN_PERM_UNIFORM, GEN_PERM_ZIPF, GEN_PROBE = range(5)
(KERNEL_SELECT, KERNEL_GEN, KERNEL_SORT_HIST, KERNEL_SORT_PASS, KERNEL_SMJ_MERGE, KERNEL_PARTITION,
 KERNEL_HJ_BUILD, KERNEL_HJ_PROBE, KERNEL_GROUP, KERNEL_SEGREDUCE, KERNEL_OTHER, KERNEL_FILTER,
 KERNEL_MATCH, KERNEL_FUSED, KERNEL_SCAN_AGG) = range(15)
KERNEL_COUNT = 15
FILTER_BITS = 16384
FILTER_BYTES = FILTER_BITS // 8


class PimdalError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}")


# ---- structs ----------------------------------------------------------------
class GenSpec(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("out_dtype", C.c_int32),
        ("seed", C.c_uint64), ("stream_id", C.c_uint64),
        ("lo", C.c_int64), ("hi", C.c_int64),
        ("perm_domain", C.c_uint64),
        ("cdf", C.c_void_p), ("cdf_n", C.c_uint64),
        ("match_permille", C.c_uint32), ("pad", C.c_uint32),
    ]


class Pred(C.Structure):
    _fields_ = [("op", C.c_int32), ("pad", C.c_int32), ("lo", C.c_int64), ("hi", C.c_int64)]


class SelArguments(C.Structure):
    _fields_ = [
        ("size", C.c_uint64), ("in_", C.c_void_p), ("in_ptr", C.c_void_p),
        ("ptr_base", C.c_uint64), ("out", C.c_void_p), ("out_ptr", C.c_void_p),
        ("pred", Pred), ("key_dtype", C.c_int32), ("layout", C.c_int32),
    ]


class SortArguments(C.Structure):
    _fields_ = [
        ("nr_elements", C.c_uint64), ("in_", C.c_void_p), ("in_ptr", C.c_void_p),
        ("ptr_base", C.c_uint64), ("out", C.c_void_p), ("out_ptr", C.c_void_p),
        ("key_dtype", C.c_int32), ("layout", C.c_int32),
        ("begin_bit", C.c_uint32), ("end_bit", C.c_uint32),
    ]


class SmjMergeArguments(C.Structure):
    _fields_ = [
        ("inner", C.c_void_p), ("inner_ptr", C.c_void_p), ("size_inner", C.c_uint64),
        ("outer", C.c_void_p), ("outer_ptr", C.c_void_p), ("size_outer", C.c_uint64),
        ("out_outer", C.c_void_p), ("out_inner", C.c_void_p), ("out_capacity", C.c_uint64),
        ("key_dtype", C.c_int32), ("pad", C.c_int32),
    ]


class SmjArguments(C.Structure):
    _fields_ = [
        ("inner_key", C.c_void_p), ("inner_payload", C.c_void_p), ("size_inner", C.c_uint64),
        ("outer_key", C.c_void_p), ("outer_payload", C.c_void_p), ("size_outer", C.c_uint64),
        ("out_inner_payload", C.c_void_p), ("out_outer_payload", C.c_void_p),
        ("out_capacity", C.c_uint64), ("key_dtype", C.c_int32), ("pad", C.c_int32),
    ]


class PartArguments(C.Structure):
    _fields_ = [
        ("in_", C.c_void_p), ("in_ptr", C.c_void_p), ("size", C.c_uint64),
        ("shift", C.c_uint32), ("part_n", C.c_uint32), ("part_out", C.c_void_p),
        ("part_out_ptr", C.c_void_p), ("part_sizes", C.c_void_p),
        ("layout", C.c_int32), ("pad", C.c_int32),
    ]


class HashArguments(C.Structure):
    _fields_ = [
        ("in_key", C.c_void_p), ("in_ptr", C.c_void_p), ("size", C.c_uint64),
        ("table_ptr", C.c_void_p), ("table_size", C.c_uint64),
    ]


class ProbeArguments(C.Structure):
    _fields_ = [
        ("table_ptr", C.c_void_p), ("table_size", C.c_uint64), ("in_key", C.c_void_p),
        ("in_ptr", C.c_void_p), ("size", C.c_uint64), ("out_outer", C.c_void_p),
        ("out_inner", C.c_void_p), ("out_capacity", C.c_uint64),
    ]


class HashJoinArguments(C.Structure):
    _fields_ = [
        ("build_key", C.c_void_p), ("build_payload", C.c_void_p), ("size_build", C.c_uint64),
        ("probe_key", C.c_void_p), ("probe_ptr", C.c_void_p), ("size_probe", C.c_uint64),
        ("out_build_payload", C.c_void_p), ("out_probe_ptr", C.c_void_p),
        ("out_capacity", C.c_uint64), ("partition_bits", C.c_uint32),
        ("load_factor_pct", C.c_uint32), ("l2_budget_bytes", C.c_uint64),
    ]


class FilterArguments(C.Structure):
    _fields_ = [
        ("in_", C.c_void_p), ("filter_ptr", C.c_void_p), ("part_sizes", C.c_void_p),
        ("part_n", C.c_uint32), ("layout", C.c_int32),
    ]


class MatchArguments(C.Structure):
    _fields_ = [
        ("filter_ptr", C.c_void_p), ("size", C.c_uint64), ("part_ptr", C.c_void_p),
        ("part_row", C.c_void_p), ("out_ptr", C.c_void_p), ("out_row", C.c_void_p),
        ("out_capacity", C.c_uint64), ("match_sizes", C.c_void_p), ("part_sizes", C.c_void_p),
        ("part_n", C.c_uint32), ("layout", C.c_int32),
    ]


FUSED_MAX_KEYS = 4096


class SelectJoinAggregateArguments(C.Structure):
    _fields_ = [
        ("size", C.c_uint64), ("date", C.c_void_p), ("date_lo", C.c_int32), ("date_hi", C.c_int32),
        ("jkey", C.c_void_p), ("table_ptr", C.c_void_p), ("table_size", C.c_uint64),
        ("flag", C.c_void_p), ("price", C.c_void_p), ("discount", C.c_void_p),
        ("attr_mult", C.c_uint32), ("key_space", C.c_uint32), ("out_key", C.c_void_p),
        ("out_sum", C.c_void_p), ("out_count", C.c_void_p), ("out_capacity", C.c_uint64),
    ]


SA_MAX_PREDS, SA_MAX_GROUP_COLS, SA_MAX_EXPRS, SA_MAX_TERMS, SA_MAX_KEYS = 4, 2, 6, 3, 1024


class ColumnPred(C.Structure):
    _fields_ = [("col", C.c_void_p), ("dtype", C.c_int32), ("pad", C.c_int32), ("pred", Pred)]


class GroupCol(C.Structure):
    _fields_ = [("col", C.c_void_p), ("dtype", C.c_int32), ("mult", C.c_uint32)]


class Term(C.Structure):
    _fields_ = [("col", C.c_void_p), ("dtype", C.c_int32), ("negate", C.c_int32),
                ("add", C.c_int64)]


class Expr(C.Structure):
    _fields_ = [("term", Term * SA_MAX_TERMS), ("n_terms", C.c_uint32), ("pad", C.c_uint32)]


class SelectAggregateArguments(C.Structure):
    _fields_ = [
        ("size", C.c_uint64), ("rows", C.c_void_p),
        ("pred", ColumnPred * SA_MAX_PREDS), ("n_preds", C.c_uint32), ("n_group", C.c_uint32),
        ("group", GroupCol * SA_MAX_GROUP_COLS), ("key_space", C.c_uint32),
        ("n_exprs", C.c_uint32), ("expr", Expr * SA_MAX_EXPRS),
        ("out_key", C.c_void_p), ("out_count", C.c_void_p),
        ("out_sum", C.c_void_p * SA_MAX_EXPRS), ("out_capacity", C.c_uint64),
    ]


class ProjectArguments(C.Structure):
    _fields_ = [("size", C.c_uint64), ("rows", C.c_void_p), ("expr", Expr), ("minus", Expr),
                ("out", C.c_void_p), ("out_dtype", C.c_int32), ("shift", C.c_uint32)]


GROUP_AUTO, GROUP_HASH, GROUP_SORT = 0, 1, 2


class AggrArguments(C.Structure):
    _fields_ = [
        ("size", C.c_uint64), ("in_", C.c_void_p), ("in_val", C.c_void_p), ("out", C.c_void_p),
        ("out_sum", C.c_void_p), ("out_count", C.c_void_p), ("out_min", C.c_void_p),
        ("out_max", C.c_void_p), ("out_capacity", C.c_uint64), ("expected_groups", C.c_uint64),
        ("key_dtype", C.c_int32), ("method", C.c_int32),
    ]


class RevenueArguments(C.Structure):
    _fields_ = [
        ("size", C.c_uint64), ("match_row", C.c_void_p), ("match_attr", C.c_void_p),
        ("sel_rows", C.c_void_p), ("price", C.c_void_p), ("discount", C.c_void_p),
        ("flag", C.c_void_p), ("attr_mult", C.c_uint32), ("pad", C.c_uint32),
        ("out_key", C.c_void_p), ("out_val", C.c_void_p),
    ]


class BatchTuning(C.Structure):
    _fields_ = [("rows_per_item", C.c_uint32), ("load_factor_pct", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]


BATCH_GROUP, BATCH_HASH_JOIN = 0, 1


class Tuning(C.Structure):
    _fields_ = [("partition_bits", C.c_uint32), ("load_factor_pct", C.c_uint32),
                ("group_mode", C.c_uint32), ("group_part_bits", C.c_uint32),
                ("ms", C.c_float), ("candidates", C.c_uint32)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}

# Exported symbols and their ctypes signatures.
_VP, _SZ, _U64, _I = C.c_void_p, C.c_size_t, C.c_uint64, C.c_int
SIGNATURES = {
    "pimdal_abi_version": (_I, []),
    "pimdal_status_string": (C.c_char_p, [_I]),
    "pimdal_ctx_create": (_I, [C.POINTER(_VP), _I]),
    "pimdal_ctx_destroy": (_I, [_VP]),
    "pimdal_ctx_set_workspace": (_I, [_VP, _VP, _SZ]),
    "pimdal_ctx_sync_status": (_I, [_VP, _VP]),
    "pimdal_ctx_launch_count": (_U64, [_VP]),
    "pimdal_ctx_set_profiling": (_I, [_VP, _I]),
    "pimdal_ctx_kernel_time": (_I, [_VP, _I, C.POINTER(_U64), C.POINTER(C.c_double)]),
    "pimdal_gen_column": (_I, [_VP, C.POINTER(GenSpec), _VP, _U64, _U64, _VP]),
    "pimdal_sel_workspace_size": (_I, [C.POINTER(SelArguments), C.POINTER(_SZ)]),
    "pimdal_sel_kernel": (_I, [_VP, C.POINTER(SelArguments), _VP, _VP]),
    "pimdal_sel_kernel_noalloc": (_I, [C.POINTER(SelArguments), _VP, _VP]),
    "pimdal_sort_workspace_size": (_I, [C.POINTER(SortArguments), C.POINTER(_SZ)]),
    "pimdal_sort_kernel": (_I, [_VP, C.POINTER(SortArguments), _VP]),
    "pimdal_smj_merge_workspace_size": (_I, [C.POINTER(SmjMergeArguments), C.POINTER(_SZ)]),
    "pimdal_smj_merge": (_I, [_VP, C.POINTER(SmjMergeArguments), _VP, _VP]),
    "pimdal_sort_merge_join_workspace_size": (_I, [C.POINTER(SmjArguments), C.POINTER(_SZ)]),
    "pimdal_sort_merge_join": (_I, [_VP, C.POINTER(SmjArguments), _VP, _VP]),
    "pimdal_part_workspace_size": (_I, [C.POINTER(PartArguments), C.POINTER(_SZ)]),
    "pimdal_part_kernel": (_I, [_VP, C.POINTER(PartArguments), _VP]),
    "pimdal_hash_table_bytes": (_SZ, [_U64]),
    "pimdal_hash_kernel": (_I, [_VP, C.POINTER(HashArguments), _VP]),
    "pimdal_hj_probe": (_I, [_VP, C.POINTER(ProbeArguments), _VP, _VP]),
    "pimdal_filter_kernel": (_I, [_VP, C.POINTER(FilterArguments), _VP]),
    "pimdal_ingest": (_I, [_VP, _VP, _SZ, _VP, _VP]),
    "pimdal_select_join_aggregate": (_I, [_VP, C.POINTER(SelectJoinAggregateArguments), _VP, _VP]),
    "pimdal_select_join_aggregate_workspace_size": (_I, [C.POINTER(SelectJoinAggregateArguments),
                                                        C.POINTER(_SZ)]),
    "pimdal_select_aggregate": (_I, [_VP, C.POINTER(SelectAggregateArguments), _VP, _VP]),
    "pimdal_project": (_I, [_VP, C.POINTER(ProjectArguments), _VP]),
    "pimdal_select_aggregate_workspace_size": (_I, [C.POINTER(SelectAggregateArguments),
                                                   C.POINTER(_SZ)]),
    "pimdal_match_workspace_size": (_I, [C.POINTER(MatchArguments), C.POINTER(_SZ)]),
    "pimdal_match_kernel": (_I, [_VP, C.POINTER(MatchArguments), _VP, _VP]),
    "pimdal_hash_join_workspace_size": (_I, [C.POINTER(HashJoinArguments), C.POINTER(_SZ)]),
    "pimdal_hash_join": (_I, [_VP, C.POINTER(HashJoinArguments), _VP, _VP]),
    "pimdal_group_workspace_size": (_I, [C.POINTER(AggrArguments), C.POINTER(_SZ)]),
    "pimdal_group_kernel": (_I, [_VP, C.POINTER(AggrArguments), _VP, _VP]),
    "pimdal_gather_u32": (_I, [_VP, _VP, _VP, _U64, _VP, _VP]),
    "pimdal_revenue_keys": (_I, [_VP, C.POINTER(RevenueArguments), _VP]),
    "pimdal_group_batch_create": (_I, [_VP, C.POINTER(AggrArguments), C.c_uint32,
                                       C.POINTER(BatchTuning), _VP, C.POINTER(_VP)]),
    "pimdal_hash_join_batch_create": (_I, [_VP, C.POINTER(HashJoinArguments), C.c_uint32,
                                           C.POINTER(BatchTuning), _VP, C.POINTER(_VP)]),
    "pimdal_batch_run": (_I, [_VP, _VP, _VP]),
    "pimdal_batch_device_bytes": (_I, [_VP, C.POINTER(_SZ)]),
    "pimdal_batch_destroy": (_I, [_VP]),
    "pimdal_batch_autotune": (_I, [_VP, _I, _VP, C.c_uint32, _VP, C.POINTER(BatchTuning),
                                   C.POINTER(_I), _VP]),
    "pimdal_hash_join_autotune": (_I, [_VP, C.POINTER(HashJoinArguments), _VP,
                                       C.POINTER(Tuning), C.POINTER(_I), _VP]),
    "pimdal_group_autotune": (_I, [_VP, C.POINTER(AggrArguments), _VP, C.POINTER(Tuning),
                                   C.POINTER(_I), _VP]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libpimdal_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m pimdal_b200.build` "
                "(there is no CPU fallback)")
        mode = getattr(os, "RTLD_LOCAL", 0)
        l = C.CDLL(str(LIB_PATH), mode=mode)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(status: int, where: str) -> None:
    if status != PIMDAL_OK:
        raise PimdalError(status, where)
