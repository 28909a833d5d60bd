"""The C-ABI library loads (no GPU needed) and exports every declared entry point."""
import ctypes
import re
from pathlib import Path

import pytest

from pimdal_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(pimdal_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_header():
    # every declared function has a ctypes signature in the Python layer
    assert set(declared_functions()) <= set(L.SIGNATURES), \
        sorted(set(declared_functions()) - set(L.SIGNATURES))


def test_status_strings_and_version():
    lib = L.lib()
    assert lib.pimdal_abi_version() == 1
    assert lib.pimdal_status_string(0) == b"ok"
    assert lib.pimdal_status_string(4) == b"hash table full"


def test_argument_errors_need_no_gpu():
    lib = L.lib()
    # null context / arguments are rejected before any CUDA call
    assert lib.pimdal_sel_kernel(None, None, None, None) == 1
    assert lib.pimdal_ctx_destroy(None) == 1
    sz = ctypes.c_size_t(7)
    assert lib.pimdal_sel_workspace_size(None, ctypes.byref(sz)) == 1


def test_batch_argument_errors_need_no_gpu():
    lib = L.lib()
    plan = ctypes.c_void_p()
    # null context, plan pointer or instance arrays are rejected before any CUDA call
    assert lib.pimdal_group_batch_create(None, None, 0, None, None, ctypes.byref(plan)) == 1
    assert lib.pimdal_hash_join_batch_create(None, None, 0, None, None, ctypes.byref(plan)) == 1
    assert lib.pimdal_batch_run(None, None, None) == 1
    assert lib.pimdal_batch_destroy(None) == 0
    sz = ctypes.c_size_t(7)
    assert lib.pimdal_batch_device_bytes(None, ctypes.byref(sz)) == 1
    best = L.BatchTuning()
    assert lib.pimdal_batch_autotune(None, 0, None, 0, None, ctypes.byref(best), None, None) == 1


def test_prefilter_fused_and_ingest_argument_errors_need_no_gpu():
    lib = L.lib()
    fa, ma = L.FilterArguments(), L.MatchArguments()
    sa = L.SelectJoinAggregateArguments()
    assert lib.pimdal_filter_kernel(None, ctypes.byref(fa), None) == 1
    assert lib.pimdal_match_kernel(None, ctypes.byref(ma), None, None) == 1
    assert lib.pimdal_select_join_aggregate(None, ctypes.byref(sa), None, None) == 1
    assert lib.pimdal_ingest(None, None, 16, None, None) == 1
    sz = ctypes.c_size_t(7)
    ma.size = 2048 * 10 + 1
    assert lib.pimdal_match_workspace_size(ctypes.byref(ma), ctypes.byref(sz)) == 0
    assert sz.value == 8 * 11  # one (first, last) partition pair per 2048-row tile
    sa.key_space = 50
    assert lib.pimdal_select_join_aggregate_workspace_size(ctypes.byref(sa), ctypes.byref(sz)) == 0
    assert sz.value == 16 * 50
    sa.key_space = L.FUSED_MAX_KEYS + 1
    assert lib.pimdal_select_join_aggregate_workspace_size(ctypes.byref(sa), ctypes.byref(sz)) == 1


def test_select_aggregate_layout_and_argument_errors_need_no_gpu():
    lib = L.lib()
    a = L.SelectAggregateArguments()
    # the ctypes mirror has the C struct's size (offsets follow from the fields)
    assert ctypes.sizeof(a) == (8 + 8 + L.SA_MAX_PREDS * 40 + 8 + L.SA_MAX_GROUP_COLS * 16 + 8
                                + L.SA_MAX_EXPRS * (L.SA_MAX_TERMS * 24 + 8) + 8 + 8
                                + L.SA_MAX_EXPRS * 8 + 8)
    assert lib.pimdal_select_aggregate(None, ctypes.byref(a), None, None) == 1
    sz = ctypes.c_size_t(7)
    a.key_space, a.n_exprs = 6, 5
    assert lib.pimdal_select_aggregate_workspace_size(ctypes.byref(a), ctypes.byref(sz)) == 0
    assert sz.value == 8 * 6 * 6
    a.key_space = L.SA_MAX_KEYS + 1
    assert lib.pimdal_select_aggregate_workspace_size(ctypes.byref(a), ctypes.byref(sz)) == 1


def test_project_layout_and_argument_errors_need_no_gpu():
    lib = L.lib()
    a = L.ProjectArguments()
    assert ctypes.sizeof(a) == 8 + 8 + 2 * (L.SA_MAX_TERMS * 24 + 8) + 8 + 4 + 4
    assert lib.pimdal_project(None, ctypes.byref(a), None) == 1


def test_autotune_layout_and_argument_errors_need_no_gpu():
    lib = L.lib()
    assert ctypes.sizeof(L.Tuning) == 24
    t, c = L.Tuning(), ctypes.c_int()
    assert lib.pimdal_hash_join_autotune(None, None, None, ctypes.byref(t), ctypes.byref(c),
                                         None) == 1
    assert lib.pimdal_group_autotune(None, None, None, ctypes.byref(t), ctypes.byref(c), None) == 1


def test_tpch_packed_dates_follow_the_reference_reader():
    from pimdal_b200 import tpch
    # read_table.cpp:8-16: day + (month << 5) + ((year - 1900) << 9)
    assert tpch.packed("1994-01-01") == 1 + (1 << 5) + (94 << 9)
    assert tpch.packed("1998-09-02") == 2 + (9 << 5) + (98 << 9)
    assert tpch.packed(tpch.Q6_DATE_LO) < tpch.packed(tpch.Q6_DATE_HI)


def test_kernel_ids_cover_the_count():
    ids = sorted(getattr(L, k) for k in dir(L) if k.startswith("KERNEL_") and k != "KERNEL_COUNT")
    assert ids == list(range(L.KERNEL_COUNT))
