"""Ingress: Arrow / parquet columns into device columns.

The reference's TPC-H pipelines read the selected columns of a parquet file
into an Arrow table (parquet_to_table, pimdal/main/tpc_h/reader/
read_table.cpp:18-34), encode dates as packed integers (date_to_int, :8-16)
and keep string columns dictionary-encoded (the segment and region
parameters of pimdal/main/tpc_h/query3/shared/param.h are codes).  Here:

* read_parquet: the selected columns of a parquet file, through pyarrow;
* date_to_int: the reference's packed date, day + (month << 5) +
  ((year - 1900) << 9), kept identical because query parameters are written
  in it;
* column_to_device: one Arrow column into a device tensor through
  pimdal_ingest (pinned staging in the library, the host copy of one chunk
  overlapping the transfer of the previous one).  Fixed-width columns keep
  their type; date32 and "YYYY-MM-DD" string columns become packed int32
  dates; dictionary-encoded columns become int32 codes on the device and
  their dictionary on the host;
* table_to_device: every column of a table.

Nulls are not supported (the operators have no validity bitmaps): a column
with nulls raises ValueError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pyarrow as pa
import torch

from . import _lib as L
from . import ops

_TORCH = {np.dtype(np.int8): torch.int8, np.dtype(np.uint8): torch.uint8,
          np.dtype(np.int16): torch.int16, np.dtype(np.int32): torch.int32,
          np.dtype(np.uint32): torch.int32, np.dtype(np.int64): torch.int64,
          np.dtype(np.uint64): torch.int64, np.dtype(np.float32): torch.float32,
          np.dtype(np.float64): torch.float64}


def read_parquet(path, columns=None) -> pa.Table:
    """The selected columns (names or indices) of a parquet file."""
    import pyarrow.parquet as pq
    if columns is not None and all(isinstance(c, int) for c in columns):
        names = pq.read_schema(path).names
        columns = [names[c] for c in columns]
    return pq.read_table(path, columns=columns)


def date_to_int(col) -> np.ndarray:
    """Packed int32 dates (day + (month << 5) + ((year - 1900) << 9)) of a
    date32/date64/timestamp array or of "YYYY-MM-DD" strings."""
    arr = col.combine_chunks() if isinstance(col, pa.ChunkedArray) else col
    if pa.types.is_string(arr.type) or pa.types.is_large_string(arr.type):
        arr = pa.compute.strptime(arr, format="%Y-%m-%d", unit="s")
    days = np.asarray(arr.cast(pa.date32()).cast(pa.int32()).to_numpy(zero_copy_only=False))
    d = days.astype("datetime64[D]")
    y = d.astype("datetime64[Y]")
    m = d.astype("datetime64[M]")
    year = y.astype(np.int64) + 1970
    month = (m - y).astype(np.int64) + 1
    day = (d - m).astype(np.int64) + 1
    return (day + (month << 5) + ((year - 1900) << 9)).astype(np.int32)


def ingest(ctx: ops.Context, host: np.ndarray, out: torch.Tensor, stream=None) -> torch.Tensor:
    """Copies a contiguous host array into a device tensor of the same size
    in bytes (pimdal_ingest).  A pageable array may be reused on return; a
    pinned one is read by the transfer and must stay unchanged until the
    stream has reached the copy."""
    host = np.ascontiguousarray(host)
    nbytes = host.nbytes
    assert out.is_cuda and out.numel() * out.element_size() == nbytes
    st = torch.cuda.current_stream() if stream is None else stream
    L.check(ctx.lib.pimdal_ingest(ctx.handle, C.c_void_p(host.ctypes.data), nbytes,
                                  C.c_void_p(out.data_ptr()), C.c_void_p(st.cuda_stream)),
            "pimdal_ingest")
    return out


def _host_values(arr: pa.Array) -> np.ndarray:
    if arr.null_count:
        raise ValueError("columns with nulls are not supported")
    return arr.to_numpy(zero_copy_only=False)


def column_to_device(ctx: ops.Context, col, *, date: bool = False, stream=None):
    """One column on the device.  Returns (tensor, dictionary or None)."""
    arr = col.combine_chunks() if isinstance(col, pa.ChunkedArray) else col
    dev = f"cuda:{ctx.device}"
    if pa.types.is_dictionary(arr.type):
        if arr.null_count:
            raise ValueError("columns with nulls are not supported")
        codes = np.asarray(arr.indices.to_numpy(zero_copy_only=False)).astype(np.int32)
        t = torch.empty(codes.size, dtype=torch.int32, device=dev)
        return ingest(ctx, codes, t, stream), arr.dictionary
    if date or pa.types.is_date(arr.type) or pa.types.is_timestamp(arr.type):
        if arr.null_count:
            raise ValueError("columns with nulls are not supported")
        v = date_to_int(arr)
    else:
        v = _host_values(arr)
    if v.dtype == np.bool_:
        v = v.astype(np.uint8)
    if v.dtype not in _TORCH:
        raise ValueError(f"unsupported column type {arr.type}")
    t = torch.empty(v.size, dtype=_TORCH[v.dtype], device=dev)
    return ingest(ctx, v, t, stream), None


def table_to_device(ctx: ops.Context, table: pa.Table, date_columns=(), stream=None) -> dict:
    """{name: (device tensor, dictionary or None)} for every column; the
    columns in date_columns (strings) are packed dates."""
    return {name: column_to_device(ctx, table.column(name), date=name in date_columns, stream=stream)
            for name in table.column_names}
