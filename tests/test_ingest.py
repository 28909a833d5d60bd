"""Ingress on the CPU: the packed-date encoding against the reference
reader's own date_to_int (golden fixture from
pimdal/main/tpc_h/reader/read_table.cpp, and the compiled reader where it is
built), for string and date32 columns; parquet column selection; nulls
rejected."""
from pathlib import Path

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest

import oracle
from pimdal_b200 import ingest

GOLD = Path(__file__).resolve().parent / "golden"


def test_date_to_int_matches_the_reference_golden():
    g = np.load(GOLD / "dates.npz")
    dates = g["dates"].tolist()
    assert np.array_equal(ingest.date_to_int(pa.array(dates)), g["packed"])
    as_date32 = pa.array(dates).cast(pa.timestamp("s")).cast(pa.date32())
    assert np.array_equal(ingest.date_to_int(as_date32), g["packed"])


@pytest.mark.skipif(not oracle.Ref.available("reader"), reason="oracle/_ref not built")
def test_date_to_int_matches_the_reference_reader_fresh():
    rng = np.random.default_rng(5)
    d = (np.datetime64("1900-01-01") + rng.integers(0, 73000, 3000).astype("timedelta64[D]"))
    d = d.astype(str).tolist()
    assert np.array_equal(ingest.date_to_int(pa.array(d)), oracle.Ref().date_to_int(d))


def test_read_parquet_selects_columns(tmp_path):
    t = pa.table({"a": pa.array([1, 2, 3], pa.int32()), "b": pa.array([4, 5, 6], pa.int64()),
                  "c": pa.array(["x", "y", "x"]).dictionary_encode()})
    path = tmp_path / "t.parquet"
    pq.write_table(t, path)
    assert ingest.read_parquet(path, [0, 2]).column_names == ["a", "c"]
    assert ingest.read_parquet(path, ["b"]).column("b").to_pylist() == [4, 5, 6]


def test_nulls_are_rejected():
    with pytest.raises(ValueError):
        ingest._host_values(pa.array([1, None, 3], pa.int32()))
