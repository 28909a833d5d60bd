"""GPU ingress: pimdal_ingest copies pageable sources (through the pinned
staging buffers: sizes of one byte, one chunk, several chunks and a ragged
tail) and pinned sources exactly; a parquet table with fixed-width,
dictionary-encoded string and date columns arrives on the device with the
same values, codes and packed dates."""
import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest
import torch

from pimdal_b200 import ingest

pytestmark = pytest.mark.gpu

CHUNK = 16 << 20


@pytest.mark.parametrize("nbytes", [1, 4097, CHUNK, 3 * CHUNK + 13])
def test_ingest_pageable_and_pinned(ctx, nbytes):
    src = np.random.default_rng(nbytes).integers(0, 256, nbytes, dtype=np.uint8)
    out = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    ingest.ingest(ctx, src, out)
    src_copy = src.copy()
    src[:] = 0  # the source may be reused as soon as the call returns
    ctx.sync()
    assert np.array_equal(out.cpu().numpy(), src_copy)
    pinned = torch.from_numpy(src_copy).pin_memory()
    out2 = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    ingest.ingest(ctx, pinned.numpy(), out2)
    ctx.sync()
    assert torch.equal(out2.cpu(), pinned)


def test_parquet_table_to_device(ctx, tmp_path):
    rng = np.random.default_rng(9)
    n = 200_001
    seg = np.array(["AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY"])
    days = rng.integers(0, 2557, n)
    dates = (np.datetime64("1992-01-01") + days.astype("timedelta64[D]"))
    t = pa.table({
        "key": pa.array(rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)),
        "price": pa.array(rng.integers(90_000, 10_500_000, n, dtype=np.int64)),
        "flag": pa.array(rng.integers(0, 3, n).astype(np.uint8)),
        "segment": pa.array(seg[rng.integers(0, 5, n)]).dictionary_encode(),
        "shipdate": pa.array(dates.astype("datetime64[D]"), pa.date32()),
        "datestr": pa.array(dates.astype(str)),
    })
    path = tmp_path / "fact.parquet"
    pq.write_table(t, path, row_group_size=50_000)
    back = ingest.read_parquet(path)
    cols = ingest.table_to_device(ctx, back, date_columns=("datestr",))
    ctx.sync()
    assert np.array_equal(cols["key"][0].cpu().numpy(), t.column("key").to_numpy())
    assert np.array_equal(cols["price"][0].cpu().numpy(), t.column("price").to_numpy())
    assert np.array_equal(cols["flag"][0].cpu().numpy(), t.column("flag").to_numpy())
    codes, dictionary = cols["segment"]
    decoded = np.asarray(dictionary.to_pylist())[codes.cpu().numpy()]
    assert decoded.tolist() == t.column("segment").to_pylist()
    packed = ingest.date_to_int(t.column("shipdate"))
    assert np.array_equal(cols["shipdate"][0].cpu().numpy(), packed)
    assert np.array_equal(cols["datestr"][0].cpu().numpy(), packed)
