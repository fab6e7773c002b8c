"""Parquet / CSV ingest: the u64 cells the reference's loader would build
(src/datasource/parquet.rs:271-460), the i32 sidecars, and the inferred
comparison types. CPU only; the device narrowing is in test_gpu_ingest.py."""
import datetime

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest

from turbogp_b200 import ingest


def _table():
    return pa.table({
        "i8": pa.array([-128, 0, 127, None], pa.int8()),
        "i16": pa.array([-30000, 5, None, 30000], pa.int16()),
        "i32": pa.array([-(2**31), -1, 2**31 - 1, None], pa.int32()),
        "i64": pa.array([-(2**63), 2**63 - 1, None, 7], pa.int64()),
        "u8": pa.array([0, 255, None, 1], pa.uint8()),
        "u32": pa.array([0, 2**32 - 1, 5, None], pa.uint32()),
        "u32s": pa.array([0, 2**31 - 1, 5, None], pa.uint32()),
        "f64": pa.array([1.5, -0.0, None, float("inf")], pa.float64()),
        "d": pa.array([datetime.date(1970, 1, 1), datetime.date(1969, 12, 31), None,
                       datetime.date(1998, 12, 1)], pa.date32()),
    })


def _cell(v: int) -> int:
    return v & 0xFFFFFFFFFFFFFFFF


def test_arrow_cells_follow_the_reference_loader(tmp_path):
    p = tmp_path / "t.parquet"
    pq.write_table(_table(), p)
    cells, side, ct = ingest.read_parquet(p)
    assert all(c.dtype == np.uint64 for c in cells.values())
    assert [int(x) for x in cells["i8"]] == [_cell(-128), 0, 127, 0]
    assert [int(x) for x in cells["i16"]] == [_cell(-30000), 5, 0, 30000]
    assert [int(x) for x in cells["i32"]] == [_cell(-(2**31)), _cell(-1), 2**31 - 1, 0]   # sign extension
    assert [int(x) for x in cells["i64"]] == [2**63, 2**63 - 1, 0, 7]
    assert [int(x) for x in cells["u8"]] == [0, 255, 0, 1]
    assert [int(x) for x in cells["u32"]] == [0, 2**32 - 1, 5, 0]                         # zero extension
    f = np.array([1.5, -0.0, 0.0, np.inf]).view(np.uint64)
    assert np.array_equal(cells["f64"], f)                                                  # f64 bits, null -> 0
    assert [int(x) for x in cells["d"]] == [0, _cell(-1), 0, 10561]                        # days since the epoch
    # Sidecars: Arrow types of at most 32 bits whose values fit i32.
    assert set(side) == {"i8", "i16", "i32", "u8", "u32s", "d"}
    for k, s in side.items():
        assert s.dtype == np.int32
        assert np.array_equal(s.astype(np.int64).view(np.uint64), cells[k])
    assert ct == {"i8": "int", "i16": "int", "i32": "int", "i64": "int", "u8": "int", "u32": "int",
                  "u32s": "int", "f64": "float", "d": "date"}


def test_csv_and_column_selection(tmp_path):
    p = tmp_path / "t.csv"
    p.write_text("a,b,c\n1,2.5,1998-12-01\n-3,4.0,1970-01-02\n")
    cells, side, ct = ingest.read_csv(p)
    assert [int(x) for x in cells["a"]] == [1, _cell(-3)]
    assert np.array_equal(cells["b"], np.array([2.5, 4.0]).view(np.uint64))
    assert [int(x) for x in cells["c"]] == [10561, 1]
    assert ct == {"a": "int", "b": "float", "c": "date"}
    assert "a" not in side  # CSV integers arrive as int64: narrowed on the device instead
    cells, _, _ = ingest.read_csv(p, columns=["c"])
    assert list(cells) == ["c"]


def test_strings_and_booleans():
    import xxhash
    words = ["", "a", "hello", "ünïcødé", "x" * 300, None]
    cells, side, ct = ingest.arrow_cells(pa.table({
        "s": pa.array(words, pa.string()),
        "ls": pa.array(words, pa.large_string()),
        "b": pa.array([True, False, None, True, False, True]),
    }))
    want = [0 if w is None else xxhash.xxh3_64_intdigest(w.encode("utf-8")) for w in words]
    assert [int(x) for x in cells["s"]] == want and [int(x) for x in cells["ls"]] == want
    assert [int(x) for x in cells["b"]] == [1, 0, 0, 1, 0, 1]
    assert ct["s"] == "int" and ct["b"] == "int" and "s" not in side and side["b"].dtype == np.int32


def test_unsupported_types_raise():
    with pytest.raises(TypeError):
        ingest.arrow_cells(pa.table({"t": pa.array([1, 2], pa.timestamp("s"))}))
    with pytest.raises(TypeError):
        ingest.arrow_cells(pa.table({"d": pa.array([1.5], pa.float32())}))
