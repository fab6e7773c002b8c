"""Loading Parquet / CSV data into HBM-resident tables.

The reference's loaders turn every Arrow column into one u64 cell per value
(src/datasource/parquet.rs:271-460): signed integers and Date32 days are cast
with sign extension (``value as u64``), unsigned integers zero-extend, Float64
keeps its bit pattern, and a null becomes the cell 0. ``arrow_cells`` builds
exactly those cells, plus an i32 sidecar for columns whose Arrow type is at
most 32 bits wide (the narrow copy the reference's CSV loader keeps,
src/datasource/table.rs:52-61); ``register_parquet`` / ``register_csv`` hand
both to ``tgp_table_register_cells``, which stores each column at the narrowest
exact width on the device. Booleans become the cells 0 / 1, and Utf8 /
LargeUtf8 strings the xxh3_64 hash of their bytes (parquet.rs:389-436), which
equality predicates on string literals compare against (the reference's
string search index for LIKE is not built).

Differences from the reference, on purpose: a column type the reference fills
with zeros (timestamps, decimals, ...) raises here instead; and comparison
types are inferred from the Arrow type (Date32 → date, Float64 → float, other
columns int) where the reference types a table without a schema as all Int
unless it is a TPC-H table (ExecTable::from_catalog,
src/engine/query_interpreter/types.rs:271-305). ``coltypes`` overrides the
inference per column, so the reference's typing can be asked for.
"""
from __future__ import annotations

import numpy as np

_SIGNED = {"int8", "int16", "int32", "int64"}
_UNSIGNED = {"uint8", "uint16", "uint32", "uint64"}


def arrow_cells(table) -> tuple[dict, dict, dict]:
    """(cells, sidecars, coltypes) of a ``pyarrow.Table``: u64 cells per
    column as the reference's loader makes them, i32 sidecars where the Arrow
    type is at most 32 bits wide and every value fits, and the coltype each
    column compares as ('int', 'date' or 'float')."""
    import pyarrow as pa

    cells, sidecars, coltypes = {}, {}, {}
    for name in table.column_names:
        arr = table.column(name).combine_chunks()
        t = arr.type
        tname = str(t)
        if pa.types.is_date32(t):
            vals = arr.cast(pa.int32()).fill_null(0).to_numpy(zero_copy_only=False).astype(np.int32)
            cells[name] = vals.astype(np.int64).view(np.uint64)
            sidecars[name] = vals
            coltypes[name] = "date"
        elif tname in _SIGNED:
            vals = arr.fill_null(0).to_numpy(zero_copy_only=False)
            cells[name] = vals.astype(np.int64).view(np.uint64)
            if vals.dtype.itemsize <= 4:
                sidecars[name] = vals.astype(np.int32)
            coltypes[name] = "int"
        elif tname in _UNSIGNED:
            vals = arr.fill_null(0).to_numpy(zero_copy_only=False)
            cells[name] = vals.astype(np.uint64)
            if vals.dtype.itemsize < 4 or (vals.dtype.itemsize == 4 and (vals.size == 0 or vals.max() <= 2**31 - 1)):
                sidecars[name] = vals.astype(np.int32)
            coltypes[name] = "int"
        elif pa.types.is_boolean(t):
            vals = arr.fill_null(False).to_numpy(zero_copy_only=False).astype(np.int32)
            cells[name] = vals.astype(np.uint64)
            sidecars[name] = vals
            coltypes[name] = "int"
        elif pa.types.is_string(t) or pa.types.is_large_string(t):
            from .engine import string_cell
            cells[name] = np.array([0 if x is None else string_cell(x) for x in arr.to_pylist()], dtype=np.uint64)
            coltypes[name] = "int"
        elif pa.types.is_float64(t):
            vals = arr.fill_null(0.0).to_numpy(zero_copy_only=False).astype(np.float64)
            cells[name] = vals.view(np.uint64)
            # A null's cell is 0 (the bits of +0.0), as in the reference.
            coltypes[name] = "float"
        else:
            raise TypeError(f"column {name!r}: Arrow type {t} is not loaded (the reference fills it with zeros)")
    return cells, sidecars, coltypes


def read_parquet(path, columns=None) -> tuple[dict, dict, dict]:
    import pyarrow.parquet as pq
    return arrow_cells(pq.read_table(path, columns=columns))


def read_csv(path, columns=None) -> tuple[dict, dict, dict]:
    import pyarrow.csv as pcsv
    opts = pcsv.ConvertOptions(include_columns=columns) if columns else None
    return arrow_cells(pcsv.read_csv(path, convert_options=opts))


def register_parquet(ctx, path, columns=None, coltypes: dict | None = None):
    """Reads a Parquet file and registers it (narrowed on the device).
    ``coltypes`` overrides the inferred comparison type per column."""
    cells, sidecars, inferred = read_parquet(path, columns)
    return ctx.register_cells(cells, {**inferred, **(coltypes or {})}, sidecars)


def register_csv(ctx, path, columns=None, coltypes: dict | None = None):
    cells, sidecars, inferred = read_csv(path, columns)
    return ctx.register_cells(cells, {**inferred, **(coltypes or {})}, sidecars)
