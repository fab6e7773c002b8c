"""turbogp_b200 — B200 (sm_100a) execution backend for turboGP's hot path:
predicate scan/filter into selection bitmaps, hash-join build and probe, and
grouped/scalar hash aggregation, behind the C ABI of include/turbogp_gpu.h."""
from .engine import (Agg, Col, Context, JoinTable, PreparedQuery, Pred, QueryOutput, Schema, Table, avg,
                     build_col, col, count_col, count_star, lit, max_, min_, string_cell, sum_)

__all__ = ["Agg", "Col", "Context", "JoinTable", "PreparedQuery", "Pred", "QueryOutput", "Schema", "Table", "avg",
           "build_col", "col", "count_col", "count_star", "lit", "max_", "min_", "string_cell", "sum_"]
