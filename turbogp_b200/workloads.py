"""The benchmark query templates, written once for the GPU engine and the oracle.

* ``filtered_group_agg`` — WHERE ship_day <= max - 90 GROUP BY (flag_a, flag_b):
  count, sum(quantity), sum(price_cents), sum(price_cents * (100 - discount_pct)),
  sum(price_cents * (100 - discount_pct) * (100 + tax_pct)), avg(quantity)
  (TPC-H Q1 shape, 6M rows).
* ``selective_scan_sum`` — ship_day in a 365-day window AND discount_pct
  BETWEEN 5 AND 7 AND quantity < 24: sum(price_cents * discount_pct), count
  (TPC-H Q6 shape, 60M rows).
* ``join_group_agg`` — dimension filtered on order_day < median, inner join on
  fact.fk = dimension.key, GROUP BY segment: sum(price_cents * (100 -
  discount_pct)), count (TPC-H Q3/Q5 shape, 60M x 1.5M rows).
* ``highcard_group`` — GROUP BY key: count, sum(value) (100M rows, ~10M groups).
"""
from __future__ import annotations

from dataclasses import dataclass

from .datagen import DAY0, NDAYS
from .engine import Pred, avg, build_col, col, count_star, sum_


@dataclass
class Template:
    name: str
    where: Pred | None
    group_by: tuple
    aggs: list
    # join: (build where, build key, probe key)
    build_where: Pred | None = None
    build_key: str | None = None
    probe_key: str | None = None


def filtered_group_agg(ship_max: int = DAY0 + NDAYS - 1 - 90) -> Template:
    p, d, t, q = col("price_cents"), col("discount_pct"), col("tax_pct"), col("quantity")
    return Template(
        "filtered_group_agg", col("ship_day") <= ship_max, ("flag_a", "flag_b"),
        [count_star(), sum_(q), sum_(p), sum_(p * (100 - d)), sum_(p * (100 - d) * (100 + t)), avg(q)])


def selective_scan_sum(day_lo: int = DAY0 + 730, days: int = 365, disc_lo: int = 5, disc_hi: int = 7,
                       qty_lt: int = 24) -> Template:
    where = ((col("ship_day") >= day_lo) & (col("ship_day") < day_lo + days) &
             col("discount_pct").between(disc_lo, disc_hi) & (col("quantity") < qty_lt))
    return Template("selective_scan_sum", where, (), [sum_(col("price_cents") * col("discount_pct")), count_star()])


def join_group_agg(order_day_lt: int = DAY0 + NDAYS // 2) -> Template:
    p, d = col("price_cents"), col("discount_pct")
    return Template("join_group_agg", None, (build_col("segment"),), [sum_(p * (100 - d)), count_star()],
                    build_where=col("order_day") < order_day_lt, build_key="key", probe_key="fk")


def highcard_group() -> Template:
    return Template("highcard_group", None, ("key",), [count_star(), sum_(col("value"))])
