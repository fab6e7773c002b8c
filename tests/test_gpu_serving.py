"""Served requests on the GPU give the same result alone and in the mix:

* the continuous-batching loop (``serving.serve_batched``) over Poisson
  arrivals of the three light templates with random literals, plus
  high-cardinality GROUP BY requests in the heavy lane on a second context:
  every request's result equals the same request run alone
  (``PreparedQuery.run``), and the oracle's for a sample;
* the same through the wire: statements from concurrent pgwire connections,
  served by the batching executor and by the plain one, return the rows the
  statement returns when executed alone."""
import threading

import numpy as np
import pytest

import oracle
from turbogp_b200 import datagen, serving, sqlfront, workloads
from turbogp_b200.engine import Context, col, count_star, sum_

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES
FCT = {**CT, "fk": "int"}
D0, ND = datagen.DAY0, datagen.NDAYS


def same_query(a, b):
    assert a.rows_selected == b.rows_selected and a.keys == b.keys
    for ra, rb in zip(a.values, b.values):
        for x, y in zip(ra, rb):
            assert (x.value, x.count) == (y.value, y.count)
            assert x.as_f64 == y.as_f64 or abs(x.as_f64 - y.as_f64) <= 1e-12 * abs(y.as_f64)


def random_request(rng, t):
    u = rng.random()
    if u < 0.03:
        return serving.Request(t, "highcard", col("value") < int(rng.integers(100, 1001)), keep=True)
    k = int(rng.integers(0, 3))
    if k == 0:
        lo = D0 + int(rng.integers(0, ND - 30))
        w = ((col("ship_day") >= lo) & (col("ship_day") < lo + int(rng.integers(30, 366))) &
             col("discount_pct").between(int(rng.integers(0, 6)), int(rng.integers(5, 11))) &
             (col("quantity") < int(rng.integers(2, 51))))
        return serving.Request(t, "scan", w, keep=True)
    if k == 1:
        return serving.Request(t, "fga", col("ship_day") <= D0 + int(rng.integers(3, ND)), keep=True)
    return serving.Request(t, "join", col("quantity") < int(rng.integers(2, 51)), keep=True)


def test_serving_loop_results_are_the_same_alone_and_in_the_mix():
    fact = datagen.fact_fk(2_000_003, 50_000, 0.8, seed=61)
    dim = datagen.dimension(50_000, seed=62)
    hc = datagen.highcard(1_000_003, 200_000, 1.1, seed=63)
    with Context(0) as ctx, Context(0) as heavy:
        f = ctx.register(fact, FCT)
        d = ctx.register(dim, datagen.DIMENSION_COLTYPES)
        h = heavy.register(hc)
        tj = workloads.join_group_agg()
        j = d.join_build("key", tj.build_where)
        ts, tf = workloads.selective_scan_sum(), workloads.filtered_group_agg()
        hc_aggs = [count_star(), sum_(col("value"))]
        templates = {
            "scan": serving.Template("scan", lambda: f.prepare(ts.aggs, ts.group_by, ts.where)),
            "fga": serving.Template("fga", lambda: f.prepare(tf.aggs, tf.group_by, tf.where)),
            "join": serving.Template("join", lambda: f.prepare(tj.aggs, tj.group_by, None, join=j, probe_key="fk")),
            "highcard": serving.Template("highcard", lambda: h.prepare(hc_aggs, ("key",), None, group_cap=1 << 18),
                                         heavy=True),
        }
        rng = np.random.default_rng(7)
        reqs = [random_request(rng, float(t)) for t in serving.poisson_arrivals(3000.0, 600, rng)]
        out = serving.serve_batched(ctx, templates, reqs, mem_budget=8 << 30)
        assert out["completed"] == len(reqs) and out["batches"] > 1
        alone = {name: tpl.make() for name, tpl in templates.items()}
        for r in reqs:
            assert r.done >= r.arrival and not isinstance(r.result, BaseException)
            same_query(r.result, alone[r.template].rebind(r.where).run())
        # A sample against the oracle, one request of each template.
        for name in ("scan", "fga", "join", "highcard"):
            r = next(x for x in reqs if x.template == name)
            if name == "join":
                e = oracle.aggregate(fact, FCT, tj.aggs, tj.group_by, r.where,
                                     build=(dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where), probe_key="fk")
            elif name == "highcard":
                e = oracle.aggregate(hc, None, hc_aggs, ("key",), r.where)
            else:
                tpl = ts if name == "scan" else tf
                e = oracle.aggregate(fact, FCT, tpl.aggs, tpl.group_by, r.where)
            same_query(r.result, e)
        j.drop()


STATEMENTS = [
    lambda rng: (f"SELECT SUM(price_cents * discount_pct), COUNT(*) FROM lineitem WHERE ship_day >= "
                 f"{D0 + int(rng.integers(0, 2000))} AND ship_day < {D0 + int(rng.integers(2000, ND))} AND "
                 f"discount_pct BETWEEN {int(rng.integers(0, 6))} AND {int(rng.integers(5, 11))} AND "
                 f"quantity < {int(rng.integers(2, 51))}"),
    lambda rng: (f"SELECT flag_a, flag_b, COUNT(*), SUM(quantity), SUM(price_cents), "
                 f"SUM(price_cents * (100 - discount_pct)), SUM(price_cents * (100 - discount_pct) * (100 + tax_pct)), "
                 f"AVG(quantity) FROM lineitem WHERE ship_day <= {D0 + int(rng.integers(3, ND))} "
                 f"GROUP BY flag_a, flag_b"),
    lambda rng: (f"SELECT segment, SUM(price_cents * (100 - discount_pct)), COUNT(*) FROM lineitem, dim "
                 f"WHERE fk = key AND order_day < {D0 + ND // 2} AND quantity < {int(rng.integers(2, 51))} "
                 f"GROUP BY segment"),
    lambda rng: "SELECT key, COUNT(*), SUM(value) FROM highcard GROUP BY key",
    lambda rng: (f"SELECT key, COUNT(*) FROM highcard WHERE value < {int(rng.integers(200, 1001))} "
                 f"GROUP BY key ORDER BY 2 DESC LIMIT 5"),
]


@pytest.mark.parametrize("batched", [True, False])
def test_wire_statements_match_alone(batched):
    from turbogp_b200 import frontend, pgwire
    fact = datagen.fact_fk(1_000_003, 20_000, 0.8, seed=71)
    dim = datagen.dimension(20_000, seed=72)
    hc = datagen.highcard(400_003, 50_000, 1.1, seed=73)
    with Context(0) as ctx, Context(0) as heavy:
        fe = frontend.Frontend(ctx, heavy)
        fe.register("lineitem", fact, FCT)
        fe.register("dim", dim, datagen.DIMENSION_COLTYPES)
        fe.register("highcard", hc, heavy=True)
        ex = frontend.BatchingExecutor(fe).start() if batched else frontend.PlainExecutor(fe).start()
        srv = pgwire.PgWireServer(ex).start()
        rng = np.random.default_rng(5)
        sqls = [STATEMENTS[int(rng.integers(0, len(STATEMENTS)))](rng) for _ in range(120)]
        got, errors = {}, []

        def client(k):
            try:
                c = pgwire.PgWireClient(*srv.address)
                for i in range(k, len(sqls), 6):
                    (names, rows, tag), = c.query(sqls[i])
                    got[i] = (names, rows, tag)
                c.close()
            except Exception as e:   # pragma: no cover - reported below
                errors.append(e)

        threads = [threading.Thread(target=client, args=(k,)) for k in range(6)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        srv.stop()
        ex.stop()
        assert not errors, errors
        # The same statements executed alone, directly on the engine.
        tables = {"lineitem": fe.tables["lineitem"][0], "highcard": fe.tables["highcard"][0]}
        for i, sql in enumerate(sqls):
            spec = sqlfront.parse(sql, fe.catalog)
            t = tables[spec.table]
            join = fe.joins[next(iter(fe.joins))] if spec.join else None
            if spec.order is not None:
                out = t.aggregate_topn(spec.aggs, spec.group_by, spec.where, spec.order[0], spec.order[1],
                                       spec.limit, join=join, probe_key="fk" if join else None)
            else:
                out = t.aggregate(spec.aggs, spec.group_by, spec.where, join=join,
                                  probe_key="fk" if join else None, group_cap=1 << 16)
            names, rows = sqlfront.format_rows(spec, out)
            assert got[i][0] == names and got[i][1] == rows, sql
            assert got[i][2] == f"SELECT {len(rows)}"
        fe.close()
