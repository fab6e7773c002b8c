"""The wire front-end on the CPU: the SQL subset lowers to the same queries
as the benchmark templates (checked with the oracle), malformed statements
get the reference's SQLSTATEs, and the protocol server answers startup,
SSL negotiation, multi-statement simple queries, errors and concurrent
connections the way a PostgreSQL client expects."""
import socket
import struct
import threading

import pytest

import oracle
from turbogp_b200 import datagen, pgwire, sqlfront, workloads
from turbogp_b200.engine import build_col

CT = datagen.LINEITEM_COLTYPES
CATALOG = {
    "lineitem": sqlfront.TableInfo("lineitem", list(CT) + ["fk"], {**CT, "fk": "int"}),
    "dim": sqlfront.TableInfo("dim", ["key", "order_day", "segment"], datagen.DIMENSION_COLTYPES),
}
D0 = datagen.DAY0


def same(a, b):
    assert a.rows_selected == b.rows_selected and a.keys == b.keys
    for ra, rb in zip(a.values, b.values):
        assert [(x.value, x.count) for x in ra] == [(y.value, y.count) for y in rb]


def test_sql_lowers_to_the_benchmark_templates():
    fact = datagen.fact_fk(30_011, 3_000, 0.8, seed=3)
    dim = datagen.dimension(3_000, seed=2)
    fct = {**CT, "fk": "int"}
    scan = workloads.selective_scan_sum(day_lo=D0 + 730, days=365, disc_lo=5, disc_hi=7, qty_lt=24)
    fga = workloads.filtered_group_agg(ship_max=D0 + 2000)
    tj = workloads.join_group_agg()
    cases = [
        (f"SELECT SUM(price_cents * discount_pct), COUNT(*) FROM lineitem WHERE ship_day >= {D0 + 730} "
         f"AND ship_day < {D0 + 1095} AND discount_pct BETWEEN 5 AND 7 AND quantity < 24", scan, None),
        (f"select flag_a, flag_b, count(*), sum(quantity), sum(price_cents), sum(price_cents*(100-discount_pct)), "
         f"sum(price_cents*(100-discount_pct)*(100+tax_pct)), avg(quantity) from lineitem "
         f"where ship_day <= {D0 + 2000} group by flag_a, flag_b", fga, None),
        (f"SELECT dim.segment, SUM(price_cents * (100 - discount_pct)), COUNT(*) FROM lineitem, dim "
         f"WHERE lineitem.fk = dim.key AND dim.order_day < {D0 + datagen.NDAYS // 2} GROUP BY dim.segment", tj,
         (dim, datagen.DIMENSION_COLTYPES, "key", tj.build_where)),
    ]
    for sql, tpl, build in cases:
        spec = sqlfront.parse(sql, CATALOG)
        got = oracle.aggregate(fact, fct, spec.aggs, spec.group_by, spec.where,
                               build=(dim, datagen.DIMENSION_COLTYPES, spec.join[1], spec.join[3]) if spec.join
                               else None, probe_key=spec.join[2] if spec.join else None)
        exp = oracle.aggregate(fact, fct, tpl.aggs, tpl.group_by, tpl.where, build=build,
                               probe_key="fk" if build else None)
        same(got, exp)
    # Statements that differ only in probe-side literals share one shape.
    a = sqlfront.parse("SELECT COUNT(*) FROM lineitem WHERE quantity < 5", CATALOG)
    b = sqlfront.parse("SELECT COUNT(*) FROM lineitem WHERE quantity < 17", CATALOG)
    c = sqlfront.parse("SELECT COUNT(*) FROM lineitem WHERE quantity <= 17", CATALOG)
    assert a.shape == b.shape != c.shape


def test_sql_errors_carry_sqlstates():
    for sql, state in [("SELECT nope FROM lineitem", "42703"), ("SELECT COUNT(*) FROM missing", "42P01"),
                       ("SELECT COUNT(*) FROM lineitem WHERE", "42601"),
                       ("SELECT quantity, COUNT(*) FROM lineitem", "42803"),
                       ("SELECT COUNT(*) FROM lineitem WHERE quantity < 3 OR quantity > 5", "0A000"),
                       ("SELECT COUNT(*) FROM lineitem, dim", "0A000"),
                       ("SELECT flag_a FROM lineitem GROUP BY flag_a", "0A000")]:
        with pytest.raises(sqlfront.SqlError) as e:
            sqlfront.parse(sql, CATALOG)
        assert e.value.sqlstate == state, sql
    spec = sqlfront.parse("SELECT flag_a, COUNT(*) AS n FROM lineitem WHERE quantity NOT BETWEEN 3 AND 5 "
                          "GROUP BY flag_a ORDER BY 2 DESC LIMIT 2", CATALOG)
    assert spec.order == (0, True) and spec.limit == 2 and [i.name for i in spec.items] == ["flag_a", "n"]
    j = sqlfront.parse("SELECT segment, COUNT(*) FROM lineitem, dim WHERE fk = key GROUP BY segment", CATALOG)
    assert j.join[:3] == ("dim", "key", "fk") and j.group_by[0].side == build_col("segment").side


class FakeExecutor:
    def __init__(self):
        self.seen = []
        self.lock = threading.Lock()

    def execute(self, sql):
        with self.lock:
            self.seen.append(sql)
        if "bad" in sql:
            raise sqlfront.SqlError("42601", "syntax error at or near bad")
        if "boom" in sql:
            raise RuntimeError("device went away")
        n = int(sql.split()[-1]) if sql.split()[-1].isdigit() else 1
        return ["k", "total", "avg"], [(str(i), str(10 * i), repr(i / 3)) for i in range(n)]


@pytest.fixture
def server():
    ex = FakeExecutor()
    s = pgwire.PgWireServer(ex).start()
    yield s, ex
    s.stop()


def test_startup_queries_and_errors(server):
    s, ex = server
    c = pgwire.PgWireClient(*s.address)
    assert c.parameters["server_version"] == "15.0"
    res = c.query("SELECT 3; SELECT 0")
    assert [r[2] for r in res] == ["SELECT 3", "SELECT 0"]
    names, rows, _ = res[0]
    assert names == ["k", "total", "avg"] and rows == [("0", "0", "0.0"), ("1", "10", repr(1 / 3)),
                                                       ("2", "20", repr(2 / 3))]
    with pytest.raises(pgwire.PgError) as e:
        c.query("SELECT 1; bad; SELECT 2")
    assert e.value.sqlstate == "42601"
    assert ex.seen[-1] == "bad"                     # statements after an error are skipped
    with pytest.raises(pgwire.PgError) as e:
        c.query("boom")
    assert e.value.sqlstate == "XX000"
    assert c.query("SELECT 1")[0][2] == "SELECT 1"  # the connection survives errors
    c.close()


def test_ssl_request_is_declined_and_startup_continues(server):
    s, _ = server
    sock = socket.create_connection(s.address)
    sock.sendall(struct.pack("!ii", 8, pgwire.SSL_REQUEST))
    assert sock.recv(1) == b"N"
    body = struct.pack("!i", pgwire.PROTOCOL_V3) + b"user\x00u\x00\x00"
    sock.sendall(struct.pack("!i", len(body) + 4) + body)
    got = b""
    while not got.endswith(b"Z\x00\x00\x00\x05I"):
        got += sock.recv(4096)
    assert got.startswith(b"R\x00\x00\x00\x08\x00\x00\x00\x00")
    sock.close()


def test_concurrent_connections(server):
    s, ex = server
    errors = []

    def client(i):
        try:
            c = pgwire.PgWireClient(*s.address)
            for j in range(20):
                (names, rows, tag), = c.query(f"SELECT {i % 5}")
                assert len(rows) == i % 5 and tag == f"SELECT {i % 5}"
            c.close()
        except Exception as e:   # pragma: no cover - reported below
            errors.append(e)

    ts = [threading.Thread(target=client, args=(i,)) for i in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors and len(ex.seen) == 160 and s.connections == 8
