"""The bounded-wait failure path on the GPU, without a fault: a scan whose
stage copy of one tile is never issued (the one-shot test hook) has its
consumers' bounded wait run out after 2 ms; the call returns TGP_TIMEOUT, and
the next queries on the same context — the same one included — are exact
against the oracle. The hook applies to one launch only."""
import pytest

import oracle
from turbogp_b200 import _capi as A
from turbogp_b200 import datagen, workloads

pytestmark = pytest.mark.gpu

CT = datagen.LINEITEM_COLTYPES


@pytest.mark.parametrize("tile", [0, 5])
def test_timeout_is_reported_and_the_context_stays_usable(ctx, tile):
    host = datagen.lineitem(2_000_003, seed=91)
    t = ctx.register(host, CT)
    for tpl in (workloads.selective_scan_sum(), workloads.filtered_group_agg()):
        expect = oracle.aggregate(host, CT, tpl.aggs, tpl.group_by, tpl.where)
        ctx.fail_next_scan(tile=tile, wait_ns=2_000_000)
        with pytest.raises(A.TgpError) as e:
            t.aggregate(tpl.aggs, tpl.group_by, tpl.where)
        assert e.value.status == A.TIMEOUT
        for _ in range(2):
            got = t.aggregate(tpl.aggs, tpl.group_by, tpl.where)
            assert got.rows_selected == expect.rows_selected and got.keys == expect.keys
            assert [[(v.value, v.count) for v in r] for r in got.values] == \
                   [[(v.value, v.count) for v in r] for r in expect.values]
    t.drop()
