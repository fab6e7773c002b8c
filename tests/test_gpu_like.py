"""LIKE on the GPU (tgp_like) against the oracle's restatement of the
reference's like(): the reference's own contains / prefix known answers,
random URL-like strings with prefix / suffix / contains / '_' / inner '%'
patterns, NOT LIKE, empty strings and patterns, the literal-'%' quirk,
sizes around warp multiples, and strings longer than a warp's staging buffer
(the unstaged path)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

WORDS = ["google", "yahoo", "bing", "shop", "game", "page_1", "page%2", "maps", "search", "a", "b", "_", "%"]


def random_strings(n, rng, long_every=0):
    out = []
    for i in range(n):
        k = int(rng.integers(0, 6))
        parts = [WORDS[int(j)] for j in rng.integers(0, len(WORDS), k)]
        s = ("https://" if rng.random() < 0.5 else "http://") + "/".join(parts) if rng.random() < 0.9 else \
            "".join(parts)
        if long_every and i % long_every == 0:
            s = s + "x" * int(rng.integers(4000, 9000)) + "google"
        out.append(s)
    return out


PATTERNS = ["%google%", "https://%", "%maps", "%page_1%", "%page%2%", "h_tp%", "%", "", "_", "%g%e%", "http://", "a%",
            "%_%", "%%google%%", "%yahoo%shop%", "%a%b%c%", "x%"]


def test_reference_known_answers(ctx, kats):
    for k in kats["like"]:
        col = ctx.register_strings(k["strings"])
        got = col.like(k["pattern"])
        exp = oracle.like(k["strings"], k["pattern"])
        assert got.count == exp.count and np.array_equal(got.bitmap, exp.bitmap), k["source"]
        col.drop()


@pytest.mark.parametrize("n, long_every", [(0, 0), (1, 0), (31, 0), (32, 0), (33, 0), (1000, 0), (100_003, 0),
                                           (5_000, 97)])
def test_like_matches_the_oracle(ctx, n, long_every):
    rng = np.random.default_rng(n + long_every)
    strings = random_strings(n, rng, long_every)
    flat = oracle.flat_strings(strings)
    col = ctx.register_strings(flat)
    for p in PATTERNS:
        for neg in (False, True):
            got = col.like(p, negated=neg)
            exp = oracle.like(flat, p, negated=neg)
            assert got.count == exp.count, (p, neg)
            assert np.array_equal(got.bitmap, exp.bitmap), (p, neg)
    col.drop()


def test_bad_offsets_are_refused(ctx):
    from turbogp_b200 import _capi as A
    data = np.frombuffer(b"abcdef", dtype=np.uint8)
    for offs in ([0, 4, 2, 6], [1, 3, 6], [0, 3, 7]):
        with pytest.raises(A.TgpError):
            ctx.register_strings((data, np.array(offs, dtype=np.uint64)))
