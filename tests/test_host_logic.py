"""Host-side helpers shared by host and device code, checked on the CPU."""
import subprocess
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_i128_to_f64_rounds_like_the_compiler(tmp_path):
    """i128_to_f64_rn (used by the device result formatter) equals the
    compiler's correctly rounded __int128 -> double on edge and random values."""
    src = tmp_path / "t.cpp"
    src.write_text(textwrap.dedent(r"""
        #include <cstdio>
        #include <cstdint>
        #include <random>
        #include "plan.hpp"
        int main() {
            std::mt19937_64 g(7);
            long bad = 0, n = 0;
            auto check = [&](__int128 v) {
                const uint64_t lo = static_cast<uint64_t>(v);
                const int64_t hi = static_cast<int64_t>(v >> 64);
                const double a = tgp::i128_to_f64_rn(lo, hi), b = static_cast<double>(v);
                ++n;
                if (a != b) { ++bad; if (bad < 5) std::printf("mismatch %.17g %.17g\n", a, b); }
            };
            const __int128 one = 1;
            for (int s = 0; s < 127; ++s) {
                for (int d = -3; d <= 3; ++d) { check((one << s) + d); check(-((one << s) + d)); }
                check((one << s) + (one << (s > 54 ? s - 53 : 0)));      // ties
                check((one << s) + 3 * (one << (s > 55 ? s - 54 : 0)));
            }
            for (int i = 0; i < 200000; ++i) {
                __int128 v = (static_cast<__int128>(static_cast<int64_t>(g())) << 64) | g();
                v >>= (g() % 127);
                check(v);
            }
            std::printf("%ld %ld\n", n, bad);
            return bad != 0;
        }
    """))
    exe = tmp_path / "t"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'turbogp_b200' / 'csrc'}", str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout


def test_tuning_cache_round_trip(tmp_path):
    """The autotuner's JSON cache keeps every entry and rejects unknown
    fields and versions."""
    import json
    from turbogp_b200.engine import VARIANT_FIELDS, load_tuning_file, save_tuning_file
    entries = {(3 << 24) | (26 << 16) | 0x45: {f: i for i, f in enumerate(VARIANT_FIELDS)},
               7: {f: 1 for f in VARIANT_FIELDS}}
    p = tmp_path / "t.json"
    save_tuning_file(p, entries)
    assert load_tuning_file(p) == entries
    doc = json.loads(p.read_text())
    assert [e["class"] for e in doc["entries"]] == sorted(entries)
    doc["entries"][0]["variant"]["bogus"] = 1
    p.write_text(json.dumps(doc))
    with pytest.raises(ValueError):
        load_tuning_file(p)
    p.write_text(json.dumps({"version": 9, "entries": []}))
    with pytest.raises(ValueError):
        load_tuning_file(p)
