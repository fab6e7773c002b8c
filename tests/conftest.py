import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100a) device")
    # Temporary files (tmp_path) stay inside the repository checkout.
    if config.option.basetemp is None:
        config.option.basetemp = str(ROOT / ".pytest_tmp")


@pytest.fixture(scope="session")
def kats():
    return json.loads((ROOT / "tests" / "golden" / "reference_kats.json").read_text())


def gen_column(spec: dict, dtype: str) -> np.ndarray:
    """Materialises a generator spec of reference_kats.json."""
    npdt = {"u64": np.uint64, "i64": np.int64, "i32": np.int32, "f64": np.float64, "u8": np.uint8}[dtype]
    (kind, arg), = spec.items()
    if kind == "list":
        return np.array(arg, dtype=npdt)
    if kind == "range":
        return np.arange(arg[0], arg[1]).astype(npdt)
    if kind == "mod":
        return (np.arange(arg[0]) % arg[1]).astype(npdt)
    if kind == "rep":
        return np.full(arg[1], arg[0], dtype=npdt)
    if kind == "f64_scaled":
        return (np.arange(arg[0], dtype=np.float64) * arg[1]).astype(npdt)
    if kind == "i32_mix":
        return (((np.arange(arg[0], dtype=np.int64) * 7) % 51) - 25).astype(npdt)
    if kind == "scaled":
        return (np.arange(arg[0]) * arg[1]).astype(npdt)
    raise ValueError(spec)


@pytest.fixture(scope="session")
def ctx():
    from turbogp_b200.engine import Context
    c = Context(0)
    yield c
    c.close()
