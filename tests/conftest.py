"""Shared test configuration.

Markers: `gpu` tests need a CUDA device and the built libkettle_b200.so; the
CPU suite (`-m "not gpu"`) covers the oracle, host logic and the C-ABI's
presence.  The oracle (oracle/) is the checker; the engine is what is tested.
"""
import json
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built engine library")


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import port as _port
    return _port()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import ref as _ref, ref_available
    if not ref_available():
        pytest.skip("reference library not built (oracle/_ref)")
    return _ref()


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN / "golden_ref.npz"))


@pytest.fixture(scope="session")
def kats():
    return json.loads((GOLDEN / "ref_kats.json").read_text())


@pytest.fixture(scope="session")
def engine():
    """The CUDA engine (skips only when no GPU is visible; a missing library is an error)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from kettle_b200 import capi
    capi.lib()
    return capi


def basis(n, index=0):
    v = np.zeros(1 << n, dtype=np.complex128)
    v[index] = 1.0
    return v


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)
