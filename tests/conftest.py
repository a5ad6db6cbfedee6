import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
for path in (ROOT, ROOT / "sparse-dft_b200"):
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")
    config.addinivalue_line("markers", "slow: long CPU reference runs")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / f"{name}.npz"))
    return load


@pytest.fixture(scope="session")
def reference():
    from oracle import ref_oracle
    if not ref_oracle.available():
        pytest.skip("reference oracle library not built (make -C oracle/ref)")
    return ref_oracle.ReferenceLibrary()


@pytest.fixture(scope="session")
def tiny_inputs():
    from sdft_b200 import synthetic
    return synthetic.tiny()


@pytest.fixture(scope="session")
def si8_inputs():
    from sdft_b200 import synthetic
    return synthetic.si8()


@pytest.fixture(scope="session")
def context():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from sdft_b200.operator import Context
    ctx = Context(0)
    yield ctx
    ctx.close()


def probe_block(npw: int, columns: int, seed: int) -> np.ndarray:
    """Same seeded probe columns as tests/golden/make_golden.py."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.asfortranarray(rng.standard_normal((npw, columns)) + 1j * rng.standard_normal((npw, columns)))


def relative_error(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
