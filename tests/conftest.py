import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcardiotrust_cuda.so")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def cuboid8(oracle_mod):
    """8x8x8 cuboid, T=500, 37 triaxial sensors, 3^3 pathological block; truth measurements from the oracle."""
    from cardiotrust_b200 import scenario as sc

    scn = sc.build(sc.workload_spec("cuboid8"))
    return sc.attach_measurements(scn, oracle_forward(oracle_mod))


def oracle_forward(oracle_mod):
    def fwd(gains, osi, coefs, delays, H, ctrl, u):
        o = oracle_mod.OracleEpoch(gains, osi, coefs, delays, np.zeros_like(coefs), H, ctrl, u)
        return o.simulate()

    return fwd


def rel_err(a, b):
    """Norm-wise relative error ||a - b|| / ||b|| in float64."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def max_rel_err(a, b):
    """max |a - b| / max |b| in float64."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    mb = np.abs(b).max() if b.size else 0.0
    return float(np.abs(a - b).max() / (mb if mb > 0 else 1.0)) if a.size else 0.0
