import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


_CACHE = {}


def small_case(nxp=6, nlev=12, ntr=6, dtlm=1800.0, seed=11, w_amp=0.05, jet=35.0):
    """Grid + transport state small enough for the oracle to finish at once."""
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import transport_state
    key = (nxp, nlev, ntr, dtlm, seed, w_amp, jet)
    if key not in _CACHE:
        g = build_grid(nxp, stretched_levels(nlev, 100.0, 30000.0), seed=seed)
        st = transport_state(g, dtlm, ntr, seed=seed, w_amp=w_amp, jet_amp=jet)
        _CACHE[key] = (g, st)
    return _CACHE[key]


@pytest.fixture(scope="session")
def case_small():
    return small_case()


def relerr(a, b):
    """Normwise relative error max|a-b| / max|b| (0 when both are 0)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / den) if den > 0 else float(np.abs(a - b).max())
