import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and the built libavism_gpu.so")


@pytest.fixture(scope="session")
def gpu():
    from avism_b200.avism import AvismGPU
    ctx = AvismGPU(0)
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def mock1():
    """64^3 periodic mock (2^18 particles, 8 underdense spheres), reader units."""
    from avism_b200 import synth
    return synth.to_reader_units(synth.mock_spheres(seed=1001))


@pytest.fixture(scope="session")
def mock_small():
    """32^3 periodic mock with 2^15 particles for quick cases."""
    from avism_b200 import synth
    return synth.to_reader_units(synth.mock_spheres(n=2 ** 15, box=64.0, nsph=3, rmin=5.0,
                                                    rmax=9.0, seed=7))


@pytest.fixture(scope="session")
def oracle_mock1(mock1):
    from avism_b200._abi import Params
    from oracle import oracle as O
    out = {}
    for per in (1, 0):
        p = Params(nx=64, periodic=per, lado0=100.0)
        out[per] = O.run_level(p, mock1)
    return out


def pcopy(parts):
    return {k: np.array(v, copy=True) if isinstance(v, np.ndarray) else v for k, v in parts.items()}
