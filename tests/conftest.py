"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and libketeb200.so; the rest
run on the CPU (oracle pins, host logic, C-ABI symbol checks)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built libketeb200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def spk_path(tmp_path_factory):
    from kete_b200 import synthetic

    p = tmp_path_factory.mktemp("spk") / "synthetic.bsp"
    synthetic.write_synthetic_spk(str(p))
    return str(p)


@pytest.fixture(scope="session")
def oracle_spk(oracle, spk_path):
    oracle.spk_reset()
    with open(spk_path, "rb") as f:
        oracle.spk_load_bytes(f.read())
    return oracle


@pytest.fixture(scope="session")
def gpu(spk_path):
    """The kete_b200 package with the synthetic SPK resident on the GPU."""
    import kete_b200
    from kete_b200 import build

    build.build()
    kete_b200.init(0)
    kete_b200.spice.kernel_reload([spk_path])
    return kete_b200


@pytest.fixture(scope="session")
def goldens():
    import json

    with open(os.path.join(ROOT, "tests", "golden", "reference_goldens.json")) as f:
        return json.load(f)


def rng(seed=0):
    return np.random.default_rng(seed)
