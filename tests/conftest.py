import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"
HA_EV = 27.21138505


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden_lih():
    return dict(np.load(GOLDEN / "lih_bulk08.npz"))


@pytest.fixture(scope="session")
def golden_synth():
    return dict(np.load(GOLDEN / "synth_small.npz"))


def instance_from_golden(d):
    """GWInstance view of a golden fixture (same Sigma grid as the fixture's oracle run)."""
    from molgw_b200.synth import GWInstance
    m_ia = d["m_ia"]
    return GWInstance(nocc=m_ia.shape[0], nvirt=m_ia.shape[1], naux=m_ia.shape[2], nomega=int(d["nomega"]),
                      energy=d["energy"], occupation=d["occupation"], m_ia=m_ia, m_sigma=d["m_sigma"],
                      nsemin=int(d["nsemin"]), nsemax=int(d["nsemax"]))


@pytest.fixture(scope="session")
def engine():
    """One library context on cuda:0 (GPU tests only)."""
    from molgw_b200 import build
    build.build()
    from molgw_b200.rigw import Engine
    eng = Engine(0)
    yield eng
    eng.close()
