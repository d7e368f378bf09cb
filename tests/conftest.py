"""Shared fixtures.  `-m "not gpu"` runs everywhere; `-m gpu` needs a B200."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    out = {}
    for name in ("ties_q005", "box2", "small"):
        with np.load(GOLDEN / f"{name}.npz") as z:
            out[name] = {k: z[k] for k in z.files}
    return out


@pytest.fixture(scope="session")
def small_x(golden):
    from gmx_correlation_b200.synth import synth_traj
    g = golden["small"]
    x = synth_traj(int(g["natoms"]), int(g["nframes"]), int(g["n_modes"]), float(g["sigma_l"]),
                   seed=int(g["seed"]))
    return x


@pytest.fixture(scope="session")
def gc():
    import gmx_correlation_b200 as gc_mod
    gc_mod.lib()  # fails loudly when the CUDA library is missing
    return gc_mod
