import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "golden_small.npz"

# The projection tolerance: results within 1e-5 of the bounding-box diagonal.
TOL_DIAG = 1e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def golden_kernel(g, name):
    from mlodsurfaces_b200.apss import Kernel

    k = Kernel()
    k.type = int(g[f"k_{name}_type"])
    k.sigma = float(g[f"k_{name}_sigma"])
    k.exponent = float(g[f"k_{name}_exponent"])
    k.constant_shift = float(g[f"k_{name}_shift"])
    k.sigmas = [float(v) for v in g[f"k_{name}_sigmas"]]
    return k


def make_kernel(kind: str, diag: float):
    """The three kernel families of the benchmark configurations, sized by the
    bounding-box diagonal: single Gaussian (sigma 0.02 diag), multi-Gaussian
    (0.01 diag, factor 2, 4 sigmas) and rational (exponent 4, shift 1e-3)."""
    from mlodsurfaces_b200.apss import Kernel

    k = Kernel()
    if kind == "gauss":
        k.type = Kernel.GAUSSIAN
        k.sigma = 0.02 * diag
    elif kind == "multi":
        k.type = Kernel.GAUSSIAN_MULTIPLE
        k.sigmas = [0.01 * diag * 2.0**i for i in range(4)]
    elif kind == "singular":
        k.type = Kernel.SINGULAR
        k.exponent = 4.0
        k.constant_shift = 1e-3
    else:
        raise ValueError(kind)
    return k


def rel_err(a, b, diag):
    return np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64), axis=1) / diag
