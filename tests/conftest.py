import ast
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "parties-vof-ibm_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    """(grid, params, planes, data, meta) of a golden fixture."""
    from pvof import abi
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = ast.literal_eval(str(d["meta"]))
    grid = abi.GridDesc()
    for k, v in meta["grid"].items():
        if isinstance(v, list):
            arr = getattr(grid, k)
            for q, x in enumerate(v):
                arr[q] = x
        else:
            setattr(grid, k, v)
    from pvof import cases
    params = cases.default_params()   # fields a fixture predates keep their defaults
    for k, v in meta["params"].items():
        if isinstance(v, list):
            arr = getattr(params, k)
            for q, x in enumerate(v):
                arr[q] = x
        else:
            setattr(params, k, v)
    planes = {k.split("/", 1)[1]: d[k] for k in d.files if k.startswith("init/")}
    return grid, params, planes, d, meta


def g_range(grid, plane, ng=False):
    """G-range part (NY, NX) of a k = 0 plane as returned by get()/get_field()."""
    from pvof import cases
    if ng:
        return plane
    NX, NY, _ = cases.dims(grid)
    G = cases.G
    return plane[G:G + NY, G:G + NX]


def physical(grid, a, field):
    """Cells each field owns in the reference (drops the aliased half cells):
    scalars i < NX-1, j < NY-1; u faces 1 <= i < NX (periodic) else < NX-1;
    v faces 1 <= j < NY-1."""
    from pvof import cases
    NX, NY, _ = cases.dims(grid)
    if field in ("U", "U_RHS", "U_EXPLICIT_OLD", "U_VISC_EXPLICIT_OLD", "FSIG_OLD_X"):
        i1 = NX if grid.periodic[0] else NX - 1
        return a[:NY - 1, 1:i1]
    if field in ("V", "V_RHS", "V_EXPLICIT_OLD", "V_VISC_EXPLICIT_OLD", "FSIG_OLD_Y"):
        j1 = NY if grid.periodic[1] else NY - 1
        return a[1:j1, :NX - 1]
    return a[:NY - 1, :NX - 1]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return d / nb if nb > 0 else d


@pytest.fixture(scope="session")
def gpu_available():
    from pvof import runtime
    return runtime.load().pvof_device_count() > 0
