"""Generate the golden fixtures of the two-phase substep from the reference.

Runs the reference's own time-step code, compiled from its sources by
oracle/ref/Makefile into oracle/_ref/ref_<case>, on small seeded cases and
stores the inputs, parameters, solver iteration counts and the fields after
every RK substep in tests/golden/<name>.npz.

    python tests/golden/make_golden.py [--refsrc PATH]

This needs the reference source tree (REFSRC, default the mounted
reference); the fixtures it writes are committed so that the tests need
neither the tree nor the binaries.
"""
import argparse
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "parties-vof-ibm_b200"))
import pyoracle as po  # noqa: E402
from pvof import abi, cases  # noqa: E402

FLOW_FIELDS = {"C_L": "C_L", "C_G": "C_G", "rho": "RHO", "mu": "MU", "ch_rhs_n": "CH_RHS_N",
               "u": "U", "v": "V", "p": "P"}
NG_FIELDS = {"u_explicit_old": "U_EXPLICIT_OLD", "v_explicit_old": "V_EXPLICIT_OLD",
             "u_visc_explicit_old": "U_VISC_EXPLICIT_OLD", "v_visc_explicit_old": "V_VISC_EXPLICIT_OLD"}
ST_FLOW = {"psi_LG": "PSI_LG"}
ST_NG = {"f_sigma_old_x": "FSIG_OLD_X", "f_sigma_old_y": "FSIG_OLD_Y"}

TIGHT = dict(ch_tol=1e-13, ch_iter_max=600, CG_ETOL=1e-15, CG_MAXIT=400, P_CG_ETOL=1e-13, P_CG_MAXIT=1000)

# name, reference case, builder kwargs, steps, dt, snapshots kept (None = all)
CASES = [
    ("rt_small", "rt2d", dict(NXM=24, NYM=48, Lx=1.0, Ly=2.0, Cn=0.04, velocity_seed=5, velocity_amp=0.1), 2, 1e-3, None),
    ("rt_st_small", "rt2d_st", dict(NXM=24, NYM=48, Lx=1.0, Ly=2.0, Cn=0.04, surface_tension=True, We=100.0,
                                   velocity_seed=11, velocity_amp=0.1), 1, 1e-3, None),
    ("rt_tight", "rt2d", dict(NXM=24, NYM=48, Lx=1.0, Ly=2.0, Cn=0.04, velocity_seed=3, velocity_amp=0.1, **TIGHT),
     2, 1e-3, ["s0", "s1_0", "s1_2", "s2_2"]),
]

PARAM_KEYS = [k for k, _ in abi.Params._fields_]
GRID_KEYS = [k for k, _ in abi.GridDesc._fields_]


def struct_to_dict(s):
    out = {}
    for k, _ in s._fields_:
        v = getattr(s, k)
        out[k] = list(v) if hasattr(v, "__len__") else v
    return out


def parse_iterations(log):
    """Per-substep solver iteration counts from the reference's progress log."""
    ch = [int(m) for m in re.findall(r"VOF diffuse biharmonic \S+ to \S+ after (\d+) iterations", log)]
    u = [int(m) for m in re.findall(r"u-component of velocity converged to \S+ after (\d+) iterations", log)]
    v = [int(m) for m in re.findall(r"v-component of velocity converged to \S+ after (\d+) iterations", log)]
    p = [int(m) for m in re.findall(r"pressure converged to \S+ after (\d+) iterations", log)]
    return np.array([ch, u, v, p], dtype=np.int64)


def g_range(grid, plane, ng):
    """G-range part (NY, NX) of a k = 0 plane."""
    if ng:
        return plane
    NX, NY, _ = cases.dims(grid)
    G = cases.G
    return plane[G:G + NY, G:G + NX]


def make(name, refcase, kw, steps, dt, keep, outdir, refsrc=None):
    grid, params, planes = cases.rayleigh_taylor(**kw)
    if not os.path.exists(po.ref_binary(refcase)):
        po.build_reference(refcase, refsrc)
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference(refcase, wd, grid, params, planes, steps, dt, 1, substeps=True)
        data = {}
        st = bool(params.surface_tension)
        tags = ["s0"] + ["s%d_%d" % (n, rk) for n in range(1, steps + 1) for rk in range(3)]
        if keep is not None:
            tags = [t for t in tags if t in keep]
        for tag in tags:
            flow = dict(FLOW_FIELDS, **(ST_FLOW if st else {}))
            ngf = dict(NG_FIELDS, **(ST_NG if st else {}))
            for fname, pname in flow.items():
                a = po.read_reference_field(wd, tag, fname, grid)
                data["%s/%s" % (tag, pname)] = g_range(grid, a, False)
            for fname, pname in ngf.items():
                a = po.read_reference_field(wd, tag, fname, grid, ng=True)
                data["%s/%s" % (tag, pname)] = a
        data["iterations"] = parse_iterations(cp.stdout)
    for k, v in planes.items():
        data["init/" + k] = v
    meta = {"grid": struct_to_dict(grid), "params": struct_to_dict(params), "steps": steps, "dt": dt,
            "refcase": refcase, "builder": kw}
    data["meta"] = np.array(repr(meta))
    path = os.path.join(outdir, name + ".npz")
    np.savez_compressed(path, **data)
    return path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--refsrc", default=None)
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    for name, refcase, kw, steps, dt, keep in CASES:
        print(make(name, refcase, kw, steps, dt, keep, a.out, a.refsrc))


if __name__ == "__main__":
    main()
