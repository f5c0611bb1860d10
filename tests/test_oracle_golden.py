"""The CPU restatement (oracle/pvof_oracle.c) against the reference's own
time step, compiled from its sources (golden fixtures, tests/golden).

The restatement keeps the reference's index ranges and operation order, so
every field must match bit for bit after every RK substep, with the same
solver iteration counts."""
import numpy as np
import pytest

from conftest import g_range, load_golden

FIELDS = ["C_L", "C_G", "RHO", "MU", "CH_RHS_N", "U", "V", "P"]
NG_FIELDS = ["U_EXPLICIT_OLD", "V_EXPLICIT_OLD", "U_VISC_EXPLICIT_OLD", "V_VISC_EXPLICIT_OLD"]


def run_case(name):
    import pyoracle as po
    grid, params, planes, d, meta = load_golden(name)
    o = po.Oracle(grid, params)
    o.set_planes(planes)
    o.initialize()
    snaps = {"s0": {}}
    iters = [[], [], [], []]
    fields = FIELDS + (["PSI_LG"] if params.surface_tension else [])
    ngf = NG_FIELDS + (["FSIG_OLD_X", "FSIG_OLD_Y"] if params.surface_tension else [])

    def take(tag):
        for f in fields:
            snaps.setdefault(tag, {})[f] = g_range(grid, o.get_field(f))
        for f in ngf:
            snaps.setdefault(tag, {})[f] = o.get_field(f)

    take("s0")
    dt = meta["dt"]
    for n in range(1, meta["steps"] + 1):
        for rk in range(3):
            if n > 1 and rk == 0:
                o.routine("CELL_CENTER")
            o.set_stage(rk, dt)
            rc, st = o.substep()
            assert rc == 0
            iters[0].append(st.ch_iters)
            iters[1].append(st.u_iters)
            iters[2].append(st.v_iters)
            iters[3].append(st.p_iters)
            take("s%d_%d" % (n, rk))
    return d, snaps, np.array(iters)


@pytest.mark.parametrize("name", ["rt_small", "rt_st_small", "rt_tight", "rt_fs_tight", "axi_small", "axi_tight",
                                  "axi_st_tight"])
def test_oracle_matches_reference_bitwise(name):
    d, snaps, iters = run_case(name)
    assert np.array_equal(iters, d["iterations"]), (iters, d["iterations"])
    checked = 0
    for key in d.files:
        if "/" not in key or key.startswith("init/"):
            continue
        tag, field = key.split("/")
        ref = d[key]
        mine = snaps[tag][field]
        assert mine.shape == ref.shape, (key, mine.shape, ref.shape)
        assert np.array_equal(mine, ref), "%s differs (max %.3e)" % (key, np.abs(mine - ref).max())
        checked += 1
    assert checked > 40
