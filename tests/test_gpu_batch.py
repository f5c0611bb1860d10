"""Batched form: independent cases advanced concurrently by
pvof_run_steps_batched (one host thread and stream per case) give the same
fields, bit for bit, as the same cases advanced one at a time -- every
kernel, reduction order included, is independent of what else runs on the
GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(32, 128), (48, 96), (24, 48), (64, 128)]
FIELDS = ["C_L", "U", "V", "P", "RHO"]


def make(NXM, NYM, seed):
    from pvof import cases, runtime
    grid, params, planes = cases.rayleigh_taylor(NXM, NYM, Lx=1.0, Ly=NYM / NXM,
                                                 Cn=0.04, velocity_seed=seed, velocity_amp=0.05, P_CG_MAXIT=2000)
    s = runtime.Solver(grid, params, device=0)
    s.set_planes(planes)
    s.initialize()
    return s


def test_batched_run_equals_one_at_a_time():
    from pvof import runtime
    alone = [make(nx, ny, q) for q, (nx, ny) in enumerate(SIZES)]
    for s in alone:
        s.run_steps(2, 1e-3)
    batch = [make(nx, ny, q) for q, (nx, ny) in enumerate(SIZES)]
    stats = runtime.run_steps_batched(batch, 2, 1e-3)
    assert len(stats) == len(SIZES)
    for a, b in zip(alone, batch):
        for f in FIELDS:
            assert np.array_equal(a.get(f), b.get(f)), f


def test_batched_run_reports_the_failing_case():
    from pvof import runtime
    ok = make(32, 64, 1)
    bad = make(32, 64, 2)
    with pytest.raises(runtime.PvofError):
        runtime.run_steps_batched([ok, bad, ok], 1, 1e-3)     # the same context twice
