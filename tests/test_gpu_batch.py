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


def test_contexts_of_any_size_order_run():
    """The cluster solvers' shared-memory limit is a property of the kernel
    shared by every context of the process: a large context created before a
    small one still launches (the limit only grows)."""
    big = make(96, 192, 1)
    small = make(24, 48, 2)
    big.run_steps(1, 1e-3)
    small.run_steps(1, 1e-3)
    big.close()
    small.close()


def test_droplet_batch_equals_one_at_a_time():
    """Four sessile-droplet cases of the batching form (static cylinder,
    surface tension, FP32 stencils, particle bookkeeping on the device) for
    eight steps -- a substep is captured the second time its launches recur
    (stage, surface-tension buffer parity, warm start), so the last steps
    replay from CUDA graphs -- advanced together by pvof_run_steps_batched:
    bit for bit the fields of each case advanced alone."""
    from pvof import cases, runtime
    batch = cases.droplet_batch(4, seed=7, nxm_min=32, nxm_max=64, P_CG_MAXIT=4000, stencil_fp32=1,
                                pressure_warm_start=1)

    def start(case):
        g, p, pl, parts = case
        s = runtime.Solver(g, p, device=0)
        s.set_particles(parts)
        s.set_planes(dict(pl, C_L=pl["F"]))
        s.initialize()
        return s

    alone = [start(c) for c in batch]
    for s in alone:
        s.run_steps(8, 1e-4)
    together = [start(c) for c in batch]
    runtime.run_steps_batched(together, 8, 1e-4)
    for a, b in zip(alone, together):
        for f in FIELDS:
            assert np.array_equal(a.get(f), b.get(f)), f
        assert np.array_equal(a.get_particles()["F"], b.get_particles()["F"])
        assert b.graph_replays() > 0
    for s in alone + together:
        s.close()
