"""The stencil tile autotuner (pvof_set_autotune): it samples every
cell-wise stencil kernel over its candidate tiles during the next substeps,
keeps the fastest, and changes no result -- the fields after eight steps are
bit for bit those of the default tile, in the FP64 and the FP32 stencil
forms, and the substeps go back to CUDA graph replay once it is done."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["C_L", "U", "V", "P", "RHO", "PSI_LG"]
TILES = {"32x8", "64x4", "128x2", "256x1", "32x4", "64x8"}


@pytest.mark.parametrize("fp32", [0, 1])
def test_autotuned_tiles_change_no_result(fp32):
    from pvof import cases, runtime
    out = []
    for tune in (False, True):
        grid, params, planes = cases.rayleigh_taylor(96, 192, Lx=1.0, Ly=2.0, Cn=0.02, surface_tension=True,
                                                     We=100.0, velocity_seed=4, velocity_amp=0.05,
                                                     P_CG_MAXIT=4000, stencil_fp32=fp32)
        s = runtime.Solver(grid, params, device=0)
        s.set_planes(planes)
        s.initialize()
        if tune:
            s.set_autotune(True)
        s.run_steps(8, 1e-4)
        out.append(({f: s.get(f) for f in FIELDS}, s.autotune_active(), s.autotune_report(), s.graph_replays()))
        s.close()
    (a, _, _, _), (b, active, report, replays) = out
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f
    assert not active
    assert len(report) >= 10 and all(r["decided"] for r in report)
    assert all(r["tile"] in TILES for r in report)
    assert any(("_f" in r["kernel"]) == bool(fp32) for r in report)
    for r in report:
        print("%-16s %-6s best %.2f us, default %.2f us" % (r["kernel"], r["tile"], r["best_us"], r["default_us"]))
    assert replays > 0
