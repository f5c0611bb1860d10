"""The C ABI boundary: the CUDA library loads on a machine without a GPU,
exports every entry point include/pvof.h declares, and the Python mirror of
the structures matches the C layout.  No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "pvof.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^[a-z][\w\s\*]*?\b(pvof_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from pvof import abi, runtime
    L = runtime.load()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(abi.EXPORTS) <= set(names)
    assert L.pvof_abi_version() == abi.ABI_VERSION


def test_field_enum_matches_header():
    from pvof import abi
    text = open(HEADER).read()
    body = text[text.index("enum pvof_field {"):]
    body = body[:body.index("};")]
    names = re.findall(r"PVOF_F_(\w+)", body)
    assert names[-1] == "COUNT"
    assert names[:-1] == abi.FIELD_NAMES


def test_struct_layout_matches_c(tmp_path):
    from pvof import abi
    src = tmp_path / "probe.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "pvof.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(pvof_grid_desc), sizeof(pvof_params),"
        " sizeof(pvof_stats), offsetof(pvof_grid_desc, slab_thickness), offsetof(pvof_params, P_CG_ETOL),"
        " offsetof(pvof_stats, clamp_mass)); return 0;}\n")
    exe = tmp_path / "probe"
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    got = [int(x) for x in out]
    want = [C.sizeof(abi.GridDesc), C.sizeof(abi.Params), C.sizeof(abi.Stats),
            abi.GridDesc.slab_thickness.offset, abi.Params.P_CG_ETOL.offset, abi.Stats.clamp_mass.offset]
    assert got == want


def test_no_device_is_an_error_not_a_fallback():
    """Without a CUDA device the library refuses to create a context."""
    from pvof import cases, runtime
    L = runtime.load()
    if L.pvof_device_count() > 0:
        pytest.skip("a CUDA device is present")
    grid, params, _ = cases.rayleigh_taylor(16, 32, Ly=2.0, Cn=0.05)
    with pytest.raises(runtime.PvofError):
        runtime.Solver(grid, params)


def test_invalid_arguments_rejected():
    from pvof import abi, runtime
    L = runtime.load()
    h = C.c_void_p()
    g = abi.GridDesc()
    p = abi.Params()
    g.ghost_nodes = 2
    assert L.pvof_create(C.byref(g), C.byref(p), 0, C.byref(h)) == abi.EINVAL
    assert L.pvof_create(None, None, 0, None) == abi.EINVAL
    assert L.pvof_set_stage(None, 0, 1e-3) == abi.EINVAL
    assert L.pvof_substep(None, None) == abi.EINVAL


def test_oracle_library_loads():
    import pyoracle as po
    L = po.lib()
    assert hasattr(L, "orc_substep")
