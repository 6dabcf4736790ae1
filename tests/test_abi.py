"""C-ABI checks that need no GPU: the library loads, exports every entry point the
header declares, and the ctypes mirror of every struct matches the C layout."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from conftest import fem, ROOT

abi = fem._abi
HEADER = os.path.join(ROOT, "include", "femtools_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(femb200_\w+)\s*\(", text, re.M)))


def test_header_declares_the_mirrored_entry_points():
    assert declared_functions() == sorted(abi.SIGNATURES)


def test_library_loads_and_exports_every_symbol():
    lib = abi.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.femb200_version()


def test_build_targets_sm_100a_only():
    import importlib.util
    spec = importlib.util.spec_from_file_location("femb_build", os.path.join(ROOT, "femtools.jl_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    assert "arch=compute_100a,code=sm_100a" in b.FLAGS


STRUCTS = {
    "femb200_stokes_material": abi.StokesMaterialC,
    "femb200_stokes_problem": abi.StokesProblemC,
    "femb200_stokes_controls": abi.StokesControlsC,
    "femb200_stokes_stats": abi.StokesStatsC,
    "femb200_thermal_problem": abi.ThermalProblemC,
    "femb200_thermal_controls": abi.ThermalControlsC,
    "femb200_thermal_stats": abi.ThermalStatsC,
    "femb200_lithostatic_problem": abi.LithostaticProblemC,
    "femb200_lithostatic_controls": abi.LithostaticControlsC,
    "femb200_cell_pressure_problem": abi.CellPressureProblemC,
    "femb200_cell_pressure_controls": abi.CellPressureControlsC,
    "femb200_cell_pressure_stats": abi.CellPressureStatsC,
    "femb200_cap_problem": abi.CapProblemC,
}


def test_struct_layouts_match_the_header():
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"femtools_b200.h\"\nint main(void){\n"
    for cname in STRUCTS:
        src += f'printf("{cname} %zu\\n", sizeof({cname}));\n'
    src += 'printf("off_mat %zu\\n", offsetof(femb200_stokes_problem, mat));\n'
    src += 'printf("off_bc %zu\\n", offsetof(femb200_stokes_problem, bc_n));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        exe = os.path.join(d, "s")
        open(c, "w").write(src)
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        out = subprocess.check_output([exe], text=True).split("\n")
    sizes = dict(line.split() for line in out if line)
    for cname, py in STRUCTS.items():
        assert int(sizes[cname]) == ctypes.sizeof(py), cname
    assert int(sizes["off_mat"]) == abi.StokesProblemC.mat.offset
    assert int(sizes["off_bc"]) == abi.StokesProblemC.bc_n.offset


def test_product_path_has_no_cpu_fallback(monkeypatch):
    # Without a CUDA device the solver refuses to run instead of computing on the host.
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    mesh = fem.structured_mixed_mesh(3, (1, 1, 1))
    with pytest.raises(RuntimeError, match="CUDA device"):
        fem.StokesDR(mesh, fem.StokesMaterial(g=(0.0, 0.0, -1.0)))
