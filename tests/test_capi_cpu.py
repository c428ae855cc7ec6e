"""The C-ABI library loads without a GPU and exports every function that
include/lattice_lbm.h declares; no compute entry point is called here."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lattice_lbm.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    names = set(re.findall(r"\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src))
    return sorted(n for n in names if n.startswith("LBM_") or n == "writeVTI")


def test_header_declares_reference_api():
    names = declared_functions()
    # the 14 functions of simulation/lib/lbm.h:59-129
    reference = ["LBM_Create", "LBM_Free", "LBM_SetSolidAABB", "LBM_InitializeFlow",
                 "LBM_Step", "LBM_GetVelocityBuffer", "LBM_ComputeDragForce",
                 "LBM_ComputeDragForceDecomposed", "LBM_ComputeDragCoefficient",
                 "LBM_ComputeLiftCoefficient", "LBM_SetSolidSphere", "LBM_AddGroundPlane",
                 "LBM_ComputeProjectedArea", "LBM_SetSolidMesh"]
    for r in reference + ["writeVTI"]:
        assert r in names, r


def test_library_exports_every_declared_symbol(solver):
    from lattice_fluid_dynamics_b200 import capi
    lib = ctypes.CDLL(capi.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
    # the ctypes table binds every declared function, nothing else
    assert sorted(capi.SIGNATURES) == declared_functions()


def test_exports_are_plain_c(solver):
    from lattice_fluid_dynamics_b200 import capi
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for name in declared_functions():
        assert name in exported, name


def test_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "lattice_lbm.h"\n'
                   "int main(void) { LBMGrid g; g.useMRT = 1; g.periodicYZ = 1;"
                   " return g.useMRT - 1; }\n")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-c", str(src), "-o", str(tmp_path / "t.o")], check=True)


def test_error_strings(solver):
    from lattice_fluid_dynamics_b200 import capi
    lib = capi.load()
    assert lib.LBM_GetErrorString(0) == b"ok"
    assert lib.LBM_GetErrorString(2) == b"out of device memory"
    assert lib.LBM_GetLastError(None) != 0


def test_create_rejects_bad_sizes_before_any_device_call(solver):
    # lbm.c:46-60 returns NULL on failure; sizes are checked on the host
    # before any allocation: non-positive extents, more than 2^31 - 1 cells,
    # an unknown storage format.  Freeing NULL is allowed (lbm.c:320-344).
    from lattice_fluid_dynamics_b200 import capi
    lib = capi.load()
    for dims in [(0, 8, 8), (8, -1, 8), (8, 8, 0), (2048, 2048, 1024), (65536, 65536, 1)]:
        assert not lib.LBM_CreateEx(*dims, 0.1, 0)
        assert not lib.LBM_Create(*dims, 0.1)
    assert not lib.LBM_CreateEx(8, 8, 8, 0.1, 99)
    lib.LBM_Free(None)
