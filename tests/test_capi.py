"""The C-ABI libraries load and export every function include/harm_b200.h declares."""
import os
import re
import subprocess

from harm_harm_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "harm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(harm_\w+)\s*\(", src)))


def exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_every_declared_symbol_is_exported():
    syms = exported(os.path.join(N.LIBDIR, "libharm_b200.so")) | exported(os.path.join(N.LIBDIR, "libharm_host.so"))
    missing = [f for f in declared_functions() if f not in syms]
    assert not missing, missing


def test_libraries_load_and_bind():
    dev = N.device_lib()
    host = N.host_lib()
    for f in N.device_symbols():
        assert hasattr(dev, f)
    for f in N.host_symbols():
        assert hasattr(host, f)
    assert set(declared_functions()) <= set(N.device_symbols()) | set(N.host_symbols())


def test_grid_setup_matches_reference_rules():
    from harm_harm_b200 import Grid
    g = Grid.torus(192, 96, 64, lim=2).g
    # MAXBND 6 for WENO5, ihor = MAXBND, horizon 1/4 cell inside face ihor (setRin coord.c:2346)
    assert g.ng == 6
    import math
    x1h = g.startx[1] + (6 + 0.25) * g.dx[1]
    assert abs(math.exp(x1h) - g.Rhor) < 1e-12
    assert abs(math.exp(g.startx[1] + 192 * g.dx[1]) - 40.0) < 1e-12


def test_host_entry_points_reject_null_arguments():
    """The multi-step host-buffer step and the mixed reciprocal check their arguments before
    any CUDA call (so this runs without a GPU): a null context is an error (1) with its text."""
    import ctypes as C
    dev = N.device_lib()
    dt = C.c_double(1e-3)
    assert dev.harm_b200_step_host_n(None, 1, 0, None, 4, C.byref(dt), None) == 1
    assert b"null" in dev.harm_b200_last_error()
    assert dev.harm_b200_mixed_reciprocal(None, None, None, 8) == 1
    assert dt.value == 1e-3
