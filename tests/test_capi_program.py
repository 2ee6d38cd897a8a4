"""A C program compiled against include/harm_b200.h alone (tests/capi/harm_step_ch.c): HARM's
[k][j][i][pl] arrays converted at the boundary, fluxcalc for the initial dt, the two RK2
substeps of step_ch_simplempi through advance / bound_prim / post_fixup, the flags into
HARM's int pflag[cell][NUMPFLAGS], and the same step through the host-buffer entry point over
a host array in HARM's layout, which must agree bit for bit.  Built here with gcc and linked
with the in-tree libraries and the CUDA runtime; run on a GPU."""
import os
import subprocess
import tempfile

import pytest

from harm_harm_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "capi", "harm_step_ch.c")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(out_dir: str) -> str:
    exe = os.path.join(out_dir, "harm_step_ch")
    lib = N.LIBDIR
    cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), SRC, "-o", exe, "-L", lib, "-lharm_b200", "-lharm_host",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{lib}",
           f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_c_caller_compiles_against_the_header():
    with tempfile.TemporaryDirectory() as d:
        assert os.access(build(d), os.X_OK)


@pytest.mark.gpu
def test_c_caller_runs_the_step_sequence(cuda):
    with tempfile.TemporaryDirectory() as d:
        exe = build(d)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.startswith("OK"), r.stdout
