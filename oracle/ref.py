"""TEST INFRASTRUCTURE ONLY: run the reference HARM binaries built by oracle/ref/build.sh.

The binaries in oracle/_ref/ are the reference code itself (its own sources, the torus
problem initboundcode/init.fishmon.c, the run configuration of oracle/ref/driver.c), so what
they write pins both the C restatement in oracle/*.c and the device path: the initial state
(init_dsandvels_torus init.fishmon.c:403 with the reference's ranc() perturbation), the
metric and connection tables (set_grid set_grid.c:114, set_connection set_grid.c:1033) and
the state after every full step (step_ch_full step_ch.c:35).

Imported by tests/ and bench.py's CPU-baseline leg only; never by the product package.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
BUILD = os.path.join(HERE, "ref", "build.sh")

# grid -> binary name; MAXBND is 4 for MC/PPM/PARALINE and 6 for WENO5 (the ghost width of
# the device grid, which also sets the inner radius through setihor, coord.c:2334)
LIM_NAMES = {0: "mc", 1: "para", 2: "weno5bnd", 3: "paraline"}
FLUX_NAMES = {0: "hll", 1: "laxf"}

# reference pflag positions [k][j][i] -> device order is the same for active cells

# metric locations of the device tables (CENT, FACE1, FACE2, CORN3) among the reference's
# eight (global.nondepnmemonics.h:1001-1008)
DEVICE_LOCS = (0, 1, 2, 6)


def binary(n1: int, n2: int, n3: int, ng: int) -> str:
    dim = "2d" if n3 == 1 else "3d"
    size = f"{n1}x{n2}" if n3 == 1 else f"{n1}x{n2}x{n3}"
    return os.path.join(REF_DIR, f"harm_ref_{dim}_{size}_b{ng}")


def available(n1: int, n2: int, n3: int, ng: int) -> bool:
    return os.access(binary(n1, n2, n3, ng), os.X_OK)


def build(*configs: str) -> None:
    r = subprocess.run(["bash", BUILD, *configs], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference build failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])


def _cache_dir() -> str:
    d = os.environ.get("HARM_REF_CACHE") or os.path.join(tempfile.gettempdir(), "harm_ref_cache")
    os.makedirs(d, exist_ok=True)
    return d


def _env(lim: int, flux: int, timeorder: int, cour: float, seed: int) -> dict:
    env = dict(os.environ)
    env.update(HREF_LIM=LIM_NAMES[lim], HREF_FLUX=FLUX_NAMES[flux], HREF_TIMEORDER=str(timeorder),
               HREF_COUR=repr(cour), HREF_SEED=str(seed))
    return env


def run(n1: int, n2: int, n3: int, ng: int, lim: int = 0, flux: int = 0, nsteps: int = 1, every: int = 1,
        timeorder: int = 2, cour: float = 0.8, seed: int = 12345, nthreads: int | None = None,
        substeps: tuple = ()) -> str:
    """Run the reference for `nsteps` full steps from its t=0 torus; returns the directory
    holding grid.npy, geom.npy, conn.npy, aux.npy, p0.npy, p_<s>.npy and steps.npy, and for the
    steps in `substeps` the inputs and outputs of every substep's advance(), fluxcalc() and
    post_fixup().  Runs are cached by their arguments (the binary's modification time
    included)."""
    exe = binary(n1, n2, n3, ng)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"reference binary {exe} not built (oracle/ref/build.sh)")
    subs = ",".join(str(int(x)) for x in substeps)
    key = f"{exe}:{os.path.getmtime(exe)}:{lim}:{flux}:{nsteps}:{every}:{timeorder}:{cour}:{seed}:{subs}"
    out = os.path.join(_cache_dir(), hashlib.sha1(key.encode()).hexdigest()[:16])
    if os.path.exists(os.path.join(out, "steps.npy")):
        return out
    os.makedirs(out, exist_ok=True)
    work = tempfile.mkdtemp(prefix="harm_ref_run_")
    # one thread: the reference's OpenMP build gives results that depend on the thread count
    # and vary from run to run in this configuration (a race); on one thread it is deterministic
    nthreads = nthreads or 1
    env = _env(lim, flux, timeorder, cour, seed)
    env["HREF_SUBSTEP_STEPS"] = subs
    r = subprocess.run([exe, "run", out, str(nthreads), str(nsteps), str(every)], cwd=work,
                       env=env, capture_output=True, text=True)
    if r.returncode != 0 or not os.path.exists(os.path.join(out, "steps.npy")):
        raise RuntimeError(f"reference run failed ({r.returncode}):\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
    subprocess.run(["rm", "-rf", work])
    return out


def points(n1: int, n2: int, n3: int, ng: int, ij: np.ndarray, U: np.ndarray, guess: np.ndarray) -> np.ndarray:
    """Utoprimgen (utoprimgen.c:32) of each record: U[n][8] (UEVOLVE) at CENT of cell
    (i, j) (active-cell indices), guess[n][8].  Returns [n][10]: P[8], pflag, Newton
    iterations."""
    exe = binary(n1, n2, n3, ng)
    rec = np.concatenate([np.asarray(ij, np.float64), np.asarray(U, np.float64), np.asarray(guess, np.float64)],
                         axis=1)
    assert rec.shape[1] == 18
    work = tempfile.mkdtemp(prefix="harm_ref_pts_")
    inp = os.path.join(work, "in.bin")
    np.ascontiguousarray(rec).tofile(inp)
    r = subprocess.run([exe, "points", work, "1", inp], cwd=work, env=_env(0, 0, 2, 0.8, 12345),
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference points failed ({r.returncode}):\n{r.stderr[-3000:]}")
    out = np.load(os.path.join(work, "points.npy"))
    subprocess.run(["rm", "-rf", work])
    return out


def fixup(n1: int, n2: int, n3: int, ng: int, P_ext: np.ndarray, flags: np.ndarray,
          finalstep: int = 1) -> tuple[np.ndarray, np.ndarray]:
    """post_fixup (fixup.c:53) of the reference on a given state: P_ext the extended state in
    the device layout [8][n3e][n2e][n1e] (ghost zones filled), flags the failure flag of each
    active cell [n3][n2][n1] (every ghost flag starts at 0), on the final substep or an
    earlier one.  Returns the extended state afterwards [8][n3e][n2e][n1e] and the extended
    flags afterwards [n3e][n2e][n1e]."""
    exe = binary(n1, n2, n3, ng)
    work = tempfile.mkdtemp(prefix="harm_ref_fix_")
    inp = os.path.join(work, "in.bin")
    aos = np.ascontiguousarray(np.moveaxis(np.asarray(P_ext, np.float64), 0, 3))
    with open(inp, "wb") as f:
        aos.tofile(f)
        np.ascontiguousarray(np.asarray(flags, np.float64)).tofile(f)
    r = subprocess.run([exe, "fixup", work, "1", inp, str(int(finalstep))], cwd=work, env=_env(0, 0, 2, 0.8, 12345),
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference fixup failed ({r.returncode}):\n{r.stderr[-3000:]}")
    out = np.ascontiguousarray(np.moveaxis(np.load(os.path.join(work, "post_fixout.npy")), 3, 0))
    fl = np.load(os.path.join(work, "post_fixflag.npy")).astype(np.int8)
    subprocess.run(["rm", "-rf", work])
    return out, fl


def time_steps(n1: int, n2: int, n3: int, ng: int, lim: int, flux: int, nsteps: int, nthreads: int,
               timeout: float | None = None) -> dict:
    """Wall time of `nsteps` full reference steps on `nthreads` OpenMP threads (after one
    untimed step); returns zone-cycles/s, seconds, steps, cells."""
    exe = binary(n1, n2, n3, ng)
    work = tempfile.mkdtemp(prefix="harm_ref_time_")
    r = subprocess.run([exe, "time", work, str(nthreads), str(nsteps)], cwd=work,
                       env=_env(lim, flux, 2, 0.8, 12345), capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference timing failed ({r.returncode}):\n{r.stderr[-3000:]}")
    v = np.load(os.path.join(work, "time.npy"))
    subprocess.run(["rm", "-rf", work])
    return {"zone_cycles_per_s": float(v[0]), "seconds": float(v[1]), "steps": int(v[2]), "cells": int(v[3])}


class RefRun:
    """The arrays of one reference run, converted to the device layout of a harm_grid:
    P[8][n3e][n2e][n1e] (active cells filled, ghosts zero), geom[4][28][n2e][n1e] at
    CENT/FACE1/FACE2/CORN3, conn[64][n2e][n1e], aux[3][n2e][n1e]."""

    def __init__(self, path: str, grid):
        self.path = path
        self.grid = grid
        g = grid.g
        self.info = np.load(os.path.join(path, "grid.npy"))
        n1, n2, n3, mb = (int(x) for x in self.info[:4])
        assert (n1, n2, n3) == (g.n1, g.n2, g.n3), "reference grid size differs"
        assert mb == g.ng, f"reference MAXBND {mb} != device ghost width {g.ng}"
        self.steps = np.load(os.path.join(path, "steps.npy"))
        self.dt0 = float(self.info[23])
        geom8 = np.load(os.path.join(path, "geom.npy"))
        self.geom8 = geom8
        self.geom = np.ascontiguousarray(geom8[list(DEVICE_LOCS)])
        self.conn = np.ascontiguousarray(np.load(os.path.join(path, "conn.npy")))
        self.aux = np.ascontiguousarray(np.load(os.path.join(path, "aux.npy")))

    def state(self, step: int) -> np.ndarray:
        name = "p0.npy" if step == 0 else f"p_{step}.npy"
        a = np.load(os.path.join(self.path, name))  # [k][j][i][pl]
        g = self.grid.g
        P = np.zeros((8, g.n3e, g.n2e, g.n1e))
        P[(slice(None),) + self.grid.active] = np.moveaxis(a, 3, 0)
        return P

    def sub(self, step: int, timeorder: int, what: str) -> np.ndarray:
        """A substep record of step `step` (1-based), substep `timeorder`: extended arrays
        (pi, pb, pf, F1..F3, fixin, fixout) as [8][n3e][n2e][n1e]; flags (pflag, fixflag) as
        int8 [n3e][n2e][n1e]; scalars (args: dt, fluxdt, timeorder, numtimeorders, CUf[4],
        Cunew[4], t, boundtime; ndt; ndtdir) as 1-D arrays."""
        a = np.load(os.path.join(self.path, f"sub_{step}_{timeorder}_{what}.npy"))
        if a.ndim == 4:
            return np.ascontiguousarray(np.moveaxis(a, 3, 0))
        if a.ndim == 3:
            return np.ascontiguousarray(a.astype(np.int8))
        return a

    def bound_calls(self, step: int):
        """The boundary calls of step `step` in call order: (direction, one_layer, input, output)
        with input/output as [8][n3e][n2e][n1e]; one_layer marks BOUNDPRIMSIMPLETYPE calls."""
        out, n = [], 0
        while os.path.exists(os.path.join(self.path, f"bnd_{step}_{n}_info.npy")):
            info = np.load(os.path.join(self.path, f"bnd_{step}_{n}_info.npy"))
            ld = lambda w: np.ascontiguousarray(np.moveaxis(np.load(os.path.join(self.path, f"bnd_{step}_{n}_{w}.npy")), 3, 0))
            out.append((int(info[0]), int(info[1]) != int(info[3]), ld("in"), ld("out")))
            n += 1
        return out

    def dt_of_step(self, step: int) -> float:
        """dt the reference used for step `step` (1-based)"""
        return float(self.steps[step, 1])
