"""Generate the golden fixtures of this directory from the reference HARM code itself.

Needs the reference binaries of oracle/_ref/ (built from the reference's sources by
oracle/ref/build.sh, which runs where the reference tree is present).  Run from the
repository root:

    python tests/golden/make_golden.py

Writes
  ref_2d_mc_32x32.npz   the 2-D torus (32 x 32, MC, HLL, Toth CT, RK2 midpoint, Courant 0.8):
                        the reference's metric, connection and floor tables
                        (set_grid set_grid.c:114, set_connection set_grid.c:1033), its t=0
                        state (init.fishmon.c:403, ranc seed 12345) and, for both substeps of
                        the first full step, the bounded input of advance() (advance.c:85),
                        its fluxes after flux-CT (fluxcalc flux.c:38), its output primitives,
                        inversion flags and ndt, and the state after the step.
  ref_utoprimgen_points.npz
                        Utoprimgen (utoprimgen.c:32) of conserved states built from the torus
                        cells -- physical ones from a perturbed guess, and ones the hot
                        inversion cannot invert (momentum beyond the light cone, negative or
                        tiny density, negative or excessive energy, NaN) -- with the primitives,
                        failure codes and Newton iteration counts the reference returns.
Arrays are in the device layout: P[8][n3e][n2e][n1e] (active cells of a 'pf' record only),
geom[4][28][n2e][n1e] at CENT/FACE1/FACE2/CORN3, conn[64][n2e][n1e], aux[3][n2e][n1e].
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from harm_harm_b200 import Grid  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import ref as R  # noqa: E402


def torus_fixture() -> None:
    n1, n2, n3, ng = 32, 32, 1, 4
    path = R.run(n1, n2, n3, ng, lim=0, flux=0, nsteps=1, every=1, substeps=(1,))
    g = Grid.torus(n1, n2, n3, lim=0)
    rr = R.RefRun(path, g)
    act = (slice(None),) + g.active
    gg = g.g
    out = dict(grid=rr.info, geom=rr.geom, conn=rr.conn, aux=rr.aux, p0=rr.state(0)[act], p1=rr.state(1)[act],
               steps=rr.steps)
    for to in (0, 1):
        out[f"s{to}_pb"] = rr.sub(1, to, "pb")
        out[f"s{to}_pf"] = rr.sub(1, to, "pf")[act]
        out[f"s{to}_pflag"] = rr.sub(1, to, "pflag")[g.active]
        out[f"s{to}_args"] = rr.sub(1, to, "args")
        out[f"s{to}_ndt"] = rr.sub(1, to, "ndt")
        out[f"s{to}_ndtdir"] = rr.sub(1, to, "ndtdir")
        for d in (1, 2):
            F = rr.sub(1, to, f"F{d}")
            k = slice(gg.ng3, gg.ng3 + gg.n3)
            j = slice(gg.ng, gg.ng + gg.n2 + (1 if d == 2 else 0))
            i = slice(gg.ng, gg.ng + gg.n1 + (1 if d == 1 else 0))
            out[f"s{to}_F{d}"] = F[:, k, j, i]
    np.savez_compressed(os.path.join(HERE, "ref_2d_mc_32x32.npz"), **out)


def points_fixture() -> None:
    n1, n2, n3, ng = 32, 32, 1, 4
    path = R.run(n1, n2, n3, ng, lim=0, flux=0, nsteps=1, every=1)
    g = Grid.torus(n1, n2, n3, lim=0)
    rr = R.RefRun(path, g)
    P0 = rr.state(0)
    rng = np.random.default_rng(2024)
    cells = rng.choice(n1 * n2, size=160, replace=False)
    ij, U, guess, kind = [], [], [], []
    for c in cells:
        j, i = divmod(int(c), n1)
        rec = rr.geom[0][:, j + ng, i + ng]
        p = P0[:, 0, j + ng, i + ng].copy()
        u0 = O.primtoU_point(rec, p)
        variants = [
            ("physical", u0, p * (1.0 + 1e-3 * rng.standard_normal(8))),
            ("physical_far_guess", u0, p * np.array([2.0, 0.3, 1.5, 1.5, 1.5, 1.0, 1.0, 1.0])),
        ]
        uu = u0.copy(); uu[2:5] *= 40.0
        variants.append(("momentum_beyond_light_cone", uu, p))
        uu = u0.copy(); uu[0] = -abs(uu[0])
        variants.append(("negative_density", uu, p))
        uu = u0.copy(); uu[0] *= 1e-14
        variants.append(("tiny_density", uu, p))
        uu = u0.copy(); uu[1] *= 0.5
        variants.append(("energy_low", uu, p))
        uu = u0.copy(); uu[1] *= 1.5
        variants.append(("energy_high", uu, p))
        uu = u0.copy(); uu[1] = np.nan
        variants.append(("nan_energy", uu, p))
        for name, uu, gp in variants:
            ij.append((i, j))
            U.append(uu)
            guess.append(gp)
            kind.append(name)
    ij = np.array(ij, dtype=np.float64)
    U = np.array(U)
    guess = np.array(guess)
    res = R.points(n1, n2, n3, ng, ij, U, guess)
    geomrec = np.stack([rr.geom[0][:, int(j) + ng, int(i) + ng] for i, j in ij], axis=1)
    np.savez_compressed(os.path.join(HERE, "ref_utoprimgen_points.npz"), ij=ij, U=U, guess=guess,
                        kind=np.array(kind), geomrec=geomrec, P=res[:, :8], pflag=res[:, 8], iters=res[:, 9],
                        grid=rr.info)


if __name__ == "__main__":
    R.build("2d_32x32_b4")
    torus_fixture()
    points_fixture()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
