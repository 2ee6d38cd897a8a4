"""Run full RK2 steps of the magnetised torus on one GPU (for timing and profiling runs).

    python -m harm_harm_b200.run_steps --grid 384 192 128 --lim weno5 --precision mixed --steps 2

Builds the torus on the host (the seeded Fishbone-Moncrief initial state), bounds it, takes
the first dt from the fluxes, runs the steps through harm_b200_step_n and prints the final dt
and the Newton iterations per cell.  Every numeric routine runs in libharm_b200.so.
"""
from __future__ import annotations

import argparse

from . import (HARM_GUESS_PREV, HARM_PREC_FP64, HARM_PREC_FP64_FMA, HARM_PREC_MIXED, Grid,
               Harm)

LIMS = {"mc": 0, "ppm": 1, "weno5": 2, "paraline": 3}
PRECS = {"fp64": HARM_PREC_FP64, "mixed": HARM_PREC_MIXED, "fp64fma": HARM_PREC_FP64_FMA}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[192, 96, 64])
    ap.add_argument("--lim", default="weno5", choices=list(LIMS))
    ap.add_argument("--flux", default="hll", choices=["hll", "laxf"])
    ap.add_argument("--precision", default="mixed", choices=list(PRECS))
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=12345)
    args = ap.parse_args()
    import torch
    g = Grid.torus(*args.grid, lim=LIMS[args.lim], fluxmethod=1 if args.flux == "laxf" else 0)
    geom, conn, aux = g.geometry()
    P = torch.from_numpy(g.torus_init(geom, aux, seed=args.seed)).cuda()
    dev = Harm(g, geom, conn, aux)
    dev.bound_prim(P)
    F = [torch.empty_like(P) for _ in range(3)]
    ndt = dev.fluxcalc(P, *F)
    del F
    dt = 1.0 / sum(1.0 / x for x in ndt if x < 1e99)
    dt, st = dev.step_ch(P, dt, precision=PRECS[args.precision], guess=HARM_GUESS_PREV, nsteps=args.steps)
    torch.cuda.synchronize()
    print(f"{args.steps} steps of {'x'.join(map(str, args.grid))} {args.lim} {args.precision}: next dt {dt:.6g}, "
          f"Newton iterations per cell {st['newton_iters'] / max(st['cells_inverted'], 1):.3f}")
    dev.close()


if __name__ == "__main__":
    main()
