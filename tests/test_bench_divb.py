"""bench.py's div B figure (torch, on whatever device holds the state) against the tests' own
corner divergence, on CPU, for a 3-D and a 2-D torus after one oracle step."""
import os
import sys

import numpy as np
import pytest
import torch

from helpers import divb_corner, make_torus
from oracle import oracle as O

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


@pytest.mark.parametrize("shape", [(24, 16, 8), (32, 32, 1)])
def test_bench_divb_matches_corner_divergence(shape):
    g, geom, conn, aux, P = make_torus(*shape)
    orc = O.Oracle(g, geom, conn, aux)
    orc.bound_prim(P)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    orc.step_ch(P, 1.0 / sum(1.0 / x for x in ndt[: (3 if g.g.n3 > 1 else 2)]))
    act = P[5][g.active]
    cell = tuple(s.start + q for s, q in zip(g.active, np.unravel_index(np.argmax(np.abs(act)), act.shape)))
    P[5][cell] *= 1.001  # the strongest B1 cell off by 0.1 %: a divergence well above round-off
    m, rel = bench.divb_max(g, torch.from_numpy(np.ascontiguousarray(geom[0, 26])), torch.from_numpy(P))
    ref = divb_corner(g, geom, P).max()
    assert m == pytest.approx(ref, rel=1e-12)
    assert rel > 1e-6
