"""The oracle's flux formula choice (fluxmethod, fluxcompute.c:243) on CPU: LAXF and HLL share
the wave speeds, so the CFL limits are identical; on a state that is the same on both sides of
every face they reduce to the physical flux; on the torus they differ."""
import numpy as np

from helpers import make_torus
from harm_harm_b200 import HARM_FLUX_HLL, HARM_FLUX_LAXF
from oracle import oracle as O


def _fluxes(fluxmethod, uniform=False):
    g, geom, conn, aux, P = make_torus(32, 24, 4, lim=0, fluxmethod=fluxmethod)
    if uniform:
        for pl, v in enumerate((1.0, 0.1, 0.02, 0.0, 0.01, 0.0, 0.0, 0.0)):
            P[pl] = v
    orc = O.Oracle(g, geom, conn, aux)
    if not uniform:
        orc.bound_prim(P)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    gg = g.g
    act = (slice(None), slice(gg.ng3, gg.ng3 + gg.n3), slice(gg.ng, gg.ng + gg.n2), slice(gg.ng, gg.ng + gg.n1))
    return ndt, [f[act][:5] for f in F]


def test_laxf_and_hll_share_the_cfl_limits_and_differ_in_flux():
    ndt_h, Fh = _fluxes(HARM_FLUX_HLL)
    ndt_l, Fl = _fluxes(HARM_FLUX_LAXF)
    assert ndt_h == ndt_l
    # x1: the Kerr-Schild frame makes the two wave speeds unequal, so HLL is not LAXF; (with
    # equal speeds, as along x2 of the initial torus where u^2 = 0, the two formulas coincide)
    assert np.abs(Fh[0] - Fl[0]).max() > 1e-6 * np.abs(Fh[0]).max()


def test_laxf_and_hll_agree_on_a_state_without_jumps():
    _, Fh = _fluxes(HARM_FLUX_HLL, uniform=True)
    _, Fl = _fluxes(HARM_FLUX_LAXF, uniform=True)
    for d in range(3):
        np.testing.assert_allclose(Fl[d], Fh[d], rtol=1e-13, atol=1e-13 * np.abs(Fh[d]).max())
