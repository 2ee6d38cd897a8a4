"""CPU tests of the oracle (the checker of the device path) against physics known answers.

The reference holds no golden vectors for this path and is not built here, so the oracle is
pinned by properties every correct restatement must satisfy: the inversion recovers the
primitives that generated U, fluxes of a uniform state are the physical flux, MC reproduces
linear data, and flux-CT keeps the corner divergence of B at round-off.
"""
import numpy as np
import pytest

from helpers import divb_corner, make_torus
from oracle import oracle as O


@pytest.fixture(scope="module")
def torus2d():
    return make_torus(64, 64, 1)


def _random_prims(rng, n, gam=4.0 / 3.0):
    rho = 10 ** rng.uniform(-6, 0, n)
    u = rho * 10 ** rng.uniform(-4, 1, n)
    ut = rng.normal(0, 1, (3, n)) * rng.uniform(0, 3, n)
    B = rng.normal(0, 1, (3, n)) * np.sqrt(rho * 10 ** rng.uniform(-3, 2, n))
    return np.vstack([rho, u, ut, B])


def test_inversion_roundtrip(torus2d):
    g, geom, conn, aux, _ = torus2d
    rng = np.random.default_rng(1)
    cent = geom[0].reshape(28, -1)
    n = 400
    cells = rng.integers(0, cent.shape[1], n)
    prims = _random_prims(rng, n)
    errs, iters = [], []
    for c in range(n):
        rec = np.ascontiguousarray(cent[:, cells[c]])
        p = prims[:, c]
        # scale the velocity so that gamma stays below the limit
        U = O.primtoU_point(rec, p)
        guess = p * (1 + 0.05 * rng.normal(size=8))
        out, flag, it = O.utoprimgen_point(g, rec, U, guess)
        assert flag == 0, (c, flag)
        err = np.abs(out[:5] - p[:5]) / (np.abs(p[:5]) + 1e-12 * np.abs(p[:2]).max())
        errs.append(err.max())
        iters.append(it)
        assert np.allclose(out[5:], p[5:], rtol=1e-14, atol=0)
    errs = np.array(errs)
    # states up to gamma ~ 50 and b^2/rho ~ 100: Newton is round-off limited for a few
    # (PRECISEINVERSION accepts errx <= MIN_NEWT_TOL after MAX_NEWT_ITER)
    assert errs.max() < 1e-5, errs.max()
    assert np.quantile(errs, 0.5) < 1e-10 and np.quantile(errs, 0.9) < 1e-7
    assert np.median(iters) <= 20


def test_uniform_state_flux_is_physical_flux(torus2d):
    g, geom, conn, aux, P = torus2d
    orc = O.Oracle(g, geom, conn, aux)
    # a uniform state: every face sees p_l = p_r, so HLL returns the physical flux
    pr = np.array([0.3, 0.02, 0.01, 0.0, 0.05, 0.0, 0.0, 0.0])
    Pu = np.broadcast_to(pr[:, None, None, None], P.shape).copy()
    F = [np.zeros_like(P) for _ in range(3)]
    orc.fluxcalc(Pu, *F)
    gg = g.g
    for (i, j) in [(10, 10), (30, 40), (50, 20)]:
        ii, jj = i + gg.ng, j + gg.ng
        for d, loc in ((1, 1), (2, 2)):
            rec = np.ascontiguousarray(geom[loc, :, jj, ii])
            Fp = O.primtoflux_point(rec, pr, d)
            got = F[d - 1][:5, 0, jj, ii]
            np.testing.assert_allclose(got, Fp[:5], rtol=1e-13, atol=1e-16)


def test_mc_reconstruction_linear():
    y = 0.5 + 0.25 * np.arange(20.0)
    yl, yr = O.reconstruct_line(0, y)
    np.testing.assert_allclose(yl[1:-1], y[1:-1] - 0.125, rtol=0, atol=1e-15)
    np.testing.assert_allclose(yr[1:-1], y[1:-1] + 0.125, rtol=0, atol=1e-15)
    # an extremum gives a flat cell
    y2 = np.array([0.0, 1.0, 3.0, 1.0, 0.0])
    yl2, yr2 = O.reconstruct_line(0, y2)
    assert yl2[2] == 3.0 and yr2[2] == 3.0


def test_divb_stays_at_roundoff_and_state_finite(torus2d):
    g, geom, conn, aux, P0 = torus2d
    P = P0.copy()
    orc = O.Oracle(g, geom, conn, aux)
    orc.bound_prim(P)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    dt = 1.0 / (1 / ndt[0] + 1 / ndt[1])
    scale = np.abs(P[5:8] * geom[0, 26][None, None]).max() / min(g.g.dx[1], g.g.dx[2])
    d0 = divb_corner(g, geom, P).max()
    for _ in range(5):
        dt, st = orc.step_ch(P, dt)
    assert np.isfinite(P).all()
    d1 = divb_corner(g, geom, P).max()
    assert d0 / scale < 1e-13 and d1 / scale < 1e-13, (d0 / scale, d1 / scale)
    assert st["newton_iters"] / st["cells_inverted"] < 10


def test_oracle_3d_runs():
    g, geom, conn, aux, P = make_torus(24, 16, 8)
    orc = O.Oracle(g, geom, conn, aux)
    orc.bound_prim(P)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    dt = 1.0 / sum(1.0 / x for x in ndt)
    scale = np.abs(P[5:8] * geom[0, 26][None, None]).max() / min(g.g.dx[1], g.g.dx[2], g.g.dx[3])
    for _ in range(2):
        dt, st = orc.step_ch(P, dt)
    assert np.isfinite(P).all()
    assert divb_corner(g, geom, P).max() / scale < 1e-12


@pytest.mark.parametrize("lim,order", [(2, 4.5), (1, 1.8)])
def test_high_order_reconstruction_convergence_and_no_overshoot(lim, order):
    errs = []
    for n in (32, 64, 128):
        x = (np.arange(n) + 0.5) / n
        y = np.sin(2 * np.pi * x) + 2.0
        yl, yr = O.reconstruct_line(lim, y)
        exact_l = np.sin(2 * np.pi * np.arange(n) / n) + 2.0
        exact_r = np.sin(2 * np.pi * (np.arange(n) + 1) / n) + 2.0
        errs.append(max(np.abs(yl[6:-6] - exact_l[6:-6]).max(), np.abs(yr[6:-6] - exact_r[6:-6]).max()))
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(rates) > order, rates
    y = np.where(np.arange(40) < 20, 1.0, 0.1)
    yl, yr = O.reconstruct_line(lim, y)
    assert yl[5:-5].min() >= 0.1 - 1e-12 and yl[5:-5].max() <= 1.0 + 1e-12
    assert yr[5:-5].min() >= 0.1 - 1e-12 and yr[5:-5].max() <= 1.0 + 1e-12


@pytest.mark.parametrize("lim", [1, 2])
def test_oracle_torus_with_ppm_and_weno5(lim):
    g, geom, conn, aux, P = make_torus(48, 48, 1, lim=lim)
    orc = O.Oracle(g, geom, conn, aux)
    orc.bound_prim(P)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    dt = 1.0 / (1 / ndt[0] + 1 / ndt[1])
    scale = np.abs(P[5:8] * geom[0, 26][None, None]).max() / min(g.g.dx[1], g.g.dx[2])
    for _ in range(4):
        dt, st = orc.step_ch(P, dt)
    assert np.isfinite(P).all()
    assert divb_corner(g, geom, P).max() / scale < 1e-13
