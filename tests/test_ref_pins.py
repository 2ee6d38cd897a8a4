"""The CPU oracle (oracle/*.c) pinned to the reference HARM code itself.

Two sources of reference output:
  - the golden fixtures of tests/golden/ (made by tests/golden/make_golden.py from the
    reference binaries): a 2-D torus step with both substeps' advance()/fluxcalc() records,
    and Utoprimgen() of physical and unphysical conserved states;
  - the reference binaries of oracle/_ref/ run live (built by oracle/ref/build.sh from the
    reference's sources where those are present), for 2-D and 3-D grids and every
    reconstruction whose parity holds.
The oracle gets the reference's own inputs (its metric, connection and floor tables and its
bounded substep input), so what is compared is the algorithm of each entry point.
"""
import os

import numpy as np
import pytest

from harm_harm_b200 import Grid
from oracle import oracle as O
from oracle import ref as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b, floor_frac=1e-12):
    """max |a-b| / (|a| + |b| + floor), floor = floor_frac * max|b|"""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    floor = floor_frac * max(np.abs(b).max(), 1e-300)
    return float((np.abs(a - b) / (np.abs(a) + np.abs(b) + floor)).max())


def normwise(a, b):
    """max |a-b| / max |b|"""
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def active_faces(g, d):
    gg = g.g
    k = slice(gg.ng3, gg.ng3 + gg.n3 + (1 if d == 3 else 0))
    j = slice(gg.ng, gg.ng + gg.n2 + (1 if d == 2 else 0))
    i = slice(gg.ng, gg.ng + gg.n1 + (1 if d == 1 else 0))
    return (slice(None), k, j, i)


# ------------------------------------------------------------------ golden fixtures

@pytest.fixture(scope="module")
def torus32():
    d = np.load(os.path.join(GOLDEN, "ref_2d_mc_32x32.npz"))
    g = Grid.torus(32, 32, 1, lim=0)
    assert abs(g.g.startx[1] - d["grid"][5]) < 1e-15 and abs(g.g.dx[1] - d["grid"][9]) < 1e-15
    orc = O.Oracle(g, d["geom"], d["conn"], d["aux"])
    return g, d, orc


@pytest.mark.parametrize("to", [0, 1])
def test_golden_fluxcalc(torus32, to):
    g, d, orc = torus32
    pb = np.ascontiguousarray(d[f"s{to}_pb"])
    F = [np.zeros_like(pb) for _ in range(3)]
    ndt = orc.fluxcalc(pb.copy(), *F)
    for dd in (1, 2):
        a = F[dd - 1][active_faces(g, dd)]
        for pl in range(8):
            assert rel(a[pl], d[f"s{to}_F{dd}"][pl]) < 1e-12, (dd, pl)
        assert abs(ndt[dd - 1] - d[f"s{to}_ndtdir"][dd - 1]) <= 1e-13 * ndt[dd - 1]


@pytest.mark.parametrize("to", [0, 1])
def test_golden_advance(torus32, to):
    """advance() of one substep from the reference's bounded input: flux, conserved update
    with sources, inversion and fixup1zone, and the next dt"""
    g, d, orc = torus32
    pb = np.ascontiguousarray(d[f"s{to}_pb"])
    pi = np.ascontiguousarray(d["s0_pb"])  # RK2 midpoint: both substeps start from P^n
    args = d[f"s{to}_args"]
    pf = pb.copy()
    flag = np.zeros(pb.shape[1:], dtype=np.int8)
    ndt, st = orc.advance(to, pi.copy(), pb.copy(), pf, flag, float(args[0]), CUf=args[4:8], Cunew=args[8:12])
    act = (slice(None),) + g.active
    for pl in range(8):
        assert rel(pf[act][pl], d[f"s{to}_pf"][pl]) < 1e-12, pl
    assert (flag[g.active] == d[f"s{to}_pflag"]).all()
    assert abs(ndt - d[f"s{to}_ndt"][0]) <= 1e-13 * ndt


PHYSICAL_AND_FAILING = ["physical", "physical_far_guess", "momentum_beyond_light_cone", "negative_density",
                        "energy_low", "energy_high", "nan_energy"]


@pytest.mark.parametrize("kind", PHYSICAL_AND_FAILING)
def test_golden_utoprimgen(kind):
    """Utoprimgen of physical states and of states the hot inversion cannot invert: the same
    primitives (NaN where the reference returns NaN) and failure codes"""
    d = np.load(os.path.join(GOLDEN, "ref_utoprimgen_points.npz"))
    g = Grid.torus(32, 32, 1, lim=0)
    sel = np.nonzero(d["kind"] == kind)[0]
    assert len(sel) > 0
    iters_equal = 0
    for p in sel:
        P, fl, it = O.utoprimgen_point(g, d["geomrec"][:, p], d["U"][p], d["guess"][p])
        assert fl == d["pflag"][p], (kind, p, fl, d["pflag"][p])
        ref = d["P"][p]
        assert (np.isnan(P) == np.isnan(ref)).all()
        m = ~np.isnan(ref)
        assert rel(P[m], ref[m]) < 1e-10, (kind, p)
        iters_equal += it == d["iters"][p]
    if kind.startswith("physical") or kind in ("negative_density", "energy_low"):
        assert iters_equal == len(sel)


# ------------------------------------------------------------------ live reference runs

LIVE = {  # name: (n1, n2, n3, ng, lim, flux, tolerance, measure)
    "2d_mc_64x64": (64, 64, 1, 4, 0, 0, 1e-12, "rel"),
    "2d_paraline_laxf_64x64": (64, 64, 1, 4, 3, 1, 1e-12, "rel"),
    "2d_weno5_48x48": (48, 48, 1, 6, 2, 0, 1e-12, "rel"),
    # the reference stores its metric per (i,j,k), and its numerically differentiated
    # Jacobian varies with x3 by ~1e-11 of each component; the oracle uses k=0's tables on
    # every plane, so 3-D fluxes agree to ~1e-10 of each field's largest face value
    "3d_mc_32x24x8": (32, 24, 8, 4, 0, 0, 2e-10, "norm"),
    "3d_para_32x24x8": (32, 24, 8, 4, 1, 0, 2e-10, "norm"),
    "3d_paraline_32x24x8": (32, 24, 8, 4, 3, 0, 2e-10, "norm"),
    "3d_paraline_laxf_32x24x8": (32, 24, 8, 4, 3, 1, 2e-10, "norm"),
    # WENO5's nonlinear weights carry the same metric difference a little further (2.1e-10)
    "3d_weno5_32x24x8": (32, 24, 8, 6, 2, 0, 1e-9, "norm"),
}

# The reference's first flux computation after init in 3-D PARALINE: its shock indicator is
# computed from a scratch array that aliases the EMF array (shocktemparray = emf,
# flux.c:1667), which init leaves holding other data; a few cells' flattening differs in that
# one call.  From the second substep on the records agree.
FIRST_SUBSTEP_SKIPPED = {"3d_paraline_32x24x8", "3d_paraline_laxf_32x24x8"}


def live_substeps(name):
    subs = [(1, 0), (1, 1), (2, 0), (2, 1)]
    return subs[1:] if name in FIRST_SUBSTEP_SKIPPED else subs


def live(name):
    n1, n2, n3, ng, lim, flux, tol, how = LIVE[name]
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built (oracle/ref/build.sh needs the reference sources)")
    path = R.run(n1, n2, n3, ng, lim=lim, flux=flux, nsteps=2, every=1, substeps=(1, 2))
    g = Grid.torus(n1, n2, n3, lim=lim, fluxmethod=flux)
    rr = R.RefRun(path, g)
    return g, rr, tol, (rel if how == "rel" else normwise)


@pytest.mark.parametrize("name", list(LIVE))
def test_live_substeps(name):
    g, rr, tol, err = live(name)
    orc = O.Oracle(g, rr.geom, rr.conn, rr.aux)
    act = (slice(None),) + g.active
    nd = 3 if g.g.n3 > 1 else 2
    for step, to in live_substeps(name):
        pb = rr.sub(step, to, "pb")
        F = [np.zeros_like(pb) for _ in range(3)]
        ndt = orc.fluxcalc(pb.copy(), *F)
        for dd in range(1, nd + 1):
            Fr = rr.sub(step, to, f"F{dd}")
            sl = active_faces(g, dd)
            for pl in range(8):
                assert err(F[dd - 1][sl][pl], Fr[sl][pl]) < tol, (step, to, dd, pl)
            assert abs(ndt[dd - 1] - rr.sub(step, to, "ndtdir")[dd - 1]) <= max(tol, 1e-13) * ndt[dd - 1]
        args = rr.sub(step, to, "args")
        pf = pb.copy()
        flag = np.zeros(pb.shape[1:], dtype=np.int8)
        ndt1, _ = orc.advance(to, rr.sub(step, to, "pi"), pb.copy(), pf, flag, float(args[0]), CUf=args[4:8],
                              Cunew=args[8:12])
        pfr = rr.sub(step, to, "pf")
        for pl in range(8):
            assert err(pf[act][pl], pfr[act][pl]) < tol, (step, to, "pf", pl)
        assert (flag[g.active] == rr.sub(step, to, "pflag")[g.active]).all()
        assert abs(ndt1 - rr.sub(step, to, "ndt")[0]) <= max(tol, 1e-13) * ndt1


def test_reference_metric_locations_shared():
    """The device keeps 4 metric locations per (i,j): in the reference's tables FACE3 equals
    CENT, CORN1 equals FACE2 and CORN2 equals FACE1 exactly"""
    g, rr, _, _ = live("2d_mc_64x64")
    G = rr.geom8
    assert np.array_equal(G[3], G[0]) and np.array_equal(G[4], G[2]) and np.array_equal(G[5], G[1])


# ------------------------------------------------------------------ boundary conditions

BOUND = {  # name: (n1, n2, n3, ng, lim, relative tolerance)
    "2d_32x32": (32, 32, 1, 4, 0, 1e-15),
    # the reference's 3-D tables vary with x3 by ~1e-11 (see LIVE), which the inflow check and
    # the Lorentz-factor limits of the ghost cells see
    "3d_32x24x8": (32, 24, 8, 4, 0, 1e-9),
}


@pytest.mark.parametrize("name", list(BOUND))
def test_live_boundary_calls(name):
    """every per-direction boundary call of a step (the one-layer bound before post_fixup and
    the full one after it, both substeps), from the reference's own input"""
    n1, n2, n3, ng, lim, tol = BOUND[name]
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built (oracle/ref/build.sh needs the reference sources)")
    g = Grid.torus(n1, n2, n3, lim=lim)
    rr = R.RefRun(R.run(n1, n2, n3, ng, lim=lim, nsteps=1, every=1, substeps=(1,)), g)
    orc = O.Oracle(g, rr.geom, rr.conn, rr.aux)
    calls = rr.bound_calls(1)
    assert len(calls) == 12
    for n, (d, one_layer, pin, pout) in enumerate(calls):
        x = pin.copy()
        orc.bound_dir(x, d, simple=one_layer)
        err = np.abs(x - pout) / np.maximum(np.abs(pout), 1e-300)
        assert float(err.max()) <= tol, (n, d, one_layer, float(err.max()))


STEPS = {  # name: (n1, n2, n3, ng, lim, flux, steps, normwise tolerance)
    "c0_2d_mc_128x128_100steps": (128, 128, 1, 4, 0, 0, 100, 1e-12),
    "2d_mc_64x64_10steps": (64, 64, 1, 4, 0, 0, 10, 1e-13),
    "3d_mc_32x24x8_4steps": (32, 24, 8, 4, 0, 0, 4, 1e-9),
    "2d_weno5_48x48_20steps": (48, 48, 1, 6, 2, 0, 20, 1e-12),
    "2d_paraline_64x64_20steps": (64, 64, 1, 4, 3, 0, 20, 1e-12),
    # 3-D WENO5 runs free for two steps only: the SMONO indicator switches between the
    # 5-point and the WENO edge where the edge derivatives are within ~1e-13 of the stencil's
    # magnitude, so the ~1e-10 metric difference of the 3-D tables (see LIVE) flips a few
    # cells near the horizon from the third step on (6e-10 of max |u^3| after two steps, 1e-7
    # after three).  Substeps 3 and 4 fed the reference's own input agree to 2e-10 like 1 and 2.
    "3d_weno5_32x24x8_2steps": (32, 24, 8, 6, 2, 0, 2, 1e-8),
}


@pytest.mark.parametrize("name", list(STEPS))
def test_live_full_steps(name):
    """full RK2 steps (advance, bound, post_fixup, bound, twice; dt from post_stepch) from the
    reference's initial torus: the state, the dt sequence and the Newton iteration count of
    every step equal the reference's"""
    n1, n2, n3, ng, lim, flux, nsteps, tol = STEPS[name]
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built (oracle/ref/build.sh needs the reference sources)")
    every = max(1, nsteps // 4)
    g = Grid.torus(n1, n2, n3, lim=lim, fluxmethod=flux)
    rr = R.RefRun(R.run(n1, n2, n3, ng, lim=lim, flux=flux, nsteps=nsteps, every=every), g)
    orc = O.Oracle(g, rr.geom, rr.conn, rr.aux)
    P = rr.state(0)
    orc.bound_prim(P)
    dt = rr.dt0
    act = (slice(None),) + g.active
    for s in range(1, nsteps + 1):
        assert abs(dt - rr.dt_of_step(s)) <= max(tol, 1e-15) * dt, (s, dt, rr.dt_of_step(s))
        dt, st = orc.step_ch(P, dt)
        if n3 == 1:
            # equal counts while the states agree to round-off; later a cell's stopping test
            # may flip by one iteration as round-off grows
            if s <= 25:
                assert st["newton_iters"] == rr.steps[s, 2], s
            else:
                assert abs(st["newton_iters"] - rr.steps[s, 2]) <= 1e-4 * rr.steps[s, 2], s
        if s % every == 0 or s == nsteps:
            b = rr.state(s)[act]
            for pl in range(8):
                assert normwise(P[act][pl], b[pl]) < tol, (s, pl)


# ------------------------------------------------------------------ post_fixup with failures

FIX_CODES = (1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 50, 51, -1)


def planted_failures(n1, n2, n3, seed=3):
    """failure flags [n3][n2][n1] of every code the inversion reports, at random cells, at cells
    next to each grid boundary, in a 3x3 block (whose centre has no usable neighbour) inside and
    at the inner radial edge (the reset region of fixup_nogood) -- the cases post_fixup treats
    differently"""
    rng = np.random.default_rng(seed)
    fl = np.zeros((n3, n2, n1))
    for c in FIX_CODES:
        for _ in range(3):
            fl[rng.integers(0, n3), rng.integers(0, n2), rng.integers(0, n1)] = c
    k0 = n3 // 2
    for c, (j, i) in zip((1, 14, 1, 9, 15, 10, 1, 14),
                         ((0, 12), (n2 - 1, 14), (10, 0), (11, n1 - 1), (1, 20), (n2 - 2, 3), (5, n1 - 2), (n2 // 2, 1))):
        fl[k0, j, i] = c
    fl[k0, n2 // 2 - 1:n2 // 2 + 2, n1 // 2 - 1:n1 // 2 + 2] = 1
    fl[k0, 3:6, 0:3] = 14
    if n3 > 1:
        fl[0, 7, 17] = 1
        fl[n3 - 1, 8, 19] = 14
        fl[0, 0, n1 - 1] = 1
    return fl


# 3-D: the reference's metric varies with x3 by ~1e-11 (see LIVE), which the Lorentz-factor
# limit of a fixed velocity sees
FIXUP = {"2d_32x32": (32, 32, 1, 4, 1e-12, "rel"), "3d_32x24x8": (32, 24, 8, 4, 1e-10, "norm")}


@pytest.mark.parametrize("finalstep", [1, 0])
@pytest.mark.parametrize("name", list(FIXUP))
def test_live_post_fixup_planted_failures(name, finalstep):
    """post_fixup of the reference on its own bounded substep state with planted failure flags
    of every code: the oracle's values (to 1e-12) and flags equal the reference's"""
    n1, n2, n3, ng, tol, how = FIXUP[name]
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built (oracle/ref/build.sh needs the reference sources)")
    g = Grid.torus(n1, n2, n3, lim=0)
    rr = R.RefRun(R.run(n1, n2, n3, ng, lim=0, nsteps=1, every=1, substeps=(1,)), g)
    P = rr.sub(1, 0, "fixin")
    fl = planted_failures(n1, n2, n3)
    out, flr = R.fixup(n1, n2, n3, ng, P, fl, finalstep=finalstep)
    orc = O.Oracle(g, rr.geom, rr.conn, rr.aux)
    Po = P.copy()
    flo = np.zeros(P.shape[1:], np.int8)
    flo[g.active] = fl.astype(np.int8)
    orc.post_fixup(Po, flo, finalstep)
    act = (slice(None),) + g.active
    err = rel if how == "rel" else normwise
    for pl in range(8):
        assert err(Po[act][pl], out[act][pl]) < tol, pl
    assert (flo[g.active] == flr[g.active]).all()
    # the planted cells were changed where the reference changed them
    assert (np.abs(out[act] - P[act]).max(axis=0) > 0).sum() > 30


# ------------------------------------------------------------------ higher-order RK steps

# setup_rktimestep (step_ch.c:1171) wiring of each substep's p_i, p_b, p_f among p and the
# two scratch states pk[0], pk[1]: 0 = p, 1 = pk[0], 2 = pk[1]
RK_WIRING = {3: ((0, 0, 1), (0, 1, 2), (0, 2, 0)),
             4: ((0, 0, 1), (0, 1, 2), (0, 2, 1), (0, 1, 0))}


def rk_step(adv, bound, post_fixup, P, dt, coefs, wiring, shape):
    """one full step of HARM's step_ch_simplempi loop (step_ch.c:524-830) with the RK step's
    conserved arrays ui, uf, ucum carried across the substeps: per substep advance, bound_prim,
    post_fixup, bound_prim; returns the next dt (post_stepch) and the Newton iterations"""
    if isinstance(P, np.ndarray):
        states = [P, np.zeros_like(P), np.zeros_like(P)]
        ui, uf, ucum = (np.zeros(shape) for _ in range(3))
        flag = np.zeros(P.shape[1:], np.int8)
    else:  # torch CUDA tensors (the device path)
        import torch
        states = [P, torch.zeros_like(P), torch.zeros_like(P)]
        ui, uf, ucum = (torch.zeros_like(P) for _ in range(3))
        flag = torch.zeros(P.shape[1:], dtype=torch.int8, device=P.device)
    n = len(wiring)
    ndt, iters = 1e300, 0.0
    for s, (i, b, f) in enumerate(wiring):
        CUf, Cun = coefs[s]
        nd, st = adv(s, n, states[i], states[b], states[f], flag, ui, uf, ucum, dt, CUf, Cun)
        ndt = min(ndt, nd)
        iters += st["newton_iters"]
        bound(states[f])
        post_fixup(states[f], flag, 1 if s == n - 1 else 0)
        bound(states[f])
    return ndt, iters


@pytest.mark.parametrize("timeorder", [3, 4])
def test_live_rk_steps(timeorder):
    """TVD RK3 and RK4 (TIMEORDER 3 and 4 of setup_rktimestep, which carry U_f and ucum across
    the substeps): four full steps of the 2-D MC torus from the reference's initial state equal
    the reference's states, dt and Newton iteration counts"""
    n1, n2, n3, ng = 64, 64, 1, 4
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built (oracle/ref/build.sh needs the reference sources)")
    g = Grid.torus(n1, n2, n3, lim=0)
    rr = R.RefRun(R.run(n1, n2, n3, ng, lim=0, nsteps=4, every=1, timeorder=timeorder, substeps=(1,)), g)
    coefs = [(rr.sub(1, s, "args")[4:8].copy(), rr.sub(1, s, "args")[8:12].copy()) for s in range(timeorder)]
    orc = O.Oracle(g, rr.geom, rr.conn, rr.aux)
    P = rr.state(0)
    orc.bound_prim(P)
    dt = rr.dt0
    act = (slice(None),) + g.active
    for s in range(1, 5):
        assert abs(dt - rr.dt_of_step(s)) <= 1e-13 * dt, (s, dt, rr.dt_of_step(s))
        ndt, iters = rk_step(orc.advance_u, orc.bound_prim, orc.post_fixup, P, dt, coefs, RK_WIRING[timeorder],
                             P.shape)
        assert iters == rr.steps[s, 2], (s, iters, rr.steps[s, 2])
        dt = min(ndt, g.g.safe * dt)
        b = rr.state(s)[act]
        for pl in range(8):
            assert normwise(P[act][pl], b[pl]) < 1e-12, (s, pl, normwise(P[act][pl], b[pl]))
