"""The device path (libharm_b200.so through the C ABI, FP64) pinned to the reference HARM code
itself: the same records as tests/test_ref_pins.py -- the golden fixtures of tests/golden/
and live runs of the reference binaries of oracle/_ref/ -- fed to the device's fluxcalc,
advance and Utoprimgen with the reference's own metric, connection and floor tables.
"""
import os

import numpy as np
import pytest

from harm_harm_b200 import Grid, Harm
from test_ref_pins import GOLDEN, LIVE, PHYSICAL_AND_FAILING, active_faces, live, live_substeps, rel

pytestmark = pytest.mark.gpu


def dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).cuda()


@pytest.fixture(scope="module")
def torus32(cuda):
    d = np.load(os.path.join(GOLDEN, "ref_2d_mc_32x32.npz"))
    g = Grid.torus(32, 32, 1, lim=0)
    h = Harm(g, d["geom"], d["conn"], d["aux"])
    yield g, d, h
    h.close()


@pytest.mark.parametrize("to", [0, 1])
def test_golden_fluxcalc_device(torus32, cuda, to):
    g, d, h = torus32
    pb = dev(cuda, d[f"s{to}_pb"])
    F = [cuda.zeros_like(pb) for _ in range(3)]
    ndt = h.fluxcalc(pb, *F)
    for dd in (1, 2):
        a = F[dd - 1].cpu().numpy()[active_faces(g, dd)]
        for pl in range(8):
            assert rel(a[pl], d[f"s{to}_F{dd}"][pl]) < 1e-12, (dd, pl)
        assert abs(ndt[dd - 1] - d[f"s{to}_ndtdir"][dd - 1]) <= 1e-13 * ndt[dd - 1]


@pytest.mark.parametrize("to", [0, 1])
def test_golden_advance_device(torus32, cuda, to):
    g, d, h = torus32
    pb = dev(cuda, d[f"s{to}_pb"])
    pi = dev(cuda, d["s0_pb"])
    pf = pb.clone()
    flag = cuda.zeros(pb.shape[1:], dtype=cuda.int8, device="cuda")
    args = d[f"s{to}_args"]
    ndt, _ = h.advance(to, pi, pb, pf, flag, float(args[0]), CUf=args[4:8], Cunew=args[8:12])
    act = (slice(None),) + g.active
    a = pf.cpu().numpy()[act]
    for pl in range(8):
        assert rel(a[pl], d[f"s{to}_pf"][pl]) < 1e-12, pl
    assert (flag.cpu().numpy()[g.active] == d[f"s{to}_pflag"]).all()
    assert abs(ndt - d[f"s{to}_ndt"][0]) <= 1e-13 * ndt


@pytest.mark.parametrize("kind", PHYSICAL_AND_FAILING)
def test_golden_utoprimgen_device(torus32, cuda, kind):
    g, _, h = torus32
    d = np.load(os.path.join(GOLDEN, "ref_utoprimgen_points.npz"))
    sel = np.nonzero(d["kind"] == kind)[0]
    U = dev(cuda, d["U"][sel].T.copy())
    P = dev(cuda, d["guess"][sel].T.copy())
    rec = dev(cuda, d["geomrec"][:, sel])
    flag = cuda.zeros(len(sel), dtype=cuda.int8, device="cuda")
    iters = cuda.zeros(len(sel), dtype=cuda.int32, device="cuda")
    h.Utoprimgen(U, rec, P, flag, iters)
    Pn = P.cpu().numpy().T
    fl = flag.cpu().numpy()
    it = iters.cpu().numpy()
    assert (fl == d["pflag"][sel]).all(), (kind, fl, d["pflag"][sel])
    ref = d["P"][sel]
    assert (np.isnan(Pn) == np.isnan(ref)).all()
    m = ~np.isnan(ref)
    assert rel(Pn[m], ref[m]) < 1e-10
    if kind.startswith("physical") or kind in ("negative_density", "energy_low"):
        assert (it == d["iters"][sel]).all()


@pytest.mark.parametrize("name", list(LIVE))
def test_live_substeps_device(cuda, name):
    g, rr, tol, err = live(name)
    h = Harm(g, rr.geom, rr.conn, rr.aux)
    act = (slice(None),) + g.active
    nd = 3 if g.g.n3 > 1 else 2
    try:
        for step, to in live_substeps(name):
            pb = dev(cuda, rr.sub(step, to, "pb"))
            F = [cuda.zeros_like(pb) for _ in range(3)]
            ndt = h.fluxcalc(pb, *F)
            for dd in range(1, nd + 1):
                Fr = rr.sub(step, to, f"F{dd}")
                sl = active_faces(g, dd)
                a = F[dd - 1].cpu().numpy()[sl]
                for pl in range(8):
                    assert err(a[pl], Fr[sl][pl]) < tol, (step, to, dd, pl)
                assert abs(ndt[dd - 1] - rr.sub(step, to, "ndtdir")[dd - 1]) <= max(tol, 1e-13) * ndt[dd - 1]
            args = rr.sub(step, to, "args")
            pf = pb.clone()
            flag = cuda.zeros(pb.shape[1:], dtype=cuda.int8, device="cuda")
            ndt1, _ = h.advance(to, dev(cuda, rr.sub(step, to, "pi")), pb, pf, flag, float(args[0]),
                                CUf=args[4:8], Cunew=args[8:12])
            pfr = rr.sub(step, to, "pf")
            a = pf.cpu().numpy()[act]
            for pl in range(8):
                assert err(a[pl], pfr[act][pl]) < tol, (step, to, "pf", pl)
            assert (flag.cpu().numpy()[g.active] == rr.sub(step, to, "pflag")[g.active]).all()
            assert abs(ndt1 - rr.sub(step, to, "ndt")[0]) <= max(tol, 1e-13) * ndt1
    finally:
        h.close()


@pytest.mark.parametrize("name", ["2d_32x32", "3d_32x24x8"])
def test_live_bound_device(cuda, name):
    """the device's bound_prim (x1, x2, x3) against the reference's full bound of both
    substeps: input of its x1 call, output of its x3 call"""
    from test_ref_pins import BOUND
    from oracle import ref as R
    n1, n2, n3, ng, lim, tol = BOUND[name]
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built")
    g = Grid.torus(n1, n2, n3, lim=lim)
    rr = R.RefRun(R.run(n1, n2, n3, ng, lim=lim, nsteps=1, every=1, substeps=(1,)), g)
    calls = rr.bound_calls(1)
    h = Harm(g, rr.geom, rr.conn, rr.aux)
    try:
        for first in (3, 9):  # the full bounds after post_fixup, substeps 0 and 1
            assert [c[0] for c in calls[first:first + 3]] == [1, 2, 3] and not calls[first][1]
            P = dev(cuda, calls[first][2])
            h.bound_prim(P)
            out = calls[first + 2][3]
            err = np.abs(P.cpu().numpy() - out) / np.maximum(np.abs(out), 1e-300)
            # exp/log of the radial extrapolation: CUDA's and glibc's may differ in the last ulp
            assert float(err.max()) <= max(tol, 1e-13), (first, float(err.max()))
    finally:
        h.close()


@pytest.mark.parametrize("name", ["c0_2d_mc_128x128_100steps", "2d_mc_64x64_10steps", "3d_mc_32x24x8_4steps"])
def test_live_full_steps_device(cuda, name):
    """full device RK2 steps (harm_b200_step_n, one step per call) from the reference's initial
    torus against the reference's states, dt and Newton iteration counts"""
    from test_ref_pins import STEPS, normwise
    from oracle import ref as R
    n1, n2, n3, ng, lim, flux, nsteps, tol = STEPS[name]
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built")
    every = max(1, nsteps // 4)
    g = Grid.torus(n1, n2, n3, lim=lim, fluxmethod=flux)
    rr = R.RefRun(R.run(n1, n2, n3, ng, lim=lim, flux=flux, nsteps=nsteps, every=every), g)
    h = Harm(g, rr.geom, rr.conn, rr.aux)
    act = (slice(None),) + g.active
    try:
        P = dev(cuda, rr.state(0))
        h.bound_prim(P)
        dt = rr.dt0
        for s in range(1, nsteps + 1):
            assert abs(dt - rr.dt_of_step(s)) <= max(tol, 1e-15) * dt, (s, dt, rr.dt_of_step(s))
            dt, st = h.step_ch(P, dt)
            if n3 == 1:
                # the device's exp, log and pow may differ from glibc's in the last bit, so a
                # cell's stopping test can flip by one iteration earlier than the oracle's
                assert abs(st["newton_iters"] - rr.steps[s, 2]) <= 1e-4 * rr.steps[s, 2], s
            if s % every == 0 or s == nsteps:
                a = P.cpu().numpy()[act]
                b = rr.state(s)[act]
                for pl in range(8):
                    assert normwise(a[pl], b[pl]) < tol, (s, pl, normwise(a[pl], b[pl]))
    finally:
        h.close()


@pytest.mark.parametrize("finalstep", [1, 0])
@pytest.mark.parametrize("name", ["2d_32x32", "3d_32x24x8"])
def test_live_post_fixup_planted_failures_device(cuda, name, finalstep):
    """the device's post_fixup (harm_b200_post_fixup) on the reference's bounded substep state
    with planted failure flags of every code (random cells, cells at every boundary, a block
    whose centre has no usable neighbour, the reset region): values and flags equal the
    reference's post_fixup"""
    from test_ref_pins import FIXUP, normwise, planted_failures
    from oracle import ref as R
    n1, n2, n3, ng, tol, how = FIXUP[name]
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built")
    g = Grid.torus(n1, n2, n3, lim=0)
    rr = R.RefRun(R.run(n1, n2, n3, ng, lim=0, nsteps=1, every=1, substeps=(1,)), g)
    P = rr.sub(1, 0, "fixin")
    fl = planted_failures(n1, n2, n3)
    out, flr = R.fixup(n1, n2, n3, ng, P, fl, finalstep=finalstep)
    h = Harm(g, rr.geom, rr.conn, rr.aux)
    try:
        Pd = dev(cuda, P)
        flh = np.zeros(P.shape[1:], np.int8)
        flh[g.active] = fl.astype(np.int8)
        fd = dev(cuda, flh)
        h.post_fixup(Pd, fd, finalstep)
        a = Pd.cpu().numpy()[(slice(None),) + g.active]
        b = out[(slice(None),) + g.active]
        err = rel if how == "rel" else normwise
        for pl in range(8):
            assert err(a[pl], b[pl]) < tol, (pl, err(a[pl], b[pl]))
        assert (fd.cpu().numpy()[g.active] == flr[g.active]).all()
    finally:
        h.close()


@pytest.mark.parametrize("timeorder", [3, 4])
def test_live_rk_steps_device(cuda, timeorder):
    """TVD RK3 and RK4 through harm_b200_advance_u (the RK step's conserved arrays ui, uf, ucum
    carried by the caller across the substeps, as HARM's advance() takes them): four full steps
    of the 2-D MC torus from the reference's initial state equal the reference's states, dt and
    Newton counts; the mixed path's steps stay within 1e-4 of each field's largest value"""
    from test_ref_pins import RK_WIRING, normwise, rk_step
    from oracle import ref as R
    from harm_harm_b200 import HARM_PREC_MIXED
    n1, n2, n3, ng = 64, 64, 1, 4
    if not R.available(n1, n2, n3, ng):
        pytest.skip("reference binary not built")
    g = Grid.torus(n1, n2, n3, lim=0)
    rr = R.RefRun(R.run(n1, n2, n3, ng, lim=0, nsteps=4, every=1, timeorder=timeorder, substeps=(1,)), g)
    coefs = [(rr.sub(1, s, "args")[4:8].copy(), rr.sub(1, s, "args")[8:12].copy()) for s in range(timeorder)]
    h = Harm(g, rr.geom, rr.conn, rr.aux)
    act = (slice(None),) + g.active
    try:
        for precision in (0, HARM_PREC_MIXED):
            P = dev(cuda, rr.state(0))
            h.bound_prim(P)
            dt = rr.dt0

            def adv(s, n, pi, pb, pf, flag, ui, uf, ucum, dt_, CUf, Cun):
                return h.advance_u(s, n, pi, pb, pf, flag, ui, uf, ucum, dt_, CUf, Cun, precision=precision)

            for s in range(1, 5):
                ndt, iters = rk_step(adv, h.bound_prim, h.post_fixup, P, dt, coefs, RK_WIRING[timeorder], P.shape)
                dt = min(ndt, g.g.safe * dt)
                b = rr.state(s)[act]
                a = P.cpu().numpy()[act]
                tol = 1e-12 if precision == 0 else 1e-4
                for pl in range(8):
                    assert normwise(a[pl], b[pl]) < tol, (precision, s, pl, normwise(a[pl], b[pl]))
                if precision == 0:
                    assert abs(iters - rr.steps[s, 2]) <= 1e-4 * rr.steps[s, 2], (s, iters, rr.steps[s, 2])
                    assert abs(dt - rr.dt_of_step(s + 1)) <= 1e-13 * dt if s < 4 else True
    finally:
        h.close()
