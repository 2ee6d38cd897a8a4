"""The device path (libharm_b200.so through the C ABI, FP64) pinned to the reference HARM code
itself: the same records as tests/test_ref_pins.py -- the golden fixtures of tests/golden/
and live runs of the reference binaries of oracle/_ref/ -- fed to the device's fluxcalc,
advance and Utoprimgen with the reference's own metric, connection and floor tables.
"""
import os

import numpy as np
import pytest

from harm_harm_b200 import Grid, Harm
from test_ref_pins import GOLDEN, LIVE, PHYSICAL_AND_FAILING, active_faces, live, rel

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
        for step in (1, 2):
            for to in (0, 1):
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
