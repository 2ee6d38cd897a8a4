"""Parity of the device path (libharm_b200.so, through the C ABI) with the CPU oracle.

FP64 path: every entry point matches the oracle to 1e-12 relative (floor 1e-12 of the
field's maximum) on the same inputs; multi-step runs to 1e-10.  Mixed precision: FP32
reconstruction/HLL/CT with FP64 update and inversion, compared with the FP64 path in L1.
"""
import numpy as np
import pytest

from helpers import divb_corner, make_torus, plant_compression, rel_err
from harm_harm_b200 import HARM_PREC_FP64, HARM_PREC_FP64_FMA, HARM_PREC_MIXED, Harm
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (n1, n2, n3, lim, planted converging pressure jump, fluxmethod); the PARALINE cases carry
# the planted jump so that its shock flattener is active along every direction; the last case
# is the reference's own torus choice of reconstruction and flux (PARALINE, LAXF)
CASES = {"2d_mc": (64, 64, 1, 0, False, 0), "3d_mc": (32, 24, 8, 0, False, 0), "3d_ppm": (32, 24, 8, 1, False, 0),
         "3d_weno5": (32, 24, 8, 2, False, 0), "2d_weno5": (48, 48, 1, 2, False, 0),
         "3d_paraline": (32, 24, 8, 3, True, 0), "2d_paraline": (48, 48, 1, 3, True, 0),
         "3d_paraline_laxf": (32, 24, 8, 3, True, 1)}


@pytest.fixture(scope="module", params=list(CASES))
def setup(request, cuda):
    n1, n2, n3, lim, plant, flux = CASES[request.param]
    g, geom, conn, aux, P = make_torus(n1, n2, n3, lim=lim, fluxmethod=flux)
    if plant:
        plant_compression(g, P)
    orc = O.Oracle(g, geom, conn, aux)
    orc.bound_prim(P)
    dev = Harm(g, geom, conn, aux)
    return g, geom, conn, aux, P, orc, dev


def dev_array(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def faces_of_active(g, d):
    """slices of the faces whose fluxes enter the update (field fluxes final there)"""
    gg = g.g
    k = slice(gg.ng3, gg.ng3 + gg.n3 + (1 if d == 3 else 0))
    j = slice(gg.ng, gg.ng + gg.n2 + (1 if d == 2 else 0))
    i = slice(gg.ng, gg.ng + gg.n1 + (1 if d == 1 else 0))
    return (slice(None), k, j, i)


def test_bound_parity(setup, cuda):
    g, geom, conn, aux, P, orc, dev = setup
    Pc = P.copy()
    Pc[:, :, :, : g.g.ng] = 7.0  # stale ghosts to be overwritten
    Po = Pc.copy()
    orc.bound_prim(Po)
    Pd = dev_array(cuda, Pc)
    dev.bound_prim(Pd)
    cuda.cuda.synchronize()
    assert rel_err(Pd.cpu().numpy(), Po) < 1e-14


def test_fluxcalc_parity_fp64(setup, cuda):
    g, geom, conn, aux, P, orc, dev = setup
    Fo = [np.zeros_like(P) for _ in range(3)]
    ndt_o = orc.fluxcalc(P, *Fo)
    Pd = dev_array(cuda, P)
    Fd = [cuda.zeros_like(Pd) for _ in range(3)]
    ndt_d = dev.fluxcalc(Pd, *Fd)
    for d in range(3 if g.g.n3 > 1 else 2):
        sl = faces_of_active(g, d + 1)
        a = Fd[d].cpu().numpy()[sl]
        b = Fo[d][sl]
        for pl in range(8):
            e = rel_err(a[pl], b[pl])
            assert e < 1e-12, (d + 1, pl, e)
    for d in range(3 if g.g.n3 > 1 else 2):
        assert abs(ndt_d[d] - ndt_o[d]) <= 1e-12 * ndt_o[d], (d, ndt_d, ndt_o)


def test_advance_parity_fp64(setup, cuda):
    g, geom, conn, aux, P, orc, dev = setup
    Fo = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *Fo)
    dt = 1.0 / sum(1.0 / x for x in ndt[: (3 if g.g.n3 > 1 else 2)])
    pf_o = np.zeros_like(P)
    fl_o = np.zeros(P.shape[1:], dtype=np.int8)
    ndt_o, st_o = orc.advance(0, P, P, pf_o, fl_o, dt)
    Pd = dev_array(cuda, P)
    pf_d = cuda.zeros_like(Pd)
    fl_d = cuda.zeros(P.shape[1:], dtype=cuda.int8, device="cuda")
    ndt_d, st_d = dev.advance(0, Pd, Pd, pf_d, fl_d, dt)
    act = (slice(None),) + g.active
    a = pf_d.cpu().numpy()[act]
    b = pf_o[act]
    for pl in range(8):
        assert rel_err(a[pl], b[pl]) < 1e-12, (pl, rel_err(a[pl], b[pl]))
    assert np.array_equal(fl_d.cpu().numpy()[g.active], fl_o[g.active])
    assert abs(ndt_d - ndt_o) <= 1e-12 * ndt_o
    assert abs(st_d["newton_iters"] - st_o["newton_iters"]) <= 1e-3 * st_o["newton_iters"]


def test_step_parity_fp64_and_divb(setup, cuda):
    g, geom, conn, aux, P, orc, dev = setup
    Fo = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *Fo)
    dt0 = 1.0 / sum(1.0 / x for x in ndt[: (3 if g.g.n3 > 1 else 2)])
    Po = P.copy()
    dto = dt0
    for _ in range(3):
        dto, _ = orc.step_ch(Po, dto)
    Pd = dev_array(cuda, P)
    dtd, st = dev.step_ch(Pd, dt0, nsteps=3)
    Pdn = Pd.cpu().numpy()
    act = (slice(None),) + g.active
    for pl in range(8):
        e = rel_err(Pdn[act][pl], Po[act][pl], floor_frac=1e-10)
        assert e < 1e-10, (pl, e)
    assert abs(dtd - dto) <= 1e-10 * dto
    scale = np.abs(Pdn[5:8] * geom[0, 26][None, None]).max() / min(g.g.dx[1], g.g.dx[2])
    assert divb_corner(g, geom, Pdn).max() / scale < 1e-12


def test_utoprimgen_points_parity(cuda):
    g, geom, conn, aux, P = make_torus(32, 32, 1)
    dev = Harm(g, geom, conn, aux)
    rng = np.random.default_rng(7)
    cent = geom[0].reshape(28, -1)
    n = 4096
    cells = rng.integers(0, cent.shape[1], n)
    rho = 10 ** rng.uniform(-6, 0, n)
    prims = np.vstack([rho, rho * 10 ** rng.uniform(-4, 1, n), rng.normal(0, 1, (3, n)),
                       rng.normal(0, 1, (3, n)) * np.sqrt(rho * 10 ** rng.uniform(-3, 2, n))])
    recs = np.ascontiguousarray(cent[:, cells])
    U = np.stack([O.primtoU_point(np.ascontiguousarray(recs[:, c]), prims[:, c]) for c in range(n)], axis=1)
    guess = prims * (1 + 0.05 * rng.normal(size=prims.shape))
    out_o = np.zeros_like(prims)
    fl_o = np.zeros(n, dtype=np.int8)
    it_o = np.zeros(n, dtype=np.int32)
    for c in range(n):
        out_o[:, c], fl_o[c], it_o[c] = O.utoprimgen_point(g, np.ascontiguousarray(recs[:, c]), U[:, c], guess[:, c])
    Ud, Gd, Pd = (dev_array(cuda, x) for x in (U, recs, guess))
    fl_d = cuda.zeros(n, dtype=cuda.int8, device="cuda")
    it_d = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    dev.Utoprimgen(Ud, Gd, Pd, fl_d, it_d)
    out_d = Pd.cpu().numpy()
    assert np.array_equal(fl_d.cpu().numpy(), fl_o)
    for pl in range(8):
        assert rel_err(out_d[pl], out_o[pl], 1e-12) < 1e-9, pl
    # iteration counts agree except where round-off moves the stop by one step
    assert np.mean(np.abs(it_d.cpu().numpy() - it_o)) < 0.5


def test_mixed_precision_close_to_fp64(setup, cuda):
    g, geom, conn, aux, P, orc, dev = setup
    Fo = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *Fo)
    dt0 = 1.0 / sum(1.0 / x for x in ndt[: (3 if g.g.n3 > 1 else 2)])
    Pa = dev_array(cuda, P)
    Pb = dev_array(cuda, P)
    dev.step_ch(Pa, dt0, precision=HARM_PREC_FP64, nsteps=5)
    dev.step_ch(Pb, dt0, precision=HARM_PREC_MIXED, nsteps=5)
    a = Pa.cpu().numpy()[(slice(None),) + g.active]
    b = Pb.cpu().numpy()[(slice(None),) + g.active]
    l1_rho = np.abs(a[0] - b[0]).mean() / np.abs(a[0]).mean()
    assert np.isfinite(b).all()
    assert l1_rho < 1e-5, l1_rho
    scale = np.abs(Pb.cpu().numpy()[5:8] * geom[0, 26][None, None]).max() / min(g.g.dx[1], g.g.dx[2])
    # flux-CT keeps the corner divergence at round-off in the mixed path too (the field
    # fluxes average their FP32 edge EMFs exactly, in FP64)
    assert divb_corner(g, geom, Pb.cpu().numpy()).max() / scale < 1e-10


def test_fp64_fma_close_to_fp64(setup, cuda):
    """The FP64 path compiled with FMA contraction and shared reciprocals (the FP64 path at
    its best speed) against the IEEE-ordered FP64 path: the fluxes of one state to 1e-12 of
    each field's largest face value, five steps to 1e-10 of each field's maximum.  WENO5's
    SMONO indicator switches a cell between the 5-point and the WENO edge where the edge
    derivatives are within ~1e-13 of the stencil's magnitude, and PARALINE's flattener and
    monotonicity checks compare against thresholds, so there round-off differences flip a few
    faces: at most 1 % of the faces differ by more than 1e-12, the fluxes agree to 1e-4 in L1
    for WENO5 and 3e-2 for PARALINE (a flipped flattening of the planted jump moves its faces'
    fluxes by up to ~10 %), and the states after five steps to 1e-5 of each field's maximum
    (of the largest component of its vector for velocity and field; measured up to 1.8e-6
    for PARALINE)."""
    g, geom, conn, aux, P, orc, dev = setup
    Pd = dev_array(cuda, P)
    Fa = [cuda.zeros_like(Pd) for _ in range(3)]
    Fb = [cuda.zeros_like(Pd) for _ in range(3)]
    ndt_a = dev.fluxcalc(Pd, *Fa, precision=HARM_PREC_FP64)
    ndt_b = dev.fluxcalc(Pd, *Fb, precision=HARM_PREC_FP64_FMA)
    nd = 3 if g.g.n3 > 1 else 2
    switching = g.g.lim in (2, 3)
    for d in range(nd):
        a = Fa[d].cpu().numpy()[faces_of_active(g, d + 1)]
        b = Fb[d].cpu().numpy()[faces_of_active(g, d + 1)]
        for pl in range(8):
            scale = max(np.abs(a[pl]).max(), 1e-300)
            diff = np.abs(a[pl] - b[pl])
            if switching:
                assert (diff > 1e-12 * scale).mean() <= 0.01, (d + 1, pl, (diff > 1e-12 * scale).mean())
                assert diff.sum() <= (1e-4 if g.g.lim == 2 else 3e-2) * max(np.abs(a[pl]).sum(), 1e-300), (d + 1, pl)
            else:
                assert diff.max() / scale < 1e-12, (d + 1, pl, diff.max() / scale)
        assert abs(ndt_a[d] - ndt_b[d]) <= (1e-6 if switching else 1e-12) * ndt_a[d]
    dt0 = 1.0 / sum(1.0 / x for x in ndt_a[:nd])
    Pa, Pb = Pd.clone(), Pd.clone()
    dta, sta = dev.step_ch(Pa, dt0, precision=HARM_PREC_FP64, nsteps=5)
    dtb, stb = dev.step_ch(Pb, dt0, precision=HARM_PREC_FP64_FMA, nsteps=5)
    a = Pa.cpu().numpy()[(slice(None),) + g.active]
    b = Pb.cpu().numpy()[(slice(None),) + g.active]
    tol = 1e-5 if switching else 1e-10
    for pl in range(8):
        # a velocity or field component against its vector's largest component (B3 of the
        # poloidal loop starts at zero, and its own maximum stays tiny in 2-D)
        grp = slice(pl, pl + 1) if pl < 2 else slice(2, 5) if pl < 5 else slice(5, 8)
        e = np.abs(a[pl] - b[pl]).max() / max(np.abs(a[grp]).max(), 1e-300)
        assert e < tol, (pl, e)
    assert abs(dta - dtb) <= tol * dta
    assert abs(stb["newton_iters"] - sta["newton_iters"]) <= 0.01 * sta["newton_iters"]


@pytest.mark.parametrize("lim", [0, 1, 2])
def test_mixed_tma_staging_equals_plain_loads(cuda, lim, monkeypatch):
    """The FP32 flux tiles staged by plain loads (the default) and by TMA
    (HARM_B200_FLUX_STAGING=tma) feed the same arithmetic (the two kernels may contract
    multiply-adds differently, so FP32 rounding may differ): after two mixed-precision steps
    the fields agree to 1e-7 in L1 and 1e-6 of their maximum, in 3-D and 2-D."""
    torch = cuda
    for n1, n2, n3 in ((40, 24, 16), (48, 40, 1)):
        g, geom, conn, aux, P = make_torus(n1, n2, n3, lim=lim)
        monkeypatch.delenv("HARM_B200_FLUX_STAGING", raising=False)
        a = Harm(g, geom, conn, aux)
        monkeypatch.setenv("HARM_B200_FLUX_STAGING", "tma")
        b = Harm(g, geom, conn, aux)
        monkeypatch.delenv("HARM_B200_FLUX_STAGING", raising=False)
        Pa = dev_array(torch, P)
        a.bound_prim(Pa)
        Pb = Pa.clone()
        dta, _ = a.step_ch(Pa, 1e-3, precision=HARM_PREC_MIXED, nsteps=2)
        dtb, _ = b.step_ch(Pb, 1e-3, precision=HARM_PREC_MIXED, nsteps=2)
        assert abs(dta - dtb) <= 1e-6 * dta
        a_, b_ = Pa.cpu().numpy(), Pb.cpu().numpy()
        for pl in range(8):
            d = np.abs(a_[pl] - b_[pl])
            l1 = d.sum() / max(np.abs(a_[pl]).sum(), 1e-300)
            mx = d.max() / max(np.abs(a_[pl]).max(), 1e-300)
            assert l1 < 1e-7 and mx < 1e-6, (lim, n3, pl, l1, mx)
        a.close()
        b.close()


def test_mixed_inversion_reciprocal(cuda):
    """The mixed inversion's FP64 reciprocal (rcp.approx.ftz.f64 and two Newton-Raphson steps)
    against IEEE 1/b: within one ulp for normal operands with normal reciprocals, over every
    binade of that range and densely over the operands the Newton residual divides by (W, X,
    gamma^2, 1+gamma, E''); at the flush-to-zero edges NaN for a zero or subnormal operand and
    0 where the reciprocal would be subnormal."""
    from helpers import make_torus
    torch = cuda
    g, geom, conn, aux, _ = make_torus(16, 16, 1)
    dev = Harm(g, geom, conn, aux)
    try:
        rng = np.random.default_rng(7)
        m = rng.uniform(1.0, 2.0, 2_000_000)
        e = rng.integers(-1022, 1022, m.size)
        wide = np.ldexp(m, e) * rng.choice([-1.0, 1.0], m.size)
        dense = np.concatenate([10.0 ** rng.uniform(-12, 12, 1_000_000), 1.0 + rng.uniform(0, 625, 500_000),
                                -(10.0 ** rng.uniform(-12, 12, 500_000))])
        for b in (wide, dense):
            bd = torch.from_numpy(b).cuda()
            r = torch.empty_like(bd)
            dev.mixed_reciprocal(bd, r)
            got = r.cpu().numpy()
            ref = 1.0 / b
            assert np.all(np.sign(got) == np.sign(ref))
            ulps = np.abs(got.view(np.int64) - ref.view(np.int64))
            assert ulps.max() <= 1, (ulps.max(), b[np.argmax(ulps)])
        edge = np.array([0.0, -0.0, 5e-324, 2.0 ** -1030, -(2.0 ** -1023), 2.0 ** 1022 * 1.5, -(2.0 ** 1023)])
        bd = torch.from_numpy(edge).cuda()
        r = torch.empty_like(bd)
        dev.mixed_reciprocal(bd, r)
        got = r.cpu().numpy()
        assert np.all(np.isnan(got[:5])), got
        assert np.all(got[5:] == 0.0), got
    finally:
        dev.close()
