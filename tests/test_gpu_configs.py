"""The torus configurations of the benchmark suite at their full grid sizes, through the C ABI:
  C0  2-D 128x128, MC, FP64: device and oracle after 10 RK2 steps, 1e-10 relative;
  C1  3-D 192x96x64, WENO5, FP64: device and oracle after 2 RK2 steps, 1e-10 relative
      (plus div B at round-off on the device after the steps);
  C2  3-D 256x128x64, WENO5, mixed precision against the FP64 device path after 20 steps:
      L1 relative density error <= 1e-6, the accuracy bound of the mixed path;
  C4  3-D 384x192x128, WENO5, mixed precision with the learned start (the benchmark's
      configuration) against the FP64 device path after 10 steps: the same bound, div B at
      round-off, at most 1% fallbacks from the learned start and no failed inversion.
The oracle runs on all host cores (OpenMP); each case takes seconds."""
import numpy as np
import pytest

from helpers import divb_corner, make_torus
from harm_harm_b200 import HARM_GUESS_MLP, HARM_PREC_FP64, HARM_PREC_MIXED, Harm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _initial_dt(orc, P):
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    return 1.0 / sum(1.0 / x for x in ndt if x < 1e99)


def _max_rel(a, b, floor_frac=1e-10):
    err = 0.0
    for pl in range(a.shape[0]):
        floor = floor_frac * max(np.abs(a[pl]).max(), np.abs(b[pl]).max(), 1e-300)
        err = max(err, float((np.abs(a[pl] - b[pl]) / (np.abs(a[pl]) + np.abs(b[pl]) + floor)).max()))
    return err


@pytest.mark.parametrize("case,n1,n2,n3,lim,steps", [("C0", 128, 128, 1, 0, 10), ("C1", 192, 96, 64, 2, 2)])
def test_fp64_config_matches_oracle(cuda, case, n1, n2, n3, lim, steps):
    torch = cuda
    g, geom, conn, aux, P = make_torus(n1, n2, n3, lim=lim)
    orc = O.Oracle(g, geom, conn, aux)
    orc.bound_prim(P)
    dt = _initial_dt(orc, P)
    dev = Harm(g, geom, conn, aux)
    Pd = torch.from_numpy(P.copy()).cuda()
    dt_d, st = dev.step_ch(Pd, dt, precision=HARM_PREC_FP64, nsteps=steps)
    Po = P.copy()
    dt_o = dt
    for _ in range(steps):
        dt_o, _ = orc.step_ch(Po, dt_o)
    act = (slice(None),) + g.active
    err = _max_rel(Pd.cpu().numpy()[act], Po[act])
    assert err < 1e-10, (case, err)
    assert abs(dt_d - dt_o) <= 1e-10 * dt_o
    dv = divb_corner(g, geom, Pd.cpu().numpy())
    bmax = np.abs(Pd.cpu().numpy()[5:8]).max()
    assert dv.max() < 1e-10 * bmax / min(g.g.dx[1], g.g.dx[2]), (case, dv.max())
    dev.close()


def test_mixed_c2_density_error_bound(cuda):
    torch = cuda
    g, geom, conn, aux, P = make_torus(256, 128, 64, lim=2)
    dev = Harm(g, geom, conn, aux)
    Pa = torch.from_numpy(P).cuda()
    dev.bound_prim(Pa)
    Pb = Pa.clone()
    dev.step_ch(Pa, 1e-3, precision=HARM_PREC_FP64, nsteps=20)
    dev.step_ch(Pb, 1e-3, precision=HARM_PREC_MIXED, nsteps=20)
    act = (slice(None),) + g.active
    a, b = Pa.cpu().numpy()[act], Pb.cpu().numpy()[act]
    l1 = float(np.abs(a[0] - b[0]).sum() / np.abs(a[0]).sum())
    assert l1 <= 1e-6, l1
    dev.close()


def test_mixed_learned_c4_full_size(cuda):
    torch = cuda
    g, geom, conn, aux, P = make_torus(384, 192, 128, lim=2)
    dev = Harm(g, geom, conn, aux)
    try:
        Pa = torch.from_numpy(P).cuda()
        dev.bound_prim(Pa)
        Pb = Pa.clone()
        # the plain method's own pairs, then a short training on the GPU
        Pt = Pa.clone()
        dev.step_ch(Pt, 1e-3, precision=HARM_PREC_MIXED)
        n = (384 * 192 * 128) // 16 + 1
        f = torch.zeros((n, 10), device="cuda")
        t = torch.zeros((n, 2), device="cuda")
        m = dev.mlp_dump(Pt, f, t, stride=16)
        f, t = f[:m].contiguous(), t[:m].contiguous()
        norm = torch.zeros(24, device="cuda")
        params = torch.zeros(9154, device="cuda")
        dev.mlp_norm(f, t, norm)
        dev.mlp_init(params, 1)
        dev.mlp_train(f, t, norm, params, steps=2000)
        dev.mlp_set(params, norm)
        dev.step_ch(Pa, 1e-3, precision=HARM_PREC_FP64, nsteps=10)
        _, st = dev.step_ch(Pb, 1e-3, precision=HARM_PREC_MIXED, guess=HARM_GUESS_MLP, nsteps=10)
        act = (slice(None),) + g.active
        a, b = Pa.cpu().numpy(), Pb.cpu().numpy()
        assert np.all(np.isfinite(b[act]))
        l1 = float(np.abs(a[act][0] - b[act][0]).sum() / np.abs(a[act][0]).sum())
        assert l1 <= 1e-6, l1
        dv = divb_corner(g, geom, b)
        bmax = np.abs(b[5:8]).max()
        assert dv.max() < 1e-10 * bmax / min(g.g.dx[1], g.g.dx[2]), dv.max()
        assert st["mlp_fallbacks"] <= 0.01 * st["cells_inverted"]
        assert st["inversion_failures"] == 0
    finally:
        dev.close()
