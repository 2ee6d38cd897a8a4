"""GPU tests of the learned inversion guess, through the C ABI:
  - synthetic pairs: device primtoU, features and targets against the oracle;
  - the FP32 forward/backward kernels: loss and gradient against the double-precision
    oracle (gradient check);
  - training on the GPU lowers the loss; BF16 tensor-core inference against the oracle's
    double forward pass;
  - grid dumps of the plain method's own run are consistent with its primitives;
  - steps with the learned guess match the plain steps within the Newton tolerance;
  - what the trained network gains: on torus states whose previous state is not known (a
    cold start: floor density and energy, zero velocity), the learned start needs fewer
    Newton iterations than the plain guess (about 5.3 against 6.1 per cell).  Where the
    previous state is known, as in a time step of a smooth flow, it is already within about
    1e-7 of the root and the learned start (BF16 inference, about 0.5% in W') costs about
    0.3 iterations per cell more; the steps test prints both counts."""
import numpy as np
import pytest

from helpers import harm_with_env, make_torus, rel_err
from harm_harm_b200 import HARM_GUESS_MLP, HARM_GUESS_PREV, HARM_PREC_FP64, HARM_PREC_MIXED, Harm
from oracle import oracle as O

pytestmark = pytest.mark.gpu
NP = 9154


@pytest.fixture(scope="module")
def torus2d(cuda):
    g, geom, conn, aux, P = make_torus(64, 64, 1)
    dev = Harm(g, geom, conn, aux)
    yield cuda, g, geom, conn, aux, P, dev
    dev.close()


def _synth(torch, dev, n, seed):
    f = torch.zeros((n, 10), device="cuda", dtype=torch.float32)
    t = torch.zeros((n, 2), device="cuda", dtype=torch.float32)
    U = torch.zeros((8, n), device="cuda", dtype=torch.float64)
    P = torch.zeros((8, n), device="cuda", dtype=torch.float64)
    cell = torch.zeros(n, device="cuda", dtype=torch.int32)
    dev.mlp_synth(f, t, seed, U, P, cell)
    return f, t, U, P, cell


def _train(torch, dev, f, t, steps, seed=1):
    norm = torch.zeros(24, device="cuda", dtype=torch.float32)
    dev.mlp_norm(f, t, norm)
    params = torch.zeros(NP, device="cuda", dtype=torch.float32)
    dev.mlp_init(params, seed=seed)
    hist = dev.mlp_train(f, t, norm, params, steps=steps, batch=8192, lr=3e-3, seed=5)
    return norm, params, hist


def _torus_pairs(torch, dev, P0, nsteps=3):
    """the plain method's own run: a few FP64 steps, then a dump of every cell"""
    P = torch.from_numpy(P0).cuda()
    dev.bound_prim(P)
    dev.step_ch(P, 1e-3, precision=HARM_PREC_FP64, nsteps=nsteps)
    g = dev.grid.g
    maxn = g.n1 * g.n2 * g.n3
    f = torch.zeros((maxn, 10), device="cuda", dtype=torch.float32)
    t = torch.zeros((maxn, 2), device="cuda", dtype=torch.float32)
    cell = torch.zeros(maxn, device="cuda", dtype=torch.int32)
    n = dev.mlp_dump(P, f, t, cell)
    return P, f[:n].contiguous(), t[:n].contiguous(), cell[:n]


def test_synthetic_pairs_match_oracle(torus2d):
    torch, g, geom, conn, aux, P0, dev = torus2d
    n = 512
    f, t, U, P, cell = _synth(torch, dev, n, 123)
    f, t, U, P, cell = f.cpu().numpy(), t.cpu().numpy(), U.cpu().numpy(), P.cpu().numpy(), cell.cpu().numpy()
    cent = geom[0].reshape(geom.shape[1], -1)
    for s in range(0, n, 7):
        rec = np.ascontiguousarray(cent[:, cell[s]])
        Uo = O.primtoU_point(rec, P[:, s])
        assert rel_err(U[:, s], Uo) < 1e-12
        fo, to = O.mlp_features(g, rec, U[:, s], P[:, s])
        assert np.allclose(f[s], fo, rtol=1e-5, atol=1e-5), (s, f[s], fo)
        assert np.allclose(t[s], to, rtol=1e-4, atol=1e-4), (s, t[s], to)


def test_gradient_matches_oracle(torus2d):
    torch, g, *_, dev = torus2d
    n = 300  # not a multiple of the 64-sample chunk
    f, t, *_ = _synth(torch, dev, 4096, 7)
    norm = torch.zeros(24, device="cuda", dtype=torch.float32)
    dev.mlp_norm(f, t, norm)
    params = torch.zeros(NP, device="cuda", dtype=torch.float32)
    dev.mlp_init(params, seed=3)
    grad = torch.zeros(NP, device="cuda", dtype=torch.float32)
    loss = dev.mlp_loss_grad(f, t, params, norm, grad, n=n)
    lo, go, _ = O.mlp_loss_grad(f[:n].cpu().numpy(), t[:n].cpu().numpy(), params.cpu().numpy(), norm.cpu().numpy())
    gd = grad.cpu().numpy().astype(np.float64)
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    assert np.linalg.norm(gd - go) <= 1e-4 * np.linalg.norm(go)
    assert np.abs(gd - go).max() <= 1e-4 * np.abs(go).max()


def test_training_lowers_loss_and_inference_matches_oracle(torus2d):
    torch, g, *_, dev = torus2d
    f, t, *_ = _synth(torch, dev, 80000, 11)
    norm, params, hist = _train(torch, dev, f, t, steps=5000)
    assert np.all(np.isfinite(hist))
    assert hist[-100:].mean() < 0.05 * hist[:5].mean(), (hist[:5], hist[-100:].mean())
    dev.mlp_set(params, norm)
    m = 2000
    out = torch.zeros((m, 2), device="cuda", dtype=torch.float32)
    dev.mlp_predict(f[:m].contiguous(), out)
    _, _, pred = O.mlp_loss_grad(f[:m].cpu().numpy(), None, params.cpu().numpy(), norm.cpu().numpy())
    tsd = norm.cpu().numpy()[22:24]
    err = np.abs(out.cpu().numpy() - pred) / tsd  # in standardised units
    print("BF16 inference |err| (standardised) mean", err.mean(0), "max", err.max(0))
    # log(W'/D), the output the Newton start uses, is the tight one; log(1+utsq) is more
    # sensitive to the BF16 rounding of the activations
    assert err[:, 0].mean() < 0.01 and err[:, 0].max() < 0.2, (err[:, 0].mean(), err[:, 0].max())
    assert err[:, 1].mean() < 0.1 and err[:, 1].max() < 1.5, (err[:, 1].mean(), err[:, 1].max())


def test_grid_dump_consistent_with_primitives(torus2d):
    torch, g, geom, conn, aux, P0, dev = torus2d
    P = torch.from_numpy(P0).cuda()
    dev.bound_prim(P)
    dev.step_ch(P, 1e-3, precision=HARM_PREC_FP64)
    n1, n2 = g.g.n1, g.g.n2
    maxn = n1 * n2
    f = torch.zeros((maxn, 10), device="cuda", dtype=torch.float32)
    t = torch.zeros((maxn, 2), device="cuda", dtype=torch.float32)
    cell = torch.zeros(maxn, device="cuda", dtype=torch.int32)
    n = dev.mlp_dump(P, f, t, cell, stride=3, phase=1)
    assert 0.9 * (maxn // 3) <= n <= maxn // 3 + 1
    f, t, cell, Ph = f[:n].cpu().numpy(), t[:n].cpu().numpy(), cell[:n].cpu().numpy(), P.cpu().numpy()
    assert np.all(cell % 3 == 1)
    gg = g.g
    cent = geom[0].reshape(geom.shape[1], -1)
    checked = 0
    for s in range(0, n, 5):
        i, j = cell[s] % n1 + gg.ng, cell[s] // n1 + gg.ng
        pr = Ph[:, 0, j, i]
        # where no floor acted, P is the converged inversion of the dumped U
        if pr[0] < 1.01 * aux[1, j, i] or pr[1] < 1.01 * aux[2, j, i]:
            continue
        rec = np.ascontiguousarray(cent[:, j * gg.n1e + i])
        U = O.primtoU_point(rec, pr)
        fo, to = O.mlp_features(g, rec, U, pr)
        assert np.allclose(f[s], fo, rtol=1e-4, atol=1e-4), (s, f[s], fo)
        assert np.allclose(t[s], to, rtol=1e-4, atol=1e-4), (s, t[s], to)
        checked += 1
    assert checked > 50


@pytest.mark.parametrize("precision", [HARM_PREC_FP64, HARM_PREC_MIXED])
def test_learned_guess_steps_match_plain_steps(torus2d, precision):
    torch, g, geom, conn, aux, P0, dev = torus2d
    _, f, t, _ = _torus_pairs(torch, dev, P0)
    norm, params, _ = _train(torch, dev, f, t, steps=3000)
    dev.mlp_set(params, norm)
    Pa = torch.from_numpy(P0).cuda()
    dev.bound_prim(Pa)
    Pb = Pa.clone()
    dta, sta = dev.step_ch(Pa, 1e-3, precision=precision, guess=HARM_GUESS_PREV, nsteps=3)
    dtb, stb = dev.step_ch(Pb, 1e-3, precision=precision, guess=HARM_GUESS_MLP, nsteps=3)
    a, b = Pa.cpu().numpy(), Pb.cpu().numpy()
    for pl in range(8):
        assert rel_err(a[pl], b[pl], 1e-8) < 1e-9, (pl, rel_err(a[pl], b[pl], 1e-8))
    assert abs(dta - dtb) <= 1e-9 * dta
    assert stb["cells_inverted"] == sta["cells_inverted"]
    assert 0 <= stb["mlp_fallbacks"] <= 0.01 * stb["cells_inverted"]
    print("iters/cell plain %.3f learned %.3f fallback rate %.5f" % (
        sta["newton_iters"] / sta["cells_inverted"], stb["newton_iters"] / stb["cells_inverted"],
        stb["mlp_fallbacks"] / stb["cells_inverted"]))


@pytest.mark.parametrize("precision", [HARM_PREC_FP64, HARM_PREC_MIXED])
def test_gated_learned_start(torus2d, precision):
    """The default engine gives the learned start only to cells whose first Newton step from
    the previous state exceeds HARM_B200_MLP_GATE of the convergence scale.  With no cell
    above the gate the step is the plain step bit for bit; with a zero gate every cell takes
    the learned start (listed, then inverted by the fused network + Newton kernel) and the
    step matches the plain step within the Newton tolerance; the default gate lies between."""
    torch, g, geom, conn, aux, P0, dev = torus2d
    _, f, t, _ = _torus_pairs(torch, dev, P0)
    norm, params, _ = _train(torch, dev, f, t, steps=3000)
    Pa = torch.from_numpy(P0).cuda()
    dev.bound_prim(Pa)
    P1 = Pa.clone()
    _, sta = dev.step_ch(Pa, 1e-3, precision=precision, guess=HARM_GUESS_PREV, nsteps=3)
    a = Pa.cpu().numpy()
    for gate in ("1e300", "0", None):
        env = {"HARM_B200_MLP_ENGINE": "gated"}
        if gate is not None:
            env["HARM_B200_MLP_GATE"] = gate
        dg = harm_with_env(g, geom, conn, aux, **env)
        try:
            dg.mlp_set(params, norm)
            Pb = P1.clone()
            _, stb = dg.step_ch(Pb, 1e-3, precision=precision, guess=HARM_GUESS_MLP, nsteps=3)
        finally:
            dg.close()
        b = Pb.cpu().numpy()
        assert stb["cells_inverted"] == sta["cells_inverted"]
        print("gate %s: listed %.0f of %.0f, iters/cell %.3f (plain %.3f), fallbacks %.0f" % (
            gate, stb["mlp_cells"], stb["cells_inverted"], stb["newton_iters"] / stb["cells_inverted"],
            sta["newton_iters"] / sta["cells_inverted"], stb["mlp_fallbacks"]))
        if gate == "1e300":
            assert np.array_equal(a, b)
            assert stb["mlp_cells"] == 0 and stb["newton_iters"] == sta["newton_iters"]
            continue
        for pl in range(8):
            assert rel_err(a[pl], b[pl], 1e-8) < 1e-9, (gate, pl, rel_err(a[pl], b[pl], 1e-8))
        assert stb["mlp_fallbacks"] <= 0.01 * max(stb["mlp_cells"], 1.0)
        if gate == "0":
            assert stb["mlp_cells"] >= 0.99 * stb["cells_inverted"]


def test_learned_guess_gains_over_a_cold_start(torus2d):
    """Torus states inverted without their previous state: the plain guess is a cold start
    (floor density and energy, zero velocity, as after a restart from conserved variables);
    the network, trained on the plain method's own pairs, starts the iteration near W'."""
    torch, g, geom, conn, aux, P0, dev = torus2d
    P, f, t, cell = _torus_pairs(torch, dev, P0)
    norm, params, _ = _train(torch, dev, f, t, steps=3000)
    dev.mlp_set(params, norm)
    gg = g.g
    Ph = P.cpu().numpy()
    cent = geom[0].reshape(geom.shape[1], -1)
    rng = np.random.default_rng(2)
    cells = rng.choice(cell.cpu().numpy(), 3000, replace=False)
    ii, jj = cells % gg.n1 + gg.ng, cells // gg.n1 + gg.ng
    prims = Ph[:, 0, jj, ii]
    recs = np.ascontiguousarray(cent[:, jj * gg.n1e + ii])
    U = np.stack([O.primtoU_point(recs[:, c], prims[:, c]) for c in range(len(cells))], axis=1)
    cold = prims.copy()
    cold[0] = aux[1, jj, ii]
    cold[1] = aux[2, jj, ii]
    cold[2:5] = 0.0
    Ud, Rd = torch.from_numpy(U).cuda(), torch.from_numpy(recs).cuda()
    res = {}
    for name, gs in (("plain", HARM_GUESS_PREV), ("learned", HARM_GUESS_MLP)):
        Pg = torch.from_numpy(cold.copy()).cuda()
        flag = torch.zeros(len(cells), device="cuda", dtype=torch.int8)
        it = torch.zeros(len(cells), device="cuda", dtype=torch.int32)
        dev.Utoprimgen(Ud, Rd, Pg, flag, it, guess=gs)
        res[name] = (it.double().mean().item(), int((flag != 0).sum().item()), Pg.cpu().numpy(), flag.cpu().numpy())
    print("cold start, mean Newton iterations: plain %.2f learned %.2f; failures plain %d learned %d" % (
        res["plain"][0], res["learned"][0], res["plain"][1], res["learned"][1]))
    assert res["learned"][0] < 0.93 * res["plain"][0]
    assert res["learned"][1] <= res["plain"][1]
    ok = (res["plain"][3] == 0) & (res["learned"][3] == 0)
    for pl in range(5):
        assert rel_err(res["plain"][2][pl][ok], res["learned"][2][pl][ok], 1e-9) < 1e-8
        assert rel_err(res["learned"][2][pl][ok], prims[pl][ok], 1e-9) < 1e-8
