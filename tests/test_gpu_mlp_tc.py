"""GPU tests of the learned start on the tcgen05 tensor cores (harm_mlp_tc.cuh), through the
C ABI.  HARM_B200_MLP_ENGINE selects the engine of a context: the mma.sync network in a kernel
ahead of the inversion (default, "mma"), the mma.sync network inside the inversion kernel
("mma-fused"), the tcgen05 network in a kernel ahead of it ("tc"), or the tcgen05 network
inside the inversion kernel ("tc-fused").  The engines compute the same
BF16 products with FP32 accumulation in different orders, so their outputs agree to the BF16
rounding of the activations; both are checked against the oracle's double-precision forward
pass.  Steps with every engine match the plain steps within the Newton tolerance."""
import os

import numpy as np
import pytest

from helpers import make_torus, rel_err
from harm_harm_b200 import HARM_GUESS_MLP, HARM_GUESS_PREV, HARM_PREC_FP64, HARM_PREC_MIXED, Harm
from oracle import oracle as O
from test_gpu_mlp import _synth, _torus_pairs, _train

pytestmark = pytest.mark.gpu


def _harm(g, geom, conn, aux, engine):
    old = os.environ.get("HARM_B200_MLP_ENGINE")
    os.environ["HARM_B200_MLP_ENGINE"] = engine
    try:
        return Harm(g, geom, conn, aux)
    finally:
        if old is None:
            del os.environ["HARM_B200_MLP_ENGINE"]
        else:
            os.environ["HARM_B200_MLP_ENGINE"] = old


@pytest.fixture(scope="module")
def engines(cuda):
    g, geom, conn, aux, P = make_torus(64, 64, 1)
    tc, mma, fused, mfused = (_harm(g, geom, conn, aux, e) for e in ("tc", "mma", "tc-fused", "mma-fused"))
    yield cuda, g, geom, conn, aux, P, tc, mma, fused, mfused
    for dev in (tc, mma, fused, mfused):
        dev.close()


def test_tensor_core_network_matches_mma_sync_and_oracle(engines):
    torch, g, geom, conn, aux, P0, tc, mma, _, _ = engines
    f, t, *_ = _synth(torch, tc, 80000, 11)
    norm, params, _ = _train(torch, tc, f, t, steps=3000)
    tc.mlp_set(params, norm)
    mma.mlp_set(params, norm)
    m = 5000  # not a multiple of the 128-row tile
    fm = f[:m].contiguous()
    out_tc = torch.zeros((m, 2), device="cuda", dtype=torch.float32)
    out_mma = torch.zeros((m, 2), device="cuda", dtype=torch.float32)
    tc.mlp_predict(fm, out_tc)
    mma.mlp_predict(fm, out_mma)
    _, _, pred = O.mlp_loss_grad(fm.cpu().numpy(), None, params.cpu().numpy(), norm.cpu().numpy())
    tsd = norm.cpu().numpy()[22:24]
    a, b = out_tc.cpu().numpy(), out_mma.cpu().numpy()
    assert np.all(np.isfinite(a))
    e_tc, e_mma, d = np.abs(a - pred) / tsd, np.abs(b - pred) / tsd, np.abs(a - b) / tsd
    print("standardised |err| vs oracle: tcgen05 mean", e_tc.mean(0), "max", e_tc.max(0),
          "| mma.sync mean", e_mma.mean(0), "max", e_mma.max(0), "| between them mean", d.mean(0), "max", d.max(0))
    # the bounds of the mma.sync inference test, and the two engines close to each other
    assert e_tc[:, 0].mean() < 0.01 and e_tc[:, 0].max() < 0.2, (e_tc[:, 0].mean(), e_tc[:, 0].max())
    assert e_tc[:, 1].mean() < 0.1 and e_tc[:, 1].max() < 1.5, (e_tc[:, 1].mean(), e_tc[:, 1].max())
    assert d[:, 0].mean() < 5e-3 and d[:, 0].max() < 0.1, (d[:, 0].mean(), d[:, 0].max())


def test_tensor_core_learned_steps_match_plain_and_mma_sync_steps(engines):
    torch, g, geom, conn, aux, P0, tc, mma, fused, mfused = engines
    _, f, t, _ = _torus_pairs(torch, tc, P0)
    norm, params, _ = _train(torch, tc, f, t, steps=3000)
    for dev in (tc, mma, fused, mfused):
        dev.mlp_set(params, norm)
    P = torch.from_numpy(P0).cuda()
    tc.bound_prim(P)
    Pa = P.clone()
    dta, sta = tc.step_ch(Pa, 1e-3, precision=HARM_PREC_MIXED, guess=HARM_GUESS_PREV, nsteps=3)
    a = Pa.cpu().numpy()
    runs = {}
    for name, dev in (("mma.sync", mma), ("mma.sync fused", mfused), ("tcgen05", tc), ("tcgen05 fused", fused)):
        Pb = P.clone()
        dtb, stb = dev.step_ch(Pb, 1e-3, precision=HARM_PREC_MIXED, guess=HARM_GUESS_MLP, nsteps=3)
        b = Pb.cpu().numpy()
        for pl in range(8):
            assert rel_err(a[pl], b[pl], 1e-8) < 1e-9, (name, pl, rel_err(a[pl], b[pl], 1e-8))
        assert abs(dta - dtb) <= 1e-9 * dta
        assert stb["cells_inverted"] == sta["cells_inverted"]
        assert 0 <= stb["mlp_fallbacks"] <= 0.01 * stb["cells_inverted"]
        runs[name] = stb["newton_iters"] / stb["cells_inverted"]
    print("iters/cell plain %.3f" % (sta["newton_iters"] / sta["cells_inverted"]),
          " ".join("%s %.3f" % kv for kv in runs.items()))
    for name in ("tcgen05", "tcgen05 fused"):
        assert abs(runs[name] - runs["mma.sync"]) < 0.05 * runs["mma.sync"]
    # the fused mma.sync kernel evaluates the same network with the same arithmetic
    assert runs["mma.sync fused"] == runs["mma.sync"]


@pytest.mark.parametrize("engine,precision", [("tc", HARM_PREC_MIXED), ("tc-fused", HARM_PREC_MIXED),
                                              ("tc", HARM_PREC_FP64), ("tc-fused", HARM_PREC_FP64),
                                              ("mma-fused", HARM_PREC_MIXED), ("mma-fused", HARM_PREC_FP64)])
def test_tensor_core_learned_steps_3d(cuda, engine, precision):
    """3-D tiles (16 i x 8 k at one j) with a ragged edge in i and k, on both arithmetic paths."""
    torch = cuda
    g, geom, conn, aux, P0 = make_torus(40, 24, 12)
    dev = _harm(g, geom, conn, aux, engine)
    try:
        _, f, t, _ = _torus_pairs(torch, dev, P0)
        norm, params, _ = _train(torch, dev, f, t, steps=2000)
        dev.mlp_set(params, norm)
        Pa = torch.from_numpy(P0).cuda()
        dev.bound_prim(Pa)
        Pb = Pa.clone()
        _, sta = dev.step_ch(Pa, 1e-3, precision=precision, guess=HARM_GUESS_PREV, nsteps=2)
        _, stb = dev.step_ch(Pb, 1e-3, precision=precision, guess=HARM_GUESS_MLP, nsteps=2)
        a, b = Pa.cpu().numpy(), Pb.cpu().numpy()
        for pl in range(8):
            assert rel_err(a[pl], b[pl], 1e-8) < 1e-9, (pl, rel_err(a[pl], b[pl], 1e-8))
        assert stb["cells_inverted"] == sta["cells_inverted"]
        assert stb["mlp_fallbacks"] <= 0.01 * stb["cells_inverted"]
    finally:
        dev.close()
