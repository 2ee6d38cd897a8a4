"""CPU checks of the oracle of the learned inversion guess (network and features):
the analytic gradient of orc_mlp_loss_grad against central finite differences of its own
loss, and the features/targets of exact (U, P) pairs against their closed forms
(D = rho gamma, W' = (rho+u+p) gamma^2 - rho gamma, utsq = gamma^2 - 1)."""
import numpy as np

from helpers import geom_records, make_torus
from oracle import oracle as O

NP = 9154


def _net(seed=3):
    rng = np.random.default_rng(seed)
    params = (rng.standard_normal(NP) * 0.3).astype(np.float32)
    norm = np.zeros(24, dtype=np.float32)
    norm[10:20] = 1.0
    norm[22:24] = 1.0
    return rng, params, norm


def test_oracle_gradient_matches_finite_differences():
    rng, params, norm = _net()
    feat = rng.standard_normal((8, 10)).astype(np.float32)
    targ = rng.standard_normal((8, 2)).astype(np.float32)
    loss, grad, _ = O.mlp_loss_grad(feat, targ, params, norm)
    assert loss > 0
    idx = np.concatenate([[0, 639, 640, 703, 704, 4799, 4800, 4864, 8959, 8960, 9024, 9151, 9152, 9153],
                          rng.choice(NP, 40, replace=False)])
    scale = np.abs(grad).max()
    for p in idx:
        w = params.copy()
        h = np.float32(1e-2)
        w[p] = params[p] + h
        lp = O.mlp_loss_grad(feat, targ, w, norm)[0]
        hp = float(w[p]) - float(params[p])
        w[p] = params[p] - h
        lm = O.mlp_loss_grad(feat, targ, w, norm)[0]
        hm = float(params[p]) - float(w[p])
        fd = (lp - lm) / (hp + hm)
        assert abs(fd - grad[p]) <= 2e-3 * scale + 2e-3 * abs(grad[p]), (p, fd, grad[p])


def test_oracle_features_and_targets_of_exact_pairs():
    g, geom, conn, aux, P = make_torus(32, 32, 1)
    gg = g.g
    rng = np.random.default_rng(5)
    gam = gg.gam
    for _ in range(20):
        i = rng.integers(gg.ng, gg.ng + gg.n1)
        j = rng.integers(gg.ng, gg.ng + gg.n2)
        rec = geom_records(geom, g, np.array([j * gg.n1e + i]))[:, 0]
        gcov = rec[0:10]
        pr = np.zeros(8)
        pr[0] = 10 ** rng.uniform(-5, 0)
        pr[1] = pr[0] * 10 ** rng.uniform(-3, 1)
        pr[2:5] = rng.standard_normal(3) * 0.3 / np.sqrt(gcov[[4, 7, 9]])
        pr[5:8] = rng.standard_normal(3) * 0.1 * np.sqrt(pr[0]) / np.sqrt(gcov[[4, 7, 9]])
        U = O.primtoU_point(rec, pr)
        f, t = O.mlp_features(g, rec, U, pr)
        u1, u2, u3 = pr[2:5]
        qsq = (gcov[4] * u1 * u1 + gcov[7] * u2 * u2 + gcov[9] * u3 * u3
               + 2 * (gcov[5] * u1 * u2 + gcov[6] * u1 * u3))
        gamma = np.sqrt(1 + qsq)
        D = pr[0] * gamma
        Wp = (pr[0] + pr[1] + (gam - 1) * pr[1]) * gamma ** 2 - D
        assert abs(f[0] - np.log(D)) < 1e-5 * max(1.0, abs(np.log(D)))
        assert abs(t[0] - np.log(Wp / D)) < 1e-5 * max(1.0, abs(np.log(Wp / D)))
        assert abs(t[1] - np.log(gamma ** 2)) < 1e-5 * max(1.0, np.log(gamma ** 2))
        assert abs(f[6] - rec[21]) < 1e-6 and abs(f[7] - np.log(abs(rec[26]))) < 1e-5
