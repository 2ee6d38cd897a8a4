"""The reference's main dump file written from device state (harm_b200_dump; dump() dump.c:256,
dump_header_general dump.c:320, dump_content dump.c:449) against the oracle's restatement of
the 52 columns, in the three layouts of dump_gen (text, binary, text header + binary rows)."""
import numpy as np
import pytest

from helpers import make_torus, read_dump
from harm_harm_b200 import HARM_PREC_FP64, Harm
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def state(cuda):
    torch = cuda
    g, geom, conn, aux, P0 = make_torus(24, 16, 4, lim=0)
    dev = Harm(g, geom, conn, aux)
    P = torch.from_numpy(P0).cuda()
    dev.bound_prim(P)
    dt, _ = dev.step_ch(P, 1e-3, precision=HARM_PREC_FP64, nsteps=2)
    yield torch, g, geom, conn, aux, dev, P, dt
    dev.close()


def _check_header(head, g, t, dt, nstep):
    gg = g.g
    assert (head["n1"], head["n2"], head["n3"]) == (gg.n1, gg.n2, gg.n3)
    assert (head["is"], head["ie"], head["js"], head["je"], head["ks"], head["ke"]) == (0, gg.n1 - 1, 0, gg.n2 - 1, 0, gg.n3 - 1)
    assert head["whichdump"] == 3 and head["version"] == 0 and head["ncol"] == 52 and head["nstep"] == nstep
    for key, val in (("t", t), ("dt", dt), ("gam", gg.gam), ("a", gg.a), ("Rin", gg.Rin), ("Rout", gg.Rout),
                     ("hslope", gg.hslope), ("startx1", gg.startx[1]), ("dx1", gg.dx[1]), ("dx2", gg.dx[2])):
        assert abs(head[key] - val) <= 1e-14 * max(abs(val), 1.0), key


@pytest.mark.parametrize("fmt", ["text", "binary", "mixed"])
def test_dump_matches_oracle_rows(state, tmp_path, fmt):
    torch, g, geom, conn, aux, dev, P, dt = state
    path = str(tmp_path / ("dump0001" + (".bin" if fmt == "binary" else "")))
    dev.dump(P, path, t=0.25, dt=dt, nstep=2, fmt=fmt)
    head, cols = read_dump(path, fmt)
    _check_header(head, g, 0.25, dt, 2)
    gg = g.g
    assert cols.shape == (gg.n1 * gg.n2 * gg.n3, 52)
    # rows in the order k, j, i (i fastest)
    k, j, i = np.meshgrid(np.arange(gg.n3), np.arange(gg.n2), np.arange(gg.n1), indexing="ij")
    assert np.array_equal(cols[:, 0], i.ravel()) and np.array_equal(cols[:, 1], j.ravel()) and np.array_equal(cols[:, 2], k.ravel())
    o = Oracle(g, geom, conn, aux, nthreads=1)
    want = o.dump_rows(P.cpu().numpy(), list(zip(i.ravel(), j.ravel(), k.ravel())))
    rtol = 1e-13 if fmt == "text" else 1e-12  # text: 15 significant digits
    for c in range(52):
        a, b = cols[:, c], want[:, c]
        if c == 28:  # divb: round-off of a vanishing divergence
            assert np.abs(a - b).max() < 1e-12, c
            continue
        scale = np.abs(b).max() + 1e-300
        err = np.abs(a - b) / (np.abs(b) + 1e-12 * scale)
        assert err.max() < rtol, (c, err.max())
    assert cols[:, 28].max() < 1e-10  # flux-CT keeps the corner divergence at round-off


def test_dump_records_the_given_conserved_state(state, tmp_path):
    torch, g, geom, conn, aux, dev, P, dt = state
    U = torch.rand_like(P)
    path = str(tmp_path / "dump_u.bin")
    dev.dump(P, path, U=U, fmt="binary")
    _, cols = read_dump(path, "binary")
    gg = g.g
    ng, ng3 = gg.ng, gg.ng3
    Ua = U.cpu().numpy()[:, ng3:ng3 + gg.n3, ng:ng + gg.n2, ng:ng + gg.n1].reshape(8, -1).T
    assert np.array_equal(cols[:, 20:28], Ua)
