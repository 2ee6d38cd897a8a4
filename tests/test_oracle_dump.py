"""The oracle's rows of the main dump file (dump_content, dump.c:449; orc_dump.c) against
closed forms: the primitive and EOS columns (pressure (gam-1)u, cs2 = gam p/(rho+u+p),
Sden = rho log(p^n/rho^(n+1)), n = 1/(gam-1)), the coordinates, u^mu u_mu = -1, b^mu = 0
and div B = 0 without a field, vmin < vmax, and U of the row equal to the point primtoU."""
import numpy as np

from helpers import make_torus
from oracle import oracle as O


def test_dump_rows_closed_forms():
    g, geom, conn, aux, P = make_torus(16, 12, 4, lim=0)
    gg = g.g
    P[5:8] = 0.0  # no field: b^mu = 0 and div B = 0 exactly
    orc = O.Oracle(g, geom, conn, aux, nthreads=1)
    orc.bound_prim(P)
    cells = [(0, 0, 0), (7, 5, 2), (15, 11, 3), (3, 6, 1)]
    rows = orc.dump_rows(P, cells)
    gam = gg.gam
    for (i, j, k), r in zip(cells, rows):
        ii, jj, kk = i + gg.ng, j + gg.ng, k + gg.ng3
        pr = P[:, kk, jj, ii]
        assert tuple(r[0:3]) == (i, j, k)
        x1 = gg.startx[1] + (i + 0.5) * gg.dx[1]
        assert abs(r[3] - x1) <= 1e-15 * abs(x1) and abs(r[6] - (gg.R0 + np.exp(x1))) <= 1e-14 * r[6]
        assert abs(r[8] - 2 * np.pi * (gg.startx[3] + (k + 0.5) * gg.dx[3])) <= 1e-14
        assert np.array_equal(r[9:17], pr)
        rho, u = pr[0], pr[1]
        p = (gam - 1.0) * u
        n = 1.0 / (gam - 1.0)
        assert r[17] == p
        assert abs(r[18] - gam * p / (rho + u + p)) <= 1e-15 * r[18]
        assert abs(r[19] - rho * np.log(p ** n / rho ** (n + 1.0))) <= 1e-12 * abs(r[19])
        rec = np.ascontiguousarray(geom[0][:, jj, ii])
        assert np.allclose(r[20:28], O.primtoU_point(rec, pr), rtol=1e-14, atol=0)
        assert r[28] == 0.0
        ucon, ucov, bcon, bcov = r[29:33], r[33:37], r[37:41], r[41:45]
        assert abs(ucon @ ucov + 1.0) < 1e-12
        assert np.all(bcon == 0.0) and np.all(bcov == 0.0)
        assert np.all(r[45:51:2] <= r[46:51:2])
        assert r[51] == geom[0, 26, jj, ii]
