"""The oracle's PARALINE (line PPM with FLASH shock flattening, interpline.para.c:8) on CPU:
known answers of the flattener, the relation to PARA4, convergence, and a torus run with a
planted converging pressure jump that switches the flattener on along every direction."""
import numpy as np
import pytest

from helpers import divb_corner, make_torus, plant_compression
from oracle import oracle as O

PARA, PARALINE = 1, 3


def test_paraline_equals_para4_on_monotone_lines():
    # the slopes differ only where the MC limiter would zero them (sign changes)
    x = np.linspace(0.0, 1.0, 40)
    y = np.exp(3 * x) + 0.3 * x ** 2
    a, b = O.reconstruct_line(PARA, y), O.reconstruct_line(PARALINE, y)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_paraline_differs_from_para4_only_next_to_extrema():
    n = 64  # two periods, phase chosen so that no two cells straddle an extremum symmetrically
    y = np.sin(2 * np.pi * ((np.arange(n) + 0.5) / n * 2 + 0.037)) + 2.0
    a, b = O.reconstruct_line(PARA, y), O.reconstruct_line(PARALINE, y)
    d1 = np.diff(y)
    ext = [c for c in range(1, n - 1) if d1[c - 1] * d1[c] <= 0]  # local extrema
    assert ext
    differ = np.nonzero((a[0] != b[0]) | (a[1] != b[1]))[0]
    assert differ.size > 0
    for c in differ:
        assert min(abs(c - e) for e in ext) == 1, (c, ext)  # the extremum's neighbours


def test_paraline_convergence_and_no_overshoot():
    errs = []
    for n in (32, 64, 128):
        x = (np.arange(n) + 0.5) / n
        y = np.sin(2 * np.pi * x) + 2.0
        yl, yr = O.reconstruct_line(PARALINE, y)
        exact_l = np.sin(2 * np.pi * np.arange(n) / n) + 2.0
        exact_r = np.sin(2 * np.pi * (np.arange(n) + 1) / n) + 2.0
        errs.append(max(np.abs(yl[6:-6] - exact_l[6:-6]).max(), np.abs(yr[6:-6] - exact_r[6:-6]).max()))
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(rates) > 1.8, rates
    y = np.where(np.arange(40) < 20, 1.0, 0.1)
    yl, yr = O.reconstruct_line(PARALINE, y)
    assert yl[5:-5].min() >= 0.1 - 1e-12 and yl[5:-5].max() <= 1.0 + 1e-12
    assert yr[5:-5].min() >= 0.1 - 1e-12 and yr[5:-5].max() <= 1.0 + 1e-12


def _step(lo, hi, n=11, at=5):
    return np.where(np.arange(n) < at, lo, hi).astype(np.float64)


def test_flattener_known_answers():
    V = -np.arange(11.0)  # converging: V[1] - V[-1] < 0 everywhere
    # pressure step 1 -> 10 between cells 4 and 5: Sp = 1 at cells 4 and 5; at cell 3 the
    # pressure difference P[1]-P[-1] is 0, so the neighbour taken is cell 4 (ties shift to +1)
    assert np.array_equal(O.paraline_flattener(V, _step(1.0, 10.0)), [0, 0, 0, 1, 1, 1, 0, 0, 0, 0, 0])
    # diverging flow: never flattened
    assert not O.paraline_flattener(-V, _step(1.0, 10.0)).any()
    # weak jump: |dP| / min(P) = 0.2 < 1/3
    assert not O.paraline_flattener(V, _step(1.0, 1.2)).any()
    # the 1/3 threshold is the long double 1/3: 1/3 rounded to a double is below it
    assert not O.paraline_flattener(V, _step(3.0, 4.0)).any()
    assert np.array_equal(O.paraline_flattener(V, _step(3.0, np.nextafter(4.0, 5.0))), [0, 0, 0, 1, 1, 1, 0, 0, 0, 0, 0])
    # spread jump: Sp = 7.2/9 = 0.8 at cell 4 -> ftilde = 10 (0.8 - 0.75) = 0.5; cell 5 has
    # Sp = 1; cells 3 and 6 have Sp <= 0.75 and take their neighbour's value (cell 3: tie,
    # shift to cell 4; cell 6: P rises, shift to cell 5)
    P = np.array([1, 1, 1, 1, 1, 8.2, 10, 10, 10, 10, 10], dtype=np.float64)
    Fi = O.paraline_flattener(V, P)
    np.testing.assert_allclose(Fi, [0, 0, 0, 0.5, 0.5, 1, 1, 0, 0, 0, 0], rtol=0, atol=1e-12)


def test_full_flattening_gives_cell_values():
    n = 16
    V = -np.arange(float(n))
    P = _step(1.0, 10.0, n, 8)
    y = np.linspace(1.0, 2.0, n) ** 2
    Fi = O.paraline_flattener(V, P)
    yl, yr = O.reconstruct_line_paraline(y, V, P)
    yl0, yr0 = O.reconstruct_line(PARALINE, y)
    flat = np.nonzero(Fi == 1.0)[0]
    assert flat.size == 3
    assert np.array_equal(yl[flat], y[flat]) and np.array_equal(yr[flat], y[flat])
    rest = [c for c in range(2, n - 2) if Fi[c] == 0.0]
    assert np.array_equal(yl[rest], yl0[rest]) and np.array_equal(yr[rest], yr0[rest])


def test_oracle_torus_with_paraline_and_planted_shock():
    g, geom, conn, aux, P = make_torus(32, 24, 8, lim=PARALINE)
    plant_compression(g, P)
    orc = O.Oracle(g, geom, conn, aux)
    orc.bound_prim(P)
    gg = g.g
    for d, (na, nb) in ((1, (gg.n2, gg.n3)), (2, (gg.n1, gg.n3)), (3, (gg.n1, gg.n2))):
        hit = sum(int((orc.paraline_line_fi(P, d, a, b) > 0).sum()) for b in range(nb) for a in range(na))
        assert hit > 40, (d, hit)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    dt = 1.0 / sum(1.0 / x for x in ndt)
    scale = np.abs(P[5:8] * geom[0, 26][None, None]).max() / min(gg.dx[1], gg.dx[2], gg.dx[3])
    for _ in range(2):
        dt, st = orc.step_ch(P, dt)
        assert st["inversion_failures"] == 0
    assert np.isfinite(P).all()
    assert divb_corner(g, geom, P).max() / scale < 1e-13
