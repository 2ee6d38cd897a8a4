"""Shared helpers of the test suite: grids, comparisons, divergence of B."""
from __future__ import annotations

import numpy as np

from harm_harm_b200 import Grid


def make_torus(n1=64, n2=64, n3=1, lim=0, seed=12345, beta=100.0, fluxmethod=0):
    g = Grid.torus(n1, n2, n3, lim=lim, fluxmethod=fluxmethod)
    geom, conn, aux = g.geometry()
    P = g.torus_init(geom, aux, beta_min=beta, seed=seed)
    return g, geom, conn, aux, P


def plant_compression(grid, P, amp=10.0, v=(0.1, 0.02, 0.05), width=3, dense_frac=0.2):
    """A strong, converging pressure jump inside the torus (in place, ghosts included): where
    rho exceeds dense_frac of its maximum, the internal energy is multiplied by amp in the
    block i >= n1/2, j >= n2/2, k >= n3/2, and within `width` cells of the block's faces the
    velocity primitives get +-v pointing at those faces, so that the PARALINE flattener
    switches on along every direction while every inversion still succeeds."""
    g = grid.g
    k_, j_, i_ = np.meshgrid(np.arange(g.n3e) - g.ng3, np.arange(g.n2e) - g.ng, np.arange(g.n1e) - g.ng,
                             indexing="ij")
    i0, j0, k0 = g.n1 // 2, g.n2 // 2, g.n3 // 2
    dense = P[0] > dense_frac * P[0].max()
    P[1][(i_ >= i0) & (j_ >= j0) & (k_ >= k0) & dense] *= amp

    def towards(x, x0):
        return np.where(x >= x0, -1.0, 1.0) * (np.abs(x - x0 + 0.5) < width) * dense

    P[2] += v[0] * towards(i_, i0)
    P[3] += v[1] * towards(j_, j0)
    if g.n3 > 1:
        P[4] += v[2] * towards(k_, k0)
    return P


def rel_err(a, b, floor_frac=1e-12):
    """max |a-b| / (|a|+|b| + floor), floor = floor_frac * max(|a|) (per array)"""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    floor = floor_frac * max(np.abs(a).max(), np.abs(b).max(), 1e-300)
    return float((np.abs(a - b) / (np.abs(a) + np.abs(b) + floor)).max())


def per_field_close(a, b, rtol, floor_frac=1e-10):
    """rel_err per primitive field; returns dict pl -> err"""
    return {pl: rel_err(a[pl], b[pl], floor_frac) for pl in range(a.shape[0])}


def divb_corner(grid, geom, P):
    """Toth corner divergence of sqrt(-g) B (the quantity flux-CT preserves) at the corners whose
    cells are all active in x1 and x2 (the corners on the radial and polar boundaries also see
    ghost cells, which the boundary conditions set, not flux-CT); x3 is periodic."""
    g = grid.g
    gd = geom[0, 26]  # CENT gdet [j][i]
    U = P[5:8] * gd[None, None, :, :]
    ng, ng3 = g.ng, g.ng3
    dx1, dx2, dx3 = g.dx[1], g.dx[2], g.dx[3]
    if g.n3 == 1:
        k = 0
        u1, u2 = U[0, k], U[1, k]
        j0, j1, i0, i1 = ng + 1, ng + g.n2, ng + 1, ng + g.n1
        J, I = np.mgrid[j0:j1, i0:i1]
        d1 = 0.5 * (u1[J, I] + u1[J - 1, I] - u1[J, I - 1] - u1[J - 1, I - 1]) / dx1
        d2 = 0.5 * (u2[J, I] + u2[J, I - 1] - u2[J - 1, I] - u2[J - 1, I - 1]) / dx2
        return np.abs(d1 + d2)
    u1, u2, u3 = U[0], U[1], U[2]
    K, J, I = np.mgrid[ng3:ng3 + g.n3 + 1, ng + 1:ng + g.n2, ng + 1:ng + g.n1]
    d1 = 0.25 * (u1[K, J, I] + u1[K, J - 1, I] + u1[K - 1, J, I] + u1[K - 1, J - 1, I]
                 - u1[K, J, I - 1] - u1[K, J - 1, I - 1] - u1[K - 1, J, I - 1] - u1[K - 1, J - 1, I - 1]) / dx1
    d2 = 0.25 * (u2[K, J, I] + u2[K, J, I - 1] + u2[K - 1, J, I] + u2[K - 1, J, I - 1]
                 - u2[K, J - 1, I] - u2[K, J - 1, I - 1] - u2[K - 1, J - 1, I] - u2[K - 1, J - 1, I - 1]) / dx2
    d3 = 0.25 * (u3[K, J, I] + u3[K, J, I - 1] + u3[K, J - 1, I] + u3[K, J - 1, I - 1]
                 - u3[K - 1, J, I] - u3[K - 1, J, I - 1] - u3[K - 1, J - 1, I] - u3[K - 1, J - 1, I - 1]) / dx3
    return np.abs(d1 + d2 + d3)


def geom_records(geom, grid, idx2d):
    """CENT records [HARM_NGF][n] at flattened (j*n1e+i) positions"""
    cent = geom[0].reshape(geom.shape[1], -1)
    return np.ascontiguousarray(cent[:, idx2d])


DUMP_NCOL = 52


def read_dump(path, fmt="text"):
    """Parse a main dump file in the reference's layout (dump_header_general dump.c:320 and
    the rows of dump_content dump.c:449): returns (header dict, columns [cells][52])."""
    import struct
    names = ["t", "n1", "n2", "n3", "startx1", "startx2", "startx3", "dx1", "dx2", "dx3", "nstep", "gam", "a",
             "R0", "Rin", "Rout", "hslope", "dt", "MBH", "QBH", "is", "ie", "js", "je", "ks", "ke", "whichdump",
             "version", "ncol"]
    with open(path, "rb") as f:
        data = f.read()
    if fmt == "binary":
        layout = "<d3i6dq9d9i"
        size = struct.calcsize(layout)
        head = dict(zip(names, struct.unpack(layout, data[:size])))
        body = np.frombuffer(data[size:], dtype=np.float64)
    else:
        nl = data.index(b"\n")
        tok = data[:nl].split()
        text_names = names[:18] + ["defcoord"] + names[18:]
        conv = [float] + [int] * 3 + [float] * 6 + [int] + [float] * 7 + [int] + [float] * 2 + [int] * 9
        head = {n: c(t) for n, c, t in zip(text_names, conv, tok)}
        rest = data[nl + 1:]
        body = np.frombuffer(rest, dtype=np.float64) if fmt == "mixed" else np.array(rest.split(), dtype=np.float64)
    return head, body.reshape(-1, head["ncol"])


def harm_with_env(g, geom, conn, aux, **env):
    """a device context created with the given environment settings (HARM_B200_MLP_ENGINE,
    HARM_B200_MLP_GATE, ...), which a context reads once at creation"""
    import os

    from harm_harm_b200 import Harm
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        return Harm(g, geom, conn, aux)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def divb_rel(grid, geom, P):
    """max of the corner divergence of sqrt(-g) B relative to max |sqrt(-g) B| / min dx (the
    size a divergence of the field itself would have)"""
    g = grid.g
    U = np.abs(P[5:8] * geom[0, 26][None, None, :, :])
    dxs = [g.dx[1], g.dx[2]] + ([g.dx[3]] if g.n3 > 1 else [])
    return float(divb_corner(grid, geom, P).max() / (U.max() / min(dxs)))
