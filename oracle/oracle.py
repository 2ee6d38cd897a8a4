"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/build/liborc.so).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
product package.  See oracle/harm_oracle.h for what the oracle restates and its parity status.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "liborc.so")


class orc(C.Structure):
    pass


def _import_grid():
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from harm_harm_b200 import _native as N  # noqa
    return N


N = _import_grid()

orc._fields_ = [("g", N.harm_grid), ("geom", C.c_void_p), ("conn", C.c_void_p), ("aux", C.c_void_p),
                ("plane", C.c_size_t), ("cells", C.c_size_t), ("nthreads", C.c_int)]

_lib = None


def build() -> str:
    r = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P, D, I = C.c_void_p, C.c_double, C.c_int
        sigs = {
            "orc_init": (None, [C.POINTER(orc), C.POINTER(N.harm_grid), P, P, P, I]),
            "orc_primtoU_point": (None, [P, P, P]),
            "orc_primtoflux_point": (None, [P, P, I, P]),
            "orc_utoprimgen_point": (I, [C.POINTER(N.harm_grid), P, P, P, P, P]),
            "orc_vchar_point": (None, [C.POINTER(N.harm_grid), P, P, I, C.POINTER(D), C.POINTER(D)]),
            "orc_bound": (I, [C.POINTER(orc), P]),
            "orc_bound_dir": (I, [C.POINTER(orc), P, I, I]),
            "orc_fluxcalc": (I, [C.POINTER(orc), P, P, P, P, P]),
            "orc_advance": (I, [C.POINTER(orc), I, I, P, P, P, P, D, P, P, C.POINTER(D), C.POINTER(N.harm_stats)]),
            "orc_post_fixup": (I, [C.POINTER(orc), P, P, I]),
            "orc_advance_u": (I, [C.POINTER(orc), I, I, P, P, P, P, P, P, P, D, P, P, P, P]),
            "orc_step": (I, [C.POINTER(orc), P, C.POINTER(D), C.POINTER(N.harm_stats)]),
            "orc_reconstruct_line": (None, [I, I, P, P, P]),
            "orc_paraline_flattener": (None, [I, P, P, P]),
            "orc_reconstruct_line_paraline": (None, [I, P, P, P, P, P]),
            "orc_paraline_line_fi": (None, [C.POINTER(orc), P, I, I, I, P]),
            "orc_mlp_nparams": (I, []),
            "orc_mlp_features": (None, [C.POINTER(N.harm_grid), P, P, P, P, P]),
            "orc_mlp_loss_grad": (D, [I, P, P, P, P, P, P]),
            "orc_dump_row": (None, [C.POINTER(orc), P, P, I, I, I, P]),
        }
        for fn, (res, args) in sigs.items():
            f = getattr(L, fn)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data


class Oracle:
    """CPU restatement of the step over the same inputs as the device path."""

    def __init__(self, grid, geom, conn, aux, nthreads: int | None = None):
        self.grid = grid
        self._keep = (np.ascontiguousarray(geom), np.ascontiguousarray(conn), np.ascontiguousarray(aux))
        self.o = orc()
        nt = nthreads or os.cpu_count() or 1
        lib().orc_init(C.byref(self.o), C.byref(grid.g), _p(self._keep[0]), _p(self._keep[1]), _p(self._keep[2]), nt)

    def bound_prim(self, P):
        lib().orc_bound(C.byref(self.o), _p(P))

    def bound_dir(self, P, d, simple=False):
        """one direction of bound_prim; simple: one ghost layer (BOUNDPRIMSIMPLETYPE)"""
        lib().orc_bound_dir(C.byref(self.o), _p(P), int(d), int(bool(simple)))

    def fluxcalc(self, pb, F1, F2, F3):
        ndt = (C.c_double * 3)()
        lib().orc_fluxcalc(C.byref(self.o), _p(pb), _p(F1), _p(F2), _p(F3), ndt)
        return tuple(ndt)

    def advance(self, timeorder, pi, pb, pf, pflag, dt, numtimeorders=2, CUf=None, Cunew=None):
        from harm_harm_b200.harm import RK2_CUF, RK2_CUNEW
        CUf = np.array(RK2_CUF[timeorder] if CUf is None else CUf, dtype=np.float64)
        Cun = np.array(RK2_CUNEW[timeorder] if Cunew is None else Cunew, dtype=np.float64)
        ndt = C.c_double()
        st = N.harm_stats()
        lib().orc_advance(C.byref(self.o), timeorder, numtimeorders, _p(pi), _p(pb), _p(pf), _p(pflag), dt, _p(CUf),
                          _p(Cun), C.byref(ndt), C.byref(st))
        return ndt.value, st.as_dict()

    def advance_u(self, timeorder, numtimeorders, pi, pb, pf, pflag, ui, uf, ucum, dt, CUf, Cunew):
        """advance with the RK step's conserved arrays ui, uf, ucum ([8][k][j][i], carried
        across the substeps by the caller)"""
        CUf = np.ascontiguousarray(CUf, dtype=np.float64)
        Cun = np.ascontiguousarray(Cunew, dtype=np.float64)
        ndt = C.c_double()
        st = N.harm_stats()
        lib().orc_advance_u(C.byref(self.o), timeorder, numtimeorders, _p(pi), _p(pb), _p(pf), _p(pflag), _p(ui),
                            _p(uf), _p(ucum), dt, _p(CUf), _p(Cun), C.byref(ndt), C.byref(st))
        return ndt.value, st.as_dict()

    def post_fixup(self, pf, pflag, finalstep: int = 1):
        lib().orc_post_fixup(C.byref(self.o), _p(pf), _p(pflag), int(finalstep))

    def dump_rows(self, P, cells, U=None):
        """the main dump's 52 columns (dump_content, dump.c:449) of the active cells (i, j, k)"""
        Pc = np.ascontiguousarray(P, dtype=np.float64)
        Uc = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        out = np.zeros((len(cells), 52))
        row = np.zeros(52)
        for n, (i, j, k) in enumerate(cells):
            lib().orc_dump_row(C.byref(self.o), _p(Pc), None if Uc is None else _p(Uc), int(i), int(j), int(k), _p(row))
            out[n] = row
        return out

    def paraline_line_fi(self, P, d, a, b):
        """PARALINE flattening coefficients fluxcalc uses on the line along direction d through
        the transverse active-relative indices (a, b); length = the line's extended size"""
        Pc = np.ascontiguousarray(P, dtype=np.float64)
        gg = self.grid.g
        n = {1: gg.n1e, 2: gg.n2e, 3: gg.n3e}[d]
        Fi = np.zeros(n)
        lib().orc_paraline_line_fi(C.byref(self.o), _p(Pc), int(d), int(a), int(b), _p(Fi))
        return Fi

    def step_ch(self, P, dt):
        d = C.c_double(dt)
        st = N.harm_stats()
        lib().orc_step(C.byref(self.o), _p(P), C.byref(d), C.byref(st))
        return d.value, st.as_dict()


def _c(a, dtype=np.float64):
    """C-contiguous array of `dtype` (the caller keeps it alive across the C call)"""
    return np.ascontiguousarray(a, dtype=dtype)


def utoprimgen_point(grid, geomrec, U, pr):
    pr = _c(pr).copy()
    rec, Uc = _c(geomrec), _c(U)
    flag = np.zeros(1, dtype=np.int8)
    it = np.zeros(1, dtype=np.int32)
    lib().orc_utoprimgen_point(C.byref(grid.g), _p(rec), _p(Uc), _p(pr), _p(flag), _p(it))
    return pr, int(flag[0]), int(it[0])


def primtoU_point(geomrec, pr):
    U = np.zeros(8)
    rec, prc = _c(geomrec), _c(pr)
    lib().orc_primtoU_point(_p(rec), _p(prc), _p(U))
    return U


def primtoflux_point(geomrec, pr, d):
    F = np.zeros(8)
    rec, prc = _c(geomrec), _c(pr)
    lib().orc_primtoflux_point(_p(rec), _p(prc), d, _p(F))
    return F


def reconstruct_line(lim, y):
    y = _c(y)
    yl = np.zeros_like(y)
    yr = np.zeros_like(y)
    lib().orc_reconstruct_line(lim, len(y), _p(y), _p(yl), _p(yr))
    return yl, yr


def paraline_flattener(V, P):
    """PARALINE flattening coefficient of each cell of a line (0 where the +-3 stencil does not fit)"""
    V, P = _c(V), _c(P)
    Fi = np.zeros_like(V)
    lib().orc_paraline_flattener(len(V), _p(V), _p(P), _p(Fi))
    return Fi


def reconstruct_line_paraline(y, V, P):
    """PARALINE edges of a line with the flattening of V = sqrt(-g) rho u^dir and P = p + b^2/2"""
    y, V, P = _c(y), _c(V), _c(P)
    yl = np.zeros_like(y)
    yr = np.zeros_like(y)
    lib().orc_reconstruct_line_paraline(len(y), _p(y), _p(V), _p(P), _p(yl), _p(yr))
    return yl, yr


def mlp_features(grid, geomrec, U, P=None):
    """features (10) and, with P, targets (2) of one point"""
    f = np.zeros(10, dtype=np.float32)
    t = np.zeros(2, dtype=np.float32)
    rec, Uc = _c(geomrec), _c(U)
    Pc = None if P is None else _c(P)
    lib().orc_mlp_features(C.byref(grid.g), _p(rec), _p(Uc), None if Pc is None else _p(Pc), _p(f), _p(t))
    return f, t


def mlp_loss_grad(feat, targ, params, norm):
    """double-precision loss, gradient and de-standardised outputs of the network"""
    feat = _c(feat, np.float32)
    n = feat.shape[0]
    params = _c(params, np.float32)
    norm = _c(norm, np.float32)
    targ = None if targ is None else _c(targ, np.float32)
    pred = np.zeros((n, 2))
    grad = np.zeros(lib().orc_mlp_nparams())
    loss = lib().orc_mlp_loss_grad(n, _p(feat), None if targ is None else _p(targ), _p(params), _p(norm), _p(pred),
                                   _p(grad))
    return loss, grad, pred
