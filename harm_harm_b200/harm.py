"""Host-side mirror of HARM's per-timestep interface over the B200 device path.

The names follow the reference's entry points so that a caller of HARM's hot path finds
the same operations:

    Grid / geometry / torus_init   set_points+set_grid+init (coord.c:2038, set_grid.c:114,
                                   initboundcode/init.fishmon.c:403)
    Harm.bound_prim                bound_prim (step_ch.c:1332)
    Harm.fluxcalc                  fluxcalc (flux.c:38)
    Harm.advance                   advance (advance.c:85)
    Harm.post_fixup                post_fixup (fixup.c:53)
    Harm.Utoprimgen                Utoprimgen (utoprimgen.c:32), over a batch of points
    Harm.step_ch                   step_ch_full (step_ch.c:35): one full RK2 step
    Harm.mlp_*                     the learned starting point of the inversion (replaces
                                   set_guess_Wp utoprim_jon.c:890 under HARM_GUESS_MLP):
                                   training pairs, training, packing, inference

Device arrays are torch CUDA tensors (torch is only the allocator and stream owner here);
every numeric routine runs in libharm_b200.so.  Errors are raised as RuntimeError with the
library's message (HARM's MYFUN/FAILSTATEMENT convention of non-zero returns).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N

RK2_CUF = ((1.0, 0.0, 0.5, 0.0), (1.0, 0.0, 1.0, 0.0))   # setup_rktimestep step_ch.c:1244-1266
RK2_CUNEW = ((0.0, 0.0, 0.0, 0.0), (0.0, 0.0, 1.0, 0.5))


def _torch_cuda():
    """torch, when it is already imported and has CUDA; None otherwise"""
    import sys
    torch = sys.modules.get("torch")
    if torch is None or not torch.cuda.is_available():
        return None
    return torch


def _ptr(a) -> int:
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    raise TypeError(type(a))


@dataclass
class Grid:
    g: N.harm_grid

    @classmethod
    def torus(cls, n1: int, n2: int, n3: int, lim: int = N.HARM_LIM_MC, a: float = 0.9375,
              hslope: float = 0.3, Rout: float = 40.0, cour: float = 0.8,
              fluxmethod: int = N.HARM_FLUX_HLL) -> "Grid":
        g = N.harm_grid()
        rc = N.host_lib().harm_grid_setup(C.byref(g), n1, n2, n3, lim, a, hslope, Rout, cour)
        if rc:
            raise RuntimeError(f"harm_grid_setup failed ({rc})")
        g.fluxmethod = fluxmethod
        return cls(g)

    @property
    def shape(self):
        return (N.HARM_NPR, self.g.n3e, self.g.n2e, self.g.n1e)

    @property
    def cells(self) -> int:
        return self.g.n1e * self.g.n2e * self.g.n3e

    @property
    def active(self):
        """slices of the active cells in a [pl][k][j][i] array"""
        g = self.g
        return (slice(g.ng3, g.ng3 + g.n3), slice(g.ng, g.ng + g.n2), slice(g.ng, g.ng + g.n1))

    def geometry(self):
        g = self.g
        plane = g.n1e * g.n2e
        geom = np.zeros((N.HARM_NLOC, N.HARM_NGF, g.n2e, g.n1e))
        conn = np.zeros((64, g.n2e, g.n1e))
        aux = np.zeros((N.HARM_NAUX, g.n2e, g.n1e))
        rc = N.host_lib().harm_geometry_build(C.byref(g), _ptr(geom), _ptr(conn), _ptr(aux))
        if rc:
            raise RuntimeError("harm_geometry_build failed")
        assert geom.size == N.HARM_NLOC * N.HARM_NGF * plane
        return geom, conn, aux

    def torus_init(self, geom, aux, beta_min: float = 100.0, seed: int = 12345) -> np.ndarray:
        P = np.zeros(self.shape)
        rc = N.host_lib().harm_torus_init(C.byref(self.g), _ptr(geom), _ptr(aux), beta_min, seed, _ptr(P))
        if rc:
            raise RuntimeError(f"harm_torus_init failed ({rc})")
        return P


class Harm:
    """One grid on one GPU: the device context of libharm_b200.so."""

    def __init__(self, grid: Grid, geom: np.ndarray | None = None, conn: np.ndarray | None = None,
                 aux: np.ndarray | None = None, device: int = 0):
        """Upload the host-built tables (geom, conn, aux), or, when all three are None, build
        the metric, connection and floor tables on the device (harm_b200_create_grid)."""
        self.grid = grid
        self.lib = N.device_lib()
        self._ctx = C.c_void_p()
        self._ext = None
        if geom is None and conn is None and aux is None:
            rc = self.lib.harm_b200_create_grid(C.byref(grid.g), device, C.byref(self._ctx))
            self._check(rc, "harm_b200_create_grid")
            return
        geom = np.ascontiguousarray(geom, dtype=np.float64)
        conn = np.ascontiguousarray(conn, dtype=np.float64)
        aux = np.ascontiguousarray(aux, dtype=np.float64)
        rc = self.lib.harm_b200_create(C.byref(grid.g), _ptr(geom), _ptr(conn), _ptr(aux), device,
                                       C.byref(self._ctx))
        self._check(rc, "harm_b200_create")

    def dump(self, P, path: str, t: float = 0.0, dt: float = 0.0, nstep: int = 0, U=None, fmt: str = "text") -> None:
        """the reference's main dump file of P (bounded ghost zones) at `path`: "text" (the
        reference's default), "binary" or "mixed" (harm_b200_dump)"""
        code = {"text": 0, "binary": 1, "mixed": 2}[fmt]
        rc = self._ordered(self.lib.harm_b200_dump, self._ctx, _ptr(P), None if U is None else _ptr(U), float(t), float(dt), int(nstep),
                                     code, path.encode())
        self._check(rc, "harm_b200_dump")

    def tables(self):
        """The context's metric, connection and floor tables as host arrays
        (geom[4][28][n2e][n1e], conn[64][n2e][n1e], aux[3][n2e][n1e])."""
        g = self.grid.g
        geom = np.empty((4, 28, g.n2e, g.n1e), dtype=np.float64)
        conn = np.empty((64, g.n2e, g.n1e), dtype=np.float64)
        aux = np.empty((3, g.n2e, g.n1e), dtype=np.float64)
        self._check(self._ordered(self.lib.harm_b200_get_tables, self._ctx, _ptr(geom), _ptr(conn), _ptr(aux)), "get_tables")
        return geom, conn, aux

    def _check(self, rc: int, what: str) -> None:
        if rc:
            raise RuntimeError(f"{what} failed ({rc}): {self.lib.harm_b200_last_error().decode()}")

    def _ordered(self, fn, *args):
        """Call a library entry point in stream order with torch: the context's stream first
        waits for the work queued so far on torch's current stream (which may still be writing
        the arguments), and torch's stream then waits for the context's (which may still be
        writing the results).  The library enqueues on its own non-blocking stream."""
        torch = _torch_cuda()
        if torch is None:
            return fn(*args)
        if self._ext is None:
            self._ext = torch.cuda.ExternalStream(self.stream_ptr)
        cur = torch.cuda.current_stream()
        self._ext.wait_stream(cur)
        rc = fn(*args)
        cur.wait_stream(self._ext)
        return rc

    def close(self) -> None:
        if self._ctx:
            self.lib.harm_b200_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(self.lib.harm_b200_launch_count(self._ctx))

    @property
    def stream_ptr(self) -> int:
        return self.lib.harm_b200_stream(self._ctx)

    # ---------------------------------------------------------------- reference API
    def bound_prim(self, P) -> None:
        self._check(self._ordered(self.lib.harm_b200_bound, self._ctx, _ptr(P)), "bound_prim")

    def fluxcalc(self, pb, F1, F2, F3, precision: int = N.HARM_PREC_FP64):
        ndt = (C.c_double * 3)()
        self._check(self._ordered(self.lib.harm_b200_fluxcalc, self._ctx, precision, _ptr(pb), _ptr(F1), _ptr(F2), _ptr(F3), ndt),
                    "fluxcalc")
        return tuple(ndt)

    def advance(self, timeorder: int, pi, pb, pf, pflag, dt: float, precision: int = N.HARM_PREC_FP64,
                guess: int = N.HARM_GUESS_PREV, numtimeorders: int = 2, CUf=None, Cunew=None):
        """one RK substep; CUf/Cunew default to the RK2 midpoint's coefficients of this substep"""
        CUf = (C.c_double * 4)(*(RK2_CUF[timeorder] if CUf is None else CUf))
        Cun = (C.c_double * 4)(*(RK2_CUNEW[timeorder] if Cunew is None else Cunew))
        ndt = C.c_double()
        st = N.harm_stats()
        self._check(self._ordered(self.lib.harm_b200_advance, self._ctx, precision, guess, timeorder, numtimeorders, _ptr(pi), _ptr(pb),
                                               _ptr(pf), _ptr(pflag), dt, CUf, Cun, C.byref(ndt), C.byref(st)),
                    "advance")
        return ndt.value, st.as_dict()

    def advance_u(self, timeorder: int, numtimeorders: int, pi, pb, pf, pflag, ui, uf, ucum, dt: float, CUf, Cunew,
                  precision: int = N.HARM_PREC_FP64, guess: int = N.HARM_GUESS_PREV):
        """one RK substep with the step's conserved arrays ui, uf, ucum (advance.c:85-91): every
        coefficient set of setup_rktimestep"""
        CUf = (C.c_double * 4)(*CUf)
        Cun = (C.c_double * 4)(*Cunew)
        ndt = C.c_double()
        st = N.harm_stats()
        self._check(self._ordered(self.lib.harm_b200_advance_u, self._ctx, precision, guess, timeorder, numtimeorders,
                                  _ptr(pi), _ptr(pb), _ptr(pf), _ptr(pflag), _ptr(ui), _ptr(uf), _ptr(ucum), dt, CUf, Cun,
                                  C.byref(ndt), C.byref(st)), "advance_u")
        return ndt.value, st.as_dict()

    def post_fixup(self, pf, pflag, finalstep: int = 1) -> None:
        self._check(self._ordered(self.lib.harm_b200_post_fixup, self._ctx, _ptr(pf), _ptr(pflag), int(finalstep)),
                    "post_fixup")

    def step_ch(self, P, dt: float, precision: int = N.HARM_PREC_FP64, guess: int = N.HARM_GUESS_PREV,
                nsteps: int = 1, stats: bool = True):
        d = C.c_double(dt)
        st = N.harm_stats()
        self._check(self._ordered(self.lib.harm_b200_step_n, self._ctx, precision, guess, _ptr(P), nsteps, C.byref(d),
                                              C.byref(st) if stats else None), "step_ch")
        return d.value, st.as_dict()

    def step_ch_host(self, P_host: np.ndarray, dt: float, precision: int = N.HARM_PREC_FP64,
                     guess: int = N.HARM_GUESS_PREV):
        d = C.c_double(dt)
        st = N.harm_stats()
        self._check(self._ordered(self.lib.harm_b200_step_host, self._ctx, precision, guess, _ptr(P_host), C.byref(d), C.byref(st)),
                    "step_ch_host")
        return d.value, st.as_dict()

    def step_ch_host_n(self, P_host: np.ndarray, dt: float, precision: int = N.HARM_PREC_FP64,
                       guess: int = N.HARM_GUESS_PREV, nsteps: int = 1):
        """nsteps steps over a host array, each copying the state in and out, with the copies
        of consecutive steps overlapped"""
        d = C.c_double(dt)
        st = N.harm_stats()
        self._check(self._ordered(self.lib.harm_b200_step_host_n, self._ctx, precision, guess, _ptr(P_host), nsteps,
                                  C.byref(d), C.byref(st)), "step_ch_host_n")
        return d.value, st.as_dict()

    def step_ch_host_harm(self, P_harm: np.ndarray, dt: float, precision: int = N.HARM_PREC_FP64,
                          guess: int = N.HARM_GUESS_PREV):
        """one step over a host array in HARM's [k][j][i][pl] layout"""
        d = C.c_double(dt)
        st = N.harm_stats()
        self._check(self._ordered(self.lib.harm_b200_step_host_harm, self._ctx, precision, guess, _ptr(P_harm), C.byref(d),
                                  C.byref(st)), "step_ch_host_harm")
        return d.value, st.as_dict()

    def from_harm_layout(self, P_harm, P) -> None:
        """[k][j][i][pl] (HARM's ORDERSTORAGE 5) -> [pl][k][j][i], device arrays"""
        self._check(self._ordered(self.lib.harm_b200_from_harm_layout, self._ctx, _ptr(P_harm), _ptr(P)), "from_harm_layout")

    def to_harm_layout(self, P, P_harm) -> None:
        self._check(self._ordered(self.lib.harm_b200_to_harm_layout, self._ctx, _ptr(P), _ptr(P_harm)), "to_harm_layout")

    def flags_to_harm(self, pflag, harm_pflag, numpflags: int) -> None:
        self._check(self._ordered(self.lib.harm_b200_flags_to_harm, self._ctx, _ptr(pflag), _ptr(harm_pflag), numpflags),
                    "flags_to_harm")

    def flags_from_harm(self, harm_pflag, pflag, numpflags: int) -> None:
        self._check(self._ordered(self.lib.harm_b200_flags_from_harm, self._ctx, _ptr(harm_pflag), _ptr(pflag), numpflags),
                    "flags_from_harm")

    def mixed_reciprocal(self, b, r) -> None:
        """r = the mixed inversion's reciprocal of b (device float64 arrays of equal size)"""
        assert b.numel() == r.numel()
        self._check(self._ordered(self.lib.harm_b200_mixed_reciprocal, self._ctx, _ptr(b), _ptr(r), b.numel()),
                    "mixed_reciprocal")

    def Utoprimgen(self, U, geomrec, P, pflag, iters=None, guess: int = N.HARM_GUESS_PREV) -> None:
        n = U.shape[-1]
        self._check(self._ordered(self.lib.harm_b200_utoprimgen_points, self._ctx, n, guess, _ptr(U), _ptr(geomrec), _ptr(P),
                                                         _ptr(pflag), _ptr(iters)), "Utoprimgen")

    def time_stages(self, P, dt: float, precision: int = N.HARM_PREC_FP64, guess: int = N.HARM_GUESS_PREV,
                    reps: int = 5) -> dict:
        ms = (C.c_double * 5)()
        self._check(self._ordered(self.lib.harm_b200_time_stages, self._ctx, precision, guess, _ptr(P), dt, reps, ms), "time_stages")
        return dict(zip(("flux", "emf", "update_invert", "bound", "post_fixup"), list(ms)))

    # ---------------------------------------------------------------- learned guess
    def mlp_dump(self, P, feat, targ, cell=None, stride: int = 1, phase: int = 0) -> int:
        """Training pairs from the most recent inversion of this context (its U and the
        primitives P it produced); returns the number written (at most len(feat))."""
        n = C.c_size_t()
        self._check(self._ordered(self.lib.harm_b200_mlp_dump, self._ctx, _ptr(P), stride, phase, feat.shape[0], _ptr(feat),
                                                _ptr(targ), _ptr(cell), C.byref(n)), "mlp_dump")
        return int(n.value)

    def mlp_synth(self, feat, targ, seed: int, U=None, P=None, cell=None) -> None:
        self._check(self._ordered(self.lib.harm_b200_mlp_synth, self._ctx, feat.shape[0], seed, _ptr(feat), _ptr(targ), _ptr(U),
                                                 _ptr(P), _ptr(cell)), "mlp_synth")

    def mlp_norm(self, feat, targ, norm, n: int | None = None) -> None:
        n = feat.shape[0] if n is None else n
        self._check(self._ordered(self.lib.harm_b200_mlp_norm, self._ctx, n, _ptr(feat), _ptr(targ), _ptr(norm)), "mlp_norm")

    def mlp_init(self, params, seed: int = 1) -> None:
        self._check(self._ordered(self.lib.harm_b200_mlp_init, self._ctx, seed, _ptr(params)), "mlp_init")

    def mlp_loss_grad(self, feat, targ, params, norm, grad, n: int | None = None) -> float:
        n = feat.shape[0] if n is None else n
        loss = C.c_double()
        self._check(self._ordered(self.lib.harm_b200_mlp_loss_grad, self._ctx, n, _ptr(feat), _ptr(targ), _ptr(params), _ptr(norm),
                                                     C.byref(loss), _ptr(grad)), "mlp_loss_grad")
        return loss.value

    def mlp_train(self, feat, targ, norm, params, steps: int, batch: int = 8192, lr: float = 3e-3, seed: int = 7,
                  n: int | None = None) -> np.ndarray:
        n = feat.shape[0] if n is None else n
        hist = np.zeros(steps, dtype=np.float32)
        self._check(self._ordered(self.lib.harm_b200_mlp_train, self._ctx, n, _ptr(feat), _ptr(targ), _ptr(norm), _ptr(params), steps,
                                                 batch, lr, seed, _ptr(hist)), "mlp_train")
        return hist

    def mlp_set(self, params, norm, start_bias: float = 0.0) -> None:
        self._check(self._ordered(self.lib.harm_b200_mlp_set, self._ctx, _ptr(params), _ptr(norm), start_bias), "mlp_set")

    def mlp_predict(self, feat, out, n: int | None = None) -> None:
        n = feat.shape[0] if n is None else n
        self._check(self._ordered(self.lib.harm_b200_mlp_predict, self._ctx, n, _ptr(feat), _ptr(out)), "mlp_predict")
