"""ctypes bindings of libharm_host.so and libharm_b200.so (include/harm_b200.h)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.environ.get("HARM_B200_LIBDIR") or os.path.join(HERE, "lib")

HARM_NPR = 8
HARM_LIM_MC, HARM_LIM_PARA, HARM_LIM_WENO5, HARM_LIM_PARALINE = 0, 1, 2, 3
HARM_FLUX_HLL, HARM_FLUX_LAXF = 0, 1
HARM_PREC_FP64, HARM_PREC_MIXED, HARM_PREC_FP64_FMA = 0, 1, 2
HARM_GUESS_PREV, HARM_GUESS_MLP = 0, 1
HARM_LOC_CENT, HARM_LOC_FACE1, HARM_LOC_FACE2, HARM_LOC_CORN3 = 0, 1, 2, 3
HARM_NLOC = 4
HARM_NGF = 28
HARM_NAUX = 3
HARM_G_GCOV, HARM_G_GCON, HARM_G_GCOVPERT_TT, HARM_G_ALPHA = 0, 10, 20, 21
HARM_G_BETASQOALPHASQ, HARM_G_BETA, HARM_G_GDET, HARM_G_IGDET = 22, 23, 26, 27
HARM_AUX_R, HARM_AUX_RHOFLOOR, HARM_AUX_UFLOOR = 0, 1, 2
HARM_NOALLOC_MAX_CELLS = 2097152
HARM_MLP_NIN, HARM_MLP_NOUT, HARM_MLP_NPARAMS, HARM_MLP_NNORM = 10, 2, 9154, 24


class harm_grid(C.Structure):
    _fields_ = [
        ("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int), ("ng", C.c_int),
        ("n1e", C.c_int), ("n2e", C.c_int), ("n3e", C.c_int), ("ng3", C.c_int),
        ("lim", C.c_int), ("fluxmethod", C.c_int),
        ("startx", C.c_double * 4), ("dx", C.c_double * 4),
        ("a", C.c_double), ("hslope", C.c_double), ("R0", C.c_double), ("Rin", C.c_double),
        ("Rout", C.c_double), ("Rhor", C.c_double), ("gam", C.c_double), ("cour", C.c_double),
        ("defcon", C.c_double), ("safe", C.c_double), ("rho_floor_coef", C.c_double),
        ("u_floor_coef", C.c_double), ("gammamax", C.c_double), ("gammafail", C.c_double),
    ]


class harm_stats(C.Structure):
    _fields_ = [("newton_iters", C.c_double), ("cells_inverted", C.c_double),
                ("mlp_fallbacks", C.c_double), ("inversion_failures", C.c_double),
                ("floor_hits", C.c_double), ("mlp_cells", C.c_double)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


P = C.c_void_p
D = C.c_double
Ip = C.c_int

_DEVICE_SIGS = {
    "harm_b200_create": (Ip, [C.POINTER(harm_grid), P, P, P, Ip, C.POINTER(P)]),
    "harm_b200_create_grid": (Ip, [C.POINTER(harm_grid), Ip, C.POINTER(P)]),
    "harm_b200_get_tables": (Ip, [P, P, P, P]),
    "harm_b200_dump": (Ip, [P, P, P, C.c_double, C.c_double, C.c_long, Ip, C.c_char_p]),
    "harm_b200_destroy": (Ip, [P]),
    "harm_b200_stream": (P, [P]),
    "harm_b200_launch_count": (C.c_ulonglong, [P]),
    "harm_b200_bound": (Ip, [P, P]),
    "harm_b200_fluxcalc": (Ip, [P, Ip, P, P, P, P, C.POINTER(D)]),
    "harm_b200_advance": (Ip, [P, Ip, Ip, Ip, Ip, P, P, P, P, D, C.POINTER(D), C.POINTER(D), C.POINTER(D),
                               C.POINTER(harm_stats)]),
    "harm_b200_post_fixup": (Ip, [P, P, P, Ip]),
    "harm_b200_advance_u": (Ip, [P, Ip, Ip, Ip, Ip, P, P, P, P, P, P, P, D, C.POINTER(D), C.POINTER(D), C.POINTER(D),
                                 C.POINTER(harm_stats)]),
    "harm_b200_from_harm_layout": (Ip, [P, P, P]),
    "harm_b200_to_harm_layout": (Ip, [P, P, P]),
    "harm_b200_flags_to_harm": (Ip, [P, P, P, Ip]),
    "harm_b200_flags_from_harm": (Ip, [P, P, P, Ip]),
    "harm_b200_mixed_reciprocal": (Ip, [P, P, P, C.c_size_t]),
    "harm_b200_step_host_harm": (Ip, [P, Ip, Ip, P, C.POINTER(D), C.POINTER(harm_stats)]),
    "harm_b200_step": (Ip, [P, Ip, Ip, P, C.POINTER(D), C.POINTER(harm_stats)]),
    "harm_b200_step_n": (Ip, [P, Ip, Ip, P, Ip, C.POINTER(D), C.POINTER(harm_stats)]),
    "harm_b200_step_host": (Ip, [P, Ip, Ip, P, C.POINTER(D), C.POINTER(harm_stats)]),
    "harm_b200_step_host_n": (Ip, [P, Ip, Ip, P, Ip, C.POINTER(D), C.POINTER(harm_stats)]),
    "harm_b200_utoprimgen_points": (Ip, [P, C.c_size_t, Ip, P, P, P, P, P]),
    "harm_b200_time_stages": (Ip, [P, Ip, Ip, P, D, Ip, C.POINTER(D)]),
    "harm_b200_fluxcalc_noalloc": (Ip, [C.POINTER(harm_grid), P, P, P, P, P, C.POINTER(D), P]),
    "harm_b200_mlp_dump": (Ip, [P, P, Ip, Ip, C.c_size_t, P, P, P, C.POINTER(C.c_size_t)]),
    "harm_b200_mlp_synth": (Ip, [P, C.c_size_t, C.c_uint64, P, P, P, P, P]),
    "harm_b200_mlp_norm": (Ip, [P, C.c_size_t, P, P, P]),
    "harm_b200_mlp_init": (Ip, [P, C.c_uint64, P]),
    "harm_b200_mlp_loss_grad": (Ip, [P, C.c_size_t, P, P, P, P, C.POINTER(D), P]),
    "harm_b200_mlp_train": (Ip, [P, C.c_size_t, P, P, P, P, Ip, Ip, C.c_float, C.c_uint64, P]),
    "harm_b200_mlp_set": (Ip, [P, P, P, D]),
    "harm_b200_mlp_predict": (Ip, [P, C.c_size_t, P, P]),
    "harm_b200_last_error": (C.c_char_p, []),
}

_HOST_SIGS = {
    "harm_grid_setup": (Ip, [C.POINTER(harm_grid), Ip, Ip, Ip, Ip, D, D, D, D]),
    "harm_geometry_build": (Ip, [C.POINTER(harm_grid), P, P, P]),
    "harm_torus_init": (Ip, [C.POINTER(harm_grid), P, P, D, C.c_uint64, P]),
}

_libs: dict[str, C.CDLL] = {}


def _load(name: str, sigs: dict) -> C.CDLL:
    if name in _libs:
        return _libs[name]
    path = os.path.join(LIBDIR, name)
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is not built; run harm_harm_b200.build.build_all() (the device path has no CPU fallback)")
    lib = C.CDLL(path)
    for fn, (res, args) in sigs.items():
        f = getattr(lib, fn)
        f.restype = res
        f.argtypes = args
    _libs[name] = lib
    return lib


def device_lib() -> C.CDLL:
    return _load("libharm_b200.so", _DEVICE_SIGS)


def host_lib() -> C.CDLL:
    return _load("libharm_host.so", _HOST_SIGS)


def device_symbols() -> list[str]:
    return list(_DEVICE_SIGS)


def host_symbols() -> list[str]:
    return list(_HOST_SIGS)
