"""harm_harm_b200 -- B200-native per-timestep GRMHD update of HARM (pseudotensor/harm_harm).

The numeric path lives in lib/libharm_b200.so (sm_100a kernels behind the C ABI declared in
include/harm_b200.h); lib/libharm_host.so produces the inputs (grid, metric tables, torus
initial state).  This package is the host-side mirror of the reference's interface.
"""
from ._native import (HARM_FLUX_HLL, HARM_FLUX_LAXF, HARM_GUESS_MLP, HARM_GUESS_PREV, HARM_LIM_MC, HARM_LIM_PARA,
                      HARM_LIM_PARALINE, HARM_LIM_WENO5, HARM_NPR, HARM_PREC_FP64, HARM_PREC_FP64_FMA, HARM_PREC_MIXED)
from .harm import Grid, Harm

__all__ = ["Grid", "Harm", "HARM_NPR", "HARM_LIM_MC", "HARM_LIM_PARA", "HARM_LIM_WENO5", "HARM_LIM_PARALINE",
           "HARM_FLUX_HLL", "HARM_FLUX_LAXF",
           "HARM_PREC_FP64", "HARM_PREC_FP64_FMA", "HARM_PREC_MIXED", "HARM_GUESS_PREV", "HARM_GUESS_MLP"]
