"""harm_b200_advance with the coefficient sets of setup_rktimestep (step_ch.c:1171): the
forward-Euler set (TIMEORDER 1) matches the oracle like the RK2 midpoint does; sets that carry
U_f or ucum from one substep to the next (TVD RK2, RK3, RK4), which the device update does not
keep, are refused with code 2 before any work is queued."""
import numpy as np
import pytest

from helpers import make_torus, rel_err
from harm_harm_b200 import Harm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _setup(cuda):
    g, geom, conn, aux, P = make_torus(32, 24, 8)
    orc = O.Oracle(g, geom, conn, aux)
    orc.bound_prim(P)
    return g, geom, conn, aux, P, orc, Harm(g, geom, conn, aux)


def test_forward_euler_substep_matches_oracle(cuda):
    g, geom, conn, aux, P, orc, dev = _setup(cuda)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    dt = 1.0 / sum(1.0 / x for x in ndt)
    CUf, Cun = (1.0, 0.0, 1.0, 0.0), (0.0, 0.0, 1.0, 0.0)
    pf_o = np.zeros_like(P)
    fl_o = np.zeros(P.shape[1:], dtype=np.int8)
    ndt_o, _ = orc.advance(0, P, P, pf_o, fl_o, dt, numtimeorders=1, CUf=CUf, Cunew=Cun)
    Pd = cuda.from_numpy(P.copy()).cuda()
    pf_d = cuda.zeros_like(Pd)
    fl_d = cuda.zeros(P.shape[1:], dtype=cuda.int8, device="cuda")
    ndt_d, _ = dev.advance(0, Pd, Pd, pf_d, fl_d, dt, numtimeorders=1, CUf=CUf, Cunew=Cun)
    act = (slice(None),) + g.active
    a, b = pf_d.cpu().numpy()[act], pf_o[act]
    for pl in range(8):
        assert rel_err(a[pl], b[pl]) < 1e-12, (pl, rel_err(a[pl], b[pl]))
    assert abs(ndt_d - ndt_o) <= 1e-12 * ndt_o
    dev.close()


@pytest.mark.parametrize("timeorder,numtimeorders,CUf,Cun", [
    (1, 2, (0.5, 0.5, 0.5, 0.0), (0.0, 0.0, 1.0, 1.0)),                  # TVD RK2, second substep
    (1, 3, (0.75, 0.25, 0.25, 0.0), (0.0, 0.0, 0.0, 1.0)),               # RK3, second substep
    (0, 4, (1.0, 0.0, 0.5, 0.0), (1.0, 1.0 / 6.0, 0.0, 0.0)),            # RK4, first substep
    (2, 2, (1.0, 0.0, 1.0, 0.0), (0.0, 0.0, 1.0, 0.5)),                  # timeorder out of range
])
def test_coefficients_that_carry_state_are_refused(cuda, timeorder, numtimeorders, CUf, Cun):
    g, geom, conn, aux, P, orc, dev = _setup(cuda)
    Pd = cuda.from_numpy(P.copy()).cuda()
    pf_d = cuda.zeros_like(Pd)
    fl_d = cuda.zeros(P.shape[1:], dtype=cuda.int8, device="cuda")
    with pytest.raises(RuntimeError) as e:
        dev.advance(timeorder, Pd, Pd, pf_d, fl_d, 1e-3, numtimeorders=numtimeorders, CUf=CUf, Cunew=Cun)
    assert "failed (2)" in str(e.value), str(e.value)
    assert float(pf_d.abs().max()) == 0.0  # nothing was written
    dev.close()
