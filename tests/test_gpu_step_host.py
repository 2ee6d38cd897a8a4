"""harm_b200_step_host (the host-buffer entry point) against harm_b200_step on the same state.
The host entry point copies the state in slabs of k-planes and starts the first substep's
flux tiles of each slab while later slabs are still in flight; the results must be those of
the device-array step, bit for bit, including the x3 tile rows that wait for planes of later
slabs (n3 = 96: four rows of 32 faces)."""
import numpy as np
import pytest

from helpers import make_torus
from harm_harm_b200 import HARM_PREC_FP64, HARM_PREC_MIXED, Harm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,lim", [((24, 16, 96), 2), ((32, 24, 16), 3), ((64, 64, 1), 0)])
@pytest.mark.parametrize("precision", [HARM_PREC_FP64, HARM_PREC_MIXED])
@pytest.mark.parametrize("pinned", [True, False])
def test_step_host_equals_device_step(cuda, shape, lim, precision, pinned):
    g, geom, conn, aux, P = make_torus(*shape, lim=lim)
    dev = Harm(g, geom, conn, aux)
    Pd = cuda.from_numpy(P.copy()).cuda()
    dev.bound_prim(Pd)
    P0 = Pd.cpu().numpy()
    Ph = cuda.from_numpy(P0.copy())
    if pinned:
        Ph = Ph.pin_memory()
    Ph = Ph.numpy()
    dt0 = 1e-3
    dt_d, st_d = dev.step_ch(Pd, dt0, precision=precision)
    dt_h, st_h = dev.step_ch_host(Ph, dt0, precision=precision)
    assert np.array_equal(Pd.cpu().numpy(), Ph)
    assert dt_h == dt_d
    assert st_h["newton_iters"] == st_d["newton_iters"]
    # a second step from the result: the copy stream and its events are reused
    dt_d2, _ = dev.step_ch(Pd, dt_d, precision=precision)
    dt_h2, _ = dev.step_ch_host(Ph, dt_h, precision=precision)
    assert np.array_equal(Pd.cpu().numpy(), Ph) and dt_h2 == dt_d2
    dev.close()
