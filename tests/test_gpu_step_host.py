"""harm_b200_step_host and harm_b200_step_host_n (the host-buffer entry points) against
harm_b200_step on the same state.
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


@pytest.mark.parametrize("shape,lim", [((24, 16, 96), 2), ((64, 64, 1), 0)])
@pytest.mark.parametrize("precision", [HARM_PREC_FP64, HARM_PREC_MIXED])
@pytest.mark.parametrize("pinned", [True, False])
def test_step_host_n_equals_device_steps(cuda, shape, lim, precision, pinned):
    """harm_b200_step_host_n: four steps whose copies out and in overlap (the next step's
    copy in of a slab waits only for the copy out of that slab) equal four device-array
    steps bit for bit, dt and Newton counts included; a second call reuses the streams."""
    g, geom, conn, aux, P = make_torus(*shape, lim=lim)
    dev = Harm(g, geom, conn, aux)
    Pd = cuda.from_numpy(P.copy()).cuda()
    dev.bound_prim(Pd)
    Ph = cuda.from_numpy(Pd.cpu().numpy())
    if pinned:
        Ph = Ph.pin_memory()
    Ph = Ph.numpy()
    dt_d, st_d = dev.step_ch(Pd, 1e-3, precision=precision, nsteps=4)
    dt_h, st_h = dev.step_ch_host_n(Ph, 1e-3, precision=precision, nsteps=4)
    assert np.array_equal(Pd.cpu().numpy(), Ph)
    assert dt_h == dt_d
    assert st_h["newton_iters"] == st_d["newton_iters"]
    dt_d2, _ = dev.step_ch(Pd, dt_d, precision=precision, nsteps=3)
    dt_h2, _ = dev.step_ch_host_n(Ph, dt_h, precision=precision, nsteps=3)
    assert np.array_equal(Pd.cpu().numpy(), Ph) and dt_h2 == dt_d2
    dev.close()


def test_harm_layout_round_trip(cuda):
    """[k][j][i][pl] <-> [pl][k][j][i] on the device, and HARM's int flags[cell][NUMPFLAGS]"""
    torch = cuda
    g, geom, conn, aux, P = make_torus(40, 24, 12, lim=2)
    dev = Harm(g, geom, conn, aux)
    aos = np.ascontiguousarray(np.moveaxis(P, 0, 3))
    A = torch.from_numpy(aos).cuda()
    S = torch.zeros_like(torch.from_numpy(P)).cuda()
    dev.from_harm_layout(A, S)
    assert np.array_equal(S.cpu().numpy(), P)
    B = torch.zeros_like(A)
    dev.to_harm_layout(S, B)
    assert np.array_equal(B.cpu().numpy(), aos)
    rng = np.random.default_rng(1)
    fl = rng.integers(-3, 60, size=P.shape[1:]).astype(np.int8)
    F = torch.from_numpy(fl).cuda()
    H = torch.full(fl.shape + (3,), 7, dtype=torch.int32, device="cuda")
    dev.flags_to_harm(F, H, 3)
    h = H.cpu().numpy()
    assert np.array_equal(h[..., 0], fl.astype(np.int32)) and (h[..., 1:] == 7).all()
    F2 = torch.zeros_like(F)
    dev.flags_from_harm(H, F2, 3)
    assert np.array_equal(F2.cpu().numpy(), fl)
    dev.close()


@pytest.mark.parametrize("shape,lim", [((24, 16, 96), 2), ((64, 64, 1), 0)])
@pytest.mark.parametrize("precision", [HARM_PREC_FP64, HARM_PREC_MIXED])
def test_step_host_harm_layout_equals_device_step(cuda, shape, lim, precision):
    """the host-buffer step over HARM's [k][j][i][pl] layout (each arriving k-slab converted on
    the device ahead of the flux tiles that stage it) equals the device-array step bit for bit"""
    torch = cuda
    g, geom, conn, aux, P = make_torus(*shape, lim=lim)
    dev = Harm(g, geom, conn, aux)
    Pd = torch.from_numpy(P.copy()).cuda()
    dev.bound_prim(Pd)
    Ph = torch.from_numpy(np.ascontiguousarray(np.moveaxis(Pd.cpu().numpy(), 0, 3))).pin_memory().numpy()
    for _ in range(2):
        dt_d, st_d = dev.step_ch(Pd, 1e-3, precision=precision)
        dt_h, st_h = dev.step_ch_host_harm(Ph, 1e-3, precision=precision)
        assert np.array_equal(np.moveaxis(Pd.cpu().numpy(), 0, 3), Ph)
        assert dt_h == dt_d and st_h["newton_iters"] == st_d["newton_iters"]
    dev.close()
