"""GPU test of harm_b200_fluxcalc_noalloc, the flux entry point for callers that cannot
allocate device memory (for example code running inside a memory pool it does not own): it
keeps its scratch in a fixed device array instead of allocating, and must return the same
fluxes and CFL limits as harm_b200_fluxcalc.  Checked through the C ABI on two calls in a
row (the second on a different state, so stale scratch from the first call would show),
with the FP64 parity tolerance of the other tests (1e-12 relative).

This file is collected last so that a run stopping at the first failure has run every other
test before it; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import make_torus, rel_err
from harm_harm_b200 import Grid, Harm
from harm_harm_b200 import _native as N

pytestmark = pytest.mark.gpu


def _faces(g, d):
    gg = g.g
    k = slice(gg.ng3, gg.ng3 + gg.n3 + (1 if d == 3 else 0))
    j = slice(gg.ng, gg.ng + gg.n2 + (1 if d == 2 else 0))
    i = slice(gg.ng, gg.ng + gg.n1 + (1 if d == 1 else 0))
    return (slice(None), k, j, i)


@pytest.mark.parametrize("shape,lim,flux", [((40, 32, 16), 0, 0), ((40, 32, 16), 1, 0), ((40, 32, 16), 2, 0),
                                            ((40, 32, 16), 3, 1), ((64, 64, 1), 0, 0), ((64, 64, 1), 2, 0)])
def test_noalloc_fluxes_equal_fluxcalc_on_two_calls(cuda, shape, lim, flux):
    """3-D grids and the 2-D branch (no x3 fluxes, ndt[2] left at its no-limit value, the
    2-D EMF form)"""
    torch = cuda
    g, geom, conn, aux, P = make_torus(*shape, lim=lim, fluxmethod=flux)
    ndirs = 3 if shape[2] > 1 else 2
    assert g.cells <= N.HARM_NOALLOC_MAX_CELLS
    dev = Harm(g, geom, conn, aux)
    lib = N.device_lib()
    P0 = torch.from_numpy(P).cuda()
    dev.bound_prim(P0)
    P1 = P0.clone()
    P1[0] *= 1.03   # a different state for the second call
    P1[1] *= 0.97
    dev.bound_prim(P1)
    Gd = torch.from_numpy(np.ascontiguousarray(geom)).cuda()
    torch.cuda.synchronize()
    for S in (P0, P1):
        Fr = [torch.zeros_like(S) for _ in range(3)]
        ndt_r = dev.fluxcalc(S, *Fr)
        Fn = [torch.full_like(S, 7.0) for _ in range(3)]
        ndt = (C.c_double * 3)()
        rc = lib.harm_b200_fluxcalc_noalloc(C.byref(g.g), Gd.data_ptr(), S.data_ptr(), Fn[0].data_ptr(),
                                            Fn[1].data_ptr(), Fn[2].data_ptr(), ndt, None)
        assert rc == 0, lib.harm_b200_last_error().decode()
        torch.cuda.synchronize()
        for d in range(ndirs):
            a = Fn[d].cpu().numpy()[_faces(g, d + 1)]
            b = Fr[d].cpu().numpy()[_faces(g, d + 1)]
            for pl in range(8):
                e = rel_err(a[pl], b[pl])
                assert e < 1e-12, (d + 1, pl, e)
        for d in range(3):
            assert abs(ndt[d] - ndt_r[d]) <= 1e-12 * ndt_r[d], (d, ndt[d], ndt_r[d])
    dev.close()


def test_noalloc_rejects_grids_above_its_maximum(cuda):
    torch = cuda
    g = Grid.torus(200, 128, 100)
    assert g.cells > N.HARM_NOALLOC_MAX_CELLS
    lib = N.device_lib()
    x = torch.zeros(8, device="cuda", dtype=torch.float64)
    ndt = (C.c_double * 3)()
    p = x.data_ptr()
    rc = lib.harm_b200_fluxcalc_noalloc(C.byref(g.g), p, p, p, p, p, ndt, None)
    assert rc == 2
    assert "maximum" in lib.harm_b200_last_error().decode()
