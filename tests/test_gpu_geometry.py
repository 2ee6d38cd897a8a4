"""The metric, connection and floor tables built on the device (harm_b200_create_grid; set_grid
set_grid.c:114, set_connection set_grid.c:1033) against the host builder's tables, which the
oracle and the other tests use: the same algorithm operation for operation, so the metric and
floor tables agree to the last bits of the math library (sin, cos, exp, pow differ by an ulp
or so between the host's and the device's) and the connection to the noise of its numerical
derivatives (Ridders' extrapolation picks among its tableau entries by their error
estimates, which that noise can reorder).  Steps on either set of tables agree."""
import numpy as np
import pytest

from helpers import make_torus, rel_err
from harm_harm_b200 import HARM_PREC_FP64, HARM_PREC_MIXED, Harm

pytestmark = pytest.mark.gpu


def _compare(geom_h, conn_h, aux_h, dev):
    geom_d, conn_d, aux_d = dev.tables()
    e_geom = max(rel_err(geom_h[loc, f], geom_d[loc, f], 1e-14) for loc in range(4) for f in range(28))
    e_aux = max(rel_err(aux_h[q], aux_d[q], 1e-14) for q in range(3))
    # the connection relative to its largest component at the same cell (components that
    # vanish analytically hold only round-off of their terms' cancellation)
    scale = np.abs(conn_h).max(axis=0)
    rel = np.abs(conn_h - conn_d) / np.maximum(scale, 1e-300)[None]
    q, j, i = np.unravel_index(np.argmax(rel), rel.shape)
    print("largest connection difference: component", q, "cell (j, i)", (j, i), "host", conn_h[q, j, i],
          "device", conn_d[q, j, i], "cell scale", scale[j, i])
    return e_geom, e_aux, float(rel.max())


@pytest.mark.parametrize("shape,lim", [((64, 64, 1), 0), ((48, 32, 8), 2)])
def test_device_tables_match_host_tables(cuda, shape, lim):
    g, geom, conn, aux, P = make_torus(*shape, lim=lim)
    dev = Harm(g)
    try:
        e_geom, e_aux, e_conn = _compare(geom, conn, aux, dev)
        print("device vs host tables: metric %.2e floors %.2e connection %.2e" % (e_geom, e_aux, e_conn))
        assert e_geom < 1e-13
        assert e_aux < 1e-13
        assert e_conn < 1e-10
    finally:
        dev.close()


@pytest.mark.parametrize("precision", [HARM_PREC_FP64, HARM_PREC_MIXED])
def test_steps_on_device_tables_match_host_tables(cuda, precision):
    torch = cuda
    g, geom, conn, aux, P0 = make_torus(48, 32, 8, lim=2)
    host, dev = Harm(g, geom, conn, aux), Harm(g)
    try:
        Pa = torch.from_numpy(P0).cuda()
        host.bound_prim(Pa)
        Pb = Pa.clone()
        dta, _ = host.step_ch(Pa, 1e-3, precision=precision, nsteps=3)
        dtb, _ = dev.step_ch(Pb, 1e-3, precision=precision, nsteps=3)
        a, b = Pa.cpu().numpy(), Pb.cpu().numpy()
        # relative to each field's largest magnitude: the velocity components cross zero, and
        # the polar boundary's Lorentz-factor limit and velocity crush are thresholds that the
        # tables' round-off (connection 4e-12) can flip in a cell next to the pole
        act = (slice(None),) + g.active
        a, b = a[act], b[act]
        errs = [float(np.abs(a[pl] - b[pl]).max() / np.abs(b[pl]).max()) for pl in range(8)]
        print("steps on device vs host tables, max rel diff per primitive", ["%.1e" % e for e in errs])
        assert max(errs) < 1e-8
        assert abs(dta - dtb) <= 1e-10 * dta
    finally:
        host.close()
        dev.close()
