"""The 2-D vortex configuration run to t = 1 through the library's driver.

mirgecom_b200.vortex advances the isentropic vortex ([0, 10] x [-5, 5],
16 x 16 x 2 triangles, order 3, beta 5 at (5, 0), velocity (1, 0), exact
prescribed boundaries, Rusanov) with RK4 at dt = 0.005 for 200 steps on the
device, as mirgecom's examples/vortex.py does on its array context.  The
oracle runs the same 200 steps on the CPU in float64; the end states agree
to 1e-11 per field, and both are within the discretisation error of the
exact solution.
"""

import numpy as np
import pytest

from cases import assert_fields_close, make_disc, vortex_np
from oracle import dg as odg
from oracle import physics as oph

pytestmark = pytest.mark.gpu


def test_vortex_run_matches_oracle(cuda):
    from mirgecom_b200 import runtime, vortex
    res = vortex.run(device=cuda)
    assert res["steps"] == 200 and abs(res["t"] - 1.0) < 1e-12
    assert runtime.read_status(res["dcoll"]) == 0
    d, od = make_disc("simplex", 2, 16, 3, (0.0, -5.0), (10.0, 5.0), False)
    q0 = vortex_np(od.nodes)
    q = q0.copy()
    obnds = {"all": odg.PrescribedBoundary(lambda x, tt: vortex_np(x, t=tt))}

    def orhs(t, qq):
        return odg.euler_operator(od, oph.make_fluid_state(qq, oph.IdealGas(), None, 2),
                                  oph.IdealGas(), obnds, time=t)

    for i in range(200):
        q = odg.rk4_step(q, i * 0.005, 0.005, orhs)
    qg = res["q"].cpu().numpy()
    # the end states, and the change over the run, field by field
    assert_fields_close(qg, q, 1e-11, what="end state")
    assert_fields_close(qg - q0, q - q0, 1e-10, what="change")
    # discretisation error against the exact solution at t = 1 (L2 over the
    # domain of area 100: |rho| ~ 10): the device run's equals the oracle's
    exact = vortex_np(od.nodes, t=1.0)
    r = q - exact
    ref_err = [float(np.sqrt(np.sum(np.abs(d.geometry.det) *
                                    np.einsum("ei,ij,ej->e", r[c], d.refel.mass, r[c]))))
               for c in range(4)]
    assert np.allclose(res["l2_error"], ref_err, rtol=1e-8), (res["l2_error"], ref_err)
    assert max(ref_err) < 0.1
