"""Adiabatic slip wall in the Euler operator (mirgecom/boundary.py:1052-1080).

CPU: the oracle's Euler RHS of a gas at rest in a closed box of slip walls
vanishes (a steady state), and the product refuses the viscous operator with
this wall on hexahedra.  GPU: the device Euler RHS with slip walls on some
sides and prescribed states on the others matches the oracle at the float64
bar (simplices: the device slip treatment; hexahedra: its state_plus
prescribed).  The viscous walls are tested in tests/test_gpu_walls.py."""

import numpy as np
import pytest
import torch

from cases import field_rel_l2, make_disc, perturbed_state_np
from mirgecom_b200.boundary import AdiabaticSlipBoundary, PrescribedFluidBoundary
from mirgecom_b200.eos import IdealSingleGas
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from oracle import dg as odg
from oracle import physics as oph

TAGS3 = ("-0", "+0", "-1", "+1", "-2", "+2")


@pytest.mark.parametrize("kind,dim,order", [("simplex", 2, 3), ("simplex", 3, 2),
                                            ("hypercube", 3, 3)])
def test_oracle_rest_state_in_slip_box_is_steady(kind, dim, order):
    _, od = make_disc(kind, dim, 3, order, (0.0,) * dim, (1.0, 2.0, 1.5)[:dim], False)
    q = np.zeros((dim + 2,) + od.nodes.shape[1:])
    q[0] = 1.2
    q[1] = 2.5
    st = oph.make_fluid_state(q, oph.IdealGas(), None, dim)
    bnd = {t: odg.AdiabaticSlipBoundary() for t in TAGS3[:2 * dim]}
    for flux in ("rusanov", "hll", "central"):
        rhs = odg.euler_operator(od, st, oph.IdealGas(), bnd, flux=flux)
        assert np.abs(rhs).max() < 1e-10, flux


def test_ns_operator_refuses_slip_wall_on_hexahedra():
    """The viscous slip wall runs on the simplex kernels' volume/face path;
    the tensor-product hexahedra evaluate only its inviscid part."""
    from mirgecom_b200.navierstokes import ns_operator
    from mirgecom_b200.transport import SimpleTransport
    d, od = make_disc("hypercube", 3, 3, 2, (0.0,) * 3, (1.0,) * 3, False)
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(viscosity=1e-3))
    q = perturbed_state_np(od.nodes, 3, 0, seed=1)
    st = make_fluid_state(ConservedVars(torch.from_numpy(q), 3), gas)
    with pytest.raises(NotImplementedError):
        ns_operator(d, gas, st, {"all": AdiabaticSlipBoundary()})


@pytest.mark.gpu
@pytest.mark.parametrize("kind,dim,order", [("simplex", 2, 3), ("simplex", 3, 3),
                                            ("hypercube", 3, 3)])
@pytest.mark.parametrize("flux", ["rusanov", "hll"])
def test_device_euler_slip_walls(cuda, kind, dim, order, flux):
    from mirgecom_b200.euler import euler_operator
    from mirgecom_b200.inviscid import inviscid_facial_flux_hll, inviscid_facial_flux_rusanov
    d, od = make_disc(kind, dim, 3, order, (0.0,) * dim, (2.0, 1.0, 1.5)[:dim], False)
    q = perturbed_state_np(od.nodes, dim, 0, seed=5)

    def ext_np(x):
        return perturbed_state_np(x, dim, 0, seed=6)

    def bfunc(dcoll, dd_bdry, gas_model, state_minus, time, nodes, **kw):
        return make_fluid_state(ConservedVars(
            torch.from_numpy(ext_np(nodes.cpu().numpy())).to(cuda), dim), gas_model)

    tags = TAGS3[:2 * dim]
    slip = set(tags[::2]) | {tags[1]}
    bnds = {t: AdiabaticSlipBoundary() if t in slip else
            PrescribedFluidBoundary(boundary_state_func=bfunc) for t in tags}
    obnds = {t: odg.AdiabaticSlipBoundary() if t in slip else
             odg.PrescribedBoundary(lambda x, tt: ext_np(x)) for t in tags}
    gas = GasModel(eos=IdealSingleGas())
    fn = {"rusanov": inviscid_facial_flux_rusanov, "hll": inviscid_facial_flux_hll}[flux]
    rhs = euler_operator(d, make_fluid_state(ConservedVars(torch.from_numpy(q).to(cuda), dim),
                                             gas), gas, bnds, inviscid_numerical_flux_func=fn)
    ref = odg.euler_operator(od, oph.make_fluid_state(q, oph.IdealGas(), None, dim),
                             oph.IdealGas(), obnds, flux=flux)
    assert field_rel_l2(rhs.q.cpu().numpy(), ref) < 1e-12
