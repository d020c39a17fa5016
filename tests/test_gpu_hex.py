"""Tensor-product hexahedra (the element of the 48^3 hex p4 Taylor-Green
configuration): the device gradient and divergence passes against the CPU
oracle -- float64 at 1e-12 relative L2 per field, the mixed form within the
mixed-form tolerance."""

import numpy as np
import pytest
import torch

from cases import field_rel_l2, flux_scale_floor, make_disc, per_field_rel_l2, \
    perturbed_state_np, tgv_np
from mirgecom_b200 import runtime
from mirgecom_b200.boundary import DummyBoundary, PrescribedFluidBoundary
from mirgecom_b200.eos import IdealSingleGas
from mirgecom_b200.euler import euler_operator
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.inviscid import (inviscid_facial_flux_central, inviscid_facial_flux_hll,
                                    inviscid_facial_flux_rusanov)
from mirgecom_b200.navierstokes import ns_operator
from mirgecom_b200.transport import PowerLawTransport, SimpleTransport
from oracle import dg as odg
from oracle import physics as oph

pytestmark = pytest.mark.gpu

TOL = 1e-12
FLUXES = {"rusanov": inviscid_facial_flux_rusanov, "hll": inviscid_facial_flux_hll,
          "central": inviscid_facial_flux_central}
MU = 1.0 / 1600
KAPPA = MU * 1.4 * 287.1 / 0.4 / 0.71


def _cv(q, dim, dev, dtype=torch.float64):
    return ConservedVars(torch.from_numpy(np.ascontiguousarray(q)).to(dev, dtype), dim)


@pytest.mark.parametrize("order", [1, 2, 4])
def test_hex_ns_taylor_green(cuda, order):
    """Viscous Taylor-Green on a periodic 3^3 hex mesh: gradients and RHS."""
    d, od = make_disc("hypercube", 3, 3, order, (-np.pi,) * 3, (np.pi,) * 3, True)
    q = tgv_np(od.nodes)
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        viscosity=MU, thermal_conductivity=KAPPA))
    rhs, gcv, gt = ns_operator(d, gas, make_fluid_state(_cv(q, 3, cuda), gas), {},
                               return_gradients=True)
    otr = oph.SimpleTransportParams(viscosity=MU, thermal_conductivity=KAPPA)
    ost = oph.make_fluid_state(q, oph.IdealGas(), otr, 3)
    ref, rgcv, rgt = odg.ns_operator(od, ost, oph.IdealGas(), otr, {}, return_gradients=True)
    h = 2 * np.pi / 3
    scale = [np.linalg.norm(q[c]) / h for c in range(q.shape[0])]
    assert field_rel_l2(gcv.q.cpu().numpy(), rgcv, floor=scale) < TOL
    tfl = np.linalg.norm(ost["temperature"]) / h
    assert field_rel_l2(gt.cpu().numpy()[None], rgt[None], floor=[tfl]) < TOL
    assert field_rel_l2(rhs.q.cpu().numpy(), ref, floor=flux_scale_floor(q, 3, h)) < TOL
    assert runtime.read_status(d) == 0


@pytest.mark.parametrize("flux", ["rusanov", "hll", "central"])
@pytest.mark.parametrize("viscous", [False, True])
def test_hex_boundaries(cuda, flux, viscous):
    """Non-periodic box of hexahedra, order 3: Dummy and Prescribed boundaries,
    Euler and Navier-Stokes (power-law transport), every inviscid flux."""
    d, od = make_disc("hypercube", 3, 3, 3, (0.0, 0.0, 0.0), (2.0, 1.0, 1.5), False)
    q = perturbed_state_np(od.nodes, 3, 0, seed=3)

    def ext_np(x):
        return perturbed_state_np(x, 3, 0, seed=4)

    def bnd(dcoll, dd_bdry, gas_model, state_minus, time, nodes, **kw):
        return make_fluid_state(_cv(ext_np(nodes.cpu().numpy()), 3, cuda), gas_model)

    tags = {"-0": "d", "+0": "p", "-1": "p", "+1": "d", "-2": "p", "+2": "d"}
    bnds = {t: (DummyBoundary() if k == "d" else PrescribedFluidBoundary(boundary_state_func=bnd))
            for t, k in tags.items()}
    obnds = {t: (odg.DummyBoundary() if k == "d" else
                 odg.PrescribedBoundary(lambda x, tt: ext_np(x))) for t, k in tags.items()}
    if viscous:
        tr = PowerLawTransport(beta=1e-2)
        gas = GasModel(eos=IdealSingleGas(), transport=tr)
        rhs = ns_operator(d, gas, make_fluid_state(_cv(q, 3, cuda), gas), bnds,
                          inviscid_numerical_flux_func=FLUXES[flux])
        otr = oph.PowerLawTransportParams(beta=1e-2)
        ref = odg.ns_operator(od, oph.make_fluid_state(q, oph.IdealGas(), otr, 3),
                              oph.IdealGas(), otr, obnds, flux=flux)
    else:
        gas = GasModel(eos=IdealSingleGas())
        rhs = euler_operator(d, make_fluid_state(_cv(q, 3, cuda), gas), gas, bnds,
                             inviscid_numerical_flux_func=FLUXES[flux])
        ref = odg.euler_operator(od, oph.make_fluid_state(q, oph.IdealGas(), None, 3),
                                 oph.IdealGas(), obnds, flux=flux)
    assert field_rel_l2(rhs.q.cpu().numpy(), ref) < TOL
    assert runtime.read_status(d) == 0


def test_hex_mixed_taylor_green(cuda):
    """Mixed form (float32 state, TF32x3 line contractions) on p4 hexahedra."""
    d, od = make_disc("hypercube", 3, 3, 4, (-np.pi,) * 3, (np.pi,) * 3, True)
    q = tgv_np(od.nodes)
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        viscosity=MU, thermal_conductivity=KAPPA))
    rhs = ns_operator(d, gas, make_fluid_state(_cv(q, 3, cuda, torch.float32), gas), {})
    otr = oph.SimpleTransportParams(viscosity=MU, thermal_conductivity=KAPPA)
    ref = odg.ns_operator(od, oph.make_fluid_state(q, oph.IdealGas(), otr, 3),
                          oph.IdealGas(), otr, {})
    # as for simplices: the float32 state's rounding of rho E, amplified by
    # the small low-Mach divergence, bounds the agreement
    out = rhs.q.double().cpu().numpy()
    assert field_rel_l2(out, ref) < 2e-2, per_field_rel_l2(out, ref)
    h = 2 * np.pi / 3
    assert field_rel_l2(out, ref, floor=flux_scale_floor(q, 3, h)) < 1e-5
    assert runtime.read_status(d) == 0
