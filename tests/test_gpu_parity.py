"""GPU parity: the CUDA RHS through the C ABI against the float64 oracle.

Tolerance: 1e-12 relative L2 per conserved field (the plain FP64 bar), on
identical nodes, reference matrices and mesh.  The oracle evaluates every
operator state the way the reference does (mirgecom/gas_model.py:728-904),
including the second Newton solve on every face trace for mixtures.
"""

import numpy as np
import pytest
import torch

from cases import (assert_fields_close, field_rel_l2, flux_scale_floor, inviscid_flux_floor,
                   make_disc, perturbed_state_np, rel_l2, tgv_np, vortex_np)
from mirgecom_b200 import runtime
from mirgecom_b200.boundary import DummyBoundary, PrescribedFluidBoundary
from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture
from mirgecom_b200.euler import euler_operator
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.integrators import rk4_step
from mirgecom_b200.inviscid import (inviscid_facial_flux_hll,
                                    inviscid_facial_flux_rusanov)
from mirgecom_b200.navierstokes import ns_operator
from mirgecom_b200.thermochemistry import UIUC_7SP
from mirgecom_b200.transport import PowerLawTransport, SimpleTransport
from oracle import dg as odg
from oracle import physics as oph

pytestmark = pytest.mark.gpu

TOL = 1e-12
FLUXES = {"rusanov": inviscid_facial_flux_rusanov, "hll": inviscid_facial_flux_hll}


def _cv(q, dim, dev):
    return ConservedVars(torch.from_numpy(np.ascontiguousarray(q)).to(dev), dim)


def _status_ok(d):
    assert runtime.read_status(d) == 0


@pytest.mark.parametrize("flux", ["rusanov", "hll"])
def test_euler_vortex_config1(cuda, flux):
    """2-D isentropic vortex, tri p3, 16x16 squares on [0,10]x[-5,5]."""
    d, od = make_disc("simplex", 2, 16, 3, (0.0, -5.0), (10.0, 5.0), False)
    t = 0.3
    q = vortex_np(od.nodes, t=t)
    gas = GasModel(eos=IdealSingleGas())

    def bnd(dcoll, dd_bdry, gas_model, state_minus, time, nodes, **kw):
        xb = nodes.cpu().numpy()
        return make_fluid_state(_cv(vortex_np(xb, t=time), 2, cuda), gas_model)

    rhs = euler_operator(d, make_fluid_state(_cv(q, 2, cuda), gas),
                         gas, {"all": PrescribedFluidBoundary(boundary_state_func=bnd)},
                         time=t, inviscid_numerical_flux_func=FLUXES[flux])
    ost = oph.make_fluid_state(q, oph.IdealGas(), None, 2)
    ref = odg.euler_operator(od, ost, oph.IdealGas(),
                             {"all": odg.PrescribedBoundary(lambda x, tt: vortex_np(x, t=tt))},
                             time=t, flux=flux)
    assert_fields_close(rhs.q.cpu().numpy(), ref, TOL)
    _status_ok(d)


@pytest.mark.parametrize("dim,order", [(3, 1), (3, 2), (3, 3), (2, 4)])
def test_euler_periodic_species(cuda, dim, order):
    d, od = make_disc("simplex", dim, 4 if dim == 3 else 6, order, (0.0,) * dim,
                      (2 * np.pi,) * dim, True)
    q = perturbed_state_np(od.nodes, dim, 2, seed=order)
    gas = GasModel(eos=IdealSingleGas())
    rhs = euler_operator(d, make_fluid_state(_cv(q, dim, cuda), gas), gas, {},
                         inviscid_numerical_flux_func=inviscid_facial_flux_rusanov)
    ref = odg.euler_operator(od, oph.make_fluid_state(q, oph.IdealGas(), None, dim),
                             oph.IdealGas(), {}, flux="rusanov")
    assert_fields_close(rhs.q.cpu().numpy(), ref, TOL)


def test_ns_taylor_green_config2_small(cuda):
    """Viscous TGV physics of config 2 on a 4^3 periodic box, tet p3."""
    d, od = make_disc("simplex", 3, 4, 3, (-np.pi,) * 3, (np.pi,) * 3, True)
    q = tgv_np(od.nodes)
    mu = 1.0 / 1600
    kappa = mu * 1.4 * 287.1 / 0.4 / 0.71
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        viscosity=mu, thermal_conductivity=kappa))
    rhs, gcv, gt = ns_operator(d, gas, make_fluid_state(_cv(q, 3, cuda), gas), {},
                               return_gradients=True)
    otr = oph.SimpleTransportParams(viscosity=mu, thermal_conductivity=kappa)
    ost = oph.make_fluid_state(q, oph.IdealGas(), otr, 3)
    ref, rgcv, rgt = odg.ns_operator(od, ost, oph.IdealGas(), otr, {},
                                     return_gradients=True)
    # natural scale of grad(q_c): |q_c| / h with h the cube edge (2 pi / 4)
    h = 2 * np.pi / 4
    scale = [np.linalg.norm(q[c]) / h for c in range(q.shape[0])]
    assert field_rel_l2(gcv.q.cpu().numpy(), rgcv, floor=scale) < TOL
    # T = p/(rho R) ~ 0.249 varies by ~1e-4 here: measure grad T against |T|/h
    tfl = np.linalg.norm(ost["temperature"]) / h
    assert field_rel_l2(gt.cpu().numpy()[None], rgt[None], floor=[tfl]) < TOL
    # Mach 0.1: the RHS is ~700x below the pressure flux; measure against |F_c|/h
    assert field_rel_l2(rhs.q.cpu().numpy(), ref, floor=flux_scale_floor(q, 3, h)) < TOL
    _status_ok(d)


@pytest.mark.parametrize("flux", ["rusanov", "hll"])
def test_ns_2d_boundaries_species(cuda, flux):
    """Mixed Dummy / Prescribed boundaries, passive species, power-law transport."""
    d, od = make_disc("simplex", 2, 5, 2, (0.0, 0.0), (2.0, 1.0), False)
    q = perturbed_state_np(od.nodes, 2, 2, seed=3)
    qext = perturbed_state_np(od.nodes, 2, 2, seed=4)
    tr = PowerLawTransport(species_diffusivity=[1e-2, 2e-2], beta=1e-2)
    gas = GasModel(eos=IdealSingleGas(), transport=tr)

    def ext_np(x):
        return perturbed_state_np(x, 2, 2, seed=4)

    def bnd(dcoll, dd_bdry, gas_model, state_minus, time, nodes, **kw):
        return make_fluid_state(_cv(ext_np(nodes.cpu().numpy()), 2, cuda), gas_model)

    bnds = {"-0": DummyBoundary(), "+0": PrescribedFluidBoundary(boundary_state_func=bnd),
            "-1": PrescribedFluidBoundary(boundary_state_func=bnd), "+1": DummyBoundary()}
    rhs = ns_operator(d, gas, make_fluid_state(_cv(q, 2, cuda), gas), bnds,
                      inviscid_numerical_flux_func=FLUXES[flux])
    otr = oph.PowerLawTransportParams(species_diffusivity=(1e-2, 2e-2), beta=1e-2)
    obnds = {"-0": odg.DummyBoundary(), "+0": odg.PrescribedBoundary(lambda x, t: ext_np(x)),
             "-1": odg.PrescribedBoundary(lambda x, t: ext_np(x)), "+1": odg.DummyBoundary()}
    ref = odg.ns_operator(od, oph.make_fluid_state(q, oph.IdealGas(), otr, 2),
                          oph.IdealGas(), otr, obnds, flux=flux)
    del qext
    # measured against each field's own norm, or its flux scale |F_c|/h with
    # h the smaller cell edge (0.2) where that is larger
    assert_fields_close(rhs.q.cpu().numpy(), ref, TOL, floor=inviscid_flux_floor(q, 2, 0.2))
    _status_ok(d)


@pytest.mark.parametrize("order", [2, 3])
def test_ns_reacting_mixture(cuda, order):
    """uiuc_7sp mixture: Newton temperature, mixture transport fluxes, sources."""
    d, od = make_disc("simplex", 3, 3, order, (0.0,) * 3, (2 * np.pi,) * 3, True)
    from mirgecom_b200.initializers import reacting_mixture_state
    x = [torch.from_numpy(od.nodes[i]) for i in range(3)]
    cv0, t_true = reacting_mixture_state(x, UIUC_7SP, seed=7)
    q = cv0.q.numpy()
    tseed = t_true.numpy() + 40.0 * np.sin(od.nodes[0])
    diff = [1e-5 * (k + 1) for k in range(7)]
    tr = SimpleTransport(viscosity=1e-5, thermal_conductivity=2e-5, species_diffusivity=diff)
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5), transport=tr)
    st = make_fluid_state(_cv(q, 3, cuda), gas,
                          temperature_seed=torch.from_numpy(tseed).to(cuda))
    rhs = ns_operator(d, gas, st, {}, species_source_temperature=st.temperature)
    ogas = oph.MixtureGas(UIUC_7SP, temperature_niter=5)
    otr = oph.SimpleTransportParams(viscosity=1e-5, thermal_conductivity=2e-5,
                                    species_diffusivity=tuple(diff))
    ost = oph.make_fluid_state(q, ogas, otr, 3, temperature_seed=tseed)
    assert rel_l2(st.temperature.cpu().numpy(), ost["temperature"]) < 1e-14
    ref = odg.ns_operator(od, ost, ogas, otr, {})
    ref = ref + oph.species_source_terms(ogas, q, ost["temperature"], 3)
    # each field against its own norm, or its inviscid flux scale |F_c|/h
    # (h the cube edge) where that is larger: only the low-Mach momentum
    # fields, whose RHS is ~15x below their pressure flux, take the latter
    floor = inviscid_flux_floor(q, 3, 2 * np.pi / 3, temperature=ost["temperature"],
                                mech=UIUC_7SP)
    assert_fields_close(rhs.q.cpu().numpy(), ref, TOL, floor=floor)
    _status_ok(d)


def test_rk4_step_vortex(cuda):
    """One RK4 step (mirgecom/integrators/explicit_rk.py:31-37) of config 1."""
    d, od = make_disc("simplex", 2, 8, 3, (0.0, -5.0), (10.0, 5.0), False)
    gas = GasModel(eos=IdealSingleGas())

    def bnd(dcoll, dd_bdry, gas_model, state_minus, time, nodes, **kw):
        return make_fluid_state(_cv(vortex_np(nodes.cpu().numpy(), t=time), 2, cuda),
                                gas_model)

    bnds = {"all": PrescribedFluidBoundary(boundary_state_func=bnd)}

    def rhs(t, cv):
        return euler_operator(d, make_fluid_state(cv, gas), gas, bnds, time=t,
                              inviscid_numerical_flux_func=inviscid_facial_flux_rusanov)

    q = vortex_np(od.nodes)
    out = rk4_step(_cv(q, 2, cuda), 0.0, 0.005, rhs)
    obnds = {"all": odg.PrescribedBoundary(lambda x, tt: vortex_np(x, t=tt))}

    def orhs(t, qq):
        return odg.euler_operator(od, oph.make_fluid_state(qq, oph.IdealGas(), None, 2),
                                  oph.IdealGas(), obnds, time=t)

    ref = odg.rk4_step(q, 0.0, 0.005, orhs)
    assert field_rel_l2(out.q.cpu().numpy() - q, ref - q) < 1e-11


@pytest.mark.parametrize("dim", [2, 3])
def test_uniform_state_rhs_zero(cuda, dim):
    """mirgecom test/test_euler.py:80-232 on the device: uniform flow, RHS = 0."""
    d, od = make_disc("simplex", dim, 4, 3, (-0.5,) * dim, (0.5,) * dim, False)
    shape = (d.nelements, d.refel.nnodes)
    q = np.zeros((dim + 2 + 2,) + shape)
    q[0] = 1.0
    q[1] = 2.5
    for i in range(dim):
        q[2 + i] = (-1.0) ** i
    q[2 + dim] = 0.1
    q[3 + dim] = 0.05
    gas = GasModel(eos=IdealSingleGas())
    for flux in FLUXES.values():
        rhs = euler_operator(d, make_fluid_state(_cv(q, dim, cuda), gas), gas,
                             {"all": DummyBoundary()}, inviscid_numerical_flux_func=flux)
        assert float(rhs.q.abs().max()) < 1e-9


@pytest.mark.parametrize("case", ["tgv", "mixture", "boundaries_hll"])
def test_rhs_paths_agree(cuda, case):
    """The volume/face path, the split divergence (flux records + surface) and
    the fused divergence pass give the same right-hand side."""
    if case == "tgv":
        d, od = make_disc("simplex", 3, 3, 3, (-np.pi,) * 3, (np.pi,) * 3, True)
        q = tgv_np(od.nodes)
        mu = 1.0 / 1600
        gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
            viscosity=mu, thermal_conductivity=mu * 1004.85 / 0.71))
        st = make_fluid_state(_cv(q, 3, cuda), gas)
        kw, bnds, flux = {}, {}, inviscid_facial_flux_rusanov
        floor = inviscid_flux_floor(q, 3, 2 * np.pi / 3)
    elif case == "mixture":
        d, od = make_disc("simplex", 3, 3, 3, (0.0,) * 3, (2 * np.pi,) * 3, True)
        from mirgecom_b200.initializers import reacting_mixture_state
        cv0, t_true = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                             UIUC_7SP, seed=5)
        gas = GasModel(eos=PyrometheusMixture(UIUC_7SP), transport=SimpleTransport(
            viscosity=1e-5, thermal_conductivity=2e-5, species_diffusivity=[1e-5] * 7))
        st = make_fluid_state(ConservedVars(cv0.q.to(cuda), 3), gas,
                              temperature_seed=t_true.to(cuda) + 10.0)
        kw, bnds, flux = {"species_source_temperature": st.temperature}, {}, \
            inviscid_facial_flux_rusanov
        floor = inviscid_flux_floor(cv0.q.numpy(), 3, 2 * np.pi / 3,
                                    temperature=st.temperature.cpu().numpy(), mech=UIUC_7SP)
    else:
        d, od = make_disc("simplex", 2, 5, 2, (0.0, 0.0), (2.0, 1.0), False)
        q = perturbed_state_np(od.nodes, 2, 2, seed=3)
        gas = GasModel(eos=IdealSingleGas(), transport=PowerLawTransport(
            species_diffusivity=[1e-2, 2e-2], beta=1e-2))

        def bnd(dcoll, dd_bdry, gas_model, state_minus, time, nodes, **k):
            return make_fluid_state(_cv(perturbed_state_np(nodes.cpu().numpy(), 2, 2, seed=4),
                                        2, cuda), gas_model)

        bnds = {"-0": DummyBoundary(), "+0": PrescribedFluidBoundary(boundary_state_func=bnd),
                "-1": PrescribedFluidBoundary(boundary_state_func=bnd), "+1": DummyBoundary()}
        st = make_fluid_state(_cv(q, 2, cuda), gas)
        kw, flux = {}, inviscid_facial_flux_hll
        floor = inviscid_flux_floor(q, 2, 0.2)
    outs = {}
    default = runtime.RHS_PATH
    for path in ("volume_face", "gradient_volume_face", "split", "fused"):
        runtime.RHS_PATH = path
        try:
            outs[path] = ns_operator(d, gas, st, bnds, inviscid_numerical_flux_func=flux,
                                     **kw).q.cpu().numpy()
        finally:
            runtime.RHS_PATH = default
    assert_fields_close(outs["split"], outs["fused"], TOL, floor=floor)
    assert_fields_close(outs["volume_face"], outs["fused"], TOL, floor=floor)
    assert_fields_close(outs["gradient_volume_face"], outs["fused"], TOL, floor=floor)
    _status_ok(d)
