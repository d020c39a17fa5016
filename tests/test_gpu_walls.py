"""Mengaldo walls and flow boundaries on the device against the oracle.

The viscous (Navier-Stokes) and inviscid (Euler) right-hand sides of boxes
whose sides carry the reference's wall and flow boundaries
(mirgecom/boundary.py:391-793: AdiabaticSlip :1052, Farfield :1146,
PressureOutflow :1231, IsothermalWall :1727, AdiabaticNoslipWall :1794),
float64 device path against the float64 oracle at 1e-12 per field (each
field against its own norm, or its inviscid flux scale |F_c|/h where that is
larger), Rusanov and HLL; the mixture with an isothermal wall; and a gas at
rest in a closed box of each wall stays at rest on the device.
"""

import numpy as np
import pytest
import torch

from cases import assert_fields_close, inviscid_flux_floor, make_disc, perturbed_state_np
from mirgecom_b200 import runtime
from mirgecom_b200.boundary import (AdiabaticNoslipWallBoundary, AdiabaticSlipBoundary,
                                    FarfieldBoundary, IsothermalWallBoundary,
                                    PressureOutflowBoundary)
from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture
from mirgecom_b200.euler import euler_operator
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.inviscid import inviscid_facial_flux_hll, inviscid_facial_flux_rusanov
from mirgecom_b200.navierstokes import ns_operator
from mirgecom_b200.thermochemistry import UIUC_7SP
from mirgecom_b200.transport import SimpleTransport
from oracle import dg as odg
from oracle import physics as oph

pytestmark = pytest.mark.gpu

TOL = 1e-12
TAGS = ("-0", "+0", "-1", "+1", "-2", "+2")
FLUX = {"rusanov": inviscid_facial_flux_rusanov, "hll": inviscid_facial_flux_hll}


def _walls(dim, t_wall, p_out, fs):
    """One boundary of each kind around the box: (device, oracle) pairs."""
    pairs = [
        (AdiabaticSlipBoundary(), odg.AdiabaticSlipBoundary()),
        (PressureOutflowBoundary(boundary_pressure=p_out),
         odg.PressureOutflowBoundary(boundary_pressure=p_out)),
        (IsothermalWallBoundary(wall_temperature=t_wall),
         odg.IsothermalWallBoundary(wall_temperature=t_wall)),
        (AdiabaticNoslipWallBoundary(), odg.AdiabaticNoslipWallBoundary()),
        (FarfieldBoundary(*fs), odg.FarfieldBoundary(*fs)),
        (AdiabaticSlipBoundary(), odg.AdiabaticSlipBoundary()),
    ]
    return ({t: p[0] for t, p in zip(TAGS[:2 * dim], pairs)},
            {t: p[1] for t, p in zip(TAGS[:2 * dim], pairs)})


@pytest.mark.parametrize("flux", ["rusanov", "hll"])
@pytest.mark.parametrize("dim,order", [(2, 3), (3, 2), (3, 3)])
def test_walls_ns_ideal_gas(cuda, dim, order, flux):
    d, od = make_disc("simplex", dim, 3, order, (0.0,) * dim, (1.0, 0.7, 1.3)[:dim], False)
    q = perturbed_state_np(od.nodes, dim, 0, seed=9)
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        viscosity=2e-2, thermal_conductivity=3e-2))
    ogas = oph.IdealGas()
    otr = oph.SimpleTransportParams(viscosity=2e-2, thermal_conductivity=3e-2)
    fs = (1.1, [0.2, -0.1, 0.05][:dim], 3.0e-3)          # p, v, T of the far field
    bnds, obnds = _walls(dim, 4.0e-3, 0.9, fs)
    st = make_fluid_state(ConservedVars(torch.from_numpy(q).to(cuda), dim), gas)
    rhs = ns_operator(d, gas, st, bnds, inviscid_numerical_flux_func=FLUX[flux])
    ref = odg.ns_operator(od, oph.make_fluid_state(q, ogas, otr, dim), ogas, otr, obnds,
                          flux=flux)
    assert_fields_close(rhs.q.cpu().numpy(), ref, TOL, floor=inviscid_flux_floor(q, dim, 0.23))
    assert runtime.read_status(d) == 0


@pytest.mark.parametrize("flux", ["rusanov", "hll"])
@pytest.mark.parametrize("dim", [2, 3])
def test_walls_euler_ideal_gas(cuda, dim, flux):
    d, od = make_disc("simplex", dim, 3, 3, (0.0,) * dim, (1.0, 0.7, 1.3)[:dim], False)
    q = perturbed_state_np(od.nodes, dim, 2, seed=4)
    gas = GasModel(eos=IdealSingleGas())
    ogas = oph.IdealGas()
    bnds, obnds = _walls(dim, 4.0e-3, 0.9, (1.1, [0.2, -0.1, 0.05][:dim], 3.0e-3,
                                            [0.1, 0.2]))
    st = make_fluid_state(ConservedVars(torch.from_numpy(q).to(cuda), dim), gas)
    rhs = euler_operator(d, st, gas, bnds, inviscid_numerical_flux_func=FLUX[flux])
    ref = odg.euler_operator(od, oph.make_fluid_state(q, ogas, None, dim), ogas, obnds,
                             flux=flux)
    assert_fields_close(rhs.q.cpu().numpy(), ref, TOL, floor=inviscid_flux_floor(q, dim, 0.23))
    assert runtime.read_status(d) == 0


def test_walls_ns_mixture(cuda):
    """uiuc_7sp: every wall and flow boundary with the mixture's Newton
    temperatures on the boundary states and species sources."""
    from mirgecom_b200.initializers import reacting_mixture_state
    d, od = make_disc("simplex", 3, 3, 2, (0.0,) * 3, (0.02, 0.014, 0.026), False)
    cv0, t_true = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                         UIUC_7SP, seed=8, t_range=(900.0, 1500.0),
                                         box=(0.02, 0.014, 0.026))
    q = cv0.q.numpy()
    tseed = t_true.numpy() + 3.0
    diff = [1e-5 * (k + 1) for k in range(7)]
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5),
                   transport=SimpleTransport(viscosity=2e-5, thermal_conductivity=3e-2,
                                             species_diffusivity=diff))
    ogas = oph.MixtureGas(UIUC_7SP, temperature_niter=5)
    otr = oph.SimpleTransportParams(viscosity=2e-5, thermal_conductivity=3e-2,
                                    species_diffusivity=tuple(diff))
    y_fs = [0.05, 0.22, 0.0, 0.0, 0.0, 0.0, 0.73]
    bnds, obnds = _walls(3, 1000.0, 101325.0, (101325.0, [3.0, -1.0, 2.0], 1200.0, y_fs))
    st = make_fluid_state(ConservedVars(torch.from_numpy(q).to(cuda), 3), gas,
                          temperature_seed=torch.from_numpy(tseed).to(cuda))
    rhs = ns_operator(d, gas, st, bnds, species_source_temperature=st.temperature)
    ost = oph.make_fluid_state(q, ogas, otr, 3, temperature_seed=tseed)
    ref = odg.ns_operator(od, ost, ogas, otr, obnds)
    ref = ref + oph.species_source_terms(ogas, q, ost["temperature"], 3)
    floor = inviscid_flux_floor(q, 3, 0.02 / 3, temperature=ost["temperature"], mech=UIUC_7SP)
    assert_fields_close(rhs.q.cpu().numpy(), ref, TOL, floor=floor)
    assert runtime.read_status(d) == 0


@pytest.mark.parametrize("wall", ["slip", "noslip", "isothermal", "outflow"])
def test_gas_at_rest_stays_at_rest(cuda, wall):
    d, od = make_disc("simplex", 3, 3, 3, (0.0,) * 3, (1.0, 0.7, 1.3), False)
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        viscosity=1e-3, thermal_conductivity=1e-2))
    q = np.zeros((5,) + od.nodes.shape[1:])
    q[0] = 1.2
    q[1] = 1.0e5 / 0.4
    t_gas = 1.0e5 / (1.2 * 287.1)
    b = {"slip": AdiabaticSlipBoundary(), "noslip": AdiabaticNoslipWallBoundary(),
         "isothermal": IsothermalWallBoundary(wall_temperature=t_gas),
         "outflow": PressureOutflowBoundary(boundary_pressure=1.0e5)}[wall]
    st = make_fluid_state(ConservedVars(torch.from_numpy(q).to(cuda), 3), gas)
    rhs = ns_operator(d, gas, st, {"all": b})
    assert float(rhs.q.abs().max()) < 1e-11 * (1.0e5 / 0.1)
    assert runtime.read_status(d) == 0
