"""The oracle's Mengaldo boundaries against the reference's own checks.

mirgecom's test/test_bc.py checks the wall states (zero momentum and the
wall temperature for the isothermal no-slip wall, :432-597; zero momentum
for the adiabatic no-slip wall, :600-778; the slip wall's state and fluxes,
:974-1178) and the far-field / outflow states (:136-429); its Navier-Stokes
tests check that a gas at rest in a closed box stays at rest.  Restated
here on the oracle (CPU), plus the equivalence of the slip wall's velocity
gradient written as a projection with the reference's rotated-frame form
where that frame is defined.
"""

import numpy as np
import pytest

from cases import make_disc
from oracle import dg as odg
from oracle import physics as oph


def _box(dim, order=2, n=3):
    return make_disc("simplex", dim, n, order, (0.0,) * dim, (1.0, 0.7, 1.3)[:dim], False)


def _rest_state(od, dim, rho=1.2, p=1.0e5, gas=None):
    shape = od.nodes[0].shape
    q = np.zeros((dim + 2,) + shape)
    q[0] = rho
    q[1] = p / (gas.gamma - 1.0)
    return q


WALLS = {
    "slip": lambda t: odg.AdiabaticSlipBoundary(),
    "noslip": lambda t: odg.AdiabaticNoslipWallBoundary(),
    "isothermal": lambda t: odg.IsothermalWallBoundary(wall_temperature=t),
    "outflow": lambda t: odg.PressureOutflowBoundary(boundary_pressure=1.0e5),
}


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("wall", sorted(WALLS))
def test_gas_at_rest_in_closed_box(dim, wall):
    """A uniform gas at rest, every boundary the same wall (the isothermal
    one at the gas temperature, the outflow at the gas pressure): the
    Navier-Stokes right-hand side vanishes."""
    _, od = _box(dim)
    gas = oph.IdealGas()
    q = _rest_state(od, dim, gas=gas)
    tr = oph.SimpleTransportParams(viscosity=1e-3, thermal_conductivity=1e-2)
    st = oph.make_fluid_state(q, gas, tr, dim)
    t_gas = float(st["temperature"].ravel()[0])
    rhs = odg.ns_operator(od, st, gas, tr, {"all": WALLS[wall](t_gas)})
    scale = 1.0e5 / 0.1          # pressure / element size
    assert np.abs(rhs).max() < 1e-11 * scale


def test_mixture_at_rest_isothermal_box():
    from mirgecom_b200.thermochemistry import UIUC_7SP
    _, od = _box(3)
    gas = oph.MixtureGas(UIUC_7SP, temperature_niter=5)
    y = np.array([0.05, 0.2, 0.05, 0.02, 0.05, 0.01, 0.62])
    t0, p0 = 1200.0, 101325.0
    shape = od.nodes[0].shape
    rho = p0 / (oph.mixture_gas_const(UIUC_7SP, y[:, None, None] * np.ones(shape)) * t0)
    e = oph.mixture_e_mass(UIUC_7SP, t0 * np.ones(shape), y[:, None, None] * np.ones(shape))
    q = np.concatenate([rho[None], (rho * e)[None], np.zeros((3,) + shape),
                        rho[None] * y[:, None, None]])
    tr = oph.SimpleTransportParams(viscosity=1e-5, thermal_conductivity=1e-5,
                                   species_diffusivity=(1e-5,) * 7)
    st = oph.make_fluid_state(q, gas, tr, 3, temperature_seed=np.full(shape, 1000.0))
    rhs = odg.ns_operator(od, st, gas, tr, {"all": odg.IsothermalWallBoundary(t0)})
    assert np.abs(rhs[:5]).max() < 1e-10 * (p0 / 0.1)
    assert np.abs(rhs[5:]).max() < 1e-10 * (rho.max() * 1.0 / 0.1)


def _boundary_state(dim, seed=0):
    rng = np.random.default_rng(seed)
    n = 7
    nb = rng.standard_normal((dim, n, 1))
    nb /= np.linalg.norm(nb, axis=0)
    q = np.zeros((dim + 2 + 2, n, 1))
    q[0] = 1.0 + 0.1 * rng.random((n, 1))
    q[2:2 + dim] = rng.standard_normal((dim, n, 1))
    q[1] = 2.5 + 0.5 * np.sum(q[2:2 + dim] ** 2, axis=0) / q[0]
    q[2 + dim:] = q[0] * np.array([0.3, 0.2])[:, None, None]
    gas = oph.IdealGas()
    return q, nb, gas, oph.make_fluid_state(q, gas, None, dim)


@pytest.mark.parametrize("dim", [2, 3])
def test_wall_states(dim):
    """test_bc.py:432-778, 974-1055 restated: no-slip states have zero
    momentum, the isothermal wall's temperature is the wall temperature, the
    slip state has no normal momentum and the reflected state reverses it."""
    q, nb, gas, sm = _boundary_state(dim)
    iso = odg.IsothermalWallBoundary(wall_temperature=2.0)
    sbc = iso.state_bc(sm, gas, None, nb, dim)
    assert np.all(sbc["cv"][2:2 + dim] == 0.0)
    assert np.allclose(sbc["temperature"], 2.0, rtol=1e-14)
    assert np.all(iso.temperature_bc(sm) == 2.0)
    nos = odg.AdiabaticNoslipWallBoundary()
    assert np.all(nos.state_bc(sm, gas, None, nb, dim)["cv"][2:2 + dim] == 0.0)
    assert np.allclose(nos.state_plus(sm, gas, None, nb, dim)["cv"][2:2 + dim],
                       -q[2:2 + dim], rtol=0, atol=0)
    slip = odg.AdiabaticSlipBoundary()
    mbc = slip.state_bc(sm, gas, None, nb, dim)["cv"][2:2 + dim]
    assert np.abs(np.sum(mbc * nb, axis=0)).max() < 1e-14
    mp = slip.state_plus(sm, gas, None, nb, dim)["cv"][2:2 + dim]
    assert np.allclose(np.sum(mp * nb, axis=0), -np.sum(q[2:2 + dim] * nb, axis=0),
                       rtol=1e-13, atol=1e-14)
    # the slip state keeps the internal energy (and so the temperature)
    assert np.allclose(slip.state_bc(sm, gas, None, nb, dim)["temperature"],
                       sm["temperature"], rtol=1e-13)


def _reference_frame(n):
    """The reference's boundary frame (mirgecom/boundary.py:75-117), for
    normals whose z component is nonzero in 3-D: rows n, t1, t2."""
    dim = n.shape[0]
    n = n / np.linalg.norm(n)
    if dim == 2:
        return np.array([n, [-n[1], n[0]]])
    x, y, z = n
    a = np.sign(z)
    b = z + a
    v2 = np.array([a * b - x * x, -x * y, -x * b])
    v2 = v2 / np.linalg.norm(v2)
    v3 = np.array([y * v2[2] - v2[1] * z, v2[0] * z - x * v2[2], x * v2[1] - y * v2[0]])
    return np.array([n, v2, v3])


@pytest.mark.parametrize("dim", [2, 3])
def test_slip_velocity_gradient_matches_rotated_frame(dim):
    q, nb, gas, sm = _boundary_state(dim, seed=3)
    rng = np.random.default_rng(5)
    gcv = rng.standard_normal((q.shape[0], dim) + q.shape[1:])
    mine = odg._grad_velocity_slip(sm, gcv, nb, dim)
    rho = q[0]
    v = q[2:2 + dim] / rho
    g = (gcv[2:2 + dim] - v[:, None] * gcv[0][None]) / rho
    for i in range(q.shape[1]):
        r = _reference_frame(nb[:, i, 0])
        gn = r @ g[:, :, i, 0] @ r.T
        for k in range(dim - 1):
            gn[k + 1][0] = 0.0
        ref = r.T @ gn @ r
        assert np.allclose(mine[:, :, i, 0], ref, rtol=1e-12, atol=1e-13)
