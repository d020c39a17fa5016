"""Time-step estimates (mirgecom/inviscid.py:379-422, viscous.py:547-607,
simutil.py:224-306) against the oracle's restatement, plus the analytic
inradius of the box meshes' cells.  CPU (torch CPU tensors)."""

import numpy as np
import pytest
import torch

from cases import make_disc, perturbed_state_np, tgv_np
from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import FluidState, GasModel
from mirgecom_b200.inviscid import get_inviscid_timestep
from mirgecom_b200.simutil import get_sim_timestep
from mirgecom_b200.thermochemistry import UIUC_7SP
from mirgecom_b200.transport import PowerLawTransport, SimpleTransport
from mirgecom_b200.viscous import get_viscous_timestep
from oracle import dg as odg
from oracle import physics as oph


def test_inradius_of_box_cells():
    """Right triangles with legs h: r = h / (2 + sqrt 2); squares: h / 2;
    the p1 triangle's nodes are its vertices, min(dr) = 2 on [-1, 1]^2."""
    n = 4
    d, _ = make_disc("simplex", 2, n, 1, (0.0, 0.0), (1.0, 1.0), True)
    h = 1.0 / n
    assert np.allclose(d.characteristic_lengthscales().numpy(), 2 * h / (2 + np.sqrt(2)))
    d, _ = make_disc("hypercube", 2, n, 1, (0.0, 0.0), (1.0, 1.0), True)
    assert np.allclose(d.characteristic_lengthscales().numpy(), 2 * h / 2)


@pytest.mark.parametrize("kind,dim,order", [("simplex", 2, 3), ("simplex", 3, 2),
                                            ("hypercube", 3, 2)])
def test_timesteps_ideal_gas(kind, dim, order):
    d, od = make_disc(kind, dim, 3, order, (0.0,) * dim, (2.0, 1.0, 1.5)[:dim], False)
    q = perturbed_state_np(od.nodes, dim, 0, seed=1)
    tr = PowerLawTransport(beta=1e-2)
    gas = GasModel(eos=IdealSingleGas(), transport=tr)
    st = FluidState(ConservedVars(torch.from_numpy(q), dim), gas)
    ost = oph.make_fluid_state(q, oph.IdealGas(), oph.PowerLawTransportParams(beta=1e-2), dim)
    assert np.allclose(d.characteristic_lengthscales().numpy(),
                       odg.characteristic_lengthscales(od), rtol=1e-13, atol=0)
    assert np.allclose(get_inviscid_timestep(d, st).numpy(), odg.inviscid_timestep(od, ost),
                       rtol=1e-12, atol=0)
    vdt = get_viscous_timestep(d, st).numpy()
    assert np.allclose(vdt, odg.viscous_timestep(od, ost), rtol=1e-12, atol=0)
    # the three modes of get_sim_timestep
    assert get_sim_timestep(d, st, t=0.0, dt=1e-3, cfl=0.5, t_final=1.0) == 1e-3
    assert get_sim_timestep(d, st, t=0.9995, dt=1e-3, cfl=0.5, t_final=1.0) == \
        pytest.approx(5e-4)
    assert get_sim_timestep(d, st, t=0.0, dt=1e-3, cfl=0.5, t_final=1.0,
                            constant_cfl=True) == pytest.approx(0.5 * vdt.min())
    local = get_sim_timestep(d, st, t=0.0, dt=1e-3, cfl=0.5, local_dt=True).numpy()
    assert np.allclose(local, 0.5 * vdt.min(axis=1, keepdims=True) * np.ones_like(vdt))


def test_timesteps_mixture():
    """Mixture sound speed from NASA-7 c_p (host torch) and species
    diffusivities, against the oracle's state at the same temperature."""
    d, od = make_disc("simplex", 3, 3, 2, (0.0,) * 3, (2 * np.pi,) * 3, True)
    from mirgecom_b200.initializers import reacting_mixture_state
    cv, t = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                   UIUC_7SP, seed=3)
    diff = [1e-5 * (k + 1) for k in range(7)]
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP),
                   transport=SimpleTransport(viscosity=2e-5, thermal_conductivity=1e-5,
                                             species_diffusivity=diff))
    st = FluidState(cv, gas, temperature=t, operator_temperature=t)
    q = cv.q.numpy()
    ost = oph.make_fluid_state(q, oph.MixtureGas(UIUC_7SP, temperature_niter=5),
                               oph.SimpleTransportParams(viscosity=2e-5, thermal_conductivity=1e-5,
                                                         species_diffusivity=tuple(diff)),
                               3, temperature_seed=t.numpy())
    assert np.allclose(st.speed_of_sound.numpy(), ost["speed_of_sound"], rtol=1e-10, atol=0)
    assert np.allclose(get_viscous_timestep(d, st).numpy(), odg.viscous_timestep(od, ost),
                       rtol=1e-10, atol=0)
