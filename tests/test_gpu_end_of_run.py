"""End of run of the reacting configuration on a reduced mesh, mixed + learned
against float64.

The 40^3 order-2 reacting configuration's physics (uiuc_7sp with Arrhenius
sources, SimpleTransport 1e-5, smooth random T in 300-2500 K, p = 101325 +-
5 %, Dirichlet(2) mass fractions, |v| <= 10 m/s) on a 4^3 x 6 tetrahedra
order-2 periodic box: 200 RK4 steps at the chemistry-resolving step (the
smallest chemical time scale rho Y_k / |W_k omega_k| of the initial state over
64, as the benchmark takes it) in the float64 form (rk4_step, the reference's
fixed-count Newton) and in the headline form (rk4_step_mixed: float64 RK
accumulation, float32 right-hand sides, the mixed Newton from a trained
network's guess and the warm step-start seed), each form seeding its
temperature solve with its own previous temperature.  Every conserved field
ends within 1e-6 relative L2 of the float64 run (momentum against the
momentum norm), and the temperatures within 1e-6, while the float64 state
itself changes by far more (the states ignite).
"""

import numpy as np
import pytest
import torch

from cases import make_disc
from mirgecom_b200 import runtime
from mirgecom_b200.eos import PyrometheusMixture
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.initializers import reacting_mixture_state
from mirgecom_b200.integrators import rk4_step, rk4_step_mixed
from mirgecom_b200.learned_guess import TemperatureMLP
from mirgecom_b200.navierstokes import ns_operator
from mirgecom_b200.thermochemistry import UIUC_7SP
from mirgecom_b200.transport import SimpleTransport

pytestmark = pytest.mark.gpu

STEPS = 200


def _transport():
    return SimpleTransport(viscosity=1e-5, thermal_conductivity=1e-5,
                           species_diffusivity=[1e-5] * 7)


def _chemical_time_scale(d, gas, q, t):
    st = make_fluid_state(ConservedVars(q, 3), gas, temperature_seed=t)
    with_src, _ = runtime.ns_rhs(d, st, gas, {}, 0.0, 0, source_temperature=st.temperature)
    without, _ = runtime.ns_rhs(d, st, gas, {}, 0.0, 0)
    src = (with_src - without)[5:]
    rhoy = q[5:]
    tau = rhoy.abs() / src.abs().clamp_min(1e-300)
    mask = (rhoy / q[0]) > 1e-3
    return float(torch.where(mask, tau, torch.full_like(tau, float("inf"))).min())


def test_reacting_200_steps_within_1e6(cuda):
    d, od = make_disc("simplex", 3, 4, 2, (0.0,) * 3, (2 * np.pi,) * 3, True)
    cv0, t_true = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                         UIUC_7SP, seed=0)
    q64 = cv0.q.to(cuda)
    t64 = (t_true + 2.0).to(cuda)
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5), transport=_transport())
    net = TemperatureMLP(cuda, seed=0)
    e, y, t = TemperatureMLP.training_pairs(UIUC_7SP, 1 << 16, cuda, seed=0)
    net.fit(e, y, t, steps=300, batch=16384, lr=3e-3, seed=0)
    gas_head = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5,
                                               learned_guess=net), transport=_transport())
    dt = _chemical_time_scale(d, gas, q64, t64) / 64

    def factory(g, box):
        def rhs(time, cv):
            st = make_fluid_state(cv, g, temperature_seed=box[0])
            return ns_operator(d, g, st, {}, species_source_temperature=st.temperature)
        return rhs

    s64 = ConservedVars(q64.clone(), 3)
    shi, slo = ConservedVars(q64.clone(), 3), None
    b64, b32 = [t64.clone()], [t64.to(torch.float32)]
    for i in range(STEPS):
        s64 = rk4_step(s64, i * dt, dt, factory(gas, b64))
        b64[0] = make_fluid_state(s64, gas, temperature_seed=b64[0]).temperature
        shi, slo = rk4_step_mixed(shi, i * dt, dt, factory(gas_head, b32), slo)
        b32[0] = make_fluid_state(slo, gas_head, temperature_seed=b32[0]).temperature
    assert runtime.read_status(d) == 0
    a, b, q0 = shi.q.cpu().numpy(), s64.q.cpu().numpy(), q64.cpu().numpy()
    mom = np.linalg.norm(b[2:5].ravel())

    def rel(x, c):
        ref = mom if 2 <= c < 5 else np.linalg.norm(b[c].ravel())
        return float(np.linalg.norm((x[c] - b[c]).ravel()) / ref)
    err = [rel(a, c) for c in range(b.shape[0])]
    moved = [rel(q0, c) for c in range(b.shape[0])]
    assert max(moved) > 1e-2, moved                 # the run does something
    assert max(err) < 1e-6, err
    tb = b64[0].cpu().numpy()
    ta = b32[0].double().cpu().numpy()
    assert np.linalg.norm(ta - tb) / np.linalg.norm(tb) < 1e-6
