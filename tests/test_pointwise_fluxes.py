"""The host-side pointwise numerical fluxes (mirgecom/inviscid.py:105-287 on
FluidState pairs, torch CPU tensors) against the oracle's, for the ideal gas
and the uiuc_7sp mixture (sound speed and gamma from NASA-7 c_p)."""

import numpy as np
import pytest
import torch

from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import FluidState, GasModel
from mirgecom_b200.inviscid import (inviscid_facial_flux_central, inviscid_facial_flux_hll,
                                    inviscid_facial_flux_rusanov)
from mirgecom_b200.thermochemistry import UIUC_7SP
from oracle import physics as oph

FLUX = {"rusanov": (inviscid_facial_flux_rusanov, oph.inviscid_facial_flux_rusanov),
        "hll": (inviscid_facial_flux_hll, oph.inviscid_facial_flux_hll),
        "central": (inviscid_facial_flux_central, oph.inviscid_facial_flux_central)}


def _ideal_pair(n, seed):
    rng = np.random.default_rng(seed)
    dim = 3
    out = []
    for _ in range(2):
        rho = rng.uniform(0.5, 2.0, n)
        v = rng.uniform(-1, 1, (dim, n))
        p = rng.uniform(0.5, 2.0, n)
        q = np.empty((dim + 2, n))
        q[0] = rho
        q[1] = p / 0.4 + 0.5 * rho * (v * v).sum(axis=0)
        q[2:] = rho * v
        out.append(q)
    return out


def _mixture_pair(n, seed):
    from mirgecom_b200.initializers import _nasa_e_rt
    from mirgecom_b200.thermochemistry import GAS_CONSTANT
    rng = np.random.default_rng(seed)
    mech = UIUC_7SP
    out = []
    for _ in range(2):
        t = rng.uniform(400.0, 2400.0, n)
        y = rng.dirichlet([2.0] * mech.nspecies, n).T
        w = mech.molecular_weights[:, None]
        rho = rng.uniform(0.2, 1.2, n)
        v = rng.uniform(-10, 10, (3, n))
        e_rt = _nasa_e_rt(mech, torch.from_numpy(t)).numpy()
        e = GAS_CONSTANT * t * (y * e_rt / w).sum(axis=0)
        q = np.concatenate([rho[None], (rho * (e + 0.5 * (v * v).sum(axis=0)))[None],
                            rho * v, rho * y])
        out.append((q, t))
    return out


@pytest.mark.parametrize("flux", sorted(FLUX))
def test_ideal_gas_fluxes(flux):
    qm, qp = _ideal_pair(200, 0)
    normal = np.random.default_rng(1).normal(size=(3, 200))
    normal /= np.linalg.norm(normal, axis=0)
    gas = GasModel(eos=IdealSingleGas())
    sm = FluidState(ConservedVars(torch.from_numpy(qm), 3), gas)
    sp = FluidState(ConservedVars(torch.from_numpy(qp), 3), gas)
    ours, ref = FLUX[flux]
    got = ours((sm, sp), gas, torch.from_numpy(normal)).numpy()
    want = ref(oph.make_fluid_state(qm, oph.IdealGas(), None, 3),
               oph.make_fluid_state(qp, oph.IdealGas(), None, 3), normal)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("flux", sorted(FLUX))
def test_mixture_fluxes(flux):
    (qm, tm), (qp, tp) = _mixture_pair(200, 2)
    normal = np.random.default_rng(3).normal(size=(3, 200))
    normal /= np.linalg.norm(normal, axis=0)
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP))
    sm = FluidState(ConservedVars(torch.from_numpy(qm), 3), gas, temperature=torch.from_numpy(tm))
    sp = FluidState(ConservedVars(torch.from_numpy(qp), 3), gas, temperature=torch.from_numpy(tp))
    ours, ref = FLUX[flux]
    got = ours((sm, sp), gas, torch.from_numpy(normal)).numpy()
    og = oph.MixtureGas(UIUC_7SP, temperature_niter=5)
    want = ref(oph.make_fluid_state(qm, og, None, 3, temperature_seed=tm),
               oph.make_fluid_state(qp, og, None, 3, temperature_seed=tp), normal)
    assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()
