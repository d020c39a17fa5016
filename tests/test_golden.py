"""Committed golden vectors (tests/golden/*.npz, made by make_golden.py).

CPU: the oracle still reproduces them (guards the checker against drift).
GPU: the device path, called through the public API, matches them at the
float64 parity bar -- without running the oracle.
"""

import os
import sys

import numpy as np
import pytest
import torch

from cases import field_errors, inviscid_flux_floor, make_disc, vortex_np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_golden  # noqa: E402

NAMES = sorted(make_golden.CASES)
TOL = 1e-12


def _load(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name):
    g = _load(name)
    new = make_golden.build(name)
    for k in ("q", "rhs", "temperature", "tseed"):
        if k in g:
            scale = max(np.abs(g[k]).max(), 1e-300)
            assert np.abs(new[k] - g[k]).max() <= 1e-13 * scale, k


def _disc(g):
    d, _ = make_disc("simplex", int(g["dim"]), int(g["n"]), int(g["order"]),
                     tuple(g["lo"]), tuple(g["hi"]), bool(g["periodic"]))
    return d


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_matches_golden(cuda, name):
    from mirgecom_b200 import runtime
    from mirgecom_b200.boundary import PrescribedFluidBoundary
    from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture
    from mirgecom_b200.euler import euler_operator
    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import GasModel, make_fluid_state
    from mirgecom_b200.inviscid import inviscid_facial_flux_rusanov
    from mirgecom_b200.navierstokes import ns_operator
    from mirgecom_b200.thermochemistry import UIUC_7SP
    from mirgecom_b200.transport import SimpleTransport

    g = _load(name)
    d = _disc(g)
    dim = int(g["dim"])
    q = torch.from_numpy(g["q"]).to(cuda)
    if name == "vortex2d_p3":
        gas = GasModel(eos=IdealSingleGas())

        def bnd(dcoll, dd_bdry, gas_model, state_minus, time, nodes, **kw):
            qb = vortex_np(nodes.cpu().numpy(), t=time)
            return make_fluid_state(ConservedVars(torch.from_numpy(qb).to(cuda), 2), gas_model)

        rhs = euler_operator(d, make_fluid_state(ConservedVars(q, dim), gas), gas,
                             {"all": PrescribedFluidBoundary(boundary_state_func=bnd)},
                             time=float(g["time"]),
                             inviscid_numerical_flux_func=inviscid_facial_flux_rusanov)
        floor = None
    elif name == "tgv3d_p3":
        gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
            viscosity=make_golden.TGV_MU, thermal_conductivity=make_golden.TGV_KAPPA))
        rhs = ns_operator(d, gas, make_fluid_state(ConservedVars(q, dim), gas), {})
        floor = inviscid_flux_floor(g["q"], 3, 2 * np.pi / int(g["n"]))
    else:
        tr = SimpleTransport(**make_golden.MIX_TRANSPORT)
        gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5), transport=tr)
        st = make_fluid_state(ConservedVars(q, dim), gas,
                              temperature_seed=torch.from_numpy(g["tseed"]).to(cuda))
        t = st.temperature.cpu().numpy()
        assert np.abs(t - g["temperature"]).max() / g["temperature"].min() < 1e-13
        rhs = ns_operator(d, gas, st, {}, species_source_temperature=st.temperature)
        # each field against its own norm, or its inviscid flux scale
        # |F_c|/h where that is larger (the low-Mach momentum fields)
        h = (float(g["hi"][0]) - float(g["lo"][0])) / int(g["n"])
        floor = inviscid_flux_floor(g["q"], dim, h, temperature=g["temperature"],
                                    mech=UIUC_7SP)
    own, scaled = field_errors(rhs.q.cpu().numpy(), g["rhs"], floor)
    assert max(scaled) < TOL, (own, scaled)
    assert runtime.read_status(d) == 0
