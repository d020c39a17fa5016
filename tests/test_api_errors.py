"""The reference's error conventions on the drop-in surface (CPU; every
check fires before any device work):

* a non-volume ``dd`` -> TypeError, a quadrature other than the base one ->
  ValueError (mirgecom/euler.py:369-372, navierstokes.py:450-453);
* ``ns_operator`` on a gas without transport -> ValueError
  (navierstokes.py:445-446);
* a mixture state without a temperature seed -> TemperatureSeedMissingError
  (eos.py:54, 796-798);
* an unspecified inviscid flux -> a warning and Rusanov (euler.py:378-383);
* CPU tensors reaching the device path -> RuntimeError (no CPU fallback).
"""

import numpy as np
import pytest
import torch

from cases import make_disc, perturbed_state_np
from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture, TemperatureSeedMissingError
from mirgecom_b200.euler import euler_operator
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.inviscid import inviscid_facial_flux_rusanov
from mirgecom_b200.navierstokes import ns_operator
from mirgecom_b200.thermochemistry import UIUC_7SP
from mirgecom_b200.transport import SimpleTransport


@pytest.fixture(scope="module")
def case():
    d, od = make_disc("simplex", 2, 3, 1, (0.0, 0.0), (1.0, 1.0), True)
    q = perturbed_state_np(od.nodes, 2, 0, seed=2)
    return d, ConservedVars(torch.from_numpy(q), 2)


def test_bad_dd_and_quadrature(case):
    d, cv = case
    gas = GasModel(eos=IdealSingleGas())
    st = make_fluid_state(cv, gas)
    with pytest.raises(TypeError):
        euler_operator(d, st, gas, {}, dd="all_faces",
                       inviscid_numerical_flux_func=inviscid_facial_flux_rusanov)
    with pytest.raises(ValueError):
        euler_operator(d, st, gas, {}, quadrature_tag="quad",
                       inviscid_numerical_flux_func=inviscid_facial_flux_rusanov)
    vgas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(viscosity=1e-3))
    with pytest.raises(TypeError):
        ns_operator(d, vgas, make_fluid_state(cv, vgas), {}, dd="all_faces")


def test_ns_operator_needs_transport(case):
    d, cv = case
    gas = GasModel(eos=IdealSingleGas())
    with pytest.raises(ValueError):
        ns_operator(d, gas, make_fluid_state(cv, gas), {})


def test_mixture_needs_temperature_seed():
    q = np.ones((4 + UIUC_7SP.nspecies, 2, 3)) * 0.1
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP))
    with pytest.raises(TemperatureSeedMissingError):
        make_fluid_state(ConservedVars(torch.from_numpy(q), 2), gas)


def test_default_flux_warns_and_cpu_tensors_are_refused(case):
    d, cv = case
    gas = GasModel(eos=IdealSingleGas())
    st = make_fluid_state(cv, gas)
    with pytest.warns(UserWarning, match="rusanov"):
        with pytest.raises(RuntimeError):
            euler_operator(d, st, gas, {})


def test_unsupported_options(case):
    d, cv = case
    gas = GasModel(eos=IdealSingleGas())
    st = make_fluid_state(cv, gas)
    with pytest.raises(NotImplementedError):
        euler_operator(d, st, gas, {}, use_esdg=True,
                       inviscid_numerical_flux_func=inviscid_facial_flux_rusanov)
    vgas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(viscosity=1e-3))
    with pytest.raises(NotImplementedError):
        ns_operator(d, vgas, make_fluid_state(cv, vgas), {}, inviscid_terms_on=False)
