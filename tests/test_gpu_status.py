"""Device status bits: problems found on the device come back in the status
word, never as a trap, and the context stays usable afterwards.

The reference raises nothing for numerical failures; its drivers check the
state's health between steps (mirgecom/simutil.py:480-506: NaN checks of
the conserved fields, temperature bounds).  Here the kernels OR bits into a
status word instead (MGC_ST_NAN for a NaN flux or right-hand side,
MGC_ST_NEWTON_MISS for a temperature solve that did not converge), which
:func:`runtime.read_status` reads.  Each test plants the problem in the host
data it uploads and checks the bit, then runs a clean evaluation and checks
that it reports nothing.
"""

import numpy as np
import pytest
import torch

from cases import make_disc, perturbed_state_np, tgv_np
from mirgecom_b200 import _lib, runtime
from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture
from mirgecom_b200.euler import euler_operator
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.navierstokes import ns_operator
from mirgecom_b200.thermochemistry import UIUC_7SP
from mirgecom_b200.transport import SimpleTransport

pytestmark = pytest.mark.gpu


def _cv(q, dim, dev, dtype=torch.float64):
    return ConservedVars(torch.from_numpy(np.ascontiguousarray(q)).to(dev, dtype), dim)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_nan_in_state_sets_nan_bit_euler(cuda, dtype):
    d, od = make_disc("simplex", 3, 3, 2, (0.0,) * 3, (2 * np.pi,) * 3, True)
    q = perturbed_state_np(od.nodes, 3, 0, seed=1)
    gas = GasModel(eos=IdealSingleGas())
    runtime.read_status(d)                       # start from a clear word
    bad = q.copy()
    bad[1, 5, 3] = np.nan                         # one node's energy
    rhs = euler_operator(d, make_fluid_state(_cv(bad, 3, cuda, dtype), gas), gas, {})
    st = runtime.read_status(d)
    assert st & _lib.ST_NAN, st
    assert torch.isnan(rhs.q).any()
    # the context is intact: a clean state reports nothing
    rhs = euler_operator(d, make_fluid_state(_cv(q, 3, cuda, dtype), gas), gas, {})
    assert runtime.read_status(d) == 0
    assert torch.isfinite(rhs.q).all()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_nan_in_state_sets_nan_bit_ns(cuda, dtype):
    d, od = make_disc("simplex", 3, 3, 3, (-np.pi,) * 3, (np.pi,) * 3, True)
    q = tgv_np(od.nodes)
    mu = 1.0 / 1600
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        viscosity=mu, thermal_conductivity=mu * 1004.85 / 0.71))
    runtime.read_status(d)
    bad = q.copy()
    bad[2, 17, 0] = np.nan                        # one node's x momentum
    ns_operator(d, gas, make_fluid_state(_cv(bad, 3, cuda, dtype), gas), {})
    assert runtime.read_status(d) & _lib.ST_NAN
    ns_operator(d, gas, make_fluid_state(_cv(q, 3, cuda, dtype), gas), {})
    assert runtime.read_status(d) == 0


def _mixture_case(cuda):
    from mirgecom_b200.initializers import reacting_mixture_state
    d, od = make_disc("simplex", 3, 3, 2, (0.0,) * 3, (2 * np.pi,) * 3, True)
    cv0, t_true = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                         UIUC_7SP, seed=3)
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5),
                   transport=SimpleTransport(viscosity=1e-5, thermal_conductivity=1e-5,
                                             species_diffusivity=[1e-5] * 7))
    return d, cv0.q.numpy(), t_true.numpy(), gas


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_energy_outside_nasa7_range_sets_newton_miss(cuda, dtype):
    """A node whose internal energy (1e9 J/kg) lies far above what the NASA-7
    fits cover (about -1.2e6 .. 6.4e6 J/kg between 300 and 6000 K for these
    mixtures): the fixed-count float64 Newton does not converge there, and
    the mixed solve fails its float64 residual check from both start
    values."""
    d, q, t_true, gas = _mixture_case(cuda)
    runtime.read_status(d)
    bad = q.copy()
    e, n = 2, 4
    ke = 0.5 * np.sum(bad[2:5, e, n] ** 2) / bad[0, e, n]
    bad[1, e, n] = bad[0, e, n] * 1e9 + ke
    seed = torch.from_numpy(t_true).to(cuda)
    st = make_fluid_state(_cv(bad, 3, cuda, dtype), gas, temperature_seed=seed)
    torch.cuda.synchronize()
    assert runtime.read_status(d) & _lib.ST_NEWTON_MISS
    # the other nodes still got their temperatures
    t = st.temperature.double().cpu().numpy()
    mask = np.ones_like(t, dtype=bool)
    mask[e, n] = False
    tol = 1e-12 if dtype == torch.float64 else 1e-6
    assert np.max(np.abs(t[mask] - t_true[mask]) / t_true[mask]) < tol
    # a clean state reports nothing
    make_fluid_state(_cv(q, 3, cuda, dtype), gas, temperature_seed=seed)
    assert runtime.read_status(d) == 0


def test_nan_in_mixture_state_sets_bits(cuda):
    """A NaN in one node's mass fraction: the temperature solve misses and the
    right-hand side carries the NaN (both bits), on the float64 path."""
    d, q, t_true, gas = _mixture_case(cuda)
    runtime.read_status(d)
    bad = q.copy()
    bad[7, 1, 2] = np.nan
    seed = torch.from_numpy(t_true).to(cuda)
    st = make_fluid_state(_cv(bad, 3, cuda), gas, temperature_seed=seed)
    ns_operator(d, gas, st, {}, species_source_temperature=st.temperature)
    s = runtime.read_status(d)
    assert s & _lib.ST_NAN and s & _lib.ST_NEWTON_MISS, s
    st = make_fluid_state(_cv(q, 3, cuda), gas, temperature_seed=seed)
    ns_operator(d, gas, st, {}, species_source_temperature=st.temperature)
    assert runtime.read_status(d) == 0
