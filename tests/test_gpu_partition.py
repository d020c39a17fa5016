"""Partitioned right-hand sides on the device, ranks emulated in one process.

Each emulated rank holds its owned elements and ghosts
(:class:`~mirgecom_b200.partition.PartitionedDiscretization`); the ghost
rows of q are exchanged, each rank makes its fluid state, runs the volume
kernel, the ranks exchange the ghosts' face records, and each runs the face
kernel.  The launches are sequential on one GPU and the data moves by device
copies (no kernel waits on another).  The owned rows of every rank together
equal the single-domain right-hand side: per element the kernels do the same
arithmetic, so the results agree to roundoff (1e-14 per field here).
"""

import numpy as np
import pytest
import torch

from cases import assert_fields_close, make_disc, tgv_np
from mirgecom_b200 import runtime
from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.navierstokes import ns_operator
from mirgecom_b200.partition import HaloExchange, LocalTransport, PartitionedDiscretization
from mirgecom_b200.thermochemistry import UIUC_7SP
from mirgecom_b200.transport import SimpleTransport

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _volume_face_layout():
    """The single-domain reference through the layout the partitioned
    phases run (the gradient, flux-volume and face kernels), so the two
    differ by roundoff of the same arithmetic only."""
    saved = runtime.RHS_PATH
    runtime.RHS_PATH = "gradient_volume_face"
    yield
    runtime.RHS_PATH = saved


def _partitioned_rhs(d, gas, q_glob, tseed_glob, nparts, dtype, sources):
    pds = [PartitionedDiscretization(d, r, nparts) for r in range(nparts)]
    tr = LocalTransport(nparts)
    exs = [HaloExchange(pd, tr) for pd in pds]
    qs = [pd.scatter(q_glob).clone() for pd in pds]
    for pd, ql in zip(pds, qs):
        ql[:, pd.nowned:] = float("nan")          # the exchange must fill every ghost row
    hs = [ex.begin_rows([ql]) for ex, ql in zip(exs, qs)]
    for ex, h in zip(exs, hs):
        ex.end(h)
    states = []
    for pd, ql in zip(pds, qs):
        ts = None if tseed_glob is None else pd.scatter(tseed_glob[None])[0]
        states.append(make_fluid_state(ConservedVars(ql.to(dtype), 3), gas,
                                       temperature_seed=ts))
    rhss = []
    for pd, st in zip(pds, states):
        src = st.temperature if sources else None
        r, _ = runtime.ns_rhs(pd, st, gas, {}, 0.0, 0, source_temperature=src, phases=1)
        rhss.append(r)
    traces = []
    for pd, st in zip(pds, states):
        dd = runtime.device_discretization(pd, st.cv.q.device)
        gs = runtime._gas_struct(gas, st.cv.nspecies, st.cv.q.device)
        traces.append(runtime.face_records(dd, gs, dtype == torch.float32, st.cv.q.shape[0]))
    hs = [ex.begin_records(t) for ex, t in zip(exs, traces)]
    for ex, h in zip(exs, hs):
        ex.end(h)
    out = torch.empty_like(q_glob, dtype=dtype)
    for pd, st, r in zip(pds, states, rhss):
        src = st.temperature if sources else None
        runtime.ns_rhs(pd, st, gas, {}, 0.0, 0, source_temperature=src, phases=2, rhs=r)
        out[:, torch.as_tensor(pd.owned, device=out.device)] = r[:, :pd.nowned]
        assert runtime.read_status(pd) == 0
    return out


@pytest.mark.parametrize("nparts", [2, 3])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_partitioned_tgv_matches_single_domain(cuda, nparts, dtype):
    d, od = make_disc("simplex", 3, 4, 3, (-np.pi,) * 3, (np.pi,) * 3, True)
    q = torch.from_numpy(tgv_np(od.nodes)).to(cuda)
    mu = 1.0 / 1600
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        viscosity=mu, thermal_conductivity=mu * 1004.85 / 0.71))
    ref = ns_operator(d, gas, make_fluid_state(ConservedVars(q.to(dtype), 3), gas), {})
    got = _partitioned_rhs(d, gas, q, None, nparts, dtype, False)
    tol = 1e-14 if dtype == torch.float64 else 1e-6
    assert_fields_close(got.double().cpu().numpy(), ref.q.double().cpu().numpy(), tol)


@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_mixture_matches_single_domain(cuda, nparts):
    from mirgecom_b200.initializers import reacting_mixture_state
    d, od = make_disc("simplex", 3, 3, 2, (0.0,) * 3, (2 * np.pi,) * 3, True)
    cv0, t_true = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                         UIUC_7SP, seed=12)
    q = cv0.q.to(cuda)
    tseed = (t_true + 4.0).to(cuda)
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5),
                   transport=SimpleTransport(viscosity=1e-5, thermal_conductivity=1e-5,
                                             species_diffusivity=[1e-5] * 7))
    st = make_fluid_state(ConservedVars(q, 3), gas, temperature_seed=tseed)
    ref = ns_operator(d, gas, st, {}, species_source_temperature=st.temperature)
    got = _partitioned_rhs(d, gas, q, tseed, nparts, torch.float64, True)
    assert_fields_close(got.cpu().numpy(), ref.q.cpu().numpy(), 1e-14)
