"""The tcgen05/TMEM gradient kernel against the mma.sync gradient kernel.

Float32 mixture states on 3-D simplices take the pipelined tcgen05 kernel
(grad_tc.cuh) unless the mma.sync kernel is selected
(``runtime.set_gradient_kernel``).  Both compute the BR1 gradients
(mirgecom/navierstokes.py:443-446) with the same element-constant shift and
TF32 three-term split, in a different summation order: they agree per field
to float32 roundoff of the shifted values, and each is as close to the
float64 gradients as the other.  Cases: periodic p3 and p1 boxes whose
element counts leave a ragged last tile, every wall and flow boundary
(prescribed and Mengaldo face values), and the owned elements of a mesh
partition.
"""

import numpy as np
import pytest
import torch

from cases import assert_fields_close, field_errors, gradient_floor, make_disc
from mirgecom_b200 import runtime
from mirgecom_b200.boundary import (AdiabaticNoslipWallBoundary, AdiabaticSlipBoundary,
                                    FarfieldBoundary, IsothermalWallBoundary,
                                    PressureOutflowBoundary)
from mirgecom_b200.eos import PyrometheusMixture
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.partition import PartitionedDiscretization
from mirgecom_b200.thermochemistry import UIUC_7SP
from mirgecom_b200.transport import SimpleTransport

pytestmark = pytest.mark.gpu

AGREE = 2e-6       # the two float32 kernels, per field against |q_c| / h


def _mixture(d, od, cuda, box, seed):
    from mirgecom_b200.initializers import reacting_mixture_state
    cv0, t_true = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                         UIUC_7SP, seed=seed, t_range=(900.0, 1500.0), box=box)
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5),
                   transport=SimpleTransport(viscosity=2e-5, thermal_conductivity=3e-2,
                                             species_diffusivity=[1e-5] * 7))
    q = cv0.q.to(cuda)
    tseed = (t_true + 3.0).to(cuda)
    st64 = make_fluid_state(ConservedVars(q, 3), gas, temperature_seed=tseed)
    st32 = make_fluid_state(ConservedVars(q.float(), 3), gas,
                            temperature_seed=st64.temperature.float())
    return gas, st64, st32


def _grads(d, gas, st, bnds, kind):
    runtime.set_gradient_kernel(kind)
    try:
        g = runtime.ns_gradients(d, st, gas, bnds, 0.0).clone()
    finally:
        runtime.set_gradient_kernel("auto")
    assert runtime.read_status(d) == 0
    return g


def _check(d, gas, st64, st32, bnds, h):
    g_tc = _grads(d, gas, st32, bnds, "auto")
    g_mma = _grads(d, gas, st32, bnds, "mma_sync")
    g64 = _grads(d, gas, st64, bnds, "auto")
    q = np.concatenate([st64.cv.q.cpu().numpy(), st64.temperature.cpu().numpy()[None]])
    floor = np.repeat(gradient_floor(q, h), 3)
    nf = g64.shape[0] * g64.shape[1]
    a = g_tc.double().cpu().numpy().reshape((nf,) + g64.shape[2:])
    b = g_mma.double().cpu().numpy().reshape((nf,) + g64.shape[2:])
    r = g64.cpu().numpy().reshape((nf,) + g64.shape[2:])
    assert_fields_close(a, b, AGREE, floor=floor, what="gradient")
    e_tc = field_errors(a, r, floor)[1]
    e_mma = field_errors(b, r, floor)[1]
    for c in range(nf):
        assert e_tc[c] <= 2.0 * e_mma[c] + 1e-7, (c, e_tc[c], e_mma[c])


@pytest.mark.parametrize("order,n", [(3, 4), (1, 5)])
def test_periodic(cuda, order, n):
    box = (0.02, 0.014, 0.026)
    d, od = make_disc("simplex", 3, n, order, (0.0,) * 3, box, True)
    assert d.nelements % (128 // 13) != 0          # a ragged last tile
    gas, st64, st32 = _mixture(d, od, cuda, box, seed=3)
    _check(d, gas, st64, st32, {}, min(box) / n)


def test_walls(cuda):
    box = (0.02, 0.014, 0.026)
    d, od = make_disc("simplex", 3, 3, 3, (0.0,) * 3, box, False)
    gas, st64, st32 = _mixture(d, od, cuda, box, seed=8)
    y_fs = [0.05, 0.22, 0.0, 0.0, 0.0, 0.0, 0.73]
    bnds = {"-0": AdiabaticSlipBoundary(),
            "+0": PressureOutflowBoundary(boundary_pressure=101325.0),
            "-1": IsothermalWallBoundary(wall_temperature=1000.0),
            "+1": AdiabaticNoslipWallBoundary(),
            "-2": FarfieldBoundary(101325.0, [3.0, -1.0, 2.0], 1200.0, y_fs),
            "+2": AdiabaticSlipBoundary()}
    _check(d, gas, st64, st32, bnds, min(box) / 3)


def test_partition_owned_rows(cuda):
    box = (0.02, 0.014, 0.026)
    d, od = make_disc("simplex", 3, 4, 3, (0.0,) * 3, box, True)
    gas, st64, st32 = _mixture(d, od, cuda, box, seed=5)
    g_all = _grads(d, gas, st32, {}, "auto")
    for rank in range(2):
        pd = PartitionedDiscretization(d, rank, 2)
        q = pd.scatter(st32.cv.q)
        t = pd.scatter(st32.temperature[None])[0]
        st = make_fluid_state(ConservedVars(q.contiguous(), 3), gas, temperature_seed=t)
        g = _grads(pd, gas, st, {}, "auto")
        own = torch.as_tensor(pd.owned, device=g.device)
        a = g[:, :, :pd.nowned].double().cpu().numpy()
        b = g_all[:, :, own].double().cpu().numpy()
        nf = a.shape[0] * a.shape[1]
        assert_fields_close(a.reshape((nf,) + a.shape[2:]), b.reshape((nf,) + b.shape[2:]),
                            1e-6, what="gradient")
