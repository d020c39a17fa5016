"""The no-allocation NS entry point against the regular one.

``mgc_ns_operator_noalloc`` serves callers that cannot allocate device
memory (their device memory belongs to their own pool, or they link the
library with no CUDA allocation layer); it keeps the gradient scratch in a
fixed library-owned device array.  Two calls in a row must reproduce the
regular two-call path (mgc_ns_grad + mgc_ns_rhs with a caller buffer) within
the parity tolerance, and a mesh too large for the array must be rejected.
This file sorts last so a failure here leaves every other test already run.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from cases import make_disc, rel_l2, tgv_np
from mirgecom_b200 import _lib, runtime
from mirgecom_b200.eos import IdealSingleGas
from mirgecom_b200.gas_model import GasModel
from mirgecom_b200.transport import SimpleTransport

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _setup(cuda):
    d, od = make_disc("simplex", 3, 4, 3, (-np.pi,) * 3, (np.pi,) * 3, True)
    q = torch.from_numpy(tgv_np(od.nodes)).to(cuda).contiguous()
    mu = 1.0 / 1600
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        viscosity=mu, thermal_conductivity=mu * 1.4 * 287.1 / 0.4 / 0.71))
    dd = runtime.device_discretization(d, cuda)
    bkind = dd.bkind_for({})
    dd.mesh.bkind = bkind.data_ptr()
    gs = gas.to_struct(0)
    return d, dd, q, gs


def test_noalloc_matches_regular_entry_points(cuda):
    lib = _lib.load()
    d, dd, q, gs = _setup(cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    stream = _lib.stream_handle()
    nc = q.shape[0]
    grad = torch.empty((nc + 1, 3) + tuple(q.shape[1:]), dtype=torch.float64, device=cuda)
    ref = torch.empty_like(q)
    assert lib.mgc_ns_grad(C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), None, None,
                           _lib.ptr(grad), _lib.ptr(status), stream) == 0
    assert lib.mgc_ns_rhs(C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), None, None,
                          _lib.ptr(grad), None, 0, 0, _lib.ptr(ref), _lib.ptr(status),
                          stream) == 0
    outs = []
    for _ in range(2):
        out = torch.full_like(q, float("nan"))
        rc = lib.mgc_ns_operator_noalloc(C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), None,
                                         None, None, 0, 0, _lib.ptr(out), _lib.ptr(status),
                                         stream)
        assert rc == 0
        outs.append(out)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    for out in outs:
        assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < TOL


def test_noalloc_matches_regular_entry_points_mixture(cuda):
    """The 7-species mixture (operator temperature, source temperature,
    Arrhenius sources, 13-row gradient) on order-2 tetrahedra."""
    from mirgecom_b200.eos import PyrometheusMixture
    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.initializers import reacting_mixture_state
    from mirgecom_b200.thermochemistry import UIUC_7SP
    lib = _lib.load()
    d, od = make_disc("simplex", 3, 3, 2, (0.0,) * 3, (2 * np.pi,) * 3, True)
    cv0, t_true = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                         UIUC_7SP, seed=11)
    q = cv0.q.to(cuda).contiguous()
    gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5),
                   transport=SimpleTransport(viscosity=1e-5, thermal_conductivity=2e-5,
                                             species_diffusivity=[1e-5] * 7))
    dd = runtime.device_discretization(d, cuda)
    bkind = dd.bkind_for({})
    dd.mesh.bkind = bkind.data_ptr()
    gs = runtime._gas_struct(gas, 7, cuda)
    t1, t2 = runtime.mixture_temperature(ConservedVars(q, 3), gas, t_true.to(cuda) + 5.0)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    stream = _lib.stream_handle()
    nc = q.shape[0]
    grad = torch.empty((nc + 1, 3) + tuple(q.shape[1:]), dtype=torch.float64, device=cuda)
    ref = torch.empty_like(q)
    assert lib.mgc_ns_grad(C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t2), None,
                           _lib.ptr(grad), _lib.ptr(status), stream) == 0
    assert lib.mgc_ns_rhs(C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t2),
                          _lib.ptr(t1), _lib.ptr(grad), None, 0, 1, _lib.ptr(ref),
                          _lib.ptr(status), stream) == 0
    outs = []
    for _ in range(2):
        out = torch.full_like(q, float("nan"))
        rc = lib.mgc_ns_operator_noalloc(C.byref(dd.mesh), C.byref(gs), _lib.ptr(q),
                                         _lib.ptr(t2), _lib.ptr(t1), None, 0, 1, _lib.ptr(out),
                                         _lib.ptr(status), stream)
        assert rc == 0
        outs.append(out)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    r = ref.cpu().numpy()
    for out in outs:
        o = out.cpu().numpy()
        # field by field: the energy's magnitude would hide the species
        assert max(rel_l2(o[c], r[c]) for c in range(nc)) < TOL


def test_noalloc_rejects_meshes_beyond_capacity(cuda):
    lib = _lib.load()
    d, dd, q, gs = _setup(cuda)
    cap = lib.mgc_ns_operator_noalloc_capacity()
    big = _lib.MeshStruct()
    C.pointer(big)[0] = dd.mesh
    # (Nc+1) * dim * E * Np doubles must exceed the array: 6 * 3 * E * 20 > cap
    big.nelem = cap // (6 * 3 * 20) + 1
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    rc = lib.mgc_ns_operator_noalloc(C.byref(big), C.byref(gs), _lib.ptr(q), None, None,
                                     None, 0, 0, _lib.ptr(q), _lib.ptr(status),
                                     _lib.stream_handle())
    assert rc == -5
