"""Device runtime: uploads, workspaces and the C-ABI launches.

One :class:`DeviceDiscretization` per (Discretization, device) holds the
uploaded index arrays and geometry, the ``mgc_mesh_t`` descriptor and the
reusable workspaces (gradients, temperatures, boundary exterior states), so
that an RHS evaluation allocates nothing after its first call.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from mirgecom_b200 import _lib

_uploaded_refops = set()     # (device index, element kind, dim, order)
_uploaded_mech = {}          # device index -> id(mechanism)
_state_status = {}           # device index -> int32 status word of the state kernels


def _dev_index(device):
    return device.index if device.index is not None else torch.cuda.current_device()


def state_status_word(device):
    """The int32 device word into which the temperature kernels of this
    device OR their status bits (a fluid state is made without a
    discretization, so its solve reports here; :func:`read_status` reads it
    together with the discretization's word)."""
    idx = _dev_index(device)
    w = _state_status.get(idx)
    if w is None:
        w = torch.zeros(1, dtype=torch.int32, device=torch.device("cuda", idx))
        _state_status[idx] = w
    return w


def ensure_reference_operators(dcoll, device):
    key = (_dev_index(device), dcoll.refel.kind, dcoll.dim, dcoll.order)
    if key in _uploaded_refops:
        return
    r = dcoll.refel
    lib = _lib.load()
    if r.kind == "hypercube":
        if not lib.mgc_supports_hex(dcoll.dim, dcoll.order, 0, _lib.EOS_IDEAL):
            raise NotImplementedError(
                f"no device kernels for {dcoll.dim}-D hexahedra of order {dcoll.order}")
        w1 = np.ascontiguousarray(r.extra["weak1d"], dtype=np.float64)
        l1 = np.ascontiguousarray(r.extra["mass1d_inv"][:, [0, -1]], dtype=np.float64)
        with torch.cuda.device(device):
            _lib.check(lib.mgc_upload_hex_operators(
                dcoll.dim, dcoll.order, _lib.ptr(w1), _lib.ptr(l1),
                float(r.face_scale_ref[0])), "mgc_upload_hex_operators")
        _uploaded_refops.add(key)
        return
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
            (r.weak, r.lift, r.ref_face_normals, r.face_scale_ref)]
    fn = np.ascontiguousarray(r.face_nodes, dtype=np.int32)
    with torch.cuda.device(device):
        _lib.check(lib.mgc_upload_reference_operators(
            dcoll.dim, dcoll.order, *[_lib.ptr(a) for a in arrs], _lib.ptr(fn)),
            "mgc_upload_reference_operators")
    _uploaded_refops.add(key)


def ensure_mechanism(eos, device):
    idx = _dev_index(device)
    if _uploaded_mech.get(idx) is eos.mechanism:
        return
    lib = _lib.load()
    ms = eos.mechanism_struct()
    with torch.cuda.device(device):
        _lib.check(lib.mgc_set_mechanism(C.byref(ms)), "mgc_set_mechanism")
    _uploaded_mech[idx] = eos.mechanism


class DeviceDiscretization:
    def __init__(self, dcoll, device):
        self.dcoll = dcoll
        self.device = device
        c = dcoll.connectivity
        g = dcoll.geometry
        self.rx = torch.from_numpy(np.ascontiguousarray(g.rx)).to(device)
        self.rx32 = self.rx.to(torch.float32)
        self.conn = torch.from_numpy(np.ascontiguousarray(c.conn, dtype=np.int32)).to(device)
        self.perm = torch.from_numpy(np.ascontiguousarray(c.perm, dtype=np.uint8)).to(device)
        self.fslot = torch.from_numpy(np.ascontiguousarray(c.fslot, dtype=np.uint8)).to(device)
        nbf = len(c.bface_elem)
        self.nbf = nbf
        self.bface_elem = torch.from_numpy(c.bface_elem).to(device)
        self.bface_nodes = torch.from_numpy(
            dcoll.refel.face_nodes[c.bface_face].astype(np.int64)).to(device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self._bkind_cache = {}
        self._work = {}
        self.mesh = _lib.MeshStruct()
        self.mesh.dim = dcoll.dim
        self.mesh.order = dcoll.order
        self.mesh.nelem = dcoll.nelements
        self.mesh.nbf = nbf
        self.mesh.nperm = len(c.perm)
        self.mesh.rx = self.rx.data_ptr()
        self.mesh.conn = self.conn.data_ptr()
        self.mesh.perm = self.perm.data_ptr()
        self.mesh.bkind = None
        self.mesh.rx32 = self.rx32.data_ptr()
        self.mesh.fslot = self.fslot.data_ptr()
        # a partition's ghost elements follow its owned ones
        self.mesh.nowned = int(getattr(dcoll, "nowned", 0))
        self.mesh.elem_kind = 1 if dcoll.refel.kind == "hypercube" else 0

    def workspace(self, name, shape, dtype=torch.float64):
        t = self._work.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=self.device)
            self._work[name] = t
        return t

    def bkind_for(self, boundaries):
        """int8 [nbf] boundary kinds for this *boundaries* dict."""
        key = tuple(sorted((str(tag), type(b).__name__) for tag, b in boundaries.items()))
        if key not in self._bkind_cache:
            kinds = np.zeros(max(self.nbf, 1), dtype=np.int8)
            covered = np.zeros(self.nbf, dtype=bool)
            for tag, bdry in boundaries.items():
                mask = self.dcoll.boundary_face_mask(tag)
                kinds[:self.nbf][mask] = bdry.device_kind
                covered |= mask
            if self.nbf and not covered.all():
                raise ValueError("some boundary faces have no boundary condition")
            self._bkind_cache[key] = torch.from_numpy(kinds).to(self.device)
        return self._bkind_cache[key]


def device_discretization(dcoll, device) -> DeviceDiscretization:
    cache = dcoll.__dict__.setdefault("_device_cache", {})
    key = _dev_index(device)
    if key not in cache:
        cache[key] = DeviceDiscretization(dcoll, device)
    ensure_reference_operators(dcoll, device)
    return cache[key]


def _gas_struct(gas_model, nspecies, device):
    if gas_model.eos.is_mixture:
        ensure_mechanism(gas_model.eos, device)
    return gas_model.to_struct(nspecies)


# float32 iteration cap per start value; relative temperature-update
# tolerance of the accepted result (the convergence check of the reference
# drivers, mirgecom examples/autoignition.py:526-530)
MIXED_NEWTON_MAXIT = 12
MIXED_NEWTON_RTOL = 1e-8


def mixture_temperature_mixed(cv, gas_model, tseed, tguess=None, iters=None, status=None,
                              learned=None):
    """Mixed-form temperature: float32 Newton from the learned guess (*learned*,
    a TemperatureMLP evaluated in the same kernel, or a precomputed *tguess*)
    else from *tseed*, float64 residual check, plain-guess fallback.  Returns
    T (float32)."""
    q = cv.q
    _lib.require_cuda(q)
    lib = _lib.load()
    gs = _gas_struct(gas_model, cv.nspecies, q.device)
    n = q[0].numel()
    tout = torch.empty_like(q[0])
    tseed = tseed.to(dtype=torch.float32).contiguous()
    if tguess is not None:
        tguess = tguess.to(dtype=torch.float32).contiguous()
    if status is None:
        status = state_status_word(q.device)
    with torch.cuda.device(q.device):
        if learned is not None:
            ms = learned.struct()
            _lib.check(lib.mgc_mixture_temperature_learned_f32(
                cv.dim, C.byref(gs), n, _lib.ptr(q), _lib.ptr(tseed), C.byref(ms),
                _lib.ptr(tout), _lib.ptr(iters), MIXED_NEWTON_MAXIT, MIXED_NEWTON_RTOL,
                _lib.ptr(status), _lib.stream_handle()), "mgc_mixture_temperature_learned_f32")
        else:
            _lib.check(lib.mgc_mixture_temperature_f32(
                cv.dim, C.byref(gs), n, _lib.ptr(q), _lib.ptr(tseed), _lib.ptr(tguess),
                _lib.ptr(tout), _lib.ptr(iters), MIXED_NEWTON_MAXIT, MIXED_NEWTON_RTOL,
                _lib.ptr(status), _lib.stream_handle()), "mgc_mixture_temperature_f32")
    return tout


def mixture_temperature(cv, gas_model, tseed, status=None):
    """Launch the Newton temperature kernel: returns (T1, T2).  Unconverged
    nodes set ST_NEWTON_MISS in *status* (default: the device's state word)."""
    q = cv.q
    _lib.require_cuda(q)
    lib = _lib.load()
    gs = _gas_struct(gas_model, cv.nspecies, q.device)
    n = q[0].numel()
    t1 = torch.empty_like(q[0])
    t2 = torch.empty_like(q[0])
    tseed = tseed.to(dtype=q.dtype).contiguous()
    if status is None:
        status = state_status_word(q.device)
    with torch.cuda.device(q.device):
        _lib.check(lib.mgc_mixture_temperature(
            cv.dim, C.byref(gs), n, _lib.ptr(q), _lib.ptr(tseed), _lib.ptr(t1),
            _lib.ptr(t2), _lib.ptr(status), _lib.stream_handle()), "mgc_mixture_temperature")
    return t1, t2


def boundary_exterior(dd, state, gas_model, boundaries, time):
    """[Nc+1, nbf, Nfp] exterior-state array of the boundary faces: the
    exterior states of the prescribed boundaries, the parameters of the
    Mengaldo ones (wall temperature, free stream, boundary pressure); None
    when no boundary needs one."""
    from mirgecom_b200.boundary import MengaldoBoundaryCondition, PrescribedFluidBoundary

    def wants(b):
        return (isinstance(b, PrescribedFluidBoundary) and b.device_kind == 1) or (
            isinstance(b, MengaldoBoundaryCondition) and type(b).exterior_parameters
            is not MengaldoBoundaryCondition.exterior_parameters)
    if not any(wants(b) for b in boundaries.values()):
        return None
    dcoll = dd.dcoll
    q = state.cv.q
    nc = q.shape[0]
    nfp = dcoll.nface_nodes
    bext = dd.workspace("bext", (nc + 1, dd.nbf, nfp), q.dtype)
    be = dd.bface_elem[:, None]
    qm = q[:, be, dd.bface_nodes]                          # [Nc, nbf, Nfp]
    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import FluidState
    tm = None
    if state.is_mixture:
        tm = state.temperature[be, dd.bface_nodes]
    for tag, bdry in boundaries.items():
        if not wants(bdry):
            continue
        mask = torch.from_numpy(dcoll.boundary_face_mask(tag)).to(q.device)
        sm = FluidState(ConservedVars(qm[:, mask], state.dim), gas_model,
                        temperature=None if tm is None else tm[mask])
        if isinstance(bdry, MengaldoBoundaryCondition):
            bext[:, mask] = bdry.exterior_parameters(dcoll, gas_model, sm, nc).to(q.dtype)
            continue
        nrm = torch.from_numpy(np.ascontiguousarray(
            dcoll.boundary_normals_numpy()[dcoll.boundary_face_mask(tag)].T)).to(q.device)
        ext = bdry.exterior_state(dcoll, tag, gas_model, sm, time,
                                  nodes=dcoll.boundary_nodes(tag, q.device),
                                  normals=nrm[:, :, None])
        bext[:nc, mask] = ext.cv.q.to(q.dtype)
        if state.is_mixture:
            bext[nc, mask] = ext.temperature.to(q.dtype)
    return bext


def _operator_temperature(state):
    if not state.is_mixture:
        return None
    if state.cv.q.dtype == torch.float32:
        # the mixed form carries one temperature for the state and its operator
        return state.temperature.contiguous()
    if state.operator_temperature is None:
        # the operator states re-solve from the state temperature
        _, t2 = mixture_temperature(state.cv, state.gas_model, state.temperature)
        state.operator_temperature = t2
    return state.operator_temperature.contiguous()


# Which device path evaluates the right-hand side of simplicial meshes:
#   "volume_face"  two kernels: volume (gradients kept on chip, pointwise
#                  fluxes, face-node records, volume divergence) and face
#                  (numerical fluxes from the records, lift) -- mgc_operator*
#   "gradient_volume_face"  three kernels through mgc_operator* (phases bit
#                  2): gradients into HBM, flux-volume (pointwise fluxes,
#                  records, volume divergence), face
#   "split"        three kernels: gradients, per-node flux records, surface
#                  and lift -- mgc_ns_grad* + mgc_rhs_split*
#   "fused"        two kernels: gradients, fused divergence -- mgc_ns_grad* +
#                  mgc_ns_rhs* (mgc_euler_rhs* for the Euler operator)
#   "auto"         "gradient_volume_face" for mixtures, Mengaldo boundaries and
#                  kernel phases (partitions); "split" otherwise (the ideal gas
#                  without walls: 0.55 ms against 0.585 ms for the 24^3 p3
#                  Taylor-Green right-hand side)
# Tensor-product hexahedra always take "split".
RHS_PATH = "auto"


def _path(dcoll, gas_model=None, boundaries=None, phased=False):
    if dcoll.refel.kind == "hypercube":
        return "split"
    if RHS_PATH != "auto":
        return RHS_PATH
    from mirgecom_b200.boundary import MengaldoBoundaryCondition
    walls = any(isinstance(b, MengaldoBoundaryCondition) for b in (boundaries or {}).values())
    mixture = gas_model is not None and gas_model.eos.is_mixture
    partitioned = getattr(dcoll, "nowned", None) is not None
    if phased or walls or mixture or partitioned:
        return "gradient_volume_face"
    return "split"


def _operator_path(path):
    return path in ("volume_face", "gradient_volume_face")


def _split_workspace(dd, gs, f32):
    lib = _lib.load()
    nbytes = lib.mgc_rhs_split_workspace_bytes(C.byref(dd.mesh), C.byref(gs), int(f32))
    if nbytes == 0:
        raise RuntimeError("split right-hand side unsupported for this configuration")
    return dd.workspace("split_ws", ((nbytes + 15) // 16 * 16,), torch.uint8)


def _operator_workspace(dd, gs, f32):
    lib = _lib.load()
    nbytes = lib.mgc_operator_workspace_bytes(C.byref(dd.mesh), C.byref(gs), int(f32))
    if nbytes == 0:
        raise RuntimeError("volume/face right-hand side unsupported for this configuration")
    # torch allocations are 256-byte aligned, as the entry point requires
    return dd.workspace("operator_ws", ((nbytes + 255) // 256 * 256,), torch.uint8)


def face_records(dd, gs, f32, nc):
    """The face-node records [E, Nf, Nfp, TW] in the operator workspace (the
    first part of its layout), as a tensor view for the halo exchange."""
    ws = _operator_workspace(dd, gs, f32)
    dtype = torch.float32 if f32 else torch.float64
    dc = dd.dcoll
    tw = -(-(nc + 4) // 4) * 4
    n = dc.nelements * dc.nfaces * dc.nface_nodes * tw
    return ws[:n * (4 if f32 else 8)].view(dtype).view(dc.nelements, dc.nfaces,
                                                        dc.nface_nodes, tw)


def _run_operator(viscous, dd, gs, q, t_op, t_src, bext, flux_kind, add_src, rhs, grad_out,
                  events=None, phases=3):
    """mgc_operator*: volume kernel then face kernel (*phases* 1: volume only,
    2: face only, 3: both).  *events* (3 CUDA events): recorded before the
    volume kernel, between the two kernels and after the face kernel."""
    lib = _lib.load()
    f32 = q.dtype == torch.float32
    ws = _operator_workspace(dd, gs, f32)
    fn = lib.mgc_operator_f32 if f32 else lib.mgc_operator
    mid = None
    if events:
        events[0].record()
        # the event exists once recorded; the library records it again
        # between its two kernels
        events[1].record()
        mid = events[1].cuda_event
    _lib.check(fn(int(viscous), C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t_op),
                  _lib.ptr(t_src), _lib.ptr(bext), flux_kind, int(add_src), _lib.ptr(rhs),
                  _lib.ptr(grad_out), _lib.ptr(ws), ws.numel(), _lib.ptr(dd.status),
                  _lib.stream_handle(), mid, int(phases)), "mgc_operator")
    if events:
        events[2].record()


def euler_rhs(dcoll, state, gas_model, boundaries, time, flux_kind):
    q = state.cv.q
    _lib.require_cuda(q)
    q = q.contiguous()
    lib = _lib.load()
    dd = device_discretization(dcoll, q.device)
    gs = _gas_struct(gas_model, state.cv.nspecies, q.device)
    path = _path(dcoll, gas_model, boundaries)
    if not _operator_path(path):
        # the inviscid slip wall needs only its state_plus: prescribe it
        from mirgecom_b200.boundary import AdiabaticSlipBoundary, _SlipStatePlus
        boundaries = {t: (_SlipStatePlus() if isinstance(b, AdiabaticSlipBoundary) else b)
                      for t, b in boundaries.items()}
    _check_boundary_path(dcoll, boundaries, path)
    bkind = dd.bkind_for(boundaries)
    dd.mesh.bkind = bkind.data_ptr()
    bext = boundary_exterior(dd, state, gas_model, boundaries, time)
    t_op = _operator_temperature(state)
    rhs = torch.empty_like(q)
    f32 = q.dtype == torch.float32
    with torch.cuda.device(q.device):
        if _operator_path(path):
            _run_operator(False, dd, gs, q, t_op, None, bext, flux_kind, False, rhs, None,
                          phases=3 | (4 if path == "gradient_volume_face" else 0))
        elif path == "split":
            ws = _split_workspace(dd, gs, f32)
            fsplit = lib.mgc_rhs_split_f32 if f32 else lib.mgc_rhs_split
            _lib.check(fsplit(0, C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t_op),
                              None, None, _lib.ptr(bext), flux_kind, 0, _lib.ptr(rhs),
                              _lib.ptr(ws), ws.numel(), _lib.ptr(dd.status),
                              _lib.stream_handle(), None), "mgc_rhs_split")
        else:
            fn = lib.mgc_euler_rhs_f32 if f32 else lib.mgc_euler_rhs
            _lib.check(fn(
                C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t_op), _lib.ptr(bext),
                flux_kind, _lib.ptr(rhs), _lib.ptr(dd.status), _lib.stream_handle()),
                "mgc_euler_rhs")
    return rhs


def set_gradient_kernel(kind):
    """Select the gradient-pass kernel process-wide: "auto" (the tcgen05
    pipelined kernel where it applies, else mma.sync) or "mma_sync"."""
    code = {"auto": 0, "mma_sync": 1}[kind]
    _lib.check(_lib.load().mgc_set_gradient_kernel(code), "mgc_set_gradient_kernel")


def gradient_kernel():
    return {0: "auto", 1: "mma_sync"}[_lib.load().mgc_get_gradient_kernel()]


def _check_boundary_path(dcoll, boundaries, path):
    """The Mengaldo boundaries are evaluated by the volume/face path only."""
    from mirgecom_b200.boundary import MengaldoBoundaryCondition
    bad = [t for t, b in boundaries.items() if isinstance(b, MengaldoBoundaryCondition)]
    if bad and not _operator_path(path):
        raise NotImplementedError(
            f"boundaries {bad}: the Mengaldo treatment runs on the volume/face path of "
            "simplicial meshes only")


def ns_rhs(dcoll, state, gas_model, boundaries, time, flux_kind, *,
           source_temperature=None, want_gradients=False, events=None, halo=None,
           phases=3, rhs=None):
    """The Navier-Stokes right-hand side; returns (rhs, gradients or None).
    Gradients [Nc+1, dim, E, Np] are returned when *want_gradients* (they are
    only written to HBM then, on the volume/face path).  *events*: on the
    volume/face path 3 CUDA events (before the volume kernel, between the
    two kernels, after the face kernel); on the gradient/volume/face path 4
    (before the gradient kernel, before the flux-volume kernel, before the
    face kernel, after it); on the other paths 3 or 4 (before the gradient
    pass, between the passes, [between the node-flux and surface kernels,]
    after the divergence).

    Mesh partitions (*dcoll* a :class:`~mirgecom_b200.partition.
    PartitionedDiscretization`, the state's ghost rows already exchanged):
    with *halo* (a :class:`~mirgecom_b200.partition.HaloExchange`) the face
    records of the ghosts are exchanged between the two kernels; or the
    caller runs the kernels one at a time (*phases* 1 then 2, passing the
    first call's *rhs* to the second) and exchanges the records of
    :func:`face_records` in between."""
    path = _path(dcoll, gas_model, boundaries, phased=(phases != 3 or halo is not None))
    _check_boundary_path(dcoll, boundaries, path)
    q = state.cv.q
    _lib.require_cuda(q)
    q = q.contiguous()
    lib = _lib.load()
    dd = device_discretization(dcoll, q.device)
    nc = q.shape[0]
    gs = _gas_struct(gas_model, state.cv.nspecies, q.device)
    bkind = dd.bkind_for(boundaries)
    dd.mesh.bkind = bkind.data_ptr()
    bext = boundary_exterior(dd, state, gas_model, boundaries, time)
    t_op = _operator_temperature(state)
    if source_temperature is not None:
        source_temperature = source_temperature.to(q.dtype)
    rhs = torch.empty_like(q) if rhs is None else rhs
    stream = _lib.stream_handle()
    add_src = source_temperature is not None
    t_src = source_temperature.contiguous() if add_src else None
    f32 = q.dtype == torch.float32
    gshape = (nc + 1, dcoll.dim) + tuple(q.shape[1:])
    if _operator_path(path):
        three = path == "gradient_volume_face"
        if three:
            grad = dd.workspace("grad", gshape, q.dtype)
        else:
            grad = torch.empty(gshape, dtype=q.dtype, device=q.device) if want_gradients else None
        # three kernels: the gradient entry point (its own launch, timed by
        # events[0..1]), then the operator with the gradients given (bit 8)
        extra = 4 | 8 if three else 0
        ops_events = events[1:] if (events and three) else events
        with torch.cuda.device(q.device):
            if three and (phases & 1):
                if events:
                    events[0].record()
                fgrad = lib.mgc_ns_grad_f32 if f32 else lib.mgc_ns_grad
                _lib.check(fgrad(
                    C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t_op), _lib.ptr(bext),
                    _lib.ptr(grad), _lib.ptr(dd.status), stream), "mgc_ns_grad")
            if halo is None:
                _run_operator(True, dd, gs, q, t_op, t_src, bext, flux_kind, add_src, rhs, grad,
                              events=ops_events, phases=phases | (extra if phases & 1 else 0))
            else:
                _run_operator(True, dd, gs, q, t_op, t_src, bext, flux_kind, add_src, rhs, grad,
                              phases=1 | extra)
                halo.exchange_records(face_records(dd, gs, f32, nc))
                _run_operator(True, dd, gs, q, t_op, t_src, bext, flux_kind, add_src, rhs, None,
                              phases=2)
        if three and want_gradients:
            grad = grad.clone()
        return rhs, (grad if want_gradients else None)
    grad = dd.workspace("grad", gshape, q.dtype)
    fgrad = lib.mgc_ns_grad_f32 if f32 else lib.mgc_ns_grad
    frhs = lib.mgc_ns_rhs_f32 if f32 else lib.mgc_ns_rhs
    with torch.cuda.device(q.device):
        if events:
            events[0].record()
        _lib.check(fgrad(
            C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t_op), _lib.ptr(bext),
            _lib.ptr(grad), _lib.ptr(dd.status), stream), "mgc_ns_grad")
        if events:
            events[1].record()
        if path == "split":
            ws = _split_workspace(dd, gs, f32)
            fsplit = lib.mgc_rhs_split_f32 if f32 else lib.mgc_rhs_split
            mid = None
            if events and len(events) == 4:
                events[2].record()
                mid = events[2].cuda_event
            _lib.check(fsplit(1, C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t_op),
                              _lib.ptr(t_src), _lib.ptr(grad), _lib.ptr(bext), flux_kind,
                              int(add_src), _lib.ptr(rhs), _lib.ptr(ws), ws.numel(),
                              _lib.ptr(dd.status), stream, mid), "mgc_rhs_split")
        else:
            _lib.check(frhs(
                C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t_op), _lib.ptr(t_src),
                _lib.ptr(grad), _lib.ptr(bext), flux_kind, int(add_src), _lib.ptr(rhs),
                _lib.ptr(dd.status), stream), "mgc_ns_rhs")
        if events:
            events[-1].record()
    return rhs, (grad.clone() if want_gradients else None)


def read_status(dcoll, device=None, reset=True):
    """Device status bits accumulated by the kernels of *dcoll* and by the
    device's temperature kernels (synchronises)."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    dd = device_discretization(dcoll, device)
    sw = state_status_word(device)
    val = int(dd.status.item()) | int(sw.item())
    if reset:
        dd.status.zero_()
        sw.zero_()
    return val


def rk4_stage(q0, k, acc, qout, stage, dt, qout_lo=None):
    lib = _lib.load()
    n = q0.numel()
    if k.dtype == torch.float32:
        _lib.check(lib.mgc_rk4_stage_mixed(
            n, _lib.ptr(q0), _lib.ptr(k), _lib.ptr(acc), _lib.ptr(qout), _lib.ptr(qout_lo),
            stage, float(dt), _lib.stream_handle()), "mgc_rk4_stage_mixed")
        return
    _lib.check(lib.mgc_rk4_stage(n, _lib.ptr(q0), _lib.ptr(k), _lib.ptr(acc), _lib.ptr(qout),
                                 _lib.ptr(qout_lo), stage, float(dt), _lib.stream_handle()),
               "mgc_rk4_stage")


def ns_gradients(dcoll, state, gas_model, boundaries, time):
    """The BR1 gradients [Nc+1, dim, E, Np] (a workspace tensor) from the
    gradient kernel mgc_ns_grad* (its Mengaldo boundary states on simplices
    included)."""
    _check_boundary_path(dcoll, boundaries, _path(dcoll, gas_model, boundaries))
    q = state.cv.q
    _lib.require_cuda(q)
    q = q.contiguous()
    lib = _lib.load()
    dd = device_discretization(dcoll, q.device)
    nc = q.shape[0]
    gs = _gas_struct(gas_model, state.cv.nspecies, q.device)
    bkind = dd.bkind_for(boundaries)
    dd.mesh.bkind = bkind.data_ptr()
    bext = boundary_exterior(dd, state, gas_model, boundaries, time)
    t_op = _operator_temperature(state)
    grad = dd.workspace("grad", (nc + 1, dcoll.dim) + tuple(q.shape[1:]), q.dtype)
    fgrad = lib.mgc_ns_grad_f32 if q.dtype == torch.float32 else lib.mgc_ns_grad
    with torch.cuda.device(q.device):
        _lib.check(fgrad(
            C.byref(dd.mesh), C.byref(gs), _lib.ptr(q), _lib.ptr(t_op), _lib.ptr(bext),
            _lib.ptr(grad), _lib.ptr(dd.status), _lib.stream_handle()), "mgc_ns_grad")
    return grad
