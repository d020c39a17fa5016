"""Element partitions of a discretization and their halo exchange.

The reference distributes a mesh over MPI ranks (meshmode's partitioning,
mirgecom/simutil.py:1050-1130 ``distribute_mesh``) and exchanges, per
Navier-Stokes right-hand side, the conserved variables and temperature on
the partition faces and then their gradients (mirgecom/gas_model.py:813-880,
mirgecom/navierstokes.py:503-531).  Here a rank owns a contiguous block of
the element order (the Morton order of the box meshes keeps blocks compact)
and holds, after its owned elements, the *ghost* elements across its
partition faces.  One right-hand side exchanges twice:

1. before the volume kernel, the ghosts' conserved variables and
   temperatures (whole element rows: the gradient pass reads the neighbour
   values at its face nodes);
2. between the volume and the face kernel, the ghosts' face-node records on
   the shared faces (F.n, |v| + c, p, c, gamma: everything the face kernel
   takes from a neighbour), so no gradients cross the partition.

:class:`PartitionedDiscretization` is one rank's view (owned elements first,
then ghosts, with the face pairing renumbered into that order) and carries
the send / receive lists of both exchanges; :class:`HaloExchange` moves the
data through ``torch.distributed`` point-to-point operations (NCCL on GPUs,
grouped; gloo on the host), or within one process for emulated ranks.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from mirgecom_b200.discretization import BTAG_ALL


def partition_elements(nelem, nparts):
    """Owner rank of every element: contiguous blocks of the element order."""
    if nparts < 1 or nparts > nelem:
        raise ValueError("need 1 <= nparts <= number of elements")
    bounds = np.linspace(0, nelem, nparts + 1).round().astype(np.int64)
    owner = np.empty(nelem, dtype=np.int64)
    for p in range(nparts):
        owner[bounds[p]:bounds[p + 1]] = p
    return owner


@dataclass
class _Plan:
    """Per peer: what this rank sends and where what it receives goes."""
    send_elems: dict       # peer -> local owned element indices (q rows)
    recv_elems: dict       # peer -> local ghost element indices
    send_faces: dict       # peer -> (local owned element, face) pairs (records)
    recv_faces: dict       # peer -> (local ghost element, face) pairs


class _LocalConnectivity:
    def __init__(self, conn, perm, fslot, bface_elem, bface_face, bface_side):
        self.conn = conn
        self.perm = perm
        self.fslot = fslot
        self.bface_elem = bface_elem
        self.bface_face = bface_face
        self.bface_side = bface_side


class _LocalGeometry:
    def __init__(self, g, elems):
        self.rx = g.rx[elems]
        self.jac = g.jac[elems]
        self.det = g.det[elems]
        self.nodes = g.nodes[:, elems]
        self.normals = g.normals[elems]
        self.fscale = g.fscale[elems]


class PartitionedDiscretization:
    """Rank *rank*'s part of *dcoll* under the owner map *owner* (default:
    :func:`partition_elements`).  Element order: the owned elements (in
    global order), then the ghosts (global order).  Quacks like the
    :class:`~mirgecom_b200.discretization.Discretization` for the runtime;
    ``nowned`` tells the kernels where the ghosts start."""

    def __init__(self, dcoll, rank, nparts, owner=None, device=None):
        if dcoll.refel.kind != "simplex":
            raise NotImplementedError("partitions run on the simplex volume/face path")
        self.global_dcoll = dcoll
        self.rank = rank
        self.nparts = nparts
        self.owner = partition_elements(dcoll.nelements, nparts) if owner is None else owner
        c = dcoll.connectivity
        nf = dcoll.nfaces
        owned = np.nonzero(self.owner == rank)[0]
        conn = c.conn[owned].astype(np.int64)
        nbr = np.where(conn >= 0, conn >> 8, -1)
        cand = np.unique(nbr[nbr >= 0])
        ghosts = cand[self.owner[cand] != rank]
        self.owned = owned
        self.ghosts = ghosts
        self.nowned = len(owned)
        elems = np.concatenate([owned, ghosts])
        self.elements = elems
        loc = np.full(dcoll.nelements, -1, dtype=np.int64)
        loc[elems] = np.arange(len(elems))
        self.local_index = loc
        # face pairing renumbered; the ghosts' own rows are never read
        lconn = np.zeros((len(elems), nf), dtype=np.int64)
        inter = conn >= 0
        lconn[:self.nowned][inter] = loc[nbr[inter]] * 256 + (conn[inter] & 255)
        # boundary faces of the owned elements, renumbered
        gbf = -(conn[~inter] + 1)
        keep = np.nonzero(np.isin(c.bface_elem, owned))[0]
        bloc = np.full(len(c.bface_elem), -1, dtype=np.int64)
        bloc[keep] = np.arange(len(keep))
        lconn[:self.nowned][~inter] = -(1 + bloc[gbf])
        if len(elems) * 256 >= 2 ** 31:
            raise ValueError("partition too large for the packed face pairing")
        self.connectivity = _LocalConnectivity(
            conn=lconn.astype(np.int32), perm=c.perm, fslot=c.fslot,
            bface_elem=loc[c.bface_elem[keep]], bface_face=c.bface_face[keep],
            bface_side=c.bface_side[keep])
        self.geometry = _LocalGeometry(dcoll.geometry, elems)
        self.refel = dcoll.refel
        self.dim = dcoll.dim
        self.order = dcoll.order
        self.mesh = dcoll.mesh
        self.nelements = len(elems)
        self._device = device
        self.plan = self._build_plan()

    # the Discretization surface the runtime uses
    @property
    def kind(self):
        return self.refel.kind

    @property
    def nfaces(self):
        return self.refel.nfaces

    @property
    def nface_nodes(self):
        return self.refel.nface_nodes

    @property
    def device(self):
        import torch
        if self._device is None:
            self._device = torch.device("cuda", torch.cuda.current_device())
        return self._device

    def boundary_face_mask(self, tag):
        side = self.connectivity.bface_side
        if tag == BTAG_ALL or tag is None:
            return np.ones(len(side), dtype=bool)
        if isinstance(tag, str) and tag[0] in "-+" and tag[1:].isdigit():
            axis = int(tag[1:])
            return side == 2 * axis + (1 if tag[0] == "+" else 0)
        raise ValueError(f"unknown boundary tag {tag!r}")

    def boundary_normals_numpy(self):
        c = self.connectivity
        return self.geometry.normals[c.bface_elem, c.bface_face]

    def boundary_nodes_numpy(self):
        c = self.connectivity
        fn = self.refel.face_nodes[c.bface_face]
        return self.geometry.nodes[:, c.bface_elem[:, None], fn]

    def boundary_nodes(self, tag=BTAG_ALL, device=None):
        import torch
        x = self.boundary_nodes_numpy()[:, self.boundary_face_mask(tag)]
        return torch.from_numpy(np.ascontiguousarray(x)).to(device or self.device)

    def nodes(self, device=None):
        import torch
        x = torch.from_numpy(np.ascontiguousarray(self.geometry.nodes)).to(
            device or self.device)
        return [x[i] for i in range(self.dim)]

    def _faces_needed(self, rank):
        """(global element, face) of every record rank *rank* reads from a
        ghost: the neighbour element and its face across each partition face
        of an element *rank* owns, sorted."""
        c = self.global_dcoll.connectivity
        nfp = self.global_dcoll.nface_nodes
        owned = np.nonzero(self.owner == rank)[0]
        conn = c.conn[owned].astype(np.int64)
        inter = conn >= 0
        nbr = np.where(inter, conn >> 8, -1)
        remote = inter & (self.owner[np.maximum(nbr, 0)] != rank)
        e_, f_ = np.nonzero(remote)
        en = nbr[e_, f_]
        fo = c.fslot[conn[e_, f_] & 255, 0].astype(np.int64) // nfp
        pairs = np.unique(np.stack([en, fo], axis=1), axis=0)
        return pairs

    def _build_plan(self):
        me = self.rank
        send_elems, recv_elems, send_faces, recv_faces = {}, {}, {}, {}
        g_owner = self.owner
        for peer in range(self.nparts):
            if peer == me:
                continue
            # q rows: the peer's ghosts owned by me (the peer sorts its ghosts
            # by global index, as I do)
            peer_pd_ghosts = self._ghosts_of(peer)
            mine = peer_pd_ghosts[g_owner[peer_pd_ghosts] == me]
            if len(mine):
                send_elems[peer] = self.local_index[mine]
            theirs = self.ghosts[g_owner[self.ghosts] == peer]
            if len(theirs):
                recv_elems[peer] = self.local_index[theirs]
            # records: faces of my elements the peer reads, and faces of the
            # peer's elements I read
            need_peer = self._faces_needed(peer)
            sel = g_owner[need_peer[:, 0]] == me if len(need_peer) else np.zeros(0, bool)
            if np.any(sel):
                pairs = need_peer[sel]
                send_faces[peer] = np.stack([self.local_index[pairs[:, 0]], pairs[:, 1]],
                                            axis=1)
            need_me = self._faces_needed(me)
            sel = g_owner[need_me[:, 0]] == peer if len(need_me) else np.zeros(0, bool)
            if np.any(sel):
                pairs = need_me[sel]
                recv_faces[peer] = np.stack([self.local_index[pairs[:, 0]], pairs[:, 1]],
                                            axis=1)
        return _Plan(send_elems, recv_elems, send_faces, recv_faces)

    def _ghosts_of(self, rank):
        c = self.global_dcoll.connectivity
        owned = np.nonzero(self.owner == rank)[0]
        conn = c.conn[owned].astype(np.int64)
        nbr = np.where(conn >= 0, conn >> 8, -1)
        cand = np.unique(nbr[nbr >= 0])
        return cand[self.owner[cand] != rank]

    def scatter(self, global_array):
        """The local rows (owned, then ghosts) of a global [..., E, Np] array."""
        return global_array[..., self.elements, :]


class HaloExchange:
    """The two exchanges of one partitioned right-hand side, each split into
    ``begin_*`` (pack and post) and ``end_*`` (wait and unpack), so that
    emulated ranks of one process can all post before any unpacks, and so
    that a driver can overlap work with an exchange in flight.

    *transport*: ``"dist"`` for ``torch.distributed`` point-to-point
    operations between the ranks of the default process group (every rank
    makes the same calls in the same order; each ``begin`` posts its sends
    and receives as one group), or a :class:`LocalTransport` shared by the
    emulated ranks of one process."""

    def __init__(self, pdcoll, transport="dist"):
        self.pd = pdcoll
        self.transport = transport

    def begin_rows(self, arrays):
        """Post the ghost rows of each [..., E_local, Np] tensor in *arrays*
        (conserved variables, temperature seeds)."""
        plan = self.pd.plan
        sends = {p: [a[..., _t(i, a), :].contiguous() for a in arrays]
                 for p, i in plan.send_elems.items()}
        recvs = {p: [_empty_rows(a, len(i)) for a in arrays]
                 for p, i in plan.recv_elems.items()}
        return ("rows", arrays, recvs, self._post(sends, recvs))

    def begin_records(self, trace):
        """Post the face-node records [E_local, Nf, Nfp, TW] of the faces the
        peers read from this rank's elements."""
        plan = self.pd.plan
        sends = {p: [trace[_t(pr[:, 0], trace), _t(pr[:, 1], trace)].contiguous()]
                 for p, pr in plan.send_faces.items()}
        recvs = {p: [trace.new_empty((len(pr),) + tuple(trace.shape[2:]))]
                 for p, pr in plan.recv_faces.items()}
        return ("records", trace, recvs, self._post(sends, recvs))

    def end(self, handle):
        what, target, recvs, reqs = handle
        for req in reqs:
            req.wait()
        plan = self.pd.plan
        if what == "rows":
            for p, idx in plan.recv_elems.items():
                for a, buf in zip(target, recvs[p]):
                    a[..., _t(idx, a), :] = buf
        else:
            for p, pr in plan.recv_faces.items():
                target[_t(pr[:, 0], target), _t(pr[:, 1], target)] = recvs[p][0]

    def exchange_rows(self, arrays):
        self.end(self.begin_rows(arrays))

    def exchange_records(self, trace):
        self.end(self.begin_records(trace))

    def _post(self, sends, recvs):
        if isinstance(self.transport, LocalTransport):
            self.transport.post(self.pd.rank, sends, recvs)
            return []
        import torch.distributed as dist
        ops = []
        for p in sorted(set(sends) | set(recvs)):
            for buf in sends.get(p, []):
                ops.append(dist.P2POp(dist.isend, buf, p))
            for buf in recvs.get(p, []):
                ops.append(dist.P2POp(dist.irecv, buf, p))
        return dist.batch_isend_irecv(ops) if ops else []


class LocalTransport:
    """Emulated ranks of one process: rank r's sends are matched with the
    receiving rank's buffers once every rank has posted (:meth:`complete`).
    Data moves by device copies; no kernel waits on another."""

    def __init__(self, nparts):
        self.nparts = nparts
        self._posted = {}

    def post(self, rank, sends, recvs):
        self._posted[rank] = (sends, recvs)
        if len(self._posted) == self.nparts:
            self.complete()

    def complete(self):
        for r, (sends, _) in self._posted.items():
            for p, bufs in sends.items():
                dst = self._posted[p][1][r]
                for d, s in zip(dst, bufs):
                    d.copy_(s)
        self._posted = {}


def _t(idx, like):
    import torch
    return torch.as_tensor(np.asarray(idx), dtype=torch.int64, device=like.device)


def _empty_rows(a, n):
    shape = list(a.shape)
    shape[-2] = n
    return a.new_empty(shape)
