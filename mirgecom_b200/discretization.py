"""Host-side flattening of the DG discretization into device index arrays.

This replaces what ``create_discretization_collection``
(mirgecom/discretization.py:41-83) obtains from grudge/meshmode: nodes,
geometric factors, face normals and the interior/boundary face pairings that
``interior_trace_pairs`` and ``op.project`` use (mirgecom/gas_model.py:813-834).
Everything is computed once on the host in float64 and uploaded once.

Device layout (all per element, elements in mesh order):

* ``rx``     float64 [E, d, d]  -- dr_r/dx_j of the affine map;
* ``conn``   int32   [E, Nf]    -- face pairing: ``nbr_elem * 256 + perm_id``
  for an interior face, ``-(1 + bface)`` for a boundary face;
* ``perm``   uint8   [nperm, Nfp] -- volume node index, inside the neighbour,
  of the point that coincides with own face node m;
* ``fslot``  uint8   [nperm, Nfp] -- the same point as the neighbour's face
  slot ``fn * Nfp + m'`` (its face fn and face-node index m'), where the
  volume kernel files the neighbour's face-node record;
* reference operators ``W`` [d, Np, Np] and ``LIFT`` [Np, Nf*Nfp].

Normals and face Jacobians are derived from ``rx`` inside the kernels
(Nanson's formula, n dS = J rx^T N dS_ref), which keeps the geometry read to
d*d values per element.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from mirgecom_b200.mesh import BoxMesh, generate_box_mesh
from mirgecom_b200.refelem import ReferenceElement, make_reference_element

BTAG_ALL = "all"


@dataclass
class FaceConnectivity:
    conn: np.ndarray           # int32 [E, Nf]
    perm: np.ndarray           # uint8 [nperm, Nfp]
    fslot: np.ndarray          # uint8 [nperm, Nfp]
    bface_elem: np.ndarray     # int64 [nbf]
    bface_face: np.ndarray     # int64 [nbf]
    bface_side: np.ndarray     # int64 [nbf]: 2*axis + (0 low, 1 high), -1 other
    nbr_node_index: np.ndarray  # int64 [E, Nf, Nfp] global node index, -1 boundary


def _face_vertex_ids(mesh, refel):
    fv = np.array(refel.face_vertices)                 # (Nf, nfv)
    return mesh.vertex_ids[:, fv]                      # (E, Nf, nfv)


def build_face_connectivity(mesh: BoxMesh, refel: ReferenceElement) -> FaceConnectivity:
    nel = mesh.nelements
    nf = refel.nfaces
    nfp = refel.nface_nodes
    fvid = _face_vertex_ids(mesh, refel)               # (E, Nf, nfv)
    nfv = fvid.shape[2]
    keys = np.sort(fvid.reshape(nel * nf, nfv), axis=1)
    order = np.lexsort(keys.T[::-1])
    sk = keys[order]
    same_next = np.all(sk[1:] == sk[:-1], axis=1)
    if np.any(same_next[1:] & same_next[:-1]):
        raise ValueError("a face is shared by more than two elements "
                         "(periodic axis too short?)")
    pair_a = order[:-1][same_next]
    pair_b = order[1:][same_next]
    matched = np.zeros(nel * nf, dtype=bool)
    matched[pair_a] = True
    matched[pair_b] = True

    nbr = np.full(nel * nf, -1, dtype=np.int64)
    nbr[pair_a] = pair_b
    nbr[pair_b] = pair_a
    own = np.nonzero(matched)[0]
    other = nbr[own]
    own_e, own_f = own // nf, own % nf
    oth_e, oth_f = other // nf, other % nf
    gv_own = fvid[own_e, own_f]                        # (n, nfv)
    gv_oth = fvid[oth_e, oth_f]
    pattern = np.argmax(gv_own[:, :, None] == gv_oth[:, None, :], axis=2)
    combo = np.concatenate([own_f[:, None], oth_f[:, None], pattern], axis=1)
    ucombo, cinv = np.unique(combo, axis=0, return_inverse=True)
    cinv = cinv.ravel()

    # node map of each (own face, neighbour face, vertex pattern) combination
    refv = refel.vertices
    rnodes = refel.nodes.T                             # (Np, d)
    combo_rows = np.zeros((len(ucombo), nfp), dtype=np.int64)
    for ci, row in enumerate(ucombo):
        f, fo, pat = int(row[0]), int(row[1]), row[2:]
        w = refel.face_param[f]                        # (Nfp, nfv)
        oth_verts = refv[np.array(refel.face_vertices[fo])[pat]]   # (nfv, d)
        pts = w @ oth_verts                            # points in neighbour frame
        cand = refel.face_nodes[fo]
        dist = np.linalg.norm(pts[:, None, :] - rnodes[cand][None, :, :], axis=2)
        best = np.argmin(dist, axis=1)
        if np.max(dist[np.arange(nfp), best]) > 1e-9:
            raise RuntimeError("face nodes of neighbouring elements do not coincide")
        combo_rows[ci] = cand[best]
    uperm, pinv = np.unique(combo_rows, axis=0, return_inverse=True)
    pinv = pinv.ravel()
    if len(uperm) > 256:
        raise ValueError("too many distinct face-node permutations")
    if nel * 256 >= 2 ** 31:
        raise ValueError("mesh too large for the packed face pairing")

    # each permutation row lists the nodes of one neighbour face: its face
    # slots fn * Nfp + m'
    fslot = np.zeros(uperm.shape, dtype=np.int64)
    fnodes = np.asarray(refel.face_nodes)
    for pi, row in enumerate(uperm):
        hits = [fo for fo in range(nf) if set(fnodes[fo]) == set(row)]
        if len(hits) != 1:
            raise RuntimeError("a face-node permutation matches no single face")
        fo = hits[0]
        pos = {int(k): i for i, k in enumerate(fnodes[fo])}
        fslot[pi] = [fo * nfp + pos[int(k)] for k in row]
    if nf * nfp > 256:
        raise ValueError("too many face nodes for the uint8 face slots")

    conn = np.zeros(nel * nf, dtype=np.int64)
    conn[own] = oth_e * 256 + pinv[cinv]
    nbr_node = np.full((nel * nf, nfp), -1, dtype=np.int64)
    nbr_node[own] = oth_e[:, None] * refel.nnodes + uperm[pinv[cinv]]

    bfaces = np.nonzero(~matched)[0]
    conn[bfaces] = -(1 + np.arange(len(bfaces)))
    be, bf = bfaces // nf, bfaces % nf
    # which box side a boundary face lies on
    side = np.full(len(bfaces), -1, dtype=np.int64)
    if len(bfaces):
        fverts = mesh.vertex_coords[be[:, None], np.array(refel.face_vertices)[bf]]
        for axis in range(mesh.dim):
            for s, val in enumerate([mesh.a[axis], mesh.b[axis]]):
                on = np.all(np.abs(fverts[:, :, axis] - val) < 1e-12, axis=1)
                side[on] = 2 * axis + s
    return FaceConnectivity(
        conn=conn.reshape(nel, nf).astype(np.int32),
        perm=uperm.astype(np.uint8),
        fslot=fslot.astype(np.uint8),
        bface_elem=be, bface_face=bf, bface_side=side,
        nbr_node_index=nbr_node.reshape(nel, nf, nfp))


@dataclass
class Geometry:
    jac: np.ndarray            # (E, d, d) dx_i/dr_r
    det: np.ndarray            # (E,)
    rx: np.ndarray             # (E, d, d) dr_r/dx_j  (index [e, r, j])
    nodes: np.ndarray          # (d, E, Np) physical node coordinates
    normals: np.ndarray        # (E, Nf, d) unit outward normals
    fscale: np.ndarray         # (E, Nf) face measure factor / volume Jacobian


def build_geometry(mesh: BoxMesh, refel: ReferenceElement) -> Geometry:
    vc = mesh.vertex_coords                           # (E, nv, d)
    d = mesh.dim
    if refel.kind == "simplex":
        jac = np.stack([(vc[:, i + 1] - vc[:, 0]) / 2 for i in range(d)], axis=2)
    else:
        # affine (parallelepiped) cells: the corner along each axis
        jac = np.stack([(vc[:, 1 << i] - vc[:, 0]) / 2 for i in range(d)], axis=2)
    det = np.linalg.det(jac)
    if np.any(det <= 0):
        raise ValueError("non-positive element Jacobian")
    rx = np.linalg.inv(jac)
    r1 = refel.nodes + 1.0                            # (d, Np)
    nodes = vc[:, 0, :].T[:, :, None] + np.einsum("eir,rn->ien", jac, r1)
    # n dS = J rx^T N dS_ref
    nvec = np.einsum("erj,fr->efj", rx, refel.ref_face_normals)
    nmag = np.linalg.norm(nvec, axis=2)
    normals = nvec / nmag[:, :, None]
    fscale = nmag * refel.face_scale_ref[None, :]
    return Geometry(jac=jac, det=det, rx=rx, nodes=nodes, normals=normals,
                    fscale=fscale)


class Discretization:
    """The build's stand-in for grudge's ``DiscretizationCollection``.

    Holds the reference element, the flattened connectivity and the geometric
    factors on the host, and uploads the device copies on first use.
    """

    def __init__(self, mesh: BoxMesh, order: int, device=None):
        self.mesh = mesh
        self.order = order
        self.dim = mesh.dim
        self.refel = make_reference_element(mesh.kind, mesh.dim, order)
        self.geometry = build_geometry(mesh, self.refel)
        self.connectivity = build_face_connectivity(mesh, self.refel)
        self.nelements = mesh.nelements
        self.nnodes_per_element = self.refel.nnodes
        self._device = device
        self._dev = {}

    # {{{ grudge-like conveniences

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
    def nbfaces(self):
        return len(self.connectivity.bface_elem)

    def nodes_numpy(self):
        return self.geometry.nodes

    def boundary_nodes_numpy(self):
        """Physical coordinates of boundary face nodes, (d, nbf, Nfp)."""
        c = self.connectivity
        fn = self.refel.face_nodes[c.bface_face]            # (nbf, Nfp)
        return self.geometry.nodes[:, c.bface_elem[:, None], fn]

    def boundary_nodes(self, tag=BTAG_ALL, device=None):
        """Boundary face node coordinates under *tag* as a tensor (d, nbf_tag, Nfp)."""
        import torch
        mask = self.boundary_face_mask(tag)
        x = self.boundary_nodes_numpy()[:, mask]
        return torch.from_numpy(np.ascontiguousarray(x)).to(device or self.device)

    def characteristic_lengthscales(self, device=None, dtype=None):
        """Per-node length scale h = min(dr) r_D for time-step estimates
        (grudge's ``dt_utils.characteristic_lengthscales``, after Hesthaven &
        Warburton 2008, sec. 6.4): min(dr) is the smallest distance between
        two nodes of the reference element (its [-1, 1] coordinates), r_D the
        element's inradius d V / sum_f F_f (for an affine element the
        Jacobian cancels: d V_ref / sum_f |rx^T N_f| F_ref,f).  Shape (E, Np)."""
        import torch
        key = ("char_len", str(device), str(dtype))
        if key not in self._dev:
            nodes = self.refel.nodes
            diff = nodes[:, :, None] - nodes[:, None, :]
            dist = np.sqrt((diff ** 2).sum(axis=0))
            min_dr = dist[np.triu_indices(nodes.shape[1], k=1)].min()
            nvec = np.einsum("erj,fr->efj", self.geometry.rx, self.refel.ref_face_normals)
            areas = np.linalg.norm(nvec, axis=2) * self.refel.ref_face_areas[None, :]
            r_d = self.dim * self.refel.ref_volume / areas.sum(axis=1)
            h = np.repeat((min_dr * r_d)[:, None], self.refel.nnodes, axis=1)
            self._dev[key] = torch.as_tensor(
                h, dtype=dtype or torch.float64,
                device=device if device is not None else self._device)
        return self._dev[key]

    def nodes(self, device=None):
        """Volume node coordinates, a list of d tensors [E, Np] (dcoll.nodes())."""
        import torch
        x = torch.from_numpy(np.ascontiguousarray(self.geometry.nodes)).to(
            device or self.device)
        return [x[i] for i in range(self.dim)]

    def zeros(self, device=None, dtype=None):
        import torch
        return torch.zeros((self.nelements, self.refel.nnodes),
                           dtype=dtype or torch.float64, device=device or self.device)

    def boundary_normals_numpy(self):
        c = self.connectivity
        return self.geometry.normals[c.bface_elem, c.bface_face]   # (nbf, d)

    def boundary_face_mask(self, tag):
        """Boolean mask over boundary faces selected by *tag*."""
        side = self.connectivity.bface_side
        if tag == BTAG_ALL or tag is None:
            return np.ones(len(side), dtype=bool)
        if isinstance(tag, str) and tag[0] in "-+" and tag[1:].isdigit():
            axis = int(tag[1:])
            return side == 2 * axis + (1 if tag[0] == "+" else 0)
        raise ValueError(f"unknown boundary tag {tag!r}")

    # }}}

    # {{{ device copies

    @property
    def device(self):
        import torch
        if self._device is None:
            self._device = torch.device("cuda", torch.cuda.current_device())
        return self._device

    def dev(self, name):
        import torch
        if name not in self._dev:
            r = self.refel
            c = self.connectivity
            g = self.geometry
            host = {
                "rx": np.ascontiguousarray(g.rx, dtype=np.float64),
                "rx32": np.ascontiguousarray(g.rx, dtype=np.float32),
                "conn": np.ascontiguousarray(c.conn, dtype=np.int32),
                "perm": np.ascontiguousarray(c.perm, dtype=np.uint8),
                "face_nodes": np.ascontiguousarray(r.face_nodes, dtype=np.int32),
                "weak": np.ascontiguousarray(r.weak, dtype=np.float64),
                "lift": np.ascontiguousarray(r.lift, dtype=np.float64),
                "ref_normals": np.ascontiguousarray(r.ref_face_normals, dtype=np.float64),
                "face_scale_ref": np.ascontiguousarray(r.face_scale_ref, dtype=np.float64),
            }
            arr = host[name]
            self._dev[name] = torch.from_numpy(arr).to(self.device)
        return self._dev[name]

    # }}}


def create_discretization_collection(mesh, order, **kwargs):
    """Counterpart of mirgecom/discretization.py:41: base nodal discretization."""
    return Discretization(mesh, order, **kwargs)


__all__ = ["BTAG_ALL", "Discretization", "create_discretization_collection",
           "generate_box_mesh", "build_face_connectivity", "build_geometry"]
