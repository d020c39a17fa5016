"""Box meshes for the DG discretization (host-side set-up only).

Plays the role of ``meshmode.mesh.generation.generate_regular_rect_mesh`` and
``mirgecom.simutil.get_box_mesh`` (mirgecom/simutil.py:141-200): a regular
grid of boxes, each split into simplices (2 triangles per square, 6 tetrahedra
per cube) or kept as tensor-product quadrilaterals/hexahedra, with optional
periodicity per axis.

Cells are visited in Morton (Z-curve) order so that face neighbours sit close
in element index, which keeps the neighbour-trace gathers of the device
kernels inside L2.  The cube split is the Kuhn (Freudenthal) triangulation:
the 6 tetrahedra share the cube's main diagonal, which is conforming across
cubes and across periodic boundaries.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np


@dataclass
class BoxMesh:
    dim: int
    kind: str                    # "simplex" or "hypercube"
    vertex_coords: np.ndarray    # (E, nverts_per_elem, dim) unwrapped coordinates
    vertex_ids: np.ndarray       # (E, nverts_per_elem) global ids, periodic-wrapped
    a: tuple
    b: tuple
    nelements_per_axis: tuple
    periodic: tuple

    @property
    def nelements(self):
        return self.vertex_ids.shape[0]

    @property
    def period(self):
        return np.array([(hi - lo) if per else 0.0
                         for lo, hi, per in zip(self.a, self.b, self.periodic)])


def _morton_order(counts):
    """Cell multi-indices (ncells, dim) sorted along a Z-curve."""
    grids = np.meshgrid(*[np.arange(n) for n in counts], indexing="ij")
    idx = np.stack([g.ravel() for g in grids], axis=1).astype(np.int64)
    code = np.zeros(len(idx), dtype=np.int64)
    nbits = int(max(counts) - 1).bit_length() if max(counts) > 1 else 1
    dim = len(counts)
    for bit in range(nbits):
        for d in range(dim):
            code |= ((idx[:, d] >> bit) & 1) << (bit * dim + d)
    return idx[np.argsort(code, kind="stable")]


def _kuhn_simplices(dim):
    """Simplices of the Kuhn split of the unit box, as corner bit-vectors."""
    simplices = []
    for perm in itertools.permutations(range(dim)):
        corner = np.zeros(dim, dtype=np.int64)
        verts = [corner.copy()]
        for axis in perm:
            corner[axis] = 1
            verts.append(corner.copy())
        simplices.append(np.array(verts))
    return simplices


def generate_box_mesh(a, b, nelements_per_axis, *, kind="simplex",
                      periodic=None):
    """Regular box mesh on [a, b] with the given cell counts per axis."""
    dim = len(a)
    counts = tuple(int(n) for n in nelements_per_axis)
    if periodic is None:
        periodic = (False,) * dim
    periodic = tuple(bool(p) for p in periodic)
    for n, per in zip(counts, periodic):
        if per and n < 3:
            raise ValueError("periodic axes need at least 3 cells")
    a = tuple(float(x) for x in a)
    b = tuple(float(x) for x in b)
    h = np.array([(hi - lo) / n for lo, hi, n in zip(a, b, counts)])
    cells = _morton_order(counts)                      # (ncells, dim)
    nvert_axis = np.array([n if per else n + 1 for n, per in zip(counts, periodic)])
    strides = np.cumprod(np.concatenate([[1], nvert_axis[:-1]]))

    def vid(corner_idx):
        wrapped = np.where(np.array(periodic), corner_idx % np.array(counts), corner_idx)
        return (wrapped * strides).sum(axis=-1)

    if kind == "simplex":
        pieces = _kuhn_simplices(dim)
    elif kind == "hypercube":
        pieces = [np.array(list(itertools.product([0, 1], repeat=dim)))[:, ::-1]]
    else:
        raise ValueError(kind)

    coords = []
    ids = []
    lo = np.array(a)
    for piece in pieces:
        corner_idx = cells[:, None, :] + piece[None, :, :]     # (ncells, nv, dim)
        xyz = lo + corner_idx * h
        gid = vid(corner_idx)
        if kind == "simplex":
            # positive orientation: swap the last two vertices if needed
            jac = xyz[:, 1:, :] - xyz[:, :1, :]
            det = np.linalg.det(jac)
            neg = det < 0
            if neg.any():
                xyz[neg, -2:] = xyz[neg][:, [-1, -2]]
                gid[neg, -2:] = gid[neg][:, [-1, -2]]
        coords.append(xyz)
        ids.append(gid)
    # interleave so the pieces of one cell are consecutive
    vertex_coords = np.stack(coords, axis=1).reshape(-1, pieces[0].shape[0], dim)
    vertex_ids = np.stack(ids, axis=1).reshape(-1, pieces[0].shape[0])
    return BoxMesh(dim=dim, kind=kind, vertex_coords=vertex_coords,
                   vertex_ids=vertex_ids.astype(np.int64), a=a, b=b,
                   nelements_per_axis=counts, periodic=periodic)
