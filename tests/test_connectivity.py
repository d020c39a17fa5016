"""Face pairings of the product's host flattening vs the oracle's
independent construction (centroid k-d tree + coordinate matching):
index maps must agree bit for bit."""

import numpy as np
import pytest

from cases import make_disc


@pytest.mark.parametrize("kind,dim,n,order,periodic", [
    ("simplex", 2, 5, 3, False), ("simplex", 2, 4, 4, True),
    ("simplex", 3, 3, 3, True), ("simplex", 3, 4, 2, False),
    ("simplex", 3, 3, 1, (True, False, True)),
    ("hypercube", 3, 3, 4, True), ("hypercube", 2, 4, 3, False),
])
def test_index_maps_bit_exact(kind, dim, n, order, periodic):
    d, od = make_disc(kind, dim, n, order, (0.0,) * dim, (1.0,) * dim, periodic)
    assert np.array_equal(d.connectivity.nbr_node_index, od.nbr_node_index)
    c = d.connectivity
    nb = np.zeros(d.nelements * d.nfaces, dtype=bool)
    nb[c.bface_elem * d.nfaces + c.bface_face] = True
    assert np.array_equal(~nb.reshape(d.nelements, d.nfaces), od.interior_mask)


def test_packed_pairing_decodes_to_index_map():
    d, _ = make_disc("simplex", 3, 3, 3, (0.0,) * 3, (1.0,) * 3, True)
    c = d.connectivity
    conn = c.conn.astype(np.int64)
    assert (conn >= 0).all()
    nbr = conn >> 8
    perm = conn & 255
    idx = nbr[:, :, None] * d.refel.nnodes + c.perm[perm].astype(np.int64)
    assert np.array_equal(idx, c.nbr_node_index)


def test_geometry_matches_oracle():
    d, od = make_disc("simplex", 3, 3, 3, (0.0,) * 3, (2.0,) * 3, False)
    assert np.allclose(d.geometry.normals, od.normals, atol=1e-15)
    assert np.allclose(d.geometry.fscale * od.jac_det[:, None],
                       od.face_area_ratio, rtol=1e-14)
    assert np.allclose(d.geometry.nodes, od.nodes, atol=1e-15)
