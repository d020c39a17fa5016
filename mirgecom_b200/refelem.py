"""Reference elements for the nodal DG discretization (host-side set-up only).

The reference builds its element groups with
``InterpolatoryEdgeClusteredGroupFactory(order)``
(mirgecom/discretization.py:74-83): warp-and-blend nodes on simplices and
Gauss-Lobatto-Legendre tensor nodes on hexahedra, with the full (exact) mass
matrix.  This module restates those published constructions:

* warp-and-blend nodes: Warburton, "An explicit construction of interpolation
  nodes on the simplex", J. Eng. Math. 56 (2006); Hesthaven & Warburton,
  "Nodal Discontinuous Galerkin Methods" (2008), sections 6.1 and 10.1;
* Gauss-Lobatto-Legendre nodes via Golub-Welsch on the Jacobi recurrence.

Nodal operators are basis independent; they are computed from a Legendre
product basis (which spans the total-degree space on simplices) and
collapsed-coordinate Gauss quadrature that integrates the mass products
exactly.  Everything here runs once at set-up on the host, in float64.

Every operator is returned in the form the DG right-hand side consumes
(mirgecom/operators.py:34-95, inverse mass folded in):

* ``W[r] = M^-1 D_r^T M``   -- weak derivative along reference axis r;
* ``LIFT[:, f*Nfp + m] = M^-1 E_f``  -- lift of face f's node m, with the
  face mass matrix taken in the face's own parametrisation (area 2 for a
  triangle face, 4 for a square face, 1 for a 0-d point face, 2 for an edge).
"""

from __future__ import annotations

import functools
import itertools
import math
from dataclasses import dataclass, field

import numpy as np

# {{{ 1-D Jacobi machinery


def jacobi_p(x, alpha, beta, n):
    """Orthonormal Jacobi polynomial P_n^(alpha,beta) at *x*."""
    x = np.asarray(x, dtype=np.float64)
    pl = np.zeros((n + 1,) + x.shape)
    gamma0 = (2 ** (alpha + beta + 1) / (alpha + beta + 1)
              * math.gamma(alpha + 1) * math.gamma(beta + 1)
              / math.gamma(alpha + beta + 1))
    pl[0] = 1.0 / math.sqrt(gamma0)
    if n == 0:
        return pl[0]
    gamma1 = (alpha + 1) * (beta + 1) / (alpha + beta + 3) * gamma0
    pl[1] = ((alpha + beta + 2) * x / 2 + (alpha - beta) / 2) / math.sqrt(gamma1)
    aold = 2 / (2 + alpha + beta) * math.sqrt(
        (alpha + 1) * (beta + 1) / (alpha + beta + 3))
    for i in range(1, n):
        h1 = 2 * i + alpha + beta
        anew = 2 / (h1 + 2) * math.sqrt(
            (i + 1) * (i + 1 + alpha + beta) * (i + 1 + alpha) * (i + 1 + beta)
            / (h1 + 1) / (h1 + 3))
        bnew = -(alpha ** 2 - beta ** 2) / h1 / (h1 + 2)
        pl[i + 1] = (-aold * pl[i - 1] + (x - bnew) * pl[i]) / anew
        aold = anew
    return pl[n]


def jacobi_gq(alpha, beta, n):
    """Gauss quadrature (n+1 points) for weight (1-x)^alpha (1+x)^beta."""
    if n == 0:
        return (np.array([(alpha - beta) / (alpha + beta + 2)]), np.array([2.0]))
    j = np.arange(n + 1, dtype=np.float64)
    h1 = 2 * j + alpha + beta
    diag = -0.5 * (alpha ** 2 - beta ** 2) / (h1 + 2) / np.where(h1 == 0, 1, h1)
    if alpha + beta < 10 * np.finfo(float).eps:
        diag[0] = 0.0
    jj = np.arange(1, n + 1, dtype=np.float64)
    h1o = 2 * jj + alpha + beta
    off = 2 / (h1o) * np.sqrt(jj * (jj + alpha + beta) * (jj + alpha) * (jj + beta)
                              / (h1o - 1) / (h1o + 1))
    mat = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
    x, v = np.linalg.eigh(mat)
    w = v[0] ** 2 * 2 ** (alpha + beta + 1) / (alpha + beta + 1) \
        * math.gamma(alpha + 1) * math.gamma(beta + 1) / math.gamma(alpha + beta + 1)
    return x, w


def jacobi_gl(alpha, beta, n):
    """Gauss-Lobatto points (n+1 of them) for the Jacobi weight."""
    if n == 1:
        return np.array([-1.0, 1.0])
    xint, _ = jacobi_gq(alpha + 1, beta + 1, n - 2)
    return np.concatenate([[-1.0], xint, [1.0]])


def legendre_and_derivative(x, n):
    """Legendre P_n (classical normalisation) and P_n' at *x*."""
    x = np.asarray(x, dtype=np.float64)
    p = np.zeros((n + 1,) + x.shape)
    dp = np.zeros_like(p)
    p[0] = 1.0
    if n >= 1:
        p[1] = x
        dp[1] = 1.0
    for k in range(1, n):
        p[k + 1] = ((2 * k + 1) * x * p[k] - k * p[k - 1]) / (k + 1)
        dp[k + 1] = dp[k - 1] + (2 * k + 1) * p[k]
    return p, dp

# }}}


# {{{ warp-and-blend nodes

_ALPHA_OPT_2D = [0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999,
                 1.2832, 1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223, 1.6258]
_ALPHA_OPT_3D = [0.0, 0.0, 0.0, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577, 1.1603,
                 1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655]


def _warp_factor(n, rout):
    """1-D edge warp: equispaced -> GLL, divided by the edge blend."""
    lglr = jacobi_gl(0, 0, n)
    req = np.linspace(-1, 1, n + 1)
    veq = np.stack([jacobi_p(req, 0, 0, i) for i in range(n + 1)], axis=1)
    pmat = np.stack([jacobi_p(rout, 0, 0, i) for i in range(n + 1)], axis=0)
    lmat = np.linalg.solve(veq.T, pmat)
    warp = lmat.T @ (lglr - req)
    zerof = (np.abs(rout) < 1.0 - 1.0e-10).astype(np.float64)
    sf = 1.0 - (zerof * rout) ** 2
    return warp / sf + warp * (zerof - 1)


def _nodes_2d_equilateral(n, alpha=None):
    if alpha is None:
        alpha = _ALPHA_OPT_2D[n - 1] if n < 16 else 5.0 / 3.0
    l1, l3 = [], []
    for i in range(n + 1):
        for j in range(n + 1 - i):
            l1.append(i / n)
            l3.append(j / n)
    l1 = np.array(l1)
    l3 = np.array(l3)
    l2 = 1.0 - l1 - l3
    x = -l2 + l3
    y = (-l2 - l3 + 2 * l1) / math.sqrt(3.0)
    blend1 = 4 * l2 * l3
    blend2 = 4 * l1 * l3
    blend3 = 4 * l1 * l2
    warpf1 = _warp_factor(n, l3 - l2)
    warpf2 = _warp_factor(n, l1 - l3)
    warpf3 = _warp_factor(n, l2 - l1)
    warp1 = blend1 * warpf1 * (1 + (alpha * l1) ** 2)
    warp2 = blend2 * warpf2 * (1 + (alpha * l2) ** 2)
    warp3 = blend3 * warpf3 * (1 + (alpha * l3) ** 2)
    x = x + warp1 + math.cos(2 * math.pi / 3) * warp2 + math.cos(4 * math.pi / 3) * warp3
    y = y + math.sin(2 * math.pi / 3) * warp2 + math.sin(4 * math.pi / 3) * warp3
    return x, y


def _xy_to_rs(x, y):
    l1 = (math.sqrt(3.0) * y + 1.0) / 3.0
    l2 = (-3.0 * x - math.sqrt(3.0) * y + 2.0) / 6.0
    l3 = (3.0 * x - math.sqrt(3.0) * y + 2.0) / 6.0
    return -l2 + l3 - l1, -l2 - l3 + l1


def _eval_warp(p, xnodes, xout):
    warp = np.zeros_like(xout)
    xeq = np.array([-1 + 2 * (p - i) / p for i in range(p + 1)])
    for i in range(p + 1):
        d = (xnodes[i] - xeq[i]) * np.ones_like(xout)
        for j in range(1, p):
            if i != j:
                d = d * (xout - xeq[j]) / (xeq[i] - xeq[j])
        if i != 0:
            d = -d / (xeq[i] - xeq[0])
        if i != p:
            d = d / (xeq[i] - xeq[p])
        warp = warp + d
    return warp


def _eval_shift(p, pval, l1, l2, l3):
    gauss_x = -jacobi_gl(0, 0, p)
    blend1 = l2 * l3
    blend2 = l1 * l3
    blend3 = l1 * l2
    warpfactor1 = 4 * _eval_warp(p, gauss_x, l3 - l2)
    warpfactor2 = 4 * _eval_warp(p, gauss_x, l1 - l3)
    warpfactor3 = 4 * _eval_warp(p, gauss_x, l2 - l1)
    warp1 = blend1 * warpfactor1 * (1 + (pval * l1) ** 2)
    warp2 = blend2 * warpfactor2 * (1 + (pval * l2) ** 2)
    warp3 = blend3 * warpfactor3 * (1 + (pval * l3) ** 2)
    dx = warp1 + math.cos(2 * math.pi / 3) * warp2 + math.cos(4 * math.pi / 3) * warp3
    dy = math.sin(2 * math.pi / 3) * warp2 + math.sin(4 * math.pi / 3) * warp3
    return dx, dy


def _nodes_3d_equilateral(p):
    alpha = _ALPHA_OPT_3D[p - 1] if p <= 15 else 1.0
    tol = 1e-10
    r, s, t = [], [], []
    for n in range(p + 1):
        for m in range(p + 1 - n):
            for q in range(p + 1 - n - m):
                r.append(-1 + q * 2 / p)
                s.append(-1 + m * 2 / p)
                t.append(-1 + n * 2 / p)
    r, s, t = (np.array(a) for a in (r, s, t))
    l1 = (1 + t) / 2
    l2 = (1 + s) / 2
    l3 = -(1 + r + s + t) / 2
    l4 = (1 + r) / 2
    v1 = np.array([-1, -1 / math.sqrt(3), -1 / math.sqrt(6)])
    v2 = np.array([1, -1 / math.sqrt(3), -1 / math.sqrt(6)])
    v3 = np.array([0, 2 / math.sqrt(3), -1 / math.sqrt(6)])
    v4 = np.array([0, 0, 3 / math.sqrt(6)])
    t1 = np.array([v2 - v1, v2 - v1, v3 - v2, v3 - v1])
    t2 = np.array([v3 - 0.5 * (v1 + v2), v4 - 0.5 * (v1 + v2),
                   v4 - 0.5 * (v2 + v3), v4 - 0.5 * (v1 + v3)])
    t1 /= np.linalg.norm(t1, axis=1)[:, None]
    t2 /= np.linalg.norm(t2, axis=1)[:, None]
    xyz = np.outer(l3, v1) + np.outer(l4, v2) + np.outer(l2, v3) + np.outer(l1, v4)
    shift = np.zeros_like(xyz)
    for face in range(4):
        la, lb, lc, ld = [(l1, l2, l3, l4), (l2, l1, l3, l4),
                          (l3, l1, l4, l2), (l4, l1, l3, l2)][face]
        warp1, warp2 = _eval_shift(p, alpha, lb, lc, ld)
        blend = lb * lc * ld
        denom = (lb + 0.5 * la) * (lc + 0.5 * la) * (ld + 0.5 * la)
        ids = denom > tol
        blend[ids] = (1 + (alpha * la[ids]) ** 2) * blend[ids] / denom[ids]
        shift += np.outer(blend * warp1, t1[face]) + np.outer(blend * warp2, t2[face])
        ids = (la < tol) & ((lb > tol).astype(int) + (lc > tol).astype(int)
                            + (ld > tol).astype(int) < 3)
        shift[ids] = (np.outer(warp1[ids], t1[face]) + np.outer(warp2[ids], t2[face]))
    xyz = xyz + shift
    # equilateral -> reference (-1,-1,-1),(1,-1,-1),(-1,1,-1),(-1,-1,1)
    rhs = xyz.T - 0.5 * (v2 + v3 + v4 - v1)[:, None]
    amat = np.stack([0.5 * (v2 - v1), 0.5 * (v3 - v1), 0.5 * (v4 - v1)], axis=1)
    return np.linalg.solve(amat, rhs)


def simplex_nodes(dim, order, face_of_3d=False):
    """Warp-and-blend nodes on the reference simplex, shape ``(dim, Np)``.

    With *face_of_3d* the 2-D set is built with the blend parameter of the
    3-D construction, so that it coincides with the trace of the 3-D nodes
    on each tetrahedron face.
    """
    if order == 0:
        return np.full((dim, 1), -1.0 / 3.0 if dim == 2 else -0.5) \
            if dim > 1 else np.zeros((1, 1))
    if dim == 1:
        return jacobi_gl(0, 0, order)[None, :]
    if dim == 2:
        alpha = None
        if face_of_3d:
            alpha = _ALPHA_OPT_3D[order - 1] if order <= 15 else 1.0
        x, y = _nodes_2d_equilateral(order, alpha)
        r, s = _xy_to_rs(x, y)
        return np.stack([r, s])
    if dim == 3:
        return _nodes_3d_equilateral(order)
    raise ValueError(f"unsupported dimension {dim}")

# }}}


# {{{ polynomial spaces and quadrature

def total_degree_exponents(dim, order):
    return [e for e in itertools.product(range(order + 1), repeat=dim)
            if sum(e) <= order]


def tensor_exponents(dim, order):
    return list(itertools.product(range(order + 1), repeat=dim))


def legendre_basis(points, exponents):
    """Legendre product basis and its gradient at *points* ``(dim, n)``."""
    dim, npts = points.shape
    order = max(max(e) for e in exponents)
    pv, dpv = zip(*(legendre_and_derivative(points[d], order) for d in range(dim)))
    vdm = np.ones((npts, len(exponents)))
    grads = np.ones((dim, npts, len(exponents)))
    for j, e in enumerate(exponents):
        for d in range(dim):
            vdm[:, j] *= pv[d][e[d]]
            for r in range(dim):
                grads[r, :, j] *= (dpv[d][e[d]] if r == d else pv[d][e[d]])
    return vdm, grads


def simplex_quadrature(dim, nq):
    """Collapsed (Duffy) Gauss rule on the reference simplex, exact to 2nq-3."""
    if dim == 1:
        x, w = jacobi_gq(0, 0, nq - 1)
        return x[None, :], w
    xg, wg = jacobi_gq(0, 0, nq - 1)
    if dim == 2:
        a, b = np.meshgrid(xg, xg, indexing="ij")
        wa, wb = np.meshgrid(wg, wg, indexing="ij")
        r = (1 + a) * (1 - b) / 2 - 1
        s = b
        w = wa * wb * (1 - b) / 2
        return np.stack([r.ravel(), s.ravel()]), w.ravel()
    if dim == 3:
        a, b, c = np.meshgrid(xg, xg, xg, indexing="ij")
        wa, wb, wc = np.meshgrid(wg, wg, wg, indexing="ij")
        # (a,b,c) in cube -> tet with vertices (-1,-1,-1),(1,-1,-1),(-1,1,-1),(-1,-1,1)
        t = c
        s = (1 + b) * (1 - c) / 2 - 1
        r = (1 + a) * (-s - t) / 2 - 1
        w = wa * wb * wc * (1 - b) / 2 * ((1 - c) / 2) ** 2
        return np.stack([r.ravel(), s.ravel(), t.ravel()]), w.ravel()
    raise ValueError(dim)


def cube_quadrature(dim, nq):
    xg, wg = jacobi_gq(0, 0, nq - 1)
    grids = np.meshgrid(*([xg] * dim), indexing="ij")
    wgrids = np.meshgrid(*([wg] * dim), indexing="ij")
    w = np.ones_like(grids[0])
    for wgd in wgrids:
        w = w * wgd
    return np.stack([g.ravel() for g in grids]), w.ravel()

# }}}


# {{{ extended-precision nodal operators

_MP_DPS = 40


def _mp_gauss_legendre(n):
    """n-point Gauss-Legendre rule on [-1, 1] in mpmath precision."""
    import mpmath as mp
    xs, ws = [], []
    for i in range(1, n + 1):
        x = mp.cos(mp.pi * (i - mp.mpf(1) / 4) / (n + mp.mpf(1) / 2))
        for _ in range(100):
            p0, p1 = mp.mpf(1), x
            for k in range(2, n + 1):
                p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
            dp = n * (x * p1 - p0) / (x * x - 1)
            dx = p1 / dp
            x -= dx
            if abs(dx) < mp.mpf(10) ** (-_MP_DPS + 5):
                break
        xs.append(x)
        ws.append(2 / ((1 - x * x) * dp * dp))
    return xs, ws


def _mp_quadrature(kind, dim, nq):
    """Gauss rule on the reference simplex (collapsed) or hypercube, mpmath."""
    import itertools as it

    import mpmath as mp
    xg, wg = _mp_gauss_legendre(nq)
    pts, wts = [], []
    for idx in it.product(range(nq), repeat=dim):
        c = [xg[i] for i in idx]
        w = mp.mpf(1)
        for i in idx:
            w *= wg[i]
        if kind == "hypercube" or dim == 1:
            pts.append(c)
            wts.append(w)
        elif dim == 2:
            a, b = c
            pts.append([(1 + a) * (1 - b) / 2 - 1, b])
            wts.append(w * (1 - b) / 2)
        else:
            a, b, cc = c
            t = cc
            s_ = (1 + b) * (1 - cc) / 2 - 1
            r = (1 + a) * (-s_ - t) / 2 - 1
            pts.append([r, s_, t])
            wts.append(w * (1 - b) / 2 * ((1 - cc) / 2) ** 2)
    return pts, wts


def _mp_basis(point, exponents, order):
    """Legendre-product basis values and gradients at one point (mpmath)."""
    import mpmath as mp
    dim = len(point)
    pv, dpv = [], []
    for d in range(dim):
        x = point[d]
        p = [mp.mpf(1), x]
        dp = [mp.mpf(0), mp.mpf(1)]
        for k in range(1, order):
            p.append(((2 * k + 1) * x * p[k] - k * p[k - 1]) / (k + 1))
            dp.append(dp[k - 1] + (2 * k + 1) * p[k])
        pv.append(p)
        dpv.append(dp)
    vals, grads = [], [[] for _ in range(dim)]
    for e in exponents:
        v = mp.mpf(1)
        for d in range(dim):
            v *= pv[d][e[d]]
        vals.append(v)
        for r in range(dim):
            g = mp.mpf(1)
            for d in range(dim):
                g *= dpv[d][e[d]] if d == r else pv[d][e[d]]
            grads[r].append(g)
    return vals, grads


def _nodal_operators_mp(nodes, exponents, kind, nq):
    """Vandermonde, exact mass matrix and derivative matrices, computed in
    mpmath (40 digits) and rounded once to float64; also returns the mpmath
    mass and derivative matrices for further exact products."""
    import mpmath as mp
    mp.mp.dps = _MP_DPS
    dim, npts = nodes.shape
    order = max(max(e) for e in exponents)
    nb = len(exponents)
    vdm = mp.matrix(npts, nb)
    gr = [mp.matrix(npts, nb) for _ in range(dim)]
    for i in range(npts):
        vals, grads = _mp_basis([mp.mpf(float(nodes[d, i])) for d in range(dim)],
                                exponents, order)
        for j in range(nb):
            vdm[i, j] = vals[j]
            for r in range(dim):
                gr[r][i, j] = grads[r][j]
    vinv = mp.inverse(vdm)
    qp, qw = _mp_quadrature(kind, dim, nq)
    # mass = sum_q w_q l_i(x_q) l_j(x_q),  l = interpolants
    lq = mp.matrix(len(qp), npts)
    for q, pt in enumerate(qp):
        vals, _ = _mp_basis(pt, exponents, order)
        row = mp.matrix([vals])
        lrow = row * vinv
        for j in range(npts):
            lq[q, j] = lrow[0, j]
    mass = mp.matrix(npts, npts)
    for q in range(len(qp)):
        for i in range(npts):
            wi = qw[q] * lq[q, i]
            for j in range(npts):
                mass[i, j] += wi * lq[q, j]
    diff = [gr[r] * vinv for r in range(dim)]
    return vdm, mass, diff


def _mp_to_np(m):
    return np.array([[float(m[i, j]) for j in range(m.cols)] for i in range(m.rows)])


def _nodal_operators(nodes, exponents, quad):
    """float64 interface (kept for the oracle-independent consistency check)."""
    vdm, grads = legendre_basis(nodes, exponents)
    vinv = np.linalg.inv(vdm)
    qx, qw = quad
    vq, _ = legendre_basis(qx, exponents)
    interp_q = vq @ vinv
    mass = interp_q.T @ (qw[:, None] * interp_q)
    diff = np.stack([g @ vinv for g in grads])
    return vdm, mass, diff

# }}}


@dataclass
class ReferenceElement:
    """Nodal reference element (simplex or hypercube) with DG operators."""

    kind: str                    # "simplex" or "hypercube"
    dim: int
    order: int
    nodes: np.ndarray            # (dim, Np) reference coordinates
    vertices: np.ndarray         # (nverts, dim) reference vertices
    face_vertices: list          # local vertex indices of each face
    face_nodes: np.ndarray       # (Nf, Nfp) volume node index of face node m
    face_param: np.ndarray       # (Nf, Nfp, nfv) vertex weights of face nodes
    mass: np.ndarray             # (Np, Np)
    mass_inv: np.ndarray
    diff: np.ndarray             # (dim, Np, Np) strong derivative
    weak: np.ndarray             # (dim, Np, Np) W_r = M^-1 D_r^T M
    lift: np.ndarray             # (Np, Nf*Nfp) M^-1 E
    face_mass: np.ndarray        # (Nfp, Nfp) face mass in face parametrisation
    face_param_area: float       # measure of the face parametrisation domain
    ref_face_normals: np.ndarray  # (Nf, dim) unit outward normals (reference)
    ref_face_areas: np.ndarray   # (Nf,) reference face measures
    ref_volume: float
    extra: dict = field(default_factory=dict)

    @property
    def nnodes(self):
        return self.nodes.shape[1]

    @property
    def nfaces(self):
        return self.face_nodes.shape[0]

    @property
    def nface_nodes(self):
        return self.face_nodes.shape[1]

    @property
    def face_scale_ref(self):
        """Reference face measure over face-parametrisation measure."""
        return self.ref_face_areas / self.face_param_area


def _simplex_vertices(dim):
    verts = -np.ones((dim + 1, dim))
    for i in range(dim):
        verts[i + 1, i] = 1.0
    return verts


_SIMPLEX_FACES = {
    1: [[0], [1]],
    2: [[0, 1], [1, 2], [2, 0]],
    3: [[0, 1, 2], [0, 1, 3], [1, 2, 3], [0, 2, 3]],
}


def _barycentric(points, verts):
    """Barycentric coordinates of *points* (dim, n) w.r.t. simplex *verts*."""
    dim = points.shape[0]
    amat = (verts[1:] - verts[0]).T
    lam_rest = np.linalg.solve(amat, points - verts[0][:, None])
    return np.vstack([1 - lam_rest.sum(axis=0), lam_rest])


def make_simplex_element(dim, order):
    nodes = simplex_nodes(dim, order)
    verts = _simplex_vertices(dim)
    exps = total_degree_exponents(dim, order)
    import mpmath as mp
    vdm_mp, mass_mp, diff_mp = _nodal_operators_mp(nodes, exps, "simplex", order + 3)
    mass_inv_mp = mp.inverse(mass_mp)
    vdm = _mp_to_np(vdm_mp)
    mass = _mp_to_np(mass_mp)
    mass_inv = _mp_to_np(mass_inv_mp)
    diff = np.stack([_mp_to_np(d) for d in diff_mp])
    weak = np.stack([_mp_to_np(mass_inv_mp * d.T * mass_mp) for d in diff_mp])
    faces = _SIMPLEX_FACES[dim]

    # face nodes ordered like the (dim-1) reference node set
    lam = _barycentric(nodes, verts)                 # (dim+1, Np)
    if dim == 1:
        fnodes_ref = np.zeros((0, 1))
        face_lam_ref = np.ones((1, 1))
    else:
        fnodes_ref = simplex_nodes(dim - 1, order, face_of_3d=(dim == 3))
        face_lam_ref = _barycentric(fnodes_ref, _simplex_vertices(dim - 1))
    nfp = face_lam_ref.shape[1]
    face_nodes = np.zeros((len(faces), nfp), dtype=np.int64)
    for f, fv in enumerate(faces):
        for m in range(nfp):
            # the volume node whose barycentrics on face f equal the face node's
            target = np.zeros(dim + 1)
            target[fv] = face_lam_ref[:, m]
            dist = np.abs(lam - target[:, None]).sum(axis=0)
            k = int(np.argmin(dist))
            if dist[k] > 1e-10:
                raise RuntimeError("face node not found in volume node set")
            face_nodes[f, m] = k

    # face mass matrix in the face's own reference parametrisation
    if dim == 1:
        face_mass_mp = mp.matrix([[1]])
        param_area = 1.0
    else:
        fexps = total_degree_exponents(dim - 1, order)
        _, face_mass_mp, _ = _nodal_operators_mp(fnodes_ref, fexps, "simplex", order + 3)
        param_area = 2.0
    face_mass = _mp_to_np(face_mass_mp)

    npn = nodes.shape[1]
    lift = np.zeros((npn, len(faces) * nfp))
    for f in range(len(faces)):
        # M^-1 E_f with E_f the face mass placed on the face's volume nodes
        for i in range(npn):
            for m in range(nfp):
                acc = mp.mpf(0)
                for mm in range(nfp):
                    acc += mass_inv_mp[i, int(face_nodes[f, mm])] * face_mass_mp[mm, m]
                lift[i, f * nfp + m] = float(acc)

    # reference outward normals and face measures
    centroid = verts.mean(axis=0)
    normals = np.zeros((len(faces), dim))
    areas = np.zeros(len(faces))
    for f, fv in enumerate(faces):
        fverts = verts[fv]
        if dim == 1:
            n = np.array([1.0]) * np.sign(fverts[0, 0] - centroid[0])
            area = 1.0
        else:
            tang = (fverts[1:] - fverts[0])
            if dim == 2:
                n = np.array([tang[0, 1], -tang[0, 0]])
                area = np.linalg.norm(tang[0])
            else:
                n = np.cross(tang[0], tang[1])
                area = 0.5 * np.linalg.norm(n)
            n = n / np.linalg.norm(n)
            if np.dot(n, fverts[0] - centroid) < 0:
                n = -n
        normals[f] = n
        areas[f] = area
    ref_volume = {1: 2.0, 2: 2.0, 3: 4.0 / 3.0}[dim]
    return ReferenceElement(
        kind="simplex", dim=dim, order=order, nodes=nodes, vertices=verts,
        face_vertices=faces, face_nodes=face_nodes,
        face_param=face_lam_ref.T[None, :, :].repeat(len(faces), axis=0),
        mass=mass, mass_inv=mass_inv, diff=diff, weak=weak, lift=lift,
        face_mass=face_mass, face_param_area=param_area,
        ref_face_normals=normals, ref_face_areas=areas, ref_volume=ref_volume,
        extra={"vandermonde": vdm})


def _hypercube_vertices(dim):
    return np.array(list(itertools.product([-1.0, 1.0], repeat=dim)))[:, ::-1]


def make_hypercube_element(dim, order):
    """Tensor-product GLL element; node index = i0 + (p+1) i1 + (p+1)^2 i2.

    The operators are Kronecker products of 1-D operators computed in
    mpmath precision (exact mass matrix on the GLL nodes)."""
    import mpmath as mp
    x1 = jacobi_gl(0, 0, order)
    n1 = order + 1
    grids = np.meshgrid(*([x1] * dim), indexing="ij")
    # axis 0 fastest
    nodes = np.stack([g.transpose(tuple(range(dim))[::-1]).ravel() for g in grids])
    v1_mp, mass1_mp, diff1_mp = _nodal_operators_mp(
        x1[None, :], [(i,) for i in range(n1)], "hypercube", order + 2)
    mass1_inv_mp = mp.inverse(mass1_mp)
    mass1 = _mp_to_np(mass1_mp)
    mass1_inv = _mp_to_np(mass1_inv_mp)
    diff1 = _mp_to_np(diff1_mp[0])
    weak1 = _mp_to_np(mass1_inv_mp * diff1_mp[0].T * mass1_mp)
    eye = np.eye(n1)

    def kron_axis(op, axis):
        # operator acting along `axis` (0 = fastest index)
        mats = [op if a == axis else eye for a in range(dim)][::-1]
        out = mats[0]
        for mmat in mats[1:]:
            out = np.kron(out, mmat)
        return out

    def kron_all(op):
        out = op
        for _ in range(dim - 1):
            out = np.kron(out, op)
        return out

    mass = kron_all(mass1)
    mass_inv = kron_all(mass1_inv)
    diff = np.stack([kron_axis(diff1, r) for r in range(dim)])
    weak = np.stack([kron_axis(weak1, r) for r in range(dim)])
    vdm = kron_all(_mp_to_np(v1_mp))

    # faces: (axis, side) -> f = 2*axis + side
    faces = []
    face_nodes = []
    verts = _hypercube_vertices(dim)
    for axis in range(dim):
        for side, val in enumerate([-1.0, 1.0]):
            fv = [i for i, v in enumerate(verts) if v[axis] == val]
            faces.append(fv)
            on = np.nonzero(np.abs(nodes[axis] - val) < 1e-12)[0]
            face_nodes.append(on)     # ascending volume index = tensor order
    face_nodes = np.array(face_nodes)
    nfp = face_nodes.shape[1]
    if dim == 1:
        face_mass = np.ones((1, 1))
        param_area = 1.0
    else:
        face_mass = mass1 if dim == 2 else np.kron(mass1, mass1)
        param_area = 2.0 ** (dim - 1)
    npn = nodes.shape[1]
    lift = np.zeros((npn, len(faces) * nfp))
    for f in range(len(faces)):
        axis, side = divmod(f, 2)
        col = 0 if side == 0 else n1 - 1
        # M^-1 E_f = (M1^-1 e_side along `axis`) x identity on the face axes
        for m in range(nfp):
            fnode = face_nodes[f, m]
            rest = [(fnode // n1 ** a) % n1 for a in range(dim)]
            for i1 in range(n1):
                idx = list(rest)
                idx[axis] = i1
                vol = sum(idx[a] * n1 ** a for a in range(dim))
                lift[vol, f * nfp + m] = mass1_inv[i1, col]
    normals = np.zeros((len(faces), dim))
    for axis in range(dim):
        normals[2 * axis, axis] = -1.0
        normals[2 * axis + 1, axis] = 1.0
    areas = np.full(len(faces), 2.0 ** (dim - 1))
    # face node vertex weights (multilinear shape functions of the face corners)
    face_param = []
    for f, fv in enumerate(faces):
        w = np.ones((nfp, len(fv)))
        for k, vi in enumerate(fv):
            for d in range(dim):
                w[:, k] *= 0.5 * (1 + verts[vi, d] * nodes[d, face_nodes[f]])
        face_param.append(w)
    return ReferenceElement(
        kind="hypercube", dim=dim, order=order, nodes=nodes, vertices=verts,
        face_vertices=faces, face_nodes=face_nodes, face_param=np.array(face_param),
        mass=mass, mass_inv=mass_inv, diff=diff, weak=weak, lift=lift,
        face_mass=face_mass, face_param_area=param_area,
        ref_face_normals=normals, ref_face_areas=areas, ref_volume=2.0 ** dim,
        extra={"vandermonde": vdm, "nodes1d": x1, "mass1d": mass1,
               "diff1d": diff1, "weak1d": weak1, "mass1d_inv": mass1_inv})


@functools.lru_cache(maxsize=None)
def make_reference_element(kind, dim, order):
    """Cached: the operators are pure functions of (kind, dim, order)."""
    if kind == "simplex":
        return make_simplex_element(dim, order)
    if kind == "hypercube":
        return make_hypercube_element(dim, order)
    raise ValueError(kind)
