"""DG operators of the oracle (float64 numpy).  Test infrastructure only.

Restates the reference's operator sequence one numpy operation at a time:

* ``grad_operator`` / ``div_operator``: mirgecom/operators.py:34-95, i.e.
  ``-M^-1 (weak_local_grad(u) - face_mass(flux))`` with grudge's
  ``weak_local_grad`` (J rx^T D^T M u), ``face_mass`` (per-face mass matrix
  times the face area ratio) and ``inverse_mass`` ((1/J) M^-1) written out
  explicitly rather than folded;
* ``euler_operator``: mirgecom/euler.py:313-416;
* ``grad_cv_operator`` / ``grad_t_operator`` / ``ns_operator``:
  mirgecom/navierstokes.py:118-575;
* the operator fluid states: mirgecom/gas_model.py:494-904
  (``project_fluid_state``, ``make_fluid_state_trace_pairs``,
  ``make_operator_fluid_states``), including the mixture temperature solve on
  both sides of every face seeded by the restricted volume temperature;
* boundaries: mirgecom/boundary.py:796-1049 (Prescribed and Dummy) and the
  Mengaldo treatment of boundary.py:391-793 with its walls and flow
  boundaries (AdiabaticSlip :1052, Farfield :1146, PressureOutflow :1231,
  IsothermalWall :1727, AdiabaticNoslipWall :1794).

The connectivity is built here independently of the product (face matching
by centroid k-d tree, node matching by coordinates), and compared with the
product's index maps bit for bit in the tests.
"""

from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree

from oracle import physics as ph


class OracleDisc:
    """Geometry and connectivity recomputed from the mesh vertices."""

    def __init__(self, mesh, refel):
        self.mesh = mesh
        self.refel = refel
        self.dim = d = mesh.dim
        vc = mesh.vertex_coords
        kind = refel.kind
        if kind == "simplex":
            jac = np.stack([(vc[:, i + 1] - vc[:, 0]) / 2 for i in range(d)], axis=2)
        else:
            jac = np.stack([(vc[:, 1 << i] - vc[:, 0]) / 2 for i in range(d)], axis=2)
        self.jac_det = np.linalg.det(jac)
        self.rx = np.linalg.inv(jac)                  # [e, r, j]
        self.nodes = vc[:, 0, :].T[:, :, None] + np.einsum(
            "eir,rn->ien", jac, refel.nodes + 1.0)   # (d, E, Np)
        self.nelements = vc.shape[0]
        fv = refel.face_vertices
        nf = len(fv)
        # physical face normals and areas from the face vertices
        cent = vc.mean(axis=1)
        normals = np.zeros((self.nelements, nf, d))
        areas = np.zeros((self.nelements, nf))
        for f, verts in enumerate(fv):
            pv = vc[:, verts]                         # (E, nfv, d)
            if d == 1:
                n = np.ones((self.nelements, 1))
                a = np.ones(self.nelements)
            elif d == 2:
                t = pv[:, 1] - pv[:, 0]
                n = np.stack([t[:, 1], -t[:, 0]], axis=1)
                a = np.linalg.norm(t, axis=1)
            else:
                if len(verts) == 3:
                    n = np.cross(pv[:, 1] - pv[:, 0], pv[:, 2] - pv[:, 0])
                    a = 0.5 * np.linalg.norm(n, axis=1)
                else:
                    # parallelogram face: the two edges from vertex 0
                    n = np.cross(pv[:, 1] - pv[:, 0], pv[:, 2] - pv[:, 0])
                    a = np.linalg.norm(n, axis=1)
            n = n / np.linalg.norm(n, axis=1)[:, None]
            sgn = np.sign(np.sum(n * (pv[:, 0] - cent), axis=1))
            normals[:, f] = n * sgn[:, None]
            areas[:, f] = a
        self.normals = normals                         # (E, Nf, d)
        self.face_area_ratio = areas / refel.face_param_area
        self._build_connectivity()

    def _build_connectivity(self):
        refel = self.refel
        mesh = self.mesh
        d = self.dim
        fn = refel.face_nodes
        nf, nfp = fn.shape
        ne = self.nelements
        fxyz = self.nodes[:, :, fn]                    # (d, E, Nf, Nfp)
        cent = fxyz.mean(axis=3).reshape(d, -1).T      # (E*Nf, d)
        lo = np.array(mesh.a)
        period = np.array([(b - a) if p else 0.0 for a, b, p in
                           zip(mesh.a, mesh.b, mesh.periodic)])
        box = np.where(period > 0, period, 1e300)
        pts = cent - lo
        pts = np.where(period > 0, np.mod(pts, np.where(period > 0, period, 1.0)), pts)
        # keep coordinates within the periodic box for cKDTree
        pts = np.where((period > 0) & (pts >= box - 1e-12), 0.0, pts)
        shift = np.where(period > 0, 0.0, -pts.min(axis=0) + 1.0)
        tree = cKDTree(pts + shift, boxsize=np.where(period > 0, period, 1e6 + 4 * np.abs(pts).max()))
        dist, idx = tree.query(pts + shift, k=2)
        hmin = np.min(np.abs(self.jac_det)) ** (1.0 / d)
        matched = dist[:, 1] < 1e-8 * max(1.0, hmin)
        self_first = idx[:, 0] == np.arange(len(idx))
        partner = np.where(self_first, idx[:, 1], idx[:, 0])
        self.nbr_node_index = np.full((ne, nf, nfp), -1, dtype=np.int64)
        own = np.nonzero(matched)[0]
        oth = partner[own]
        oe, of = own // nf, own % nf
        te, tf = oth // nf, oth % nf
        a = fxyz[:, oe, of]                            # (d, n, Nfp)
        b = fxyz[:, te, tf]
        diff = a[:, :, :, None] - b[:, :, None, :]     # (d, n, Nfp, Nfp)
        if np.any(period > 0):
            per = period.reshape(d, 1, 1, 1)
            diff = np.where(per > 0, diff - np.round(diff / np.where(per > 0, per, 1.0)) * per, diff)
        dd = np.sqrt(np.sum(diff ** 2, axis=0))        # (n, Nfp, Nfp)
        best = np.argmin(dd, axis=2)
        self.nbr_node_index[oe, of] = te[:, None] * refel.nnodes + fn[tf][np.arange(len(tf))[:, None], best]
        bmask = ~matched
        self.bface_elem = np.nonzero(bmask)[0] // nf
        self.bface_face = np.nonzero(bmask)[0] % nf
        self.interior_mask = matched.reshape(ne, nf)

    # {{{ grudge operations

    def to_faces(self, u):
        """Volume -> all-faces restriction (op.project vol -> all_faces)."""
        return u[..., self.refel.face_nodes]           # (..., E, Nf, Nfp)

    def exterior(self, u):
        """Neighbour values at own face nodes (interior_trace_pairs .ext)."""
        flat = u.reshape(u.shape[:-2] + (-1,))
        idx = np.where(self.nbr_node_index >= 0, self.nbr_node_index, 0)
        return flat[..., idx]                          # (..., E, Nf, Nfp)

    def weak_local_grad(self, u):
        """grudge op.weak_local_grad: (..., E, Np) -> (d, ..., E, Np)."""
        r = self.refel
        out = []
        for j in range(self.dim):
            acc = 0.0
            for k in range(self.dim):
                dtm = r.diff[k].T @ r.mass             # D_r^T M
                acc = acc + self.jac_det[:, None] * self.rx[:, k, j][:, None] \
                    * np.einsum("ab,...eb->...ea", dtm, u)
            out.append(acc)
        return np.array(out)

    def weak_local_div(self, v):
        """v: (..., d, E, Np) -> (..., E, Np)."""
        wg = [self.weak_local_grad(v[..., j, :, :])[j] for j in range(self.dim)]
        return sum(wg)

    def face_mass(self, flux):
        """flux (..., E, Nf, Nfp) -> (..., E, Np)."""
        r = self.refel
        out = np.zeros(flux.shape[:-2] + (r.nnodes,))
        for f in range(r.nfaces):
            contrib = self.face_area_ratio[:, f][:, None] * np.einsum(
                "mk,...ek->...em", r.face_mass, flux[..., f, :])
            out[..., r.face_nodes[f]] += contrib
        return out

    def inverse_mass(self, u):
        return np.einsum("ab,...eb->...ea", self.refel.mass_inv, u) / self.jac_det[:, None]

    # }}}


def grad_operator(disc, u, flux):
    """mirgecom/operators.py:34-63.  flux: (d, ..., E, Nf, Nfp)."""
    wg = disc.weak_local_grad(u)
    fm = np.array([disc.face_mass(flux[j]) for j in range(disc.dim)])
    return -disc.inverse_mass(wg - fm)


def div_operator(disc, v, flux):
    """mirgecom/operators.py:66-95.  v: (Nc, d, E, Np); flux: (Nc, E, Nf, Nfp)."""
    return -disc.inverse_mass(disc.weak_local_div(v) - disc.face_mass(flux))


def scalar_gradient(disc, u, exact):
    """Weak gradient of a scalar with the central flux on interior faces and
    the exact value *exact(x)* on boundary faces (the set-up of
    test/test_operators.py:208-228 and :330-417)."""
    nrm = _face_normals(disc)
    avg = ph.num_flux_central(disc.to_faces(u), disc.exterior(u))
    flux = np.array([avg * nrm[j] for j in range(disc.dim)])
    flux = flux * disc.interior_mask[None, :, :, None]
    be, bf = disc.bface_elem, disc.bface_face
    xb = disc.nodes[:, be[:, None], disc.refel.face_nodes[bf]]
    ub = exact(xb)                                        # (nbf, Nfp)
    bn = _bnormals(disc)
    mask = np.ones(len(be), dtype=bool)
    for j in range(disc.dim):
        flux[j] = flux[j] + _scatter_boundary(disc, ub * bn[j], flux[j].shape, mask)
    return grad_operator(disc, u, flux)


# {{{ boundaries (mirgecom/boundary.py)

class DummyBoundary:
    """mirgecom/boundary.py:1012-1049: exterior state = interior state."""


class PrescribedBoundary:
    """mirgecom/boundary.py:796-1009 with the default helpers: the callback
    returns the exterior conserved state (and, for mixtures, temperature) at
    the boundary face nodes, ``func(nodes (d, nbf, Nfp), time) -> q or (q, T)``.
    """

    def __init__(self, func):
        self.func = func


# {{{ Mengaldo boundaries

def _internal_energy(gas, t, y):
    """eos.get_internal_energy: mass-specific internal energy at T (and Y)
    (mirgecom/eos.py:459-470 ideal, :690-700 mixture)."""
    if isinstance(gas, ph.IdealGas):
        return gas.gas_const / (gas.gamma - 1.0) * t
    return ph.mixture_e_mass(gas.mech, t, y)


def _gas_const(gas, y):
    if isinstance(gas, ph.IdealGas):
        return gas.gas_const
    return ph.mixture_gas_const(gas.mech, y)


def _replace_state(sm, gas, transport, dim, energy=None, momentum=None):
    """mirgecom/gas_model.py:907-997 (replace_fluid_state): the interior
    state's conserved variables with *energy* / *momentum* replaced, its
    temperature re-solved from the interior temperature."""
    q = sm["cv"].copy()
    if energy is not None:
        q[1] = energy
    if momentum is not None:
        q[2:2 + dim] = momentum
    seed = sm["temperature"] if isinstance(gas, ph.MixtureGas) else None
    return ph.make_fluid_state(q, gas, transport, dim, temperature_seed=seed)


def _dot(a, b):
    return np.sum(a * b, axis=0)


def _grad_species_impermeable(sm, gcv, nb, dim):
    """mirgecom/boundary.py:187-204: the species mass fractions' normal
    gradient removed, grad(rho Y)_bc = rho grad(Y)_bc + Y grad(rho)."""
    q = sm["cv"]
    rho = q[0]
    ns = q.shape[0] - 2 - dim
    out = gcv[2 + dim:].copy()
    for k in range(ns):
        y = q[2 + dim + k] / rho
        gy = (gcv[2 + dim + k] - y * gcv[0]) / rho          # fluid.py:400-427
        gy_bc = gy - _dot(gy, nb) * nb
        out[k] = rho * gy_bc + y * gcv[0]
    return out


def _grad_velocity_slip(sm, gcv, nb, dim):
    """mirgecom/boundary.py:156-172: the velocity gradient rotated into the
    boundary frame (normal, tangents), the tangential velocities' normal
    derivatives zeroed, rotated back.  Written as the equivalent projection
    G - (I - n n^T) G n n^T, G[i][j] = d v_i / d x_j: the reference's
    frame (boundary.py:75-117) divides by the normal's z component, which
    vanishes on x and y walls in 3-D; the projection is the same tensor
    wherever that frame is defined (tests/test_mengaldo_oracle.py)."""
    q = sm["cv"]
    rho = q[0]
    v = q[2:2 + dim] / rho
    g = (gcv[2:2 + dim] - v[:, None] * gcv[0][None]) / rho    # fluid.py:355-397
    gn = np.einsum("ij...,j...->i...", g, nb)                 # G n
    tang = gn - _dot(gn, nb) * nb                             # (I - n n^T) G n
    return g - tang[:, None] * nb[None, :]


class MengaldoBoundary:
    """mirgecom/boundary.py:391-793.  Inviscid flux: the numerical flux
    between the interior state and :meth:`state_plus`; gradient fluxes:
    state_bc.cv (x) n and temperature_bc n (:732-793); viscous flux:
    F_V(state_bc, grad_cv_bc, grad_t_bc) . n (:654-730, not the central
    flux).  States are functions of the interior boundary state *sm*, the
    normals *nb* (dim, nbf, 1) and the gas."""

    def state_plus(self, sm, gas, tr, nb, dim):
        raise NotImplementedError

    def state_bc(self, sm, gas, tr, nb, dim):
        raise NotImplementedError

    def temperature_bc(self, sm):
        return sm["temperature"]

    def grad_cv_bc(self, sm, sbc, gcv, nb, dim):
        return gcv

    def grad_t_bc(self, gt, nb):
        return gt


class AdiabaticSlipBoundary(MengaldoBoundary):
    """mirgecom/boundary.py:1052-1143 with the slip, impermeable and
    adiabatic components (:149-204)."""

    def state_plus(self, sm, gas, tr, nb, dim):
        m = sm["cv"][2:2 + dim]
        return _replace_state(sm, gas, tr, dim, momentum=m - 2.0 * _dot(m, nb) * nb)

    def state_bc(self, sm, gas, tr, nb, dim):
        q = sm["cv"]
        m = q[2:2 + dim]
        m_bc = m - _dot(m, nb) * nb
        rho_e = q[1] - 0.5 * _dot(m, m) / q[0]                 # eos.internal_energy
        return _replace_state(sm, gas, tr, dim, energy=rho_e + 0.5 * _dot(m_bc, m_bc) / q[0],
                              momentum=m_bc)

    def grad_cv_bc(self, sm, sbc, gcv, nb, dim):
        gv_bc = _grad_velocity_slip(sm, gcv, nb, dim)
        v_bc = sbc["cv"][2:2 + dim] / sbc["cv"][0]
        out = gcv.copy()
        out[2:2 + dim] = sbc["cv"][0] * gv_bc + v_bc[:, None] * gcv[0][None]
        out[2 + dim:] = _grad_species_impermeable(sm, gcv, nb, dim)
        return out

    def grad_t_bc(self, gt, nb):
        return gt - _dot(gt, nb) * nb


class AdiabaticNoslipWallBoundary(MengaldoBoundary):
    """mirgecom/boundary.py:1794-1858."""

    def state_plus(self, sm, gas, tr, nb, dim):
        return _replace_state(sm, gas, tr, dim, momentum=-sm["cv"][2:2 + dim])

    def _t_wall(self, sm):
        return sm["temperature"]

    def state_bc(self, sm, gas, tr, nb, dim):
        q = sm["cv"]
        y = q[2 + dim:] / q[0]
        e_bc = q[0] * _internal_energy(gas, self._t_wall(sm), y)
        return _replace_state(sm, gas, tr, dim, energy=e_bc, momentum=0.0 * q[2:2 + dim])

    def temperature_bc(self, sm):
        return self._t_wall(sm)

    def grad_cv_bc(self, sm, sbc, gcv, nb, dim):
        out = gcv.copy()
        out[2 + dim:] = _grad_species_impermeable(sm, gcv, nb, dim)
        return out

    def grad_t_bc(self, gt, nb):
        return gt - _dot(gt, nb) * nb


class IsothermalWallBoundary(AdiabaticNoslipWallBoundary):
    """mirgecom/boundary.py:1727-1792."""

    def __init__(self, wall_temperature=300.0):
        self.wall_temperature = wall_temperature

    def _t_wall(self, sm):
        return np.zeros_like(sm["temperature"]) + self.wall_temperature

    def grad_t_bc(self, gt, nb):
        return gt


class FarfieldBoundary(MengaldoBoundary):
    """mirgecom/boundary.py:1146-1228: both states are the free stream."""

    def __init__(self, free_stream_pressure, free_stream_velocity, free_stream_temperature,
                 free_stream_mass_fractions=None):
        self.p = free_stream_pressure
        self.v = np.asarray(free_stream_velocity, dtype=np.float64)
        self.t = free_stream_temperature
        self.y = (None if free_stream_mass_fractions is None
                  else np.asarray(free_stream_mass_fractions, dtype=np.float64))

    def state_plus(self, sm, gas, tr, nb, dim):
        shape = sm["cv"][0].shape
        ns = sm["cv"].shape[0] - 2 - dim
        t = np.zeros(shape) + self.t
        y = (np.zeros((ns,) + shape) + self.y.reshape((-1,) + (1,) * len(shape))
             if ns else np.zeros((0,) + shape))
        rho = self.p / (_gas_const(gas, y) * t)
        v = np.zeros((dim,) + shape) + self.v.reshape((-1,) + (1,) * len(shape))
        e = _internal_energy(gas, t, y)
        q = np.concatenate([rho[None], (rho * (e + 0.5 * _dot(v, v)))[None], rho * v, rho * y])
        seed = t if isinstance(gas, ph.MixtureGas) else None
        return ph.make_fluid_state(q, gas, tr, dim, temperature_seed=seed)

    def state_bc(self, sm, gas, tr, nb, dim):
        return self.state_plus(sm, gas, tr, nb, dim)

    def temperature_bc(self, sm):
        return np.zeros_like(sm["temperature"]) + self.t


class PressureOutflowBoundary(MengaldoBoundary):
    """mirgecom/boundary.py:1231-1403: mass, momentum and species from the
    interior; the energy from the prescribed pressure where the outflow is
    subsonic (|v . n| <= c), from the interior where it is supersonic."""

    def __init__(self, boundary_pressure=101325.0):
        self.p = boundary_pressure

    def _state(self, sm, gas, tr, nb, dim, pressure_plus):
        q = sm["cv"]
        rho = q[0]
        m = q[2:2 + dim]
        v = m / rho
        vn = _dot(v, nb)
        speed = np.sqrt(_dot(vn * nb, vn * nb))
        ke = 0.5 * _dot(m, m) / rho
        supersonic = speed > sm["speed_of_sound"]
        if isinstance(gas, ph.MixtureGas):
            y = q[2 + dim:] / rho
            t_plus = np.where(supersonic, sm["temperature"],
                              pressure_plus / (rho * _gas_const(gas, y)))
            rho_e = rho * _internal_energy(gas, t_plus, y)
        else:
            pb = np.where(supersonic, sm["pressure"], pressure_plus)
            rho_e = pb / (sm["gamma"] - 1.0)
        return _replace_state(sm, gas, tr, dim, energy=rho_e + ke)

    def state_plus(self, sm, gas, tr, nb, dim):
        p_plus = np.where(sm["pressure"] > 2.0 * self.p, sm["pressure"],
                          2.0 * self.p - sm["pressure"])
        return self._state(sm, gas, tr, nb, dim, p_plus)

    def state_bc(self, sm, gas, tr, nb, dim):
        return self._state(sm, gas, tr, nb, dim, self.p + 0.0 * sm["pressure"])

# }}}


def _normalize_boundaries(boundaries):
    return boundaries or {}


def _bface_selection(disc, tag):
    """Boundary faces under *tag*: "all", or "-k"/"+k" for the low/high box
    side along axis k."""
    if tag in ("all", None):
        return np.ones(len(disc.bface_elem), dtype=bool)
    axis = int(tag[1:])
    val = disc.mesh.a[axis] if tag[0] == "-" else disc.mesh.b[axis]
    fverts = disc.mesh.vertex_coords[disc.bface_elem[:, None],
                                     np.array(disc.refel.face_vertices)[disc.bface_face]]
    return np.all(np.abs(fverts[:, :, axis] - val) < 1e-12, axis=1)

# }}}


def _face_normals(disc):
    return np.moveaxis(disc.normals, 2, 0)[:, :, :, None]      # (d, E, Nf, 1)


def make_operator_fluid_states(disc, state, gas, transport, boundaries, time):
    """mirgecom/gas_model.py:728-904 on the base discretization."""
    dim = disc.dim
    q = state["cv"]
    is_mix = isinstance(gas, ph.MixtureGas)
    tseed_vol = state["temperature"] if is_mix else None
    vol = ph.make_fluid_state(q, gas, transport, dim, temperature_seed=tseed_vol)
    q_m = disc.to_faces(q)
    q_p = disc.exterior(q)
    ts_m = disc.to_faces(tseed_vol) if is_mix else None
    ts_p = disc.exterior(tseed_vol) if is_mix else None
    st_m = ph.make_fluid_state(q_m, gas, transport, dim, temperature_seed=ts_m)
    st_p = ph.make_fluid_state(q_p, gas, transport, dim, temperature_seed=ts_p)
    # boundary states: minus side and the prescribed/dummy plus side
    bst = {}
    for tag, bdry in _normalize_boundaries(boundaries).items():
        be, bf = disc.bface_elem, disc.bface_face
        fnodes = disc.refel.face_nodes[bf]
        qb = q[:, be[:, None], fnodes]                              # (Nc, nbf, Nfp)
        tb = tseed_vol[be[:, None], fnodes] if is_mix else None
        sm = ph.make_fluid_state(qb, gas, transport, dim, temperature_seed=tb)
        if isinstance(bdry, DummyBoundary):
            sp = sm
        elif isinstance(bdry, MengaldoBoundary):
            nb = _bnormals(disc)
            sp = bdry.state_plus(sm, gas, transport, nb, dim)
            sp["bc"] = bdry.state_bc(sm, gas, transport, nb, dim)
            sp["temperature_bc"] = bdry.temperature_bc(sm)
        else:
            xb = disc.nodes[:, be[:, None], fnodes]
            ext = bdry.func(xb, time)
            if is_mix:
                qe, te = ext
                sp = ph.make_fluid_state(qe, gas, transport, dim, temperature_seed=te)
            else:
                sp = ph.make_fluid_state(ext, gas, transport, dim)
        bst[tag] = (bdry, sm, sp, _bface_selection(disc, tag))
    return vol, (st_m, st_p), bst


def _scatter_boundary(disc, values, shape, mask):
    """Boundary-face values (..., nbf, Nfp) -> all-faces array (op.project)."""
    out = np.zeros(shape)
    out[..., disc.bface_elem[mask], disc.bface_face[mask], :] = values[..., mask, :]
    return out


def _bnormals(disc):
    n = disc.normals[disc.bface_elem, disc.bface_face]     # (nbf, d)
    return n.T[:, :, None]                                   # (d, nbf, 1)


def inviscid_flux_on_element_boundary(disc, ostates, flux_name):
    """mirgecom/inviscid.py:290-376."""
    _, (st_m, st_p), bst = ostates
    num_flux = ph.INVISCID_FLUXES[flux_name]
    nrm = _face_normals(disc)
    fint = num_flux(st_m, st_p, nrm)
    fint = fint * disc.interior_mask[None, :, :, None]
    for tag, (bdry, sm, sp, mask) in bst.items():
        bn = _bnormals(disc)
        if isinstance(bdry, DummyBoundary):
            fb = ph.dot_normal(ph.inviscid_flux(sm), bn)        # boundary.py:1027
        else:
            fb = num_flux(sm, sp, bn)                            # boundary.py:929-944
        fint = fint + _scatter_boundary(disc, fb, fint.shape, mask)
    return fint


def euler_operator(disc, state, gas, boundaries, time=0.0, flux="rusanov",
                   operator_states=None):
    """mirgecom/euler.py:313-416 (non-ESDG branch)."""
    ostates = operator_states or make_operator_fluid_states(
        disc, state, gas, None, boundaries, time)
    vol = ostates[0]
    fvol = ph.inviscid_flux(vol)
    fbnd = inviscid_flux_on_element_boundary(disc, ostates, flux)
    return -div_operator(disc, fvol, fbnd)


def _grad_flux_interior(disc, u_m, u_p):
    """mirgecom/navierstokes.py:118-126: outer(central(u-, u+), n)."""
    nrm = _face_normals(disc)
    avg = ph.num_flux_central(u_m, u_p)
    return np.array([avg * nrm[j] for j in range(disc.dim)])    # (d, ..., E, Nf, Nfp)


def grad_cv_operator(disc, ostates, time=0.0):
    """mirgecom/navierstokes.py:129-235; returns (Nc, d, E, Np)."""
    vol, (st_m, st_p), bst = ostates
    flux = _grad_flux_interior(disc, st_m["cv"], st_p["cv"])
    flux = flux * disc.interior_mask[None, None, :, :, None]
    bn = _bnormals(disc)
    for tag, (bdry, sm, sp, mask) in bst.items():
        if isinstance(bdry, DummyBoundary):
            fb = np.array([sm["cv"] * bn[j] for j in range(disc.dim)])   # :1031
        elif isinstance(bdry, MengaldoBoundary):
            fb = np.array([sp["bc"]["cv"] * bn[j] for j in range(disc.dim)])  # :732-760
        else:
            fb = np.array([sp["cv"] * bn[j] for j in range(disc.dim)])   # :895-907
        flux = flux + _scatter_boundary(disc, fb, flux.shape, mask)
    g = grad_operator(disc, vol["cv"], flux)                  # (d, Nc, E, Np)
    return np.swapaxes(g, 0, 1)


def grad_t_operator(disc, ostates, time=0.0):
    """mirgecom/navierstokes.py:238-347; returns (d, E, Np)."""
    vol, (st_m, st_p), bst = ostates
    flux = _grad_flux_interior(disc, st_m["temperature"], st_p["temperature"])
    flux = flux * disc.interior_mask[None, :, :, None]
    bn = _bnormals(disc)
    for tag, (bdry, sm, sp, mask) in bst.items():
        if isinstance(bdry, DummyBoundary):
            tb = sm["temperature"]
        elif isinstance(bdry, MengaldoBoundary):
            tb = sp["temperature_bc"]                                     # :762-793
        else:
            tb = sp["temperature"]
        fb = np.array([tb * bn[j] for j in range(disc.dim)])
        flux = flux + _scatter_boundary(disc, fb, flux.shape, mask)
    return grad_operator(disc, vol["temperature"], flux)


def viscous_flux_on_element_boundary(disc, ostates, grad_cv, grad_t):
    """mirgecom/viscous.py:431-544 with the central numerical flux."""
    vol, (st_m, st_p), bst = ostates
    nrm = _face_normals(disc)
    gcv_m = disc.to_faces(grad_cv)
    gcv_p = disc.exterior(grad_cv)
    gt_m = disc.to_faces(grad_t)
    gt_p = disc.exterior(grad_t)
    f = ph.viscous_facial_flux_central(st_m, st_p, gcv_m, gcv_p, gt_m, gt_p, nrm)
    f = f * disc.interior_mask[None, :, :, None]
    bn = _bnormals(disc)
    be, bf = disc.bface_elem, disc.bface_face
    fnodes = disc.refel.face_nodes[bf]
    gcv_b = grad_cv[:, :, be[:, None], fnodes]
    gt_b = grad_t[:, be[:, None], fnodes]
    for tag, (bdry, sm, sp, mask) in bst.items():
        if isinstance(bdry, DummyBoundary):
            fb = ph.dot_normal(ph.viscous_flux(sm, gcv_b, gt_b), bn)     # :1047
        elif isinstance(bdry, MengaldoBoundary):
            # F_V(state_bc, grad_cv_bc, grad_t_bc) . n (boundary.py:654-730)
            sbc = sp["bc"]
            gcv_bc = bdry.grad_cv_bc(sm, sbc, gcv_b, bn, disc.dim)
            gt_bc = bdry.grad_t_bc(gt_b, bn)
            fb = ph.dot_normal(ph.viscous_flux(sbc, gcv_bc, gt_bc), bn)
        else:
            # central flux, exterior gradients = interior (boundary.py:141-146)
            fb = ph.viscous_facial_flux_central(sm, sp, gcv_b, gcv_b, gt_b, gt_b, bn)
        f = f + _scatter_boundary(disc, fb, f.shape, mask)
    return f


def ns_operator(disc, state, gas, transport, boundaries, time=0.0,
                flux="rusanov", return_gradients=False):
    """mirgecom/navierstokes.py:350-575 (default, fused inviscid branch)."""
    ostates = make_operator_fluid_states(disc, state, gas, transport, boundaries, time)
    vol = ostates[0]
    grad_cv = grad_cv_operator(disc, ostates, time)
    grad_t = grad_t_operator(disc, ostates, time)
    vol_term = ph.viscous_flux(vol, grad_cv, grad_t)
    bnd_term = viscous_flux_on_element_boundary(disc, ostates, grad_cv, grad_t)
    vol_term = vol_term - ph.inviscid_flux(vol)
    bnd_term = bnd_term - inviscid_flux_on_element_boundary(disc, ostates, flux)
    rhs = div_operator(disc, vol_term, bnd_term)
    if return_gradients:
        return rhs, grad_cv, grad_t
    return rhs


def rk4_step(q, t, dt, rhs):
    """mirgecom/integrators/explicit_rk.py:31-37."""
    k1 = rhs(t, q)
    k2 = rhs(t + dt / 2, q + dt / 2 * k1)
    k3 = rhs(t + dt / 2, q + dt / 2 * k2)
    k4 = rhs(t + dt, q + dt * k3)
    return q + dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4)


# {{{ time-step estimates (mirgecom/inviscid.py:379-422, viscous.py:547-607)

def characteristic_lengthscales(od):
    """grudge's ``dt_utils.characteristic_lengthscales`` restated (grudge is
    not installed; Hesthaven & Warburton 2008, sec. 6.4): h = min(dr) r_D with
    min(dr) the smallest distance between two reference-element nodes and
    r_D = d V / sum_f F_f the inradius, here from the element's vertices
    (volume from the vertex Jacobian, face areas from the face vertices)."""
    nodes = od.refel.nodes
    n = nodes.shape[1]
    min_dr = min(float(np.linalg.norm(nodes[:, i] - nodes[:, j]))
                 for i in range(n) for j in range(i + 1, n))
    vol = np.abs(od.jac_det) * od.refel.ref_volume
    areas = od.face_area_ratio * od.refel.face_param_area
    r_d = od.dim * vol / areas.sum(axis=1)
    return np.repeat((min_dr * r_d)[:, None], n, axis=1)


def inviscid_timestep(od, st):
    return characteristic_lengthscales(od) / ph.wavespeed(st)


def viscous_timestep(od, st):
    h = characteristic_lengthscales(od)
    nu = st["mu"] / st["cv"][0] if "mu" in st else 0.0
    dmax = st["diff"].max(axis=0) if "diff" in st and len(st["diff"]) else 0.0
    return h / (ph.wavespeed(st) + (nu + dmax) / h)

# }}}
