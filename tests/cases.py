"""Matched product / oracle set-ups for the parity tests."""

from __future__ import annotations

import math

import numpy as np
import torch

from mirgecom_b200.discretization import Discretization
from mirgecom_b200.mesh import generate_box_mesh
from oracle import dg as odg
from oracle import physics as oph


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def field_errors(a, b, floor=None):
    """Per-field relative L2 errors (fields along axis 0), two ways.

    Returns (own, floored): *own* divides by each field's own norm; *floored*
    divides by the larger of that norm and ``floor[c]``, the field's natural
    physical scale (|q_c|/h for a gradient, |F_c|/h for a divergence: see
    :func:`flux_scale_floor`), for fields whose value is a small difference of
    large fluxes (low-Mach momentum, a uniform density's gradient).  Without
    *floor* the two are equal."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    own, fl = [], []
    for c in range(b.shape[0]):
        err = np.linalg.norm((a[c] - b[c]).ravel())
        nb = np.linalg.norm(b[c].ravel())
        own.append(float(err / max(nb, 1e-300)))
        f = 0.0 if floor is None else float(floor[c])
        fl.append(float(err / max(nb, f, 1e-300)))
    return own, fl


def field_rel_l2(a, b, floor=None):
    """Largest per-field relative L2 error, each field against the larger of
    its own norm and its natural scale ``floor[c]`` (no floor by default)."""
    return max(field_errors(a, b, floor)[1])


def assert_fields_close(a, b, tol, floor=None, what="field"):
    """Every field within *tol* (against its own norm, or its natural scale
    where *floor* is given); the message lists both errors per field."""
    own, fl = field_errors(a, b, floor)
    bad = [c for c in range(len(fl)) if not fl[c] < tol]
    msg = "; ".join(f"{what} {c}: own {own[c]:.2e} scaled {fl[c]:.2e}" for c in range(len(fl)))
    assert not bad, f"fields {bad} above {tol:g}: {msg}"


def make_disc(kind, dim, n, order, lo, hi, periodic):
    mesh = generate_box_mesh(lo, hi, (n,) * dim, kind=kind, periodic=(periodic,) * dim
                             if isinstance(periodic, bool) else periodic)
    d = Discretization(mesh, order)
    od = odg.OracleDisc(mesh, d.refel)
    return d, od


def vortex_np(x, t=0.0, beta=5.0, center=(5.0, 0.0), vel=(1.0, 0.0), gamma=1.4):
    xr = x[0] - center[0] - t * vel[0]
    yr = x[1] - center[1] - t * vel[1]
    r = np.sqrt(xr ** 2 + yr ** 2)
    ex = beta * np.exp(1 - r ** 2)
    u = vel[0] - ex * yr / (2 * np.pi)
    v = vel[1] + ex * xr / (2 * np.pi)
    rho = (1 - (gamma - 1) / (16 * gamma * np.pi ** 2) * ex ** 2) ** (1 / (gamma - 1))
    p = rho ** gamma
    return np.array([rho, p / (gamma - 1) + rho / 2 * (u ** 2 + v ** 2), rho * u, rho * v])


def tgv_np(x, gamma=1.4, mach=0.1):
    u = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
    v = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    w = np.zeros_like(u)
    p0 = 1.0 / (gamma * mach ** 2)
    p = p0 + 1.0 / 16 * (np.cos(2 * x[0]) + np.cos(2 * x[1])) * (np.cos(2 * x[2]) + 2)
    rho = np.ones_like(u)
    return np.array([rho, p / (gamma - 1) + 0.5 * (u * u + v * v), u, v, w])


def perturbed_state_np(x, dim, nspecies, seed=0):
    """Smooth non-uniform ideal-gas state with passive species."""
    rng = np.random.default_rng(seed)
    k = rng.uniform(0.5, 1.5, size=(6, dim))
    ph = rng.uniform(0, 2 * np.pi, size=6)
    def f(i):
        return np.cos(sum(k[i, d] * x[d] for d in range(dim)) + ph[i])
    rho = 1.0 + 0.2 * f(0)
    vel = [0.3 * f(1 + (j % 3)) for j in range(dim)]
    p = 1.0 + 0.1 * f(4)
    e = p / 0.4 + 0.5 * rho * sum(v * v for v in vel)
    q = [rho, e] + [rho * v for v in vel]
    for s in range(nspecies):
        q.append(rho * (0.1 + 0.05 * (s + 1) * (1 + f(5))))
    return np.array(q)


def per_field_rel_l2(a, b, floor=None):
    """Per-field relative L2 errors (same normalisation as field_rel_l2)."""
    return field_errors(a, b, floor)[1]


def flux_scale_floor(q, dim, h, gamma=1.4):
    """Per-field natural scale of a divergence of the ideal-gas inviscid
    flux: |F_c| / h (for low-Mach states the RHS is orders of magnitude
    below its fluxes and roundoff scales with the fluxes)."""
    from oracle import physics as oph
    st = oph.make_fluid_state(q, oph.IdealGas(gamma=gamma), None, dim)
    return state_flux_floor(st, h)


def state_flux_floor(st, h):
    """|F_c| / h per conserved field for an oracle fluid state *st* (any gas:
    ideal or mixture), F the inviscid flux."""
    from oracle import physics as oph
    f = oph.inviscid_flux(st)
    return [np.linalg.norm(f[c]) / h for c in range(f.shape[0])]


def gradient_floor(q, h):
    """|q_c| / h per field: the natural scale of a gradient of q_c."""
    q = np.asarray(q)
    return [np.linalg.norm(q[c]) / h for c in range(q.shape[0])]


def inviscid_flux_floor(q, dim, h, temperature=None, mech=None, gamma=1.4):
    """|F_c| / h per conserved field from the state alone (numpy, no
    oracle): F the inviscid flux, the pressure of the ideal gas (gamma) or,
    with *temperature* and *mech*, of the mixture (p = rho R_u T sum Y_k/W_k)."""
    q = np.asarray(q, dtype=np.float64)
    rho = q[0]
    v = q[2:2 + dim] / rho
    if mech is None:
        p = (gamma - 1) * (q[1] - 0.5 * np.sum(q[2:2 + dim] * v, axis=0))
    else:
        from mirgecom_b200.thermochemistry import GAS_CONSTANT
        w = np.asarray(mech.molecular_weights).reshape((-1,) + (1,) * (q.ndim - 1))
        p = GAS_CONSTANT * np.asarray(temperature) * np.sum(q[2 + dim:] / w, axis=0)
    out = [np.linalg.norm(q[0] * v), np.linalg.norm((q[1] + p) * v)]
    for i in range(dim):
        fi = q[2 + i] * v
        fi[i] = fi[i] + p
        out.append(np.linalg.norm(fi))
    for k in range(q.shape[0] - 2 - dim):
        out.append(np.linalg.norm(q[2 + dim + k] * v))
    return [x / h for x in out]
