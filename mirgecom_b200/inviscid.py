"""Inviscid facial fluxes, mirroring mirgecom/inviscid.py:105-287.

Each function is the selector the operators pass to the device kernels
(``.flux_kind``); calling one evaluates the flux pointwise on a pair of
:class:`~mirgecom_b200.gas_model.FluidState` objects with torch ops.
"""

from __future__ import annotations

import torch

from mirgecom_b200 import _lib
from mirgecom_b200.flux import num_flux_hll, num_flux_lfr


def inviscid_flux(state):
    """mirgecom/inviscid.py:65-102 as a tensor (Nc, dim, ...)."""
    cv = state.cv
    d = cv.dim
    v = cv.velocity
    p = state.pressure
    rows = [cv.momentum, v * (cv.energy + p)]
    for i in range(d):
        row = cv.mass * v[i] * v
        row[i] = row[i] + p
        rows.append(row)
    for k in range(cv.nspecies):
        rows.append(v * cv.species_mass[k])
    return torch.stack([torch.as_tensor(r) for r in rows])


def _dot_n(f, normal):
    return (f * normal[None]).sum(dim=1)


def _gamma(eos, state):
    if state.is_mixture:
        return eos.gamma(state.cv, state.temperature)
    return eos.gamma()


def inviscid_facial_flux_rusanov(state_pair, gas_model=None, normal=None):
    sm, sp = state_pair
    lam = torch.maximum(sm.wavespeed, sp.wavespeed)
    return num_flux_lfr(_dot_n(inviscid_flux(sm), normal), _dot_n(inviscid_flux(sp), normal),
                        sm.cv.q, sp.cv.q, lam)


def inviscid_facial_flux_central(state_pair, gas_model=None, normal=None):
    sm, sp = state_pair
    return num_flux_lfr(_dot_n(inviscid_flux(sm), normal), _dot_n(inviscid_flux(sp), normal),
                        sm.cv.q, sp.cv.q, 0)


def inviscid_facial_flux_hll(state_pair, gas_model=None, normal=None):
    sm, sp = state_pair
    eos = (gas_model or sm.gas_model).eos
    p_int, p_ext = sm.pressure, sp.pressure
    u_int = (sm.velocity * normal).sum(dim=0)
    u_ext = (sp.velocity * normal).sum(dim=0)
    rho_int, rho_ext = sm.cv.mass, sp.cv.mass
    c_int, c_ext = sm.speed_of_sound, sp.speed_of_sound
    p_star = (0.5 * (p_int + p_ext) + (1. / 8.) * (u_int - u_ext)
              * (rho_int + rho_ext) * (c_int + c_ext))
    g_int, g_ext = _gamma(eos, sm), _gamma(eos, sp)
    q_int = 1 + (g_int + 1) / (2 * g_int) * (p_star / p_int - 1)
    q_ext = 1 + (g_ext + 1) / (2 * g_ext) * (p_star / p_ext - 1)
    q_int_rt = torch.where(p_star > p_int, q_int, torch.ones_like(q_int)).sqrt()
    q_ext_rt = torch.where(p_star > p_ext, q_ext, torch.ones_like(q_ext)).sqrt()
    s_minus = u_int - c_int * q_int_rt
    s_plus = u_ext + c_ext * q_ext_rt
    return num_flux_hll(_dot_n(inviscid_flux(sm), normal), _dot_n(inviscid_flux(sp), normal),
                        sm.cv.q, sp.cv.q, s_minus, s_plus)


inviscid_facial_flux_rusanov.flux_kind = _lib.FLUX_RUSANOV
inviscid_facial_flux_hll.flux_kind = _lib.FLUX_HLL
inviscid_facial_flux_central.flux_kind = _lib.FLUX_CENTRAL


def flux_kind_of(func):
    kind = getattr(func, "flux_kind", None)
    if kind is None:
        raise NotImplementedError(
            f"{func!r} is not a device-supported inviscid numerical flux; use "
            "inviscid_facial_flux_rusanov, _hll or _central")
    return kind


def get_inviscid_timestep(dcoll, state, dd=None):
    """Node-local stable time step of an inviscid fluid, h / (|v| + c)
    (mirgecom/inviscid.py:379-422), h the characteristic length scale of
    :meth:`~mirgecom_b200.discretization.Discretization.characteristic_lengthscales`.
    Returns a tensor shaped like the state's fields (E, Np)."""
    if dd is not None and dd != "vol":
        raise TypeError("dd must represent the volume")
    ws = state.wavespeed
    h = dcoll.characteristic_lengthscales(device=ws.device, dtype=ws.dtype)
    return h / ws
