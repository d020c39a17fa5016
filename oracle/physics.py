"""Pointwise physics of the oracle (float64 numpy).  Test infrastructure only.

Conserved variables are arrays ``q[Nc, ...]`` in the reference's field order
[mass, energy, momentum[dim], species_mass[nspecies]]
(mirgecom/fluid.py:300-312).  Flux vectors are ``f[Nc, dim, ...]``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GAS_CONSTANT = 8314.46261815324
ONE_ATM = 101325.0


# {{{ gas models

@dataclass
class IdealGas:
    """mirgecom/eos.py:302-537 (IdealSingleGas)."""
    gamma: float = 1.4
    gas_const: float = 287.1


@dataclass
class MixtureGas:
    """mirgecom/eos.py:540-888 (PyrometheusMixture) with the pyrometheus
    wrapper of mirgecom/thermochemistry.py:51-183."""
    mech: object                 # mirgecom_b200.thermochemistry.Mechanism data
    temperature_niter: int = 5
    zero_level: float = 0.0


@dataclass
class SimpleTransportParams:
    """mirgecom/transport.py:143-202."""
    viscosity: float = 0.0
    bulk_viscosity: float = 0.0
    thermal_conductivity: float = 0.0
    species_diffusivity: tuple = ()


@dataclass
class PowerLawTransportParams:
    """mirgecom/transport.py:205-321."""
    alpha: float = 0.6
    beta: float = 4.093e-7
    sigma: float = 2.5
    n: float = 0.666
    species_diffusivity: tuple = ()
    lewis: tuple | None = None

# }}}


def split(q, dim):
    rho = q[0]
    rhoe = q[1]
    mom = q[2:2 + dim]
    rhoy = q[2 + dim:]
    return rho, rhoe, mom, rhoy


# {{{ NASA-7 / pyrometheus-style thermochemistry

def _nasa(mech, temperature):
    """Coefficients per species selected by range, shape (Ns, 7, ...)."""
    t = np.asarray(temperature)
    hi = t[None] > mech.t_mid.reshape((-1,) + (1,) * t.ndim)
    lo_c = mech.nasa_low.reshape(mech.nasa_low.shape + (1,) * t.ndim)
    hi_c = mech.nasa_high.reshape(mech.nasa_high.shape + (1,) * t.ndim)
    return np.where(hi[:, None], hi_c, lo_c)


def species_cp_r(mech, t):
    a = _nasa(mech, t)
    return a[:, 0] + a[:, 1] * t + a[:, 2] * t**2 + a[:, 3] * t**3 + a[:, 4] * t**4


def species_h_rt(mech, t):
    a = _nasa(mech, t)
    return (a[:, 0] + a[:, 1] / 2 * t + a[:, 2] / 3 * t**2 + a[:, 3] / 4 * t**3
            + a[:, 4] / 5 * t**4 + a[:, 5] / t)


def species_s_r(mech, t):
    a = _nasa(mech, t)
    return (a[:, 0] * np.log(t) + a[:, 1] * t + a[:, 2] / 2 * t**2
            + a[:, 3] / 3 * t**3 + a[:, 4] / 4 * t**4 + a[:, 6])


def _wcol(mech, ndim):
    return mech.molecular_weights.reshape((-1,) + (1,) * ndim)


def mixture_gas_const(mech, y):
    return GAS_CONSTANT * np.sum(y / _wcol(mech, y.ndim - 1), axis=0)


def mixture_cp_mass(mech, t, y):
    return GAS_CONSTANT * np.sum(y * species_cp_r(mech, t) / _wcol(mech, y.ndim - 1), axis=0)


def mixture_cv_mass(mech, t, y):
    return GAS_CONSTANT * np.sum(y * (species_cp_r(mech, t) - 1.0)
                                 / _wcol(mech, y.ndim - 1), axis=0)


def mixture_e_mass(mech, t, y):
    return GAS_CONSTANT * t * np.sum(y * (species_h_rt(mech, t) - 1.0)
                                     / _wcol(mech, y.ndim - 1), axis=0)


def newton_temperature(mech, e, t_guess, y, niter):
    """Fixed-count Newton, mirgecom/thermochemistry.py:99-102,126-167."""
    t = t_guess
    for _ in range(niter):
        t = t + (e - mixture_e_mass(mech, t, y)) / mixture_cv_mass(mech, t, y)
    return t


def species_enthalpies(mech, t):
    """mirgecom/eos.py:733-742: (R/W_k) T (h/RT)_k."""
    return (GAS_CONSTANT / _wcol(mech, np.ndim(t))) * t * species_h_rt(mech, t)


def net_production_rates(mech, rho, t, y, zero_level=0.0):
    """Molar production rates (kmol/m^3/s), pyrometheus semantics with the
    concentration floor of mirgecom/thermochemistry.py:87-94."""
    w = _wcol(mech, np.ndim(t))
    conc = rho * y / w
    conc = np.where(conc < zero_level, 0.0, conc)
    g_rt = species_h_rt(mech, t) - species_s_r(mech, t)
    rates = []
    for i in range(mech.nreactions):
        kf = np.exp(mech.log_a[i] + mech.beta[i] * np.log(t) - mech.t_act[i] / t)
        rf = kf * np.ones_like(t)
        for k in range(mech.nspecies):
            if mech.orders_fwd[i, k] != 0:
                rf = rf * conc[k] ** mech.orders_fwd[i, k]
        r = rf
        if mech.reversible[i]:
            nu = mech.nu_prod[i] - mech.nu_reac[i]
            dg = np.tensordot(nu, g_rt, axes=(0, 0))
            log_kc = -dg + nu.sum() * np.log(ONE_ATM / (GAS_CONSTANT * t))
            rr = kf * np.exp(-log_kc)
            for k in range(mech.nspecies):
                if mech.nu_prod[i, k] != 0:
                    rr = rr * conc[k] ** mech.nu_prod[i, k]
            r = rf - rr
        rates.append(r)
    rates = np.array(rates)
    return np.tensordot(mech.nu_prod - mech.nu_reac, rates, axes=(0, 0))


def species_source_terms(gas, q, t, dim):
    """mirgecom/eos.py:858-875: W_k omega_k on the species equations."""
    mech = gas.mech
    rho, _, _, rhoy = split(q, dim)
    y = rhoy / rho
    omega = net_production_rates(mech, rho, t, y, gas.zero_level)
    src = np.zeros_like(q)
    src[2 + dim:] = _wcol(mech, np.ndim(t)) * omega
    return src

# }}}


# {{{ fluid state (mirgecom/gas_model.py:302-430)

def make_fluid_state(q, gas, transport, dim, temperature_seed=None):
    rho, rhoe, mom, rhoy = split(q, dim)
    ke = 0.5 * np.sum(mom * mom, axis=0) / rho
    st = {"cv": q, "dim": dim}
    if isinstance(gas, IdealGas):
        eint = rhoe - ke
        p = eint * (gas.gamma - 1.0)
        t = ((gas.gamma - 1.0) / gas.gas_const) * eint / rho
        c = np.sqrt(gas.gamma / rho * p)
        st.update(temperature=t, pressure=p, speed_of_sound=c,
                  gamma=gas.gamma * np.ones_like(rho),
                  cv_heat=gas.gas_const / (gas.gamma - 1.0) * np.ones_like(rho),
                  cp_heat=gas.gas_const * gas.gamma / (gas.gamma - 1.0) * np.ones_like(rho),
                  mass_fractions=rhoy / rho)
    else:
        if temperature_seed is None:
            raise ValueError("mixture temperature requires a seed")
        mech = gas.mech
        y = rhoy / rho
        e = (rhoe - ke) / rho
        tseed = temperature_seed * np.ones_like(rho)
        t = newton_temperature(mech, e, tseed, y, gas.temperature_niter)
        rmix = mixture_gas_const(mech, y)
        p = rho * rmix * t
        cp = mixture_cp_mass(mech, t, y)
        gamma = cp / (cp - rmix)
        c = np.sqrt(gamma * p / rho)
        st.update(temperature=t, pressure=p, speed_of_sound=c, gamma=gamma,
                  cp_heat=cp, cv_heat=cp - rmix, mass_fractions=y,
                  species_enthalpies=species_enthalpies(mech, t))
    if transport is not None:
        st.update(transport_vars(transport, st, gas))
    return st


def transport_vars(tr, st, gas):
    rho = st["cv"][0]
    ones = np.ones_like(rho)
    nspec = st["mass_fractions"].shape[0]
    if isinstance(tr, SimpleTransportParams):
        d = np.array(tr.species_diffusivity, dtype=np.float64).reshape(
            (-1,) + (1,) * rho.ndim) * ones
        return {"mu": tr.viscosity * ones, "mu_b": tr.bulk_viscosity * ones,
                "kappa": tr.thermal_conductivity * ones, "diff": d[:nspec]}
    if isinstance(tr, PowerLawTransportParams):
        mu = tr.beta * st["temperature"] ** tr.n
        kappa = tr.sigma * mu * st["cv_heat"]
        if tr.lewis is not None:
            le = np.array(tr.lewis).reshape((-1,) + (1,) * rho.ndim)
            d = tr.sigma * mu / (rho * le * st["gamma"])
        else:
            d = np.array(tr.species_diffusivity, dtype=np.float64).reshape(
                (-1,) + (1,) * rho.ndim) * ones
        return {"mu": mu, "mu_b": tr.alpha * mu, "kappa": kappa, "diff": d[:nspec]}
    raise TypeError(type(tr))

# }}}


# {{{ fluxes

def velocity(st):
    q = st["cv"]
    return q[2:2 + st["dim"]] / q[0]


def wavespeed(st):
    """mirgecom/gas_model.py:224-226: |v| + c."""
    v = velocity(st)
    return np.sqrt(np.sum(v * v, axis=0)) + st["speed_of_sound"]


def inviscid_flux(st):
    """mirgecom/inviscid.py:65-102."""
    q = st["cv"]
    dim = st["dim"]
    rho, rhoe, mom, rhoy = split(q, dim)
    v = mom / rho
    p = st["pressure"]
    f = np.zeros((q.shape[0], dim) + q.shape[1:])
    f[0] = mom
    f[1] = v * (rhoe + p)
    for i in range(dim):
        f[2 + i] = rho * v[i] * v
        f[2 + i, i] += p
    f[2 + dim:] = v[None] * rhoy[:, None]
    return f


def dot_normal(f, normal):
    """``flux @ normal`` with ``normal[dim, ...]``."""
    return np.sum(f * normal[None], axis=1)


def num_flux_lfr(f_minus_n, f_plus_n, q_minus, q_plus, lam):
    """mirgecom/flux.py:45-84."""
    return (f_minus_n + f_plus_n + lam * (q_minus - q_plus)) / 2


def num_flux_central(f_minus, f_plus):
    """mirgecom/flux.py:87-110."""
    return (f_plus + f_minus) / 2


def num_flux_hll(f_minus_n, f_plus_n, q_minus, q_plus, s_minus, s_plus):
    """mirgecom/flux.py:113-177."""
    f_star = (s_plus * f_minus_n - s_minus * f_plus_n
              + s_plus * s_minus * (q_plus - q_minus)) / (s_plus - s_minus)
    f = np.where(s_minus >= 0, f_minus_n, f_star)
    f = np.where(s_plus <= 0, f_plus_n, f)
    return f


def inviscid_facial_flux_rusanov(st_m, st_p, normal):
    """mirgecom/inviscid.py:105-152."""
    lam = np.maximum(wavespeed(st_m), wavespeed(st_p))
    return num_flux_lfr(dot_normal(inviscid_flux(st_m), normal),
                        dot_normal(inviscid_flux(st_p), normal),
                        st_m["cv"], st_p["cv"], lam)


def inviscid_facial_flux_central(st_m, st_p, normal):
    """mirgecom/inviscid.py:155-199."""
    return num_flux_lfr(dot_normal(inviscid_flux(st_m), normal),
                        dot_normal(inviscid_flux(st_p), normal),
                        st_m["cv"], st_p["cv"], 0.0)


def inviscid_facial_flux_hll(st_m, st_p, normal):
    """mirgecom/inviscid.py:202-287."""
    p_int = st_m["pressure"]
    p_ext = st_p["pressure"]
    u_int = np.sum(velocity(st_m) * normal, axis=0)
    u_ext = np.sum(velocity(st_p) * normal, axis=0)
    rho_int = st_m["cv"][0]
    rho_ext = st_p["cv"][0]
    c_int = st_m["speed_of_sound"]
    c_ext = st_p["speed_of_sound"]
    p_star = (0.5 * (p_int + p_ext) + (1. / 8.) * (u_int - u_ext)
              * (rho_int + rho_ext) * (c_int + c_ext))
    g_int = st_m["gamma"]
    g_ext = st_p["gamma"]
    q_int = 1 + (g_int + 1) / (2 * g_int) * (p_star / p_int - 1)
    q_ext = 1 + (g_ext + 1) / (2 * g_ext) * (p_star / p_ext - 1)
    q_int_rt = np.sqrt(np.where(p_star > p_int, q_int, 1.0))
    q_ext_rt = np.sqrt(np.where(p_star > p_ext, q_ext, 1.0))
    s_minus = u_int - c_int * q_int_rt
    s_plus = u_ext + c_ext * q_ext_rt
    return num_flux_hll(dot_normal(inviscid_flux(st_m), normal),
                        dot_normal(inviscid_flux(st_p), normal),
                        st_m["cv"], st_p["cv"], s_minus, s_plus)


INVISCID_FLUXES = {
    "rusanov": inviscid_facial_flux_rusanov,
    "hll": inviscid_facial_flux_hll,
    "central": inviscid_facial_flux_central,
}


def viscous_flux(st, grad_cv, grad_t):
    """mirgecom/viscous.py:232-293 with :72-73 (stress), :110-112 (diffusive
    flux), :158-229 (heat fluxes).  ``grad_cv[Nc, dim, ...]``,
    ``grad_t[dim, ...]``."""
    q = st["cv"]
    dim = st["dim"]
    rho, rhoe, mom, rhoy = split(q, dim)
    v = mom / rho
    # velocity_gradient, mirgecom/fluid.py:355-397
    grad_v = (grad_cv[2:2 + dim] - v[:, None] * grad_cv[0][None]) / rho
    mu = st["mu"]
    mu_b = st["mu_b"]
    div_v = sum(grad_v[i, i] for i in range(dim))
    tau = mu * (grad_v + np.swapaxes(grad_v, 0, 1))
    for i in range(dim):
        tau[i, i] = tau[i, i] + (mu_b - 2 * mu / 3) * div_v
    nspec = rhoy.shape[0]
    f = np.zeros((q.shape[0], dim) + q.shape[1:])
    # energy: tau . v - q_diffusive - q_conductive
    e_flux = np.einsum("ij...,j...->i...", tau, v)
    e_flux = e_flux + st["kappa"] * grad_t
    if nspec:
        y = rhoy / rho
        grad_y = (grad_cv[2 + dim:] - y[:, None] * grad_cv[0][None]) / rho
        d = st["diff"]
        dgy = d[:, None] * grad_y
        if "species_enthalpies" in st:
            j = -rho * (dgy - y[:, None] * np.sum(dgy, axis=0)[None])
            e_flux = e_flux - np.sum(st["species_enthalpies"][:, None] * j, axis=0)
        else:
            j = -rho * dgy
        f[2 + dim:] = -j
    f[1] = e_flux
    f[2:2 + dim] = tau
    return f


def viscous_facial_flux_central(st_m, st_p, gcv_m, gcv_p, gt_m, gt_p, normal):
    """mirgecom/viscous.py:296-349."""
    f_int = viscous_flux(st_m, gcv_m, gt_m)
    f_ext = viscous_flux(st_p, gcv_p, gt_p)
    return dot_normal(num_flux_central(f_int, f_ext), normal)

# }}}
