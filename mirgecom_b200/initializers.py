"""Initial states for the benchmark and test configurations.

* :class:`Vortex2D` -- the isentropic vortex of mirgecom/initializers.py:143-225
  (Zhou 2003; Hesthaven & Warburton 2008, sec. 6.6).
* :func:`taylor_green_state` -- the viscous Taylor-Green vortex
  u = sin x cos y cos z, v = -cos x sin y cos z, w = 0,
  p = p0 + rho0 V0^2/16 (cos 2x + cos 2y)(cos 2z + 2), p0 = rho0 V0^2/(gamma M^2),
  rho = rho0 (the textbook fields; the reference's own inviscid initializer,
  mirgecom/initializers.py:1523-1591, mixes up z and is not used).
* :func:`reacting_mixture_state` -- seeded smooth random fields for the
  reacting-mixture configurations: T in [300, 2500] K, p = 101325 (1 +- 5%),
  mass fractions from a Dirichlet(alpha=2) draw modulated by smooth positive
  fields and renormalised, |v| <= 10 m/s; rho = p / (R_mix T) and the energy
  from the NASA-7 internal energy (mirgecom/eos.py:540-888 conventions).

All functions take/return torch tensors on the nodes' device.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.thermochemistry import GAS_CONSTANT


class Vortex2D:
    def __init__(self, *, beta=5, center=(0, 0), velocity=(0, 0)):
        self._beta = beta
        self._center = np.array(center, dtype=np.float64)
        self._velocity = np.array(velocity, dtype=np.float64)

    def __call__(self, x_vec, *, time=0, eos=None, **kwargs):
        gamma = 1.4 if eos is None else eos.gamma()
        loc = self._center + time * self._velocity
        x_rel = x_vec[0] - loc[0]
        y_rel = x_vec[1] - loc[1]
        r = torch.sqrt(x_rel ** 2 + y_rel ** 2)
        expterm = self._beta * torch.exp(1 - r ** 2)
        u = self._velocity[0] - expterm * y_rel / (2 * np.pi)
        v = self._velocity[1] + expterm * x_rel / (2 * np.pi)
        mass = (1 - (gamma - 1) / (16 * gamma * np.pi ** 2)
                * expterm ** 2) ** (1 / (gamma - 1))
        p = mass ** gamma
        energy = p / (gamma - 1) + mass / 2 * (u ** 2 + v ** 2)
        return ConservedVars(torch.stack([mass, energy, mass * u, mass * v]), 2)


def taylor_green_state(x_vec, *, gamma=1.4, mach=0.1, rho0=1.0, v0=1.0):
    x, y, z = x_vec
    u = v0 * torch.sin(x) * torch.cos(y) * torch.cos(z)
    v = -v0 * torch.cos(x) * torch.sin(y) * torch.cos(z)
    w = torch.zeros_like(u)
    p0 = rho0 * v0 ** 2 / (gamma * mach ** 2)
    p = p0 + rho0 * v0 ** 2 / 16 * (torch.cos(2 * x) + torch.cos(2 * y)) * (torch.cos(2 * z) + 2)
    rho = torch.full_like(u, rho0)
    energy = p / (gamma - 1) + 0.5 * rho * (u * u + v * v + w * w)
    return ConservedVars(torch.stack([rho, energy, rho * u, rho * v, rho * w]), 3)


def taylor_green_transport_params(gamma=1.4, gas_const=287.1, reynolds=1600.0,
                                  prandtl=0.71, rho0=1.0, v0=1.0, length=1.0):
    mu = rho0 * v0 * length / reynolds
    cp = gamma * gas_const / (gamma - 1)
    return {"viscosity": mu, "thermal_conductivity": mu * cp / prandtl}


def _smooth_field(x_vec, gen, nmodes=4, kmax=4, box=None):
    """Sum of low-wavenumber Fourier modes, scaled to [-1, 1]."""
    dim = len(x_vec)
    box = box or [2 * math.pi] * dim
    f = torch.zeros_like(x_vec[0])
    for _ in range(nmodes):
        k = torch.randint(0, kmax + 1, (dim,), generator=gen)
        if int(k.sum()) == 0:
            k[0] = 1
        phase = float(torch.rand(1, generator=gen)) * 2 * math.pi
        amp = float(torch.rand(1, generator=gen)) + 0.5
        arg = sum(2 * math.pi * int(k[d]) * x_vec[d] / box[d] for d in range(dim))
        f = f + amp * torch.cos(arg + phase)
    fmax = f.abs().max().clamp_min(1e-30)
    return f / fmax


def _nasa_e_rt(mech, t):
    """(h/RT - 1) per species, shape (Ns, ...), torch."""
    lo = torch.as_tensor(mech.nasa_low, dtype=t.dtype, device=t.device)
    hi = torch.as_tensor(mech.nasa_high, dtype=t.dtype, device=t.device)
    tmid = torch.as_tensor(mech.t_mid, dtype=t.dtype, device=t.device)
    shape = (-1,) + (1,) * t.ndim
    sel = t[None] > tmid.reshape(shape)
    a = [torch.where(sel, hi[:, j].reshape(shape), lo[:, j].reshape(shape)) for j in range(6)]
    h_rt = (a[0] + a[1] / 2 * t + a[2] / 3 * t ** 2 + a[3] / 4 * t ** 3
            + a[4] / 5 * t ** 4 + a[5] / t)
    return h_rt - 1.0


def reacting_mixture_state(x_vec, mech, *, seed=0, t_range=(300.0, 2500.0),
                           p_mean=101325.0, p_rel=0.05, vmax=10.0, alpha=2.0,
                           box=None):
    """Returns (ConservedVars, temperature) on the given node coordinates."""
    gen = torch.Generator().manual_seed(seed)
    dim = len(x_vec)
    tlo, thi = t_range
    t = 0.5 * (tlo + thi) + 0.5 * (thi - tlo) * _smooth_field(x_vec, gen, box=box)
    p = p_mean * (1 + p_rel * _smooth_field(x_vec, gen, box=box))
    ns = mech.nspecies
    base = _dirichlet(ns, alpha, gen)
    ys = []
    for k in range(ns):
        ys.append(float(base[k]) * torch.exp(0.5 * _smooth_field(x_vec, gen, box=box)))
    y = torch.stack(ys)
    y = y / y.sum(dim=0, keepdim=True)
    w = torch.as_tensor(mech.molecular_weights, dtype=t.dtype, device=t.device)
    w = w.reshape((-1,) + (1,) * t.ndim)
    rmix = GAS_CONSTANT * (y / w).sum(dim=0)
    rho = p / (rmix * t)
    vel = [vmax / math.sqrt(dim) * _smooth_field(x_vec, gen, box=box) for _ in range(dim)]
    e = GAS_CONSTANT * t * (y * _nasa_e_rt(mech, t) / w).sum(dim=0)
    ke = 0.5 * sum(v * v for v in vel)
    q = torch.cat([rho[None], (rho * (e + ke))[None], torch.stack([rho * v for v in vel]),
                   rho[None] * y])
    return ConservedVars(q.contiguous(), dim), t


def _dirichlet(n, alpha, gen):
    """Dirichlet(alpha) draw; alpha = 2 is a sum of two unit exponentials."""
    if float(alpha) != 2.0:
        raise ValueError("only alpha = 2 is supported")
    u = torch.rand((2, n), generator=gen, dtype=torch.float64).clamp_min(1e-300)
    g = -torch.log(u).sum(dim=0)
    return g / g.sum()
