"""Equations of state, mirroring mirgecom/eos.py.

The classes carry parameters; the arithmetic runs in the device kernels
(``csrc/physics.cuh``).  ``IdealSingleGas`` follows mirgecom/eos.py:302-537,
``PyrometheusMixture`` mirgecom/eos.py:540-888 with the fixed-iteration
Newton temperature solve of mirgecom/thermochemistry.py:126-167.
"""

from __future__ import annotations

import numpy as np

from mirgecom_b200 import _lib
from mirgecom_b200.thermochemistry import GAS_CONSTANT, Mechanism


class TemperatureSeedMissingError(Exception):
    """mirgecom/eos.py:54: mixtures need a temperature seed."""


class GasEOS:
    is_mixture = False


class IdealSingleGas(GasEOS):
    """p = rho R T with constant gamma (defaults gamma=1.4, R=287.1)."""

    def __init__(self, gamma=1.4, gas_const=287.1):
        self._gamma = float(gamma)
        self._gas_const = float(gas_const)

    def gamma(self, cv=None, temperature=None):
        return self._gamma

    def gas_const(self, cv=None, temperature=None, species_mass_fractions=None):
        return self._gas_const

    def heat_capacity_cp(self, cv=None, temperature=None):
        return self._gas_const * self._gamma / (self._gamma - 1)

    def heat_capacity_cv(self, cv=None, temperature=None):
        return self._gas_const / (self._gamma - 1)

    def get_density(self, pressure, temperature, species_mass_fractions=None):
        return pressure / (self._gas_const * temperature)

    def kinetic_energy(self, cv):
        mom = cv.momentum
        return 0.5 * (mom * mom).sum(dim=0) / cv.mass

    def internal_energy(self, cv):
        return cv.energy - self.kinetic_energy(cv)

    def pressure(self, cv, temperature=None):
        return self.internal_energy(cv) * (self._gamma - 1.0)

    def sound_speed(self, cv, temperature=None):
        return (self._gamma / cv.mass * self.pressure(cv)).sqrt()

    def temperature(self, cv, temperature_seed=None):
        return (((self._gamma - 1.0) / self._gas_const)
                * self.internal_energy(cv) / cv.mass)

    def total_energy(self, cv, pressure, temperature=None):
        return pressure / (self._gamma - 1.0) + self.kinetic_energy(cv)

    def get_internal_energy(self, temperature, species_mass_fractions=None):
        return self._gas_const * temperature / (self._gamma - 1)

    def fill_struct(self, s: _lib.GasStruct):
        s.eos_kind = _lib.EOS_IDEAL
        s.gamma = self._gamma
        s.gas_const = self._gas_const


class MixtureEOS(GasEOS):
    is_mixture = True


class PyrometheusMixture(MixtureEOS):
    """Ideal-gas mixture with NASA-7 thermodynamics and Arrhenius kinetics.

    *pyrometheus_mech* is a :class:`~mirgecom_b200.thermochemistry.Mechanism`
    (the role the pyrometheus class plays in the reference);
    *temperature_niter* is the Newton iteration count of the reference's
    wrapper class (``get_pyrometheus_wrapper_class(temperature_niter=5)``).
    """

    def __init__(self, pyrometheus_mech: Mechanism, temperature_guess=300.0,
                 temperature_niter=5, zero_level=0.0, learned_guess=None):
        if pyrometheus_mech.nspecies > _lib.MAX_SPECIES \
                or pyrometheus_mech.nreactions > _lib.MAX_REACTIONS:
            raise ValueError("mechanism too large for the device tables")
        self._mech = pyrometheus_mech
        self._tguess = float(temperature_guess)
        self._niter = int(temperature_niter)
        self._zero_level = float(zero_level)
        # optional learned Newton initial guess (mixed form only), e.g. a
        # mirgecom_b200.learned_guess.TemperatureMLP
        self.learned_guess = learned_guess

    def learned_temperature_guess(self, cv):
        return self.learned_guess.predict(cv)

    @property
    def mechanism(self):
        return self._mech

    @property
    def temperature_niter(self):
        return self._niter

    def get_temperature_seed(self, ary=None, temperature_seed=None):
        import torch
        tseed = self._tguess if temperature_seed is None else temperature_seed
        if isinstance(tseed, torch.Tensor):
            return tseed
        if ary is None:
            raise ValueError("Requires *ary* for shaping temperature seed.")
        return torch.full_like(ary, float(tseed))

    def get_species_molecular_weights(self):
        return self._mech.molecular_weights

    def gas_const(self, cv=None, temperature=None, species_mass_fractions=None):
        y = species_mass_fractions if cv is None else cv.species_mass_fractions
        w = _wcol(self._mech.molecular_weights, y)
        return GAS_CONSTANT * (y / w).sum(dim=0)

    def kinetic_energy(self, cv):
        mom = cv.momentum
        return 0.5 * (mom * mom).sum(dim=0) / cv.mass

    def internal_energy(self, cv):
        return cv.energy - self.kinetic_energy(cv)

    def _species_cp_r(self, temperature):
        """NASA-7 c_p,k / R per species, (Ns, ...), the range chosen by T."""
        import torch
        m = self._mech
        t = temperature
        shape = (-1,) + (1,) * t.ndim
        lo = torch.as_tensor(m.nasa_low, dtype=t.dtype, device=t.device)
        hi = torch.as_tensor(m.nasa_high, dtype=t.dtype, device=t.device)
        sel = t[None] > torch.as_tensor(m.t_mid, dtype=t.dtype, device=t.device).reshape(shape)
        a = [torch.where(sel, hi[:, j].reshape(shape), lo[:, j].reshape(shape)) for j in range(5)]
        return a[0] + t * (a[1] + t * (a[2] + t * (a[3] + t * a[4])))

    def heat_capacity_cp(self, cv, temperature):
        """Mixture c_p per unit mass (mirgecom/eos.py:631-635)."""
        y = cv.species_mass_fractions
        w = _wcol(self._mech.molecular_weights, y)
        return GAS_CONSTANT * (y * self._species_cp_r(temperature) / w).sum(dim=0)

    def heat_capacity_cv(self, cv, temperature):
        """c_v = c_p - R_mix (mirgecom/eos.py:637-642)."""
        return self.heat_capacity_cp(cv, temperature) - self.gas_const(cv)

    def gamma(self, cv, temperature):
        """c_p / (c_p - R_mix) (mirgecom/eos.py:644-650)."""
        return self.heat_capacity_cp(cv, temperature) / self.heat_capacity_cv(cv, temperature)

    def get_density(self, pressure, temperature, species_mass_fractions):
        """rho = p / (R_mix T) (mirgecom/eos.py:702-718)."""
        return pressure / (self.gas_const(species_mass_fractions=species_mass_fractions)
                           * temperature)

    def get_internal_energy(self, temperature, species_mass_fractions):
        """Mass-specific internal energy e(T, Y) = sum_k Y_k (R/W_k) T
        (h_k/RT - 1) (mirgecom/eos.py:690-700)."""
        from mirgecom_b200.initializers import _nasa_e_rt
        y = species_mass_fractions
        t = temperature
        w = _wcol(self._mech.molecular_weights, y)
        return GAS_CONSTANT * t * (y / w * _nasa_e_rt(self._mech, t)).sum(dim=0)

    def pressure(self, cv, temperature):
        """p = rho R_mix T (mirgecom/eos.py:751-761)."""
        return cv.mass * self.gas_const(cv) * temperature

    def sound_speed(self, cv, temperature):
        """c = sqrt(gamma p / rho) (mirgecom/eos.py:763-776)."""
        return (self.gamma(cv, temperature) * self.pressure(cv, temperature) / cv.mass).sqrt()

    def fill_struct(self, s: _lib.GasStruct):
        s.eos_kind = _lib.EOS_MIXTURE
        s.niter = self._niter
        s.zero_level = self._zero_level

    def mechanism_struct(self) -> _lib.MechanismStruct:
        return mechanism_struct(self._mech)


def _wcol(w, like):
    import torch
    t = torch.as_tensor(np.asarray(w), dtype=like.dtype, device=like.device)
    return t.reshape((-1,) + (1,) * (like.ndim - 1))


def mechanism_struct(mech: Mechanism) -> _lib.MechanismStruct:
    ms = _lib.MechanismStruct()
    ms.nspecies = mech.nspecies
    ms.nreactions = mech.nreactions
    for k in range(mech.nspecies):
        ms.mw[k] = mech.molecular_weights[k]
        ms.inv_mw[k] = 1.0 / mech.molecular_weights[k]
        ms.t_mid[k] = mech.t_mid[k]
        for j in range(7):
            ms.a_lo[k][j] = mech.nasa_low[k, j]
            ms.a_hi[k][j] = mech.nasa_high[k, j]
    for i in range(mech.nreactions):
        for k in range(mech.nspecies):
            ms.ord_f[i][k] = mech.orders_fwd[i, k]
            ms.nu_p[i][k] = mech.nu_prod[i, k]
            ms.nu_net[i][k] = mech.nu_prod[i, k] - mech.nu_reac[i, k]
        ms.dnu[i] = float(np.sum(mech.nu_prod[i] - mech.nu_reac[i]))
        ms.log_a[i] = mech.log_a[i]
        ms.beta[i] = mech.beta[i]
        ms.t_act[i] = mech.t_act[i]
        ms.reversible[i] = int(bool(mech.reversible[i]))
    return ms
