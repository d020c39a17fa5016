"""Transport models, mirroring mirgecom/transport.py.

``SimpleTransport`` (mirgecom/transport.py:143-202): constant mu, mu_B,
kappa and species diffusivities.  ``PowerLawTransport`` (:205-321):
mu = beta T^n, mu_B = alpha mu, kappa = sigma mu c_v, and diffusivities
either given or from Lewis numbers, d = sigma mu / (rho Le gamma).
The values are evaluated per node inside the device kernels.
"""

from __future__ import annotations

import numpy as np

from mirgecom_b200 import _lib


class TransportModel:
    pass


class SimpleTransport(TransportModel):
    def __init__(self, bulk_viscosity=0, viscosity=0, thermal_conductivity=0,
                 species_diffusivity=None):
        if species_diffusivity is None:
            species_diffusivity = np.empty((0,))
        self._mu_bulk = float(bulk_viscosity)
        self._mu = float(viscosity)
        self._kappa = float(thermal_conductivity)
        self._d_alpha = np.asarray(species_diffusivity, dtype=np.float64)

    def viscosity(self, cv=None, dv=None, eos=None):
        return self._mu

    def bulk_viscosity(self, cv=None, dv=None, eos=None):
        return self._mu_bulk

    def volume_viscosity(self, cv=None, dv=None, eos=None):
        return self._mu_bulk - 2 * self._mu / 3

    def thermal_conductivity(self, cv=None, dv=None, eos=None):
        return self._kappa

    def species_diffusivity(self, cv=None, dv=None, eos=None):
        return self._d_alpha

    def fill_struct(self, s: _lib.GasStruct, nspecies: int):
        s.transport_kind = _lib.TR_SIMPLE
        s.mu = self._mu
        s.mu_b = self._mu_bulk
        s.kappa = self._kappa
        _fill_diff(s, self._d_alpha, nspecies)


class PowerLawTransport(TransportModel):
    def __init__(self, alpha=0.6, beta=4.093e-7, sigma=2.5, n=.666,
                 species_diffusivity=None, lewis=None):
        if species_diffusivity is None and lewis is None:
            species_diffusivity = np.empty((0,))
        self._alpha = float(alpha)
        self._beta = float(beta)
        self._sigma = float(sigma)
        self._n = float(n)
        self._d_alpha = (None if species_diffusivity is None
                         else np.asarray(species_diffusivity, dtype=np.float64))
        self._lewis = None if lewis is None else np.asarray(lewis, dtype=np.float64)

    # host evaluations (mirgecom/transport.py:255-321); dv is the fluid state
    # (its temperature), as the reference passes its dependent variables
    def viscosity(self, cv=None, dv=None, eos=None):
        """mu = beta T^n."""
        return self._beta * dv.temperature ** self._n

    def bulk_viscosity(self, cv=None, dv=None, eos=None):
        return self._alpha * self.viscosity(cv, dv)

    def volume_viscosity(self, cv=None, dv=None, eos=None):
        return (self._alpha - 2.0 / 3.0) * self.viscosity(cv, dv)

    def thermal_conductivity(self, cv=None, dv=None, eos=None):
        """kappa = sigma mu c_v."""
        return self._sigma * self.viscosity(cv, dv) * eos.heat_capacity_cv(cv, dv.temperature)

    def species_diffusivity(self, cv=None, dv=None, eos=None):
        """Given diffusivities, or sigma mu / (rho Le gamma) from Lewis numbers."""
        if self._lewis is not None:
            import torch
            le = torch.as_tensor(self._lewis, dtype=cv.mass.dtype, device=cv.mass.device)
            le = le.reshape((-1,) + (1,) * cv.mass.ndim)
            return (self._sigma * self.viscosity(cv, dv)
                    / (cv.mass * le * eos.gamma(cv, dv.temperature)))
        return self._d_alpha

    def fill_struct(self, s: _lib.GasStruct, nspecies: int):
        s.transport_kind = _lib.TR_POWERLAW
        s.pl_alpha = self._alpha
        s.pl_beta = self._beta
        s.pl_sigma = self._sigma
        s.pl_n = self._n
        if self._lewis is not None:
            s.use_lewis = 1
            for k in range(nspecies):
                s.lewis[k] = self._lewis[k]
        else:
            _fill_diff(s, self._d_alpha, nspecies)


def _fill_diff(s, d, nspecies):
    if nspecies > _lib.MAX_SPECIES:
        raise ValueError("too many species")
    for k in range(nspecies):
        s.diff[k] = float(d[k]) if k < len(d) else 0.0
