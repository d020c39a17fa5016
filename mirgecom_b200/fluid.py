"""Conserved variables, mirroring mirgecom/fluid.py.

``ConservedVars`` keeps the reference's field order
[mass, energy, momentum[dim], species_mass[nspecies]]
(mirgecom/fluid.py:57-275, ``_split_conserved`` :300-312) in ONE contiguous
tensor ``q[Nc, E, Np]`` (float64 on the plain path).  Each field is a view,
so handing the state to a kernel costs nothing.
"""

from __future__ import annotations

import torch


class ConservedVars:
    """Fluid conserved variables ``q[Nc, ...]`` with named field views."""

    __array_priority__ = 100

    def __init__(self, q: torch.Tensor, dim: int):
        if q.shape[0] < dim + 2:
            raise ValueError("ConservedVars needs at least dim + 2 fields")
        self.q = q
        self.dim = dim

    # {{{ fields (fluid.py:57-275)

    @property
    def nspecies(self):
        return self.q.shape[0] - self.dim - 2

    @property
    def mass(self):
        return self.q[0]

    @property
    def energy(self):
        return self.q[1]

    @property
    def momentum(self):
        return self.q[2:2 + self.dim]

    @property
    def species_mass(self):
        return self.q[2 + self.dim:]

    @property
    def velocity(self):
        return self.momentum / self.mass

    @property
    def speed(self):
        """|v| (mirgecom/fluid.py:241-244)."""
        return (self.velocity ** 2).sum(dim=0).sqrt()

    @property
    def species_mass_fractions(self):
        return self.species_mass / self.mass

    @property
    def array_context(self):
        return None

    def join(self):
        return self.q

    def replace(self, **kwargs):
        q = self.q.clone()
        if "mass" in kwargs:
            q[0] = kwargs["mass"]
        if "energy" in kwargs:
            q[1] = kwargs["energy"]
        if "momentum" in kwargs:
            q[2:2 + self.dim] = kwargs["momentum"]
        if "species_mass" in kwargs:
            q[2 + self.dim:] = kwargs["species_mass"]
        return ConservedVars(q, self.dim)

    # }}}

    # {{{ arithmetic (the reference's dataclass_array_container arithmetic)

    def _wrap(self, q):
        return ConservedVars(q, self.dim)

    def _val(self, other):
        return other.q if isinstance(other, ConservedVars) else other

    def __add__(self, other):
        return self._wrap(self.q + self._val(other))

    __radd__ = __add__

    def __sub__(self, other):
        return self._wrap(self.q - self._val(other))

    def __rsub__(self, other):
        return self._wrap(self._val(other) - self.q)

    def __mul__(self, other):
        return self._wrap(self.q * self._val(other))

    __rmul__ = __mul__

    def __truediv__(self, other):
        return self._wrap(self.q / self._val(other))

    def __neg__(self):
        return self._wrap(-self.q)

    # }}}

    def __repr__(self):
        return (f"ConservedVars(dim={self.dim}, nspecies={self.nspecies}, "
                f"shape={tuple(self.q.shape)}, dtype={self.q.dtype})")


def make_conserved(dim, mass=None, energy=None, momentum=None, species_mass=None,
                   q=None, scalar_quantities=None, vector_quantities=None):
    """Counterpart of mirgecom/fluid.py:338-352."""
    if q is not None:
        return ConservedVars(q, dim)
    parts = [mass[None], energy[None], momentum]
    if species_mass is not None and len(species_mass):
        parts.append(species_mass)
    return ConservedVars(torch.cat([torch.as_tensor(p) for p in parts], dim=0).contiguous(), dim)


def velocity_gradient(cv: ConservedVars, grad_cv: ConservedVars):
    """mirgecom/fluid.py:355-397: (grad(rho v) - v grad(rho)) / rho."""
    d = cv.dim
    v = cv.velocity
    return (grad_cv.q[2:2 + d] - v[:, None] * grad_cv.q[0][None]) / cv.mass


def species_mass_fraction_gradient(cv: ConservedVars, grad_cv: ConservedVars):
    """mirgecom/fluid.py:400-427."""
    d = cv.dim
    y = cv.species_mass_fractions
    return (grad_cv.q[2 + d:] - y[:, None] * grad_cv.q[0][None]) / cv.mass
