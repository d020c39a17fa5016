"""Fluid boundary conditions, mirroring mirgecom/boundary.py.

The device kernels treat a boundary face in one of these ways:

* ``DummyBoundary`` (mirgecom/boundary.py:1012-1049): every flux uses the
  interior state only -- inviscid F_I(q-).n, gradient flux q- n, viscous
  F_V(q-, grad q-).n;
* ``PrescribedFluidBoundary`` (mirgecom/boundary.py:796-1009) with its
  default helpers: the exterior state comes from *boundary_state_func*
  (evaluated here, on the boundary face nodes, as in the reference); the
  inviscid flux is the numerical flux between interior and exterior states,
  the gradient flux sends the exterior value (boundary.py:70-72), and the
  viscous flux is the central flux with the interior gradients on both
  sides (boundary.py:141-146, 944-970).

* the Mengaldo walls and flow boundaries (mirgecom/boundary.py:391-793):
  ``AdiabaticSlipBoundary``, ``AdiabaticNoslipWallBoundary``,
  ``IsothermalWallBoundary``, ``FarfieldBoundary``,
  ``PressureOutflowBoundary`` -- their boundary states and gradients are
  evaluated in the kernels from the interior trace (simplicial meshes).

``boundary_state_func(dcoll, dd_bdry, gas_model, state_minus, **kwargs)``
keeps the reference signature; ``kwargs`` carries ``time`` and ``nodes``
(the boundary face node coordinates, a tensor (dim, nbf, Nfp)).
"""

from __future__ import annotations

import warnings

import numpy as np

from mirgecom_b200.gas_model import FluidState


class FluidBoundary:
    device_kind = 0


class DummyBoundary(FluidBoundary):
    device_kind = 0

    def __init__(self):
        warnings.warn("Using dummy boundary: copies interior solution.", stacklevel=2)


class PrescribedFluidBoundary(FluidBoundary):
    device_kind = 1

    def __init__(self, inviscid_flux_func=None, boundary_state_func=None,
                 temperature_gradient_flux_func=None, boundary_temperature_func=None,
                 cv_gradient_flux_func=None, gradient_numerical_flux_func=None,
                 viscous_flux_func=None, boundary_gradient_cv_func=None,
                 boundary_gradient_temperature_func=None):
        unsupported = [n for n, f in dict(
            inviscid_flux_func=inviscid_flux_func,
            temperature_gradient_flux_func=temperature_gradient_flux_func,
            boundary_temperature_func=boundary_temperature_func,
            cv_gradient_flux_func=cv_gradient_flux_func,
            gradient_numerical_flux_func=gradient_numerical_flux_func,
            viscous_flux_func=viscous_flux_func,
            boundary_gradient_cv_func=boundary_gradient_cv_func,
            boundary_gradient_temperature_func=boundary_gradient_temperature_func,
        ).items() if f is not None]
        if unsupported:
            raise NotImplementedError(
                "custom boundary flux callbacks are not supported by the device "
                f"kernels: {unsupported}")
        if boundary_state_func is None:
            warnings.warn("Using dummy boundary: copies interior solution.", stacklevel=2)
            self.device_kind = 0
        self._bnd_state_func = boundary_state_func

    def exterior_state(self, dcoll, dd_bdry, gas_model, state_minus: FluidState, time,
                       nodes=None, normals=None) -> FluidState:
        if self._bnd_state_func is None:
            return state_minus
        return self._bnd_state_func(dcoll=dcoll, dd_bdry=dd_bdry, gas_model=gas_model,
                                    state_minus=state_minus, time=time, nodes=nodes)


class MengaldoBoundaryCondition(FluidBoundary):
    """The Mengaldo boundary treatment (mirgecom/boundary.py:391-793): the
    inviscid flux is the numerical flux between the interior state and
    ``state_plus``; the gradient fluxes send ``state_bc.cv`` and
    ``temperature_bc``; the viscous flux is F_V(state_bc, grad_cv_bc,
    grad_t_bc) . n.  On the device every one of these is evaluated per
    boundary face node from the interior trace (``device_kind`` selects the
    wall); :meth:`exterior_parameters` gives the per-node parameters the
    kernels read from the exterior-state array (None: none)."""

    device_kind = -1

    def exterior_parameters(self, dcoll, gas_model, state_minus, nc):
        return None


class AdiabaticSlipBoundary(MengaldoBoundaryCondition):
    """mirgecom/boundary.py:1052-1143: state_plus reflects the normal
    momentum, state_bc removes it (internal energy kept); temperature_bc is
    the interior temperature; grad_cv_bc zeroes the tangential velocities'
    normal derivatives and the mass fractions' normal gradients;
    grad_temperature_bc removes the normal component (adiabatic)."""

    device_kind = 2


class AdiabaticNoslipWallBoundary(MengaldoBoundaryCondition):
    """mirgecom/boundary.py:1794-1858: state_plus reverses the momentum,
    state_bc has zero momentum and the internal energy at the interior
    temperature; grad_cv_bc impermeable to species; adiabatic grad_t_bc."""

    device_kind = 3


class IsothermalWallBoundary(MengaldoBoundaryCondition):
    """mirgecom/boundary.py:1727-1792: as the adiabatic no-slip wall, but
    state_bc and temperature_bc at *wall_temperature* and grad_t_bc the
    interior one."""

    device_kind = 4

    def __init__(self, wall_temperature=300):
        self._wall_temp = wall_temperature

    def exterior_parameters(self, dcoll, gas_model, state_minus, nc):
        import torch
        t = torch.as_tensor(self._wall_temp, dtype=state_minus.cv.q.dtype,
                            device=state_minus.cv.q.device)
        out = torch.zeros((nc + 1,) + tuple(state_minus.cv.q.shape[1:]),
                          dtype=state_minus.cv.q.dtype, device=state_minus.cv.q.device)
        out[nc] = t
        return out


class FarfieldBoundary(MengaldoBoundaryCondition):
    """mirgecom/boundary.py:1146-1228: state_plus = state_bc = the free
    stream (density from p, T and Y; total energy from the internal energy
    at T and the free-stream velocity), temperature_bc the free-stream
    temperature, gradients the interior ones.  The free-stream state and its
    temperature (the mixture Newton solve seeded by the free-stream
    temperature, as make_fluid_state does) are computed here and passed to
    the kernels in the exterior-state array."""

    device_kind = 5

    def __init__(self, free_stream_pressure, free_stream_velocity,
                 free_stream_temperature, free_stream_mass_fractions=None):
        self._pressure = free_stream_pressure
        self._velocity = free_stream_velocity
        self._temperature = free_stream_temperature
        self._mass_fractions = free_stream_mass_fractions

    def exterior_parameters(self, dcoll, gas_model, state_minus, nc):
        import torch

        from mirgecom_b200.fluid import ConservedVars
        from mirgecom_b200.gas_model import make_fluid_state
        q = state_minus.cv.q
        dim = state_minus.dim
        shape = tuple(q.shape[1:])
        kw = dict(dtype=q.dtype, device=q.device)
        t = torch.full(shape, float(self._temperature), **kw)
        p = torch.full(shape, float(self._pressure), **kw)
        v = torch.as_tensor(np.asarray(self._velocity, dtype=np.float64), **kw).reshape(
            (dim,) + (1,) * len(shape)) * torch.ones(shape, **kw)
        ns = nc - 2 - dim
        if ns:
            y = torch.as_tensor(np.asarray(self._mass_fractions, dtype=np.float64), **kw)
            y = y.reshape((ns,) + (1,) * len(shape)) * torch.ones(shape, **kw)
        else:
            y = torch.zeros((0,) + shape, **kw)
        eos = gas_model.eos
        rho = eos.get_density(p, t, species_mass_fractions=y)
        e = eos.get_internal_energy(t, species_mass_fractions=y)
        energy = rho * (e + 0.5 * (v * v).sum(dim=0))
        cv = ConservedVars(torch.cat([rho[None], energy[None], rho * v, rho * y]), dim)
        out = torch.zeros((nc + 1,) + shape, **kw)
        out[:nc] = cv.q
        if eos.is_mixture:
            out[nc] = make_fluid_state(cv, gas_model, temperature_seed=t).temperature
        else:
            out[nc] = t
        return out


class PressureOutflowBoundary(MengaldoBoundaryCondition):
    """mirgecom/boundary.py:1231-1403: mass, momentum and species from the
    interior; the energy from the boundary pressure (state_bc) or its
    reflection about the interior pressure (state_plus) where the outflow is
    subsonic, from the interior where it is supersonic; gradients the
    interior ones."""

    device_kind = 6

    def __init__(self, boundary_pressure=101325):
        self._pressure = boundary_pressure

    def exterior_parameters(self, dcoll, gas_model, state_minus, nc):
        import torch
        q = state_minus.cv.q
        out = torch.zeros((nc + 1,) + tuple(q.shape[1:]), dtype=q.dtype, device=q.device)
        out[0] = float(self._pressure)
        return out


class _SlipStatePlus(PrescribedFluidBoundary):
    """The slip wall's state_plus (boundary.py:1075-1080: the interior state
    with its normal momentum reflected, m+ = m - 2 (m . n) n) computed here
    from the interior trace and handed to the kernels as a prescribed
    exterior state.  The Euler operator needs nothing else from the wall,
    so meshes whose kernels lack the device slip treatment (tensor-product
    hexahedra) evaluate the inviscid slip wall this way."""

    device_kind = 1

    def __init__(self):
        self._bnd_state_func = None

    def exterior_state(self, dcoll, dd_bdry, gas_model, state_minus: FluidState, time,
                       nodes=None, normals=None) -> FluidState:
        from mirgecom_b200.fluid import ConservedVars
        d = state_minus.dim
        q = state_minus.cv.q.clone()
        n = normals.to(q.dtype)
        mom = q[2:2 + d]
        q[2:2 + d] = mom - 2.0 * (mom * n).sum(dim=0) * n
        return FluidState(ConservedVars(q, d), gas_model,
                          temperature=state_minus._temperature,
                          operator_temperature=state_minus.operator_temperature)
