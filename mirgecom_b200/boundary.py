"""Fluid boundary conditions, mirroring mirgecom/boundary.py.

The device kernels treat a boundary face in one of two ways:

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

``boundary_state_func(dcoll, dd_bdry, gas_model, state_minus, **kwargs)``
keeps the reference signature; ``kwargs`` carries ``time`` and ``nodes``
(the boundary face node coordinates, a tensor (dim, nbf, Nfp)).
"""

from __future__ import annotations

import warnings

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


class AdiabaticSlipBoundary(PrescribedFluidBoundary):
    """Adiabatic slip wall, inviscid part (mirgecom/boundary.py:1052-1080):
    the exterior state of the inviscid numerical flux is the interior state
    with its normal momentum reflected, m+ = m - 2 (m . n) n
    (``_SlipBoundaryComponent.momentum_plus``, boundary.py:152-153); density,
    total energy, species and temperature are the interior ones.  On the
    device it is a prescribed boundary whose exterior state is computed here
    from the interior trace.  The viscous wall treatment of the reference
    (``state_bc``, ``grad_cv_bc``, ``grad_temperature_bc``, boundary.py:
    1082-1143) is not built: ``euler_operator`` accepts this boundary,
    ``ns_operator`` raises ``NotImplementedError``."""

    device_kind = 1
    inviscid_only = True

    def __init__(self):
        self._bnd_state_func = None

    def exterior_state(self, dcoll, dd_bdry, gas_model, state_minus: FluidState, time,
                       nodes=None, normals=None) -> FluidState:
        from mirgecom_b200.fluid import ConservedVars
        if normals is None:
            raise ValueError("the slip wall needs the boundary normals")
        d = state_minus.dim
        q = state_minus.cv.q.clone()
        n = normals.to(q.dtype)
        mom = q[2:2 + d]
        q[2:2 + d] = mom - 2.0 * (mom * n).sum(dim=0) * n
        return FluidState(ConservedVars(q, d), gas_model,
                          temperature=state_minus._temperature,
                          operator_temperature=state_minus.operator_temperature)
