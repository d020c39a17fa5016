"""Navier-Stokes operator, mirroring mirgecom/navierstokes.py:129-575.

``ns_operator`` keeps the reference signature and computes
div(F_V - F_I) with BR1 gradients on the device (``runtime.ns_rhs``): on
simplicial meshes in two kernels through ``mgc_operator`` (a volume kernel
that keeps the gradients on chip and evaluates the pointwise fluxes and the
volume part of the divergence, and a face kernel for the numerical fluxes and
the lift); on hexahedra as a gradient pass and a split divergence pass.
For a reacting mixture the species source terms (the driver-side
``eos.get_species_source_terms`` of examples/gas-in-box.py:702-705) are
fused into the volume kernel by passing ``species_source_temperature``.
"""

from __future__ import annotations

from mirgecom_b200 import runtime
from mirgecom_b200.euler import DD_VOLUME_ALL, DISCR_TAG_BASE, _check_dd
from mirgecom_b200.flux import num_flux_central
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.inviscid import flux_kind_of, inviscid_facial_flux_rusanov
from mirgecom_b200.viscous import viscous_facial_flux_central


def _check_fluxes(gradient_numerical_flux_func, viscous_numerical_flux_func):
    if gradient_numerical_flux_func is not num_flux_central:
        raise NotImplementedError("the device gradient pass uses the central (BR1) flux")
    if viscous_numerical_flux_func is not viscous_facial_flux_central:
        raise NotImplementedError("the device divergence pass uses the central viscous flux")


def _split_grad(grad, state):
    nc = state.cv.q.shape[0]
    return ConservedVars(grad[:nc], state.dim), grad[nc]


def grad_cv_operator(dcoll, gas_model, boundaries, state, *, time=0.0,
                     numerical_flux_func=num_flux_central,
                     quadrature_tag=DISCR_TAG_BASE, dd=DD_VOLUME_ALL, comm_tag=None,
                     operator_states_quad=None, limiter_func=None, entropy_min=None,
                     use_esdg=False):
    """Gradient of the conserved variables, ConservedVars of (Nc, dim, E, Np)."""
    _check_dd(dd, quadrature_tag)
    _check_fluxes(numerical_flux_func, viscous_facial_flux_central)
    grad = runtime.ns_gradients(dcoll, state, gas_model, boundaries or {}, time)
    return _split_grad(grad.clone(), state)[0]


def grad_t_operator(dcoll, gas_model, boundaries, state, *, time=0.0,
                    numerical_flux_func=num_flux_central,
                    quadrature_tag=DISCR_TAG_BASE, dd=DD_VOLUME_ALL, comm_tag=None,
                    operator_states_quad=None, limiter_func=None, entropy_min=None,
                    use_esdg=False):
    """Gradient of the temperature, a tensor (dim, E, Np)."""
    _check_dd(dd, quadrature_tag)
    _check_fluxes(numerical_flux_func, viscous_facial_flux_central)
    grad = runtime.ns_gradients(dcoll, state, gas_model, boundaries or {}, time)
    return _split_grad(grad.clone(), state)[1]


def ns_operator(dcoll, gas_model, state, boundaries, *, time=0.0,
                inviscid_fluid_operator=None,
                inviscid_numerical_flux_func=inviscid_facial_flux_rusanov,
                gradient_numerical_flux_func=num_flux_central,
                viscous_numerical_flux_func=viscous_facial_flux_central,
                return_gradients=False, quadrature_tag=DISCR_TAG_BASE,
                dd=DD_VOLUME_ALL, comm_tag=None, limiter_func=None,
                entropy_min=None, operator_states_quad=None, use_esdg=False,
                grad_cv=None, grad_t=None, inviscid_terms_on=True,
                entropy_conserving_flux_func=None,
                species_source_temperature=None):
    """RHS of the Navier-Stokes equations, div(F_V - F_I)."""
    if not state.is_viscous:
        raise ValueError("Navier-Stokes operator expects viscous gas model.")
    _check_dd(dd, quadrature_tag)
    _check_fluxes(gradient_numerical_flux_func, viscous_numerical_flux_func)
    if use_esdg or inviscid_fluid_operator is not None or not inviscid_terms_on:
        raise NotImplementedError("only the fused inviscid branch is implemented")
    if grad_cv is not None or grad_t is not None:
        raise NotImplementedError("precomputed gradients are not supported")
    if limiter_func is not None or operator_states_quad is not None:
        raise NotImplementedError("limiters / precomputed operator states are not supported")
    kind = flux_kind_of(inviscid_numerical_flux_func)
    rhs, grad = runtime.ns_rhs(dcoll, state, gas_model, boundaries or {}, time, kind,
                               source_temperature=species_source_temperature,
                               want_gradients=return_gradients)
    out = ConservedVars(rhs, state.dim)
    if return_gradients:
        gcv, gt = _split_grad(grad, state)
        return out, gcv, gt
    return out
