"""Euler operator, mirroring mirgecom/euler.py:313-416.

``euler_operator`` keeps the reference signature.  The RHS
``-div_operator(F_I, F*_I)`` -- volume flux, trace pairs, numerical flux,
boundary fluxes, weak divergence, face lift and inverse mass -- runs on the
device (``runtime.euler_rhs``): on simplicial meshes two kernels through
``mgc_operator`` (a volume kernel for the pointwise fluxes, face-node records
and the volume part of the divergence, a face kernel for the numerical
fluxes and the lift); on hexahedra the split divergence pass.
"""

from __future__ import annotations

import warnings

from mirgecom_b200 import runtime
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.inviscid import flux_kind_of, inviscid_facial_flux_rusanov

DD_VOLUME_ALL = "vol"
DISCR_TAG_BASE = "base"


def _check_dd(dd, quadrature_tag):
    if dd not in (None, DD_VOLUME_ALL):
        raise TypeError("dd must represent a volume")
    if quadrature_tag not in (None, DISCR_TAG_BASE):
        raise ValueError("only the base discretization is supported "
                         "(overintegration is not implemented)")


def euler_operator(dcoll, state, gas_model, boundaries, time=0.0,
                   inviscid_numerical_flux_func=None,
                   quadrature_tag=DISCR_TAG_BASE, dd=DD_VOLUME_ALL,
                   comm_tag=None, use_esdg=False, operator_states_quad=None,
                   entropy_conserving_flux_func=None, limiter_func=None,
                   entropy_min=None):
    """RHS of the Euler equations, -div(F_I) with the numerical face flux."""
    _check_dd(dd, quadrature_tag)
    if use_esdg:
        raise NotImplementedError("the entropy-stable DG operator is not implemented")
    if limiter_func is not None or operator_states_quad is not None:
        raise NotImplementedError("limiters / precomputed operator states are not supported")
    if inviscid_numerical_flux_func is None:
        warnings.warn("inviscid_numerical_flux_func unspecified, defaulting to "
                      "inviscid_facial_flux_rusanov.", stacklevel=2)
        inviscid_numerical_flux_func = inviscid_facial_flux_rusanov
    kind = flux_kind_of(inviscid_numerical_flux_func)
    rhs = runtime.euler_rhs(dcoll, state, gas_model, boundaries or {}, time, kind)
    return ConservedVars(rhs, state.dim)
