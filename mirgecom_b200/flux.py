"""Low-level numerical fluxes, mirroring mirgecom/flux.py.

Elementwise functions on tensors (or numpy arrays).  The same formulas run
inside the device kernels (``csrc/physics.cuh``); these host versions serve
pointwise use and the flux-selection API.
"""

from __future__ import annotations


def _where(cond, a, b):
    try:
        import torch
        if isinstance(cond, torch.Tensor):
            return torch.where(cond, a, b)
    except ImportError:   # pragma: no cover
        pass
    import numpy as np
    return np.where(cond, a, b)


def num_flux_lfr(f_minus_normal, f_plus_normal, q_minus, q_plus, lam):
    """mirgecom/flux.py:45-84."""
    return (f_minus_normal + f_plus_normal + lam * (q_minus - q_plus)) / 2


def num_flux_central(f_minus_normal, f_plus_normal):
    """mirgecom/flux.py:87-110."""
    return (f_plus_normal + f_minus_normal) / 2


def num_flux_hll(f_minus_normal, f_plus_normal, q_minus, q_plus, s_minus, s_plus):
    """mirgecom/flux.py:113-177."""
    f_star = (s_plus * f_minus_normal - s_minus * f_plus_normal
              + s_plus * s_minus * (q_plus - q_minus)) / (s_plus - s_minus)
    f = _where(s_minus >= 0, f_minus_normal + 0 * f_star, f_star)
    f = _where(s_plus <= 0, f_plus_normal + 0 * f, f)
    return f
