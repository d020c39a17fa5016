"""Viscous facial flux selector, mirroring mirgecom/viscous.py:296-349.

The central viscous flux 1/2 (F_V+ + F_V-) . n is evaluated inside the
device kernels; this function is the selector ``ns_operator`` accepts.
"""


def viscous_facial_flux_central(dcoll=None, state_pair=None, grad_cv_pair=None,
                                grad_t_pair=None, gas_model=None):
    raise NotImplementedError("evaluated inside the device kernels only")


viscous_facial_flux_central.device_supported = True


def get_local_max_species_diffusivity(actx, d_alpha):
    """Largest species diffusivity at every node (mirgecom/viscous.py:641-665);
    0 without species.  *actx* is accepted for the reference's signature."""
    import numpy as np
    import torch
    if d_alpha is None or len(d_alpha) == 0:
        return 0
    if isinstance(d_alpha, torch.Tensor):
        return d_alpha.max(dim=0).values if d_alpha.ndim > 1 else float(d_alpha.max())
    return float(np.max(d_alpha))


def get_viscous_timestep(dcoll, state, *, dd=None):
    """Node-local stable time step of a viscous fluid,
    h / (|v| + c + (mu / rho + max_a D_a) / h) (mirgecom/viscous.py:547-607).
    Returns a tensor shaped like the state's fields (E, Np)."""
    if dd is not None and dd != "vol":
        raise TypeError("dd must represent the volume")
    ws = state.wavespeed
    h = dcoll.characteristic_lengthscales(device=ws.device, dtype=ws.dtype)
    nu = 0
    d_alpha_max = 0
    if state.is_viscous:
        nu = state.viscosity / state.mass_density
        d_alpha_max = get_local_max_species_diffusivity(None, state.species_diffusivity)
    return h / (ws + (nu + d_alpha_max) / h)
