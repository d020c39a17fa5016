"""Viscous facial flux selector, mirroring mirgecom/viscous.py:296-349.

The central viscous flux 1/2 (F_V+ + F_V-) . n is evaluated inside the
device kernels; this function is the selector ``ns_operator`` accepts.
"""


def viscous_facial_flux_central(dcoll=None, state_pair=None, grad_cv_pair=None,
                                grad_t_pair=None, gas_model=None):
    raise NotImplementedError("evaluated inside the device kernels only")


viscous_facial_flux_central.device_supported = True
