"""ctypes binding of ``libmgc_b200.so`` (the C ABI of include/mgc_b200.h).

The shared library is built in-tree by ``python -m mirgecom_b200.build``.
There is no CPU fallback: if the library or a GPU is missing, every compute
call raises.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmgc_b200.so")

MAX_SPECIES = 16
MAX_REACTIONS = 8

EOS_IDEAL, EOS_MIXTURE = 0, 1
TR_NONE, TR_SIMPLE, TR_POWERLAW = 0, 1, 2
FLUX_RUSANOV, FLUX_HLL, FLUX_CENTRAL = 0, 1, 2

ERRORS = {-1: "invalid argument", -2: "unsupported configuration",
          -3: "reference operators or mechanism not uploaded", -4: "CUDA error",
          -5: "mesh too large for the fixed no-allocation scratch array"}

ST_NAN, ST_BAD_INDEX, ST_NEWTON_MISS = 1, 2, 4


class GasStruct(C.Structure):
    _fields_ = [
        ("eos_kind", C.c_int32), ("nspecies", C.c_int32), ("niter", C.c_int32),
        ("transport_kind", C.c_int32),
        ("gamma", C.c_double), ("gas_const", C.c_double),
        ("mu", C.c_double), ("mu_b", C.c_double), ("kappa", C.c_double),
        ("pl_alpha", C.c_double), ("pl_beta", C.c_double), ("pl_sigma", C.c_double),
        ("pl_n", C.c_double),
        ("use_lewis", C.c_int32), ("pad_", C.c_int32),
        ("diff", C.c_double * MAX_SPECIES), ("lewis", C.c_double * MAX_SPECIES),
        ("zero_level", C.c_double),
    ]


class MechanismStruct(C.Structure):
    _fields_ = [
        ("nspecies", C.c_int32), ("nreactions", C.c_int32),
        ("mw", C.c_double * MAX_SPECIES), ("inv_mw", C.c_double * MAX_SPECIES),
        ("t_mid", C.c_double * MAX_SPECIES),
        ("a_lo", (C.c_double * 7) * MAX_SPECIES), ("a_hi", (C.c_double * 7) * MAX_SPECIES),
        ("ord_f", (C.c_double * MAX_SPECIES) * MAX_REACTIONS),
        ("nu_p", (C.c_double * MAX_SPECIES) * MAX_REACTIONS),
        ("nu_net", (C.c_double * MAX_SPECIES) * MAX_REACTIONS),
        ("dnu", C.c_double * MAX_REACTIONS), ("log_a", C.c_double * MAX_REACTIONS),
        ("beta", C.c_double * MAX_REACTIONS), ("t_act", C.c_double * MAX_REACTIONS),
        ("reversible", C.c_int32 * MAX_REACTIONS),
    ]


class MeshStruct(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("order", C.c_int32), ("nelem", C.c_int32),
        ("nbf", C.c_int32), ("nperm", C.c_int32), ("elem_kind", C.c_int32),
        ("rx", C.c_void_p), ("conn", C.c_void_p), ("perm", C.c_void_p),
        ("bkind", C.c_void_p), ("rx32", C.c_void_p), ("fslot", C.c_void_p),
        ("nowned", C.c_int32), ("pad_", C.c_int32),
    ]


class MLPStruct(C.Structure):
    _fields_ = [
        ("params", C.c_void_p), ("w1_bf16", C.c_void_p), ("w2_bf16", C.c_void_p),
        ("w2t_bf16", C.c_void_p), ("in_shift", C.c_float * 8), ("in_scale", C.c_float * 8),
        ("out_shift", C.c_float), ("out_scale", C.c_float),
    ]


_P = C.c_void_p
_SIGNATURES = {
    "mgc_version": ([], C.c_int),
    "mgc_supports": ([C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
    "mgc_upload_reference_operators": (
        [C.c_int, C.c_int, _P, _P, _P, _P, _P], C.c_int),
    "mgc_set_mechanism": ([_P], C.c_int),
    "mgc_supports_hex": ([C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
    "mgc_upload_hex_operators": ([C.c_int, C.c_int, _P, _P, C.c_double], C.c_int),
    "mgc_mixture_temperature": ([C.c_int, _P, C.c_int64, _P, _P, _P, _P, _P, _P], C.c_int),
    "mgc_euler_rhs": ([_P, _P, _P, _P, _P, C.c_int, _P, _P, _P], C.c_int),
    "mgc_ns_grad": ([_P, _P, _P, _P, _P, _P, _P, _P], C.c_int),
    "mgc_ns_rhs": ([_P, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P], C.c_int),
    "mgc_rk4_stage": ([C.c_int64, _P, _P, _P, _P, _P, C.c_int, C.c_double, _P], C.c_int),
    "mgc_euler_rhs_f32": ([_P, _P, _P, _P, _P, C.c_int, _P, _P, _P], C.c_int),
    "mgc_ns_grad_f32": ([_P, _P, _P, _P, _P, _P, _P, _P], C.c_int),
    "mgc_ns_rhs_f32": ([_P, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P], C.c_int),
    "mgc_mixture_temperature_f32": (
        [C.c_int, _P, C.c_int64, _P, _P, _P, _P, _P, C.c_int, C.c_float, _P, _P], C.c_int),
    "mgc_mixture_temperature_learned_f32": (
        [C.c_int, _P, C.c_int64, _P, _P, _P, _P, _P, C.c_int, C.c_float, _P, _P], C.c_int),
    "mgc_rk4_stage_mixed": ([C.c_int64, _P, _P, _P, _P, _P, C.c_int, C.c_double, _P], C.c_int),
    "mgc_rhs_split_workspace_bytes": ([_P, _P, C.c_int], C.c_size_t),
    "mgc_rhs_split": ([C.c_int, _P, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P,
                       C.c_size_t, _P, _P, _P], C.c_int),
    "mgc_rhs_split_f32": ([C.c_int, _P, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P,
                           C.c_size_t, _P, _P, _P], C.c_int),
    "mgc_mlp_nparams": ([], C.c_int),
    "mgc_mlp_refresh": ([_P, _P], C.c_int),
    "mgc_mlp_infer": ([C.c_int, C.c_int, C.c_int64, _P, _P, _P, _P], C.c_int),
    "mgc_mlp_train_workspace_bytes": ([C.c_int64], C.c_size_t),
    "mgc_mlp_train_grad": ([C.c_int64, _P, _P, _P, _P, C.c_size_t, _P, _P, _P], C.c_int),
    "mgc_mlp_adam": ([_P, _P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, _P],
                     C.c_int),
    "mgc_ns_operator_noalloc_capacity": ([], C.c_size_t),
    "mgc_ns_operator_noalloc": (
        [_P, _P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P], C.c_int),
    "mgc_operator_workspace_bytes": ([_P, _P, C.c_int], C.c_size_t),
    "mgc_operator": ([C.c_int, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P,
                      C.c_size_t, _P, _P, _P, C.c_int], C.c_int),
    "mgc_operator_f32": ([C.c_int, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P,
                          C.c_size_t, _P, _P, _P, C.c_int], C.c_int),
    "mgc_fp64_probe_flops": ([C.c_int, C.c_int, C.c_int, C.c_int], C.c_double),
    "mgc_fp64_probe": ([C.c_int, C.c_int, C.c_int, C.c_int, _P, _P], C.c_int),
    "mgc_set_gradient_kernel": ([C.c_int], C.c_int),
    "mgc_get_gradient_kernel": ([], C.c_int),
}

_lib = None


def exported_symbols():
    return list(_SIGNATURES)


def load():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with 'python -m mirgecom_b200.build'")
        lib = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed: {ERRORS.get(rc, rc)} ({rc})")


def ptr(t):
    """Device (or host) pointer of a tensor/ndarray, or None."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data_as(C.c_void_p)
    return C.c_void_p(t.data_ptr())


def stream_handle(device=None):
    import torch
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda(t):
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("mirgecom_b200 needs a CUDA device: no CPU fallback exists")
    if not t.is_cuda:
        raise RuntimeError("mirgecom_b200 operators take CUDA tensors")
