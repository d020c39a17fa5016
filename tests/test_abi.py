"""The C-ABI library loads and exports every symbol include/mgc_b200.h declares."""

import ctypes
import os
import re

from mirgecom_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "mgc_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mgc_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "mgc_euler_rhs" in names and "mgc_ns_rhs" in names


def test_library_exports_all_declared_symbols():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_version_and_supports_without_gpu():
    lib = _lib.load()
    assert lib.mgc_version() >= 1
    assert lib.mgc_supports(3, 3, 0, 0) == 1
    assert lib.mgc_supports(3, 3, 7, 1) == 1
    assert lib.mgc_supports(3, 5, 0, 0) == 0
    assert lib.mgc_supports(2, 4, 2, 0) == 1


def test_invalid_arguments_rejected_without_gpu():
    lib = _lib.load()
    assert lib.mgc_euler_rhs(None, None, None, None, None, 0, None, None, None) == -1
    assert lib.mgc_rk4_stage(-1, None, None, None, None, None, 0, 0.1, None) == -1


_QUERIES = {"mgc_version", "mgc_supports", "mgc_supports_hex", "mgc_mlp_nparams",
            "mgc_rhs_split_workspace_bytes", "mgc_mlp_train_workspace_bytes",
            "mgc_ns_operator_noalloc_capacity", "mgc_fp64_probe_flops",
            "mgc_operator_workspace_bytes", "mgc_set_gradient_kernel",
            "mgc_get_gradient_kernel"}


def test_gradient_kernel_option_without_gpu():
    lib = _lib.load()
    assert lib.mgc_get_gradient_kernel() == 0
    assert lib.mgc_set_gradient_kernel(7) == -1
    assert lib.mgc_set_gradient_kernel(-1) == -1
    assert lib.mgc_get_gradient_kernel() == 0
    assert lib.mgc_set_gradient_kernel(1) == 0
    assert lib.mgc_get_gradient_kernel() == 1
    assert lib.mgc_set_gradient_kernel(0) == 0


def _null_call_script():
    """Python source that calls every non-query entry point with null
    pointers, zero dimensions and negative sizes and prints the codes."""
    return r'''
import ctypes as C, json, sys
sys.path.insert(0, %r)
from mirgecom_b200 import _lib
lib = _lib.load()
out = {}
for name, (args, res) in _lib._SIGNATURES.items():
    if name in %r:
        continue
    vals = []
    for a in args:
        if a is C.c_void_p:
            vals.append(None)
        elif a is C.c_int64:
            vals.append(-1)
        elif a in (C.c_float, C.c_double):
            vals.append(0.0)
        elif a is C.c_size_t:
            vals.append(0)
        else:
            vals.append(0)
    out[name] = getattr(lib, name)(*vals)
print(json.dumps(out))
''' % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))), sorted(_QUERIES))


def test_every_entry_point_rejects_null_arguments():
    """Null pointers, zero dimensions and negative sizes come back as a
    negative code from every entry point, before any device work, in a child
    process (so that a crash would fail this test, not the run)."""
    import json
    import subprocess
    import sys
    res = subprocess.run([sys.executable, "-c", _null_call_script()], capture_output=True,
                         text=True, timeout=120)
    assert res.returncode == 0, res.stderr[-2000:]
    codes = json.loads(res.stdout.strip().splitlines()[-1])
    assert set(codes) == set(_lib.exported_symbols()) - _QUERIES
    bad = {k: v for k, v in codes.items() if v >= 0}
    assert not bad, bad


def test_noalloc_capacity_edge_without_gpu():
    """The allocation-free NS entry point accepts a mesh whose gradient
    buffer fills its fixed array exactly and rejects one element more
    (MGC_E_TOO_LARGE), checked before any device work: the child process
    sees no GPU, so the accepted size stops at the device lookup
    (MGC_E_CUDA) and nothing is launched."""
    import json
    import subprocess
    import sys
    script = r'''
import ctypes as C, json, sys
sys.path.insert(0, %r)
from mirgecom_b200 import _lib
lib = _lib.load()
cap = lib.mgc_ns_operator_noalloc_capacity()
gas = _lib.GasStruct()
gas.eos_kind = _lib.EOS_IDEAL
gas.nspecies = 0
mesh = _lib.MeshStruct()
mesh.dim, mesh.order, mesh.elem_kind = 3, 3, 0
per_elem = (3 + 2 + 1) * 3 * 20          # (Nc+1) * dim * Np doubles per element
out = {}
for key, nel in (("edge", cap // per_elem), ("over", cap // per_elem + 1)):
    mesh.nelem = nel
    out[key] = lib.mgc_ns_operator_noalloc(C.byref(mesh), C.byref(gas), None, None, None,
                                           None, 0, 0, None, None, None)
bad = _lib.MeshStruct()
bad.dim, bad.order, bad.elem_kind, bad.nelem = 3, 3, 7, 10
out["bad_kind"] = lib.mgc_ns_operator_noalloc(C.byref(bad), C.byref(gas), None, None, None,
                                              None, 0, 0, None, None, None)
bad.elem_kind, bad.order = 0, 1 << 20
out["huge_order"] = lib.mgc_ns_operator_noalloc(C.byref(bad), C.byref(gas), None, None,
                                                None, None, 0, 0, None, None, None)
print(json.dumps(out))
''' % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    res = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True,
                         timeout=120, env=env)
    assert res.returncode == 0, res.stderr[-2000:]
    codes = json.loads(res.stdout.strip().splitlines()[-1])
    assert codes["edge"] == -4, codes          # past the size check, no device
    assert codes["over"] == -5, codes          # MGC_E_TOO_LARGE
    assert codes["bad_kind"] == -1, codes      # invalid element kind
    assert codes["huge_order"] == -2, codes    # unsupported order, no overflow
