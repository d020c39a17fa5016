"""Measured FP64 peaks of this GPU: the float64 path's compute roofline.

The float64 right-hand side is bound by the lower of HBM bandwidth and its
FP64 compute: contractions on the float64 tensor cores (DMMA) and pointwise
math on the FP64 FMA pipe.  Neither rate is published for this part, so
:func:`measure` times the library's probe kernels (``mgc_fp64_probe``:
independent instruction chains over a grid that fills every SM) with CUDA
events and returns TFLOP/s.
"""

from __future__ import annotations

from mirgecom_b200 import _lib


def measure(device, threads=256, iters=4096, repeats=5):
    """{"dfma_tflops": .., "dmma_tflops": ..}: best of *repeats* launches."""
    import torch
    lib = _lib.load()
    props = torch.cuda.get_device_properties(device)
    nblocks = props.multi_processor_count * 8
    sink = torch.empty(nblocks * threads, dtype=torch.float64, device=device)
    out = {}
    with torch.cuda.device(device):
        stream = _lib.stream_handle()
        for kind, name in ((0, "dfma_tflops"), (1, "dmma_tflops")):
            flops = lib.mgc_fp64_probe_flops(kind, nblocks, threads, iters)
            _lib.check(lib.mgc_fp64_probe(kind, nblocks, threads, 16, _lib.ptr(sink), stream),
                       "mgc_fp64_probe")
            best = None
            for _ in range(repeats):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                _lib.check(lib.mgc_fp64_probe(kind, nblocks, threads, iters, _lib.ptr(sink),
                                              stream), "mgc_fp64_probe")
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                best = ms if best is None else min(best, ms)
            out[name] = flops / (best / 1e3) / 1e12
            out[name.replace("tflops", "ms")] = best
    out["how"] = (f"{nblocks} blocks x {threads} threads, {iters} rounds of 8 independent "
                  "chains per thread (DFMA) / per warp (DMMA m8n8k4), best of "
                  f"{repeats}, CUDA events")
    return out
