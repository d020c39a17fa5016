"""Benchmark of the DG Navier-Stokes right-hand side on B200.

One step = one RHS evaluation of the named workload over its whole mesh
(the hot path: temperature solve where the gas is a mixture, gradient pass,
divergence pass).  The metric is DOF-RHS evaluations per second:
(nodes x conserved fields) x RHS evaluations / second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tgv_p3_tet24]

Timing: CUDA events around each step on the launching stream, after W
warm-up steps; the L2 is flushed (a 512 MiB write) between timed steps and
the flush is outside the events.  Under torchrun every rank runs its own
replica of the workload (the RHS of one mesh partition needs no collective)
and the reported time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


# {{{ workloads

WORKLOADS = {
    "tgv_p3_tet24": dict(
        desc="3-D viscous Taylor-Green vortex, periodic [-pi,pi]^3, 24^3 hexes x 6 tets "
             "(82,944 tets), order 3 (20 nodes/tet), ideal gas gamma=1.4, Mach 0.1, "
             "Re 1600, Pr 0.71, Rusanov + BR1, plain FP64",
        n=24, order=3, kind="tgv"),
}


def build_workload(name, device):
    import torch

    from mirgecom_b200.discretization import Discretization
    from mirgecom_b200.eos import IdealSingleGas
    from mirgecom_b200.gas_model import GasModel
    from mirgecom_b200.initializers import (taylor_green_state,
                                            taylor_green_transport_params)
    from mirgecom_b200.mesh import generate_box_mesh
    from mirgecom_b200.transport import SimpleTransport
    w = WORKLOADS[name]
    mesh = generate_box_mesh((-np.pi,) * 3, (np.pi,) * 3, (w["n"],) * 3,
                             periodic=(True,) * 3)
    dcoll = Discretization(mesh, w["order"], device=device)
    x = [t for t in dcoll.nodes(device)]
    cv = taylor_green_state(x)
    gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
        **taylor_green_transport_params()))
    torch.cuda.synchronize()
    return dcoll, cv, gas


def algorithmic_bytes(dcoll, nc, s=8):
    """Compulsory HBM bytes per launch of each kernel of one NS RHS.

    grad: read q (Nc) + write grad ((Nc+1) d) per node, + rx and face
    pairing per element.  rhs: read q (Nc) + grad ((Nc+1) d), write rhs
    (Nc) per node, + rx and face pairing per element.
    """
    d = dcoll.dim
    nn = dcoll.nelements * dcoll.refel.nnodes
    geo = dcoll.nelements * (d * d * s + dcoll.nfaces * 4)
    grad = nn * (nc + (nc + 1) * d) * s + geo
    rhs = nn * (nc + (nc + 1) * d + nc) * s + geo
    return {"grad": grad, "rhs": rhs}

# }}}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        if not getattr(self, "lines", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except (ValueError, IndexError):
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_baseline(name, seconds=10.0):
    """The float64 oracle (numpy) on a bounded sample of the same physics."""
    from mirgecom_b200.discretization import Discretization
    from mirgecom_b200.mesh import generate_box_mesh
    from oracle import dg as odg
    from oracle import physics as oph
    w = WORKLOADS[name]
    n_sample = 6
    mesh = generate_box_mesh((-np.pi,) * 3, (np.pi,) * 3, (n_sample,) * 3,
                             periodic=(True,) * 3)
    d = Discretization(mesh, w["order"])
    od = odg.OracleDisc(mesh, d.refel)
    x = od.nodes
    u = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
    v = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    p = 1 / (1.4 * 0.01) + (np.cos(2 * x[0]) + np.cos(2 * x[1])) * (np.cos(2 * x[2]) + 2) / 16
    q = np.array([np.ones_like(u), p / 0.4 + 0.5 * (u * u + v * v), u, v, 0 * u])
    mu = 1 / 1600
    otr = oph.SimpleTransportParams(viscosity=mu, thermal_conductivity=mu * 1004.85 / 0.71)
    gas = oph.IdealGas()
    odg.ns_operator(od, oph.make_fluid_state(q, gas, otr, 3), gas, otr, {})
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < seconds or reps < 2:
        odg.ns_operator(od, oph.make_fluid_state(q, gas, otr, 3), gas, otr, {})
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    dof = q.size
    return {"value": dof / dt, "unit": "DOF-RHS/s", "cores": 1, "kind": "port",
            "sample": f"{n_sample}^3 x 6 tets ({mesh.nelements} tets, {dof} DOF), same "
                      f"physics and order, {reps} RHS evaluations, numpy float64 oracle"}


def run_reference(args):
    rank, world, _ = _dist_env()
    if rank != 0:
        return
    t0 = time.perf_counter()
    res = cpu_baseline(args.workload, seconds=max(5.0, 2.0 * args.steps))
    line = {"impl": "reference", "metric": "DOF-RHS evals/s", "value": res["value"],
            "unit": "DOF-RHS/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "sample": res["sample"]},
            "cpu_baseline": {"value": res["value"], "unit": res["unit"],
                             "cores": res["cores"], "kind": res["kind"],
                             "sample": res["sample"]},
            "e2e": {"value": res["value"], "unit": "DOF-RHS/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from mirgecom_b200 import runtime
    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import make_fluid_state
    from mirgecom_b200.navierstokes import ns_operator

    rank, world, local = _dist_env()
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dcoll, cv, gas = build_workload(args.workload, dev)
    q = cv.q.contiguous()
    nc = q.shape[0]
    dof = q.numel()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(qq):
        st = make_fluid_state(ConservedVars(qq, 3), gas)
        return ns_operator(dcoll, gas, st, {})

    for _ in range(args.warmup):
        step(q)
    torch.cuda.synchronize()
    if runtime.read_status(dcoll, dev) != 0:
        raise RuntimeError("device status error during warm-up")

    # timed region: K steps, per-step events, L2 flush between steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    kev = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.fill_(float(i))
            kern = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[i][0].record(stream)
            runtime.ns_rhs(dcoll, make_fluid_state(ConservedVars(q, 3), gas), gas, {}, 0.0,
                           0, events=kern)
            ev[i][1].record(stream)
            kev.append(kern)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    grad_ms = [k[0].elapsed_time(k[1]) for k in kev]
    rhs_ms = [k[1].elapsed_time(k[2]) for k in kev]
    total_ms = float(np.sum(step_ms))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * dof * args.steps / (total_ms / 1e3)

    # end to end through the public API with host buffers
    q_host = q.cpu().pin_memory()
    out_host = torch.empty_like(q_host).pin_memory()
    qd = torch.empty_like(q)
    e2e_ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    for _ in range(2):
        qd.copy_(q_host, non_blocking=True)
        out_host.copy_(step(qd).q, non_blocking=True)
    torch.cuda.synchronize()
    e2e_ms = 0.0
    for i in range(args.steps):
        flush.fill_(float(i))
        e2e_ev[0].record(stream)
        qd.copy_(q_host, non_blocking=True)
        out_host.copy_(step(qd).q, non_blocking=True)
        e2e_ev[1].record(stream)
        torch.cuda.synchronize()
        e2e_ms += e2e_ev[0].elapsed_time(e2e_ev[1])
    e2e_value = world * dof * args.steps / (e2e_ms / 1e3)

    # roofline of the dominant kernel
    hbm, peak_kind = _peaks()
    ab = algorithmic_bytes(dcoll, nc)
    kt = {"grad": float(np.mean(grad_ms)), "rhs": float(np.mean(rhs_ms))}
    top = max(kt, key=kt.get)
    achieved = ab[top] / (kt[top] / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(args.workload, {}).get(top)

    if rank != 0:
        return
    cpu = cpu_baseline(args.workload) if world == 1 and not args.no_cpu else None
    line = {
        "metric": "DOF-RHS evals/s", "value": value, "unit": "DOF-RHS/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"],
                   "elements": dcoll.nelements, "dof": dof,
                   "l2": "flushed between timed steps (512 MiB write, untimed)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "DOF-RHS/s",
                "h2d_bytes_per_step": q.numel() * 8, "d2h_bytes_per_step": q.numel() * 8},
        "gpu_launches": 2 * args.steps,
        "kernels_ms": kt,
        "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                     "algorithmic_bytes": ab[top], "traffic": traffic},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tgv_p3_tet24", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
