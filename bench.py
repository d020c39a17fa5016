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
    "reacting_p3_tet80": dict(
        desc="3-D reacting Navier-Stokes, uiuc_7sp ethylene/air (7 species, 3 Arrhenius "
             "reactions, NASA-7), periodic [0,2pi]^3 m box, 80^3 hexes x 6 tets "
             "(3,072,000 tets), order 3 (20 nodes/tet), 61.4M nodes x 12 fields; seeded "
             "smooth random T in [300,2500] K, p = 101325 +-5%, Dirichlet(2) mass "
             "fractions, |v| <= 10 m/s; SimpleTransport mu = kappa = D = 1e-5; Newton "
             "seeded with the step-start temperature; reactions on",
        n=80, order=3, kind="reacting"),
    "reacting_p2_tet40": dict(
        desc="3-D reacting Navier-Stokes, uiuc_7sp, 40^3 hexes x 6 tets (384,000 tets), "
             "order 2 (10 nodes/tet), same fields and models as reacting_p3_tet80",
        n=40, order=2, kind="reacting"),
    "reacting_p3_tet20": dict(
        desc="3-D reacting Navier-Stokes, uiuc_7sp, 20^3 hexes x 6 tets (48,000 tets), "
             "order 3 (20 nodes/tet): the reacting_p3_tet80 physics at a size for profiling",
        n=20, order=3, kind="reacting"),
    "reacting_p3_tet32": dict(
        desc="3-D reacting Navier-Stokes, uiuc_7sp, 32^3 hexes x 6 tets (196,608 tets), "
             "order 3 (20 nodes/tet, 3.9M nodes): the reacting_p3_tet80 physics with inputs "
             "larger than L2 and a few GB on the device, for kernel captures",
        n=32, order=3, kind="reacting"),
    "tgv_p4_hex48": dict(
        desc="3-D viscous Taylor-Green vortex, periodic [-pi,pi]^3, 48^3 tensor-product "
             "hexahedra (110,592), order 4 (125 nodes/element, 13.8M nodes), ideal gas "
             "gamma=1.4, Mach 0.1, Re 1600, Pr 0.71, Rusanov + BR1; sum-factorised "
             "contractions",
        n=48, order=4, kind="tgv", elem="hypercube"),
    "tgv_p3_tet24": dict(
        desc="3-D viscous Taylor-Green vortex, periodic [-pi,pi]^3, 24^3 hexes x 6 tets "
             "(82,944 tets), order 3 (20 nodes/tet), ideal gas gamma=1.4, Mach 0.1, "
             "Re 1600, Pr 0.71, Rusanov + BR1",
        n=24, order=3, kind="tgv"),
}
DEFAULT_WORKLOAD = "reacting_p3_tet80"


def build_workload(name, device):
    import torch

    from mirgecom_b200.discretization import Discretization
    from mirgecom_b200.eos import IdealSingleGas, PyrometheusMixture
    from mirgecom_b200.gas_model import GasModel
    from mirgecom_b200.initializers import (reacting_mixture_state, taylor_green_state,
                                            taylor_green_transport_params)
    from mirgecom_b200.mesh import generate_box_mesh
    from mirgecom_b200.thermochemistry import UIUC_7SP
    from mirgecom_b200.transport import SimpleTransport
    w = WORKLOADS[name]
    elem = w.get("elem", "simplex")
    if w["kind"] == "tgv":
        mesh = generate_box_mesh((-np.pi,) * 3, (np.pi,) * 3, (w["n"],) * 3,
                                 kind=elem, periodic=(True,) * 3)
    else:
        mesh = generate_box_mesh((0.0,) * 3, (2 * np.pi,) * 3, (w["n"],) * 3,
                                 kind=elem, periodic=(True,) * 3)
    dcoll = Discretization(mesh, w["order"], device=device)
    x = [t for t in dcoll.nodes(device)]
    if w["kind"] == "tgv":
        cv = taylor_green_state(x)
        gas = GasModel(eos=IdealSingleGas(), transport=SimpleTransport(
            **taylor_green_transport_params()))
        tseed = None
    else:
        cv, tseed = reacting_mixture_state(x, UIUC_7SP, seed=0)
        gas = GasModel(eos=PyrometheusMixture(UIUC_7SP, temperature_niter=5),
                       transport=SimpleTransport(viscosity=1e-5, thermal_conductivity=1e-5,
                                                 species_diffusivity=[1e-5] * 7))
        # the step-start temperature: the exact temperature of a nearby state
        tseed = tseed + 2.0
    del x
    torch.cuda.synchronize()
    return dcoll, cv, gas, tseed


def contraction_flops(dcoll, nc):
    """Tensor-core flops per launch of the volume and face kernels on
    simplices (dense reference matrices, inverse mass folded in): volume =
    the gradient pass (Nc+1) d 2 Np^2 + its lift (Nc+1) 2 Np Nf Nfp, plus the
    volume divergence Nc d 2 Np^2; face = the lift Nc 2 Np Nf Nfp; per
    element.  The three-kernel layout splits volume into grad (the gradient
    pass) and flux_volume (the divergence)."""
    d = dcoll.dim
    npn = dcoll.refel.nnodes
    nfn = dcoll.nfaces * dcoll.nface_nodes
    e = dcoll.nelements
    grad = (nc + 1) * d * 2 * npn * npn + (nc + 1) * 2 * npn * nfn
    div = nc * d * 2 * npn * npn
    return {"volume": float(e * (grad + div)), "grad": float(e * grad),
            "flux_volume": float(e * div), "face": float(e * nc * 2 * npn * nfn)}


KERNEL_NAMES = {"state": "k_mixture_state*", "grad": "k_grad*", "node_flux": "k_node_flux",
                "surface": "k_surface", "volume": "k_volume", "flux_volume": "k_flux_volume",
                "face": "k_face"}


def algorithmic_bytes(dcoll, nc, s=8, mixture=False):
    """Compulsory HBM bytes per launch of each kernel of one NS RHS.

    state (mixture): read q (Nc) and the seed, write T (1, plus the operator
    temperature on the float64 path).  grad: read q (Nc) [+ T], write grad
    ((Nc+1) d) per node.  node_flux: read q, grad [+ T, T_src], write the
    flux record (FW values: Nc d fluxes, p, c, gamma, |v| + c, padded) [+ Ns
    sources].  surface: read the records, q [+ sources], write the rhs (Nc).
    rhs: the divergence pass as one (q + grad + rhs [+ 2 T] per node, no
    records).  Plus rx and the face pairing per element where used.
    """
    d = dcoll.dim
    nn = dcoll.nelements * dcoll.refel.nnodes
    geo = dcoll.nelements * (d * d * s + dcoll.nfaces * 4)
    t_in = 1 if mixture else 0
    ns = nc - d - 2
    fw = -(-(nc * d + 4) // 4) * 4
    nfn = dcoll.nfaces * dcoll.nface_nodes
    tw = -(-(nc + 4) // 4) * 4
    ne = dcoll.nelements
    out = {
        # volume: read q [+ T (+ source T on the float64 path)], write the
        # volume part of the rhs, the face-node records (Nf Nfp x TW per
        # element) and the node-0 shifts (Nf Nc per element)
        "volume": nn * (nc + t_in * (2 if s == 8 else 1) + nc) * s
                  + ne * (nfn * tw + dcoll.nfaces * nc) * s + geo,
        # face: read the own records and the node-0 shifts, q at the own face
        # nodes, the rhs, write the rhs (the neighbours' records and q come
        # from L2 when the element order keeps neighbours close)
        "face": ne * (nfn * tw + dcoll.nfaces * nc) * s + nn * (nc + 2 * nc) * s + geo,
        "grad": nn * (nc + t_in + (nc + 1) * d) * s + geo,
        # flux-volume: the volume kernel's traffic plus reading the gradients
        "flux_volume": nn * (nc + t_in * (2 if s == 8 else 1) + nc + (nc + 1) * d) * s
                       + ne * (nfn * tw + dcoll.nfaces * nc) * s + geo,
        "node_flux": nn * (nc + (nc + 1) * d + 2 * t_in + fw + (ns if mixture else 0)) * s,
        "surface": nn * (fw + nc + (ns if mixture else 0) + nc) * s + geo,
        "rhs": nn * (nc + (nc + 1) * d + nc + 2 * t_in) * s + geo,
    }
    if mixture:
        out["state"] = nn * (nc + 1 + (2 if s == 8 else 1)) * s
    return out

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


def _max_over_ranks(xs, device):
    """Element-wise maximum of the float list *xs* over all ranks (the
    device times of a multi-process run); *xs* itself when not distributed.
    Every rank must call it at the same point."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(x) for x in xs]
    t = torch.tensor([float(x) for x in xs], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def _oracle_setup(name):
    """Oracle discretization and gas of a bounded sample of the workload
    (numpy only; no torch, so spawned CPU workers stay light)."""
    from mirgecom_b200.discretization import Discretization
    from mirgecom_b200.mesh import generate_box_mesh
    from mirgecom_b200.thermochemistry import UIUC_7SP
    from oracle import dg as odg
    from oracle import physics as oph
    w = WORKLOADS[name]
    if w["kind"] == "tgv":
        n_sample = 6
        mesh = generate_box_mesh((-np.pi,) * 3, (np.pi,) * 3, (n_sample,) * 3,
                                 kind=w.get("elem", "simplex"), periodic=(True,) * 3)
        mu = 1 / 1600
        otr = oph.SimpleTransportParams(viscosity=mu, thermal_conductivity=mu * 1004.85 / 0.71)
        gas = oph.IdealGas()
    else:
        n_sample = 3
        mesh = generate_box_mesh((0.0,) * 3, (2 * np.pi,) * 3, (n_sample,) * 3,
                                 periodic=(True,) * 3)
        otr = oph.SimpleTransportParams(viscosity=1e-5, thermal_conductivity=1e-5,
                                        species_diffusivity=(1e-5,) * 7)
        gas = oph.MixtureGas(UIUC_7SP, temperature_niter=5)
    d = Discretization(mesh, w["order"])
    od = odg.OracleDisc(mesh, d.refel)
    return od, gas, otr, mesh.nelements, n_sample


def _oracle_state(name, od):
    """The workload's state on the sample's nodes: (q, temperature seed)."""
    w = WORKLOADS[name]
    x = od.nodes
    if w["kind"] == "tgv":
        u = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
        v = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
        p = 1 / (1.4 * 0.01) + (np.cos(2 * x[0]) + np.cos(2 * x[1])) * (np.cos(2 * x[2]) + 2) / 16
        q = np.array([np.ones_like(u), p / 0.4 + 0.5 * (u * u + v * v), u, v, 0 * u])
        return q, None
    import torch

    from mirgecom_b200.initializers import reacting_mixture_state
    from mirgecom_b200.thermochemistry import UIUC_7SP
    cv, t = reacting_mixture_state([torch.from_numpy(x[i]) for i in range(3)], UIUC_7SP, seed=0)
    return cv.q.numpy(), t.numpy() + 2.0


def _oracle_rhs(od, q, tseed, gas, otr):
    from oracle import dg as odg
    from oracle import physics as oph
    st = oph.make_fluid_state(q, gas, otr, 3, temperature_seed=tseed)
    rhs = odg.ns_operator(od, st, gas, otr, {})
    if isinstance(gas, oph.MixtureGas):
        rhs = rhs + oph.species_source_terms(gas, q, st["temperature"], 3)
    return rhs


def _time_oracle(name, q, tseed, seconds):
    """RHS evaluations of the oracle on the sample for about *seconds*."""
    od, gas, otr, nel, n_sample = _oracle_setup(name)
    _oracle_rhs(od, q, tseed, gas, otr)
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < seconds or reps < 2:
        _oracle_rhs(od, q, tseed, gas, otr)
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    return q.size / dt, reps, nel, n_sample


def cpu_baseline(name, seconds=10.0):
    """The float64 oracle (numpy, one process) on a bounded sample of the
    same physics and order; the sample is stated in the result."""
    od, _, _, _, _ = _oracle_setup(name)
    q, tseed = _oracle_state(name, od)
    value, reps, nel, n_sample = _time_oracle(name, q, tseed, seconds)
    return {"value": value, "unit": "DOF-RHS/s", "cores": 1, "kind": "port",
            "sample": f"{n_sample}^3 mesh ({nel} elements, {q.size} DOF), same physics, "
                      f"element and "
                      f"order as {name}, {reps} RHS evaluations, numpy float64 oracle, "
                      f"one process"}


def _reference_worker(job):
    name, q, tseed, seconds = job
    return _time_oracle(name, q, tseed, seconds)


def run_reference(args):
    """The reference's CPU path (restated by the oracle: the reference's own
    runtime is not installed) on every host core: one spawned process per
    core, each evaluating the RHS of the bounded sample; the value is the sum
    of their rates."""
    rank, world, _ = _dist_env()
    if rank != 0:
        return
    t0 = time.perf_counter()
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    od, _, _, _, _ = _oracle_setup(args.workload)
    q, tseed = _oracle_state(args.workload, od)
    seconds = max(5.0, 2.0 * args.steps)
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(ncores) as pool:
        res = pool.map(_reference_worker, [(args.workload, q, tseed, seconds)] * ncores)
    value = float(sum(r[0] for r in res))
    reps = sum(r[1] for r in res)
    _, _, nel, n_sample = res[0]
    sample = (f"{n_sample}^3 mesh ({nel} elements, {q.size} DOF), same physics, element "
              f"and order as {args.workload}, {reps} RHS evaluations over {ncores} processes, numpy "
              f"float64 oracle (the reference's CPU path restated; its runtime is not "
              f"installed)")
    line = {"impl": "reference", "metric": "DOF-RHS evals/s", "value": value,
            "unit": "DOF-RHS/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "sample": sample},
            "cpu_baseline": {"value": value, "unit": "DOF-RHS/s", "cores": ncores,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "DOF-RHS/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}
    print(json.dumps(line), flush=True)


def _rhs_call(dcoll, gas, q, tseed, events=None):
    """One RHS evaluation of the workload through the public API."""
    from mirgecom_b200 import runtime
    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import make_fluid_state
    if events:
        events[0].record()
    st = make_fluid_state(ConservedVars(q, 3), gas, temperature_seed=tseed)
    src = st.temperature if st.is_mixture else None
    rhs, _ = runtime.ns_rhs(dcoll, st, gas, {}, 0.0, 0, source_temperature=src,
                            events=events[1:] if events else None)
    return rhs


def _time_form(dcoll, gas, q, tseed, steps, warmup, flush, stream):
    import torch

    from mirgecom_b200 import runtime
    path = runtime._path(dcoll, gas)
    vf = path == "volume_face"
    three = path == "gradient_volume_face"
    nev = 4 if vf else 5
    for _ in range(warmup):
        _rhs_call(dcoll, gas, q, tseed)
    torch.cuda.synchronize()
    evs = []
    for i in range(steps):
        flush.fill_(float(i))
        # start | state | volume | face,  start | state | grad | flux_volume | face
        # or  start | state | grad | node_flux | surface
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(nev)]
        _rhs_call(dcoll, gas, q, tseed, events=ev)
        evs.append(ev)
    torch.cuda.synchronize()
    step_ms = [e[0].elapsed_time(e[-1]) for e in evs]

    def mean(i, j):
        return float(np.mean([e[i].elapsed_time(e[j]) for e in evs]))
    if vf:
        kern = {"state": mean(0, 1), "volume": mean(1, 2), "face": mean(2, 3),
                "rhs": mean(1, 3)}
    elif three:
        kern = {"state": mean(0, 1), "grad": mean(1, 2), "flux_volume": mean(2, 3),
                "face": mean(3, 4), "rhs": mean(1, 4)}
    else:
        kern = {"state": mean(0, 1), "grad": mean(1, 2), "node_flux": mean(2, 3),
                "surface": mean(3, 4), "rhs": mean(2, 4)}
    return float(np.sum(step_ms)), kern


def _newton_stats(dcoll, gas, q, tseed):
    """Float32 Newton iterations per node for one temperature solve."""
    import torch

    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import make_fluid_state
    it = torch.zeros(q[0].shape, dtype=torch.int32, device=q.device)
    make_fluid_state(ConservedVars(q, 3), gas, temperature_seed=tseed, newton_iterations=it)
    fb = it >= 1000
    base = torch.where(fb, it - 1000, it)
    warm = base >= 100            # learned form: network skipped for a warm warp
    base = torch.where(warm, base - 100, base).float()
    return {"mean": float(base.mean()), "max": int(base.max()),
            "fallback_nodes": int(fb.sum()),
            "network_skipped_nodes": int(warm.sum()), "nodes": int(it.numel())}


def _train_guess(dev, seed=0, steps=2000, samples=1 << 20):
    import torch

    from mirgecom_b200.learned_guess import TemperatureMLP
    from mirgecom_b200.thermochemistry import UIUC_7SP
    t0 = time.perf_counter()
    net = TemperatureMLP(dev, seed=seed)
    e, y, t = TemperatureMLP.training_pairs(UIUC_7SP, samples, dev, seed=seed)
    hist = net.fit(e, y, t, steps=steps, batch=min(65536, samples), lr=3e-3, seed=seed)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    from mirgecom_b200.fluid import ConservedVars
    e2, y2, t2 = TemperatureMLP.training_pairs(UIUC_7SP, 1 << 16, dev, seed=seed + 1)
    q = torch.cat([torch.ones_like(e2)[None], e2[None],
                   torch.zeros((3, e2.numel()), dtype=torch.float64, device=dev), y2])
    guess = net.predict(ConservedVars(q.float().contiguous(), 3))
    rms = float(((guess.double() - t2) ** 2).mean().sqrt())
    return net, {"samples": samples, "steps": steps, "train_s": train_s,
                 "loss_first": hist[0], "loss_final": hist[-1], "heldout_rms_K": rms}


def _end_of_run(dcoll, gas, q64, nsteps, n_axis):
    """*nsteps* RK4 steps of the float64 form and of the mixed form (float64
    RK accumulation, float32 right-hand sides) from the same state: the
    per-field relative L2 difference at the end, next to how far the state
    moved.  The float64 device path stands in for the oracle at this size (it
    matches the oracle to 1e-12 in the parity tests)."""
    import torch

    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import make_fluid_state
    from mirgecom_b200.integrators import rk4_step, rk4_step_mixed
    from mirgecom_b200.navierstokes import ns_operator
    h = 2 * np.pi / n_axis
    p = dcoll.order
    # acoustic CFL 0.3 with the (p+1)^2 DG scaling: |u| + c <= 11 at Mach 0.1
    dt = 0.3 * h / (p + 1) ** 2 / 11.0

    def rhs(t, cv):
        return ns_operator(dcoll, gas, make_fluid_state(cv, gas), {})

    s64 = ConservedVars(q64.clone(), 3)
    shi = ConservedVars(q64.clone(), 3)
    slo = None
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(nsteps):
        s64 = rk4_step(s64, i * dt, dt, rhs)
        shi, slo = rk4_step_mixed(shi, i * dt, dt, rhs, slo)
    torch.cuda.synchronize()
    a, b, q0 = shi.q.cpu().numpy(), s64.q.cpu().numpy(), q64.cpu().numpy()

    def rel(x, y):
        # momentum components against the norm of the momentum field (the
        # Taylor-Green z momentum starts at zero)
        mom = np.linalg.norm(y[2:5].ravel())
        return [float(np.linalg.norm((x[c] - y[c]).ravel()) /
                      max(mom if 2 <= c < 5 else np.linalg.norm(y[c].ravel()), 1e-300))
                for c in range(y.shape[0])]
    return {"steps": nsteps, "dt": dt, "t_final": nsteps * dt,
            "fields": ["mass", "energy", "momentum_x", "momentum_y", "momentum_z"],
            "mixed_vs_fp64_rel_l2": rel(a, b), "fp64_change_rel_l2": rel(b, q0),
            "wall_s": time.perf_counter() - t0}


def chemical_time_scale(dcoll, gas, q64, t64):
    """Smallest chemical time scale of the state: min over nodes and species
    with Y_k > 1e-3 of rho Y_k / |W_k omega_k|, the sources taken as the
    difference of the float64 right-hand sides with and without them."""
    import torch

    from mirgecom_b200 import runtime
    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import make_fluid_state
    st = make_fluid_state(ConservedVars(q64, 3), gas, temperature_seed=t64)
    with_src, _ = runtime.ns_rhs(dcoll, st, gas, {}, 0.0, 0, source_temperature=st.temperature)
    without, _ = runtime.ns_rhs(dcoll, st, gas, {}, 0.0, 0)
    src = (with_src - without)[5:]
    rhoy = q64[5:]
    mask = (rhoy / q64[0]) > 1e-3
    tau = rhoy.abs() / src.abs().clamp_min(1e-300)
    return float(torch.where(mask, tau, torch.full_like(tau, float("inf"))).min())


def _end_of_run_mixture(dcoll, gas, gas_head, q64, t64, nsteps, dt=None):
    """*nsteps* RK4 steps of the reacting workload in the float64 form and in
    the headline form (mixed precision + learned guess: float64 RK
    accumulation, float32 right-hand sides) from the same state, species
    sources on, each form's temperature seeded with its own previous
    temperature.  dt (default) resolves the chemistry: the smallest chemical
    time scale of the initial state over 64.  The synthetic states ignite,
    and over longer horizons the flow itself amplifies float32-level
    differences (on the float64 oracle alone a 6e-8 perturbation of the
    initial state grows to 4.5e-6 over 200 steps of 5e-9 s, tests/
    end_of_run_sensitivity.py).  Returns the per-field relative L2 difference
    at the end and the temperatures' difference."""
    import torch

    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import make_fluid_state
    from mirgecom_b200.integrators import rk4_step, rk4_step_mixed
    from mirgecom_b200.navierstokes import ns_operator

    tau = chemical_time_scale(dcoll, gas, q64, t64)
    dt_rule = "given"
    if dt is None:
        dt = tau / 64
        dt_rule = "smallest chemical time scale / 64"

    def factory(g, box):
        def rhs(t, cv):
            st = make_fluid_state(cv, g, temperature_seed=box[0])
            return ns_operator(dcoll, g, st, {}, species_source_temperature=st.temperature)
        return rhs

    s64 = ConservedVars(q64.clone(), 3)
    shi = ConservedVars(q64.clone(), 3)
    slo = None
    b64 = [t64.clone()]
    b32 = [t64.to(torch.float32)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(nsteps):
        s64 = rk4_step(s64, i * dt, dt, factory(gas, b64))
        b64[0] = make_fluid_state(s64, gas, temperature_seed=b64[0]).temperature
        shi, slo = rk4_step_mixed(shi, i * dt, dt, factory(gas_head, b32), slo)
        b32[0] = make_fluid_state(slo, gas_head, temperature_seed=b32[0]).temperature
    torch.cuda.synchronize()
    a, b, q0 = shi.q.cpu().numpy(), s64.q.cpu().numpy(), q64.cpu().numpy()

    def rel(x, y):
        mom = np.linalg.norm(y[2:5].ravel())
        return [float(np.linalg.norm((x[c] - y[c]).ravel()) /
                      max(mom if 2 <= c < 5 else np.linalg.norm(y[c].ravel()), 1e-300))
                for c in range(y.shape[0])]
    ta, tb = b32[0].double().cpu().numpy(), b64[0].cpu().numpy()
    species = list(gas.eos.mechanism.species)
    return {"steps": nsteps, "dt": dt, "dt_rule": dt_rule, "tau_chem_min": tau,
            "t_final": nsteps * dt,
            "form": "mixed_learned vs plain_fp64",
            "fields": ["mass", "energy", "momentum_x", "momentum_y", "momentum_z"] +
                      [f"rho_{sp}" for sp in species],
            "mixed_vs_fp64_rel_l2": rel(a, b), "fp64_change_rel_l2": rel(b, q0),
            "temperature_rel_l2": float(np.linalg.norm(ta - tb) / np.linalg.norm(tb)),
            "wall_s": time.perf_counter() - t0}


def run_vortex(args):
    """The 2-D vortex configuration run to t = 1 (200 RK4 steps of 0.005)
    through the library's driver (mirgecom_b200.vortex) on the GPU, and the
    float64 oracle's same run on one host core: wall times, L2 errors
    against the exact solution, and the largest per-field difference of the
    two end states."""
    import torch

    from mirgecom_b200 import vortex
    rank, world, local = _dist_env()
    if rank != 0:
        return
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    vortex.run(device=dev, nsteps=2)            # warm-up: uploads, kernel set-up
    res = vortex.run(device=dev)
    q_gpu = res["q"].cpu().numpy()
    from mirgecom_b200.discretization import Discretization
    from mirgecom_b200.mesh import generate_box_mesh
    from oracle import dg as odg
    from oracle import physics as oph
    c = vortex.CASE
    mesh = generate_box_mesh(c["a"], c["b"], (c["nel"], c["nel"]))
    d = Discretization(mesh, c["order"])
    od = odg.OracleDisc(mesh, d.refel)
    init = vortex.Vortex2D(beta=c["beta"], center=c["center"], velocity=c["velocity"])

    def exact(x, t):
        return init([torch.from_numpy(x[i]) for i in range(2)], time=t).q.numpy()

    obnds = {"all": odg.PrescribedBoundary(exact)}

    def orhs(t, qq):
        return odg.euler_operator(od, oph.make_fluid_state(qq, oph.IdealGas(), None, 2),
                                  oph.IdealGas(), obnds, time=t)

    q = exact(od.nodes, 0.0)
    t0 = time.perf_counter()
    for i in range(res["steps"]):
        q = odg.rk4_step(q, i * c["dt"], c["dt"], orhs)
    cpu_wall = time.perf_counter() - t0
    r = q - exact(od.nodes, res["t"])
    det = np.abs(d.geometry.det)
    cpu_err = [float(np.sqrt(np.sum(det * np.einsum("ei,ij,ej->e", r[k], d.refel.mass, r[k]))))
               for k in range(4)]
    diff = [float(np.linalg.norm(q_gpu[k] - q[k]) / np.linalg.norm(q[k])) for k in range(4)]
    nrhs = 4 * res["steps"]
    fields = ["mass", "energy", "momentum_x", "momentum_y"]
    print(json.dumps({
        "case": "vortex2d_p3", "desc": "2-D Euler isentropic vortex, [0,10]x[-5,5], 16x16x2 "
        "triangles, order 3, beta 5 at (5,0), velocity (1,0), exact prescribed boundaries, "
        "Rusanov, RK4 dt 0.005 to t = 1", "steps": res["steps"], "t_final": res["t"],
        "gpu": {"wall_s": res["wall_s"], "dof_rhs_per_s": res["dof"] * nrhs / res["wall_s"],
                "l2_error_vs_exact": dict(zip(fields, res["l2_error"]))},
        "cpu_oracle": {"wall_s": cpu_wall, "cores": 1, "dof_rhs_per_s":
                       res["dof"] * nrhs / cpu_wall,
                       "l2_error_vs_exact": dict(zip(fields, cpu_err))},
        "end_state_rel_l2_gpu_vs_oracle": dict(zip(fields, diff))}), flush=True)


def run_ours(args):
    import torch.distributed as dist
    try:
        if _dist_env()[1] > 1:
            _run_partitioned(args)
        else:
            _run_ours(args)
    finally:
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


def _run_partitioned(args):
    """N GPUs, one process each: the workload's mesh split into N contiguous
    element blocks (strong scaling), each rank's right-hand side on its
    owned elements with the two halo exchanges per right-hand side (ghost
    rows of q and the temperature seed before, the ghosts' face records
    between the volume and face kernels) as NCCL point-to-point groups.
    Time per step = max over ranks of the CUDA-event time; value = the whole
    mesh's DOF x steps / that time.  e2e: each rank uploads its owned rows
    of q and the seed from pinned host memory and downloads its owned rows
    of the right-hand side every step."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from mirgecom_b200 import runtime
    from mirgecom_b200.eos import PyrometheusMixture
    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import GasModel, make_fluid_state
    from mirgecom_b200.partition import HaloExchange, PartitionedDiscretization

    rank, world, local = _dist_env()
    dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    mixture = w["kind"] == "reacting"
    dcoll, cv, gas, tseed = build_workload(args.workload, dev)
    dof_global = cv.q.numel()
    pd = PartitionedDiscretization(dcoll, rank, world, device=dev)
    halo = HaloExchange(pd, "dist")
    q64 = pd.scatter(cv.q).contiguous()
    t64 = pd.scatter(tseed[None])[0].contiguous() if mixture else None
    del cv, tseed
    q32 = q64.to(torch.float32)
    t32 = t64.to(torch.float32) if mixture else None
    gas_learn = None
    if mixture:
        net, _ = _train_guess(dev)
        eos = gas.eos
        gas_learn = GasModel(eos=PyrometheusMixture(eos.mechanism,
                                                    temperature_niter=eos.temperature_niter,
                                                    learned_guess=net),
                             transport=gas.transport)
    forms = [("plain_fp64", gas, q64, t64), ("mixed_plain_guess", gas, q32, t32)]
    if mixture:
        forms.append(("mixed_learned", gas_learn, q32, t32))
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step(g, q, t):
        halo.exchange_rows([q] if t is None else [q, t])
        st = make_fluid_state(ConservedVars(q, 3), g, temperature_seed=t)
        rhs, _ = runtime.ns_rhs(pd, st, g, {}, 0.0, 0,
                                source_temperature=st.temperature if mixture else None,
                                halo=halo)
        return rhs

    res = {}
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for name, g, q, t in forms:
            for _ in range(args.warmup):
                step(g, q, t)
            torch.cuda.synchronize()
            dist.barrier()
            total = 0.0
            for i in range(args.steps):
                flush.fill_(float(i))
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                step(g, q, t)
                e1.record()
                torch.cuda.synchronize()
                total += e0.elapsed_time(e1)
            res[name] = total
    dist.barrier()
    names = [f[0] for f in forms]
    tot = _max_over_ranks([res[n] for n in names], dev)
    values = {n: dof_global * args.steps / (ms / 1e3) for n, ms in zip(names, tot)}
    head = "mixed_learned" if mixture else "mixed_plain_guess"
    hg, hq, ht = (gas_learn if mixture else gas), q32, t32
    # end to end: owned rows in from pinned host memory, owned rows out
    nown = pd.nowned
    q_host = hq[:, :nown].cpu().pin_memory()
    t_host = ht[:nown].cpu().pin_memory() if ht is not None else None
    out_host = torch.empty_like(q_host).pin_memory()
    for it in range(2 + args.steps):
        if it == 2:
            torch.cuda.synchronize()
            dist.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record()
        hq[:, :nown].copy_(q_host, non_blocking=True)
        if t_host is not None:
            ht[:nown].copy_(t_host, non_blocking=True)
        rhs = step(hg, hq, ht)
        out_host.copy_(rhs[:, :nown], non_blocking=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = _max_over_ranks([e0.elapsed_time(e1)], dev)[0]
    status = runtime.read_status(pd, dev)
    status = int(_max_over_ranks([status], dev)[0])
    if rank != 0:
        return
    line = {
        "metric": "DOF-RHS evals/s", "value": values[head], "unit": "DOF-RHS/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot[names.index(head)] / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 state and pointwise math, tf32x3 contractions (f64 RK accumulation, "
                 "f64 Newton inputs and residual check)",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"],
                   "elements": dcoll.nelements, "dof": dof_global,
                   "form": head.replace("_", " "),
                   "l2": "flushed between timed steps (512 MiB write, untimed)",
                   "parallelism": f"element partition x{world}: halo exchange of q rows and "
                                  "face records, NCCL point-to-point"},
        "forms": {n: {"value": values[n], "ms_per_step": ms / args.steps}
                  for n, ms in zip(names, tot)},
        "mixed_over_fp64": values[head] / values["plain_fp64"],
        "e2e": {"value": dof_global * args.steps / (e2e_ms / 1e3), "unit": "DOF-RHS/s",
                "h2d_bytes_per_step": (q_host.numel() + (t_host.numel() if t_host is not None
                                                         else 0)) * 4 * world,
                "d2h_bytes_per_step": out_host.numel() * 4 * world,
                "schedule": "per rank: owned rows in, RHS with halo exchanges, owned rows out, "
                            "serialised on one stream"},
        "gpu_launches": ((1 if mixture else 0) + 2) * args.steps,
        "device_status": status,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def _run_ours(args):
    import torch
    import torch.distributed as dist

    from mirgecom_b200 import runtime
    from mirgecom_b200.eos import PyrometheusMixture
    from mirgecom_b200.gas_model import GasModel

    rank, world, local = _dist_env()
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    mixture = w["kind"] == "reacting"
    dcoll, cv, gas, tseed = build_workload(args.workload, dev)
    q64 = cv.q.contiguous()
    q32 = q64.to(torch.float32)
    t64 = tseed.contiguous() if mixture else None
    t32 = tseed.to(torch.float32) if mixture else None
    nc = q64.shape[0]
    dof = q64.numel()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    learned = None
    gas_learn = None
    if mixture:
        # the profiling run trains a short network: only the inference kernel is timed
        net, learned = (_train_guess(dev, steps=50, samples=1 << 16) if args.profile
                        else _train_guess(dev))
        eos = gas.eos
        gas_learn = GasModel(eos=PyrometheusMixture(eos.mechanism,
                                                    temperature_niter=eos.temperature_niter,
                                                    learned_guess=net),
                             transport=gas.transport)

    forms = [("plain_fp64", gas, q64, t64), ("mixed_plain_guess", gas, q32, t32)]
    if mixture:
        forms.append(("mixed_learned", gas_learn, q32, t32))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    res = {}
    with ClockSampler(local) as clk:
        for name, g, q, t in forms:
            res[name] = _time_form(dcoll, g, q, t, args.steps, args.warmup, flush, stream)
    if world > 1:
        dist.barrier()
    status = runtime.read_status(dcoll, dev)
    eor = None
    # RK4 steps of the end-of-run comparison: the configuration's own count
    # (reacting 200, Taylor-Green 100) unless given
    n_eor = args.end_of_run if args.end_of_run is not None else (
        200 if w["kind"] == "reacting" else 100)
    if n_eor > 0 and world == 1 and not args.profile:
        if mixture:
            eor = _end_of_run_mixture(dcoll, gas, gas_learn, q64, t64, n_eor,
                                      dt=args.end_of_run_dt)
        else:
            eor = _end_of_run(dcoll, gas, q64, n_eor, w["n"])
        status |= runtime.read_status(dcoll, dev)
    names = [f[0] for f in forms]
    tot = _max_over_ranks([res[n][0] for n in names], dev)
    values = {n: world * dof * args.steps / (ms / 1e3) for n, ms in zip(names, tot)}
    head = "mixed_learned" if gas_learn is not None else "mixed_plain_guess"
    hq, ht, hgas = q32, t32, (gas_learn if gas_learn is not None else gas)
    if args.profile:
        print(json.dumps({"profile_run": args.workload, "values": values,
                          "kernels_ms": {n: res[n][1] for n in names}}), flush=True)
        return

    if gas_learn is not None:
        from mirgecom_b200.initializers import reacting_mixture_state  # noqa: F401
        cold = torch.full_like(t32, 300.0)
        learned["newton_warm_seed"] = {
            "plain_guess": _newton_stats(dcoll, gas, q32, t32),
            "learned_guess": _newton_stats(dcoll, gas_learn, q32, t32)}
        learned["newton_cold_start_300K"] = {
            "plain_guess": _newton_stats(dcoll, gas, q32, cold),
            "learned_guess": _newton_stats(dcoll, gas_learn, q32, cold)}
        learned["fp64_plain_iterations"] = "fixed 5 (+5 for the operator states)"

    # the headline form's right-hand side against the float64 one on the
    # benchmark state (the float64 path matches the oracle at 1e-12 in the
    # parity tests): per-field relative L2, each field measured against the
    # larger of its own norm and its natural scale |F_c| / h (the inviscid
    # flux of field c over the element size; a low-Mach divergence is orders
    # of magnitude below its fluxes, and roundoff scales with the fluxes)
    from mirgecom_b200.fluid import ConservedVars
    from mirgecom_b200.gas_model import make_fluid_state
    r64 = _rhs_call(dcoll, gas, q64, t64).double()
    rmx = _rhs_call(dcoll, hgas, hq, ht).double()
    st = make_fluid_state(ConservedVars(q64, 3), gas, temperature_seed=t64)
    vel = q64[2:5] / q64[0]
    pres = st.pressure
    flux = [q64[0] * vel, (q64[1] + pres) * vel]
    flux += [q64[2 + i] * vel + pres * torch.eye(3, dtype=q64.dtype, device=dev)[i].view(
        3, *([1] * (q64.dim() - 1))) for i in range(3)]
    flux += [q64[5 + k] * vel for k in range(nc - 5)]
    h = 2 * np.pi / w["n"]
    rhs_err = [float(torch.linalg.vector_norm(rmx[c] - r64[c]) /
                     max(float(torch.linalg.vector_norm(r64[c])),
                         float(torch.linalg.vector_norm(flux[c])) / h, 1e-300))
               for c in range(nc)]
    del r64, rmx, st, vel, pres, flux

    # end to end through the public API with host buffers (headline form: the
    # float32 state goes in, the float32 right-hand side comes out), as a
    # pipelined driver runs it: step i's host-to-device copy, step i's RHS and
    # step i-1's device-to-host copy run on three streams, so the two copy
    # directions and the kernels overlap.  Every step still copies its whole
    # state in and its whole RHS out; the inputs (2.9 GB at 80^3) exceed L2.
    q_host = hq.cpu().pin_memory()
    out_host = [torch.empty_like(q_host).pin_memory() for _ in range(2)]
    qd = [torch.empty_like(hq) for _ in range(2)]
    # a driver holds the step-start temperature on the host with the state
    # and uploads it with q (mixtures)
    t_host = ht.cpu().pin_memory() if ht is not None else None
    td = [torch.empty_like(ht) for _ in range(2)] if ht is not None else [None, None]
    h2d, d2h = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def pipelined(nsteps):
        read_done = [None, None]      # compute has finished reading qd[b]
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(h2d)
        for i in range(nsteps):
            b = i % 2
            if read_done[b] is not None:
                h2d.wait_event(read_done[b])
            with torch.cuda.stream(h2d):
                qd[b].copy_(q_host, non_blocking=True)
                if t_host is not None:
                    td[b].copy_(t_host, non_blocking=True)
            loaded = torch.cuda.Event()
            loaded.record(h2d)
            stream.wait_event(loaded)
            rhs = _rhs_call(dcoll, hgas, qd[b], td[b])
            read_done[b] = torch.cuda.Event()
            read_done[b].record(stream)
            d2h.wait_event(read_done[b])
            with torch.cuda.stream(d2h):
                out_host[b].copy_(rhs, non_blocking=True)
            rhs.record_stream(d2h)
            del rhs
        ev1.record(d2h)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    pipelined(2)
    e2e_ms = _max_over_ranks([pipelined(args.steps)], dev)[0]
    e2e_value = world * dof * args.steps / (e2e_ms / 1e3)

    # roofline of the dominant kernel of the headline form
    hbm, peak_kind = _peaks()
    ab = algorithmic_bytes(dcoll, nc, s=4, mixture=mixture)
    k32 = res[head][1]
    kt = {k: v for k, v in k32.items() if k in ab and k != "rhs"}
    top = max(kt, key=kt.get)
    achieved = ab[top] / (kt[top] / 1e3) / 1e9
    ab64 = algorithmic_bytes(dcoll, nc, s=8, mixture=mixture)
    k64 = res["plain_fp64"][1]
    # the float64 path's compute roofline: its contractions run on the
    # float64 tensor cores (DMMA); the peak is measured here by a probe
    fp64 = None
    if "face" in k64 and world == 1:
        from mirgecom_b200 import fp64_peak
        pk = fp64_peak.measure(dev)
        fl = contraction_flops(dcoll, nc)
        fp64 = {"dmma_peak_tflops": pk["dmma_tflops"], "dfma_peak_tflops": pk["dfma_tflops"],
                "peak_how": pk["how"], "kernels": {}}
        for kname in ("volume", "grad", "flux_volume", "face"):
            if kname not in k64:
                continue
            tf = fl[kname] / (k64[kname] / 1e3) / 1e12
            fp64["kernels"][KERNEL_NAMES[kname]] = {
                "contraction_flops": fl[kname], "achieved_tflops": tf,
                "dmma_frac": tf / pk["dmma_tflops"]}
    kt64 = {k: v for k, v in k64.items() if k in ab64 and k != "rhs"}
    top64 = max(kt64, key=kt64.get)
    traffic = traffic64 = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f).get(args.workload, {})
        traffic = tj.get("mixed_" + top)
        traffic64 = tj.get("plain_fp64_" + top64)

    if rank != 0:
        return
    cpu = cpu_baseline(args.workload) if world == 1 and not args.no_cpu else None
    # this library's kernels per step: temperature (mixtures), gradient, and
    # the divergence pass (node flux + surface on the split path)
    from mirgecom_b200 import runtime as _rt
    per_step = (1 if mixture else 0) + {"volume_face": 2, "gradient_volume_face": 3}.get(
        _rt._path(dcoll, gas), 3)
    line = {
        "metric": "DOF-RHS evals/s", "value": values[head], "unit": "DOF-RHS/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot[names.index(head)] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state and pointwise math, tf32x3 contractions (f64 RK accumulation, "
                 "f64 Newton inputs and residual check)",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"],
                   "elements": dcoll.nelements, "dof": dof,
                   "form": head.replace("_", " "),
                   "l2": "flushed between timed steps (512 MiB write, untimed)",
                   "parallelism": f"replicas x{world}"},
        "forms": {n: {"value": values[n], "ms_per_step": ms / args.steps,
                      "kernels_ms": res[n][1]} for n, ms in zip(names, tot)},
        "mixed_over_fp64": values[head] / values["plain_fp64"],
        "kernels_ms": k32,
        "learned_guess": learned,
        "e2e": {"value": e2e_value, "unit": "DOF-RHS/s",
                "h2d_bytes_per_step": hq.numel() * 4 + (ht.numel() * 4 if ht is not None else 0),
                "d2h_bytes_per_step": hq.numel() * 4,
                "schedule": "pipelined: host-to-device copy of step i (state and, for "
                            "mixtures, the step-start temperature), RHS of step i and "
                            "device-to-host copy of step i-1 on separate streams; pinned host "
                            "buffers; inputs larger than L2"},
        "gpu_launches": per_step * args.steps,
        "gpu_launches_note": "headline form's timed steps; each form launches the same "
                             f"{per_step} kernels per step",
        "roofline": {"bound": "hbm", "kernel": KERNEL_NAMES.get(top, top), "phase": top,
                     "achieved": achieved, "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                     "algorithmic_bytes": ab[top], "traffic": traffic},
        "roofline_plain_fp64": {"kernel": KERNEL_NAMES.get(top64, top64), "phase": top64,
                                "achieved": ab64[top64] / (kt64[top64] / 1e3) / 1e9,
                                "frac": ab64[top64] / (kt64[top64] / 1e3) / 1e9 / hbm,
                                "algorithmic_bytes": ab64[top64], "traffic": traffic64,
                                "compute": fp64},
        "device_status": status,
        "rhs_rel_l2_vs_fp64": rhs_err,
        "end_of_run": eor,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--end-of-run", type=int, default=None,
                    help="after timing, run this many RK4 steps in the float64 and the "
                         "headline mixed form from the same state and report their "
                         "per-field difference (0: skip; default: 200 for the reacting "
                         "workloads, 100 for Taylor-Green, the configurations' counts)")
    ap.add_argument("--end-of-run-dt", type=float, default=None,
                    help="time step of the reacting end-of-run comparison (s); default: "
                         "the state's smallest chemical time scale / 64")
    ap.add_argument("--vortex-run", action="store_true",
                    help="run the 2-D vortex configuration to t = 1 on the GPU and with the "
                         "float64 oracle on one host core, and report both")
    ap.add_argument("--profile", action="store_true",
                    help="time the plain and mixed forms only (no network training, "
                         "end-to-end or CPU legs): the command profiled with ncu")
    ap.add_argument("--gradient-kernel", default="auto", choices=["auto", "mma_sync"],
                    help="gradient-pass kernel: the tcgen05 pipelined kernel where it "
                         "applies (auto) or the mma.sync kernel")
    args = ap.parse_args(argv)
    if args.impl != "reference" and args.gradient_kernel != "auto":
        from mirgecom_b200 import runtime
        runtime.set_gradient_kernel(args.gradient_kernel)
    if args.impl == "reference":
        run_reference(args)
    elif args.vortex_run:
        run_vortex(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
