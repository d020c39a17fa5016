"""How far float32-level perturbations grow over a reacting run (CPU, oracle).

The mixed-precision form stores the right-hand side's input and output in
float32 (relative rounding 6e-8).  Whether its end-of-run fields can stay
within 1e-6 of the float64 run depends on how much the reacting flow itself
amplifies perturbations of that size over the run.  This script measures it
with the float64 oracle alone on the reacting physics of the 40^3 order-2
workload (smooth random T in 300-2500 K, p = 101325 +- 5 %, Dirichlet(2)
mass fractions, |v| <= 10 m/s, uiuc_7sp with sources, SimpleTransport
1e-5) on a 3^3 x 6 tetrahedra order-2 mesh, 200 RK4 steps, against the
unperturbed float64 run:

  perturbed   the initial state times (1 + 6e-8 N(0,1)), then float64 throughout
  q_f32       every right-hand side evaluated from q rounded to float32
              (float64 arithmetic, species sources from the unrounded q)
  rhs_f32     every right-hand side rounded to float32
  src_f32in   species sources from T, rho, Y rounded to float32
  src_f32     species sources in float32 arithmetic from float32 inputs

It prints the largest per-field relative L2 difference at the end (momentum
against the momentum norm) and the smallest chemical time scale
rho Y_k / |W_k omega_k| (species above Y = 1e-3) of the initial state.

    python tests/end_of_run_sensitivity.py [--dt 5e-9] [--steps 200]
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

VARIANTS = ("perturbed", "q_f32", "rhs_f32", "src_f32in", "src_f32")


def _f32(a):
    return a.astype(np.float32).astype(np.float64)


def _rates_f32(mech, rho, t, y, zero_level=0.0):
    """Net molar production rates in float32 arithmetic (the oracle's
    net_production_rates with every operand rounded to float32)."""
    f = np.float32
    rho, t, y = rho.astype(f), t.astype(f), y.astype(f)
    w = mech.molecular_weights.astype(f).reshape((-1,) + (1,) * t.ndim)
    conc = rho * y / w
    conc = np.where(conc < f(zero_level), f(0), conc)
    sel = t[None] > mech.t_mid.astype(f).reshape((-1,) + (1,) * t.ndim)

    def coef(i):
        lo = mech.nasa_low[:, i].astype(f).reshape((-1,) + (1,) * t.ndim)
        hi = mech.nasa_high[:, i].astype(f).reshape((-1,) + (1,) * t.ndim)
        return np.where(sel, hi, lo)
    a = [coef(i) for i in range(7)]
    h = (a[0] + a[1] * t / f(2) + a[2] * t ** 2 / f(3) + a[3] * t ** 3 / f(4)
         + a[4] * t ** 4 / f(5) + a[5] / t)
    s = (a[0] * np.log(t) + a[1] * t + a[2] * t ** 2 / f(2) + a[3] * t ** 3 / f(3)
         + a[4] * t ** 4 / f(4) + a[6])
    g_rt = h - s
    rates = []
    for i in range(mech.nreactions):
        kf = np.exp(f(mech.log_a[i]) + f(mech.beta[i]) * np.log(t) - f(mech.t_act[i]) / t)
        rf = kf
        for k in range(mech.nspecies):
            if mech.orders_fwd[i, k] != 0:
                rf = rf * conc[k] ** f(mech.orders_fwd[i, k])
        r = rf
        if mech.reversible[i]:
            nu = (mech.nu_prod[i] - mech.nu_reac[i]).astype(f)
            dg = np.tensordot(nu, g_rt, axes=(0, 0))
            log_kc = -dg + nu.sum() * np.log(f(101325.0) / (f(8314.46261815324) * t))
            rr = kf * np.exp(-log_kc)
            for k in range(mech.nspecies):
                if mech.nu_prod[i, k] != 0:
                    rr = rr * conc[k] ** f(mech.nu_prod[i, k])
            r = rf - rr
        rates.append(r)
    nu_net = (mech.nu_prod - mech.nu_reac).astype(f)
    return np.tensordot(nu_net, np.array(rates), axes=(0, 0)).astype(np.float64)


def run(dt=5e-9, nsteps=200, variants=VARIANTS, n=3, seed=0):
    import torch

    from cases import make_disc
    from mirgecom_b200.initializers import reacting_mixture_state
    from mirgecom_b200.thermochemistry import UIUC_7SP
    from oracle import dg as odg
    from oracle import physics as oph

    _, od = make_disc("simplex", 3, n, 2, (0.0,) * 3, (2 * np.pi,) * 3, True)
    cv0, t0 = reacting_mixture_state([torch.from_numpy(od.nodes[i]) for i in range(3)],
                                     UIUC_7SP, seed=seed)
    q0 = cv0.q.numpy().copy()
    t0 = t0.numpy() + 2.0
    gas = oph.MixtureGas(UIUC_7SP, temperature_niter=5)
    tr = oph.SimpleTransportParams(viscosity=1e-5, thermal_conductivity=1e-5,
                                   species_diffusivity=(1e-5,) * 7)
    w = UIUC_7SP.molecular_weights[:, None, None]

    def make_rhs(kind, box):
        def rhs(t, q):
            qin = _f32(q) if kind == "q_f32" else q
            st = oph.make_fluid_state(qin, gas, tr, 3, temperature_seed=box[0])
            r = odg.ns_operator(od, st, gas, tr, {})
            temp = st["temperature"]
            if kind == "src_f32":
                qs = _f32(q)
                src = np.zeros_like(q)
                src[5:] = w * _rates_f32(UIUC_7SP, qs[0], _f32(temp), qs[5:] / qs[0])
            elif kind == "src_f32in":
                qs = q.copy()
                qs[0] = _f32(q[0])
                qs[5:] = _f32(q[5:])
                src = oph.species_source_terms(gas, qs, _f32(temp), 3)
            else:
                src = oph.species_source_terms(gas, q, temp, 3)
            r = r + src
            return _f32(r) if kind == "rhs_f32" else r
        return rhs

    finals = {}
    walls = {}
    for kind in ("reference",) + tuple(variants):
        q = q0.copy()
        if kind == "perturbed":
            q = q * (1 + 6e-8 * np.random.default_rng(1).standard_normal(q.shape))
        box = [t0.copy()]
        rhs = make_rhs(kind, box)
        tic = time.perf_counter()
        for i in range(nsteps):
            q = odg.rk4_step(q, i * dt, dt, rhs)
            box[0] = oph.make_fluid_state(q, gas, tr, 3, temperature_seed=box[0])["temperature"]
        walls[kind] = time.perf_counter() - tic
        finals[kind] = q
    ref = finals["reference"]
    mom = np.linalg.norm(ref[2:5].ravel())

    def rel(a, b):
        return [float(np.linalg.norm((a[c] - b[c]).ravel()) /
                      (mom if 2 <= c < 5 else np.linalg.norm(b[c].ravel())))
                for c in range(b.shape[0])]
    st0 = oph.make_fluid_state(q0, gas, tr, 3, temperature_seed=t0)
    src0 = oph.species_source_terms(gas, q0, st0["temperature"], 3)[5:]
    mask = (q0[5:] / q0[0]) > 1e-3
    tau = np.abs(q0[5:][mask]) / np.maximum(np.abs(src0[mask]), 1e-300)
    return {"dt": dt, "steps": nsteps, "t_final": dt * nsteps,
            "tau_chem_min": float(tau.min()), "tau_chem_p1": float(np.percentile(tau, 1)),
            "fp64_change_max": max(rel(ref, q0)),
            "o2_consumed": float(1 - ref[6].sum() / q0[6].sum()),
            "max_rel_l2": {k: max(rel(finals[k], ref)) for k in variants},
            "wall_s": walls}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--dt", type=float, default=5e-9)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--variants", default=",".join(VARIANTS))
    args = ap.parse_args(argv)
    print(json.dumps(run(args.dt, args.steps, tuple(args.variants.split(",")))))


if __name__ == "__main__":
    main()
