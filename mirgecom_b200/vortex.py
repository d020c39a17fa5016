"""Isentropic-vortex driver: the 2-D Euler configuration run to a final time.

The counterpart of mirgecom's examples/vortex.py:99-133,350-383 (an
``euler_operator`` right-hand side with the exact solution prescribed on
every boundary, advanced with ``rk4_step`` at a fixed dt, the final state
compared with the exact solution), on this library's device path.  The
default case is the 2-D benchmark configuration: [0, 10] x [-5, 5] split
into 16 x 16 squares of 2 triangles, order 3, ideal gas gamma = 1.4, vortex
strength beta = 5 centred at (5, 0) advected at velocity (1, 0), Rusanov
flux, RK4 with dt = 0.005 to t = 1 (200 steps).  (The reference example
itself uses [-5, 5]^2, centre (0, 0), velocity (1, 1) and t_final = 0.01.)

    python -m mirgecom_b200.vortex [--steps 200] [--dt 0.005]
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from mirgecom_b200.boundary import PrescribedFluidBoundary
from mirgecom_b200.discretization import Discretization
from mirgecom_b200.eos import IdealSingleGas
from mirgecom_b200.euler import euler_operator
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.initializers import Vortex2D
from mirgecom_b200.integrators import advance_state, rk4_step
from mirgecom_b200.inviscid import inviscid_facial_flux_rusanov
from mirgecom_b200.mesh import generate_box_mesh

CASE = dict(a=(0.0, -5.0), b=(10.0, 5.0), nel=16, order=3, beta=5.0, center=(5.0, 0.0),
            velocity=(1.0, 0.0), dt=0.005, t_final=1.0)


def setup(device, nel=CASE["nel"], order=CASE["order"]):
    """Discretization, gas model, initializer and boundaries of the case."""
    mesh = generate_box_mesh(CASE["a"], CASE["b"], (nel, nel))
    dcoll = Discretization(mesh, order, device=device)
    gas = GasModel(eos=IdealSingleGas())
    init = Vortex2D(beta=CASE["beta"], center=CASE["center"], velocity=CASE["velocity"])

    def boundary_solution(dcoll, dd_bdry, gas_model, state_minus, time=0.0, nodes=None,
                          **kwargs):
        x = [nodes[i] for i in range(nodes.shape[0])]
        return make_fluid_state(init(x, eos=gas_model.eos, time=time), gas_model)

    boundaries = {"all": PrescribedFluidBoundary(boundary_state_func=boundary_solution)}
    return dcoll, gas, init, boundaries


def l2_error(dcoll, q, q_exact):
    """Per-field L2 norm of q - q_exact over the domain: sqrt(sum_e det(J_e)
    r_e^T M r_e), M the reference mass matrix."""
    r = (q - q_exact).double().cpu().numpy()                 # (Nc, E, Np)
    mass = dcoll.refel.mass
    det = np.abs(dcoll.geometry.det)
    return [float(np.sqrt(np.sum(det * np.einsum("ei,ij,ej->e", r[c], mass, r[c]))))
            for c in range(r.shape[0])]


def run(device=None, nsteps=None, dt=CASE["dt"], nel=CASE["nel"], order=CASE["order"]):
    """Advance the vortex; returns a dict with the final state, the final
    time, the per-field L2 error against the exact solution and the wall
    time of the stepping (synchronised)."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    dcoll, gas, init, boundaries = setup(device, nel, order)
    x = dcoll.nodes(device)
    cv = init(x, eos=gas.eos)

    def rhs(t, state):
        return euler_operator(dcoll, make_fluid_state(state, gas), gas, boundaries, time=t,
                              inviscid_numerical_flux_func=inviscid_facial_flux_rusanov)

    t_final = CASE["t_final"] if nsteps is None else nsteps * dt
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    steps, t, cv = advance_state(rhs, rk4_step, cv, t_final, dt=dt)
    torch.cuda.synchronize(device)
    wall = time.perf_counter() - t0
    exact = init(x, eos=gas.eos, time=t)
    return {"q": cv.q, "t": t, "steps": steps, "dt": dt, "wall_s": wall,
            "l2_error": l2_error(dcoll, cv.q, exact.q),
            "dof": int(cv.q.numel()), "dcoll": dcoll}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=None, help="default: to t = 1")
    ap.add_argument("--dt", type=float, default=CASE["dt"])
    args = ap.parse_args(argv)
    res = run(nsteps=args.steps, dt=args.dt)
    print(json.dumps({"case": "vortex2d_p3", "steps": res["steps"], "t": res["t"],
                      "dt": res["dt"], "wall_s": res["wall_s"],
                      "l2_error": dict(zip(["mass", "energy", "momentum_x", "momentum_y"],
                                           res["l2_error"]))}))


if __name__ == "__main__":
    main()
