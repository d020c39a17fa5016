"""Generate the golden input/output vectors of tests/golden/ with the CPU oracle.

Run from the repository root:  python tests/golden/make_golden.py

Each case stores its mesh parameters, the seeded input state and the oracle's
float64 outputs.  tests/test_golden.py checks that the oracle still
reproduces them (CPU) and that the device path matches them (GPU).
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))                   # tests/
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))  # repository root

from cases import make_disc, tgv_np, vortex_np  # noqa: E402

from mirgecom_b200.thermochemistry import UIUC_7SP  # noqa: E402
from oracle import dg as odg  # noqa: E402
from oracle import physics as oph  # noqa: E402

CASES = {
    # 2-D Euler, isentropic vortex (beta 5, centre (5, 0), velocity (1, 0))
    # at t = 0.3 on [0,10]x[-5,5], 4x4 squares x 2 triangles, order 3,
    # exact-solution prescribed boundaries, Rusanov
    "vortex2d_p3": dict(dim=2, n=4, order=3, lo=(0.0, -5.0), hi=(10.0, 5.0), periodic=False),
    # 3-D Navier-Stokes Taylor-Green, periodic [-pi,pi]^3, 3^3 x 6 tets,
    # order 3, mu = 1/1600, Prandtl 0.71
    "tgv3d_p3": dict(dim=3, n=3, order=3, lo=(-np.pi,) * 3, hi=(np.pi,) * 3, periodic=True),
    # 3-D reacting Navier-Stokes, uiuc_7sp, periodic [0,2pi]^3, 3^3 x 6 tets,
    # order 2, Newton from the exact temperature + 25 K, sources on
    "mixture3d_p2": dict(dim=3, n=3, order=2, lo=(0.0,) * 3, hi=(2 * np.pi,) * 3,
                         periodic=True),
}

TGV_MU = 1.0 / 1600
TGV_KAPPA = TGV_MU * 287.1 * 1.4 / 0.4 / 0.71
MIX_TRANSPORT = dict(viscosity=1e-5, thermal_conductivity=2e-5,
                     species_diffusivity=tuple(1e-5 * (k + 1) for k in range(7)))


def mixture_inputs(nodes, seed=11):
    """Seeded smooth reacting state (float64): q and its exact temperature."""
    import torch

    from mirgecom_b200.initializers import reacting_mixture_state
    cv, t = reacting_mixture_state([torch.from_numpy(nodes[i]) for i in range(3)],
                                   UIUC_7SP, seed=seed)
    return cv.q.numpy(), t.numpy()


def build(name):
    c = CASES[name]
    _, od = make_disc("simplex", c["dim"], c["n"], c["order"], c["lo"], c["hi"],
                      c["periodic"])
    out = {k: np.asarray(v) for k, v in c.items()}
    if name == "vortex2d_p3":
        t = 0.3
        q = vortex_np(od.nodes, t)
        gas = oph.IdealGas()
        st = oph.make_fluid_state(q, gas, None, 2)
        bnd = {"all": odg.PrescribedBoundary(lambda x, tt: vortex_np(x, tt))}
        out.update(q=q, time=np.array(t), rhs=odg.euler_operator(od, st, gas, bnd, time=t))
    elif name == "tgv3d_p3":
        q = tgv_np(od.nodes)
        gas = oph.IdealGas()
        tr = oph.SimpleTransportParams(viscosity=TGV_MU, thermal_conductivity=TGV_KAPPA)
        st = oph.make_fluid_state(q, gas, tr, 3)
        out.update(q=q, rhs=odg.ns_operator(od, st, gas, tr, {}))
    else:
        q, t_exact = mixture_inputs(od.nodes)
        tseed = t_exact + 25.0
        gas = oph.MixtureGas(UIUC_7SP, temperature_niter=5)
        tr = oph.SimpleTransportParams(**MIX_TRANSPORT)
        st = oph.make_fluid_state(q, gas, tr, 3, temperature_seed=tseed)
        rhs = odg.ns_operator(od, st, gas, tr, {})
        rhs = rhs + oph.species_source_terms(gas, q, st["temperature"], 3)
        out.update(q=q, tseed=tseed, temperature=st["temperature"], rhs=rhs)
    return out


def main():
    for name in CASES:
        data = build(name)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(path, {k: v.shape for k, v in data.items() if v.ndim})


if __name__ == "__main__":
    main()
