"""Simulation time-step selection, mirroring mirgecom/simutil.py:224-306."""

from __future__ import annotations

import torch

from mirgecom_b200.viscous import get_viscous_timestep


def _global_min(x):
    """Minimum over all nodes, and over all ranks when a process group is
    active (the reference's ``nodal_min`` is an MPI collective: every rank
    must call it)."""
    import torch.distributed as dist
    m = x.min()
    if dist.is_available() and dist.is_initialized():
        m = m.detach().clone()
        dist.all_reduce(m, op=dist.ReduceOp.MIN)
    return float(m)


def get_sim_timestep(dcoll, state, t, dt, cfl, t_final=0.0, constant_cfl=False,
                     local_dt=False, fluid_dd=None):
    """Constraint-limited time step (mirgecom/simutil.py:224-306).

    * constant dt (default): min(dt, t_final - t), not below 0;
    * constant CFL: min(cfl * global min of the viscous time step, t_final - t);
    * local dt: cfl times the element-wise minimum of the viscous time step,
      as a tensor shaped like the fields (*t_final* ignored).
    """
    if local_dt:
        vdt = get_viscous_timestep(dcoll, state, dd=fluid_dd)
        emin = vdt.min(dim=-1, keepdim=True).values
        return cfl * torch.ones_like(vdt) * emin
    my_dt = dt
    t_remaining = max(0, t_final - t)
    if constant_cfl:
        my_dt = cfl * _global_min(get_viscous_timestep(dcoll, state, dd=fluid_dd))
    return min(t_remaining, my_dt)
