"""Time integration, mirroring mirgecom/integrators/explicit_rk.py:31-37.

``rk4_step`` keeps the reference signature and arithmetic.  With a
:class:`ConservedVars` state on the GPU the stage combinations run in one
fused FP64 kernel per stage (``mgc_rk4_stage``) whose roundings reproduce
the reference's array-by-array evaluation exactly.
"""

from __future__ import annotations

import torch

from mirgecom_b200 import runtime
from mirgecom_b200.fluid import ConservedVars


def rk4_step(state, t, dt, rhs):
    """Take one step using the fourth-order classical Runge-Kutta method."""
    if not (isinstance(state, ConservedVars) and state.q.is_cuda
            and state.q.dtype == torch.float64):
        k1 = rhs(t, state)
        k2 = rhs(t + dt / 2, state + dt / 2 * k1)
        k3 = rhs(t + dt / 2, state + dt / 2 * k2)
        k4 = rhs(t + dt, state + dt * k3)
        return state + dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
    q0 = state.q.contiguous()
    acc = torch.empty_like(q0)
    qs = torch.empty_like(q0)
    tt = [t + dt / 2, t + dt / 2, t + dt]
    k = rhs(t, state)
    for stage in range(3):
        runtime.rk4_stage(q0, k.q.contiguous(), acc, qs, stage, dt)
        k = rhs(tt[stage], ConservedVars(qs, state.dim))
        qs = torch.empty_like(q0) if stage < 2 else qs
    out = torch.empty_like(q0)
    runtime.rk4_stage(q0, k.q.contiguous(), acc, out, 3, dt)
    return ConservedVars(out, state.dim)


def rk4_step_mixed(state, t, dt, rhs, state_lo=None):
    """RK4 of the mixed-precision form.

    *state* is the float64 ConservedVars; *rhs(t, cv32)* takes and returns
    float32 ConservedVars.  Stage states and the stage sum are accumulated in
    float64 (the only float64 arithmetic of the form besides the Newton
    residual check); each stage kernel also emits the float32 copy the next
    right-hand side reads.  Returns (new float64 state, its float32 copy).
    """
    q0 = state.q.contiguous()
    q32 = state_lo.q if state_lo is not None else q0.to(torch.float32)
    acc = torch.empty_like(q0)
    qs = torch.empty_like(q0)
    qs32 = torch.empty_like(q32)
    tt = [t + dt / 2, t + dt / 2, t + dt]
    k = rhs(t, ConservedVars(q32, state.dim))
    for stage in range(3):
        runtime.rk4_stage(q0, k.q.contiguous(), acc, qs, stage, dt, qout_lo=qs32)
        k = rhs(tt[stage], ConservedVars(qs32, state.dim))
    out = torch.empty_like(q0)
    out32 = torch.empty_like(q32)
    runtime.rk4_stage(q0, k.q.contiguous(), acc, out, 3, dt, qout_lo=out32)
    return ConservedVars(out, state.dim), ConservedVars(out32, state.dim)


def advance_state(rhs, timestepper, state, t_final, t=0.0, dt=None, istep=0,
                  pre_step_callback=None, post_step_callback=None, max_steps=None):
    """Thin counterpart of mirgecom/steppers.py:350-449 (fixed dt)."""
    nsteps = 0
    while t < t_final - 1e-14 * max(1.0, abs(t_final)):
        if max_steps is not None and nsteps >= max_steps:
            break
        step_dt = min(dt, t_final - t)
        if pre_step_callback is not None:
            state, step_dt = pre_step_callback(step=istep, t=t, dt=step_dt, state=state)
        state = timestepper(state=state, t=t, dt=step_dt, rhs=rhs)
        t += step_dt
        istep += 1
        nsteps += 1
        if post_step_callback is not None:
            state, step_dt = post_step_callback(step=istep, t=t, dt=step_dt, state=state)
    return istep, t, state
