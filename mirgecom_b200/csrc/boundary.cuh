// Mengaldo boundary treatment on the device (mirgecom/boundary.py:391-793).
//
// At a boundary face node, from the interior state (q-, its operator
// temperature T-, p-, c-, gamma-), the outward unit normal n and the
// boundary's parameters (its row of the exterior-state array):
//   state_plus   the exterior state of the inviscid numerical flux
//   state_bc     the state whose conserved variables the gradient flux
//                sends (state_bc.cv (x) n) and at which the viscous flux is
//                evaluated: F_V(state_bc, grad_cv_bc, grad_t_bc) . n
//   temperature_bc   the temperature the temperature-gradient flux sends
//   grad_cv_bc, grad_t_bc   the interior gradients modified by the wall
// For mixtures the plus and bc states' temperatures are re-solved by the
// fixed-count Newton from T- (replace_fluid_state, gas_model.py:907-997).
#pragma once
#include "physics.cuh"

namespace mgc {

// Boundary face kinds (int8 per boundary face).  Prescribed: exterior state
// from the caller (boundary.py:796-1009).  The others are the Mengaldo
// treatment (boundary.py:391-793) with their states computed on the device
// from the interior trace; their parameters travel in the exterior-state
// array: the wall temperature in the temperature row (isothermal), the free
// stream state (far field), the boundary pressure in row 0 (outflow).
enum BoundaryKind {
  BK_DUMMY = 0,
  BK_PRESCRIBED = 1,
  BK_SLIP = 2,          // AdiabaticSlipBoundary          boundary.py:1052-1143
  BK_NOSLIP = 3,        // AdiabaticNoslipWallBoundary    boundary.py:1794-1858
  BK_ISOTHERMAL = 4,    // IsothermalWallBoundary         boundary.py:1727-1792
  BK_FARFIELD = 5,      // FarfieldBoundary               boundary.py:1146-1228
  BK_OUTFLOW = 6,       // PressureOutflowBoundary        boundary.py:1231-1403
};
__host__ __device__ constexpr bool bk_mengaldo(int k) { return k >= BK_SLIP && k <= BK_OUTFLOW; }
// kinds whose exterior-state array entries are read
__host__ __device__ constexpr bool bk_needs_bext(int k) {
  return k == BK_PRESCRIBED || k == BK_ISOTHERMAL || k == BK_FARFIELD || k == BK_OUTFLOW;
}

template <class R, int NS>
__device__ __forceinline__ R bc_internal_energy(const GasParams& g, const R* y, R t) {
  if (g.eos_kind == EOS_IDEAL) return (R)g.gas_const / ((R)g.gamma - R(1)) * t;
  if constexpr (NS > 0) {
    R e, cv;
    mixture_e_cv<R, NS>(y, t, e, cv);
    return e;
  }
  return R(0);
}

// PressureOutflowBoundary energy density (boundary.py:1281-1330) for the
// pressure *pp* where the flow out is subsonic
template <class R, int DIM, int NS>
__device__ __forceinline__ R bc_outflow_energy(const GasParams& g, const R* qm, R tm, R pm,
                                               R cm, R gm, const R* n, R pp) {
  const R rho = qm[0];
  R vn = R(0), mm = R(0);
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    vn += qm[2 + i] / rho * n[i];
    mm += qm[2 + i] * qm[2 + i];
  }
  R sp2 = R(0);
#pragma unroll
  for (int i = 0; i < DIM; ++i) sp2 += (vn * n[i]) * (vn * n[i]);
  const bool supersonic = sqrt(sp2) > cm;
  const R ke = R(0.5) * mm / rho;
  R rho_e;
  if (g.eos_kind == EOS_IDEAL) {
    rho_e = (supersonic ? pm : pp) / (gm - R(1));
  } else {
    R y[NS > 0 ? NS : 1];
#pragma unroll
    for (int k = 0; k < NS; ++k) y[k] = qm[2 + DIM + k] / rho;
    R tp = tm;
    if constexpr (NS > 0)
      if (!supersonic) tp = pp / (rho * mixture_gas_const<R, NS>(y));
    rho_e = rho * bc_internal_energy<R, NS>(g, y, tp);
  }
  return rho_e + ke;
}

// state_bc.cv into qbc; returns temperature_bc.  par: the boundary's
// exterior-state row (NC + 1 values), read by the kinds that need it.
template <class R, int DIM, int NS>
__device__ __forceinline__ R bc_state_cv(int kind, const GasParams& g, const R* qm, R tm, R pm,
                                         R cm, R gm, const R* n, const R* par, R* qbc) {
  constexpr int NC = DIM + 2 + NS;
#pragma unroll
  for (int c = 0; c < NC; ++c) qbc[c] = qm[c];
  const R rho = qm[0];
  R y[NS > 0 ? NS : 1];
#pragma unroll
  for (int k = 0; k < NS; ++k) y[k] = qm[2 + DIM + k] / rho;
  if (kind == BK_SLIP) {
    R mn = R(0), mm = R(0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
      mn += qm[2 + i] * n[i];
      mm += qm[2 + i] * qm[2 + i];
    }
    R mb2 = R(0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
      qbc[2 + i] = qm[2 + i] - mn * n[i];
      mb2 += qbc[2 + i] * qbc[2 + i];
    }
    const R rho_e = qm[1] - R(0.5) * mm / rho;
    qbc[1] = rho_e + R(0.5) * mb2 / rho;
    return tm;
  }
  if (kind == BK_NOSLIP || kind == BK_ISOTHERMAL) {
    const R tw = (kind == BK_ISOTHERMAL) ? par[NC] : tm;
#pragma unroll
    for (int i = 0; i < DIM; ++i) qbc[2 + i] = R(0);
    qbc[1] = rho * bc_internal_energy<R, NS>(g, y, tw);
    return tw;
  }
  if (kind == BK_FARFIELD) {
#pragma unroll
    for (int c = 0; c < NC; ++c) qbc[c] = par[c];
    return par[NC];
  }
  if (kind == BK_OUTFLOW) {
    qbc[1] = bc_outflow_energy<R, DIM, NS>(g, qm, tm, pm, cm, gm, n, par[0]);
    return tm;
  }
  return tm;
}

// state_plus.cv into qp
template <class R, int DIM, int NS>
__device__ __forceinline__ void bc_plus_cv(int kind, const GasParams& g, const R* qm, R tm, R pm,
                                           R cm, R gm, const R* n, const R* par, R* qp) {
  constexpr int NC = DIM + 2 + NS;
#pragma unroll
  for (int c = 0; c < NC; ++c) qp[c] = qm[c];
  if (kind == BK_SLIP) {
    R mn = R(0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) mn += qm[2 + i] * n[i];
#pragma unroll
    for (int i = 0; i < DIM; ++i) qp[2 + i] = qm[2 + i] - R(2) * mn * n[i];
  } else if (kind == BK_NOSLIP || kind == BK_ISOTHERMAL) {
#pragma unroll
    for (int i = 0; i < DIM; ++i) qp[2 + i] = -qm[2 + i];
  } else if (kind == BK_FARFIELD) {
#pragma unroll
    for (int c = 0; c < NC; ++c) qp[c] = par[c];
  } else if (kind == BK_OUTFLOW) {
    const R pb = par[0];
    const R pp = (pm > R(2) * pb) ? pm : R(2) * pb - pm;
    qp[1] = bc_outflow_energy<R, DIM, NS>(g, qm, tm, pm, cm, gm, n, pp);
  }
}

// The wall's gradients: grad_cv_bc (boundary.py:1118-1143 slip, :1772-1781
// isothermal, :1843-1852 no-slip; far field and outflow keep the interior
// ones) and grad_t_bc (adiabatic walls remove the normal component).
// gq [NC][DIM] and gt [DIM] in place; qm the interior state, qbc state_bc.
template <class R, int DIM, int NS>
__device__ __forceinline__ void bc_gradients(int kind, const R* qm, const R* qbc, const R* n,
                                             R (*gq)[DIM], R* gt) {
  constexpr int NC = DIM + 2 + NS;
  (void)NC;
  const R rho = qm[0];
  if (kind == BK_SLIP) {
    // velocity gradient G[i][j] = d v_i / d x_j without the tangential
    // velocities' normal derivatives: G - (I - n n^T) G n n^T
    R g[DIM][DIM], gn[DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
      const R vi = qm[2 + i] / rho;
#pragma unroll
      for (int j = 0; j < DIM; ++j) g[i][j] = (gq[2 + i][j] - vi * gq[0][j]) / rho;
    }
    R ngn = R(0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
      R a = R(0);
#pragma unroll
      for (int j = 0; j < DIM; ++j) a += g[i][j] * n[j];
      gn[i] = a;
      ngn += a * n[i];
    }
    const R rho_bc = qbc[0];
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
      const R ti = gn[i] - ngn * n[i];
      const R vbc = qbc[2 + i] / rho_bc;
#pragma unroll
      for (int j = 0; j < DIM; ++j) gq[2 + i][j] = rho_bc * (g[i][j] - ti * n[j]) + vbc * gq[0][j];
    }
  }
  if (kind == BK_SLIP || kind == BK_NOSLIP || kind == BK_ISOTHERMAL) {
    // impermeable: the mass fractions' normal gradient removed
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const R y = qm[2 + DIM + k] / rho;
      R gy[DIM], gyn = R(0);
#pragma unroll
      for (int j = 0; j < DIM; ++j) {
        gy[j] = (gq[2 + DIM + k][j] - y * gq[0][j]) / rho;
        gyn += gy[j] * n[j];
      }
#pragma unroll
      for (int j = 0; j < DIM; ++j) gq[2 + DIM + k][j] = rho * (gy[j] - gyn * n[j]) + y * gq[0][j];
    }
  }
  if (kind == BK_SLIP || kind == BK_NOSLIP) {
    R tn = R(0);
#pragma unroll
    for (int j = 0; j < DIM; ++j) tn += gt[j] * n[j];
#pragma unroll
    for (int j = 0; j < DIM; ++j) gt[j] = gt[j] - tn * n[j];
  }
}

}  // namespace mgc
