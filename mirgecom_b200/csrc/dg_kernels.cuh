// DG right-hand-side kernels for simplicial elements.
//
// Three kernels make one Navier-Stokes RHS (mirgecom/navierstokes.py:350-575):
//
//   mixture_state  T1 = Newton(e, Y; seed), T2 = Newton(e, Y; T1) per node.
//                  T1 is the state's temperature (gas_model.py:388-389), T2 is
//                  the temperature the operator states carry: every operator
//                  state (volume quad, both sides of each face, boundary) is
//                  re-solved from the restricted state temperature
//                  (gas_model.py:494-588, 661-682, 803-904), and with
//                  interpolatory nodes the restriction is the node value.
//   grad           grad_cv_operator + grad_t_operator (navierstokes.py:129-347):
//                  -M^-1 (S^T u - E (u*) n), u* the BR1 central trace value
//                  (navierstokes.py:118-126) or the boundary value.
//   rhs            div_operator(F_V - F_I, F*_V - F*_I) (navierstokes.py:536-563)
//                  or, without viscous terms, -div_operator(F_I, F*_I)
//                  (euler.py:402-416), plus optional Arrhenius sources.
//
// Element-tile organisation (one CTA = EPB consecutive elements):
//   phase 1  coalesced load of the tile's conserved fields into shared memory
//   phase 2  pointwise volume flux per node, metric-combined into
//            G_r = sum_j (dr_r/dx_j) F_j                       (shared)
//   phase 3  one thread per face node: gather the neighbour trace straight
//            from HBM/L2 through the packed face pairing, evaluate the
//            numerical flux, scale by the face Jacobian factor  (shared)
//   phase 4  one thread per (element, field): operands in registers,
//            reference matrices as constant-memory operands of fully
//            unrolled FMAs:  out = LIFT * S - sum_r W_r * G_r
//
// Face fluxes are owner-computed (each side evaluates its own copy), so
// there are no atomics and results are deterministic run to run.
// Device-detected problems go to *status* (bit mask) and never trap.
#pragma once
#include "dg_refops.cuh"
#include "physics.cuh"

namespace mgc {

template <class R>
struct DGArgs {
  int32_t nelem, nbf, nperm, flux_kind;
  const R* q;          // [NC][E][NP]
  const R* t_op;       // [E][NP] operator temperature (mixture only)
  const R* t_src;      // [E][NP] temperature for source terms (mixture only)
  const R* grad;       // [NC+1][DIM][E][NP] gradients (NS rhs input)
  R* out;              // grad: [NC+1][DIM][E][NP]; rhs: [NC][E][NP]
  const R* rx;         // [E][DIM][DIM]  dr_r/dx_j
  const int32_t* conn; // [E][NF]
  const uint8_t* perm; // [nperm][NFP]
  const int8_t* bkind; // [nbf]  0 = copy interior, 1 = prescribed exterior
  const R* bext;       // [NC+1][nbf][NFP] prescribed exterior q (+ T)
  int32_t* status;
  int32_t add_sources;
  int32_t pad_;
};

enum BoundaryKind { BK_DUMMY = 0, BK_PRESCRIBED = 1 };

__host__ __device__ constexpr int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int round_up(int a, int b) { return (a + b - 1) / b * b; }

template <class R, int DIM, int ORDER, int NS, bool MIX>
struct Cfg {
  using S = Simplex<DIM, ORDER>;
  static constexpr int NP = S::NP, NF = S::NF, NFP = S::NFP;
  static constexpr int NFN = NF * NFP;
  static constexpr int NC = DIM + 2 + NS;
  static constexpr int NU = NC + 1;      // conserved fields + temperature
  static constexpr int SMEM_BUDGET = 96 * 1024;
  // per-element shared bytes
  static constexpr int GEO = DIM * DIM + NF * (DIM + 1);
  static constexpr int BYTES_GRAD = (NU * NP + NU * NFN + GEO) * (int)sizeof(R);
  static constexpr int BYTES_RHS =
      (NC * NP + (MIX ? 2 * NP : 0) + DIM * NC * NP + NC * NFN + NS * NP + GEO) * (int)sizeof(R);
  static constexpr int EPB_GRAD = imax(1, imin(imin(128 / NU, 32), SMEM_BUDGET / BYTES_GRAD));
  static constexpr int EPB_RHS = imax(1, imin(imin(128 / NC, 32), SMEM_BUDGET / BYTES_RHS));
  // 256 threads leave up to 255 registers per thread for the register-resident
  // contraction operands; the pointwise phases stride over the tile
  static constexpr int NT_GRAD = 256;
  static constexpr int NT_RHS = 256;
  static constexpr int PERM_MAX = 256 * NFP;
};

// Per-element geometry: rx copy, unit normals and face factors derived from rx
// (n dS = J rx^T N dS_ref;  fscale = |rx^T N| * face_scale_ref).
template <class R, int DIM, int ORDER>
__device__ __forceinline__ void load_geometry(const R* __restrict__ rx_g, int e0, int ne,
                                              R* rx_s, R* nrm_s, R* fs_s) {
  using S = Simplex<DIM, ORDER>;
  constexpr int NF = S::NF;
  for (int idx = threadIdx.x; idx < ne * DIM * DIM; idx += blockDim.x)
    rx_s[idx] = rx_g[(size_t)e0 * DIM * DIM + idx];
  __syncthreads();
  for (int idx = threadIdx.x; idx < ne * NF; idx += blockDim.x) {
    const int e = idx / NF, f = idx % NF;
    R nv[DIM];
    R mag2 = 0;
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      R a = 0;
#pragma unroll
      for (int r = 0; r < DIM; ++r)
        a += rx_s[e * DIM * DIM + r * DIM + j] * RefBank<R>::get(S::OFF_NREF + f * DIM + r);
      nv[j] = a;
      mag2 += a * a;
    }
    const R mag = sqrt(mag2);
#pragma unroll
    for (int j = 0; j < DIM; ++j) nrm_s[(e * NF + f) * DIM + j] = nv[j] / mag;
    fs_s[e * NF + f] = mag * RefBank<R>::get(S::OFF_FSR + f);
  }
}

// {{{ mixture temperature: T1 = Newton(seed), T2 = Newton(T1)

template <class R, int DIM, int NS>
__global__ void __launch_bounds__(256) k_mixture_state(int64_t nnodes, const R* __restrict__ q,
                                                       const R* __restrict__ tseed,
                                                       R* __restrict__ t1, R* __restrict__ t2,
                                                       GasParams g) {
  constexpr int NC = DIM + 2 + NS;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nnodes; n += stride) {
    R qq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qq[c] = q[(int64_t)c * nnodes + n];
    const R ta = node_temperature<R, DIM, NS>(qq, tseed[n], g);
    t1[n] = ta;
    if (t2) t2[n] = node_temperature<R, DIM, NS>(qq, ta, g);
  }
}

// }}}

// {{{ gradient kernel

template <class R, int DIM, int ORDER, int NS, bool MIX>
__global__ void __launch_bounds__((Cfg<R, DIM, ORDER, NS, MIX>::NT_GRAD))
    k_grad(DGArgs<R> a, GasParams g) {
  using C = Cfg<R, DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = C::NP, NF = C::NF, NFP = C::NFP, NFN = C::NFN, NC = C::NC, NU = C::NU;
  constexpr int EPB = C::EPB_GRAD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* u_s = reinterpret_cast<R*>(smem_raw);                 // [NU][EPB][NP]
  R* f_s = u_s + NU * EPB * NP;                            // [NU][EPB][NFN]
  R* rx_s = f_s + NU * EPB * NFN;                          // [EPB][DIM][DIM]
  R* nrm_s = rx_s + EPB * DIM * DIM;                       // [EPB][NF][DIM]
  R* fs_s = nrm_s + EPB * NF * DIM;                        // [EPB][NF]
  int* fn_s = reinterpret_cast<int*>(fs_s + EPB * NF);     // [NF*NFP]
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(fn_s + NFN);

  const int E = a.nelem;
  const int e0 = blockIdx.x * EPB;
  const int ne = imin(EPB, E - e0);
  const int64_t EN = (int64_t)E * NP;

  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];
  // phase 1: tile load
  for (int c = 0; c < NC; ++c)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x)
      u_s[(c * EPB) * NP + idx] = a.q[c * EN + (int64_t)e0 * NP + idx];
  if (MIX)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x)
      u_s[(NC * EPB) * NP + idx] = a.t_op[(int64_t)e0 * NP + idx];
  load_geometry<R, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);
  __syncthreads();
  if (!MIX) {
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
      R qq[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) qq[c] = u_s[(c * EPB) * NP + idx];
      u_s[(NC * EPB) * NP + idx] = node_temperature<R, DIM, NS>(qq, (R)0, g);
    }
    __syncthreads();
  }

  // phase 3: face values  fscale * u*   (u* = central / boundary value)
  for (int idx = threadIdx.x; idx < ne * NFN; idx += blockDim.x) {
    const int e = idx / NFN, fm = idx % NFN, f = fm / NFP, m = fm % NFP;
    const int k = fn_s[fm];
    const int cn = a.conn[(int64_t)(e0 + e) * NF + f];
    const R fsc = fs_s[e * NF + f];
    R up[NU];
    bool central = true;
    if (cn >= 0) {
      const int en = cn >> 8, pr = cn & 255;
      const int kn = (pr < a.nperm) ? perm_s[pr * NFP + m] : NP;
      if (en >= E || kn >= NP) {
        atomicOr(a.status, ST_BAD_INDEX);
#pragma unroll
        for (int c = 0; c < NU; ++c) up[c] = u_s[(c * EPB + e) * NP + k];
      } else {
        const int64_t gi = (int64_t)en * NP + kn;
#pragma unroll
        for (int c = 0; c < NC; ++c) up[c] = a.q[c * EN + gi];
        up[NC] = MIX ? a.t_op[gi] : node_temperature<R, DIM, NS>(up, (R)0, g);
      }
    } else {
      const int bf = -(cn + 1);
      const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
      if (kind == BK_PRESCRIBED) {
        const int64_t bs = (int64_t)a.nbf * NFP;
#pragma unroll
        for (int c = 0; c < NC; ++c) up[c] = a.bext[c * bs + (int64_t)bf * NFP + m];
        up[NC] = MIX ? a.bext[NC * bs + (int64_t)bf * NFP + m]
                     : node_temperature<R, DIM, NS>(up, (R)0, g);
        central = false;   // gradient flux sends the exterior value
      } else {
        if (kind < 0) atomicOr(a.status, ST_BAD_INDEX);
#pragma unroll
        for (int c = 0; c < NU; ++c) up[c] = u_s[(c * EPB + e) * NP + k];
      }
    }
#pragma unroll
    for (int c = 0; c < NU; ++c) {
      const R um = u_s[(c * EPB + e) * NP + k];
      const R ustar = central ? (up[c] + um) / (R)2 : up[c];
      f_s[(c * EPB + e) * NFN + fm] = fsc * ustar;
    }
  }
  __syncthreads();

  // phase 4: one thread per (element, field)
  for (int p = threadIdx.x; p < EPB * NU; p += blockDim.x) {
    const int e = p % EPB, c = p / EPB;
    if (e >= ne) continue;
    R uk[NP];
    R sk[NFN];
#pragma unroll
    for (int k = 0; k < NP; ++k) uk[k] = u_s[(c * EPB + e) * NP + k];
#pragma unroll
    for (int k = 0; k < NFN; ++k) sk[k] = f_s[(c * EPB + e) * NFN + k];
    R rxe[DIM][DIM], nre[NF][DIM];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int j = 0; j < DIM; ++j) rxe[r][j] = rx_s[e * DIM * DIM + r * DIM + j];
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int j = 0; j < DIM; ++j) nre[f][j] = nrm_s[(e * NF + f) * DIM + j];
    R* outp = a.out + ((int64_t)c * DIM) * EN + (int64_t)(e0 + e) * NP;
    // operands stay in registers; the row index is warp-uniform, so the
    // reference-matrix entries are broadcast constant loads
#pragma unroll 1
    for (int i = 0; i < NP; ++i) {
      R du[DIM];
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        R acc = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k)
          acc += RefBank<R>::get(S::OFF_W + (r * NP + i) * NP + k) * uk[k];
        du[r] = acc;
      }
      R lf[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        R acc = 0;
#pragma unroll
        for (int m = 0; m < NFP; ++m)
          acc += RefBank<R>::get(S::OFF_LIFT + i * NFN + f * NFP + m) * sk[f * NFP + m];
        lf[f] = acc;
      }
#pragma unroll
      for (int j = 0; j < DIM; ++j) {
        R gsum = 0;
#pragma unroll
        for (int f = 0; f < NF; ++f) gsum += nre[f][j] * lf[f];
#pragma unroll
        for (int r = 0; r < DIM; ++r) gsum -= rxe[r][j] * du[r];
        outp[(int64_t)j * EN + i] = gsum;
      }
    }
  }
}

// }}}

// {{{ rhs kernel (Euler when VISC is false)

template <class R, int DIM, int ORDER, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__((Cfg<R, DIM, ORDER, NS, MIX>::NT_RHS))
    k_rhs(DGArgs<R> a, GasParams g) {
  using C = Cfg<R, DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = C::NP, NF = C::NF, NFP = C::NFP, NFN = C::NFN, NC = C::NC, NU = C::NU;
  constexpr int EPB = C::EPB_RHS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* q_s = reinterpret_cast<R*>(smem_raw);                 // [NC][EPB][NP]
  R* t_s = q_s + NC * EPB * NP;                            // [2][EPB][NP] (MIX)
  R* g_s = t_s + (MIX ? 2 * EPB * NP : 0);                 // [DIM][NC][EPB][NP]
  R* f_s = g_s + DIM * NC * EPB * NP;                      // [NC][EPB][NFN]
  R* src_s = f_s + NC * EPB * NFN;                         // [NS][EPB][NP]
  R* rx_s = src_s + NS * EPB * NP;                         // [EPB][DIM][DIM]
  R* nrm_s = rx_s + EPB * DIM * DIM;
  R* fs_s = nrm_s + EPB * NF * DIM;
  int* fn_s = reinterpret_cast<int*>(fs_s + EPB * NF);
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(fn_s + NFN);

  const int E = a.nelem;
  const int e0 = blockIdx.x * EPB;
  const int ne = imin(EPB, E - e0);
  const int64_t EN = (int64_t)E * NP;
  const bool sources = MIX && a.add_sources;

  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];
  for (int c = 0; c < NC; ++c)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x)
      q_s[(c * EPB) * NP + idx] = a.q[c * EN + (int64_t)e0 * NP + idx];
  if (MIX)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
      t_s[idx] = a.t_op[(int64_t)e0 * NP + idx];
      t_s[EPB * NP + idx] = sources ? a.t_src[(int64_t)e0 * NP + idx] : (R)0;
    }
  load_geometry<R, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);
  __syncthreads();

  // phase 2: volume flux F = F_V - F_I, metric-combined
  for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
    const int e = idx / NP;
    R qq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qq[c] = q_s[(c * EPB) * NP + idx];
    NodeState<R, DIM, NS> st;
    make_state<R, DIM, NS>(qq, MIX ? t_s[idx] : (R)0, g, st);
    R fl[NC][DIM];
    inviscid_flux<R, DIM, NS>(st, fl);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int j = 0; j < DIM; ++j) fl[c][j] = -fl[c][j];
    if (VISC) {
      R gq[NC][DIM], gt[DIM];
      const int64_t gi = (int64_t)e0 * NP + idx;
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) gq[c][j] = a.grad[((int64_t)c * DIM + j) * EN + gi];
#pragma unroll
      for (int j = 0; j < DIM; ++j) gt[j] = a.grad[((int64_t)NC * DIM + j) * EN + gi];
      R fv[NC][DIM];
      viscous_flux<R, DIM, NS, MIX>(st, gq, gt, fv);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) fl[c][j] = fv[c][j] + fl[c][j];
    }
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        R acc = 0;
#pragma unroll
        for (int j = 0; j < DIM; ++j) acc += rx_s[e * DIM * DIM + r * DIM + j] * fl[c][j];
        g_s[((r * NC + c) * EPB) * NP + idx] = acc;
      }
    if constexpr (MIX && NS > 0) {
      if (sources) {
        R om[NS];
        const R tsrc = t_s[EPB * NP + idx];
        production_rates<R, NS>(st.rho, tsrc, st.y, (R)g.zero_level, om);
#pragma unroll
        for (int k = 0; k < NS; ++k) src_s[(k * EPB) * NP + idx] = (R)c_mech.mw[k] * om[k];
      }
    }
  }
  __syncthreads();

  // phase 3: numerical face flux  fscale * (F*_V - F*_I)
  for (int idx = threadIdx.x; idx < ne * NFN; idx += blockDim.x) {
    const int e = idx / NFN, fm = idx % NFN, f = fm / NFP, m = fm % NFP;
    const int k = fn_s[fm];
    const int cn = a.conn[(int64_t)(e0 + e) * NF + f];
    const R fsc = fs_s[e * NF + f];
    R n[DIM];
#pragma unroll
    for (int j = 0; j < DIM; ++j) n[j] = nrm_s[(e * NF + f) * DIM + j];
    R qm[NC], qp[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qm[c] = q_s[(c * EPB + e) * NP + k];
    NodeState<R, DIM, NS> sm, sp;
    make_state<R, DIM, NS>(qm, MIX ? t_s[e * NP + k] : (R)0, g, sm);
    // own total flux . n from the metric-combined volume flux
    R nmag2 = 0;
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      R a2 = 0;
#pragma unroll
      for (int r = 0; r < DIM; ++r)
        a2 += rx_s[e * DIM * DIM + r * DIM + j] * RefBank<R>::get(S::OFF_NREF + f * DIM + r);
      nmag2 += a2 * a2;
    }
    const R inmag = (R)1 / sqrt(nmag2);
    R ftm[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      R acc = 0;
#pragma unroll
      for (int r = 0; r < DIM; ++r)
        acc += RefBank<R>::get(S::OFF_NREF + f * DIM + r) * g_s[((r * NC + c) * EPB + e) * NP + k];
      ftm[c] = acc * inmag;
    }
    int mode = 0;   // 0 interior, 1 dummy (copy interior), 2 prescribed
    int64_t gi = 0;
    if (cn >= 0) {
      const int en = cn >> 8, pr = cn & 255;
      const int kn = (pr < a.nperm) ? perm_s[pr * NFP + m] : NP;
      if (en >= E || kn >= NP) {
        atomicOr(a.status, ST_BAD_INDEX);
        mode = 1;
      } else {
        gi = (int64_t)en * NP + kn;
#pragma unroll
        for (int c = 0; c < NC; ++c) qp[c] = a.q[c * EN + gi];
        make_state<R, DIM, NS>(qp, MIX ? a.t_op[gi] : (R)0, g, sp);
      }
    } else {
      const int bf = -(cn + 1);
      const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
      if (kind == BK_PRESCRIBED) {
        mode = 2;
        const int64_t bs = (int64_t)a.nbf * NFP;
#pragma unroll
        for (int c = 0; c < NC; ++c) qp[c] = a.bext[c * bs + (int64_t)bf * NFP + m];
        make_state<R, DIM, NS>(qp, MIX ? a.bext[NC * bs + (int64_t)bf * NFP + m] : (R)0, g, sp);
      } else {
        if (kind < 0) atomicOr(a.status, ST_BAD_INDEX);
        mode = 1;
      }
    }
    R out[NC];
    if (mode == 1) {
      // DummyBoundary: F_V(q-).n - F_I(q-).n  (boundary.py:1027-1049)
#pragma unroll
      for (int c = 0; c < NC; ++c) out[c] = ftm[c];
    } else {
      R fi[NC];
      inviscid_num_flux<R, DIM, NS>(sm, sp, qm, qp, n, a.flux_kind, fi);
#pragma unroll
      for (int c = 0; c < NC; ++c) out[c] = -fi[c];
      if (VISC) {
        // own viscous part: F_V- . n = (F_V - F_I)- . n + F_I- . n
        R fim[NC];
        inviscid_flux_n<R, DIM, NS>(sm, n, fim);
        R gq[NC][DIM], gt[DIM];
        const int64_t gsrc = (mode == 0) ? gi : (int64_t)(e0 + e) * NP + k;
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int j = 0; j < DIM; ++j) gq[c][j] = a.grad[((int64_t)c * DIM + j) * EN + gsrc];
#pragma unroll
        for (int j = 0; j < DIM; ++j) gt[j] = a.grad[((int64_t)NC * DIM + j) * EN + gsrc];
        R fvp[NC][DIM];
        viscous_flux<R, DIM, NS, MIX>(sp, gq, gt, fvp);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          R fvpn = 0;
#pragma unroll
          for (int j = 0; j < DIM; ++j) fvpn += fvp[c][j] * n[j];
          const R fvmn = ftm[c] + fim[c];
          out[c] += (fvmn + fvpn) / (R)2;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) f_s[(c * EPB + e) * NFN + fm] = fsc * out[c];
  }
  __syncthreads();

  // phase 4: rhs = LIFT * S - sum_r W_r G_r  (+ sources)
  for (int p = threadIdx.x; p < EPB * NC; p += blockDim.x) {
    const int e = p % EPB, c = p / EPB;
    if (e >= ne) continue;
    R acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = 0;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      R sk[NFP];
#pragma unroll
      for (int m = 0; m < NFP; ++m) sk[m] = f_s[(c * EPB + e) * NFN + f * NFP + m];
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        R s = 0;
#pragma unroll
        for (int m = 0; m < NFP; ++m)
          s += RefBank<R>::get(S::OFF_LIFT + i * NFN + f * NFP + m) * sk[m];
        acc[i] += s;
      }
    }
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
      R gk[NP];
#pragma unroll
      for (int k = 0; k < NP; ++k) gk[k] = g_s[((r * NC + c) * EPB + e) * NP + k];
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        R s = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) s += RefBank<R>::get(S::OFF_W + (r * NP + i) * NP + k) * gk[k];
        acc[i] -= s;
      }
    }
    if (sources && c >= 2 + DIM) {
      const int sidx = c - 2 - DIM;
#pragma unroll
      for (int i = 0; i < NP; ++i) acc[i] += src_s[(sidx * EPB + e) * NP + i];
    }
    R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
    bool bad = false;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      outp[i] = acc[i];
      bad |= !(acc[i] == acc[i]);
    }
    if (bad) atomicOr(a.status, ST_NAN);
  }
}

// }}}

// {{{ RK4 (mirgecom/integrators/explicit_rk.py:31-37), FP64 accumulation

// stage s of 4:  sum (+)= w_s k ;  q_stage = q0 + a_s k   (s < 3)
//                q_new = q0 + (dt/6) (sum + k)             (s == 3)
template <class R>
__global__ void k_rk4_stage(int64_t n, const double* __restrict__ q0, const double* __restrict__ k,
                            double* __restrict__ sum, double* __restrict__ qout,
                            R* __restrict__ qout_lo, int stage, double dt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    // explicit roundings (no FMA contraction) reproduce the reference's
    // array-by-array evaluation order bit for bit
    const double kv = k[i];
    double qn;
    if (stage == 0) {
      sum[i] = kv;
      qn = __dadd_rn(q0[i], __dmul_rn(dt / 2, kv));
    } else if (stage == 1) {
      sum[i] = __dadd_rn(sum[i], __dmul_rn(2.0, kv));
      qn = __dadd_rn(q0[i], __dmul_rn(dt / 2, kv));
    } else if (stage == 2) {
      sum[i] = __dadd_rn(sum[i], __dmul_rn(2.0, kv));
      qn = __dadd_rn(q0[i], __dmul_rn(dt, kv));
    } else {
      qn = __dadd_rn(q0[i], __dmul_rn(dt / 6, __dadd_rn(sum[i], kv)));
    }
    qout[i] = qn;
    if (qout_lo) qout_lo[i] = (R)qn;
  }
}

// }}}

}  // namespace mgc
