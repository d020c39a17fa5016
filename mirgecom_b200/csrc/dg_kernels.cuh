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

// Padded row stride (in doubles) of a shared-memory operand matrix read as
// m8n8k4 f64 MMA fragments: rows hold K entries (rounded to the k-step 4),
// and stride = 4 (mod 16) keeps each half-warp's 16 loads on distinct banks.
__host__ __device__ constexpr int mma_stride(int k) {
  return round_up(k, 4) + ((4 - round_up(k, 4) % 16) + 16) % 16;
}

template <int DIM, int ORDER, int NS, bool MIX>
struct Cfg {
  using S = Simplex<DIM, ORDER>;
  static constexpr int NP = S::NP, NF = S::NF, NFP = S::NFP;
  static constexpr int NFN = NF * NFP;
  static constexpr int NC = DIM + 2 + NS;
  static constexpr int NU = NC + 1;      // conserved fields + temperature
  static constexpr int MP = round_up(NP, 8);           // output rows, padded
  static constexpr int MT = MP / 8;                    // m-tiles
  static constexpr int NT = 256;                       // threads per CTA
  // two resident CTAs per SM (<= 128 registers) unless the species make the
  // pointwise flux state too large for that
  static constexpr int MINB = (NC <= 7) ? 2 : 1;
  static constexpr int SMEM_BUDGET = 112 * 1024;
  static constexpr int GEO = DIM * DIM + NF * (DIM + 1);

  // gradient kernel operands: U [col][KU], face values [col][KS] with
  // col = field * EPB + element; matrices AW [DIM][MP][KU], AL [NF][MP][KL]
  static constexpr int NFP4 = round_up(NFP, 4);
  static constexpr int KU = mma_stride(NP);
  static constexpr int KS = mma_stride(NF * NFP4);
  static constexpr int KL = mma_stride(NFP4);
  static constexpr int G_MAT = DIM * MP * KU + NF * MP * KL;
  static constexpr int G_PER_ELEM = NU * (KU + KS) + GEO;
  static constexpr int EPB_G_RAW = (SMEM_BUDGET / 8 - G_MAT - 512) / G_PER_ELEM;
  static constexpr int EPB_GRAD = imax(8, imin(32, EPB_G_RAW / 8 * 8));
  static constexpr int NCOL_G = round_up(NU * EPB_GRAD, 8);

  // rhs kernel operands: B [col][KB] = [G_0 .. G_{DIM-1} | S] per column,
  // A [MP][KB] = [-W_0 .. -W_{DIM-1} | LIFT]
  static constexpr int KR = DIM * NP + NFN;
  static constexpr int KB = mma_stride(KR);
  static constexpr int R_MAT = MP * KB;
  static constexpr int R_PER_ELEM = NC * KB + NC * NP + (MIX ? 2 * NP : 0) + NS * NP + GEO;
  static constexpr int EPB_R_RAW = (SMEM_BUDGET / 8 - R_MAT - 512) / R_PER_ELEM;
  static constexpr int EPB_RHS = imax(4, imin(32, EPB_R_RAW >= 8 ? EPB_R_RAW / 8 * 8
                                                                 : EPB_R_RAW / 4 * 4));
  static constexpr int NCOL_R = round_up(NC * EPB_RHS, 8);

  static size_t smem_grad(int nperm) {
    return (size_t)(G_MAT + NCOL_G * (KU + KS) + EPB_GRAD * GEO) * 8 + NFN * 4 +
           (size_t)nperm * NFP + 64;
  }
  static size_t smem_rhs(int nperm) {
    return (size_t)(R_MAT + NCOL_R * KB + EPB_RHS * (NC * NP + (MIX ? 2 * NP : 0) + NS * NP + GEO)) * 8 +
           NFN * 4 + (size_t)nperm * NFP + 64;
  }
};

// D(8x8) += A(8x4) * B(4x8), float64 tensor-core MMA.  Fragments:
//   A: lane holds A[lane/4][lane%4];  B: lane holds B[lane%4][lane/4];
//   D: lane holds D[lane/4][2*(lane%4) + {0,1}].
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

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

template <int DIM, int ORDER, int NS, bool MIX>
__global__ void __launch_bounds__(256, (Cfg<DIM, ORDER, NS, MIX>::MINB)) k_grad(DGArgs<double> a, GasParams g) {
  using C = Cfg<DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = C::NP, NF = C::NF, NFP = C::NFP, NFN = C::NFN, NC = C::NC, NU = C::NU;
  constexpr int EPB = C::EPB_GRAD, MP = C::MP, MT = C::MT;
  constexpr int KU = C::KU, KS = C::KS, KL = C::KL, NFP4 = C::NFP4, NCOL = C::NCOL_G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* aw = reinterpret_cast<double*>(smem_raw);        // [DIM][MP][KU]
  double* al = aw + DIM * MP * KU;                         // [NF][MP][KL]
  double* bu = al + NF * MP * KL;                          // [NCOL][KU]
  double* bs = bu + NCOL * KU;                              // [NCOL][KS]
  double* rx_s = bs + NCOL * KS;                           // [EPB][DIM][DIM]
  double* nrm_s = rx_s + EPB * DIM * DIM;                  // [EPB][NF][DIM]
  double* fs_s = nrm_s + EPB * NF * DIM;                   // [EPB][NF]
  int* fn_s = reinterpret_cast<int*>(fs_s + EPB * NF);     // [NF*NFP]
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(fn_s + NFN);

  const int E = a.nelem;
  const int e0 = blockIdx.x * EPB;
  const int ne = imin(EPB, E - e0);
  const int64_t EN = (int64_t)E * NP;

  // reference operators (zero padded) and zeroed operand tiles
  for (int i = threadIdx.x; i < DIM * MP * KU; i += blockDim.x) {
    const int r = i / (MP * KU), row = (i / KU) % MP, k = i % KU;
    aw[i] = (row < NP && k < NP) ? c_ref64[S::OFF_W + (r * NP + row) * NP + k] : 0.0;
  }
  for (int i = threadIdx.x; i < NF * MP * KL; i += blockDim.x) {
    const int f = i / (MP * KL), row = (i / KL) % MP, m = i % KL;
    al[i] = (row < NP && m < NFP) ? c_ref64[S::OFF_LIFT + row * NFN + f * NFP + m] : 0.0;
  }
  for (int i = threadIdx.x; i < NCOL * (KU + KS); i += blockDim.x) bu[i] = 0.0;
  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];
  load_geometry<double, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);   // syncs once
  __syncthreads();

  // phase 1: conserved fields (and temperature) of the tile into U
  for (int c = 0; c < NC; ++c)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
      const int e = idx / NP, k = idx % NP;
      bu[(c * EPB + e) * KU + k] = a.q[c * EN + (int64_t)e0 * NP + idx];
    }
  if (MIX)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
      const int e = idx / NP, k = idx % NP;
      bu[(NC * EPB + e) * KU + k] = a.t_op[(int64_t)e0 * NP + idx];
    }
  __syncthreads();
  if (!MIX) {
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
      const int e = idx / NP, k = idx % NP;
      double qq[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) qq[c] = bu[(c * EPB + e) * KU + k];
      bu[(NC * EPB + e) * KU + k] = node_temperature<double, DIM, NS>(qq, 0.0, g);
    }
    __syncthreads();
  }

  // phase 3: face values  fscale * u*   (u* = central average or boundary value)
  for (int idx = threadIdx.x; idx < ne * NFN; idx += blockDim.x) {
    const int e = idx / NFN, fm = idx % NFN, f = fm / NFP, m = fm % NFP;
    const int k = fn_s[fm];
    const int cn = a.conn[(int64_t)(e0 + e) * NF + f];
    const double fsc = fs_s[e * NF + f];
    double up[NU];
    bool central = true;
    if (cn >= 0) {
      const int en = cn >> 8, pr = cn & 255;
      const int kn = (pr < a.nperm) ? perm_s[pr * NFP + m] : NP;
      if (en >= E || kn >= NP) {
        atomicOr(a.status, ST_BAD_INDEX);
#pragma unroll
        for (int c = 0; c < NU; ++c) up[c] = bu[(c * EPB + e) * KU + k];
      } else {
        const int64_t gi = (int64_t)en * NP + kn;
#pragma unroll
        for (int c = 0; c < NC; ++c) up[c] = a.q[c * EN + gi];
        up[NC] = MIX ? a.t_op[gi] : node_temperature<double, DIM, NS>(up, 0.0, g);
      }
    } else {
      const int bf = -(cn + 1);
      const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
      if (kind == BK_PRESCRIBED) {
        const int64_t bstride = (int64_t)a.nbf * NFP;
#pragma unroll
        for (int c = 0; c < NC; ++c) up[c] = a.bext[c * bstride + (int64_t)bf * NFP + m];
        up[NC] = MIX ? a.bext[NC * bstride + (int64_t)bf * NFP + m]
                     : node_temperature<double, DIM, NS>(up, 0.0, g);
        central = false;   // the gradient flux sends the exterior value
      } else {
        if (kind < 0) atomicOr(a.status, ST_BAD_INDEX);
#pragma unroll
        for (int c = 0; c < NU; ++c) up[c] = bu[(c * EPB + e) * KU + k];
      }
    }
#pragma unroll
    for (int c = 0; c < NU; ++c) {
      const double um = bu[(c * EPB + e) * KU + k];
      const double ustar = central ? (up[c] + um) / 2 : up[c];
      bs[(c * EPB + e) * KS + f * NFP4 + m] = fsc * ustar;
    }
  }
  __syncthreads();

  // phase 4: per 8-column tile, du_r = W_r U and L_f = LIFT_f S on the
  // float64 tensor cores, then grad_j = sum_f n_fj L_f - sum_r rx_rj du_r
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  for (int nt = warp; nt < NCOL / 8; nt += blockDim.x >> 5) {
    double du[DIM][MT][2], lf[NF][MT][2];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int t = 0; t < MT; ++t) du[r][t][0] = du[r][t][1] = 0.0;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int t = 0; t < MT; ++t) lf[f][t][0] = lf[f][t][1] = 0.0;
    const double* bcol = bu + (nt * 8 + gq) * KU + tq;
#pragma unroll
    for (int ks = 0; ks < KU / 4; ++ks) {
      if (ks * 4 >= NP) break;
      const double b = bcol[ks * 4];
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int t = 0; t < MT; ++t)
          dmma884(du[r][t], aw[(r * MP + t * 8 + gq) * KU + ks * 4 + tq], b);
    }
    const double* scol = bs + (nt * 8 + gq) * KS + tq;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int ks = 0; ks < NFP4 / 4; ++ks) {
        const double b = scol[f * NFP4 + ks * 4];
#pragma unroll
        for (int t = 0; t < MT; ++t)
          dmma884(lf[f][t], al[(f * MP + t * 8 + gq) * KL + ks * 4 + tq], b);
      }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int col = nt * 8 + 2 * tq + h;
      const int c = col / EPB, e = col % EPB;
      if (c >= NU || e >= ne) continue;
      double rxe[DIM][DIM], nre[NF][DIM];
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int j = 0; j < DIM; ++j) rxe[r][j] = rx_s[e * DIM * DIM + r * DIM + j];
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < DIM; ++j) nre[f][j] = nrm_s[(e * NF + f) * DIM + j];
      double* outp = a.out + ((int64_t)c * DIM) * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        const int i = t * 8 + gq;
        if (i >= NP) continue;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
          double gsum = 0.0;
#pragma unroll
          for (int f = 0; f < NF; ++f) gsum += nre[f][j] * lf[f][t][h];
#pragma unroll
          for (int r = 0; r < DIM; ++r) gsum -= rxe[r][j] * du[r][t][h];
          outp[(int64_t)j * EN + i] = gsum;
        }
      }
    }
  }
}

// }}}

// {{{ rhs kernel (Euler when VISC is false)

template <int DIM, int ORDER, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__(256, (Cfg<DIM, ORDER, NS, MIX>::MINB)) k_rhs(DGArgs<double> a, GasParams g) {
  using C = Cfg<DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = C::NP, NF = C::NF, NFP = C::NFP, NFN = C::NFN, NC = C::NC;
  constexpr int EPB = C::EPB_RHS, MP = C::MP, MT = C::MT, KB = C::KB, KR = C::KR;
  constexpr int NCOL = C::NCOL_R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* am = reinterpret_cast<double*>(smem_raw);        // [MP][KB]
  double* bm = am + MP * KB;                               // [NCOL][KB]
  double* q_s = bm + NCOL * KB;                            // [NC][EPB][NP]
  double* t_s = q_s + NC * EPB * NP;                       // [2][EPB][NP] (MIX)
  double* src_s = t_s + (MIX ? 2 * EPB * NP : 0);          // [NS][EPB][NP] (MIX)
  double* rx_s = src_s + NS * EPB * NP;                    // [EPB][DIM][DIM]
  double* nrm_s = rx_s + EPB * DIM * DIM;
  double* fs_s = nrm_s + EPB * NF * DIM;
  int* fn_s = reinterpret_cast<int*>(fs_s + EPB * NF);
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(fn_s + NFN);

  const int E = a.nelem;
  const int e0 = blockIdx.x * EPB;
  const int ne = imin(EPB, E - e0);
  const int64_t EN = (int64_t)E * NP;
  const bool sources = MIX && a.add_sources;

  // A = [-W_0 .. -W_{DIM-1} | LIFT], zero padded
  for (int i = threadIdx.x; i < MP * KB; i += blockDim.x) {
    const int row = i / KB, k = i % KB;
    double v = 0.0;
    if (row < NP && k < KR) {
      if (k < DIM * NP) {
        const int r = k / NP, kk = k % NP;
        v = -c_ref64[S::OFF_W + (r * NP + row) * NP + kk];
      } else {
        v = c_ref64[S::OFF_LIFT + row * NFN + (k - DIM * NP)];
      }
    }
    am[i] = v;
  }
  for (int i = threadIdx.x; i < NCOL * KB; i += blockDim.x) bm[i] = 0.0;
  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];
  for (int c = 0; c < NC; ++c)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x)
      q_s[(c * EPB) * NP + idx] = a.q[c * EN + (int64_t)e0 * NP + idx];
  if (MIX)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
      t_s[idx] = a.t_op[(int64_t)e0 * NP + idx];
      t_s[EPB * NP + idx] = sources ? a.t_src[(int64_t)e0 * NP + idx] : 0.0;
    }
  load_geometry<double, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);
  __syncthreads();

  // phase 2: volume flux F = F_V - F_I, metric-combined into B[col][r*NP + k]
  for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
    const int e = idx / NP, k = idx % NP;
    double qq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qq[c] = q_s[(c * EPB) * NP + idx];
    NodeState<double, DIM, NS> st;
    make_state<double, DIM, NS>(qq, MIX ? t_s[idx] : 0.0, g, st);
    double fl[NC][DIM];
    inviscid_flux<double, DIM, NS>(st, fl);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int j = 0; j < DIM; ++j) fl[c][j] = -fl[c][j];
    if (VISC) {
      double gq[NC][DIM], gt[DIM];
      const int64_t gi = (int64_t)e0 * NP + idx;
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) gq[c][j] = a.grad[((int64_t)c * DIM + j) * EN + gi];
#pragma unroll
      for (int j = 0; j < DIM; ++j) gt[j] = a.grad[((int64_t)NC * DIM + j) * EN + gi];
      double fv[NC][DIM];
      viscous_flux<double, DIM, NS, MIX>(st, gq, gt, fv);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) fl[c][j] = fv[c][j] + fl[c][j];
    }
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < DIM; ++j) acc += rx_s[e * DIM * DIM + r * DIM + j] * fl[c][j];
        bm[(c * EPB + e) * KB + r * NP + k] = acc;
      }
    if constexpr (MIX && NS > 0) {
      if (sources) {
        double om[NS];
        production_rates<double, NS>(st.rho, t_s[EPB * NP + idx], st.y, g.zero_level, om);
#pragma unroll
        for (int s = 0; s < NS; ++s) src_s[(s * EPB) * NP + idx] = c_mech.mw[s] * om[s];
      }
    }
  }
  __syncthreads();

  // phase 3: numerical face flux fscale * (F*_V - F*_I) into B[col][DIM*NP + fm]
  for (int idx = threadIdx.x; idx < ne * NFN; idx += blockDim.x) {
    const int e = idx / NFN, fm = idx % NFN, f = fm / NFP, m = fm % NFP;
    const int k = fn_s[fm];
    const int cn = a.conn[(int64_t)(e0 + e) * NF + f];
    const double fsc = fs_s[e * NF + f];
    double n[DIM];
#pragma unroll
    for (int j = 0; j < DIM; ++j) n[j] = nrm_s[(e * NF + f) * DIM + j];
    double qm[NC], qp[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qm[c] = q_s[(c * EPB + e) * NP + k];
    NodeState<double, DIM, NS> sm, sp;
    make_state<double, DIM, NS>(qm, MIX ? t_s[e * NP + k] : 0.0, g, sm);
    // own total flux . n from the metric-combined volume flux:
    // F.n = (sum_r N_r G_r) / |rx^T N|
    double nmag2 = 0.0;
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      double a2 = 0.0;
#pragma unroll
      for (int r = 0; r < DIM; ++r)
        a2 += rx_s[e * DIM * DIM + r * DIM + j] * c_ref64[S::OFF_NREF + f * DIM + r];
      nmag2 += a2 * a2;
    }
    const double inmag = 1.0 / sqrt(nmag2);
    double ftm[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double acc = 0.0;
#pragma unroll
      for (int r = 0; r < DIM; ++r)
        acc += c_ref64[S::OFF_NREF + f * DIM + r] * bm[(c * EPB + e) * KB + r * NP + k];
      ftm[c] = acc * inmag;
    }
    int mode = 0;   // 0 interior, 1 dummy (interior only), 2 prescribed exterior
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
        make_state<double, DIM, NS>(qp, MIX ? a.t_op[gi] : 0.0, g, sp);
      }
    } else {
      const int bf = -(cn + 1);
      const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
      if (kind == BK_PRESCRIBED) {
        mode = 2;
        const int64_t bstride = (int64_t)a.nbf * NFP;
#pragma unroll
        for (int c = 0; c < NC; ++c) qp[c] = a.bext[c * bstride + (int64_t)bf * NFP + m];
        make_state<double, DIM, NS>(qp, MIX ? a.bext[NC * bstride + (int64_t)bf * NFP + m] : 0.0,
                                    g, sp);
      } else {
        if (kind < 0) atomicOr(a.status, ST_BAD_INDEX);
        mode = 1;
      }
    }
    double out[NC];
    if (mode == 1) {
      // DummyBoundary: F_V(q-).n - F_I(q-).n  (boundary.py:1027-1049)
#pragma unroll
      for (int c = 0; c < NC; ++c) out[c] = ftm[c];
    } else {
      double fi[NC];
      inviscid_num_flux<double, DIM, NS>(sm, sp, qm, qp, n, a.flux_kind, fi);
#pragma unroll
      for (int c = 0; c < NC; ++c) out[c] = -fi[c];
      if (VISC) {
        // own viscous part: F_V- . n = (F_V - F_I)- . n + F_I- . n
        double fim[NC];
        inviscid_flux_n<double, DIM, NS>(sm, n, fim);
        double gqp[NC][DIM], gtp[DIM];
        const int64_t gsrc = (mode == 0) ? gi : (int64_t)(e0 + e) * NP + k;
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int j = 0; j < DIM; ++j) gqp[c][j] = a.grad[((int64_t)c * DIM + j) * EN + gsrc];
#pragma unroll
        for (int j = 0; j < DIM; ++j) gtp[j] = a.grad[((int64_t)NC * DIM + j) * EN + gsrc];
        double fvp[NC][DIM];
        viscous_flux<double, DIM, NS, MIX>(sp, gqp, gtp, fvp);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double fvpn = 0.0;
#pragma unroll
          for (int j = 0; j < DIM; ++j) fvpn += fvp[c][j] * n[j];
          const double fvmn = ftm[c] + fim[c];
          out[c] += (fvmn + fvpn) / 2;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) bm[(c * EPB + e) * KB + DIM * NP + fm] = fsc * out[c];
  }
  __syncthreads();

  // phase 4: rhs = [-W | LIFT] [G ; S] on the float64 tensor cores (+ sources)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  bool bad = false;
  for (int nt = warp; nt < NCOL / 8; nt += blockDim.x >> 5) {
    double d[MT][2];
#pragma unroll
    for (int t = 0; t < MT; ++t) d[t][0] = d[t][1] = 0.0;
    const double* bcol = bm + (nt * 8 + gq) * KB + tq;
#pragma unroll 5
    for (int ks = 0; ks < (KR + 3) / 4; ++ks) {
      const double b = bcol[ks * 4];
#pragma unroll
      for (int t = 0; t < MT; ++t) dmma884(d[t], am[(t * 8 + gq) * KB + ks * 4 + tq], b);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int col = nt * 8 + 2 * tq + h;
      const int c = col / EPB, e = col % EPB;
      if (c >= NC || e >= ne) continue;
      double* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        const int i = t * 8 + gq;
        if (i >= NP) continue;
        double v = d[t][h];
        if (sources && c >= 2 + DIM) v += src_s[((c - 2 - DIM) * EPB + e) * NP + i];
        outp[i] = v;
        bad |= !(v == v);
      }
    }
  }
  if (bad) atomicOr(a.status, ST_NAN);
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
