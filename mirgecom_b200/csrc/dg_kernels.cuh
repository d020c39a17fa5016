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
#include "boundary.cuh"
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
  R* fbuf;             // split path: per-node flux record [E*NP][FW]
  R* srcbuf;           // split path: species sources [NS][E][NP]
  void* mid_event;     // host side: cudaEvent_t recorded between the two
                       // kernels of a two-kernel pass, or null
  // volume/face path
  R* trace;            // [E][NF][NFP][TW] face-node records: F.n, lambda, p, c, gamma
  R* s0;               // [E][NF][NC] node-0 flux . n per face (element-constant shift)
  R* btrace;           // [nbf][NFP][TW] exterior records of boundary faces
  R* bplus;            // [NC][nbf][NFP] exterior q of the inviscid flux at boundary faces
  const uint8_t* fslot;  // [nperm][NFP] neighbour face slot fn * NFP + m'
  R* grad_out;         // optional [NC+1][DIM][E][NP] gradients (return_gradients)
  int32_t nowned;      // elements [0, nowned) are evaluated; the rest (up to nelem)
                       // are ghosts of a mesh partition, read as neighbours only
  int32_t phases;      // volume/face path: bit 0 volume stage, bit 1 face stage,
                       // bit 2 the volume stage as gradient kernel (into grad_out)
                       // then flux-volume kernel
  int32_t grad_kernel; // gradient pass: 0 tcgen05 where it applies, else mma.sync;
                       // 1 always mma.sync
  int32_t pad2_;
};

__host__ __device__ constexpr int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Flux record of the split divergence: NC*DIM total-flux values, then p, c,
// gamma and the node's wave speed |v| + c, padded to 16 bytes.
__host__ __device__ constexpr int flux_record_width(int dim, int nc) {
  return round_up(nc * dim + 4, 4);
}

// Tensor-core tiling per arithmetic type.
//   double: mma.m8n8k4.f64        -- m-tile 8,  k-step 4, 8-byte banks;
//   float : mma.m16n8k8.tf32 x 3  -- m-tile 16, k-step 8, 4-byte banks.
// A row stride of MODK (mod 2*KSTEP... see mma_stride) keeps every fragment
// load of a warp (8 rows x 4 consecutive k) on distinct shared-memory banks.
template <class R> struct Tile;
template <> struct Tile<double> {
  static constexpr int MROW = 8, KSTEP = 4;
  // stride = 4 (mod 8) doubles: rows g=0..3 of a half-warp hit 4 disjoint bank quads
  static constexpr __host__ __device__ int stride(int k) {
    return round_up(k, 4) % 8 == 4 ? round_up(k, 4) : round_up(k, 4) + 4;
  }
};
template <> struct Tile<float> {
  static constexpr int MROW = 16, KSTEP = 8;
  // stride = 4 (mod 8) floats: rows g=0..7 x 4 consecutive k cover 32 banks
  static constexpr __host__ __device__ int stride(int k) {
    return round_up(k, 8) + 4;
  }
};

template <class R, int DIM, int ORDER, int NS, bool MIX>
struct Cfg {
  using S = Simplex<DIM, ORDER>;
  using T = Tile<R>;
  static constexpr int RB = (int)sizeof(R);
  static constexpr bool TF32 = sizeof(R) == 4;
  static constexpr int NP = S::NP, NF = S::NF, NFP = S::NFP;
  static constexpr int NFN = NF * NFP;
  static constexpr int NC = DIM + 2 + NS;
  static constexpr int NU = NC + 1;      // conserved fields + temperature
  static constexpr int MP = round_up(NP, T::MROW);     // output rows, padded
  static constexpr int MT = MP / T::MROW;              // m-tiles
  static constexpr int NAC = TF32 ? 2 : 1;             // A copies: tf32 hi/lo split
  static constexpr int NT = 256;                       // threads per CTA
  // two resident CTAs per SM unless the species make the pointwise flux
  // state too large for <= 128 registers
  static constexpr int MINB = (NC <= 7 || TF32) ? 2 : 1;
  static constexpr int SMEM_BUDGET = 112 * 1024;
  static constexpr int GEO = DIM * DIM + NF * (DIM + 1);

  // gradient kernel operands: U [col][KU], face values [col][KS] with
  // col = field * EPB + element; matrices AW [DIM][MP][KU], AL [NF][MP][KL]
  static constexpr int KUR = round_up(NP, T::KSTEP);     // k extent, volume
  static constexpr int NFPK = round_up(NFP, T::KSTEP);   // k extent per face
  static constexpr int KU = T::stride(KUR);
  static constexpr int KS = T::stride(NF * NFPK);
  static constexpr int KL = T::stride(NFPK);
  static constexpr int G_MAT = NAC * (DIM * MP * KU + NF * MP * KL);
  static constexpr int G_PER_ELEM = NU * (KU + KS + 1) + GEO;
  static constexpr int EPB_G_RAW = (SMEM_BUDGET / RB - G_MAT - 1024 / RB) / G_PER_ELEM;
  // elements per tile, a multiple of 4: the float32 7-species p3 tile of 12
  // gives the 256 threads 240 nodes, 480 face nodes and 40 (n-tile, m-tile)
  // items for the 8 warps, with little idle time at the tile's barriers
  static constexpr int EPB_GRAD = imax(8, imin(32, EPB_G_RAW / 4 * 4));
  static constexpr int NCOL_G = round_up(NU * EPB_GRAD, 8);

  // rhs kernel operands: B [col][KB] = [G_0 .. G_{DIM-1} | S] per column,
  // A [MP][KB] = [-W_0 .. -W_{DIM-1} | LIFT]
  static constexpr int KR = DIM * NP + NFN;
  static constexpr int KRR = round_up(KR, T::KSTEP);
  static constexpr int KB = T::stride(KRR);
  static constexpr int R_MAT = NAC * MP * KB;
  static constexpr int R_PER_ELEM =
      NC * KB + NC * NP + (MIX ? 2 * NP : 0) + NS * NP + 3 * NP + GEO;
  static constexpr int EPB_R_RAW = (SMEM_BUDGET / RB - R_MAT - 1024 / RB) / R_PER_ELEM;
  static constexpr int EPB_RHS = imax(4, imin(32, EPB_R_RAW >= 8 ? EPB_R_RAW / 8 * 8
                                                                 : EPB_R_RAW / 4 * 4));
  static constexpr int NCOL_R = round_up(NC * EPB_RHS, 8);

  // split right-hand side: per-node flux record = total flux F[c][j] then
  // p, c, gamma, |v| + c (padded to 16 bytes); the surface kernel holds only
  // the contraction operands in shared memory
  static constexpr int FW = flux_record_width(DIM, NC);
  static constexpr int S_BUDGET = (RB == 8 ? 100 : 92) * 1024;
  // resident blocks: float64 mixture state needs more registers per thread
  static constexpr int MINB_NODE = (RB == 8 && NS > 2) ? 3 : 4;
  static constexpr int MINB_SURF = 2;
  static constexpr int S_PER_ELEM = NC * KB + GEO;
  static constexpr int EPB_S_RAW = (S_BUDGET / RB - R_MAT - 1024 / RB) / S_PER_ELEM;
  static constexpr int EPB_SURF = imax(4, imin(32, EPB_S_RAW / 4 * 4));
  static constexpr int NCOL_S = round_up(NC * EPB_SURF, 8);
  static size_t smem_surface(int nperm) {
    return (size_t)(R_MAT + NCOL_S * KB + EPB_SURF * GEO) * RB + NFN * 4 + EPB_SURF * NF * 4 +
           (size_t)nperm * NFP + 64;
  }

  static constexpr int MINB_GRAD = 2;
  static size_t smem_grad(int nperm) {
    return (size_t)(G_MAT + NCOL_G * (KU + KS) + EPB_GRAD * GEO + NU * EPB_GRAD) * RB +
           NFN * 4 + EPB_GRAD * NF * 4 + (size_t)nperm * NFP + 64;
  }
  static size_t smem_rhs(int nperm) {
    return (size_t)(R_MAT + NCOL_R * KB +
                    EPB_RHS * (NC * NP + (MIX ? 2 * NP : 0) + NS * NP + 3 * NP + GEO)) * RB +
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

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

// D(16x8) += A(16x8) * B(8x8) with tf32 operands, f32 accumulate.  Fragments
// (g = lane/4, t = lane%4):  A: a0 A[g][t], a1 A[g+8][t], a2 A[g][t+4],
// a3 A[g+8][t+4];  B: b0 B[t][g], b1 B[t+4][g];  D: d0 D[g][2t], d1 D[g][2t+1],
// d2 D[g+8][2t], d3 D[g+8][2t+1].
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Three-term split product  A*B ~= Ahi*Bhi + Ahi*Blo + Alo*Bhi  on tf32
// tensor cores; A arrives pre-split (hi/lo in shared memory), B is split here.
__device__ __forceinline__ void mma_tf32x3(float (&d)[4], const uint32_t (&ahi)[4],
                                           const uint32_t (&alo)[4], float b0, float b1) {
  const uint32_t bh0 = to_tf32(b0), bh1 = to_tf32(b1);
  const uint32_t bl0 = to_tf32(b0 - __uint_as_float(bh0));
  const uint32_t bl1 = to_tf32(b1 - __uint_as_float(bh1));
  mma_tf32(d, alo, bh0, bh1);
  mma_tf32(d, ahi, bl0, bl1);
  mma_tf32(d, ahi, bh0, bh1);
}

// B operand split once into tf32 hi/lo words (shared by several A operands)
struct SplitB {
  uint32_t h0, h1, l0, l1;
  SplitB() = default;
  __device__ __forceinline__ SplitB(float b0, float b1) {
    h0 = to_tf32(b0);
    h1 = to_tf32(b1);
    l0 = to_tf32(b0 - __uint_as_float(h0));
    l1 = to_tf32(b1 - __uint_as_float(h1));
  }
};

// the same three-term product with B already split
__device__ __forceinline__ void mma_tf32x3(float (&d)[4], const uint32_t (&ahi)[4],
                                           const uint32_t (&alo)[4], const SplitB& b) {
  mma_tf32(d, alo, b.h0, b.h1);
  mma_tf32(d, ahi, b.l0, b.l1);
  mma_tf32(d, ahi, b.h0, b.h1);
}

// A fragment of the tf32 m16n8k8 product (16 rows from m0, 8 columns from
// k0, row stride `stride` floats, rows 16-byte aligned) in one ldmatrix.x4:
// the four 8x8 b16 matrices are the 8x4-word blocks (rows 0-7 | 8-15) x
// (k 0-3 | 4-7); lane l gives the row address of block l / 8, and receives
// word (l % 4) of row (l / 4) of each block -- exactly a0..a3.
__device__ __forceinline__ void load_a_tf32_ldsm(uint32_t (&a)[4], const float* am, int stride,
                                                 int m0, int k0, int lane) {
  const int row = m0 + (lane & 7) + ((lane >> 3) & 1) * 8;
  const int kk = k0 + ((lane >> 4) << 2);
  const uint32_t addr = (uint32_t)__cvta_generic_to_shared(am + row * stride + kk);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
               : "r"(addr));
}

// hi/lo tf32 split of a float64 reference-matrix entry
__device__ __forceinline__ void split_tf32(double v, float& hi, float& lo) {
  hi = __uint_as_float(to_tf32((float)v));
  lo = __uint_as_float(to_tf32((float)(v - (double)hi)));
}

// Store one reference-matrix entry into the A operand copies of type R.
template <class R>
__device__ __forceinline__ void put_a(R* a, int stride_copy, int i, double v) {
  if constexpr (sizeof(R) == 8) {
    a[i] = v;
  } else {
    float hi, lo;
    split_tf32(v, hi, lo);
    a[i] = hi;
    a[stride_copy + i] = lo;
  }
}

// A fragment (tf32) of rows m0.., k columns k0.. from a shared copy
__device__ __forceinline__ void load_a_tf32(uint32_t (&a)[4], const float* am, int stride, int m0,
                                            int k0, int g, int t) {
  a[0] = __float_as_uint(am[(m0 + g) * stride + k0 + t]);
  a[1] = __float_as_uint(am[(m0 + g + 8) * stride + k0 + t]);
  a[2] = __float_as_uint(am[(m0 + g) * stride + k0 + t + 4]);
  a[3] = __float_as_uint(am[(m0 + g + 8) * stride + k0 + t + 4]);
}

// Everything below has internal linkage: every translation unit that
// includes this file launches its own copies of the kernels, which read that
// unit's constant banks.  (With external linkage the host linker may keep one
// unit's launch stub for an instantiation that two units share.)
namespace {

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

// Face pairing of the tile's elements into shared memory (read back after
// the next barrier), so that a face-node item starts its neighbour gathers
// one global-memory round trip earlier.
template <int NF>
__device__ __forceinline__ void stage_conn(const int32_t* __restrict__ conn_g, int e0, int ne,
                                           int32_t* conn_s) {
  for (int idx = threadIdx.x; idx < ne * NF; idx += blockDim.x)
    conn_s[idx] = conn_g[(int64_t)e0 * NF + idx];
}

// Interior state of a boundary face node: q- from HBM, the operator
// temperature (mixtures) or the ideal gas's, and p, c, gamma.
template <class R, int DIM, int NS, bool MIX>
__device__ __forceinline__ void boundary_minus(const DGArgs<R>& a, const GasParams& g, int64_t EN,
                                               int64_t gm, R* qm, NodeState<R, DIM, NS>& sm) {
  constexpr int NC = DIM + 2 + NS;
#pragma unroll
  for (int c = 0; c < NC; ++c) qm[c] = a.q[c * EN + gm];
  make_state<R, DIM, NS>(qm, MIX ? a.t_op[gm] : R(0), g, sm);
}

// The gradient pass's face value at a Mengaldo boundary face node:
// (state_bc.cv, temperature_bc) into up[NC + 1] (boundary.py:732-793).
template <class R, int DIM, int NS, bool MIX>
__device__ __noinline__ void mengaldo_grad_value(const DGArgs<R> a, const GasParams g, int kind,
                                                 int bf, int m, int nfp, int64_t EN, int64_t gm,
                                                 R n0, R n1, R n2, R* up) {
  constexpr int NC = DIM + 2 + NS;
  const R n[3] = {n0, n1, n2};
  R qm[NC];
  NodeState<R, DIM, NS> sm;
  boundary_minus<R, DIM, NS, MIX>(a, g, EN, gm, qm, sm);
  R par[NC + 1];
  const int64_t bstride = (int64_t)a.nbf * nfp, bo = (int64_t)bf * nfp + m;
#pragma unroll
  for (int c = 0; c <= NC; ++c) par[c] = bk_needs_bext(kind) ? a.bext[c * bstride + bo] : R(0);
  R qbc[NC];
  const R tbc = bc_state_cv<R, DIM, NS>(kind, g, qm, sm.t, sm.p, sm.c, sm.gamma, n, par, qbc);
#pragma unroll
  for (int c = 0; c < NC; ++c) up[c] = qbc[c];
  up[NC] = tbc;
}


// {{{ mixture temperature

// plain form: T1 = Newton(seed), T2 = Newton(T1), fixed iteration count.
// The reference's fixed-count solve has no convergence check (its drivers
// check the temperature update: mirgecom examples/autoignition.py:526-530);
// here a node whose T2 (or, without T2, one further Newton step) moved by
// more than 1e-6 of T1, or whose temperature is not positive and finite,
// sets ST_NEWTON_MISS in *status*.  The temperatures written are the
// reference's either way.
template <class R, int DIM, int NS>
__global__ void __launch_bounds__(256) k_mixture_state(int64_t nnodes, const R* __restrict__ q,
                                                       const R* __restrict__ tseed,
                                                       R* __restrict__ t1, R* __restrict__ t2,
                                                       int32_t* status, GasParams g) {
  constexpr int NC = DIM + 2 + NS;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  bool miss = false;
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nnodes; n += stride) {
    R qq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qq[c] = q[(int64_t)c * nnodes + n];
    const R ta = node_temperature<R, DIM, NS>(qq, tseed[n], g);
    t1[n] = ta;
    R tb;
    if (t2) {
      tb = node_temperature<R, DIM, NS>(qq, ta, g);
      t2[n] = tb;
    } else {
      GasParams g1 = g;
      g1.niter = 1;
      tb = node_temperature<R, DIM, NS>(qq, ta, g1);
    }
    miss |= !(ta > R(0) && tb > R(0) && fabs(tb - ta) <= R(1e-6) * ta && ta < R(1e30));
  }
  if (miss && status) atomicOr(status, ST_NEWTON_MISS);
}

// mixed form: float32 Newton from the learned guess (if given) else the
// seed, stopped once the update falls below 1e-5 of T (float32 cannot
// resolve e_mix(T) much further once formation enthalpies of ~1e7 J/kg enter
// e); then the float64 residual check
//   |e(q) - e_mix(T)| / (c_v(T) T) <= rtol
// accepts the result and applies that float64 residual as the final Newton
// step (quadratic convergence: the remaining error is of order rtol^2).  A
// rejected result is recomputed from the plain guess (seed).  iters
// (optional) receives the float32 iteration count per node, with 1000
// added when the fallback ran; ST_NEWTON_MISS flags nodes that fail both.
template <int DIM, int NS>
__global__ void __launch_bounds__(256) k_mixture_state_mixed(
    int64_t nnodes, const float* __restrict__ q, const float* __restrict__ tseed,
    const float* __restrict__ tguess, float* __restrict__ tout, int32_t* __restrict__ iters,
    int maxit, float rtol, int32_t* status, GasParams g) {
  constexpr int NC = DIM + 2 + NS;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  bool miss = false;
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nnodes; n += stride) {
    float qq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qq[c] = q[(int64_t)c * nnodes + n];
    float y[NS], e32;
    double yd[NS], e64;
    mixed_newton_inputs<DIM, NS>(qq, y, yd, e32, e64);
    int used = 0;
    float t = 0.f;
    bool ok = false;
    // attempt 0: learned guess (when given); attempt 1: the plain guess (seed)
    for (int attempt = tguess ? 0 : 1; attempt < 2 && !ok; ++attempt) {
      t = (attempt == 0) ? tguess[n] : tseed[n];
      ok = mixed_newton<NS>(y, yd, e32, e64, t, maxit, (double)rtol, used);
      if (!ok && attempt == 0) used += 1000;
    }
    if (!ok) miss = true;
    tout[n] = t;
    if (iters) iters[n] = used;
  }
  if (miss) atomicOr(status, ST_NEWTON_MISS);
}

// }}}

// {{{ gradient kernel

// Gradient pass (grad_cv_operator + grad_t_operator): a persistent kernel
// that builds W_r and LIFT_f once per CTA and loops over element tiles:
//   phase 1  U = u - u0 per node (u0 the element's node-0 value; the discrete
//            gradient of a constant vanishes, so the shift keeps large means
//            out of the contraction and changes nothing in exact arithmetic)
//   phase 2  S = fscale (u* - u0) per face node and group of four fields,
//            u* the BR1 central value, the prescribed exterior value, or the
//            interior value (dummy boundary)
//   phase 3  du_r = W_r U, L_f = LIFT_f S on the tensor cores per (n-tile,
//            m-tile), grad_j = sum_f n_fj L_f - sum_r (dr_r/dx_j) du_r
template <class R, int DIM, int ORDER, int NS, bool MIX>
__global__ void __launch_bounds__(256, (Cfg<R, DIM, ORDER, NS, MIX>::MINB_GRAD))
    k_grad(DGArgs<R> a, GasParams g) {
  using C = Cfg<R, DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = C::NP, NF = C::NF, NFP = C::NFP, NFN = C::NFN, NC = C::NC, NU = C::NU;
  constexpr int EPB = C::EPB_GRAD, MP = C::MP, MT = C::MT, NAC = C::NAC;
  constexpr int KU = C::KU, KS = C::KS, KL = C::KL, NFPK = C::NFPK, NCOL = C::NCOL_G;
  constexpr int KUR = C::KUR;
  constexpr int AWN = DIM * MP * KU, ALN = NF * MP * KL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* aw = reinterpret_cast<R*>(smem_raw);                  // [NAC][DIM][MP][KU]
  R* al = aw + NAC * AWN;                                  // [NAC][NF][MP][KL]
  R* bu = al + NAC * ALN;                                  // [NCOL][KU]
  R* bs = bu + NCOL * KU;                                  // [NCOL][KS]
  R* rx_s = bs + NCOL * KS;                                // [EPB][DIM][DIM]
  R* nrm_s = rx_s + EPB * DIM * DIM;                       // [EPB][NF][DIM]
  R* fs_s = nrm_s + EPB * NF * DIM;                        // [EPB][NF]
  R* u0_s = fs_s + EPB * NF;                               // [NU][EPB]
  int* fn_s = reinterpret_cast<int*>(u0_s + NU * EPB);     // [NF*NFP]
  int32_t* conn_s = fn_s + NFN;                            // [EPB][NF]
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(conn_s + EPB * NF);

  const int E = a.nelem;
  const int64_t EN = (int64_t)E * NP;
  // whole rows of NP floats can be moved in 16-byte pieces
  const bool rows16 =
      ((reinterpret_cast<uintptr_t>(a.q) | reinterpret_cast<uintptr_t>(a.t_op)) & 15) == 0 &&
      (KU * sizeof(R)) % 16 == 0;

  // reference operators (zero padded; hi/lo tf32 split on the mixed path)
  for (int i = threadIdx.x; i < AWN; i += blockDim.x) {
    const int r = i / (MP * KU), row = (i / KU) % MP, k = i % KU;
    put_a<R>(aw, AWN, i, (row < NP && k < NP) ? c_ref64[S::OFF_W + (r * NP + row) * NP + k] : 0.0);
  }
  for (int i = threadIdx.x; i < ALN; i += blockDim.x) {
    const int f = i / (MP * KL), row = (i / KL) % MP, m = i % KL;
    put_a<R>(al, ALN, i,
             (row < NP && m < NFP) ? c_ref64[S::OFF_LIFT + row * NFN + f * NFP + m] : 0.0);
  }
  // padding rows/columns of the B operands stay zero for the whole kernel
  for (int i = threadIdx.x; i < NCOL * (KU + KS); i += blockDim.x) bu[i] = R(0);
  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const int nwarps = blockDim.x >> 5;
  constexpr int NACC = C::TF32 ? 4 : 2;     // accumulator entries per lane per m-tile
  // elements [0, nowned) of a partition (0: all)
  const int EOWN = a.nowned > 0 ? a.nowned : E;
  const int ntiles = (EOWN + EPB - 1) / EPB;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * EPB;
    const int ne = imin(EPB, EOWN - e0);
    // the previous tile's phase 3 reads rx_s and nrm_s, which load_geometry
    // overwrites before its own first barrier
    __syncthreads();
    stage_conn<NF>(a.conn, e0, ne, conn_s);
    load_geometry<R, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);

    // phase 1: shifted conserved fields and temperature.  With the operator
    // temperature given (mixtures) one (element, field) row per item: the
    // row's NP values in 16-byte loads, shifted by its first; otherwise one
    // node per item (the ideal-gas temperature needs all fields of a node)
    bool rows_done = false;
    if constexpr (MIX && NP % 4 == 0 && sizeof(R) == 4) {
      if (rows16) {
        for (int it = threadIdx.x; it < ne * NU; it += blockDim.x) {
          const int e = it % ne, c = it / ne;
          const float* src = (c < NC ? a.q + c * EN : a.t_op) + (int64_t)(e0 + e) * NP;
          float4 v[NP / 4];
#pragma unroll
          for (int i = 0; i < NP / 4; ++i) v[i] = reinterpret_cast<const float4*>(src)[i];
          const float u0 = v[0].x;
          float4* dst = reinterpret_cast<float4*>(bu + (c * EPB + e) * KU);
#pragma unroll
          for (int i = 0; i < NP / 4; ++i)
            dst[i] = make_float4(v[i].x - u0, v[i].y - u0, v[i].z - u0, v[i].w - u0);
          u0_s[c * EPB + e] = u0;
        }
        rows_done = true;
      }
    }
    if (!rows_done) {
      for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
        const int e = idx / NP, k = idx % NP;
        const int64_t gn = (int64_t)e0 * NP + idx, g0 = (int64_t)(e0 + e) * NP;
        R qq[NC], q0[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          qq[c] = a.q[c * EN + gn];
          q0[c] = a.q[c * EN + g0];
        }
        const R t = MIX ? a.t_op[gn] : node_temperature<R, DIM, NS>(qq, R(0), g);
        const R t0 = MIX ? a.t_op[g0] : node_temperature<R, DIM, NS>(q0, R(0), g);
#pragma unroll
        for (int c = 0; c < NC; ++c) bu[(c * EPB + e) * KU + k] = qq[c] - q0[c];
        bu[(NC * EPB + e) * KU + k] = t - t0;
        if (k == 0) {
#pragma unroll
          for (int c = 0; c < NC; ++c) u0_s[c * EPB + e] = q0[c];
          u0_s[NC * EPB + e] = t0;
        }
      }
    }
    __syncthreads();

    // phase 2: face values  fscale * (u* - u0), one face node per item
    for (int fnode = threadIdx.x; fnode < ne * NFN; fnode += blockDim.x) {
      const int e = fnode / NFN, fm = fnode % NFN, f = fm / NFP, m = fm % NFP;
      const int k = fn_s[fm];
      const int cn = conn_s[e * NF + f];
      const R fsc = fs_s[e * NF + f];
      // 0: two-sided average with node gi; 1: prescribed exterior; 2: interior
      // value; 3: Mengaldo boundary state (becomes 1)
      int mode = 2;
      int64_t gi = 0;
      int bf = 0;
      if (cn >= 0) {
        const int en = cn >> 8, pr = cn & 255;
        const int kn = (pr < a.nperm) ? perm_s[pr * NFP + m] : NP;
        if (en >= E || kn >= NP) {
          atomicOr(a.status, ST_BAD_INDEX);
        } else {
          gi = (int64_t)en * NP + kn;
          mode = 0;
        }
      } else {
        bf = -(cn + 1);
        int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
        if ((bk_needs_bext(kind) && !a.bext) || kind > BK_OUTFLOW) kind = -1;
        if (kind == BK_PRESCRIBED) {
          mode = 1;
        } else if (bk_mengaldo(kind)) {
          mode = 3;
        } else if (kind < 0) {
          atomicOr(a.status, ST_BAD_INDEX);
        }
      }
      R* bcol = bs + e * KS + f * NFPK + m;
      if (mode == 2) {
#pragma unroll
        for (int c = 0; c < NU; ++c) bcol[c * EPB * KS] = fsc * bu[(c * EPB + e) * KU + k];
        continue;
      }
      const int64_t bstride = (int64_t)a.nbf * NFP, bo = (int64_t)bf * NFP + m;
      R up[NU];
      if (mode == 3) {
        const R* nf = nrm_s + (e * NF + f) * DIM;
        mengaldo_grad_value<R, DIM, NS, MIX>(a, g, a.bkind[bf], bf, m, NFP, EN,
                                             (int64_t)(e0 + e) * NP + k, nf[0], nf[1],
                                             DIM > 2 ? nf[DIM - 1] : R(0), up);
        mode = 1;
      } else {
#pragma unroll
        for (int c = 0; c < NC; ++c)
          up[c] = (mode == 0) ? a.q[c * EN + gi] : a.bext[c * bstride + bo];
        if (MIX)
          up[NC] = (mode == 0) ? a.t_op[gi] : a.bext[NC * bstride + bo];
        else
          up[NC] = node_temperature<R, DIM, NS>(up, R(0), g);
      }
#pragma unroll
      for (int c = 0; c < NU; ++c) {
        const R um = bu[(c * EPB + e) * KU + k];           // u- - u0
        const R u0 = u0_s[c * EPB + e];
        const R v = (mode == 0) ? ((up[c] - u0) + um) * R(0.5) : up[c] - u0;
        bcol[c * EPB * KS] = fsc * v;
      }
    }
    __syncthreads();

    // phase 3: contraction and metric combination.  float32: one item per
    // n-tile and every m-tile, each B value split into tf32 hi/lo once
    if constexpr (C::TF32) {
      for (int nt = warp; nt < NCOL / 8; nt += nwarps) {
        float du[MT][DIM][4], lf[MT][NF][4];
#pragma unroll
        for (int t = 0; t < MT; ++t)
#pragma unroll
          for (int v = 0; v < 4; ++v) {
#pragma unroll
            for (int r = 0; r < DIM; ++r) du[t][r][v] = 0.f;
#pragma unroll
            for (int f = 0; f < NF; ++f) lf[t][f][v] = 0.f;
          }
        const R* bcol = bu + (nt * 8 + gq) * KU + tq;
        const R* scol = bs + (nt * 8 + gq) * KS + tq;
#pragma unroll
        for (int ks = 0; ks < KUR / 8; ++ks) {
          const SplitB b(bcol[ks * 8], bcol[ks * 8 + 4]);
#pragma unroll
          for (int t = 0; t < MT; ++t)
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
              uint32_t ah[4], alo[4];
              load_a_tf32_ldsm(ah, aw + r * MP * KU, KU, t * 16, ks * 8, lane);
              load_a_tf32_ldsm(alo, aw + AWN + r * MP * KU, KU, t * 16, ks * 8, lane);
              mma_tf32x3(du[t][r], ah, alo, b);
            }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
          for (int ks = 0; ks < NFPK / 8; ++ks) {
            const SplitB b(scol[f * NFPK + ks * 8], scol[f * NFPK + ks * 8 + 4]);
#pragma unroll
            for (int t = 0; t < MT; ++t) {
              uint32_t ah[4], alo[4];
              load_a_tf32_ldsm(ah, al + f * MP * KL, KL, t * 16, ks * 8, lane);
              load_a_tf32_ldsm(alo, al + ALN + f * MP * KL, KL, t * 16, ks * 8, lane);
              mma_tf32x3(lf[t][f], ah, alo, b);
            }
          }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int col = nt * 8 + 2 * tq + h;
          const int c = col / EPB, e = col % EPB;
          if (c >= NU || e >= ne) continue;
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
#pragma unroll
          for (int t = 0; t < MT; ++t)
#pragma unroll
            for (int half = 0; half < 2; ++half) {
              const int i = t * Tile<R>::MROW + gq + 8 * half;
              if (i >= NP) continue;
              const int v = 2 * half + h;
#pragma unroll
              for (int j = 0; j < DIM; ++j) {
                R gsum = R(0);
#pragma unroll
                for (int f = 0; f < NF; ++f) gsum += nre[f][j] * lf[t][f][v];
#pragma unroll
                for (int r = 0; r < DIM; ++r) gsum -= rxe[r][j] * du[t][r][v];
                outp[(int64_t)j * EN + i] = gsum;
              }
            }
        }
      }
    } else
    for (int w = warp; w < (NCOL / 8) * MT; w += nwarps) {
      const int nt = w / MT, t = w % MT;
      R du[DIM][NACC], lf[NF][NACC];
#pragma unroll
      for (int v = 0; v < NACC; ++v) {
#pragma unroll
        for (int r = 0; r < DIM; ++r) du[r][v] = R(0);
#pragma unroll
        for (int f = 0; f < NF; ++f) lf[f][v] = R(0);
      }
      const R* bcol = bu + (nt * 8 + gq) * KU + tq;
      const R* scol = bs + (nt * 8 + gq) * KS + tq;
      if constexpr (!C::TF32) {
#pragma unroll
        for (int ks = 0; ks < KUR / 4; ++ks) {
          const double b = bcol[ks * 4];
#pragma unroll
          for (int r = 0; r < DIM; ++r)
            dmma884(du[r], aw[(r * MP + t * 8 + gq) * KU + ks * 4 + tq], b);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
          for (int ks = 0; ks < NFPK / 4; ++ks)
            dmma884(lf[f], al[(f * MP + t * 8 + gq) * KL + ks * 4 + tq], scol[f * NFPK + ks * 4]);
      } else {
        // B split once per k-step and shared by the DIM operators; A
        // fragments by ldmatrix
#pragma unroll
        for (int ks = 0; ks < KUR / 8; ++ks) {
          const SplitB b(bcol[ks * 8], bcol[ks * 8 + 4]);
#pragma unroll
          for (int r = 0; r < DIM; ++r) {
            uint32_t ah[4], alo[4];
            load_a_tf32_ldsm(ah, aw + r * MP * KU, KU, t * 16, ks * 8, lane);
            load_a_tf32_ldsm(alo, aw + AWN + r * MP * KU, KU, t * 16, ks * 8, lane);
            mma_tf32x3(du[r], ah, alo, b);
          }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
          for (int ks = 0; ks < NFPK / 8; ++ks) {
            const SplitB b(scol[f * NFPK + ks * 8], scol[f * NFPK + ks * 8 + 4]);
            uint32_t ah[4], alo[4];
            load_a_tf32_ldsm(ah, al + f * MP * KL, KL, t * 16, ks * 8, lane);
            load_a_tf32_ldsm(alo, al + ALN + f * MP * KL, KL, t * 16, ks * 8, lane);
            mma_tf32x3(lf[f], ah, alo, b);
          }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int col = nt * 8 + 2 * tq + h;
        const int c = col / EPB, e = col % EPB;
        if (c >= NU || e >= ne) continue;
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
#pragma unroll
        for (int half = 0; half < NACC / 2; ++half) {
          const int i = t * Tile<R>::MROW + gq + 8 * half;
          if (i >= NP) continue;
          const int v = 2 * half + h;
#pragma unroll
          for (int j = 0; j < DIM; ++j) {
            R gsum = R(0);
#pragma unroll
            for (int f = 0; f < NF; ++f) gsum += nre[f][j] * lf[f][v];
#pragma unroll
            for (int r = 0; r < DIM; ++r) gsum -= rxe[r][j] * du[r][v];
            outp[(int64_t)j * EN + i] = gsum;
          }
        }
      }
    }
  }
}

// }}}

// {{{ rhs kernel (Euler when VISC is false)

template <class R, int DIM, int ORDER, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__(256, (Cfg<R, DIM, ORDER, NS, MIX>::MINB))
    k_rhs(DGArgs<R> a, GasParams g) {
  using C = Cfg<R, DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = C::NP, NF = C::NF, NFP = C::NFP, NFN = C::NFN, NC = C::NC;
  constexpr int EPB = C::EPB_RHS, MP = C::MP, MT = C::MT, KB = C::KB, KR = C::KR;
  constexpr int KRR = C::KRR, NCOL = C::NCOL_R, NAC = C::NAC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* am = reinterpret_cast<R*>(smem_raw);                  // [NAC][MP][KB]
  R* bm = am + NAC * MP * KB;                              // [NCOL][KB]
  R* q_s = bm + NCOL * KB;                                 // [NC][EPB][NP]
  R* t_s = q_s + NC * EPB * NP;                            // [2][EPB][NP] (MIX)
  R* src_s = t_s + (MIX ? 2 * EPB * NP : 0);               // [NS][EPB][NP] (MIX)
  R* pcg_s = src_s + NS * EPB * NP;                        // [3][EPB][NP] p, c, gamma
  R* rx_s = pcg_s + 3 * EPB * NP;                          // [EPB][DIM][DIM]
  R* nrm_s = rx_s + EPB * DIM * DIM;
  R* fs_s = nrm_s + EPB * NF * DIM;
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
    put_a<R>(am, MP * KB, i, v);
  }
  for (int i = threadIdx.x; i < NCOL * KB; i += blockDim.x) bm[i] = R(0);
  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];
  for (int c = 0; c < NC; ++c)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x)
      q_s[(c * EPB) * NP + idx] = a.q[c * EN + (int64_t)e0 * NP + idx];
  if (MIX)
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
      t_s[idx] = a.t_op[(int64_t)e0 * NP + idx];
      t_s[EPB * NP + idx] = sources ? a.t_src[(int64_t)e0 * NP + idx] : R(0);
    }
  load_geometry<R, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);
  __syncthreads();

  // phase 2: volume flux F = F_V - F_I, metric-combined into B[col][r*NP + k]
  for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
    const int e = idx / NP, k = idx % NP;
    R qq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qq[c] = q_s[(c * EPB) * NP + idx];
    NodeState<R, DIM, NS> st;
    make_state<R, DIM, NS>(qq, MIX ? t_s[idx] : R(0), g, st);
    pcg_s[idx] = st.p;
    pcg_s[EPB * NP + idx] = st.c;
    pcg_s[2 * EPB * NP + idx] = st.gamma;
    R fl[NC][DIM];
    inviscid_flux<R, DIM, NS>(st, fl);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int j = 0; j < DIM; ++j) fl[c][j] = -fl[c][j];
    if (VISC) {
      R gqv[NC][DIM], gt[DIM];
      const int64_t gi = (int64_t)e0 * NP + idx;
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) gqv[c][j] = a.grad[((int64_t)c * DIM + j) * EN + gi];
#pragma unroll
      for (int j = 0; j < DIM; ++j) gt[j] = a.grad[((int64_t)NC * DIM + j) * EN + gi];
      R fv[NC][DIM];
      viscous_flux<R, DIM, NS, MIX>(st, gqv, gt, fv);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) fl[c][j] = fv[c][j] + fl[c][j];
    }
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        R acc = R(0);
#pragma unroll
        for (int j = 0; j < DIM; ++j) acc += rx_s[e * DIM * DIM + r * DIM + j] * fl[c][j];
        bm[(c * EPB + e) * KB + r * NP + k] = acc;
      }
    if constexpr (MIX && NS > 0) {
      if (sources) {
        R om[NS];
        production_rates<R, NS>(st.rho, t_s[EPB * NP + idx], st.y, (R)g.zero_level, om);
#pragma unroll
        for (int s = 0; s < NS; ++s) src_s[(s * EPB) * NP + idx] = mech<R>().mw[s] * om[s];
      }
    }
  }
  __syncthreads();

  // phase 3: numerical face flux fscale * (F*_V - F*_I) into B[col][DIM*NP + fm]
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
    // own side: the inviscid flux needs q, p, c, gamma only, kept from phase 2
    make_state_light<R, DIM, NS>(qm, pcg_s[e * NP + k], pcg_s[EPB * NP + e * NP + k],
                                 pcg_s[2 * EPB * NP + e * NP + k], sm);
    // own total flux . n from the metric-combined volume flux:
    // F.n = (sum_r N_r G_r) / |rx^T N|
    R nmag2 = R(0);
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      R a2 = R(0);
#pragma unroll
      for (int r = 0; r < DIM; ++r)
        a2 += rx_s[e * DIM * DIM + r * DIM + j] * RefBank<R>::get(S::OFF_NREF + f * DIM + r);
      nmag2 += a2 * a2;
    }
    const R inmag = R(1) / sqrt(nmag2);
    R ftm[NC], f0n[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      R acc = R(0), acc0 = R(0);
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        const R nr = RefBank<R>::get(S::OFF_NREF + f * DIM + r);
        acc += nr * bm[(c * EPB + e) * KB + r * NP + k];
        acc0 += nr * bm[(c * EPB + e) * KB + r * NP];
      }
      ftm[c] = acc * inmag;
      f0n[c] = acc0 * inmag;     // element-constant shift: node-0 flux . n
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
        make_state<R, DIM, NS>(qp, MIX ? a.t_op[gi] : R(0), g, sp);
      }
    } else {
      const int bf = -(cn + 1);
      const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
      if (kind == BK_PRESCRIBED) {
        mode = 2;
        const int64_t bstride = (int64_t)a.nbf * NFP;
#pragma unroll
        for (int c = 0; c < NC; ++c) qp[c] = a.bext[c * bstride + (int64_t)bf * NFP + m];
        make_state<R, DIM, NS>(qp, MIX ? a.bext[NC * bstride + (int64_t)bf * NFP + m] : R(0),
                               g, sp);
      } else {
        if (kind != BK_DUMMY) atomicOr(a.status, ST_BAD_INDEX);
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
        R gqp[NC][DIM], gtp[DIM];
        const int64_t gsrc = (mode == 0) ? gi : (int64_t)(e0 + e) * NP + k;
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int j = 0; j < DIM; ++j) gqp[c][j] = a.grad[((int64_t)c * DIM + j) * EN + gsrc];
#pragma unroll
        for (int j = 0; j < DIM; ++j) gtp[j] = a.grad[((int64_t)NC * DIM + j) * EN + gsrc];
        R fvp[NC][DIM];
        viscous_flux<R, DIM, NS, MIX>(sp, gqp, gtp, fvp);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          R fvpn = R(0);
#pragma unroll
          for (int j = 0; j < DIM; ++j) fvpn += fvp[c][j] * n[j];
          const R fvmn = ftm[c] + fim[c];
          out[c] += (fvmn + fvpn) * R(0.5);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) bm[(c * EPB + e) * KB + DIM * NP + fm] = fsc * (out[c] - f0n[c]);
  }
  __syncthreads();
  // subtract the node-0 flux from the volume terms: with the face terms
  // shifted by F0 . n above, the divergence is unchanged in exact arithmetic
  for (int p = threadIdx.x; p < NC * ne * DIM; p += blockDim.x) {
    const int r = p % DIM, ce = p / DIM, c = ce / ne, e = ce % ne;
    R* row = bm + (c * EPB + e) * KB + r * NP;
    const R g0 = row[0];
#pragma unroll 4
    for (int k = 0; k < NP; ++k) row[k] -= g0;
  }
  __syncthreads();

  // phase 4: rhs = [-W | LIFT] [G ; S] on the tensor cores (+ sources)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  constexpr int NACC = C::TF32 ? 4 : 2;
  bool bad = false;
  for (int nt = warp; nt < NCOL / 8; nt += blockDim.x >> 5) {
    R d[MT][NACC];
#pragma unroll
    for (int t = 0; t < MT; ++t)
#pragma unroll
      for (int v = 0; v < NACC; ++v) d[t][v] = R(0);
    const R* bcol = bm + (nt * 8 + gq) * KB + tq;
    if constexpr (!C::TF32) {
#pragma unroll 5
      for (int ks = 0; ks < KRR / 4; ++ks) {
        const double b = bcol[ks * 4];
#pragma unroll
        for (int t = 0; t < MT; ++t) dmma884(d[t], am[(t * 8 + gq) * KB + ks * 4 + tq], b);
      }
    } else {
#pragma unroll 2
      for (int ks = 0; ks < KRR / 8; ++ks) {
        const float b0 = bcol[ks * 8], b1 = bcol[ks * 8 + 4];
#pragma unroll
        for (int t = 0; t < MT; ++t) {
          uint32_t ah[4], alo[4];
          load_a_tf32(ah, am, KB, t * 16, ks * 8, gq, tq);
          load_a_tf32(alo, am + MP * KB, KB, t * 16, ks * 8, gq, tq);
          mma_tf32x3(d[t], ah, alo, b0, b1);
        }
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int col = nt * 8 + 2 * tq + h;
      const int c = col / EPB, e = col % EPB;
      if (c >= NC || e >= ne) continue;
      R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
      for (int t = 0; t < MT; ++t)
#pragma unroll
        for (int half = 0; half < NACC / 2; ++half) {
          const int i = t * Tile<R>::MROW + gq + 8 * half;
          if (i >= NP) continue;
          R v = d[t][2 * half + h];
          if (sources && c >= 2 + DIM) v += src_s[((c - 2 - DIM) * EPB + e) * NP + i];
          outp[i] = v;
          bad |= !(v == v);
        }
    }
  }
  if (bad) atomicOr(a.status, ST_NAN);
}

// }}}

// {{{ split right-hand side: pointwise flux kernel + surface/lift kernel
//
// k_node_flux evaluates every node's state and total flux F = F_V - F_I once
// (plus p, c, gamma, the wave speed |v| + c and the Arrhenius sources) and
// writes a flux record per node.  k_surface then builds, per element tile, the metric-combined volume
// terms from the records, the numerical face fluxes from the records of both
// sides of each face node (the neighbour's flux is gathered, not
// recomputed), and contracts on the tensor cores exactly as k_rhs does.
// The split trades one record write + read per node for the 2-3x repeated
// neighbour-state evaluations of the fused kernel.

// resident 128-thread blocks of the node-flux kernel: the float64 mixture
// state needs more registers per thread
__host__ __device__ constexpr int node_flux_minb(int rb, int ns) { return (rb == 8 && ns > 2) ? 3 : 4; }

template <class R, int DIM, int NP, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__(128, node_flux_minb((int)sizeof(R), NS))
    k_node_flux(DGArgs<R> a, GasParams g) {
  constexpr int NC = DIM + 2 + NS, FW = flux_record_width(DIM, NC);
  const int64_t EN = (int64_t)a.nelem * NP;
  const bool sources = MIX && a.add_sources;
  bool bad = false;
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < EN;
       n += (int64_t)gridDim.x * blockDim.x) {
    R qq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qq[c] = a.q[c * EN + n];
    NodeState<R, DIM, NS> st;
    make_state<R, DIM, NS>(qq, MIX ? a.t_op[n] : R(0), g, st);
    R fl[NC][DIM];
    inviscid_flux<R, DIM, NS>(st, fl);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int j = 0; j < DIM; ++j) fl[c][j] = -fl[c][j];
    if (VISC) {
      R gqv[NC][DIM], gt[DIM];
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) gqv[c][j] = a.grad[((int64_t)c * DIM + j) * EN + n];
#pragma unroll
      for (int j = 0; j < DIM; ++j) gt[j] = a.grad[((int64_t)NC * DIM + j) * EN + n];
      R fv[NC][DIM];
      viscous_flux<R, DIM, NS, MIX>(st, gqv, gt, fv);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) fl[c][j] = fv[c][j] + fl[c][j];
    }
    R rec[FW];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int j = 0; j < DIM; ++j) rec[c * DIM + j] = fl[c][j];
    rec[NC * DIM] = st.p;
    rec[NC * DIM + 1] = st.c;
    rec[NC * DIM + 2] = st.gamma;
    {
      R v2 = R(0);
#pragma unroll
      for (int j = 0; j < DIM; ++j) v2 += st.v[j] * st.v[j];
      rec[NC * DIM + 3] = sqrt(v2) + st.c;
    }
#pragma unroll
    for (int i = NC * DIM + 4; i < FW; ++i) rec[i] = R(0);
    bad |= !(st.p == st.p) || !(st.c == st.c);
    R* dst = a.fbuf + n * FW;
    if constexpr (sizeof(R) == 4) {
#pragma unroll
      for (int i = 0; i < FW; i += 4)
        *reinterpret_cast<float4*>(dst + i) = make_float4(rec[i], rec[i + 1], rec[i + 2], rec[i + 3]);
    } else {
#pragma unroll
      for (int i = 0; i < FW; i += 2)
        *reinterpret_cast<double2*>(dst + i) = make_double2(rec[i], rec[i + 1]);
    }
    if constexpr (MIX && NS > 0) {
      if (sources) {
        R om[NS];
        production_rates<R, NS>(st.rho, a.t_src[n], st.y, (R)g.zero_level, om);
#pragma unroll
        for (int s = 0; s < NS; ++s) a.srcbuf[s * EN + n] = mech<R>().mw[s] * om[s];
      }
    }
  }
  if (bad) atomicOr(a.status, ST_NAN);
}

// flux record of one node into registers
template <class R, int FW>
__device__ __forceinline__ void load_record(const R* __restrict__ src, R (&rec)[FW]) {
  if constexpr (sizeof(R) == 4) {
#pragma unroll
    for (int i = 0; i < FW; i += 4) {
      const float4 v = *reinterpret_cast<const float4*>(src + i);
      rec[i] = v.x;
      rec[i + 1] = v.y;
      rec[i + 2] = v.z;
      rec[i + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < FW; i += 2) {
      const double2 v = *reinterpret_cast<const double2*>(src + i);
      rec[i] = v.x;
      rec[i + 1] = v.y;
    }
  }
}

// Record values [v0, v0 + GV) of one node into registers, in 16-byte loads;
// chunks that start at or beyond *lim* (the end of the flux part of the
// record) are skipped.
template <class R, int GV>
__device__ __forceinline__ void load_group(const R* __restrict__ src, int v0, int lim,
                                           R (&v)[GV]) {
  if constexpr (sizeof(R) == 4) {
#pragma unroll
    for (int i = 0; i < GV; i += 4) {
      float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
      if (v0 + i < lim) x = *reinterpret_cast<const float4*>(src + v0 + i);
      v[i] = x.x;
      v[i + 1] = x.y;
      v[i + 2] = x.z;
      v[i + 3] = x.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < GV; i += 2) {
      double2 x = make_double2(0.0, 0.0);
      if (v0 + i < lim) x = *reinterpret_cast<const double2*>(src + v0 + i);
      v[i] = x.x;
      v[i + 1] = x.y;
    }
  }
}

// One face node of the surface pass evaluated from full face states: HLL on
// interior faces, prescribed and dummy boundaries, and pairings that fail the
// index checks.  Follows mirgecom/inviscid.py:290-376 and viscous.py:431-544
// (F* = central(F_V) - numflux(F_I)), boundary.py:141-146 (prescribed: the
// exterior state with the interior gradients) and boundary.py:1027-1049
// (dummy: the interior flux).  Writes S_c = fsc (F*_c - F0_c . n) for every
// field c to bcol[c * cstride].  Out of line (arguments by value, no
// address of a caller variable taken), so that its face states do not enter
// the register allocation of the interior fast path.
template <class R, int DIM, int NP, int NFP, int NS, bool MIX, bool VISC>
__device__ __noinline__ void surface_face_general(const DGArgs<R> a, const GasParams g,
                                                  int64_t EN, int64_t gm, int64_t g0, int m,
                                                  int cn, R n0, R n1, R n2, R fsc,
                                                  const uint8_t* perm_s, R* bcol, int cstride) {
  const R n[3] = {n0, n1, n2};
  constexpr int NC = DIM + 2 + NS, FW = flux_record_width(DIM, NC);
  const int E = a.nelem;
  R fr[FW], f0[FW];
  load_record<R, FW>(a.fbuf + gm * FW, fr);
  load_record<R, FW>(a.fbuf + g0 * FW, f0);
  R qm[NC], qp[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) qm[c] = a.q[c * EN + gm];
  NodeState<R, DIM, NS> sm, sp;
  make_state_light<R, DIM, NS>(qm, fr[NC * DIM], fr[NC * DIM + 1], fr[NC * DIM + 2], sm);
  R ftm[NC], f0n[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    R acc = R(0), acc0 = R(0);
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      acc += fr[c * DIM + j] * n[j];
      acc0 += f0[c * DIM + j] * n[j];
    }
    ftm[c] = acc;
    f0n[c] = acc0;
  }
  int mode = 0;   // 0 two-sided, 1 interior flux only (dummy / bad pairing)
  R fpn[NC];
  if (cn >= 0) {
    const int en = cn >> 8, pr = cn & 255;
    const int kn = (pr < a.nperm) ? perm_s[pr * NFP + m] : NP;
    if (en >= E || kn >= NP) {
      atomicOr(a.status, ST_BAD_INDEX);
      mode = 1;
    } else {
      const int64_t gi = (int64_t)en * NP + kn;
      load_record<R, FW>(a.fbuf + gi * FW, fr);     // reuse: neighbour record
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        qp[c] = a.q[c * EN + gi];
        R acc = R(0);
#pragma unroll
        for (int j = 0; j < DIM; ++j) acc += fr[c * DIM + j] * n[j];
        fpn[c] = acc;
      }
      make_state_light<R, DIM, NS>(qp, fr[NC * DIM], fr[NC * DIM + 1], fr[NC * DIM + 2], sp);
    }
  } else {
    const int bf = -(cn + 1);
    const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
    if (kind == BK_PRESCRIBED) {
      const int64_t bstride = (int64_t)a.nbf * NFP;
#pragma unroll
      for (int c = 0; c < NC; ++c) qp[c] = a.bext[c * bstride + (int64_t)bf * NFP + m];
      make_state<R, DIM, NS>(qp, MIX ? a.bext[NC * bstride + (int64_t)bf * NFP + m] : R(0), g,
                             sp);
      R fe[NC][DIM];
      inviscid_flux<R, DIM, NS>(sp, fe);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) fe[c][j] = -fe[c][j];
      if (VISC) {
        R gqp[NC][DIM], gtp[DIM];
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int j = 0; j < DIM; ++j) gqp[c][j] = a.grad[((int64_t)c * DIM + j) * EN + gm];
#pragma unroll
        for (int j = 0; j < DIM; ++j) gtp[j] = a.grad[((int64_t)NC * DIM + j) * EN + gm];
        R fv[NC][DIM];
        viscous_flux<R, DIM, NS, MIX>(sp, gqp, gtp, fv);
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int j = 0; j < DIM; ++j) fe[c][j] += fv[c][j];
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        R acc = R(0);
#pragma unroll
        for (int j = 0; j < DIM; ++j) acc += fe[c][j] * n[j];
        fpn[c] = acc;
      }
    } else {
      if (kind != BK_DUMMY) atomicOr(a.status, ST_BAD_INDEX);
      mode = 1;
    }
  }
  if (mode == 1) {
#pragma unroll
    for (int c = 0; c < NC; ++c) bcol[c * cstride] = fsc * (ftm[c] - f0n[c]);
  } else {
    // F_V . n = F . n + F_I . n on each side
    R fi[NC], fim[NC], fip[NC];
    inviscid_num_flux<R, DIM, NS>(sm, sp, qm, qp, n, a.flux_kind, fi);
    inviscid_flux_n<R, DIM, NS>(sm, n, fim);
    inviscid_flux_n<R, DIM, NS>(sp, n, fip);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      R out = -fi[c];
      if (VISC) out += ((ftm[c] + fim[c]) + (fpn[c] + fip[c])) * R(0.5);
      bcol[c * cstride] = fsc * (out - f0n[c]);
    }
  }
}

// Surface and lift pass of the split divergence: a persistent kernel (one
// grid of resident CTAs) that builds the [-W | LIFT] operand once per CTA and
// then loops over element tiles:
//   volume  G_r = sum_j (dr_r/dx_j)(F_j - F0_j) from the flux records, one
//           (node, group of four fields) per work item
//   faces   one (face node, field group) per work item.  On interior faces
//           with the Rusanov or central flux the records already hold the
//           total flux F = F_V - F_I on both sides, so
//               F*_V - F*_I = (F^- + F^+) . n / 2 - lambda (q^- - q^+) / 2
//           (lambda = max(|v| + c) for Rusanov, the node wave speeds the
//           records carry; 0 for central): no face state is rebuilt.  Other
//           faces take surface_face_general.  The tile's face pairing is
//           read from shared memory, so the neighbour gathers start one
//           global round trip earlier.
//   lift    rhs = [-W | LIFT] [G ; S] on the tensor cores, one (n-tile,
//           m-tile) per warp work item, plus the species sources.
// F0 is the record of the element's node 0: subtracting an element-constant
// flux from every volume and face value leaves the discrete divergence
// unchanged and keeps the contraction operands small.
template <class R, int DIM, int ORDER, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__(256, (Cfg<R, DIM, ORDER, NS, MIX>::MINB_SURF))
    k_surface(DGArgs<R> a, GasParams g) {
  using C = Cfg<R, DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = C::NP, NF = C::NF, NFP = C::NFP, NFN = C::NFN, NC = C::NC, FW = C::FW;
  constexpr int EPB = C::EPB_SURF, MP = C::MP, MT = C::MT, KB = C::KB, KR = C::KR;
  constexpr int KRR = C::KRR, NCOL = C::NCOL_S;
  constexpr int CG = 4;                     // fields per work item
  constexpr int NG = (NC + CG - 1) / CG;    // field groups
  constexpr int GV = CG * DIM;              // record values per group
  constexpr int LIM = NC * DIM;             // end of the flux part of a record
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* am = reinterpret_cast<R*>(smem_raw);                  // [NAC][MP][KB]
  R* bm = am + C::NAC * MP * KB;                           // [NCOL][KB]
  R* rx_s = bm + NCOL * KB;                                // [EPB][DIM][DIM]
  R* nrm_s = rx_s + EPB * DIM * DIM;
  R* fs_s = nrm_s + EPB * NF * DIM;
  int* fn_s = reinterpret_cast<int*>(fs_s + EPB * NF);
  int32_t* conn_s = fn_s + NFN;
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(conn_s + EPB * NF);

  const int E = a.nelem;
  const int64_t EN = (int64_t)E * NP;
  const bool sources = MIX && a.add_sources;

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
    put_a<R>(am, MP * KB, i, v);
  }
  // padding rows/columns of B stay zero for the whole kernel
  for (int i = threadIdx.x; i < NCOL * KB; i += blockDim.x) bm[i] = R(0);
  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const int nwarps = blockDim.x >> 5;
  constexpr int NACC = C::TF32 ? 4 : 2;
  const int ntiles = (E + EPB - 1) / EPB;
  bool bad = false;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * EPB;
    const int ne = imin(EPB, E - e0);
    // (no barrier needed before these writes: the previous tile's last
    // phase reads only am / bm, and the first barrier of load_geometry
    // orders those reads before this tile's writes of bm)
    stage_conn<NF>(a.conn, e0, ne, conn_s);
    load_geometry<R, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);
    __syncthreads();

    // volume terms
    for (int it = threadIdx.x; it < ne * NP * NG; it += blockDim.x) {
      const int grp = it % NG, node = it / NG;
      const int e = node / NP, k = node % NP;
      R fv[GV], f0v[GV];
      load_group<R, GV>(a.fbuf + ((int64_t)e0 * NP + node) * FW, grp * GV, LIM, fv);
      load_group<R, GV>(a.fbuf + ((int64_t)(e0 + e) * NP) * FW, grp * GV, LIM, f0v);
      const R* rxe = rx_s + e * DIM * DIM;
#pragma unroll
      for (int cc = 0; cc < CG; ++cc) {
        const int c = grp * CG + cc;
        if (c >= NC) break;
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          R acc = R(0);
#pragma unroll
          for (int j = 0; j < DIM; ++j)
            acc += rxe[r * DIM + j] * (fv[cc * DIM + j] - f0v[cc * DIM + j]);
          bm[(c * EPB + e) * KB + r * NP + k] = acc;
        }
      }
    }

    // face terms, one face node per item: the pairing and the wave speed
    // once, then the field groups
    for (int fnode = threadIdx.x; fnode < ne * NFN; fnode += blockDim.x) {
      const int e = fnode / NFN, fm = fnode % NFN, f = fm / NFP, m = fm % NFP;
      const int k = fn_s[fm];
      const int cn = conn_s[e * NF + f];
      const R fsc = fs_s[e * NF + f];
      R n[DIM];
#pragma unroll
      for (int j = 0; j < DIM; ++j) n[j] = nrm_s[(e * NF + f) * DIM + j];
      const int64_t gm = (int64_t)(e0 + e) * NP + k, g0 = (int64_t)(e0 + e) * NP;
      R* bcol = bm + e * KB + DIM * NP + fm;
      int64_t gi = -1;
      if (cn >= 0 && a.flux_kind != FLUX_HLL) {
        const int en = cn >> 8, pr = cn & 255;
        const int kn = (pr < a.nperm) ? perm_s[pr * NFP + m] : NP;
        if (en < E && kn < NP) gi = (int64_t)en * NP + kn;
      }
      if (gi >= 0) {
        // Rusanov: lambda = max(|v| + c) of the two sides, from the records
        const R lm = a.fbuf[gm * FW + LIM + 3], lp = a.fbuf[gi * FW + LIM + 3];
        const R lam = (a.flux_kind == FLUX_RUSANOV) ? fmax(lm, lp) : R(0);
#pragma unroll 1
        for (int grp = 0; grp < NG; ++grp) {
          R fmv[GV], fpv[GV], f0v[GV];
          load_group<R, GV>(a.fbuf + gm * FW, grp * GV, LIM, fmv);
          load_group<R, GV>(a.fbuf + gi * FW, grp * GV, LIM, fpv);
          load_group<R, GV>(a.fbuf + g0 * FW, grp * GV, LIM, f0v);
#pragma unroll
          for (int cc = 0; cc < CG; ++cc) {
            const int c = grp * CG + cc;
            if (c >= NC) break;
            R sm_ = R(0), sp_ = R(0), s0 = R(0);
#pragma unroll
            for (int j = 0; j < DIM; ++j) {
              sm_ += fmv[cc * DIM + j] * n[j];
              sp_ += fpv[cc * DIM + j] * n[j];
              s0 += f0v[cc * DIM + j] * n[j];
            }
            const R dq = a.q[c * EN + gm] - a.q[c * EN + gi];
            const R out = (sm_ + sp_) * R(0.5) - lam * dq * R(0.5);
            bcol[c * EPB * KB] = fsc * (out - s0);
          }
        }
      } else {
        surface_face_general<R, DIM, NP, NFP, NS, MIX, VISC>(
            a, g, EN, gm, g0, m, cn, n[0], n[1], DIM > 2 ? n[DIM - 1] : R(0), fsc, perm_s,
            bcol, EPB * KB);
      }
    }
    __syncthreads();

    // rhs = [-W | LIFT] [G ; S] on the tensor cores (+ sources).  float32:
    // one warp item per group of NTG n-tiles and every m-tile, each B value
    // split into its tf32 hi/lo words once; float64: one m-tile and NTG
    // n-tiles per item, so each A fragment load serves NTG products
    constexpr int NNT = NCOL / 8;
    constexpr int NTG = (NNT % 3 == 0) ? 3 : ((NNT % 2 == 0) ? 2 : 1);
    if constexpr (C::TF32) {
      for (int ng = warp; ng < NNT / NTG; ng += nwarps) {
        float d[MT][NTG][NACC];
#pragma unroll
        for (int t = 0; t < MT; ++t)
#pragma unroll
          for (int u = 0; u < NTG; ++u)
#pragma unroll
            for (int v = 0; v < NACC; ++v) d[t][u][v] = 0.f;
        const R* bcol = bm + (ng * NTG * 8 + gq) * KB + tq;
#pragma unroll 2
        for (int ks = 0; ks < KRR / 8; ++ks) {
          SplitB bs[NTG];
#pragma unroll
          for (int u = 0; u < NTG; ++u)
            bs[u] = SplitB(bcol[u * 8 * KB + ks * 8], bcol[u * 8 * KB + ks * 8 + 4]);
#pragma unroll
          for (int t = 0; t < MT; ++t) {
            uint32_t ah[4], alo[4];
            load_a_tf32_ldsm(ah, am, KB, t * 16, ks * 8, lane);
            load_a_tf32_ldsm(alo, am + MP * KB, KB, t * 16, ks * 8, lane);
#pragma unroll
            for (int u = 0; u < NTG; ++u) mma_tf32x3(d[t][u], ah, alo, bs[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < NTG; ++u)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int col = (ng * NTG + u) * 8 + 2 * tq + h;
            const int c = col / EPB, e = col % EPB;
            if (c >= NC || e >= ne) continue;
            R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
            for (int t = 0; t < MT; ++t)
#pragma unroll
              for (int half = 0; half < NACC / 2; ++half) {
                const int i = t * Tile<R>::MROW + gq + 8 * half;
                if (i >= NP) continue;
                R v = d[t][u][2 * half + h];
                if (sources && c >= 2 + DIM)
                  v += a.srcbuf[(int64_t)(c - 2 - DIM) * EN + (int64_t)(e0 + e) * NP + i];
                outp[i] = v;
                bad |= !(v == v);
              }
          }
      }
    } else
    for (int w = warp; w < (NNT / NTG) * MT; w += nwarps) {
      const int ng = w / MT, t = w % MT;
      R d[NTG][NACC];
#pragma unroll
      for (int u = 0; u < NTG; ++u)
#pragma unroll
        for (int v = 0; v < NACC; ++v) d[u][v] = R(0);
      const R* bcol = bm + (ng * NTG * 8 + gq) * KB + tq;
      if constexpr (!C::TF32) {
#pragma unroll 5
        for (int ks = 0; ks < KRR / 4; ++ks) {
          const double av = am[(t * 8 + gq) * KB + ks * 4 + tq];
#pragma unroll
          for (int u = 0; u < NTG; ++u) dmma884(d[u], av, bcol[u * 8 * KB + ks * 4]);
        }
      } else {
#pragma unroll 2
        for (int ks = 0; ks < KRR / 8; ++ks) {
          uint32_t ah[4], alo[4];
          load_a_tf32_ldsm(ah, am, KB, t * 16, ks * 8, lane);
          load_a_tf32_ldsm(alo, am + MP * KB, KB, t * 16, ks * 8, lane);
#pragma unroll
          for (int u = 0; u < NTG; ++u)
            mma_tf32x3(d[u], ah, alo, bcol[u * 8 * KB + ks * 8], bcol[u * 8 * KB + ks * 8 + 4]);
        }
      }
#pragma unroll
      for (int u = 0; u < NTG; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int col = (ng * NTG + u) * 8 + 2 * tq + h;
          const int c = col / EPB, e = col % EPB;
          if (c >= NC || e >= ne) continue;
          R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
          for (int half = 0; half < NACC / 2; ++half) {
            const int i = t * Tile<R>::MROW + gq + 8 * half;
            if (i >= NP) continue;
            R v = d[u][2 * half + h];
            if (sources && c >= 2 + DIM)
              v += a.srcbuf[(int64_t)(c - 2 - DIM) * EN + (int64_t)(e0 + e) * NP + i];
            outp[i] = v;
            bad |= !(v == v);
          }
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

// mixed form: k arrives in float32, the state and the sum stay float64, and
// the float32 copy of the new state feeds the next right-hand side
__global__ void k_rk4_stage_mixed(int64_t n, const double* __restrict__ q0,
                                  const float* __restrict__ k, double* __restrict__ sum,
                                  double* __restrict__ qout, float* __restrict__ qout_lo,
                                  int stage, double dt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double kv = (double)k[i];
    double qn;
    if (stage == 0) {
      sum[i] = kv;
      qn = q0[i] + dt / 2 * kv;
    } else if (stage == 1) {
      sum[i] = sum[i] + 2.0 * kv;
      qn = q0[i] + dt / 2 * kv;
    } else if (stage == 2) {
      sum[i] = sum[i] + 2.0 * kv;
      qn = q0[i] + dt * kv;
    } else {
      qn = q0[i] + dt / 6 * (sum[i] + kv);
    }
    qout[i] = qn;
    qout_lo[i] = (float)qn;
  }
}

// }}}

}  // namespace

}  // namespace mgc
