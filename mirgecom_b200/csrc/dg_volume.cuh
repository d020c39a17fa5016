// Two-kernel right-hand side for simplicial elements: a volume kernel and a
// face kernel.
//
// k_volume (one persistent CTA per SM slot, a loop over element tiles):
//   gradients  grad_cv_operator + grad_t_operator (navierstokes.py:129-347)
//              exactly as k_grad computes them, but kept in shared memory
//              (node-major); written to HBM only when the caller asks for
//              them (return_gradients, navierstokes.py:573-574)
//   pointwise  per node: state, total flux F = F_V - F_I (viscous.py:232-293,
//              inviscid.py:65-102), Arrhenius sources (eos.py:858-875); the
//              metric-combined volume flux G_r = sum_j (dr_r/dx_j) F_j into
//              shared memory; for each face the node lies on, a face-node
//              record {F.n, |v| + c, p, c, gamma} into HBM; the node-0 flux
//              F0.n per face (the element-constant shift) into HBM; at
//              prescribed boundary faces the exterior state's record
//   volume     rhs = -sum_r W_r (G_r - G0_r) + sources on the tensor cores,
//              written to HBM
// k_face (persistent as well):
//   faces      per face node: the two records of the face (own, and the
//              neighbour's through the face pairing), q on both sides, and
//              the numerical flux F*_V - F*_I (Rusanov / central from the
//              records alone, HLL through the general path) minus F0.n,
//              scaled by the face factor
//   lift       rhs += LIFT S on the tensor cores
//
// Against the three-pass split (gradients, per-node flux records, surface)
// this never writes the gradients to HBM, writes compact face-node records
// instead of full per-node flux records, and leaves the face kernel a small
// contraction (K = Nf * Nfp).  Subtracting the element-constant flux F0 from
// the volume terms (volume kernel) and from the face terms (face kernel)
// leaves the discrete divergence unchanged: -W c + LIFT (c.n) = 0 for a
// constant c.
#pragma once
#include "boundary.cuh"
#include "dg_kernels.cuh"

namespace mgc {

// Face-node record: F.n (NC values, n the element's own outward unit normal),
// then |v| + c, p, c, gamma, padded to 16 bytes.
__host__ __device__ constexpr int trace_width(int nc) { return round_up(nc + 4, 4); }

template <class R, int DIM, int ORDER, int NS, bool MIX>
struct VCfg {
  using G = Cfg<R, DIM, ORDER, NS, MIX>;
  static constexpr int RB = (int)sizeof(R);
  static constexpr bool TF32 = G::TF32;
  static constexpr int NP = G::NP, NF = G::NF, NFP = G::NFP, NFN = G::NFN;
  static constexpr int NC = G::NC, NU = G::NU;
  static constexpr int MP = G::MP, MT = G::MT, NAC = G::NAC, MROW = Tile<R>::MROW;
  static constexpr int KSTEP = Tile<R>::KSTEP;
  static constexpr int KU = G::KU, KS = G::KS, KL = G::KL, NFPK = G::NFPK, KUR = G::KUR;
  static constexpr int GEO = G::GEO;
  static constexpr int TW = trace_width(NC);
  // node-major staging rows (odd strides: a warp reading one row per lane,
  // or the tensor-core fragment pattern, hits distinct banks)
  static constexpr int GST = (NU * DIM) | 1;     // gradients of one node
  static constexpr int FST = (NC * DIM) | 1;     // metric-combined fluxes of one node

  // ---- volume kernel: threads, elements per tile, shared memory
  static constexpr int NT = TF32 ? 256 : 128;
  static constexpr int MINB = 2;
  static constexpr int BUDGET = 111 * 1024;
  static constexpr int A_VOL = NAC * (DIM * MP * KU + NF * MP * KL);
  static constexpr __host__ __device__ int nnode(int epb) { return epb * NP + (KUR - NP) + 4; }
  static constexpr __host__ __device__ int ncol_g(int epb) { return round_up(NU * epb, 8); }
  static constexpr __host__ __device__ int w1(int epb) {
    return imax(ncol_g(epb) * (KU + KS), nnode(epb) * FST + NS * epb * NP);
  }
  static constexpr __host__ __device__ int vol_reals(int epb) {
    return A_VOL + w1(epb) + nnode(epb) * GST + epb * GEO + NU * epb;
  }
  static constexpr __host__ __device__ size_t vol_bytes(int epb, int nperm) {
    return (size_t)vol_reals(epb) * RB + NFN * 4 + epb * NF * 4 + NP * NF * 2 +
           (size_t)nperm * NFP + 64;
  }
  // largest multiple of 4 elements (8 on the float32 path) within the budget
  // with up to 32 face-pairing permutations
  static constexpr __host__ __device__ int pick_epb() {
    int best = 4;
    for (int e = 4; e <= 32; e += (TF32 ? 4 : 4))
      if (vol_bytes(e, 32) <= (size_t)BUDGET && (!TF32 || e % 8 == 0 || e == 4)) best = e;
    return best;
  }
  static constexpr int EPB = pick_epb();
  static constexpr int NNODE = nnode(EPB);
  static constexpr int NCOL = ncol_g(EPB);
  static constexpr int W1 = w1(EPB);
  static constexpr int NCOLD = round_up(NC * EPB, 8);      // divergence columns

  // ---- flux-volume kernel (gradients from HBM): no gradient operands or
  // staging; element tiles sized so the pointwise phase fills the block
  static constexpr int NT3 = TF32 ? 256 : 128;
  static constexpr int A_FLUX = NAC * DIM * MP * KU;
  static constexpr __host__ __device__ int nnode3(int epb) { return epb * NP + (KUR - NP) + 4; }
  static constexpr __host__ __device__ size_t flux_bytes(int epb, int nperm) {
    return (size_t)(A_FLUX + nnode3(epb) * FST + NS * epb * NP + epb * GEO) * RB + NFN * 4 +
           epb * NF * 4 + NP * NF * 2 + (size_t)nperm * NFP + 64;
  }
  // the largest tile with at most one node per thread and two blocks per SM
  static constexpr __host__ __device__ int pick_epb3() {
    int best = 1;
    for (int e = 1; e * NP <= NT3; ++e)
      if (flux_bytes(e, 32) <= (size_t)BUDGET) best = e;
    return best;
  }
  static constexpr int EPB3 = pick_epb3();
  static constexpr int NCOL3 = round_up(NC * EPB3, 8);

  // ---- face kernel
  // float32: 8-element tiles in six resident blocks per SM (the face pass is
  // bound by its gathers' latency: 8.7 ms against 9.8 ms for four blocks of
  // 16 elements at 80^3)
  static constexpr int NT2 = 128;
  static constexpr int MINB2 = TF32 ? 6 : 3;
  static constexpr int KFR = round_up(NFN, KSTEP);
  static constexpr int KF = Tile<R>::stride(KFR);
  static constexpr int A_FACE = NAC * MP * KF;
  static constexpr int EPB2 = 8;
  static constexpr int NCOL2 = round_up(NC * EPB2, 8);
  static size_t face_bytes(int nperm) {
    return (size_t)(A_FACE + NCOL2 * KF + EPB2 * GEO) * RB + NFN * 4 + EPB2 * NF * 4 +
           2 * (size_t)nperm * NFP + 64;
  }
};

namespace {

// The exterior state's record at face node m of prescribed boundary face bf
// (boundary.py:141-146 for the viscous part: the exterior state with the
// interior gradients *gq* [NU][DIM] of the face node), in the neighbour's
// convention: -F_ext.n with n the interior's outward normal.  Out of line,
// arguments by value, so that its state does not enter the register
// allocation of the pointwise phase.
template <class R, int DIM, int NS, bool MIX, bool VISC>
__device__ __noinline__ void boundary_record(const DGArgs<R> a, const GasParams g, int bf, int m,
                                             int nfp, const R* gq, int64_t gs, R n0, R n1, R n2,
                                             R* dst) {
  constexpr int NC = DIM + 2 + NS, TW = trace_width(NC);
  const R n[3] = {n0, n1, n2};
  const int64_t bstride = (int64_t)a.nbf * nfp, bo = (int64_t)bf * nfp + m;
  R qp[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) qp[c] = a.bext[c * bstride + bo];
  NodeState<R, DIM, NS> sp;
  make_state<R, DIM, NS>(qp, MIX ? a.bext[NC * bstride + bo] : R(0), g, sp);
  R fe[NC][DIM];
  inviscid_flux<R, DIM, NS>(sp, fe);
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int j = 0; j < DIM; ++j) fe[c][j] = -fe[c][j];
  if (VISC) {
    R gqv[NC][DIM], gt[DIM];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int j = 0; j < DIM; ++j) gqv[c][j] = gq[(c * DIM + j) * gs];
#pragma unroll
    for (int j = 0; j < DIM; ++j) gt[j] = gq[(NC * DIM + j) * gs];
    R fv[NC][DIM];
    viscous_flux<R, DIM, NS, MIX>(sp, gqv, gt, fv);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int j = 0; j < DIM; ++j) fe[c][j] += fv[c][j];
  }
  R rec[TW];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    R acc = R(0);
#pragma unroll
    for (int j = 0; j < DIM; ++j) acc += fe[c][j] * n[j];
    rec[c] = -acc;
  }
  rec[NC] = wavespeed<R, DIM, NS>(sp);
  rec[NC + 1] = sp.p;
  rec[NC + 2] = sp.c;
  rec[NC + 3] = sp.gamma;
#pragma unroll
  for (int i = NC + 4; i < TW; ++i) rec[i] = R(0);
#pragma unroll
  for (int i = 0; i < TW; ++i) dst[i] = rec[i];
#pragma unroll
  for (int c = 0; c < NC; ++c) a.bplus[c * bstride + bo] = qp[c];
}

// The exterior record of a Mengaldo boundary face node (neighbour
// convention) and its state_plus q into bplus.  The face kernel combines it
// with the interior record as for an interior face: central(F_V) from the
// pair gives F_V(state_bc, grad_cv_bc, grad_t_bc) . n when the exterior
// viscous part is 2 F_V,bc - F_V-; the inviscid part is the numerical flux
// between the interior state and state_plus (boundary.py:583-730).
template <class R, int DIM, int NS, bool MIX, bool VISC>
__device__ __noinline__ void mengaldo_record(const DGArgs<R> a, const GasParams g, int kind,
                                             int bf, int m, int nfp, int64_t EN, int64_t gm,
                                             const R* gq, int64_t gs, R n0, R n1, R n2, R* dst) {
  constexpr int NC = DIM + 2 + NS, TW = trace_width(NC);
  const R n[3] = {n0, n1, n2};
  R qm[NC];
  NodeState<R, DIM, NS> sm;
  boundary_minus<R, DIM, NS, MIX>(a, g, EN, gm, qm, sm);
  R par[NC + 1];
  const int64_t bstride = (int64_t)a.nbf * nfp, bo = (int64_t)bf * nfp + m;
#pragma unroll
  for (int c = 0; c <= NC; ++c) par[c] = bk_needs_bext(kind) ? a.bext[c * bstride + bo] : R(0);
  R qp[NC];
  bc_plus_cv<R, DIM, NS>(kind, g, qm, sm.t, sm.p, sm.c, sm.gamma, n, par, qp);
  // mixtures: the plus state's temperature re-solved from T- (the far field
  // state comes with its own)
  R tp = R(0);
  if (MIX) tp = (kind == BK_FARFIELD) ? par[NC] : node_temperature<R, DIM, NS>(qp, sm.t, g);
  NodeState<R, DIM, NS> sp;
  make_state<R, DIM, NS>(qp, tp, g, sp);
  R fip[NC];
  inviscid_flux_n<R, DIM, NS>(sp, n, fip);
  R rec[TW];
#pragma unroll
  for (int c = 0; c < NC; ++c) rec[c] = fip[c];
  if (VISC) {
    R qbc[NC];
    bc_state_cv<R, DIM, NS>(kind, g, qm, sm.t, sm.p, sm.c, sm.gamma, n, par, qbc);
    R tb = R(0);
    if (MIX) tb = (kind == BK_FARFIELD) ? par[NC] : node_temperature<R, DIM, NS>(qbc, sm.t, g);
    NodeState<R, DIM, NS> sb;
    make_state<R, DIM, NS>(qbc, tb, g, sb);
    R gqv[NC][DIM], gt[DIM];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int j = 0; j < DIM; ++j) gqv[c][j] = gq[(c * DIM + j) * gs];
#pragma unroll
    for (int j = 0; j < DIM; ++j) gt[j] = gq[(NC * DIM + j) * gs];
    R fvm[NC][DIM];
    viscous_flux<R, DIM, NS, MIX>(sm, gqv, gt, fvm);
    bc_gradients<R, DIM, NS>(kind, qm, qbc, n, gqv, gt);
    R fvb[NC][DIM];
    viscous_flux<R, DIM, NS, MIX>(sb, gqv, gt, fvb);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      R vb = R(0), vm = R(0);
#pragma unroll
      for (int j = 0; j < DIM; ++j) {
        vb += fvb[c][j] * n[j];
        vm += fvm[c][j] * n[j];
      }
      // -(F_V+ - F_I+) . n with F_V+ . n = 2 F_V,bc . n - F_V- . n
      rec[c] = -((R(2) * vb - vm) - fip[c]);
    }
  }
  rec[NC] = wavespeed<R, DIM, NS>(sp);
  rec[NC + 1] = sp.p;
  rec[NC + 2] = sp.c;
  rec[NC + 3] = sp.gamma;
#pragma unroll
  for (int i = NC + 4; i < TW; ++i) rec[i] = R(0);
#pragma unroll
  for (int i = 0; i < TW; ++i) dst[i] = rec[i];
#pragma unroll
  for (int c = 0; c < NC; ++c) a.bplus[c * bstride + bo] = qp[c];
}

// Ask L2 for the 128-byte lines of [p, p + bytes), the work spread over the
// block's threads: the next tile's contiguous inputs are fetched while the
// current tile computes (prefetch.global.L2 does not block and takes no
// registers; a line already resident costs nothing).
__device__ __forceinline__ void prefetch_l2(const void* p, size_t bytes) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(p) & ~uintptr_t(127);
  const uintptr_t a1 = reinterpret_cast<uintptr_t>(p) + bytes;
  for (uintptr_t a = a0 + (uintptr_t)threadIdx.x * 128; a < a1; a += (uintptr_t)blockDim.x * 128)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
}

// 16-byte vector store / load of one record (TW values, 16-byte aligned)
template <class R, int TW>
__device__ __forceinline__ void store_rec(R* dst, const R (&rec)[TW]) {
  if constexpr (sizeof(R) == 4) {
#pragma unroll
    for (int i = 0; i < TW; i += 4)
      *reinterpret_cast<float4*>(dst + i) = make_float4(rec[i], rec[i + 1], rec[i + 2], rec[i + 3]);
  } else {
#pragma unroll
    for (int i = 0; i < TW; i += 2)
      *reinterpret_cast<double2*>(dst + i) = make_double2(rec[i], rec[i + 1]);
  }
}

// Volume kernel: gradients, pointwise fluxes, face-node records and the
// volume part of the divergence.  VISC false: the Euler operator (no
// gradient pass, F = -F_I).
template <class R, int DIM, int ORDER, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__((VCfg<R, DIM, ORDER, NS, MIX>::NT),
                                  (VCfg<R, DIM, ORDER, NS, MIX>::MINB))
    k_volume(DGArgs<R> a, GasParams g) {
  using V = VCfg<R, DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = V::NP, NF = V::NF, NFP = V::NFP, NFN = V::NFN, NC = V::NC, NU = V::NU;
  constexpr int EPB = V::EPB, MP = V::MP, MT = V::MT, NAC = V::NAC, MROW = V::MROW;
  constexpr int KU = V::KU, KS = V::KS, KL = V::KL, NFPK = V::NFPK, KUR = V::KUR;
  constexpr int NCOL = V::NCOL, NCOLD = V::NCOLD, NNODE = V::NNODE;
  constexpr int GST = V::GST, FST = V::FST, TW = V::TW;
  constexpr int AWN = DIM * MP * KU, ALN = NF * MP * KL;
  constexpr int ENP = EPB * NP;
  static_assert(NCOL * (KU + KS) <= V::W1 && NNODE * FST + NS * ENP <= V::W1, "work region");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* aw = reinterpret_cast<R*>(smem_raw);                  // [NAC][DIM][MP][KU]
  R* al = aw + NAC * AWN;                                  // [NAC][NF][MP][KL]
  R* w1 = al + NAC * ALN;                                  // work region
  R* bu = w1;                                              //   [NCOL][KU]  (gradient pass)
  R* bs = bu + NCOL * KU;                                  //   [NCOL][KS]  (gradient pass)
  R* gfl = w1;                                             //   [NNODE][FST] (after it)
  R* src_s = w1 + NNODE * FST;                             //   [NS][ENP]
  R* gn = w1 + V::W1;                                      // [NNODE][GST] gradients
  R* rx_s = gn + NNODE * GST;                              // [EPB][DIM][DIM]
  R* nrm_s = rx_s + EPB * DIM * DIM;                       // [EPB][NF][DIM]
  R* fs_s = nrm_s + EPB * NF * DIM;                        // [EPB][NF]
  R* u0_s = fs_s + EPB * NF;                               // [NU][EPB]
  int* fn_s = reinterpret_cast<int*>(u0_s + NU * EPB);     // [NFN]
  int32_t* conn_s = fn_s + NFN;                            // [EPB][NF]
  int16_t* slot_s = reinterpret_cast<int16_t*>(conn_s + EPB * NF);   // [NP][NF]
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(slot_s + NP * NF);

  const int E = a.nelem;
  const int64_t EN = (int64_t)E * NP;
  const bool sources = MIX && a.add_sources;
  const bool rows16 =
      ((reinterpret_cast<uintptr_t>(a.q) | reinterpret_cast<uintptr_t>(a.t_op)) & 15) == 0 &&
      (KU * sizeof(R)) % 16 == 0;

  // operators W_r (gradient and divergence) and LIFT_f (gradient), zero padded
  for (int i = threadIdx.x; i < AWN; i += blockDim.x) {
    const int r = i / (MP * KU), row = (i / KU) % MP, k = i % KU;
    put_a<R>(aw, AWN, i, (row < NP && k < NP) ? c_ref64[S::OFF_W + (r * NP + row) * NP + k] : 0.0);
  }
  if (VISC)
    for (int i = threadIdx.x; i < ALN; i += blockDim.x) {
      const int f = i / (MP * KL), row = (i / KL) % MP, m = i % KL;
      put_a<R>(al, ALN, i,
               (row < NP && m < NFP) ? c_ref64[S::OFF_LIFT + row * NFN + f * NFP + m] : 0.0);
    }
  for (int i = threadIdx.x; i < V::W1 + NNODE * GST; i += blockDim.x) w1[i] = R(0);
  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];
  if (threadIdx.x == 0) {
    // face slots f * NFP + m of each volume node (-1: none)
    for (int i = 0; i < NP * NF; ++i) slot_s[i] = -1;
    for (int fm = 0; fm < NFN; ++fm) {
      const int k = c_face_nodes<DIM, ORDER>(fm);
      for (int s = 0; s < NF; ++s)
        if (slot_s[k * NF + s] < 0) {
          slot_s[k * NF + s] = (int16_t)fm;
          break;
        }
    }
  }

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const int nwarps = blockDim.x >> 5;
  constexpr int NACC = V::TF32 ? 4 : 2;
  const int ntiles = (a.nowned + EPB - 1) / EPB;
  bool bad = false;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * EPB;
    const int ne = imin(EPB, a.nowned - e0);
    // the previous tile's last phase reads the work region, src_s and the
    // geometry, which this tile overwrites
    __syncthreads();
    stage_conn<NF>(a.conn, e0, ne, conn_s);
    load_geometry<R, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);
    // the normals and face factors load_geometry computes last are read by
    // other threads in every phase below (the Euler operator goes straight
    // to the pointwise phase)
    __syncthreads();

    if constexpr (VISC) {
      // ---- gradient pass (as k_grad), results into gn
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
          const int64_t gnd = (int64_t)e0 * NP + idx, g0 = (int64_t)(e0 + e) * NP;
          R qq[NC], q0[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            qq[c] = a.q[c * EN + gnd];
            q0[c] = a.q[c * EN + g0];
          }
          const R t = MIX ? a.t_op[gnd] : node_temperature<R, DIM, NS>(qq, R(0), g);
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

      // face values fscale * (u* - u0), one face node per item
      for (int fnode = threadIdx.x; fnode < ne * NFN; fnode += blockDim.x) {
        const int e = fnode / NFN, fm = fnode % NFN, f = fm / NFP, m = fm % NFP;
        const int k = fn_s[fm];
        const int cn = conn_s[e * NF + f];
        const R fsc = fs_s[e * NF + f];
        int mode = 2;      // 0 two-sided average, 1 prescribed exterior, 2 interior value
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
          const R um = bu[(c * EPB + e) * KU + k];
          const R u0 = u0_s[c * EPB + e];
          const R v = (mode == 0) ? ((up[c] - u0) + um) * R(0.5) : up[c] - u0;
          bcol[c * EPB * KS] = fsc * v;
        }
      }
      __syncthreads();

      // the next tile's rows of q and the temperatures, its geometry and
      // face pairing, into L2 while this tile computes
      {
        const int tn = tile + gridDim.x;
        if (tn < ntiles) {
          const int e1 = tn * EPB, n1 = imin(EPB, a.nowned - e1);
          const size_t row = (size_t)n1 * NP * sizeof(R);
          for (int c = 0; c < NC; ++c) prefetch_l2(a.q + c * EN + (int64_t)e1 * NP, row);
          if (MIX) prefetch_l2(a.t_op + (int64_t)e1 * NP, row);
          if (MIX && a.add_sources) prefetch_l2(a.t_src + (int64_t)e1 * NP, row);
          prefetch_l2(a.rx + (int64_t)e1 * DIM * DIM, (size_t)n1 * DIM * DIM * sizeof(R));
          prefetch_l2(a.conn + (int64_t)e1 * NF, (size_t)n1 * NF * 4);
        }
      }

      // contraction and metric combination into gn[node][c * DIM + j]
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
        if constexpr (!V::TF32) {
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
#pragma unroll
          for (int half = 0; half < NACC / 2; ++half) {
            const int i = t * MROW + gq + 8 * half;
            if (i >= NP) continue;
            const int v = 2 * half + h;
#pragma unroll
            for (int j = 0; j < DIM; ++j) {
              R gsum = R(0);
#pragma unroll
              for (int f = 0; f < NF; ++f) gsum += nre[f][j] * lf[f][v];
#pragma unroll
              for (int r = 0; r < DIM; ++r) gsum -= rxe[r][j] * du[r][v];
              gn[(e * NP + i) * GST + c * DIM + j] = gsum;
              if (a.grad_out)
                a.grad_out[((int64_t)c * DIM + j) * EN + (int64_t)(e0 + e) * NP + i] = gsum;
            }
          }
        }
      }
      // every contraction has read bu/bs (the region gfl and src_s reuse)
      // and every gradient is in gn
      __syncthreads();
    }

    // ---- pointwise: fluxes, records, sources; G_r into gfl[node][c * DIM + r]
    for (int n = threadIdx.x; n < ne * NP; n += blockDim.x) {
      const int e = n / NP, k = n % NP;
      const int64_t gnd = (int64_t)(e0 + e) * NP + k;
      R qq[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) qq[c] = a.q[c * EN + gnd];
      NodeState<R, DIM, NS> st;
      make_state<R, DIM, NS>(qq, MIX ? a.t_op[gnd] : R(0), g, st);
      R fl[NC][DIM];
      inviscid_flux<R, DIM, NS>(st, fl);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) fl[c][j] = -fl[c][j];
      if constexpr (VISC) {
        // the gradients are read from the node's shared-memory row where the
        // viscous flux uses them (no register copy of all (NC+1) DIM values)
        const R* gr = gn + n * GST;
        R fv[NC][DIM];
        viscous_flux<R, DIM, NS, MIX>(st, reinterpret_cast<const R(*)[DIM]>(gr), gr + NC * DIM,
                                      fv);
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int j = 0; j < DIM; ++j) fl[c][j] = fv[c][j] + fl[c][j];
      }
      bad |= !(st.p == st.p) || !(st.c == st.c);
      const R* rxe = rx_s + e * DIM * DIM;
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          R acc = R(0);
#pragma unroll
          for (int j = 0; j < DIM; ++j) acc += rxe[r * DIM + j] * fl[c][j];
          gfl[n * FST + c * DIM + r] = acc;
        }
      if constexpr (MIX && NS > 0) {
        if (sources) {
          R om[NS];
          production_rates<R, NS>(st.rho, a.t_src[gnd], st.y, (R)g.zero_level, om);
#pragma unroll
          for (int s = 0; s < NS; ++s) src_s[s * ENP + n] = mech<R>().mw[s] * om[s];
        }
      }
      R v2 = R(0);
#pragma unroll
      for (int j = 0; j < DIM; ++j) v2 += st.v[j] * st.v[j];
      const R lam = sqrt(v2) + st.c;
      // one record per face slot of this node
#pragma unroll 1
      for (int sl = 0; sl < NF; ++sl) {
        const int fm = slot_s[k * NF + sl];
        if (fm < 0) break;
        const int f = fm / NFP, m = fm % NFP;
        const R* nf = nrm_s + (e * NF + f) * DIM;
        R rec[TW];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          R acc = R(0);
#pragma unroll
          for (int j = 0; j < DIM; ++j) acc += fl[c][j] * nf[j];
          rec[c] = acc;
        }
        rec[NC] = lam;
        rec[NC + 1] = st.p;
        rec[NC + 2] = st.c;
        rec[NC + 3] = st.gamma;
#pragma unroll
        for (int i = NC + 4; i < TW; ++i) rec[i] = R(0);
        store_rec<R, TW>(a.trace + (((int64_t)(e0 + e) * NF + f) * NFP + m) * TW, rec);
      }
      if (k == 0) {
        // element-constant shift of the face terms: F0 . n_f, every face
        R* s0e = a.s0 + (int64_t)(e0 + e) * NF * NC;
#pragma unroll 1
        for (int f = 0; f < NF; ++f) {
          const R* nf = nrm_s + (e * NF + f) * DIM;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            R acc = R(0);
#pragma unroll
            for (int j = 0; j < DIM; ++j) acc += fl[c][j] * nf[j];
            s0e[f * NC + c] = acc;
          }
        }
      }
    }
    // exterior records of the tile's boundary face nodes, in a loop of their
    // own: out of line calls inside the pointwise loop would make the
    // compiler spill that loop's registers around them for every node
    for (int fnode = threadIdx.x; fnode < ne * NFN; fnode += blockDim.x) {
      const int e = fnode / NFN, fm = fnode % NFN, f = fm / NFP, m = fm % NFP;
      const int cn = conn_s[e * NF + f];
      if (cn >= 0) continue;
      const int bf = -(cn + 1);
      const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
      if ((bk_needs_bext(kind) && !a.bext) || (kind != BK_PRESCRIBED && !bk_mengaldo(kind)))
        continue;
      const int k = fn_s[fm];
      const int n = e * NP + k;
      const R* nf = nrm_s + (e * NF + f) * DIM;
      R* dst = a.btrace + ((int64_t)bf * NFP + m) * TW;
      if (kind == BK_PRESCRIBED)
        boundary_record<R, DIM, NS, MIX, VISC>(a, g, bf, m, NFP, VISC ? gn + n * GST : nullptr,
                                               1, nf[0], nf[1], DIM > 2 ? nf[DIM - 1] : R(0),
                                               dst);
      else
        mengaldo_record<R, DIM, NS, MIX, VISC>(a, g, kind, bf, m, NFP, EN,
                                               (int64_t)(e0 + e) * NP + k,
                                               VISC ? gn + n * GST : nullptr, 1, nf[0], nf[1],
                                               DIM > 2 ? nf[DIM - 1] : R(0), dst);
    }
    __syncthreads();

    // ---- volume divergence: rhs = -sum_r W_r (G_r - G0_r) (+ sources); one
    // m-tile and NTG n-tiles per warp item.  Column col = c * EPB + e reads
    // node rows of element e; rows k >= NP of the operator are zero, so the
    // padded k reach into the next rows harmlessly (finite, zero-filled).
    constexpr int NNT = NCOLD / 8;
    constexpr int NTG = (NNT % 3 == 0) ? 3 : ((NNT % 2 == 0) ? 2 : 1);
    for (int w = warp; w < (NNT / NTG) * MT; w += nwarps) {
      const int ngp = w / MT, t = w % MT;
      R d[NTG][NACC];
#pragma unroll
      for (int u = 0; u < NTG; ++u)
#pragma unroll
        for (int v = 0; v < NACC; ++v) d[u][v] = R(0);
      // this lane's B column per n-tile: element row base and field offset
      int cbase[NTG];
#pragma unroll
      for (int u = 0; u < NTG; ++u) {
        const int col = (ngp * NTG + u) * 8 + gq;
        const int c = col / EPB, e = col % EPB;
        cbase[u] = (c < NC) ? (e * NP) * FST + c * DIM : -1;
      }
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        R g0[NTG];
#pragma unroll
        for (int u = 0; u < NTG; ++u) g0[u] = cbase[u] >= 0 ? gfl[cbase[u] + r] : R(0);
        if constexpr (!V::TF32) {
#pragma unroll
          for (int ks = 0; ks < KUR / 4; ++ks) {
            const double av = aw[(r * MP + t * 8 + gq) * KU + ks * 4 + tq];
            const int kk = ks * 4 + tq;
#pragma unroll
            for (int u = 0; u < NTG; ++u) {
              const double b = cbase[u] >= 0 ? gfl[cbase[u] + kk * FST + r] - g0[u] : 0.0;
              dmma884(d[u], av, b);
            }
          }
        } else {
#pragma unroll
          for (int ks = 0; ks < KUR / 8; ++ks) {
            uint32_t ah[4], alo[4];
            load_a_tf32_ldsm(ah, aw + r * MP * KU, KU, t * 16, ks * 8, lane);
            load_a_tf32_ldsm(alo, aw + AWN + r * MP * KU, KU, t * 16, ks * 8, lane);
            const int k0 = ks * 8 + tq;
#pragma unroll
            for (int u = 0; u < NTG; ++u) {
              float b0 = 0.f, b1 = 0.f;
              if (cbase[u] >= 0) {
                b0 = gfl[cbase[u] + k0 * FST + r] - g0[u];
                b1 = gfl[cbase[u] + (k0 + 4) * FST + r] - g0[u];
              }
              mma_tf32x3(d[u], ah, alo, b0, b1);
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < NTG; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int col = (ngp * NTG + u) * 8 + 2 * tq + h;
          const int c = col / EPB, e = col % EPB;
          if (c >= NC || e >= ne) continue;
          R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
          for (int half = 0; half < NACC / 2; ++half) {
            const int i = t * MROW + gq + 8 * half;
            if (i >= NP) continue;
            R v = -d[u][2 * half + h];
            if (sources && c >= 2 + DIM) v += src_s[(c - 2 - DIM) * ENP + e * NP + i];
            outp[i] = v;
          }
        }
    }
  }
  if (bad) atomicOr(a.status, ST_NAN);
}

// Flux-volume kernel: the pointwise phase and the volume divergence of
// k_volume with the gradients read from HBM (written by k_grad), for the
// three-kernel pass gradient -> flux-volume -> face.  Without the gradient
// operands and staging its tiles fill the block: 12 order-3 tetrahedra (240
// nodes) per 256 threads on the float32 path.
template <class R, int DIM, int ORDER, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__((VCfg<R, DIM, ORDER, NS, MIX>::NT3), 2)
    k_flux_volume(DGArgs<R> a, GasParams g) {
  using V = VCfg<R, DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = V::NP, NF = V::NF, NFP = V::NFP, NFN = V::NFN, NC = V::NC;
  constexpr int EPB = V::EPB3, MP = V::MP, MT = V::MT, MROW = V::MROW;
  constexpr int KU = V::KU, KUR = V::KUR, NCOLD = V::NCOL3, NNODE = V::nnode3(V::EPB3);
  constexpr int FST = V::FST, TW = V::TW;
  constexpr int AWN = DIM * MP * KU;
  constexpr int ENP = EPB * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* aw = reinterpret_cast<R*>(smem_raw);                  // [NAC][DIM][MP][KU]
  R* gfl = aw + V::A_FLUX;                                 // [NNODE][FST]
  R* src_s = gfl + NNODE * FST;                            // [NS][ENP]
  R* rx_s = src_s + NS * ENP;                              // [EPB][DIM][DIM]
  R* nrm_s = rx_s + EPB * DIM * DIM;                       // [EPB][NF][DIM]
  R* fs_s = nrm_s + EPB * NF * DIM;                        // [EPB][NF]
  int* fn_s = reinterpret_cast<int*>(fs_s + EPB * NF);     // [NFN]
  int32_t* conn_s = fn_s + NFN;                            // [EPB][NF]
  int16_t* slot_s = reinterpret_cast<int16_t*>(conn_s + EPB * NF);   // [NP][NF]

  const int E = a.nelem;
  const int64_t EN = (int64_t)E * NP;
  const bool sources = MIX && a.add_sources;
  for (int i = threadIdx.x; i < AWN; i += blockDim.x) {
    const int r = i / (MP * KU), row = (i / KU) % MP, k = i % KU;
    put_a<R>(aw, AWN, i, (row < NP && k < NP) ? c_ref64[S::OFF_W + (r * NP + row) * NP + k] : 0.0);
  }
  for (int i = threadIdx.x; i < NNODE * FST + NS * ENP; i += blockDim.x) gfl[i] = R(0);
  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  if (threadIdx.x == 0) {
    for (int i = 0; i < NP * NF; ++i) slot_s[i] = -1;
    for (int fm = 0; fm < NFN; ++fm) {
      const int k = c_face_nodes<DIM, ORDER>(fm);
      for (int sl = 0; sl < NF; ++sl)
        if (slot_s[k * NF + sl] < 0) {
          slot_s[k * NF + sl] = (int16_t)fm;
          break;
        }
    }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const int nwarps = blockDim.x >> 5;
  constexpr int NACC = V::TF32 ? 4 : 2;
  const int ntiles = (a.nowned + EPB - 1) / EPB;
  bool bad = false;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * EPB;
    const int ne = imin(EPB, a.nowned - e0);
    __syncthreads();
    stage_conn<NF>(a.conn, e0, ne, conn_s);
    load_geometry<R, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);
    __syncthreads();

    for (int n = threadIdx.x; n < ne * NP; n += blockDim.x) {
      const int e = n / NP, k = n % NP;
      const int64_t gnd = (int64_t)(e0 + e) * NP + k;
      R qq[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) qq[c] = a.q[c * EN + gnd];
      NodeState<R, DIM, NS> st;
      make_state<R, DIM, NS>(qq, MIX ? a.t_op[gnd] : R(0), g, st);
      R fl[NC][DIM];
      inviscid_flux<R, DIM, NS>(st, fl);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < DIM; ++j) fl[c][j] = -fl[c][j];
      if constexpr (VISC) {
        R gqv[NC][DIM], gt[DIM];
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int j = 0; j < DIM; ++j) gqv[c][j] = a.grad[((int64_t)c * DIM + j) * EN + gnd];
#pragma unroll
        for (int j = 0; j < DIM; ++j) gt[j] = a.grad[((int64_t)NC * DIM + j) * EN + gnd];
        R fv[NC][DIM];
        viscous_flux<R, DIM, NS, MIX>(st, gqv, gt, fv);
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int j = 0; j < DIM; ++j) fl[c][j] = fv[c][j] + fl[c][j];
      }
      bad |= !(st.p == st.p) || !(st.c == st.c);
      const R* rxe = rx_s + e * DIM * DIM;
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          R acc = R(0);
#pragma unroll
          for (int j = 0; j < DIM; ++j) acc += rxe[r * DIM + j] * fl[c][j];
          gfl[n * FST + c * DIM + r] = acc;
        }
      if constexpr (MIX && NS > 0) {
        if (sources) {
          R om[NS];
          production_rates<R, NS>(st.rho, a.t_src[gnd], st.y, (R)g.zero_level, om);
#pragma unroll
          for (int sp = 0; sp < NS; ++sp) src_s[sp * ENP + n] = mech<R>().mw[sp] * om[sp];
        }
      }
      R v2 = R(0);
#pragma unroll
      for (int j = 0; j < DIM; ++j) v2 += st.v[j] * st.v[j];
      const R lam = sqrt(v2) + st.c;
#pragma unroll 1
      for (int sl = 0; sl < NF; ++sl) {
        const int fm = slot_s[k * NF + sl];
        if (fm < 0) break;
        const int f = fm / NFP, m = fm % NFP;
        const R* nf = nrm_s + (e * NF + f) * DIM;
        R rec[TW];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          R acc = R(0);
#pragma unroll
          for (int j = 0; j < DIM; ++j) acc += fl[c][j] * nf[j];
          rec[c] = acc;
        }
        rec[NC] = lam;
        rec[NC + 1] = st.p;
        rec[NC + 2] = st.c;
        rec[NC + 3] = st.gamma;
#pragma unroll
        for (int i = NC + 4; i < TW; ++i) rec[i] = R(0);
        store_rec<R, TW>(a.trace + (((int64_t)(e0 + e) * NF + f) * NFP + m) * TW, rec);
      }
      if (k == 0) {
        R* s0e = a.s0 + (int64_t)(e0 + e) * NF * NC;
#pragma unroll 1
        for (int f = 0; f < NF; ++f) {
          const R* nf = nrm_s + (e * NF + f) * DIM;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            R acc = R(0);
#pragma unroll
            for (int j = 0; j < DIM; ++j) acc += fl[c][j] * nf[j];
            s0e[f * NC + c] = acc;
          }
        }
      }
    }
    // exterior records of the tile's boundary face nodes (own loop: see k_volume)
    for (int fnode = threadIdx.x; fnode < ne * NFN; fnode += blockDim.x) {
      const int e = fnode / NFN, fm = fnode % NFN, f = fm / NFP, m = fm % NFP;
      const int cn = conn_s[e * NF + f];
      if (cn >= 0) continue;
      const int bf = -(cn + 1);
      const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
      if ((bk_needs_bext(kind) && !a.bext) || (kind != BK_PRESCRIBED && !bk_mengaldo(kind)))
        continue;
      const int64_t gnd = (int64_t)(e0 + e) * NP + fn_s[fm];
      const R* nf = nrm_s + (e * NF + f) * DIM;
      R* dst = a.btrace + ((int64_t)bf * NFP + m) * TW;
      if (kind == BK_PRESCRIBED)
        boundary_record<R, DIM, NS, MIX, VISC>(a, g, bf, m, NFP, VISC ? a.grad + gnd : nullptr,
                                               EN, nf[0], nf[1], DIM > 2 ? nf[DIM - 1] : R(0),
                                               dst);
      else
        mengaldo_record<R, DIM, NS, MIX, VISC>(a, g, kind, bf, m, NFP, EN, gnd,
                                               VISC ? a.grad + gnd : nullptr, EN, nf[0], nf[1],
                                               DIM > 2 ? nf[DIM - 1] : R(0), dst);
    }
    __syncthreads();

    // volume divergence.  float32: one item per group of NTG column tiles
    // and every m-tile, so each shifted flux value is read and split into
    // its tf32 hi/lo words once
    constexpr int NNT = NCOLD / 8;
    constexpr int NTG = (NNT % 3 == 0) ? 3 : ((NNT % 2 == 0) ? 2 : 1);
    if constexpr (V::TF32) {
      for (int w = warp; w < NNT / NTG; w += nwarps) {
        const int ngp = w;
        float d[MT][NTG][NACC];
#pragma unroll
        for (int t = 0; t < MT; ++t)
#pragma unroll
          for (int u = 0; u < NTG; ++u)
#pragma unroll
            for (int v = 0; v < NACC; ++v) d[t][u][v] = 0.f;
        int cbase[NTG];
#pragma unroll
        for (int u = 0; u < NTG; ++u) {
          const int col = (ngp * NTG + u) * 8 + gq;
          const int c = col / EPB, e = col % EPB;
          cbase[u] = (c < NC) ? (e * NP) * FST + c * DIM : -1;
        }
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          float g0[NTG];
#pragma unroll
          for (int u = 0; u < NTG; ++u) g0[u] = cbase[u] >= 0 ? gfl[cbase[u] + r] : 0.f;
#pragma unroll
          for (int ks = 0; ks < KUR / 8; ++ks) {
            const int k0 = ks * 8 + tq;
            SplitB bs[NTG] = {};
#pragma unroll
            for (int u = 0; u < NTG; ++u) {
              float b0 = 0.f, b1 = 0.f;
              if (cbase[u] >= 0) {
                b0 = gfl[cbase[u] + k0 * FST + r] - g0[u];
                b1 = gfl[cbase[u] + (k0 + 4) * FST + r] - g0[u];
              }
              bs[u] = SplitB(b0, b1);
            }
#pragma unroll
            for (int t = 0; t < MT; ++t) {
              uint32_t ah[4], alo[4];
              load_a_tf32_ldsm(ah, aw + r * MP * KU, KU, t * 16, ks * 8, lane);
              load_a_tf32_ldsm(alo, aw + AWN + r * MP * KU, KU, t * 16, ks * 8, lane);
#pragma unroll
              for (int u = 0; u < NTG; ++u) mma_tf32x3(d[t][u], ah, alo, bs[u]);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < NTG; ++u)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int col = (ngp * NTG + u) * 8 + 2 * tq + h;
            const int c = col / EPB, e = col % EPB;
            if (c >= NC || e >= ne) continue;
            R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
            for (int t = 0; t < MT; ++t)
#pragma unroll
              for (int half = 0; half < NACC / 2; ++half) {
                const int i = t * MROW + gq + 8 * half;
                if (i >= NP) continue;
                R v = -d[t][u][2 * half + h];
                if (sources && c >= 2 + DIM) v += src_s[(c - 2 - DIM) * ENP + e * NP + i];
                outp[i] = v;
              }
          }
      }
    } else
    for (int w = warp; w < (NNT / NTG) * MT; w += nwarps) {
      const int ngp = w / MT, t = w % MT;
      R d[NTG][NACC];
#pragma unroll
      for (int u = 0; u < NTG; ++u)
#pragma unroll
        for (int v = 0; v < NACC; ++v) d[u][v] = R(0);
      int cbase[NTG];
#pragma unroll
      for (int u = 0; u < NTG; ++u) {
        const int col = (ngp * NTG + u) * 8 + gq;
        const int c = col / EPB, e = col % EPB;
        cbase[u] = (c < NC) ? (e * NP) * FST + c * DIM : -1;
      }
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        R g0[NTG];
#pragma unroll
        for (int u = 0; u < NTG; ++u) g0[u] = cbase[u] >= 0 ? gfl[cbase[u] + r] : R(0);
        if constexpr (!V::TF32) {
#pragma unroll
          for (int ks = 0; ks < KUR / 4; ++ks) {
            const double av = aw[(r * MP + t * 8 + gq) * KU + ks * 4 + tq];
            const int kk = ks * 4 + tq;
#pragma unroll
            for (int u = 0; u < NTG; ++u) {
              const double b = cbase[u] >= 0 ? gfl[cbase[u] + kk * FST + r] - g0[u] : 0.0;
              dmma884(d[u], av, b);
            }
          }
        } else {
#pragma unroll
          for (int ks = 0; ks < KUR / 8; ++ks) {
            uint32_t ah[4], alo[4];
            load_a_tf32_ldsm(ah, aw + r * MP * KU, KU, t * 16, ks * 8, lane);
            load_a_tf32_ldsm(alo, aw + AWN + r * MP * KU, KU, t * 16, ks * 8, lane);
            const int k0 = ks * 8 + tq;
#pragma unroll
            for (int u = 0; u < NTG; ++u) {
              float b0 = 0.f, b1 = 0.f;
              if (cbase[u] >= 0) {
                b0 = gfl[cbase[u] + k0 * FST + r] - g0[u];
                b1 = gfl[cbase[u] + (k0 + 4) * FST + r] - g0[u];
              }
              mma_tf32x3(d[u], ah, alo, b0, b1);
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < NTG; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int col = (ngp * NTG + u) * 8 + 2 * tq + h;
          const int c = col / EPB, e = col % EPB;
          if (c >= NC || e >= ne) continue;
          R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
          for (int half = 0; half < NACC / 2; ++half) {
            const int i = t * MROW + gq + 8 * half;
            if (i >= NP) continue;
            R v = -d[u][2 * half + h];
            if (sources && c >= 2 + DIM) v += src_s[(c - 2 - DIM) * ENP + e * NP + i];
            outp[i] = v;
          }
        }
    }
  }
  if (bad) atomicOr(a.status, ST_NAN);
}

// Face pass on interior faces with HLL, and wherever a face needs more than
// the records' Rusanov / central combination: the HLL inviscid flux from the
// two states (q, p, c, gamma), the viscous parts central
// (inviscid.py:202-287, viscous.py:296-349).  recm / recp: own and
// neighbour-convention records; qp_g: the exterior q (stride qstride).
template <class R, int DIM, int NS, bool VISC>
__device__ __noinline__ void face_flux_general(const DGArgs<R> a, int64_t EN, int64_t gm,
                                               const R* recm, const R* recp, const R* qp_g,
                                               int64_t qstride, R n0, R n1, R n2, R fsc,
                                               const R* s0, R* bcol, int cstride) {
  constexpr int NC = DIM + 2 + NS;
  const R n[3] = {n0, n1, n2};
  R qm[NC], qp[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    qm[c] = a.q[c * EN + gm];
    qp[c] = qp_g[c * qstride];
  }
  NodeState<R, DIM, NS> sm, sp;
  make_state_light<R, DIM, NS>(qm, recm[NC + 1], recm[NC + 2], recm[NC + 3], sm);
  make_state_light<R, DIM, NS>(qp, recp[NC + 1], recp[NC + 2], recp[NC + 3], sp);
  R fi[NC], fim[NC], fip[NC];
  inviscid_num_flux<R, DIM, NS>(sm, sp, qm, qp, n, FLUX_HLL, fi);
  inviscid_flux_n<R, DIM, NS>(sm, n, fim);
  inviscid_flux_n<R, DIM, NS>(sp, n, fip);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    R out = -fi[c];
    // F_V . n = F . n + F_I . n on each side; the neighbour record holds -F . n
    if (VISC) out += ((recm[c] + fim[c]) + (-recp[c] + fip[c])) * R(0.5);
    bcol[c * cstride] = fsc * (out - s0[c]);
  }
}

// Face kernel: numerical fluxes from the face-node records, lift, added to
// the volume kernel's result.
template <class R, int DIM, int ORDER, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__((VCfg<R, DIM, ORDER, NS, MIX>::NT2),
                                  (VCfg<R, DIM, ORDER, NS, MIX>::MINB2))
    k_face(DGArgs<R> a, GasParams g) {
  using V = VCfg<R, DIM, ORDER, NS, MIX>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = V::NP, NF = V::NF, NFP = V::NFP, NFN = V::NFN, NC = V::NC, TW = V::TW;
  constexpr int EPB = V::EPB2, MP = V::MP, MT = V::MT, KF = V::KF, KFR = V::KFR;
  constexpr int NCOL = V::NCOL2, MROW = V::MROW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* am = reinterpret_cast<R*>(smem_raw);                  // [NAC][MP][KF] LIFT
  R* bm = am + V::A_FACE;                                  // [NCOL][KF]
  R* rx_s = bm + NCOL * KF;
  R* nrm_s = rx_s + EPB * DIM * DIM;
  R* fs_s = nrm_s + EPB * NF * DIM;
  int* fn_s = reinterpret_cast<int*>(fs_s + EPB * NF);
  int32_t* conn_s = fn_s + NFN;
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(conn_s + EPB * NF);
  uint8_t* fslot_s = perm_s + a.nperm * NFP;

  const int E = a.nelem;
  const int64_t EN = (int64_t)E * NP;
  for (int i = threadIdx.x; i < MP * KF; i += blockDim.x) {
    const int row = i / KF, k = i % KF;
    put_a<R>(am, MP * KF, i, (row < NP && k < NFN) ? c_ref64[S::OFF_LIFT + row * NFN + k] : 0.0);
  }
  for (int i = threadIdx.x; i < NCOL * KF; i += blockDim.x) bm[i] = R(0);
  for (int i = threadIdx.x; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) {
    perm_s[i] = a.perm[i];
    fslot_s[i] = a.fslot[i];
  }

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const int nwarps = blockDim.x >> 5;
  constexpr int NACC = V::TF32 ? 4 : 2;
  const int ntiles = (a.nowned + EPB - 1) / EPB;
  const int64_t bstride = (int64_t)a.nbf * NFP;
  bool bad = false;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * EPB;
    const int ne = imin(EPB, a.nowned - e0);
    // (the previous tile's contraction reads am / bm only; load_geometry's
    // first barrier orders it before this tile's writes of bm)
    stage_conn<NF>(a.conn, e0, ne, conn_s);
    load_geometry<R, DIM, ORDER>(a.rx, e0, ne, rx_s, nrm_s, fs_s);
    __syncthreads();

    for (int fnode = threadIdx.x; fnode < ne * NFN; fnode += blockDim.x) {
      const int e = fnode / NFN, fm = fnode % NFN, f = fm / NFP, m = fm % NFP;
      const int k = fn_s[fm];
      const int cn = conn_s[e * NF + f];
      const R fsc = fs_s[e * NF + f];
      const int64_t gm = (int64_t)(e0 + e) * NP + k;
      const R* recm = a.trace + (((int64_t)(e0 + e) * NF + f) * NFP + m) * TW;
      const R* s0 = a.s0 + ((int64_t)(e0 + e) * NF + f) * NC;
      R* bcol = bm + e * KF + fm;
      // neighbour record and exterior q; mode 0 interior, 1 prescribed,
      // 2 interior flux only (dummy boundary, or a pairing that fails its
      // index checks)
      int mode = 2;
      const R* recp = nullptr;
      const R* qp_g = nullptr;
      int64_t qstride = EN;
      if (cn >= 0) {
        const int en = cn >> 8, pr = cn & 255;
        int kn = NP, sl = NFN;
        if (pr < a.nperm) {
          kn = perm_s[pr * NFP + m];
          sl = fslot_s[pr * NFP + m];
        }
        if (en < E && kn < NP && sl < NFN) {
          recp = a.trace + ((int64_t)en * NFN + sl) * TW;
          qp_g = a.q + (int64_t)en * NP + kn;
          mode = 0;
        } else {
          atomicOr(a.status, ST_BAD_INDEX);
        }
      } else {
        const int bf = -(cn + 1);
        int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
        if ((bk_needs_bext(kind) && !a.bext) || kind > BK_OUTFLOW) kind = -1;
        if (kind >= BK_PRESCRIBED) {
          // the volume kernel filed the exterior record and state_plus
          recp = a.btrace + ((int64_t)bf * NFP + m) * TW;
          qp_g = a.bplus + (int64_t)bf * NFP + m;
          qstride = bstride;
          mode = 1;
        } else if (kind < 0) {
          atomicOr(a.status, ST_BAD_INDEX);
        }
      }
      if (mode == 2) {
        // DummyBoundary: F* = F(q-) . n (boundary.py:1027-1049)
#pragma unroll
        for (int c = 0; c < NC; ++c) bcol[c * EPB * KF] = fsc * (recm[c] - s0[c]);
        continue;
      }
      if (a.flux_kind == FLUX_HLL) {
        const R* nf = nrm_s + (e * NF + f) * DIM;
        face_flux_general<R, DIM, NS, VISC>(a, EN, gm, recm, recp, qp_g, qstride, nf[0], nf[1],
                                            DIM > 2 ? nf[DIM - 1] : R(0), fsc, s0, bcol,
                                            EPB * KF);
        continue;
      }
      R rm[TW], rp[TW];
      load_record<R, TW>(recm, rm);
      load_record<R, TW>(recp, rp);
      R qm[NC], qp[NC], sh[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        qm[c] = a.q[c * EN + gm];
        qp[c] = qp_g[c * qstride];
        sh[c] = s0[c];
      }
      const R lam = (a.flux_kind == FLUX_RUSANOV) ? fmax(rm[NC], rp[NC]) : R(0);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const R out = (rm[c] - rp[c]) * R(0.5) - lam * (qm[c] - qp[c]) * R(0.5);
        bcol[c * EPB * KF] = fsc * (out - sh[c]);
      }
    }
    __syncthreads();

    // rhs += LIFT S on the tensor cores.  float32: one item per group of NTG
    // column tiles and every m-tile, each face value split into its tf32
    // hi/lo words once; float64: one m-tile and NTG column tiles per item
    constexpr int NNT = NCOL / 8;
    constexpr int NTG = (NNT % 3 == 0) ? 3 : ((NNT % 2 == 0) ? 2 : 1);
    if constexpr (V::TF32) {
      for (int ngp = warp; ngp < NNT / NTG; ngp += nwarps) {
        float d[MT][NTG][NACC];
#pragma unroll
        for (int t = 0; t < MT; ++t)
#pragma unroll
          for (int u = 0; u < NTG; ++u)
#pragma unroll
            for (int v = 0; v < NACC; ++v) d[t][u][v] = 0.f;
        const R* bcol = bm + (ngp * NTG * 8 + gq) * KF + tq;
#pragma unroll
        for (int ks = 0; ks < KFR / 8; ++ks) {
          SplitB bs[NTG];
#pragma unroll
          for (int u = 0; u < NTG; ++u)
            bs[u] = SplitB(bcol[u * 8 * KF + ks * 8], bcol[u * 8 * KF + ks * 8 + 4]);
#pragma unroll
          for (int t = 0; t < MT; ++t) {
            uint32_t ah[4], alo[4];
            load_a_tf32_ldsm(ah, am, KF, t * 16, ks * 8, lane);
            load_a_tf32_ldsm(alo, am + MP * KF, KF, t * 16, ks * 8, lane);
#pragma unroll
            for (int u = 0; u < NTG; ++u) mma_tf32x3(d[t][u], ah, alo, bs[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < NTG; ++u)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int col = (ngp * NTG + u) * 8 + 2 * tq + h;
            const int c = col / EPB, e = col % EPB;
            if (c >= NC || e >= ne) continue;
            R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
            for (int t = 0; t < MT; ++t)
#pragma unroll
              for (int half = 0; half < NACC / 2; ++half) {
                const int i = t * MROW + gq + 8 * half;
                if (i >= NP) continue;
                const R v = outp[i] + d[t][u][2 * half + h];
                outp[i] = v;
                bad |= !(v == v);
              }
          }
      }
    } else
    for (int w = warp; w < (NNT / NTG) * MT; w += nwarps) {
      const int ngp = w / MT, t = w % MT;
      R d[NTG][NACC];
#pragma unroll
      for (int u = 0; u < NTG; ++u)
#pragma unroll
        for (int v = 0; v < NACC; ++v) d[u][v] = R(0);
      const R* bcol = bm + (ngp * NTG * 8 + gq) * KF + tq;
      if constexpr (!V::TF32) {
#pragma unroll
        for (int ks = 0; ks < KFR / 4; ++ks) {
          const double av = am[(t * 8 + gq) * KF + ks * 4 + tq];
#pragma unroll
          for (int u = 0; u < NTG; ++u) dmma884(d[u], av, bcol[u * 8 * KF + ks * 4]);
        }
      } else {
#pragma unroll
        for (int ks = 0; ks < KFR / 8; ++ks) {
          uint32_t ah[4], alo[4];
          load_a_tf32_ldsm(ah, am, KF, t * 16, ks * 8, lane);
          load_a_tf32_ldsm(alo, am + MP * KF, KF, t * 16, ks * 8, lane);
#pragma unroll
          for (int u = 0; u < NTG; ++u)
            mma_tf32x3(d[u], ah, alo, bcol[u * 8 * KF + ks * 8], bcol[u * 8 * KF + ks * 8 + 4]);
        }
      }
#pragma unroll
      for (int u = 0; u < NTG; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int col = (ngp * NTG + u) * 8 + 2 * tq + h;
          const int c = col / EPB, e = col % EPB;
          if (c >= NC || e >= ne) continue;
          R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
#pragma unroll
          for (int half = 0; half < NACC / 2; ++half) {
            const int i = t * MROW + gq + 8 * half;
            if (i >= NP) continue;
            const R v = outp[i] + d[u][2 * half + h];
            outp[i] = v;
            bad |= !(v == v);
          }
        }
    }
  }
  if (bad) atomicOr(a.status, ST_NAN);
}

}  // namespace

}  // namespace mgc
