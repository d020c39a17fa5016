// Gradient and surface/lift passes for tensor-product (GLL) hexahedra.
//
// Same mathematics as the simplex passes (mirgecom/operators.py:34-95,
// navierstokes.py:118-575, euler.py:313-416), with sum factorisation: every
// operator of the reference hexahedron is a Kronecker product of 1-D
// operators, so it acts on the N1 = p+1 nodes of each line of nodes along
// one reference axis.  For an affine element the face terms combine with
// the same metric factors as the volume terms: the outward normal of face
// (a, side) times its surface factor is (side ? +1 : -1) rx[a][:] FSR
// (n dS = J rx^T N dS_ref), so along a line of axis a
//
//   gradient    grad_j += rx[a][j] v_a,
//               v_a = -W1 u' - FSR L1[:,0] s'_lo + FSR L1[:,1] s'_hi
//   divergence  rhs    += -W1 G_a + L1[:,0] S_lo + L1[:,1] S_hi,
//               G_a = sum_j rx[a][j] (F_j - F0_j)
//
// with W1 = M1^-1 D1^T M1 (1-D weak derivative), L1 = M1^-1 e_{0,p} (1-D lift
// of the two line ends), u' = u - u0 and s' = u* - u0 the values shifted by
// the element's node-0 value, and S the face fluxes of the split divergence
// (fsc (F* - F0) . n).  Each line is one column of a small matrix product
// A [N1 x (N1+2)] x B [(N1+2) x lines]; it runs on the tensor cores --
// float64 mma m8n8k4, or the TF32 three-term split on mma m16n8k8 -- with
// the 25 lines of an axis as the N dimension and A held in registers.
#pragma once
#include "dg_dispatch.cuh"

namespace mgc {

// {{{ 1-D operators in constant memory

// packed per order p = 1..4:  W1 [N1][N1], L1 [N1][2], FSR
__host__ __device__ constexpr int hexops_size(int order) {
  return (order + 1) * (order + 1) + 2 * (order + 1) + 1;
}
__host__ __device__ constexpr int hexops_offset(int order) {
  int off = 0;
  for (int o = 1; o < order; ++o) off += hexops_size(o);
  return off;
}
constexpr int kHexMaxOrder = 4;
constexpr int kHexOpsTotal = hexops_offset(kHexMaxOrder + 1);

static __constant__ double c_hex64[kHexOpsTotal];

template <int ORDER>
struct Hex {
  static constexpr int N1 = ORDER + 1;
  static constexpr int NP = N1 * N1 * N1, NF = 6, NFP = N1 * N1, NFN = NF * NFP;
  static constexpr int NL = N1 * N1;                 // lines per axis
  static constexpr int NNT = (NL + 7) / 8;           // 8-line n-tiles per axis
  static constexpr int KH = N1 + 2;                  // k extent of the line operator
  static constexpr int OFF_W = hexops_offset(ORDER);
  static constexpr int OFF_L = OFF_W + N1 * N1;
  static constexpr int OFF_FSR = OFF_L + 2 * N1;
  static_assert(KH <= 8, "line operator must fit one k-step of 8");
};

// volume node of position k along axis a on line n (n runs over the other
// two axes, the lower one fastest); line n of axis a is also face node n of
// faces (a, 0) and (a, 1)
template <int N1>
__device__ __forceinline__ int hex_node(int a, int n, int k) {
  const int lo = n % N1, hi = n / N1;
  return a == 0 ? k + N1 * (lo + N1 * hi) : a == 1 ? lo + N1 * (k + N1 * hi)
                                                   : lo + N1 * (hi + N1 * k);
}

// Entry (i, k) of the line operator [-W1 | cl L1[:,0] | ch L1[:,1]]
template <int ORDER>
__device__ __forceinline__ double hex_line_op(int i, int k, double cl, double ch) {
  using H = Hex<ORDER>;
  if (i >= H::N1 || k >= H::KH) return 0.0;
  if (k < H::N1) return -c_hex64[H::OFF_W + i * H::N1 + k];
  return (k == H::N1 ? cl : ch) * c_hex64[H::OFF_L + i * 2 + (k - H::N1)];
}

// Line-operator fragments of one lane, kept in registers for the kernel.
//   double: mma m8n8k4, A[g][t] of the two k-steps
//   float : mma m16n8k8, a0 = A[g][t], a2 = A[g][t+4] (rows >= 8 are zero),
//           TF32 hi/lo split
template <class R> struct LineOp;
template <> struct LineOp<double> {
  double a[2];
  template <int ORDER>
  __device__ __forceinline__ void init(double cl, double ch, int g, int t) {
    a[0] = hex_line_op<ORDER>(g, t, cl, ch);
    a[1] = hex_line_op<ORDER>(g, t + 4, cl, ch);
  }
  // d[0], d[1] = D[g][2t], D[g][2t+1]; b0, b1 = B[t][g], B[t+4][g]
  __device__ __forceinline__ void apply(double (&d)[2], double b0, double b1) const {
    d[0] = d[1] = 0.0;
    dmma884(d, a[0], b0);
    dmma884(d, a[1], b1);
  }
};
template <> struct LineOp<float> {
  uint32_t hi[4], lo[4];
  template <int ORDER>
  __device__ __forceinline__ void init(double cl, double ch, int g, int t) {
    float h, l;
    split_tf32(hex_line_op<ORDER>(g, t, cl, ch), h, l);
    hi[0] = __float_as_uint(h);
    lo[0] = __float_as_uint(l);
    split_tf32(hex_line_op<ORDER>(g, t + 4, cl, ch), h, l);
    hi[2] = __float_as_uint(h);
    lo[2] = __float_as_uint(l);
    hi[1] = hi[3] = lo[1] = lo[3] = 0u;
  }
  __device__ __forceinline__ void apply(float (&d)[2], float b0, float b1) const {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    mma_tf32x3(acc, hi, lo, b0, b1);
    d[0] = acc[0];
    d[1] = acc[1];
  }
};

// }}}

namespace {

template <class R, int ORDER, int NS, bool MIX>
struct HexCfg {
  using H = Hex<ORDER>;
  static constexpr int NC = 5 + NS, NU = NC + 1, RB = (int)sizeof(R);
  static constexpr int NT = 256;
  static constexpr int NW = NT / 32;
  // element tiles: gradient [u][NU][NP] + [s'][NU][NF][NFP]; surface
  // [G][NC][3][NP] + [S][NC][NF][NFP]; per-warp accumulators
  static constexpr int G_ELEM = NU * (H::NP + H::NFN) + 9;
  static constexpr int S_ELEM = NC * (3 * H::NP + H::NFN) + 9;
  static constexpr int BUDGET = 96 * 1024 / RB;
  static constexpr int EPB_G = imax(1, imin(4, (BUDGET - NW * 3 * H::NP) / G_ELEM));
  static constexpr int EPB_S = imax(1, imin(4, (BUDGET - NW * H::NP) / S_ELEM));
  static size_t smem_grad(int nperm) {
    return (size_t)(EPB_G * G_ELEM + NW * 3 * H::NP) * RB + EPB_G * 6 * 4 +
           (size_t)nperm * H::NFP + 64;
  }
  static size_t smem_surface(int nperm) {
    return (size_t)(EPB_S * S_ELEM + NW * H::NP) * RB + EPB_S * 6 * 4 +
           (size_t)nperm * H::NFP + 64;
  }
};

// {{{ gradient

template <class R, int ORDER, int NS, bool MIX>
__global__ void __launch_bounds__(256, 2) k_hex_grad(DGArgs<R> a, GasParams g) {
  using C = HexCfg<R, ORDER, NS, MIX>;
  using H = Hex<ORDER>;
  constexpr int N1 = H::N1, NP = H::NP, NFP = H::NFP, NFN = H::NFN, NL = H::NL;
  constexpr int NC = C::NC, NU = C::NU, EPB = C::EPB_G, DIM = 3;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* u_s = reinterpret_cast<R*>(smem_raw);             // [EPB][NU][NP]
  R* s_s = u_s + EPB * NU * NP;                         // [EPB][NU][NF][NFP]
  R* rx_s = s_s + EPB * NU * NFN;                       // [EPB][9]
  R* acc_all = rx_s + EPB * 9;                          // [NW][3][NP]
  int32_t* conn_s = reinterpret_cast<int32_t*>(acc_all + C::NW * 3 * NP);  // [EPB][6]
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(conn_s + EPB * 6);

  const int E = a.nelem;
  const int64_t EN = (int64_t)E * NP;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const double fsr = c_hex64[H::OFF_FSR];
  LineOp<R> op;
  op.template init<ORDER>(-fsr, fsr, gq, tq);
  R* acc = acc_all + warp * 3 * NP;
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];

  const int ntiles = (E + EPB - 1) / EPB;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * EPB;
    const int ne = imin(EPB, E - e0);
    __syncthreads();   // the previous tile's contraction reads are done
    for (int i = threadIdx.x; i < ne * 9; i += blockDim.x)
      rx_s[i] = a.rx[(int64_t)e0 * 9 + i];
    stage_conn<6>(a.conn, e0, ne, conn_s);
    // conserved fields and temperature of the tile
    for (int idx = threadIdx.x; idx < ne * NP; idx += blockDim.x) {
      const int e = idx / NP, k = idx % NP;
      const int64_t gn = (int64_t)e0 * NP + idx;
      R qq[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        qq[c] = a.q[c * EN + gn];
        u_s[(e * NU + c) * NP + k] = qq[c];
      }
      u_s[(e * NU + NC) * NP + k] = MIX ? a.t_op[gn] : node_temperature<R, DIM, NS>(qq, R(0), g);
    }
    __syncthreads();

    // face values s' = u* - u0, one face node per item
    for (int fnode = threadIdx.x; fnode < ne * NFN; fnode += blockDim.x) {
      const int e = fnode / NFN, fm = fnode % NFN, f = fm / NFP, m = fm % NFP;
      const int k = hex_node<N1>(f >> 1, m, (f & 1) ? N1 - 1 : 0);
      const int cn = conn_s[e * 6 + f];
      int mode = 2;   // 0 two-sided average, 1 prescribed exterior, 2 interior value
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
        const int kind = (bf < a.nbf) ? a.bkind[bf] : -1;
        if (kind == BK_PRESCRIBED)
          mode = 1;
        else if (kind != BK_DUMMY)   // unknown, or a kind the hexahedra do not evaluate
          atomicOr(a.status, ST_BAD_INDEX);
      }
      R* scol = s_s + e * NU * NFN + fm;
      if (mode == 2) {
#pragma unroll
        for (int c = 0; c < NU; ++c)
          scol[c * NFN] = u_s[(e * NU + c) * NP + k] - u_s[(e * NU + c) * NP];
        continue;
      }
      const int64_t bstride = (int64_t)a.nbf * NFP, bo = (int64_t)bf * NFP + m;
      R up[NU];
#pragma unroll
      for (int c = 0; c < NC; ++c) up[c] = (mode == 0) ? a.q[c * EN + gi] : a.bext[c * bstride + bo];
      if (MIX)
        up[NC] = (mode == 0) ? a.t_op[gi] : a.bext[NC * bstride + bo];
      else
        up[NC] = node_temperature<R, DIM, NS>(up, R(0), g);
#pragma unroll
      for (int c = 0; c < NU; ++c) {
        const R u0 = u_s[(e * NU + c) * NP];
        const R um = u_s[(e * NU + c) * NP + k] - u0;
        scol[c * NFN] = (mode == 0) ? ((up[c] - u0) + um) * R(0.5) : up[c] - u0;
      }
    }
    __syncthreads();

    // line contractions, one (element, field) per warp
    for (int unit = warp; unit < ne * NU; unit += C::NW) {
      const int e = unit / NU, c = unit % NU;
      const R* u = u_s + (e * NU + c) * NP;
      const R* sf = s_s + (e * NU + c) * NFN;
      const R u0 = u[0];
      for (int i = lane; i < 3 * NP; i += 32) acc[i] = R(0);
      __syncwarp();
#pragma unroll 1
      for (int ax = 0; ax < 3; ++ax) {
        R rxa[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) rxa[j] = rx_s[e * 9 + ax * 3 + j];
#pragma unroll
        for (int nt = 0; nt < H::NNT; ++nt) {
          const int n = nt * 8 + gq;
          R b[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int k = tq + 4 * h;
            R v = R(0);
            if (n < NL) {
              if (k < N1) v = u[hex_node<N1>(ax, n, k)] - u0;
              else if (k == N1) v = sf[(2 * ax) * NFP + n];
              else if (k == N1 + 1) v = sf[(2 * ax + 1) * NFP + n];
            }
            b[h] = v;
          }
          R d[2];
          op.apply(d, b[0], b[1]);
          if (gq < N1) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int line = nt * 8 + 2 * tq + h;
              if (line < NL) {
                const int node = hex_node<N1>(ax, line, gq);
#pragma unroll
                for (int j = 0; j < 3; ++j) acc[j * NP + node] += rxa[j] * d[h];
              }
            }
          }
        }
        __syncwarp();
      }
      R* outp = a.out + ((int64_t)c * DIM) * EN + (int64_t)(e0 + e) * NP;
      for (int i = lane; i < 3 * NP; i += 32) {
        const int j = i / NP, k = i % NP;
        outp[(int64_t)j * EN + k] = acc[i];
      }
      __syncwarp();
    }
  }
}

// }}}

// {{{ surface and lift

template <class R, int ORDER, int NS, bool MIX, bool VISC>
__global__ void __launch_bounds__(256, 2) k_hex_surface(DGArgs<R> a, GasParams g) {
  using C = HexCfg<R, ORDER, NS, MIX>;
  using H = Hex<ORDER>;
  constexpr int N1 = H::N1, NP = H::NP, NFP = H::NFP, NFN = H::NFN, NL = H::NL;
  constexpr int NC = C::NC, EPB = C::EPB_S, DIM = 3;
  constexpr int FW = flux_record_width(DIM, NC);
  constexpr int CG = 4, NG = (NC + CG - 1) / CG, GV = CG * DIM, LIM = NC * DIM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* g_s = reinterpret_cast<R*>(smem_raw);              // [EPB][NC][3][NP]
  R* s_s = g_s + EPB * NC * 3 * NP;                     // [EPB][NC][NF][NFP]
  R* rx_s = s_s + EPB * NC * NFN;                       // [EPB][9]
  R* acc_all = rx_s + EPB * 9;                          // [NW][NP]
  int32_t* conn_s = reinterpret_cast<int32_t*>(acc_all + C::NW * NP);  // [EPB][6]
  uint8_t* perm_s = reinterpret_cast<uint8_t*>(conn_s + EPB * 6);

  const int E = a.nelem;
  const int64_t EN = (int64_t)E * NP;
  const bool sources = MIX && a.add_sources;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const R fsr = (R)c_hex64[H::OFF_FSR];
  LineOp<R> op;
  op.template init<ORDER>(1.0, 1.0, gq, tq);
  R* acc = acc_all + warp * NP;
  for (int i = threadIdx.x; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];

  const int ntiles = (E + EPB - 1) / EPB;
  bool bad = false;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * EPB;
    const int ne = imin(EPB, E - e0);
    __syncthreads();
    for (int i = threadIdx.x; i < ne * 9; i += blockDim.x)
      rx_s[i] = a.rx[(int64_t)e0 * 9 + i];
    stage_conn<6>(a.conn, e0, ne, conn_s);
    __syncthreads();

    // volume: G_a = sum_j rx[a][j] (F_j - F0_j)
    for (int it = threadIdx.x; it < ne * NP * NG; it += blockDim.x) {
      const int grp = it % NG, node = it / NG;
      const int e = node / NP, k = node % NP;
      R fv[GV], f0v[GV];
      load_group<R, GV>(a.fbuf + ((int64_t)e0 * NP + node) * FW, grp * GV, LIM, fv);
      load_group<R, GV>(a.fbuf + ((int64_t)(e0 + e) * NP) * FW, grp * GV, LIM, f0v);
      const R* rxe = rx_s + e * 9;
#pragma unroll
      for (int cc = 0; cc < CG; ++cc) {
        const int c = grp * CG + cc;
        if (c >= NC) break;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          R s = R(0);
#pragma unroll
          for (int j = 0; j < 3; ++j) s += rxe[r * 3 + j] * (fv[cc * DIM + j] - f0v[cc * DIM + j]);
          g_s[((e * NC + c) * 3 + r) * NP + k] = s;
        }
      }
    }

    // faces: S = fsc (F* - F0) . n, one face node per item
    for (int fnode = threadIdx.x; fnode < ne * NFN; fnode += blockDim.x) {
      const int e = fnode / NFN, fm = fnode % NFN, f = fm / NFP, m = fm % NFP;
      const int ax = f >> 1;
      const int k = hex_node<N1>(ax, m, (f & 1) ? N1 - 1 : 0);
      const int cn = conn_s[e * 6 + f];
      // n dS = J rx^T N dS_ref: the normal is +-rx[ax][:] normalised
      R n[3], mag2 = R(0);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        n[j] = (f & 1) ? rx_s[e * 9 + ax * 3 + j] : -rx_s[e * 9 + ax * 3 + j];
        mag2 += n[j] * n[j];
      }
      const R mag = sqrt(mag2);
#pragma unroll
      for (int j = 0; j < 3; ++j) n[j] = n[j] / mag;
      const R fsc = mag * fsr;
      const int64_t gm = (int64_t)(e0 + e) * NP + k, g0 = (int64_t)(e0 + e) * NP;
      R* bcol = s_s + (e * NC) * NFN + fm;
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
            bcol[c * NFN] = fsc * (out - s0);
          }
        }
      } else {
        surface_face_general<R, DIM, NP, NFP, NS, MIX, VISC>(a, g, EN, gm, g0, m, cn, n[0], n[1],
                                                             n[2], fsc, perm_s, bcol, NFN);
      }
    }
    __syncthreads();

    // line contractions and the sum over axes, one (element, field) per warp
    for (int unit = warp; unit < ne * NC; unit += C::NW) {
      const int e = unit / NC, c = unit % NC;
      const R* gc = g_s + (e * NC + c) * 3 * NP;
      const R* sf = s_s + (e * NC + c) * NFN;
      for (int i = lane; i < NP; i += 32) acc[i] = R(0);
      __syncwarp();
#pragma unroll 1
      for (int ax = 0; ax < 3; ++ax) {
#pragma unroll
        for (int nt = 0; nt < H::NNT; ++nt) {
          const int n = nt * 8 + gq;
          R b[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int k = tq + 4 * h;
            R v = R(0);
            if (n < NL) {
              if (k < N1) v = gc[ax * NP + hex_node<N1>(ax, n, k)];
              else if (k == N1) v = sf[(2 * ax) * NFP + n];
              else if (k == N1 + 1) v = sf[(2 * ax + 1) * NFP + n];
            }
            b[h] = v;
          }
          R d[2];
          op.apply(d, b[0], b[1]);
          if (gq < N1) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int line = nt * 8 + 2 * tq + h;
              if (line < NL) acc[hex_node<N1>(ax, line, gq)] += d[h];
            }
          }
        }
        __syncwarp();
      }
      R* outp = a.out + (int64_t)c * EN + (int64_t)(e0 + e) * NP;
      for (int i = lane; i < NP; i += 32) {
        R v = acc[i];
        if (sources && c >= 2 + DIM)
          v += a.srcbuf[(int64_t)(c - 2 - DIM) * EN + (int64_t)(e0 + e) * NP + i];
        outp[i] = v;
        bad |= !(v == v);
      }
      __syncwarp();
    }
  }
  if (bad) atomicOr(a.status, ST_NAN);
}

// }}}

// {{{ launches

template <class R, int ORDER, int NS, bool MIX>
struct HexLaunch {
  using C = HexCfg<R, ORDER, NS, MIX>;
  using H = Hex<ORDER>;
  static int grad(const DGArgs<R>& a, const GasParams& g, cudaStream_t s) {
    const size_t smem = C::smem_grad(a.nperm);
    auto kern = k_hex_grad<R, ORDER, NS, MIX>;
    int rc = prepare_kernel(kern, smem);
    if (rc) return rc;
    int nblk = 0;
    rc = persistent_grid(kern, C::NT, smem, (a.nelem + C::EPB_G - 1) / C::EPB_G, &nblk);
    if (rc) return rc;
    kern<<<nblk, C::NT, smem, s>>>(a, g);
    return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
  }
  template <bool VISC>
  static int rhs_split(const DGArgs<R>& a, const GasParams& g, cudaStream_t s) {
    const int64_t nn = (int64_t)a.nelem * H::NP;
    int64_t nb = (nn + 127) / 128;
    if (nb > 148 * 64) nb = 148 * 64;
    k_node_flux<R, 3, H::NP, NS, MIX, VISC><<<(unsigned)nb, 128, 0, s>>>(a, g);
    if (cudaGetLastError() != cudaSuccess) return MGC_E_CUDA;
    if (a.mid_event && cudaEventRecord(static_cast<cudaEvent_t>(a.mid_event), s) != cudaSuccess)
      return MGC_E_CUDA;
    const size_t smem = C::smem_surface(a.nperm);
    auto kern = k_hex_surface<R, ORDER, NS, MIX, VISC>;
    int rc = prepare_kernel(kern, smem);
    if (rc) return rc;
    int nblk = 0;
    rc = persistent_grid(kern, C::NT, smem, (a.nelem + C::EPB_S - 1) / C::EPB_S, &nblk);
    if (rc) return rc;
    kern<<<nblk, C::NT, smem, s>>>(a, g);
    return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
  }
  static size_t split_workspace_bytes(int64_t nelem) {
    constexpr int FW = flux_record_width(3, 5 + NS);
    return ((size_t)nelem * H::NP * FW + (size_t)NS * nelem * H::NP) * sizeof(R) + 256;
  }
};

// op: 0 = grad, 3 = euler (split), 4 = ns (split); hexahedra carry no fused
// divergence pass
template <class R, int ORDER>
inline int hex_dispatch_order(int op, int ns, bool mix, const DGArgs<R>& a, const GasParams& g,
                              cudaStream_t s) {
  if (ns != 0 || mix) return MGC_E_UNSUPPORTED;
  using L = HexLaunch<R, ORDER, 0, false>;
  if (op == 0) return L::grad(a, g, s);
  if (op == 3) return L::template rhs_split<false>(a, g, s);
  if (op == 4) return L::template rhs_split<true>(a, g, s);
  return MGC_E_UNSUPPORTED;
}

template <class R>
inline int hex_dispatch(int op, int order, int ns, bool mix, const DGArgs<R>& a,
                        const GasParams& g, cudaStream_t s) {
  switch (order) {
    case 1: return hex_dispatch_order<R, 1>(op, ns, mix, a, g, s);
    case 2: return hex_dispatch_order<R, 2>(op, ns, mix, a, g, s);
    case 3: return hex_dispatch_order<R, 3>(op, ns, mix, a, g, s);
    case 4: return hex_dispatch_order<R, 4>(op, ns, mix, a, g, s);
    default: return MGC_E_UNSUPPORTED;
  }
}

template <class R>
inline size_t hex_split_workspace(int order, int ns, bool mix, int64_t nelem) {
  if (ns != 0 || mix) return 0;
  switch (order) {
    case 1: return HexLaunch<R, 1, 0, false>::split_workspace_bytes(nelem);
    case 2: return HexLaunch<R, 2, 0, false>::split_workspace_bytes(nelem);
    case 3: return HexLaunch<R, 3, 0, false>::split_workspace_bytes(nelem);
    case 4: return HexLaunch<R, 4, 0, false>::split_workspace_bytes(nelem);
    default: return 0;
  }
}

inline int upload_hexops_local(const double* packed) {
  return cudaMemcpyToSymbol(c_hex64, packed, kHexOpsTotal * sizeof(double)) == cudaSuccess
             ? MGC_OK
             : MGC_E_CUDA;
}

// }}}

}  // namespace

}  // namespace mgc
