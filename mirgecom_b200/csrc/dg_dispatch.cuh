// Per-translation-unit dispatch from runtime (dim, order, nspecies, eos)
// to the compiled kernel instantiations.  Each unit that includes this file
// owns its own constant-memory banks, so it also provides the upload hooks.
#pragma once
#include <cuda_runtime.h>

#include <cstring>

#include "dg_kernels.cuh"
#include "dg_volume.cuh"
#include "grad_tc.cuh"
#include "../../include/mgc_b200.h"

namespace mgc {

static_assert(sizeof(GasParams) == sizeof(mgc_gas_t), "gas struct mismatch");
// device mechanism = the C ABI table followed by derived coefficient tables
inline Mechanism expand_mechanism(const mgc_mechanism_t& m) {
  Mechanism d;
  memset(&d, 0, sizeof(d));
  memcpy(&d, &m, sizeof(m));
  for (int s = 0; s < MGC_MAX_SPECIES; ++s) {
    for (int r = 0; r < 2; ++r) {
      const double* a = r ? m.a_hi[s] : m.a_lo[s];
      double* h = r ? d.h_hi[s] : d.h_lo[s];
      double* e = r ? d.s_hi[s] : d.s_lo[s];
      h[0] = a[0];
      h[1] = a[1] / 2;
      h[2] = a[2] / 3;
      h[3] = a[3] / 4;
      h[4] = a[4] / 5;
      h[5] = a[5];
      e[0] = a[0];
      e[1] = a[1];
      e[2] = a[2] / 2;
      e[3] = a[3] / 3;
      e[4] = a[4] / 4;
      e[5] = a[6];
    }
  }
  // Newton convergence constant: max over species and T in [200, 6000] K of
  // |c_v'| / (2 c_v), c_v/R = a0 - 1 + a1 T + ... + a4 T^4 (1 K steps)
  double kmax = 0.0;
  for (int s = 0; s < m.nspecies && s < MGC_MAX_SPECIES; ++s) {
    for (int ti = 200; ti <= 6000; ++ti) {
      const double t = ti;
      const double* a = (t > m.t_mid[s]) ? m.a_hi[s] : m.a_lo[s];
      const double cv = a[0] - 1.0 + t * (a[1] + t * (a[2] + t * (a[3] + t * a[4])));
      const double dcv = a[1] + t * (2.0 * a[2] + t * (3.0 * a[3] + t * 4.0 * a[4]));
      if (cv > 0.0) {
        const double k = 0.5 * (dcv < 0 ? -dcv : dcv) / cv;
        if (k > kmax) kmax = k;
      }
    }
  }
  d.newton_k = kmax;
  return d;
}

// The helpers below touch this translation unit's own constant banks and
// kernels, so they have internal linkage: a shared (inline, external) copy
// could be kept by the linker from any one unit and would then upload to,
// or launch from, that unit only.
namespace {

inline int upload_refops_local(int dim, int order, const double* packed64, const float* packed32,
                               const int* fnodes) {
  const int off = refops_offset(dim, order);
  const int n = refops_size(dim, order);
  const int foff = fnodes_offset(dim, order);
  const int fn = fnodes_size(dim, order);
  if (off < 0) return MGC_E_UNSUPPORTED;
  if (cudaMemcpyToSymbol(c_ref64, packed64, n * sizeof(double), off * sizeof(double)) != cudaSuccess)
    return MGC_E_CUDA;
  if (cudaMemcpyToSymbol(c_ref32, packed32, n * sizeof(float), off * sizeof(float)) != cudaSuccess)
    return MGC_E_CUDA;
  if (cudaMemcpyToSymbol(c_fnodes, fnodes, fn * sizeof(int), foff * sizeof(int)) != cudaSuccess)
    return MGC_E_CUDA;
  return MGC_OK;
}

inline int upload_mechanism_local(const Mechanism* m) {
  if (cudaMemcpyToSymbol(c_mech, m, sizeof(Mechanism)) != cudaSuccess) return MGC_E_CUDA;
  const MechanismT<float> f = narrow_mechanism(*m);
  return cudaMemcpyToSymbol(c_mech32, &f, sizeof(f)) == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

template <class Kern>
inline int prepare_kernel(Kern kern, size_t smem) {
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return MGC_E_CUDA;
  }
  return MGC_OK;
}

// Grid of a persistent kernel: every CTA that fits on the device at once
// (occupancy for this block size and shared memory times the SM count),
// capped at the number of work tiles.
template <class Kern>
inline int persistent_grid(Kern kern, int threads, size_t smem, int64_t tiles, int* nblk) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess)
    return MGC_E_CUDA;
  int64_t nb = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
  if (nb > tiles) nb = tiles;
  *nblk = (int)(nb > 0 ? nb : 1);
  return MGC_OK;
}

template <class R, int DIM, int ORDER, int NS, bool MIX>
struct Launch {
  using C = Cfg<R, DIM, ORDER, NS, MIX>;
  // the gradient kernel over the owned elements of a partition (its tile
  // loop runs to nelem): elements [nowned, nelem) are ghosts
  static int grad_owned(const DGArgs<R>& a, const GasParams& g, cudaStream_t s) {
    return grad(a, g, s);
  }
  static int grad(const DGArgs<R>& a, const GasParams& g, cudaStream_t s) {
    if constexpr (sizeof(R) == 4 && MIX && DIM == 3) {
      if constexpr (TcGrad<DIM, ORDER, NS>::OK) {
        if (a.grad_kernel == 0 && grad_tc_applies(a)) return grad_tc(a, g, s);
      }
    }
    const size_t smem = C::smem_grad(a.nperm);
    auto kern = k_grad<R, DIM, ORDER, NS, MIX>;
    int rc = prepare_kernel(kern, smem);
    if (rc) return rc;
    const int ntiles = (a.nelem + C::EPB_GRAD - 1) / C::EPB_GRAD;
    int nblk = 0;
    rc = persistent_grid(kern, C::NT, smem, ntiles, &nblk);
    if (rc) return rc;
    kern<<<nblk, C::NT, smem, s>>>(a, g);
    return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
  }
  // the tcgen05 gradient kernel reads rows of q and T in 16-byte pieces
  static bool grad_tc_applies(const DGArgs<R>& a) {
    const uintptr_t al = reinterpret_cast<uintptr_t>(a.q) | reinterpret_cast<uintptr_t>(a.t_op) |
                         reinterpret_cast<uintptr_t>(a.out);
    return a.t_op != nullptr && (al & 15) == 0 && a.nperm <= 64;
  }
  static int grad_tc(const DGArgs<R>& a, const GasParams& g, cudaStream_t s) {
    using T = TcGrad<DIM, ORDER, NS>;
    const size_t smem = T::smem_bytes(a.nperm);
    auto kern = k_grad_tc<DIM, ORDER, NS>;
    int rc = prepare_kernel(kern, smem);
    if (rc) return rc;
    const int eown = a.nowned > 0 ? a.nowned : a.nelem;
    const int ntiles = (eown + T::EPB - 1) / T::EPB;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return MGC_E_CUDA;
    const int nblk = ntiles < sms ? (ntiles > 0 ? ntiles : 1) : sms;
    kern<<<nblk, T::NT, smem, s>>>(a, g);
    return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
  }
  template <bool VISC>
  static int rhs_split(const DGArgs<R>& a, const GasParams& g, cudaStream_t s) {
    const int64_t nn = (int64_t)a.nelem * C::NP;
    int64_t nb = (nn + 127) / 128;
    if (nb > 148 * 64) nb = 148 * 64;
    k_node_flux<R, DIM, C::NP, NS, MIX, VISC><<<(unsigned)nb, 128, 0, s>>>(a, g);
    if (cudaGetLastError() != cudaSuccess) return MGC_E_CUDA;
    if (a.mid_event && cudaEventRecord(static_cast<cudaEvent_t>(a.mid_event), s) != cudaSuccess)
      return MGC_E_CUDA;
    const size_t smem = C::smem_surface(a.nperm);
    auto kern = k_surface<R, DIM, ORDER, NS, MIX, VISC>;
    int rc = prepare_kernel(kern, smem);
    if (rc) return rc;
    const int ntiles = (a.nelem + C::EPB_SURF - 1) / C::EPB_SURF;
    int nblk = 0;
    rc = persistent_grid(kern, C::NT, smem, ntiles, &nblk);
    if (rc) return rc;
    kern<<<nblk, C::NT, smem, s>>>(a, g);
    return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
  }
  static size_t split_workspace_bytes(int64_t nelem) {
    return ((size_t)nelem * C::NP * C::FW + (size_t)NS * nelem * C::NP) * sizeof(R) + 256;
  }
  // volume kernel then face kernel (dg_volume.cuh)
  // a.phases: bit 0 the volume stage, bit 1 the face kernel; bit 2 runs the
  // volume stage as the gradient kernel (gradients into a.grad_out) and the
  // flux-volume kernel instead of the fused volume kernel; bit 3 (with bit
  // 2) skips the gradient kernel, a.grad_out holding the gradients already
  template <bool VISC>
  static int vol_face(const DGArgs<R>& a, const GasParams& g, cudaStream_t s) {
    using V = VCfg<R, DIM, ORDER, NS, MIX>;
    const int phases = a.phases;
    int nblk = 0, rc = MGC_OK;
    if ((phases & 1) && (phases & 4)) {
      DGArgs<R> b = a;
      if (VISC) {
        // the gradient kernel writes its gradients to ga.out (bit 3: the
        // caller has computed them)
        if (!(phases & 8)) {
          DGArgs<R> ga = a;
          ga.out = a.grad_out;
          rc = grad_owned(ga, g, s);
          if (rc) return rc;
        }
        b.grad = a.grad_out;
      }
      const size_t smem3 = V::flux_bytes(V::EPB3, a.nperm);
      auto k3 = k_flux_volume<R, DIM, ORDER, NS, MIX, VISC>;
      rc = prepare_kernel(k3, smem3);
      if (rc) return rc;
      rc = persistent_grid(k3, V::NT3, smem3, (a.nowned + V::EPB3 - 1) / V::EPB3, &nblk);
      if (rc) return rc;
      k3<<<nblk, V::NT3, smem3, s>>>(b, g);
      if (cudaGetLastError() != cudaSuccess) return MGC_E_CUDA;
    } else if (phases & 1) {
      const size_t smem1 = V::vol_bytes(V::EPB, a.nperm);
      auto k1 = k_volume<R, DIM, ORDER, NS, MIX, VISC>;
      rc = prepare_kernel(k1, smem1);
      if (rc) return rc;
      rc = persistent_grid(k1, V::NT, smem1, (a.nowned + V::EPB - 1) / V::EPB, &nblk);
      if (rc) return rc;
      k1<<<nblk, V::NT, smem1, s>>>(a, g);
      if (cudaGetLastError() != cudaSuccess) return MGC_E_CUDA;
    }
    if (a.mid_event && cudaEventRecord(static_cast<cudaEvent_t>(a.mid_event), s) != cudaSuccess)
      return MGC_E_CUDA;
    if (phases & 2) {
      const size_t smem2 = V::face_bytes(a.nperm);
      auto k2 = k_face<R, DIM, ORDER, NS, MIX, VISC>;
      rc = prepare_kernel(k2, smem2);
      if (rc) return rc;
      rc = persistent_grid(k2, V::NT2, smem2, (a.nowned + V::EPB2 - 1) / V::EPB2, &nblk);
      if (rc) return rc;
      k2<<<nblk, V::NT2, smem2, s>>>(a, g);
      if (cudaGetLastError() != cudaSuccess) return MGC_E_CUDA;
    }
    return MGC_OK;
  }
  // workspace of vol_face: face-node records, node-0 shifts, boundary
  // records, boundary plus states, each 256-byte aligned
  static size_t vol_workspace_parts(int64_t nelem, int64_t nbf, size_t* off_s0,
                                    size_t* off_btrace, size_t* off_bplus) {
    using V = VCfg<R, DIM, ORDER, NS, MIX>;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t nb = (size_t)(nbf > 0 ? nbf : 1);
    const size_t tr = al((size_t)nelem * V::NFN * V::TW * sizeof(R));
    const size_t s0 = al((size_t)nelem * V::NF * V::NC * sizeof(R));
    const size_t bt = al(nb * V::NFP * V::TW * sizeof(R));
    const size_t bp = al(nb * V::NFP * V::NC * sizeof(R));
    if (off_s0) *off_s0 = tr;
    if (off_btrace) *off_btrace = tr + s0;
    if (off_bplus) *off_bplus = tr + s0 + bt;
    return tr + s0 + bt + bp;
  }
  template <bool VISC>
  static int rhs(const DGArgs<R>& a, const GasParams& g, cudaStream_t s) {
    const size_t smem = C::smem_rhs(a.nperm);
    auto kern = k_rhs<R, DIM, ORDER, NS, MIX, VISC>;
    int rc = prepare_kernel(kern, smem);
    if (rc) return rc;
    const int nblk = (a.nelem + C::EPB_RHS - 1) / C::EPB_RHS;
    kern<<<nblk, C::NT, smem, s>>>(a, g);
    return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
  }
};

// op: 0 = grad, 1 = euler rhs, 2 = ns rhs
template <class R, int DIM, int ORDER>
inline int dispatch_order(int op, int ns, bool mix, const DGArgs<R>& a, const GasParams& g,
                          cudaStream_t s) {
#define MGC_CASE(NSV, MIXV)                                              \
  if (ns == NSV && mix == MIXV) {                                        \
    using L = Launch<R, DIM, ORDER, NSV, MIXV>;                          \
    if (op == 0) return L::grad(a, g, s);                                \
    if (op == 1) return L::template rhs<false>(a, g, s);                 \
    if (op == 2) return L::template rhs<true>(a, g, s);                  \
    if (op == 3) return L::template rhs_split<false>(a, g, s);           \
    if (op == 4) return L::template rhs_split<true>(a, g, s);            \
    if (op == 5) return L::template vol_face<false>(a, g, s);            \
    return L::template vol_face<true>(a, g, s);                          \
  }
  if constexpr (sizeof(R) == 8) {
    MGC_CASE(0, false)
    MGC_CASE(2, false)
    MGC_CASE(7, false)
    MGC_CASE(7, true)
  } else {
    MGC_CASE(0, false)
    MGC_CASE(7, true)
  }
#undef MGC_CASE
  return MGC_E_UNSUPPORTED;
}

template <class R, int DIM, int ORDER>
inline size_t vol_workspace_order(int ns, bool mix, int64_t nelem, int64_t nbf, size_t* off_s0,
                                  size_t* off_bt, size_t* off_bp) {
#define MGC_WS(NSV, MIXV)                                                                  \
  if (ns == NSV && mix == MIXV)                                                            \
    return Launch<R, DIM, ORDER, NSV, MIXV>::vol_workspace_parts(nelem, nbf, off_s0, off_bt,   \
                                                                 off_bp);
  if constexpr (sizeof(R) == 8) {
    MGC_WS(0, false)
    MGC_WS(2, false)
    MGC_WS(7, false)
    MGC_WS(7, true)
  } else {
    MGC_WS(0, false)
    MGC_WS(7, true)
  }
#undef MGC_WS
  return 0;
}

template <class R, int DIM, int ORDER>
inline size_t split_workspace_order(int ns, bool mix, int64_t nelem) {
#define MGC_WS(NSV, MIXV) \
  if (ns == NSV && mix == MIXV) return Launch<R, DIM, ORDER, NSV, MIXV>::split_workspace_bytes(nelem);
  if constexpr (sizeof(R) == 8) {
    MGC_WS(0, false)
    MGC_WS(2, false)
    MGC_WS(7, false)
    MGC_WS(7, true)
  } else {
    MGC_WS(0, false)
    MGC_WS(7, true)
  }
#undef MGC_WS
  return 0;
}

inline bool supported_species(int ns, bool mix) {
  return (ns == 0 && !mix) || (ns == 2 && !mix) || (ns == 7);
}

inline bool supported_species_f32(int ns, bool mix) {
  return (ns == 0 && !mix) || (ns == 7 && mix);
}

template <int DIM>
inline int mixture_state_mixed_dim(int ns, int64_t nnodes, const float* q, const float* tseed,
                                   const float* tguess, float* tout, int32_t* iters, int maxit,
                                   float rtol, int32_t* status, const GasParams& g,
                                   cudaStream_t s) {
  if (ns != 7) return MGC_E_UNSUPPORTED;
  const int nt = 256;
  // grid-stride loop: one wave of resident blocks, so that no second,
  // partly filled wave runs at a fraction of the machine
  auto kern = k_mixture_state_mixed<DIM, 7>;
  int nb = 0;
  const int rc = persistent_grid(kern, nt, 0, (nnodes + nt - 1) / nt, &nb);
  if (rc) return rc;
  kern<<<(unsigned)nb, nt, 0, s>>>(nnodes, q, tseed, tguess, tout, iters, maxit, rtol, status, g);
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

template <class R, int DIM>
inline int mixture_state_dim(int ns, int64_t nnodes, const R* q, const R* tseed, R* t1, R* t2,
                             int32_t* status, const GasParams& g, cudaStream_t s) {
  if (ns != 7) return MGC_E_UNSUPPORTED;
  const int nt = 256;
  auto kern = k_mixture_state<R, DIM, 7>;   // grid-stride: one wave of resident blocks
  int nb = 0;
  const int rc = persistent_grid(kern, nt, 0, (nnodes + nt - 1) / nt, &nb);
  if (rc) return rc;
  kern<<<(unsigned)nb, nt, 0, s>>>(nnodes, q, tseed, t1, t2, status, g);
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

}  // namespace

}  // namespace mgc
