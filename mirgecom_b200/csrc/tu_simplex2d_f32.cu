// Kernel instantiations for 2-D simplices, mixed-precision path (float32
// storage and pointwise math, tf32 x3 tensor-core contractions).
#include "dg_dispatch.cuh"

namespace mgc {

int tu2f_upload_refops(int dim, int order, const double* p64, const float* p32, const int* fn) {
  return upload_refops_local(dim, order, p64, p32, fn);
}

int tu2f_upload_mechanism(const Mechanism* m) { return upload_mechanism_local(m); }

int tu2f_dispatch(int op, int order, int ns, bool mix, const DGArgs<float>& a,
                     const GasParams& g, cudaStream_t s) {
  switch (order) {
    case 1: return dispatch_order<float, 2, 1>(op, ns, mix, a, g, s);
    case 2: return dispatch_order<float, 2, 2>(op, ns, mix, a, g, s);
    case 3: return dispatch_order<float, 2, 3>(op, ns, mix, a, g, s);
    case 4: return dispatch_order<float, 2, 4>(op, ns, mix, a, g, s);
    default: return MGC_E_UNSUPPORTED;
  }
}

int tu2f_mixture_state(int ns, int64_t nnodes, const float* q, const float* tseed,
                          const float* tguess, float* tout, int32_t* iters, int maxit,
                          float rtol, int32_t* status, const GasParams& g, cudaStream_t s) {
  return mixture_state_mixed_dim<2>(ns, nnodes, q, tseed, tguess, tout, iters, maxit, rtol,
                                       status, g, s);
}

size_t tu2f_split_workspace(int order, int ns, bool mix, int64_t nelem) {
  switch (order) {
    case 1: return split_workspace_order<float, 2, 1>(ns, mix, nelem);
    case 2: return split_workspace_order<float, 2, 2>(ns, mix, nelem);
    case 3: return split_workspace_order<float, 2, 3>(ns, mix, nelem);
    case 4: return split_workspace_order<float, 2, 4>(ns, mix, nelem);
    default: return 0;
  }
}

size_t tu2f_vol_workspace(int order, int ns, bool mix, int64_t nelem, int64_t nbf,
                          size_t* off_s0, size_t* off_bt, size_t* off_bp) {
  switch (order) {
    case 1: return vol_workspace_order<float, 2, 1>(ns, mix, nelem, nbf, off_s0, off_bt, off_bp);
    case 2: return vol_workspace_order<float, 2, 2>(ns, mix, nelem, nbf, off_s0, off_bt, off_bp);
    case 3: return vol_workspace_order<float, 2, 3>(ns, mix, nelem, nbf, off_s0, off_bt, off_bp);
    case 4: return vol_workspace_order<float, 2, 4>(ns, mix, nelem, nbf, off_s0, off_bt, off_bp);
    default: return 0;
  }
}

}  // namespace mgc
