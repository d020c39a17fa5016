// Kernel instantiations for 3-D tensor-product hexahedra (float32).
#include "dg_dispatch.cuh"
#include "hex_kernels.cuh"

namespace mgc {

int tuhf_upload_hexops(const double* packed) { return upload_hexops_local(packed); }

int tuhf_dispatch(int op, int order, int ns, bool mix, const DGArgs<float>& a,
                 const GasParams& g, cudaStream_t s) {
  return hex_dispatch<float>(op, order, ns, mix, a, g, s);
}

size_t tuhf_split_workspace(int order, int ns, bool mix, int64_t nelem) {
  return hex_split_workspace<float>(order, ns, mix, nelem);
}

}  // namespace mgc
