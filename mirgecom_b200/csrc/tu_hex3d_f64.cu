// Kernel instantiations for 3-D tensor-product hexahedra (float64).
#include "dg_dispatch.cuh"
#include "hex_kernels.cuh"

namespace mgc {

int tuh_upload_hexops(const double* packed) { return upload_hexops_local(packed); }

int tuh_dispatch(int op, int order, int ns, bool mix, const DGArgs<double>& a,
                 const GasParams& g, cudaStream_t s) {
  return hex_dispatch<double>(op, order, ns, mix, a, g, s);
}

size_t tuh_split_workspace(int order, int ns, bool mix, int64_t nelem) {
  return hex_split_workspace<double>(order, ns, mix, nelem);
}

}  // namespace mgc
