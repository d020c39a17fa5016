// Navier-Stokes right-hand side for callers that must not allocate device
// memory.
//
// The full NS operator needs one scratch buffer between its two passes: the
// gradients of the conserved variables and of the temperature
// ([Nc+1][dim][E][Np] doubles).  The regular entry points take that buffer
// from the caller.  Some callers cannot provide it: a solver whose device
// memory is owned by its own pool allocator and that forbids driver
// allocations once a run has started, or a host code that links this
// library without any CUDA allocation layer of its own.  For them this file
// keeps the scratch in a fixed, file-scope device array and exposes one
// entry point that allocates nothing.
//
// Costs and limits:
//   * every GPU that loads the library holds kNoAllocScratchDoubles doubles
//     (32 MiB) until the process exits;
//   * meshes whose gradient buffer would not fit are rejected with
//     MGC_E_TOO_LARGE (e.g. at most 11,650 order-3 tetrahedra of a
//     single-species gas, or 5,377 for the 7-species mixture);
//   * all calls share the one array: calls that overlap on the GPU (two
//     streams, two host threads) race on it and must be serialised by the
//     caller.  Nothing in the array needs clearing between calls: the
//     gradient pass writes every entry the divergence pass reads.
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before capturing any stream.  The address is kept for the life of the
//     process: it does not survive cudaDeviceReset (or any other teardown of
//     the device's primary context), after which this entry point must not
//     be called again in that process.
#include <cuda_runtime.h>

#include <atomic>

#include "dg_refops.cuh"
#include "../../include/mgc_b200.h"

namespace {

constexpr size_t kNoAllocScratchDoubles = size_t(4) << 20;   // 32 MiB of float64
constexpr int kMaxDevices = 64;
// highest simplex order with device kernels (2-D); bounds the node count
// before the size check
constexpr int kNoAllocMaxOrder = 4;

static __device__ __align__(256) double g_noalloc_grad[kNoAllocScratchDoubles];

// host-side record of the array's device address, per device.  Two host
// threads making their first call on one device at once may both look the
// address up; they store the same value, and the atomics make that benign.
std::atomic<double*> g_noalloc_ptr[kMaxDevices] = {};

int noalloc_scratch(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MGC_E_CUDA;
  double* p = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    void* sym = nullptr;
    if (cudaGetSymbolAddress(&sym, g_noalloc_grad) != cudaSuccess || !sym) return MGC_E_CUDA;
    p = static_cast<double*>(sym);
    g_noalloc_ptr[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return MGC_OK;
}

}  // namespace

extern "C" {

size_t mgc_ns_operator_noalloc_capacity(void) { return kNoAllocScratchDoubles; }

int mgc_ns_operator_noalloc(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                            const double* t_op, const double* t_src, const double* bext,
                            int flux_kind, int add_sources, double* rhs, int32_t* status,
                            void* stream) {
  if (!mesh || !gas || mesh->nelem <= 0 || gas->nspecies < 0 ||
      gas->nspecies > MGC_MAX_SPECIES || (mesh->dim != 2 && mesh->dim != 3))
    return MGC_E_INVALID;
  // an element kind that is neither is an invalid mesh (as for mgc_ns_rhs)
  if (mesh->elem_kind != MGC_ELEM_SIMPLEX && mesh->elem_kind != MGC_ELEM_HEX)
    return MGC_E_INVALID;
  // simplicial meshes only: hexahedra have no fused divergence pass; orders
  // without device kernels are unsupported (and bounding the order here
  // keeps the node count below from overflowing)
  if (mesh->elem_kind != MGC_ELEM_SIMPLEX) return MGC_E_UNSUPPORTED;
  if (mesh->order < 1 || mesh->order > kNoAllocMaxOrder) return MGC_E_UNSUPPORTED;
  const size_t np = (size_t)mgc::simplex_npts(mesh->dim, mesh->order);
  const size_t nc = (size_t)(mesh->dim + 2 + gas->nspecies);
  const size_t need = (nc + 1) * (size_t)mesh->dim * (size_t)mesh->nelem * np;
  if (need > kNoAllocScratchDoubles) return MGC_E_TOO_LARGE;
  double* grad = nullptr;
  int rc = noalloc_scratch(&grad);
  if (rc) return rc;
  rc = mgc_ns_grad(mesh, gas, q, t_op, bext, grad, status, stream);
  if (rc) return rc;
  return mgc_ns_rhs(mesh, gas, q, t_op, t_src, grad, bext, flux_kind, add_sources, rhs, status,
                    stream);
}

}  // extern "C"
