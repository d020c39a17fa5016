// extern "C" entry points of libmgc_b200 (declared in include/mgc_b200.h).
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <vector>

#include "dg_dispatch.cuh"
#include "hex_kernels.cuh"

namespace mgc {
int tu2_upload_refops(int, int, const double*, const float*, const int*);
int tu3_upload_refops(int, int, const double*, const float*, const int*);
int tu2_upload_mechanism(const Mechanism*);
int tu3_upload_mechanism(const Mechanism*);
int tu2_dispatch(int, int, int, bool, const DGArgs<double>&, const GasParams&, cudaStream_t);
int tu3_dispatch(int, int, int, bool, const DGArgs<double>&, const GasParams&, cudaStream_t);
int tu2_mixture_state(int, int64_t, const double*, const double*, double*, double*,
                      int32_t*, const GasParams&, cudaStream_t);
int tu2f_upload_refops(int, int, const double*, const float*, const int*);
int tu3f_upload_refops(int, int, const double*, const float*, const int*);
int tu2f_upload_mechanism(const Mechanism*);
int tu3f_upload_mechanism(const Mechanism*);
int mlp_upload_mechanism(const Mechanism*);
int tu2f_dispatch(int, int, int, bool, const DGArgs<float>&, const GasParams&, cudaStream_t);
int tu3f_dispatch(int, int, int, bool, const DGArgs<float>&, const GasParams&, cudaStream_t);
int tu2f_mixture_state(int, int64_t, const float*, const float*, const float*, float*, int32_t*,
                       int, float, int32_t*, const GasParams&, cudaStream_t);
int tu3f_mixture_state(int, int64_t, const float*, const float*, const float*, float*, int32_t*,
                       int, float, int32_t*, const GasParams&, cudaStream_t);
int tu3_mixture_state(int, int64_t, const double*, const double*, double*, double*,
                      int32_t*, const GasParams&, cudaStream_t);
size_t tu2_split_workspace(int, int, bool, int64_t);
size_t tu3_split_workspace(int, int, bool, int64_t);
size_t tu2f_split_workspace(int, int, bool, int64_t);
size_t tu3f_split_workspace(int, int, bool, int64_t);
size_t tu2_vol_workspace(int, int, bool, int64_t, int64_t, size_t*, size_t*, size_t*);
size_t tu3_vol_workspace(int, int, bool, int64_t, int64_t, size_t*, size_t*, size_t*);
size_t tu2f_vol_workspace(int, int, bool, int64_t, int64_t, size_t*, size_t*, size_t*);
size_t tu3f_vol_workspace(int, int, bool, int64_t, int64_t, size_t*, size_t*, size_t*);
int tuh_upload_hexops(const double*);
int tuhf_upload_hexops(const double*);
int tuh_dispatch(int, int, int, bool, const DGArgs<double>&, const GasParams&, cudaStream_t);
int tuhf_dispatch(int, int, int, bool, const DGArgs<float>&, const GasParams&, cudaStream_t);
size_t tuh_split_workspace(int, int, bool, int64_t);
size_t tuhf_split_workspace(int, int, bool, int64_t);
}  // namespace mgc

using namespace mgc;

namespace {

// per-device record of which reference operators / mechanism were uploaded
constexpr int kMaxDevices = 64;
bool g_refops_ready[kMaxDevices][8] = {};
bool g_hexops_ready[kMaxDevices][8] = {};
bool g_mech_ready[kMaxDevices] = {};

// 1-D operators of the tensor-product hexahedra uploaded so far (host copy
// of the packed constant block; each upload adds one order)
constexpr int kHexPacked = 200;
double g_hexops_host[kHexPacked] = {};

constexpr int kElemSimplex = 0, kElemHex = 1;

int mesh_npts(const mgc_mesh_t* m) {
  return m->elem_kind == kElemHex ? (m->order + 1) * (m->order + 1) * (m->order + 1)
                                  : simplex_npts(m->dim, m->order);
}

int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) return -1;
  return d;
}

bool mesh_ok(const mgc_mesh_t* m) {
  return m && (m->dim == 2 || m->dim == 3) && m->nelem > 0 && m->rx && m->conn &&
         (m->elem_kind == kElemSimplex || (m->elem_kind == kElemHex && m->dim == 3)) &&
         m->nperm > 0 && m->nperm <= 256 && m->perm && m->nbf >= 0 &&
         (m->nbf == 0 || m->bkind) && (int64_t)m->nelem * 256 < (int64_t)1 << 31;
}

bool gas_ok(const mgc_gas_t* g) {
  return g && (g->eos_kind == MGC_EOS_IDEAL || g->eos_kind == MGC_EOS_MIXTURE) &&
         g->nspecies >= 0 && g->nspecies <= MGC_MAX_SPECIES && g->niter >= 0;
}

int ready(const mgc_mesh_t* m, const mgc_gas_t* g) {
  const int dev = current_device();
  if (dev < 0) return MGC_E_CUDA;
  if (m->elem_kind == kElemHex) {
    if (m->order < 1 || m->order > kHexMaxOrder) return MGC_E_UNSUPPORTED;
    if (!g_hexops_ready[dev][m->order]) return MGC_E_NOT_READY;
  } else {
    const int slot = refops_slot(m->dim, m->order);
    if (slot < 0) return MGC_E_UNSUPPORTED;
    if (!g_refops_ready[dev][slot]) return MGC_E_NOT_READY;
  }
  if (g->eos_kind == MGC_EOS_MIXTURE && !g_mech_ready[dev]) return MGC_E_NOT_READY;
  return MGC_OK;
}

// gradient-pass kernel choice (mgc_set_gradient_kernel), process-wide
std::atomic<int> g_grad_kernel{MGC_GRAD_AUTO};

template <class R>
DGArgs<R> make_args(const mgc_mesh_t* m, const R* q, const R* t_op, const R* t_src,
                    const R* grad, R* out, const R* bext, int flux_kind, int add_sources,
                    int32_t* status) {
  DGArgs<R> a;
  std::memset(&a, 0, sizeof(a));
  a.nelem = m->nelem;
  a.nbf = m->nbf;
  a.nperm = m->nperm;
  a.flux_kind = flux_kind;
  a.q = q;
  a.t_op = t_op;
  a.t_src = t_src;
  a.grad = grad;
  a.out = out;
  if constexpr (sizeof(R) == 8) {
    a.rx = m->rx;
  } else {
    a.rx = m->rx32;
  }
  a.conn = m->conn;
  a.perm = m->perm;
  a.bkind = m->bkind;
  a.bext = bext;
  a.status = status;
  a.add_sources = add_sources;
  a.grad_kernel = g_grad_kernel.load(std::memory_order_relaxed) == MGC_GRAD_MMA_SYNC ? 1 : 0;
  return a;
}

GasParams to_params(const mgc_gas_t* g) {
  GasParams p;
  std::memcpy(&p, g, sizeof(p));
  return p;
}

int dispatch(int op, const mgc_mesh_t* m, const mgc_gas_t* g, const DGArgs<double>& a,
             cudaStream_t s) {
  const bool mix = g->eos_kind == MGC_EOS_MIXTURE;
  if (!supported_species(g->nspecies, mix)) return MGC_E_UNSUPPORTED;
  const GasParams p = to_params(g);
  if (m->elem_kind == kElemHex) return tuh_dispatch(op, m->order, g->nspecies, mix, a, p, s);
  if (m->dim == 2) return tu2_dispatch(op, m->order, g->nspecies, mix, a, p, s);
  return tu3_dispatch(op, m->order, g->nspecies, mix, a, p, s);
}

int dispatch(int op, const mgc_mesh_t* m, const mgc_gas_t* g, const DGArgs<float>& a,
             cudaStream_t s) {
  const bool mix = g->eos_kind == MGC_EOS_MIXTURE;
  if (!supported_species_f32(g->nspecies, mix)) return MGC_E_UNSUPPORTED;
  if (!m->rx32) return MGC_E_INVALID;
  const GasParams p = to_params(g);
  if (m->elem_kind == kElemHex) return tuhf_dispatch(op, m->order, g->nspecies, mix, a, p, s);
  if (m->dim == 2) return tu2f_dispatch(op, m->order, g->nspecies, mix, a, p, s);
  return tu3f_dispatch(op, m->order, g->nspecies, mix, a, p, s);
}

template <class R>
int euler_rhs_impl(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const R* q, const R* t_op,
                   const R* bext, int flux_kind, R* rhs, int32_t* status, void* stream) {
  if (!mesh_ok(mesh) || !gas_ok(gas) || !q || !rhs || !status) return MGC_E_INVALID;
  if (flux_kind < 0 || flux_kind > 2) return MGC_E_INVALID;
  if (gas->eos_kind == MGC_EOS_MIXTURE && !t_op) return MGC_E_INVALID;
  int rc = ready(mesh, gas);
  if (rc) return rc;
  const DGArgs<R> a =
      make_args<R>(mesh, q, t_op, nullptr, nullptr, rhs, bext, flux_kind, 0, status);
  return dispatch(1, mesh, gas, a, (cudaStream_t)stream);
}

template <class R>
int ns_grad_impl(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const R* q, const R* t_op,
                 const R* bext, R* grad, int32_t* status, void* stream) {
  if (!mesh_ok(mesh) || !gas_ok(gas) || !q || !grad || !status) return MGC_E_INVALID;
  if (gas->eos_kind == MGC_EOS_MIXTURE && !t_op) return MGC_E_INVALID;
  int rc = ready(mesh, gas);
  if (rc) return rc;
  const DGArgs<R> a = make_args<R>(mesh, q, t_op, nullptr, nullptr, grad, bext, 0, 0, status);
  return dispatch(0, mesh, gas, a, (cudaStream_t)stream);
}

template <class R>
int ns_rhs_impl(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const R* q, const R* t_op,
                const R* t_src, const R* grad, const R* bext, int flux_kind, int add_sources,
                R* rhs, int32_t* status, void* stream) {
  if (!mesh_ok(mesh) || !gas_ok(gas) || !q || !grad || !rhs || !status) return MGC_E_INVALID;
  if (flux_kind < 0 || flux_kind > 2) return MGC_E_INVALID;
  if (gas->eos_kind == MGC_EOS_MIXTURE && !t_op) return MGC_E_INVALID;
  if (add_sources && (gas->eos_kind != MGC_EOS_MIXTURE || !t_src)) return MGC_E_INVALID;
  int rc = ready(mesh, gas);
  if (rc) return rc;
  const DGArgs<R> a =
      make_args<R>(mesh, q, t_op, t_src, grad, rhs, bext, flux_kind, add_sources, status);
  return dispatch(2, mesh, gas, a, (cudaStream_t)stream);
}

template <class R>
size_t split_ws(const mgc_mesh_t* m, const mgc_gas_t* g) {
  const bool mix = g->eos_kind == MGC_EOS_MIXTURE;
  if (m->elem_kind == kElemHex)
    return sizeof(R) == 8 ? tuh_split_workspace(m->order, g->nspecies, mix, m->nelem)
                          : tuhf_split_workspace(m->order, g->nspecies, mix, m->nelem);
  if constexpr (sizeof(R) == 8)
    return m->dim == 2 ? tu2_split_workspace(m->order, g->nspecies, mix, m->nelem)
                       : tu3_split_workspace(m->order, g->nspecies, mix, m->nelem);
  return m->dim == 2 ? tu2f_split_workspace(m->order, g->nspecies, mix, m->nelem)
                     : tu3f_split_workspace(m->order, g->nspecies, mix, m->nelem);
}

template <class R>
int rhs_split_impl(int visc, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const R* q,
                   const R* t_op, const R* t_src, const R* grad, const R* bext, int flux_kind,
                   int add_sources, R* rhs, void* workspace, size_t workspace_bytes,
                   int32_t* status, void* stream, void* mid_event) {
  if (!mesh_ok(mesh) || !gas_ok(gas) || !q || !rhs || !status || !workspace)
    return MGC_E_INVALID;
  if (visc && !grad) return MGC_E_INVALID;
  if (flux_kind < 0 || flux_kind > 2) return MGC_E_INVALID;
  if (gas->eos_kind == MGC_EOS_MIXTURE && !t_op) return MGC_E_INVALID;
  if (add_sources && (gas->eos_kind != MGC_EOS_MIXTURE || !t_src)) return MGC_E_INVALID;
  if (reinterpret_cast<uintptr_t>(workspace) % 16) return MGC_E_INVALID;
  int rc = ready(mesh, gas);
  if (rc) return rc;
  const size_t need = split_ws<R>(mesh, gas);
  if (need == 0) return MGC_E_UNSUPPORTED;
  if (workspace_bytes < need) return MGC_E_INVALID;
  DGArgs<R> a = make_args<R>(mesh, q, t_op, t_src, grad, rhs, bext, flux_kind, add_sources,
                             status);
  a.fbuf = static_cast<R*>(workspace);
  a.mid_event = mid_event;
  // sources after the flux records, 16-byte aligned
  const size_t rec_bytes =
      need - 256 - (size_t)gas->nspecies * mesh->nelem * mesh_npts(mesh) * sizeof(R);
  a.srcbuf = reinterpret_cast<R*>(static_cast<char*>(workspace) + ((rec_bytes + 15) / 16) * 16);
  return dispatch(visc ? 4 : 3, mesh, gas, a, (cudaStream_t)stream);
}

template <class R>
size_t vol_ws(const mgc_mesh_t* m, const mgc_gas_t* g, size_t* off_s0, size_t* off_bt,
              size_t* off_bp) {
  if (m->elem_kind != kElemSimplex) return 0;
  const bool mix = g->eos_kind == MGC_EOS_MIXTURE;
  if constexpr (sizeof(R) == 8)
    return m->dim == 2 ? tu2_vol_workspace(m->order, g->nspecies, mix, m->nelem, m->nbf, off_s0, off_bt, off_bp)
                       : tu3_vol_workspace(m->order, g->nspecies, mix, m->nelem, m->nbf, off_s0, off_bt, off_bp);
  return m->dim == 2 ? tu2f_vol_workspace(m->order, g->nspecies, mix, m->nelem, m->nbf, off_s0, off_bt, off_bp)
                     : tu3f_vol_workspace(m->order, g->nspecies, mix, m->nelem, m->nbf, off_s0, off_bt, off_bp);
}

template <class R>
int operator_impl(int visc, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const R* q,
                  const R* t_op, const R* t_src, const R* bext, int flux_kind, int add_sources,
                  R* rhs, R* grad_out, void* workspace, size_t workspace_bytes, int32_t* status,
                  void* stream, void* mid_event, int phases) {
  if (phases < 1 || phases > 15 || (phases & 3) == 0) return MGC_E_INVALID;
  if ((phases & 8) && !(phases & 4)) return MGC_E_INVALID;
  if ((phases & 4) && (phases & 1) && visc && !grad_out) return MGC_E_INVALID;
  if (!mesh_ok(mesh) || !gas_ok(gas) || !q || !rhs || !status || !workspace)
    return MGC_E_INVALID;
  if (flux_kind < 0 || flux_kind > 2) return MGC_E_INVALID;
  if (gas->eos_kind == MGC_EOS_MIXTURE && !t_op) return MGC_E_INVALID;
  if (add_sources && (gas->eos_kind != MGC_EOS_MIXTURE || !t_src)) return MGC_E_INVALID;
  if (grad_out && !visc) return MGC_E_INVALID;
  if (mesh->elem_kind != kElemSimplex) return MGC_E_UNSUPPORTED;
  if (!mesh->fslot) return MGC_E_INVALID;
  if (mesh->nowned < 0 || mesh->nowned > mesh->nelem) return MGC_E_INVALID;
  if (reinterpret_cast<uintptr_t>(workspace) % 256) return MGC_E_INVALID;
  int rc = ready(mesh, gas);
  if (rc) return rc;
  size_t off_s0 = 0, off_bt = 0, off_bp = 0;
  const size_t need = vol_ws<R>(mesh, gas, &off_s0, &off_bt, &off_bp);
  if (need == 0) return MGC_E_UNSUPPORTED;
  if (workspace_bytes < need) return MGC_E_INVALID;
  DGArgs<R> a = make_args<R>(mesh, q, t_op, t_src, nullptr, rhs, bext, flux_kind, add_sources,
                             status);
  char* ws = static_cast<char*>(workspace);
  a.trace = reinterpret_cast<R*>(ws);
  a.s0 = reinterpret_cast<R*>(ws + off_s0);
  a.btrace = reinterpret_cast<R*>(ws + off_bt);
  a.bplus = reinterpret_cast<R*>(ws + off_bp);
  a.fslot = mesh->fslot;
  a.grad_out = grad_out;
  a.mid_event = mid_event;
  a.nowned = mesh->nowned > 0 ? mesh->nowned : mesh->nelem;
  a.phases = phases;
  return dispatch(visc ? 6 : 5, mesh, gas, a, (cudaStream_t)stream);
}

}  // namespace

extern "C" {

int mgc_set_gradient_kernel(int kind) {
  if (kind != MGC_GRAD_AUTO && kind != MGC_GRAD_MMA_SYNC) return MGC_E_INVALID;
  g_grad_kernel.store(kind);
  return MGC_OK;
}

int mgc_get_gradient_kernel(void) { return g_grad_kernel.load(); }

size_t mgc_operator_workspace_bytes(const mgc_mesh_t* mesh, const mgc_gas_t* gas,
                                    int single_precision) {
  if (!mesh_ok(mesh) || !gas_ok(gas)) return 0;
  return single_precision ? vol_ws<float>(mesh, gas, nullptr, nullptr, nullptr)
                          : vol_ws<double>(mesh, gas, nullptr, nullptr, nullptr);
}

int mgc_operator(int viscous, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                 const double* t_op, const double* t_src, const double* bext, int flux_kind,
                 int add_sources, double* rhs, double* grad_out, void* workspace,
                 size_t workspace_bytes, int32_t* status, void* stream, void* mid_event,
                 int phases) {
  return operator_impl<double>(viscous, mesh, gas, q, t_op, t_src, bext, flux_kind, add_sources,
                               rhs, grad_out, workspace, workspace_bytes, status, stream,
                               mid_event, phases);
}

int mgc_operator_f32(int viscous, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                     const float* t_op, const float* t_src, const float* bext, int flux_kind,
                     int add_sources, float* rhs, float* grad_out, void* workspace,
                     size_t workspace_bytes, int32_t* status, void* stream, void* mid_event,
                     int phases) {
  return operator_impl<float>(viscous, mesh, gas, q, t_op, t_src, bext, flux_kind, add_sources,
                              rhs, grad_out, workspace, workspace_bytes, status, stream,
                              mid_event, phases);
}

size_t mgc_rhs_split_workspace_bytes(const mgc_mesh_t* mesh, const mgc_gas_t* gas,
                                     int single_precision) {
  if (!mesh_ok(mesh) || !gas_ok(gas)) return 0;
  return single_precision ? split_ws<float>(mesh, gas) : split_ws<double>(mesh, gas);
}

int mgc_rhs_split(int viscous, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                  const double* t_op, const double* t_src, const double* grad,
                  const double* bext, int flux_kind, int add_sources, double* rhs,
                  void* workspace, size_t workspace_bytes, int32_t* status, void* stream,
                  void* mid_event) {
  return rhs_split_impl<double>(viscous, mesh, gas, q, t_op, t_src, grad, bext, flux_kind,
                                add_sources, rhs, workspace, workspace_bytes, status, stream,
                                mid_event);
}

int mgc_rhs_split_f32(int viscous, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                      const float* t_op, const float* t_src, const float* grad,
                      const float* bext, int flux_kind, int add_sources, float* rhs,
                      void* workspace, size_t workspace_bytes, int32_t* status, void* stream,
                      void* mid_event) {
  return rhs_split_impl<float>(viscous, mesh, gas, q, t_op, t_src, grad, bext, flux_kind,
                               add_sources, rhs, workspace, workspace_bytes, status, stream,
                               mid_event);
}


int mgc_version(void) { return 1; }

int mgc_supports(int dim, int order, int nspecies, int eos_kind) {
  if (refops_slot(dim, order) < 0) return 0;
  return supported_species(nspecies, eos_kind == MGC_EOS_MIXTURE) ? 1 : 0;
}

int mgc_supports_hex(int dim, int order, int nspecies, int eos_kind) {
  return (dim == 3 && order >= 1 && order <= kHexMaxOrder && nspecies == 0 &&
          eos_kind == MGC_EOS_IDEAL) ? 1 : 0;
}

int mgc_upload_hex_operators(int dim, int order, const double* weak1d_host,
                             const double* lift1d_host, double face_scale_ref) {
  if (dim != 3 || order < 1 || order > kHexMaxOrder) return MGC_E_UNSUPPORTED;
  if (!weak1d_host || !lift1d_host || !(face_scale_ref > 0.0)) return MGC_E_INVALID;
  static_assert(kHexOpsTotal <= kHexPacked, "hex operator block");
  const int n1 = order + 1;
  double* p = g_hexops_host + hexops_offset(order);
  for (int i = 0; i < n1 * n1; ++i) p[i] = weak1d_host[i];
  for (int i = 0; i < 2 * n1; ++i) p[n1 * n1 + i] = lift1d_host[i];
  p[n1 * n1 + 2 * n1] = face_scale_ref;
  int rc = tuh_upload_hexops(g_hexops_host);
  if (rc) return rc;
  rc = tuhf_upload_hexops(g_hexops_host);
  if (rc) return rc;
  const int dev = current_device();
  if (dev < 0) return MGC_E_CUDA;
  g_hexops_ready[dev][order] = true;
  return MGC_OK;
}

int mgc_upload_reference_operators(int dim, int order, const double* weak_host,
                                   const double* lift_host, const double* ref_normals_host,
                                   const double* face_scale_ref_host,
                                   const int32_t* face_nodes_host) {
  const int slot = refops_slot(dim, order);
  if (slot < 0) return MGC_E_UNSUPPORTED;
  if (!weak_host || !lift_host || !ref_normals_host || !face_scale_ref_host || !face_nodes_host)
    return MGC_E_INVALID;
  const int np = simplex_npts(dim, order);
  const int nf = dim + 1;
  const int nfp = simplex_npts(dim - 1, order);
  const int n = refops_size(dim, order);
  std::vector<double> p64(n);
  int o = 0;
  for (int i = 0; i < dim * np * np; ++i) p64[o++] = weak_host[i];
  for (int i = 0; i < np * nf * nfp; ++i) p64[o++] = lift_host[i];
  for (int i = 0; i < nf * dim; ++i) p64[o++] = ref_normals_host[i];
  for (int i = 0; i < nf; ++i) p64[o++] = face_scale_ref_host[i];
  std::vector<float> p32(n);
  for (int i = 0; i < n; ++i) p32[i] = (float)p64[i];
  std::vector<int> fn(nf * nfp);
  for (int i = 0; i < nf * nfp; ++i) {
    if (face_nodes_host[i] < 0 || face_nodes_host[i] >= np) return MGC_E_INVALID;
    fn[i] = face_nodes_host[i];
  }
  int rc = tu2_upload_refops(dim, order, p64.data(), p32.data(), fn.data());
  if (rc) return rc;
  rc = tu3_upload_refops(dim, order, p64.data(), p32.data(), fn.data());
  if (rc) return rc;
  rc = tu2f_upload_refops(dim, order, p64.data(), p32.data(), fn.data());
  if (rc) return rc;
  rc = tu3f_upload_refops(dim, order, p64.data(), p32.data(), fn.data());
  if (rc) return rc;
  rc = upload_refops_local(dim, order, p64.data(), p32.data(), fn.data());
  if (rc) return rc;
  const int dev = current_device();
  if (dev < 0) return MGC_E_CUDA;
  g_refops_ready[dev][slot] = true;
  return MGC_OK;
}

int mgc_set_mechanism(const mgc_mechanism_t* mech_host) {
  if (!mech_host || mech_host->nspecies < 1 || mech_host->nspecies > MGC_MAX_SPECIES ||
      mech_host->nreactions < 0 || mech_host->nreactions > MGC_MAX_REACTIONS)
    return MGC_E_INVALID;
  const Mechanism m = expand_mechanism(*mech_host);
  int rc = tu2_upload_mechanism(&m);
  if (rc) return rc;
  rc = tu3_upload_mechanism(&m);
  if (rc) return rc;
  rc = tu2f_upload_mechanism(&m);
  if (rc) return rc;
  rc = tu3f_upload_mechanism(&m);
  if (rc) return rc;
  rc = mlp_upload_mechanism(&m);
  if (rc) return rc;
  rc = upload_mechanism_local(&m);
  if (rc) return rc;
  const int dev = current_device();
  if (dev < 0) return MGC_E_CUDA;
  g_mech_ready[dev] = true;
  return MGC_OK;
}

int mgc_mixture_temperature(int dim, const mgc_gas_t* gas, int64_t nnodes, const double* q,
                            const double* t_seed, double* t1, double* t2, int32_t* status,
                            void* stream) {
  if (!gas_ok(gas) || gas->eos_kind != MGC_EOS_MIXTURE || nnodes < 0 || !q || !t_seed || !t1)
    return MGC_E_INVALID;
  if (nnodes == 0) return MGC_OK;
  const int dev = current_device();
  if (dev < 0) return MGC_E_CUDA;
  if (!g_mech_ready[dev]) return MGC_E_NOT_READY;
  const GasParams p = to_params(gas);
  cudaStream_t s = (cudaStream_t)stream;
  if (dim == 2) return tu2_mixture_state(gas->nspecies, nnodes, q, t_seed, t1, t2, status, p, s);
  if (dim == 3) return tu3_mixture_state(gas->nspecies, nnodes, q, t_seed, t1, t2, status, p, s);
  return MGC_E_UNSUPPORTED;
}

int mgc_euler_rhs(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                  const double* t_op, const double* bext, int flux_kind, double* rhs,
                  int32_t* status, void* stream) {
  return euler_rhs_impl<double>(mesh, gas, q, t_op, bext, flux_kind, rhs, status, stream);
}

int mgc_euler_rhs_f32(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                      const float* t_op, const float* bext, int flux_kind, float* rhs,
                      int32_t* status, void* stream) {
  return euler_rhs_impl<float>(mesh, gas, q, t_op, bext, flux_kind, rhs, status, stream);
}

int mgc_ns_grad(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                const double* t_op, const double* bext, double* grad, int32_t* status,
                void* stream) {
  return ns_grad_impl<double>(mesh, gas, q, t_op, bext, grad, status, stream);
}

int mgc_ns_grad_f32(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                    const float* t_op, const float* bext, float* grad, int32_t* status,
                    void* stream) {
  return ns_grad_impl<float>(mesh, gas, q, t_op, bext, grad, status, stream);
}

int mgc_ns_rhs(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
               const double* t_op, const double* t_src, const double* grad,
               const double* bext, int flux_kind, int add_sources, double* rhs,
               int32_t* status, void* stream) {
  return ns_rhs_impl<double>(mesh, gas, q, t_op, t_src, grad, bext, flux_kind, add_sources,
                             rhs, status, stream);
}

int mgc_ns_rhs_f32(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                   const float* t_op, const float* t_src, const float* grad,
                   const float* bext, int flux_kind, int add_sources, float* rhs,
                   int32_t* status, void* stream) {
  return ns_rhs_impl<float>(mesh, gas, q, t_op, t_src, grad, bext, flux_kind, add_sources, rhs,
                            status, stream);
}

int mgc_mixture_temperature_f32(int dim, const mgc_gas_t* gas, int64_t nnodes, const float* q,
                                const float* t_seed, const float* t_guess, float* t_out,
                                int32_t* iters, int maxit, float rtol, int32_t* status,
                                void* stream) {
  if (!gas_ok(gas) || gas->eos_kind != MGC_EOS_MIXTURE || nnodes < 0 || !q || !t_seed ||
      !t_out || !status || maxit < 1 || maxit > 100 || !(rtol > 0.f))
    return MGC_E_INVALID;
  if (nnodes == 0) return MGC_OK;
  const int dev = current_device();
  if (dev < 0) return MGC_E_CUDA;
  if (!g_mech_ready[dev]) return MGC_E_NOT_READY;
  const GasParams p = to_params(gas);
  cudaStream_t s = (cudaStream_t)stream;
  if (dim == 2)
    return tu2f_mixture_state(gas->nspecies, nnodes, q, t_seed, t_guess, t_out, iters, maxit,
                              rtol, status, p, s);
  if (dim == 3)
    return tu3f_mixture_state(gas->nspecies, nnodes, q, t_seed, t_guess, t_out, iters, maxit,
                              rtol, status, p, s);
  return MGC_E_UNSUPPORTED;
}

int mgc_rk4_stage_mixed(int64_t n, const double* q0, const float* k, double* sum,
                        double* q_out, float* q_out_lo, int stage, double dt, void* stream) {
  if (n < 0 || !q0 || !k || !sum || !q_out || !q_out_lo || stage < 0 || stage > 3)
    return MGC_E_INVALID;
  if (n == 0) return MGC_OK;
  const int nt = 256;
  int64_t nb = (n + nt - 1) / nt;
  if (nb > 148 * 32) nb = 148 * 32;
  k_rk4_stage_mixed<<<(unsigned)nb, nt, 0, (cudaStream_t)stream>>>(n, q0, k, sum, q_out,
                                                                   q_out_lo, stage, dt);
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

int mgc_rk4_stage(int64_t n, const double* q0, const double* k, double* sum, double* q_out,
                  float* q_out_lo, int stage, double dt, void* stream) {
  if (n < 0 || !q0 || !k || !sum || !q_out || stage < 0 || stage > 3) return MGC_E_INVALID;
  if (n == 0) return MGC_OK;
  const int nt = 256;
  int64_t nb = (n + nt - 1) / nt;
  if (nb > 148 * 32) nb = 148 * 32;
  k_rk4_stage<float><<<(unsigned)nb, nt, 0, (cudaStream_t)stream>>>(n, q0, k, sum, q_out,
                                                                    q_out_lo, stage, dt);
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

}  // extern "C"
