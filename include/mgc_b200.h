/*
 * mgc_b200.h -- C ABI of the B200 DG compressible Euler / Navier-Stokes
 * right-hand side.
 *
 * All array pointers are DEVICE pointers (CUDA global memory) unless the
 * parameter name ends in _host.  Streams are passed as `void*` (a
 * cudaStream_t, NULL for the legacy default stream).  Every call is
 * stream-ordered and asynchronous; none allocates device memory except where
 * noted.  Return value: 0 on success, a negative MGC_E* code for invalid
 * arguments or an unsupported configuration; problems found on the device
 * (NaN, corrupt index, ...) are OR-ed into the caller's `status` word as
 * MGC_ST* bits and never trap.
 *
 * Array layouts (E elements, Np nodes per element, Nc = dim + 2 + nspecies):
 *   q, rhs        [Nc][E][Np]  float64, field order of ConservedVars:
 *                 mass, energy, momentum[dim], species_mass[nspecies]
 *                 (mirgecom/fluid.py:300-312)
 *   temperature   [E][Np]
 *   grad          [Nc+1][dim][E][Np]  gradient of q then of temperature
 *   rx            [E][dim][dim]  dr_r/dx_j
 *   conn          [E][Nf]  nbr_elem*256 + perm_id, or -(1 + boundary face)
 *   perm          [nperm][Nfp]  neighbour volume node of own face node m
 *   bkind         [nbf]  0 = exterior copies interior (DummyBoundary),
 *                        1 = prescribed exterior state
 *   bext          [Nc+1][nbf][Nfp]  prescribed exterior q, then temperature
 */
#ifndef MGC_B200_H
#define MGC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGC_OK 0
#define MGC_E_INVALID (-1)
#define MGC_E_UNSUPPORTED (-2)
#define MGC_E_NOT_READY (-3)
#define MGC_E_CUDA (-4)
#define MGC_E_TOO_LARGE (-5)

#define MGC_ST_NAN 1
#define MGC_ST_BAD_INDEX 2
#define MGC_ST_NEWTON_MISS 4
#define MGC_ST_NONPOSITIVE 8
#define MGC_ST_WAIT_TIMEOUT 16

#define MGC_MAX_SPECIES 16
#define MGC_MAX_REACTIONS 8

#define MGC_EOS_IDEAL 0
#define MGC_EOS_MIXTURE 1
#define MGC_TRANSPORT_NONE 0
#define MGC_TRANSPORT_SIMPLE 1
#define MGC_TRANSPORT_POWERLAW 2
#define MGC_FLUX_RUSANOV 0
#define MGC_FLUX_HLL 1
#define MGC_FLUX_CENTRAL 2
#define MGC_ELEM_SIMPLEX 0
#define MGC_ELEM_HEX 1       /* tensor-product (GLL) hexahedra, affine */

/* Gas model: GasModel(eos, transport), mirgecom/gas_model.py:82-97, with
 * IdealSingleGas (mirgecom/eos.py:302), PyrometheusMixture (eos.py:540),
 * SimpleTransport (mirgecom/transport.py:143), PowerLawTransport (:205). */
typedef struct {
  int32_t eos_kind;
  int32_t nspecies;
  int32_t niter;            /* Newton iterations, thermochemistry.py:51 */
  int32_t transport_kind;
  double gamma, gas_const;
  double mu, mu_b, kappa;
  double pl_alpha, pl_beta, pl_sigma, pl_n;
  int32_t use_lewis;
  int32_t pad_;
  double diff[MGC_MAX_SPECIES];
  double lewis[MGC_MAX_SPECIES];
  double zero_level;
} mgc_gas_t;

/* Thermochemistry tables in SI units (pyrometheus conventions). */
typedef struct {
  int32_t nspecies, nreactions;
  double mw[MGC_MAX_SPECIES];
  double inv_mw[MGC_MAX_SPECIES];
  double t_mid[MGC_MAX_SPECIES];
  double a_lo[MGC_MAX_SPECIES][7];
  double a_hi[MGC_MAX_SPECIES][7];
  double ord_f[MGC_MAX_REACTIONS][MGC_MAX_SPECIES];
  double nu_p[MGC_MAX_REACTIONS][MGC_MAX_SPECIES];
  double nu_net[MGC_MAX_REACTIONS][MGC_MAX_SPECIES];
  double dnu[MGC_MAX_REACTIONS];
  double log_a[MGC_MAX_REACTIONS];
  double beta[MGC_MAX_REACTIONS];
  double t_act[MGC_MAX_REACTIONS];
  int32_t reversible[MGC_MAX_REACTIONS];
} mgc_mechanism_t;

/* Flattened discretization (the host-side replacement of grudge's
 * DiscretizationCollection connectivity, mirgecom/discretization.py:41-83). */
typedef struct {
  int32_t dim, order, nelem, nbf, nperm;
  int32_t elem_kind;        /* MGC_ELEM_SIMPLEX or MGC_ELEM_HEX */
  const double* rx;
  const int32_t* conn;
  const uint8_t* perm;
  const int8_t* bkind;
  const float* rx32;        /* float32 copy of rx, for the *_f32 entry points */
  const uint8_t* fslot;     /* [nperm][Nfp] neighbour face slot fn*Nfp + m' of own face
                               node m (mgc_operator*; may be NULL for the others) */
  int32_t nowned;           /* mgc_operator*: elements [0, nowned) are evaluated, the
                               rest are ghost elements of a mesh partition (neighbours
                               only); 0 = all nelem */
  int32_t pad_;
} mgc_mesh_t;

/* Library version and the list of supported (dim, order) pairs. */
int mgc_version(void);
int mgc_supports(int dim, int order, int nspecies, int eos_kind);

/* Upload the reference-element operators of one (dim, order) pair to every
 * device-side constant bank of the library, on the current device.
 * weak_host [dim][Np][Np], lift_host [Np][Nf*Nfp], ref_normals_host
 * [Nf][dim], face_scale_ref_host [Nf], face_nodes_host [Nf][Nfp].
 * Replaces grudge's reference matrices behind op.weak_local_grad/div,
 * op.face_mass and op.inverse_mass (mirgecom/operators.py:60-63,92-95). */
int mgc_upload_reference_operators(int dim, int order, const double* weak_host,
                                   const double* lift_host,
                                   const double* ref_normals_host,
                                   const double* face_scale_ref_host,
                                   const int32_t* face_nodes_host);

/* Tensor-product hexahedra (TensorProductElementGroup meshes,
 * mirgecom/discretization.py:41-83 with tensor-product groups; the operators
 * of operators.py:34-95 applied by sum factorisation).  Upload the 1-D
 * operators of order p: weak1d [p+1][p+1] = M1^-1 D1^T M1, lift1d [p+1][2] =
 * columns 0 and p of M1^-1, and the reference face scale.  Supported: dim 3,
 * p = 1..4, single ideal gas; the gradient pass (mgc_ns_grad*) and the split
 * divergence (mgc_rhs_split*) -- the fused mgc_euler_rhs / mgc_ns_rhs return
 * MGC_E_UNSUPPORTED for hexahedra. */
int mgc_supports_hex(int dim, int order, int nspecies, int eos_kind);
int mgc_upload_hex_operators(int dim, int order, const double* weak1d_host,
                             const double* lift1d_host, double face_scale_ref);

/* Upload a thermochemistry mechanism (pyrometheus class data used by
 * PyrometheusMixture, mirgecom/eos.py:540-888) on the current device. */
int mgc_set_mechanism(const mgc_mechanism_t* mech_host);

/* Mixture temperature (mirgecom/eos.py:777-803 -> thermochemistry.py:126-167):
 * t1 = Newton(e, Y; t_seed), t2 = Newton(e, Y; t1) (t2 may be NULL).
 * nnodes = E*Np.  A node whose solve has not converged (t2, or one further
 * Newton step when t2 is NULL, moves by more than 1e-6 of t1) or whose
 * temperature is not positive and finite sets MGC_ST_NEWTON_MISS in *status
 * (may be NULL); the reference leaves this to its drivers' health checks. */
int mgc_mixture_temperature(int dim, const mgc_gas_t* gas, int64_t nnodes,
                            const double* q, const double* t_seed, double* t1,
                            double* t2, int32_t* status, void* stream);

/* euler_operator (mirgecom/euler.py:313-416), non-ESDG branch. t_op is the
 * operator temperature for mixtures (NULL for the ideal gas). */
int mgc_euler_rhs(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                  const double* t_op, const double* bext, int flux_kind,
                  double* rhs, int32_t* status, void* stream);

/* grad_cv_operator + grad_t_operator (mirgecom/navierstokes.py:129-347). */
int mgc_ns_grad(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                const double* t_op, const double* bext, double* grad,
                int32_t* status, void* stream);

/* The divergence part of ns_operator (mirgecom/navierstokes.py:533-563) given
 * the gradients; with add_sources != 0 adds the species source terms
 * (mirgecom/eos.py:858-875) evaluated at t_src. */
int mgc_ns_rhs(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
               const double* t_op, const double* t_src, const double* grad,
               const double* bext, int flux_kind, int add_sources, double* rhs,
               int32_t* status, void* stream);

/* One stage of rk4_step (mirgecom/integrators/explicit_rk.py:31-37):
 * stage 0..2: sum (+)= w k, q_out = q0 + c dt k; stage 3: q_out = q0 +
 * dt/6 (sum + k).  q_out_lo (float32 copy of q_out) may be NULL. */
int mgc_rk4_stage(int64_t n, const double* q0, const double* k, double* sum,
                  double* q_out, float* q_out_lo, int stage, double dt,
                  void* stream);

/* ---- mixed-precision form (float32 storage and pointwise math, tf32 x3
 * tensor-core contractions with float32 accumulation).  Same semantics and
 * layouts as the float64 entry points above, with float arrays; the
 * operator temperature t_op is the single temperature of the state. ---- */

int mgc_euler_rhs_f32(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                      const float* t_op, const float* bext, int flux_kind, float* rhs,
                      int32_t* status, void* stream);

int mgc_ns_grad_f32(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                    const float* t_op, const float* bext, float* grad, int32_t* status,
                    void* stream);

int mgc_ns_rhs_f32(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                   const float* t_op, const float* t_src, const float* grad,
                   const float* bext, int flux_kind, int add_sources, float* rhs,
                   int32_t* status, void* stream);

/* Mixture temperature, mixed form (extends mirgecom/thermochemistry.py:126-167,
 * which runs a fixed number of float64 iterations).  Float32 Newton from
 * t_guess (the learned guess; NULL to start from t_seed), stopped once the
 * predicted remaining error k dT^2 (k = max |c_v'| / (2 c_v) of the
 * mechanism, quadratic convergence) is small enough for the last step; then
 * the float64 residual correction corr = (e - e(T)) / c_v(T) is applied when
 * its own predicted remainder k corr^2 is at most rtol |T| -- the relative
 * temperature-update tolerance the reference drivers check, e.g. 1e-8 in
 * mirgecom examples/autoignition.py:526-530.  A rejected result is recomputed
 * from the plain guess t_seed.  iters (nullable) receives the float32
 * iteration count per node (+1000 when the fallback ran); nodes failing both
 * set MGC_ST_NEWTON_MISS. */
int mgc_mixture_temperature_f32(int dim, const mgc_gas_t* gas, int64_t nnodes,
                                const float* q, const float* t_seed, const float* t_guess,
                                float* t_out, int32_t* iters, int maxit, float rtol,
                                int32_t* status, void* stream);

/* rk4 stage with a float32 right-hand side k: the state and the stage sum
 * stay float64, q_out_lo receives the float32 copy of q_out. */
int mgc_rk4_stage_mixed(int64_t n, const double* q0, const float* k, double* sum,
                        double* q_out, float* q_out_lo, int stage, double dt,
                        void* stream);

/* ---- split right-hand side: the divergence pass of mgc_euler_rhs (viscous
 * = 0) or mgc_ns_rhs (viscous = 1) as two kernels -- every node's total
 * flux, p, c and gamma (and species sources) once into a caller-provided
 * workspace, then the numerical face fluxes from the records of both sides
 * and the tensor-core contraction.  Same arguments and results as the fused
 * entry points plus the workspace (16-byte aligned, at least
 * mgc_rhs_split_workspace_bytes(mesh, gas, single_precision) bytes) and
 * mid_event, a cudaEvent_t recorded on the stream between the two kernels
 * (NULL for none; for timing the surface kernel on its own). ---- */
size_t mgc_rhs_split_workspace_bytes(const mgc_mesh_t* mesh, const mgc_gas_t* gas,
                                     int single_precision);
int mgc_rhs_split(int viscous, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                  const double* t_op, const double* t_src, const double* grad,
                  const double* bext, int flux_kind, int add_sources, double* rhs,
                  void* workspace, size_t workspace_bytes, int32_t* status, void* stream,
                  void* mid_event);
int mgc_rhs_split_f32(int viscous, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                      const float* t_op, const float* t_src, const float* grad,
                      const float* bext, int flux_kind, int add_sources, float* rhs,
                      void* workspace, size_t workspace_bytes, int32_t* status, void* stream,
                      void* mid_event);

/* Gradient-pass kernel of every entry point that computes gradients
 * (mgc_ns_grad*, mgc_ns_rhs*'s callers, mgc_operator* with phases bit 4):
 * MGC_GRAD_AUTO (default) runs the tcgen05/TMEM pipelined kernel where it
 * applies (float32, 3-D simplices, mixtures, rows of Np floats in 16-byte
 * pieces) and the mma.sync kernel elsewhere; MGC_GRAD_MMA_SYNC always runs
 * the mma.sync kernel.  Process-wide; returns MGC_E_INVALID for other
 * values.  Replaces no reference interface (the reference has one gradient
 * code path, grad_operator, mirgecom/navierstokes.py:443-446). */
#define MGC_GRAD_AUTO 0
#define MGC_GRAD_MMA_SYNC 1
int mgc_set_gradient_kernel(int kind);
int mgc_get_gradient_kernel(void);

/* ---- euler_operator (viscous = 0; mirgecom/euler.py:313-416, non-ESDG
 * branch) or ns_operator (viscous = 1; mirgecom/navierstokes.py:350-575,
 * with return_gradients when grad_out is non-NULL) in one call on
 * simplicial meshes: a volume kernel (BR1 gradients kept on chip, pointwise
 * fluxes and sources, face-node flux records, the volume part of the weak
 * divergence) and a face kernel (numerical face fluxes from the records of
 * both sides, lift).  t_op: operator temperature (mixtures); t_src: the
 * temperature of the species sources (add_sources != 0); bext: prescribed
 * exterior states [Nc+1][nbf][Nfp] (may be NULL when no boundary face is
 * prescribed); grad_out: optional [Nc+1][dim][E][Np] gradients.  The mesh
 * needs fslot.  workspace: 256-byte aligned, at least
 * mgc_operator_workspace_bytes(mesh, gas, single_precision) bytes (face-node
 * records [E][Nf][Nfp][round_up(Nc+4, 4)], node-0 fluxes [E][Nf][Nc],
 * boundary records, boundary plus states).  mid_event: a cudaEvent_t
 * recorded between the two kernels, or NULL.  phases: 1 the volume kernel
 * only, 2 the face kernel only, 3 both (a partitioned mesh exchanges the
 * ghost elements' face-node records between the two); | 4 runs the volume
 * stage as two kernels, the gradient kernel (gradients into grad_out,
 * required when viscous) then a flux-volume kernel that reads them; | 8
 * (with 4) skips that gradient kernel: grad_out already holds the
 * gradients (from mgc_ns_grad*).  With
 * mesh->nowned > 0 only elements [0, nowned) are evaluated; elements
 * [nowned, nelem) are ghosts (q, temperatures and, before the face kernel,
 * their face-node records filled by the caller's halo exchange).  Hexahedral
 * meshes return MGC_E_UNSUPPORTED (use mgc_ns_grad* + mgc_rhs_split*). ---- */
size_t mgc_operator_workspace_bytes(const mgc_mesh_t* mesh, const mgc_gas_t* gas,
                                    int single_precision);
int mgc_operator(int viscous, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                 const double* t_op, const double* t_src, const double* bext, int flux_kind,
                 int add_sources, double* rhs, double* grad_out, void* workspace,
                 size_t workspace_bytes, int32_t* status, void* stream, void* mid_event,
                 int phases);
int mgc_operator_f32(int viscous, const mgc_mesh_t* mesh, const mgc_gas_t* gas, const float* q,
                     const float* t_op, const float* t_src, const float* bext, int flux_kind,
                     int add_sources, float* rhs, float* grad_out, void* workspace,
                     size_t workspace_bytes, int32_t* status, void* stream, void* mid_event,
                     int phases);

/* ---- learned initial guess of the mixture temperature (no counterpart in
 * the reference, whose Newton solve always starts from the seed): an
 * 8 -> 64 -> 64 -> 1 tanh MLP, bf16 tensor-core matrix products with float32
 * accumulation.  Inputs: mixture internal energy and the 7 species mass
 * fractions, normalised by (x - in_shift) * in_scale; output T = out_shift +
 * out_scale * y.  params is the float32 master vector (mgc_mlp_nparams()
 * entries: W1 [64][16] with input columns 8..15 zero, b1 [64], W2 [64][64],
 * b2 [64], w3 [64], b3); the bf16 copies are refreshed by mgc_mlp_refresh
 * and by every mgc_mlp_adam step. ---- */
typedef struct {
  float* params;
  void* w1_bf16;            /* [64][16] */
  void* w2_bf16;            /* [64][64] (out, in) */
  void* w2t_bf16;           /* [64][64] (in, out) */
  float in_shift[8], in_scale[8];
  float out_shift, out_scale;
} mgc_mlp_t;

int mgc_mlp_nparams(void);
int mgc_mlp_refresh(const mgc_mlp_t* w, void* stream);

/* Mixed-form mixture temperature with the learned guess computed in the same
 * kernel (no counterpart in the reference, which has no learned guess): per
 * node the network's guess, then the solve of mgc_mixture_temperature_f32
 * with t_seed as the fallback.  Nodes are taken 32 at a time: when the first
 * Newton step from t_seed is at most 4 K for all 32 (a seed the network cannot
 * improve on), the network is skipped and the solve continues from the seed;
 * iters then carries + 100.  Same arguments and status as
 * mgc_mixture_temperature_f32 plus the network w; requires mgc_set_mechanism. */
int mgc_mixture_temperature_learned_f32(int dim, const mgc_gas_t* gas, int64_t nnodes,
                                        const float* q, const float* t_seed,
                                        const mgc_mlp_t* w, float* t_out, int32_t* iters,
                                        int maxit, float rtol, int32_t* status, void* stream);

/* Guess T for every node of a float32 state q [Nc][n] (nspecies == 7). */
int mgc_mlp_infer(int dim, int nspecies, int64_t n, const float* q, const mgc_mlp_t* w,
                  float* t_out, void* stream);

/* Gradient of the mean squared error over n normalised samples x [n][8],
 * target [n]: grad (mgc_mlp_nparams() floats, overwritten) and loss (one
 * float, overwritten).  workspace: caller-provided device memory of
 * mgc_mlp_train_workspace_bytes(n) bytes. */
size_t mgc_mlp_train_workspace_bytes(int64_t n);
int mgc_mlp_train_grad(int64_t n, const float* x, const float* target, const mgc_mlp_t* w,
                       void* workspace, size_t workspace_bytes, float* grad, float* loss,
                       void* stream);

/* One Adam step on the master vector (m, v: optimiser state, step >= 1). */
int mgc_mlp_adam(const mgc_mlp_t* w, const float* grad, float* m, float* v, float lr,
                 float beta1, float beta2, float eps, int step, void* stream);

/* ---- FP64 throughput probes (the float64 path's compute roofline).
 * No counterpart in the reference (a measurement aid).  kind 0 runs
 * independent fma.rn.f64 chains (the FP64 FMA pipe), kind 1 independent
 * mma.m8n8k4.f64 chains (the float64 tensor cores) over nblocks x threads
 * (threads <= 256, a multiple of 32) for iters rounds; sink receives
 * nblocks*threads doubles.  mgc_fp64_probe_flops gives the flops one launch
 * performs, for the caller's event timing. */
double mgc_fp64_probe_flops(int kind, int nblocks, int threads, int iters);
int mgc_fp64_probe(int kind, int nblocks, int threads, int iters, double* sink,
                   void* stream);

/* ---- Navier-Stokes right-hand side without device allocation.
 * No counterpart in the reference: it exists for callers that cannot
 * allocate device memory -- a solver that owns all device memory through
 * its own pool and forbids driver allocations during a run, or a host code
 * linked without a CUDA allocation layer.  It runs mgc_ns_grad then
 * mgc_ns_rhs with the gradient buffer taken from a fixed library-owned
 * device array of mgc_ns_operator_noalloc_capacity() doubles (32 MiB, held
 * by every GPU that loads the library until exit).  Meshes whose gradient
 * buffer ((Nc+1)*dim*E*Np doubles) exceeds it return MGC_E_TOO_LARGE.
 * All calls share that array: calls overlapping on the GPU race and must be
 * serialised by the caller.  The first call on a device looks up the
 * array's device address; make it before any stream capture.  That address
 * is kept for the life of the process and does not survive cudaDeviceReset
 * (or any other teardown of the device's primary context): do not call this
 * entry point after one.  Arguments and results are those of mgc_ns_rhs. ---- */
size_t mgc_ns_operator_noalloc_capacity(void);

int mgc_ns_operator_noalloc(const mgc_mesh_t* mesh, const mgc_gas_t* gas, const double* q,
                            const double* t_op, const double* t_src, const double* bext,
                            int flux_kind, int add_sources, double* rhs, int32_t* status,
                            void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MGC_B200_H */
