// Reference-element operators of the nodal DG discretization, held in
// constant memory so that the fully unrolled contractions read them as
// instruction operands (one broadcast per warp, no shared-memory traffic).
//
// For every supported (dim, order) the packed block holds, in order:
//   W     [dim][Np][Np]   W_r = M^-1 D_r^T M          (weak derivative)
//   LIFT  [Np][Nf*Nfp]    M^-1 E                      (face lift)
//   NREF  [Nf][dim]       unit outward reference normals
//   FSR   [Nf]            reference face measure / face-parametrisation measure
// The host computes them once (refelem.py) and uploads them through
// mgc_upload_reference_operators().
#pragma once
#include <cstdint>

namespace mgc {

__host__ __device__ constexpr int simplex_npts(int dim, int order) {
  return dim == 0 ? 1
       : dim == 1 ? order + 1
       : dim == 2 ? (order + 1) * (order + 2) / 2
                  : (order + 1) * (order + 2) * (order + 3) / 6;
}

__host__ __device__ constexpr int refops_size(int dim, int order) {
  return dim * simplex_npts(dim, order) * simplex_npts(dim, order) +
         simplex_npts(dim, order) * (dim + 1) * simplex_npts(dim - 1, order) +
         (dim + 1) * dim + (dim + 1);
}

// supported simplex discretizations, in packing order
__host__ __device__ constexpr int refops_slot(int dim, int order) {
  return (dim == 2 && order >= 1 && order <= 4) ? order - 1
       : (dim == 3 && order >= 1 && order <= 3) ? 4 + order - 1
                                                : -1;
}

__host__ __device__ constexpr int refops_offset(int dim, int order) {
  int off = 0;
  for (int o = 1; o <= 4; ++o) {
    if (dim == 2 && o == order) return off;
    off += refops_size(2, o);
  }
  for (int o = 1; o <= 3; ++o) {
    if (dim == 3 && o == order) return off;
    off += refops_size(3, o);
  }
  return -1;
}

constexpr int kRefOpsTotal = refops_offset(3, 3) + refops_size(3, 3);

// Every translation unit that launches kernels holds its own copy (internal
// linkage, no relocatable device code); mgc_upload_reference_operators()
// fills the copy of each unit.
static __constant__ double c_ref64[kRefOpsTotal];
static __constant__ float c_ref32[kRefOpsTotal];

__host__ __device__ constexpr int fnodes_size(int dim, int order) {
  return (dim + 1) * simplex_npts(dim - 1, order);
}

__host__ __device__ constexpr int fnodes_offset(int dim, int order) {
  int off = 0;
  for (int o = 1; o <= 4; ++o) {
    if (dim == 2 && o == order) return off;
    off += fnodes_size(2, o);
  }
  for (int o = 1; o <= 3; ++o) {
    if (dim == 3 && o == order) return off;
    off += fnodes_size(3, o);
  }
  return -1;
}

constexpr int kFaceNodesTotal = fnodes_offset(3, 3) + fnodes_size(3, 3);

// volume node index of face node m of face f, at [f * Nfp + m]
static __constant__ int c_fnodes[kFaceNodesTotal];

template <int DIM, int ORDER>
__device__ __forceinline__ int c_face_nodes(int i) {
  return c_fnodes[fnodes_offset(DIM, ORDER) + i];
}

template <int DIM, int ORDER>
struct Simplex {
  static constexpr int NP = simplex_npts(DIM, ORDER);
  static constexpr int NF = DIM + 1;
  static constexpr int NFP = simplex_npts(DIM - 1, ORDER);
  static constexpr int OFF = refops_offset(DIM, ORDER);
  static constexpr int OFF_W = OFF;
  static constexpr int OFF_LIFT = OFF_W + DIM * NP * NP;
  static constexpr int OFF_NREF = OFF_LIFT + NP * NF * NFP;
  static constexpr int OFF_FSR = OFF_NREF + NF * DIM;
  static_assert(OFF >= 0, "unsupported simplex discretization");
};

template <class R> struct RefBank;
template <> struct RefBank<double> {
  static __device__ __forceinline__ double get(int i) { return c_ref64[i]; }
};
template <> struct RefBank<float> {
  static __device__ __forceinline__ float get(int i) { return c_ref32[i]; }
};

}  // namespace mgc
