// BR1 gradient pass on the 5th-generation tensor cores (tcgen05, TMEM).
//
// The same arithmetic as k_grad (dg_kernels.cuh) -- the weak-form gradient
//   grad_j u = sum_f n_fj LIFT_f (fscale_f u*_f) - sum_r rx_rj W_r u
// of every conserved field and the temperature, with the element-constant
// shift u - u_0 and the TF32 three-term split A_hi B_hi + A_hi B_lo +
// A_lo B_hi -- organised as a warp-specialised pipeline over tiles of
// EPB elements (grad_operator, mirgecom/navierstokes.py:443-446, and
// grad_facial_flux, mirgecom/gradient.py):
//
//   producer warps 0-11  load the tile's rows of q and T (shifted by their
//                        first node), the face values fscale (u* - u_0) of
//                        the neighbours or the boundary, and the element
//                        geometry; they write the hi/lo copies of the A
//                        operand [row = (field, element)][k] into one of two
//                        shared-memory stages and arrive on full[s]; after
//                        the next tile barrier the group's last thread waits
//                        on full[s] (complete by then), issues the tcgen05.mma
//                        products
//                        D[row][(r, i)] = sum_k U[row][k] W_r[i][k]  (k nodes)
//                        D[row][(f, i)] = sum_k S[row][k] LIFT_f[i][k]
//                        into TMEM buffer s and commits to done[s]
//   epilogue warps 12-15 wait on done[s], read their TMEM lanes (one row per
//                        thread), combine with the metric terms and normals,
//                        store the gradients and arrive on empty[s]
//
// so the loads of tile i+1 overlap the products and the epilogue of tile i.
// Operands use the K-major, non-swizzled canonical layout of the UMMA
// descriptors: 8-row x 16-byte core matrices, row groups SBO = 128 bytes
// apart, k chunks LBO bytes apart.  Every mbarrier wait is bounded: after
// kWaitNs the waiting role sets ST_WAIT_TIMEOUT in the status word and an
// abort flag that ends the other roles' loops; the kernel then releases its
// TMEM and returns.
#pragma once
#include <cstdint>

#include "dg_kernels.cuh"

namespace mgc {

// {{{ tcgen05 / mbarrier primitives

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\tmbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n\t}" ::"r"(
          smem_addr(b))
      : "memory");
}
// one test of the phase, the thread suspended until it completes or for at
// most kSuspendNs
constexpr uint32_t kSuspendNs = 200000;
__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(addr), "r"(parity), "n"(kSuspendNs)
      : "memory");
  return ok != 0;
}
// one test of the phase without suspending
__device__ __forceinline__ bool mbar_test(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// a waiting role gives up after this long (the whole kernel normally takes
// milliseconds)
constexpr uint64_t kWaitNs = 2000000000ull;
// Bounded wait for the completion of phase *parity* of barrier *b*; false
// when the time limit ran out or another role raised *abort* (if given).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity,
                                          const volatile int* abort) {
  const uint32_t a = smem_addr(b);
  if (mbar_try(a, parity)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try(a, parity)) return true;
    if (abort && *abort) return false;
    if (global_ns() - t0 > kWaitNs) return false;
  }
}
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// TMEM allocation by one whole warp; the base address lands in *dst
__device__ __forceinline__ void tc_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
// Shared-memory matrix descriptor: K-major, no swizzle (layout type 0),
// descriptor version 1; addresses and offsets in 16-byte units.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::tf32: f32 accumulator, tf32 A and B, both
// K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}
// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void tc_mma_tf32(uint32_t d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on *b once every product issued so far by this thread has completed
__device__ __forceinline__ void tc_commit(uint64_t* b) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_addr(b))
      : "memory");
}
// four consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tc_ld4(uint32_t taddr, uint32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}
// wait for this thread's TMEM loads; the registers are tied to the wait so
// that no use is scheduled before it
template <int N>
__device__ __forceinline__ void tc_wait_ld(uint32_t (&v)[N][4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < N; ++i)
    asm volatile("" : "+r"(v[i][0]), "+r"(v[i][1]), "+r"(v[i][2]), "+r"(v[i][3]));
}

// }}}

// {{{ configuration

template <int DIM, int ORDER, int NS>
struct TcGrad {
  using S = Simplex<DIM, ORDER>;
  static constexpr int NP = S::NP, NF = S::NF, NFP = S::NFP, NFN = NF * NFP;
  static constexpr int NC = DIM + 2 + NS, NU = NC + 1;
  static constexpr int ROWS = 128;                    // MMA M: rows (field, element)
  static constexpr int EPB = ROWS / NU;               // elements per tile
  static constexpr int KV = round_up(NP, 8);          // k extent of the volume product
  static constexpr int KL = round_up(NFN, 8);         // k extent of the lift product
  static constexpr int KA = KV + KL;                  // A operand k extent
  static constexpr int NV = round_up(DIM * NP, 16);   // N of the volume product
  static constexpr int NL = round_up(NF * NP, 16);    // N of the lift product
  static constexpr int NACC = NV + NL;                // TMEM columns per buffer
  static constexpr int TCOLS = 512;                   // allocated TMEM columns (2 buffers)
  static constexpr int BUF_COLS = 256;
  // byte strides of the canonical layouts
  static constexpr int SBO = 128;
  static constexpr int LBO_A = ROWS / 8 * 128;
  static constexpr int LBO_V = NV / 8 * 128;
  static constexpr int LBO_L = NL / 8 * 128;
  static constexpr int A_BYTES = KA / 4 * LBO_A;      // one copy (hi or lo) of one stage
  static constexpr int BV_BYTES = KV / 4 * LBO_V;
  static constexpr int BL_BYTES = KL / 4 * LBO_L;
  static constexpr int GEO = DIM * DIM + NF * DIM;    // rx, unit normals per element
  // one producer group of GW warps filling the block's tiles (tile it into
  // stage it % 2); four epilogue warps.  A single group is what the
  // deferred product issue assumes: the previous tile's products are issued
  // after the next tile's barrier, which waits for the stage of the tile
  // before (two producer groups, each reusing its own stage, would wait for
  // their own unissued products)
  static constexpr int NGRP = 1;
  static constexpr int GW = 12, GT = GW * 32;
  static constexpr int NPROD = NGRP * GT, NEPI = 128;
  // producer work items per tile and the rounds of a group they take
  static constexpr int ROW_ITEMS = NP / 4 * NU * EPB;
  static constexpr int FACE_ITEMS = NFN * EPB;
  static constexpr int ROW_ROUNDS = (ROW_ITEMS + GT - 1) / GT;
  static constexpr int FACE_ROUNDS = (FACE_ITEMS + GT - 1) / GT;
  static constexpr int NT = NPROD + NEPI;
  static constexpr int EPI_WARP0 = NPROD / 32;        // a multiple of 4: warp w reads TMEM
                                                      // lanes 32 (w % 4) ..
  // per-tile data of a group's tile: face pairing, rx and unit normals,
  // face scales, the row shifts u_0 (floats/ints), staged one tile ahead
  static constexpr int SMALL = EPB * NF + EPB * GEO + EPB * NF + NU * EPB;
  // shared-memory carve-up (bytes)
  static constexpr int OFF_BAR = 0;                   // full[2], done[2], empty[2]
  static constexpr int OFF_TMEM = 48;                 // TMEM base address
  static constexpr int OFF_ABORT = 52;                // any role gave up
  static constexpr int OFF_PABORT = 64;               // each group's copy of it [NGRP]
  static constexpr int OFF_A = 1024;                  // [stage][hi, lo]
  static constexpr int OFF_BV = OFF_A + 4 * A_BYTES;  // [hi, lo]
  static constexpr int OFF_BL = OFF_BV + 2 * BV_BYTES;
  static constexpr int OFF_GEO = OFF_BL + 2 * BL_BYTES;          // [stage][EPB][GEO] float
  static constexpr int OFF_SMALL = OFF_GEO + 2 * EPB * GEO * 4;  // [group][2][SMALL] 4-byte
  static constexpr int OFF_RAW = round_up(OFF_SMALL + NGRP * 2 * SMALL * 4, 16);
  // [group][NU * EPB][NP] float
  static constexpr int OFF_FN = OFF_RAW + NGRP * NU * EPB * NP * 4;  // [NFN] int
  static constexpr int OFF_PERM = OFF_FN + NFN * 4;               // [nperm][NFP] uint8
  static size_t smem_bytes(int nperm) { return (size_t)OFF_PERM + (size_t)nperm * NFP + 16; }
  // whole rows of NP floats in 16-byte pieces; products within the
  // instruction shapes; two TMEM buffers; the per-tile data one item per
  // group thread
  static constexpr bool OK = (NP % 4 == 0) && EPB >= 1 && EPB * NF + NU * EPB <= GT &&
                             NV <= 256 && NL <= 256 && NACC <= BUF_COLS &&
                             OFF_PERM + 64 * NFP <= 227 * 1024;
};

// the benchmark's configuration (order-3 tetrahedra, 7 species) fits
static_assert(TcGrad<3, 3, 7>::OK, "tcgen05 gradient kernel no longer fits order-3 tets");

// byte offset of element (row, k) in a canonical K-major no-swizzle operand
__device__ __forceinline__ int canon_off(int row, int k, int lbo) {
  return (k >> 2) * lbo + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ void split_f32(float v, float& hi, float& lo) {
  const uint32_t h = to_tf32(v);
  hi = __uint_as_float(h);
  lo = __uint_as_float(to_tf32(v - hi));
}

// }}}

namespace {

template <int DIM, int ORDER, int NS>
__global__ void __launch_bounds__(TcGrad<DIM, ORDER, NS>::NT, 1)
    k_grad_tc(DGArgs<float> a, GasParams g) {
  using C = TcGrad<DIM, ORDER, NS>;
  using S = Simplex<DIM, ORDER>;
  constexpr int NP = C::NP, NF = C::NF, NFP = C::NFP, NFN = C::NFN, NC = C::NC, NU = C::NU;
  constexpr int EPB = C::EPB, KV = C::KV, GEO = C::GEO, GT = C::GT;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + C::OFF_BAR);
  uint64_t* done = full + 2;
  uint64_t* empty = full + 4;
  uint32_t* tmem_s = reinterpret_cast<uint32_t*>(smem_raw + C::OFF_TMEM);
  volatile int* abort_s = reinterpret_cast<volatile int*>(smem_raw + C::OFF_ABORT);
  volatile int* pabort_s = reinterpret_cast<volatile int*>(smem_raw + C::OFF_PABORT);
  float* geo_s = reinterpret_cast<float*>(smem_raw + C::OFF_GEO);
  int* fn_s = reinterpret_cast<int*>(smem_raw + C::OFF_FN);
  uint8_t* perm_s = smem_raw + C::OFF_PERM;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int E = a.nelem;
  const int64_t EN = (int64_t)E * NP;
  const int EOWN = a.nowned > 0 ? a.nowned : E;
  const int ntiles = (EOWN + EPB - 1) / EPB;

  // ---- setup: barriers, zeroed A stages, operator B copies, TMEM
  if (tid == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(full + s, C::GT);
      mbar_init(done + s, 1);
      mbar_init(empty + s, C::NEPI);
    }
    *abort_s = 0;
    for (int i = 0; i < C::NGRP; ++i) pabort_s[i] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    float4* az = reinterpret_cast<float4*>(smem_raw + C::OFF_A);
    for (int i = tid; i < 4 * C::A_BYTES / 16; i += blockDim.x) az[i] = make_float4(0, 0, 0, 0);
    float* bvh = reinterpret_cast<float*>(smem_raw + C::OFF_BV);
    float* bvl = reinterpret_cast<float*>(smem_raw + C::OFF_BV + C::BV_BYTES);
    for (int i = tid; i < C::NV * KV; i += blockDim.x) {
      const int n = i / KV, k = i % KV, r = n / NP, row = n % NP;
      const double v = (n < DIM * NP && k < NP) ? c_ref64[S::OFF_W + (r * NP + row) * NP + k] : 0.0;
      float hi, lo;
      split_tf32(v, hi, lo);
      const int o = canon_off(n, k, C::LBO_V) >> 2;
      bvh[o] = hi;
      bvl[o] = lo;
    }
    float* blh = reinterpret_cast<float*>(smem_raw + C::OFF_BL);
    float* bll = reinterpret_cast<float*>(smem_raw + C::OFF_BL + C::BL_BYTES);
    for (int i = tid; i < C::NL * C::KL; i += blockDim.x) {
      const int n = i / C::KL, k = i % C::KL, f = n / NP, row = n % NP;
      const double v = (n < NF * NP && k < NFN && k / NFP == f)
                           ? c_ref64[S::OFF_LIFT + row * NFN + k]
                           : 0.0;
      float hi, lo;
      split_tf32(v, hi, lo);
      const int o = canon_off(n, k, C::LBO_L) >> 2;
      blh[o] = hi;
      bll[o] = lo;
    }
    for (int i = tid; i < NFN; i += blockDim.x) fn_s[i] = c_face_nodes<DIM, ORDER>(i);
    for (int i = tid; i < a.nperm * NFP; i += blockDim.x) perm_s[i] = a.perm[i];
  }
  if (warp == 0) tc_alloc(tmem_s, C::TCOLS);
  // generic-proxy writes of the operands become visible to the tensor cores
  fence_async_shared();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_s;

  if (warp < C::NPROD / 32) {
    // ================= producers: group grp fills the block's tiles
    // it = grp, grp + NGRP, ..., tile it into stage it % 2
    constexpr int RR = C::ROW_ROUNDS, FR = C::FACE_ROUNDS;
    const int grp = tid / GT, gtid = tid % GT;
    // group buffers: per-tile data [2][SMALL], shifted rows [NU * EPB][NP]
    float* small_g = reinterpret_cast<float*>(smem_raw + C::OFF_SMALL) + grp * 2 * C::SMALL;
    float* raw = reinterpret_cast<float*>(smem_raw + C::OFF_RAW) + grp * NU * EPB * NP;
    auto conn_of = [&](int b) { return reinterpret_cast<int32_t*>(small_g + b * C::SMALL); };
    auto geo_of = [&](int b) { return small_g + b * C::SMALL + EPB * NF; };
    auto fs_of = [&](int b) { return small_g + b * C::SMALL + EPB * NF + EPB * GEO; };
    auto u0_of = [&](int b) { return small_g + b * C::SMALL + 2 * EPB * NF + EPB * GEO; };
    // per-tile data of tile *tl*: loads, then (after this tile's work) the
    // derived values into buffer *b*
    struct Small {
      int32_t cn;
      float rxe[DIM * DIM];
      float u0;
      bool gok, uok;
    };
    auto small_load = [&](int tl, Small& sm) {
      const int e1 = tl * EPB, n1 = imin(EPB, EOWN - e1);
      const int gi = gtid, ui = gtid - EPB * NF;
      sm.gok = gi < n1 * NF;
      sm.uok = ui >= 0 && ui < NU * EPB && ui % EPB < n1;
      if (sm.gok) {
        sm.cn = __ldg(a.conn + (int64_t)e1 * NF + gi);
        const float* rxg = a.rx + (int64_t)(e1 + gi / NF) * DIM * DIM;
#pragma unroll
        for (int i = 0; i < DIM * DIM; ++i) sm.rxe[i] = __ldg(rxg + i);
      }
      if (sm.uok) {
        const int c = ui / EPB, e = ui % EPB;
        sm.u0 = __ldg((c < NC ? a.q + c * EN : a.t_op) + (int64_t)(e1 + e) * NP);
      }
    };
    auto small_store = [&](const Small& sm, int b) {
      if (sm.gok) {
        const int gi = gtid, e = gi / NF, f = gi % NF;
        float* pg = geo_of(b) + e * GEO;
        conn_of(b)[gi] = sm.cn;
        float nv[DIM];
        float mag2 = 0;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
          float acc = 0;
#pragma unroll
          for (int r = 0; r < DIM; ++r)
            acc += sm.rxe[r * DIM + j] * RefBank<float>::get(S::OFF_NREF + f * DIM + r);
          nv[j] = acc;
          mag2 += acc * acc;
        }
        const float mag = sqrtf(mag2);
#pragma unroll
        // approximate quotient: an IEEE division site (with its out-of-line
        // slow path) cost this whole kernel 1.1 ms at 80^3; the normals
        // differ from the other kernels' by a few ulp
        for (int j = 0; j < DIM; ++j) pg[DIM * DIM + f * DIM + j] = __fdividef(nv[j], mag);
        fs_of(b)[gi] = mag * RefBank<float>::get(S::OFF_FSR + f);
        if (f == 0) {
#pragma unroll
          for (int i = 0; i < DIM * DIM; ++i) pg[i] = sm.rxe[i];
        }
      }
      if (sm.uok) u0_of(b)[gtid - EPB * NF] = sm.u0;
    };
    // D[s] = A[s] B^T: the volume products into columns [0, NV), the lift
    // products into [NV, NV + NL), three split terms per k step
    auto issue_products = [&](int s) {
      constexpr uint32_t IDV = umma_idesc_tf32(C::ROWS, C::NV);
      constexpr uint32_t IDL = umma_idesc_tf32(C::ROWS, C::NL);
      const uint32_t ah = smem_addr(smem_raw + C::OFF_A) + (2 * s) * C::A_BYTES;
      const uint32_t al = ah + C::A_BYTES;
      const uint32_t bvh = smem_addr(smem_raw + C::OFF_BV), bvl = bvh + C::BV_BYTES;
      const uint32_t blh = smem_addr(smem_raw + C::OFF_BL), bll = blh + C::BL_BYTES;
      const uint32_t d = tmem + (uint32_t)(s * C::BUF_COLS);
#pragma unroll
      for (int ks = 0; ks < KV / 8; ++ks) {
        const uint32_t ao = 2 * ks * C::LBO_A, bo = 2 * ks * C::LBO_V;
        tc_mma_tf32(d, umma_desc(al + ao, C::LBO_A, C::SBO), umma_desc(bvh + bo, C::LBO_V, C::SBO),
                    IDV, ks > 0);
        tc_mma_tf32(d, umma_desc(ah + ao, C::LBO_A, C::SBO), umma_desc(bvl + bo, C::LBO_V, C::SBO),
                    IDV, 1);
        tc_mma_tf32(d, umma_desc(ah + ao, C::LBO_A, C::SBO), umma_desc(bvh + bo, C::LBO_V, C::SBO),
                    IDV, 1);
      }
#pragma unroll
      for (int ks = 0; ks < C::KL / 8; ++ks) {
        const uint32_t ao = (KV / 4 + 2 * ks) * C::LBO_A, bo = 2 * ks * C::LBO_L;
        const uint32_t dl = d + C::NV;
        tc_mma_tf32(dl, umma_desc(al + ao, C::LBO_A, C::SBO),
                    umma_desc(blh + bo, C::LBO_L, C::SBO), IDL, ks > 0);
        tc_mma_tf32(dl, umma_desc(ah + ao, C::LBO_A, C::SBO),
                    umma_desc(bll + bo, C::LBO_L, C::SBO), IDL, 1);
        tc_mma_tf32(dl, umma_desc(ah + ao, C::LBO_A, C::SBO),
                    umma_desc(blh + bo, C::LBO_L, C::SBO), IDL, 1);
      }
    };
    int issued = 0, last_issued = -1;
    int pending = -1;          // a filled tile whose products are not issued yet
    const int first = blockIdx.x + grp * (int)gridDim.x;
    const int step = C::NGRP * (int)gridDim.x;
    if (first < ntiles) {
      Small sm0;
      small_load(first, sm0);
      small_store(sm0, 0);
    }
    for (int u = 0, tile = first; tile < ntiles; ++u, tile += step) {
      const int b = u & 1;
      const int it = grp + u * C::NGRP;
      const int s = it & 1;
      const uint32_t use = (uint32_t)it >> 1;
      if (gtid == 0) {
        bool ok = true;
        if (use >= 1) ok = mbar_wait(empty + s, (use - 1) & 1, abort_s);
        if (!ok) {
          atomicOr(a.status, ST_WAIT_TIMEOUT);
          *abort_s = 1;
        }
        pabort_s[grp] = *abort_s;
      }
      // this tile's staged data is complete, the group is done with the
      // other buffer and with the shifted rows, and stage s is free
      asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "n"(GT) : "memory");
      if (pabort_s[grp]) break;
      // the previous tile's products, issued by the group's last thread (it
      // has no face item and one row piece at most): its wait and issue
      // overlap the other threads' loads instead of delaying the barrier
      if (gtid == GT - 1 && pending >= 0) {
        const int ps = pending & 1;
        if (!mbar_wait(full + ps, ((uint32_t)pending >> 1) & 1, abort_s)) {
          atomicOr(a.status, ST_WAIT_TIMEOUT);
          *abort_s = 1;
        } else {
          tc_fence_after();
          issue_products(ps);
          tc_commit(done + ps);
          ++issued;
          last_issued = pending;
        }
        pending = -1;
      }
      const int e0 = tile * EPB;
      const int ne = imin(EPB, EOWN - e0);
      const int32_t* conn_b = conn_of(b);
      const float* fs_b = fs_of(b);
      const float* u0_b = u0_of(b);
      const float* pg_b = geo_of(b);
      unsigned char* ahi = smem_raw + C::OFF_A + (2 * s) * C::A_BYTES;
      unsigned char* alo = ahi + C::A_BYTES;

      // ---- every global load of this thread's items first: rows of q and T
      // in 16-byte pieces (item -> piece kc, field c, element e), the
      // neighbours' values at this thread's face nodes (item -> face node
      // fm, element e)
      float4 rv[RR];
#pragma unroll
      for (int j = 0; j < RR; ++j) {
        const int idx = gtid + j * GT;
        const int e = idx % EPB, c = (idx / EPB) % NU, kc = idx / (EPB * NU);
        if (idx < C::ROW_ITEMS && e < ne) {
          const float* src = (c < NC ? a.q + c * EN : a.t_op) + (int64_t)(e0 + e) * NP;
          rv[j] = __ldg(reinterpret_cast<const float4*>(src) + kc);
        }
      }
      float nb[FR][NU];
      int fmode[FR];
#pragma unroll
      for (int j = 0; j < FR; ++j) {
        const int idx = gtid + j * GT;
        const int e = idx % EPB, fm = idx / EPB, f = fm / NFP, m = fm % NFP;
        fmode[j] = -1;
        if (idx < C::FACE_ITEMS && e < ne) {
          const int cn = conn_b[e * NF + f];
          // 0 two-sided average, 1 exterior value, 2 interior value, 3 Mengaldo
          int mode = 2;
          if (cn >= 0) {
            const int en = cn >> 8, pr = cn & 255;
            const int kn = (pr < a.nperm) ? perm_s[pr * NFP + m] : NP;
            if (en >= E || kn >= NP) {
              atomicOr(a.status, ST_BAD_INDEX);
            } else {
              const int64_t gi = (int64_t)en * NP + kn;
#pragma unroll
              for (int c = 0; c < NU; ++c)
                nb[j][c] = __ldg((c < NC ? a.q + c * EN : a.t_op) + gi);
              mode = 0;
            }
          } else {
            const int bf = -(cn + 1);
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
          fmode[j] = mode;
        }
      }
      // one group: the next tile's per-tile data loads with this tile's
      const bool more = tile + step < ntiles;
      Small sm;
      sm.gok = sm.uok = false;
      if (C::NGRP == 1 && more) small_load(tile + step, sm);

      // ---- rows: shift, keep the shifted row, split, store
#pragma unroll
      for (int j = 0; j < RR; ++j) {
        const int idx = gtid + j * GT;
        const int e = idx % EPB, c = (idx / EPB) % NU, kc = idx / (EPB * NU);
        if (idx < C::ROW_ITEMS && e < ne) {
          const float u0 = u0_b[c * EPB + e];
          const float4 x = make_float4(rv[j].x - u0, rv[j].y - u0, rv[j].z - u0, rv[j].w - u0);
          *reinterpret_cast<float4*>(raw + (c * EPB + e) * NP + kc * 4) = x;
          float4 h, l;
          split_f32(x.x, h.x, l.x);
          split_f32(x.y, h.y, l.y);
          split_f32(x.z, h.z, l.z);
          split_f32(x.w, h.w, l.w);
          const int o = canon_off(c * EPB + e, kc * 4, C::LBO_A);
          *reinterpret_cast<float4*>(ahi + o) = h;
          *reinterpret_cast<float4*>(alo + o) = l;
        }
      }
      // the shifted rows are complete
      asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "n"(GT) : "memory");
      // ---- face values fscale * (u* - u0), own values from the shifted rows
#pragma unroll
      for (int j = 0; j < FR; ++j) {
        if (fmode[j] < 0) continue;
        const int idx = gtid + j * GT;
        const int e = idx % EPB, fm = idx / EPB, f = fm / NFP, m = fm % NFP;
        const int k = fn_s[fm];
        const float fsc = fs_b[e * NF + f];
        int mode = fmode[j];
        if (mode == 1 || mode == 3) {
          const int bf = -(conn_b[e * NF + f] + 1);
          float up[NU];
          if (mode == 3) {
            const float* nf = pg_b + e * GEO + DIM * DIM + f * DIM;
            mengaldo_grad_value<float, DIM, NS, true>(a, g, a.bkind[bf], bf, m, NFP, EN,
                                                      (int64_t)(e0 + e) * NP + k, nf[0], nf[1],
                                                      DIM > 2 ? nf[DIM - 1] : 0.f, up);
          } else {
            const int64_t bstride = (int64_t)a.nbf * NFP, bo = (int64_t)bf * NFP + m;
#pragma unroll
            for (int c = 0; c < NU; ++c) up[c] = a.bext[c * bstride + bo];
          }
#pragma unroll
          for (int c = 0; c < NU; ++c) nb[j][c] = up[c];
          mode = 1;
        }
        const int kk = KV + fm;
#pragma unroll
        for (int c = 0; c < NU; ++c) {
          const float u0 = u0_b[c * EPB + e];
          const float um = raw[(c * EPB + e) * NP + k];
          float v;
          if (mode == 0)
            v = ((nb[j][c] - u0) + um) * 0.5f;
          else if (mode == 1)
            v = nb[j][c] - u0;
          else
            v = um;
          float hi, lo;
          split_f32(fsc * v, hi, lo);
          const int o = canon_off(c * EPB + e, kk, C::LBO_A);
          *reinterpret_cast<float*>(ahi + o) = hi;
          *reinterpret_cast<float*>(alo + o) = lo;
        }
      }
      // ---- the epilogue's copy of the geometry; the group's next tile's
      // data (its latency hidden by the other group's work)
      float* geo = geo_s + s * EPB * GEO;
      for (int i = gtid; i < ne * GEO; i += GT) geo[i] = pg_b[i];
      if (more) {
        if (C::NGRP > 1) small_load(tile + step, sm);
        small_store(sm, b ^ 1);
      }
      fence_async_shared();
      mbar_arrive(full + s);
      if (gtid == GT - 1) pending = it;
    }
    // the last tile's products (after a normal end of the loop)
    if (gtid == GT - 1 && pending >= 0 && !*abort_s) {
      const int ps = pending & 1;
      if (!mbar_wait(full + ps, ((uint32_t)pending >> 1) & 1, abort_s)) {
        atomicOr(a.status, ST_WAIT_TIMEOUT);
        *abort_s = 1;
      } else {
        tc_fence_after();
        issue_products(ps);
        tc_commit(done + ps);
        ++issued;
        last_issued = pending;
      }
    }
    // on an early exit, let the products already issued finish before the
    // TMEM is released
    if (gtid == GT - 1 && *abort_s && issued > 0) {
      if (!mbar_wait(done + (last_issued & 1), ((uint32_t)last_issued >> 1) & 1, nullptr))
        atomicOr(a.status, ST_WAIT_TIMEOUT);
    }
  } else {
    // ================= epilogue: one TMEM lane (row) per thread
    const int q4 = warp & 3;
    const int row = 32 * q4 + lane;
    const int c = row / EPB, e = row % EPB;
    const uint32_t lane_base = tmem + ((uint32_t)(32 * q4) << 16);
    for (int it = 0, tile = blockIdx.x; tile < ntiles; ++it, tile += gridDim.x) {
      const int s = it & 1;
      const uint32_t use = (uint32_t)it >> 1;
      // the products of this tile, then (already complete) the producers'
      // arrival, whose release covers the geometry they wrote
      bool ok = mbar_wait(done + s, use & 1, abort_s);
      ok = ok && mbar_wait(full + s, use & 1, abort_s);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) {
          atomicOr(a.status, ST_WAIT_TIMEOUT);
          *abort_s = 1;
        }
        break;
      }
      tc_fence_after();
      const int e0 = tile * EPB;
      const int ne = imin(EPB, EOWN - e0);
      const bool valid = c < NU && e < ne;
      const float* ge = geo_s + s * EPB * GEO + e * GEO;
      float rxe[DIM][DIM], nre[NF][DIM];
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int j = 0; j < DIM; ++j) rxe[r][j] = ge[r * DIM + j];
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < DIM; ++j) nre[f][j] = ge[DIM * DIM + f * DIM + j];
      const uint32_t tb = lane_base + (uint32_t)(s * C::BUF_COLS);
      float* outp = a.out + ((int64_t)(valid ? c : 0) * DIM) * EN + (int64_t)(e0 + e) * NP;
#pragma unroll 1
      for (int i0 = 0; i0 < NP; i0 += 4) {
        uint32_t v[DIM + NF][4];
#pragma unroll
        for (int r = 0; r < DIM; ++r) tc_ld4(tb + r * NP + i0, v[r]);
#pragma unroll
        for (int f = 0; f < NF; ++f) tc_ld4(tb + C::NV + f * NP + i0, v[DIM + f]);
        tc_wait_ld<DIM + NF>(v);
        if (valid) {
#pragma unroll
          for (int j = 0; j < DIM; ++j) {
            float o[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              float gsum = 0.f;
#pragma unroll
              for (int f = 0; f < NF; ++f) gsum += nre[f][j] * __uint_as_float(v[DIM + f][i]);
#pragma unroll
              for (int r = 0; r < DIM; ++r) gsum -= rxe[r][j] * __uint_as_float(v[r][i]);
              o[i] = gsum;
            }
            *reinterpret_cast<float4*>(outp + (int64_t)j * EN + i0) =
                make_float4(o[0], o[1], o[2], o[3]);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(empty + s);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    __syncwarp();
    tc_dealloc(tmem, C::TCOLS);
  }
}

}  // namespace

}  // namespace mgc
