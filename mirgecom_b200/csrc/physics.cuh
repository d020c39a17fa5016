// Pointwise gas physics for the DG right-hand side kernels.
//
// Restates, per node and in registers:
//   * IdealSingleGas            mirgecom/eos.py:302-537
//   * PyrometheusMixture        mirgecom/eos.py:540-888 with the fixed-count
//                               Newton of mirgecom/thermochemistry.py:99-167
//   * SimpleTransport           mirgecom/transport.py:143-202
//   * PowerLawTransport         mirgecom/transport.py:205-321
//   * inviscid flux             mirgecom/inviscid.py:65-102
//   * viscous flux              mirgecom/viscous.py:72-293
//   * Rusanov / HLL / central   mirgecom/flux.py:45-177, inviscid.py:105-287
//   * Arrhenius source terms    mirgecom/eos.py:858-875 (pyrometheus rates,
//                               concentration floor thermochemistry.py:87-94)
// Templated on the arithmetic type R (double for the plain path, float for
// the mixed-precision path).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <cstring>

#define MGC_MAX_SPECIES 16
#define MGC_MAX_REACTIONS 8

namespace mgc {

enum EosKind { EOS_IDEAL = 0, EOS_MIXTURE = 1 };
enum TransportKind { TR_NONE = 0, TR_SIMPLE = 1, TR_POWERLAW = 2 };
enum FluxKind { FLUX_RUSANOV = 0, FLUX_HLL = 1, FLUX_CENTRAL = 2 };

// Gas model parameters, passed by value to every kernel.
struct GasParams {
  int32_t eos_kind;
  int32_t nspecies;
  int32_t niter;            // Newton iterations of the mixture temperature
  int32_t transport_kind;
  double gamma, gas_const;  // ideal gas
  double mu, mu_b, kappa;   // simple transport
  double pl_alpha, pl_beta, pl_sigma, pl_n;   // power-law transport
  int32_t use_lewis;
  int32_t pad_;
  double diff[MGC_MAX_SPECIES];
  double lewis[MGC_MAX_SPECIES];
  double zero_level;        // concentration floor
};

// Mechanism tables (SI units), uploaded once.  T is the coefficient type:
// the float64 kernels read MechanismT<double>, the float32 ones a float copy
// (each coefficient rounded once on the host), so no kernel converts
// coefficients at run time.
template <class T>
struct MechanismT {
  int32_t nspecies, nreactions;
  T mw[MGC_MAX_SPECIES];
  T inv_mw[MGC_MAX_SPECIES];
  T t_mid[MGC_MAX_SPECIES];
  T a_lo[MGC_MAX_SPECIES][7];
  T a_hi[MGC_MAX_SPECIES][7];
  T ord_f[MGC_MAX_REACTIONS][MGC_MAX_SPECIES];
  T nu_p[MGC_MAX_REACTIONS][MGC_MAX_SPECIES];
  T nu_net[MGC_MAX_REACTIONS][MGC_MAX_SPECIES];
  T dnu[MGC_MAX_REACTIONS];
  T log_a[MGC_MAX_REACTIONS];
  T beta[MGC_MAX_REACTIONS];
  T t_act[MGC_MAX_REACTIONS];
  int32_t reversible[MGC_MAX_REACTIONS];
  // derived at upload: enthalpy coefficients (a0, a1/2, a2/3, a3/4, a4/5, a5)
  // and entropy coefficients (a0, a1, a2/2, a3/3, a4/4, a6), low / high range
  T h_lo[MGC_MAX_SPECIES][6], h_hi[MGC_MAX_SPECIES][6];
  T s_lo[MGC_MAX_SPECIES][6], s_hi[MGC_MAX_SPECIES][6];
  // derived at upload: bound on |c_v'(T)| / (2 c_v(T)) (1/K) over the
  // species and the NASA-7 temperature range, the quadratic-convergence
  // constant of the temperature Newton iteration
  T newton_k;
};
using Mechanism = MechanismT<double>;

// one copy of each per translation unit, filled by mgc_set_mechanism()
static __constant__ MechanismT<double> c_mech;
static __constant__ MechanismT<float> c_mech32;

template <class R> __device__ __forceinline__ const MechanismT<R>& mech();
template <> __device__ __forceinline__ const MechanismT<double>& mech<double>() { return c_mech; }
template <> __device__ __forceinline__ const MechanismT<float>& mech<float>() { return c_mech32; }

// float copy of the device mechanism (every coefficient rounded to nearest)
static inline MechanismT<float> narrow_mechanism(const Mechanism& d) {
  MechanismT<float> f;
  memset(&f, 0, sizeof(f));
  f.nspecies = d.nspecies;
  f.nreactions = d.nreactions;
  auto cp = [](float* dst, const double* src, int n) {
    for (int i = 0; i < n; ++i) dst[i] = (float)src[i];
  };
  constexpr int S = MGC_MAX_SPECIES, R = MGC_MAX_REACTIONS;
  cp(f.mw, d.mw, S);
  cp(f.inv_mw, d.inv_mw, S);
  cp(f.t_mid, d.t_mid, S);
  cp(&f.a_lo[0][0], &d.a_lo[0][0], S * 7);
  cp(&f.a_hi[0][0], &d.a_hi[0][0], S * 7);
  cp(&f.ord_f[0][0], &d.ord_f[0][0], R * S);
  cp(&f.nu_p[0][0], &d.nu_p[0][0], R * S);
  cp(&f.nu_net[0][0], &d.nu_net[0][0], R * S);
  cp(f.dnu, d.dnu, R);
  cp(f.log_a, d.log_a, R);
  cp(f.beta, d.beta, R);
  cp(f.t_act, d.t_act, R);
  for (int i = 0; i < R; ++i) f.reversible[i] = d.reversible[i];
  cp(&f.h_lo[0][0], &d.h_lo[0][0], S * 6);
  cp(&f.h_hi[0][0], &d.h_hi[0][0], S * 6);
  cp(&f.s_lo[0][0], &d.s_lo[0][0], S * 6);
  cp(&f.s_hi[0][0], &d.s_hi[0][0], S * 6);
  f.newton_k = (float)d.newton_k;
  return f;
}

constexpr double kGasConstant = 8314.46261815324;
constexpr double kOneAtm = 101325.0;

// status bits written by kernels (never trapped)
enum StatusBits {
  ST_NAN = 1,
  ST_BAD_INDEX = 2,
  ST_NEWTON_MISS = 4,
  ST_NONPOSITIVE = 8,
  ST_WAIT_TIMEOUT = 16,   // a bounded wait inside a pipelined kernel ran out
};

template <class R> __device__ __forceinline__ R rsqrt_(R x);
template <> __device__ __forceinline__ double rsqrt_<double>(double x) { return 1.0 / sqrt(x); }
template <> __device__ __forceinline__ float rsqrt_<float>(float x) { return rsqrtf(x); }

// {{{ NASA-7 thermochemistry

// Powers of T shared by every species of one NASA-7 evaluation.
template <class R>
struct TPow {
  R t, t2, t3, t4, it;
  __device__ __forceinline__ explicit TPow(R tt)
      : t(tt), t2(tt * tt), t3(tt * tt * tt), t4(tt * tt * tt * tt), it(R(1) / tt) {}
};

// cp/R and h/RT of species s (high range when t > t_mid).  Both ranges are
// evaluated and the result selected: the coefficient addresses then depend
// on the species only, so every lane of a warp reads the same constants
// (a per-lane choice of table would serialise the constant-cache reads).
template <class R>
__device__ __forceinline__ void nasa_cp_h(int s, const TPow<R>& p, R& cp, R& h) {
  const MechanismT<R>& m = mech<R>();
  const R* al = m.a_lo[s];
  const R* ah = m.a_hi[s];
  const R* bl = m.h_lo[s];
  const R* bh = m.h_hi[s];
  const R cpl = al[0] + al[1] * p.t + al[2] * p.t2 + al[3] * p.t3 + al[4] * p.t4;
  const R cph = ah[0] + ah[1] * p.t + ah[2] * p.t2 + ah[3] * p.t3 + ah[4] * p.t4;
  const R hl = bl[0] + bl[1] * p.t + bl[2] * p.t2 + bl[3] * p.t3 + bl[4] * p.t4 + bl[5] * p.it;
  const R hh = bh[0] + bh[1] * p.t + bh[2] * p.t2 + bh[3] * p.t3 + bh[4] * p.t4 + bh[5] * p.it;
  const bool hi = p.t > m.t_mid[s];
  cp = hi ? cph : cpl;
  h = hi ? hh : hl;
}

template <class R>
__device__ __forceinline__ R species_cp_r(int s, R t) {
  R cp, h;
  nasa_cp_h<R>(s, TPow<R>(t), cp, h);
  return cp;
}

template <class R>
__device__ __forceinline__ R species_h_rt(int s, R t) {
  R cp, h;
  nasa_cp_h<R>(s, TPow<R>(t), cp, h);
  return h;
}

// s/R of species s given log(t) (both ranges evaluated, as in nasa_cp_h)
template <class R>
__device__ __forceinline__ R species_s_r(int s, const TPow<R>& p, R logt) {
  const MechanismT<R>& m = mech<R>();
  const R* cl = m.s_lo[s];
  const R* ch = m.s_hi[s];
  const R sl = cl[0] * logt + cl[1] * p.t + cl[2] * p.t2 + cl[3] * p.t3 + cl[4] * p.t4 + cl[5];
  const R sh = ch[0] * logt + ch[1] * p.t + ch[2] * p.t2 + ch[3] * p.t3 + ch[4] * p.t4 + ch[5];
  return p.t > m.t_mid[s] ? sh : sl;
}

// mixture e (J/kg) and c_v (J/kg/K) at temperature t
template <class R, int NS>
__device__ __forceinline__ void mixture_e_cv(const R* y, R t, R& e, R& cv) {
  const TPow<R> p(t);
  R se = 0, scv = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    R cps, hs;
    nasa_cp_h<R>(s, p, cps, hs);
    const R yw = y[s] * mech<R>().inv_mw[s];
    se += yw * (hs - (R)1);
    scv += yw * (cps - (R)1);
  }
  e = (R)kGasConstant * t * se;
  cv = (R)kGasConstant * scv;
}

template <class R, int NS>
__device__ __forceinline__ R mixture_gas_const(const R* y) {
  R s = 0;
#pragma unroll
  for (int k = 0; k < NS; ++k) s += y[k] * mech<R>().inv_mw[k];
  return (R)kGasConstant * s;
}

// mixture c_p and the species enthalpies (J/kg) in one NASA-7 pass
template <class R, int NS>
__device__ __forceinline__ R mixture_cp_and_h(const R* y, R t, R* h) {
  const TPow<R> p(t);
  R s = 0;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    R cps, hs;
    nasa_cp_h<R>(k, p, cps, hs);
    s += y[k] * cps * mech<R>().inv_mw[k];
    h[k] = ((R)kGasConstant * mech<R>().inv_mw[k]) * t * hs;
  }
  return (R)kGasConstant * s;
}

template <class R, int NS>
__device__ __forceinline__ R mixture_cp(const R* y, R t) {
  R h[NS];
  return mixture_cp_and_h<R, NS>(y, t, h);
}

// c^o for a concentration c >= 0 and a positive order o
template <class R>
__device__ __forceinline__ R conc_pow(R c, R o) {
  if (o == R(1)) return c;
  if constexpr (sizeof(R) == 4) {
    return c > 0.f ? expf(o * logf(c)) : 0.f;
  } else {
    return pow(c, o);
  }
}

// T_{i+1} = T_i + (e - e(T_i)) / c_v(T_i), fixed count
template <class R, int NS>
__device__ __forceinline__ R newton_temperature(R e, R tguess, const R* y, int niter) {
  R t = tguess;
  for (int it = 0; it < niter; ++it) {
    R em, cv;
    mixture_e_cv<R, NS>(y, t, em, cv);
    t = t + (e - em) / cv;
  }
  return t;
}

// Newton inputs of the mixed form from a float32 conserved state: mass
// fractions and specific internal energy in float64 (one reciprocal of rho)
// and their float32 roundings.
template <int DIM, int NS>
__device__ __forceinline__ void mixed_newton_inputs(const float* qq, float* y, double* yd,
                                                    float& e32, double& e64) {
  const double irho = 1.0 / (double)qq[0];
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    yd[k] = (double)qq[2 + DIM + k] * irho;
    y[k] = (float)yd[k];
  }
  double ked = 0;
#pragma unroll
  for (int i = 0; i < DIM; ++i) ked += (double)qq[2 + i] * (double)qq[2 + i];
  e64 = ((double)qq[1] - 0.5 * ked * irho) * irho;
  e32 = (float)e64;
}

// Mixed-precision temperature solve of one node from the start value *t*.
// Newton converges quadratically: after a step dT the remaining error is
// about k dT^2, k = max |c_v'| / (2 c_v) (Mechanism::newton_k).  The float32
// iterations stop once that predicted error is a quarter of the error the
// final float64 step can absorb; the float64 residual then gives the last
// correction, accepted when its own predicted remainder k corr^2 is at most
// rtol |T| (the relative temperature-update tolerance the reference drivers
// check: mirgecom examples/autoignition.py:526-530).  Returns acceptance;
// *used* counts float32 iterations.
template <int NS>
__device__ __forceinline__ bool mixed_newton(const float* y, const double* yd, float e32,
                                             double e64, float& t, int maxit, double rtol,
                                             int& used) {
  const float k = mech<float>().newton_k;
  const float rt = (float)rtol;
  for (int it = 0; it < maxit; ++it) {
    float em, cv;
    mixture_e_cv<float, NS>(y, t, em, cv);
    const float dt = (e32 - em) / cv;
    t += dt;
    ++used;
    if (k * dt * dt <= 0.25f * sqrtf(rt * fabsf(t) / k)) break;
  }
  double em, cv;
  mixture_e_cv<double, NS>(yd, (double)t, em, cv);
  const double corr = (e64 - em) / cv;
  const bool ok = t > 0.f && corr == corr &&
                  mech<double>().newton_k * corr * corr <= rtol * fabs((double)t);
  if (ok) t = (float)((double)t + corr);
  return ok;
}

// net molar production rates (kmol/m^3/s)
template <class R, int NS>
__device__ __forceinline__ void production_rates(R rho, R t, const R* y, R zero_level,
                                                 R* omega) {
  R conc[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    R c = mech<R>().inv_mw[k] * rho * y[k];
    conc[k] = (c < zero_level) ? (R)0 : c;
    omega[k] = 0;
  }
  const R logt = log(t);
  const R invt = (R)1 / t;
  const TPow<R> tp(t);
  for (int i = 0; i < mech<R>().nreactions; ++i) {
    const R kf = exp(mech<R>().log_a[i] + mech<R>().beta[i] * logt - mech<R>().t_act[i] * invt);
    R rf = kf;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const R o = mech<R>().ord_f[i][k];
      if (o != (R)0) rf = rf * conc_pow<R>(conc[k], o);
    }
    R r = rf;
    if (mech<R>().reversible[i]) {
      R dg = 0;
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const R nu = mech<R>().nu_net[i][k];
        if (nu != (R)0) {
          R cps, hs;
          nasa_cp_h<R>(k, tp, cps, hs);
          dg += nu * (hs - species_s_r<R>(k, tp, logt));
        }
      }
      const R log_kc = -dg + mech<R>().dnu[i] * log((R)kOneAtm / ((R)kGasConstant * t));
      R rr = kf * exp(-log_kc);
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const R o = mech<R>().nu_p[i][k];
        if (o != (R)0) rr = rr * conc_pow<R>(conc[k], o);
      }
      r = rf - rr;
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) omega[k] += mech<R>().nu_net[i][k] * r;
  }
}

// }}}

// {{{ fluid state at one node

template <class R, int DIM, int NS>
struct NodeState {
  R rho, rhoe, mom[DIM], rhoy[NS > 0 ? NS : 1];
  R v[DIM], y[NS > 0 ? NS : 1];
  R p, t, c, gamma, cv;
  R h[NS > 0 ? NS : 1];
  R mu, mub, kappa, d[NS > 0 ? NS : 1];
};

// Fill the thermodynamic state.  For the ideal gas the temperature is
// computed from q; for mixtures *t_in* is the converged temperature.
//
// Per-node quotients by the density: float64 divides as the reference does;
// float32 multiplies by the correctly rounded reciprocal (one division per
// node instead of ~40 in the state and the viscous flux; at most one more
// rounding per quotient).
template <class R>
__device__ __forceinline__ R per_rho(R x, R rho, R irho) {
  if constexpr (sizeof(R) == 4) {
    return x * irho;
  } else {
    (void)irho;
    return x / rho;
  }
}

template <class R, int DIM, int NS>
__device__ __forceinline__ void make_state(const R* q, R t_in, const GasParams& g,
                                           NodeState<R, DIM, NS>& s) {
  s.rho = q[0];
  s.rhoe = q[1];
  R ke = 0;
  const R irho = (R)1 / s.rho;
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    s.mom[i] = q[2 + i];
    ke += s.mom[i] * s.mom[i];
  }
  ke = per_rho((R)0.5 * ke, s.rho, irho);
#pragma unroll
  for (int i = 0; i < DIM; ++i) s.v[i] = per_rho(s.mom[i], s.rho, irho);
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    s.rhoy[k] = q[2 + DIM + k];
    s.y[k] = per_rho(s.rhoy[k], s.rho, irho);
  }
  if (g.eos_kind == EOS_IDEAL) {
    const R gam = (R)g.gamma;
    const R eint = s.rhoe - ke;
    s.p = eint * (gam - (R)1);
    s.t = (((gam - (R)1) / (R)g.gas_const) * eint) / s.rho;
    s.c = sqrt(gam / s.rho * s.p);
    s.gamma = gam;
    s.cv = (R)g.gas_const / (gam - (R)1);
  } else {
    if constexpr (NS > 0) {
      s.t = t_in;
      const R rmix = mixture_gas_const<R, NS>(s.y);
      s.p = s.rho * rmix * s.t;
      const R cp = mixture_cp_and_h<R, NS>(s.y, s.t, s.h);
      s.gamma = cp / (cp - rmix);
      s.cv = cp - rmix;
      s.c = sqrt(s.gamma * s.p / s.rho);
    }
  }
  // transport
  if (g.transport_kind == TR_SIMPLE) {
    s.mu = (R)g.mu;
    s.mub = (R)g.mu_b;
    s.kappa = (R)g.kappa;
#pragma unroll
    for (int k = 0; k < NS; ++k) s.d[k] = (R)g.diff[k];
  } else if (g.transport_kind == TR_POWERLAW) {
    s.mu = (R)g.pl_beta * pow(s.t, (R)g.pl_n);
    s.mub = (R)g.pl_alpha * s.mu;
    s.kappa = (R)g.pl_sigma * s.mu * s.cv;
#pragma unroll
    for (int k = 0; k < NS; ++k)
      s.d[k] = g.use_lewis ? (R)g.pl_sigma * s.mu / (s.rho * (R)g.lewis[k] * s.gamma)
                           : (R)g.diff[k];
  } else {
    s.mu = s.mub = s.kappa = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k) s.d[k] = 0;
  }
}

// Inviscid-only state from q and the node's p, c, gamma (computed before by
// make_state): all the numerical inviscid fluxes need.
template <class R, int DIM, int NS>
__device__ __forceinline__ void make_state_light(const R* q, R p, R c, R gamma,
                                                 NodeState<R, DIM, NS>& s) {
  s.rho = q[0];
  s.rhoe = q[1];
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    s.mom[i] = q[2 + i];
    s.v[i] = s.mom[i] / s.rho;
  }
#pragma unroll
  for (int k = 0; k < NS; ++k) s.rhoy[k] = q[2 + DIM + k];
  s.p = p;
  s.c = c;
  s.gamma = gamma;
}

// Temperature of a node from q (ideal: closed form; mixture: Newton from seed)
template <class R, int DIM, int NS>
__device__ __forceinline__ R node_temperature(const R* q, R seed, const GasParams& g) {
  R ke = 0;
#pragma unroll
  for (int i = 0; i < DIM; ++i) ke += q[2 + i] * q[2 + i];
  ke = (R)0.5 * ke / q[0];
  if (g.eos_kind == EOS_IDEAL) {
    const R gam = (R)g.gamma;
    return (((gam - (R)1) / (R)g.gas_const) * (q[1] - ke)) / q[0];
  }
  if constexpr (NS > 0) {
    R y[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) y[k] = q[2 + DIM + k] / q[0];
    const R e = (q[1] - ke) / q[0];
    return newton_temperature<R, NS>(e, seed, y, g.niter);
  }
  return seed;
}

template <class R, int DIM, int NS>
__device__ __forceinline__ R wavespeed(const NodeState<R, DIM, NS>& s) {
  R v2 = 0;
#pragma unroll
  for (int i = 0; i < DIM; ++i) v2 += s.v[i] * s.v[i];
  return sqrt(v2) + s.c;
}

// }}}

// {{{ fluxes

// inviscid flux dotted with n: F_I(q) . n   (mirgecom/inviscid.py:65-102)
template <class R, int DIM, int NS>
__device__ __forceinline__ void inviscid_flux_n(const NodeState<R, DIM, NS>& s, const R* n,
                                                R* fn) {
  R vn = 0, mn = 0;
#pragma unroll
  for (int j = 0; j < DIM; ++j) {
    vn += s.v[j] * n[j];
    mn += s.mom[j] * n[j];
  }
  fn[0] = mn;
  fn[1] = vn * (s.rhoe + s.p);
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    R a = 0;
#pragma unroll
    for (int j = 0; j < DIM; ++j) a += (s.rho * s.v[i] * s.v[j] + ((i == j) ? s.p : (R)0)) * n[j];
    fn[2 + i] = a;
  }
#pragma unroll
  for (int k = 0; k < NS; ++k) fn[2 + DIM + k] = vn * s.rhoy[k];
}

// full inviscid flux F_I[c][j]
template <class R, int DIM, int NS>
__device__ __forceinline__ void inviscid_flux(const NodeState<R, DIM, NS>& s,
                                              R (*f)[DIM]) {
#pragma unroll
  for (int j = 0; j < DIM; ++j) {
    f[0][j] = s.mom[j];
    f[1][j] = s.v[j] * (s.rhoe + s.p);
#pragma unroll
    for (int i = 0; i < DIM; ++i)
      f[2 + i][j] = s.rho * s.v[i] * s.v[j] + ((i == j) ? s.p : (R)0);
#pragma unroll
    for (int k = 0; k < NS; ++k) f[2 + DIM + k][j] = s.v[j] * s.rhoy[k];
  }
}

// viscous flux F_V[c][j] from gradients gq[c][j] (c < NC) and gt[j]
template <class R, int DIM, int NS, bool MIXTURE>
__device__ __forceinline__ void viscous_flux(const NodeState<R, DIM, NS>& s,
                                             const R (*gq)[DIM], const R* gt,
                                             R (*f)[DIM]) {
  const R irho = (R)1 / s.rho;
  R gv[DIM][DIM];
  R divv = 0;
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
#pragma unroll
    for (int j = 0; j < DIM; ++j) gv[i][j] = per_rho(gq[2 + i][j] - s.v[i] * gq[0][j], s.rho, irho);
    divv += gv[i][i];
  }
  R tau[DIM][DIM];
  const R lam = (s.mub - (R)2 * s.mu / (R)3) * divv;
#pragma unroll
  for (int i = 0; i < DIM; ++i)
#pragma unroll
    for (int j = 0; j < DIM; ++j)
      tau[i][j] = s.mu * (gv[i][j] + gv[j][i]) + ((i == j) ? lam : (R)0);
#pragma unroll
  for (int j = 0; j < DIM; ++j) {
    f[0][j] = 0;
    R ef = 0;
#pragma unroll
    for (int i = 0; i < DIM; ++i) ef += tau[j][i] * s.v[i];
    ef = ef + s.kappa * gt[j];
#pragma unroll
    for (int i = 0; i < DIM; ++i) f[2 + i][j] = tau[i][j];
    f[1][j] = ef;
  }
  if constexpr (NS > 0) {
    R gy[NS][DIM];
#pragma unroll
    for (int k = 0; k < NS; ++k)
#pragma unroll
      for (int j = 0; j < DIM; ++j)
        gy[k][j] = per_rho(gq[2 + DIM + k][j] - s.y[k] * gq[0][j], s.rho, irho);
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      if constexpr (MIXTURE) {
        R sum_dgy = 0;
#pragma unroll
        for (int k = 0; k < NS; ++k) sum_dgy += s.d[k] * gy[k][j];
        R qd = 0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          const R jk = -s.rho * (s.d[k] * gy[k][j] - s.y[k] * sum_dgy);
          qd += s.h[k] * jk;
          f[2 + DIM + k][j] = -jk;
        }
        f[1][j] = f[1][j] - qd;
      } else {
#pragma unroll
        for (int k = 0; k < NS; ++k) f[2 + DIM + k][j] = s.rho * (s.d[k] * gy[k][j]);
      }
    }
  }
}

// numerical inviscid flux F*_I . n between interior (m) and exterior (p)
template <class R, int DIM, int NS>
__device__ __forceinline__ void inviscid_num_flux(const NodeState<R, DIM, NS>& sm,
                                                  const NodeState<R, DIM, NS>& sp,
                                                  const R* qm, const R* qp, const R* n,
                                                  int kind, R* out) {
  constexpr int NC = DIM + 2 + NS;
  R fm[NC], fp[NC];
  inviscid_flux_n<R, DIM, NS>(sm, n, fm);
  inviscid_flux_n<R, DIM, NS>(sp, n, fp);
  if (kind == FLUX_HLL) {
    R u_int = 0, u_ext = 0;
#pragma unroll
    for (int j = 0; j < DIM; ++j) {
      u_int += sm.v[j] * n[j];
      u_ext += sp.v[j] * n[j];
    }
    const R p_star = ((R)0.5 * (sm.p + sp.p) +
                      ((R)1 / (R)8) * (u_int - u_ext) * (sm.rho + sp.rho) * (sm.c + sp.c));
    const R q_int = (R)1 + (sm.gamma + (R)1) / ((R)2 * sm.gamma) * (p_star / sm.p - (R)1);
    const R q_ext = (R)1 + (sp.gamma + (R)1) / ((R)2 * sp.gamma) * (p_star / sp.p - (R)1);
    const R q_int_rt = sqrt((p_star > sm.p) ? q_int : (R)1);
    const R q_ext_rt = sqrt((p_star > sp.p) ? q_ext : (R)1);
    const R s_minus = u_int - sm.c * q_int_rt;
    const R s_plus = u_ext + sp.c * q_ext_rt;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      R f = (s_plus * fm[c] - s_minus * fp[c] + s_plus * s_minus * (qp[c] - qm[c])) /
            (s_plus - s_minus);
      if (s_minus >= (R)0) f = fm[c];
      if (s_plus <= (R)0) f = fp[c];
      out[c] = f;
    }
  } else {
    const R lam = (kind == FLUX_RUSANOV)
                      ? fmax(wavespeed<R, DIM, NS>(sm), wavespeed<R, DIM, NS>(sp))
                      : (R)0;
#pragma unroll
    for (int c = 0; c < NC; ++c) out[c] = (fm[c] + fp[c] + lam * (qm[c] - qp[c])) * (R)0.5;
  }
}

// }}}

}  // namespace mgc
