// The elec pair potential for the B200 kernels: Coulomb energy with a
// sigmoidal distance-dependent dielectric,
//   eps(d) = D - (D - D0) / 2 * (2 + 2 d S + d^2 S^2) * exp(-d S),
//   E(d)   = q1 q2 * (C1 / (d eps(d)) - C2),   C2 = C1 / (max_dis eps(max_dis)),
// flat below min_dis - 0.25, a cubic Hermite bridge over
// [min_dis - 0.25, min_dis + 0.25], a cubic fade to zero over
// [max_dis - 1, max_dis], zero beyond (tmol/score/elec/potentials/
// potentials.hh:32-215).  Every region is q1 q2 times a function of d
// alone, so the flat value and both splines are reduced, once per plan, to
// per-unit-charge constants (ElecK) and the kernels evaluate
//   E = q1 q2 * f(d),  dE/dd = q1 q2 * f'(d).
// The constants are computed on the host the way the reference evaluates
// them, including that eps(min_dis) and eps(max_dis) are taken in single
// precision whatever the precision of the op (the reference's template
// deduces its Real from the float argument).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace tmol_b200 {

constexpr int N_ELEC_K = 20;

// Per-unit-charge constants of one plan, in the order of the device array.
template <typename Real>
struct ElecK {
  Real lo_start, lo_end, hi_start, hi_end;  // region bounds
  Real inv_lo_w, inv_hi_w;                  // 1 / spline widths
  Real C1, C2, D, hDD0, S;                  // Coulomb region; hDD0 = (D - D0) / 2
  Real e_min;                               // flat region value
  Real lo[4], hi[4];  // spline coefficients in t = (d - start) / width
};

static_assert(sizeof(ElecK<float>) == N_ELEC_K * sizeof(float), "ElecK layout");

template <typename Real>
__device__ __forceinline__ ElecK<Real> load_elec_k(const Real* k) {
  ElecK<Real> K;
  Real* o = reinterpret_cast<Real*>(&K);
#pragma unroll
  for (int i = 0; i < N_ELEC_K; ++i) o[i] = k[i];
  return K;
}

__device__ __forceinline__ float elec_exp(float x) { return __expf(x); }
__device__ __forceinline__ double elec_exp(double x) { return exp(x); }

// f(d) and f'(d) per unit q1 q2 for d < hi_end (the caller's range test).
template <typename Real, bool GRAD>
__device__ __forceinline__ void elec_eval(Real d, const ElecK<Real>& K, Real& f, Real& df) {
  if (d >= K.lo_end && d < K.hi_start) {
    const Real x = d * K.S;
    const Real ex = elec_exp(-x);
    const Real eps = K.D - K.hDD0 * (Real(2) + x * (Real(2) + x)) * ex;
    const Real r = Real(1) / (d * eps);
    f = K.C1 * r - K.C2;
    if (GRAD) {
      const Real deps = K.hDD0 * x * x * K.S * ex;
      df = -K.C1 * (eps + d * deps) * r * r;
    }
  } else {
    const bool lo = d < K.lo_end;
    const bool flat = d < K.lo_start;
    const Real iw = lo ? K.inv_lo_w : K.inv_hi_w;
    const Real t = (d - (lo ? K.lo_start : K.hi_start)) * iw;
    const Real c0 = flat ? K.e_min : (lo ? K.lo[0] : K.hi[0]);
    const Real c1 = flat ? Real(0) : (lo ? K.lo[1] : K.hi[1]);
    const Real c2 = flat ? Real(0) : (lo ? K.lo[2] : K.hi[2]);
    const Real c3 = flat ? Real(0) : (lo ? K.lo[3] : K.hi[3]);
    f = c0 + t * (c1 + t * (c2 + t * c3));
    if (GRAD) df = (c1 + t * (Real(2) * c2 + Real(3) * t * c3)) * iw;
    if (d >= K.hi_end) {
      f = Real(0);
      df = Real(0);
    }
  }
}

// Host: the constants of ElecK from the five global parameters (in double;
// the kernels round them to their Real).
inline void elec_constants(float D, float D0, float S, float min_dis, float max_dis,
                           double out[N_ELEC_K]) {
  // D - D0 is a float difference in the reference
  const float DD0 = D - D0;
  auto eps_d = [&](double d) {
    return (double)D - 0.5 * DD0 * (2 + 2 * d * S + d * d * S * S) * std::exp(-d * S);
  };
  auto deps_d = [&](double d) { return 0.5 * DD0 * d * d * S * S * S * std::exp(-d * S); };
  auto eps_f = [&](float d) {
    return (float)((double)D - 0.5 * DD0 * (2 + 2 * d * S + d * d * S * S) * std::exp(-d * S));
  };
  const double C1 = 322.0637;
  const double lo_start = min_dis - 0.25, lo_end = min_dis + 0.25;
  const double hi_start = max_dis - 1.0, hi_end = max_dis;
  const double C2 = C1 / (double)(max_dis * eps_f(max_dis));
  const double e_min = C1 / (double)(min_dis * eps_f(min_dis)) - C2;
  auto coulomb = [&](double d, double& E, double& dE) {
    const double e = eps_d(d), de = deps_d(d);
    E = C1 / (d * e) - C2;
    dE = -C1 * (e + d * de) / (d * d * e * e);
  };
  // Hermite from (x0, p0, m0) to (x1, p1, m1) as p0 + t (c1 + t (c2 + t c3)),
  // t = (x - x0) / (x1 - x0) (tmol/score/common/cubic_hermite_polynomial.hh)
  auto hermite = [](double x0, double p0, double m0, double x1, double p1, double m1, double* c) {
    const double h = x1 - x0, dp0 = m0 * h, dp1 = m1 * h;
    c[0] = p0;
    c[1] = dp0;
    c[2] = -2 * dp0 - dp1 - 3 * p0 + 3 * p1;
    c[3] = dp0 + dp1 + 2 * p0 - 2 * p1;
  };
  double E_le, dE_le, E_hs, dE_hs;
  coulomb(lo_end, E_le, dE_le);
  coulomb(hi_start, E_hs, dE_hs);
  out[0] = lo_start;
  out[1] = lo_end;
  out[2] = hi_start;
  out[3] = hi_end;
  out[4] = 1.0 / (lo_end - lo_start);
  out[5] = 1.0 / (hi_end - hi_start);
  out[6] = C1;
  out[7] = C2;
  out[8] = D;
  out[9] = 0.5 * DD0;
  out[10] = S;
  out[11] = e_min;
  hermite(lo_start, e_min, 0.0, lo_end, E_le, dE_le, out + 12);
  hermite(hi_start, E_hs, dE_hs, hi_end, 0.0, 0.0, out + 16);
}

}  // namespace tmol_b200
