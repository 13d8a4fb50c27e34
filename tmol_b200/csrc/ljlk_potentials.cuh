// LJ and LK isotropic pair potentials for the B200 kernels.
//
// The mathematics is tmol's (beta_nov2016 LJ with linear region, cubic
// fade-out and atr/rep split; Lazaridis-Karplus Gaussian solvation with
// flat/close-spline/exact/far-spline regions), restated for device code:
//   count-pair weight   tmol/score/ljlk/potentials/common.hh:14-22
//   LJ sigma rule       tmol/score/ljlk/potentials/common.hh:25-44
//   LJ                  tmol/score/ljlk/potentials/lj.hh:22-178
//   LK                  tmol/score/ljlk/potentials/lk_isotropic.hh:23-361
//   Hermite splines     tmol/score/common/cubic_hermite_polynomial.hh:34-137
// Type parameters arrive as struct AtomParams (one per atom, staged in
// shared memory by the scoring kernel); sqrt/exp/floor/division are CUDA's.
#pragma once

#include <cuda_runtime.h>

namespace tmol_b200 {

enum AtomFlags : int {
  kDonor = 1,
  kHydroxyl = 2,
  kPolarH = 4,
  kAcceptor = 8,
  kCarbonLK = 16,
  kHeavy = 32,
};

template <typename Real>
struct GlobalParams {
  Real max_dis;
  Real lj_dlin_sigma_factor;
  Real lj_hbond_dis;
  Real lj_hbond_OH_donor_dis;
  Real lj_hbond_hdis;
};

template <typename Real>
struct AtomParams {
  Real lj_radius, lj_wdepth, lk_dgfree, lk_lambda, lk_volume;
  int flags;
};

template <typename Real>
__device__ __forceinline__ Real connectivity_weight(int sep) {
  return sep > 4 ? Real(1) : (sep == 4 ? Real(0.2) : Real(0));
}

template <typename Real>
__device__ __forceinline__ Real lj_sigma(int fi, Real ri, int fj, Real rj,
                                         const GlobalParams<Real>& g) {
  bool di = fi & kDonor, dj = fj & kDonor;
  bool ai = fi & kAcceptor, aj = fj & kAcceptor;
  if ((di && aj) || (dj && ai)) {
    if ((di && (fi & kHydroxyl)) || (dj && (fj & kHydroxyl)))
      return g.lj_hbond_OH_donor_dis;
    return g.lj_hbond_dis;
  }
  if (((fi & kPolarH) && aj) || ((fj & kPolarH) && ai)) return g.lj_hbond_hdis;
  return ri + rj;
}

template <typename Real>
__device__ __forceinline__ Real hermite(Real x, Real x0, Real p0, Real dpdx0,
                                        Real x1, Real p1, Real dpdx1) {
  Real h = x1 - x0;
  Real t = (x - x0) / h;
  Real dp0 = dpdx0 * h, dp1 = dpdx1 * h;
  return p0 + t * (dp0 + t * (-2 * dp0 - dp1 - 3 * p0 + 3 * p1 +
                              t * (dp0 + dp1 + 2 * p0 - 2 * p1)));
}

template <typename Real>
__device__ __forceinline__ void hermite_V_dV(Real x, Real x0, Real p0,
                                             Real dpdx0, Real x1, Real p1,
                                             Real dpdx1, Real& V, Real& dV) {
  Real h = x1 - x0;
  Real t = (x - x0) / h;
  Real dp0 = dpdx0 * h, dp1 = dpdx1 * h;
  V = p0 + t * (dp0 + t * (-2 * dp0 - dp1 - 3 * p0 + 3 * p1 +
                           t * (dp0 + dp1 + 2 * p0 - 2 * p1)));
  dV = (dp0 + t * (-4 * dp0 - 2 * dp1 - 6 * p0 + 6 * p1 +
                   t * (3 * dp0 + 3 * dp1 + 6 * p0 - 6 * p1))) /
       h;
}

template <typename Real>
__device__ __forceinline__ Real hermite_to_zero(Real x, Real x0, Real p0,
                                                Real dpdx0, Real x1) {
  Real h = x1 - x0;
  Real t = (x - x0) / h;
  Real dp0 = dpdx0 * h;
  return p0 + t * (dp0 + t * (-2 * dp0 - 3 * p0 + t * (dp0 + 2 * p0)));
}

template <typename Real>
__device__ __forceinline__ void hermite_to_zero_V_dV(Real x, Real x0, Real p0,
                                                     Real dpdx0, Real x1,
                                                     Real& V, Real& dV) {
  Real h = x1 - x0;
  Real t = (x - x0) / h;
  Real dp0 = dpdx0 * h;
  V = p0 + t * (dp0 + t * (-2 * dp0 - 3 * p0 + t * (dp0 + 2 * p0)));
  dV = (dp0 + t * (-4 * dp0 - 6 * p0 + t * (3 * dp0 + 6 * p0))) / h;
}

template <typename Real>
__device__ __forceinline__ void vdw_V_dV(Real dist, Real sigma, Real eps,
                                         Real& V, Real& dV) {
  Real sd = sigma / dist;
  Real sd2 = sd * sd;
  Real sd6 = sd2 * sd2 * sd2;
  Real sd12 = sd6 * sd6;
  V = eps * (sd12 - Real(2) * sd6);
  dV = eps * (Real(-12) * sd12 + Real(12) * sd6) / dist;
}

template <typename Real>
__device__ __forceinline__ Real vdw_V(Real dist, Real sigma, Real eps) {
  Real sd = sigma / dist;
  Real sd2 = sd * sd;
  Real sd6 = sd2 * sd2 * sd2;
  return eps * (sd6 * sd6 - Real(2) * sd6);
}

// LJ knots for one atom pair.
template <typename Real>
struct LJPair {
  Real sigma, eps, d_lin, dmin, dmax;
};

template <typename Real>
__device__ __forceinline__ LJPair<Real> lj_pair(const AtomParams<Real>& i,
                                                const AtomParams<Real>& j,
                                                const GlobalParams<Real>& g) {
  LJPair<Real> q;
  q.sigma = lj_sigma(i.flags, i.lj_radius, j.flags, j.lj_radius, g);
  q.eps = sqrt(i.lj_wdepth * j.lj_wdepth);
  q.d_lin = q.sigma * g.lj_dlin_sigma_factor;
  q.dmax = g.max_dis;
  Real dmin = g.max_dis - Real(1.5);
  if (q.sigma > dmin) dmin = q.sigma;
  if (dmin > q.dmax - Real(0.1)) dmin = q.dmax - Real(0.1);
  q.dmin = dmin;
  return q;
}

// Unweighted LJ energy split into (atr, rep); caller applies the count-pair
// weight.  Matches lj_score::V (lj.hh:65-113) for dist <= max_dis.
template <typename Real>
__device__ __forceinline__ void lj_V(Real dist, const LJPair<Real>& q,
                                     Real& atr, Real& rep) {
  Real lj;
  if (dist > q.dmin) {
    Real v0, dv0;
    vdw_V_dV(q.dmin, q.sigma, q.eps, v0, dv0);
    lj = hermite_to_zero(dist, q.dmin, v0, dv0, q.dmax);
  } else if (dist > q.d_lin) {
    lj = vdw_V(dist, q.sigma, q.eps);
  } else {
    Real v0, dv0;
    vdw_V_dV(q.d_lin, q.sigma, q.eps, v0, dv0);
    lj = v0 + dv0 * (dist - q.d_lin);
  }
  if (dist < q.sigma) {
    atr = -q.eps;
    rep = lj + q.eps;
  } else {
    atr = lj;
    rep = 0;
  }
}

// Unweighted LJ energies and distance derivatives (lj_score::V_dV,
// lj.hh:115-177).
template <typename Real>
__device__ __forceinline__ void lj_V_dV(Real dist, const LJPair<Real>& q,
                                        Real& atr, Real& rep, Real& datr,
                                        Real& drep) {
  Real lj, dlj;
  if (dist < q.d_lin) {
    Real v0, dv0;
    vdw_V_dV(q.d_lin, q.sigma, q.eps, v0, dv0);
    lj = v0 + dv0 * (dist - q.d_lin);
    dlj = dv0;
  } else if (dist < q.dmin) {
    vdw_V_dV(dist, q.sigma, q.eps, lj, dlj);
  } else if (dist < q.dmax) {
    Real v0, dv0;
    vdw_V_dV(q.dmin, q.sigma, q.eps, v0, dv0);
    hermite_to_zero_V_dV(dist, q.dmin, v0, dv0, q.dmax, lj, dlj);
  } else {
    lj = 0;
    dlj = 0;
  }
  if (dist < q.sigma) {
    atr = -q.eps;
    rep = lj + q.eps;
    datr = 0;
    drep = dlj;
  } else {
    atr = lj;
    rep = 0;
    datr = dlj;
    drep = 0;
  }
}

// One direction of the LK Gaussian, f_desolv (lk_isotropic.hh:30-94).
template <typename Real>
__device__ __forceinline__ Real desolv_V(Real dist, Real r_i, Real dg_i,
                                         Real lam_i, Real vol_j) {
  const Real pi_pow1p5 = Real(5.56832799683f);  // a float literal in tmol
  Real x = dist - r_i;
  return -vol_j * dg_i / (Real(2) * pi_pow1p5 * lam_i) / (dist * dist) *
         exp(-x * x / (lam_i * lam_i));
}

template <typename Real>
__device__ __forceinline__ void desolv_V_dV(Real dist, Real r_i, Real dg_i,
                                            Real lam_i, Real vol_j, Real& V,
                                            Real& dV) {
  const Real pi_pow1p5 = Real(5.56832799683f);  // a float literal in tmol
  Real x = dist - r_i;
  Real e = exp(-x * x / (lam_i * lam_i));
  Real c = -vol_j * dg_i / (Real(2) * pi_pow1p5 * lam_i);
  Real inv_d2 = Real(1) / (dist * dist);
  V = c * inv_d2 * e;
  dV = c * e * inv_d2 * (Real(-2) / dist - Real(2) * (dist - r_i) / (lam_i * lam_i));
}

// Shared knots of both LK directions (they depend on sigma and the C-C flag
// only): the flat region ends at close_dmin, the close spline spans
// [close_dmin, close_dmax] with knots on 1/20 A^2 etable bins
// (lk_isotropic.hh:132-143).
template <typename Real>
struct LKKnots {
  Real d_min, close_dmin, close_dmax, far_dmin, far_dmax;
};

template <typename Real>
__device__ __forceinline__ LKKnots<Real> lk_knots(Real sigma, bool cc,
                                                  Real max_dis) {
  LKKnots<Real> k;
  // sigma * .89 is formed in double and rounded, as the reference does
  Real dm = Real(double(sigma) * 0.89);
  if (cc && dm < Real(4.2)) dm = Real(4.2);
  Real n = floor(Real(20) * dm * dm);
  Real lo = n - Real(29);
  Real hi = n + Real(21);
  k.d_min = dm;
  k.close_dmin = sqrt((lo > Real(0) ? lo : Real(0)) / Real(20));
  k.close_dmax = sqrt((hi < Real(405) ? hi : Real(405)) / Real(20));
  k.far_dmax = max_dis;
  k.far_dmin = max_dis - Real(1.5);
  return k;
}

// One LK direction (i desolvated by j), unweighted; lk_isotropic_pair
// (lk_isotropic.hh:97-236).
template <typename Real>
__device__ __forceinline__ Real lk_dir_V(Real dist, const LKKnots<Real>& k,
                                         Real r_i, Real dg_i, Real lam_i,
                                         Real vol_j) {
  if (dist < k.close_dmin) {
    return desolv_V(k.d_min, r_i, dg_i, lam_i, vol_j);
  } else if (dist < k.close_dmax) {
    Real v1, dv1;
    desolv_V_dV(k.close_dmax, r_i, dg_i, lam_i, vol_j, v1, dv1);
    return hermite(dist, k.close_dmin, desolv_V(k.d_min, r_i, dg_i, lam_i, vol_j),
                   Real(0), k.close_dmax, v1, dv1);
  } else if (dist < k.far_dmin) {
    return desolv_V(dist, r_i, dg_i, lam_i, vol_j);
  } else if (dist < k.far_dmax) {
    Real v0, dv0;
    desolv_V_dV(k.far_dmin, r_i, dg_i, lam_i, vol_j, v0, dv0);
    return hermite_to_zero(dist, k.far_dmin, v0, dv0, k.far_dmax);
  }
  return Real(0);
}

template <typename Real>
__device__ __forceinline__ void lk_dir_V_dV(Real dist, const LKKnots<Real>& k,
                                            Real r_i, Real dg_i, Real lam_i,
                                            Real vol_j, Real& V, Real& dV) {
  if (dist < k.close_dmin) {
    V = desolv_V(k.d_min, r_i, dg_i, lam_i, vol_j);
    dV = 0;
  } else if (dist < k.close_dmax) {
    Real v1, dv1;
    desolv_V_dV(k.close_dmax, r_i, dg_i, lam_i, vol_j, v1, dv1);
    hermite_V_dV(dist, k.close_dmin, desolv_V(k.d_min, r_i, dg_i, lam_i, vol_j),
                 Real(0), k.close_dmax, v1, dv1, V, dV);
  } else if (dist < k.far_dmin) {
    desolv_V_dV(dist, r_i, dg_i, lam_i, vol_j, V, dV);
  } else if (dist < k.far_dmax) {
    Real v0, dv0;
    desolv_V_dV(k.far_dmin, r_i, dg_i, lam_i, vol_j, v0, dv0);
    hermite_to_zero_V_dV(dist, k.far_dmin, v0, dv0, k.far_dmax, V, dV);
  } else {
    V = 0;
    dV = 0;
  }
}

// LK isotropic, both directions, unweighted.
template <typename Real>
__device__ __forceinline__ Real lk_V(Real dist, Real sigma,
                                     const AtomParams<Real>& i,
                                     const AtomParams<Real>& j, Real max_dis) {
  bool cc = (i.flags & kCarbonLK) && (j.flags & kCarbonLK);
  LKKnots<Real> k = lk_knots(sigma, cc, max_dis);
  return lk_dir_V(dist, k, i.lj_radius, i.lk_dgfree, i.lk_lambda, j.lk_volume) +
         lk_dir_V(dist, k, j.lj_radius, j.lk_dgfree, j.lk_lambda, i.lk_volume);
}

template <typename Real>
__device__ __forceinline__ void lk_V_dV(Real dist, Real sigma,
                                        const AtomParams<Real>& i,
                                        const AtomParams<Real>& j, Real max_dis,
                                        Real& V, Real& dV) {
  bool cc = (i.flags & kCarbonLK) && (j.flags & kCarbonLK);
  LKKnots<Real> k = lk_knots(sigma, cc, max_dis);
  Real v1, d1, v2, d2;
  lk_dir_V_dV(dist, k, i.lj_radius, i.lk_dgfree, i.lk_lambda, j.lk_volume, v1, d1);
  lk_dir_V_dV(dist, k, j.lj_radius, j.lk_dgfree, j.lk_lambda, i.lk_volume, v2, d2);
  V = v1 + v2;
  dV = d1 + d2;
}

}  // namespace tmol_b200

namespace tmol_b200 {

// ---------------------------------------------------------------------------
// Type-pair tables.  Everything in the two potentials that depends only on
// the two atom types (sigma, epsilon, region boundaries and the function
// values and slopes at the spline knots) is computed once per plan for every
// ordered pair of the atom types a PoseStack uses.  Per atom pair the kernels
// then evaluate one region: the LJ linear extension, the 12-6 form or the
// fade-out cubic; the LK flat value, the close cubic, the two Gaussians, or
// the fade-out cubic.  LK splines of the two directions share their knots,
// so the table stores the sums of both directions' knot values and one
// cubic is evaluated for the pair.

template <typename Real>
struct alignas(4 * sizeof(Real)) LJRecord {  // 8 values, two groups of four
  Real sigma, eps, d_lin, dmin;
  Real inv_h;   // 1 / (max_dis - dmin), the fade-out interval
  Real spl_V;   // 12-6 value at dmin (start of the fade)
  Real spl_dp;  // 12-6 slope at dmin times the fade-out interval
  Real pad;
};

template <typename Real>
struct alignas(4 * sizeof(Real)) LKRecord {  // 16 values (13 used), four groups of four
  Real close_dmin, close_dmax;
  Real flat_V;                // both directions at d_min
  Real inv_hc;                // 1 / (close_dmax - close_dmin)
  Real cmax_V, cmax_dp;       // both directions at close_dmax; slope times the close interval
  Real fmin_V, fmin_dp;       // both directions at far_dmin; slope times the fade-out interval
  Real c_i, r_i, il2_i;       // i desolvated by j: c * exp(-(d-r)^2 * il2) / d^2
  Real pad1;
  Real c_j, r_j, il2_j;       // j desolvated by i
  Real pad2;
};

// A group of four table values, read with one vector load.
template <typename Real>
struct alignas(4 * sizeof(Real)) Quad {
  Real a, b, c, d;
};

template <typename Real>
__device__ __forceinline__ void build_records(const AtomParams<Real>& i,
                                              const AtomParams<Real>& j,
                                              const GlobalParams<Real>& g,
                                              LJRecord<Real>& lj,
                                              LKRecord<Real>& lk) {
  LJPair<Real> q = lj_pair(i, j, g);
  lj.sigma = q.sigma;
  lj.eps = q.eps;
  lj.d_lin = q.d_lin;
  lj.dmin = q.dmin;
  {
    Real spl_dV;
    vdw_V_dV(q.dmin, q.sigma, q.eps, lj.spl_V, spl_dV);
    const Real h = g.max_dis - q.dmin;
    lj.inv_h = Real(1) / h;
    lj.spl_dp = spl_dV * h;
    lj.pad = Real(0);
  }

  bool cc = (i.flags & kCarbonLK) && (j.flags & kCarbonLK);
  LKKnots<Real> k = lk_knots(q.sigma, cc, g.max_dis);
  lk.close_dmin = k.close_dmin;
  lk.close_dmax = k.close_dmax;
  lk.flat_V = desolv_V(k.d_min, i.lj_radius, i.lk_dgfree, i.lk_lambda, j.lk_volume) +
              desolv_V(k.d_min, j.lj_radius, j.lk_dgfree, j.lk_lambda, i.lk_volume);
  Real v1, d1, v2, d2;
  desolv_V_dV(k.close_dmax, i.lj_radius, i.lk_dgfree, i.lk_lambda, j.lk_volume, v1, d1);
  desolv_V_dV(k.close_dmax, j.lj_radius, j.lk_dgfree, j.lk_lambda, i.lk_volume, v2, d2);
  lk.cmax_V = v1 + v2;
  lk.inv_hc = Real(1) / (k.close_dmax - k.close_dmin);
  lk.cmax_dp = (d1 + d2) * (k.close_dmax - k.close_dmin);
  desolv_V_dV(k.far_dmin, i.lj_radius, i.lk_dgfree, i.lk_lambda, j.lk_volume, v1, d1);
  desolv_V_dV(k.far_dmin, j.lj_radius, j.lk_dgfree, j.lk_lambda, i.lk_volume, v2, d2);
  lk.fmin_V = v1 + v2;
  lk.fmin_dp = (d1 + d2) * (k.far_dmax - k.far_dmin);
  const Real pi_pow1p5 = Real(5.56832799683f);
  lk.c_i = -j.lk_volume * i.lk_dgfree / (Real(2) * pi_pow1p5 * i.lk_lambda);
  lk.r_i = i.lj_radius;
  lk.il2_i = Real(1) / (i.lk_lambda * i.lk_lambda);
  lk.c_j = -i.lk_volume * j.lk_dgfree / (Real(2) * pi_pow1p5 * j.lk_lambda);
  lk.r_j = j.lj_radius;
  lk.il2_j = Real(1) / (j.lk_lambda * j.lk_lambda);
  lk.pad1 = lk.pad2 = Real(0);
}

// Unweighted LJ (atr, rep) and, with DERIV, their distance derivatives;
// inv = 1 / d.  The fade-out cubic runs on t = (d - dmin) / (max_dis - dmin)
// with the record's stored reciprocal and pre-scaled slope; the linear
// extension's knot value and slope (clashes only) are the 12-6 form's at
// d_lin, computed here.  The record's second group of four is read only in
// the fade-out region.
template <typename Real, bool DERIV>
__device__ __forceinline__ void lj_eval(Real d, Real inv, const LJRecord<Real>* rp,
                                        Real& atr, Real& rep, Real& datr, Real& drep) {
  const Quad<Real>* q = reinterpret_cast<const Quad<Real>*>(rp);
  const Quad<Real> r = q[0];  // sigma, eps, d_lin, dmin
  Real lj, dlj = 0;
  if (d < r.c) {
    Real lin_V, lin_dV;
    vdw_V_dV(r.c, r.a, r.b, lin_V, lin_dV);
    lj = lin_V + lin_dV * (d - r.c);
    dlj = lin_dV;
  } else if (d < r.d) {
    Real sd = r.a * inv;
    Real sd2 = sd * sd;
    Real sd6 = sd2 * sd2 * sd2;
    Real sd12 = sd6 * sd6;
    lj = r.b * (sd12 - Real(2) * sd6);
    if (DERIV) dlj = r.b * (Real(12) * (sd6 - sd12)) * inv;
  } else {
    const Quad<Real> f = q[1];  // 1 / interval, value, interval-scaled slope
    Real t = (d - r.d) * f.a;
    Real p0 = f.b, dp0 = f.c;
    lj = p0 + t * (dp0 + t * (-2 * dp0 - 3 * p0 + t * (dp0 + 2 * p0)));
    if (DERIV) dlj = (dp0 + t * (-4 * dp0 - 6 * p0 + t * (3 * dp0 + 6 * p0))) * f.a;
  }
  if (d < r.a) {
    atr = -r.b;
    rep = lj + r.b;
    datr = 0;
    drep = dlj;
  } else {
    atr = lj;
    rep = 0;
    datr = dlj;
    drep = 0;
  }
}

// The fade-out cubic of LK beyond far_dmin from its knot value and slope.
template <typename Real, bool DERIV>
__device__ __forceinline__ void lk_far(Real d, Real fmin_V, Real fmin_dp, Real far_dmin, Real inv_hf,
                                       Real& V, Real& dV) {
  Real t = (d - far_dmin) * inv_hf;
  Real p0 = fmin_V, dp0 = fmin_dp;
  V = p0 + t * (dp0 + t * (-2 * dp0 - 3 * p0 + t * (dp0 + 2 * p0)));
  if (DERIV) dV = (dp0 + t * (-4 * dp0 - 6 * p0 + t * (3 * dp0 + 6 * p0))) * inv_hf;
}

// Unweighted LK (both directions) and, with DERIV, its distance
// derivative; inv_d = 1 / d.  The regions are tested in the order flat,
// close cubic, Gaussians, fade-out; beyond far_first = max(far_dmin, 4.5 A)
// only the fade-out can apply (every close cubic ends by sqrt(405 / 20) =
// 4.5 A), so that, the most populated region, is tested first.  Only the
// group of four record values a region needs is read.
template <typename Real, bool DERIV>
__device__ __forceinline__ void lk_eval(Real d, Real inv_d, const LKRecord<Real>* rp,
                                        Real far_dmin, Real far_first, Real inv_hf, Real& V,
                                        Real& dV) {
  const Quad<Real>* q = reinterpret_cast<const Quad<Real>*>(rp);
  dV = 0;
  if (d >= far_first) {
    const Quad<Real> k = q[1];  // cmax_V, cmax_dp, fmin_V, fmin_dp
    lk_far<Real, DERIV>(d, k.c, k.d, far_dmin, inv_hf, V, dV);
    return;
  }
  const Quad<Real> b = q[0];  // close_dmin, close_dmax, flat_V, 1 / close interval
  if (d < b.a) {
    V = b.c;
  } else if (d < b.b) {
    const Quad<Real> k = q[1];
    Real t = (d - b.a) * b.d;
    Real p0 = b.c, p1 = k.a, dp1 = k.b;
    V = p0 + t * (t * (-dp1 - 3 * p0 + 3 * p1 + t * (dp1 + 2 * p0 - 2 * p1)));
    if (DERIV) dV = (t * (-2 * dp1 - 6 * p0 + 6 * p1 + t * (3 * dp1 + 6 * p0 - 6 * p1))) * b.d;
  } else if (d < far_dmin) {
    const Quad<Real> gi = q[2], gj = q[3];  // (c, r, il2) of each direction
    Real inv_d2 = inv_d * inv_d;
    Real xi = d - gi.b, xj = d - gj.b;
    Real ei = gi.a * exp(-xi * xi * gi.c);
    Real ej = gj.a * exp(-xj * xj * gj.c);
    V = (ei + ej) * inv_d2;
    if (DERIV) {
      dV = inv_d2 * (ei * (Real(-2) * inv_d - Real(2) * xi * gi.c) +
                     ej * (Real(-2) * inv_d - Real(2) * xj * gj.c));
    }
  } else {
    const Quad<Real> k = q[1];
    lk_far<Real, DERIV>(d, k.c, k.d, far_dmin, inv_hf, V, dV);
  }
}

}  // namespace tmol_b200
