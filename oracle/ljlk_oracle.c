/*
 * CPU restatement of tmol's LJ + LK pose scoring, used ONLY as a test oracle.
 *
 * This file is test infrastructure.  Nothing in the product links or calls
 * it; tests, the smoke check and the benchmark's CPU-baseline leg load it
 * through ctypes to check the CUDA path.
 *
 * It follows, function by function, the reference's CPU execution of the
 * pose-score op (one thread per work group, work groups in index order), in
 * the same floating-point operation order, so that the float build agrees
 * with the compiled reference op to the last bit in most cases:
 *
 *   count-pair weight      tmol/score/ljlk/potentials/common.hh:14-22
 *   LJ sigma rule          tmol/score/ljlk/potentials/common.hh:25-44
 *   vdw / lj_score         tmol/score/ljlk/potentials/lj.hh:22-178
 *   f_desolv / LK pair     tmol/score/ljlk/potentials/lk_isotropic.hh:23-236
 *   LK isotropic score     tmol/score/ljlk/potentials/lk_isotropic.hh:239-361
 *   Hermite splines        tmol/score/common/cubic_hermite_polynomial.hh:34-137
 *   distance + gradient    tmol/score/common/geom.hh:20-40
 *   block spheres          tmol/score/common/sphere_overlap.impl.hh:109-196
 *   block neighbours       tmol/score/common/sphere_overlap.impl.hh:287-351
 *   inter-block count pair tmol/score/common/count_pair.hh:162-207,
 *                          tmol/score/ljlk/potentials/ljlk_pose_score.impl.hh:47-67
 *   intra-block count pair ljlk_pose_score.impl.hh:115-134, 176-206
 *   tile walk              tmol/score/common/tile_atom_pair_evaluation.hh:79-173, 358-505
 *   whole-pose forward     ljlk_pose_score.impl.hh:953-1156
 *   block-pair forward     ljlk_pose_score.impl.hh:803-951
 *   block-pair backward    ljlk_pose_score.impl.hh:1160-1477
 *
 * Compile with -DORACLE_REAL=float (default) or -DORACLE_REAL=double and
 * -ffp-contract=off (no fused multiply-add, as the reference's x86-64 build).
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#if defined(ORACLE_DOUBLE)
#define ORACLE_REAL double
#else
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;

#define TILE 32
#define MAX_N_CONN 4
#define MAX_IMPORTANT_BOND_SEPARATION 4

typedef struct {
  real lj_radius, lj_wdepth, lk_dgfree, lk_lambda, lk_volume;
  real is_donor, is_hydroxyl, is_polarh, is_acceptor, is_carbon_lk;
} type_params_t;

typedef struct {
  real max_dis, lj_dlin_sigma_factor, lj_hbond_dis, lj_hbond_OH_donor_dis,
      lj_hbond_hdis;
} global_params_t;

static real rsqrt_(real x) {
#if defined(ORACLE_DOUBLE)
  return sqrt(x);
#else
  return sqrtf(x);
#endif
}
static real rexp_(real x) {
#if defined(ORACLE_DOUBLE)
  return exp(x);
#else
  return expf(x);
#endif
}
static real rfloor_(real x) {
#if defined(ORACLE_DOUBLE)
  return floor(x);
#else
  return floorf(x);
#endif
}
static real rmax_(real a, real b) { return a < b ? b : a; }
static real rmin_(real a, real b) { return b < a ? b : a; }

/* common.hh:14-22 */
static real connectivity_weight(int bonded_path_length) {
  if (bonded_path_length > 4) return (real)1.0;
  if (bonded_path_length == 4) return (real)0.2;
  return (real)0.0;
}

/* common.hh:25-44 */
static real lj_sigma(const type_params_t* i, const type_params_t* j,
                     const global_params_t* g) {
  if ((i->is_donor != 0 && j->is_acceptor != 0) ||
      (j->is_donor != 0 && i->is_acceptor != 0)) {
    if ((i->is_donor != 0 && i->is_hydroxyl != 0) ||
        (j->is_donor != 0 && j->is_hydroxyl != 0)) {
      return g->lj_hbond_OH_donor_dis;
    }
    return g->lj_hbond_dis;
  } else if ((i->is_polarh != 0 && j->is_acceptor != 0) ||
             (j->is_polarh != 0 && i->is_acceptor != 0)) {
    return g->lj_hbond_hdis;
  }
  return i->lj_radius + j->lj_radius;
}

/* cubic_hermite_polynomial.hh:48-63 */
static real interpolate(real x, real x0, real p0, real dpdx0, real x1, real p1,
                        real dpdx1) {
  real t = (x - x0) / (x1 - x0);
  real dp0 = dpdx0 * (x1 - x0);
  real dp1 = dpdx1 * (x1 - x0);
  return p0 + t * (dp0 + t * (-2 * dp0 - dp1 - 3 * p0 + 3 * p1 +
                              t * (dp0 + dp1 + 2 * p0 - 2 * p1)));
}

/* cubic_hermite_polynomial.hh:83-102 */
static void interpolate_V_dV(real x, real x0, real p0, real dpdx0, real x1,
                             real p1, real dpdx1, real* V, real* dV) {
  real t = (x - x0) / (x1 - x0);
  real dp0 = dpdx0 * (x1 - x0);
  real dp1 = dpdx1 * (x1 - x0);
  real p = p0 + t * (dp0 + t * (-2 * dp0 - dp1 - 3 * p0 + 3 * p1 +
                                t * (dp0 + dp1 + 2 * p0 - 2 * p1)));
  real dp = dp0 + t * (-4 * dp0 - 2 * dp1 - 6 * p0 + 6 * p1 +
                       t * (3 * dp0 + 3 * dp1 + 6 * p0 - 6 * p1));
  *V = p;
  *dV = dp / (x1 - x0);
}

/* cubic_hermite_polynomial.hh:104-113 */
static real interpolate_to_zero(real x, real x0, real p0, real dpdx0, real x1) {
  real t = (x - x0) / (x1 - x0);
  real dp0 = dpdx0 * (x1 - x0);
  return p0 + t * (dp0 + t * (-2 * dp0 - 3 * p0 + t * (dp0 + 2 * p0)));
}

/* cubic_hermite_polynomial.hh:127-137 */
static void interpolate_to_zero_V_dV(real x, real x0, real p0, real dpdx0,
                                     real x1, real* V, real* dV) {
  real t = (x - x0) / (x1 - x0);
  real dp0 = dpdx0 * (x1 - x0);
  *V = p0 + t * (dp0 + t * (-2 * dp0 - 3 * p0 + t * (dp0 + 2 * p0)));
  *dV = (dp0 + t * (-4 * dp0 - 6 * p0 + t * (3 * dp0 + 6 * p0))) / (x1 - x0);
}

/* lj.hh:32-36 */
static real vdw_V(real dist, real sigma, real epsilon) {
  real sd = (sigma / dist);
  real sd2 = sd * sd;
  real sd6 = sd2 * sd2 * sd2;
  real sd12 = sd6 * sd6;
  return epsilon * (sd12 - 2 * sd6);
}

/* lj.hh:38-47 */
static void vdw_V_dV(real dist, real sigma, real epsilon, real* V, real* dV) {
  real sd = (sigma / dist);
  real sd2 = sd * sd;
  real sd6 = sd2 * sd2 * sd2;
  real sd12 = sd6 * sd6;
  *V = epsilon * (sd12 - (real)2.0 * sd6);
  *dV = epsilon * (((real)-12.0 * sd12 / dist) - ((real)-12.0 * sd6 / dist));
}

/* lj.hh:65-113 (energy only) */
void oracle_lj_score_V(real dist, real bonded_path_length,
                       const type_params_t* i, const type_params_t* j,
                       const global_params_t* g, real out[2]) {
  real cpoly_dmax = g->max_dis;
  real spline_start = g->max_dis - (real)1.5;
  real weight, Vatr, Vrep;
  if (dist > cpoly_dmax) {
    Vatr = 0;
    Vrep = 0;
    weight = 0;
  } else {
    real sigma = lj_sigma(i, j, g);
    real epsilon = rsqrt_(i->lj_wdepth * j->lj_wdepth);
    real d_lin = sigma * g->lj_dlin_sigma_factor;
    real cpoly_dmin =
        sigma > spline_start
            ? (sigma > cpoly_dmax - (real)0.1 ? cpoly_dmax - (real)0.1 : sigma)
            : spline_start;
    weight = connectivity_weight((int)bonded_path_length);
    if (dist > cpoly_dmin) {
      real v0, dv0;
      vdw_V_dV(cpoly_dmin, sigma, epsilon, &v0, &dv0);
      Vatr = interpolate_to_zero(dist, cpoly_dmin, v0, dv0, cpoly_dmax);
    } else if (dist > d_lin) {
      Vatr = vdw_V(dist, sigma, epsilon);
    } else {
      real v0, dv0;
      vdw_V_dV(d_lin, sigma, epsilon, &v0, &dv0);
      Vatr = (v0 + dv0 * (dist - d_lin));
    }
    if (dist < sigma) {
      Vrep = Vatr + epsilon;
      Vatr = -epsilon;
    } else {
      Vrep = 0;
    }
  }
  out[0] = weight * Vatr;
  out[1] = weight * Vrep;
}

/* lj.hh:115-177: out = {Vatr, Vrep, dVatr/dd, dVrep/dd} */
void oracle_lj_score_V_dV(real dist, real bonded_path_length,
                          const type_params_t* i, const type_params_t* j,
                          const global_params_t* g, real out[4]) {
  real sigma = lj_sigma(i, j, g);
  real weight = connectivity_weight((int)bonded_path_length);
  real epsilon = rsqrt_(i->lj_wdepth * j->lj_wdepth);
  real d_lin = sigma * g->lj_dlin_sigma_factor;
  real cpoly_dmax = g->max_dis;
  real cpoly_dmin = g->max_dis - (real)1.5;
  if (sigma > cpoly_dmin) cpoly_dmin = sigma;
  if (cpoly_dmin > cpoly_dmax - (real)0.1) cpoly_dmin = cpoly_dmax - (real)0.1;
  real lj, dlj;
  if (dist < d_lin) {
    real v0, dv0;
    vdw_V_dV(d_lin, sigma, epsilon, &v0, &dv0);
    lj = v0 + dv0 * (dist - d_lin);
    dlj = dv0;
  } else if (dist < cpoly_dmin) {
    vdw_V_dV(dist, sigma, epsilon, &lj, &dlj);
  } else if (dist < cpoly_dmax) {
    real v0, dv0;
    vdw_V_dV(cpoly_dmin, sigma, epsilon, &v0, &dv0);
    interpolate_to_zero_V_dV(dist, cpoly_dmin, v0, dv0, cpoly_dmax, &lj, &dlj);
  } else {
    lj = 0;
    dlj = 0;
  }
  real Vatr, Vrep, dVatr, dVrep;
  if (dist < sigma) {
    Vatr = -epsilon;
    Vrep = lj + epsilon;
    dVatr = 0;
    dVrep = dlj;
  } else {
    Vatr = lj;
    Vrep = 0;
    dVatr = dlj;
    dVrep = 0;
  }
  out[0] = weight * Vatr;
  out[1] = weight * Vrep;
  out[2] = weight * dVatr;
  out[3] = weight * dVrep;
}

static const real pi_pow1p5 = (real)5.56832799683f;

/* lk_isotropic.hh:30-51 */
static real f_desolv_V(real dist, real lj_radius_i, real lk_dgfree_i,
                       real lk_lambda_i, real lk_volume_j) {
  return (-lk_volume_j * lk_dgfree_i / (2 * pi_pow1p5 * lk_lambda_i) /
          (dist * dist) *
          rexp_(-(dist - lj_radius_i) * (dist - lj_radius_i) /
                (lk_lambda_i * lk_lambda_i)));
}

/* lk_isotropic.hh:53-94 */
static void f_desolv_V_dV(real dist, real lj_radius_i, real lk_dgfree_i,
                          real lk_lambda_i, real lk_volume_j, real* V,
                          real* dV) {
  real exp_val = rexp_(-(dist - lj_radius_i) * (dist - lj_radius_i) /
                       (lk_lambda_i * lk_lambda_i));
  *V = (-lk_volume_j * lk_dgfree_i / (2 * pi_pow1p5 * lk_lambda_i) /
        (dist * dist) * exp_val);
  *dV = (-lk_volume_j * lk_dgfree_i / (2 * pi_pow1p5 * lk_lambda_i) * exp_val *
         ((-2 / (dist * dist * dist)) +
          (1 / (dist * dist) * -(2 * dist - 2 * lj_radius_i) /
           (lk_lambda_i * lk_lambda_i))));
}

/* close-spline knots, lk_isotropic.hh:132-143 */
static void lk_knots(real lj_sigma_ij, int is_cc_pair, real* d_min,
                     real* close_dmin, real* close_dmax) {
  real dm = (real)(lj_sigma_ij * .89);
  if (is_cc_pair) dm = rmax_(dm, (real)4.2);
  real n = rfloor_((real)20 * dm * dm);
  *d_min = dm;
  *close_dmin = rsqrt_(rmax_((real)0, n - 29) / 20);
  *close_dmax = rsqrt_(rmin_(n + 21, (real)405) / 20);
}

/* lk_isotropic.hh:167-236 */
static void lk_isotropic_pair_V_dV(real dist, real bonded_path_length,
                                   real lj_sigma_ij, real lj_radius_i,
                                   real lk_dgfree_i, real lk_lambda_i,
                                   real lk_volume_j, real max_dis,
                                   int is_cc_pair, real* V, real* dV) {
  real d_min, close_dmin, close_dmax;
  lk_knots(lj_sigma_ij, is_cc_pair, &d_min, &close_dmin, &close_dmax);
  real far_dmax = max_dis;
  real far_dmin = max_dis - (real)1.5;
  real weight = connectivity_weight((int)bonded_path_length);
  real lk, dlk;
  if (dist < close_dmin) {
    lk = f_desolv_V(d_min, lj_radius_i, lk_dgfree_i, lk_lambda_i, lk_volume_j);
    dlk = 0;
  } else if (dist < close_dmax) {
    real v1, dv1;
    f_desolv_V_dV(close_dmax, lj_radius_i, lk_dgfree_i, lk_lambda_i,
                  lk_volume_j, &v1, &dv1);
    interpolate_V_dV(
        dist, close_dmin,
        f_desolv_V(d_min, lj_radius_i, lk_dgfree_i, lk_lambda_i, lk_volume_j),
        (real)0.0, close_dmax, v1, dv1, &lk, &dlk);
  } else if (dist < far_dmin) {
    f_desolv_V_dV(dist, lj_radius_i, lk_dgfree_i, lk_lambda_i, lk_volume_j,
                  &lk, &dlk);
  } else if (dist < far_dmax) {
    real v0, dv0;
    f_desolv_V_dV(far_dmin, lj_radius_i, lk_dgfree_i, lk_lambda_i, lk_volume_j,
                  &v0, &dv0);
    interpolate_to_zero_V_dV(dist, far_dmin, v0, dv0, far_dmax, &lk, &dlk);
  } else {
    lk = 0;
    dlk = 0;
  }
  *V = weight * lk;
  *dV = weight * dlk;
}

/* lk_isotropic.hh:248-326 (energy only) */
real oracle_lk_score_V(real dist, real bonded_path_length,
                       const type_params_t* i, const type_params_t* j,
                       const global_params_t* g) {
  real sigma = lj_sigma(i, j, g);
  int is_cc = (i->is_carbon_lk != 0) && (j->is_carbon_lk != 0);
  real d_min, close_dmin, close_dmax;
  lk_knots(sigma, is_cc, &d_min, &close_dmin, &close_dmax);
  real far_dmax = g->max_dis;
  real far_dmin = g->max_dis - (real)1.5;
  real weight = connectivity_weight((int)bonded_path_length);
  real lk;
  if (dist > far_dmax) {
    lk = 0;
  } else if (dist > far_dmin) {
    real v0, dv0;
    f_desolv_V_dV(far_dmin, i->lj_radius, i->lk_dgfree, i->lk_lambda,
                  j->lk_volume, &v0, &dv0);
    lk = interpolate_to_zero(dist, far_dmin, v0, dv0, far_dmax);
    f_desolv_V_dV(far_dmin, j->lj_radius, j->lk_dgfree, j->lk_lambda,
                  i->lk_volume, &v0, &dv0);
    lk += interpolate_to_zero(dist, far_dmin, v0, dv0, far_dmax);
  } else if (dist > close_dmax) {
    lk = f_desolv_V(dist, i->lj_radius, i->lk_dgfree, i->lk_lambda,
                    j->lk_volume) +
         f_desolv_V(dist, j->lj_radius, j->lk_dgfree, j->lk_lambda,
                    i->lk_volume);
  } else if (dist > close_dmin) {
    real v1, dv1;
    f_desolv_V_dV(close_dmax, i->lj_radius, i->lk_dgfree, i->lk_lambda,
                  j->lk_volume, &v1, &dv1);
    lk = interpolate(dist, close_dmin,
                     f_desolv_V(d_min, i->lj_radius, i->lk_dgfree, i->lk_lambda,
                                j->lk_volume),
                     (real)0.0, close_dmax, v1, dv1);
    f_desolv_V_dV(close_dmax, j->lj_radius, j->lk_dgfree, j->lk_lambda,
                  i->lk_volume, &v1, &dv1);
    lk += interpolate(dist, close_dmin,
                      f_desolv_V(d_min, j->lj_radius, j->lk_dgfree,
                                 j->lk_lambda, i->lk_volume),
                      (real)0.0, close_dmax, v1, dv1);
  } else {
    lk = f_desolv_V(d_min, i->lj_radius, i->lk_dgfree, i->lk_lambda,
                    j->lk_volume) +
         f_desolv_V(d_min, j->lj_radius, j->lk_dgfree, j->lk_lambda,
                    i->lk_volume);
  }
  return weight * lk;
}

/* lk_isotropic.hh:328-361: out = {V, dV/dd} */
void oracle_lk_score_V_dV(real dist, real bonded_path_length,
                          const type_params_t* i, const type_params_t* j,
                          const global_params_t* g, real out[2]) {
  real sigma = lj_sigma(i, j, g);
  int is_cc = (i->is_carbon_lk != 0) && (j->is_carbon_lk != 0);
  real v1, d1, v2, d2;
  lk_isotropic_pair_V_dV(dist, bonded_path_length, sigma, i->lj_radius,
                         i->lk_dgfree, i->lk_lambda, j->lk_volume, g->max_dis,
                         is_cc, &v1, &d1);
  lk_isotropic_pair_V_dV(dist, bonded_path_length, sigma, j->lj_radius,
                         j->lk_dgfree, j->lk_lambda, i->lk_volume, g->max_dis,
                         is_cc, &v2, &d2);
  out[0] = v1 + v2;
  out[1] = d1 + d2;
}

/* ---------------------------------------------------------------------- */
/* Pose scoring.                                                           */

typedef struct {
  /* inputs (row-major, int32 tables, `real` floats) */
  const real* coords; /* [n_atoms][3] */
  const int32_t* rot_coord_offset;      /* [n_rots] */
  const int32_t* first_rot_block_type;  /* [P][B] */
  const int32_t* block_ind_for_rot;     /* [n_rots] */
  const int32_t* pose_ind_for_rot;      /* [n_rots] */
  const int32_t* block_type_ind_for_rot;/* [n_rots] */
  const int32_t* rot_offset_for_block;  /* [P][B] */
  const int32_t* min_bondsep;           /* [P][B][B] */
  const int32_t* inter_block_bondsep;   /* [P][B][B][C][C] */
  const int32_t* bt_n_atoms;            /* [nbt] */
  const int32_t* bt_n_heavy_in_tile;    /* [nbt][ntiles] */
  const int32_t* bt_heavy_in_tile;      /* [nbt][32*ntiles] */
  const int32_t* bt_atom_types;         /* [nbt][A] */
  const int32_t* bt_n_conn;             /* [nbt] */
  const int32_t* bt_conn_atom;          /* [nbt][C] */
  const int32_t* bt_path_distance;      /* [nbt][A][A] */
  const int32_t* bt_is_ligand;          /* [nbt] */
  const real* type_params;              /* [T][10] */
  const real* global_params;            /* [5] */
  real max_dis;
  int n_atoms, n_rots, P, B, nbt, A, C, ntiles, T;
  const int32_t* n_rots_for_block;      /* [P][B] (rotamer scoring) */
  /* the elec term (term == 1): per block-type atom partial charges, path
   * distances to each atom's count-pair representative (conn-atom lookups;
   * bt_path_distance then holds the representative-to-representative
   * table), and the sigmoidal-dielectric parameters */
  int term;
  const real* bt_charge;                /* [nbt][A] */
  const int32_t* bt_pd_inter;           /* [nbt][A][A] */
  float elec_D, elec_D0, elec_S, elec_min_dis, elec_max_dis;
} oracle_inputs_t;

typedef struct {
  int pose, b1, b2, rot1, rot2, bt1, bt2, n1, n2, off1, off2;
  int n_conn1, n_conn2, min_sep, striking;
  unsigned char conn_ats1[MAX_N_CONN], conn_ats2[MAX_N_CONN];
  unsigned char conn_seps[MAX_N_CONN * MAX_N_CONN];
  int lig_pair;
} pair_ctx_t;

static const type_params_t* tparams(const oracle_inputs_t* in, int bt,
                                    int atom) {
  int t = in->bt_atom_types[bt * in->A + atom];
  return (const type_params_t*)(in->type_params + 10 * (size_t)t);
}

/* count_pair.hh:162-207 + ljlk_pose_score.impl.hh:47-67 */
static int inter_separation(const oracle_inputs_t* in, const pair_ctx_t* c,
                            int a1, int a2) {
  int sep = c->min_sep;
  const int32_t* pd = in->bt_pd_inter ? in->bt_pd_inter : in->bt_path_distance;
  if (sep <= MAX_IMPORTANT_BOND_SEPARATION) {
    sep = MAX_IMPORTANT_BOND_SEPARATION + 1;
    for (int ii = 0; ii < c->n_conn1; ++ii) {
      unsigned char pd1 = (unsigned char)pd
          [((size_t)c->bt1 * in->A + c->conn_ats1[ii]) * in->A + a1];
      for (int jj = 0; jj < c->n_conn2; ++jj) {
        int cs = c->conn_seps[ii * c->n_conn2 + jj];
        unsigned char pd2 = (unsigned char)pd
            [((size_t)c->bt2 * in->A + c->conn_ats2[jj]) * in->A + a2];
        int s = pd1 + cs + pd2;
        if (s < sep) sep = s;
      }
    }
  }
  if (c->lig_pair && (sep == 3 || sep == 4)) sep = 5;
  return sep;
}

static int intra_separation(const oracle_inputs_t* in, int bt, int a1,
                            int a2) {
  return in->bt_path_distance[((size_t)bt * in->A + a1) * in->A + a2];
}

/* geom.hh:20-40; Eigen's norm() sums the squares as x^2 + (y^2 + z^2) */
static void dist_and_grad(const real* x1, const real* x2, real* d,
                          real g1[3]) {
  real dx = x1[0] - x2[0], dy = x1[1] - x2[1], dz = x1[2] - x2[2];
  real V = rsqrt_(dx * dx + (dy * dy + dz * dz));
  *d = V;
  if (V != 0) {
    g1[0] = dx / V;
    g1[1] = dy / V;
    g1[2] = dz / V;
  } else {
    g1[0] = g1[1] = g1[2] = 0;
  }
}

static void acc3(real* dst, const real* g, real s) {
  for (int k = 0; k < 3; ++k) {
    real v = s * g[k];
    if (v != 0) dst[k] += v;
  }
}
static void acc3_neg(real* dst, const real* g, real s) {
  for (int k = 0; k < 3; ++k) {
    real v = s * -g[k];
    if (v != 0) dst[k] += v;
  }
}

/* Modes of the per-atom-pair evaluation. */
enum { MODE_ENERGY = 0, MODE_ENERGY_AND_DERIVS = 1, MODE_WEIGHTED_DERIVS = 2 };

typedef struct {
  int mode;
  real* dV;       /* MODE 1: [3][n_atoms][3]; MODE 2: [n_atoms][3] */
  real w[3];      /* MODE 2 weights for atr, rep, lk */
} eval_t;

static void eval_lj(const oracle_inputs_t* in, const eval_t* ev, int bt1,
                    int a1, int at1, int bt2, int a2, int at2, int sep,
                    real* atr, real* rep) {
  const global_params_t* g = (const global_params_t*)in->global_params;
  const real* x1 = in->coords + 3 * (size_t)at1;
  const real* x2 = in->coords + 3 * (size_t)at2;
  const type_params_t* t1 = tparams(in, bt1, a1);
  const type_params_t* t2 = tparams(in, bt2, a2);
  if (ev->mode == MODE_ENERGY) {
    real dx = x1[0] - x2[0], dy = x1[1] - x2[1], dz = x1[2] - x2[2];
    real d = rsqrt_(dx * dx + (dy * dy + dz * dz));
    real out[2];
    oracle_lj_score_V(d, (real)sep, t1, t2, g, out);
    *atr = out[0];
    *rep = out[1];
    return;
  }
  real d, gr[3];
  dist_and_grad(x1, x2, &d, gr);
  real o[4];
  oracle_lj_score_V_dV(d, (real)sep, t1, t2, g, o);
  if (ev->mode == MODE_ENERGY_AND_DERIVS) {
    size_t N3 = 3 * (size_t)in->n_atoms;
    /* ljlk.hh:629-664: atom 1 (atr, rep per component), then atom 2 */
    for (int k = 0; k < 3; ++k) {
      real va = o[2] * gr[k];
      real vr = o[3] * gr[k];
      if (va != 0) ev->dV[0 * N3 + 3 * (size_t)at1 + k] += va;
      if (vr != 0) ev->dV[1 * N3 + 3 * (size_t)at1 + k] += vr;
    }
    for (int k = 0; k < 3; ++k) {
      real va = o[2] * -gr[k];
      real vr = o[3] * -gr[k];
      if (va != 0) ev->dV[0 * N3 + 3 * (size_t)at2 + k] += va;
      if (vr != 0) ev->dV[1 * N3 + 3 * (size_t)at2 + k] += vr;
    }
  } else {
    /* ljlk.hh:531-594 */
    for (int k = 0; k < 3; ++k) {
      real va = ev->w[0] * o[2] * gr[k];
      real vr = ev->w[1] * o[3] * gr[k];
      if (va != 0) ev->dV[3 * (size_t)at1 + k] += va;
      if (vr != 0) ev->dV[3 * (size_t)at1 + k] += vr;
    }
    for (int k = 0; k < 3; ++k) {
      real va = ev->w[0] * o[2] * -gr[k];
      real vr = ev->w[1] * o[3] * -gr[k];
      if (va != 0) ev->dV[3 * (size_t)at2 + k] += va;
      if (vr != 0) ev->dV[3 * (size_t)at2 + k] += vr;
    }
  }
  *atr = o[0];
  *rep = o[1];
}

static real eval_lk(const oracle_inputs_t* in, const eval_t* ev, int bt1,
                    int a1, int at1, int bt2, int a2, int at2, int sep) {
  const global_params_t* g = (const global_params_t*)in->global_params;
  const real* x1 = in->coords + 3 * (size_t)at1;
  const real* x2 = in->coords + 3 * (size_t)at2;
  const type_params_t* t1 = tparams(in, bt1, a1);
  const type_params_t* t2 = tparams(in, bt2, a2);
  if (ev->mode == MODE_ENERGY) {
    real dx = x1[0] - x2[0], dy = x1[1] - x2[1], dz = x1[2] - x2[2];
    real d = rsqrt_(dx * dx + (dy * dy + dz * dz));
    return oracle_lk_score_V(d, (real)sep, t1, t2, g);
  }
  real d, gr[3];
  dist_and_grad(x1, x2, &d, gr);
  real o[2];
  oracle_lk_score_V_dV(d, (real)sep, t1, t2, g, o);
  if (ev->mode == MODE_ENERGY_AND_DERIVS) {
    size_t N3 = 3 * (size_t)in->n_atoms;
    acc3(ev->dV + 2 * N3 + 3 * (size_t)at1, gr, o[1]);
    acc3_neg(ev->dV + 2 * N3 + 3 * (size_t)at2, gr, o[1]);
  } else {
    acc3(ev->dV + 3 * (size_t)at1, gr, ev->w[2] * o[1]);
    acc3_neg(ev->dV + 3 * (size_t)at2, gr, ev->w[2] * o[1]);
  }
  return o[0];
}

/* ---------------------------------------------------------------------- */
/* The elec term (tmol/score/elec/potentials/potentials.hh:32-215): a      */
/* sigmoidal distance-dependent dielectric Coulomb energy, flat below       */
/* min_dis - 0.25, cubic fades over [min_dis - 0.25, min_dis + 0.25] and    */
/* [max_dis - 1, max_dis].  The parameters are floats and the literals      */
/* doubles, as in the reference, so intermediate values are promoted the    */
/* same way before the result is rounded to `real`.                         */

static real elec_eps(real dist, float D, float D0, float S) {
  return (real)(D - 0.5 * (D - D0) * (2 + 2 * dist * S + dist * dist * S * S) *
                        rexp_(-dist * S));
}

/* eps called with a float distance (min_dis, max_dis): the reference's
 * template deduces Real = float from that argument, so these values are
 * float in both precisions of the op (and so are their products with
 * min_dis / max_dis). */
static float elec_eps_f(float dist, float D, float D0, float S) {
  return (float)(D - 0.5 * (D - D0) * (2 + 2 * dist * S + dist * dist * S * S) *
                         expf(-dist * S));
}

static real elec_deps_ddist(real dist, float D, float D0, float S) {
  return (real)(0.5 * (D - D0) * dist * dist * S * S * S * rexp_(-dist * S));
}

/* elec_delec_ddist (potentials.hh:50-127) when dE != NULL, else elec
 * (:129-205). */
static real elec_pair(const oracle_inputs_t* in, real dist, real e_i, real e_j,
                      real bonded_path_length, real* dE) {
  const float D = in->elec_D, D0 = in->elec_D0, S = in->elec_S;
  const float min_dis = in->elec_min_dis, max_dis = in->elec_max_dis;
  real low_poly_start = min_dis - 0.25;
  real low_poly_end = min_dis + 0.25;
  real hi_poly_start = max_dis - 1.0;
  real hi_poly_end = max_dis;
  real weight = connectivity_weight(bonded_path_length);
  real C1 = 322.0637;
  real C2 = C1 / (max_dis * elec_eps_f(max_dis, D, D0, S));
  real eiej = e_i * e_j;
  real E = 0, dE_ = 0;
  if (dE) *dE = 0;
  if (eiej == 0) return 0;
  if (dist < low_poly_start) {
    real min_dis_score = C1 / (min_dis * elec_eps_f(min_dis, D, D0, S)) - C2;
    E = eiej * min_dis_score;
    dE_ = 0;
  } else if (dist < low_poly_end) {
    real min_dis_score = C1 / (min_dis * elec_eps_f(min_dis, D, D0, S)) - C2;
    real eps_elec = elec_eps(low_poly_end, D, D0, S);
    real deps_elec_d_dist = elec_deps_ddist(low_poly_end, D, D0, S);
    real dmax_elec = eiej * (C1 / (low_poly_end * eps_elec) - C2);
    real dmax_elec_d_dist = -C1 * eiej * (eps_elec + low_poly_end * deps_elec_d_dist) /
                            (low_poly_end * low_poly_end * eps_elec * eps_elec);
    if (dE) {
      interpolate_V_dV(dist, low_poly_start, eiej * min_dis_score, 0.0, low_poly_end,
                       dmax_elec, dmax_elec_d_dist, &E, &dE_);
    } else {
      E = interpolate(dist, low_poly_start, eiej * min_dis_score, 0.0, low_poly_end,
                      dmax_elec, dmax_elec_d_dist);
    }
  } else if (dist < hi_poly_start) {
    real eps_elec = elec_eps(dist, D, D0, S);
    real deps_elec_d_dist = elec_deps_ddist(dist, D, D0, S);
    E = eiej * (C1 / (dist * eps_elec) - C2);
    dE_ = -C1 * eiej * (eps_elec + dist * deps_elec_d_dist) /
          (dist * dist * eps_elec * eps_elec);
  } else if (dist < hi_poly_end) {
    real eps_elec = elec_eps(hi_poly_start, D, D0, S);
    real deps_elec_d_dist = elec_deps_ddist(hi_poly_start, D, D0, S);
    real dmin_elec = eiej * (C1 / (hi_poly_start * eps_elec) - C2);
    real dmin_elec_d_dist = -C1 * eiej * (eps_elec + hi_poly_start * deps_elec_d_dist) /
                            (hi_poly_start * hi_poly_start * eps_elec * eps_elec);
    if (dE) {
      interpolate_to_zero_V_dV(dist, hi_poly_start, dmin_elec, dmin_elec_d_dist,
                               hi_poly_end, &E, &dE_);
    } else {
      E = interpolate_to_zero(dist, hi_poly_start, dmin_elec, dmin_elec_d_dist, hi_poly_end);
    }
  }
  if (dE) *dE = weight * dE_;
  return weight * E;
}

/* elec_atom_energy / _derivs / _energy_and_derivs_full (elec.hh:405-545) */
static real eval_elec(const oracle_inputs_t* in, const eval_t* ev, int bt1, int a1,
                      int at1, int bt2, int a2, int at2, int sep) {
  const real* x1 = in->coords + 3 * (size_t)at1;
  const real* x2 = in->coords + 3 * (size_t)at2;
  const real q1 = in->bt_charge[(size_t)bt1 * in->A + a1];
  const real q2 = in->bt_charge[(size_t)bt2 * in->A + a2];
  if (ev->mode == MODE_ENERGY) {
    real dx = x1[0] - x2[0], dy = x1[1] - x2[1], dz = x1[2] - x2[2];
    real d = rsqrt_(dx * dx + (dy * dy + dz * dz));
    return elec_pair(in, d, q1, q2, (real)sep, NULL);
  }
  real d, gr[3], dE;
  dist_and_grad(x1, x2, &d, gr);
  real E = elec_pair(in, d, q1, q2, (real)sep, &dE);
  if (ev->mode == MODE_ENERGY_AND_DERIVS) {
    acc3(ev->dV + 3 * (size_t)at1, gr, dE);
    acc3_neg(ev->dV + 3 * (size_t)at2, gr, dE);
  } else {
    acc3(ev->dV + 3 * (size_t)at1, gr, ev->w[0] * dE);
    acc3_neg(ev->dV + 3 * (size_t)at2, gr, ev->w[0] * dE);
  }
  return E;
}

/* One work group of the pose kernel: all atom pairs of one block pair,
 * walked tile by tile (tile_atom_pair_evaluation.hh:358-505).  Returns the
 * three block-pair totals. */
static void eval_block_pair(const oracle_inputs_t* in, const eval_t* ev,
                            const pair_ctx_t* c, real tot[3]) {
  real t_atr = 0, t_rep = 0, t_lk = 0;
  int nt_tiles = in->ntiles;
  if (c->b1 != c->b2) {
    int n_it1 = (c->n1 - 1) / TILE + 1;
    int n_it2 = (c->n2 - 1) / TILE + 1;
    for (int i = 0; i < n_it1; ++i) {
      int s1 = TILE * i;
      int nr1 = c->n1 - s1 < TILE ? c->n1 - s1 : TILE;
      int nh1 = in->term == 0 ? in->bt_n_heavy_in_tile[c->bt1 * nt_tiles + i] : 0;
      for (int j = 0; j < n_it2; ++j) {
        int s2 = TILE * j;
        int nr2 = c->n2 - s2 < TILE ? c->n2 - s2 : TILE;
        int nh2 = in->term == 0 ? in->bt_n_heavy_in_tile[c->bt2 * nt_tiles + j] : 0;
        real la = 0, lr = 0, lk = 0;
        for (int k = 0; k < nr1 * nr2; ++k) {
          int a1 = s1 + k / nr2, a2 = s2 + k % nr2;
          int sep = inter_separation(in, c, a1, a2);
          real atr, rep = 0;
          if (in->term == 1)
            atr = eval_elec(in, ev, c->bt1, a1, c->off1 + a1, c->bt2, a2, c->off2 + a2, sep);
          else
            eval_lj(in, ev, c->bt1, a1, c->off1 + a1, c->bt2, a2, c->off2 + a2,
                    sep, &atr, &rep);
          la += atr;
          lr += rep;
        }
        t_atr += la;
        t_rep += lr;
        if (in->term == 0 && nh1 > 0 && nh2 > 0) {
          for (int k = 0; k < nh1 * nh2; ++k) {
            int h1 = k / nh2, h2 = k % nh2;
            int a1 = s1 + in->bt_heavy_in_tile[c->bt1 * TILE * nt_tiles + s1 + h1];
            int a2 = s2 + in->bt_heavy_in_tile[c->bt2 * TILE * nt_tiles + s2 + h2];
            int sep = inter_separation(in, c, a1, a2);
            lk += eval_lk(in, ev, c->bt1, a1, c->off1 + a1, c->bt2, a2,
                          c->off2 + a2, sep);
          }
        }
        t_lk += lk;
      }
    }
  } else {
    int n_it = (c->n1 - 1) / TILE + 1;
    for (int i = 0; i < n_it; ++i) {
      int s1 = TILE * i;
      int nr1 = c->n1 - s1 < TILE ? c->n1 - s1 : TILE;
      int nh1 = in->term == 0 ? in->bt_n_heavy_in_tile[c->bt1 * nt_tiles + i] : 0;
      for (int j = i; j < n_it; ++j) {
        int s2 = TILE * j;
        int nr2 = c->n1 - s2 < TILE ? c->n1 - s2 : TILE;
        int nh2 = in->term == 0 ? in->bt_n_heavy_in_tile[c->bt1 * nt_tiles + j] : 0;
        real la = 0, lr = 0, lk = 0;
        for (int k = 0; k < nr1 * nr2; ++k) {
          int a1 = s1 + k / nr2, a2 = s2 + k % nr2;
          if (a1 >= a2) continue;
          int sep = intra_separation(in, c->bt1, a1, a2);
          real atr, rep = 0;
          if (in->term == 1)
            atr = eval_elec(in, ev, c->bt1, a1, c->off1 + a1, c->bt1, a2, c->off1 + a2, sep);
          else
            eval_lj(in, ev, c->bt1, a1, c->off1 + a1, c->bt1, a2, c->off1 + a2,
                    sep, &atr, &rep);
          la += atr;
          lr += rep;
        }
        t_atr += la;
        t_rep += lr;
        if (in->term == 0 && nh1 > 0 && nh2 > 0) {
          for (int k = 0; k < nh1 * nh2; ++k) {
            int h1 = k / nh2, h2 = k % nh2;
            if (h1 + s1 >= h2 + s2) continue;
            int a1 = s1 + in->bt_heavy_in_tile[c->bt1 * TILE * nt_tiles + s1 + h1];
            int a2 = s2 + in->bt_heavy_in_tile[c->bt1 * TILE * nt_tiles + s2 + h2];
            int sep = intra_separation(in, c->bt1, a1, a2);
            lk += eval_lk(in, ev, c->bt1, a1, c->off1 + a1, c->bt1, a2,
                          c->off1 + a2, sep);
          }
        }
        t_lk += lk;
      }
    }
  }
  tot[0] = t_atr;
  tot[1] = t_rep;
  tot[2] = t_lk;
}

/* sphere_overlap.impl.hh:109-196: per rotamer centroid + radius */
static void compute_spheres(const oracle_inputs_t* in, real* spheres) {
  for (size_t k = 0; k < (size_t)in->P * in->B * 4; ++k) spheres[k] = 0;
  for (int r = 0; r < in->n_rots; ++r) {
    int p = in->pose_ind_for_rot[r];
    int b = in->block_ind_for_rot[r];
    int bt = in->block_type_ind_for_rot[r];
    int off = in->rot_coord_offset[r];
    if (bt < 0) continue;
    int n = in->bt_n_atoms[bt];
    real c[3] = {0, 0, 0};
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) c[k] += in->coords[3 * (size_t)(off + i) + k];
    for (int k = 0; k < 3; ++k) c[k] /= n;
    real d2max = 0;
    for (int i = 0; i < n; ++i) {
      const real* x = in->coords + 3 * (size_t)(off + i);
      real d2 = ((x[0] - c[0]) * (x[0] - c[0]) + (x[1] - c[1]) * (x[1] - c[1]) +
                 (x[2] - c[2]) * (x[2] - c[2]));
      if (d2 > d2max) d2max = d2;
    }
    real* s = spheres + 4 * ((size_t)p * in->B + b);
    s[0] = c[0];
    s[1] = c[1];
    s[2] = c[2];
    s[3] = rsqrt_(d2max);
  }
}

/* sphere_overlap.impl.hh:287-351 */
static void detect_neighbors(const oracle_inputs_t* in, const real* spheres,
                             int32_t* nbr) {
  int B = in->B;
  memset(nbr, 0, sizeof(int32_t) * (size_t)in->P * B * B);
  for (int p = 0; p < in->P; ++p)
    for (int i = 0; i < B; ++i)
      for (int j = i; j < B; ++j) {
        if (in->first_rot_block_type[p * B + i] < 0) continue;
        if (in->first_rot_block_type[p * B + j] < 0) continue;
        const real* s1 = spheres + 4 * ((size_t)p * B + i);
        const real* s2 = spheres + 4 * ((size_t)p * B + j);
        real d2 = ((s1[0] - s2[0]) * (s1[0] - s2[0]) +
                   (s1[1] - s2[1]) * (s1[1] - s2[1]) +
                   (s1[2] - s2[2]) * (s1[2] - s2[2]));
        real thr = s1[3] + s2[3] + in->max_dis;
        if (d2 < thr * thr) nbr[((size_t)p * B + i) * B + j] = 1;
      }
}

/* Context of one evaluation: rotamer rot1 of block b1 against rotamer rot2
 * of block b2 of pose p (b1 == b2 means rot1 == rot2, intra-block). */
static int setup_rot_pair(const oracle_inputs_t* in, int p, int b1, int b2,
                          int rot1, int rot2, pair_ctx_t* c) {
  int B = in->B;
  c->pose = p;
  c->b1 = b1;
  c->b2 = b2;
  c->rot1 = rot1;
  c->rot2 = rot2;
  if (c->rot1 < 0 || c->rot2 < 0) return 0;
  c->bt1 = in->block_type_ind_for_rot[c->rot1];
  c->bt2 = in->block_type_ind_for_rot[c->rot2];
  if (c->bt1 < 0 || c->bt2 < 0) return 0;
  c->n1 = in->bt_n_atoms[c->bt1];
  c->n2 = in->bt_n_atoms[c->bt2];
  c->off1 = in->rot_coord_offset[c->rot1];
  c->off2 = in->rot_coord_offset[c->rot2];
  c->n_conn1 = in->bt_n_conn[c->bt1];
  c->n_conn2 = in->bt_n_conn[c->bt2];
  c->min_sep = in->min_bondsep[((size_t)p * B + b1) * B + b2];
  c->striking = c->min_sep <= MAX_IMPORTANT_BOND_SEPARATION;
  c->lig_pair = in->bt_is_ligand[c->bt1] && in->bt_is_ligand[c->bt2];
  if (c->striking) {
    for (int k = 0; k < c->n_conn1; ++k)
      c->conn_ats1[k] = (unsigned char)in->bt_conn_atom[c->bt1 * in->C + k];
    for (int k = 0; k < c->n_conn2; ++k)
      c->conn_ats2[k] = (unsigned char)in->bt_conn_atom[c->bt2 * in->C + k];
    for (int k1 = 0; k1 < c->n_conn1; ++k1)
      for (int k2 = 0; k2 < c->n_conn2; ++k2)
        c->conn_seps[k1 * c->n_conn2 + k2] =
            (unsigned char)in->inter_block_bondsep
                [((((size_t)p * B + b1) * B + b2) * in->C + k1) * in->C + k2];
  }
  return 1;
}

/* The pose op: each block's first (only) rotamer. */
static int setup_pair(const oracle_inputs_t* in, int p, int b1, int b2,
                      pair_ctx_t* c) {
  int B = in->B;
  return setup_rot_pair(in, p, b1, b2, in->rot_offset_for_block[p * B + b1],
                        in->rot_offset_for_block[p * B + b2], c);
}

/*
 * The pose-score op forward (ljlk_pose_score.impl.hh:628-1158).
 *   block_pair == 0: out_E[3][P] (whole pose); if out_dV != NULL, the
 *     per-term gradients [3][n_atoms][3] are accumulated and energies use the
 *     V_dV evaluators, as the reference does when coords require grad.
 *   block_pair != 0: out_E[3][P][B][B], energies only.
 *   out_nbr[P][B][B] receives the block-neighbour matrix.
 */
int oracle_ljlk_pose_scores(const oracle_inputs_t* in, int block_pair,
                            real* out_E, real* out_dV, int32_t* out_nbr) {
  int P = in->P, B = in->B;
  real* spheres = (real*)malloc(sizeof(real) * 4 * (size_t)P * B + 16);
  if (!spheres) return 1;
  compute_spheres(in, spheres);
  detect_neighbors(in, spheres, out_nbr);
  free(spheres);
  size_t n_out = block_pair ? (size_t)3 * P * B * B : (size_t)3 * P;
  for (size_t k = 0; k < n_out; ++k) out_E[k] = 0;
  eval_t ev;
  ev.mode = (!block_pair && out_dV) ? MODE_ENERGY_AND_DERIVS : MODE_ENERGY;
  ev.dV = out_dV;
  if (out_dV && !block_pair)
    for (size_t k = 0; k < (size_t)9 * in->n_atoms; ++k) out_dV[k] = 0;
  for (int p = 0; p < P; ++p)
    for (int b1 = 0; b1 < B; ++b1)
      for (int b2 = b1; b2 < B; ++b2) {
        if (out_nbr[((size_t)p * B + b1) * B + b2] == 0) continue;
        pair_ctx_t c;
        if (!setup_pair(in, p, b1, b2, &c)) continue;
        real tot[3];
        eval_block_pair(in, &ev, &c, tot);
        for (int t = 0; t < 3; ++t) {
          if (block_pair)
            out_E[(((size_t)t * P + p) * B + b1) * B + b2] = tot[t];
          else
            out_E[(size_t)t * P + p] += tot[t];
        }
      }
  return 0;
}

/*
 * Recompute adjoint: dL/dx[n_atoms][3] = sum over neighbouring block pairs
 * (b1 <= b2) of dTdV[t][p][b1][b2] * dE_t(b1, b2)/dx, as the reference's
 * block-pair backward (ljlk_pose_score.impl.hh:1160-1477).  With
 * per_pose_weights != 0, dTdV is [3][P] and applies to every block pair of
 * the pose (the whole-pose adjoint).
 */
int oracle_ljlk_backward(const oracle_inputs_t* in, const int32_t* nbr,
                         const real* dTdV, int per_pose_weights, real* out_dx) {
  int P = in->P, B = in->B;
  for (size_t k = 0; k < (size_t)3 * in->n_atoms; ++k) out_dx[k] = 0;
  eval_t ev;
  ev.mode = MODE_WEIGHTED_DERIVS;
  ev.dV = out_dx;
  for (int p = 0; p < P; ++p)
    for (int b1 = 0; b1 < B; ++b1)
      for (int b2 = b1; b2 < B; ++b2) {
        if (nbr[((size_t)p * B + b1) * B + b2] == 0) continue;
        pair_ctx_t c;
        if (!setup_pair(in, p, b1, b2, &c)) continue;
        for (int t = 0; t < 3; ++t)
          ev.w[t] = per_pose_weights
                        ? dTdV[(size_t)t * P + p]
                        : dTdV[(((size_t)t * P + p) * B + b1) * B + b2];
        real tot[3];
        eval_block_pair(in, &ev, &c, tot);
      }
  return 0;
}

/* Number of atom pairs and heavy-atom pairs the neighbour list covers: the
 * benchmark's unit of work (inter: n1*n2, intra: n(n-1)/2). */
void oracle_count_pairs(const oracle_inputs_t* in, const int32_t* nbr,
                        int64_t* atom_pairs, int64_t* heavy_pairs) {
  int64_t ap = 0, hp = 0;
  int P = in->P, B = in->B;
  for (int p = 0; p < P; ++p)
    for (int b1 = 0; b1 < B; ++b1)
      for (int b2 = b1; b2 < B; ++b2) {
        if (nbr[((size_t)p * B + b1) * B + b2] == 0) continue;
        pair_ctx_t c;
        if (!setup_pair(in, p, b1, b2, &c)) continue;
        int h1 = 0, h2 = 0;
        for (int t = 0; in->term == 0 && t < in->ntiles; ++t) {
          h1 += in->bt_n_heavy_in_tile[c.bt1 * in->ntiles + t];
          h2 += in->bt_n_heavy_in_tile[c.bt2 * in->ntiles + t];
        }
        if (b1 != b2) {
          ap += (int64_t)c.n1 * c.n2;
          hp += (int64_t)h1 * h2;
        } else {
          ap += (int64_t)c.n1 * (c.n1 - 1) / 2;
          hp += (int64_t)h1 * (h1 - 1) / 2;
        }
      }
  *atom_pairs = ap;
  *heavy_pairs = hp;
}

int oracle_sizeof_real(void) { return (int)sizeof(real); }

/* ---------------------------------------------------------------------- */
/* Rotamer scoring (ljlk_pose_score.impl.hh:1479-2126).                    */

/* compute_rot_spheres (sphere_overlap.impl.hh:23-107) with the CPU launch
 * box (one thread): per rotamer, centroid of its atoms in order and the
 * largest centroid distance. */
static void rot_spheres(const oracle_inputs_t* in, real* rs) {
  for (int r = 0; r < in->n_rots; ++r) {
    real* s = rs + 4 * (size_t)r;
    s[0] = s[1] = s[2] = s[3] = 0;
    int bt = in->block_type_ind_for_rot[r];
    if (bt < 0) continue;
    int off = in->rot_coord_offset[r];
    int n = in->bt_n_atoms[bt];
    real c[3] = {0, 0, 0};
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) c[k] += in->coords[3 * (size_t)(off + i) + k];
    for (int k = 0; k < 3; ++k) c[k] /= n;
    real d2max = 0;
    for (int i = 0; i < n; ++i) {
      const real* x = in->coords + 3 * (size_t)(off + i);
      real d2 = ((x[0] - c[0]) * (x[0] - c[0]) + (x[1] - c[1]) * (x[1] - c[1]) +
                 (x[2] - c[2]) * (x[2] - c[2]));
      if (d2 > d2max) d2max = d2;
    }
    s[0] = c[0];
    s[1] = c[1];
    s[2] = c[2];
    s[3] = rsqrt_(d2max);
  }
}

/* compute_block_spheres_from_rot_spheres (sphere_overlap.impl.hh:455-510):
 * the mean of the block's rotamer centres and the largest centre distance
 * plus rotamer radius. */
static void block_spheres_from_rots(const oracle_inputs_t* in, const real* rs,
                                    real* bs) {
  for (int i = 0; i < in->P * in->B; ++i) {
    real* s = bs + 4 * (size_t)i;
    s[0] = s[1] = s[2] = s[3] = 0;
    int n = in->n_rots_for_block[i];
    int r0 = in->rot_offset_for_block[i];
    if (n <= 0 || r0 < 0) continue;
    real cx = 0, cy = 0, cz = 0;
    for (int r = 0; r < n; ++r) {
      cx += rs[4 * (size_t)(r0 + r) + 0];
      cy += rs[4 * (size_t)(r0 + r) + 1];
      cz += rs[4 * (size_t)(r0 + r) + 2];
    }
    cx /= n;
    cy /= n;
    cz /= n;
    real rmax = 0;
    for (int r = 0; r < n; ++r) {
      const real* q = rs + 4 * (size_t)(r0 + r);
      real dx = q[0] - cx, dy = q[1] - cy, dz = q[2] - cz;
      real d = rsqrt_(dx * dx + dy * dy + dz * dz) + q[3];
      if (d > rmax) rmax = d;
    }
    s[0] = cx;
    s[1] = cy;
    s[2] = cz;
    s[3] = rmax;
  }
}

/* Block neighbours of the rotamer op into nbr[P][B][B]; returns the number
 * of rotamer pairs it dispatches (rot_neighbor_indices_from_block_neighbors,
 * sphere_overlap.impl.hh:512-610): n_rots(b1) self pairs on the diagonal,
 * n_rots(b1) * n_rots(b2) pairs off it. */
int64_t oracle_ljlk_rotamer_count(const oracle_inputs_t* in, int32_t* nbr) {
  int P = in->P, B = in->B;
  real* rs = (real*)malloc(sizeof(real) * 4 * (size_t)(in->n_rots + 1));
  real* bs = (real*)malloc(sizeof(real) * 4 * ((size_t)P * B + 1));
  if (!rs || !bs) {
    free(rs);
    free(bs);
    return -1;
  }
  rot_spheres(in, rs);
  block_spheres_from_rots(in, rs, bs);
  detect_neighbors(in, bs, nbr);
  free(rs);
  free(bs);
  int64_t total = 0;
  for (int p = 0; p < P; ++p)
    for (int b1 = 0; b1 < B; ++b1)
      for (int b2 = b1; b2 < B; ++b2) {
        if (!nbr[((size_t)p * B + b1) * B + b2]) continue;
        int64_t n1 = in->n_rots_for_block[p * B + b1];
        int64_t n2 = in->n_rots_for_block[p * B + b2];
        total += b1 == b2 ? n1 : n1 * n2;
      }
  return total;
}

/* Visit every dispatched rotamer pair in the reference's order (pose, b1,
 * b2, rotamer of b1, rotamer of b2); fn(k, p, b1, b2, rot1, rot2). */
typedef void (*rot_pair_fn)(const oracle_inputs_t*, int64_t, int, int, int, int,
                            int, void*);
static void for_rot_pairs(const oracle_inputs_t* in, const int32_t* nbr,
                          rot_pair_fn fn, void* arg) {
  int P = in->P, B = in->B;
  int64_t k = 0;
  for (int p = 0; p < P; ++p)
    for (int b1 = 0; b1 < B; ++b1)
      for (int b2 = b1; b2 < B; ++b2) {
        if (!nbr[((size_t)p * B + b1) * B + b2]) continue;
        int n1 = in->n_rots_for_block[p * B + b1];
        int n2 = in->n_rots_for_block[p * B + b2];
        int o1 = in->rot_offset_for_block[p * B + b1];
        int o2 = in->rot_offset_for_block[p * B + b2];
        if (o1 < 0 || o2 < 0) continue;
        if (b1 == b2) {
          for (int i = 0; i < n1; ++i) fn(in, k++, p, b1, b2, o1 + i, o1 + i, arg);
        } else {
          for (int i = 0; i < n1; ++i)
            for (int j = 0; j < n2; ++j) fn(in, k++, p, b1, b2, o1 + i, o2 + j, arg);
        }
      }
}

typedef struct {
  eval_t ev;
  real* E;          /* [3][n] */
  int32_t* idx;     /* [3][n] */
  const real* dTdV; /* [3][n] */
  int64_t n;
} rot_job_t;

static void rot_pair_energy(const oracle_inputs_t* in, int64_t k, int p, int b1,
                            int b2, int rot1, int rot2, void* arg) {
  rot_job_t* job = (rot_job_t*)arg;
  job->idx[k] = p;
  job->idx[job->n + k] = rot1;
  job->idx[2 * job->n + k] = rot2;
  real tot[3] = {0, 0, 0};
  pair_ctx_t c;
  if (setup_rot_pair(in, p, b1, b2, rot1, rot2, &c)) eval_block_pair(in, &job->ev, &c, tot);
  for (int t = 0; t < 3; ++t) job->E[t * job->n + k] = tot[t];
}

static void rot_pair_adjoint(const oracle_inputs_t* in, int64_t k, int p, int b1,
                             int b2, int rot1, int rot2, void* arg) {
  rot_job_t* job = (rot_job_t*)arg;
  pair_ctx_t c;
  if (!setup_rot_pair(in, p, b1, b2, rot1, rot2, &c)) return;
  for (int t = 0; t < 3; ++t) job->ev.w[t] = job->dTdV[t * job->n + k];
  real tot[3];
  eval_block_pair(in, &job->ev, &c, tot);
}

/*
 * The rotamer-score op forward: out_E[3][n] energies of the n dispatched
 * rotamer pairs and out_idx[3][n] their (pose, rot1, rot2), n from
 * oracle_ljlk_rotamer_count (nbr as it returned).
 */
int oracle_ljlk_rotamer_scores(const oracle_inputs_t* in, const int32_t* nbr,
                               int64_t n, real* out_E, int32_t* out_idx) {
  rot_job_t job;
  job.ev.mode = MODE_ENERGY;
  job.ev.dV = NULL;
  job.E = out_E;
  job.idx = out_idx;
  job.dTdV = NULL;
  job.n = n;
  for_rot_pairs(in, nbr, rot_pair_energy, &job);
  return 0;
}

/* Its adjoint: out_dx[n_atoms][3] = sum_k sum_t dTdV[t][k] dE_t(pair k)/dx
 * (ljlk_pose_score.impl.hh:1826-2126). */
int oracle_ljlk_rotamer_backward(const oracle_inputs_t* in, const int32_t* nbr,
                                 int64_t n, const real* dTdV, real* out_dx) {
  for (size_t k = 0; k < (size_t)3 * in->n_atoms; ++k) out_dx[k] = 0;
  rot_job_t job;
  job.ev.mode = MODE_WEIGHTED_DERIVS;
  job.ev.dV = out_dx;
  job.E = NULL;
  job.idx = NULL;
  job.dTdV = dTdV;
  job.n = n;
  for_rot_pairs(in, nbr, rot_pair_adjoint, &job);
  return 0;
}

/* ====================================================================== */
/* LK-ball (tmol/score/lk_ball/potentials): waters built on polar atoms    */
/* (water.hh:330-601, gen_pose_waters.impl.hh:30-250, acceptor bases       */
/* hbond/identification.hh:27-160, bond walk bonded_atom.hh:157-270) and   */
/* the four-term pair potential (lk_ball.hh:34-540) over polar / occluder  */
/* pairs of neighbouring blocks (lk_ball.hh:1270-1360,                     */
/* lk_ball_pose_score.impl.hh:330-540).  Shared inputs come in             */
/* oracle_inputs_t: bt_path_distance is the plain bond separation and      */
/* bt_is_ligand all zero (LK-ball has no ligand count-pair rule).  Sums    */
/* run in pair order, not the reference's tile order, so results agree to */
/* rounding, not bit for bit.                                              */

#define LKB_NW 4
#define LKB_NP 9

typedef struct {
  const int32_t* irc;          /* [P][B][C][2] */
  const int32_t* all_bonds;    /* [nbt][NB][3] */
  const int32_t* bond_ranges;  /* [nbt][A][2] */
  int NB, NT;
  const int32_t* tile_n_donH;  /* [nbt][NT] */
  const int32_t* tile_n_acc;
  const int32_t* tile_donH_inds; /* [nbt][NT][32] */
  const int32_t* tile_donH_hvy;
  const int32_t* tile_which_donH;
  const int32_t* tile_acc_inds;
  const int32_t* tile_acc_hyb;
  const int32_t* tile_acc_nH;
  const int32_t* is_hydrogen;  /* [nbt][A] */
  const int32_t* tile_n_polar; /* [nbt][NT] */
  const int32_t* tile_n_occ;
  const int32_t* tile_pol_occ; /* [nbt][NT][32] */
  const real* tile_params;     /* [nbt][NT][32][9] */
  real water_dist, ang_sp2, ang_sp3, ang_ring;
  const real* tors_sp2;
  const real* tors_sp3;
  const real* tors_ring;
  int n_sp2, n_sp3, n_ring;
  real hbond_dis, hbond_OH_donor_dis, hbond_hdis, max_dis;
} lkb_inputs_t;

typedef struct {
  int block, bt, atom;
} bcat_t;

static int bcat_eq(bcat_t a, bcat_t b) { return a.block == b.block && a.bt == b.bt && a.atom == b.atom; }

/* the k-th bonded neighbour of (block, bt, atom) in pose p: an intra-block
 * bond, or across connection c to the partner's connection atom; an
 * unresolved connection gives atom -1 */
static bcat_t lkb_bonded(const oracle_inputs_t* in, const lkb_inputs_t* k, int p, bcat_t x, int bidx) {
  const int32_t* e = k->all_bonds + ((size_t)x.bt * k->NB + bidx) * 3;
  bcat_t r = {x.block, x.bt, e[1]};
  if (e[1] >= 0) return r;
  const int32_t* t = k->irc + (((size_t)p * in->B + x.block) * in->C + e[2]) * 2;
  if (t[1] < 0) {
    r.block = r.bt = r.atom = -1;
    return r;
  }
  r.block = t[0];
  r.bt = in->first_rot_block_type[(size_t)p * in->B + t[0]];
  if (r.bt < 0) {
    /* a partner block without a rotamer (a rotamer set may leave blocks
     * out): the bond does not resolve */
    r.block = r.atom = -1;
    return r;
  }
  r.atom = in->bt_conn_atom[(size_t)r.bt * in->C + t[1]];
  return r;
}

static int lkb_is_h(const lkb_inputs_t* k, const oracle_inputs_t* in, bcat_t x) {
  return x.atom >= 0 && k->is_hydrogen[(size_t)x.bt * in->A + x.atom];
}

static void lkb_range(const oracle_inputs_t* in, const lkb_inputs_t* k, bcat_t x, int* lo, int* hi) {
  const int32_t* r = k->bond_ranges + ((size_t)x.bt * in->A + x.atom) * 2;
  *lo = r[0];
  *hi = r[1];
}

/* identification.hh:35-148; hyb 1 sp2, 2 sp3, 3 ring.  Returns 0 when the
 * water frame is undefined (no base, or B0 == B). */
static int lkb_acc_bases(const oracle_inputs_t* in, const lkb_inputs_t* k, int p, bcat_t A, int hyb, bcat_t* B,
                         bcat_t* B0) {
  bcat_t none = {-1, -1, -1};
  int lo, hi;
  *B = none;
  *B0 = none;
  if (hyb < 1 || hyb > 3) return 0;
  lkb_range(in, k, A, &lo, &hi);
  for (int i = lo; i < hi; ++i) {
    bcat_t o = lkb_bonded(in, k, p, A, i);
    if (o.atom >= 0 && !lkb_is_h(k, in, o)) {
      *B = o;
      break;
    }
  }
  if (hyb == 1) {
    if (B->atom < 0) return 0;
    int lo2, hi2;
    lkb_range(in, k, *B, &lo2, &hi2);
    for (int i = lo2; i < hi2; ++i) {
      bcat_t o = lkb_bonded(in, k, p, *B, i);
      if (o.atom < 0) continue;
      if (B->block != A.block && o.block == A.block) continue;
      if (!bcat_eq(o, A)) {
        *B0 = o;
        break;
      }
    }
    if (B0->atom < 0) return 0;
  } else if (hyb == 2) {
    for (int i = lo; i < hi; ++i) {
      bcat_t o = lkb_bonded(in, k, p, A, i);
      if (o.atom >= 0 && !bcat_eq(o, *B) && lkb_is_h(k, in, o)) {
        *B0 = o;
        break;
      }
    }
    if (B0->atom < 0)
      for (int i = lo; i < hi; ++i) {
        bcat_t o = lkb_bonded(in, k, p, A, i);
        if (o.atom >= 0 && !bcat_eq(o, *B)) {
          *B0 = o;
          break;
        }
      }
    if (B0->atom < 0) *B0 = *B;
  } else {
    if (B->atom < 0) return 0;
    for (int i = lo; i < hi; ++i) {
      bcat_t o = lkb_bonded(in, k, p, A, i);
      if (o.atom >= 0 && !bcat_eq(o, *B) && !lkb_is_h(k, in, o)) {
        *B0 = o;
        break;
      }
    }
    if (B0->atom < 0) return 0;
  }
  if (B->atom < 0 || bcat_eq(*B0, *B)) return 0;
  return 1;
}

static size_t lkb_atom_row(const oracle_inputs_t* in, int p, bcat_t x) {
  int rot = in->rot_offset_for_block[(size_t)p * in->B + x.block];
  return (size_t)in->rot_coord_offset[rot] + x.atom;
}

static void v3_load(const real* c, size_t row, real v[3]) {
  v[0] = c[3 * row];
  v[1] = c[3 * row + 1];
  v[2] = c[3 * row + 2];
}
static real v3_dot(const real* a, const real* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void v3_cross(const real* a, const real* b, real* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

/* gen_coord.hh:40-74: the point at `dist` from A, angle(W, A, B) = angle,
 * torsion(W, A, B, C) = torsion.  M = [e0, e1, e2] with e0 = (A - B) / |A - B|,
 * e2 = e0 x (C - B) normalised, e1 = e2 x e0. */
typedef struct {
  real e0[3], e1[3], e2[3], u[3], c[3], nd, nu, v[3];
} frame_t;

static void lkb_frame(const real* A, const real* Bp, const real* C, real dist, real angle, real tor, frame_t* f) {
  const real pi = (real)3.14159265358979323846;
  real d[3];
  for (int i = 0; i < 3; ++i) {
    d[i] = A[i] - Bp[i];
    f->c[i] = C[i] - Bp[i];
  }
  f->nd = rsqrt_(v3_dot(d, d));
  for (int i = 0; i < 3; ++i) f->e0[i] = d[i] / f->nd;
  v3_cross(f->e0, f->c, f->u);
  f->nu = rsqrt_(v3_dot(f->u, f->u));
  if (f->nu == 0) {
    real alt[3] = {1, 0, 0};
    if (f->e0[0] == 1 || f->e0[0] == -1) {
      alt[0] = 0;
      alt[1] = 1;
    }
    v3_cross(f->e0, alt, f->u);
    f->nu = rsqrt_(v3_dot(f->u, f->u));
  }
  for (int i = 0; i < 3; ++i) f->e2[i] = f->u[i] / f->nu;
  v3_cross(f->e2, f->e0, f->e1);
  real sa = (real)sin(pi - angle), ca = (real)cos(pi - angle);
  f->v[0] = dist * ca;
  f->v[1] = dist * sa * (real)cos(tor);
  f->v[2] = dist * sa * (real)sin(tor);
}

static void lkb_build(const real* A, const frame_t* f, real* W) {
  for (int i = 0; i < 3; ++i) W[i] = A[i] + f->v[0] * f->e0[i] + f->v[1] * f->e1[i] + f->v[2] * f->e2[i];
}

/* vector-Jacobian product of lkb_build: gA, gB, gC += d(g . W)/d(A, B, C) */
static void lkb_build_vjp(const frame_t* f, const real* g, real* gA, real* gB, real* gC) {
  real ge0[3], ge1[3], ge2[3], t[3], gu[3], gd[3];
  for (int i = 0; i < 3; ++i) {
    gA[i] += g[i];
    ge0[i] = f->v[0] * g[i];
    ge1[i] = f->v[1] * g[i];
    ge2[i] = f->v[2] * g[i];
  }
  /* e1 = e2 x e0 */
  v3_cross(f->e0, ge1, t);
  for (int i = 0; i < 3; ++i) ge2[i] += t[i];
  v3_cross(ge1, f->e2, t);
  for (int i = 0; i < 3; ++i) ge0[i] += t[i];
  /* e2 = u / |u| */
  real s = v3_dot(f->e2, ge2);
  for (int i = 0; i < 3; ++i) gu[i] = (ge2[i] - f->e2[i] * s) / f->nu;
  /* u = e0 x c */
  v3_cross(f->c, gu, t);
  for (int i = 0; i < 3; ++i) ge0[i] += t[i];
  real gc[3];
  v3_cross(gu, f->e0, gc);
  /* e0 = (A - B) / |A - B| */
  s = v3_dot(f->e0, ge0);
  for (int i = 0; i < 3; ++i) gd[i] = (ge0[i] - f->e0[i] * s) / f->nd;
  for (int i = 0; i < 3; ++i) {
    gA[i] += gd[i];
    gB[i] -= gd[i] + gc[i];
    gC[i] += gc[i];
  }
}

/* one water site: its atoms and how it is built */
typedef struct {
  int kind;  /* 0 none, 1 donor (D, H), 2 acceptor (A, B, B0) */
  int hyb;
  size_t rowA, rowB, rowB0; /* donor: rowA = D, rowB = H */
  real tor, ang;
} lkb_site_t;

/* the coordinate row of x for waters built on rotamer `rot` (block b at
 * offset off): its own block from the rotamer's coordinates, other blocks
 * from their first rotamer's (water.hh:318-327) */
static size_t lkb_row(const oracle_inputs_t* in, int p, int b, size_t off, bcat_t x) {
  return x.block == b ? off + x.atom : lkb_atom_row(in, p, x);
}

/* the site of water slot `w` of each atom of rotamer `rot`, or kind 0
 * (gen_pose_waters.impl.hh:112-175, per rotamer as the reference runs it;
 * in the pose op each block's one rotamer) */
static void lkb_sites_for_rot(const oracle_inputs_t* in, const lkb_inputs_t* k, int rot,
                              lkb_site_t* sites /* [n_atoms][4] */) {
  int bt = in->block_type_ind_for_rot[rot];
  int p = in->pose_ind_for_rot[rot], b = in->block_ind_for_rot[rot];
  size_t off = in->rot_coord_offset[rot];
  int n = in->bt_n_atoms[bt];
  for (int i = 0; i < n * LKB_NW; ++i) sites[i].kind = 0;
  for (int t = 0; t < k->NT; ++t) {
    size_t tb = ((size_t)bt * k->NT + t);
    for (int q = 0; q < k->tile_n_donH[tb]; ++q) {
      int H = t * TILE + k->tile_donH_inds[tb * TILE + q];
      int D = k->tile_donH_hvy[tb * TILE + q];
      int which = k->tile_which_donH[tb * TILE + q];
      bcat_t dh = {b, bt, D}, hh = {b, bt, H};
      lkb_site_t* s = &sites[D * LKB_NW + which];
      s->kind = 1;
      s->rowA = lkb_row(in, p, b, off, dh);
      s->rowB = lkb_row(in, p, b, off, hh);
    }
    for (int q = 0; q < k->tile_n_acc[tb]; ++q) {
      int Aat = t * TILE + k->tile_acc_inds[tb * TILE + q];
      int hyb = k->tile_acc_hyb[tb * TILE + q];
      int nH = k->tile_acc_nH[tb * TILE + q];
      bcat_t A = {b, bt, Aat}, Bb, B0;
      if (!lkb_acc_bases(in, k, p, A, hyb, &Bb, &B0)) continue;
      const real* tors = hyb == 1 ? k->tors_sp2 : hyb == 2 ? k->tors_sp3 : k->tors_ring;
      int nt = hyb == 1 ? k->n_sp2 : hyb == 2 ? k->n_sp3 : k->n_ring;
      real ang = hyb == 1 ? k->ang_sp2 : hyb == 2 ? k->ang_sp3 : k->ang_ring;
      for (int w = 0; w < LKB_NW && w < nt; ++w) {
        if (w + nH >= LKB_NW) break;
        lkb_site_t* s = &sites[Aat * LKB_NW + w + nH];
        s->kind = 2;
        s->hyb = hyb;
        s->rowA = lkb_row(in, p, b, off, A);
        s->rowB = lkb_row(in, p, b, off, Bb);
        s->rowB0 = lkb_row(in, p, b, off, B0);
        s->tor = tors[w];
        s->ang = ang;
      }
    }
  }
}

static void lkb_site_water(const oracle_inputs_t* in, const lkb_inputs_t* k, const lkb_site_t* s, real* W,
                           frame_t* f) {
  real A[3], Bv[3], B0v[3];
  v3_load(in->coords, s->rowA, A);
  v3_load(in->coords, s->rowB, Bv);
  if (s->kind == 1) {
    /* water.hh:42-44: D + dist * (H - D) / |H - D| */
    real h[3] = {Bv[0] - A[0], Bv[1] - A[1], Bv[2] - A[2]};
    real nh = rsqrt_(v3_dot(h, h));
    for (int i = 0; i < 3; ++i) W[i] = A[i] + k->water_dist * (h[i] / nh);
    return;
  }
  v3_load(in->coords, s->rowB0, B0v);
  if (s->hyb == 3)
    for (int i = 0; i < 3; ++i) Bv[i] = (Bv[i] + B0v[i]) / 2;
  lkb_frame(A, Bv, B0v, k->water_dist, s->ang, s->tor, f);
  lkb_build(A, f, W);
}

/* gen_pose_waters: W [n_atoms][4][3], NAN where no water is built */
int oracle_lkb_waters(const oracle_inputs_t* in, const lkb_inputs_t* k, real* W) {
  for (size_t i = 0; i < (size_t)in->n_atoms * LKB_NW * 3; ++i) W[i] = (real)NAN;
  lkb_site_t* sites = (lkb_site_t*)malloc(sizeof(lkb_site_t) * (size_t)in->A * LKB_NW);
  if (!sites) return 2;
  for (int rot = 0; rot < in->n_rots; ++rot) {
    int bt = in->block_type_ind_for_rot[rot];
    if (bt < 0) continue;
    lkb_sites_for_rot(in, k, rot, sites);
    size_t off = in->rot_coord_offset[rot];
    for (int a = 0; a < in->bt_n_atoms[bt]; ++a)
      for (int w = 0; w < LKB_NW; ++w) {
        frame_t f;
        if (sites[a * LKB_NW + w].kind)
          lkb_site_water(in, k, &sites[a * LKB_NW + w], W + ((off + a) * LKB_NW + w) * 3, &f);
      }
  }
  free(sites);
  return 0;
}

/* lk_ball.hh:34-39 */
static const real lkb_overlap_gap = (real)0.5, lkb_overlap_width = (real)2.6;
#define LKB_ANGLE_OVERLAP ((real)2.8 * lkb_overlap_width)
static const real lkb_ramp_width = (real)3.709;
static real sq_(real v) { return v * v; }

/* lk_fraction (lk_ball.hh:42-124): value and d/dJ, d/dWI */
static real lkb_fraction(const real* WI, const real* J, real lj_radius_j, real* dJ, real* dWI) {
  real d2_low = sq_((real)1.4 + lj_radius_j) - lkb_ramp_width;
  if (d2_low < 0) d2_low = 0;
  real wsum = 0, gJ[3] = {0, 0, 0}, gW[LKB_NW * 3] = {0};
  for (int w = 0; w < LKB_NW; ++w) {
    real dl[3] = {J[0] - WI[3 * w], J[1] - WI[3 * w + 1], J[2] - WI[3 * w + 2]};
    real d2 = v3_dot(dl, dl) - d2_low;
    if (isnan(d2)) continue;
    real e = rexp_(-d2);
    wsum += e;
    for (int i = 0; i < 3; ++i) {
      gJ[i] += 2 * e * dl[i];
      gW[3 * w + i] = -2 * e * dl[i];
    }
  }
  if (wsum != 0)
    for (int i = 0; i < 3; ++i) {
      gJ[i] /= wsum;
      for (int w = 0; w < LKB_NW; ++w) gW[3 * w + i] /= wsum;
    }
  real x = -(real)log(wsum);
  real frac = 0, df = 0;
  if (x < 0)
    frac = 1;
  else if (x < lkb_ramp_width)
    frac = sq_(1 - sq_(x / lkb_ramp_width));
  if (x > 0 && x < lkb_ramp_width)
    df = -4 * x * (sq_(lkb_ramp_width) - sq_(x)) / sq_(sq_(lkb_ramp_width));
  if (dJ)
    for (int i = 0; i < 3; ++i) dJ[i] = gJ[i] * df;
  if (dWI)
    for (int i = 0; i < LKB_NW * 3; ++i) dWI[i] = gW[i] * df;
  return frac;
}

/* lk_bridge_fraction (lk_ball.hh:126-277) */
static real lkb_bridge(const real* I, const real* J, const real* WI, const real* WJ, real water_dist, real* dI,
                       real* dJ, real* dWI, real* dWJ) {
  real wsum = 0, gWI[LKB_NW * 3] = {0}, gWJ[LKB_NW * 3] = {0};
  for (int a = 0; a < LKB_NW; ++a)
    for (int c = 0; c < LKB_NW; ++c) {
      real dl[3] = {WI[3 * a] - WJ[3 * c], WI[3 * a + 1] - WJ[3 * c + 1], WI[3 * a + 2] - WJ[3 * c + 2]};
      real d2 = v3_dot(dl, dl) - lkb_overlap_gap;
      if (isnan(d2)) continue;
      real e = rexp_(-d2);
      for (int i = 0; i < 3; ++i) {
        gWI[3 * a + i] += 2 * e * dl[i];
        gWJ[3 * c + i] -= 2 * e * dl[i];
      }
      wsum += e;
    }
  if (wsum != 0)
    for (int i = 0; i < LKB_NW * 3; ++i) {
      gWI[i] /= wsum;
      gWJ[i] /= wsum;
    }
  real x = -(real)log(wsum);
  real ofrac, dof;
  if (x > lkb_overlap_width) {
    ofrac = 0;
    dof = 0;
  } else if (x > 0) {
    ofrac = sq_(1 - sq_(x / lkb_overlap_width));
    dof = -4 * x * (sq_(lkb_overlap_width) - sq_(x)) / sq_(sq_(lkb_overlap_width));
  } else {
    ofrac = 1;
    dof = 0;
  }
  real target = (real)(8.0 / 3.0) * sq_(water_dist);
  real dIJ[3] = {I[0] - J[0], I[1] - J[1], I[2] - J[2]};
  real base = v3_dot(dIJ, dIJ) - target;
  real afrac, daf;
  real ab = base < 0 ? -base : base;
  if (ab > LKB_ANGLE_OVERLAP) {
    afrac = 0;
    daf = 0;
  } else if (ab > 0) {
    afrac = sq_(1 - sq_(base / LKB_ANGLE_OVERLAP));
    daf = -4 * base * (sq_(LKB_ANGLE_OVERLAP) - sq_(base)) / sq_(sq_(LKB_ANGLE_OVERLAP));
  } else {
    afrac = 1;
    daf = 0;
  }
  if (dI)
    for (int i = 0; i < 3; ++i) {
      dI[i] = ofrac * daf * 2 * dIJ[i];
      dJ[i] = -ofrac * daf * 2 * dIJ[i];
    }
  if (dWI)
    for (int i = 0; i < LKB_NW * 3; ++i) {
      dWI[i] = afrac * dof * gWI[i];
      dWJ[i] = afrac * dof * gWJ[i];
    }
  return ofrac * afrac;
}

typedef struct {
  real lj_radius, lk_dgfree, lk_lambda, lk_volume, is_donor, is_hydroxyl, is_polarh, is_acceptor, is_carbon_lk;
} lkb_params_t;

/* ljlk common.hh:25-44 with LK-ball's atom parameters */
static real lkb_sigma(const lkb_params_t* i, const lkb_params_t* j, const lkb_inputs_t* k) {
  if ((i->is_donor != 0 && j->is_acceptor != 0) || (j->is_donor != 0 && i->is_acceptor != 0)) {
    if ((i->is_donor != 0 && i->is_hydroxyl != 0) || (j->is_donor != 0 && j->is_hydroxyl != 0))
      return k->hbond_OH_donor_dis;
    return k->hbond_dis;
  } else if ((i->is_polarh != 0 && j->is_acceptor != 0) || (j->is_polarh != 0 && i->is_acceptor != 0)) {
    return k->hbond_hdis;
  }
  return i->lj_radius + j->lj_radius;
}

/* lk_ball_score (lk_ball.hh:335-500) for polar I (waters WI) against
 * occluder J (waters WJ): E[4]; with g (dL/dE[4]) the adjoint adds to
 * gI, gJ, gWI, gWJ */
static void lkb_pair(const real* I, const real* J, const real* WI, const real* WJ, int sep, const lkb_params_t* pi,
                     const lkb_params_t* pj, const lkb_inputs_t* k, real* E, const real* g, real* gI, real* gJ,
                     real* gWI, real* gWJ) {
  E[0] = E[1] = E[2] = E[3] = 0;
  if (sep <= 3) return;
  real dv[3] = {I[0] - J[0], I[1] - J[1], I[2] - J[2]};
  real dist = rsqrt_(v3_dot(dv, dv));
  if (dist >= k->max_dis) return;
  if (isnan(WI[0])) return;
  real sigma = lkb_sigma(pi, pj, k);
  real iso, diso;
  lk_isotropic_pair_V_dV(dist, (real)sep, sigma, pi->lj_radius, pi->lk_dgfree, pi->lk_lambda, pj->lk_volume,
                         k->max_dis, pi->is_carbon_lk != 0 && pj->is_carbon_lk != 0, &iso, &diso);
  real fdJ[3], fdWI[LKB_NW * 3];
  real fdes = lkb_fraction(WI, J, pj->lj_radius, fdJ, fdWI);
  real bdI[3] = {0, 0, 0}, bdJ[3] = {0, 0, 0}, bdWI[LKB_NW * 3] = {0}, bdWJ[LKB_NW * 3] = {0};
  real fov = 0;
  if (pj->is_donor != 0 || pj->is_acceptor != 0) fov = lkb_bridge(I, J, WI, WJ, k->water_dist, bdI, bdJ, bdWI, bdWJ);
  E[0] = iso;
  E[1] = iso * fdes;
  E[2] = iso * fov;
  E[3] = fov / 2;
  if (!g) return;
  /* unit vector of the distance, zero at coincidence (geom.hh:20-40) */
  real u[3] = {0, 0, 0};
  if (dist != 0)
    for (int i = 0; i < 3; ++i) u[i] = dv[i] / dist;
  real giso = g[0] + g[1] * fdes + g[2] * fov;
  for (int i = 0; i < 3; ++i) {
    gI[i] += giso * diso * u[i] + g[2] * iso * bdI[i] + g[3] * bdI[i] / 2;
    gJ[i] += -giso * diso * u[i] + g[1] * iso * fdJ[i] + g[2] * iso * bdJ[i] + g[3] * bdJ[i] / 2;
  }
  for (int i = 0; i < LKB_NW * 3; ++i) {
    gWI[i] += g[1] * iso * fdWI[i] + g[2] * iso * bdWI[i] + g[3] * bdWI[i] / 2;
    gWJ[i] += g[2] * iso * bdWJ[i] + g[3] * bdWJ[i] / 2;
  }
}

/* polar / occluder lists of one block (all tiles): block-type atom index
 * and parameters */
static int lkb_lists(const oracle_inputs_t* in, const lkb_inputs_t* k, int bt, int* pol, int* occ, int* n_pol,
                     const real** ppar, const real** opar) {
  int np = 0, no = 0;
  for (int t = 0; t < k->NT; ++t) {
    size_t tb = (size_t)bt * k->NT + t;
    int npt = k->tile_n_polar[tb], nott = k->tile_n_occ[tb];
    for (int q = 0; q < nott; ++q) {
      int a = t * TILE + k->tile_pol_occ[tb * TILE + q];
      const real* par = k->tile_params + (tb * TILE + q) * LKB_NP;
      if (q < npt) {
        pol[np] = a;
        ppar[np++] = par;
      }
      occ[no] = a;
      opar[no++] = par;
    }
  }
  *n_pol = np;
  return no;
}

/* scratch for the polar / occluder lists of the two sides of a pair */
typedef struct {
  int *pol1, *occ1, *pol2, *occ2;
  const real **ppar1, **opar1, **ppar2, **opar2;
  void* mem;
} lkb_lists_t;

static int lkb_lists_alloc(lkb_lists_t* L, int A) {
  int* ib = (int*)malloc(sizeof(int) * 4 * (size_t)(A + 1));
  const real** pb = (const real**)malloc(sizeof(real*) * 4 * (size_t)(A + 1));
  if (!ib || !pb) {
    free(ib);
    free((void*)pb);
    return 0;
  }
  L->pol1 = ib, L->occ1 = ib + (A + 1), L->pol2 = ib + 2 * (A + 1), L->occ2 = ib + 3 * (A + 1);
  L->ppar1 = pb, L->opar1 = pb + (A + 1), L->ppar2 = pb + 2 * (A + 1), L->opar2 = pb + 3 * (A + 1);
  L->mem = pb;
  return 1;
}

static void lkb_lists_free(lkb_lists_t* L) {
  free(L->pol1);
  free(L->mem);
}

/* Every polar / occluder pair of the rotamer pair in c (one side's polars
 * against the other side's occluders, both ways; within one rotamer,
 * ordered pairs of distinct atoms; lk_ball.hh:1270-1360): energies added
 * to e4[4]; with g4, the adjoint of g4 . E added to dx (directly) and gW
 * (the waters). */
static void lkb_eval_ctx(const oracle_inputs_t* in, const lkb_inputs_t* k, const real* W, const pair_ctx_t* c,
                         lkb_lists_t* L, const real* g4, real* e4, real* dx, real* gW) {
  const int same = c->rot1 == c->rot2;
  int np1, np2;
  int no1 = lkb_lists(in, k, c->bt1, L->pol1, L->occ1, &np1, L->ppar1, L->opar1);
  int no2 = lkb_lists(in, k, c->bt2, L->pol2, L->occ2, &np2, L->ppar2, L->opar2);
  for (int side = 0; side < 2; ++side) {
    if (same && side == 1) break;
    const int* pol = side ? L->pol2 : L->pol1;
    const real** ppar = side ? L->ppar2 : L->ppar1;
    int npol = side ? np2 : np1;
    const int* occ = same ? L->occ1 : (side ? L->occ1 : L->occ2);
    const real** opar = same ? L->opar1 : (side ? L->opar1 : L->opar2);
    int nocc = same ? no1 : (side ? no1 : no2);
    size_t offp = side ? c->off2 : c->off1, offo = same ? c->off1 : (side ? c->off1 : c->off2);
    for (int x = 0; x < npol; ++x)
      for (int y = 0; y < nocc; ++y) {
        int ap = pol[x], ao = occ[y];
        if (same && ap == ao) continue;
        int sep;
        if (same)
          sep = in->bt_path_distance[((size_t)c->bt1 * in->A + ap) * in->A + ao];
        else
          sep = side ? inter_separation(in, c, ao, ap) : inter_separation(in, c, ap, ao);
        size_t rp = offp + ap, ro = offo + ao;
        real I[3], J[3], e[4];
        v3_load(in->coords, rp, I);
        v3_load(in->coords, ro, J);
        lkb_params_t pi, pj;
        memcpy(&pi, ppar[x], sizeof(pi));
        memcpy(&pj, opar[y], sizeof(pj));
        real gI[3] = {0, 0, 0}, gJ[3] = {0, 0, 0}, gWI[LKB_NW * 3] = {0}, gWJ[LKB_NW * 3] = {0};
        lkb_pair(I, J, W + rp * LKB_NW * 3, W + ro * LKB_NW * 3, sep, &pi, &pj, k, e, g4, gI, gJ, gWI, gWJ);
        for (int t = 0; t < 4; ++t) e4[t] += e[t];
        if (g4) {
          for (int i = 0; i < 3; ++i) {
            dx[3 * rp + i] += gI[i];
            dx[3 * ro + i] += gJ[i];
          }
          for (int i = 0; i < LKB_NW * 3; ++i) {
            gW[rp * LKB_NW * 3 + i] += gWI[i];
            gW[ro * LKB_NW * 3 + i] += gWJ[i];
          }
        }
      }
  }
}

/* The waters' adjoint onto the atoms that place them: dx += d(waters)/dx^T
 * gW (water.hh:412-600), every rotamer's waters. */
static int lkb_waters_adjoint(const oracle_inputs_t* in, const lkb_inputs_t* k, const real* gW, real* dx) {
  lkb_site_t* sites = (lkb_site_t*)malloc(sizeof(lkb_site_t) * (size_t)(in->A + 1) * LKB_NW);
  if (!sites) return 2;
  for (int rot = 0; rot < in->n_rots; ++rot) {
    int bt = in->block_type_ind_for_rot[rot];
    if (bt < 0) continue;
    lkb_sites_for_rot(in, k, rot, sites);
    size_t off = in->rot_coord_offset[rot];
    for (int a = 0; a < in->bt_n_atoms[bt]; ++a)
      for (int w = 0; w < LKB_NW; ++w) {
        const lkb_site_t* s = &sites[a * LKB_NW + w];
        if (!s->kind) continue;
        const real* g = gW + ((off + a) * LKB_NW + w) * 3;
        if (g[0] == 0 && g[1] == 0 && g[2] == 0) continue;
        real Av[3], Bv[3];
        v3_load(in->coords, s->rowA, Av);
        v3_load(in->coords, s->rowB, Bv);
        if (s->kind == 1) {
          real h[3] = {Bv[0] - Av[0], Bv[1] - Av[1], Bv[2] - Av[2]};
          real nh = rsqrt_(v3_dot(h, h));
          real n[3] = {h[0] / nh, h[1] / nh, h[2] / nh};
          real gn[3] = {k->water_dist * g[0], k->water_dist * g[1], k->water_dist * g[2]};
          real sdot = v3_dot(n, gn);
          for (int i = 0; i < 3; ++i) {
            real gh = (gn[i] - n[i] * sdot) / nh;
            dx[3 * s->rowA + i] += g[i] - gh;
            dx[3 * s->rowB + i] += gh;
          }
          continue;
        }
        real B0v[3], Bm[3];
        v3_load(in->coords, s->rowB0, B0v);
        for (int i = 0; i < 3; ++i) Bm[i] = s->hyb == 3 ? (Bv[i] + B0v[i]) / 2 : Bv[i];
        frame_t f;
        lkb_frame(Av, Bm, B0v, k->water_dist, s->ang, s->tor, &f);
        real gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0}, gC[3] = {0, 0, 0};
        lkb_build_vjp(&f, g, gA, gB, gC);
        for (int i = 0; i < 3; ++i) {
          dx[3 * s->rowA + i] += gA[i];
          if (s->hyb == 3) {
            dx[3 * s->rowB + i] += gB[i] / 2;
            dx[3 * s->rowB0 + i] += gB[i] / 2;
          } else {
            dx[3 * s->rowB + i] += gB[i];
          }
          dx[3 * s->rowB0 + i] += gC[i];
        }
      }
  }
  free(sites);
  return 0;
}

/* lk_ball_pose_score, whole-pose: E [4][P]; with wts [4][P] the gradient of
 * sum_t wts[t][p] E[t][p] w.r.t. the coordinates (through the waters) goes
 * to dx [n_atoms][3]; nbr [P][B][B] gets the block-neighbour matrix. */
int oracle_lkb_pose_scores(const oracle_inputs_t* in, const lkb_inputs_t* k, const real* W, real* E,
                           const real* wts, real* dx, int32_t* nbr) {
  const int P = in->P, B = in->B;
  real* spheres = (real*)malloc(sizeof(real) * 4 * ((size_t)P * B + 1));
  real* gW = dx ? (real*)calloc((size_t)in->n_atoms * LKB_NW * 3 + 1, sizeof(real)) : NULL;
  lkb_lists_t L;
  if (!spheres || (dx && !gW) || !lkb_lists_alloc(&L, in->A)) return 2;
  compute_spheres(in, spheres);
  detect_neighbors(in, spheres, nbr);
  for (size_t i = 0; i < (size_t)4 * P; ++i) E[i] = 0;
  if (dx)
    for (size_t i = 0; i < (size_t)in->n_atoms * 3; ++i) dx[i] = 0;
  for (int p = 0; p < P; ++p)
    for (int b1 = 0; b1 < B; ++b1)
      for (int b2 = b1; b2 < B; ++b2) {
        if (!nbr[((size_t)p * B + b1) * B + b2]) continue;
        pair_ctx_t c;
        if (!setup_pair(in, p, b1, b2, &c)) continue;
        real g4[4], e4[4] = {0, 0, 0, 0};
        if (dx)
          for (int t = 0; t < 4; ++t) g4[t] = wts[(size_t)t * P + p];
        lkb_eval_ctx(in, k, W, &c, &L, dx ? g4 : NULL, e4, dx, gW);
        for (int t = 0; t < 4; ++t) E[(size_t)t * P + p] += e4[t];
      }
  int rc = dx ? lkb_waters_adjoint(in, k, gW, dx) : 0;
  free(spheres);
  lkb_lists_free(&L);
  free(gW);
  return rc;
}

/* lk_ball_rotamer_score (LKBallRotamerScoreDispatch, lk_ball_pose_score.impl.hh:
 * 1005-1380): the four energies E [4][n] of the n rotamer pairs that
 * oracle_ljlk_rotamer_count dispatched (nbr as it returned), in its order,
 * with their (pose, rot1, rot2) in idx [3][n]; with dTdV [4][n], dx
 * [n_atoms][3] gets the gradient of sum dTdV * E through the waters. */
int oracle_lkb_rotamer_scores(const oracle_inputs_t* in, const lkb_inputs_t* k, const real* W,
                              const int32_t* nbr, int64_t n, real* E, int32_t* idx, const real* dTdV, real* dx) {
  const int P = in->P, B = in->B;
  real* gW = dx ? (real*)calloc((size_t)in->n_atoms * LKB_NW * 3 + 1, sizeof(real)) : NULL;
  lkb_lists_t L;
  if ((dx && !gW) || !lkb_lists_alloc(&L, in->A)) return 2;
  if (dx)
    for (size_t i = 0; i < (size_t)in->n_atoms * 3; ++i) dx[i] = 0;
  int64_t q = 0;
  for (int p = 0; p < P; ++p)
    for (int b1 = 0; b1 < B; ++b1)
      for (int b2 = b1; b2 < B; ++b2) {
        if (!nbr[((size_t)p * B + b1) * B + b2]) continue;
        int n1 = in->n_rots_for_block[p * B + b1], n2 = in->n_rots_for_block[p * B + b2];
        int o1 = in->rot_offset_for_block[p * B + b1], o2 = in->rot_offset_for_block[p * B + b2];
        if (o1 < 0 || o2 < 0) continue;
        for (int i = 0; i < n1; ++i)
          for (int j = 0; j < (b1 == b2 ? 1 : n2); ++j) {
            int r1 = o1 + i, r2 = b1 == b2 ? o1 + i : o2 + j;
            if (q >= n) return 3;
            idx[q] = p;
            idx[n + q] = r1;
            idx[2 * n + q] = r2;
            real e4[4] = {0, 0, 0, 0}, g4[4];
            pair_ctx_t c;
            if (setup_rot_pair(in, p, b1, b2, r1, r2, &c)) {
              if (dx)
                for (int t = 0; t < 4; ++t) g4[t] = dTdV[(size_t)t * n + q];
              lkb_eval_ctx(in, k, W, &c, &L, dx ? g4 : NULL, e4, dx, gW);
            }
            for (int t = 0; t < 4; ++t) E[(size_t)t * n + q] = e4[t];
            ++q;
          }
      }
  int rc = q == n ? 0 : 3;
  if (!rc && dx) rc = lkb_waters_adjoint(in, k, gW, dx);
  lkb_lists_free(&L);
  free(gW);
  return rc;
}
