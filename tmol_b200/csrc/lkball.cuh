// LK-ball on B200: water sites, water building and its adjoint, and the
// four-term polar / occluder pair potential (tmol/score/lk_ball/potentials:
// water.hh, lk_ball.hh; acceptor bases tmol/score/hbond/identification.hh:26-168).
// Included by ljlk.cu inside namespace tmol_b200, after ScoreArgs and the
// LJ/LK kernels, whose plan (neighbour detection, count-pair tables, work
// items) the LK-ball kernels share.
//
// A plan resolves, once, every water a PoseStack can carry into a "site":
// the coordinate rows of the atoms that place it (donor: heavy atom and
// hydrogen; acceptor: the acceptor and its two base atoms, which may sit in
// bonded blocks) and its torsion / angle.  Per call, one thread per (atom,
// slot) builds the waters; the scoring kernel walks the plan's work items
// like score_kernel and evaluates every polar / occluder pair of each
// neighbouring block pair, lanes striding over the pairs; the adjoint
// accumulates d/dcoords and d/dwaters with atomics, and a second pass moves
// d/dwaters onto the placing atoms.

constexpr int LKB_NW = 4;    // waters per polar atom
constexpr int LKB_NPAR = 9;  // per-atom parameters

enum LkbSiteKind : int { kLkbNone = 0, kLkbDonor = 1, kLkbSp2 = 2, kLkbSp3 = 3, kLkbRing = 4 };

template <typename Real>
struct LkbSite {
  int kind;
  int rowA, rowB, rowB0;  // donor: rowA = heavy atom, rowB = hydrogen
  Real tor, ang;
};

template <typename Real>
struct LkbArgs {
  const LkbSite<Real>* sites;  // [n_atoms * 4]
  int64_t n_sites;
  const int* active;  // the occupied sites (kind != none), ascending
  int64_t n_active;
  const Real* waters;   // [n_atoms][4][3]
  Real* waters_out;
  const Real* dwaters;  // adjoint in
  Real* dwaters_out;    // adjoint out
  const int* pol;       // [nbt][maxpol] polar atoms of each block type
  const int* npol;      // [nbt]
  const int* occ;       // [nbt][maxocc] heavy atoms (polar ones included), donors / acceptors first
  const int* nocc;
  const int* nbocc;     // [nbt] leading occluders that are donors or acceptors (the bridge term)
  int maxpol, maxocc;
  const Real* par;      // [nbt][A][9]
  Real water_dist, hbond_dis, hbond_oh, hbond_h, max_dis;
};

// ---------------------------------------------------------------------------
// plan time: sites

struct LkbTables {
  const int32_t* irc;          // [P][B][C][2]
  const int32_t* all_bonds;    // [nbt][NB][3]
  const int32_t* ranges;       // [nbt][A][2]
  int NB, NT;
  const int32_t* tile_n_donH;  // [nbt][NT]
  const int32_t* tile_n_acc;
  const int32_t* tile_donH;    // [nbt][NT][32]
  const int32_t* tile_donH_hvy;
  const int32_t* tile_which;
  const int32_t* tile_acc;
  const int32_t* tile_hyb;
  const int32_t* tile_nH;
  const int32_t* is_h;         // [nbt][A]
  const int32_t* bt_conn_atom; // [nbt][C]
};

struct LkbAtom {
  int block, bt, atom;
};

__device__ __forceinline__ bool lkb_same(LkbAtom a, LkbAtom b) {
  return a.block == b.block && a.bt == b.bt && a.atom == b.atom;
}

// bonded neighbour k of x (bonded_atom.hh:157-260): intra-block, or the
// partner's connection atom across a connection; atom -1 if unresolved
__device__ inline LkbAtom lkb_bonded(const LkbTables& t, const int* blk_bt, int p, int B, int C, LkbAtom x,
                                     int bidx) {
  const int32_t* e = t.all_bonds + ((int64_t)x.bt * t.NB + bidx) * 3;
  LkbAtom r = {x.block, x.bt, e[1]};
  if (e[1] >= 0) return r;
  if (e[2] < 0 || e[2] >= C) return LkbAtom{-1, -1, -1};
  const int32_t* c = t.irc + (((int64_t)p * B + x.block) * C + e[2]) * 2;
  if (c[1] < 0 || c[1] >= C || c[0] < 0 || c[0] >= B) return LkbAtom{-1, -1, -1};
  r.block = c[0];
  r.bt = blk_bt[p * B + c[0]];
  if (r.bt < 0) return LkbAtom{-1, -1, -1};
  r.atom = t.bt_conn_atom[(int64_t)r.bt * C + c[1]];
  return r;
}

__device__ __forceinline__ bool lkb_is_h(const LkbTables& t, int A, LkbAtom x) {
  return x.atom >= 0 && x.atom < A && t.is_h[(int64_t)x.bt * A + x.atom];
}

// an atom's bond range, clamped to the table
__device__ __forceinline__ void lkb_range(const LkbTables& t, int A, LkbAtom x, int& lo, int& hi) {
  lo = hi = 0;
  if (x.atom < 0 || x.atom >= A) return;
  const int32_t* r = t.ranges + ((int64_t)x.bt * A + x.atom) * 2;
  lo = r[0] < 0 ? 0 : r[0];
  hi = r[1] > t.NB ? t.NB : r[1];
}

// acceptor bases (identification.hh:32-150); false when the water frame
// is undefined
__device__ inline bool lkb_bases(const LkbTables& t, const int* blk_bt, int p, int B, int C, int A, LkbAtom a,
                                 int hyb, LkbAtom& b, LkbAtom& b0) {
  const LkbAtom none = {-1, -1, -1};
  b = none;
  b0 = none;
  if (hyb < 1 || hyb > 3) return false;
  int lo, hi;
  lkb_range(t, A, a, lo, hi);
  for (int i = lo; i < hi; ++i) {
    LkbAtom o = lkb_bonded(t, blk_bt, p, B, C, a, i);
    if (o.atom >= 0 && !lkb_is_h(t, A, o)) {
      b = o;
      break;
    }
  }
  if (hyb == 1) {
    if (b.atom < 0) return false;
    int lo2, hi2;
    lkb_range(t, A, b, lo2, hi2);
    for (int i = lo2; i < hi2; ++i) {
      LkbAtom o = lkb_bonded(t, blk_bt, p, B, C, b, i);
      if (o.atom < 0) continue;
      if (b.block != a.block && o.block == a.block) continue;
      if (!lkb_same(o, a)) {
        b0 = o;
        break;
      }
    }
    if (b0.atom < 0) return false;
  } else if (hyb == 2) {
    for (int i = lo; i < hi; ++i) {
      LkbAtom o = lkb_bonded(t, blk_bt, p, B, C, a, i);
      if (o.atom >= 0 && !lkb_same(o, b) && lkb_is_h(t, A, o)) {
        b0 = o;
        break;
      }
    }
    if (b0.atom < 0)
      for (int i = lo; i < hi; ++i) {
        LkbAtom o = lkb_bonded(t, blk_bt, p, B, C, a, i);
        if (o.atom >= 0 && !lkb_same(o, b)) {
          b0 = o;
          break;
        }
      }
    if (b0.atom < 0) b0 = b;
  } else {
    if (b.atom < 0) return false;
    for (int i = lo; i < hi; ++i) {
      LkbAtom o = lkb_bonded(t, blk_bt, p, B, C, a, i);
      if (o.atom >= 0 && !lkb_same(o, b) && !lkb_is_h(t, A, o)) {
        b0 = o;
        break;
      }
    }
    if (b0.atom < 0) return false;
  }
  return b.atom >= 0 && !lkb_same(b0, b);
}

// The rotamer-set indexing the sites are built from (the op's own
// arguments, read at plan time): waters are built per rotamer, with atoms of
// other blocks taken from those blocks' first rotamers (water.hh:318-327).
struct LkbRots {
  const int32_t* rot_coord_offset;      // [R]
  const int32_t* pose_ind_for_rot;      // [R]
  const int32_t* block_ind_for_rot;     // [R]
  const int32_t* block_type_ind_for_rot;// [R]
  const int32_t* first_rot_for_block;   // [P][B]
  const int32_t* first_rot_block_type;  // [P][B]
  const int32_t* bt_n_atoms;            // [nbt]
  int R, nbt;
  int64_t N;
};

// x's coordinate row for waters of rotamer (p, b, off); -1 if unresolved
__device__ __forceinline__ int64_t lkb_row(const LkbRots& r, int p, int B, int b, int off, LkbAtom x) {
  if (x.block == b) return (int64_t)off + x.atom;
  const int fr = r.first_rot_for_block[p * B + x.block];
  if (fr < 0 || fr >= r.R) return -1;
  return (int64_t)r.rot_coord_offset[fr] + x.atom;
}

// One thread per rotamer: its water sites, the donor and acceptor waters
// the reference builds per rotamer (gen_pose_waters.impl.hh:112-175;
// water.hh:332-445).  In the pose op every block has one rotamer.
template <typename Real>
__global__ void lkb_sites_kernel(LkbRots rs, int P, int B, int C, int A, LkbTables t,
                                 const Real* tors_sp2, int n_sp2, const Real* tors_sp3, int n_sp3,
                                 const Real* tors_ring, int n_ring, Real ang_sp2, Real ang_sp3, Real ang_ring,
                                 LkbSite<Real>* sites, int* status) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rs.R; r += gridDim.x * blockDim.x) {
    const int bt = rs.block_type_ind_for_rot[r];
    if (bt < 0) continue;
    const int p = rs.pose_ind_for_rot[r], b = rs.block_ind_for_rot[r];
    const int off = rs.rot_coord_offset[r];
    if (bt >= rs.nbt || p < 0 || p >= P || b < 0 || b >= B || off < 0) {
      atomicOr(status, kStIndex);
      continue;
    }
    const int n = rs.bt_n_atoms[bt];
    if ((int64_t)off + n > rs.N) {
      atomicOr(status, kStIndex);
      continue;
    }
    for (int tt = 0; tt < t.NT; ++tt) {
      const int64_t tb = (int64_t)bt * t.NT + tt;
      for (int q = 0; q < t.tile_n_donH[tb]; ++q) {
        const int h = tt * TILE + t.tile_donH[tb * TILE + q];
        const int d = t.tile_donH_hvy[tb * TILE + q];
        const int w = t.tile_which[tb * TILE + q];
        if (d < 0 || d >= n || h < 0 || h >= n || w < 0 || w >= LKB_NW) {
          atomicOr(status, kStIndex);
          continue;
        }
        LkbSite<Real> s;
        s.kind = kLkbDonor;
        s.rowA = off + d;
        s.rowB = off + h;
        s.rowB0 = off + d;
        s.tor = s.ang = 0;
        sites[(int64_t)(off + d) * LKB_NW + w] = s;
      }
      for (int q = 0; q < t.tile_n_acc[tb]; ++q) {
        const int a = tt * TILE + t.tile_acc[tb * TILE + q];
        const int hyb = t.tile_hyb[tb * TILE + q];
        const int nh = t.tile_nH[tb * TILE + q];
        if (a < 0 || a >= n || nh < 0) {
          atomicOr(status, kStIndex);
          continue;
        }
        LkbAtom x = {b, bt, a}, bb, b0;
        if (!lkb_bases(t, rs.first_rot_block_type, p, B, C, A, x, hyb, bb, b0)) continue;
        const int64_t rb = lkb_row(rs, p, B, b, off, bb), rb0 = lkb_row(rs, p, B, b, off, b0);
        if (bb.atom >= rs.bt_n_atoms[bb.bt] || b0.atom >= rs.bt_n_atoms[b0.bt] || rb < 0 || rb0 < 0 ||
            rb >= rs.N || rb0 >= rs.N) {
          atomicOr(status, kStIndex);
          continue;
        }
        const Real* tors = hyb == 1 ? tors_sp2 : (hyb == 2 ? tors_sp3 : tors_ring);
        const int nt = hyb == 1 ? n_sp2 : (hyb == 2 ? n_sp3 : n_ring);
        const Real ang = hyb == 1 ? ang_sp2 : (hyb == 2 ? ang_sp3 : ang_ring);
        for (int w = 0; w < nt && w + nh < LKB_NW; ++w) {
          LkbSite<Real> s;
          s.kind = kLkbDonor + hyb;
          s.rowA = off + a;
          s.rowB = (int)rb;
          s.rowB0 = (int)rb0;
          s.tor = tors[w];
          s.ang = ang;
          sites[(int64_t)(off + a) * LKB_NW + w + nh] = s;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// water building (water.hh:42-44; gen_coord.hh:40-74) and its adjoint

template <typename Real>
struct LkbFrame {
  Real e0[3], e1[3], e2[3], c[3], nd, nu, v[3];
};

template <typename Real>
__device__ __forceinline__ void lkb_cross(const Real* a, const Real* b, Real* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

template <typename Real>
__device__ __forceinline__ Real lkb_dot(const Real* a, const Real* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ float lkb_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double lkb_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float lkb_exp(float x) { return expf(x); }
__device__ __forceinline__ double lkb_exp(double x) { return exp(x); }
__device__ __forceinline__ float lkb_log(float x) { return logf(x); }
__device__ __forceinline__ double lkb_log(double x) { return log(x); }
__device__ __forceinline__ void lkb_sincos(float x, float* s, float* c) { sincosf(x, s, c); }
__device__ __forceinline__ void lkb_sincos(double x, double* s, double* c) { sincos(x, s, c); }

template <typename Real>
__device__ inline void lkb_frame(const Real* A, const Real* Bp, const Real* C, Real dist, Real angle, Real tor,
                                 LkbFrame<Real>& f) {
  Real d[3], u[3];
  for (int i = 0; i < 3; ++i) {
    d[i] = A[i] - Bp[i];
    f.c[i] = C[i] - Bp[i];
  }
  f.nd = lkb_sqrt(lkb_dot(d, d));
  for (int i = 0; i < 3; ++i) f.e0[i] = d[i] / f.nd;
  lkb_cross(f.e0, f.c, u);
  f.nu = lkb_sqrt(lkb_dot(u, u));
  if (f.nu == Real(0)) {
    Real alt[3] = {1, 0, 0};
    if (f.e0[0] == Real(1) || f.e0[0] == Real(-1)) {
      alt[0] = 0;
      alt[1] = 1;
    }
    lkb_cross(f.e0, alt, u);
    f.nu = lkb_sqrt(lkb_dot(u, u));
  }
  for (int i = 0; i < 3; ++i) f.e2[i] = u[i] / f.nu;
  lkb_cross(f.e2, f.e0, f.e1);
  Real sa, ca, st, ct;
  lkb_sincos(Real(3.14159265358979323846) - angle, &sa, &ca);
  lkb_sincos(tor, &st, &ct);
  f.v[0] = dist * ca;
  f.v[1] = dist * sa * ct;
  f.v[2] = dist * sa * st;
}

template <typename Real>
__device__ __forceinline__ void lkb_load3(const Real* c, int64_t row, Real* v) {
  v[0] = c[3 * row];
  v[1] = c[3 * row + 1];
  v[2] = c[3 * row + 2];
}

template <typename Real>
__device__ inline void lkb_site_water(const LkbSite<Real>& s, const Real* coords, Real dist, Real* W) {
  Real A[3], Bv[3];
  lkb_load3(coords, s.rowA, A);
  lkb_load3(coords, s.rowB, Bv);
  if (s.kind == kLkbDonor) {
    Real h[3] = {Bv[0] - A[0], Bv[1] - A[1], Bv[2] - A[2]};
    const Real nh = lkb_sqrt(lkb_dot(h, h));
    for (int i = 0; i < 3; ++i) W[i] = A[i] + dist * (h[i] / nh);
    return;
  }
  Real B0v[3];
  lkb_load3(coords, s.rowB0, B0v);
  if (s.kind == kLkbRing)
    for (int i = 0; i < 3; ++i) Bv[i] = (Bv[i] + B0v[i]) / 2;
  LkbFrame<Real> f;
  lkb_frame(A, Bv, B0v, dist, s.ang, s.tor, f);
  for (int i = 0; i < 3; ++i) W[i] = A[i] + f.v[0] * f.e0[i] + f.v[1] * f.e1[i] + f.v[2] * f.e2[i];
}

// The waters of the occupied sites (the empty slots hold NaN, written
// beforehand as a byte fill)
template <typename Real>
__global__ void lkb_waters_kernel(LkbArgs<Real> k, const Real* coords) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < k.n_active;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = k.active[j];
    const LkbSite<Real> s = k.sites[i];
    Real W[3];
    lkb_site_water(s, coords, k.water_dist, W);
    k.waters_out[3 * i] = W[0];
    k.waters_out[3 * i + 1] = W[1];
    k.waters_out[3 * i + 2] = W[2];
  }
}

// dcoords += the adjoint of each occupied site's water
template <typename Real>
__global__ void lkb_waters_backward_kernel(LkbArgs<Real> k, const Real* coords, Real* dcoords) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < k.n_active;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = k.active[j];
    const LkbSite<Real> s = k.sites[i];
    const Real g[3] = {k.dwaters[3 * i], k.dwaters[3 * i + 1], k.dwaters[3 * i + 2]};
    if (g[0] == Real(0) && g[1] == Real(0) && g[2] == Real(0)) continue;
    Real A[3], Bv[3];
    lkb_load3(coords, s.rowA, A);
    lkb_load3(coords, s.rowB, Bv);
    Real gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0}, gC[3] = {0, 0, 0};
    if (s.kind == kLkbDonor) {
      Real h[3] = {Bv[0] - A[0], Bv[1] - A[1], Bv[2] - A[2]};
      const Real nh = lkb_sqrt(lkb_dot(h, h));
      Real n[3] = {h[0] / nh, h[1] / nh, h[2] / nh};
      Real gn[3] = {k.water_dist * g[0], k.water_dist * g[1], k.water_dist * g[2]};
      const Real sd = lkb_dot(n, gn);
      for (int j = 0; j < 3; ++j) {
        const Real gh = (gn[j] - n[j] * sd) / nh;
        gA[j] = g[j] - gh;
        gB[j] = gh;
      }
      for (int j = 0; j < 3; ++j) {
        atomicAdd(&dcoords[3 * (int64_t)s.rowA + j], gA[j]);
        atomicAdd(&dcoords[3 * (int64_t)s.rowB + j], gB[j]);
      }
      continue;
    }
    Real B0v[3], Bm[3];
    lkb_load3(coords, s.rowB0, B0v);
    for (int j = 0; j < 3; ++j) Bm[j] = s.kind == kLkbRing ? (Bv[j] + B0v[j]) / 2 : Bv[j];
    LkbFrame<Real> f;
    lkb_frame(A, Bm, B0v, k.water_dist, s.ang, s.tor, f);
    // reverse mode through W = A + v0 e0 + v1 e1 + v2 e2
    Real ge0[3], ge1[3], ge2[3], tmp[3], gu[3];
    for (int j = 0; j < 3; ++j) {
      gA[j] = g[j];
      ge0[j] = f.v[0] * g[j];
      ge1[j] = f.v[1] * g[j];
      ge2[j] = f.v[2] * g[j];
    }
    lkb_cross(f.e0, ge1, tmp);  // e1 = e2 x e0
    for (int j = 0; j < 3; ++j) ge2[j] += tmp[j];
    lkb_cross(ge1, f.e2, tmp);
    for (int j = 0; j < 3; ++j) ge0[j] += tmp[j];
    Real sd = lkb_dot(f.e2, ge2);  // e2 = u / |u|
    for (int j = 0; j < 3; ++j) gu[j] = (ge2[j] - f.e2[j] * sd) / f.nu;
    lkb_cross(f.c, gu, tmp);  // u = e0 x c
    for (int j = 0; j < 3; ++j) ge0[j] += tmp[j];
    Real gc[3];
    lkb_cross(gu, f.e0, gc);
    sd = lkb_dot(f.e0, ge0);  // e0 = (A - B) / |A - B|
    for (int j = 0; j < 3; ++j) {
      const Real gd = (ge0[j] - f.e0[j] * sd) / f.nd;
      gA[j] += gd;
      gB[j] = -gd - gc[j];
      gC[j] = gc[j];
    }
    for (int j = 0; j < 3; ++j) {
      atomicAdd(&dcoords[3 * (int64_t)s.rowA + j], gA[j]);
      if (s.kind == kLkbRing) {
        atomicAdd(&dcoords[3 * (int64_t)s.rowB + j], gB[j] / 2);
        atomicAdd(&dcoords[3 * (int64_t)s.rowB0 + j], gB[j] / 2);
      } else {
        atomicAdd(&dcoords[3 * (int64_t)s.rowB + j], gB[j]);
      }
      atomicAdd(&dcoords[3 * (int64_t)s.rowB0 + j], gC[j]);
    }
  }
}

// ---------------------------------------------------------------------------
// the pair potential (lk_ball.hh:34-500)

template <typename Real>
struct LkbParams {
  Real lj_radius, lk_dgfree, lk_lambda, lk_volume, is_donor, is_hydroxyl, is_polarh, is_acceptor, is_carbon_lk;
};

template <typename Real>
__device__ __forceinline__ Real lkb_sq(Real v) {
  return v * v;
}

// lk_fraction: value, d/dJ, d/dWI
template <typename Real, bool GRAD>
__device__ inline Real lkb_fraction(const Real* WI, const Real* J, Real lj_radius_j, Real* dJ, Real* dWI) {
  const Real ramp = Real(3.709);
  Real d2_low = lkb_sq(Real(1.4) + lj_radius_j) - ramp;
  if (d2_low < Real(0)) d2_low = 0;
  Real wsum = 0, gJ[3] = {0, 0, 0}, gW[LKB_NW * 3];
#pragma unroll
  for (int i = 0; i < LKB_NW * 3; ++i) gW[i] = 0;
#pragma unroll
  for (int w = 0; w < LKB_NW; ++w) {
    const Real dl[3] = {J[0] - WI[3 * w], J[1] - WI[3 * w + 1], J[2] - WI[3 * w + 2]};
    const Real d2 = lkb_dot(dl, dl) - d2_low;
    if (isnan(d2)) continue;
    const Real e = lkb_exp(-d2);
    wsum += e;
    if (GRAD)
      for (int i = 0; i < 3; ++i) {
        gJ[i] += 2 * e * dl[i];
        gW[3 * w + i] = -2 * e * dl[i];
      }
  }
  const Real x = -lkb_log(wsum);
  Real frac = 0;
  if (x < Real(0))
    frac = 1;
  else if (x < ramp)
    frac = lkb_sq(Real(1) - lkb_sq(x / ramp));
  if (GRAD) {
    Real df = 0;
    if (x > Real(0) && x < ramp) df = -4 * x * (lkb_sq(ramp) - lkb_sq(x)) / lkb_sq(lkb_sq(ramp));
    const Real inv = wsum != Real(0) ? Real(1) / wsum : Real(1);
    for (int i = 0; i < 3; ++i) dJ[i] = gJ[i] * inv * df;
    for (int i = 0; i < LKB_NW * 3; ++i) dWI[i] = gW[i] * inv * df;
  }
  return frac;
}

// lk_bridge_fraction
template <typename Real, bool GRAD>
__device__ inline Real lkb_bridge(const Real* I, const Real* J, const Real* WI, const Real* WJ, Real water_dist,
                                  Real* dI, Real* dJ, Real* dWI, Real* dWJ) {
  const Real gap = Real(0.5), width = Real(2.6), aover = Real(2.8) * Real(2.6);
  Real wsum = 0;
  if (GRAD)
    for (int i = 0; i < LKB_NW * 3; ++i) dWI[i] = dWJ[i] = 0;
#pragma unroll 1
  for (int a = 0; a < LKB_NW; ++a)
#pragma unroll
    for (int c = 0; c < LKB_NW; ++c) {
      const Real dl[3] = {WI[3 * a] - WJ[3 * c], WI[3 * a + 1] - WJ[3 * c + 1], WI[3 * a + 2] - WJ[3 * c + 2]};
      const Real d2 = lkb_dot(dl, dl) - gap;
      if (isnan(d2)) continue;
      const Real e = lkb_exp(-d2);
      if (GRAD)
        for (int i = 0; i < 3; ++i) {
          dWI[3 * a + i] += 2 * e * dl[i];
          dWJ[3 * c + i] -= 2 * e * dl[i];
        }
      wsum += e;
    }
  const Real x = -lkb_log(wsum);
  Real ofrac, dof = 0;
  if (x > width) {
    ofrac = 0;
  } else if (x > Real(0)) {
    ofrac = lkb_sq(Real(1) - lkb_sq(x / width));
    dof = -4 * x * (lkb_sq(width) - lkb_sq(x)) / lkb_sq(lkb_sq(width));
  } else {
    ofrac = 1;
  }
  const Real dIJ[3] = {I[0] - J[0], I[1] - J[1], I[2] - J[2]};
  const Real base = lkb_dot(dIJ, dIJ) - Real(8.0 / 3.0) * lkb_sq(water_dist);
  const Real ab = base < Real(0) ? -base : base;
  Real afrac, daf = 0;
  if (ab > aover) {
    afrac = 0;
  } else if (ab > Real(0)) {
    afrac = lkb_sq(Real(1) - lkb_sq(base / aover));
    daf = -4 * base * (lkb_sq(aover) - lkb_sq(base)) / lkb_sq(lkb_sq(aover));
  } else {
    afrac = 1;
  }
  if (GRAD) {
    const Real inv = wsum != Real(0) ? Real(1) / wsum : Real(1);
    for (int i = 0; i < 3; ++i) {
      dI[i] = ofrac * daf * 2 * dIJ[i];
      dJ[i] = -ofrac * daf * 2 * dIJ[i];
    }
    for (int i = 0; i < LKB_NW * 3; ++i) {
      dWI[i] *= afrac * dof * inv;
      dWJ[i] *= afrac * dof * inv;
    }
  }
  return ofrac * afrac;
}

template <typename Real, typename K>
__device__ __forceinline__ Real lkb_sigma(const LkbParams<Real>& i, const LkbParams<Real>& j, const K& k) {
  const bool di = i.is_donor != 0, dj = j.is_donor != 0, ai = i.is_acceptor != 0, aj = j.is_acceptor != 0;
  if ((di && aj) || (dj && ai)) {
    if ((di && i.is_hydroxyl != 0) || (dj && j.is_hydroxyl != 0)) return k.hbond_oh;
    return k.hbond_dis;
  }
  if ((i.is_polarh != 0 && aj) || (j.is_polarh != 0 && ai)) return k.hbond_h;
  return i.lj_radius + j.lj_radius;
}

// one direction of lk_isotropic (lk_isotropic.hh:97-236)
template <typename Real>
__device__ inline void lkb_lk_pair(Real dist, int sep, Real sigma, Real ri, Real dgi, Real lami, Real volj,
                                   Real max_dis, bool cc, Real& V, Real& dV) {
  Real d_min = sigma * Real(.89);
  if (cc) d_min = d_min > Real(4.2) ? d_min : Real(4.2);
  const Real n = floor(Real(20) * d_min * d_min);
  const Real close_dmin = lkb_sqrt((n - 29 > Real(0) ? n - 29 : Real(0)) / 20);
  const Real close_dmax = lkb_sqrt((n + 21 < Real(405) ? n + 21 : Real(405)) / 20);
  const Real far_dmax = max_dis, far_dmin = max_dis - Real(1.5);
  const Real weight = sep > 4 ? Real(1) : (sep == 4 ? Real(0.2) : Real(0));
  const Real pref = -volj * dgi / (2 * Real(5.56832799683f) * lami);  // pi^1.5 as a float literal, as tmol has it
  auto f = [&](Real d, Real& v, Real& dv) {
    const Real z = (d - ri) / lami;
    const Real ex = lkb_exp(-z * z);
    v = pref / (d * d) * ex;
    dv = pref * ex * (Real(-2) / (d * d * d) + Real(1) / (d * d) * -(2 * d - 2 * ri) / (lami * lami));
  };
  Real lk = 0, dlk = 0;
  if (dist < close_dmin) {
    Real v, dv;
    f(d_min, v, dv);
    lk = v;
  } else if (dist < close_dmax) {
    Real v0, dv0, v1, dv1;
    f(d_min, v0, dv0);
    f(close_dmax, v1, dv1);
    hermite_V_dV(dist, close_dmin, v0, Real(0), close_dmax, v1, dv1, lk, dlk);
  } else if (dist < far_dmin) {
    f(dist, lk, dlk);
  } else if (dist < far_dmax) {
    Real v0, dv0;
    f(far_dmin, v0, dv0);
    hermite_V_dV(dist, far_dmin, v0, dv0, far_dmax, Real(0), Real(0), lk, dlk);
  }
  V = weight * lk;
  dV = weight * dlk;
}

// lk_ball_score (lk_ball.hh:335-500) for polar I against occluder J: E[4]
// and, with GRAD, the adjoint of g . E onto I, J, WI, WJ (added).  Returns
// 0 when the pair is out of reach (bond separation, distance, no water),
// 1 when evaluated, 2 when evaluated with the water-bridge term.
template <typename Real, bool GRAD, typename K>
__device__ inline int lkb_pair(const Real* I, const Real* J, const Real* WI, const Real* WJ, int sep,
                                const LkbParams<Real>& pi, const LkbParams<Real>& pj, const K& k,
                                Real* E, const Real* g, Real* gI, Real* gJ, Real* gWI, Real* gWJ) {
  E[0] = E[1] = E[2] = E[3] = 0;
  if (sep <= 3) return 0;
  const Real dv[3] = {I[0] - J[0], I[1] - J[1], I[2] - J[2]};
  const Real dist = lkb_sqrt(lkb_dot(dv, dv));
  if (dist >= k.max_dis) return 0;
  if (isnan(WI[0])) return 0;
  const Real sigma = lkb_sigma(pi, pj, k);
  Real iso, diso;
  lkb_lk_pair(dist, sep, sigma, pi.lj_radius, pi.lk_dgfree, pi.lk_lambda, pj.lk_volume, k.max_dis,
              pi.is_carbon_lk != 0 && pj.is_carbon_lk != 0, iso, diso);
  Real fdJ[3], fdWI[LKB_NW * 3];
  const Real fdes = lkb_fraction<Real, GRAD>(WI, J, pj.lj_radius, fdJ, fdWI);
  Real bdI[3] = {0, 0, 0}, bdJ[3] = {0, 0, 0}, bdWI[LKB_NW * 3], bdWJ[LKB_NW * 3];
  Real fov = 0;
  const bool bridged = pj.is_donor != 0 || pj.is_acceptor != 0;
  if (bridged) {
    fov = lkb_bridge<Real, GRAD>(I, J, WI, WJ, k.water_dist, bdI, bdJ, bdWI, bdWJ);
  } else if (GRAD) {
    for (int i = 0; i < LKB_NW * 3; ++i) bdWI[i] = bdWJ[i] = 0;
  }
  E[0] = iso;
  E[1] = iso * fdes;
  E[2] = iso * fov;
  E[3] = fov / 2;
  if (!GRAD) return bridged ? 2 : 1;
  Real u[3] = {0, 0, 0};
  if (dist != Real(0))
    for (int i = 0; i < 3; ++i) u[i] = dv[i] / dist;
  const Real giso = g[0] + g[1] * fdes + g[2] * fov;
  for (int i = 0; i < 3; ++i) {
    gI[i] += giso * diso * u[i] + g[2] * iso * bdI[i] + g[3] * bdI[i] / 2;
    gJ[i] += -giso * diso * u[i] + g[1] * iso * fdJ[i] + g[2] * iso * bdJ[i] + g[3] * bdJ[i] / 2;
  }
  for (int i = 0; i < LKB_NW * 3; ++i) {
    gWI[i] += g[1] * iso * fdWI[i] + g[2] * iso * bdWI[i] + g[3] * bdWI[i] / 2;
    gWJ[i] += g[2] * iso * bdWJ[i] + g[3] * bdWJ[i] / 2;
  }
  return bridged ? 2 : 1;
}

// ---------------------------------------------------------------------------
// scoring kernel: the plan's work items (pose, b1, candidate blocks), the
// neighbour rule as score_kernel applies it, then every polar / occluder
// pair of each neighbouring block pair (intra-block: ordered pairs of
// distinct atoms; inter-block: polars of either block against occluders of
// the other), lanes striding over the pairs.

template <typename Real>
__device__ __forceinline__ int lkb_inter_sep(const ScoreArgs<Real>& s, int bt1, int bt2, int nc1, int nc2,
                                             const uint8_t* seps, int a1, int a2) {
  int sep = 5;  // one past the largest separation that matters (4)
  for (int u = 0; u < nc1; ++u) {
    const int pd1 = s.bt_conn_pd[((int64_t)bt1 * s.C + u) * s.A + a1];
    for (int v = 0; v < nc2; ++v) {
      const int t = pd1 + seps[u * 4 + v] + s.bt_conn_pd[((int64_t)bt2 * s.C + v) * s.A + a2];
      sep = t < sep ? t : sep;
    }
  }
  return sep;
}

template <typename Real, typename K>
__device__ __forceinline__ LkbParams<Real> lkb_params(const K& k, int A, int bt, int atom) {
  const Real* q = k.par + ((int64_t)bt * A + atom) * LKB_NPAR;
  LkbParams<Real> r;
  r.lj_radius = q[0];
  r.lk_dgfree = q[1];
  r.lk_lambda = q[2];
  r.lk_volume = q[3];
  r.is_donor = q[4];
  r.is_hydroxyl = q[5];
  r.is_polarh = q[6];
  r.is_acceptor = q[7];
  r.is_carbon_lk = q[8];
  return r;
}

// Pairs in reach wait in two per-warp queues, those whose occluder bridges
// (donor or acceptor: the 4 x 4 water-pair term) and the rest, and are
// evaluated 32 at a time with every lane busy on the same branch.
constexpr int LKB_Q = 64;
// warps per CTA of the LK-ball kernels (launches clamp to it)
constexpr int LKB_MAX_WARPS = 8;

template <bool TAGGED>
struct LkbQueue {
  int rp[LKB_Q], ro[LKB_Q], pi[LKB_Q], oi[LKB_Q];  // coordinate rows; (bt * A + atom) of the polar / occluder
  int tag[TAGGED ? LKB_Q : 1];  // the output row each pair belongs to (tagged queues only)
  uint8_t sep[LKB_Q];
};

// What evaluating a queued pair needs (a compact by-value context).
template <typename Real>
struct LkbEval {
  const Real* coords;
  const Real* waters;
  const Real* par;
  Real* dcoords;
  Real* dwaters;
  int A;
  Real water_dist, hbond_dis, hbond_oh, hbond_h, max_dis;
};

template <typename Real>
struct Lkb4 {
  Real v[4];
};

// Evaluates entry `lane` of q when lane < n: returns its four energies and,
// with GRAD, adds the adjoint of w . E to dcoords / dwaters.
// inlined: an out-of-line copy (smaller code) measured 34% slower, its
// calling convention spilling the kernel's state
#ifndef TMOL_B200_LKB_DRAIN_ATTR
#define TMOL_B200_LKB_DRAIN_ATTR __forceinline__
#endif
// two 256-thread CTAs per SM (128 registers): measured faster than one
// (182 registers) and than three (80 registers, spilling)
#ifndef TMOL_B200_LKB_MIN_CTAS
#define TMOL_B200_LKB_MIN_CTAS 2
#endif

template <typename Real, bool GRAD, typename Queue>
__device__ TMOL_B200_LKB_DRAIN_ATTR Lkb4<Real> lkb_drain(const LkbEval<Real> ev, const Queue& q, int n, int lane,
                                             const Lkb4<Real> w) {
  Lkb4<Real> out = {{0, 0, 0, 0}};
  if (lane >= n) return out;
  const int64_t rp = q.rp[lane], ro = q.ro[lane];
  const int pidx = q.pi[lane], oidx = q.oi[lane], sep = q.sep[lane];
  Real I[3], J[3], WI[LKB_NW * 3], WJ[LKB_NW * 3];
  lkb_load3(ev.coords, rp, I);
  lkb_load3(ev.coords, ro, J);
#pragma unroll
  for (int c = 0; c < LKB_NW * 3; ++c) {
    WI[c] = ev.waters[rp * LKB_NW * 3 + c];
    WJ[c] = ev.waters[ro * LKB_NW * 3 + c];
  }
  const LkbParams<Real> pp = lkb_params<Real>(ev, 0, 0, pidx);  // row bt * A + atom
  const LkbParams<Real> po = lkb_params<Real>(ev, 0, 0, oidx);
  Real gI[3] = {0, 0, 0}, gJ[3] = {0, 0, 0}, gWI[LKB_NW * 3], gWJ[LKB_NW * 3];
  if (GRAD)
#pragma unroll
    for (int c = 0; c < LKB_NW * 3; ++c) gWI[c] = gWJ[c] = 0;
  lkb_pair<Real, GRAD>(I, J, WI, WJ, sep, pp, po, ev, out.v, w.v, gI, gJ, gWI, gWJ);
  if (GRAD) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (gI[c] != Real(0)) atomicAdd(&ev.dcoords[3 * rp + c], gI[c]);
      if (gJ[c] != Real(0)) atomicAdd(&ev.dcoords[3 * ro + c], gJ[c]);
    }
#pragma unroll
    for (int c = 0; c < LKB_NW * 3; ++c) {
      if (gWI[c] != Real(0)) atomicAdd(&ev.dwaters[rp * LKB_NW * 3 + c], gWI[c]);
      if (gWJ[c] != Real(0)) atomicAdd(&ev.dwaters[ro * LKB_NW * 3 + c], gWJ[c]);
    }
  }
  return out;
}

// Per-warp queue state: the two queues (plain, bridged) in shared memory,
// their fill (warp-uniform) and the work counters.
template <typename Real, bool TAGGED>
struct LkbWarp {
  LkbQueue<TAGGED>* qs;
  int nq[2];
  int lane;
  unsigned lt_mask;
  unsigned long long n_bp, n_pairs, n_bridge, n_eval;
};

// Where tagged entries' energies go and their weights come from:
// out[t * n + tag] (rotamer op: energies [4, n_pairs], dTdV [4, n_pairs]).
template <typename Real>
struct LkbTagged {
  Real* energies;
  const Real* dTdV;
  int64_t n;
};

// Evaluates full queues (or, with `all`, everything queued) under the
// weights w, adding energies to e4, and shifts what is left to the front.
// TAGGED: each entry's weights and energies are those of its tag's row.
template <typename Real, bool GRAD, bool TAGGED>
__device__ __forceinline__ void lkb_pump(const LkbEval<Real>& ev, LkbWarp<Real, TAGGED>& q, bool all, const Lkb4<Real> w,
                                         Real* e4, const LkbTagged<Real> tg) {
  for (;;) {
    int which, n;
    if (q.nq[0] >= 32) {
      which = 0, n = 32;
    } else if (q.nq[1] >= 32) {
      which = 1, n = 32;
    } else if (all && q.nq[0] > 0) {
      which = 0, n = q.nq[0];
    } else if (all && q.nq[1] > 0) {
      which = 1, n = q.nq[1];
    } else {
      break;
    }
    LkbQueue<TAGGED>& Q = q.qs[which];
    const int lane = q.lane;
    __syncwarp();
    Lkb4<Real> wl = w;
    const int tag = TAGGED && lane < n ? Q.tag[lane] : 0;
    if (TAGGED && GRAD && lane < n)
      for (int c = 0; c < 4; ++c) wl.v[c] = tg.dTdV[(int64_t)c * tg.n + tag];
    const Lkb4<Real> got = lkb_drain<Real, GRAD>(ev, Q, n, lane, wl);
    if (TAGGED) {
      if (!GRAD && lane < n)
        for (int c = 0; c < 4; ++c)
          if (got.v[c] != Real(0)) atomicAdd(&tg.energies[(int64_t)c * tg.n + tag], got.v[c]);
    } else {
      for (int c = 0; c < 4; ++c) e4[c] += got.v[c];
    }
    const int rest = (which ? q.nq[1] : q.nq[0]) - n;
    int a = 0, b = 0, c = 0, d = 0, e = 0, f = 0;
    if (lane < rest) {
      a = Q.rp[n + lane], b = Q.ro[n + lane], c = Q.pi[n + lane], d = Q.oi[n + lane], e = Q.sep[n + lane];
      if (TAGGED) f = Q.tag[n + lane];
    }
    __syncwarp();
    if (lane < rest) {
      Q.rp[lane] = a, Q.ro[lane] = b, Q.pi[lane] = c, Q.oi[lane] = d, Q.sep[lane] = (uint8_t)e;
      if (TAGGED) Q.tag[lane] = f;
    }
    __syncwarp();
    if (which)
      q.nq[1] = rest;
    else
      q.nq[0] = rest;
  }
}

// One side of a pair of blocks (or rotamers): block type, first coordinate
// row, polar / occluder counts.
struct LkbSide {
  int bt, off, npol, nocc, nbr;
};

template <typename Real>
__device__ __forceinline__ LkbSide lkb_side(const LkbArgs<Real>& k, int bt, int off) {
  return LkbSide{bt, off, k.npol[bt], k.nocc[bt], k.nbocc[bt]};
}

// Every polar / occluder pair of sides 1 and 2 (intra: ordered pairs of
// distinct atoms of side 1; else both directions): filtered on bond
// separation (intra: the block type's path distances; inter: through the
// connections when `striking`), distance and the polar atom's waters, and
// queued; full queues are evaluated under w into e4.
template <typename Real, bool GRAD, bool TAGGED, bool COUNT = true>
__device__ __forceinline__ void lkb_enqueue_pairs(const ScoreArgs<Real>& s, const LkbArgs<Real>& k,
                                                  const LkbEval<Real>& ev, LkbWarp<Real, TAGGED>& q, const LkbSide& a,
                                                  const LkbSide& b, bool intra, bool striking, int nc1, int nc2,
                                                  const uint8_t* seps, const Lkb4<Real> w, Real* e4, int tag,
                                                  const LkbTagged<Real> tg) {
  const int lane = q.lane;
  const int no = intra ? a.nocc : b.nocc;
  const int n01 = a.npol * no;
  const int total = intra ? n01 : n01 + a.nocc * b.npol;
  // idx / no in float: exact for these sizes (idx < 2^16, no <= 256: the
  // error is far below 0.5 / no)
  const float inv_no = no > 0 ? 1.0f / float(no) : 0.0f;
  const float inv_nocc1 = a.nocc > 0 ? 1.0f / float(a.nocc) : 0.0f;
  if (COUNT) {
    q.n_bp += 1;
    q.n_pairs += total;
  }
  for (int base = 0; base < total; base += 32) {
    const int idx = base + lane;
    bool in_reach = false, bridged = false;
    int rp = 0, ro = 0, pidx = 0, oidx = 0, sep = 0;
    if (idx < total) {
      int ap, ao, btp, bto, offp, offo, y;
      if (idx < n01) {
        const int x = (int)((float(idx) + 0.5f) * inv_no);
        y = idx - x * no;
        btp = a.bt;
        bto = intra ? a.bt : b.bt;
        ap = k.pol[(int64_t)btp * k.maxpol + x];
        ao = k.occ[(int64_t)bto * k.maxocc + y];
        offp = a.off;
        offo = intra ? a.off : b.off;
        if (intra)
          sep = ap == ao ? 0 : s.bt_pd[((int64_t)a.bt * s.A + ap) * s.A + ao];
        else
          sep = striking ? lkb_inter_sep(s, a.bt, b.bt, nc1, nc2, seps, ap, ao) : 6;
        bridged = y < (intra ? a.nbr : b.nbr);
      } else {
        const int j = idx - n01;
        const int x = (int)((float(j) + 0.5f) * inv_nocc1);
        y = j - x * a.nocc;
        btp = b.bt;
        bto = a.bt;
        ap = k.pol[(int64_t)btp * k.maxpol + x];
        ao = k.occ[(int64_t)bto * k.maxocc + y];
        offp = b.off;
        offo = a.off;
        sep = striking ? lkb_inter_sep(s, a.bt, b.bt, nc1, nc2, seps, ao, ap) : 6;
        bridged = y < a.nbr;
      }
      if (sep > 3) {
        rp = offp + ap;
        ro = offo + ao;
        Real I[3], J[3];
        lkb_load3(s.coords, rp, I);
        lkb_load3(s.coords, ro, J);
        const Real dv[3] = {I[0] - J[0], I[1] - J[1], I[2] - J[2]};
        const Real dist = lkb_sqrt(lkb_dot(dv, dv));
        in_reach = dist < k.max_dis && !isnan(k.waters[(int64_t)rp * LKB_NW * 3]);
        pidx = btp * s.A + ap;
        oidx = bto * s.A + ao;
      }
    }
    const unsigned m1 = __ballot_sync(0xffffffffu, in_reach && bridged);
    const unsigned m0 = __ballot_sync(0xffffffffu, in_reach && !bridged);
    if (in_reach) {
      const int which = bridged ? 1 : 0;
      LkbQueue<TAGGED>& Q = q.qs[which];
      const int pos = (bridged ? q.nq[1] : q.nq[0]) + __popc((bridged ? m1 : m0) & q.lt_mask);
      Q.rp[pos] = rp;
      Q.ro[pos] = ro;
      Q.pi[pos] = pidx;
      Q.oi[pos] = oidx;
      Q.sep[pos] = (uint8_t)(sep > 255 ? 255 : sep);
      if (TAGGED) Q.tag[pos] = tag;
    }
    q.nq[0] += __popc(m0);
    q.nq[1] += __popc(m1);
    if (COUNT) {
      q.n_eval += __popc(m0 | m1);
      q.n_bridge += __popc(m1);
    }
    lkb_pump<Real, GRAD, TAGGED>(ev, q, false, w, e4, tg);
  }
}

// The count-pair data of block pair (row i1, block b2): whether any atom
// pair is within 4 bonds and, if so, the connection-to-connection
// separations.
template <typename Real>
__device__ __forceinline__ bool lkb_striking(const ScoreArgs<Real>& s, int64_t i1, int b2, int cp_b2, int cp_min,
                                             uint8_t* seps) {
  const unsigned pm = __ballot_sync(0xffffffffu, cp_b2 == b2);
  bool striking = false;
  if (pm) {
    const int src = __ffs(pm) - 1;
    striking = __shfl_sync(0xffffffffu, cp_min, src) <= 4;
    const int64_t e = i1 * CP_CAP + src;
    if (striking)
      for (int c = 0; c < 16; ++c) seps[c] = s.cp_seps[e * 16 + c];
  }
  return striking;
}

template <typename Real>
__device__ __forceinline__ LkbEval<Real> lkb_eval_of(const ScoreArgs<Real>& s, const LkbArgs<Real>& k) {
  LkbEval<Real> ev;
  ev.coords = s.coords;
  ev.waters = k.waters;
  ev.par = k.par;
  ev.dcoords = s.dcoords;
  ev.dwaters = k.dwaters_out;
  ev.A = s.A;
  ev.water_dist = k.water_dist;
  ev.hbond_dis = k.hbond_dis;
  ev.hbond_oh = k.hbond_oh;
  ev.hbond_h = k.hbond_h;
  ev.max_dis = k.max_dis;
  return ev;
}

template <typename Real, bool TAGGED>
__device__ __forceinline__ void lkb_flush_counts(const ScoreArgs<Real>& s, const LkbWarp<Real, TAGGED>& q) {
  if (s.counts && q.lane == 0) {
    if (q.n_bp) atomicAdd(&s.counts[0], q.n_bp);
    if (q.n_pairs) atomicAdd(&s.counts[1], q.n_pairs);
    if (q.n_bridge) atomicAdd(&s.counts[2], q.n_bridge);
    if (q.n_eval) atomicAdd(&s.counts[3], q.n_eval);
  }
}

// The pose op: the plan's work items (pose, b1, candidate blocks b2 >= b1),
// the neighbour rule as score_kernel applies it, then every polar /
// occluder pair of each neighbouring block pair.
// COUNT: the work counters (registers and instructions in the pair loop),
// compiled into a separate instantiation used on request
template <typename Real, bool GRAD, bool BLOCK_PAIR, bool COUNT>
__global__ void __launch_bounds__(256, TMOL_B200_LKB_MIN_CTAS) lkb_score_kernel(ScoreArgs<Real> s, LkbArgs<Real> k, int items_per_ticket) {
  if (s.done && *s.done) return;  // a speculative gradient was taken
  // [warp][plain, bridged]; block-pair mode tags queued pairs with their
  // block pair (p * B + b1) * B + b2
  __shared__ LkbQueue<BLOCK_PAIR> queues[LKB_MAX_WARPS][2];
  LkbWarp<Real, BLOCK_PAIR> q;
  q.lane = threadIdx.x & 31;
  q.qs = queues[threadIdx.x >> 5];
  q.lt_mask = (1u << q.lane) - 1u;
  q.nq[0] = q.nq[1] = 0;
  q.n_bp = q.n_pairs = q.n_bridge = q.n_eval = 0;
  const int lane = q.lane;
  const int64_t stride = (int64_t)s.P * s.B * s.B;
  const LkbEval<Real> ev = lkb_eval_of(s, k);
  LkbTagged<Real> tg;
  tg.energies = s.energies;
  tg.dTdV = s.dTdV;
  tg.n = stride;
  const Lkb4<Real> none = {{0, 0, 0, 0}};
  const int n_work = s.ticket[2];  // the plan's item count (a rebalance may split items)
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(s.ticket, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    const int it0 = t * items_per_ticket;
    if (it0 >= n_work) break;
    const int it1 = min(it0 + items_per_ticket, n_work);
    for (int item = it0; item < it1; ++item) {
      const long long t_item = COUNT ? clock64() : 0;  // item costs: the counting instantiation
      const int4 wi = s.work[item];
      const int p = wi.x, b1 = wi.y, cand0 = wi.z, cand1 = wi.w;
      const int i1 = p * s.B + b1;
      const int bt1 = s.blk_bt[i1];
      if (bt1 < 0) {
        if (s.item_cost && lane == 0) s.item_cost[item] = 0;
        continue;
      }
      const Real* sph1 = s.spheres + 4 * (int64_t)i1;
      const Real c1x = sph1[0], c1y = sph1[1], c1z = sph1[2], rad1 = sph1[3];
      unsigned my_mask = 0;
      const int n_batches = (cand1 - cand0 + 31) / 32;
      for (int bi = 0; bi < n_batches; ++bi) {
        const int b2 = cand0 + bi * 32 + lane;
        bool hit = false;
        if (b2 < cand1) {
          const int i2 = p * s.B + b2;
          if (s.blk_bt[i2] >= 0) {
            const Real* s2 = s.spheres + 4 * (int64_t)i2;
            const Real dx = sub_rn(c1x, s2[0]), dy = sub_rn(c1y, s2[1]), dz = sub_rn(c1z, s2[2]);
            const Real d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
            const Real thr = add_rn(add_rn(rad1, s2[3]), s.reach);
            hit = d2 < mul_rn(thr, thr);
          }
          if (s.nbr) s.nbr[(int64_t)i1 * s.B + b2] = hit ? 1 : 0;
        }
        const unsigned mk = __ballot_sync(0xffffffffu, hit);
        if (lane == bi) my_mask = mk;
      }
      // the row's count-pair partners, one per lane
      const int ncp = s.cp_count[i1];
      const int cp_b2 = lane < ncp ? s.cp_b2[i1 * CP_CAP + lane] : -1;
      const int cp_min = lane < ncp ? s.cp_minsep[i1 * CP_CAP + lane] : 6;
      Lkb4<Real> w = {{0, 0, 0, 0}};
      if (GRAD && !BLOCK_PAIR)
        for (int c = 0; c < 4; ++c) w.v[c] = s.dTdV[(int64_t)c * s.P + p];
      Real acc[4] = {0, 0, 0, 0};
      const LkbSide side1 = lkb_side(k, bt1, s.blk_off[i1]);
      for (int bi = 0; bi < n_batches; ++bi) {
        unsigned mask = __shfl_sync(0xffffffffu, my_mask, bi);
        while (mask) {
          const int kk = __ffs(mask) - 1;
          mask &= mask - 1;
          const int b2 = cand0 + bi * 32 + kk;
          const int i2 = p * s.B + b2;
          const bool intra = b2 == b1;
          uint8_t seps[16];
          const bool striking = !intra && lkb_striking(s, i1, b2, cp_b2, cp_min, seps);
          const LkbSide side2 = lkb_side(k, s.blk_bt[i2], s.blk_off[i2]);
          const int nc1 = striking ? s.bt_n_conn[bt1] : 0, nc2 = striking ? s.bt_n_conn[side2.bt] : 0;
          lkb_enqueue_pairs<Real, GRAD, BLOCK_PAIR, COUNT>(s, k, ev, q, side1, side2, intra, striking, nc1, nc2, seps,
                                                    BLOCK_PAIR ? none : w, acc,
                                                    BLOCK_PAIR ? (int)((int64_t)i1 * s.B + b2) : 0, tg);
        }
      }
      if (!BLOCK_PAIR) lkb_pump<Real, GRAD, BLOCK_PAIR>(ev, q, true, w, acc, tg);
      // whole-pose energies (also in the adjoint when asked for: one pass
      // for energy and gradient)
      if (!BLOCK_PAIR && s.energies)
        for (int c = 0; c < 4; ++c) {
          const Real v = warp_sum(acc[c]);
          if (lane == 0 && v != Real(0)) atomicAdd(&s.energies[(int64_t)c * s.P + p], v);
        }
      // the item's cost, for ordering the work longest-first
      if (COUNT && s.item_cost && lane == 0)
        s.item_cost[item] = (int)min((clock64() - t_item) >> 4, (long long)0x7fffffff);
    }
  }
  if (BLOCK_PAIR) {
    Real unused[4] = {0, 0, 0, 0};  // tagged entries add their energies to their rows
    lkb_pump<Real, GRAD, BLOCK_PAIR>(ev, q, true, none, unused, tg);
  }
  lkb_flush_counts(s, q);
}

// The rotamer op: work items (rot1, first rot2, n rot2, first pair) from
// the rotamer dispatch; every polar / occluder pair of rot1 against each
// rot2 (itself on the diagonal), energies per dispatched pair
// (energies[t * n_pairs + d], added by atomics), the adjoint under
// dTdV[t * n_pairs + d].  Queued pairs carry d, so the queues fill across
// rotamer pairs and items (a rotamer pair has few pairs in reach).
template <typename Real, bool GRAD, bool COUNT>
__global__ void __launch_bounds__(256, TMOL_B200_LKB_MIN_CTAS)
    lkb_rotamer_kernel(ScoreArgs<Real> s, LkbArgs<Real> k, RotArgs ra, const Real* rot_spheres) {
  __shared__ LkbQueue<true> queues[LKB_MAX_WARPS][2];
  LkbWarp<Real, true> q;
  q.lane = threadIdx.x & 31;
  q.qs = queues[threadIdx.x >> 5];
  q.lt_mask = (1u << q.lane) - 1u;
  q.nq[0] = q.nq[1] = 0;
  q.n_bp = q.n_pairs = q.n_bridge = q.n_eval = 0;
  const int lane = q.lane;
  const LkbEval<Real> ev = lkb_eval_of(s, k);
  LkbTagged<Real> tg;
  tg.energies = s.energies;
  tg.dTdV = s.dTdV;
  tg.n = ra.n_pairs;
  const Lkb4<Real> none = {{0, 0, 0, 0}};
  Real unused[4] = {0, 0, 0, 0};  // tagged entries add their energies to their rows
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(s.ticket, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= ra.n_items) break;
    const int4 item = ra.items[it];
    const int rot1 = item.x, rot2_first = item.y, n_rot2 = item.z;
    const long long pair_first = item.w;
    const int p = ra.rot_pose[rot1], b1 = ra.rot_block[rot1];
    const int64_t i1 = (int64_t)p * s.B + b1;
    const LkbSide side1 = lkb_side(k, ra.rot_bt[rot1], ra.rot_off[rot1]);
    const int ncp = s.cp_count[i1];
    const int cp_b2 = lane < ncp ? s.cp_b2[i1 * CP_CAP + lane] : -1;
    const int cp_min = lane < ncp ? s.cp_minsep[i1 * CP_CAP + lane] : 6;
    // b2 and its count-pair data are the same for every rot2 of the item
    const int b2 = n_rot2 > 0 ? ra.rot_block[rot2_first] : b1;
    uint8_t seps[16];
    const bool striking = b2 != b1 && lkb_striking(s, i1, b2, cp_b2, cp_min, seps);
    const Real* sp1 = rot_spheres + 4 * (int64_t)rot1;
    const Real c1x = sp1[0], c1y = sp1[1], c1z = sp1[2], r1 = sp1[3];
    for (int j = 0; j < n_rot2; ++j) {
      const int rot2 = rot2_first + j;
      const bool intra = rot2 == rot1;
      if (!intra) {
        // no atom pair of two rotamers whose bounding spheres are farther
        // apart than max_dis (with a margin far above rounding) is in
        // reach: their energies are zero
        const Real* sp2 = rot_spheres + 4 * (int64_t)rot2;
        const Real dx = c1x - sp2[0], dy = c1y - sp2[1], dz = c1z - sp2[2];
        const Real thr = r1 + sp2[3] + k.max_dis + Real(0.01);
        if (dx * dx + dy * dy + dz * dz > thr * thr) continue;
      }
      const LkbSide side2 = lkb_side(k, ra.rot_bt[rot2], ra.rot_off[rot2]);
      const int nc1 = striking ? s.bt_n_conn[side1.bt] : 0, nc2 = striking ? s.bt_n_conn[side2.bt] : 0;
      lkb_enqueue_pairs<Real, GRAD, true, COUNT>(s, k, ev, q, side1, side2, intra, striking, nc1, nc2, seps, none, unused,
                                          (int)(pair_first + j), tg);
    }
  }
  // entries carry their pair: the queues drain across items, once at the end
  lkb_pump<Real, GRAD, true>(ev, q, true, none, unused, tg);
  lkb_flush_counts(s, q);
}
