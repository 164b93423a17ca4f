// H-matrix generator: HACApK's construction rules restated in C++ for a point
// kernel.  See include/hacapk_hgen.h for the reference routines each part
// follows.  Everything here is host code; it produces the inputs that the HMVM
// library consumes (in memory, or as hmatrix_1.bin / hmatrix_2.bin files).

#include "hacapk_hgen.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Seeded point clouds (splitmix64 stream -> doubles in [0,1)).
struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

void make_points(int64_t n, int geometry, uint64_t seed, double* xyz) {
  SplitMix rng{seed * 0x2545F4914F6CDD1Dull + 0x1234567ull};
  for (int64_t i = 0; i < n; i++) {
    double* p = xyz + 3 * i;
    if (geometry == HGEN_SPHERE) {
      // Archimedes: z uniform in [-1,1], azimuth uniform -> uniform on the sphere.
      double z = 2.0 * rng.uniform() - 1.0;
      double phi = 2.0 * kPi * rng.uniform();
      double r = std::sqrt(std::max(0.0, 1.0 - z * z));
      p[0] = r * std::cos(phi);
      p[1] = r * std::sin(phi);
      p[2] = z;
    } else if (geometry == HGEN_CUBE_SURFACE) {
      // Six faces of equal area: pick a face, then a uniform point on it.
      int face = (int)(rng.uniform() * 6.0);
      if (face > 5) face = 5;
      double u = rng.uniform(), v = rng.uniform();
      int axis = face >> 1;
      double fixed = (face & 1) ? 1.0 : 0.0;
      p[axis] = fixed;
      p[(axis + 1) % 3] = u;
      p[(axis + 2) % 3] = v;
    } else {
      p[0] = 2.0 * rng.uniform();
      p[1] = rng.uniform();
      p[2] = 0.0;
    }
  }
}

// Kernel entry between original points i and j (0-based).
inline double kernel_entry(const double* xyz, int32_t i, int32_t j) {
  if (i == j) return 1.0;
  double dx = xyz[3 * i] - xyz[3 * j];
  double dy = xyz[3 * i + 1] - xyz[3 * j + 1];
  double dz = xyz[3 * i + 2] - xyz[3 * j + 2];
  return 1.0 / (4.0 * kPi * std::sqrt(dx * dx + dy * dy + dz * dz));
}

// ppohBEM's collocation kernel (face_integral, src_hdump/m_ppohBEM_user_func.f90:
// 49-100): the potential at (x, y, z) of a uniform unit charge density on the
// triangle (xs, ys, zs), from the closed-form edge terms.  The module's PI and
// EPSILON_0 are default-kind (single precision) Fortran literals promoted to
// double; they are reproduced as such.  Operation order follows the source.
inline void cross3(const double* u, const double* v, double* w) {
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}
double face_integral(const double* xs, const double* ys, const double* zs, double x, double y, double z) {
  const double pi_f = (double)3.141592653589793f;
  const double eps0 = (double)8.854187818f * 1e-12;
  double r[3];
  for (int k = 0; k < 3; k++)
    r[k] = std::sqrt((xs[k] - x) * (xs[k] - x) + (ys[k] - y) * (ys[k] - y) + (zs[k] - z) * (zs[k] - z));
  double u[3] = {xs[1] - xs[0], ys[1] - ys[0], zs[1] - zs[0]};
  double v[3] = {xs[2] - xs[1], ys[2] - ys[1], zs[2] - zs[1]};
  double w[3];
  cross3(u, v, w);
  const double wn = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  for (int k = 0; k < 3; k++) w[k] = w[k] / wn;
  u[0] = x - xs[0];
  u[1] = y - ys[0];
  u[2] = z - zs[0];
  const double zp = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
  const double ox = x - zp * w[0], oy = y - zp * w[1], oz = z - zp * w[2];
  const double zpabs = std::fabs(zp);
  double sum = 0.0;
  for (int i = 0; i < 3; i++) {
    const int j = (i + 1) % 3;
    u[0] = xs[j] - ox;
    u[1] = ys[j] - oy;
    u[2] = zs[j] - oz;
    const double xj = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    for (int k = 0; k < 3; k++) u[k] = u[k] / xj;
    cross3(w, u, v);
    const double xi = (xs[i] - ox) * u[0] + (ys[i] - oy) * u[1] + (zs[i] - oz) * u[2];
    const double yi = (xs[i] - ox) * v[0] + (ys[i] - oy) * v[1] + (zs[i] - oz) * v[2];
    const double dx = xj - xi, dy = -yi;  // yj = 0
    const double t = std::sqrt(dx * dx + dy * dy);
    const double l = dx / t, mm = dy / t;
    const double d = l * yi - mm * xi;
    const double ti = l * xi + mm * yi, tj = l * xj;
    const double theta = std::atan2(yi, xi);
    const double omega = theta - std::atan2(r[i] * d, zpabs * ti) + std::atan2(r[j] * d, zpabs * tj);
    const double q = std::log((r[j] + tj) / (r[i] + ti));
    const double g = d * q - zpabs * omega;
    sum = sum + g;
  }
  return std::fabs(sum) / (4.0 * pi_f * eps0);
}

// The matrix entry between original points (or faces) i and j, 0-based: the
// point kernel, or for a mesh ppohBEM_matrix_element_ij
// (src_hdump/m_ppohBEM_matrix_element_ij.f90): face j's integral at the
// centroid of face i.
struct Kernel {
  const double* xyz;
  const hgen_mesh* mesh;
  double operator()(int32_t i, int32_t j) const {
    if (!mesh) return kernel_entry(xyz, i, j);
    const int32_t* fi = mesh->face2node + (int64_t)i * mesh->nond_on_face;
    const int32_t* fj = mesh->face2node + (int64_t)j * mesh->nond_on_face;
    const double* np = mesh->nodes;
    const double xp = (np[3 * fi[0]] + np[3 * fi[1]] + np[3 * fi[2]]) / 3.0;
    const double yp = (np[3 * fi[0] + 1] + np[3 * fi[1] + 1] + np[3 * fi[2] + 1]) / 3.0;
    const double zp = (np[3 * fi[0] + 2] + np[3 * fi[1] + 2] + np[3 * fi[2] + 2]) / 3.0;
    const double xf[3] = {np[3 * fj[0]], np[3 * fj[1]], np[3 * fj[2]]};
    const double yf[3] = {np[3 * fj[0] + 1], np[3 * fj[1] + 1], np[3 * fj[2] + 1]};
    const double zf[3] = {np[3 * fj[0] + 2], np[3 * fj[1] + 2], np[3 * fj[2] + 2]};
    return face_integral(xf, yf, zf, xp, yp, zp);
  }
};

// ---------------------------------------------------------------------------
// Cluster tree (HACApK_generate_cbitree, m_HACApK_base.f90:994-1054) with
// bounding boxes (HACApK_bndbox, :953-991).
struct Cluster {
  int32_t nstrt;  // 1-based first position
  int32_t nsize;
  int32_t son[2] = {-1, -1};
  int32_t nson = 0;
  double bmin[3], bmax[3];
  double zwdth = 0.0;
};

struct Tree {
  std::vector<Cluster> c;
  const double* xyz;
  std::vector<int32_t> lod;  // 0-based point index at each 0-based position
  int minsz;

  // Bisection at the bounding-box midpoint of the longest axis, with HACApK's
  // in-place two-pointer partition (:1021-1027).  Recursion is iterative-safe
  // in depth because bisection depth is O(log n) for non-degenerate inputs;
  // degenerate (coincident) inputs peel one point per level.
  int32_t build(int32_t nsrt, int32_t nd) {
    int32_t id = (int32_t)c.size();
    c.emplace_back();
    c[id].nstrt = nsrt;
    c[id].nsize = nd;
    if (nd <= minsz) return id;
    int32_t* l = lod.data() + (nsrt - 1);  // l[0..nd-1]
    double zlmin[3], zlmax[3];
    for (int d = 0; d < 3; d++) {
      zlmin[d] = xyz[3 * l[0] + d];
      zlmax[d] = zlmin[d];
      for (int32_t il = 1; il < nd; il++) {
        double zg = xyz[3 * l[il] + d];
        if (zg < zlmin[d]) zlmin[d] = zg;
        else if (zlmax[d] < zg) zlmax[d] = zg;
      }
    }
    double zdiff = zlmax[0] - zlmin[0];
    int ncut = 0;
    for (int d = 0; d < 3; d++) {
      double zidiff = zlmax[d] - zlmin[d];
      if (zidiff > zdiff) { zdiff = zidiff; ncut = d; }
    }
    double zlmid = (zlmax[ncut] + zlmin[ncut]) / 2;
    // 1-based nl/nr as in the reference loop.
    int32_t nl = 1, nr = nd;
    auto g = [&](int32_t k) { return xyz[3 * l[k - 1] + ncut]; };
    while (nl < nr) {
      while (nl < nd && g(nl) <= zlmid) nl++;
      while (nr >= 1 && g(nr) > zlmid) nr--;
      if (nl < nr) std::swap(l[nl - 1], l[nr - 1]);
    }
    c[id].nson = 2;
    int32_t s0 = build(nsrt, nl - 1);
    int32_t s1 = build(nsrt + nl - 1, nd - nl + 1);
    c[id].son[0] = s0;
    c[id].son[1] = s1;
    return id;
  }

  void bndbox(int32_t id) {
    Cluster& k = c[id];
    if (k.nson == 0) {
      const int32_t* l = lod.data() + (k.nstrt - 1);
      for (int d = 0; d < 3; d++) {
        k.bmin[d] = k.nsize > 0 ? xyz[3 * l[0] + d] : 0.0;
        k.bmax[d] = k.bmin[d];
        for (int32_t il = 1; il < k.nsize; il++) {
          double v = xyz[3 * l[il] + d];
          if (v < k.bmin[d]) k.bmin[d] = v;
          if (k.bmax[d] < v) k.bmax[d] = v;
        }
      }
    } else {
      bndbox(k.son[0]);
      bndbox(k.son[1]);
      Cluster& kk = c[id];
      for (int d = 0; d < 3; d++) {
        kk.bmin[d] = c[kk.son[0]].bmin[d];
        kk.bmax[d] = c[kk.son[0]].bmax[d];
        if (c[kk.son[1]].bmin[d] < kk.bmin[d]) kk.bmin[d] = c[kk.son[1]].bmin[d];
        if (kk.bmax[d] < c[kk.son[1]].bmax[d]) kk.bmax[d] = c[kk.son[1]].bmax[d];
      }
    }
    Cluster& kk = c[id];
    double w = 0.0;
    for (int d = 0; d < 3; d++) w += (kk.bmax[d] - kk.bmin[d]) * (kk.bmax[d] - kk.bmin[d]);
    kk.zwdth = std::sqrt(w);
  }
};

struct Leaf {
  int32_t ltmtx, ndl, ndt, nstrtl, nstrtt, kt;
};

// Block tree (HACApK_generate_leafmtx, :845-891).
void block_tree(const Tree& t, int32_t cl, int32_t ct, int32_t nleaf, int64_t nlmax, double eta,
                std::vector<Leaf>& out) {
  const Cluster& L = t.c[cl];
  const Cluster& T = t.c[ct];
  int32_t ndl = L.nsize, ndt = T.nsize;
  double zs = 0.0;
  for (int d = 0; d < 3; d++) {
    if (L.bmax[d] < T.bmin[d]) zs += (T.bmin[d] - L.bmax[d]) * (T.bmin[d] - L.bmax[d]);
    else if (T.bmax[d] < L.bmin[d]) zs += (L.bmin[d] - T.bmax[d]) * (L.bmin[d] - T.bmax[d]);
  }
  double zdistlt = std::sqrt(zs);
  if ((L.zwdth <= eta * zdistlt || T.zwdth <= eta * zdistlt) &&
      (ndl >= nleaf && ndt >= nleaf && ndl <= nlmax && ndt <= nlmax)) {
    out.push_back(Leaf{1, ndl, ndt, L.nstrt, T.nstrt, 0});
  } else if (L.nson == 0 || T.nson == 0 || ndl <= nleaf || ndt <= nleaf) {
    out.push_back(Leaf{2, ndl, ndt, L.nstrt, T.nstrt, 0});
  } else {
    for (int il = 0; il < L.nson; il++)
      for (int it = 0; it < T.nson; it++) block_tree(t, L.son[il], T.son[it], nleaf, nlmax, eta, out);
  }
}

// HACApK_med3 (src_hdump/HACApK_lib.f90:156-162).
inline int32_t med3(int32_t nl, int32_t nr, int32_t nlr2) {
  if (nl < nr) {
    if (nr < nlr2) return nr;
    if (nlr2 < nl) return nl;
    return nlr2;
  }
  if (nlr2 < nr) return nr;
  if (nl < nlr2) return nl;
  return nlr2;
}

// HACApK_qsort_row_leafmtx / HACApK_qsort_col_leafmtx (:893-935): Hoare
// partition around a median-of-three key; 1-based inclusive bounds.
template <class Key>
void hqsort(std::vector<Leaf>& a, int32_t s, int32_t e, Key key) {
  if (s >= e) return;
  int32_t nl = s, nr = e, nlr2 = nl + (nr - nl) / 2;
  int32_t nmid = med3(key(a[nl - 1]), key(a[nr - 1]), key(a[nlr2 - 1]));
  for (;;) {
    while (key(a[nl - 1]) < nmid) nl++;
    while (key(a[nr - 1]) > nmid) nr--;
    if (nl >= nr) break;
    std::swap(a[nl - 1], a[nr - 1]);
    nl++;
    nr--;
  }
  hqsort(a, s, nl - 1, key);
  hqsort(a, nr + 1, e, key);
}

// HACApK_unrm_d (src_hdump/HACApK_lib.f90:31-46): scaled 2-norm skipping |v|<1e-30.
double unrm(const double* za, int32_t n) {
  double zscl = 0.0, zzz = 1.0;
  for (int32_t i = 0; i < n; i++) {
    double zza = std::fabs(za[i]);
    if (zza < 1.0e-30) continue;
    if (zscl < zza) {
      zzz = 1.0 + zzz * (zscl / zza) * (zscl / zza);
      zscl = zza;
    } else {
      zzz = zzz + (zza / zscl) * (zza / zscl);
    }
  }
  return zscl * std::sqrt(zzz);
}

// HACApK_maxabsvallocm_d (HACApK_lib.f90:59-70): 1-based argmax |v| over
// unmasked entries, 0 if none exceeds 0.
int32_t maxabs_masked(const double* za, int32_t n, const std::vector<uint8_t>& msk, double* zz) {
  int32_t il = 0;
  *zz = 0.0;
  for (int32_t it = 0; it < n; it++) {
    if (msk[it]) continue;
    if (std::fabs(za[it]) > *zz) {
      il = it + 1;
      *zz = std::fabs(za[it]);
    }
  }
  return il;
}

struct AcaOut {
  int32_t kt = 0;
  bool incomplete = false;
  std::vector<double> V;  // ndt x kt, column-major (zab)
  std::vector<double> U;  // ndl x kt, column-major (zaa)
};

// Partially pivoted ACA (HACApK_aca, m_HACApK_base.f90:494-577) with
// param(61)=1 (the k=1 term's norm is the block norm), param(64)=1.
void aca(const Kernel& K, const int32_t* lod, const Leaf& lf, int32_t kmax, double eps, double aca_eps,
         AcaOut& o) {
  const int32_t ndl = lf.ndl, ndt = lf.ndt, nstrtl = lf.nstrtl, nstrtt = lf.nstrtt;
  const int32_t krank = std::min(ndl, ndt);
  const int32_t kstop = std::min(kmax, krank);
  std::vector<uint8_t> rmsk(ndl, 0), cmsk(ndt, 0);
  std::vector<double>& U = o.U;
  std::vector<double>& V = o.V;
  U.clear();
  V.clear();
  int32_t ist = (nstrtl > nstrtt) ? 1 : ndl;
  int32_t k = 1;
  double znrm = 0.0, zeps = 0.0;
  std::vector<double> zau;
  // Entry of the permuted matrix at 1-based positions (lod holds 1-based point ids).
  auto ent = [&](int32_t ill, int32_t itt) { return K(lod[ill - 1] - 1, lod[itt - 1] - 1); };
  for (;;) {
    V.resize((size_t)ndt * k);
    U.resize((size_t)ndl * k);
    double* prow = V.data() + (size_t)ndt * (k - 1);
    double* pcol = U.data() + (size_t)ndl * (k - 1);
    // HACApK_calc_vec row direction (:467-488, ld=0): fresh entries of row ist
    // on unmasked columns, minus sum_j V(:,j)*U(ist,j), masked entries -> 0.
    for (int32_t ii = 0; ii < ndt; ii++)
      if (!cmsk[ii]) prow[ii] = ent(ist + nstrtl - 1, ii + nstrtt);
    if (k > 1) {
      zau.assign(ndt, 0.0);
      for (int32_t j = 0; j < k - 1; j++) {
        double zu = U[(size_t)ndl * j + (ist - 1)];
        const double* col = V.data() + (size_t)ndt * j;
        for (int32_t ii = 0; ii < ndt; ii++) zau[ii] = zau[ii] + col[ii] * zu;
      }
      for (int32_t ii = 0; ii < ndt; ii++) prow[ii] = prow[ii] - zau[ii];
      for (int32_t ii = 0; ii < ndt; ii++)
        if (cmsk[ii]) prow[ii] = 0.0;
    }
    double row_maxval;
    int32_t jst = maxabs_masked(prow, ndt, cmsk, &row_maxval);
    if (jst == 0) {
      // The residual row is exactly zero (HACApK would divide by it): the block
      // is already represented; keep k-1 terms (one zero term if k == 1).
      if (k == 1) {
        std::fill(prow, prow + ndt, 0.0);
        std::fill(pcol, pcol + ndl, 0.0);
      } else {
        k--;
        V.resize((size_t)ndt * k);
        U.resize((size_t)ndl * k);
      }
      zeps = 0.0;
      break;
    }
    double zdltinv = 1.0 / prow[jst - 1];
    for (int32_t ii = 0; ii < ndt; ii++) prow[ii] = prow[ii] * zdltinv;
    // Column direction (ld=1).
    for (int32_t ii = 0; ii < ndl; ii++)
      if (!rmsk[ii]) pcol[ii] = ent(ii + nstrtl, jst + nstrtt - 1);
    if (k > 1) {
      zau.assign(ndl, 0.0);
      for (int32_t j = 0; j < k - 1; j++) {
        double zu = V[(size_t)ndt * j + (jst - 1)];
        const double* col = U.data() + (size_t)ndl * j;
        for (int32_t ii = 0; ii < ndl; ii++) zau[ii] = zau[ii] + col[ii] * zu;
      }
      for (int32_t ii = 0; ii < ndl; ii++) pcol[ii] = pcol[ii] - zau[ii];
      for (int32_t ii = 0; ii < ndl; ii++)
        if (rmsk[ii]) pcol[ii] = 0.0;
    }
    rmsk[ist - 1] = 1;
    double col_maxval;
    int32_t istn = maxabs_masked(pcol, ndl, rmsk, &col_maxval);
    cmsk[jst - 1] = 1;
    ist = istn > 0 ? istn : ist;
    if (std::fabs(row_maxval) < aca_eps && std::fabs(col_maxval) < aca_eps && k >= 1) break;
    zeps = unrm(pcol, ndl) * unrm(prow, ndt);
    if (k == 1) znrm = zeps;
    zeps = znrm > 0.0 ? zeps / znrm : 0.0;
    bool lstop = (zeps < eps || k == kstop);
    if (lstop && k >= 1) break;
    if (istn == 0) break;  // every row pivoted: nothing left to approximate
    k++;
  }
  o.kt = k;
  o.incomplete = (zeps > eps && k < krank);
}

}  // namespace

extern "C" {

void hgen_default_params(hgen_params* p) {
  p->n = 8192;
  p->geometry = HGEN_SPHERE;
  p->leaf_size = 32;
  p->eta = 2.0;
  p->eps = 1.0e-4;
  p->aca_eps_factor = 1.0e-3;
  p->kmax = 1000;
  p->nthreads = 0;
  p->seed = 1;
}

void hgen_free(hgen_hmatrix* m) {
  if (!m) return;
  free(m->ltmtx); free(m->kt); free(m->ndl); free(m->ndt); free(m->nstrtl); free(m->nstrtt);
  free(m->a1); free(m->a2); free(m->rowmat); free(m->lod); free(m->coords);
  free(m);
}

// Cluster tree, block tree and leaf order over m->coords (m->nd points);
// frees m on failure.
static int build_tree_points(const hgen_params* p, hgen_hmatrix* m, hgen_hmatrix** out) {
  const int32_t n = m->nd;
  std::vector<Leaf> leaves;
  try {
    Tree t;
    t.xyz = m->coords;
    t.minsz = p->leaf_size;
    t.lod.resize(n);
    for (int32_t i = 0; i < n; i++) t.lod[i] = i;
    t.c.reserve((size_t)4 * (n / std::max(1, p->leaf_size / 2) + 1));
    t.build(1, n);
    t.bndbox(0);
    for (int32_t i = 0; i < n; i++) m->lod[i] = t.lod[i] + 1;
    block_tree(t, 0, 0, p->leaf_size + 1, (int64_t)n, p->eta, leaves);
  } catch (const std::bad_alloc&) {
    hgen_free(m);
    return HGEN_ENOMEM;
  }
  int32_t nlf = (int32_t)leaves.size();
  // Row sort, then a column sort inside every row group except the last one
  // (the reference loop only sorts a group when the next one starts,
  // m_HACApK_base.f90:247-255).
  hqsort(leaves, 1, nlf, [](const Leaf& a) { return a.nstrtl; });
  {
    int32_t ilp = 1, ips = 1;
    for (int32_t ip = 1; ip <= nlf; ip++) {
      int32_t il = leaves[ip - 1].nstrtl;
      if (il > ilp) {
        hqsort(leaves, ips, ip - 1, [](const Leaf& a) { return a.nstrtt; });
        ilp = il;
        ips = ip;
      }
    }
  }

  // Structural arrays in file order; no leaf data yet.
  m->nlf = nlf;
  size_t nb = (size_t)(nlf > 0 ? nlf : 1);
  m->ltmtx = (int32_t*)malloc(nb * 4); m->kt = (int32_t*)calloc(nb, 4);
  m->ndl = (int32_t*)malloc(nb * 4); m->ndt = (int32_t*)malloc(nb * 4);
  m->nstrtl = (int32_t*)malloc(nb * 4); m->nstrtt = (int32_t*)malloc(nb * 4);
  m->a1 = (int64_t*)calloc(nb, 8); m->a2 = (int64_t*)calloc(nb, 8);
  if (!m->ltmtx || !m->kt || !m->ndl || !m->ndt || !m->nstrtl || !m->nstrtt || !m->a1 || !m->a2) {
    hgen_free(m);
    return HGEN_ENOMEM;
  }
  for (int32_t i = 0; i < nlf; i++) {
    const Leaf& lf = leaves[i];
    m->ltmtx[i] = lf.ltmtx; m->ndl[i] = lf.ndl; m->ndt[i] = lf.ndt;
    m->nstrtl[i] = lf.nstrtl; m->nstrtt[i] = lf.nstrtt;
    if (lf.ltmtx == 1) m->n_lowrank++;
    else m->n_dense++;
  }
  *out = m;
  return HGEN_OK;
}

static bool tree_params_ok(const hgen_params* p) {
  return p && p->leaf_size >= 1 && p->eta >= 0.0 && p->eps > 0.0 && p->kmax >= 1;
}

int hgen_build_tree(const hgen_params* p, hgen_hmatrix** out) {
  if (!out) return HGEN_EINVAL;
  *out = nullptr;
  if (!tree_params_ok(p) || p->n < 1 || p->n > INT32_MAX || p->geometry < 0 || p->geometry > 2)
    return HGEN_EINVAL;
#ifdef _OPENMP
  if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
  const int32_t n = (int32_t)p->n;
  hgen_hmatrix* m = (hgen_hmatrix*)calloc(1, sizeof(hgen_hmatrix));
  if (!m) return HGEN_ENOMEM;
  m->nd = n;
  m->coords = (double*)malloc(sizeof(double) * 3 * (size_t)n);
  m->lod = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  if (!m->coords || !m->lod) { hgen_free(m); return HGEN_ENOMEM; }
  make_points(n, p->geometry, p->seed, m->coords);
  return build_tree_points(p, m, out);
}

int hgen_build_tree_mesh(const hgen_params* p, const hgen_mesh* mesh, hgen_hmatrix** out) {
  if (!out) return HGEN_EINVAL;
  *out = nullptr;
  if (!tree_params_ok(p) || !mesh || mesh->nofc < 1 || mesh->nond_on_face != 3 || !mesh->nodes ||
      !mesh->face2node)
    return HGEN_EINVAL;
  for (int64_t k = 0; k < (int64_t)mesh->nofc * 3; k++)
    if (mesh->face2node[k] < 0 || mesh->face2node[k] >= mesh->nond) return HGEN_EINVAL;
#ifdef _OPENMP
  if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
  const int32_t n = mesh->nofc;
  hgen_hmatrix* m = (hgen_hmatrix*)calloc(1, sizeof(hgen_hmatrix));
  if (!m) return HGEN_ENOMEM;
  m->nd = n;
  m->mesh = mesh;
  m->coords = (double*)malloc(sizeof(double) * 3 * (size_t)n);
  m->lod = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  if (!m->coords || !m->lod) { hgen_free(m); return HGEN_ENOMEM; }
  // cluster points: face centroids (m_ppohBEM_bembb2hacapk.f90, "center of balance")
  const double* np = mesh->nodes;
  for (int32_t f = 0; f < n; f++) {
    const int32_t* fn = mesh->face2node + 3 * (int64_t)f;
    for (int d = 0; d < 3; d++) m->coords[3 * f + d] = (np[3 * fn[0] + d] + np[3 * fn[1] + d] + np[3 * fn[2] + d]) / 3.0;
  }
  return build_tree_points(p, m, out);
}

int hgen_fill_leaves(hgen_hmatrix* m, const hgen_params* p) {
  if (!m || !p || m->rowmat || !(p->eps > 0.0) || p->kmax < 1) return HGEN_EINVAL;
#ifdef _OPENMP
  if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
  const int32_t nlf = m->nlf;
  std::vector<Leaf> leaves((size_t)nlf);
  for (int32_t i = 0; i < nlf; i++)
    leaves[i] = Leaf{m->ltmtx[i], m->ndl[i], m->ndt[i], m->nstrtl[i], m->nstrtt[i], 0};
  // ACA for every low-rank leaf (independent per leaf; results do not depend on
  // the thread count).
  std::vector<AcaOut> fac(nlf);
  std::vector<int32_t> order;
  for (int32_t i = 0; i < nlf; i++)
    if (leaves[i].ltmtx == 1) order.push_back(i);
  std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    int64_t ca = (int64_t)leaves[a].ndl + leaves[a].ndt, cb = (int64_t)leaves[b].ndl + leaves[b].ndt;
    return ca != cb ? ca > cb : a < b;
  });
  const double aca_eps = p->aca_eps_factor * p->eps;
  int64_t incomplete = 0;
  bool oom = false;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : incomplete)
  for (size_t oi = 0; oi < order.size(); oi++) {
    int32_t i = order[oi];
    try {
      aca(Kernel{m->coords, m->mesh}, m->lod, leaves[i], p->kmax, p->eps, aca_eps, fac[i]);
    } catch (const std::bad_alloc&) {
#pragma omp critical
      oom = true;
    }
    leaves[i].kt = fac[i].kt;
    if (fac[i].incomplete) incomplete++;
  }
  if (oom) return HGEN_ENOMEM;

  // Offsets in file order, then the single packed array.
  int64_t off = 0;
  int32_t ktmax = 0;
  for (int32_t i = 0; i < nlf; i++) {
    const Leaf& lf = leaves[i];
    m->kt[i] = lf.kt;
    if (lf.ltmtx == 1) {
      m->a1[i] = off;
      off += (int64_t)lf.kt * lf.ndt;
      m->a2[i] = off;
      off += (int64_t)lf.kt * lf.ndl;
      if (lf.kt > ktmax) ktmax = lf.kt;
    } else {
      m->a1[i] = off;
      m->a2[i] = 0;
      off += (int64_t)lf.ndl * lf.ndt;
    }
  }
  m->len = off;
  m->ktmax = ktmax;
  m->aca_incomplete = incomplete;
  m->rowmat = (double*)malloc(sizeof(double) * (size_t)(off > 0 ? off : 1));
  if (!m->rowmat) return HGEN_ENOMEM;
  const Kernel K{m->coords, m->mesh};
#pragma omp parallel for schedule(dynamic, 16)
  for (int32_t i = 0; i < nlf; i++) {
    const Leaf& lf = leaves[i];
    if (lf.ltmtx == 1) {
      // a1 = zab(ndt,kt), a2 = zaa(ndl,kt), both column-major (:625-626).
      std::memcpy(m->rowmat + m->a1[i], fac[i].V.data(), sizeof(double) * (size_t)lf.kt * lf.ndt);
      std::memcpy(m->rowmat + m->a2[i], fac[i].U.data(), sizeof(double) * (size_t)lf.kt * lf.ndl);
      std::vector<double>().swap(fac[i].V);
      std::vector<double>().swap(fac[i].U);
    } else {
      // a1(ndt,ndl): a1(it,il) = K(row il, col it) (:637-649).
      double* a = m->rowmat + m->a1[i];
      for (int32_t il = 0; il < lf.ndl; il++) {
        int32_t pi = m->lod[il + lf.nstrtl - 1] - 1;
        for (int32_t it = 0; it < lf.ndt; it++)
          a[it + (int64_t)il * lf.ndt] = K(pi, m->lod[it + lf.nstrtt - 1] - 1);
      }
    }
  }
  return HGEN_OK;
}

int hgen_build(const hgen_params* p, hgen_hmatrix** out) {
  if (!out) return HGEN_EINVAL;
  *out = nullptr;
  hgen_hmatrix* m = nullptr;
  int rc = hgen_build_tree(p, &m);
  if (rc) return rc;
  rc = hgen_fill_leaves(m, p);
  if (rc) {
    hgen_free(m);
    return rc;
  }
  *out = m;
  return HGEN_OK;
}

// ---- .pbf meshes --------------------------------------------------------------
namespace {
// Whitespace-separated tokens of a list-directed Fortran text file (numbers
// may use d / D exponents).
struct Tokens {
  FILE* f;
  bool next(char* buf, size_t cap) {
    int c;
    do c = fgetc(f);
    while (c != EOF && (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == ','));
    if (c == EOF) return false;
    size_t n = 0;
    while (c != EOF && c != ' ' && c != '\t' && c != '\n' && c != '\r' && c != ',') {
      if (n + 1 < cap) buf[n++] = (c == 'd' || c == 'D') ? 'e' : (char)c;
      c = fgetc(f);
    }
    buf[n] = 0;
    return true;
  }
  bool real(double* v) {
    char b[128], *end;
    if (!next(b, sizeof b)) return false;
    *v = std::strtod(b, &end);
    return end != b && *end == 0;
  }
  bool integer(int32_t* v) {
    char b[64], *end;
    if (!next(b, sizeof b)) return false;
    const long x = std::strtol(b, &end, 10);
    if (end == b || *end != 0 || x < INT32_MIN || x > INT32_MAX) return false;
    *v = (int32_t)x;
    return true;
  }
};
}  // namespace

void hgen_free_mesh(hgen_mesh* mesh) {
  if (!mesh) return;
  free(mesh->nodes);
  free(mesh->face2node);
  free(mesh->int_para_fc);
  free(mesh->dble_para_fc);
  free(mesh);
}

int hgen_read_pbf(const char* fname, hgen_mesh** out) {
  if (!fname || !out) return HGEN_EINVAL;
  *out = nullptr;
  FILE* f = fopen(fname, "r");
  if (!f) return HGEN_EIO;
  Tokens T{f};
  hgen_mesh* m = (hgen_mesh*)calloc(1, sizeof(hgen_mesh));
  int rc = m ? HGEN_OK : HGEN_ENOMEM;
  auto bad = [&]() { rc = HGEN_EIO; };
  if (!rc && (!T.integer(&m->nond) || m->nond < 1)) bad();
  if (!rc && !(m->nodes = (double*)malloc(sizeof(double) * 3 * (size_t)m->nond))) rc = HGEN_ENOMEM;
  for (int64_t k = 0; !rc && k < 3 * (int64_t)m->nond; k++)
    if (!T.real(&m->nodes[k])) bad();
  if (!rc && (!T.integer(&m->nofc) || m->nofc < 1 || !T.integer(&m->nond_on_face) || m->nond_on_face < 1 ||
              !T.integer(&m->nint_para_fc) || m->nint_para_fc < 0 || !T.integer(&m->ndble_para_fc) ||
              m->ndble_para_fc < 0))
    bad();
  const int64_t nfn = rc ? 0 : (int64_t)m->nofc * m->nond_on_face;
  if (!rc && !(m->face2node = (int32_t*)malloc(sizeof(int32_t) * (size_t)nfn))) rc = HGEN_ENOMEM;
  for (int64_t k = 0; !rc && k < nfn; k++)
    if (!T.integer(&m->face2node[k]) || m->face2node[k] < 0 || m->face2node[k] >= m->nond) bad();
  const int64_t ni = rc ? 0 : (int64_t)m->nofc * m->nint_para_fc;
  if (!rc && ni && !(m->int_para_fc = (int32_t*)malloc(sizeof(int32_t) * (size_t)ni))) rc = HGEN_ENOMEM;
  for (int64_t k = 0; !rc && k < ni; k++)
    if (!T.integer(&m->int_para_fc[k])) bad();
  const int64_t nr = rc ? 0 : (int64_t)m->nofc * m->ndble_para_fc;
  if (!rc && nr && !(m->dble_para_fc = (double*)malloc(sizeof(double) * (size_t)nr))) rc = HGEN_ENOMEM;
  for (int64_t k = 0; !rc && k < nr; k++)
    if (!T.real(&m->dble_para_fc[k])) bad();
  fclose(f);
  if (rc) {
    hgen_free_mesh(m);
    return rc;
  }
  *out = m;
  return HGEN_OK;
}

double hgen_entry(const hgen_hmatrix* m, int32_t ill, int32_t itt) {
  return Kernel{m->coords, m->mesh}(m->lod[ill - 1] - 1, m->lod[itt - 1] - 1);
}

// Fortran unformatted sequential records: int32 byte count, payload, byte count.
static int put_record(FILE* f, const void* p, int64_t nbytes) {
  if (nbytes > INT32_MAX) return HGEN_ERANGE;
  int32_t mk = (int32_t)nbytes;
  if (fwrite(&mk, 4, 1, f) != 1) return HGEN_EIO;
  if (nbytes && fwrite(p, 1, (size_t)nbytes, f) != (size_t)nbytes) return HGEN_EIO;
  if (fwrite(&mk, 4, 1, f) != 1) return HGEN_EIO;
  return HGEN_OK;
}

static int write_leaf_data(FILE* f, const hgen_hmatrix* m, int32_t i) {
  int rc;
  if (m->ltmtx[i] == 1) {
    if ((rc = put_record(f, m->rowmat + m->a1[i], 8 * (int64_t)m->kt[i] * m->ndt[i]))) return rc;
    return put_record(f, m->rowmat + m->a2[i], 8 * (int64_t)m->kt[i] * m->ndl[i]);
  }
  if (m->ltmtx[i] == 2) return put_record(f, m->rowmat + m->a1[i], 8 * (int64_t)m->ndl[i] * m->ndt[i]);
  return HGEN_OK;
}

int hgen_write_bin1(const hgen_hmatrix* m, const char* fname) {
  FILE* f = fopen(fname, "wb");
  if (!f) return HGEN_EIO;
  int32_t hdr[3] = {m->nd, m->nlf, m->ktmax};
  int rc = put_record(f, hdr, sizeof hdr);
  for (int32_t i = 0; rc == HGEN_OK && i < m->nlf; i++) {
    int32_t h6[6] = {m->ltmtx[i], m->ndl[i], m->ndt[i], m->nstrtl[i], m->nstrtt[i], m->kt[i]};
    rc = put_record(f, h6, sizeof h6);
    if (rc == HGEN_OK) rc = write_leaf_data(f, m, i);
  }
  if (fclose(f) != 0 && rc == HGEN_OK) rc = HGEN_EIO;
  return rc;
}

// bin2 and its 64-bit variant differ only in the width of the header's len.
static int write_bin2_like(const hgen_hmatrix* m, const char* fname, bool len64) {
  FILE* f = fopen(fname, "wb");
  if (!f) return HGEN_EIO;
  unsigned char hdr[20];
  const int32_t h3[3] = {m->nd, m->nlf, m->ktmax};
  std::memcpy(hdr, h3, 12);
  if (len64) {
    const int64_t len = m->len;
    std::memcpy(hdr + 12, &len, 8);
  } else {
    const int32_t len32 = m->len > INT32_MAX ? INT32_MAX : (int32_t)m->len;
    std::memcpy(hdr + 12, &len32, 4);
  }
  int rc = put_record(f, hdr, len64 ? 20 : 16);
  const int32_t* cols[6] = {m->ltmtx, m->ndl, m->ndt, m->nstrtl, m->nstrtt, m->kt};
  for (int c = 0; rc == HGEN_OK && c < 6; c++) rc = put_record(f, cols[c], 4 * (int64_t)m->nlf);
  for (int32_t i = 0; rc == HGEN_OK && i < m->nlf; i++) rc = write_leaf_data(f, m, i);
  if (fclose(f) != 0 && rc == HGEN_OK) rc = HGEN_EIO;
  return rc;
}

int hgen_write_bin2(const hgen_hmatrix* m, const char* fname) { return write_bin2_like(m, fname, false); }
int hgen_write_bin64(const hgen_hmatrix* m, const char* fname) { return write_bin2_like(m, fname, true); }

}  // extern "C"
