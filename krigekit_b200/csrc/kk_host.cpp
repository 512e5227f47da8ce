// kk_host.cpp -- host-side preparation for the kriging solve path:
// rotation matrices, variogram lookup tables and the kd-tree used by the
// device tie fallback.  Arithmetic follows the reference build exactly
// (gfortran -O2, IEEE double, no fused multiply-add): this file is compiled
// with -ffp-contract=off.
#include <cmath>
#include <cstring>
#include <functional>

#include "kk_host.h"

namespace kk {

static double kpi() { return 4.0 * std::atan(1.0); }  // common.f90:7

// corefunc_fn, vgmfunc.f90:28-67
static double corefunc(int vtype, double r) {
  const double pi = kpi();
  switch (vtype) {
    case KK_NUG: return 0.0;
    case KK_SPH: return (r < 1.0) ? 1.0 - 1.5 * r + 0.5 * (r * r * r) : 0.0;
    case KK_EXP: return std::exp(-3.0 * r);
    case KK_GAU: return std::exp(-3.0625 * (r * r));
    case KK_HOL: return std::cos(pi * r);
    case KK_POW: return (r < 1.0) ? 1.0 - std::pow(r, 1.5) : 0.0;
    case KK_BSQ: { double t = 1.0 - r * r; return (r < 1.0) ? t * t : 0.0; }
    case KK_CIR:
      return (r < 1.0) ? 1.0 - (2.0 * r * std::sqrt(1.0 - r * r) + 2.0 * std::asin(r)) / pi : 0.0;
    case KK_LIN: return (r < 1.0) ? 1.0 - r : 0.0;
    case KK_CYC: { double s = std::sin(pi * r); return std::exp(-2.0 * (s * s)); }
    case KK_DCO: return std::exp(-3.0 * r) * std::cos(pi * r);
    default: return 0.0;
  }
}

// corefunc_has_analytic_tail, vgmfunc.f90:71-80
static int has_tail(int v) {
  return v == KK_EXP || v == KK_GAU || v == KK_HOL || v == KK_CYC || v == KK_DCO;
}

static void mat3_mul(const double* a, const double* b, double* c) {
  double t[9];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + a[i + 3 * k] * b[k + 3 * j];
      t[i + 3 * j] = s;
    }
  std::memcpy(c, t, sizeof t);
}

// calc_rotmat, rotation.f90:51-95 (column-major)
void calc_rotmat(double ang1, double ang2, double ang3, double anis1, double anis2, double* m) {
  const double deg2rad = kpi() / 180.0;
  const double eps = 1.0e-10;
  for (int i = 0; i < 9; ++i) m[i] = 0.0;
  m[0] = 1.0 / anis1;
  m[4] = 1.0;
  m[8] = 1.0 / anis2;
  if (std::fabs(ang3) > eps) {
    double al = -ang3 * deg2rad, sa = std::sin(al), ca = std::cos(al);
    double t[9] = {ca, 0.0, sa, 0.0, 1.0, 0.0, -sa, 0.0, ca};
    mat3_mul(m, t, m);
  }
  if (std::fabs(ang2) > eps) {
    double al = -ang2 * deg2rad, sa = std::sin(al), ca = std::cos(al);
    double t[9] = {1.0, 0.0, 0.0, 0.0, ca, sa, 0.0, -sa, ca};
    mat3_mul(m, t, m);
  }
  if (std::fabs(ang1) > eps) {
    double al = ang1 * deg2rad, sa = std::sin(al), ca = std::cos(al);
    double t[9] = {ca, sa, 0.0, -sa, ca, 0.0, 0.0, 0.0, 1.0};
    mat3_mul(m, t, m);
  }
}

// zone layout, alloc_zones (variogram.f90:223-256) with the fixed bounds of
// kriging.F90:416-417
static const double HB[KK_TAB_NZ + 1] = {0.0, 0.1, 0.5, 3.5};
static const double DH[KK_TAB_NZ] = {1e-5, 1e-4, 1e-3};

static void zones(int* zn, int* off, double* inv_dh) {
  int o = 0;
  for (int k = 0; k < KK_TAB_NZ; ++k) {
    int n = (int)std::lround((HB[k + 1] - HB[k]) / DH[k]);
    if (n < 1) n = 1;
    zn[k] = n;
    off[k] = o;
    inv_dh[k] = (double)n / (HB[k + 1] - HB[k]);
    o += n;
  }
}

// Append a table tab[0..N] as double2 {tab[i], tab[i+1]-tab[i]}, i = 0..N-1,
// plus a terminal entry {tab[N], 0}; returns its offset.
static int push_table(std::vector<double2>& out, const std::vector<double>& tab) {
  int off = (int)out.size();
  for (size_t i = 0; i + 1 < tab.size(); ++i) out.push_back(make_double2(tab[i], tab[i + 1] - tab[i]));
  out.push_back(make_double2(tab.back(), 0.0));
  return off;
}

static void comp_from_spec(const StructSpec& s, int ndim, KkComp& c) {
  std::memset(&c, 0, sizeof c);
  c.vtype = s.vtype;
  c.is_product = s.is_product;
  c.sill = s.sill;
  c.nugget = s.nugget;
  c.a_major = s.a_major;
  c.tab_off = -1;
  c.tail = has_tail(s.vtype);
  // build_aniso_mat, variogram.f90:185-192
  calc_rotmat(s.az, s.dip, s.plunge, s.a_minor1 / s.a_major, s.a_minor2 / s.a_major, c.mat);
  for (int i = 0; i < 9; ++i) c.mat[i] = c.mat[i] / s.a_major;
  (void)ndim;
}

// struct_recompute_cov0, variogram.f90:853-869
static double model_cov0(const std::vector<StructSpec>& sp) {
  double total = 0.0;
  size_t iv = 0;
  while (iv < sp.size()) {
    double g = sp[iv].sill + sp[iv].nugget;
    while (iv + 1 < sp.size() && sp[iv + 1].is_product) {
      ++iv;
      g = g * (sp[iv].sill + sp[iv].nugget);
    }
    total = total + g;
    ++iv;
  }
  return total;
}

// struct_build_table (variogram.f90:497-537) with Level A (541-556) and
// Level B (572-679) tables; mode KK_ANALYTIC when no table is built.
static void build_model(const std::vector<StructSpec>& sp, int ndim, bool want_table, KkModel& m,
                        std::vector<double2>& tables) {
  std::memset(&m, 0, sizeof m);
  m.ndim = ndim;
  m.nstruct = (int)sp.size();
  m.cov0 = model_cov0(sp);
  m.btab_off = -1;
  for (int i = 0; i < m.nstruct; ++i) comp_from_spec(sp[i], ndim, m.comp[i]);
  m.mode = KK_ANALYTIC;
  if (!want_table) return;
  int zn[KK_TAB_NZ], off[KK_TAB_NZ];
  double inv_dh[KK_TAB_NZ];
  zones(zn, off, inv_dh);
  int ntab = off[KK_TAB_NZ - 1] + zn[KK_TAB_NZ - 1];
  int ref = -1;
  bool level_a = false;
  for (int iv = 0; iv < m.nstruct; ++iv) {
    if (sp[iv].vtype == KK_NUG) continue;
    if (ref < 0) { ref = iv; continue; }
    bool mismatch;
    if (sp[iv].is_product) {
      mismatch = std::fabs(sp[iv].az - sp[ref].az) > 1.0e-4 || std::fabs(sp[iv].dip - sp[ref].dip) > 1.0e-4 ||
                 std::fabs(sp[iv].plunge - sp[ref].plunge) > 1.0e-4;
    } else {
      double mx = 0.0;
      for (int q = 0; q < 9; ++q) mx = std::fmax(mx, std::fabs(m.comp[iv].mat[q] - m.comp[ref].mat[q]));
      mismatch = mx > 1.0e-6;
    }
    if (mismatch) { level_a = true; break; }
  }
  if (level_a) {
    m.mode = KK_LEVEL_A;
    for (int iv = 0; iv < m.nstruct; ++iv) {
      std::vector<double> tab(ntab + 1);
      tab[0] = sp[iv].sill + sp[iv].nugget;
      int o = 0;
      for (int k = 0; k < KK_TAB_NZ; ++k) {
        double step = 1.0 / inv_dh[k];
        for (int i = 1; i <= zn[k]; ++i) {
          double r = HB[k] + (double)i * step;
          tab[o + i] = sp[iv].sill * corefunc(sp[iv].vtype, r);
        }
        o += zn[k];
      }
      m.comp[iv].tab_off = push_table(tables, tab);
    }
    return;
  }
  if (ref < 0) return;  // all nugget: analytic (variogram.f90:531-533)
  m.mode = KK_LEVEL_B;
  const double aref = sp[ref].a_major;
  std::vector<double> tab(ntab + 1);
  tab[0] = m.cov0;
  for (int k = 0; k < KK_TAB_NZ; ++k) {
    double step = 1.0 / inv_dh[k];
    for (int i = 1; i <= zn[k]; ++i) {
      double r = HB[k] + (double)i * step;
      double val = 0.0;
      int iv = 0;
      while (iv < m.nstruct) {
        if (sp[iv].vtype == KK_NUG) { ++iv; continue; }
        double rk = r * aref / sp[iv].a_major;
        double g = sp[iv].sill * corefunc(sp[iv].vtype, rk);
        while (iv < m.nstruct - 1) {
          if (!sp[iv + 1].is_product) break;
          ++iv;
          rk = r * aref / sp[iv].a_major;
          g = g * sp[iv].sill * corefunc(sp[iv].vtype, rk);
        }
        val = val + g;
        ++iv;
      }
      tab[off[k] + i] = val;
    }
  }
  int tail = 0, iv = 0;
  while (iv < m.nstruct) {
    if (has_tail(sp[iv].vtype) && sp[iv].vtype != KK_NUG) {
      int gt = 1;
      while (iv < m.nstruct - 1 && sp[iv + 1].is_product) {
        ++iv;
        gt = gt && has_tail(sp[iv].vtype);
      }
      tail = tail || gt;
    }
    ++iv;
  }
  m.btail = tail;
  m.btab_off = push_table(tables, tab);
  std::memcpy(m.bmat, m.comp[ref].mat, sizeof m.bmat);
}

void build_models(const Engine& e, std::vector<KkModel>& mdl, std::vector<KkSTModel>& smdl,
                  std::vector<double2>& tables) {
  const int nv = e.nvar;
  mdl.assign(nv * nv, KkModel{});
  smdl.clear();
  tables.clear();
  if (!e.st) {
    // tables only for vgm(a, b) with b >= a (kriging.F90:412-421); the other
    // orientation evaluates analytically (variogram.f90:358)
    for (int a = 0; a < nv; ++a)
      for (int b = 0; b < nv; ++b) {
        int lo = a < b ? a : b, hi = a < b ? b : a;
        build_model(e.vgm[lo][hi], e.ndim, a <= b, mdl[a * nv + b], tables);
      }
    return;
  }
  smdl.assign(nv * nv, KkSTModel{});
  for (int a = 0; a < nv; ++a)
    for (int b = 0; b < nv; ++b) {
      int lo = a < b ? a : b, hi = a < b ? b : a;
      KkSTModel& s = smdl[a * nv + b];
      std::memset(&s, 0, sizeof s);
      build_model(e.vgm[lo][hi], e.ndim, true, s.cs, tables);
      build_model(e.vgm_t[lo][hi], 1, true, s.ct, tables);
      s.model = e.st_model;
      s.tvtype = e.st_transform;
      s.t_nugget = e.st_time_nugget;
      s.t_sill = e.st_time_sill;
      s.at = e.st_at;
      s.k_ps = e.st_k_ps;
      const std::vector<double>& j = e.joint[lo][hi];
      s.has_joint = j.empty() ? 0 : 1;
      for (size_t k = 0; k < j.size() && k < KK_MAXSTRUCT; ++k) s.joint[k] = j[k];
      // compute_cov0_vgm_st, variogram_st.f90:344-371
      if (s.model == 1) {
        s.cov0 = s.k_ps * s.cs.cov0 * s.ct.cov0 + s.cs.cov0 + s.ct.cov0;
      } else {
        s.cov0 = s.cs.cov0 + s.ct.cov0;
        if (s.has_joint)
          for (int k = 0; k < s.cs.nstruct; ++k)
            if (s.cs.comp[k].vtype != KK_NUG) s.cov0 = s.cov0 + s.joint[k];
      }
    }
}

// ---------------------------------------------------------------------------
// kd-tree build, restating kdtree2 (M. Kennel, AFL 1.1) as bundled in the
// reference (kdtree2_maxidx.f90:629-916): mean split on the dimension of
// largest spread, bucket size 12, boxes refined from the children.
// ---------------------------------------------------------------------------
#ifndef KK_KD_SPLIT_MIN
#define KK_KD_SPLIT_MIN (1 << 14)  // points from which subtrees build in threads
#endif

namespace {
constexpr int KD_EXT = -2;  // the parent is a node of another builder (a subtree's root)

struct TreeBuild {
  int D = 0;
  int* ind = nullptr;     // shared by every builder: disjoint ranges
  // the points in the order of ind (row i = data row ind[i]): every pass over
  // a node's range reads them in sequence instead of gathering
  double* pts = nullptr;
  std::vector<int> ni;      // 5 per node
  std::vector<double> nd;   // 3 per node
  std::vector<double> box;  // 2*D per node
  // the parent of a subtree's root, in the builder above it
  int ext_cut = -1;
  const double* ext_box = nullptr;
  // the builder above the subtrees: ranges left for them, and the nodes whose
  // boxes wait for their children
  struct Job { int l, u, parent, side; };
  int split_depth = -1;
  std::vector<Job> jobs;
  std::vector<int> pending;

  double v(int c, int i) const { return pts[(size_t)i * D + c]; }  // coordinate c of range position i

  void spread(int c, int l, int u, double& smin, double& smax) const {
    smin = v(c, l);
    smax = smin;
    int i;
    for (i = l + 2; i <= u; i += 2) {
      double lmin = v(c, i - 1), lmax = v(c, i);
      if (lmin > lmax) std::swap(lmin, lmax);
      if (smin > lmin) smin = lmin;
      if (smax < lmax) smax = lmax;
    }
    if (i == u + 1) {
      double last = v(c, u);
      if (smin > last) smin = last;
      if (smax < last) smax = last;
    }
  }
  void swap_pos(int a, int b) {
    std::swap(ind[a], ind[b]);
    for (int k = 0; k < D; ++k) std::swap(pts[(size_t)a * D + k], pts[(size_t)b * D + k]);
  }
  int select_value(int c, double alpha, int lb, int rb) {
    while (lb < rb) {
      if (v(c, lb) <= alpha) ++lb;
      else { swap_pos(lb, rb); --rb; }
    }
    return v(c, lb) <= alpha ? lb : lb - 1;
  }
  int node(int l, int u, int parent, int depth = 0, int side = 0) {
    if (u < l) return -1;
    if (depth == split_depth) {  // left for a subtree builder
      jobs.push_back({l, u, parent, side});
      return -1;
    }
    int me = (int)(ni.size() / 5);
    ni.resize(ni.size() + 5);
    nd.resize(nd.size() + 3);
    box.resize(box.size() + 2 * D);
    ni[me * 5 + 1] = l;
    ni[me * 5 + 2] = u;
    ni[me * 5 + 3] = -1;
    ni[me * 5 + 4] = -1;
    double* bx = &box[(size_t)me * 2 * D];
    if (u - l <= 12) {
      for (int i = 0; i < D; ++i) spread(i, l, u, bx[2 * i], bx[2 * i + 1]);
      ni[me * 5 + 0] = 0;
      nd[me * 3 + 0] = 0.0;
      return me;
    }
    const int pcut = parent >= 0 ? ni[parent * 5 + 0] : (parent == KD_EXT ? ext_cut : -1);
    const double* pbox = parent >= 0 ? &box[(size_t)parent * 2 * D] : (parent == KD_EXT ? ext_box : nullptr);
    for (int i = 0; i < D; ++i) {
      if (pbox && i != pcut) {
        box[(size_t)me * 2 * D + 2 * i] = pbox[2 * i];
        box[(size_t)me * 2 * D + 2 * i + 1] = pbox[2 * i + 1];
      } else {
        double lo, hi;
        spread(i, l, u, lo, hi);
        box[(size_t)me * 2 * D + 2 * i] = lo;
        box[(size_t)me * 2 * D + 2 * i + 1] = hi;
      }
    }
    int c = 0;
    double best = box[(size_t)me * 2 * D + 1] - box[(size_t)me * 2 * D];
    for (int i = 1; i < D; ++i) {
      double s = box[(size_t)me * 2 * D + 2 * i + 1] - box[(size_t)me * 2 * D + 2 * i];
      if (s > best) { best = s; c = i; }
    }
    double sum = 0.0;
    for (int i = l; i <= u; ++i) sum = sum + v(c, i);
    double average = sum / (double)(u - l + 1);
    nd[me * 3 + 0] = average;
    int m = select_value(c, average, l, u);
    ni[me * 5 + 0] = c;
    int left = node(l, m, me, depth + 1, 3);
    int right = node(m + 1, u, me, depth + 1, 4);
    ni[me * 5 + 3] = left;
    ni[me * 5 + 4] = right;
    if (split_depth >= 0) pending.push_back(me);  // children may still be subtrees
    else refine(me);
    return me;
  }
  // the box and split bounds of node me from its children
  void refine(int me) {
    const int c = ni[me * 5 + 0], left = ni[me * 5 + 3], right = ni[me * 5 + 4];
    double* b = &box[(size_t)me * 2 * D];
    if (right < 0) {
      for (int i = 0; i < 2 * D; ++i) b[i] = box[(size_t)left * 2 * D + i];
      nd[me * 3 + 1] = box[(size_t)left * 2 * D + 2 * c + 1];
      nd[me * 3 + 0] = nd[me * 3 + 1];
    } else if (left < 0) {
      for (int i = 0; i < 2 * D; ++i) b[i] = box[(size_t)right * 2 * D + i];
      nd[me * 3 + 2] = box[(size_t)right * 2 * D + 2 * c];
      nd[me * 3 + 0] = nd[me * 3 + 2];
    } else {
      nd[me * 3 + 2] = box[(size_t)right * 2 * D + 2 * c];
      nd[me * 3 + 1] = box[(size_t)left * 2 * D + 2 * c + 1];
      nd[me * 3 + 0] = (nd[me * 3 + 1] + nd[me * 3 + 2]) / 2.0;
      for (int i = 0; i < D; ++i) {
        b[2 * i + 1] = std::fmax(box[(size_t)left * 2 * D + 2 * i + 1], box[(size_t)right * 2 * D + 2 * i + 1]);
        b[2 * i] = std::fmin(box[(size_t)left * 2 * D + 2 * i], box[(size_t)right * 2 * D + 2 * i]);
      }
    }
  }
};
}  // namespace

void build_kdtree(const double* data, int D, int n, std::vector<int>& node_i,
                  std::vector<double>& node_d, std::vector<double>& box, std::vector<int>& ind,
                  std::vector<double>& rdata, int& root) {
  ind.resize(n);
  for (int i = 0; i < n; ++i) ind[i] = i;
  rdata.assign(data, data + (size_t)D * n);  // becomes the points in tree order
  TreeBuild t;
  t.D = D;
  t.ind = ind.data();
  t.pts = rdata.data();
  // large sets: the nodes above depth 3 here, the (up to) eight subtrees below
  // them in threads over their disjoint ranges, then merged and the upper
  // boxes refined from their children (the same tree as a serial build)
  t.split_depth = n >= KK_KD_SPLIT_MIN ? 3 : -1;
  root = t.node(0, n - 1, -1);
  if (!t.jobs.empty()) {
    std::vector<TreeBuild> sub(t.jobs.size());
    std::vector<std::vector<double>> pbox(t.jobs.size());
    for (size_t j = 0; j < t.jobs.size(); ++j) {
      const TreeBuild::Job& jb = t.jobs[j];
      TreeBuild& b = sub[j];
      b.D = D;
      b.ind = t.ind;
      b.pts = t.pts;
      b.ext_cut = t.ni[jb.parent * 5 + 0];
      pbox[j].assign(&t.box[(size_t)jb.parent * 2 * D], &t.box[(size_t)jb.parent * 2 * D] + 2 * D);
      b.ext_box = pbox[j].data();
    }
    std::vector<int> sroot(t.jobs.size(), -1);
    par_for(t.jobs.size(), 1, [&](size_t j0, size_t j1) {
      for (size_t j = j0; j < j1; ++j) sroot[j] = sub[j].node(t.jobs[j].l, t.jobs[j].u, KD_EXT);
    });
    for (size_t j = 0; j < t.jobs.size(); ++j) {
      const int off = (int)(t.ni.size() / 5);
      const TreeBuild& b = sub[j];
      for (size_t k = 0; k < b.ni.size(); ++k) {
        int x = b.ni[k];
        if ((k % 5 == 3 || k % 5 == 4) && x >= 0) x += off;
        t.ni.push_back(x);
      }
      t.nd.insert(t.nd.end(), b.nd.begin(), b.nd.end());
      t.box.insert(t.box.end(), b.box.begin(), b.box.end());
      t.ni[t.jobs[j].parent * 5 + t.jobs[j].side] = sroot[j] >= 0 ? sroot[j] + off : -1;
    }
  }
  for (int me : t.pending) t.refine(me);  // listed after their children (post-order)
  node_i.swap(t.ni);
  node_d.swap(t.nd);
  box.swap(t.box);
}

}  // namespace kk
