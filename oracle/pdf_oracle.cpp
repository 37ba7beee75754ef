/*
 * pdf_oracle.cpp — FP64 CPU oracle of the projective-dynamics step loop with
 * dry frictional contact.
 *
 * TEST INFRASTRUCTURE ONLY: a plain restatement of the reference algorithm
 * used as the checker by tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py.  Nothing in the product links or calls this file.
 *
 * Each function cites the reference file:line it restates (paths relative to
 * the reference project root; "SFE" = src/physics/SimulationFrictionEstimation.cpp).
 * Build with -ffp-contract=off so that the detection arithmetic rounds like
 * the reference compiled without FMA contraction.
 *
 * Declared deviations (both sides of every parity test share them):
 *  - Eigen SimplicialLLT (AMD ordering) is replaced by an up-looking sparse
 *    LL^T with a nested-dissection ordering: the same factorisation up to
 *    rounding.
 *  - CGAL box_intersection_d emits candidates in an unspecified order; here
 *    candidates are visited in canonical order (vertex asc, triangle asc).
 *  - Local forces of contacts whose storage slot is new are zero (the
 *    reference leaves them uninitialised; SFE:336 resize).
 *  - Self collision is detected per mesh with scene-global vertex indices (the
 *    reference uses mesh-local indices, geometry_util.cpp:196, which is only
 *    correct for the first mesh).
 */
#include "pdf_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static thread_local std::string g_error;

/* ------------------------------------------------------------------ V3 */
struct V3 {
  double x, y, z;
};
static inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline double sqn(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline double nrm(V3 a) { return std::sqrt(sqn(a)); }
static inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
/* Eigen normalized(): divide by the norm unless the vector is zero. */
static inline V3 normalized(V3 a) {
  double z = sqn(a);
  if (z > 0.) {
    double s = std::sqrt(z);
    return {a.x / s, a.y / s, a.z / s};
  }
  return a;
}
static inline V3 ld(const double* p, int64_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
static inline void st(double* p, int64_t i, V3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}
static inline double comp(V3 v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

/* 3x3 basis stored by columns: col0 = normal, col1 = tangent, col2 = bitangent. */
struct Basis {
  V3 c0, c1, c2;
};
/* B^T v : component k = column_k . v */
static inline V3 btv(const Basis& b, V3 v) { return {dot(b.c0, v), dot(b.c1, v), dot(b.c2, v)}; }
/* B r : component i = (B(i,0) r0 + B(i,1) r1) + B(i,2) r2 */
static inline V3 bv(const Basis& b, V3 r) {
  return {b.c0.x * r.x + b.c1.x * r.y + b.c2.x * r.z, b.c0.y * r.x + b.c1.y * r.y + b.c2.y * r.z,
          b.c0.z * r.x + b.c1.z * r.y + b.c2.z * r.z};
}

/* computeBasis SFE:91-105 */
static Basis compute_basis(V3 n) {
  const V3 t1{1., 0., 0.}, t2{0., 1., 0.};
  V3 t = cross(n, t1);
  if (nrm(t) < 1.e-15) t = cross(n, t2);
  t = normalized(t);
  V3 bt = normalized(cross(n, t));
  return {n, t, bt};
}

/* ------------------------------------------------------- closest point */
/* closestPointToTriangle, src/geometry/geometry_util.cpp:506-616 (Ericson) with
 * the reference's early exit (tol2 is whatever the caller passes). */
static void closest_point(V3 p, V3 a, V3 b, V3 c, double tol2, V3& cp, V3& bary) {
  const V3 ap = p - a, ab = b - a, ac = c - a;
  if (sqn(ap) - sqn(ab) - sqn(ac) > tol2) {
    cp = a;
    bary = {1, 0, 0};
    return;
  }
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) {
    cp = a;
    bary = {1, 0, 0};
    return;
  }
  const V3 bp = p - b;
  const double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) {
    cp = b;
    bary = {0, 1, 0};
    return;
  }
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
    const double v = d1 / (d1 - d3);
    cp = a + v * ab;
    bary = {1 - v, v, 0};
    return;
  }
  const V3 cpv = p - c;
  const double d5 = dot(ab, cpv), d6 = dot(ac, cpv);
  if (d6 >= 0.0 && d5 <= d6) {
    cp = c;
    bary = {0, 0, 1};
    return;
  }
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    const double w = d2 / (d2 - d6);
    cp = a + w * ac;
    bary = {1 - w, 0, w};
    return;
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
    const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    cp = b + w * (c - b);
    bary = {0, 1 - w, w};
    return;
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  cp = a + ab * v + ac * w;
  bary = {1. - v - w, v, w};
}

/* Matrix [a b c] times barycentric vector: ((a_i b0 + b_i b1) + c_i b2). */
static inline V3 tri_point(V3 a, V3 b, V3 c, V3 w) {
  return {a.x * w.x + b.x * w.y + c.x * w.z, a.y * w.x + b.y * w.y + c.y * w.z,
          a.z * w.x + b.z * w.y + c.z * w.z};
}

/* ------------------------------------------------- candidate detection */
/* getMeshPotentialTriangleCollision + getToleranceBoundingBox
 * (geometry_util.cpp:284-327): closed-box overlap between each triangle's
 * bounding box and [x - t, x + t].  A uniform grid only accelerates the search;
 * the exact overlap test defines the set.  Output per vertex, triangle-sorted. */
static void box_candidates(const std::vector<V3>& verts, const std::vector<std::array<int, 3>>& tris,
                           const std::vector<V3>& tri_pos_src, double t,
                           std::vector<std::vector<int>>& out) {
  (void)tri_pos_src;
  const int64_t nv = (int64_t)verts.size();
  out.assign(nv, {});
  if (tris.empty() || nv == 0) return;
  /* tri_pos_src holds the triangle's own vertex array (may differ from verts) */
  const std::vector<V3>& tp = tri_pos_src;
  const int64_t nt = (int64_t)tris.size();
  std::vector<V3> tmin(nt), tmax(nt);
  double ext = 0.;
  V3 lo{1e300, 1e300, 1e300};
  for (int64_t i = 0; i < nt; ++i) {
    V3 a = tp[tris[i][0]], b = tp[tris[i][1]], c = tp[tris[i][2]];
    tmin[i] = {std::min(std::min(a.x, b.x), c.x), std::min(std::min(a.y, b.y), c.y),
               std::min(std::min(a.z, b.z), c.z)};
    tmax[i] = {std::max(std::max(a.x, b.x), c.x), std::max(std::max(a.y, b.y), c.y),
               std::max(std::max(a.z, b.z), c.z)};
    ext = std::max(ext, std::max(tmax[i].x - tmin[i].x,
                                 std::max(tmax[i].y - tmin[i].y, tmax[i].z - tmin[i].z)));
    lo.x = std::min(lo.x, tmin[i].x);
    lo.y = std::min(lo.y, tmin[i].y);
    lo.z = std::min(lo.z, tmin[i].z);
  }
  double h = std::max(ext, 2.0 * t);
  if (!(h > 0.) || !std::isfinite(h)) h = 1.0;
  auto cell = [&](double x, double o) { return (int64_t)std::floor((x - o) / h); };
  auto key = [](int64_t i, int64_t j, int64_t k) {
    return (uint64_t)((i + (1 << 20)) & 0x1fffff) | ((uint64_t)((j + (1 << 20)) & 0x1fffff) << 21) |
           ((uint64_t)((k + (1 << 20)) & 0x1fffff) << 42);
  };
  std::unordered_map<uint64_t, std::vector<int>> grid;
  grid.reserve(nt * 2);
  for (int64_t i = 0; i < nt; ++i) {
    for (int64_t a = cell(tmin[i].x, lo.x); a <= cell(tmax[i].x, lo.x); ++a)
      for (int64_t b = cell(tmin[i].y, lo.y); b <= cell(tmax[i].y, lo.y); ++b)
        for (int64_t c = cell(tmin[i].z, lo.z); c <= cell(tmax[i].z, lo.z); ++c)
          grid[key(a, b, c)].push_back((int)i);
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t v = 0; v < nv; ++v) {
    const V3 x = verts[v];
    const V3 bmin{x.x - t, x.y - t, x.z - t}, bmax{x.x + t, x.y + t, x.z + t};
    std::vector<int>& res = out[v];
    for (int64_t a = cell(bmin.x, lo.x) - 1; a <= cell(bmax.x, lo.x) + 1; ++a)
      for (int64_t b = cell(bmin.y, lo.y) - 1; b <= cell(bmax.y, lo.y) + 1; ++b)
        for (int64_t c = cell(bmin.z, lo.z) - 1; c <= cell(bmax.z, lo.z) + 1; ++c) {
          auto it = grid.find(key(a, b, c));
          if (it == grid.end()) continue;
          for (int tI : it->second) {
            if (tmin[tI].x <= bmax.x && bmin.x <= tmax[tI].x && tmin[tI].y <= bmax.y &&
                bmin.y <= tmax[tI].y && tmin[tI].z <= bmax.z && bmin.z <= tmax[tI].z)
              res.push_back(tI);
          }
        }
    std::sort(res.begin(), res.end());
    res.erase(std::unique(res.begin(), res.end()), res.end());
  }
}

struct Hit {
  int tri;
  V3 bary;
};

/* checkMeshAllCollision, geometry_util.cpp:229-262: candidates with box
 * half-width 1.1*tol, closest point with the early exit passed the UNSQUARED
 * tolerance, kept if the squared distance is below tol^2. */
static void all_collisions(const std::vector<V3>& verts, const std::vector<V3>& tri_verts,
                           const std::vector<std::array<int, 3>>& tris, double tol,
                           std::vector<std::vector<Hit>>& out) {
  std::vector<std::vector<int>> cand;
  box_candidates(verts, tris, tri_verts, 1.1 * tol, cand);
  const double tol_sq = tol * tol;
  out.assign(verts.size(), {});
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t v = 0; v < (int64_t)verts.size(); ++v) {
    for (int tI : cand[v]) {
      const V3 x = verts[v];
      V3 cp, bary;
      closest_point(x, tri_verts[tris[tI][0]], tri_verts[tris[tI][1]], tri_verts[tris[tI][2]], tol,
                    cp, bary);
      if (sqn(cp - x) < tol_sq) out[v].push_back({tI, bary});
    }
  }
}

struct SelfInfo {
  int vertex;
  int face[3];
  V3 normal;
  V3 bary;
  double mu;
};

/* checkMeshSelfCollisions(const Mesh&, double), geometry_util.cpp:94-219.
 * verts: this mesh's vertices (mesh-local), tris mesh-local, rings: 1-rings
 * (mesh-local). */
static std::vector<SelfInfo> self_collisions(const std::vector<V3>& verts,
                                             const std::vector<std::array<int, 3>>& tris,
                                             const std::vector<std::vector<int>>& rings,
                                             double tolerance) {
  std::vector<std::vector<Hit>> hits;
  all_collisions(verts, verts, tris, tolerance, hits);
  std::vector<SelfInfo> result;
  std::vector<std::vector<int>> registered(verts.size());
  /* isTriangleVertexIndexIn, geometry_util.cpp:211-219 */
  auto tri_in = [&](const std::array<int, 3>& t, const std::vector<int>& lst) -> int {
    for (int i = 0; i < 3; ++i)
      for (int x : lst)
        if (t[i] == x) return i;
    return 3;
  };
  for (int v = 0; v < (int)verts.size(); ++v) {
    for (const Hit& h : hits[v]) {
      const std::array<int, 3>& t = tris[h.tri];
      V3 bary = h.bary;
      if (t[0] == v || t[1] == v || t[2] == v || bary.x == 0 || bary.y == 0 || bary.z == 0) continue;
      if (tri_in(t, registered[v]) < 3) continue;
      bool cand[3] = {true, true, true};
      for (int r : rings[v]) {
        int k = tri_in(t, registered[r]);
        if (k < 3) cand[k] = false;
      }
      int best = 3;
      double best_b = 0;
      for (int k = 0; k < 3; ++k) {
        if (!cand[k]) continue;
        double bk = comp(bary, k);
        if (bk > best_b) {
          best = k;
          best_b = bk;
        }
      }
      if (best >= 3) continue;
      V3 cpt = tri_point(verts[t[0]], verts[t[1]], verts[t[2]], bary);
      SelfInfo info;
      info.normal = normalized(verts[v] - cpt);
      int paired = t[best];
      double b3[3] = {0, 0, 0};
      b3[best] = 1.;
      info.bary = {b3[0], b3[1], b3[2]};
      registered[paired].push_back(v);
      registered[v].push_back(paired);
      info.face[0] = t[0];
      info.face[1] = t[1];
      info.face[2] = t[2];
      info.vertex = v;
      info.mu = 0;
      result.push_back(info);
    }
  }
  return result;
}

/* ---------------------------------------------------------- topology */
struct Topo {
  std::vector<std::array<int, 2>> edges; /* per mesh in CGAL creation order */
  std::vector<std::vector<int>> ring;    /* clockwise 1-ring of interior vertices */
  std::vector<std::vector<int>> nbrs;    /* 1-ring (any order) of every vertex */
  std::vector<char> border;
  std::vector<std::vector<int>> vfaces; /* faces incident to each vertex */
};

/* Mesh topology of CGAL::Surface_mesh as used by Mesh (src/geometry/Mesh.cpp:31-56,
 * 219-292): edges numbered in order of first appearance while adding faces,
 * vertices_around_target circulating clockwise (h -> opposite(next(h))),
 * border = some incident halfedge without a face on one side. */
static void build_topology(int nv, const std::vector<std::array<int, 3>>& tris, int v0, int v1,
                           int t0, int t1, Topo& tp) {
  std::unordered_map<uint64_t, int> he; /* (u,v) -> halfedge id */
  auto k = [&](int u, int v) { return ((uint64_t)(uint32_t)u << 32) | (uint32_t)v; };
  he.reserve((size_t)(t1 - t0) * 3 * 2);
  for (int f = t0; f < t1; ++f)
    for (int i = 0; i < 3; ++i) he[k(tris[f][i], tris[f][(i + 1) % 3])] = 3 * f + i;
  for (int f = t0; f < t1; ++f)
    for (int i = 0; i < 3; ++i) {
      int a = tris[f][i], b = tris[f][(i + 1) % 3];
      auto it = he.find(k(b, a));
      bool exists_before = (it != he.end() && it->second < 3 * f + i);
      if (!exists_before) tp.edges.push_back({b, a});
      if (it == he.end()) {
        tp.border[a] = 1;
        tp.border[b] = 1;
      }
      tp.vfaces[a].push_back(f);
      tp.nbrs[a].push_back(b);
      tp.nbrs[b].push_back(a);
    }
  for (int v = v0; v < v1; ++v) {
    std::sort(tp.nbrs[v].begin(), tp.nbrs[v].end());
    tp.nbrs[v].erase(std::unique(tp.nbrs[v].begin(), tp.nbrs[v].end()), tp.nbrs[v].end());
    if (tp.vfaces[v].empty()) tp.border[v] = 1;
    if (tp.border[v]) continue;
    /* incoming halfedge to v in its first face */
    int f = tp.vfaces[v][0];
    int i = 0;
    while (tris[f][i] != v) ++i;
    int h = 3 * f + (i + 2) % 3; /* (prev -> v) */
    const int h0 = h;
    int guard = 0;
    do {
      int hf = h / 3, hi = h % 3;
      int src = tris[hf][hi];
      tp.ring[v].push_back(src);
      int nx = 3 * hf + (hi + 1) % 3; /* next(h): v -> w */
      int a = tris[hf][(hi + 1) % 3], b = tris[hf][(hi + 2) % 3];
      auto it = he.find(k(b, a)); /* opposite(next(h)) : w -> v */
      (void)nx;
      if (it == he.end()) {
        tp.border[v] = 1;
        tp.ring[v].clear();
        break;
      }
      h = it->second;
    } while (h != h0 && ++guard < 1000);
  }
  (void)nv;
}

/* getMeanValue / getSine / getCosine, geometry_util.cpp:766-791 */
static double get_sine(V3 v1, V3 v2, V3 v3) {
  V3 e1 = v1 - v2, e2 = v3 - v2;
  return nrm(cross(e1, e2)) / (nrm(e1) * nrm(e2));
}
static double get_cosine(V3 v1, V3 v2, V3 v3) {
  V3 e1 = v1 - v2, e2 = v3 - v2;
  return dot(e1, e2) / (nrm(e1) * nrm(e2));
}
static double get_mean_value(V3 v1, V3 v2, V3 v3) {
  double num = (1 - get_cosine(v1, v2, v3));
  if (num == 0) return 0;
  return num / get_sine(v1, v2, v3);
}
/* getLaplaceBeltramiDiscretisationMeanValueCoefficients, geometry_util.cpp:673-710 */
static std::vector<double> mean_value_coeffs(V3 mid, const std::vector<V3>& ring) {
  std::vector<double> res;
  const size_t n = ring.size();
  for (size_t i = 0; i < n; ++i) {
    V3 vtx = ring[i], cw = ring[(i + 1) % n], ccw = ring[(i + n - 1) % n];
    double dist = nrm(vtx - mid);
    double cwm = get_mean_value(vtx, mid, cw);
    double ccwm = get_mean_value(vtx, ccw, mid);
    res.push_back((cwm + ccwm) / dist);
  }
  return res;
}

/* ---------------------------------------------------------- sparse */
struct CSR {
  int n = 0, m = 0;
  std::vector<int64_t> ptr;
  std::vector<int> col;
  std::vector<double> val;
};

/* Up-looking sparse Cholesky LL^T (the published CSparse cs_chol algorithm,
 * T. Davis, "Direct Methods for Sparse Linear Systems", ch. 4) on P A P^T with a
 * nested-dissection ordering P.  Replaces Eigen::SimplicialLLT
 * (include/physics/SimulationSpeed.hpp:102, SimulationSpeed.cpp:53). */
struct Chol {
  int n = 0;
  std::vector<int> perm, iperm;
  std::vector<int64_t> Lp;
  std::vector<int> Li;
  std::vector<double> Lx;

  static void nd_order(const CSR& A, const std::vector<V3>& pos, std::vector<int>& ids,
                       std::vector<char>& side, std::vector<int>& out) {
    if (ids.size() <= 48) {
      out.insert(out.end(), ids.begin(), ids.end());
      return;
    }
    V3 lo{1e300, 1e300, 1e300}, hi{-1e300, -1e300, -1e300};
    for (int v : ids) {
      lo = {std::min(lo.x, pos[v].x), std::min(lo.y, pos[v].y), std::min(lo.z, pos[v].z)};
      hi = {std::max(hi.x, pos[v].x), std::max(hi.y, pos[v].y), std::max(hi.z, pos[v].z)};
    }
    V3 e = hi - lo;
    int ax = (e.x >= e.y && e.x >= e.z) ? 0 : (e.y >= e.z ? 1 : 2);
    size_t mid = ids.size() / 2;
    std::nth_element(ids.begin(), ids.begin() + mid, ids.end(), [&](int a, int b) {
      double ca = comp(pos[a], ax), cb = comp(pos[b], ax);
      return ca < cb || (ca == cb && a < b);
    });
    std::vector<int> s1(ids.begin(), ids.begin() + mid), s2(ids.begin() + mid, ids.end());
    for (int v : s1) side[v] = 1;
    std::vector<int> s2r, sep;
    for (int v : s2) {
      bool touch = false;
      for (int64_t p = A.ptr[v]; p < A.ptr[v + 1] && !touch; ++p) touch = side[A.col[p]] == 1;
      (touch ? sep : s2r).push_back(v);
    }
    for (int v : s1) side[v] = 0;
    ids.clear();
    ids.shrink_to_fit();
    nd_order(A, pos, s1, side, out);
    nd_order(A, pos, s2r, side, out);
    out.insert(out.end(), sep.begin(), sep.end());
  }

  bool factor(const CSR& A, const std::vector<V3>& pos) {
    n = A.n;
    std::vector<int> ids(n);
    for (int i = 0; i < n; ++i) ids[i] = i;
    std::vector<char> side(n, 0);
    perm.clear();
    nd_order(A, pos, ids, side, perm);
    iperm.assign(n, 0);
    for (int k = 0; k < n; ++k) iperm[perm[k]] = k;
    /* column k of C = P A P^T, upper part (rows <= k) */
    auto col_of = [&](int k, std::vector<std::pair<int, double>>& c) {
      c.clear();
      int r = perm[k];
      for (int64_t p = A.ptr[r]; p < A.ptr[r + 1]; ++p) {
        int i = iperm[A.col[p]];
        if (i <= k) c.push_back({i, A.val[p]});
      }
    };
    /* elimination tree (cs_etree) */
    std::vector<int> parent(n, -1), anc(n, -1);
    std::vector<std::pair<int, double>> ck;
    for (int k = 0; k < n; ++k) {
      col_of(k, ck);
      for (auto& e : ck) {
        int i = e.first;
        while (i != -1 && i < k) {
          int inext = anc[i];
          anc[i] = k;
          if (inext == -1) parent[i] = k;
          i = inext;
        }
      }
    }
    std::vector<int> w(n, -1), s(n);
    auto ereach = [&](int k, const std::vector<std::pair<int, double>>& c) {
      int top = n;
      w[k] = k;
      for (auto& e : c) {
        int i = e.first;
        if (i > k) continue;
        int len = 0;
        while (w[i] != k) {
          s[len++] = i;
          w[i] = k;
          i = parent[i];
        }
        while (len > 0) s[--top] = s[--len];
      }
      return top;
    };
    /* symbolic: column counts */
    std::vector<int64_t> cnt(n, 1);
    for (int k = 0; k < n; ++k) {
      col_of(k, ck);
      int top = ereach(k, ck);
      for (int p = top; p < n; ++p) cnt[s[p]]++;
    }
    Lp.assign(n + 1, 0);
    for (int k = 0; k < n; ++k) Lp[k + 1] = Lp[k] + cnt[k];
    Li.assign(Lp[n], 0);
    Lx.assign(Lp[n], 0.);
    std::vector<int64_t> c(Lp.begin(), Lp.end() - 1);
    std::vector<double> x(n, 0.);
    std::fill(w.begin(), w.end(), -1);
    for (int k = 0; k < n; ++k) {
      col_of(k, ck);
      int top = ereach(k, ck);
      x[k] = 0;
      for (auto& e : ck) x[e.first] = e.second;
      double d = x[k];
      x[k] = 0;
      for (; top < n; ++top) {
        int i = s[top];
        double lki = x[i] / Lx[Lp[i]];
        x[i] = 0;
        for (int64_t q = Lp[i] + 1; q < c[i]; ++q) x[Li[q]] -= Lx[q] * lki;
        d -= lki * lki;
        int64_t q = c[i]++;
        Li[q] = k;
        Lx[q] = lki;
      }
      if (!(d > 0.)) return false;
      int64_t q = c[k]++;
      Li[q] = k;
      Lx[q] = std::sqrt(d);
    }
    return true;
  }

  /* x <- A^-1 x for one right-hand side */
  void solve(double* b, std::vector<double>& x) const {
    x.resize(n);
    for (int k = 0; k < n; ++k) x[k] = b[perm[k]];
    for (int j = 0; j < n; ++j) {
      x[j] /= Lx[Lp[j]];
      for (int64_t q = Lp[j] + 1; q < Lp[j + 1]; ++q) x[Li[q]] -= Lx[q] * x[j];
    }
    for (int j = n - 1; j >= 0; --j) {
      for (int64_t q = Lp[j] + 1; q < Lp[j + 1]; ++q) x[j] -= Lx[q] * x[Li[q]];
      x[j] /= Lx[Lp[j]];
    }
    for (int k = 0; k < n; ++k) b[perm[k]] = x[k];
  }
};

/* --------------------------------------------------------- obstacles */
struct Obstacle {
  int type, material;
  V3 center;
  double radius;
  V3 rot; /* angular_speed * axis.normalized() */
  double time_before_start;
  V3 point, normal;
  std::vector<V3> mverts;
  std::vector<std::array<int, 3>> mtris;
  double threshold;
  int mesh; /* -1: every dynamic mesh; else only vertices of that mesh */
  V3 size;  /* box: extents; center = the corner with the smallest coordinates */
  /* moving mesh (MovingMesh.cpp:28-41): every key frame, the clock, the index
   * of the next key frame; mverts is the current (interpolated) mesh */
  std::vector<std::vector<V3>> frames;
  double interval = 0., clock = 0.;
  int next = 1;
  double frame_time(int f) const { return (double)f * interval; }
  /* MovingMesh::isInMovement MovingMesh.cpp:253-257 */
  bool in_movement() const { return clock >= frame_time(next - 1) && clock <= frame_time(next); }
};

struct CInfo {
  int vertex;
  V3 cp, normal, speed;
  double mu;
  double gap; /* signed distance to the obstacle surface (warm-start feature) */
};

/* -------------------------------------------------------------- sim */
struct Sim {
  int N = 0;
  pdf_params prm;
  std::vector<V3> rest;
  std::vector<double> q, v;    /* scene generalized positions / speeds (3N) */
  std::vector<double> mass;    /* lumped masses */
  std::vector<std::array<int, 3>> tris;
  std::vector<pdf_mesh_desc> meshes;
  std::vector<int> vmesh;      /* containing mesh of each vertex */
  Topo topo;
  /* constraints in row order */
  struct Spring {
    int i, j;
    double w, L;
  };
  struct Bend {
    std::vector<int> idx;     /* centre then ring */
    std::vector<double> coef; /* beltrami coefficients (unweighted) */
    double w, rest_norm;
  };
  struct Pin {
    int i;
    double w;
    V3 x0;
  };
  /* row -> (kind, index) */
  std::vector<std::pair<int, int>> rows;
  std::vector<Spring> springs;
  std::vector<Bend> bends;
  std::vector<Pin> pins;
  CSR At;   /* A^T in CSR: rows = vertices, entries (constraint row, value) */
  CSR ATA;  /* A^T A */
  CSR LHS;  /* M + dt^2 A^T A */
  int64_t nnzA = 0;
  Chol chol;
  std::vector<Obstacle> obstacles;
  int n_mat = 0;
  std::vector<double> friction;
  double time = 0;

  /* per step */
  std::vector<double> tn, vnext, qnext, damping, rhs, proj, forces, last_rhs;
  std::vector<CInfo> contacts;
  std::vector<SelfInfo> selfc;
  std::vector<Basis> cbasis, sbasis;
  std::vector<V3> c_local_forces, s_local_forces;
  std::vector<double> c_ac, s_ac;
  std::vector<std::vector<int>> levels;
  std::vector<V3> remember;
  std::vector<double> contact_forces[2], self_forces[2];
  int cur = 0, nxt = 1;
  std::vector<double> residual_hist;
  /* per-iteration (tangential, |normal|) Alart-Curnier norms of every contact
   * of the last step, obstacle contacts first (the PRINT_ALART_CURNIER_ERROR
   * output of SFE:720-752) */
  bool trace_ac = false;
  std::vector<double> ac_trace;
  int trace_nc = 0, trace_ns = 0;
  pdf_step_report last{};
  std::vector<double> tmpx;

  /* learned warm start (restates climatenet_b200/csrc/mlp.cu for checking) */
  std::vector<float> mlp_w;
  bool mlp_ready = false;
  std::vector<char> c_active;   /* last projection of the contact was not a take-off */
  std::vector<char> s_active;   /* same for the self contacts */
  /* per iteration: mean AC norm with the force each contact actually applied
   * in that iteration (zero after a take-off) instead of the stale local force
   * the reference keeps for it */
  std::vector<double> residual_applied_hist;
  std::vector<double> rprev;    /* world impulse per vertex, end of the tagged step */
  std::vector<int> rprev_tag;
  int mlp_tag = 0;
  std::vector<float> feat, pred; /* C x 10, C x 3 */
  std::vector<float> log_X, log_T;
  int log_cap = 0, log_n = 0;

  int partner(const SelfInfo& s) const {
    const V3& a = s.bary;
    return s.face[(a.x > a.y) ? ((a.x > a.z) ? 0 : 2) : ((a.y > a.z) ? 1 : 2)];
  }
};

static void spmv3(const CSR& A, const double* x, double* y) {
#pragma omp parallel for schedule(static, 1024)
  for (int i = 0; i < A.n; ++i) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t p = A.ptr[i]; p < A.ptr[i + 1]; ++p) {
      const double a = A.val[p];
      const int j = A.col[p];
      s0 += a * x[3 * j];
      s1 += a * x[3 * j + 1];
      s2 += a * x[3 * j + 2];
    }
    y[3 * i] = s0;
    y[3 * i + 1] = s1;
    y[3 * i + 2] = s2;
  }
}

/* computeProjections SimulationBase.cpp:314-323 with
 * SpringConstraint::addConstraintProjection SpringConstraint.cpp:57-69,
 * BendingConstraint::addConstraintProjection BendingConstraint.cpp:106-138,
 * AttachmentConstraint::addConstraintProjection AttachmentConstraint.cpp:45-51. */
static void projections(Sim& s, const double* x, double* p) {
  const int64_t R = (int64_t)s.rows.size();
#pragma omp parallel for schedule(static, 1024)
  for (int64_t r = 0; r < R; ++r) {
    const int kind = s.rows[r].first, id = s.rows[r].second;
    V3 out{0, 0, 0};
    if (kind == 0) {
      const auto& sp = s.springs[id];
      V3 e = normalized(ld(x, sp.i) - ld(x, sp.j));
      out = (sp.w * sp.L) * e;
    } else if (kind == 1) {
      const auto& b = s.bends[id];
      V3 lb{0, 0, 0};
      for (size_t k = 0; k < b.idx.size(); ++k) lb = lb + b.coef[k] * ld(x, b.idx[k]);
      double lbn = nrm(lb);
      if (lbn > 1e-25) {
        lb = lb * (b.rest_norm / lbn);
        out = b.w * lb;
      } else {
        out = {0, 0, 0};
      }
    } else {
      const auto& pn = s.pins[id];
      out = pn.w * pn.x0;
    }
    st(p, r, out);
  }
}

/* SimulationSpeed::computeRhs SimulationSpeed.cpp:238-278 (base RHS). */
static void rhs_base(Sim& s, const double* qn, const double* tn, const double* vk,
                     const double* qk, double* rhs) {
  const int N = s.N;
  projections(s, qk, s.proj.data());
  std::vector<double> atp(3 * N), ataq(3 * N);
  spmv3(s.At, s.proj.data(), atp.data());
  spmv3(s.ATA, qn, ataq.data());
  const double dt = s.prm.time_step;
#pragma omp parallel for schedule(static, 1024)
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) {
      const int64_t d = 3 * (int64_t)i + c;
      rhs[d] = s.mass[i] * tn[d] + dt * (atp[d] - s.damping[i] * vk[d] - ataq[d]);
    }
}

static std::vector<double> alart_curnier(V3 u, V3 r, double mu, double* an, double* at) {
  /* coulomb_util.cpp:92-152 (rho = 1) */
  auto mx = [](double a, double b) { return (a < b) ? b : a; };
  auto mn = [](double a, double b) { return (b < a) ? b : a; };
  double N = mx(0., r.x - u.x) - r.x;
  double dtx = r.y - u.y, dty = r.z - u.z;
  double dn = std::sqrt(dtx * dtx + dty * dty);
  double radius = mx(0., mu * r.x / dn);
  double m = mn(1., radius);
  double Tx = dtx * m - r.y, Ty = dty * m - r.z;
  *an = std::abs(N);
  *at = std::sqrt(Tx * Tx + Ty * Ty);
  return {N, Tx, Ty};
}

/* SFE:161-293 computeCollisionComputationOrder & co. */
static void compute_order(Sim& s) {
  const int N = s.N;
  struct Nb {
    int index, cid;
  };
  std::vector<std::vector<Nb>> graph(N);
  for (size_t c = 0; c < s.selfc.size(); ++c) {
    int tgt = s.partner(s.selfc[c]);
    int src = s.selfc[c].vertex;
    graph[src].push_back({tgt, (int)c});
    graph[tgt].push_back({src, (int)c});
  }
  s.levels.clear();
  std::vector<char> visited(s.selfc.size(), 0);
  auto fill = [&](const std::vector<int>& start) {
    std::vector<int> last = start, visiting;
    size_t ci = 0;
    while (!last.empty()) {
      if (s.levels.size() <= ci) s.levels.emplace_back();
      for (int vx : last)
        for (const Nb& nb : graph[vx]) {
          if (visited[nb.cid]) continue;
          visiting.push_back(nb.index);
          visited[nb.cid] = 1;
          s.levels[ci].push_back(nb.cid);
        }
      last = std::move(visiting);
      visiting.clear();
      ++ci;
    }
  };
  auto vis = [&](int vx) {
    for (const Nb& nb : graph[vx])
      if (!visited[nb.cid]) return false;
    return true;
  };
  std::vector<int> start;
  for (auto& c : s.contacts) start.push_back(c.vertex);
  fill(start);
  for (int vx = 0; vx < N; ++vx) {
    if (vis(vx)) continue;
    if (graph[vx].size() == 1u) fill({vx});
  }
  for (int vx = 0; vx < N; ++vx) {
    if (vis(vx)) continue;
    if (graph[vx].size() > 1u) fill({vx});
  }
}

/* Obstacle detection: PhysicScene::getCollisionsInfoExceptFor PhysicScene.cpp:115-181
 * with Obstacle::checkCollision Obstacle.cpp:24-45 and the obstacle types. */
static void detect_obstacles(Sim& s) {
  s.contacts.clear();
  const int N = s.N;
  std::vector<V3> verts(N);
  for (int i = 0; i < N; ++i) verts[i] = ld(s.q.data(), i);
  for (auto& ob : s.obstacles) {
    std::vector<CInfo> found;
    if (ob.type == PDF_OBSTACLE_SPHERE || ob.type == PDF_OBSTACLE_ROTATING_SPHERE) {
      for (int i = 0; i < N; ++i) {
        /* Sphere::isInside Sphere.cpp:93-98, Sphere::project :104-113 */
        V3 r = verts[i] - ob.center;
        if (!(nrm(r) < ob.radius + 1e-2)) continue;
        V3 rn = normalized(verts[i] - ob.center);
        CInfo c;
        c.vertex = i;
        c.gap = nrm(r) - ob.radius;
        c.cp = ob.center + ob.radius * rn;
        c.normal = rn;
        c.speed = {0, 0, 0};
        if (ob.type == PDF_OBSTACLE_ROTATING_SPHERE && ob.time_before_start < 0) {
          /* RotatingSphere::checkCollision RotatingSphere.cpp:71-93 */
          c.speed = cross(ob.rot, c.cp - ob.center);
        }
        found.push_back(c);
      }
    } else if (ob.type == PDF_OBSTACLE_PLANE) {
      /* StaticPlane::checkCollision StaticPlane.cpp:57-73 */
      for (int i = 0; i < N; ++i) {
        double d = dot(verts[i] - ob.point, ob.normal);
        if (!(d < 1.5e-2)) continue;
        CInfo c;
        c.vertex = i;
        c.gap = d;
        c.cp = verts[i] - ob.normal * d;
        c.normal = ob.normal;
        c.speed = {0, 0, 0};
        found.push_back(c);
      }
    } else if (ob.type == PDF_OBSTACLE_BOX) {
      /* StaticAxisAlignedBox::checkCollision StaticAxisAlignedBox.cpp:41-58:
       * relative = x - position - size/2; inside when |relative_i| <= size_i/2
       * for every axis; nearest side by std::min_element over TOP, BOTTOM,
       * LEFT, RIGHT, FRONT, BACK (:67-80, first of equal distances) with
       * distance |relative[axis] - sign size[axis]/2| (:96-105); contact point
       * the projection on that side (:84-94), normal the side's axis vector. */
      const int ax[6] = {1, 1, 0, 0, 2, 2};
      const double sg[6] = {1., -1., -1., 1., 1., -1.};
      for (int i = 0; i < N; ++i) {
        const V3 x = verts[i];
        const double r[3] = {(x.x - ob.center.x) - 0.5 * ob.size.x, (x.y - ob.center.y) - 0.5 * ob.size.y,
                             (x.z - ob.center.z) - 0.5 * ob.size.z};
        const double sz[3] = {ob.size.x, ob.size.y, ob.size.z};
        bool in = true;
        for (int k = 0; k < 3; ++k)
          if (std::abs(r[k]) > sz[k] / 2) in = false;
        if (!in) continue;
        int b = 0;
        double best = std::abs(r[ax[0]] - sg[0] * 0.5 * sz[ax[0]]);
        for (int k = 1; k < 6; ++k) {
          const double d = std::abs(r[ax[k]] - sg[k] * 0.5 * sz[ax[k]]);
          if (d < best) {
            best = d;
            b = k;
          }
        }
        double cpr[3] = {r[0], r[1], r[2]};
        cpr[ax[b]] = sg[b] * 0.5 * sz[ax[b]];
        CInfo c;
        c.vertex = i;
        c.cp = {(cpr[0] + ob.center.x) + 0.5 * sz[0], (cpr[1] + ob.center.y) + 0.5 * sz[1],
                (cpr[2] + ob.center.z) + 0.5 * sz[2]};
        c.normal = {ax[b] == 0 ? sg[b] : 0., ax[b] == 1 ? sg[b] : 0., ax[b] == 2 ? sg[b] : 0.};
        c.gap = -best;
        c.speed = {0, 0, 0};
        found.push_back(c);
      }
    } else if (ob.type == PDF_OBSTACLE_MESH || ob.type == PDF_OBSTACLE_MOVING_MESH) {
      /* StaticMesh::checkCollision StaticMesh.cpp:33-48 and
       * MovingMesh::checkCollision MovingMesh.cpp:164-192 -> checkMeshCollision
       * (vector form) geometry_util.cpp:32-92 */
      double tol = std::sqrt(ob.threshold * ob.threshold);
      std::vector<std::vector<Hit>> hits;
      all_collisions(verts, ob.mverts, ob.mtris, tol, hits);
      double tol_sq = tol * tol;
      for (int i = 0; i < N; ++i) {
        double best = INFINITY;
        V3 bp{0, 0, 0}, bw{0, 0, 0};
        int bt = -1;
        for (const Hit& h : hits[i]) {
          const auto& t = ob.mtris[h.tri];
          V3 p = tri_point(ob.mverts[t[0]], ob.mverts[t[1]], ob.mverts[t[2]], h.bary);
          double d2 = sqn(p - verts[i]);
          if (d2 < best) {
            best = d2;
            bp = p;
            bw = h.bary;
            bt = h.tri;
          }
        }
        if (best < tol_sq) {
          const auto& t = ob.mtris[bt];
          CInfo c;
          c.vertex = i;
          c.cp = bp;
          c.normal = normalized(cross(ob.mverts[t[1]] - ob.mverts[t[0]], ob.mverts[t[2]] - ob.mverts[t[0]]));
          c.gap = dot(verts[i] - bp, c.normal);
          c.speed = {0, 0, 0};
          if (ob.type == PDF_OBSTACLE_MOVING_MESH && ob.in_movement()) {
            /* MovingMesh::getPointSpeed MovingMesh.cpp:232-249: the contact's
             * barycentric point on the two key frames around the clock */
            const std::vector<V3>& fp = ob.frames[ob.next - 1];
            const std::vector<V3>& fn = ob.frames[ob.next];
            const V3 pn = tri_point(fn[t[0]], fn[t[1]], fn[t[2]], bw);
            const V3 pp = tri_point(fp[t[0]], fp[t[1]], fp[t[2]], bw);
            const double span = ob.frame_time(ob.next) - ob.frame_time(ob.next - 1);
            const V3 dp = pn - pp;
            c.speed = {dp.x / span, dp.y / span, dp.z / span};
          }
          found.push_back(c);
        }
      }
    }
    for (auto& c : found) {
      if (ob.mesh >= 0 && s.vmesh[c.vertex] != ob.mesh) continue;
      int mm = s.meshes[s.vmesh[c.vertex]].material;
      c.mu = s.friction[(size_t)mm * s.n_mat + ob.material];
      s.contacts.push_back(c);
    }
  }
}

/* ------------------------------------------------- learned warm start
 * No counterpart in the reference: restates the product's warm start
 * (climatenet_b200/csrc/mlp.cu) so that its steps can be checked.  The MLP
 * forward emulates the tensor-core arithmetic: inputs, weights and hidden
 * activations rounded to bfloat16 (round to nearest even), products summed per
 * 16-wide k block in double and accumulated in float, biases added in float. */
static const int kMIn = 10, kMH = 64, kMOut = 3;
static const int kMParams = kMH * kMIn + kMH + kMH * kMH + kMH + kMOut * kMH + kMOut;

static float to_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return f;
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  std::memcpy(&f, &u, 4);
  return f;
}

static void mlp_layer(const float* W, const float* b, int nout, int nin, const float* in, float* out, bool relu) {
  for (int o = 0; o < nout; ++o) {
    float acc = 0.f;
    for (int k0 = 0; k0 < nin; k0 += 16) {
      double blk = 0.;
      for (int k = k0; k < std::min(nin, k0 + 16); ++k)
        blk += (double)to_bf16(in[k]) * (double)to_bf16(W[(size_t)o * nin + k]);
      acc = (float)((double)acc + blk);
    }
    const float z = acc + b[o];
    out[o] = relu ? (z > 0.f ? z : 0.f) : z;
  }
}

static void mlp_forward_one(const float* w, const float* x, float* y) {
  const float* W1 = w;
  const float* b1 = W1 + kMH * kMIn;
  const float* W2 = b1 + kMH;
  const float* b2 = W2 + kMH * kMH;
  const float* W3 = b2 + kMH;
  const float* b3 = W3 + kMOut * kMH;
  float h1[kMH], h2[kMH];
  mlp_layer(W1, b1, kMH, kMIn, x, h1, true);
  mlp_layer(W2, b2, kMH, kMH, h1, h2, true);
  mlp_layer(W3, b3, kMOut, kMH, h2, y, false);
}

static double gravity_norm(const Sim& s) {
  const double* g = s.prm.gravity;
  const double gn = std::sqrt((g[0] * g[0] + g[1] * g[1]) + g[2] * g[2]);
  return gn > 1e-12 ? gn : 1e-12;
}

/* Features of every obstacle contact (definitions in mlp.cu's header). */
static void mlp_features(Sim& s) {
  const int C = (int)s.contacts.size();
  const double g = gravity_norm(s);
  const double sv = g * s.prm.time_step;
  const V3 gv{s.prm.gravity[0], s.prm.gravity[1], s.prm.gravity[2]};
  s.feat.assign((size_t)C * kMIn, 0.f);
  for (int k = 0; k < C; ++k) {
    const CInfo& ci = s.contacts[k];
    const Basis& B = s.cbasis[k];
    const int v = ci.vertex;
    const V3 d = ld(s.tn.data(), v) - ci.speed;
    float* x = &s.feat[(size_t)k * kMIn];
    x[0] = (float)(dot(B.c0, d) / sv);
    x[1] = (float)(dot(B.c1, d) / sv);
    x[2] = (float)(dot(B.c2, d) / sv);
    x[3] = (float)(ci.gap / 1e-2);
    const double sr = s.mass[v] * sv;
    if (s.rprev_tag[v] == s.mlp_tag - 1) {
      const V3 R = ld(s.rprev.data(), v);
      x[4] = (float)(dot(B.c0, R) / sr);
      x[5] = (float)(dot(B.c1, R) / sr);
      x[6] = (float)(dot(B.c2, R) / sr);
    }
    x[7] = (float)ci.mu;
    x[8] = (float)(dot(B.c0, gv) / g);
    x[9] = 1.f;
  }
}

/* End of step: impulse memory and optional sample log (contact order). */
static void mlp_record(Sim& s) {
  const int C = (int)s.contacts.size();
  const double sv = gravity_norm(s) * s.prm.time_step;
  for (int k = 0; k < C; ++k) {
    const int v = s.contacts[k].vertex;
    st(s.rprev.data(), v, {0, 0, 0});
    s.rprev_tag[v] = s.mlp_tag;
  }
  const int base = s.log_n;
  for (int k = 0; k < C; ++k) {
    const int v = s.contacts[k].vertex;
    const bool active = s.c_active[k] != 0;
    const V3 r = active ? s.c_local_forces[k] : V3{0, 0, 0};
    if (active) {
      const V3 g = bv(s.cbasis[k], r);
      for (int c = 0; c < 3; ++c) s.rprev[3 * (size_t)v + c] += comp(g, c);
    }
    if (s.log_cap > 0 && (int64_t)base + k < s.log_cap) {
      const size_t o = (size_t)base + k;
      for (int d = 0; d < kMIn; ++d) s.log_X[o * kMIn + d] = s.feat[(size_t)k * kMIn + d];
      const double sr = s.mass[v] * sv;
      s.log_T[o * kMOut] = (float)(r.x / sr);
      s.log_T[o * kMOut + 1] = (float)(r.y / sr);
      s.log_T[o * kMOut + 2] = (float)(r.z / sr);
    }
  }
  if (s.log_cap > 0) s.log_n = (int)std::min<int64_t>((int64_t)s.log_n + C, s.log_cap);
}

/* One SimulationBase::step(), SimulationBase.cpp:103-173, with the
 * SimulationSpeed / SimulationFrictionEstimation overrides. */
static void step(Sim& s) {
  const int N = s.N;
  const double dt = s.prm.time_step;
  const bool self = s.prm.self_collision != 0;
  /* initializeStep SimulationSpeed.cpp:62-76; external force SimulationBase.cpp:266-287
   * (gravity functor m g, simulation_building.cpp:86-92); t_n :294-301 */
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) {
      const int64_t d = 3 * (int64_t)i + c;
      double f = s.mass[i] * s.prm.gravity[c];
      s.tn[d] = s.v[d] + dt * ((1. / s.mass[i]) * f);
      s.vnext[d] = s.tn[d];
      s.qnext[d] = s.q[d] + dt * s.vnext[d];
    }
  /* baseUpdateColisions SimulationBase.cpp:333-413 */
  detect_obstacles(s);
  const double damp = std::max(s.prm.air_damping, 0.);
  std::fill(s.damping.begin(), s.damping.end(), damp);
  if (damp > 0.)
    for (auto& c : s.contacts) s.damping[c.vertex] = 0.;
  s.selfc.clear();
  if (self) {
    double tol2 = s.prm.self_collision_tolerance * s.prm.self_collision_tolerance;
    double tol = std::sqrt(tol2);
    for (size_t m = 0; m < s.meshes.size(); ++m) {
      const auto& md = s.meshes[m];
      std::vector<V3> verts(md.n_vertices);
      for (int i = 0; i < md.n_vertices; ++i) verts[i] = ld(s.q.data(), md.vertex_offset + i);
      std::vector<std::array<int, 3>> tl(md.n_triangles);
      for (int t = 0; t < md.n_triangles; ++t)
        for (int k = 0; k < 3; ++k) tl[t][k] = s.tris[md.triangle_offset + t][k] - md.vertex_offset;
      std::vector<std::vector<int>> rings(md.n_vertices);
      for (int i = 0; i < md.n_vertices; ++i) {
        for (int r : s.topo.nbrs[md.vertex_offset + i]) rings[i].push_back(r - md.vertex_offset);
      }
      auto res = self_collisions(verts, tl, rings, tol);
      double mu = s.friction[(size_t)md.material * s.n_mat + md.material];
      for (auto& r : res) {
        r.vertex += md.vertex_offset;
        for (int k = 0; k < 3; ++k) r.face[k] += md.vertex_offset;
        r.mu = mu;
        s.selfc.push_back(r);
      }
    }
    if (damp > 0.)
      for (auto& c : s.selfc) {
        s.damping[c.vertex] = 0.;
        s.damping[s.partner(c)] = 0.;
      }
  }
  /* SFE::updateCollision SFE:107-152 */
  s.cbasis.resize(s.contacts.size());
  for (size_t c = 0; c < s.contacts.size(); ++c) s.cbasis[c] = compute_basis(s.contacts[c].normal);
  s.sbasis.resize(s.selfc.size());
  for (size_t c = 0; c < s.selfc.size(); ++c) s.sbasis[c] = compute_basis(s.selfc[c].normal);
  s.remember.assign(s.selfc.size(), {0, 0, 0});
  s.levels.clear();
  if (self && !s.selfc.empty()) compute_order(s);

  const int C = (int)s.contacts.size(), S = (int)s.selfc.size();
  const bool warm = s.prm.warm_start == PDF_WARM_MLP;
  const bool mlp_on = warm || s.log_cap > 0;
  if (warm && !s.mlp_ready) throw std::invalid_argument("PDF_WARM_MLP needs weights");
  if (mlp_on) {
    mlp_features(s);
    if (warm) {
      s.pred.assign((size_t)C * kMOut, 0.f);
      for (int k = 0; k < C; ++k) mlp_forward_one(s.mlp_w.data(), &s.feat[(size_t)k * kMIn], &s.pred[(size_t)k * kMOut]);
    }
  }
  if ((int)s.c_active.size() < C) s.c_active.resize(C, 0);
  const double pred_sv = gravity_norm(s) * dt;
  s.residual_hist.clear();
  s.residual_applied_hist.clear();
  s.s_active.assign(S, 0);
  s.ac_trace.clear();
  s.trace_nc = C;
  s.trace_ns = S;
  int it = 0;
  double res_mean = 0, res_max = 0, res_n = 0, res_t = 0;
  for (; it < s.prm.local_global_iterations; ++it) {
    /* SFE::computeRhs SFE:307-588 */
    rhs_base(s, s.q.data(), s.tn.data(), s.vnext.data(), s.qnext.data(), s.rhs.data());
    /* SFE:334-335 resize: slots keep whatever an earlier step left there
     * (storage only ever grows; never-used slots hold zero). */
    if ((int)s.c_local_forces.size() < C) s.c_local_forces.resize(C, {0, 0, 0});
    if ((int)s.s_local_forces.size() < S) s.s_local_forces.resize(S, {0, 0, 0});
    if (!((C == 0) && (!self || S == 0))) {
      /* forces = rhs - dt^2 A^T A v  (SFE:337-347) */
      std::vector<double> atav(3 * (size_t)N);
      spmv3(s.ATA, s.vnext.data(), atav.data());
      const double dt2 = std::pow(dt, 2);
      for (int64_t d = 0; d < 3 * (int64_t)N; ++d) s.forces[d] = s.rhs[d] - dt2 * atav[d];
      /* obstacle contacts SFE:350-423 */
      for (int c = 0; c < C; ++c) {
        const CInfo& ci = s.contacts[c];
        const int vid = ci.vertex;
        const Basis& B = s.cbasis[c];
        const double mu = ci.mu;
        V3 r;
        bool predicted = false;
        if (warm && it == 0) {
          /* first iteration under the learned warm start: the predicted force,
           * projected on the cone; non-finite -> the projection below */
          const double sr = s.mass[vid] * pred_sv;
          r = {sr * (double)s.pred[3 * (size_t)c], sr * (double)s.pred[3 * (size_t)c + 1],
               sr * (double)s.pred[3 * (size_t)c + 2]};
          if (std::isfinite(r.x) && std::isfinite(r.y) && std::isfinite(r.z)) {
            predicted = true;
            if (!(r.x > 0.)) {
              s.c_local_forces[c] = {0, 0, 0};
              s.c_active[c] = 0;
              continue;
            }
            const double rtn = std::sqrt(r.y * r.y + r.z * r.z);
            if (rtn > mu * r.x) {
              r.y *= mu * r.x / rtn;
              r.z *= mu * r.x / rtn;
            }
          }
        }
        if (!predicted) {
          V3 f = ld(s.forces.data(), vid);
          if (self) f = f + ld(s.self_forces[s.cur].data(), vid);
          V3 fl = btv(B, f - s.mass[vid] * ci.speed);
          if (fl.x > 0.) {
            s.c_active[c] = 0;
            continue;
          }
          r = {-fl.x, -fl.y, -fl.z};
          const double rtn = std::sqrt(r.y * r.y + r.z * r.z);
          if (rtn > mu * r.x) {
            r.y *= mu * r.x / rtn;
            r.z *= mu * r.x / rtn;
          }
        }
        s.c_active[c] = 1;
        s.c_local_forces[c] = r;
        V3 g = bv(B, r);
        if (!self || S == 0) {
          s.rhs[3 * (int64_t)vid] += g.x;
          s.rhs[3 * (int64_t)vid + 1] += g.y;
          s.rhs[3 * (int64_t)vid + 2] += g.z;
        }
        if (self) st(s.contact_forces[s.nxt].data(), vid, g);
      }
      if (self && S > 0) {
        /* self-contact levels SFE:431-576 */
        for (const auto& lvl : s.levels) {
          struct Add {
            int plus, minus;
            V3 f;
          };
          std::vector<Add> adds(lvl.size());
          for (size_t i = 0; i < lvl.size(); ++i) {
            const int sc = lvl[i];
            const SelfInfo& si = s.selfc[sc];
            const int vid = si.vertex;
            const Basis& B = s.sbasis[sc];
            const double mu = si.mu;
            const double mA = s.mass[vid];
            const int idB = s.partner(si);
            const double mB = s.mass[idB];
            V3 fA = ld(s.forces.data(), vid) + ld(s.contact_forces[s.nxt].data(), vid) +
                    ld(s.self_forces[s.cur].data(), vid) + ld(s.self_forces[s.nxt].data(), vid) -
                    s.remember[sc];
            V3 fB = ld(s.forces.data(), idB) + ld(s.contact_forces[s.nxt].data(), idB) +
                    ld(s.self_forces[s.cur].data(), idB) + ld(s.self_forces[s.nxt].data(), idB) +
                    s.remember[sc];
            V3 fl = btv(B, (1. / mA) * fA - (1. / mB) * fB);
            if (fl.x > 0.) {
              adds[i] = {vid, idB, {0, 0, 0}};
              s.s_active[sc] = 0;
              continue;
            }
            V3 r = -fl;
            const double rtn = std::sqrt(r.y * r.y + r.z * r.z);
            if (rtn > mu * r.x) {
              r.y *= mu * r.x / rtn;
              r.z *= mu * r.x / rtn;
            }
            r = ((mA * mB) / (mA + mB)) * r;
            s.s_local_forces[sc] = r;
            s.s_active[sc] = 1;
            adds[i] = {vid, idB, bv(B, r)};
          }
          for (size_t i = 0; i < lvl.size(); ++i) {
            const int sc = lvl[i];
            const V3 prev = s.remember[sc];
            const Add& a = adds[i];
            double* cu = s.self_forces[s.cur].data();
            double* nx = s.self_forces[s.nxt].data();
            for (int c = 0; c < 3; ++c) {
              cu[3 * (int64_t)a.plus + c] -= comp(prev, c);
              cu[3 * (int64_t)a.minus + c] += comp(prev, c);
              nx[3 * (int64_t)a.plus + c] += comp(a.f, c);
              nx[3 * (int64_t)a.minus + c] -= comp(a.f, c);
            }
            s.remember[sc] = a.f;
          }
        }
        for (int64_t d = 0; d < 3 * (int64_t)N; ++d)
          s.rhs[d] += s.contact_forces[s.nxt][d] + s.self_forces[s.nxt][d];
      }
      if (self) {
        s.cur = s.nxt;
        s.nxt = s.nxt ? 0 : 1;
        std::fill(s.contact_forces[s.nxt].begin(), s.contact_forces[s.nxt].end(), 0.);
        std::fill(s.self_forces[s.nxt].begin(), s.self_forces[s.nxt].end(), 0.);
      }
    }
    s.last_rhs = s.rhs;
    /* SimulationSpeed::solve :171-187 (one thread per component, like the
     * reference's omp loop over x/y/z) */
#pragma omp parallel for num_threads(3)
    for (int c = 0; c < 3; ++c) {
      std::vector<double> b(N), scratch;
      for (int i = 0; i < N; ++i) b[i] = s.rhs[3 * (int64_t)i + c];
      s.chol.solve(b.data(), scratch);
      for (int i = 0; i < N; ++i) s.vnext[3 * (int64_t)i + c] = b[i];
    }
    for (int64_t d = 0; d < 3 * (int64_t)N; ++d) s.qnext[d] = s.q[d] + dt * s.vnext[d];
    /* updateIterationData SFE:720-753 -> AC norms SFE:590-652 */
    s.c_ac.assign(C, 0.);
    s.s_ac.assign(S, 0.);
    double sum = 0, mxv = 0, sn = 0, stt = 0, sum_app = 0;
    for (int c = 0; c < C; ++c) {
      const CInfo& ci = s.contacts[c];
      V3 u = btv(s.cbasis[c], ld(s.vnext.data(), ci.vertex) - ci.speed);
      double an, at;
      auto acv = alart_curnier(u, s.c_local_forces[c], ci.mu, &an, &at);
      double n3 = std::sqrt(acv[0] * acv[0] + acv[1] * acv[1] + acv[2] * acv[2]);
      s.c_ac[c] = n3;
      sum += n3;
      {
        const V3 ra = s.c_active[c] ? s.c_local_forces[c] : V3{0, 0, 0};
        double an2, at2;
        auto ap = alart_curnier(u, ra, ci.mu, &an2, &at2);
        sum_app += std::sqrt(ap[0] * ap[0] + ap[1] * ap[1] + ap[2] * ap[2]);
      }
      mxv = std::max(mxv, n3);
      sn += an;
      stt += at;
      if (s.trace_ac) {
        s.ac_trace.push_back(at);
        s.ac_trace.push_back(an);
      }
    }
    for (int c = 0; c < S; ++c) {
      const SelfInfo& si = s.selfc[c];
      V3 u = btv(s.sbasis[c], ld(s.vnext.data(), si.vertex) - ld(s.vnext.data(), s.partner(si)));
      double an, at;
      auto acv = alart_curnier(u, s.s_local_forces[c], si.mu, &an, &at);
      double n3 = std::sqrt(acv[0] * acv[0] + acv[1] * acv[1] + acv[2] * acv[2]);
      s.s_ac[c] = n3;
      sum += n3;
      {
        const V3 ra = s.s_active[c] ? s.s_local_forces[c] : V3{0, 0, 0};
        double an2, at2;
        auto ap = alart_curnier(u, ra, si.mu, &an2, &at2);
        sum_app += std::sqrt(ap[0] * ap[0] + ap[1] * ap[1] + ap[2] * ap[2]);
      }
      mxv = std::max(mxv, n3);
      sn += an;
      stt += at;
      if (s.trace_ac) {
        s.ac_trace.push_back(at);
        s.ac_trace.push_back(an);
      }
    }
    const int nc = C + S;
    res_mean = nc ? sum / nc : 0.;
    res_max = mxv;
    res_n = nc ? sn / nc : 0.;
    res_t = nc ? stt / nc : 0.;
    s.residual_hist.push_back(res_mean);
    s.residual_applied_hist.push_back(nc ? sum_app / nc : 0.);
    if (s.prm.residual_tolerance > 0. && nc > 0 && res_mean <= s.prm.residual_tolerance) {
      ++it;
      break;
    }
  }
  if (mlp_on) mlp_record(s);
  s.mlp_tag += 1;
  /* SFE::updateScene SFE:64-87 */
  s.q = s.qnext;
  s.v = s.vnext;
  for (auto& ob : s.obstacles) {
    if (ob.type == PDF_OBSTACLE_ROTATING_SPHERE) ob.time_before_start -= dt;
    if (ob.type == PDF_OBSTACLE_MOVING_MESH) {
      /* MovingMesh::update MovingMesh.cpp:43-84: advance the clock, at most
       * one key frame, then interpolate the current mesh while in movement */
      ob.clock += dt;
      if (ob.frame_time(ob.next) < ob.clock && ob.next + 1 < (int)ob.frames.size()) ob.next += 1;
      if (ob.in_movement()) {
        const double t0 = ob.frame_time(ob.next - 1), t1 = ob.frame_time(ob.next);
        const double a = (ob.clock - t0) / (t1 - t0);
        const std::vector<V3>& fp = ob.frames[ob.next - 1];
        const std::vector<V3>& fn = ob.frames[ob.next];
        for (size_t k = 0; k < ob.mverts.size(); ++k) ob.mverts[k] = fp[k] * (1 - a) + fn[k] * a;
      }
    }
  }
  if (self) {
    s.cur = 0;
    s.nxt = 1;
    for (int i = 0; i < 2; ++i) {
      std::fill(s.contact_forces[i].begin(), s.contact_forces[i].end(), 0.);
      std::fill(s.self_forces[i].begin(), s.self_forces[i].end(), 0.);
    }
  }
  s.time += dt;
  s.last.n_contacts = C;
  s.last.n_self_contacts = S;
  s.last.n_levels = (int)s.levels.size();
  s.last.iterations = it;
  s.last.residual = res_mean;
  s.last.residual_max = res_max;
  s.last.normal_residual = res_n;
  s.last.tangential_residual = res_t;
  s.last.time = s.time;
}

static void build(Sim& s, const pdf_scene_desc* sc, const pdf_params* p) {
  if (!sc || !p || sc->n_vertices <= 0 || !sc->rest_positions || sc->n_meshes <= 0 || !sc->meshes)
    throw std::invalid_argument("invalid scene description");
  if (!(p->time_step > 0.)) throw std::invalid_argument("time step must be positive");
  s.prm = *p;
  const int N = sc->n_vertices;
  s.N = N;
  s.rest.resize(N);
  for (int i = 0; i < N; ++i) s.rest[i] = ld(sc->rest_positions, i);
  s.q.assign(sc->rest_positions, sc->rest_positions + 3 * (size_t)N);
  if (sc->positions) s.q.assign(sc->positions, sc->positions + 3 * (size_t)N);
  s.v.assign(3 * (size_t)N, 0.);
  s.rprev.assign(3 * (size_t)N, 0.);
  s.rprev_tag.assign(N, -0x40000000);
  if (sc->velocities) s.v.assign(sc->velocities, sc->velocities + 3 * (size_t)N);
  for (double x : s.q)
    if (!std::isfinite(x)) throw std::invalid_argument("non-finite position");
  s.tris.resize(sc->n_triangles);
  for (int t = 0; t < sc->n_triangles; ++t)
    for (int k = 0; k < 3; ++k) {
      int ix = sc->triangles[3 * (size_t)t + k];
      if (ix < 0 || ix >= N) throw std::invalid_argument("triangle index out of range");
      s.tris[t][k] = ix;
    }
  s.meshes.assign(sc->meshes, sc->meshes + sc->n_meshes);
  s.vmesh.assign(N, 0);
  s.n_mat = sc->n_materials;
  s.friction.assign(sc->friction, sc->friction + (size_t)s.n_mat * s.n_mat);
  s.topo.ring.assign(N, {});
  s.topo.nbrs.assign(N, {});
  s.topo.border.assign(N, 0);
  s.topo.vfaces.assign(N, {});
  s.mass.assign(N, 0.);
  /* per mesh: topology, masses (PhysicMesh::initializeMasses PhysicMesh.cpp:115-151),
   * constraints (PhysicMesh::initializeConstraints :70-113) */
  for (int m = 0; m < sc->n_meshes; ++m) {
    const pdf_mesh_desc& md = sc->meshes[m];
    if (md.material < 0 || md.material >= s.n_mat) throw std::invalid_argument("mesh material out of range");
    for (int i = md.vertex_offset; i < md.vertex_offset + md.n_vertices; ++i) s.vmesh[i] = m;
    size_t e0 = s.topo.edges.size();
    build_topology(N, s.tris, md.vertex_offset, md.vertex_offset + md.n_vertices, md.triangle_offset,
                   md.triangle_offset + md.n_triangles, s.topo);
    for (int i = md.vertex_offset; i < md.vertex_offset + md.n_vertices; ++i) {
      double acc = 0.;
      for (int f : s.topo.vfaces[i]) {
        /* Mesh::getTriangleArea Mesh.cpp:112-118: sqrt(CGAL::squared_area) */
        V3 a = s.rest[s.tris[f][0]], b = s.rest[s.tris[f][1]], c = s.rest[s.tris[f][2]];
        V3 cr = cross(b - a, c - a);
        double area = std::sqrt(sqn(cr) / 4);
        acc += md.area_density * area;
      }
      s.mass[i] = acc / 3;
    }
    /* springs (SpringConstraint ctor + addConstraintMatrix SpringConstraint.cpp:30-54) */
    for (size_t e = e0; e < s.topo.edges.size(); ++e) {
      int a = s.topo.edges[e][0], b = s.topo.edges[e][1];
      Sim::Spring sp{a, b, std::sqrt(md.stretching), nrm(s.rest[a] - s.rest[b])};
      s.rows.push_back({0, (int)s.springs.size()});
      s.springs.push_back(sp);
    }
    /* bending (BendingConstraint ctor BendingConstraint.cpp:47-83) */
    for (int i = md.vertex_offset; i < md.vertex_offset + md.n_vertices; ++i) {
      if (s.topo.border[i]) continue;
      const auto& ring = s.topo.ring[i];
      std::vector<V3> rp;
      for (int r : ring) rp.push_back(s.rest[r]);
      auto co = mean_value_coeffs(s.rest[i], rp);
      Sim::Bend b;
      b.idx.push_back(i);
      b.idx.insert(b.idx.end(), ring.begin(), ring.end());
      b.coef.push_back(0.);
      for (double c : co) {
        b.coef[0] += c;
        b.coef.push_back(-c);
      }
      b.w = std::sqrt(md.bending);
      V3 lb{0, 0, 0};
      for (size_t k = 0; k < b.idx.size(); ++k) lb = lb + b.coef[k] * s.rest[b.idx[k]];
      b.rest_norm = nrm(lb);
      s.rows.push_back({1, (int)s.bends.size()});
      s.bends.push_back(b);
    }
  }
  for (int k = 0; k < sc->n_pins; ++k) {
    Sim::Pin pn{sc->pin_vertices[k], std::sqrt(sc->pin_weights[k]), ld(sc->pin_positions, k)};
    if (pn.i < 0 || pn.i >= N) throw std::invalid_argument("pin vertex out of range");
    s.rows.push_back({2, (int)s.pins.size()});
    s.pins.push_back(pn);
  }
  for (int i = 0; i < N; ++i)
    if (!(s.mass[i] > 0.)) throw std::invalid_argument("vertex with zero mass (not on any triangle)");
  /* A^T (CSR over vertices) — SimulationBase.cpp:71-78 */
  const int64_t R = (int64_t)s.rows.size();
  std::vector<std::vector<std::pair<int, double>>> at(N);
  for (int64_t r = 0; r < R; ++r) {
    int kind = s.rows[r].first, id = s.rows[r].second;
    if (kind == 0) {
      at[s.springs[id].i].push_back({(int)r, s.springs[id].w});
      at[s.springs[id].j].push_back({(int)r, -s.springs[id].w});
      s.nnzA += 2;
    } else if (kind == 1) {
      const auto& b = s.bends[id];
      for (size_t k = 0; k < b.idx.size(); ++k) at[b.idx[k]].push_back({(int)r, b.w * b.coef[k]});
      s.nnzA += (int64_t)b.idx.size();
    } else {
      at[s.pins[id].i].push_back({(int)r, s.pins[id].w});
      s.nnzA += 1;
    }
  }
  s.At.n = N;
  s.At.m = (int)R;
  s.At.ptr.assign(N + 1, 0);
  for (int i = 0; i < N; ++i) {
    std::sort(at[i].begin(), at[i].end());
    s.At.ptr[i + 1] = s.At.ptr[i] + (int64_t)at[i].size();
  }
  for (int i = 0; i < N; ++i)
    for (auto& e : at[i]) {
      s.At.col.push_back(e.first);
      s.At.val.push_back(e.second);
    }
  /* A rows (for A^T A) */
  std::vector<std::vector<std::pair<int, double>>> arow(R);
  for (int i = 0; i < N; ++i)
    for (auto& e : at[i]) arow[e.first].push_back({i, e.second});
  /* A^T A and LHS = M + dt^2 A^T A (SimulationSpeed::computeLhs :230-236) */
  s.ATA.n = N;
  s.ATA.m = N;
  s.ATA.ptr.assign(N + 1, 0);
  {
    std::vector<double> acc(N, 0.);
    std::vector<int> mark(N, -1), list;
    for (int i = 0; i < N; ++i) {
      list.clear();
      for (auto& e : at[i])
        for (auto& f : arow[e.first]) {
          if (mark[f.first] != i) {
            mark[f.first] = i;
            acc[f.first] = 0.;
            list.push_back(f.first);
          }
          acc[f.first] += e.second * f.second;
        }
      std::sort(list.begin(), list.end());
      for (int j : list) {
        s.ATA.col.push_back(j);
        s.ATA.val.push_back(acc[j]);
      }
      s.ATA.ptr[i + 1] = (int64_t)s.ATA.col.size();
    }
  }
  s.LHS = s.ATA;
  const double dt2 = std::pow(s.prm.time_step, 2);
  for (int i = 0; i < N; ++i)
    for (int64_t p2 = s.LHS.ptr[i]; p2 < s.LHS.ptr[i + 1]; ++p2) {
      s.LHS.val[p2] = dt2 * s.ATA.val[p2];
      if (s.LHS.col[p2] == i) s.LHS.val[p2] += s.mass[i];
    }
  /* one-time factorisation (SimulationSpeed.cpp:53) */
  if (!s.chol.factor(s.LHS, s.rest)) throw std::runtime_error("LHS is not positive definite");
  /* obstacles */
  for (int k = 0; k < sc->n_obstacles; ++k) {
    const pdf_obstacle& o = sc->obstacles[k];
    Obstacle ob;
    ob.type = o.type;
    ob.material = o.material;
    if (o.material < 0 || o.material >= s.n_mat) throw std::invalid_argument("obstacle material out of range");
    ob.center = {o.center[0], o.center[1], o.center[2]};
    ob.radius = o.radius;
    V3 ax{o.axis[0], o.axis[1], o.axis[2]};
    ob.rot = o.angular_speed * normalized(ax);
    ob.time_before_start = o.rotation_start_time;
    ob.point = {o.point[0], o.point[1], o.point[2]};
    ob.normal = normalized(V3{o.normal[0], o.normal[1], o.normal[2]});
    ob.threshold = o.threshold;
    ob.mesh = o.mesh;
    ob.size = {o.size[0], o.size[1], o.size[2]};
    if (ob.mesh >= sc->n_meshes) throw std::invalid_argument("obstacle mesh out of range");
    if (o.type == PDF_OBSTACLE_MESH || o.type == PDF_OBSTACLE_MOVING_MESH) {
      if (o.n_vertices <= 0 || o.n_triangles <= 0 || !o.vertices || !o.triangles)
        throw std::invalid_argument("mesh obstacle without geometry");
      for (int i = 0; i < o.n_vertices; ++i) ob.mverts.push_back(ld(o.vertices, i));
      for (int t = 0; t < o.n_triangles; ++t) {
        ob.mtris.push_back({o.triangles[3 * t], o.triangles[3 * t + 1], o.triangles[3 * t + 2]});
        for (int c = 0; c < 3; ++c)
          if (o.triangles[3 * t + c] < 0 || o.triangles[3 * t + c] >= o.n_vertices)
            throw std::invalid_argument("mesh obstacle index out of range");
      }
      if (o.type == PDF_OBSTACLE_MOVING_MESH) {
        if (o.n_frames < 2 || !(o.frame_interval > 0.))
          throw std::invalid_argument("moving mesh needs at least two key frames and a positive interval");
        ob.interval = o.frame_interval;
        for (int f = 0; f < o.n_frames; ++f) {
          std::vector<V3> fr;
          for (int i = 0; i < o.n_vertices; ++i) fr.push_back(ld(o.vertices, (size_t)f * o.n_vertices + i));
          ob.frames.push_back(std::move(fr));
        }
      }
    } else if (o.type < 0 || o.type > 5) {
      throw std::invalid_argument("unknown obstacle type");
    }
    s.obstacles.push_back(ob);
  }
  s.tn.assign(3 * (size_t)N, 0.);
  s.vnext.assign(3 * (size_t)N, 0.);
  s.qnext = s.q;
  s.damping.assign(N, 0.);
  s.rhs.assign(3 * (size_t)N, 0.);
  s.forces.assign(3 * (size_t)N, 0.);
  s.proj.assign(3 * (size_t)R, 0.);
  for (int i = 0; i < 2; ++i) {
    s.contact_forces[i].assign(3 * (size_t)N, 0.);
    s.self_forces[i].assign(3 * (size_t)N, 0.);
  }
}

static void fill_contact(pdf_contact& o, int vertex, int partner, const int* face, V3 n, V3 sp,
                         double mu, V3 f, double ac) {
  o.vertex = vertex;
  o.partner = partner;
  for (int k = 0; k < 3; ++k) o.face[k] = face ? face[k] : -1;
  o.normal[0] = n.x;
  o.normal[1] = n.y;
  o.normal[2] = n.z;
  o.speed[0] = sp.x;
  o.speed[1] = sp.y;
  o.speed[2] = sp.z;
  o.mu = mu;
  o.force[0] = f.x;
  o.force[1] = f.y;
  o.force[2] = f.z;
  o.ac = ac;
}

}  // namespace orc

using namespace orc;

struct orc_sim {
  Sim s;
};

extern "C" {

const char* orc_last_error(void) { return g_error.c_str(); }

int orc_create(const pdf_scene_desc* scene, const pdf_params* params, orc_sim** out) {
  if (!out) return PDF_INVALID_ARG;
  *out = nullptr;
  orc_sim* h = new orc_sim();
  try {
    build(h->s, scene, params);
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    delete h;
    return PDF_INVALID_ARG;
  } catch (const std::exception& e) {
    g_error = e.what();
    delete h;
    return PDF_NOT_SPD;
  }
  *out = h;
  return PDF_OK;
}

int orc_step(orc_sim* h, int32_t nsteps, pdf_step_report* report) {
  if (!h || nsteps < 0) return PDF_INVALID_ARG;
  try {
    for (int i = 0; i < nsteps; ++i) step(h->s);
  } catch (const std::exception& e) {
    g_error = e.what();
    return PDF_INVALID_ARG;
  }
  if (report) *report = h->s.last;
  return PDF_OK;
}

int orc_mlp_set_weights(orc_sim* h, const float* w, int32_t count) {
  if (!h || !w || count != kMParams) return PDF_INVALID_ARG;
  h->s.mlp_w.assign(w, w + kMParams);
  h->s.mlp_ready = true;
  return PDF_OK;
}

int orc_mlp_log(orc_sim* h, int32_t capacity) {
  if (!h || capacity < 0) return PDF_INVALID_ARG;
  h->s.log_cap = capacity;
  h->s.log_n = 0;
  h->s.log_X.assign((size_t)capacity * kMIn, 0.f);
  h->s.log_T.assign((size_t)capacity * kMOut, 0.f);
  return PDF_OK;
}

int orc_mlp_samples(orc_sim* h, float* X, float* T, int32_t cap, int32_t* n) {
  if (!h || !n) return PDF_INVALID_ARG;
  *n = h->s.log_n;
  const int m = std::min(h->s.log_n, cap);
  if (X) std::memcpy(X, h->s.log_X.data(), sizeof(float) * (size_t)m * kMIn);
  if (T) std::memcpy(T, h->s.log_T.data(), sizeof(float) * (size_t)m * kMOut);
  return PDF_OK;
}

int orc_mlp_forward(const float* w, const float* X, int32_t n, float* Y) {
  if (!w || n < 0 || (n > 0 && (!X || !Y))) return PDF_INVALID_ARG;
  for (int i = 0; i < n; ++i) mlp_forward_one(w, X + (size_t)i * kMIn, Y + (size_t)i * kMOut);
  return PDF_OK;
}

int orc_get_state(orc_sim* h, double* q, double* v) {
  if (!h) return PDF_INVALID_ARG;
  if (q) std::memcpy(q, h->s.q.data(), sizeof(double) * h->s.q.size());
  if (v) std::memcpy(v, h->s.v.data(), sizeof(double) * h->s.v.size());
  return PDF_OK;
}

int orc_set_state(orc_sim* h, const double* q, const double* v) {
  if (!h) return PDF_INVALID_ARG;
  if (q) std::memcpy(h->s.q.data(), q, sizeof(double) * h->s.q.size());
  if (v) std::memcpy(h->s.v.data(), v, sizeof(double) * h->s.v.size());
  h->s.mlp_tag += 2; /* the previous step's contact impulses no longer apply */
  return PDF_OK;
}

int orc_get_contacts(orc_sim* h, pdf_contact* out, int32_t cap, int32_t* n) {
  if (!h) return PDF_INVALID_ARG;
  Sim& s = h->s;
  const int C = (int)s.contacts.size();
  if (n) *n = C;
  if (!out) return PDF_OK;
  for (int c = 0; c < C && c < cap; ++c) {
    const CInfo& ci = s.contacts[c];
    fill_contact(out[c], ci.vertex, -1, nullptr, ci.normal, ci.speed, ci.mu,
                 c < (int)s.c_local_forces.size() ? s.c_local_forces[c] : V3{0, 0, 0},
                 c < (int)s.c_ac.size() ? s.c_ac[c] : 0.);
  }
  return C > cap ? PDF_CAPACITY_EXCEEDED : PDF_OK;
}

int orc_get_self_contacts(orc_sim* h, pdf_contact* out, int32_t cap, int32_t* n) {
  if (!h) return PDF_INVALID_ARG;
  Sim& s = h->s;
  const int S = (int)s.selfc.size();
  if (n) *n = S;
  if (!out) return PDF_OK;
  for (int c = 0; c < S && c < cap; ++c) {
    const SelfInfo& si = s.selfc[c];
    fill_contact(out[c], si.vertex, s.partner(si), si.face, si.normal, {0, 0, 0}, si.mu,
                 c < (int)s.s_local_forces.size() ? s.s_local_forces[c] : V3{0, 0, 0},
                 c < (int)s.s_ac.size() ? s.s_ac[c] : 0.);
  }
  return S > cap ? PDF_CAPACITY_EXCEEDED : PDF_OK;
}

int orc_get_self_levels(orc_sim* h, int32_t* level_ptr, int32_t level_cap, int32_t* order,
                        int32_t order_cap, int32_t* n_levels) {
  if (!h) return PDF_INVALID_ARG;
  Sim& s = h->s;
  if (n_levels) *n_levels = (int)s.levels.size();
  if (!level_ptr || !order) return PDF_OK;
  int pos = 0;
  for (size_t l = 0; l < s.levels.size(); ++l) {
    if ((int)l < level_cap) level_ptr[l] = pos;
    for (int c : s.levels[l]) {
      if (pos < order_cap) order[pos] = c;
      ++pos;
    }
  }
  if ((int)s.levels.size() < level_cap) level_ptr[s.levels.size()] = pos;
  return PDF_OK;
}

int orc_get_residual_history(orc_sim* h, double* out, int32_t cap, int32_t* n) {
  if (!h) return PDF_INVALID_ARG;
  const auto& r = h->s.residual_hist;
  if (n) *n = (int)r.size();
  if (out)
    for (int i = 0; i < (int)r.size() && i < cap; ++i) out[i] = r[i];
  return PDF_OK;
}

int orc_get_residual_applied_history(orc_sim* h, double* out, int32_t cap, int32_t* n) {
  if (!h) return PDF_INVALID_ARG;
  const auto& r = h->s.residual_applied_hist;
  if (n) *n = (int)r.size();
  if (out)
    for (int i = 0; i < (int)r.size() && i < cap; ++i) out[i] = r[i];
  return PDF_OK;
}

int orc_trace_alart_curnier(orc_sim* h, int32_t enable) {
  if (!h) return PDF_INVALID_ARG;
  h->s.trace_ac = enable != 0;
  h->s.ac_trace.clear();
  return PDF_OK;
}

int orc_get_alart_curnier_trace(orc_sim* h, double* out, int64_t cap, int32_t* iterations,
                                int32_t* n_contacts, int32_t* n_self) {
  if (!h) return PDF_INVALID_ARG;
  const Sim& s = h->s;
  const int64_t per = 2 * (int64_t)(s.trace_nc + s.trace_ns);
  if (iterations) *iterations = per ? (int32_t)((int64_t)s.ac_trace.size() / per) : 0;
  if (n_contacts) *n_contacts = s.trace_nc;
  if (n_self) *n_self = s.trace_ns;
  if (out)
    for (int64_t i = 0; i < (int64_t)s.ac_trace.size() && i < cap; ++i) out[i] = s.ac_trace[i];
  return PDF_OK;
}

int orc_get_sizes(orc_sim* h, int64_t* sz) {
  if (!h || !sz) return PDF_INVALID_ARG;
  sz[0] = (int64_t)h->s.rows.size();
  sz[1] = h->s.nnzA;
  sz[2] = (int64_t)h->s.LHS.col.size();
  sz[3] = h->s.chol.Lp.empty() ? 0 : h->s.chol.Lp.back();
  return PDF_OK;
}

int orc_projections(orc_sim* h, const double* q, double* p) {
  if (!h || !q || !p) return PDF_INVALID_ARG;
  projections(h->s, q, p);
  return PDF_OK;
}

int orc_rhs_base(orc_sim* h, const double* qn, const double* tn, const double* vk, double* rhs) {
  if (!h || !qn || !tn || !vk || !rhs) return PDF_INVALID_ARG;
  Sim& s = h->s;
  std::vector<double> qk(3 * (size_t)s.N);
  for (size_t d = 0; d < qk.size(); ++d) qk[d] = qn[d] + s.prm.time_step * vk[d];
  rhs_base(s, qn, tn, vk, qk.data(), rhs);
  return PDF_OK;
}

int orc_last_rhs(orc_sim* h, double* rhs) {
  if (!h || !rhs) return PDF_INVALID_ARG;
  if (h->s.last_rhs.empty()) return PDF_INVALID_ARG;
  std::memcpy(rhs, h->s.last_rhs.data(), sizeof(double) * h->s.last_rhs.size());
  return PDF_OK;
}

int orc_solve(orc_sim* h, double* x) {
  if (!h || !x) return PDF_INVALID_ARG;
  Sim& s = h->s;
  std::vector<double> b(s.N);
  for (int c = 0; c < 3; ++c) {
    for (int i = 0; i < s.N; ++i) b[i] = x[3 * (int64_t)i + c];
    s.chol.solve(b.data(), s.tmpx);
    for (int i = 0; i < s.N; ++i) x[3 * (int64_t)i + c] = b[i];
  }
  return PDF_OK;
}

int orc_lhs_csr(orc_sim* h, int32_t* row_ptr, int32_t* col, double* val, int64_t* nnz) {
  if (!h) return PDF_INVALID_ARG;
  const CSR& L = h->s.LHS;
  if (nnz) *nnz = (int64_t)L.col.size();
  if (row_ptr)
    for (int i = 0; i <= L.n; ++i) row_ptr[i] = (int32_t)L.ptr[i];
  if (col)
    for (size_t k = 0; k < L.col.size(); ++k) col[k] = L.col[k];
  if (val) std::memcpy(val, L.val.data(), sizeof(double) * L.val.size());
  return PDF_OK;
}

int orc_masses(orc_sim* h, double* m) {
  if (!h || !m) return PDF_INVALID_ARG;
  std::memcpy(m, h->s.mass.data(), sizeof(double) * h->s.mass.size());
  return PDF_OK;
}

double orc_time(orc_sim* h) { return h ? h->s.time : 0.; }

void orc_destroy(orc_sim* h) { delete h; }

int orc_self_candidates(const double* pos, int32_t nv, const int32_t* tris, int32_t nt, double tolerance,
                        int32_t* pairs, int32_t cap, int32_t* n) {
  if (!pos || nv < 0 || nt < 0 || (nt > 0 && !tris)) return PDF_INVALID_ARG;
  std::vector<V3> verts(nv);
  for (int i = 0; i < nv; ++i) verts[i] = ld(pos, i);
  std::vector<std::array<int, 3>> tl(nt);
  for (int t = 0; t < nt; ++t)
    for (int k = 0; k < 3; ++k) tl[t][k] = tris[3 * t + k];
  std::vector<std::vector<int>> cand;
  box_candidates(verts, tl, verts, 1.1 * tolerance, cand);
  int64_t total = 0;
  for (int v = 0; v < nv; ++v)
    for (int t : cand[v]) {
      if (pairs && total < cap) {
        pairs[2 * total] = v;
        pairs[2 * total + 1] = t;
      }
      ++total;
    }
  if (n) *n = (int32_t)total;
  return total > cap ? PDF_CAPACITY_EXCEEDED : PDF_OK;
}

int orc_self_collisions(const double* pos, int32_t nv, const int32_t* tris, int32_t nt, double tolerance,
                        pdf_contact* out, int32_t cap, int32_t* n) {
  if (!pos || nv < 0 || nt < 0 || (nt > 0 && !tris)) return PDF_INVALID_ARG;
  std::vector<V3> verts(nv);
  for (int i = 0; i < nv; ++i) verts[i] = ld(pos, i);
  std::vector<std::array<int, 3>> tl(nt);
  Topo tp;
  tp.ring.assign(nv, {});
  tp.nbrs.assign(nv, {});
  tp.border.assign(nv, 0);
  tp.vfaces.assign(nv, {});
  for (int t = 0; t < nt; ++t)
    for (int k = 0; k < 3; ++k) tl[t][k] = tris[3 * t + k];
  build_topology(nv, tl, 0, nv, 0, nt, tp);
  auto res = self_collisions(verts, tl, tp.nbrs, tolerance);
  if (n) *n = (int32_t)res.size();
  if (out)
    for (size_t i = 0; i < res.size() && (int)i < cap; ++i) {
      const SelfInfo& si = res[i];
      const V3& a = si.bary;
      int p = si.face[(a.x > a.y) ? ((a.x > a.z) ? 0 : 2) : ((a.y > a.z) ? 1 : 2)];
      fill_contact(out[i], si.vertex, p, si.face, si.normal, {0, 0, 0}, 0., {0, 0, 0}, 0.);
    }
  return (int)res.size() > cap ? PDF_CAPACITY_EXCEEDED : PDF_OK;
}

void orc_closest_point(const double* p, const double* a, const double* b, const double* c, double tol2,
                       double* cp, double* bary) {
  V3 o, w;
  closest_point(ld(p, 0), ld(a, 0), ld(b, 0), ld(c, 0), tol2, o, w);
  st(cp, 0, o);
  st(bary, 0, w);
}

}  // extern "C"
