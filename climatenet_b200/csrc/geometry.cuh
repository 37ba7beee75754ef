// geometry.cuh — exact FP64 proximity queries shared by obstacle and
// self-collision detection.  Include only from translation units compiled with
// --fmad=false: the operation order below follows the reference line by line
// and must round identically.
#pragma once
#include "device.cuh"

namespace pdfb {

// closestPointToTriangle (src/geometry/geometry_util.cpp:506-616): Ericson's
// region test with the reference's early exit `|ap|^2 - |ab|^2 - |ac|^2 > tol2`
// (callers pass the UNSQUARED tolerance there, as the reference does).
__device__ __forceinline__ void closest_point(double3 p, double3 a, double3 b, double3 c, double tol2, double3* cp,
                                              double3* bary) {
  const double3 ap = p - a, ab = b - a, ac = c - a;
  if (dot3(ap, ap) - dot3(ab, ab) - dot3(ac, ac) > tol2) {
    *cp = a;
    *bary = make_double3(1, 0, 0);
    return;
  }
  const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) {
    *cp = a;
    *bary = make_double3(1, 0, 0);
    return;
  }
  const double3 bp = p - b;
  const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) {
    *cp = b;
    *bary = make_double3(0, 1, 0);
    return;
  }
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
    const double v = d1 / (d1 - d3);
    *cp = a + v * ab;
    *bary = make_double3(1 - v, v, 0);
    return;
  }
  const double3 cpv = p - c;
  const double d5 = dot3(ab, cpv), d6 = dot3(ac, cpv);
  if (d6 >= 0.0 && d5 <= d6) {
    *cp = c;
    *bary = make_double3(0, 0, 1);
    return;
  }
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    const double w = d2 / (d2 - d6);
    *cp = a + w * ac;
    *bary = make_double3(1 - w, 0, w);
    return;
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
    const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    *cp = b + w * (c - b);
    *bary = make_double3(0, 1 - w, w);
    return;
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  // a + ab*v + ac*w evaluated left to right
  *cp = make_double3((a.x + ab.x * v) + ac.x * w, (a.y + ab.y * v) + ac.y * w, (a.z + ab.z * v) + ac.z * w);
  *bary = make_double3(1. - v - w, v, w);
}

// [a b c] * w : ((a_i w0 + b_i w1) + c_i w2)
__device__ __forceinline__ double3 tri_point(double3 a, double3 b, double3 c, double3 w) {
  return make_double3(a.x * w.x + b.x * w.y + c.x * w.z, a.y * w.x + b.y * w.y + c.y * w.z,
                      a.z * w.x + b.z * w.y + c.z * w.z);
}

// Closed-box overlap of a triangle's bounding box with [x - t, x + t]
// (CGAL box_intersection_d default closed topology; geometry_util.cpp:284-327).
__device__ __forceinline__ bool box_overlap(double3 x, double t, double3 lo, double3 hi) {
  return lo.x <= x.x + t && x.x - t <= hi.x && lo.y <= x.y + t && x.y - t <= hi.y && lo.z <= x.z + t &&
         x.z - t <= hi.z;
}

__device__ __forceinline__ void tri_box(double3 a, double3 b, double3 c, double3* lo, double3* hi) {
  *lo = make_double3(fmin(fmin(a.x, b.x), c.x), fmin(fmin(a.y, b.y), c.y), fmin(fmin(a.z, b.z), c.z));
  *hi = make_double3(fmax(fmax(a.x, b.x), c.x), fmax(fmax(a.y, b.y), c.y), fmax(fmax(a.z, b.z), c.z));
}

// StaticMesh detection (StaticMesh.cpp:33-48 -> checkMeshCollision, vector
// form, geometry_util.cpp:32-92): candidates with box half-width 1.1 tol,
// closest point, kept if |c - x|^2 < tol^2, closest kept triangle (first on
// ties, triangles ascending), contact if its distance^2 < tol^2.
__device__ __forceinline__ bool mesh_obstacle_closest(double3 x, const double* mv, const int* mt, int nt, double tol,
                                                      int* tri_out, double3* cp_out, double3* w_out = nullptr) {
  const double t = 1.1 * tol, tol_sq = tol * tol;
  double best = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  int bt = -1;
  double3 bp = make_double3(0., 0., 0.), bw = bp;
  for (int k = 0; k < nt; ++k) {
    const double3 a = ld3(mv, mt[3 * k]), b = ld3(mv, mt[3 * k + 1]), c = ld3(mv, mt[3 * k + 2]);
    double3 lo, hi;
    tri_box(a, b, c, &lo, &hi);
    if (!box_overlap(x, t, lo, hi)) continue;
    double3 cp, w;
    closest_point(x, a, b, c, tol, &cp, &w);
    const double3 dd = cp - x;
    if (!(dot3(dd, dd) < tol_sq)) continue;
    const double3 p = tri_point(a, b, c, w);
    const double3 e = p - x;
    const double d2 = dot3(e, e);
    if (d2 < best) {
      best = d2;
      bt = k;
      bp = p;
      bw = w;
    }
  }
  *tri_out = bt;
  *cp_out = bp;
  if (w_out) *w_out = bw;
  return best < tol_sq;
}

}  // namespace pdfb
