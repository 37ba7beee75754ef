// detect_kernels.cu — obstacle detection and contact bookkeeping.
// Compiled with --fmad=false so that every multiply and add rounds separately,
// exactly like the reference compiled for plain x86-64: detection decisions
// (inside / outside, closest-point region) must come out bit-identical.
#include <cuda_runtime.h>

#include <algorithm>
#include <cub/cub.cuh>
#include <stdexcept>
#include <string>

#include "device.cuh"
#include "geometry.cuh"
#include "kernels.hpp"
#include "lbvh.cuh"

namespace pdfb {

// Axis-aligned box (StaticAxisAlignedBox.cpp:41-135): coordinates relative to
// the box centre; a vertex is in contact when inside (no margin); the contact
// side is the first of TOP (+y), BOTTOM (-y), LEFT (-x), RIGHT (+x),
// FRONT (+z), BACK (-z) at the smallest distance.
__device__ __forceinline__ double3 box_relative(double3 x, const DObstacle& ob) {
  return make_double3((x.x - ob.c[0]) - 0.5 * ob.s[0], (x.y - ob.c[1]) - 0.5 * ob.s[1],
                      (x.z - ob.c[2]) - 0.5 * ob.s[2]);
}
__device__ __forceinline__ double comp3(double3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ bool box_inside(double3 x, const DObstacle& ob) {
  const double3 r = box_relative(x, ob);
  for (int i = 0; i < 3; ++i)
    if (fabs(comp3(r, i)) > ob.s[i] / 2) return false;
  return true;
}
// nearest side: its axis and sign; *dist = distance to it
__device__ __forceinline__ void box_side(double3 r, const DObstacle& ob, int* axis, double* sign, double* dist) {
  const int ax[6] = {1, 1, 0, 0, 2, 2};
  const double sg[6] = {1., -1., -1., 1., 1., -1.};
  double best = 0.;
  int b = -1;
  for (int k = 0; k < 6; ++k) {
    const double d = fabs(comp3(r, ax[k]) - sg[k] * 0.5 * ob.s[ax[k]]);
    if (b < 0 || d < best) {
      best = d;
      b = k;
    }
  }
  *axis = ax[b];
  *sign = sg[b];
  *dist = best;
}

// Closest kept triangle of a mesh obstacle through its LBVH: the same
// candidates (closed box test with half-width 1.1 tol), filter and ranking as
// mesh_obstacle_closest's scan in triangle order, which keeps the first of
// equal distances: here ties go to the lower triangle index.  Returns the
// triangle, or -1 when none is within tol.
__device__ int mesh_obstacle_bvh(double3 x, const double* mv, const int* mt, const WNode* nodes, double tol) {
  const double t = 1.1 * tol, tol_sq = tol * tol;
  double best = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  int bt = -1;
  int stack[64];
  int sp = 0;
  int node = 0;
  while (node >= 0) {
    const double2* r = reinterpret_cast<const double2*>(nodes + node);
    const double2 b01 = __ldg(r), b23 = __ldg(r + 1), b45 = __ldg(r + 2), b67 = __ldg(r + 3), b89 = __ldg(r + 4),
                  b1011 = __ldg(r + 5);
    const int4 chv = __ldg(reinterpret_cast<const int4*>(r + 6));
    const int ch[2] = {chv.x, chv.y};
    const bool ov[2] = {box_overlap(x, t, make_double3(b01.x, b01.y, b23.x), make_double3(b23.y, b45.x, b45.y)),
                        box_overlap(x, t, make_double3(b67.x, b67.y, b89.x), make_double3(b89.y, b1011.x, b1011.y))};
    int next = -1;
    for (int c = 0; c < 2; ++c) {
      if (!ov[c]) continue;
      if (ch[c] < 0) {
        const int k = ~ch[c];
        const double3 a = ld3(mv, mt[3 * k]), b = ld3(mv, mt[3 * k + 1]), cc = ld3(mv, mt[3 * k + 2]);
        double3 cp, w;
        closest_point(x, a, b, cc, tol, &cp, &w);
        const double3 dd = cp - x;
        if (!(dot3(dd, dd) < tol_sq)) continue;
        const double3 e = tri_point(a, b, cc, w) - x;
        const double d2 = dot3(e, e);
        if (d2 < best || (d2 == best && k < bt)) {
          best = d2;
          bt = k;
        }
      } else if (next < 0) {
        next = ch[c];
      } else if (sp < 64) {
        stack[sp++] = ch[c];
      } else {
        return -2;  // deeper than the stack: the caller falls back to the scan
      }
    }
    node = next >= 0 ? next : (sp > 0 ? stack[--sp] : -1);
  }
  return best < tol_sq ? bt : -1;
}

struct MeshBVH {
  int nv = 0, nt = 0;
  int *mval = nullptr, *mval_in = nullptr, *left = nullptr, *right = nullptr, *parent = nullptr,
      *leaf_parent = nullptr, *visits = nullptr;
  unsigned long long *keys = nullptr, *keys_sorted = nullptr, *bbox = nullptr;
  double *tlo = nullptr, *thi = nullptr;
  WNode* nodes = nullptr;
  void* cub_tmp = nullptr;
  size_t cub_bytes = 0;
};

namespace {
template <typename T>
T* balloc(size_t n) {
  T* p = nullptr;
  const cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(1, n) * sizeof(T));
  if (e != cudaSuccess) throw std::runtime_error(std::string("mesh obstacle BVH: ") + cudaGetErrorString(e));
  return p;
}
void bck(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("mesh obstacle BVH: ") + cudaGetErrorString(e));
}
}  // namespace

MeshBVH* mesh_bvh_create(int nv, int nt) {
  MeshBVH* b = new MeshBVH();
  b->nv = nv;
  b->nt = nt;
  b->mval = balloc<int>(nt);
  b->mval_in = balloc<int>(nt);
  b->left = balloc<int>(nt);
  b->right = balloc<int>(nt);
  b->parent = balloc<int>(nt);
  b->leaf_parent = balloc<int>(nt);
  b->visits = balloc<int>(nt);
  b->keys = balloc<unsigned long long>(nt);
  b->keys_sorted = balloc<unsigned long long>(nt);
  b->bbox = balloc<unsigned long long>(6);
  b->tlo = balloc<double>(3 * (size_t)nt);
  b->thi = balloc<double>(3 * (size_t)nt);
  b->nodes = balloc<WNode>(nt);
  bck(cub::DeviceRadixSort::SortPairs(nullptr, b->cub_bytes, b->keys, b->keys_sorted, b->mval_in, b->mval, nt));
  b->cub_tmp = balloc<char>(b->cub_bytes);
  return b;
}

void mesh_bvh_refit(MeshBVH* b, const double* verts, const int* tris, cudaStream_t st) {
  const int nt = b->nt, tb = 256;
  if (nt < 2) return;
  bck(cudaMemsetAsync(b->visits, 0, sizeof(int) * nt, st));
  k_refit_wide<<<(nt + tb - 1) / tb, tb, 0, st>>>(nt, b->mval, verts, tris, b->left, b->parent, b->leaf_parent,
                                                  b->nodes, b->visits);
}

void mesh_bvh_build(MeshBVH* b, const double* verts, const int* tris, cudaStream_t st) {
  const int nt = b->nt, nv = b->nv, tb = 256;
  if (nt < 2) return;
  const unsigned long long init[6] = {~0ULL, ~0ULL, ~0ULL, 0ULL, 0ULL, 0ULL};
  bck(cudaMemcpyAsync(b->bbox, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_bbox<<<std::min(1024, (nv + tb - 1) / tb), tb, 0, st>>>(nv, verts, b->bbox);
  k_tri_keys<<<(nt + tb - 1) / tb, tb, 0, st>>>(nt, verts, tris, 0, b->bbox, b->tlo, b->thi, b->keys, b->mval_in);
  size_t bytes = b->cub_bytes;
  bck(cub::DeviceRadixSort::SortPairs(b->cub_tmp, bytes, b->keys, b->keys_sorted, b->mval_in, b->mval, nt, 32, 62,
                                      st));
  k_build<<<(nt - 1 + tb - 1) / tb, tb, 0, st>>>(nt, b->keys_sorted, b->left, b->right, b->parent, b->leaf_parent);
  mesh_bvh_refit(b, verts, tris, st);
}

const void* mesh_bvh_nodes(const MeshBVH* b) { return b->nt >= 2 ? b->nodes : nullptr; }

void mesh_bvh_free(MeshBVH* b) {
  if (!b) return;
  void* ptrs[] = {b->mval, b->mval_in, b->left, b->right, b->parent, b->leaf_parent, b->visits, b->keys,
                  b->keys_sorted, b->bbox, b->tlo, b->thi, b->nodes, b->cub_tmp};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete b;
}

// Per (obstacle, vertex) flag, obstacle-major so that a stable compaction gives
// the reference's order (obstacles in scene order, vertices ascending:
// PhysicScene::getCollisionsInfoExceptFor PhysicScene.cpp:115-181 and
// Obstacle::checkCollision Obstacle.cpp:24-45).
__global__ void k_obstacle_flags(int N, const double* __restrict__ q, DObstacles obs, unsigned char* __restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double3 x = ld3(q, i);
  const int mi = obs.vmesh[i];
  for (int o = 0; o < obs.n; ++o) {
    const DObstacle& ob = obs.o[o];
    bool hit = false;
    if (ob.mesh >= 0 && ob.mesh != mi) {
      hit = false;  // obstacle restricted to another mesh
    } else if (ob.type == 0 || ob.type == 1) {
      // Sphere::isInside Sphere.cpp:93-98 (hard-coded 1 cm margin)
      const double3 r = x - make_double3(ob.c[0], ob.c[1], ob.c[2]);
      hit = sqrt(dot3(r, r)) < ob.R + 1e-2;
    } else if (ob.type == 2) {
      // StaticPlane::checkCollision StaticPlane.cpp:57-73 (hard-coded 1.5 cm)
      const double d = dot3(x - make_double3(ob.p[0], ob.p[1], ob.p[2]), make_double3(ob.n[0], ob.n[1], ob.n[2]));
      hit = d < 1.5e-2;
    } else if (ob.type == 4) {
      hit = box_inside(x, ob);
    } else {
      int tri = -2;
      if (ob.bvh) tri = mesh_obstacle_bvh(x, ob.mv, ob.mt, static_cast<const WNode*>(ob.bvh), ob.tol);
      if (tri == -2) {  // no hierarchy (one triangle) or a walk deeper than the stack: scan
        double3 cp;
        if (!mesh_obstacle_closest(x, ob.mv, ob.mt, ob.n_tri, ob.tol, &tri, &cp)) tri = -1;
      }
      hit = tri >= 0;
      obs.best[(int64_t)o * N + i] = tri;
    }
    flags[(int64_t)o * N + i] = hit ? 1 : 0;
  }
}

// MovingMesh::updateCurrentMesh MovingMesh.cpp:67-84: the current mesh is
// prev * (1 - a) + next * a, componentwise.
__global__ void k_moving_mesh_lerp(int n3, const double* __restrict__ prev, const double* __restrict__ next, double a,
                                   double* __restrict__ cur) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += gridDim.x * blockDim.x)
    cur[k] = prev[k] * (1 - a) + next[k] * a;
}

void launch_moving_mesh_lerp(cudaStream_t st, int n3, const double* prev, const double* next, double a, double* cur) {
  k_moving_mesh_lerp<<<std::min((n3 + 255) / 256, 1184), 256, 0, st>>>(n3, prev, next, a, cur);
}

// Obstacle contacts beyond the capacity are dropped: the count is clamped and
// bit 1 of the handle's error word is set (the step then reports
// PDF_CAPACITY_EXCEEDED).
__global__ void k_clamp_contacts(int* n, int cap, int* err) {
  if (*n > cap) {
    *n = cap;
    atomicOr(err, 2);
  }
}

// contact basis, computeBasis SFE:91-105
__device__ void write_basis(double* B, double3 n) {
  double3 t = cross3(n, make_double3(1., 0., 0.));
  if (sqrt(dot3(t, t)) < 1.e-15) t = cross3(n, make_double3(0., 1., 0.));
  t = normalized3(t);
  const double3 bt = normalized3(cross3(n, t));
  B[0] = n.x;
  B[1] = n.y;
  B[2] = n.z;
  B[3] = t.x;
  B[4] = t.y;
  B[5] = t.z;
  B[6] = bt.x;
  B[7] = bt.y;
  B[8] = bt.z;
}

__global__ void k_obstacle_materialize(int N, const double* __restrict__ q, DObstacles obs, const int* __restrict__ idx,
                                       const int* __restrict__ vmat, const double* __restrict__ friction, int n_mat,
                                       DContacts c) {
  const int C = *c.n_contacts;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
    const int o = idx[k] / N, i = idx[k] % N;
    const DObstacle& ob = obs.o[o];
    const double3 x = ld3(q, i);
    double3 nrm, sp = make_double3(0., 0., 0.);
    double gap;  // signed distance to the surface (warm-start feature)
    if (ob.type == 0 || ob.type == 1) {
      // Sphere::project Sphere.cpp:104-113
      const double3 ctr = make_double3(ob.c[0], ob.c[1], ob.c[2]);
      const double3 rel = x - ctr;
      gap = sqrt(dot3(rel, rel)) - ob.R;
      nrm = normalized3(rel);
      const double3 cp = ctr + ob.R * nrm;
      if (ob.type == 1 && ob.time_before_start < 0) {
        // RotatingSphere::checkCollision RotatingSphere.cpp:71-93: omega x (p - c)
        sp = cross3(make_double3(ob.rot[0], ob.rot[1], ob.rot[2]), cp - ctr);
      }
    } else if (ob.type == 2) {
      nrm = make_double3(ob.n[0], ob.n[1], ob.n[2]);
      gap = dot3(x - make_double3(ob.p[0], ob.p[1], ob.p[2]), nrm);
    } else if (ob.type == 4) {
      int axis;
      double sign, dist;
      box_side(box_relative(x, ob), ob, &axis, &sign, &dist);
      nrm = make_double3(axis == 0 ? sign : 0., axis == 1 ? sign : 0., axis == 2 ? sign : 0.);
      gap = -dist;
    } else {
      // the triangle k_obstacle_flags chose; its closest point again (the
      // contact point is the barycentric point, as in the ranking)
      const int tri = obs.best[idx[k]];
      const int i0 = ob.mt[3 * tri], i1 = ob.mt[3 * tri + 1], i2 = ob.mt[3 * tri + 2];
      const double3 a = ld3(ob.mv, i0), b = ld3(ob.mv, i1), cc = ld3(ob.mv, i2);
      double3 cp0, w;
      closest_point(x, a, b, cc, ob.tol, &cp0, &w);
      const double3 cp = tri_point(a, b, cc, w);
      nrm = normalized3(cross3(b - a, cc - a));  // Mesh::getTriangleNormal Mesh.cpp:120-126
      gap = dot3(x - cp, nrm);
      if (ob.type == 5 && ob.moving) {
        // MovingMesh::getPointSpeed MovingMesh.cpp:232-249
        const double3 pn = tri_point(ld3(ob.fnext, i0), ld3(ob.fnext, i1), ld3(ob.fnext, i2), w);
        const double3 pp = tri_point(ld3(ob.fprev, i0), ld3(ob.fprev, i1), ld3(ob.fprev, i2), w);
        const double3 dp = pn - pp;
        sp = make_double3(dp.x / ob.frame_dt, dp.y / ob.frame_dt, dp.z / ob.frame_dt);
      }
    }
    c.c_gap[k] = gap;
    c.c_vertex[k] = i;
    st3(c.c_normal, k, nrm);
    st3(c.c_speed, k, sp);
    c.c_mu[k] = friction[(int64_t)vmat[i] * n_mat + ob.material];
    write_basis(c.c_basis + 9 * (int64_t)k, nrm);
  }
}

// Involved-vertex slots: every contact vertex, self-contact vertex and partner
// gets a compact slot for the per-contact force buffers.
__device__ __forceinline__ void claim_slot(DContacts& c, int v) {
  if (atomicCAS(c.slot_of + v, -1, -2) == -1) {
    const int s = atomicAdd(c.n_slots, 1);
    if (s < c.slot_cap) {
      c.slot_vertex[s] = v;
      c.slot_of[v] = s;
    }
  }
}

__global__ void k_contact_slots(DContacts c) {
  const int C = *c.n_contacts, S = *c.n_self;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C + S; k += gridDim.x * blockDim.x) {
    if (k < C) {
      claim_slot(c, c.c_vertex[k]);
    } else {
      claim_slot(c, c.s_vertex[k - C]);
      claim_slot(c, c.s_partner[k - C]);
    }
  }
}

__global__ void k_contact_slots_fill(DContacts c) {
  const int C = *c.n_contacts, S = *c.n_self;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C + S; k += gridDim.x * blockDim.x) {
    if (k < C) {
      c.c_slot[k] = c.slot_of[c.c_vertex[k]];
    } else {
      c.s_slota[k - C] = c.slot_of[c.s_vertex[k - C]];
      c.s_slotb[k - C] = c.slot_of[c.s_partner[k - C]];
      st3(c.s_remember, k - C, make_double3(0., 0., 0.));
    }
  }
  const int ns = min(*c.n_slots, c.slot_cap);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < 3 * ns; s += gridDim.x * blockDim.x) {
    c.cf[0][s] = 0.;
    c.cf[1][s] = 0.;
    c.sf[0][s] = 0.;
    c.sf[1][s] = 0.;
  }
}

__global__ void k_contact_slots_reset(DContacts c) {
  const int ns = min(*c.n_slots, c.slot_cap);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) c.slot_of[c.slot_vertex[s]] = -1;
}

}  // namespace pdfb
