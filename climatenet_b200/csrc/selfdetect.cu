// selfdetect.cu — self-collision detection on the GPU (compiled with
// --fmad=false: every decision below must round like the reference).
//
//  1. LBVH over the mesh's triangles (Morton codes of the centroids, radix
//     sort, Karras hierarchy, bottom-up box refit).  Node boxes are exact
//     unions of the triangles' own bounding boxes, so a traversal with the
//     closed query box [x - 1.1 tol, x + 1.1 tol] finds exactly the candidate
//     set of getMeshPotentialTriangleCollision (geometry_util.cpp:284-327).
//  2. Per candidate: closest point with the reference's early exit and the
//     |c - x|^2 < tol^2 filter (checkMeshAllCollision geometry_util.cpp:229-262).
//     Hits that the pairing would skip without side effect (vertex in the
//     triangle, a zero barycentric coordinate; geometry_util.cpp:127-135) are
//     dropped here.
//  3. Hits are sorted by (vertex, triangle): the canonical candidate order.
//  4. Greedy node-node pairing in that order (geometry_util.cpp:94-219), one
//     thread: the pairing of a vertex depends on the pairings of its 1-ring.
//  5. Breadth-first Gauss-Seidel levels of the self-contact graph
//     (SFE:161-293) in one CTA, from the closed-form equivalent of the
//     reference's three BFS passes: edge level = min(dist(a), dist(b)) with
//     dist the BFS distance from the component's seeds (obstacle-contact
//     vertices; else its lowest-index degree-1 vertex; else its lowest-index
//     vertex).
#include <cuda_runtime.h>

#include <cub/cub.cuh>
#include <cuda/atomic>
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "device.cuh"
#include "geometry.cuh"
#include "handle.hpp"
#include "kernels.hpp"
#include "lbvh.cuh"

namespace pdfb {
namespace {

constexpr int kRegCap = 16;   // pairing partners remembered per vertex
constexpr int kHitSlots = 32; // step path: candidate triangles kept per vertex
constexpr int kRebuildEvery = 8;  // step path: hierarchy rebuilt every k steps, refit in between

// Error bits of the handle's device error word set by the step path (read at
// the end of pdf_step): more partners or self contacts than the buffers hold,
// more hits than kHitSlots per vertex or than the hit buffer, BVH stack.
constexpr int kErrSelfContacts = 4, kErrSelfHits = 8, kErrSelfStack = 16;

struct SelfWS {
  int max_nt = 0, max_nv = 0, hit_cap = 0;
  double *tlo = nullptr, *thi = nullptr;             // 3 nt leaf boxes (triangle order)
  unsigned long long *mkey = nullptr, *mkey2 = nullptr;
  int *mval = nullptr, *mval2 = nullptr;             // sorted leaf -> triangle
  int *left = nullptr, *right = nullptr, *parent = nullptr, *leaf_parent = nullptr;
  double *nlo = nullptr, *nhi = nullptr;             // 3 (nt-1) node boxes
  int* visits = nullptr;
  unsigned long long* bbox = nullptr;                // 6 ordered-bit min/max
  int* n_hits = nullptr;
  unsigned long long *hkey = nullptr, *hkey2 = nullptr;
  int *hval = nullptr, *hval2 = nullptr;
  double* hbary = nullptr;
  int *reg = nullptr, *reg_n = nullptr, *touched = nullptr, *n_touched = nullptr, *err = nullptr;
  // BFS scratch (slot space)
  int *deg = nullptr, *uf = nullptr, *dist = nullptr, *seed = nullptr, *cobst = nullptr, *cdeg1 = nullptr,
      *cmin = nullptr, *elev = nullptr, *lcount = nullptr;
  void* cub_tmp = nullptr;
  size_t cub_bytes = 0;
  // step path: one persistent hierarchy per mesh (regions at the mesh's
  // triangle offset, all meshes' triangles in total), per-vertex hit slots
  // and counts (shared by the meshes, consumed within the step)
  WNode* wnodes = nullptr;
  int *s_mval = nullptr, *s_left = nullptr, *s_right = nullptr, *s_parent = nullptr, *s_leaf_parent = nullptr,
      *s_visits = nullptr;
  int *hcount = nullptr, *hoff = nullptr, *slot_tri = nullptr, *n_total = nullptr;
  std::vector<int> since_build;  // per mesh: steps since its hierarchy was built (0 = never)
};

#define CKS(x)                                                                                    \
  do {                                                                                            \
    cudaError_t e_ = (x);                                                                         \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
T* salloc(size_t n) {
  T* p = nullptr;
  CKS(cudaMalloc((void**)&p, std::max<size_t>(1, n) * sizeof(T)));
  return p;
}

__device__ __forceinline__ void child_box(int c, const int* mval, const double* tlo, const double* thi,
                                          const double* nlo, const double* nhi, double3* lo, double3* hi) {
  if (c < 0) {
    const int t = mval[~c];
    *lo = make_double3(__ldcg(tlo + 3 * t), __ldcg(tlo + 3 * t + 1), __ldcg(tlo + 3 * t + 2));
    *hi = make_double3(__ldcg(thi + 3 * t), __ldcg(thi + 3 * t + 1), __ldcg(thi + 3 * t + 2));
  } else {
    *lo = make_double3(__ldcg(nlo + 3 * c), __ldcg(nlo + 3 * c + 1), __ldcg(nlo + 3 * c + 2));
    *hi = make_double3(__ldcg(nhi + 3 * c), __ldcg(nhi + 3 * c + 1), __ldcg(nhi + 3 * c + 2));
  }
}

// Bottom-up refit: the second child to arrive computes the parent's box.
__global__ void k_refit(int n, const int* __restrict__ mval, const double* tlo, const double* thi, const int* left,
                        const int* right, const int* parent, const int* leaf_parent, double* nlo, double* nhi,
                        int* visits) {
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n) return;
  int p = leaf_parent[leaf];
  while (p >= 0) {
    __threadfence();
    if (atomicAdd(visits + p, 1) == 0) return;
    __threadfence();
    double3 l0, h0, l1, h1;
    child_box(left[p], mval, tlo, thi, nlo, nhi, &l0, &h0);
    child_box(right[p], mval, tlo, thi, nlo, nhi, &l1, &h1);
    const double3 lo = make_double3(fmin(l0.x, l1.x), fmin(l0.y, l1.y), fmin(l0.z, l1.z));
    const double3 hi = make_double3(fmax(h0.x, h1.x), fmax(h0.y, h1.y), fmax(h0.z, h1.z));
    __stcg(nlo + 3 * p, lo.x);
    __stcg(nlo + 3 * p + 1, lo.y);
    __stcg(nlo + 3 * p + 2, lo.z);
    __stcg(nhi + 3 * p, hi.x);
    __stcg(nhi + 3 * p + 1, hi.y);
    __stcg(nhi + 3 * p + 2, hi.z);
    p = parent[p];
  }
}

// Step-path traversal: both children are tested at their parent (one node
// record load), overlapping leaf children are handled on the spot, the walk
// continues into the first overlapping internal child and keeps the other on
// a per-thread stack in shared memory (column-major: no bank conflicts).  A
// candidate is a triangle whose box overlaps the vertex's query box and that
// does not contain the vertex; candidates go to the vertex's slots,
// unordered, and the closest-point filter runs in k_filter_candidates.
constexpr int kTraverseThreads = 128, kTraverseStack = 48;
__global__ void __launch_bounds__(kTraverseThreads)
    k_traverse_slots(int nv, int nt, const double* __restrict__ q, const int* __restrict__ tris, int v0, double tol,
                     const WNode* __restrict__ nodes, int* __restrict__ hcount, int* __restrict__ slot_tri,
                     int* err) {
  __shared__ int stack[kTraverseStack * kTraverseThreads];
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const double t = 1.1 * tol;
  const double3 x = ld3(q, v0 + v);
  int count = 0;
  int* slots = slot_tri + (int64_t)v * kHitSlots;
  const int gv = v0 + v;
  auto candidate = [&](int tri) {
    if (__ldg(tris + 3 * tri) == gv || __ldg(tris + 3 * tri + 1) == gv || __ldg(tris + 3 * tri + 2) == gv) return;
    if (count < kHitSlots) slots[count] = tri;
    ++count;
  };
  if (nt == 1) {
    double3 tl, th;
    tri_box(ld3(q, tris[0]), ld3(q, tris[1]), ld3(q, tris[2]), &tl, &th);
    if (box_overlap(x, t, tl, th)) candidate(0);
  } else {
    int* st = stack + threadIdx.x;
    int sp = 0;
    int node = 0;
    while (node >= 0) {
      // the 112-byte record in seven 16-byte loads
      const double2* r = reinterpret_cast<const double2*>(nodes + node);
      const double2 b01 = __ldg(r), b23 = __ldg(r + 1), b45 = __ldg(r + 2), b67 = __ldg(r + 3),
                    b89 = __ldg(r + 4), b1011 = __ldg(r + 5);
      const int4 chv = __ldg(reinterpret_cast<const int4*>(r + 6));
      const int c0 = chv.x, c1 = chv.y;
      const bool o0 = box_overlap(x, t, make_double3(b01.x, b01.y, b23.x), make_double3(b23.y, b45.x, b45.y));
      const bool o1 = box_overlap(x, t, make_double3(b67.x, b67.y, b89.x), make_double3(b89.y, b1011.x, b1011.y));
      if (o0 && c0 < 0) candidate(~c0);
      if (o1 && c1 < 0) candidate(~c1);
      const bool d0 = o0 && c0 >= 0, d1 = o1 && c1 >= 0;
      if (d0 && d1) {
        if (sp >= kTraverseStack) {
          atomicOr(err, kErrSelfStack);
          break;
        }
        st[sp++ * kTraverseThreads] = c1;
        node = c0;
      } else if (d0) {
        node = c0;
      } else if (d1) {
        node = c1;
      } else {
        node = sp > 0 ? st[--sp * kTraverseThreads] : -1;
      }
    }
  }
  if (count > kHitSlots) {
    atomicOr(err, kErrSelfHits);
    count = kHitSlots;
  }
  hcount[v] = count;
}

// The closest-point filter and the pairing precondition of mode 1 below on
// each vertex's candidates; survivors stay in the vertex's slots (in place,
// order kept) and hcount becomes their number.
__global__ void k_filter_candidates(int nv, const double* __restrict__ q, const int* __restrict__ tris, int v0,
                                    double tol, int* __restrict__ hcount, int* __restrict__ slot_tri) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int cnt = hcount[v];
  if (cnt == 0) return;
  int* slots = slot_tri + (int64_t)v * kHitSlots;
  const double3 x = ld3(q, v0 + v);
  const double tol_sq = tol * tol;
  int kept = 0;
  for (int k = 0; k < cnt; ++k) {
    const int tri = slots[k];
    double3 cp, w;
    closest_point(x, ld3(q, tris[3 * tri]), ld3(q, tris[3 * tri + 1]), ld3(q, tris[3 * tri + 2]), tol, &cp, &w);
    const double3 dd = cp - x;
    if (!(dot3(dd, dd) < tol_sq)) continue;
    if (w.x == 0 || w.y == 0 || w.z == 0) continue;
    slots[kept++] = tri;
  }
  hcount[v] = kept;
}

// Hits in canonical (vertex, triangle) order without a global sort: vertex v
// owns [hoff[v], hoff[v] + hcount[v]); its triangles are sorted in place and
// the barycentric coordinates recomputed (same arithmetic as the filter).
__global__ void k_compact_hits(int nv, const double* __restrict__ q, const int* __restrict__ tris, int v0, double tol,
                               const int* __restrict__ hcount, const int* __restrict__ hoff,
                               const int* __restrict__ slot_tri, int cap, unsigned long long* hkey, int* hval,
                               double* hbary, int* n_total, int* err) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int cnt = hcount[v], o = hoff[v];
  if (v == nv - 1) {
    const int total = o + cnt;
    if (total > cap) atomicOr(err, kErrSelfHits);
    *n_total = min(total, cap);
  }
  if (cnt == 0) return;
  int tl[kHitSlots];
  for (int k = 0; k < cnt; ++k) {
    const int tv = slot_tri[(int64_t)v * kHitSlots + k];
    int j = k;
    while (j > 0 && tl[j - 1] > tv) {
      tl[j] = tl[j - 1];
      --j;
    }
    tl[j] = tv;
  }
  const double3 x = ld3(q, v0 + v);
  for (int k = 0; k < cnt; ++k) {
    const int h = o + k;
    if (h >= cap) return;
    const int tri = tl[k];
    double3 cp, w;
    closest_point(x, ld3(q, tris[3 * tri]), ld3(q, tris[3 * tri + 1]), ld3(q, tris[3 * tri + 2]), tol, &cp, &w);
    hkey[h] = ((unsigned long long)v << 32) | (unsigned int)tri;
    hval[h] = h;
    st3(hbary, h, w);
  }
}

// Per-vertex traversal.  mode 0: emit every box candidate (v, t);
// mode 1: emit hits that survive the closest-point filter and can pair.
__global__ void k_traverse(int nv, int nt, const double* __restrict__ q, const int* __restrict__ tris, int v0,
                           double tol, const int* __restrict__ mval, const double* __restrict__ tlo,
                           const double* __restrict__ thi, const int* __restrict__ left, const int* __restrict__ right,
                           const double* __restrict__ nlo, const double* __restrict__ nhi, int mode, int* n_hits,
                           int cap, unsigned long long* hkey, int* hval, double* hbary, int* err) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const double t = 1.1 * tol;
  const double tol_sq = tol * tol;
  const double3 x = ld3(q, v0 + v);
  int stack[64];
  int sp = 0;
  stack[sp++] = (nt == 1) ? ~0 : 0;
  while (sp > 0) {
    const int node = stack[--sp];
    if (node < 0) {
      const int tri = mval[~node];
      const double3 lo = ld3(tlo, tri), hi = ld3(thi, tri);
      if (!box_overlap(x, t, lo, hi)) continue;
      if (mode == 0) {
        const int k = atomicAdd(n_hits, 1);
        if (k < cap) {
          hkey[k] = ((unsigned long long)v << 32) | (unsigned int)tri;
          hval[k] = k;
        }
        continue;
      }
      const int ia = tris[3 * tri] - v0, ib = tris[3 * tri + 1] - v0, ic = tris[3 * tri + 2] - v0;
      if (ia == v || ib == v || ic == v) continue;
      double3 cp, w;
      closest_point(x, ld3(q, v0 + ia), ld3(q, v0 + ib), ld3(q, v0 + ic), tol, &cp, &w);
      const double3 dd = cp - x;
      if (!(dot3(dd, dd) < tol_sq)) continue;
      if (w.x == 0 || w.y == 0 || w.z == 0) continue;
      const int k = atomicAdd(n_hits, 1);
      if (k < cap) {
        hkey[k] = ((unsigned long long)v << 32) | (unsigned int)tri;
        hval[k] = k;
        st3(hbary, k, w);
      }
      continue;
    }
    const double3 lo = ld3(nlo, node), hi = ld3(nhi, node);
    if (!box_overlap(x, t, lo, hi)) continue;
    if (sp + 2 > 64) {
      atomicExch(err, 2);
      return;
    }
    stack[sp++] = left[node];
    stack[sp++] = right[node];
  }
}

// Greedy node-node pairing (checkMeshSelfCollisions, geometry_util.cpp:94-219)
// over hits in canonical order; emits self contacts in the order found.
// n_hits_dev (if not null) holds the hit count on the device; err_word (if
// not null) receives kErrSelfContacts instead of *err being set, and the
// contacts paired so far are kept.
__global__ void k_pair(int n_hits, const unsigned long long* __restrict__ hkey, const int* __restrict__ hval,
                       const double* __restrict__ hbary, const double* __restrict__ q, const int* __restrict__ tris,
                       int v0, const int* __restrict__ ring_ptr, const int* __restrict__ ring_idx, double mu,
                       int* reg, int* reg_n, int* touched, int* n_touched, int touched_cap, DContacts c, int* err,
                       const int* n_hits_dev = nullptr, int* err_word = nullptr) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int S = *c.n_self;
  int nt = *n_touched;
  if (n_hits_dev) n_hits = *n_hits_dev;
  for (int h = 0; h < n_hits; ++h) {
    const int v = (int)(hkey[h] >> 32);
    const int tri = (int)(hkey[h] & 0xffffffffu);
    const int gv = v0 + v;
    const double3 w = ld3(hbary, hval[h]);
    const int tv[3] = {tris[3 * tri], tris[3 * tri + 1], tris[3 * tri + 2]};
    // already paired with a vertex of this triangle?
    bool skip = false;
    for (int k = 0; k < 3 && !skip; ++k)
      for (int r = 0; r < reg_n[gv]; ++r)
        if (reg[gv * kRegCap + r] == tv[k]) {
          skip = true;
          break;
        }
    if (skip) continue;
    bool cand[3] = {true, true, true};
    for (int s = ring_ptr[gv]; s < ring_ptr[gv + 1]; ++s) {
      const int rv = ring_idx[s];
      // first triangle slot present in registered[rv] (isTriangleVertexIndexIn)
      int found = 3;
      for (int k = 0; k < 3 && found == 3; ++k)
        for (int r = 0; r < reg_n[rv]; ++r)
          if (reg[rv * kRegCap + r] == tv[k]) {
            found = k;
            break;
          }
      if (found < 3) cand[found] = false;
    }
    int best = 3;
    double bb = 0;
    const double wv[3] = {w.x, w.y, w.z};
    for (int k = 0; k < 3; ++k) {
      if (!cand[k]) continue;
      if (wv[k] > bb) {
        best = k;
        bb = wv[k];
      }
    }
    if (best >= 3) continue;
    const double3 xa = ld3(q, tv[0]), xb = ld3(q, tv[1]), xc = ld3(q, tv[2]);
    const double3 cpt = tri_point(xa, xb, xc, w);
    const double3 nrm = normalized3(ld3(q, gv) - cpt);
    const int paired = tv[best];
    if (reg_n[paired] >= kRegCap || reg_n[gv] >= kRegCap) {
      if (err_word) {
        atomicOr(err_word, kErrSelfContacts);
        break;
      }
      *err = 3;
      return;
    }
    if (reg_n[paired] == 0 && nt < touched_cap) touched[nt++] = paired;
    reg[paired * kRegCap + reg_n[paired]++] = gv;
    if (reg_n[gv] == 0 && nt < touched_cap) touched[nt++] = gv;
    reg[gv * kRegCap + reg_n[gv]++] = paired;
    if (S >= c.self_cap) {
      if (err_word) {
        atomicOr(err_word, kErrSelfContacts);
        break;
      }
      *err = 4;
      return;
    }
    c.s_vertex[S] = gv;
    c.s_partner[S] = paired;
    c.s_face[3 * S] = tv[0];
    c.s_face[3 * S + 1] = tv[1];
    c.s_face[3 * S + 2] = tv[2];
    st3(c.s_normal, S, nrm);
    c.s_mu[S] = mu;
    ++S;
  }
  *c.n_self = S;
  *n_touched = nt;
}

__global__ void k_reset_registered(int* reg_n, int* touched, int* n_touched) {
  const int n = *n_touched;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) reg_n[touched[i]] = 0;
}

__device__ void write_basis_s(double* B, double3 n) {
  double3 t = cross3(n, make_double3(1., 0., 0.));
  if (sqrt(dot3(t, t)) < 1.e-15) t = cross3(n, make_double3(0., 1., 0.));
  t = normalized3(t);
  const double3 bt = normalized3(cross3(n, t));
  B[0] = n.x; B[1] = n.y; B[2] = n.z;
  B[3] = t.x; B[4] = t.y; B[5] = t.z;
  B[6] = bt.x; B[7] = bt.y; B[8] = bt.z;
}

__global__ void k_self_bases(DContacts c) {
  const int S = *c.n_self;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x)
    write_basis_s(c.s_basis + 9 * (int64_t)k, ld3(c.s_normal, k));
}

__device__ int uf_find(int* uf, int x) {
  while (true) {
    const int p = uf[x];
    if (p == x) return x;
    const int gp = uf[p];
    if (gp != p) atomicCAS(uf + x, p, gp);
    x = p;
  }
}

// Breadth-first levels (one CTA).  Slot space: every contact vertex has a slot.
__global__ void k_levels(DContacts c, int* deg, int* uf, int* dist, int* seed, int* cobst, int* cdeg1, int* cmin,
                         int* elev, int* lcount, int cap_levels) {
  __shared__ int changed;
  __shared__ int maxlvl;
  const int S = *c.n_self, C = *c.n_contacts;
  const int V = min(*c.n_slots, c.slot_cap);
  const int tid = threadIdx.x, nth = blockDim.x;
  const int INF = 0x3fffffff;
  if (S == 0) {
    if (tid == 0) {
      *c.n_levels = 0;
      c.level_ptr[0] = 0;
    }
    return;
  }
  for (int s = tid; s < V; s += nth) {
    deg[s] = 0;
    uf[s] = s;
    dist[s] = INF;
    seed[s] = 0;
    cobst[s] = 0;
    cdeg1[s] = INF;
    cmin[s] = INF;
  }
  __syncthreads();
  for (int e = tid; e < S; e += nth) {
    atomicAdd(deg + c.s_slota[e], 1);
    atomicAdd(deg + c.s_slotb[e], 1);
  }
  for (int k = tid; k < C; k += nth) seed[c.c_slot[k]] = 1;
  __syncthreads();
  // connected components: hook the larger root under the smaller until stable
  do {
    __syncthreads();
    if (tid == 0) changed = 0;
    __syncthreads();
    for (int e = tid; e < S; e += nth) {
      const int ra = uf_find(uf, c.s_slota[e]), rb = uf_find(uf, c.s_slotb[e]);
      if (ra != rb) {
        atomicMin(uf + max(ra, rb), min(ra, rb));
        changed = 1;
      }
    }
    __syncthreads();
  } while (changed);
  for (int s = tid; s < V; s += nth) uf[s] = uf_find(uf, s);
  __syncthreads();
  for (int s = tid; s < V; s += nth) {
    const int r = uf[s];
    const int vx = c.slot_vertex[s];
    if (seed[s]) atomicOr(cobst + r, 1);
    if (deg[s] == 1) atomicMin(cdeg1 + r, vx);
    if (deg[s] >= 1) atomicMin(cmin + r, vx);
  }
  __syncthreads();
  for (int s = tid; s < V; s += nth) {
    const int r = uf[s];
    const int vx = c.slot_vertex[s];
    bool src;
    if (cobst[r])
      src = seed[s] != 0;
    else
      src = vx == (cdeg1[r] != INF ? cdeg1[r] : cmin[r]);
    dist[s] = src ? 0 : INF;
  }
  __syncthreads();
  int d = 0;
  do {
    __syncthreads();
    if (tid == 0) changed = 0;
    __syncthreads();
    for (int e = tid; e < S; e += nth) {
      const int a = c.s_slota[e], b = c.s_slotb[e];
      if (dist[a] == d && dist[b] == INF) {
        dist[b] = d + 1;
        changed = 1;
      }
      if (dist[b] == d && dist[a] == INF) {
        dist[a] = d + 1;
        changed = 1;
      }
    }
    __syncthreads();
    ++d;
  } while (changed);
  if (tid == 0) maxlvl = 0;
  for (int l = tid; l < cap_levels + 1; l += nth) lcount[l] = 0;
  __syncthreads();
  for (int e = tid; e < S; e += nth) elev[e] = min(dist[c.s_slota[e]], dist[c.s_slotb[e]]);
  // the reference opens one level per breadth-first frontier, including the
  // last frontier that finds no new edge: levels = max reached distance + 1
  for (int s = tid; s < V; s += nth)
    if (dist[s] < INF) atomicMax(&maxlvl, dist[s]);
  __syncthreads();
  const int nl = min(maxlvl + 1, cap_levels);
  for (int e = tid; e < S; e += nth) atomicAdd(lcount + min(elev[e], nl - 1), 1);
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int l = 0; l < nl; ++l) {
      c.level_ptr[l] = acc;
      acc += lcount[l];
      lcount[l] = c.level_ptr[l];
    }
    c.level_ptr[nl] = acc;
    *c.n_levels = nl;
    // stable fill in contact order
    for (int e = 0; e < S; ++e) c.level_order[lcount[min(elev[e], nl - 1)]++] = e;
  }
}

void ws_alloc(SelfWS& w, int nv, int nt, int hit_cap, int slot_cap) {
  w.max_nv = nv;
  w.max_nt = nt;
  w.hit_cap = hit_cap;
  w.tlo = salloc<double>(3 * (size_t)nt);
  w.thi = salloc<double>(3 * (size_t)nt);
  w.mkey = salloc<unsigned long long>(nt);
  w.mkey2 = salloc<unsigned long long>(nt);
  w.mval = salloc<int>(nt);
  w.mval2 = salloc<int>(nt);
  w.left = salloc<int>(nt);
  w.right = salloc<int>(nt);
  w.parent = salloc<int>(nt);
  w.leaf_parent = salloc<int>(nt);
  w.nlo = salloc<double>(3 * (size_t)nt);
  w.nhi = salloc<double>(3 * (size_t)nt);
  w.visits = salloc<int>(nt);
  w.bbox = salloc<unsigned long long>(6);
  w.n_hits = salloc<int>(1);
  w.hkey = salloc<unsigned long long>(hit_cap);
  w.hkey2 = salloc<unsigned long long>(hit_cap);
  w.hval = salloc<int>(hit_cap);
  w.hval2 = salloc<int>(hit_cap);
  w.hbary = salloc<double>(3 * (size_t)hit_cap);
  w.err = salloc<int>(1);
  w.hcount = salloc<int>(nv);
  w.hoff = salloc<int>(nv);
  w.slot_tri = salloc<int>((size_t)nv * kHitSlots);
  w.n_total = salloc<int>(1);
  size_t b1 = 0, b2 = 0, b3 = 0;
  CKS(cub::DeviceScan::ExclusiveSum(nullptr, b3, w.hcount, w.hoff, nv));
  CKS(cub::DeviceRadixSort::SortPairs(nullptr, b1, w.mkey, w.mkey2, w.mval, w.mval2, nt));
  CKS(cub::DeviceRadixSort::SortPairs(nullptr, b2, w.hkey, w.hkey2, w.hval, w.hval2, hit_cap));
  w.cub_bytes = std::max(std::max(b1, b2), b3);
  w.cub_tmp = salloc<char>(w.cub_bytes);
  (void)slot_cap;
}

void ws_free(SelfWS& w) {
  void* ptrs[] = {w.tlo, w.thi, w.mkey, w.mkey2, w.mval, w.mval2, w.left, w.right, w.parent, w.leaf_parent,
                  w.nlo, w.nhi, w.visits, w.bbox, w.n_hits, w.hkey, w.hkey2, w.hval, w.hval2, w.hbary,
                  w.reg, w.reg_n, w.touched, w.n_touched, w.err, w.deg, w.uf, w.dist, w.seed, w.cobst, w.cdeg1,
                  w.cmin, w.elev, w.lcount, w.cub_tmp, w.wnodes, w.hcount, w.hoff, w.slot_tri, w.n_total,
                  w.s_mval, w.s_left, w.s_right, w.s_parent, w.s_leaf_parent, w.s_visits};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  w = SelfWS{};
}

// Builds the LBVH over triangles [t0, t0+nt) (scene-global vertex indices
// with vertices [v0, v0+nv)) and traverses it from every vertex of the range.
// Returns the number of emitted records (may exceed the capacity).
int detect_mesh(SelfWS& w, const double* q, const int* tris_global, int v0, int nv, int nt, double tol, int mode,
                cudaStream_t st) {
  const int tb = 256;
  const unsigned long long init[6] = {~0ULL, ~0ULL, ~0ULL, 0ULL, 0ULL, 0ULL};
  CKS(cudaMemcpyAsync(w.bbox, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_bbox<<<std::min(1024, (nv + tb - 1) / tb), tb, 0, st>>>(nv, q + 3 * (size_t)v0, w.bbox);
  k_tri_keys<<<(nt + tb - 1) / tb, tb, 0, st>>>(nt, q, tris_global, v0, w.bbox, w.tlo, w.thi, w.mkey, w.mval);
  size_t bytes = w.cub_bytes;
  CKS(cub::DeviceRadixSort::SortPairs(w.cub_tmp, bytes, w.mkey, w.mkey2, w.mval, w.mval2, nt, 0, 64, st));
  if (nt > 1) {
    k_build<<<(nt - 1 + tb - 1) / tb, tb, 0, st>>>(nt, w.mkey2, w.left, w.right, w.parent, w.leaf_parent);
    CKS(cudaMemsetAsync(w.visits, 0, sizeof(int) * nt, st));
    k_refit<<<(nt + tb - 1) / tb, tb, 0, st>>>(nt, w.mval2, w.tlo, w.thi, w.left, w.right, w.parent, w.leaf_parent,
                                               w.nlo, w.nhi, w.visits);
  }
  CKS(cudaMemsetAsync(w.n_hits, 0, sizeof(int), st));
  CKS(cudaMemsetAsync(w.err, 0, sizeof(int), st));
  k_traverse<<<(nv + tb - 1) / tb, tb, 0, st>>>(nv, nt, q, tris_global, v0, tol, w.mval2, w.tlo, w.thi, w.left,
                                               w.right, w.nlo, w.nhi, mode, w.n_hits, w.hit_cap, w.hkey, w.hval,
                                               w.hbary, w.err);
  int nh = 0, err = 0;
  CKS(cudaMemcpyAsync(&nh, w.n_hits, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKS(cudaMemcpyAsync(&err, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKS(cudaStreamSynchronize(st));
  if (err) throw std::overflow_error("BVH traversal stack overflow (a vertex's walk needs more than the stack holds)");
  if (nh > 0 && nh <= w.hit_cap) {
    int bits = 64;
    CKS(cub::DeviceRadixSort::SortPairs(w.cub_tmp, bytes, w.hkey, w.hkey2, w.hval, w.hval2, nh, 0, bits, st));
  }
  return nh;
}

// Step path of detect_mesh: same candidate semantics, no host round trip.
// The hits of mesh [v0, v0+nv) end in hkey2 / hval2 / hbary in canonical
// order with their count in *w.n_total; errors go to err_word.
void detect_mesh_step(SelfWS& w, const double* q, const int* tris_global, int v0, int nv, int nt, int t0,
                      bool rebuild, double tol, cudaStream_t st, int* err_word) {
  const int tb = 256;
  int* mval = w.s_mval + t0;
  int* left = w.s_left + t0;
  int* parent = w.s_parent + t0;
  int* leaf_parent = w.s_leaf_parent + t0;
  WNode* nodes = w.wnodes + t0;
  if (rebuild) {
    const unsigned long long init[6] = {~0ULL, ~0ULL, ~0ULL, 0ULL, 0ULL, 0ULL};
    CKS(cudaMemcpyAsync(w.bbox, init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_bbox<<<std::min(1024, (nv + tb - 1) / tb), tb, 0, st>>>(nv, q + 3 * (size_t)v0, w.bbox);
    k_tri_keys<<<(nt + tb - 1) / tb, tb, 0, st>>>(nt, q, tris_global, v0, w.bbox, w.tlo, w.thi, w.mkey, w.mval);
    // key = morton << 32 | triangle and the sort is stable on triangles in
    // ascending order: the 30 Morton bits give the full key order
    size_t bytes = w.cub_bytes;
    CKS(cub::DeviceRadixSort::SortPairs(w.cub_tmp, bytes, w.mkey, w.mkey2, w.mval, mval, nt, 32, 62, st));
    if (nt > 1)
      k_build<<<(nt - 1 + tb - 1) / tb, tb, 0, st>>>(nt, w.mkey2, left, w.s_right + t0, parent, leaf_parent);
  }
  if (nt > 1) {
    CKS(cudaMemsetAsync(w.s_visits + t0, 0, sizeof(int) * nt, st));
    k_refit_wide<<<(nt + tb - 1) / tb, tb, 0, st>>>(nt, mval, q, tris_global, left, parent, leaf_parent, nodes,
                                                    w.s_visits + t0);
  }
  k_traverse_slots<<<(nv + kTraverseThreads - 1) / kTraverseThreads, kTraverseThreads, 0, st>>>(
      nv, nt, q, tris_global, v0, tol, nodes, w.hcount, w.slot_tri, err_word);
  k_filter_candidates<<<(nv + tb - 1) / tb, tb, 0, st>>>(nv, q, tris_global, v0, tol, w.hcount, w.slot_tri);
  size_t bytes = w.cub_bytes;
  CKS(cub::DeviceScan::ExclusiveSum(w.cub_tmp, bytes, w.hcount, w.hoff, nv, st));
  k_compact_hits<<<(nv + tb - 1) / tb, tb, 0, st>>>(nv, q, tris_global, v0, tol, w.hcount, w.hoff, w.slot_tri,
                                                    w.hit_cap, w.hkey2, w.hval2, w.hbary, w.n_total, err_word);
}

// pairing / level scratch sized by the scene
void ws_alloc_pairing(SelfWS& w, int N, int slot_cap, int cap_levels) {
  w.reg = salloc<int>((size_t)N * kRegCap);
  w.reg_n = salloc<int>(N);
  CKS(cudaMemset(w.reg_n, 0, sizeof(int) * N));
  w.touched = salloc<int>(N);
  w.n_touched = salloc<int>(1);
  CKS(cudaMemset(w.n_touched, 0, sizeof(int)));
  w.deg = salloc<int>(slot_cap);
  w.uf = salloc<int>(slot_cap);
  w.dist = salloc<int>(slot_cap);
  w.seed = salloc<int>(slot_cap);
  w.cobst = salloc<int>(slot_cap);
  w.cdeg1 = salloc<int>(slot_cap);
  w.cmin = salloc<int>(slot_cap);
  w.elev = salloc<int>(cap_levels);
  w.lcount = salloc<int>(cap_levels + 1);
}

}  // namespace

int self_detect_init(pdf_handle* h) {
  try {
    SelfWS* w = new SelfWS();
    int max_nt = 1, max_nv = 1;
    for (const auto& md : h->model.meshes) {
      max_nt = std::max(max_nt, md.n_triangles);
      max_nv = std::max(max_nv, md.n_vertices);
    }
    ws_alloc(*w, max_nv, max_nt, std::max(1024, 8 * max_nv), h->model.N);
    ws_alloc_pairing(*w, h->model.N, h->model.N, h->cap_self);
    const size_t T = std::max<size_t>(1, h->model.tris.size() / 3);
    w->wnodes = salloc<WNode>(T);
    w->s_mval = salloc<int>(T);
    w->s_left = salloc<int>(T);
    w->s_right = salloc<int>(T);
    w->s_parent = salloc<int>(T);
    w->s_leaf_parent = salloc<int>(T);
    w->s_visits = salloc<int>(T);
    w->since_build.assign(h->model.meshes.size(), 0);
    h->d.self_ws = w;
  } catch (const std::exception& e) {
    h->err = e.what();
    return PDF_CUDA_ERROR;
  }
  return PDF_OK;
}

void self_detect_free(pdf_handle* h) {
  if (!h->d.self_ws) return;
  SelfWS* w = (SelfWS*)h->d.self_ws;
  ws_free(*w);
  delete w;
  h->d.self_ws = nullptr;
}

int self_detect_step(pdf_handle* h) {
  SelfWS& w = *(SelfWS*)h->d.self_ws;
  cudaStream_t st = h->stream;
  DContacts& c = h->d.c;
  // PhysicScene::getSelfCollisionsInfo(tol^2) -> checkMeshSelfCollisions(mesh, sqrt(tol^2))
  const double tol2 = h->prm.self_collision_tolerance * h->prm.self_collision_tolerance;
  const double tol = std::sqrt(tol2);
  CKS(cudaMemsetAsync(c.n_self, 0, sizeof(int), st));
  k_reset_registered<<<64, 256, 0, st>>>(w.reg_n, w.touched, w.n_touched);
  CKS(cudaMemsetAsync(w.n_touched, 0, sizeof(int), st));
  // no host round trip: counts stay on the device, errors go to the handle's
  // error word (read at the end of pdf_step)
  for (size_t mi = 0; mi < h->model.meshes.size(); ++mi) {
    const auto& md = h->model.meshes[mi];
    const int* mtris = h->d.tris + 3 * (size_t)md.triangle_offset;
    // the hierarchy only steers the search: its boxes are refit exactly every
    // step, so rebuilding it every step or every k steps finds the same set
    int& since = w.since_build[mi];
    const bool rebuild = since == 0 || since >= kRebuildEvery;
    since = rebuild ? 1 : since + 1;
    detect_mesh_step(w, h->d.q, mtris, md.vertex_offset, md.n_vertices, md.n_triangles, md.triangle_offset, rebuild,
                     tol, st, h->d.sync.err);
    const double mu = h->model.friction[(size_t)md.material * h->model.n_materials + md.material];
    k_pair<<<1, 1, 0, st>>>(0, w.hkey2, w.hval2, w.hbary, h->d.q, mtris, md.vertex_offset, h->d.ring_ptr,
                            h->d.ring_idx, mu, w.reg, w.reg_n, w.touched, w.n_touched, h->model.N, c, w.err, w.n_total,
                            h->d.sync.err);
  }
  k_self_bases<<<64, 256, 0, st>>>(c);
  return PDF_OK;
}

void self_levels_step(pdf_handle* h) {
  SelfWS& w = *(SelfWS*)h->d.self_ws;
  k_levels<<<1, 1024, 0, h->stream>>>(h->d.c, w.deg, w.uf, w.dist, w.seed, w.cobst, w.cdeg1, w.cmin, w.elev,
                                      w.lcount, h->cap_self);
}

int standalone_candidates(const double* pos, int nv, const int* tris, int nt, double tol, int* pairs, int cap, int* n,
                          int device, std::string& err) {
  if (!pos || nv <= 0 || nt <= 0 || !tris) {
    err = "invalid mesh";
    return PDF_INVALID_ARG;
  }
  CKS(cudaSetDevice(device));
  SelfWS w;
  double* dq = salloc<double>(3 * (size_t)nv);
  int* dt = salloc<int>(3 * (size_t)nt);
  int status = PDF_OK;
  try {
    CKS(cudaMemcpy(dq, pos, 3 * sizeof(double) * nv, cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(dt, tris, 3 * sizeof(int) * nt, cudaMemcpyHostToDevice));
    int hit_cap = std::max(1024, cap);
    ws_alloc(w, nv, nt, hit_cap, nv);
    int nh = detect_mesh(w, dq, dt, 0, nv, nt, tol, 0, 0);
    if (n) *n = nh;
    if (nh > hit_cap || nh > cap) {
      err = "candidate buffer too small";
      status = PDF_CAPACITY_EXCEEDED;
    } else if (pairs && nh > 0) {
      std::vector<unsigned long long> keys(nh);
      CKS(cudaMemcpy(keys.data(), w.hkey2, nh * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
      for (int k = 0; k < nh; ++k) {
        pairs[2 * k] = (int)(keys[k] >> 32);
        pairs[2 * k + 1] = (int)(keys[k] & 0xffffffffu);
      }
    }
  } catch (...) {
    ws_free(w);
    cudaFree(dq);
    cudaFree(dt);
    throw;
  }
  ws_free(w);
  cudaFree(dq);
  cudaFree(dt);
  return status;
}

int standalone_self(const double* pos, int nv, const int* tris, int nt, double tol, pdf_contact* out, int cap, int* n,
                    int device, std::string& err) {
  if (!pos || nv <= 0 || nt <= 0 || !tris) {
    err = "invalid mesh";
    return PDF_INVALID_ARG;
  }
  // a one-mesh scene: rings from the triangles
  std::vector<std::vector<int>> nb(nv);
  for (int t = 0; t < nt; ++t)
    for (int k = 0; k < 3; ++k) {
      int a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
      if (a < 0 || a >= nv || b < 0 || b >= nv) {
        err = "triangle index out of range";
        return PDF_INVALID_ARG;
      }
      nb[a].push_back(b);
      nb[b].push_back(a);
    }
  std::vector<int> rp(nv + 1, 0), ri;
  for (int v = 0; v < nv; ++v) {
    std::sort(nb[v].begin(), nb[v].end());
    nb[v].erase(std::unique(nb[v].begin(), nb[v].end()), nb[v].end());
    rp[v + 1] = rp[v] + (int)nb[v].size();
    ri.insert(ri.end(), nb[v].begin(), nb[v].end());
  }
  CKS(cudaSetDevice(device));
  SelfWS w;
  std::vector<void*> mem;
  auto track = [&](void* p) {
    mem.push_back(p);
    return p;
  };
  int status = PDF_OK;
  try {
    double* dq = (double*)track(salloc<double>(3 * (size_t)nv));
    int* dt = (int*)track(salloc<int>(3 * (size_t)nt));
    int* drp = (int*)track(salloc<int>(nv + 1));
    int* dri = (int*)track(salloc<int>(ri.size()));
    CKS(cudaMemcpy(dq, pos, 3 * sizeof(double) * nv, cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(dt, tris, 3 * sizeof(int) * nt, cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(drp, rp.data(), sizeof(int) * (nv + 1), cudaMemcpyHostToDevice));
    if (!ri.empty()) CKS(cudaMemcpy(dri, ri.data(), sizeof(int) * ri.size(), cudaMemcpyHostToDevice));
    const int scap = std::max(1, 2 * nv);
    DContacts c{};
    c.cap = 1;
    c.n_self = (int*)track(salloc<int>(1));
    c.s_vertex = (int*)track(salloc<int>(scap));
    c.s_partner = (int*)track(salloc<int>(scap));
    c.s_face = (int*)track(salloc<int>(3 * (size_t)scap));
    c.s_normal = (double*)track(salloc<double>(3 * (size_t)scap));
    c.s_mu = (double*)track(salloc<double>(scap));
    c.self_cap = scap;
    CKS(cudaMemset(c.n_self, 0, sizeof(int)));
    ws_alloc(w, nv, nt, std::max(1024, 4 * nv), nv);
    ws_alloc_pairing(w, nv, 1, 1);
    int nh = detect_mesh(w, dq, dt, 0, nv, nt, tol, 1, 0);
    if (nh > w.hit_cap) {
      err = "hit buffer too small";
      status = PDF_CAPACITY_EXCEEDED;
    } else {
      if (nh > 0)
        k_pair<<<1, 1>>>(nh, w.hkey2, w.hval2, w.hbary, dq, dt, 0, drp, dri, 0., w.reg, w.reg_n, w.touched,
                         w.n_touched, nv, c, w.err);
      int S = 0, e2 = 0;
      CKS(cudaMemcpy(&S, c.n_self, sizeof(int), cudaMemcpyDeviceToHost));
      CKS(cudaMemcpy(&e2, w.err, sizeof(int), cudaMemcpyDeviceToHost));
      if (e2) {
        err = "pairing capacity exceeded";
        status = PDF_CAPACITY_EXCEEDED;
      }
      if (n) *n = S;
      if (out && status == PDF_OK) {
        const int m = std::min(S, cap);
        std::vector<int> vx(m), pa(m), fa(3 * m);
        std::vector<double> nr(3 * m);
        if (m > 0) {
          CKS(cudaMemcpy(vx.data(), c.s_vertex, m * sizeof(int), cudaMemcpyDeviceToHost));
          CKS(cudaMemcpy(pa.data(), c.s_partner, m * sizeof(int), cudaMemcpyDeviceToHost));
          CKS(cudaMemcpy(fa.data(), c.s_face, 3 * m * sizeof(int), cudaMemcpyDeviceToHost));
          CKS(cudaMemcpy(nr.data(), c.s_normal, 3 * m * sizeof(double), cudaMemcpyDeviceToHost));
        }
        for (int k = 0; k < m; ++k) {
          pdf_contact& o = out[k];
          std::memset(&o, 0, sizeof(o));
          o.vertex = vx[k];
          o.partner = pa[k];
          for (int j = 0; j < 3; ++j) {
            o.face[j] = fa[3 * k + j];
            o.normal[j] = nr[3 * k + j];
          }
        }
        if (S > cap) {
          err = "output buffer too small";
          status = PDF_CAPACITY_EXCEEDED;
        }
      }
    }
  } catch (...) {
    ws_free(w);
    for (void* p : mem) cudaFree(p);
    throw;
  }
  ws_free(w);
  for (void* p : mem) cudaFree(p);
  return status;
}

// ---------------------------------------------------------------------------
// Allocation-free candidate detection (pdf_detect_candidates_noalloc).
//
// Some callers cannot allocate device memory at the point where they need
// the candidate pairs: code running inside another framework's memory pool
// that must not grow the process footprint, real-time loops with a fixed
// memory budget that forbid cudaMalloc/cudaFree after start-up, and hosts whose
// allocator is not the CUDA runtime's.  For them the whole workspace of the
// detection (LBVH boxes and nodes, Morton keys, candidate keys, radix-sort
// temporary storage) lives in one file-scope device array of fixed size.
// Every GPU that loads this library holds that array until the process exits.
constexpr int kNoAllocMaxTriangles = 65536;
constexpr int kNoAllocMaxPairs = 262144;
constexpr size_t kNoAllocSortBytes = size_t(8) << 20;
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
// byte layout of the array (each block 256-byte aligned)
constexpr size_t kTriBytes = align256(sizeof(double) * 3 * kNoAllocMaxTriangles);      // tlo, thi, nlo, nhi
constexpr size_t kTriKeyBytes = align256(sizeof(unsigned long long) * kNoAllocMaxTriangles);  // mkey, mkey2
constexpr size_t kTriIntBytes = align256(sizeof(int) * kNoAllocMaxTriangles);  // mval, mval2, left, right, parent, leaf_parent, visits
constexpr size_t kPairKeyBytes = align256(sizeof(unsigned long long) * kNoAllocMaxPairs);  // hkey, hkey2
constexpr size_t kPairIntBytes = align256(sizeof(int) * kNoAllocMaxPairs);                  // hval, hval2
constexpr size_t kPairBaryBytes = align256(sizeof(double) * 3 * kNoAllocMaxPairs);          // hbary (unused in mode 0)
constexpr size_t kSmallBytes = 256 * 3;                                                     // bbox, n_hits, err
constexpr size_t kNoAllocScratchBytes = 4 * kTriBytes + 2 * kTriKeyBytes + 7 * kTriIntBytes + 2 * kPairKeyBytes +
                                        2 * kPairIntBytes + kPairBaryBytes + kSmallBytes + kNoAllocSortBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

__global__ void k_keys_to_pairs(int n, const unsigned long long* __restrict__ keys, int* __restrict__ pairs) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  pairs[2 * k] = (int)(keys[k] >> 32);
  pairs[2 * k + 1] = (int)(keys[k] & 0xffffffffu);
}

int noalloc_candidates(const double* positions, int nv, const int* triangles, int nt, double tol, int* pairs,
                       int cap, int* n_out, cudaStream_t st, std::string& err) {
  if (!positions || !triangles || nv <= 0 || nt <= 0 || cap < 0 || !n_out) {
    err = "invalid arguments";
    return PDF_INVALID_ARG;
  }
  if (nt > kNoAllocMaxTriangles) {
    err = "pdf_detect_candidates_noalloc handles at most " + std::to_string(kNoAllocMaxTriangles) +
          " triangles (got " + std::to_string(nt) + ")";
    return PDF_CAPACITY_EXCEEDED;
  }
  // Set-up, repeated on every call with the caller's device current: the
  // array's device address on this device (the name is only a host-side
  // stand-in; cudaGetSymbolAddress allocates nothing) and the check that the
  // radix sort's workspace fits the reserved block.  Looking the address up on
  // every call keeps it valid after a cudaDeviceReset and needs no lock when
  // several host threads call.
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    err = std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e);
    return PDF_CUDA_ERROR;
  }
  size_t b1 = 0, b2 = 0;
  CKS(cub::DeviceRadixSort::SortPairs(nullptr, b1, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                      (int*)nullptr, (int*)nullptr, kNoAllocMaxTriangles));
  CKS(cub::DeviceRadixSort::SortPairs(nullptr, b2, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                      (int*)nullptr, (int*)nullptr, kNoAllocMaxPairs));
  if (std::max(b1, b2) > kNoAllocSortBytes) {
    err = "radix-sort workspace larger than the reserved scratch";
    return PDF_CAPACITY_EXCEEDED;
  }
  unsigned char* base = (unsigned char*)p;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char* q = base + off;
    off += bytes;
    return q;
  };
  SelfWS w;
  w.max_nt = nt;
  w.max_nv = nv;
  w.hit_cap = kNoAllocMaxPairs;
  w.tlo = (double*)take(kTriBytes);
  w.thi = (double*)take(kTriBytes);
  w.nlo = (double*)take(kTriBytes);
  w.nhi = (double*)take(kTriBytes);
  w.mkey = (unsigned long long*)take(kTriKeyBytes);
  w.mkey2 = (unsigned long long*)take(kTriKeyBytes);
  w.mval = (int*)take(kTriIntBytes);
  w.mval2 = (int*)take(kTriIntBytes);
  w.left = (int*)take(kTriIntBytes);
  w.right = (int*)take(kTriIntBytes);
  w.parent = (int*)take(kTriIntBytes);
  w.leaf_parent = (int*)take(kTriIntBytes);
  w.visits = (int*)take(kTriIntBytes);
  w.hkey = (unsigned long long*)take(kPairKeyBytes);
  w.hkey2 = (unsigned long long*)take(kPairKeyBytes);
  w.hval = (int*)take(kPairIntBytes);
  w.hval2 = (int*)take(kPairIntBytes);
  w.hbary = (double*)take(kPairBaryBytes);
  w.bbox = (unsigned long long*)take(256);
  w.n_hits = (int*)take(256);
  w.err = (int*)take(256);
  w.cub_tmp = take(kNoAllocSortBytes);
  w.cub_bytes = kNoAllocSortBytes;
  const int nh = detect_mesh(w, positions, triangles, 0, nv, nt, tol, 0, st);
  *n_out = nh;
  if (nh > kNoAllocMaxPairs || nh > cap) {
    err = "candidate pairs exceed the output capacity or the scratch limit (" + std::to_string(kNoAllocMaxPairs) + ")";
    return PDF_CAPACITY_EXCEEDED;
  }
  if (nh > 0) k_keys_to_pairs<<<(nh + 255) / 256, 256, 0, st>>>(nh, w.hkey2, pairs);
  CKS(cudaGetLastError());
  CKS(cudaStreamSynchronize(st));
  return PDF_OK;
}

}  // namespace pdfb

extern "C" int pdf_detect_candidates_noalloc(const double* positions, int32_t n_vertices, const int32_t* triangles,
                                             int32_t n_triangles, double tolerance, int32_t* pairs, int32_t cap,
                                             int32_t* n, void* cuda_stream) {
  std::string err;
  int st;
  try {
    st = pdfb::noalloc_candidates(positions, n_vertices, triangles, n_triangles, tolerance, pairs, cap, n,
                                  (cudaStream_t)cuda_stream, err);
  } catch (const std::overflow_error& e) {
    err = e.what();
    st = PDF_CAPACITY_EXCEEDED;
  } catch (const std::exception& e) {
    err = e.what();
    st = PDF_CUDA_ERROR;
  }
  if (st != PDF_OK) pdfb::set_global_error(err);
  return st;
}
