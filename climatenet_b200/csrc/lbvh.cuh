// lbvh.cuh — linear BVH over triangles, shared by self-collision detection
// (selfdetect.cu) and mesh-obstacle detection (detect_kernels.cu): Morton
// codes of the triangle boxes' centres, radix sort (by the caller, with CUB),
// Karras (2012) hierarchy, and a bottom-up refit into node records that hold
// both children's boxes.  Node boxes are exact unions of the triangles' own
// bounding boxes (tri_box), so a traversal with a closed query box finds
// exactly the triangles whose boxes overlap it, whatever the tree's shape.
// Everything here has internal linkage: each including source gets its own
// copy of the kernels.
#pragma once
#include <cuda/atomic>

#include "device.cuh"
#include "geometry.cuh"

namespace pdfb {
namespace {

// LBVH node: both children's boxes and ids in one 112-byte
// record, so a traversal tests both children with one node load.  Child id
// >= 0: internal node; < 0: ~triangle (leaf).
struct __align__(16) WNode {
  double b[12];  // child 0 lo xyz, hi xyz; child 1 lo xyz, hi xyz
  int ch[2];
  int pad[2];
};
static_assert(sizeof(WNode) == 112, "WNode is read as seven 16-byte vectors");

__device__ __forceinline__ unsigned long long ord_bits(double x) {
  // order-preserving map of doubles to unsigned integers
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u & 0x8000000000000000ULL) ? ~u : (u | 0x8000000000000000ULL);
}
__device__ __forceinline__ double from_ord(unsigned long long u) {
  u = (u & 0x8000000000000000ULL) ? (u & 0x7fffffffffffffffULL) : ~u;
  return __longlong_as_double((long long)u);
}

// Bounding box of the vertices (order-preserving integer images of the
// coordinates): warp and block reductions, then one atomic per block and bound.
__global__ void k_bbox(int nv, const double* __restrict__ q, unsigned long long* bbox) {
  __shared__ unsigned long long red[6][32];
  unsigned long long v[6] = {~0ULL, ~0ULL, ~0ULL, 0ULL, 0ULL, 0ULL};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
    for (int c = 0; c < 3; ++c) {
      unsigned long long u = ord_bits(q[3 * (int64_t)i + c]);
      v[c] = min(v[c], u);
      v[3 + c] = max(v[3 + c], u);
    }
  for (int o = 16; o > 0; o >>= 1)
    for (int c = 0; c < 3; ++c) {
      v[c] = min(v[c], __shfl_xor_sync(0xffffffffu, v[c], o));
      v[3 + c] = max(v[3 + c], __shfl_xor_sync(0xffffffffu, v[3 + c], o));
    }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (lane == 0)
    for (int c = 0; c < 6; ++c) red[c][warp] = v[c];
  __syncthreads();
  if (threadIdx.x < 6) {
    const int c = threadIdx.x;
    unsigned long long r = red[c][0];
    for (int k = 1; k < nw; ++k) r = c < 3 ? min(r, red[c][k]) : max(r, red[c][k]);
    if (c < 3)
      atomicMin(bbox + c, r);
    else
      atomicMax(bbox + c, r);
  }
}

__device__ __forceinline__ unsigned int spread10(unsigned int v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

// Leaf boxes and Morton keys (key = morton << 32 | triangle, unique).
__global__ void k_tri_keys(int nt, const double* __restrict__ q, const int* __restrict__ tris, int v0,
                           const unsigned long long* __restrict__ bbox, double* tlo, double* thi,
                           unsigned long long* key, int* val) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const double3 a = ld3(q, tris[3 * t]), b = ld3(q, tris[3 * t + 1]), c = ld3(q, tris[3 * t + 2]);
  double3 lo, hi;
  tri_box(a, b, c, &lo, &hi);
  st3(tlo, t, lo);
  st3(thi, t, hi);
  (void)v0;
  const double bl[3] = {from_ord(bbox[0]), from_ord(bbox[1]), from_ord(bbox[2])};
  const double bh[3] = {from_ord(bbox[3]), from_ord(bbox[4]), from_ord(bbox[5])};
  const double cc[3] = {(lo.x + hi.x) * 0.5, (lo.y + hi.y) * 0.5, (lo.z + hi.z) * 0.5};
  unsigned int code = 0;
  for (int k = 0; k < 3; ++k) {
    const double ext = bh[k] - bl[k];
    double u = ext > 0 ? (cc[k] - bl[k]) / ext : 0.;
    u = fmin(fmax(u, 0.), 1.);
    unsigned int qv = (unsigned int)fmin(u * 1024., 1023.);
    code |= spread10(qv) << (2 - k);
  }
  key[t] = ((unsigned long long)code << 32) | (unsigned int)t;
  val[t] = t;
}

__device__ __forceinline__ int delta(const unsigned long long* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  return __clzll(k[i] ^ k[j]);
}

// Karras (2012) hierarchy.  Children: >= 0 internal node, < 0 leaf ~c.
__global__ void k_build(int n, const unsigned long long* __restrict__ k, int* left, int* right, int* parent,
                        int* leaf_parent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(k, n, i, i - d);
  int lmax = 2;
  while (delta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(k, n, i, j);
  int s = 0;
  int div = 2;
  while (true) {
    const int t = (l + div - 1) / div;
    if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
    div <<= 1;
  }
  const int gamma = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int lc = (lo == gamma) ? ~gamma : gamma;
  const int rc = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
  left[i] = lc;
  right[i] = rc;
  if (lc >= 0) parent[lc] = i; else leaf_parent[~lc] = i;
  if (rc >= 0) parent[rc] = i; else leaf_parent[~rc] = i;
  if (i == 0) parent[0] = -1;
}

// Bottom-up refit into wide nodes: each finished box (a leaf's triangle box,
// or the union of a node's two children) is written into its slot of the
// parent's record; the second child to arrive at a node computes its union.
__device__ __forceinline__ void put_child(WNode* nodes, const int* left, int p, int self_id, int enc, double3 lo,
                                          double3 hi) {
  const int side = left[p] == self_id ? 0 : 1;
  double* b = nodes[p].b + 6 * side;
  __stcg(b + 0, lo.x);
  __stcg(b + 1, lo.y);
  __stcg(b + 2, lo.z);
  __stcg(b + 3, hi.x);
  __stcg(b + 4, hi.y);
  __stcg(b + 5, hi.z);
  __stcg(nodes[p].ch + side, enc);
}

// Leaf boxes come straight from the positions (a triangle's own bounding
// box, as tri_box computes it everywhere else).
__global__ void k_refit_wide(int n, const int* __restrict__ mval, const double* __restrict__ q,
                             const int* __restrict__ tris, const int* __restrict__ left, const int* __restrict__ parent,
                             const int* __restrict__ leaf_parent, WNode* nodes, int* visits) {
  const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n) return;
  const int tri = mval[leaf];
  int p = leaf_parent[leaf];
  double3 tl, th;
  tri_box(ld3(q, tris[3 * tri]), ld3(q, tris[3 * tri + 1]), ld3(q, tris[3 * tri + 2]), &tl, &th);
  put_child(nodes, left, p, ~leaf, ~tri, tl, th);
  while (p >= 0) {
    // release our child box, acquire the sibling's
    cuda::atomic_ref<int, cuda::thread_scope_device> arrivals(visits[p]);
    if (arrivals.fetch_add(1, cuda::memory_order_acq_rel) == 0) return;
    const double* b = nodes[p].b;
    double v[12];
    for (int k = 0; k < 12; ++k) v[k] = __ldcg(b + k);
    const double3 lo = make_double3(fmin(v[0], v[6]), fmin(v[1], v[7]), fmin(v[2], v[8]));
    const double3 hi = make_double3(fmax(v[3], v[9]), fmax(v[4], v[10]), fmax(v[5], v[11]));
    const int pp = parent[p];
    if (pp >= 0) put_child(nodes, left, pp, p, p, lo, hi);
    p = pp;
  }
}

}  // namespace
}  // namespace pdfb
