// sweep_kernels.cu — level-scheduled supernodal triangular sweeps for three
// right-hand sides (x, y, z), replacing the three Eigen::SimplicialLLT::solve
// calls of SimulationSpeed::solve (src/physics/SimulationSpeed.cpp:171-187).
//
// Each supernode s (columns [c0, c0+ns), rows R_s) carries
// W_s = [D^-1 ; L_R D^-1] (see factor.hpp).  A sweep over one elimination-tree
// level is one launch; a warp owns a task of consecutive rows (forward) or
// columns (backward) of one supernode, with g lanes cooperating on each
// row/column so that short rows do not idle a whole warp.
//   forward : y_s = D^-1 b_s ; b_R -= (L_R D^-1) b_s      (atomics into b_R)
//   backward: x_s = W_s^T [y_s ; -x_R]                    (gather from ancestors)
// Both read their copy of W once, coalesced (row-major for forward,
// column-major for backward).
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.hpp"

namespace pdfb {

__device__ __forceinline__ void atomic_sub3(double* p, double a, double b, double c) {
  atomicAdd(p, -a);
  atomicAdd(p + 1, -b);
  atomicAdd(p + 2, -c);
}
__device__ __forceinline__ void atomic_sub3(float* p, float a, float b, float c) {
  atomicAdd(p, -a);
  atomicAdd(p + 1, -b);
  atomicAdd(p + 2, -c);
}

template <typename T>
__device__ __forceinline__ void group_reduce(T& a, T& b, T& c, int g) {
  for (int o = g >> 1; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_sweep_forward(const SweepTask* __restrict__ tasks, int ntasks,
                                                       const SnInfo* __restrict__ sn, const int* __restrict__ rows,
                                                       const T* __restrict__ W, T* __restrict__ b,
                                                       T* __restrict__ y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= ntasks) return;
  const int lane = threadIdx.x & 31;
  const SweepTask t = tasks[warp];
  const SnInfo s = sn[t.sn];
  const int g = t.g;
  const int grp = lane / g, sub = lane % g;
  const int row = t.first + grp;
  const bool active = grp < t.count;
  T ax = 0, ay = 0, az = 0;
  if (active) {
    const int len = row < s.ns ? row + 1 : s.ns;
    const int64_t base = s.woff + (row < s.ns ? (int64_t)row * (row + 1) / 2
                                              : (int64_t)s.ns * (s.ns + 1) / 2 + (int64_t)(row - s.ns) * s.ns);
    const T* wr = W + base;
    const T* bs = b + 3 * (int64_t)s.c0;
    int j = sub;
    for (; j + 3 * g < len; j += 4 * g) {
      const T w0 = wr[j], w1 = wr[j + g], w2 = wr[j + 2 * g], w3 = wr[j + 3 * g];
      const T* b0 = bs + 3 * j;
      const T* b1 = bs + 3 * (j + g);
      const T* b2 = bs + 3 * (j + 2 * g);
      const T* b3 = bs + 3 * (j + 3 * g);
      ax += w0 * b0[0] + w1 * b1[0] + w2 * b2[0] + w3 * b3[0];
      ay += w0 * b0[1] + w1 * b1[1] + w2 * b2[1] + w3 * b3[1];
      az += w0 * b0[2] + w1 * b1[2] + w2 * b2[2] + w3 * b3[2];
    }
    for (; j < len; j += g) {
      const T w = wr[j];
      ax += w * bs[3 * j];
      ay += w * bs[3 * j + 1];
      az += w * bs[3 * j + 2];
    }
  }
  group_reduce(ax, ay, az, g);
  if (active && sub == 0) {
    if (row < s.ns) {
      T* o = y + 3 * ((int64_t)s.c0 + row);
      o[0] = ax;
      o[1] = ay;
      o[2] = az;
    } else {
      atomic_sub3(b + 3 * (int64_t)rows[s.roff + row - s.ns], ax, ay, az);
    }
  }
}

// mode 0: v[perm] = x (direct FP64 solve); mode 1: v[perm] += x (increment).
template <typename T>
__global__ void __launch_bounds__(256) k_sweep_backward(const SweepTask* __restrict__ tasks, int ntasks,
                                                        const SnInfo* __restrict__ sn, const int* __restrict__ rows,
                                                        const T* __restrict__ W, const T* __restrict__ y,
                                                        T* __restrict__ x, const int* __restrict__ perm,
                                                        double* __restrict__ v, double* __restrict__ qk,
                                                        const double* __restrict__ q, double dt, int mode) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= ntasks) return;
  const int lane = threadIdx.x & 31;
  const SweepTask t = tasks[warp];
  const SnInfo s = sn[t.sn];
  const int g = t.g;
  const int grp = lane / g, sub = lane % g;
  const int col = t.first + grp;
  const bool active = grp < t.count;
  T ax = 0, ay = 0, az = 0;
  if (active) {
    const int nd = s.ns - col;  // entries of D^-1 in this column
    const int len = nd + s.nr;
    const int64_t base = s.woff + (int64_t)col * (s.ns + s.nr) - (int64_t)col * (col - 1) / 2;
    const T* wc = W + base;
    const T* ys = y + 3 * ((int64_t)s.c0 + col);
    const int* rr = rows + s.roff - nd;
    for (int k = sub; k < len; k += g) {
      const T w = wc[k];
      if (k < nd) {
        ax += w * ys[3 * k];
        ay += w * ys[3 * k + 1];
        az += w * ys[3 * k + 2];
      } else {
        const T* xr = x + 3 * (int64_t)rr[k];
        ax -= w * xr[0];
        ay -= w * xr[1];
        az -= w * xr[2];
      }
    }
  }
  group_reduce(ax, ay, az, g);
  if (active && sub == 0) {
    const int64_t pc = (int64_t)s.c0 + col;
    T* o = x + 3 * pc;
    o[0] = ax;
    o[1] = ay;
    o[2] = az;
    const int64_t vtx = perm[pc];
    double vx = (double)ax, vy = (double)ay, vz = (double)az;
    if (mode == 1) {
      vx += v[3 * vtx];
      vy += v[3 * vtx + 1];
      vz += v[3 * vtx + 2];
    }
    v[3 * vtx] = vx;
    v[3 * vtx + 1] = vy;
    v[3 * vtx + 2] = vz;
    qk[3 * vtx] = q[3 * vtx] + dt * vx;
    qk[3 * vtx + 1] = q[3 * vtx + 1] + dt * vy;
    qk[3 * vtx + 2] = q[3 * vtx + 2] + dt * vz;
  }
}

template __global__ void k_sweep_forward<double>(const SweepTask*, int, const SnInfo*, const int*, const double*,
                                                 double*, double*);
template __global__ void k_sweep_forward<float>(const SweepTask*, int, const SnInfo*, const int*, const float*,
                                                float*, float*);
template __global__ void k_sweep_backward<double>(const SweepTask*, int, const SnInfo*, const int*, const double*,
                                                  const double*, double*, const int*, double*, double*,
                                                  const double*, double, int);
template __global__ void k_sweep_backward<float>(const SweepTask*, int, const SnInfo*, const int*, const float*,
                                                 const float*, float*, const int*, double*, double*,
                                                 const double*, double, int);

}  // namespace pdfb
