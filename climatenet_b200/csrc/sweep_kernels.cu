// sweep_kernels.cu — level-scheduled supernodal triangular sweeps for three
// right-hand sides (x, y, z), replacing the three Eigen::SimplicialLLT::solve
// calls of SimulationSpeed::solve (src/physics/SimulationSpeed.cpp:171-187).
//
// Each supernode s (columns [c0, c0+ns), rows R_s) carries
// W_s = [D^-1 ; L_R D^-1] (see factor.hpp).  A sweep over one elimination-tree
// level is one launch; a warp owns a task of consecutive rows (forward) or
// columns (backward) of one supernode, with g lanes cooperating on each
// row/column so that short rows do not idle a whole warp.  Warps walk the
// level's task list with a grid stride, so the grid stays a few CTAs per SM.
//   forward : y_s = D^-1 b_s ; b_R -= (L_R D^-1) b_s      (atomics into b_R)
//   backward: x_s = W_s^T [y_s ; -x_R]                    (gather from ancestors)
// Both read their copy of W once, coalesced (row-major for forward,
// column-major for backward).  The three right-hand sides are stored as three
// planes of n values (structure of arrays), so every vector access of a lane
// group is contiguous.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.hpp"

namespace pdfb {

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
                                                       T* __restrict__ y, int n) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ntasks; w += nwarps) {
    const SweepTask t = tasks[w];
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
      const T* bx = b + s.c0;
      const T* by = bx + n;
      const T* bz = by + n;
      int j = sub;
      for (; j + 3 * g < len; j += 4 * g) {
        const T w0 = wr[j], w1 = wr[j + g], w2 = wr[j + 2 * g], w3 = wr[j + 3 * g];
        ax += w0 * bx[j] + w1 * bx[j + g] + w2 * bx[j + 2 * g] + w3 * bx[j + 3 * g];
        ay += w0 * by[j] + w1 * by[j + g] + w2 * by[j + 2 * g] + w3 * by[j + 3 * g];
        az += w0 * bz[j] + w1 * bz[j + g] + w2 * bz[j + 2 * g] + w3 * bz[j + 3 * g];
      }
      for (; j < len; j += g) {
        const T wv = wr[j];
        ax += wv * bx[j];
        ay += wv * by[j];
        az += wv * bz[j];
      }
    }
    group_reduce(ax, ay, az, g);
    if (active && sub == 0) {
      if (row < s.ns) {
        const int64_t o = (int64_t)s.c0 + row;
        y[o] = ax;
        y[o + n] = ay;
        y[o + 2 * (int64_t)n] = az;
      } else {
        const int64_t r = rows[s.roff + row - s.ns];
        atomicAdd(b + r, -ax);
        atomicAdd(b + r + n, -ay);
        atomicAdd(b + r + 2 * (int64_t)n, -az);
      }
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
                                                        const double* __restrict__ q, double dt, int mode, int n) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ntasks; w += nwarps) {
    const SweepTask t = tasks[w];
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
      const T* yx = y + s.c0 + col;
      const T* yy = yx + n;
      const T* yz = yy + n;
      int k = sub;
      for (; k < nd; k += g) {
        const T wv = wc[k];
        ax += wv * yx[k];
        ay += wv * yy[k];
        az += wv * yz[k];
      }
      const int* rr = rows + s.roff - nd;
      for (; k < len; k += g) {
        const T wv = wc[k];
        const int64_t r = rr[k];
        ax -= wv * x[r];
        ay -= wv * x[r + n];
        az -= wv * x[r + 2 * (int64_t)n];
      }
    }
    group_reduce(ax, ay, az, g);
    if (active && sub == 0) {
      const int64_t pc = (int64_t)s.c0 + col;
      x[pc] = ax;
      x[pc + n] = ay;
      x[pc + 2 * (int64_t)n] = az;
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
}

// At most kSweepCtasPerSm CTAs of 8 warps per SM; warps stride over tasks.
constexpr int kSweepCtas = 148 * 8;

template <typename T>
void launch_sweep_forward(cudaStream_t st, const SweepTask* tasks, int ntasks, const SnInfo* sn, const int* rows,
                          const T* W, T* b, T* y, int n) {
  const int grid = std::min(kSweepCtas, (ntasks + 7) / 8);
  k_sweep_forward<T><<<grid, 256, 0, st>>>(tasks, ntasks, sn, rows, W, b, y, n);
}
template <typename T>
void launch_sweep_backward(cudaStream_t st, const SweepTask* tasks, int ntasks, const SnInfo* sn, const int* rows,
                           const T* W, const T* y, T* x, const int* perm, double* v, double* qk, const double* q,
                           double dt, int mode, int n) {
  const int grid = std::min(kSweepCtas, (ntasks + 7) / 8);
  k_sweep_backward<T><<<grid, 256, 0, st>>>(tasks, ntasks, sn, rows, W, y, x, perm, v, qk, q, dt, mode, n);
}
template void launch_sweep_forward<double>(cudaStream_t, const SweepTask*, int, const SnInfo*, const int*,
                                           const double*, double*, double*, int);
template void launch_sweep_forward<float>(cudaStream_t, const SweepTask*, int, const SnInfo*, const int*, const float*,
                                          float*, float*, int);
template void launch_sweep_backward<double>(cudaStream_t, const SweepTask*, int, const SnInfo*, const int*,
                                            const double*, const double*, double*, const int*, double*, double*,
                                            const double*, double, int, int);
template void launch_sweep_backward<float>(cudaStream_t, const SweepTask*, int, const SnInfo*, const int*,
                                           const float*, const float*, float*, const int*, double*, double*,
                                           const double*, double, int, int);

}  // namespace pdfb
