// sweep_kernels.cu — supernodal triangular sweeps for three right-hand sides
// (x, y, z), replacing the three Eigen::SimplicialLLT::solve calls of
// SimulationSpeed::solve (src/physics/SimulationSpeed.cpp:171-187).
//
// Each supernode s (columns [c0, c0+ns), rows R_s) carries
// W_s = [D^-1 ; L_R D^-1] (see factor.hpp) in 32-lane tiles.  A sweep is ONE
// persistent launch: warps take work items from a queue in elimination-tree
// order and wait (bounded spin) only for the supernodes they depend on, so
// independent subtrees and tree levels overlap instead of being separated by
// kernel boundaries.
//   forward : y_s = D^-1 b_s ; b_R -= (L_R D^-1) b_s   (a work item: one row tile
//             x one column chunk; partial sums land in y / b_R with atomics);
//             s may start once all its children are complete.
//   backward: x_s = W_s^T [y_s ; -x_R]                 (a work item: one column
//             tile x one row chunk; partial sums land in x with atomics);
//             s may start once its parent is complete.
// Every element of W is read once per sweep with one coalesced 32-lane load;
// the vector entries a tile needs are loaded 32 at a time and broadcast by
// warp shuffles.  Vectors that other warps update during the sweep are read
// through L2 (ld.global.cg) so that no stale L1 line is used.
// Completion counters are cumulative over solves: supernode s has finished
// solve number e when its counter reaches e * (work items of s).  A wait that
// exceeds kMaxSpins sets the error flag and gives up instead of hanging.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.hpp"

namespace pdfb {

constexpr int kMaxSpins = 1 << 22;
constexpr int kTicketBatch = 2;

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}

__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

// Release / acquire fence at device scope (lighter than the sequentially
// consistent __threadfence()).
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// lane 0 waits until *ctr >= target; false (and error flag set) on timeout
__device__ __forceinline__ bool wait_counter(const unsigned long long* ctr, unsigned long long target, int* err) {
  int spins = 0;
  while (ld_volatile_u64(ctr) < target) {
    if (++spins > kMaxSpins) {
      atomicOr(err, 1);
      return false;
    }
    __nanosleep(32);
  }
  fence_acq_rel_gpu();
  return true;
}

// Issues the (up to) 32 loads of one 32-wide slab of a tile: lane l reads
// element (l, u) at p[stride u]; absent columns (u >= m) and lanes outside the
// tile (act false) read as zero.
template <typename T>
__device__ __forceinline__ void load_tile(T (&w)[32], const T* p, int m, int stride = kTile, bool act = true) {
#pragma unroll
  for (int u = 0; u < 32; ++u) w[u] = (act && u < m) ? __ldg(p + u * stride) : T(0);
}

template <typename T>
__global__ void __launch_bounds__(256) k_sweep_forward(const SweepTask* __restrict__ tasks, int ntasks,
                                                       const SnInfo* __restrict__ sn, const int* __restrict__ rows,
                                                       const T* __restrict__ W, T* b, T* y, int n, SweepSync sy) {
  trace_stamp(sy.trace, DTrace::kSolve);
  const int lane = threadIdx.x & 31;
  const unsigned long long ep = *reinterpret_cast<const volatile unsigned long long*>(sy.epoch);
  // tickets are taken kTicketBatch at a time and processed in order: every
  // item with a smaller ticket is held by a running warp, so the waits below
  // always end
  int t = 0, tend = 0;
  for (;; ++t) {
    if (t >= tend) {
      if (lane == 0) t = atomicAdd(sy.queue + 0, kTicketBatch);
      t = __shfl_sync(0xffffffffu, t, 0);
      tend = t + kTicketBatch;
    }
    if (t >= ntasks) return;
    const SweepTask tk = tasks[t];
    const SnInfo s = sn[tk.sn];
    // the factor does not depend on the wait: its first 32 tile columns are
    // already in flight while lane 0 checks the children
    const int mrows = min(kTile, s.ns + s.nr - tk.tile * kTile);
    const T* wbase = W + tk.off + lane;
    T w[32];
    load_tile(w, wbase + (int64_t)tk.a0 * mrows, min(32, tk.a1 - tk.a0), mrows, lane < mrows);
    int ok = 1;
    if (lane == 0 && s.nchild > 0) ok = wait_counter(sy.fchild + tk.sn, ep * (unsigned long long)s.nchild, sy.err);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    const int row = tk.tile * kTile + lane;
    T ax = 0, ay = 0, az = 0;
    if (ok) {
      const T* bx = b + s.c0;
      const T* by = bx + n;
      const T* bz = by + n;
      for (int j0 = tk.a0; j0 < tk.a1; j0 += 32) {
        const int jl = j0 + lane;
        if (j0 != tk.a0) load_tile(w, wbase + (int64_t)j0 * mrows, min(32, tk.a1 - j0), mrows, lane < mrows);
        T vx = 0, vy = 0, vz = 0;
        if (jl < tk.a1) {
          vx = ldcg(bx + jl);
          vy = ldcg(by + jl);
          vz = ldcg(bz + jl);
        }
#pragma unroll
        for (int u = 0; u < 32; ++u) {
          ax += w[u] * __shfl_sync(0xffffffffu, vx, u);
          ay += w[u] * __shfl_sync(0xffffffffu, vy, u);
          az += w[u] * __shfl_sync(0xffffffffu, vz, u);
        }
      }
      if (row < s.ns) {
        const int64_t o = (int64_t)s.c0 + row;
        atomicAdd(y + o, ax);
        atomicAdd(y + o + n, ay);
        atomicAdd(y + o + 2 * (int64_t)n, az);
      } else if (row < s.ns + s.nr) {
        const int64_t r = rows[s.roff + row - s.ns];
        atomicAdd(b + r, -ax);
        atomicAdd(b + r + n, -ay);
        atomicAdd(b + r + 2 * (int64_t)n, -az);
      }
    }
    fence_acq_rel_gpu();
    __syncwarp();
    if (lane == 0) {
      const unsigned long long done = atomicAdd(sy.fdone + tk.sn, 1ULL) + 1ULL;
      if (done == ep * (unsigned long long)s.ntf && s.parent >= 0) {
        fence_acq_rel_gpu();
        atomicAdd(sy.fchild + s.parent, 1ULL);
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_sweep_backward(const SweepTask* __restrict__ tasks, int ntasks,
                                                        const SnInfo* __restrict__ sn, const int* __restrict__ rows,
                                                        const T* __restrict__ W, const T* __restrict__ y, T* x, int n,
                                                        SweepSync sy) {
  const int lane = threadIdx.x & 31;
  const unsigned long long ep = *reinterpret_cast<const volatile unsigned long long*>(sy.epoch);
  int t = 0, tend = 0;
  for (;; ++t) {
    if (t >= tend) {
      if (lane == 0) t = atomicAdd(sy.queue + 1, kTicketBatch);
      t = __shfl_sync(0xffffffffu, t, 0);
      tend = t + kTicketBatch;
    }
    if (t >= ntasks) return;
    const SweepTask tk = tasks[t];
    const SnInfo s = sn[tk.sn];
    const int mcols = min(kTile, s.ns - tk.tile * kTile);
    const T* wbase = W + tk.off + lane;
    T w[32];
    load_tile(w, wbase + (int64_t)tk.a0 * mcols, min(32, tk.a1 - tk.a0), mcols, lane < mcols);
    int ok = 1;
    if (lane == 0 && s.parent >= 0)
      ok = wait_counter(sy.bdone + s.parent, ep * (unsigned long long)sn[s.parent].ntb, sy.err);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    const int j0t = tk.tile * kTile;
    const int col = j0t + lane;
    const int nd = s.ns - j0t;  // local rows belonging to D^-1
    T ax = 0, ay = 0, az = 0;
    if (ok) {
      for (int i0 = tk.a0; i0 < tk.a1; i0 += 32) {
        const int il = i0 + lane;
        if (i0 != tk.a0) load_tile(w, wbase + (int64_t)i0 * mcols, min(32, tk.a1 - i0), mcols, lane < mcols);
        T vx = 0, vy = 0, vz = 0;
        if (il < tk.a1) {
          if (il < nd) {
            const int64_t o = (int64_t)s.c0 + j0t + il;
            vx = y[o];
            vy = y[o + n];
            vz = y[o + 2 * (int64_t)n];
          } else {
            const int64_t r = rows[s.roff + il - nd];
            vx = -ldcg(x + r);
            vy = -ldcg(x + r + n);
            vz = -ldcg(x + r + 2 * (int64_t)n);
          }
        }
#pragma unroll
        for (int u = 0; u < 32; ++u) {
          ax += w[u] * __shfl_sync(0xffffffffu, vx, u);
          ay += w[u] * __shfl_sync(0xffffffffu, vy, u);
          az += w[u] * __shfl_sync(0xffffffffu, vz, u);
        }
      }
      if (col < s.ns) {
        const int64_t o = (int64_t)s.c0 + col;
        atomicAdd(x + o, ax);
        atomicAdd(x + o + n, ay);
        atomicAdd(x + o + 2 * (int64_t)n, az);
      }
    }
    fence_acq_rel_gpu();
    __syncwarp();
    if (lane == 0) atomicAdd(sy.bdone + tk.sn, 1ULL);
  }
}

// After the backward sweep: v[perm] = x (mode 0) or v[perm] += x (mode 1),
// q^k = q_n + dt v; x and y are cleared for the next solve; one thread
// rewinds the work queues and advances the solve counter.
template <typename T>
__global__ void k_solve_post(int n, const int* __restrict__ perm, T* x, T* y, double* __restrict__ v,
                             double* __restrict__ qk, const double* __restrict__ q, double dt, int mode, SweepSync sy) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int64_t vtx = perm[k];
    double vv[3];
    for (int c = 0; c < 3; ++c) {
      const int64_t o = k + (int64_t)c * n;
      vv[c] = (double)x[o];
      x[o] = 0;
      y[o] = 0;
    }
    for (int c = 0; c < 3; ++c) {
      double val = vv[c];
      if (mode == 1) val += v[3 * vtx + c];
      v[3 * vtx + c] = val;
      qk[3 * vtx + c] = q[3 * vtx + c] + dt * val;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sy.queue[0] = 0;
    sy.queue[1] = 0;
    *sy.epoch += 1ULL;
  }
}

// Clears the solve vectors and rewinds the queues (first use / timing runs).
template <typename T>
__global__ void k_solve_prep(int n, T* x, T* y, SweepSync sy) {
  for (int64_t k = blockIdx.x * blockDim.x + threadIdx.x; k < 3 * (int64_t)n; k += gridDim.x * blockDim.x) {
    x[k] = 0;
    y[k] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sy.queue[0] = 0;
    sy.queue[1] = 0;
  }
}

// Persistent grid: as many CTAs as can be resident at once.
template <typename K>
int resident_ctas(K kernel) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
  return std::max(1, per_sm) * sms;
}

template <typename T>
void launch_solve_sweeps(cudaStream_t st, const SweepTask* ftasks, int nf, const SweepTask* btasks, int nb,
                         const SnInfo* sn, const int* rows, const T* Wf, const T* Wb, T* b, T* y, T* x, int n,
                         SweepSync sy) {
  static const int gf = resident_ctas(k_sweep_forward<T>);
  static const int gb = resident_ctas(k_sweep_backward<T>);
  k_sweep_forward<T><<<std::min(gf, (nf + 7) / 8), 256, 0, st>>>(ftasks, nf, sn, rows, Wf, b, y, n, sy);
  k_sweep_backward<T><<<std::min(gb, (nb + 7) / 8), 256, 0, st>>>(btasks, nb, sn, rows, Wb, y, x, n, sy);
}
template <typename T>
void launch_solve_post(cudaStream_t st, int n, const int* perm, T* x, T* y, double* v, double* qk, const double* q,
                       double dt, int mode, SweepSync sy) {
  k_solve_post<T><<<std::min(148 * 4, (n + 255) / 256), 256, 0, st>>>(n, perm, x, y, v, qk, q, dt, mode, sy);
}
template <typename T>
void launch_solve_prep(cudaStream_t st, int n, T* x, T* y, SweepSync sy) {
  k_solve_prep<T><<<std::min(148 * 4, (3 * n + 255) / 256), 256, 0, st>>>(n, x, y, sy);
}

template void launch_solve_sweeps<double>(cudaStream_t, const SweepTask*, int, const SweepTask*, int, const SnInfo*,
                                          const int*, const double*, const double*, double*, double*, double*, int,
                                          SweepSync);
template void launch_solve_sweeps<float>(cudaStream_t, const SweepTask*, int, const SweepTask*, int, const SnInfo*,
                                         const int*, const float*, const float*, float*, float*, float*, int,
                                         SweepSync);
template void launch_solve_post<double>(cudaStream_t, int, const int*, double*, double*, double*, double*,
                                        const double*, double, int, SweepSync);
template void launch_solve_post<float>(cudaStream_t, int, const int*, float*, float*, double*, double*, const double*,
                                       double, int, SweepSync);
template void launch_solve_prep<double>(cudaStream_t, int, double*, double*, SweepSync);
template void launch_solve_prep<float>(cudaStream_t, int, float*, float*, SweepSync);

}  // namespace pdfb
