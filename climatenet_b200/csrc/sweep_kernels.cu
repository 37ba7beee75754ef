// sweep_kernels.cu — supernodal triangular sweeps for three right-hand sides
// (x, y, z), replacing the three Eigen::SimplicialLLT::solve calls of
// SimulationSpeed::solve (src/physics/SimulationSpeed.cpp:171-187).
//
// Each supernode s (columns [c0, c0+ns), rows R_s) carries
// W_s = [D^-1 ; L_R D^-1] (see factor.hpp) in 32-lane tiles:
//   forward : y_s = D^-1 b_s ; b_R -= (L_R D^-1) b_s
//   backward: x_s = W_s^T [y_s ; -x_R]
// A sweep is ONE persistent launch with two kinds of work (factor.hpp,
// SweepPlan):
//  * subtree blocks — the lower levels of the elimination tree, cut into
//    subtrees with contiguous columns.  One CTA solves a block alone: the
//    block's slice of the vector sits in shared memory, its levels are
//    separated by CTA barriers, each tile of each supernode is one warp's
//    item, and only rows of the block's ancestors are updated in global
//    memory.  No dependency counter is touched inside a block.
//  * upper work items — the supernodes above the blocks, split into 32-row
//    (forward) / 32-column (backward) tiles times column / row chunks, taken
//    by warps from a queue in elimination-tree order; a warp waits (bounded
//    spin) only for the supernodes its item depends on: forward, all children
//    complete (block roots signal once per block); backward, the parent
//    complete.  Partial sums land in y / b_R / x with atomics.
// The forward launch runs the blocks first (they depend on nothing), then the
// upper items; the backward launch runs the upper items first, then the
// blocks, whose write-back of v and q^k is fused in.  Every element of W is
// read once per sweep with coalesced 32-lane loads that stream past the
// caches (__ldcs); vectors other CTAs update during the sweep are read
// through L2 (ld.global.cg).  Completion counters are cumulative over solves:
// supernode s has finished solve number e when its counter reaches
// e * (its work items).  A wait that exceeds SweepSync::max_spins sets the
// error flag and gives up instead of hanging.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.cuh"
#include "kernels.hpp"

namespace pdfb {

constexpr int kTicketBatch = 2;
constexpr int kSweepThreads = 256;

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}

__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
// factor elements are read once per sweep: evict-first, so that the vectors
// stay in L2
__device__ __forceinline__ float ldw(const float* p) { return __ldcs(p); }
__device__ __forceinline__ double ldw(const double* p) { return __ldcs(p); }

// Release / acquire fence at device scope (lighter than the sequentially
// consistent __threadfence()).
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// waits until *ctr >= target; false (and error flag set) after max_spins polls
__device__ __forceinline__ bool wait_counter(const unsigned long long* ctr, unsigned long long target, int* err,
                                             int max_spins) {
  int spins = 0;
  while (ld_volatile_u64(ctr) < target) {
    if (++spins > max_spins) {
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
  for (int u = 0; u < 32; ++u) w[u] = (act && u < m) ? ldw(p + u * stride) : T(0);
}

// ---------------------------------------------------------------- blocks

// Slab width of the block tiles: 16 columns (forward) / rows (backward), so
// that a slab of W and the vector entries it multiplies fit the register
// budget of two resident CTAs per SM (32-wide slabs took 206-220 registers).
constexpr int kSlab = 16;

template <typename T>
__device__ __forceinline__ void load_slab(T (&w)[kSlab], const T* p, int m, int stride, bool act) {
#pragma unroll
  for (int u = 0; u < kSlab; ++u) w[u] = (act && u < m) ? ldw(p + u * stride) : T(0);
}

// Forward tile of a block: rows [32 tile, 32 tile + m) of W_s times the
// block's slice sv of b; y_s rows are written (each by exactly one lane), the
// R rows are subtracted from the slice (ancestors inside the block, shared
// atomics) or from b (ancestors above the block, global atomics).
template <typename T>
__device__ __forceinline__ void block_fwd_item(const BlockItem& I, int c0b, int c1b, int nc, T* sv, const T* W,
                                               T* b, T* y, const int* rows, int n, int lane) {
  const int m = min(kTile, I.ns + I.nr - kTile * I.tile);
  const int w = min(I.ns, kTile * I.tile + kTile);
  const bool act = lane < m;
  const T* wp = W + I.off + lane;
  const T* vx = sv + I.c0l;
  const T* vy = vx + nc;
  const T* vz = vy + nc;
  T ax = 0, ay = 0, az = 0;
#pragma unroll 1
  for (int j0 = 0; j0 < w; j0 += kSlab) {
    const int cnt = min(kSlab, w - j0);
    T wv[kSlab];
    load_slab(wv, wp + (int64_t)j0 * m, cnt, m, act);
    if (cnt == kSlab) {
#pragma unroll
      for (int u = 0; u < kSlab; ++u) {
        ax += wv[u] * vx[j0 + u];
        ay += wv[u] * vy[j0 + u];
        az += wv[u] * vz[j0 + u];
      }
    } else {
#pragma unroll
      for (int u = 0; u < kSlab; ++u)
        if (u < cnt) {
          ax += wv[u] * vx[j0 + u];
          ay += wv[u] * vy[j0 + u];
          az += wv[u] * vz[j0 + u];
        }
    }
  }
  const int row = kTile * I.tile + lane;
  if (row < I.ns) {
    const int64_t o = (int64_t)c0b + I.c0l + row;
    y[o] = ax;
    y[o + n] = ay;
    y[o + 2 * (int64_t)n] = az;
  } else if (row < I.ns + I.nr) {
    const int r = rows[I.roff + row - I.ns];
    if (r < c1b) {
      T* s = sv + (r - c0b);
      atomicAdd(s, -ax);
      atomicAdd(s + nc, -ay);
      atomicAdd(s + 2 * nc, -az);
    } else {
      atomicAdd(b + r, -ax);
      atomicAdd(b + r + n, -ay);
      atomicAdd(b + r + 2 * (int64_t)n, -az);
    }
  }
}

// Backward tile of a block: columns [32 tile, 32 tile + mc) of W_s (lane =
// column) over its rows: y_s from the forward sweep, then -x_R from the slice
// sx (ancestors inside the block, already final) or from x (ancestors above
// the block, final once the block's parent is).  The vector entries of a slab
// are staged in the warp's shared buffer stage[3][kSlab] and read back as
// broadcasts (fewer live registers than shuffled values).
template <typename T>
__device__ __forceinline__ void block_bwd_item(const BlockItem& I, int c0b, int c1b, int nc, T* sx, const T* W,
                                               const T* y, const T* x, const int* rows, int n, int lane,
                                               T* stage) {
  const int j0t = kTile * I.tile, nd = I.ns - j0t, mc = min(kTile, nd), h = nd + I.nr;
  const bool act = lane < mc;
  const T* wp = W + I.off + lane;
  T ax = 0, ay = 0, az = 0;
#pragma unroll 1
  for (int i0 = 0; i0 < h; i0 += kSlab) {
    const int cnt = min(kSlab, h - i0);
    T wv[kSlab];
    load_slab(wv, wp + (int64_t)i0 * mc, cnt, mc, act);
    const int il = i0 + lane;
    T vx = 0, vy = 0, vz = 0;
    if (lane < cnt) {
      if (il < nd) {
        const int64_t o = (int64_t)c0b + I.c0l + j0t + il;
        vx = y[o];
        vy = y[o + n];
        vz = y[o + 2 * (int64_t)n];
      } else {
        const int r = rows[I.roff + il - nd];
        if (r < c1b) {
          const T* s = sx + (r - c0b);
          vx = -s[0];
          vy = -s[nc];
          vz = -s[2 * nc];
        } else {
          vx = -ldcg(x + r);
          vy = -ldcg(x + r + n);
          vz = -ldcg(x + r + 2 * (int64_t)n);
        }
      }
    }
    __syncwarp();  // the previous slab's reads of stage are done
    if (lane < kSlab) {
      stage[lane] = vx;
      stage[kSlab + lane] = vy;
      stage[2 * kSlab + lane] = vz;
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < kSlab; ++u) {
      ax += wv[u] * stage[u];
      ay += wv[u] * stage[kSlab + u];
      az += wv[u] * stage[2 * kSlab + u];
    }
  }
  if (act) {
    T* s = sx + I.c0l + j0t + lane;
    s[0] = ax;
    s[nc] = ay;
    s[2 * nc] = az;
  }
}

// CTA-wide ticket: thread 0 draws, everyone reads it after the barrier.
__device__ __forceinline__ int cta_ticket(int* queue, int* slot) {
  __syncthreads();  // every thread has read the previous ticket
  if (threadIdx.x == 0) *slot = atomicAdd(queue, 1);
  __syncthreads();
  return *slot;
}

// ---------------------------------------------------------------- sweeps

template <typename T>
__global__ void __launch_bounds__(kSweepThreads) k_sweep_forward(DPlan P, const T* __restrict__ W, T* b, T* y, int n,
                                                                 SweepSync sy) {
  trace_stamp(sy.trace, DTrace::kSolve);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_ticket;
  T* sv = reinterpret_cast<T*>(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned long long ep = ld_volatile_u64(sy.epoch);
  // ---- subtree blocks
  for (;;) {
    const int bi = cta_ticket(sy.queue + 2, &s_ticket);
    if (bi >= P.nblk) break;
    const SweepBlock& B = P.fblk[bi];
    const int c0b = B.c0, c1b = B.c1, nc = c1b - c0b, item0 = B.item0, nlev = B.nlev;
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
      sv[k] = b[c0b + k];
      sv[nc + k] = b[(int64_t)n + c0b + k];
      sv[2 * nc + k] = b[2 * (int64_t)n + c0b + k];
    }
    __syncthreads();
    for (int L = 0; L < nlev; ++L) {
      const int i1 = item0 + B.lev[L + 1];
#pragma unroll 1
      for (int it = item0 + B.lev[L] + warp; it < i1; it += nw)
        block_fwd_item<T>(P.fitem[it], c0b, c1b, nc, sv, W, b, y, P.rows, n, lane);
      __syncthreads();
    }
    if (B.parent >= 0) {
      // the block's global updates of its ancestors' rows happen before the
      // parent sees the block complete
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) atomicAdd(sy.fchild + B.parent, 1ULL);
    }
  }
  // ---- upper work items.  Tickets are taken kTicketBatch at a time and
  // processed in order, the next batch drawn while the current one runs:
  // every item with a smaller ticket is held by a running warp (and every
  // block by a running CTA), so the waits below always end.
  int t = 0, tend = 0, next = 0;
  if (lane == 0) next = atomicAdd(sy.queue + 0, kTicketBatch);
  for (;; ++t) {
    if (t >= tend) {
      t = __shfl_sync(0xffffffffu, next, 0);
      tend = t + kTicketBatch;
      if (t >= P.nfup) return;
      if (lane == 0) next = atomicAdd(sy.queue + 0, kTicketBatch);
    }
    if (t >= P.nfup) return;
    const UpperItem tk = P.fup[t];
    // the factor does not depend on the wait: its first 32 tile columns are
    // already in flight while lane 0 checks the children
    const int mrows = min(kTile, tk.ns + tk.nr - tk.tile * kTile);
    const T* wbase = W + tk.off + lane;
    T w[32];
    load_tile(w, wbase + (int64_t)tk.a0 * mrows, min(32, tk.a1 - tk.a0), mrows, lane < mrows);
    int ok = 1;
    if (lane == 0 && tk.wait > 0)
      ok = wait_counter(sy.fchild + tk.sn, ep * (unsigned long long)tk.wait, sy.err, sy.max_spins);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    const int row = tk.tile * kTile + lane;
    T ax = 0, ay = 0, az = 0;
    if (ok) {
      const T* bx = b + tk.c0;
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
      if (row < tk.ns) {
        const int64_t o = (int64_t)tk.c0 + row;
        atomicAdd(y + o, ax);
        atomicAdd(y + o + n, ay);
        atomicAdd(y + o + 2 * (int64_t)n, az);
      } else if (row < tk.ns + tk.nr) {
        const int64_t r = P.rows[tk.roff + row - tk.ns];
        atomicAdd(b + r, -ax);
        atomicAdd(b + r + n, -ay);
        atomicAdd(b + r + 2 * (int64_t)n, -az);
      }
    }
    fence_acq_rel_gpu();
    __syncwarp();
    if (lane == 0) {
      const unsigned long long done = atomicAdd(sy.fdone + tk.sn, 1ULL) + 1ULL;
      if (done == ep * (unsigned long long)tk.ntf && tk.parent >= 0) {
        fence_acq_rel_gpu();
        atomicAdd(sy.fchild + tk.parent, 1ULL);
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kSweepThreads) k_sweep_backward(DPlan P, const T* __restrict__ W,
                                                                  const T* __restrict__ y, T* x, int n,
                                                                  SweepSync sy, WriteBack wb) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_ticket, s_ok;
  __shared__ T s_stage[kSweepThreads / 32][3 * kSlab];
  T* sx = reinterpret_cast<T*>(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned long long ep = ld_volatile_u64(sy.epoch);
  // ---- upper work items (top-down); tickets as in the forward sweep
  int t = 0, tend = 0, next = 0;
  if (lane == 0) next = atomicAdd(sy.queue + 1, kTicketBatch);
  for (;; ++t) {
    if (t >= tend) {
      t = __shfl_sync(0xffffffffu, next, 0);
      tend = t + kTicketBatch;
      if (t >= P.nbup) break;
      if (lane == 0) next = atomicAdd(sy.queue + 1, kTicketBatch);
    }
    if (t >= P.nbup) break;
    const UpperItem tk = P.bup[t];
    const int mcols = min(kTile, tk.ns - tk.tile * kTile);
    const T* wbase = W + tk.off + lane;
    T w[32];
    load_tile(w, wbase + (int64_t)tk.a0 * mcols, min(32, tk.a1 - tk.a0), mcols, lane < mcols);
    int ok = 1;
    if (lane == 0 && tk.parent >= 0)
      ok = wait_counter(sy.bdone + tk.parent, ep * (unsigned long long)tk.wait, sy.err, sy.max_spins);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    const int j0t = tk.tile * kTile;
    const int col = j0t + lane;
    const int nd = tk.ns - j0t;  // local rows belonging to D^-1
    T ax = 0, ay = 0, az = 0;
    if (ok) {
      for (int i0 = tk.a0; i0 < tk.a1; i0 += 32) {
        const int il = i0 + lane;
        if (i0 != tk.a0) load_tile(w, wbase + (int64_t)i0 * mcols, min(32, tk.a1 - i0), mcols, lane < mcols);
        T vx = 0, vy = 0, vz = 0;
        if (il < tk.a1) {
          if (il < nd) {
            const int64_t o = (int64_t)tk.c0 + j0t + il;
            vx = ldcg(y + o);
            vy = ldcg(y + o + n);
            vz = ldcg(y + o + 2 * (int64_t)n);
          } else {
            const int64_t r = P.rows[tk.roff + il - nd];
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
      if (col < tk.ns) {
        const int64_t o = (int64_t)tk.c0 + col;
        atomicAdd(x + o, ax);
        atomicAdd(x + o + n, ay);
        atomicAdd(x + o + 2 * (int64_t)n, az);
      }
    }
    fence_acq_rel_gpu();
    __syncwarp();
    if (lane == 0) atomicAdd(sy.bdone + tk.sn, 1ULL);
  }
  // ---- subtree blocks (top-down inside each), write-back of v and q^k
  for (;;) {
    const int bi = cta_ticket(sy.queue + 3, &s_ticket);
    if (bi >= P.nblk) break;
    const SweepBlock& B = P.bblk[bi];
    const int c0b = B.c0, c1b = B.c1, nc = c1b - c0b, item0 = B.item0, nlev = B.nlev;
    if (threadIdx.x == 0)
      s_ok = B.parent < 0 ||
             wait_counter(sy.bdone + B.parent, ep * (unsigned long long)P.sn[B.parent].ntb, sy.err, sy.max_spins);
    __syncthreads();
    if (!s_ok) continue;  // uniform: the error flag is set, the state is left as it was
    for (int L = 0; L < nlev; ++L) {
      const int i1 = item0 + B.lev[L + 1];
#pragma unroll 1
      for (int it = item0 + B.lev[L] + warp; it < i1; it += nw)
        block_bwd_item<T>(P.bitem[it], c0b, c1b, nc, sx, W, y, x, P.rows, n, lane, s_stage[warp]);
      __syncthreads();
    }
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
      const int64_t vtx = P.perm[c0b + k];
      for (int c = 0; c < 3; ++c) {
        double val = (double)sx[k + c * nc];
        if (wb.mode == 1) val += wb.v[3 * vtx + c];
        wb.v[3 * vtx + c] = val;
        wb.qk[3 * vtx + c] = wb.q[3 * vtx + c] + wb.dt * val;
      }
    }
  }
}

// After the backward sweep, for the upper supernodes' columns: v[perm] = x
// (mode 0) or v[perm] += x (mode 1), q^k = q_n + dt v, and x, y cleared for
// the next solve (the blocks' columns are written back by the backward sweep
// and their y is overwritten by the next forward sweep); one thread rewinds
// the work queues and advances the solve counter.
template <typename T>
__global__ void k_solve_post(DPlan P, T* x, T* y, int n, WriteBack wb, SweepSync sy) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P.n_upper; k += gridDim.x * blockDim.x) {
    const int col = P.upper_cols[k];
    const int64_t vtx = P.perm[col];
    for (int c = 0; c < 3; ++c) {
      const int64_t o = col + (int64_t)c * n;
      double val = (double)x[o];
      x[o] = 0;
      y[o] = 0;
      if (wb.mode == 1) val += wb.v[3 * vtx + c];
      wb.v[3 * vtx + c] = val;
      wb.qk[3 * vtx + c] = wb.q[3 * vtx + c] + wb.dt * val;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x < 4) sy.queue[threadIdx.x] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *sy.epoch += 1ULL;
}

// Clears the solve vectors and rewinds the queues (first use / timing runs).
template <typename T>
__global__ void k_solve_prep(int n, T* x, T* y, SweepSync sy) {
  for (int64_t k = blockIdx.x * blockDim.x + threadIdx.x; k < 3 * (int64_t)n; k += gridDim.x * blockDim.x) {
    x[k] = 0;
    y[k] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x < 4) sy.queue[threadIdx.x] = 0;
}

// Persistent grid: as many CTAs as can be resident at once with this dynamic
// shared memory.
template <typename K>
int resident_ctas(K kernel, size_t smem) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSweepThreads, smem);
  return std::max(1, per_sm) * sms;
}

template <typename T>
void configure_solve(DPlan& P) {
  const size_t smem = 3 * (size_t)std::max(1, P.max_cols) * sizeof(T);
  P.smem = (int)smem;
  P.grid_f = resident_ctas(k_sweep_forward<T>, smem);
  P.grid_b = resident_ctas(k_sweep_backward<T>, smem);
}

template <typename T>
void launch_solve_sweeps(cudaStream_t st, const DPlan& P, const T* Wf, const T* Wb, T* b, T* y, T* x, int n,
                         SweepSync sy, WriteBack wb) {
  k_sweep_forward<T><<<P.grid_f, kSweepThreads, P.smem, st>>>(P, Wf, b, y, n, sy);
  k_sweep_backward<T><<<P.grid_b, kSweepThreads, P.smem, st>>>(P, Wb, y, x, n, sy, wb);
  k_solve_post<T><<<std::max(1, std::min(148 * 4, (P.n_upper + 255) / 256)), 256, 0, st>>>(P, x, y, n, wb, sy);
}
template <typename T>
void launch_solve_prep(cudaStream_t st, int n, T* x, T* y, SweepSync sy) {
  k_solve_prep<T><<<std::min(148 * 4, (3 * n + 255) / 256), 256, 0, st>>>(n, x, y, sy);
}

template void configure_solve<double>(DPlan&);
template void configure_solve<float>(DPlan&);
template void launch_solve_sweeps<double>(cudaStream_t, const DPlan&, const double*, const double*, double*, double*,
                                          double*, int, SweepSync, WriteBack);
template void launch_solve_sweeps<float>(cudaStream_t, const DPlan&, const float*, const float*, float*, float*,
                                         float*, int, SweepSync, WriteBack);
template void launch_solve_prep<double>(cudaStream_t, int, double*, double*, SweepSync);
template void launch_solve_prep<float>(cudaStream_t, int, float*, float*, SweepSync);

}  // namespace pdfb
