// sweep_kernels.cu — supernodal triangular sweeps for three right-hand sides
// (x, y, z), replacing the three Eigen::SimplicialLLT::solve calls of
// SimulationSpeed::solve (src/physics/SimulationSpeed.cpp:171-187).
//
// Each supernode s (columns [c0, c0+ns), rows R_s) carries
// W_s = [D^-1 ; L_R D^-1] (see factor.hpp) in 32-lane tiles:
//   forward : y_s = D^-1 b_s ; b_R -= (L_R D^-1) b_s
//   backward: x_s = W_s^T [y_s ; -x_R]
// One solve, in launch order (factor.hpp, SweepPlan):
//  1. k_block_forward — the lower levels of the elimination tree, cut into
//     subtrees with contiguous columns ("blocks"), one CTA per block at a
//     time: the block's slice of b and its rows outside the block ("ext"
//     rows, the row set of the block's root) sit in shared memory, the
//     block's levels are separated by a barrier among the consumer warps,
//     each tile of each supernode (each span of kBlockSpanF columns /
//     kBlockSpanB rows of a longer tile, the spans meeting in atomics) is one
//     consumer warp's item, and a producer warp streams the factor through
//     bulk asynchronous copies (cp.async.bulk, global -> shared, completion
//     on an mbarrier) into a ring of slots shared by the CTA, ahead of the
//     consumers and across their level barriers (the factor does not depend
//     on the data).  The ext rows' updates are added to b with one atomic
//     each per block.
//  2. the supernodes above the blocks, forward, split into 32-row tiles x
//     column chunks: either k_upper_level_forward, one launch per
//     elimination-tree level (items spread over all warps, the launch
//     boundary ordering the levels), or k_upper_forward, one launch whose
//     warps take items from a queue in elimination-tree order and wait
//     (bounded spin) until every work item of the supernode's upper children
//     is counted (each item counts itself without reading the counter back).
//     Partial sums land in y / b_R with atomics.
//  3. the same supernodes backward, top-down, in 32-column tiles x row
//     chunks (k_upper_level_backward per level, or k_upper_backward with an
//     item waiting until its parent is complete); sums land in x.
//  4. k_block_backward — the blocks top-down: their y slice and the final x
//     of their ext rows are loaded into shared memory, the factor and, per
//     slab, the row-index list of the tile stream in as in launch 1, and x of
//     the block's columns is written back into v and q^k directly.
//  5. k_solve_post — the write-back of the upper supernodes' columns.
// The launches after the first are programmatic dependents of the one before
// them (griddepcontrol).  Completion counters are cumulative over solves:
// supernode s has finished solve number e when its counter reaches e * (its
// work items).  Every wait (counter or mbarrier) gives up after
// SweepSync::max_spins polls, sets the error flag and returns instead of
// hanging.
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>

#include "device.cuh"
#include "kernels.hpp"

namespace pdfb {

constexpr int kTicketBatch = 2;
constexpr int kSweepThreads = 256;
// block kernels: up to 17 warps per CTA (16 consumers and the producer), at
// most 112 registers a thread, so that 2 CTAs of 9 warps fit an SM
constexpr int kBlockMaxThreads = 576;

// A slab (one bulk copy) is 32 rows x kCols columns (forward) or kCols rows
// x 32 columns (backward): 4 KB, except FP32 backward slabs of 16 rows (2 KB,
// measured faster there: the per-row index staging is half as long).  A
// block kernel's CTA has a ring of R slots (DPlan::ring_f / ring_b): the
// largest in [kMinSlots, kMaxSlots] with which the launch shape's CTAs fit an
// SM.
template <typename T, bool kFwd>
struct Stages {
  static constexpr int kCols = (sizeof(T) == 4 && kFwd) ? kSlabMax : kSlab;
  static constexpr int kElems = kTile * kCols;
};
constexpr int kMinSlots = 4, kMaxSlots = 64;

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

// ---- mbarrier and bulk-copy primitives (PTX, sm_90+; no multicast)
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Programmatic dependent launch: a kernel launched with the programmatic
// stream serialization attribute may start while the kernel before it in the
// stream still runs; griddep_wait() returns once that kernel has completed
// and its memory operations are visible.  Before it, such a kernel reads
// only data no kernel of the solve writes (the factor, the plan).
// griddep_launch_dependents() lets the next such kernel start launching.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// orders generic-proxy accesses of shared memory before the bulk copies that
// follow (a slot's earlier reads before the copy that overwrites it)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// global -> shared bulk copy of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completing `bytes` transactions on `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int max_spins) {
  for (int k = 0; k < max_spins; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// every lane waits (each needs the barrier's acquire to see the copied data);
// the outcome is made uniform across the warp
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, int max_spins) {
  return __all_sync(0xffffffffu, mbar_wait(bar, parity, max_spins)) != 0;
}
__device__ __forceinline__ uint32_t round16(uint32_t bytes) { return (bytes + 15u) & ~15u; }

// Issues the (up to) 32 loads of one 32-wide slab of a tile: lane l reads
// element (l, u) at p[stride u]; absent columns (u >= m) and lanes outside the
// tile (act false) read as zero.
template <typename T>
__device__ __forceinline__ void load_tile(T (&w)[32], const T* p, int m, int stride = kTile, bool act = true) {
#pragma unroll
  for (int u = 0; u < 32; ++u) w[u] = (act && u < m) ? ldw(p + u * stride) : T(0);
}

// Asynchronous global -> shared copy of N = 4, 8 or 16 bytes (both
// addresses N-byte aligned); cp_async_wait_all() waits for this thread's.
template <int N>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// A block's item descriptors into shared memory (32 bytes each, two copies).
__device__ __forceinline__ void stage_items(BlockItem* dst, const BlockItem* src, int nitems) {
  for (int k = threadIdx.x; k < nitems; k += blockDim.x) {
    cp_async<16>(reinterpret_cast<char*>(dst + k), reinterpret_cast<const char*>(src + k));
    cp_async<16>(reinterpret_cast<char*>(dst + k) + 16, reinterpret_cast<const char*>(src + k) + 16);
  }
}

// Block tickets: thread 0 draws the first one before the loop and the next
// one when a block enters its last level (its round trip overlaps that
// level, and blocks are still claimed in about the order CTAs free up); the
// ticket is published in shared memory between two barriers at the block's
// end, after every thread has read the current one.

// ---------------------------------------------------------------- blocks
//
// A block kernel's CTA is `ncw` consumer warps and one producer warp.  The
// producer's lane 0 streams the block's factor, slab by slab in item order
// (the items are stored level by level), into a ring of R slots shared by
// the CTA: slot q % R holds the block's slab number q (counted over the CTA's
// lifetime), its `full` mbarrier completes when the copy lands, its `empty`
// mbarrier when the consuming warp has read it.  Consumer warps take the
// items of each level round-robin, wait for each slab's `full` barrier, and
// release it; levels are separated by a barrier among the consumers only, so
// the producer keeps copying the next levels' slabs while a level finishes.
// A slab is only copied into a slot whose previous slab (issued R slabs
// earlier, so of the same or an earlier level) was read, which its consumer
// reaches without waiting on anything issued later: the pipeline cannot
// stall on itself.  A consumer may reach a slot two uses ahead of the copy
// in it (its slab belongs to a warp that is ahead of the one reading the
// slot's previous slab), where a parity wait on `full` would mistake an
// earlier phase for its own; so the producer posts the use number of each
// slot (`use`) before the copy, and a consumer waits for its use number
// first, then for `full`.  Every wait is bounded.

// the ring's parts in shared memory
template <typename T>
struct BlockSmem {
  T* ring;          // R slots of Stages::kElems
  int* iring;       // backward: R slots of kCols row indices
  uint64_t* full;   // R
  uint64_t* empty;  // R
  int* use;         // R: the use number of the copy issued into each slot (-1: none yet)
  T* sv;
  T* ys;
  T* vstage;        // this consumer warp's 3 x kCols vector entries (backward)
  BlockItem* items;
  int* slab0;       // first slab of each item, relative to the block
};

template <typename T, bool kFwd>
__device__ __forceinline__ BlockSmem<T> block_smem(unsigned char* base, int ncw, int warp, int max_ld, int max_cols,
                                                   int max_items, int R) {
  constexpr int KE = Stages<T, kFwd>::kElems, kCols = Stages<T, kFwd>::kCols;
  BlockSmem<T> s;
  size_t off = 0;
  s.ring = reinterpret_cast<T*>(base);
  off += (size_t)R * KE * sizeof(T);
  s.iring = reinterpret_cast<int*>(base + off);
  if (!kFwd) off += (size_t)R * kCols * sizeof(int);
  s.full = reinterpret_cast<uint64_t*>(base + off);
  s.empty = s.full + R;
  off += 2 * (size_t)R * sizeof(uint64_t);
  s.use = reinterpret_cast<int*>(base + off);
  off += (size_t)R * sizeof(uint64_t);
  s.sv = reinterpret_cast<T*>(base + off);
  off += 3 * (size_t)max_ld * sizeof(T);
  s.ys = reinterpret_cast<T*>(base + off);
  if (!kFwd) off += 3 * (size_t)max_cols * sizeof(T);
  s.vstage = reinterpret_cast<T*>(base + off) + (size_t)min(warp, ncw - 1) * 3 * kCols;
  if (!kFwd) off += (size_t)ncw * 3 * kCols * sizeof(T);
  off = (off + 15) & ~size_t(15);
  s.items = reinterpret_cast<BlockItem*>(base + off);
  off += (size_t)max_items * sizeof(BlockItem);
  s.slab0 = reinterpret_cast<int*>(base + off);
  return s;
}

template <typename T, bool kFwd>
size_t block_smem_bytes(int ncw, int max_ld, int max_cols, int max_items, int R) {
  constexpr int KE = Stages<T, kFwd>::kElems, kCols = Stages<T, kFwd>::kCols;
  size_t b = (size_t)R * KE * sizeof(T) + 3 * (size_t)R * sizeof(uint64_t) + 3 * (size_t)max_ld * sizeof(T);
  if (!kFwd) b += (size_t)R * kCols * sizeof(int) + 3 * (size_t)max_cols * sizeof(T) + (size_t)ncw * 3 * kCols * sizeof(T);
  return ((b + 15) & ~size_t(15)) + (size_t)max_items * (sizeof(BlockItem) + sizeof(int));
}

// A consumer warp's wait for slab q: its slot's use number posted, then the
// slot's `full` barrier (bounded; false when either wait gave up).
__device__ __forceinline__ bool wait_slab(const int* use, uint64_t* full, int q, int R, int max_spins) {
  const int slot = q % R, u = q / R;
  int ok = 1;
  if ((threadIdx.x & 31) == 0) {
    ok = 0;
    for (int k = 0; k < max_spins; ++k)
      if (*reinterpret_cast<const volatile int*>(use + slot) == u) {
        ok = 1;
        break;
      }
  }
  if (!__shfl_sync(0xffffffffu, ok, 0)) return false;
  return mbar_wait_warp(full + slot, u & 1, max_spins);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// barrier 1 among the consumer warps only (the producer does not take part)
__device__ __forceinline__ void consumers_sync(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Warp 0: slab0[k] = the number of slabs of items [0, k) (kCols columns /
// rows each, from a0); returns the total (every lane).
template <int kCols>
__device__ __forceinline__ int scan_slabs(const BlockItem* items, int nitems, int* slab0, int lane) {
  int total = 0;
  for (int k0 = 0; k0 < nitems; k0 += 32) {
    const int k = k0 + lane;
    const int c = k < nitems ? (items[k].a1 - items[k].a0 + kCols - 1) / kCols : 0;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (k < nitems) slab0[k] = total + incl - c;
    total += __shfl_sync(0xffffffffu, incl, 31);
  }
  return total;
}

// Producer lane: copies the block's slabs, numbered from q_base, into the
// ring in item order; returns the number after the last one issued and sets
// ok false when a wait for a free slot gave up.
template <typename T, bool kFwd>
__device__ __forceinline__ int produce_block(const BlockSmem<T>& sm, const BlockItem* items, int nitems, int q_base,
                                             int R, const T* W, const int* bidx, int max_spins, bool& ok) {
  constexpr int KE = Stages<T, kFwd>::kElems, kCols = Stages<T, kFwd>::kCols;
  int q = q_base;
  for (int it = 0; it < nitems; ++it) {
    const BlockItem I = items[it];
    // forward: rows of the tile m, a slab = columns j0.. (column-major, m per
    // column); backward: columns of the tile mc, a slab = rows j0.. (mc per row)
    const int width = kFwd ? min(kTile, I.ns + I.nr - kTile * I.tile) : min(kTile, I.ns - kTile * I.tile);
    for (int j0 = I.a0; j0 < I.a1; j0 += kCols, ++q) {
      const int slot = q % R, use = q / R;
      if (use > 0 && !mbar_wait(sm.empty + slot, (use - 1) & 1, max_spins)) {
        ok = false;
        return q;
      }
      fence_proxy_async();  // the consumer's reads of the slot before the copy over it
      // the slot's `full` barrier has completed every phase before this use
      *reinterpret_cast<volatile int*>(sm.use + slot) = use;
      const int cnt = min(kCols, I.a1 - j0);
      const uint32_t wbytes = round16((uint32_t)(width * cnt) * (uint32_t)sizeof(T));
      const uint32_t ibytes = kFwd ? 0u : (uint32_t)(kCols * sizeof(int));
      mbar_expect_tx(sm.full + slot, wbytes + ibytes);
      bulk_g2s(sm.ring + (size_t)slot * KE, W + I.off + (int64_t)width * j0, wbytes, sm.full + slot);
      if (!kFwd) bulk_g2s(sm.iring + (size_t)slot * kCols, bidx + I.idx0 + j0, ibytes, sm.full + slot);
    }
  }
  return q;
}

// After a wait gave up: the producer waits (bounded) for the copies it
// issued into each slot's last use, so that none lands after the CTA exits.
__device__ __forceinline__ void drain_ring(uint64_t* full, int q_end, int R, int max_spins) {
  for (int q = max(0, q_end - R); q < q_end; ++q) mbar_wait(full + q % R, (q / R) & 1, max_spins);
}

template <typename T>
__global__ void __launch_bounds__(kBlockMaxThreads, 1) k_block_forward(DPlan P, const T* __restrict__ W, T* b, T* y,
                                                                    int n, SweepSync sy) {
  trace_stamp(sy.trace, DTrace::kSolve);
  griddep_launch_dependents();  // the first upper level may start on SMs this sweep leaves
  constexpr int KE = Stages<T, true>::kElems, kCols = Stages<T, true>::kCols;
  const int R = P.ring_f;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int s_ticket, s_nslab, s_failed;
  __shared__ int s_lev[kMaxBlockLevels + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, ncw = (blockDim.x >> 5) - 1;
  const bool producer = warp == ncw;
  const BlockSmem<T> sm =
      block_smem<T, true>(smem_raw, ncw, warp, P.max_cols + P.max_ext, P.max_cols, P.max_items, R);
  if (threadIdx.x == 0) {
    for (int k = 0; k < R; ++k) {
      mbar_init(sm.full + k, 1);
      mbar_init(sm.empty + k, 1);
      sm.use[k] = -1;
    }
    fence_mbar_init();
  }
  int q_base = 0;       // the CTA's slabs before this block
  int q_issued = 0;     // producer lane 0: slabs issued
  bool failed = false;  // a bounded wait gave up (this thread's view)
  int next_ticket = 0;  // thread 0
  if (threadIdx.x == 0) {
    s_ticket = atomicAdd(sy.queue + 2, 1);
    s_failed = 0;
  }
  __syncthreads();
  for (;;) {
    const int bi = s_ticket;
    if (bi >= P.nblk) break;
    const SweepBlock& B = P.fblk[bi];
    const int c0b = B.c0, nc = B.c1 - B.c0, ld = nc + B.next, nlev = B.nlev, nitems = B.lev[B.nlev];
    T* sv = sm.sv;
    // b of the block's columns and the item descriptors: every copy in
    // flight at once
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
      cp_async<sizeof(T)>(sv + k, b + c0b + k);
      cp_async<sizeof(T)>(sv + ld + k, b + (int64_t)n + c0b + k);
      cp_async<sizeof(T)>(sv + 2 * ld + k, b + 2 * (int64_t)n + c0b + k);
    }
    stage_items(sm.items, P.fitem + B.item0, nitems);
    for (int e = threadIdx.x; e < B.next; e += blockDim.x) sv[nc + e] = sv[ld + nc + e] = sv[2 * ld + nc + e] = T(0);
    if (threadIdx.x <= nlev) s_lev[threadIdx.x] = B.lev[threadIdx.x];
    cp_async_wait_all();
    __syncthreads();
    if (warp == 0) {
      const int t = scan_slabs<kCols>(sm.items, nitems, sm.slab0, lane);
      if (lane == 0) s_nslab = t;
    }
    __syncthreads();
    const BlockItem* items = sm.items;
    if (producer) {
      int q_end = q_base;
      bool ok = !failed;
      if (lane == 0 && ok) {
        q_end = produce_block<T, true>(sm, items, nitems, q_base, R, W, P.bidx, sy.max_spins, ok);
        q_issued = q_end;
        if (!ok) {
          atomicOr(sy.err, 1);
          s_failed = 1;
        }
      }
      failed = failed || !__shfl_sync(0xffffffffu, ok, 0);
    } else {
      for (int L = 0; L < nlev; ++L) {
        if (L == nlev - 1 && threadIdx.x == 0) next_ticket = atomicAdd(sy.queue + 2, 1);
        const int i1 = s_lev[L + 1];
#pragma unroll 1
        for (int it = s_lev[L] + warp; it < i1; it += ncw) {
          const BlockItem I = items[it];
          const int m = min(kTile, I.ns + I.nr - kTile * I.tile);
          const int w = min((int)I.ns, kTile * I.tile + kTile);
          const int a1 = I.a1;
          const int row = kTile * I.tile + lane;
          const int loc = (row >= I.ns && row < I.ns + I.nr) ? P.rows_loc[I.roff + row - I.ns] : -1;
          const T* vx = sv + I.c0l;
          T ax = 0, ay = 0, az = 0;
          int q = q_base + sm.slab0[it];
#pragma unroll 1
          for (int j0 = I.a0; j0 < a1; j0 += kCols, ++q) {
            const int slot = q % R;
            if (!failed && !wait_slab(sm.use, sm.full, q, R, sy.max_spins)) {
              failed = true;
              if (lane == 0) {
                atomicOr(sy.err, 1);
                s_failed = 1;
              }
            }
            if (!failed) {
              const T* sp = sm.ring + (size_t)slot * KE;
              const int cnt = min(kCols, a1 - j0);
              if (lane < m) {
#pragma unroll
                for (int u = 0; u < kCols; ++u)
                  if (u < cnt) {
                    const T wv = sp[m * u + lane];
                    ax += wv * vx[j0 + u];
                    ay += wv * vx[ld + j0 + u];
                    az += wv * vx[2 * ld + j0 + u];
                  }
              }
              __syncwarp();
              if (lane == 0) mbar_arrive(sm.empty + slot);  // the slot is read
            }
          }
          if (row < I.ns) {
            const int64_t o = (int64_t)c0b + I.c0l + row;
            if (I.a0 == 0 && a1 == w) {
              y[o] = ax;
              y[o + n] = ay;
              y[o + 2 * (int64_t)n] = az;
            } else {  // one span of a split tile (y starts at zero)
              atomicAdd(y + o, ax);
              atomicAdd(y + o + n, ay);
              atomicAdd(y + o + 2 * (int64_t)n, az);
            }
          } else if (loc >= 0) {
            atomicAdd(sv + loc, -ax);
            atomicAdd(sv + ld + loc, -ay);
            atomicAdd(sv + 2 * ld + loc, -az);
          }
        }
        consumers_sync(ncw * 32);
      }
    }
    q_base += s_nslab;
    __syncthreads();  // every level done, every slab of the block issued
    // the ext rows' updates, once per block
    for (int e = threadIdx.x; e < B.next; e += blockDim.x) {
      const int64_t r = P.rows[B.ext0 + e];
      atomicAdd(b + r, sv[nc + e]);
      atomicAdd(b + r + n, sv[ld + nc + e]);
      atomicAdd(b + r + 2 * (int64_t)n, sv[2 * ld + nc + e]);
    }
    __syncthreads();  // the shared vector is free, every thread has read s_ticket and s_nslab
    if (threadIdx.x == 0) s_ticket = next_ticket;
    __syncthreads();
  }
  // a wait gave up somewhere: every copy the producer issued lands before
  // the CTA exits
  if (s_failed && producer && lane == 0) drain_ring(sm.full, q_issued, R, sy.max_spins);
}

// v[perm[k]] = x_k (mode 0) or += x_k (mode 1) and q^k = q_n + dt v for the
// nc columns of a block, x in shared memory (3 planes of stride ld).  Each
// thread takes kWbCols columns a pass and issues every load of the pass
// before its stores, so that a pass costs two dependent memory round trips
// (the permutation, then the vertex gathers) instead of several per column.
constexpr int kWbCols = 2;
constexpr int kExtBatch = 4;  // ext rows per thread whose indices are loaded together
template <typename T>
__device__ __forceinline__ void write_back_columns(const T* sv, int ld, int nc, const int* __restrict__ perm,
                                                   const WriteBack& wb) {
  double* __restrict__ v = wb.v;
  double* __restrict__ qk = wb.qk;
  const double* __restrict__ q = wb.q;
  for (int k0 = threadIdx.x; k0 < nc; k0 += kWbCols * blockDim.x) {
    int64_t vtx[kWbCols];
    double val[kWbCols][3], qv[kWbCols][3];
#pragma unroll
    for (int j = 0; j < kWbCols; ++j) {
      const int k = k0 + j * blockDim.x;
      vtx[j] = k < nc ? perm[k] : -1;
    }
#pragma unroll
    for (int j = 0; j < kWbCols; ++j)
      if (vtx[j] >= 0) {
        const int k = k0 + j * blockDim.x;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          val[j][c] = (double)sv[k + c * ld];
          qv[j][c] = q[3 * vtx[j] + c];
          if (wb.mode == 1) val[j][c] += v[3 * vtx[j] + c];
        }
      }
#pragma unroll
    for (int j = 0; j < kWbCols; ++j)
      if (vtx[j] >= 0)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          v[3 * vtx[j] + c] = val[j][c];
          qk[3 * vtx[j] + c] = qv[j][c] + wb.dt * val[j][c];
        }
  }
}

template <typename T>
__global__ void __launch_bounds__(kBlockMaxThreads, 1) k_block_backward(DPlan P, const T* __restrict__ W,
                                                                     const T* __restrict__ y, const T* x, int n,
                                                                     SweepSync sy, WriteBack wb) {
  griddep_launch_dependents();
  constexpr int KE = Stages<T, false>::kElems, kCols = Stages<T, false>::kCols;
  const int R = P.ring_b;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int s_ticket, s_nslab, s_failed;
  __shared__ int s_lev[kMaxBlockLevels + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, ncw = (blockDim.x >> 5) - 1;
  const bool producer = warp == ncw;
  const BlockSmem<T> sm =
      block_smem<T, false>(smem_raw, ncw, warp, P.max_cols + P.max_ext, P.max_cols, P.max_items, R);
  if (threadIdx.x == 0) {
    for (int k = 0; k < R; ++k) {
      mbar_init(sm.full + k, 1);
      mbar_init(sm.empty + k, 1);
      sm.use[k] = -1;
    }
    fence_mbar_init();
  }
  int q_base = 0, q_issued = 0;
  bool failed = false;
  int next_ticket = 0;  // thread 0
  if (threadIdx.x == 0) {
    s_ticket = atomicAdd(sy.queue + 3, 1);
    s_failed = 0;
  }
  __syncthreads();
  for (;;) {
    const int bi = s_ticket;
    if (bi >= P.nblk) break;
    const SweepBlock& B = P.bblk[bi];
    const int c0b = B.c0, nc = B.c1 - B.c0, ld = nc + B.next, nlev = B.nlev, nitems = B.lev[B.nlev];
    T* sv = sm.sv;
    T* ys = sm.ys;
    stage_items(sm.items, P.bitem + B.item0, nitems);
    if (threadIdx.x <= nlev) s_lev[threadIdx.x] = B.lev[threadIdx.x];
    // the ext rows' indices (constant), then the y slice and the final x of
    // the ext rows (the upper supernodes finished in the previous launches:
    // this kernel is their programmatic dependent), every copy in flight at once
    const int* ext_rows = P.rows + B.ext0;
    int64_t er[kExtBatch];
#pragma unroll
    for (int j = 0; j < kExtBatch; ++j) {
      const int e = threadIdx.x + j * blockDim.x;
      er[j] = e < B.next ? ext_rows[e] : -1;
    }
    griddep_wait();
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
      cp_async<sizeof(T)>(ys + k, y + c0b + k);
      cp_async<sizeof(T)>(ys + nc + k, y + (int64_t)n + c0b + k);
      cp_async<sizeof(T)>(ys + 2 * nc + k, y + 2 * (int64_t)n + c0b + k);
    }
#pragma unroll
    for (int j = 0; j < kExtBatch; ++j)
      if (er[j] >= 0) {
        const int e = threadIdx.x + j * blockDim.x;
        cp_async<sizeof(T)>(sv + nc + e, x + er[j]);
        cp_async<sizeof(T)>(sv + ld + nc + e, x + er[j] + n);
        cp_async<sizeof(T)>(sv + 2 * ld + nc + e, x + er[j] + 2 * (int64_t)n);
      }
    for (int e = threadIdx.x + kExtBatch * blockDim.x; e < B.next; e += blockDim.x) {  // beyond the batch
      const int64_t r = ext_rows[e];
      cp_async<sizeof(T)>(sv + nc + e, x + r);
      cp_async<sizeof(T)>(sv + ld + nc + e, x + r + n);
      cp_async<sizeof(T)>(sv + 2 * ld + nc + e, x + r + 2 * (int64_t)n);
    }
    // the block's columns start at zero: the spans of a split tile add into them
    for (int k = threadIdx.x; k < nc; k += blockDim.x) sv[k] = sv[ld + k] = sv[2 * ld + k] = T(0);
    cp_async_wait_all();
    __syncthreads();
    if (warp == 0) {
      const int t = scan_slabs<kCols>(sm.items, nitems, sm.slab0, lane);
      if (lane == 0) s_nslab = t;
    }
    __syncthreads();
    const BlockItem* items = sm.items;
    if (producer) {
      bool ok = !failed;
      if (lane == 0 && ok) {
        q_issued = produce_block<T, false>(sm, items, nitems, q_base, R, W, P.bidx, sy.max_spins, ok);
        if (!ok) {
          atomicOr(sy.err, 1);
          s_failed = 1;
        }
      }
      failed = failed || !__shfl_sync(0xffffffffu, ok, 0);
    } else {
      for (int L = 0; L < nlev; ++L) {
        if (L == nlev - 1 && threadIdx.x == 0) next_ticket = atomicAdd(sy.queue + 3, 1);
        const int i1 = s_lev[L + 1];
#pragma unroll 1
        for (int it = s_lev[L] + warp; it < i1; it += ncw) {
          const BlockItem I = items[it];
          const int j0t = kTile * I.tile, nd = I.ns - j0t, mc = min(kTile, nd), h = nd + I.nr;
          const int a1 = I.a1;
          T ax = 0, ay = 0, az = 0;
          int q = q_base + sm.slab0[it];
#pragma unroll 1
          for (int i0 = I.a0; i0 < a1; i0 += kCols, ++q) {
            const int slot = q % R;
            if (!failed && !wait_slab(sm.use, sm.full, q, R, sy.max_spins)) {
              failed = true;
              if (lane == 0) {
                atomicOr(sy.err, 1);
                s_failed = 1;
              }
            }
            if (failed) continue;
            const int cnt = min(kCols, a1 - i0);
            if (lane < kCols) {
              T vx = 0, vy = 0, vz = 0;
              if (lane < cnt) {
                const int idx = sm.iring[(size_t)slot * kCols + lane];
                if (idx < 0) {
                  const int k = -1 - idx;
                  vx = ys[k];
                  vy = ys[nc + k];
                  vz = ys[2 * nc + k];
                } else {
                  vx = -sv[idx];
                  vy = -sv[ld + idx];
                  vz = -sv[2 * ld + idx];
                }
              }
              sm.vstage[lane] = vx;
              sm.vstage[kCols + lane] = vy;
              sm.vstage[2 * kCols + lane] = vz;
            }
            __syncwarp();
            if (lane < mc) {
              const T* sp = sm.ring + (size_t)slot * KE;
#pragma unroll
              for (int u = 0; u < kCols; ++u)
                if (u < cnt) {
                  const T wv = sp[mc * u + lane];
                  ax += wv * sm.vstage[u];
                  ay += wv * sm.vstage[kCols + u];
                  az += wv * sm.vstage[2 * kCols + u];
                }
            }
            __syncwarp();  // the slot and the staged entries are read
            if (lane == 0) mbar_arrive(sm.empty + slot);
          }
          if (lane < mc) {
            T* s = sv + I.c0l + j0t + lane;
            if (I.a0 == 0 && a1 == h) {
              s[0] = ax;
              s[ld] = ay;
              s[2 * ld] = az;
            } else {  // one span of a split tile
              atomicAdd(s, ax);
              atomicAdd(s + ld, ay);
              atomicAdd(s + 2 * ld, az);
            }
          }
        }
        consumers_sync(ncw * 32);
      }
    }
    q_base += s_nslab;
    __syncthreads();  // every level done, every slab of the block issued
    if (!failed) write_back_columns(sv, ld, nc, P.perm + c0b, wb);
    __syncthreads();  // the shared vectors are free, every thread has read s_ticket and s_nslab
    if (threadIdx.x == 0) s_ticket = next_ticket;
    __syncthreads();
  }
  if (s_failed && producer && lane == 0) drain_ring(sm.full, q_issued, R, sy.max_spins);
  griddep_wait();  // a CTA without a block completes after the launch before it too
}

// ---------------------------------------------------------- upper items

// Tickets are taken kTicketBatch at a time and processed in order, the next
// batch drawn while the current one runs: every item with a smaller ticket is
// held by a running warp, so the waits below always end.
template <typename T>
__global__ void __launch_bounds__(kSweepThreads) k_upper_forward(DPlan P, const T* __restrict__ W, T* b, T* y, int n,
                                                                 SweepSync sy) {
  const int lane = threadIdx.x & 31;
  const unsigned long long ep = ld_volatile_u64(sy.epoch);
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
    if (lane == 0)
      for (int c = 0; c < tk.wait && ok; ++c) {
        const int2 ch = reinterpret_cast<const int2*>(P.child)[tk.child0 + c];
        ok = wait_counter(sy.fdone + ch.x, ep * (unsigned long long)ch.y, sy.err, sy.max_spins);
      }
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
    // the item's updates are performed before its count: a parent item that
    // sees every item of this supernode counted sees all of them
    fence_acq_rel_gpu();
    __syncwarp();
    if (lane == 0) atomicAdd(sy.fdone + tk.sn, 1ULL);
  }
}

template <typename T>
__global__ void __launch_bounds__(kSweepThreads) k_upper_backward(DPlan P, const T* __restrict__ W,
                                                                  const T* __restrict__ y, T* x, int n, SweepSync sy) {
  const int lane = threadIdx.x & 31;
  const unsigned long long ep = ld_volatile_u64(sy.epoch);
  int t = 0, tend = 0, next = 0;
  if (lane == 0) next = atomicAdd(sy.queue + 1, kTicketBatch);
  for (;; ++t) {
    if (t >= tend) {
      t = __shfl_sync(0xffffffffu, next, 0);
      tend = t + kTicketBatch;
      if (t >= P.nbup) return;
      if (lane == 0) next = atomicAdd(sy.queue + 1, kTicketBatch);
    }
    if (t >= P.nbup) return;
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
}

// ---------------------------------------------- upper items, level by level

// One elimination-tree level of upper items per launch, [lo, hi), spread
// over all warps (grid-stride); the launches follow one another in sweep
// order, so an item needs no dependency wait and signals nothing.  Launched
// as programmatic dependents: an item's factor tile and row indices are
// loaded before the wait for the previous launch, its vector after it.
// Resident CTAs per SM the level kernels are compiled for: 3 in FP32 (its
// 32-element tiles leave room; measured 4 % faster solves), 2 in FP64 (at 3
// the FP64 kernels spill and the solve is 26 % slower).
template <typename T>
struct LevelOccupancy {
  static constexpr int kCtas = sizeof(T) == 4 ? 3 : 2;
};

template <typename T>
__global__ void __launch_bounds__(kSweepThreads, LevelOccupancy<T>::kCtas) k_upper_level_forward(DPlan P, int lo, int hi,
                                                                       const T* __restrict__ W, T* b, T* y, int n) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  griddep_launch_dependents();
  bool waited = false;
#pragma unroll 1
  for (int t = lo + gw; t < hi; t += nwarps) {
    const UpperItem tk = P.fup[t];
    const int mrows = min(kTile, tk.ns + tk.nr - tk.tile * kTile);
    const T* wbase = W + tk.off + lane;
    const int row = tk.tile * kTile + lane;
    const int64_t r = (row >= tk.ns && row < tk.ns + tk.nr) ? P.rows[tk.roff + row - tk.ns] : -1;
    const T* bx = b + tk.c0;
    const T* by = bx + n;
    const T* bz = by + n;
    T ax = 0, ay = 0, az = 0;
    for (int j0 = tk.a0; j0 < tk.a1; j0 += 32) {
      T w[32];
      load_tile(w, wbase + (int64_t)j0 * mrows, min(32, tk.a1 - j0), mrows, lane < mrows);
      if (!waited) {  // the factor is in flight; b comes from the previous launches
        griddep_wait();
        waited = true;
      }
      const int jl = j0 + lane;
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
    } else if (r >= 0) {
      atomicAdd(b + r, -ax);
      atomicAdd(b + r + n, -ay);
      atomicAdd(b + r + 2 * (int64_t)n, -az);
    }
  }
  // every thread waits before it exits, so that this launch completes only
  // after the one before it (the next programmatic dependent relies on it)
  if (!waited) griddep_wait();
}

template <typename T>
__global__ void __launch_bounds__(kSweepThreads, LevelOccupancy<T>::kCtas) k_upper_level_backward(DPlan P, int lo, int hi,
                                                                        const T* __restrict__ W,
                                                                        const T* __restrict__ y, T* x, int n) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  griddep_launch_dependents();
  bool waited = false;
#pragma unroll 1
  for (int t = lo + gw; t < hi; t += nwarps) {
    const UpperItem tk = P.bup[t];
    const int mcols = min(kTile, tk.ns - tk.tile * kTile);
    const T* wbase = W + tk.off + lane;
    const int j0t = tk.tile * kTile;
    const int col = j0t + lane;
    const int nd = tk.ns - j0t;
    T ax = 0, ay = 0, az = 0;
    for (int i0 = tk.a0; i0 < tk.a1; i0 += 32) {
      T w[32];
      load_tile(w, wbase + (int64_t)i0 * mcols, min(32, tk.a1 - i0), mcols, lane < mcols);
      const int il = i0 + lane;
      const int64_t r = (il < tk.a1 && il >= nd) ? P.rows[tk.roff + il - nd] : 0;
      if (!waited) {  // the factor and row indices are in flight; y and x come from the previous launches
        griddep_wait();
        waited = true;
      }
      T vx = 0, vy = 0, vz = 0;
      if (il < tk.a1) {
        if (il < nd) {
          const int64_t o = (int64_t)tk.c0 + j0t + il;
          vx = ldcg(y + o);
          vy = ldcg(y + o + n);
          vz = ldcg(y + o + 2 * (int64_t)n);
        } else {
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
  // every thread waits before it exits, so that this launch completes only
  // after the one before it (the next programmatic dependent relies on it)
  if (!waited) griddep_wait();
}

// After the backward sweep, for the upper supernodes' columns: v[perm] = x
// (mode 0) or v[perm] += x (mode 1), q^k = q_n + dt v, and x, y cleared for
// the next solve (the blocks' columns are written back by the backward sweep
// and their y is overwritten by the next forward sweep); one thread rewinds
// the work queues and advances the solve counter.
template <typename T>
__global__ void k_solve_post(DPlan P, T* __restrict__ x, T* __restrict__ y, int n, WriteBack wb, SweepSync sy) {
  griddep_wait();  // launched as a programmatic dependent of the block backward sweep
  double* __restrict__ v = wb.v;
  double* __restrict__ qk = wb.qk;
  const double* __restrict__ q = wb.q;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P.n_upper; k += gridDim.x * blockDim.x) {
    const int col = P.upper_cols[k];
    const int64_t vtx = P.perm[col];
    // every load before the first store (the arrays do not alias)
    double val[3], qv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      val[c] = (double)x[col + (int64_t)c * n];
      qv[c] = q[3 * vtx + c];
    }
    if (wb.mode == 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) val[c] += v[3 * vtx + c];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t o = col + (int64_t)c * n;
      x[o] = 0;
      y[o] = 0;
      v[3 * vtx + c] = val[c];
      qk[3 * vtx + c] = qv[c] + wb.dt * val[c];
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
// shared memory (0 when the kernel does not fit).
// The kernel's dynamic shared-memory limit is raised to the device's
// opt-in maximum, not to this plan's need: the attribute belongs to the
// kernel, shared by every handle of the process, and a later handle with a
// smaller plan must not lower it under an earlier handle's launches (or the
// launches captured in its graphs).
template <typename K>
int resident_ctas(K kernel, size_t smem, int threads = kSweepThreads) {
  int dev = 0, sms = 148, per_sm = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  const int dyn_max = optin - (int)fa.sharedSizeBytes;  // static shared memory counts against the limit
  if (smem > (size_t)dyn_max) return 0;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * sms;
}

// The largest ring (kMinSlots .. kMaxSlots slots per CTA) with which `ctas`
// CTAs of `warps` consumer warps and the producer warp of this block kernel
// are resident per SM; 0 if none.
template <typename T, bool kFwd, typename K>
int ring_for(K kernel, const DPlan& P, int warps, int ctas, int* smem) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int max_ld = std::max(1, P.max_cols + P.max_ext);
  for (int R = kMaxSlots; R >= kMinSlots; --R) {
    const size_t b = block_smem_bytes<T, kFwd>(warps, max_ld, std::max(1, P.max_cols), std::max(1, P.max_items), R);
    if (resident_ctas(kernel, b, 32 * (warps + 1)) >= ctas * sms) {
      *smem = (int)b;
      return R;
    }
  }
  return 0;
}

template <typename T>
bool configure_solve(DPlan& P, int shape) {
  if (shape < 0 || shape >= kBlockShapes) return false;
  const int warps = kBlockShapeWarps[shape], ctas = kBlockShapeCtas[shape];
  P.block_shape = shape;
  P.block_warps = warps;
  P.block_ctas = ctas;
  P.ring_f = ring_for<T, true>(k_block_forward<T>, P, warps, ctas, &P.smem_f);
  P.ring_b = ring_for<T, false>(k_block_backward<T>, P, warps, ctas, &P.smem_b);
  if (!P.ring_f || !P.ring_b) return false;
  const int rf = resident_ctas(k_block_forward<T>, P.smem_f, 32 * (warps + 1));
  const int rb = resident_ctas(k_block_backward<T>, P.smem_b, 32 * (warps + 1));
  P.grid_bf = std::max(1, std::min(rf, std::max(1, P.nblk)));
  P.grid_bb = std::max(1, std::min(rb, std::max(1, P.nblk)));
  P.grid_uf = std::max(1, resident_ctas(k_upper_forward<T>, 0));
  P.grid_ub = std::max(1, resident_ctas(k_upper_backward<T>, 0));
  // the level kernels use the same launch shape; make sure they can launch
  resident_ctas(k_upper_level_forward<T>, 0);
  resident_ctas(k_upper_level_backward<T>, 0);
  return rf > 0 && rb > 0;
}

// Launch as a programmatic dependent of the previous kernel in the stream
// (the kernel calls griddep_wait() before it reads what that kernel writes).
template <typename... Params, typename... Args>
void launch_dependent(void (*kernel)(Params...), int grid, int block, size_t smem, cudaStream_t st,
                      Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <typename T>
void launch_solve_sweeps(cudaStream_t st, const DPlan& P, const T* Wf, const T* Wb, T* b, T* y, T* x, int n,
                         SweepSync sy, WriteBack wb, cudaEvent_t* marks) {
  // marks (optional): 4 events recorded between the five launches
  k_block_forward<T><<<P.grid_bf, 32 * (P.block_warps + 1), P.smem_f, st>>>(P, Wf, b, y, n, sy);
  if (marks) cudaEventRecord(marks[0], st);
  if (P.upper_mode == 1) {
    const int wpc = kSweepThreads / 32;
    for (int k = 0; k < P.n_flev; ++k) {
      const int lo = P.flev[k], hi = P.flev[k + 1];
      const int grid = std::max(1, std::min(P.grid_uf, (hi - lo + wpc - 1) / wpc));
      launch_dependent(k_upper_level_forward<T>, grid, kSweepThreads, 0, st, P, lo, hi, Wf, b, y, n);
    }
  } else {
    k_upper_forward<T><<<P.grid_uf, kSweepThreads, 0, st>>>(P, Wf, b, y, n, sy);
  }
  if (marks) cudaEventRecord(marks[1], st);
  if (P.upper_mode == 1) {
    const int wpc = kSweepThreads / 32;
    for (int k = 0; k < P.n_blev; ++k) {
      const int lo = P.blev[k], hi = P.blev[k + 1];
      const int grid = std::max(1, std::min(P.grid_ub, (hi - lo + wpc - 1) / wpc));
      launch_dependent(k_upper_level_backward<T>, grid, kSweepThreads, 0, st, P, lo, hi, Wb,
                       static_cast<const T*>(y), x, n);
    }
  } else {
    k_upper_backward<T><<<P.grid_ub, kSweepThreads, 0, st>>>(P, Wb, y, x, n, sy);
  }
  if (marks) cudaEventRecord(marks[2], st);
  launch_dependent(k_block_backward<T>, P.grid_bb, 32 * (P.block_warps + 1), (size_t)P.smem_b, st, P, Wb,
                   static_cast<const T*>(y), static_cast<const T*>(x), n, sy, wb);
  if (marks) cudaEventRecord(marks[3], st);
  launch_dependent(k_solve_post<T>, std::max(1, std::min(148 * 4, (P.n_upper + 255) / 256)), 256, 0, st, P, x, y, n,
                   wb, sy);
}
template <typename T>
void launch_solve_prep(cudaStream_t st, int n, T* x, T* y, SweepSync sy) {
  k_solve_prep<T><<<std::min(148 * 4, (3 * n + 255) / 256), 256, 0, st>>>(n, x, y, sy);
}

template bool configure_solve<double>(DPlan&, int);
template bool configure_solve<float>(DPlan&, int);
template void launch_solve_sweeps<double>(cudaStream_t, const DPlan&, const double*, const double*, double*, double*,
                                          double*, int, SweepSync, WriteBack, cudaEvent_t*);
template void launch_solve_sweeps<float>(cudaStream_t, const DPlan&, const float*, const float*, float*, float*,
                                         float*, int, SweepSync, WriteBack, cudaEvent_t*);
template void launch_solve_prep<double>(cudaStream_t, int, double*, double*, SweepSync);
template void launch_solve_prep<float>(cudaStream_t, int, float*, float*, SweepSync);

}  // namespace pdfb
