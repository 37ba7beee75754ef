// kernels.hpp — declarations of the device kernels and their launch records.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"
#include "factor.hpp"

namespace pdfb {

// Work queues (4 ints: forward / backward upper items, forward / backward
// blocks), solve counter and cumulative completion counters.
struct SweepSync {
  int* queue;
  unsigned long long* epoch;
  unsigned long long* fdone;   // per supernode: forward work items finished
  unsigned long long* bdone;   // per supernode: backward work items finished
  int* err;                    // set when a dependency wait gives up
  int max_spins;               // polls of a dependency counter before giving up
  DTrace trace;                // iteration clock (forward sweep row)
};

constexpr int kMaxUpperLevels = 32;

// Launch shapes of the block kernels: warps per CTA and CTAs per SM (the
// ring of bulk-copy stages shrinks to fit); the schedule autotuner picks one.
constexpr int kBlockShapes = 5;
constexpr int kBlockShapeWarps[kBlockShapes] = {8, 8, 4, 4, 16};
constexpr int kBlockShapeCtas[kBlockShapes] = {1, 2, 3, 4, 1};

// Device view of a SweepPlan (factor.hpp) and its launch shape.
struct DPlan {
  const UpperItem* fup;
  const UpperItem* bup;
  int nfup, nbup;
  const SnInfo* sn;
  const int* rows;
  const SweepBlock* fblk;
  const SweepBlock* bblk;
  int nblk;
  const BlockItem* fitem;
  const BlockItem* bitem;
  const int* upper_cols;
  int n_upper;
  const int* perm;      // pivot position -> vertex
  const int* rows_loc;  // block supernodes: place of each row in the block's shared vector
  const int* bidx;      // backward block tiles: per-row vector index lists
  const int* child;     // forward upper items: (child, its work items) pairs
  int max_cols;         // widest block (shared-memory slice, 3 planes)
  int max_ext;          // most rows outside a block
  int max_items;        // most tiles of a block in one sweep
  int smem_f, smem_b;   // dynamic shared memory of the forward / backward block kernels
  int grid_bf, grid_bb, grid_uf, grid_ub;
  // launch shape of the block kernels (kBlockShapes): warps per CTA, CTAs
  // per SM it was sized for, and bulk-copy stages per warp (forward, backward)
  int block_shape, block_warps, block_ctas, ring_f, ring_b;
  // upper supernodes: 0 = dependency-driven items in one launch per sweep,
  // 1 = one launch per elimination-tree level (no waits; the launch boundary
  // orders the levels), with the level boundaries of fup / bup
  int upper_mode;
  int n_flev, n_blev;
  int flev[kMaxUpperLevels + 1], blev[kMaxUpperLevels + 1];
};

// Write-back of the solution: v[perm] = x (mode 0) or v[perm] += x (mode 1,
// FP32 correction), q^k = q_n + dt v.
struct WriteBack {
  double* v;
  double* qk;
  const double* q;
  double dt;
  int mode;
};

// Analytic and mesh obstacles (device array, refreshed every step for the
// rotating spheres' clocks).
struct DObstacle {
  int type, material, n_tri, mesh;  // mesh: -1 = every dynamic mesh
  double c[3], R;
  double rot[3], time_before_start;
  double p[3], n[3];
  double tol;
  double s[3];  // box: size (c = the corner with the smallest coordinates)
  const double* mv;  // mesh obstacles: current vertex positions
  const int* mt;
  // moving mesh: the key frames around its clock, their time span, and
  // whether the clock lies between them (contact speed is zero otherwise)
  const double* fprev;
  const double* fnext;
  double frame_dt;
  int moving;
  const void* bvh;  // mesh obstacles: LBVH node records over mv / mt (null: scan every triangle)
};
struct DObstacles {
  int n;
  const DObstacle* o;
  const int* vmesh;  // containing mesh of every vertex
  int* best;         // per (obstacle, vertex), obstacle-major: closest mesh-obstacle triangle, -1 if none
};

// LBVH over a mesh obstacle's triangles (lbvh.cuh), kept on the device: built
// once (static mesh) or rebuilt every few steps and refit every step (moving
// mesh).  Host-side handle; the node records go to DObstacle::bvh.
struct MeshBVH;
MeshBVH* mesh_bvh_create(int nv, int nt);
void mesh_bvh_build(MeshBVH* b, const double* verts, const int* tris, cudaStream_t st);
void mesh_bvh_refit(MeshBVH* b, const double* verts, const int* tris, cudaStream_t st);
const void* mesh_bvh_nodes(const MeshBVH* b);
void mesh_bvh_free(MeshBVH* b);

__global__ void k_step_init(DModel m, const double* q, double* v, double* tn, double* qk, double* cstep, double gx,
                            double gy, double gz, double dt);
// residual_mode 1: writes p_b - A_b q (the bending force's row value)
__global__ void k_bend_proj(DModel m, const double* qk, double* bp, int residual_mode);
// Iteration control of one step, on the device.  iter = PD iterations
// completed in this step (kernels of iteration k read k from it); the last
// block of the Alart-Curnier kernel closes the iteration: it advances iter and
// iter_total and, inside a conditional WHILE graph body, sets the loop
// condition (continue while iter < kmax and not (tol > 0, contacts > 0 and
// mean |AC| <= tol)).
struct IterCtl {
  int* iter;
  long long* iter_total;
  unsigned int* blocks_done;
  double tol;
  int kmax;
  int set_cond;
  cudaGraphConditionalHandle cond;
  DTrace trace;  // iteration clock (Alart-Curnier rows)
};
__global__ void k_alart_curnier(DContacts c, const double* v, double* hist, IterCtl ctl);
// End-of-step record that k_finalize copies into host-mapped memory: the
// step's counters and its iteration clock (null counts: no record).
struct StepOut {
  const int* n_contacts;
  const int* n_self;
  const int* n_levels;
  const int* iter;
  const unsigned long long* stamps;
  int n_stamps;
  int* counts;                     // contacts, self contacts, levels, iterations
  unsigned long long* stamps_out;  // n_stamps
};
__global__ void k_finalize(int n3, const double* qk, double* q, StepOut o);
__global__ void k_gather_vertices(int n, const int* idx, const double* q, const double* v, double* out);
__global__ void k_check_state(int64_t n, const double* a, const double* cur, int* flags);

// Templated kernels are launched through host wrappers defined (and
// instantiated for float and double) next to the kernels, so that every
// launch goes through the translation unit that registers the kernel.
template <typename T>
void launch_vertex_rhs(dim3 grid, dim3 block, cudaStream_t st, DModel m, const double* qk, const double* v,
                       const double* cstep, const double* bp, double air_damping, const int* slot_of, double* fslot,
                       T* b, double dt, int residual_mode);
// The contact kernels take the iteration index from *iter: the parity selects
// the current / next self-contact force buffers, and iteration 0 uses the
// learned prediction when pred is given.
template <typename T>
void launch_friction_obstacle(dim3 grid, dim3 block, cudaStream_t st, DModel m, DContacts c, T* b, int self_mode,
                              const int* iter, const float* pred = nullptr, double pred_sv = 0.);
template <typename T>
void launch_friction_self(dim3 grid, dim3 block, cudaStream_t st, DModel m, DContacts c, T* b, double* newf,
                          const int* iter);
// Solve vectors b, y, x are three planes of n values (x, y, z components) in
// pivot order.  y and x of the upper supernodes must be zero before a solve
// (the previous solve's write-back, or launch_solve_prep).  One solve is the
// forward sweep, the backward sweep (with the blocks' write-back) and the
// write-back of the upper columns.
template <typename T>
bool configure_solve(DPlan& P, int shape);  // shared memory and grids; false if the shape does not fit
template <typename T>
void launch_solve_sweeps(cudaStream_t st, const DPlan& P, const T* Wf, const T* Wb, T* b, T* y, T* x, int n,
                         SweepSync sy, WriteBack wb, cudaEvent_t* marks = nullptr);
template <typename T>
void launch_solve_prep(cudaStream_t st, int n, T* x, T* y, SweepSync sy);

// detection (detect_kernels.cu, compiled without FMA contraction)
__global__ void k_obstacle_flags(int N, const double* q, DObstacles obs, unsigned char* flags);
__global__ void k_obstacle_materialize(int N, const double* q, DObstacles obs, const int* idx, const int* vmat,
                                       const double* friction, int n_mat, DContacts c);
__global__ void k_clamp_contacts(int* n, int cap, int* err);
void launch_moving_mesh_lerp(cudaStream_t st, int n3, const double* prev, const double* next, double a, double* cur);
__global__ void k_contact_slots(DContacts c);
__global__ void k_contact_slots_fill(DContacts c);
__global__ void k_contact_slots_reset(DContacts c);

}  // namespace pdfb
