// handle.hpp — the state behind a pdf_handle (host orchestration of the
// device step loop).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/pdf.h"
#include "factor.hpp"
#include "kernels.hpp"
#include "mlp.hpp"
#include "model.hpp"

namespace pdfb {

struct DeviceBuffers {
  // model tables
  double *mass = nullptr, *ring_kappa = nullptr, *ring_bend = nullptr, *self_bend = nullptr;
  int *ring_ptr = nullptr, *ring_idx = nullptr, *bend_of = nullptr, *bend_ptr = nullptr, *bend_idx = nullptr;
  double *bend_coef = nullptr, *bend_w = nullptr, *bend_rest = nullptr, *pin_term = nullptr;
  double *spring_k = nullptr, *pin_w = nullptr;
  int *ata_ptr = nullptr, *ata_col = nullptr;
  double* ata_val = nullptr;
  int *perm = nullptr, *iperm = nullptr, *vmat = nullptr;
  double* friction = nullptr;
  int* tris = nullptr;  // 3T scene-global
  std::vector<double*> obstacle_v;
  std::vector<int*> obstacle_t;
  DObstacle* obstacles = nullptr;
  int* vmesh = nullptr;
  int* ob_best = nullptr;  // per (obstacle, vertex): closest mesh-obstacle triangle
  // state
  double *q = nullptr, *v = nullptr, *tn = nullptr, *qk = nullptr, *cstep = nullptr, *bp = nullptr;
  // solve
  DPlan plan{};       // device copy of the sweep plan (blocks, upper items)
  SweepPlan host_plan;
  SnInfo* sn = nullptr;
  int* rows = nullptr;
  double *Wf64 = nullptr, *Wb64 = nullptr;  // tiled factor copies (forward / backward)
  float *Wf32 = nullptr, *Wb32 = nullptr;
  SweepSync sync{};
  double *b64 = nullptr, *y64 = nullptr, *x64 = nullptr;
  float *b32 = nullptr, *y32 = nullptr, *x32 = nullptr;
  // contacts
  DContacts c{};
  unsigned char* flags = nullptr;
  int* sel_idx = nullptr;
  void* cub_tmp = nullptr;
  size_t cub_tmp_bytes = 0;
  double* newf = nullptr;
  double* ac_hist = nullptr;  // 4 per iteration
  // device iteration control (IterCtl): iterations of the current step, of
  // the handle's lifetime, and the AC kernel's block-completion counter
  int* iter = nullptr;
  unsigned long long* stamps = nullptr;  // DTrace::kRows * K iteration clock
  long long* iter_total = nullptr;
  unsigned int* blocks_done = nullptr;
  // self-collision detection scratch (selfdetect.cu)
  void* self_ws = nullptr;
};

}  // namespace pdfb

// Clock of one key-framed moving-mesh obstacle (MovingMesh.cpp:28-84):
// every key frame stays resident on the device; `cur` is the interpolated mesh
// that detection reads.
struct MovingClock {
  int n_frames = 0, n_vertices = 0, next = 1;
  double interval = 0., clock = 0.;
  const double* frames = nullptr;
  double* cur = nullptr;
  double frame_time(int f) const { return (double)f * interval; }
  bool in_movement() const { return clock >= frame_time(next - 1) && clock <= frame_time(next); }
};

// One step's timing record: CUDA events around its phases, and the
// host-mapped counters and iteration clock that k_finalize fills.  Events:
// 0 step start, 1 after obstacle detection, 2 after self detection, 3 after
// self-contact ordering, 4 iterations begin, 5 iterations end, 6 step end.
struct StepRecord {
  cudaEvent_t ev[7] = {};
  int* counts = nullptr;                 // contacts, self contacts, levels, iterations
  unsigned long long* stamps = nullptr;  // DTrace::kRows * K, ns
  int* counts_dev = nullptr;             // device views of the same memory
  unsigned long long* stamps_dev = nullptr;
  bool pending = false;
};

// Per-sample statistics, in microseconds, of the reference's stats file
// (SimulationBase::exportStats SimulationBase.cpp:474-494 and
// SimulationFrictionEstimation::exportStats SFE:756-771).
struct StatSamples {
  std::vector<double> iteration, detection, self_detection, solver, rhs, step, rhs_base, friction, self_friction,
      ordering;
  std::vector<int64_t> collisions, self_collisions;
};

struct pdf_handle {
  pdfb::Model model;
  pdfb::Factor fac;
  pdf_params prm{};
  pdfb::DeviceBuffers d;
  pdfb::DModel dm{};
  pdfb::DObstacles obs{};
  std::vector<pdfb::DObstacle> host_obs;
  std::vector<MovingClock> moving;  // one per obstacle (n_frames = 0: not moving)
  std::vector<pdfb::MeshBVH*> mesh_bvh;  // one per obstacle (null: not a mesh obstacle)
  std::vector<int> bvh_since;           // moving meshes: steps since the hierarchy was built
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[8] = {};
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  int n_levels = 0;
  int cap_contacts = 0, cap_self = 0;
  double time = 0.;
  std::string err;
  pdf_step_report last{};
  pdf_stats stats{};
  std::vector<double> residual_hist;
  int64_t launches_outside = 0;  // kernels launched outside PD iterations so far
  // step records, reused round-robin; a record is harvested (its events
  // waited for) before reuse and at the end of every pdf_step call
  std::vector<StepRecord> ring;
  int ring_head = 0;
  void* ring_host = nullptr;  // host-mapped memory of all records
  StatSamples samples;
  double lhs_ms = 0.;  // model and LHS assembly (host)
  // frame output: two pinned copies of q filled on a copy stream; frame_guard
  // is the slot whose copy the next write-back of q must wait for (-1: none)
  double* frame_host[2] = {nullptr, nullptr};
  cudaEvent_t frame_ev[2] = {nullptr, nullptr};
  cudaEvent_t frame_ready = nullptr;
  cudaStream_t copy_stream = nullptr;
  int frame_guard = -1;
  // state upload: device staging copies of q, v, the non-finite flag and its
  // pinned host image
  double* stage = nullptr;  // 6N: q then v
  int* bad_dev = nullptr;
  int* bad_host = nullptr;
  // log reads: device index list and gathered q, v
  int* gather_idx = nullptr;
  double* gather_out = nullptr;
  int gather_cap = 0;
  // iterate-to-tolerance graph: the iterations are one conditional WHILE node
  cudaGraphConditionalHandle cond{};
  bool capturing_cond = false;
  std::vector<double> host_time_before_start;
  bool fp32 = false;
  // learned warm start (mlp.cu): device weights, per-contact features and
  // predictions, the per-vertex impulse memory of the previous step (valid
  // where rprev_tag == mlp_tag - 1) and the optional sample log
  float* mlp_w = nullptr;
  bool mlp_ready = false;
  float *mlp_X = nullptr, *mlp_Y = nullptr;
  double* rprev = nullptr;
  int* rprev_tag = nullptr;
  int mlp_tag = 0;
  float *log_X = nullptr, *log_T = nullptr;
  int* log_n = nullptr;
  int log_cap = 0;
};

namespace pdfb {
// api.cu: message returned by pdf_global_error()
void set_global_error(const std::string& msg);
// selfdetect.cu
int self_detect_init(pdf_handle* h);
int self_detect_step(pdf_handle* h);  // self contacts of the step (detection + pairing)
void self_levels_step(pdf_handle* h); // breadth-first Gauss-Seidel levels (after slots)
void self_detect_free(pdf_handle* h);
int standalone_candidates(const double* pos, int nv, const int* tris, int nt, double tol, int* pairs, int cap,
                          int* n, int device, std::string& err);
int standalone_self(const double* pos, int nv, const int* tris, int nt, double tol, pdf_contact* out, int cap,
                    int* n, int device, std::string& err);
}  // namespace pdfb
