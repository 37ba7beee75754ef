// device.cuh — shared device types and small helpers for the step-loop kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pdfb {

// Per-iteration device clock of the current step: the first thread of block 0
// of a few kernels writes %globaltimer (ns) at entry, indexed by the PD
// iteration the kernel belongs to.  Rows of stamps[kRows * k]: local step
// start, obstacle friction entry, self friction entry, forward sweep entry,
// Alart-Curnier entry, Alart-Curnier end (written by its last block).
struct DTrace {
  const int* iter;               // PD iterations completed in this step
  unsigned long long* stamps;    // kRows * k, or null (no trace)
  int k;                         // iteration capacity
  static constexpr int kRows = 6;
  enum Row { kLocal = 0, kFriction = 1, kSelfFriction = 2, kSolve = 3, kAcBegin = 4, kAcEnd = 5 };
};

#ifdef __CUDACC__
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// called by every thread; only thread 0 of block 0 writes
__device__ __forceinline__ void trace_stamp(const DTrace& t, int row) {
  if (t.stamps && blockIdx.x == 0 && threadIdx.x == 0) {
    const int it = *t.iter;
    if (it >= 0 && it < t.k) t.stamps[(int64_t)row * t.k + it] = global_ns();
  }
}
#endif

// Read-only model tables (original vertex order unless stated).
struct DModel {
  int N, B;                 // vertices, bending rows
  const double* mass;       // N
  const int* ring_ptr;      // N+1
  const int* ring_idx;
  const double* ring_kappa; // spring sqrt(k)*(sqrt(k)*L)
  const double* ring_bend;  // coefficient of i in the bending row of the neighbour
  const int* bend_of;       // N: own bending row or -1
  const double* self_bend;  // N
  const int* bend_ptr;      // B+1
  const int* bend_idx;
  const double* bend_coef;
  const double* bend_w;     // B
  const double* bend_rest;  // B
  const double* pin_term;   // 3N or null
  const double* spring_k;   // N: stiffness of the vertex's springs
  const double* pin_w;      // N or null: summed pin weight of the vertex
  const double* tn;         // 3N: predictor t_n of the current step
  const int* ata_ptr;       // N+1, A^T A in CSR
  const int* ata_col;
  const double* ata_val;
  const int* perm;          // pivot position -> vertex
  const int* iperm;         // vertex -> pivot position
  DTrace trace;             // iteration clock (local step and friction rows)
};

// Contacts of the current step (device-resident, counts on the device).
struct DContacts {
  int* n_contacts;          // [1]
  int* c_vertex;            // cap
  double* c_normal;         // 3 cap
  double* c_speed;          // 3 cap
  double* c_mu;             // cap
  double* c_basis;          // 9 cap (columns n, t, b)
  double* c_force;          // 3 cap persistent local forces
  double* c_ac;             // cap
  int* c_slot;              // cap: slot of the contact vertex
  double* c_gap;            // cap: signed distance to the obstacle surface
  int* c_active;            // cap: 1 if the last projection was not a take-off
  int* n_self;              // [1]
  int* s_vertex;            // cap
  int* s_partner;           // cap
  int* s_face;              // 3 cap
  double* s_normal;         // 3 cap
  double* s_mu;             // cap
  double* s_basis;          // 9 cap
  double* s_force;          // 3 cap persistent local forces
  double* s_ac;             // cap
  int* s_slota;             // cap
  int* s_slotb;             // cap
  double* s_remember;       // 3 cap
  int* n_levels;            // [1]
  int* level_ptr;           // cap+1
  int* level_order;         // cap
  int* slot_of;             // N, -1 when not involved
  int* n_slots;             // [1]
  int* slot_vertex;         // cap slots
  double* f;                // 3 * slots: forces f = rhs - dt^2 A^T A v at slots
  double* cf[2];            // contact forces per slot (self mode)
  double* sf[2];            // self contact forces per slot
  int cap, slot_cap, self_cap;
  // per-iteration Alart-Curnier norms (tangential, |normal|) of every
  // contact, [iteration][contact][2] with contact stride trace_stride; null
  // unless tracing is on
  double* ac_trace;
  int trace_stride, trace_k;
};

__device__ __forceinline__ double3 ld3(const double* p, int64_t i) {
  return make_double3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
__device__ __forceinline__ void st3(double* p, int64_t i, double3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}
__device__ __forceinline__ double3 operator+(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 operator-(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 operator*(double s, double3 a) { return make_double3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// Eigen-style normalized(): divide by the norm unless zero.
__device__ __forceinline__ double3 normalized3(double3 a) {
  double z = dot3(a, a);
  if (z > 0.) {
    double s = sqrt(z);
    return make_double3(a.x / s, a.y / s, a.z / s);
  }
  return a;
}

}  // namespace pdfb
