// step_kernels.cu — device kernels of one projective-dynamics step:
// predictor, local step (projections + right-hand side), per-contact
// Coulomb/Signorini projection, self-contact Gauss-Seidel levels,
// Alart-Curnier residual.  Reference citations are relative to the reference
// project root ("SFE" = src/physics/SimulationFrictionEstimation.cpp).
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.hpp"

namespace pdfb {

// ---------------------------------------------------------------------------
// Predictor and per-step constant (SimulationSpeed::initializeStep,
// SimulationSpeed.cpp:62-76; external force SimulationBase.cpp:266-287 with the
// gravity functor m g of simulation_building.cpp:86-92; t_n :294-301).
// c = M t_n - dt A^T A q_n + dt * (attachment part of A^T p), which is the
// part of SimulationSpeed::computeRhs (:238-278) that is constant over a step.
__global__ void k_step_init(DModel m, const double* __restrict__ q, double* __restrict__ v,
                            double* __restrict__ tn, double* __restrict__ qk, double* __restrict__ cstep,
                            double gx, double gy, double gz, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.N) return;
  const double mi = m.mass[i];
  const double g[3] = {gx, gy, gz};
  double ax = 0, ay = 0, az = 0;
  for (int k = m.ata_ptr[i]; k < m.ata_ptr[i + 1]; ++k) {
    const double a = m.ata_val[k];
    const int j = m.ata_col[k];
    ax += a * q[3 * (int64_t)j];
    ay += a * q[3 * (int64_t)j + 1];
    az += a * q[3 * (int64_t)j + 2];
  }
  const double ataq[3] = {ax, ay, az};
  for (int c = 0; c < 3; ++c) {
    const int64_t d = 3 * (int64_t)i + c;
    const double f = mi * g[c];
    const double t = v[d] + dt * ((1. / mi) * f);
    tn[d] = t;
    v[d] = t;
    qk[d] = q[d] + dt * t;
    double cc = mi * t - dt * ataq[c];
    if (m.pin_term) cc += dt * m.pin_term[d];
    cstep[d] = cc;
  }
}

// Bending projections (BendingConstraint::addConstraintProjection,
// BendingConstraint.cpp:106-138): p_b = sqrt(b) * (rest/|L x|) L x, or 0 when
// |L x| <= 1e-25, with L x the mean-value Laplacian at the current iterate.
// Residual mode (FP32 solves) writes p_b - A_b x instead (A_b x = sqrt(b) L x),
// the row's part of the bending force A_b^T (p_b - A_b x).
__global__ void k_bend_proj(DModel m, const double* __restrict__ qk, double* __restrict__ bp, int residual_mode) {
  trace_stamp(m.trace, DTrace::kLocal);
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= m.B) return;
  double3 lb = make_double3(0., 0., 0.);
  for (int k = m.bend_ptr[b]; k < m.bend_ptr[b + 1]; ++k) lb = lb + m.bend_coef[k] * ld3(qk, m.bend_idx[k]);
  const double n = sqrt(dot3(lb, lb));
  const double w = m.bend_w[b];
  double3 p = make_double3(0., 0., 0.);
  if (n > 1e-25) {
    const double s = m.bend_rest[b] / n;
    p = w * make_double3(lb.x * s, lb.y * s, lb.z * s);
  }
  if (residual_mode) p = p - w * lb;
  st3(bp, b, p);
}

// Vertex-centric local step + right-hand side (SimulationBase::computeProjections
// SimulationBase.cpp:314-323, SpringConstraint.cpp:57-69, SimulationSpeed::computeRhs
// SimulationSpeed.cpp:238-278):
//   rhs_i = c_i + dt * ( sum_j kappa_ij normalize(q_i - q_j)          springs
//                        + sum_{rows b containing i} A[b,i] p_b        bending
//                        - d_i v_i )                                   damping
// Vertex i gathers from its 1-ring, so no atomics are needed.  Output goes
// straight to the solve's pivot order.  At contact vertices (slot >= 0) the
// force estimate f = rhs - dt^2 (A^T A v)_i of SFE:337-347 is written too.
// Residual mode (FP32 solves) writes r = rhs - (M + dt^2 A^T A) v instead, in
// its force form r = M (t_n - v) + dt (A^T p - A^T A q^k) - dt D v with
// q^k = q_n + dt v: per spring k (L e - (q_i - q_j)), per bending row
// A[b,i] (p_b - A_b q^k) (k_bend_proj's residual mode), per pin
// w (x0 - q_i) — the same quantity without the A^T A product, each term a
// small force instead of a difference of large ones; f = r + M v.
template <typename T>
__global__ void __launch_bounds__(256, 4) k_vertex_rhs(DModel m, const double* __restrict__ qk, const double* __restrict__ v,
                             const double* __restrict__ cstep, const double* __restrict__ bp,
                             double air_damping, const int* __restrict__ slot_of,
                             double* __restrict__ fslot, T* __restrict__ b, double dt, int residual_mode) {
  if (m.B == 0) trace_stamp(m.trace, DTrace::kLocal);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.N) return;
  const double3 qi = ld3(qk, i);
  double3 acc = make_double3(0., 0., 0.);
  const int bo = m.bend_of[i];
  if (bo >= 0) acc = acc + m.self_bend[i] * ld3(bp, bo);
  const double ks = residual_mode ? m.spring_k[i] : 0.;
  for (int s = m.ring_ptr[i]; s < m.ring_ptr[i + 1]; ++s) {
    const int j = m.ring_idx[s];
    const double3 d = qi - ld3(qk, j);
    acc = acc + m.ring_kappa[s] * normalized3(d);
    if (residual_mode) acc = acc - ks * d;
    const int bj = m.bend_of[j];
    if (bj >= 0) acc = acc + m.ring_bend[s] * ld3(bp, bj);
  }
  const double3 vi = ld3(v, i);
  const int slot = slot_of[i];
  // air damping is switched off at every contact vertex (SimulationBase.cpp:347-396)
  const double di = slot >= 0 ? 0. : air_damping;
  double3 out;
  if (residual_mode) {
    if (m.pin_term) {
      const double pw = m.pin_w[i];
      const double3 pt = ld3(m.pin_term, i);
      acc = acc + make_double3(pt.x - pw * qi.x, pt.y - pw * qi.y, pt.z - pw * qi.z);
    }
    const double mi = m.mass[i];
    const double3 t = ld3(m.tn, i);
    out = make_double3(mi * (t.x - vi.x) + dt * (acc.x - di * vi.x), mi * (t.y - vi.y) + dt * (acc.y - di * vi.y),
                       mi * (t.z - vi.z) + dt * (acc.z - di * vi.z));
    if (slot >= 0) st3(fslot, slot, make_double3(out.x + mi * vi.x, out.y + mi * vi.y, out.z + mi * vi.z));
  } else {
    const double3 c = ld3(cstep, i);
    const double3 rhs = make_double3(c.x + dt * (acc.x - di * vi.x), c.y + dt * (acc.y - di * vi.y),
                                     c.z + dt * (acc.z - di * vi.z));
    out = rhs;
    if (slot >= 0) {
      double ax = 0, ay = 0, az = 0;
      for (int k = m.ata_ptr[i]; k < m.ata_ptr[i + 1]; ++k) {
        const double a = m.ata_val[k];
        const int j = m.ata_col[k];
        ax += a * v[3 * (int64_t)j];
        ay += a * v[3 * (int64_t)j + 1];
        az += a * v[3 * (int64_t)j + 2];
      }
      const double dt2 = dt * dt;
      st3(fslot, slot, make_double3(rhs.x - dt2 * ax, rhs.y - dt2 * ay, rhs.z - dt2 * az));
    }
  }
  const int64_t p = m.iperm[i];
  b[p] = (T)out.x;
  b[p + m.N] = (T)out.y;
  b[p + 2 * (int64_t)m.N] = (T)out.z;
}

template <typename T>
void launch_vertex_rhs(dim3 grid, dim3 block, cudaStream_t st, DModel m, const double* qk, const double* v,
                       const double* cstep, const double* bp, double air_damping, const int* slot_of, double* fslot,
                       T* b, double dt, int residual_mode) {
  k_vertex_rhs<T><<<grid, block, 0, st>>>(m, qk, v, cstep, bp, air_damping, slot_of, fslot, b, dt, residual_mode);
}
template void launch_vertex_rhs<double>(dim3, dim3, cudaStream_t, DModel, const double*, const double*, const double*,
                                        const double*, double, const int*, double*, double*, double, int);
template void launch_vertex_rhs<float>(dim3, dim3, cudaStream_t, DModel, const double*, const double*, const double*,
                                       const double*, double, const int*, double*, float*, double, int);

// Adds g into entry p of the three planes (stride n) of a solve vector.
__device__ __forceinline__ void atomic_add3(double* b, int64_t p, int n, double3 g) {
  atomicAdd(b + p, g.x);
  atomicAdd(b + p + n, g.y);
  atomicAdd(b + p + 2 * (int64_t)n, g.z);
}
__device__ __forceinline__ void atomic_add3(float* b, int64_t p, int n, double3 g) {
  atomicAdd(b + p, (float)g.x);
  atomicAdd(b + p + n, (float)g.y);
  atomicAdd(b + p + 2 * (int64_t)n, (float)g.z);
}

__device__ __forceinline__ double3 basis_t(const double* B, double3 v) {
  // B^T v with B stored by columns (n, t, b)
  return make_double3(B[0] * v.x + B[1] * v.y + B[2] * v.z, B[3] * v.x + B[4] * v.y + B[5] * v.z,
                      B[6] * v.x + B[7] * v.y + B[8] * v.z);
}
__device__ __forceinline__ double3 basis_v(const double* B, double3 r) {
  // B r : component i = (B(i,0) r0 + B(i,1) r1) + B(i,2) r2
  return make_double3(B[0] * r.x + B[3] * r.y + B[6] * r.z, B[1] * r.x + B[4] * r.y + B[7] * r.z,
                      B[2] * r.x + B[5] * r.y + B[8] * r.z);
}

// Friction-cone projection shared by obstacle and self contacts (SFE:376-394,
// 503-520): r = -forceLoc, tangential part clamped to mu r_N.
__device__ __forceinline__ double3 cone_project(double3 fl, double mu) {
  double3 r = make_double3(-fl.x, -fl.y, -fl.z);
  const double rtn = sqrt(r.y * r.y + r.z * r.z);
  if (rtn > mu * r.x) {
    r.y *= mu * r.x / rtn;
    r.z *= mu * r.x / rtn;
  }
  return r;
}

// Obstacle contacts (SFE:350-423).  One thread per contact.
// pred (learned warm start, first iteration of a step only): the predicted
// local force y_k, in units of s_r = m |g| dt (pred_sv = |g| dt), replaces the
// projection; it is projected on the friction cone, and a non-finite
// prediction falls back to the projection for that contact.
template <typename T>
__global__ void k_friction_obstacle(DModel m, DContacts c, T* __restrict__ b, int self_mode, const int* __restrict__ iter,
                                    const float* __restrict__ pred, double pred_sv) {
  trace_stamp(m.trace, DTrace::kFriction);
  const int C = *c.n_contacts;
  const int S = self_mode ? *c.n_self : 0;
  const int it = *iter;
  const int cur = it & 1, nxt = 1 - cur;
  if (it != 0) pred = nullptr;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
    const int vid = c.c_vertex[k];
    const int slot = c.c_slot[k];
    const double* B = c.c_basis + 9 * (int64_t)k;
    const double mv = m.mass[vid];
    double3 r;
    bool predicted = false;
    if (pred) {
      const double sr = mv * pred_sv;
      r = make_double3(sr * (double)pred[3 * (int64_t)k], sr * (double)pred[3 * (int64_t)k + 1],
                       sr * (double)pred[3 * (int64_t)k + 2]);
      if (isfinite(r.x) && isfinite(r.y) && isfinite(r.z)) {
        predicted = true;
        if (!(r.x > 0.)) {  // predicted separation
          st3(c.c_force, k, make_double3(0., 0., 0.));
          c.c_active[k] = 0;
          continue;
        }
        const double mu = c.c_mu[k];
        const double rtn = sqrt(r.y * r.y + r.z * r.z);
        if (rtn > mu * r.x) {
          r.y *= mu * r.x / rtn;
          r.z *= mu * r.x / rtn;
        }
      }
    }
    if (!predicted) {
      double3 f = ld3(c.f, slot);
      if (self_mode) f = f + ld3(c.sf[cur], slot);
      const double3 sp = ld3(c.c_speed, k);
      const double3 fl = basis_t(B, make_double3(f.x - mv * sp.x, f.y - mv * sp.y, f.z - mv * sp.z));
      if (fl.x > 0.) {  // take-off: the stored local force keeps its old value
        c.c_active[k] = 0;
        continue;
      }
      r = cone_project(fl, c.c_mu[k]);
    }
    c.c_active[k] = 1;
    st3(c.c_force, k, r);
    const double3 g = basis_v(B, r);
    if (!self_mode || S == 0) atomic_add3(b, m.iperm[vid], m.N, g);
    if (self_mode) st3(c.cf[nxt], slot, g);
  }
}
template <typename T>
void launch_friction_obstacle(dim3 grid, dim3 block, cudaStream_t st, DModel m, DContacts c, T* b, int self_mode,
                              const int* iter, const float* pred, double pred_sv) {
  k_friction_obstacle<T><<<grid, block, 0, st>>>(m, c, b, self_mode, iter, pred, pred_sv);
}
template void launch_friction_obstacle<double>(dim3, dim3, cudaStream_t, DModel, DContacts, double*, int, const int*,
                                               const float*, double);
template void launch_friction_obstacle<float>(dim3, dim3, cudaStream_t, DModel, DContacts, float*, int, const int*,
                                              const float*, double);

// Self contacts (SFE:431-587).  One CTA walks the breadth-first levels in
// order; inside a level every contact is estimated from the buffers as they
// stood before the level (compute phase), then the previous forces are removed
// and the new ones added (update phase).  At the end the contact and
// self-contact forces are added to the right-hand side and the buffer that
// becomes "next" is cleared.
template <typename T>
__global__ void k_friction_self(DModel m, DContacts c, T* __restrict__ b, double* __restrict__ newf,
                                const int* __restrict__ iter) {
  trace_stamp(m.trace, DTrace::kSelfFriction);
  const int cur = (*iter) & 1, nxt = 1 - cur;
  const int S = *c.n_self;
  const int C = *c.n_contacts;
  const int nl = *c.n_levels;
  if (S > 0) {
    for (int l = 0; l < nl; ++l) {
      const int l0 = c.level_ptr[l], l1 = c.level_ptr[l + 1];
      for (int i = l0 + threadIdx.x; i < l1; i += blockDim.x) {
        const int sc = c.level_order[i];
        const int sa = c.s_slota[sc], sb = c.s_slotb[sc];
        const int va = c.s_vertex[sc], vb = c.s_partner[sc];
        const double* Bm = c.s_basis + 9 * (int64_t)sc;
        const double mA = m.mass[va], mB = m.mass[vb];
        const double3 rem = ld3(c.s_remember, sc);
        const double3 fA = ld3(c.f, sa) + ld3(c.cf[nxt], sa) + ld3(c.sf[cur], sa) + ld3(c.sf[nxt], sa) - rem;
        const double3 fB = ld3(c.f, sb) + ld3(c.cf[nxt], sb) + ld3(c.sf[cur], sb) + ld3(c.sf[nxt], sb) + rem;
        const double ia = 1. / mA, ib = 1. / mB;
        const double3 fl = basis_t(Bm, make_double3(ia * fA.x - ib * fB.x, ia * fA.y - ib * fB.y, ia * fA.z - ib * fB.z));
        double3 g = make_double3(0., 0., 0.);
        if (!(fl.x > 0.)) {
          double3 r = cone_project(fl, c.s_mu[sc]);
          const double sc2 = (mA * mB) / (mA + mB);
          r = make_double3(sc2 * r.x, sc2 * r.y, sc2 * r.z);
          st3(c.s_force, sc, r);
          g = basis_v(Bm, r);
        }
        st3(newf, sc, g);
      }
      __syncthreads();
      for (int i = l0 + threadIdx.x; i < l1; i += blockDim.x) {
        const int sc = c.level_order[i];
        const int sa = c.s_slota[sc], sb = c.s_slotb[sc];
        const double3 prev = ld3(c.s_remember, sc);
        const double3 g = ld3(newf, sc);
        atomicAdd(c.sf[cur] + 3 * sa, -prev.x);
        atomicAdd(c.sf[cur] + 3 * sa + 1, -prev.y);
        atomicAdd(c.sf[cur] + 3 * sa + 2, -prev.z);
        atomicAdd(c.sf[cur] + 3 * sb, prev.x);
        atomicAdd(c.sf[cur] + 3 * sb + 1, prev.y);
        atomicAdd(c.sf[cur] + 3 * sb + 2, prev.z);
        atomicAdd(c.sf[nxt] + 3 * sa, g.x);
        atomicAdd(c.sf[nxt] + 3 * sa + 1, g.y);
        atomicAdd(c.sf[nxt] + 3 * sa + 2, g.z);
        atomicAdd(c.sf[nxt] + 3 * sb, -g.x);
        atomicAdd(c.sf[nxt] + 3 * sb + 1, -g.y);
        atomicAdd(c.sf[nxt] + 3 * sb + 2, -g.z);
        st3(c.s_remember, sc, g);
      }
      __syncthreads();
    }
    const int ns = *c.n_slots;
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
      const double3 g = ld3(c.cf[nxt], s) + ld3(c.sf[nxt], s);
      const int64_t p = m.iperm[c.slot_vertex[s]];
      atomic_add3(b, p, m.N, g);
    }
    __syncthreads();
  }
  (void)C;
  // buffer swap: the old "current" buffers become "next" and start from zero
  if (S > 0 || C > 0) {
    const int ns = *c.n_slots;
    for (int s = threadIdx.x; s < 3 * ns; s += blockDim.x) {
      c.cf[cur][s] = 0.;
      c.sf[cur][s] = 0.;
    }
  }
}
template <typename T>
void launch_friction_self(dim3 grid, dim3 block, cudaStream_t st, DModel m, DContacts c, T* b, double* newf,
                          const int* iter) {
  k_friction_self<T><<<grid, block, 0, st>>>(m, c, b, newf, iter);
}
template void launch_friction_self<double>(dim3, dim3, cudaStream_t, DModel, DContacts, double*, double*, const int*);
template void launch_friction_self<float>(dim3, dim3, cudaStream_t, DModel, DContacts, float*, double*, const int*);

// Alart-Curnier residual with rho = 1 (coulomb_util.cpp:92-152) for every
// contact after the solve (SFE:590-652).  acc[4] += {sum |AC|, max |AC|,
// sum |AC_N|, sum |AC_T|}.
__device__ __forceinline__ double dmax0(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin0(double a, double b) { return (b < a) ? b : a; }

__device__ double ac_norm(double3 u, double3 r, double mu, double* an, double* at) {
  const double N = dmax0(0., r.x - u.x) - r.x;
  const double dx = r.y - u.y, dy = r.z - u.z;
  const double dn = sqrt(dx * dx + dy * dy);
  const double radius = dmax0(0., mu * r.x / dn);
  const double mm = dmin0(1., radius);
  const double tx = dx * mm - r.y, ty = dy * mm - r.z;
  *an = fabs(N);
  *at = sqrt(tx * tx + ty * ty);
  return sqrt(N * N + tx * tx + ty * ty);
}

__device__ __forceinline__ void atomic_max_pos(double* addr, double val) {
  // valid for non-negative doubles: their bit patterns order like int64
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(val));
}

__global__ void k_alart_curnier(DContacts c, const double* __restrict__ v, double* __restrict__ hist, IterCtl ctl) {
  trace_stamp(ctl.trace, DTrace::kAcBegin);
  const int C = *c.n_contacts, S = *c.n_self;
  const int it = *ctl.iter;
  double* acc = hist + 4 * (int64_t)it;
  double s = 0, mx = 0, sn = 0, st = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C + S; k += gridDim.x * blockDim.x) {
    double an, at, n;
    if (k < C) {
      const double* B = c.c_basis + 9 * (int64_t)k;
      const double3 u = basis_t(B, ld3(v, c.c_vertex[k]) - ld3(c.c_speed, k));
      n = ac_norm(u, ld3(c.c_force, k), c.c_mu[k], &an, &at);
      c.c_ac[k] = n;
    } else {
      const int q = k - C;
      const double* B = c.s_basis + 9 * (int64_t)q;
      const double3 u = basis_t(B, ld3(v, c.s_vertex[q]) - ld3(v, c.s_partner[q]));
      n = ac_norm(u, ld3(c.s_force, q), c.s_mu[q], &an, &at);
      c.s_ac[q] = n;
    }
    if (c.ac_trace && it < c.trace_k) {
      double* tr = c.ac_trace + 2 * ((int64_t)it * c.trace_stride + k);
      tr[0] = at;
      tr[1] = an;
    }
    s += n;
    mx = fmax(mx, n);
    sn += an;
    st += at;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    sn += __shfl_xor_sync(0xffffffffu, sn, o);
    st += __shfl_xor_sync(0xffffffffu, st, o);
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  // block reduction, then one set of atomics per block that had work
  __shared__ double red[4][32];
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][warp] = s;
    red[1][warp] = mx;
    red[2][warp] = sn;
    red[3][warp] = st;
  }
  __syncthreads();
  if (threadIdx.x == 0 && (int64_t)blockIdx.x * blockDim.x < (int64_t)(C + S)) {
    for (int k = 1; k < nw; ++k) {
      s += red[0][k];
      mx = fmax(mx, red[1][k]);
      sn += red[2][k];
      st += red[3][k];
    }
    atomicAdd(acc, s);
    atomic_max_pos(acc + 1, mx);
    atomicAdd(acc + 2, sn);
    atomicAdd(acc + 3, st);
  }
  // the last block to finish closes the iteration
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(ctl.blocks_done, 1u);
    if (prev == gridDim.x - 1) {
      *ctl.blocks_done = 0u;
      if (ctl.trace.stamps && it >= 0 && it < ctl.trace.k)
        ctl.trace.stamps[(int64_t)DTrace::kAcEnd * ctl.trace.k + it] = global_ns();
      const int k1 = it + 1;
      *ctl.iter = k1;
      *ctl.iter_total += 1;
      if (ctl.set_cond) {
        const int nc = C + S;
        const double mean = nc > 0 ? __ldcg(acc) / nc : 0.;
        const bool stop = k1 >= ctl.kmax || (ctl.tol > 0. && nc > 0 && mean <= ctl.tol);
        cudaGraphSetConditional(ctl.cond, stop ? 0u : 1u);
      }
    }
  }
}

// Check of an uploaded array against the one it would replace: flags[0]
// becomes non-zero if any of the n values is NaN or infinite, flags[1] if any
// differs bitwise from cur.
__global__ void k_check_state(int64_t n, const double* __restrict__ a, const double* __restrict__ cur, int* flags) {
  int bad = 0, diff = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    bad |= !isfinite(a[k]);
    diff |= __double_as_longlong(a[k]) != __double_as_longlong(cur[k]);
  }
  bad = __any_sync(0xffffffffu, bad);
  diff = __any_sync(0xffffffffu, diff);
  if ((threadIdx.x & 31) == 0) {
    if (bad) atomicOr(flags, 1);
    if (diff) atomicOr(flags + 1, 1);
  }
}

// Positions and velocities of listed vertices: out[0 .. 3n) = q, out[3n .. 6n) = v.
__global__ void k_gather_vertices(int n, const int* __restrict__ idx, const double* __restrict__ q,
                                  const double* __restrict__ v, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  st3(out, k, ld3(q, idx[k]));
  st3(out + 3 * (int64_t)n, k, ld3(v, idx[k]));
}

// End of step (SFE::updateScene SFE:64-87): q <- q^K.  Block 0 also copies
// the step's counters and iteration clock to the host-mapped record.
__global__ void k_finalize(int n3, const double* __restrict__ qk, double* __restrict__ q, StepOut o) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n3) q[d] = qk[d];
  if (o.counts && blockIdx.x == 0) {
    if (threadIdx.x == 0) {
      o.counts[0] = *o.n_contacts;
      o.counts[1] = *o.n_self;
      o.counts[2] = *o.n_levels;
      o.counts[3] = *o.iter;
    }
    for (int k = threadIdx.x; k < o.n_stamps; k += blockDim.x) o.stamps_out[k] = o.stamps[k];
  }
}

}  // namespace pdfb
