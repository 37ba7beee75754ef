// api.cu — the C ABI (include/pdf.h): handle creation, the step loop and
// state / contact / statistics read-back.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <fstream>
#include <sstream>
#include <ios>
#include <limits>
#include <ostream>
#include <random>
#include <stdexcept>
#include <string>

#include "../../include/pdf.h"
#include "handle.hpp"

using namespace pdfb;

namespace {

thread_local std::string g_error;

struct CudaFail : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define CK(x)                                                                                  \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess)                                                                     \
      throw CudaFail(std::string(#x) + ": " + cudaGetErrorString(e_));                         \
  } while (0)

template <typename T>
T* dalloc(size_t n) {
  T* p = nullptr;
  if (n == 0) n = 1;
  CK(cudaMalloc((void**)&p, n * sizeof(T)));
  return p;
}
template <typename T>
T* upload(const std::vector<T>& v) {
  T* p = dalloc<T>(v.size());
  if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return p;
}

constexpr int kThreads = 256;
inline int blocks_for(int64_t n) { return (int)std::max<int64_t>(1, (n + kThreads - 1) / kThreads); }
constexpr int kStrideBlocks = 592;  // 4 x 148 SMs for grid-stride kernels

// Work items of the upper supernodes are at most 32 x chunk elements and the
// subtree blocks reach up to the cut level; both are chosen per scene by the
// autotuner in create_impl among these.
constexpr int kChunk = 64;
constexpr int kCutLevel = 4;  // host emulation check (pdf_factor_check)
constexpr int kRecords = 64;  // step records in flight before the oldest is harvested
constexpr int kChunkCandidates[3] = {32, 64, 128};
constexpr int kCutCandidates = 8;  // cut levels 0 .. 7
constexpr int kBlockShape = 1;     // block kernels: 2 CTAs of 8 warps per SM
// the launch shapes tried at every cut level and mode (2 CTAs of 8 consumer
// warps, 4 CTAs of 4 per SM); the others only at the best of those
constexpr int kStageOneShapes[2] = {1, 3};
// polls of a dependency counter before a sweep gives up (each poll sleeps
// about 32 ns): far above any legitimate wait
constexpr int kMaxSpins = 1 << 22;

template <typename T>
void free_dev(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

void free_plan(DPlan& P) {
  free_dev(P.fup);
  free_dev(P.bup);
  free_dev(P.fblk);
  free_dev(P.bblk);
  free_dev(P.fitem);
  free_dev(P.bitem);
  free_dev(P.upper_cols);
  free_dev(P.rows_loc);
  free_dev(P.bidx);
  free_dev(P.child);
}

// Sweep plan (subtree blocks + upper work items, factor.hpp) on the device.
// The completion counters are cumulative per schedule, so they restart here.
void build_schedule(pdf_handle* h, int chunk, int cut_level, int upper_mode = 0, int shape = kBlockShape) {
  const Factor& f = h->fac;
  SweepPlan& hp = h->d.host_plan;
  build_sweep_plan(f, chunk, cut_level, hp);
  DPlan& P = h->d.plan;
  free_plan(P);
  if (h->d.sn) cudaFree(h->d.sn);
  h->d.sn = upload(hp.sn);
  if (!h->d.rows) h->d.rows = upload(f.rows);
  P.fup = upload(hp.fupi);
  P.bup = upload(hp.bupi);
  P.nfup = (int)hp.fupi.size();
  P.nbup = (int)hp.bupi.size();
  P.sn = h->d.sn;
  P.rows = h->d.rows;
  P.fblk = upload(hp.fblk);
  P.bblk = upload(hp.bblk);
  P.nblk = (int)hp.fblk.size();
  P.fitem = upload(hp.fitem);
  P.bitem = upload(hp.bitem);
  P.upper_cols = upload(hp.upper_cols);
  P.n_upper = (int)hp.upper_cols.size();
  P.perm = h->d.perm;
  P.rows_loc = upload(hp.rows_loc);
  P.bidx = upload(hp.bidx.empty() ? std::vector<int>(kSlabMax, 0) : hp.bidx);
  P.child = upload(hp.child.empty() ? std::vector<int>(2, 0) : hp.child);
  P.max_cols = hp.max_block_cols;
  P.max_ext = hp.max_block_ext;
  P.max_items = hp.max_block_items;
  P.n_flev = (int)hp.fup_lev.size() - 1;
  P.n_blev = (int)hp.bup_lev.size() - 1;
  const bool levels_fit = P.n_flev <= kMaxUpperLevels && P.n_blev <= kMaxUpperLevels;
  P.upper_mode = upper_mode == 1 && levels_fit ? 1 : 0;
  for (int k = 0; k <= kMaxUpperLevels; ++k) {
    P.flev[k] = levels_fit && k <= P.n_flev ? hp.fup_lev[k] : 0;
    P.blev[k] = levels_fit && k <= P.n_blev ? hp.bup_lev[k] : 0;
  }
  // the requested launch shape of the block kernels, else one CTA of 8 warps
  // per SM (P.block_shape tells which)
  auto configure = [&](int sh) { return h->fp32 ? configure_solve<float>(P, sh) : configure_solve<double>(P, sh); };
  if (!configure(shape) && !configure(0))
    throw CudaFail("the sweep's block kernels do not fit the device's shared memory");
  h->n_levels = f.n_levels;
  h->stats.sweep_chunk = chunk;
  h->stats.sweep_cut_level = cut_level;
  h->stats.sweep_upper_mode = P.upper_mode;
  h->stats.sweep_block_shape = P.block_shape;
  h->stats.sweep_block_warps = P.block_warps;
  h->stats.sweep_block_ctas = P.block_ctas;
  h->stats.sweep_ring_stages[0] = P.ring_f;
  h->stats.sweep_ring_stages[1] = P.ring_b;
  h->stats.sweep_upper_levels = P.n_flev;
  h->stats.sweep_blocks = P.nblk;
  h->stats.sweep_block_elems = hp.block_elems;
  h->stats.sweep_upper_elems = hp.upper_elems;
  // dependency counters start at zero, the solve counter at one
  SweepSync& sy = h->d.sync;
  if (!sy.queue) {
    sy.queue = dalloc<int>(4);
    sy.epoch = dalloc<unsigned long long>(1);
    sy.fdone = dalloc<unsigned long long>(f.n_sn);
    sy.bdone = dalloc<unsigned long long>(f.n_sn);
    sy.err = dalloc<int>(1);
    sy.max_spins = kMaxSpins;
  }
  CK(cudaMemset(sy.queue, 0, 4 * sizeof(int)));
  const unsigned long long one = 1ULL;
  CK(cudaMemcpy(sy.epoch, &one, sizeof(one), cudaMemcpyHostToDevice));
  CK(cudaMemset(sy.fdone, 0, f.n_sn * sizeof(unsigned long long)));
  CK(cudaMemset(sy.bdone, 0, f.n_sn * sizeof(unsigned long long)));
  CK(cudaMemset(sy.err, 0, sizeof(int)));
  sy.trace = DTrace{h->d.iter, h->d.stamps, std::max(1, h->prm.local_global_iterations)};
}

void autotune_schedule(pdf_handle* h);

// Warm-start feature / prediction buffers and the impulse memory.
void ensure_mlp_buffers(pdf_handle* h) {
  if (h->mlp_X) return;
  const size_t cc = h->cap_contacts;
  h->mlp_X = dalloc<float>(kMlpIn * cc);
  h->mlp_Y = dalloc<float>(kMlpOut * cc);
  h->rprev = dalloc<double>(3 * (size_t)h->dm.N);
  h->rprev_tag = dalloc<int>(h->dm.N);
  CK(cudaMemset(h->rprev, 0, 3 * (size_t)h->dm.N * sizeof(double)));
  CK(cudaMemset(h->rprev_tag, 0x80, h->dm.N * sizeof(int)));  // large negative tags: no memory yet
}

// Weights file: "PDFMLP01", int32 {in, hidden, out, count}, count floats.
constexpr char kMlpMagic[8] = {'P', 'D', 'F', 'M', 'L', 'P', '0', '1'};
void load_weights_file(const std::string& path, float* w) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::ios_base::failure("cannot open MLP weights file " + path);
  char magic[8];
  int32_t hdr[4];
  in.read(magic, 8);
  in.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
  if (!in || std::memcmp(magic, kMlpMagic, 8) != 0) throw std::ios_base::failure("not an MLP weights file: " + path);
  if (hdr[0] != kMlpIn || hdr[1] != kMlpHidden || hdr[2] != kMlpOut || hdr[3] != kMlpParams)
    throw std::invalid_argument("MLP weights file has another network shape: " + path);
  in.read(reinterpret_cast<char*>(w), kMlpParams * sizeof(float));
  if (!in) throw std::ios_base::failure("truncated MLP weights file " + path);
  for (int i = 0; i < kMlpParams; ++i)
    if (!std::isfinite(w[i])) throw std::invalid_argument("non-finite value in MLP weights file " + path);
}

// Seeded He initialisation: W ~ N(0, 2 / fan_in) (output layer scaled by 0.1), b = 0.
void mlp_init_host(float* w, uint64_t seed);
}  // namespace
namespace pdfb {
void mlp_init_params(float* w, uint64_t seed) { mlp_init_host(w, seed); }
}  // namespace pdfb
namespace {
void mlp_init_host(float* w, uint64_t seed) {
  std::mt19937_64 rng(seed);
  std::normal_distribution<double> nd(0., 1.);
  int o = 0;
  auto layer = [&](int nout, int nin, double scale) {
    const double sd = scale * std::sqrt(2. / nin);
    for (int i = 0; i < nout * nin; ++i) w[o++] = (float)(sd * nd(rng));
    for (int i = 0; i < nout; ++i) w[o++] = 0.f;
  };
  layer(kMlpHidden, kMlpIn, 1.);
  layer(kMlpHidden, kMlpHidden, 1.);
  layer(kMlpOut, kMlpHidden, 0.1);
}

double gravity_dt(const pdf_handle* h) {
  const double* g = h->prm.gravity;
  double gn = std::sqrt((g[0] * g[0] + g[1] * g[1]) + g[2] * g[2]);
  if (!(gn > 1e-12)) gn = 1e-12;
  return gn * h->prm.time_step;
}

void create_impl(pdf_handle* h, const pdf_scene_desc* sc, const pdf_params* p) {
  auto t0 = std::chrono::steady_clock::now();
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw std::domain_error("no CUDA device");
  if (p->device < 0 || p->device >= ndev) throw std::invalid_argument("device ordinal out of range");
  CK(cudaSetDevice(p->device));
  h->prm = *p;
  h->fp32 = p->precision == PDF_FP32_REFINE;
  if (p->precision != PDF_FP64 && p->precision != PDF_FP32_REFINE) throw std::invalid_argument("unknown precision mode");
  const auto tl = std::chrono::steady_clock::now();
  build_model(*sc, *p, h->model);
  h->lhs_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tl).count();
  const Model& m = h->model;
  std::string ferr;
  if (!factorize(m, p->time_step, 40, h->fac, ferr)) throw std::range_error(ferr);
  const Factor& f = h->fac;
  const int N = m.N;
  CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  for (auto& e : h->ev) CK(cudaEventCreate(&e));
  DeviceBuffers& d = h->d;
  d.mass = upload(m.mass);
  d.ring_ptr = upload(m.ring_ptr);
  d.ring_idx = upload(m.ring_idx);
  d.ring_kappa = upload(m.ring_kappa);
  d.ring_bend = upload(m.ring_bend);
  d.bend_of = upload(m.bend_of);
  d.self_bend = upload(m.self_bend);
  d.bend_ptr = upload(m.bend_ptr);
  d.bend_idx = upload(m.bend_idx);
  d.bend_coef = upload(m.bend_coef);
  d.bend_w = upload(m.bend_w);
  d.bend_rest = upload(m.bend_rest);
  d.pin_term = m.has_pins ? upload(m.pin_term) : nullptr;
  d.spring_k = upload(m.spring_k);
  d.pin_w = m.has_pins ? upload(m.pin_w) : nullptr;
  d.ata_ptr = upload(m.ata_ptr);
  d.ata_col = upload(m.ata_col);
  d.ata_val = upload(m.ata_val);
  d.perm = upload(f.perm);
  d.iperm = upload(f.iperm);
  std::vector<int> vmat(N);
  for (int i = 0; i < N; ++i) vmat[i] = m.meshes[m.vmesh[i]].material;
  d.vmat = upload(vmat);
  d.friction = upload(m.friction);
  d.tris = upload(m.tris);
  DModel& dm = h->dm;
  dm.N = N;
  dm.B = (int)m.bend_w.size();
  dm.mass = d.mass;
  dm.ring_ptr = d.ring_ptr;
  dm.ring_idx = d.ring_idx;
  dm.ring_kappa = d.ring_kappa;
  dm.ring_bend = d.ring_bend;
  dm.bend_of = d.bend_of;
  dm.self_bend = d.self_bend;
  dm.bend_ptr = d.bend_ptr;
  dm.bend_idx = d.bend_idx;
  dm.bend_coef = d.bend_coef;
  dm.bend_w = d.bend_w;
  dm.bend_rest = d.bend_rest;
  dm.pin_term = d.pin_term;
  dm.spring_k = d.spring_k;
  dm.pin_w = d.pin_w;
  dm.ata_ptr = d.ata_ptr;
  dm.ata_col = d.ata_col;
  dm.ata_val = d.ata_val;
  dm.perm = d.perm;
  dm.iperm = d.iperm;
  // obstacles
  h->obs.n = (int)m.obstacles.size();
  h->host_obs.assign(h->obs.n, DObstacle{});
  h->moving.assign(h->obs.n, MovingClock{});
  for (int k = 0; k < h->obs.n; ++k) {
    const pdf_obstacle& o = m.obstacles[k];
    DObstacle& ob = h->host_obs[k];
    ob.type = o.type;
    ob.material = o.material;
    ob.mesh = o.mesh;
    if (o.mesh >= (int)m.meshes.size()) throw std::invalid_argument("obstacle mesh out of range");
    for (int c = 0; c < 3; ++c) {
      ob.c[c] = o.center[c];
      ob.p[c] = o.point[c];
      ob.s[c] = o.size[c];
    }
    ob.R = o.radius;
    // RotatingSphere ctor (RotatingSphere.cpp:29-37): omega * axis.normalized()
    double ax = o.axis[0], ay = o.axis[1], az = o.axis[2];
    double an2 = ax * ax + ay * ay + az * az;
    if (an2 > 0) {
      double an = std::sqrt(an2);
      ax /= an;
      ay /= an;
      az /= an;
    }
    ob.rot[0] = o.angular_speed * ax;
    ob.rot[1] = o.angular_speed * ay;
    ob.rot[2] = o.angular_speed * az;
    // StaticPlane ctor normalises the normal (StaticPlane.cpp:46-53)
    double nx = o.normal[0], ny = o.normal[1], nz = o.normal[2];
    double nn2 = nx * nx + ny * ny + nz * nz;
    if (nn2 > 0) {
      double nn = std::sqrt(nn2);
      nx /= nn;
      ny /= nn;
      nz /= nn;
    }
    ob.n[0] = nx;
    ob.n[1] = ny;
    ob.n[2] = nz;
    // StaticMesh keeps tol^2 and passes sqrt(tol^2) (StaticMesh.cpp:25-31)
    ob.tol = std::sqrt(o.threshold * o.threshold);
    if (o.type == PDF_OBSTACLE_MESH || o.type == PDF_OBSTACLE_MOVING_MESH) {
      d.obstacle_v.push_back(upload(m.obstacle_vertices[k]));
      d.obstacle_t.push_back(upload(m.obstacle_triangles[k]));
      ob.mv = d.obstacle_v.back();
      ob.mt = d.obstacle_t.back();
      ob.n_tri = (int)m.obstacle_triangles[k].size() / 3;
    }
    if (o.type == PDF_OBSTACLE_MOVING_MESH) {
      // every key frame resident; the current mesh starts as key frame 0
      MovingClock& mc = h->moving[k];
      mc.n_frames = o.n_frames;
      mc.n_vertices = o.n_vertices;
      mc.interval = o.frame_interval;
      mc.frames = ob.mv;
      mc.cur = dalloc<double>(3 * (size_t)o.n_vertices);
      d.obstacle_v.push_back(mc.cur);
      CK(cudaMemcpy(mc.cur, mc.frames, 3 * (size_t)o.n_vertices * sizeof(double), cudaMemcpyDeviceToDevice));
      ob.mv = mc.cur;
    }
    h->host_time_before_start.push_back(o.rotation_start_time);
  }
  d.obstacles = dalloc<DObstacle>(std::max(1, h->obs.n));
  d.vmesh = upload(m.vmesh);
  h->obs.o = d.obstacles;
  h->obs.vmesh = d.vmesh;
  d.ob_best = dalloc<int>(std::max<size_t>(1, (size_t)h->obs.n * N));
  h->obs.best = d.ob_best;
  // mesh obstacles: LBVH over their triangles (a moving mesh's over its
  // current mesh, refit every step)
  h->mesh_bvh.assign(h->obs.n, nullptr);
  h->bvh_since.assign(h->obs.n, 1);
  for (int k = 0; k < h->obs.n; ++k) {
    DObstacle& ob = h->host_obs[k];
    if (ob.type != PDF_OBSTACLE_MESH && ob.type != PDF_OBSTACLE_MOVING_MESH) continue;
    const int nvo = (int)(ob.type == PDF_OBSTACLE_MOVING_MESH ? h->moving[k].n_vertices
                                                              : m.obstacle_vertices[k].size() / 3);
    h->mesh_bvh[k] = mesh_bvh_create(nvo, ob.n_tri);
    mesh_bvh_build(h->mesh_bvh[k], ob.mv, ob.mt, h->stream);
    ob.bvh = mesh_bvh_nodes(h->mesh_bvh[k]);
  }
  CK(cudaStreamSynchronize(h->stream));
  // state
  d.q = upload(m.q0);
  d.v = upload(m.v0);
  d.tn = dalloc<double>(3 * (size_t)N);
  h->dm.tn = d.tn;
  d.qk = upload(m.q0);
  d.cstep = dalloc<double>(3 * (size_t)N);
  d.bp = dalloc<double>(3 * (size_t)std::max(1, dm.B));
  // solve
  build_schedule(h, kChunk, kCutLevel);
  if (h->fp32) {
    d.Wf32 = upload(std::vector<float>(f.Wf.begin(), f.Wf.end()));
    d.Wb32 = upload(std::vector<float>(f.Wb.begin(), f.Wb.end()));
    d.b32 = dalloc<float>(3 * (size_t)N);
    d.y32 = dalloc<float>(3 * (size_t)N);
    d.x32 = dalloc<float>(3 * (size_t)N);
    launch_solve_prep<float>(h->stream, N, d.x32, d.y32, d.sync);
  } else {
    d.Wf64 = upload(f.Wf);
    d.Wb64 = upload(f.Wb);
    d.b64 = dalloc<double>(3 * (size_t)N);
    d.y64 = dalloc<double>(3 * (size_t)N);
    d.x64 = dalloc<double>(3 * (size_t)N);
    launch_solve_prep<double>(h->stream, N, d.x64, d.y64, d.sync);
  }
  // contacts
  // at most one contact per (obstacle, vertex of the meshes it acts on)
  int64_t cap_auto = 0;
  for (const DObstacle& ob : h->host_obs) cap_auto += ob.mesh >= 0 ? m.meshes[ob.mesh].n_vertices : N;
  cap_auto = std::max<int64_t>(1, cap_auto);
  if (cap_auto > (int64_t)INT32_MAX) throw std::overflow_error("contact capacity above 2^31");
  h->cap_contacts = p->contact_capacity > 0 ? p->contact_capacity : (int)cap_auto;
  h->cap_self = p->contact_capacity > 0 ? p->contact_capacity : 2 * N;
  DContacts& c = d.c;
  c.cap = h->cap_contacts;
  c.slot_cap = N;
  c.self_cap = h->cap_self;
  if (p->trace_alart_curnier) {
    c.trace_stride = c.cap + c.self_cap;
    c.trace_k = std::max(1, p->local_global_iterations);
    c.ac_trace = dalloc<double>(2 * (size_t)c.trace_stride * c.trace_k);
  }
  c.n_contacts = dalloc<int>(1);
  c.n_self = dalloc<int>(1);
  c.n_levels = dalloc<int>(1);
  c.n_slots = dalloc<int>(1);
  CK(cudaMemset(c.n_contacts, 0, sizeof(int)));
  CK(cudaMemset(c.n_self, 0, sizeof(int)));
  CK(cudaMemset(c.n_levels, 0, sizeof(int)));
  CK(cudaMemset(c.n_slots, 0, sizeof(int)));
  const size_t cc = h->cap_contacts, cs = h->cap_self;
  c.c_vertex = dalloc<int>(cc);
  c.c_normal = dalloc<double>(3 * cc);
  c.c_speed = dalloc<double>(3 * cc);
  c.c_mu = dalloc<double>(cc);
  c.c_basis = dalloc<double>(9 * cc);
  c.c_force = dalloc<double>(3 * cc);
  CK(cudaMemset(c.c_force, 0, 3 * cc * sizeof(double)));
  c.c_ac = dalloc<double>(cc);
  c.c_slot = dalloc<int>(cc);
  c.c_gap = dalloc<double>(cc);
  c.c_active = dalloc<int>(cc);
  CK(cudaMemset(c.c_active, 0, cc * sizeof(int)));
  c.s_vertex = dalloc<int>(cs);
  c.s_partner = dalloc<int>(cs);
  c.s_face = dalloc<int>(3 * cs);
  c.s_normal = dalloc<double>(3 * cs);
  c.s_mu = dalloc<double>(cs);
  c.s_basis = dalloc<double>(9 * cs);
  c.s_force = dalloc<double>(3 * cs);
  CK(cudaMemset(c.s_force, 0, 3 * cs * sizeof(double)));
  c.s_ac = dalloc<double>(cs);
  c.s_slota = dalloc<int>(cs);
  c.s_slotb = dalloc<int>(cs);
  c.s_remember = dalloc<double>(3 * cs);
  c.level_ptr = dalloc<int>(cs + 2);
  c.level_order = dalloc<int>(cs);
  c.slot_of = dalloc<int>(N);
  CK(cudaMemset(c.slot_of, 0xff, N * sizeof(int)));
  c.slot_vertex = dalloc<int>(N);
  c.f = dalloc<double>(3 * (size_t)N);
  for (int k = 0; k < 2; ++k) {
    c.cf[k] = dalloc<double>(3 * (size_t)N);
    c.sf[k] = dalloc<double>(3 * (size_t)N);
    CK(cudaMemset(c.cf[k], 0, 3 * (size_t)N * sizeof(double)));
    CK(cudaMemset(c.sf[k], 0, 3 * (size_t)N * sizeof(double)));
  }
  d.newf = dalloc<double>(3 * cs);
  d.ac_hist = dalloc<double>(4 * (size_t)std::max(1, p->local_global_iterations));
  d.iter = dalloc<int>(1);
  d.iter_total = dalloc<long long>(1);
  d.blocks_done = dalloc<unsigned int>(1);
  CK(cudaMemset(d.iter, 0, sizeof(int)));
  CK(cudaMemset(d.iter_total, 0, sizeof(long long)));
  CK(cudaMemset(d.blocks_done, 0, sizeof(unsigned int)));
  // iteration clock and the step records that carry it to the host
  {
    const int K = std::max(1, p->local_global_iterations);
    const size_t nst = (size_t)DTrace::kRows * K;
    d.stamps = dalloc<unsigned long long>(nst);
    CK(cudaMemset(d.stamps, 0, nst * sizeof(unsigned long long)));
    h->dm.trace = DTrace{d.iter, d.stamps, K};
    h->d.sync.trace = h->dm.trace;
    const size_t per = 64 + nst * sizeof(unsigned long long);  // counts padded to 64 bytes
    h->ring.resize(kRecords);
    CK(cudaHostAlloc(&h->ring_host, per * kRecords, cudaHostAllocMapped));
    std::memset(h->ring_host, 0, per * kRecords);
    for (int r = 0; r < kRecords; ++r) {
      StepRecord& rec = h->ring[r];
      char* base = static_cast<char*>(h->ring_host) + per * r;
      rec.counts = reinterpret_cast<int*>(base);
      rec.stamps = reinterpret_cast<unsigned long long*>(base + 64);
      CK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&rec.counts_dev), rec.counts, 0));
      CK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&rec.stamps_dev), rec.stamps, 0));
      for (auto& e : rec.ev) CK(cudaEventCreate(&e));
    }
  }
  if (h->obs.n > 0) {
    const int nitems = h->obs.n * N;
    d.flags = dalloc<unsigned char>(nitems);
    d.sel_idx = dalloc<int>(nitems);
    thrust::counting_iterator<int> it(0);
    CK(cub::DeviceSelect::Flagged(nullptr, d.cub_tmp_bytes, it, d.flags, d.sel_idx, c.n_contacts, nitems,
                                  h->stream));
    d.cub_tmp = dalloc<char>(d.cub_tmp_bytes);
  }
  if (p->self_collision) {
    int st = self_detect_init(h);
    if (st != PDF_OK) throw CudaFail("self-collision workspace: " + h->err);
  }
  // learned warm start
  if (p->warm_start != PDF_WARM_NONE && p->warm_start != PDF_WARM_MLP) throw std::invalid_argument("unknown warm start");
  h->mlp_w = dalloc<float>(kMlpParams);
  if (p->warm_start == PDF_WARM_MLP) {
    ensure_mlp_buffers(h);
    const size_t len = strnlen(p->mlp_weights, sizeof(p->mlp_weights));
    if (len == sizeof(p->mlp_weights)) throw std::invalid_argument("mlp_weights path is not terminated");
    if (len > 0) {
      std::vector<float> w(kMlpParams);
      load_weights_file(std::string(p->mlp_weights, len), w.data());
      CK(cudaMemcpy(h->mlp_w, w.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
      h->mlp_ready = true;
    }
  }
  CK(cudaDeviceSynchronize());
  autotune_schedule(h);
  // the timing solves overwrote v and q^k: restore the initial state
  CK(cudaMemcpy(d.v, m.v0.data(), m.v0.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.qk, m.q0.data(), m.q0.size() * sizeof(double), cudaMemcpyHostToDevice));
  h->stats.factor_ms = f.factor_ms;
  h->stats.factor_nnz = f.nnz_w;
  h->stats.factor_nnz_true = f.nnz_l_true;
  h->stats.n_supernodes = f.n_sn;
  h->stats.n_levels = f.n_levels;
  h->stats.lhs_nnz = (int64_t)m.ata_col.size();
  h->stats.n_constraint_rows = m.n_rows;
  h->stats.setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Local step: bending projections + vertex right-hand side (or residual).
template <typename T>
void launch_local(pdf_handle* h, T* b, int mode) {
  DeviceBuffers& d = h->d;
  const DModel& dm = h->dm;
  cudaStream_t st = h->stream;
  if (dm.B > 0) k_bend_proj<<<blocks_for(dm.B), kThreads, 0, st>>>(dm, d.qk, d.bp, mode);
  launch_vertex_rhs<T>(blocks_for(dm.N), kThreads, st, dm, d.qk, d.v, d.cstep, d.bp,
                       std::max(h->prm.air_damping, 0.), d.c.slot_of, d.c.f, b, h->prm.time_step, mode);
}

// Global solve: one persistent forward and one backward sweep (which writes
// back v and q^k of the blocks' columns), then the write-back of the upper
// columns (which also clears their x, y for the next solve).
template <typename T>
void launch_solve(pdf_handle* h, T* b, T* y, T* x, const T* Wf, const T* Wb, int mode) {
  DeviceBuffers& d = h->d;
  launch_solve_sweeps<T>(h->stream, d.plan, Wf, Wb, b, y, x, h->dm.N, d.sync,
                         WriteBack{d.v, d.qk, d.q, h->prm.time_step, mode});
}

template <typename T>
void launch_solve_with(pdf_handle* h, const SweepSync& sy, T* b, T* y, T* x, const T* Wf, const T* Wb, int mode) {
  DeviceBuffers& d = h->d;
  launch_solve_sweeps<T>(h->stream, d.plan, Wf, Wb, b, y, x, h->dm.N, sy,
                         WriteBack{d.v, d.qk, d.q, h->prm.time_step, mode});
}

// Schedule autotuner: times the global solve of this scene's factor with
// each candidate cut level and both upper modes (work-item width 64, block
// kernels at 2 CTAs of 8 or 4 CTAs of 4 consumer warps per SM where they
// fit), then with each launch shape of the block kernels at the best cut
// level and mode, then with each work-item width, and keeps the fastest.  The right-hand side is
// zero (the sweeps read the same data and wait on the same dependencies
// whatever the values); v and q^k, which the solve writes, are restored.
void autotune_schedule(pdf_handle* h) {
  DeviceBuffers& d = h->d;
  const int N = h->dm.N;
  cudaStream_t st = h->stream;
  std::vector<double> vsave(3 * (size_t)N), qsave(3 * (size_t)N);
  CK(cudaMemcpy(vsave.data(), d.v, vsave.size() * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(qsave.data(), d.qk, qsave.size() * sizeof(double), cudaMemcpyDeviceToHost));
  // 0 when the schedule built is not the one asked for (upper levels beyond
  // the launch table, or a block shape that does not fit)
  auto time_plan = [&](int chunk, int cut, int mode, int shape, bool exact_shape) {
    build_schedule(h, chunk, cut, mode, shape);
    if (h->d.plan.upper_mode != mode || (exact_shape && h->d.plan.block_shape != shape)) return 0.;
    double total = 0.;
    for (int r = 0; r < 4; ++r) {
      if (h->fp32) {
        CK(cudaMemsetAsync(d.b32, 0, 3 * (size_t)N * sizeof(float), st));
        launch_solve_prep<float>(st, N, d.x32, d.y32, d.sync);
      } else {
        CK(cudaMemsetAsync(d.b64, 0, 3 * (size_t)N * sizeof(double), st));
        launch_solve_prep<double>(st, N, d.x64, d.y64, d.sync);
      }
      CK(cudaEventRecord(h->ev[5], st));
      if (h->fp32)
        launch_solve<float>(h, d.b32, d.y32, d.x32, d.Wf32, d.Wb32, 1);
      else
        launch_solve<double>(h, d.b64, d.y64, d.x64, d.Wf64, d.Wb64, 0);
      CK(cudaEventRecord(h->ev[6], st));
      CK(cudaEventSynchronize(h->ev[6]));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, h->ev[5], h->ev[6]));
      if (r > 0) total += ms;  // first run warms up
    }
    int derr = 0;
    CK(cudaMemcpy(&derr, d.sync.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (derr) throw CudaFail("a supernodal sweep gave up waiting for a dependency while tuning");
    return total / 3.;
  };
  double best = 1e300;
  int best_cut = kCutLevel, best_chunk = kChunk, best_mode = 0, best_shape = kBlockShape;
  double cut_ms[2][kCutCandidates] = {};
  int cut_shape[2][kCutCandidates] = {};
  for (int cut = 0; cut < kCutCandidates; ++cut)
    for (int mode = 0; mode < 2; ++mode)
      for (int sh : kStageOneShapes) {
        const double ms = time_plan(kChunk, cut, mode, sh, true);
        if (ms > 0. && (cut_ms[mode][cut] == 0. || ms < cut_ms[mode][cut])) {
          cut_ms[mode][cut] = ms;
          cut_shape[mode][cut] = sh;
        }
        if (ms > 0. && ms < best) {
          best = ms;
          best_cut = cut;
          best_mode = mode;
        }
      }
  if (best == 1e300) {  // neither first-stage shape fits any cut: one CTA of 8 warps
    for (int cut = 0; cut < kCutCandidates; ++cut)
      for (int mode = 0; mode < 2; ++mode) {
        const double ms = time_plan(kChunk, cut, mode, 0, false);
        cut_ms[mode][cut] = ms;
        cut_shape[mode][cut] = h->d.plan.block_shape;
        if (ms > 0. && ms < best) {
          best = ms;
          best_cut = cut;
          best_mode = mode;
        }
      }
  }
  for (int cut = 0; cut < kCutCandidates; ++cut) {
    h->stats.sweep_cut_ms[cut] = cut_ms[0][cut];
    h->stats.sweep_cut_level_ms[cut] = cut_ms[1][cut];
  }
  // the block kernels' launch shapes at the best cut level and mode
  best_shape = cut_shape[best_mode][best_cut];
  for (int sh = 0; sh < kBlockShapes; ++sh) {
    const double ms = sh == best_shape ? best : time_plan(kChunk, best_cut, best_mode, sh, true);
    h->stats.sweep_shape_ms[sh] = ms;
    if (ms > 0. && ms < best) {
      best = ms;
      best_shape = sh;
    }
  }
  const double best_default_chunk = best;
  for (int ci = 0; ci < 3; ++ci) {
    const int chunk = kChunkCandidates[ci];
    const double ms =
        chunk == kChunk ? best_default_chunk : time_plan(chunk, best_cut, best_mode, best_shape, true);
    h->stats.sweep_chunk_ms[ci] = ms;
    if (ms > 0. && ms < best) {
      best = ms;
      best_chunk = chunk;
    }
  }
  build_schedule(h, best_chunk, best_cut, best_mode, best_shape);
  if (h->fp32)
    launch_solve_prep<float>(st, N, d.x32, d.y32, d.sync);
  else
    launch_solve_prep<double>(st, N, d.x64, d.y64, d.sync);
  CK(cudaMemcpy(d.v, vsave.data(), vsave.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.qk, qsave.data(), qsave.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaStreamSynchronize(st));
}

// One PD iteration (SimulationBase.cpp:119-157): local step + friction
// (SFE::computeRhs), global solve (SimulationSpeed::solve), AC residual.
// The iteration index comes from the device counter d.iter (advanced by the
// AC kernel), so the same launches serve fixed and iterate-to-tolerance runs.
template <typename T>
void launch_iteration(pdf_handle* h, T* b, T* y, T* x, const T* Wf, const T* Wb, int mode) {
  DeviceBuffers& d = h->d;
  const DModel& dm = h->dm;
  cudaStream_t st = h->stream;
  const int self_mode = h->prm.self_collision ? 1 : 0;
  launch_local<T>(h, b, mode);
  // learned warm start: the first iteration of the step takes the predicted forces
  const bool warm = h->prm.warm_start == PDF_WARM_MLP;
  launch_friction_obstacle<T>(kStrideBlocks, kThreads, st, dm, d.c, b, self_mode, d.iter, warm ? h->mlp_Y : nullptr,
                              warm ? gravity_dt(h) : 0.);
  if (self_mode) launch_friction_self<T>(1, 1024, st, dm, d.c, b, d.newf, d.iter);
  launch_solve<T>(h, b, y, x, Wf, Wb, mode);
  IterCtl ctl{d.iter, d.iter_total, d.blocks_done, h->prm.residual_tolerance, h->prm.local_global_iterations,
              h->capturing_cond ? 1 : 0, h->cond, h->dm.trace};
  k_alart_curnier<<<kStrideBlocks, kThreads, 0, st>>>(d.c, d.v, d.ac_hist, ctl);
}

// Kernels of this library launched by one PD iteration (CUB's not counted):
// [bending], vertex rhs, friction, [self friction], forward, backward, post, AC.
int64_t launches_per_iteration(const pdf_handle* h) {
  return 6 + (h->dm.B > 0 ? 1 : 0) + (h->prm.self_collision ? 1 : 0);
}

// Per step outside the iterations: predictor, obstacle flags + clamp + materialise,
// slots (2), slot reset, finalize; self-collision: register reset, per mesh
// bbox/keys/build/refit/traverse/filter/compact/pair, bases, levels.
int64_t launches_per_step_extra(const pdf_handle* h) {
  int64_t n = 1 + (h->obs.n > 0 ? 3 : 0) + 2 + 1 + 1;
  if (h->prm.self_collision) n += 1 + 8 * (int64_t)h->model.meshes.size() + 1 + 1;
  // warm start: features, forward; record (clear + accumulate [+ count])
  const bool warm = h->prm.warm_start == PDF_WARM_MLP;
  if (warm || h->log_cap > 0) n += 1 + 2 + (h->log_cap > 0 ? 1 : 0) + (warm ? 1 : 0);
  return n;
}

void launch_iterations(pdf_handle* h, int count) {
  DeviceBuffers& d = h->d;
  for (int k = 0; k < count; ++k) {
    if (h->fp32)
      launch_iteration<float>(h, d.b32, d.y32, d.x32, d.Wf32, d.Wb32, 1);
    else
      launch_iteration<double>(h, d.b64, d.y64, d.x64, d.Wf64, d.Wb64, 0);
  }
}

// Iterate-to-tolerance graph: one conditional WHILE node whose body is one PD
// iteration; the AC kernel's last block decides whether the body runs again.
void build_tolerance_graph(pdf_handle* h) {
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  CK(cudaGraphConditionalHandleCreate(&h->cond, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h->cond;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  h->capturing_cond = true;
  CK(cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  launch_iterations(h, 1);
  cudaGraph_t captured;
  const cudaError_t e = cudaStreamEndCapture(h->stream, &captured);
  h->capturing_cond = false;
  CK(e);
  CK(cudaGraphInstantiate(&h->graph, g, 0));
  CK(cudaGraphDestroy(g));
}

// Reads one finished step record into the per-sample statistics and the
// cumulative phase times (the reference's timers: SimulationBase.cpp:103-173,
// 333-405; SFE:135-151, 307-426, 430-572).
void harvest_record(pdf_handle* h, StepRecord& rec) {
  CK(cudaEventSynchronize(rec.ev[6]));
  float e[7] = {0.f};
  for (int k = 1; k < 7; ++k) CK(cudaEventElapsedTime(&e[k], rec.ev[0], rec.ev[k]));
  const bool self = h->prm.self_collision != 0;
  const int C = rec.counts[0], S = rec.counts[1], iters = rec.counts[3];
  const int K = std::max(1, h->prm.local_global_iterations);
  StatSamples& sm = h->samples;
  pdf_stats& st = h->stats;
  sm.detection.push_back(1e3 * e[1]);
  st.detection_ms += e[1];
  if (C > 0) sm.collisions.push_back(C);
  if (self) {
    sm.self_detection.push_back(1e3 * (e[2] - e[1]));
    st.self_detection_ms += e[2] - e[1];
    if (S > 0) {
      sm.self_collisions.push_back(S);
      sm.ordering.push_back(1e3 * (e[3] - e[2]));
      st.ordering_ms += e[3] - e[2];
    }
  }
  st.solve_ms += e[5] - e[4];
  st.step_ms += e[6];
  sm.step.push_back(1e3 * e[6]);
  const unsigned long long* t = rec.stamps;
  auto us = [](unsigned long long a, unsigned long long b) { return b >= a ? 1e-3 * (double)(b - a) : 0.; };
  for (int k = 0; k < std::min(iters, K); ++k) {
    const unsigned long long t0 = t[DTrace::kLocal * K + k], tf = t[DTrace::kFriction * K + k],
                             ts = t[DTrace::kSelfFriction * K + k], tv = t[DTrace::kSolve * K + k],
                             ta = t[DTrace::kAcBegin * K + k], te = t[DTrace::kAcEnd * K + k];
    sm.iteration.push_back(us(t0, te));
    sm.rhs.push_back(us(t0, tv));
    sm.solver.push_back(us(tv, ta));
    sm.rhs_base.push_back(us(t0, tf));
    st.rhs_ms += 1e-3 * us(t0, tf);
    if (C + S > 0) {
      sm.friction.push_back(us(tf, self ? ts : tv));
      st.friction_ms += 1e-3 * us(tf, self ? ts : tv);
    }
    if (self && S > 0) {
      sm.self_friction.push_back(us(ts, tv));
      st.self_friction_ms += 1e-3 * us(ts, tv);
    }
  }
  rec.pending = false;
}

// Harvests every pending record, oldest first.
void harvest_all(pdf_handle* h) {
  for (int k = 0; k < kRecords; ++k) {
    StepRecord& rec = h->ring[(h->ring_head + k) % kRecords];
    if (rec.pending) harvest_record(h, rec);
  }
}

void step_once(pdf_handle* h, bool want_report) {
  DeviceBuffers& d = h->d;
  const DModel& dm = h->dm;
  cudaStream_t st = h->stream;
  const double dt = h->prm.time_step;
  const int N = dm.N;
  const int K = h->prm.local_global_iterations;
  StepRecord& rec = h->ring[h->ring_head];
  if (rec.pending) harvest_record(h, rec);
  CK(cudaEventRecord(rec.ev[0], st));
  k_step_init<<<blocks_for(N), kThreads, 0, st>>>(dm, d.q, d.v, d.tn, d.qk, d.cstep, h->prm.gravity[0],
                                                  h->prm.gravity[1], h->prm.gravity[2], dt);
  // obstacle detection on the start-of-step positions (SimulationBase.cpp:333-366)
  if (h->obs.n > 0) {
    for (int k = 0; k < h->obs.n; ++k) {
      DObstacle& ob = h->host_obs[k];
      ob.time_before_start = h->host_time_before_start[k];
      const MovingClock& mc = h->moving[k];
      if (mc.n_frames > 0) {
        ob.fprev = mc.frames + 3 * (size_t)mc.n_vertices * (mc.next - 1);
        ob.fnext = mc.frames + 3 * (size_t)mc.n_vertices * mc.next;
        ob.frame_dt = mc.frame_time(mc.next) - mc.frame_time(mc.next - 1);
        ob.moving = mc.in_movement() ? 1 : 0;
      }
    }
    CK(cudaMemcpyAsync(d.obstacles, h->host_obs.data(), h->obs.n * sizeof(DObstacle), cudaMemcpyHostToDevice, st));
    k_obstacle_flags<<<blocks_for(N), kThreads, 0, st>>>(N, d.q, h->obs, d.flags);
    thrust::counting_iterator<int> it(0);
    CK(cub::DeviceSelect::Flagged(d.cub_tmp, d.cub_tmp_bytes, it, d.flags, d.sel_idx, d.c.n_contacts,
                                  h->obs.n * N, st));
    k_clamp_contacts<<<1, 1, 0, st>>>(d.c.n_contacts, d.c.cap, d.sync.err);
    k_obstacle_materialize<<<kStrideBlocks, kThreads, 0, st>>>(N, d.q, h->obs, d.sel_idx, d.vmat, d.friction,
                                                               h->model.n_materials, d.c);
  } else {
    CK(cudaMemsetAsync(d.c.n_contacts, 0, sizeof(int), st));
  }
  CK(cudaEventRecord(rec.ev[1], st));
  if (h->prm.self_collision) {
    int sst = self_detect_step(h);
    if (sst != PDF_OK) throw std::overflow_error(h->err);
  } else {
    CK(cudaMemsetAsync(d.c.n_self, 0, sizeof(int), st));
    CK(cudaMemsetAsync(d.c.n_levels, 0, sizeof(int), st));
  }
  CK(cudaEventRecord(rec.ev[2], st));
  // compact slots of every vertex touched by a contact (force buffers of SFE:45-60)
  k_contact_slots<<<kStrideBlocks, kThreads, 0, st>>>(d.c);
  k_contact_slots_fill<<<kStrideBlocks, kThreads, 0, st>>>(d.c);
  if (h->prm.self_collision) self_levels_step(h);
  CK(cudaEventRecord(rec.ev[3], st));
  // learned warm start: features of every obstacle contact, predicted forces
  const bool warm = h->prm.warm_start == PDF_WARM_MLP;
  const bool mlp_features = warm || h->log_cap > 0;
  if (mlp_features) {
    launch_mlp_features(st, d.c, d.tn, d.mass, h->rprev, h->rprev_tag, h->mlp_tag - 1, h->prm.gravity, dt, h->mlp_X);
    if (warm) mlp_forward_counted(h->mlp_w, h->mlp_X, d.c.n_contacts, h->cap_contacts, h->mlp_Y, st);
  }
  CK(cudaEventRecord(rec.ev[4], st));
  CK(cudaMemsetAsync(d.ac_hist, 0, 4 * (size_t)K * sizeof(double), st));
  CK(cudaMemsetAsync(d.iter, 0, sizeof(int), st));
  // iterations
  int iters = -1;  // -1: known on the device only
  if (h->prm.residual_tolerance > 0.) {
    // iterate to tolerance: stop after the first iteration whose mean
    // Alart-Curnier residual is at or below the tolerance (LocalGlobal caps it)
    if (h->prm.use_graph) {
      if (!h->graph) build_tolerance_graph(h);
      CK(cudaGraphLaunch(h->graph, st));
    } else {
      int counts[2];
      CK(cudaMemcpyAsync(&counts[0], d.c.n_contacts, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(&counts[1], d.c.n_self, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      const int nc = counts[0] + counts[1];
      iters = 0;
      while (iters < K) {
        launch_iterations(h, 1);
        ++iters;
        if (nc == 0) continue;
        double sum = 0.;
        CK(cudaMemcpyAsync(&sum, d.ac_hist + 4 * (size_t)(iters - 1), sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (sum / nc <= h->prm.residual_tolerance) break;
      }
    }
  } else if (h->prm.use_graph) {
    if (!h->graph) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      launch_iterations(h, K);
      CK(cudaStreamEndCapture(st, &g));
      CK(cudaGraphInstantiate(&h->graph, g, 0));
      CK(cudaGraphDestroy(g));
    }
    CK(cudaGraphLaunch(h->graph, st));
    iters = K;
  } else {
    launch_iterations(h, K);
    iters = K;
  }
  CK(cudaEventRecord(rec.ev[5], st));
  if (mlp_features) {
    const bool log = h->log_cap > 0;
    launch_mlp_record(st, d.c, d.mass, h->rprev, h->rprev_tag, h->mlp_tag, h->prm.gravity, dt, h->mlp_X,
                      log ? h->log_X : nullptr, h->log_T, h->log_n, h->log_cap);
  }
  h->mlp_tag += 1;
  k_contact_slots_reset<<<kStrideBlocks, kThreads, 0, st>>>(d.c);
  CK(cudaMemsetAsync(d.c.n_slots, 0, sizeof(int), st));
  // a frame copy of q still in flight must end before q is overwritten
  if (h->frame_guard >= 0) {
    CK(cudaStreamWaitEvent(st, h->frame_ev[h->frame_guard], 0));
    h->frame_guard = -1;
  }
  const StepOut out{d.c.n_contacts, d.c.n_self, d.c.n_levels, d.iter, d.stamps,
                    DTrace::kRows * std::max(1, K), rec.counts_dev, rec.stamps_dev};
  k_finalize<<<blocks_for(3 * (int64_t)N), kThreads, 0, st>>>(3 * N, d.qk, d.q, out);
  CK(cudaEventRecord(rec.ev[6], st));
  rec.pending = true;
  h->ring_head = (h->ring_head + 1) % kRecords;
  CK(cudaGetLastError());
  // RotatingSphere::update (RotatingSphere.cpp:39-43)
  for (auto& t : h->host_time_before_start) t -= dt;
  // MovingMesh::update (MovingMesh.cpp:43-84): advance the clock, at most one
  // key frame, then interpolate the current mesh while in movement
  for (MovingClock& mc : h->moving) {
    if (mc.n_frames == 0) continue;
    mc.clock += dt;
    if (mc.frame_time(mc.next) < mc.clock && mc.next + 1 < mc.n_frames) mc.next += 1;
    if (mc.in_movement()) {
      const double t0 = mc.frame_time(mc.next - 1), t1 = mc.frame_time(mc.next);
      const size_t nv3 = 3 * (size_t)mc.n_vertices;
      launch_moving_mesh_lerp(st, (int)nv3, mc.frames + nv3 * (mc.next - 1), mc.frames + nv3 * mc.next,
                              (mc.clock - t0) / (t1 - t0), mc.cur);
      h->launches_outside += 1;
      // its hierarchy follows: refit every step, rebuilt every 8
      const size_t k = &mc - h->moving.data();
      if (h->mesh_bvh[k]) {
        if (++h->bvh_since[k] > 8) {
          mesh_bvh_build(h->mesh_bvh[k], mc.cur, h->host_obs[k].mt, st);
          h->bvh_since[k] = 1;
          h->launches_outside += 4;
        } else {
          mesh_bvh_refit(h->mesh_bvh[k], mc.cur, h->host_obs[k].mt, st);
          h->launches_outside += 1;
        }
      }
    }
  }
  h->time += dt;
  h->stats.steps += 1;
  h->launches_outside += launches_per_step_extra(h);
  if (want_report) {
    CK(cudaStreamSynchronize(st));
    harvest_all(h);
    const int counts[3] = {rec.counts[0], rec.counts[1], rec.counts[2]};
    if (iters < 0) iters = rec.counts[3];
    std::vector<double> hist(4 * (size_t)K);
    CK(cudaMemcpy(hist.data(), d.ac_hist, hist.size() * sizeof(double), cudaMemcpyDeviceToHost));
    const int nc = counts[0] + counts[1];
    h->residual_hist.resize(iters);
    for (int k = 0; k < iters; ++k) h->residual_hist[k] = nc ? hist[4 * k] / nc : 0.;
    pdf_step_report& r = h->last;
    r.n_contacts = counts[0];
    r.n_self_contacts = counts[1];
    r.n_levels = counts[2];
    r.iterations = iters;
    const int kl = std::max(iters, 1) - 1;
    r.residual = nc ? hist[4 * kl] / nc : 0.;
    r.residual_max = hist[4 * kl + 1];
    r.normal_residual = nc ? hist[4 * kl + 2] / nc : 0.;
    r.tangential_residual = nc ? hist[4 * kl + 3] / nc : 0.;
    r.time = h->time;
  }
}

int fail(pdf_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  g_error = msg;
  return code;
}

template <typename F>
int guarded(pdf_handle* h, F&& fn) {
  try {
    return fn();
  } catch (const CudaFail& e) {
    return fail(h, PDF_CUDA_ERROR, e.what());
  } catch (const std::ios_base::failure& e) {
    return fail(h, PDF_IO_ERROR, e.what());
  } catch (const std::overflow_error& e) {
    return fail(h, PDF_CAPACITY_EXCEEDED, e.what());
  } catch (const std::range_error& e) {
    return fail(h, PDF_NOT_SPD, e.what());
  } catch (const std::domain_error& e) {
    return fail(h, PDF_NO_DEVICE, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(h, PDF_INVALID_ARG, e.what());
  } catch (const std::runtime_error& e) {
    return fail(h, PDF_CUDA_ERROR, e.what());
  } catch (const std::exception& e) {
    return fail(h, PDF_INVALID_ARG, e.what());
  }
}

void free_handle(pdf_handle* h) {
  if (!h) return;
  cudaSetDevice(h->prm.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  self_detect_free(h);
  DeviceBuffers& d = h->d;
  void* ptrs[] = {d.spring_k, d.pin_w, d.mass, d.ring_kappa, d.ring_bend, d.self_bend, d.ring_ptr, d.ring_idx, d.bend_of, d.bend_ptr,
                  d.bend_idx, d.bend_coef, d.bend_w, d.bend_rest, d.pin_term, d.ata_ptr, d.ata_col, d.ata_val,
                  d.perm, d.iperm, d.vmat, d.friction, d.tris, d.obstacles, d.vmesh, d.q, d.v, d.tn, d.qk,
                  d.cstep, d.bp, d.sn, d.rows, d.Wf64, d.Wb64, d.Wf32, d.Wb32, d.sync.queue, d.sync.epoch,
                  d.sync.fdone, d.sync.bdone, d.sync.err, d.b64, d.y64, d.x64, d.b32, d.y32,
                  d.x32, d.flags, d.sel_idx, d.cub_tmp, d.newf, d.ac_hist, d.c.n_contacts, d.c.c_vertex,
                  d.c.c_normal, d.c.c_speed, d.c.c_mu, d.c.c_basis, d.c.c_force, d.c.c_ac, d.c.c_slot, d.c.n_self,
                  d.c.s_vertex, d.c.s_partner, d.c.s_face, d.c.s_normal, d.c.s_mu, d.c.s_basis, d.c.s_force,
                  d.c.s_ac, d.c.s_slota, d.c.s_slotb, d.c.s_remember, d.c.n_levels, d.c.level_ptr,
                  d.c.level_order, d.c.slot_of, d.c.n_slots, d.c.slot_vertex, d.c.f, d.c.cf[0], d.c.cf[1],
                  d.c.sf[0], d.c.sf[1], d.c.c_gap, d.c.c_active, h->mlp_w, h->mlp_X, h->mlp_Y, h->rprev,
                  h->rprev_tag, h->log_X, h->log_T, h->log_n, d.iter, d.iter_total, d.blocks_done, d.stamps,
                  d.c.ac_trace, h->gather_idx, h->gather_out, h->stage, h->bad_dev, d.ob_best};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  free_plan(d.plan);
  for (auto p : d.obstacle_v) cudaFree(p);
  for (auto b : h->mesh_bvh) mesh_bvh_free(b);
  for (auto p : d.obstacle_t) cudaFree(p);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  for (StepRecord& rec : h->ring)
    for (auto& e : rec.ev)
      if (e) cudaEventDestroy(e);
  if (h->ring_host) cudaFreeHost(h->ring_host);
  if (h->bad_host) cudaFreeHost(h->bad_host);
  for (int k = 0; k < 2; ++k) {
    if (h->frame_host[k]) cudaFreeHost(h->frame_host[k]);
    if (h->frame_ev[k]) cudaEventDestroy(h->frame_ev[k]);
  }
  if (h->frame_ready) cudaEventDestroy(h->frame_ready);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

void fill_contact(pdf_contact& o, int vertex, int partner, const int* face, const double* n, const double* sp,
                  double mu, const double* f, double ac) {
  o.vertex = vertex;
  o.partner = partner;
  for (int k = 0; k < 3; ++k) {
    o.face[k] = face ? face[k] : -1;
    o.normal[k] = n[k];
    o.speed[k] = sp ? sp[k] : 0.;
    o.force[k] = f[k];
  }
  o.mu = mu;
  o.ac = ac;
}

}  // namespace

namespace pdfb {
void set_global_error(const std::string& msg) { g_error = msg; }
}  // namespace pdfb

extern "C" {

void pdf_params_default(pdf_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->time_step = 1e-3;
  p->local_global_iterations = 20;
  p->gravity[2] = -9.81;
  p->precision = PDF_FP64;
  p->refine_max = 4;
  p->refine_tolerance = 1e-10;
  p->use_graph = 1;
}

const char* pdf_global_error(void) { return g_error.c_str(); }
const char* pdf_last_error(const pdf_handle* h) { return h ? h->err.c_str() : g_error.c_str(); }

int pdf_create(const pdf_scene_desc* scene, const pdf_params* params, pdf_handle** out) {
  if (!out) return fail(nullptr, PDF_INVALID_ARG, "null output handle");
  *out = nullptr;
  if (!scene || !params) return fail(nullptr, PDF_INVALID_ARG, "null scene or parameters");
  pdf_handle* h = new pdf_handle();
  int st = guarded(h, [&] {
    create_impl(h, scene, params);
    return PDF_OK;
  });
  if (st != PDF_OK) {
    g_error = h->err;
    free_handle(h);
    return st;
  }
  *out = h;
  return PDF_OK;
}

int pdf_step(pdf_handle* h, int32_t nsteps, pdf_step_report* report) {
  if (!h || nsteps < 0) return fail(h, PDF_INVALID_ARG, "invalid handle or step count");
  if (h->prm.warm_start == PDF_WARM_MLP && !h->mlp_ready)
    return fail(h, PDF_INVALID_ARG, "PDF_WARM_MLP needs weights (mlp_weights, pdf_mlp_set_weights or pdf_mlp_train)");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaEventRecord(h->ev[5], h->stream));
    for (int s = 0; s < nsteps; ++s) step_once(h, s == nsteps - 1);
    CK(cudaEventRecord(h->ev[6], h->stream));
    CK(cudaStreamSynchronize(h->stream));
    harvest_all(h);
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev[5], h->ev[6]));
    h->last.device_ms = ms;
    if (report) *report = h->last;
    int derr = 0;
    CK(cudaMemcpy(&derr, h->d.sync.err, sizeof(int), cudaMemcpyDeviceToHost));
    // error word bits: 1 sweep wait gave up, 2 obstacle contacts, 4 self
    // contacts or partners, 8 self-collision hits, 16 BVH stack
    if (derr & 2) return fail(h, PDF_CAPACITY_EXCEEDED, "more obstacle contacts than contact_capacity");
    if (derr & 4)
      return fail(h, PDF_CAPACITY_EXCEEDED,
                  "more self contacts than the self-contact buffer, or a vertex with more than 16 partners");
    if (derr & 8)
      return fail(h, PDF_CAPACITY_EXCEEDED, "more than 32 self-collision candidates at a vertex, or hit buffer full");
    if (derr & 16) return fail(h, PDF_CAPACITY_EXCEEDED, "self-collision BVH deeper than the traversal stack");
    if (derr) return fail(h, PDF_DEVICE_TIMEOUT, "a supernodal sweep gave up waiting for a dependency");
    return PDF_OK;
  });
}

int pdf_time_phase(pdf_handle* h, int32_t phase, int32_t reps, double* ms_out, double* bytes_out) {
  if (!h || reps <= 0 || phase < 0 || phase > 3) return fail(h, PDF_INVALID_ARG, "invalid phase timing request");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    DeviceBuffers& d = h->d;
    const DModel& dm = h->dm;
    cudaStream_t st = h->stream;
    const Factor& f = h->fac;
    const double s = h->fp32 ? 4. : 8.;
    const double N = dm.N;
    double bytes = 0;
    int64_t idx_rows = (int64_t)f.rows.size();
    if (phase == 0) {
      // 2 [l s + idx_bytes(L)] + 2 (2 * 3 s N) + FP64 write-back (q read; v, q^k
      // written), with l = structural nnz(L) (padding and explicit zeros of the
      // stored tiles are not counted)
      bytes = 2. * ((double)f.nnz_l_true * s + 4. * (double)idx_rows) + 2. * (2. * 3. * s * N) + 72. * N;
    } else if (phase == 1) {
      // 4*3sN + E (8 + s) + sum_b [(r_b + 1)(4 + s) + s], s = 8 (FP64 local step)
      const double E = (double)h->model.ring_idx.size() / 2.;
      double bsum = 0;
      for (size_t b = 0; b + 1 < h->model.bend_ptr.size(); ++b)
        bsum += (h->model.bend_ptr[b + 1] - h->model.bend_ptr[b]) * 12. + 8.;
      bytes = 4. * 24. * N + E * 16. + bsum;
    } else if (phase == 3) {
      // obstacle tests: positions read, one flag byte per (obstacle, vertex);
      // self collision (when on): positions and triangles read (24 N + 12 T),
      // the 112-byte node records written by the refit and read once by the
      // traversal, and the triangle boxes (48 T) written and read
      const double T = (double)h->model.tris.size() / 3.;
      bytes = (double)h->obs.n * (24. * N + N);
      if (h->prm.self_collision) bytes += 24. * N + 12. * T + 2. * 112. * std::max(0., T - 1.) + 2. * 48. * T;
    }
    // phase 0 works on a saved right-hand side restored between repetitions
    double* save64 = nullptr;
    float* save32 = nullptr;
    if (phase == 0) {
      if (h->fp32) {
        save32 = dalloc<float>(3 * (size_t)dm.N);
        CK(cudaMemcpyAsync(save32, d.b32, 3 * (size_t)dm.N * sizeof(float), cudaMemcpyDeviceToDevice, st));
      } else {
        save64 = dalloc<double>(3 * (size_t)dm.N);
        CK(cudaMemcpyAsync(save64, d.b64, 3 * (size_t)dm.N * sizeof(double), cudaMemcpyDeviceToDevice, st));
      }
    }
    std::vector<double> vsave(3 * (size_t)dm.N), qsave(3 * (size_t)dm.N);
    CK(cudaMemcpyAsync(vsave.data(), d.v, vsave.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(qsave.data(), d.qk, qsave.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    double total = 0;
    for (int r = 0; r < reps; ++r) {
      if (phase == 0) {
        if (h->fp32)
          CK(cudaMemcpyAsync(d.b32, save32, 3 * (size_t)dm.N * sizeof(float), cudaMemcpyDeviceToDevice, st));
        else
          CK(cudaMemcpyAsync(d.b64, save64, 3 * (size_t)dm.N * sizeof(double), cudaMemcpyDeviceToDevice, st));
      }
      CK(cudaEventRecord(h->ev[5], st));
      if (phase == 0) {
        if (h->fp32)
          launch_solve<float>(h, d.b32, d.y32, d.x32, d.Wf32, d.Wb32, 1);
        else
          launch_solve<double>(h, d.b64, d.y64, d.x64, d.Wf64, d.Wb64, 0);
      } else if (phase == 1) {
        if (h->fp32)
          launch_local<float>(h, d.b32, 1);
        else
          launch_local<double>(h, d.b64, 0);
      } else if (phase == 2) {
        if (h->fp32)
          launch_friction_obstacle<float>(kStrideBlocks, kThreads, st, dm, d.c, d.b32, 0, d.iter);
        else
          launch_friction_obstacle<double>(kStrideBlocks, kThreads, st, dm, d.c, d.b64, 0, d.iter);
      } else {
        if (h->obs.n > 0) {
          k_obstacle_flags<<<blocks_for(dm.N), kThreads, 0, st>>>(dm.N, d.q, h->obs, d.flags);
          thrust::counting_iterator<int> it(0);
          CK(cub::DeviceSelect::Flagged(d.cub_tmp, d.cub_tmp_bytes, it, d.flags, d.sel_idx, d.c.n_contacts,
                                        h->obs.n * dm.N, st));
        }
        if (h->prm.self_collision) {
          int sst = self_detect_step(h);
          if (sst != PDF_OK) throw std::overflow_error(h->err);
        }
      }
      CK(cudaEventRecord(h->ev[6], st));
      CK(cudaEventSynchronize(h->ev[6]));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, h->ev[5], h->ev[6]));
      total += ms;
    }
    CK(cudaMemcpyAsync(d.v, vsave.data(), vsave.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d.qk, qsave.data(), qsave.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    if (save64) cudaFree(save64);
    if (save32) cudaFree(save32);
    if (ms_out) *ms_out = total / reps;
    if (bytes_out) *bytes_out = bytes;
    return PDF_OK;
  });
}

int pdf_get_state(pdf_handle* h, double* q, double* v) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    const size_t n = 3 * (size_t)h->dm.N * sizeof(double);
    // ordered after the enqueued steps on the handle's stream; pinned
    // destinations make these true asynchronous DMA copies
    if (q) CK(cudaMemcpyAsync(q, h->d.q, n, cudaMemcpyDeviceToHost, h->stream));
    if (v) CK(cudaMemcpyAsync(v, h->d.v, n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PDF_OK;
  });
}

// The state is uploaded to staging buffers and checked on the device; only a
// finite state replaces the handle's (a rejected one leaves it unchanged).
// Uploading the state the handle already holds (a caller feeding back what it
// read) changes nothing, so the warm start's memory of the last step's
// contact impulses is kept; any other state invalidates it.
int pdf_set_state(pdf_handle* h, const double* q, const double* v) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  if (!q && !v) return PDF_OK;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    cudaStream_t st = h->stream;
    const size_t n3 = 3 * (size_t)h->dm.N, bytes = n3 * sizeof(double);
    if (!h->stage) {
      h->stage = dalloc<double>(2 * n3);
      h->bad_dev = dalloc<int>(2);
      CK(cudaHostAlloc(reinterpret_cast<void**>(&h->bad_host), 2 * sizeof(int), cudaHostAllocDefault));
    }
    if (h->copy_stream) CK(cudaStreamSynchronize(h->copy_stream));
    CK(cudaMemsetAsync(h->bad_dev, 0, 2 * sizeof(int), st));
    if (q) {
      CK(cudaMemcpyAsync(h->stage, q, bytes, cudaMemcpyHostToDevice, st));
      k_check_state<<<kStrideBlocks, kThreads, 0, st>>>((int64_t)n3, h->stage, h->d.q, h->bad_dev);
      h->launches_outside += 1;
    }
    if (v) {
      CK(cudaMemcpyAsync(h->stage + n3, v, bytes, cudaMemcpyHostToDevice, st));
      k_check_state<<<kStrideBlocks, kThreads, 0, st>>>((int64_t)n3, h->stage + n3, h->d.v, h->bad_dev);
      h->launches_outside += 1;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->bad_host, h->bad_dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h->bad_host[0]) return fail(h, PDF_NAN_DETECTED, "non-finite value in the state passed to pdf_set_state");
    if (!h->bad_host[1]) return PDF_OK;  // the state the handle holds already
    if (q) CK(cudaMemcpyAsync(h->d.q, h->stage, bytes, cudaMemcpyDeviceToDevice, st));
    if (v) CK(cudaMemcpyAsync(h->d.v, h->stage + n3, bytes, cudaMemcpyDeviceToDevice, st));
    h->mlp_tag += 2;  // the previous step's contact impulses no longer apply
    return PDF_OK;
  });
}

int pdf_device_state(pdf_handle* h, double** q_dev, double** v_dev, void** stream) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  if (q_dev) *q_dev = h->d.q;
  if (v_dev) *v_dev = h->d.v;
  if (stream) *stream = (void*)h->stream;
  return PDF_OK;
}

int pdf_get_contacts(pdf_handle* h, pdf_contact* out, int32_t cap, int32_t* n) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  return guarded(h, [&]() -> int {
    CK(cudaStreamSynchronize(h->stream));
    int C = 0;
    CK(cudaMemcpy(&C, h->d.c.n_contacts, sizeof(int), cudaMemcpyDeviceToHost));
    if (n) *n = C;
    if (!out) return PDF_OK;
    const int m = std::min(C, cap);
    std::vector<int> vx(m);
    std::vector<double> nr(3 * m), sp(3 * m), mu(m), fo(3 * m), ac(m);
    const DContacts& c = h->d.c;
    if (m > 0) {
      CK(cudaMemcpy(vx.data(), c.c_vertex, m * sizeof(int), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(nr.data(), c.c_normal, 3 * m * sizeof(double), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(sp.data(), c.c_speed, 3 * m * sizeof(double), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(mu.data(), c.c_mu, m * sizeof(double), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(fo.data(), c.c_force, 3 * m * sizeof(double), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(ac.data(), c.c_ac, m * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (int k = 0; k < m; ++k)
      fill_contact(out[k], vx[k], -1, nullptr, &nr[3 * k], &sp[3 * k], mu[k], &fo[3 * k], ac[k]);
    return C > cap ? fail(h, PDF_CAPACITY_EXCEEDED, "contact buffer too small") : PDF_OK;
  });
}

int pdf_get_self_contacts(pdf_handle* h, pdf_contact* out, int32_t cap, int32_t* n) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  return guarded(h, [&]() -> int {
    CK(cudaStreamSynchronize(h->stream));
    int S = 0;
    CK(cudaMemcpy(&S, h->d.c.n_self, sizeof(int), cudaMemcpyDeviceToHost));
    if (n) *n = S;
    if (!out) return PDF_OK;
    const int m = std::min(S, cap);
    std::vector<int> vx(m), pa(m), fa(3 * m);
    std::vector<double> nr(3 * m), mu(m), fo(3 * m), ac(m);
    const DContacts& c = h->d.c;
    if (m > 0) {
      CK(cudaMemcpy(vx.data(), c.s_vertex, m * sizeof(int), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(pa.data(), c.s_partner, m * sizeof(int), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(fa.data(), c.s_face, 3 * m * sizeof(int), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(nr.data(), c.s_normal, 3 * m * sizeof(double), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(mu.data(), c.s_mu, m * sizeof(double), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(fo.data(), c.s_force, 3 * m * sizeof(double), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(ac.data(), c.s_ac, m * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (int k = 0; k < m; ++k)
      fill_contact(out[k], vx[k], pa[k], &fa[3 * k], &nr[3 * k], nullptr, mu[k], &fo[3 * k], ac[k]);
    return S > cap ? fail(h, PDF_CAPACITY_EXCEEDED, "self-contact buffer too small") : PDF_OK;
  });
}

int pdf_get_self_levels(pdf_handle* h, int32_t* level_ptr, int32_t level_cap, int32_t* order, int32_t order_cap,
                        int32_t* n_levels) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  return guarded(h, [&]() -> int {
    CK(cudaStreamSynchronize(h->stream));
    int nl = 0, S = 0;
    CK(cudaMemcpy(&nl, h->d.c.n_levels, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&S, h->d.c.n_self, sizeof(int), cudaMemcpyDeviceToHost));
    if (n_levels) *n_levels = nl;
    if (level_ptr && level_cap > 0)
      CK(cudaMemcpy(level_ptr, h->d.c.level_ptr, std::min(level_cap, nl + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    if (order && order_cap > 0 && S > 0)
      CK(cudaMemcpy(order, h->d.c.level_order, std::min(order_cap, S) * sizeof(int), cudaMemcpyDeviceToHost));
    return PDF_OK;
  });
}

int pdf_get_stats(pdf_handle* h, pdf_stats* out) {
  if (!h || !out) return fail(h, PDF_INVALID_ARG, "null argument");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaStreamSynchronize(h->stream));
    long long total = 0;
    CK(cudaMemcpy(&total, h->d.iter_total, sizeof(long long), cudaMemcpyDeviceToHost));
    h->stats.iterations = total;
    h->stats.kernel_launches = h->launches_outside + total * launches_per_iteration(h);
    *out = h->stats;
    return PDF_OK;
  });
}

}  // extern "C"

namespace {
// computeAndWriteStats (template/physics/io.tpp:23-63): a title line, then
// "(No data)", " Value : x" for one sample, or the number, minimum, mean and
// maximum of the samples (default stream formatting), then a dashed separator.
// Counts are integers: their mean is truncated like the reference's
// conversion of the double mean to the element type.
template <typename T>
void write_stats_section(std::ostream& of, const char* name, const std::vector<T>& v) {
  of << name << std::endl;
  if (v.empty()) {
    of << "\t(No data)" << std::endl;
  } else if (v.size() == 1) {
    of << "\t Value : " << v[0] << std::endl;
  } else {
    double mn = std::numeric_limits<double>::max(), mx = std::numeric_limits<double>::min(), sum = 0.;
    for (const T& x : v) {
      mn = std::min(mn, (double)x);
      mx = std::max(mx, (double)x);
      sum += (double)x;
    }
    of << "\t Number      : " << v.size() << std::endl
       << "\t Min value   : " << (T)mn << std::endl
       << "\t Mean value  : " << (T)(sum / (double)v.size()) << std::endl
       << "\t Max value   : " << (T)mx << std::endl;
  }
  of << std::endl << "-------------------" << std::endl << std::endl;
}
}  // namespace

extern "C" {

// The stats file's text (SimulationFrictionEstimation::exportStats SFE:756-771
// around SimulationBase::exportStats SimulationBase.cpp:474-494).
void write_stats(pdf_handle* h, std::ostream& of) {
  CK(cudaSetDevice(h->prm.device));
  CK(cudaStreamSynchronize(h->stream));
  harvest_all(h);
  const StatSamples& sm = h->samples;
  const bool self = h->prm.self_collision != 0;
  write_stats_section(of, "LHS computation time (µs)", std::vector<double>{1e3 * h->lhs_ms});
  write_stats_section(of, "Cholesky computation time (µs)", std::vector<double>{1e3 * h->stats.factor_ms});
  write_stats_section(of, "Iteration time (µs)", sm.iteration);
  write_stats_section(of, "Collision detection time (µs)", sm.detection);
  if (self) {
    write_stats_section(of, "Number of collisions", sm.collisions);
    write_stats_section(of, "Self collision detection time (µs)", sm.self_detection);
  }
  write_stats_section(of, "Number of self collisions", sm.self_collisions);
  write_stats_section(of, "Solver time (µs)", sm.solver);
  write_stats_section(of, "Full RHS computation time (µs)", sm.rhs);
  write_stats_section(of, "Step time (µs)", sm.step);
  write_stats_section(of, "RHS base computation time (µs)", sm.rhs_base);
  write_stats_section(of, "RHS friction overhead (µs)", sm.friction);
  if (self) {
    write_stats_section(of, "Self collision time (µs)", sm.self_friction);
    write_stats_section(of, "Self collision ordering time (µs)", sm.ordering);
  }
}

int pdf_export_stats(pdf_handle* h, const char* path) {
  if (!h || !path) return fail(h, PDF_INVALID_ARG, "null argument");
  std::ofstream of(path);
  if (!of) return fail(h, PDF_IO_ERROR, std::string("cannot open ") + path);
  return guarded(h, [&]() -> int {
    write_stats(h, of);
    if (!of) return fail(h, PDF_IO_ERROR, std::string("cannot write ") + path);
    return PDF_OK;
  });
}

int pdf_export_stats_text(pdf_handle* h, char* buf, int64_t cap, int64_t* len) {
  if (!h || !len || (cap > 0 && !buf)) return fail(h, PDF_INVALID_ARG, "null argument");
  return guarded(h, [&]() -> int {
    std::ostringstream os;
    write_stats(h, os);
    const std::string t = os.str();
    *len = (int64_t)t.size();
    if (cap > 0) {
      const int64_t n = std::min<int64_t>(cap - 1, (int64_t)t.size());
      std::memcpy(buf, t.data(), (size_t)n);
      buf[n] = '\0';
    }
    return PDF_OK;
  });
}

int pdf_frame_capture(pdf_handle* h, int32_t slot) {
  if (!h || slot < 0 || slot > 1) return fail(h, PDF_INVALID_ARG, "invalid handle or frame slot");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    const size_t bytes = 3 * (size_t)h->dm.N * sizeof(double);
    if (!h->copy_stream) {
      CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&h->frame_ready, cudaEventDisableTiming));
      for (int k = 0; k < 2; ++k) {
        CK(cudaHostAlloc(reinterpret_cast<void**>(&h->frame_host[k]), bytes, cudaHostAllocDefault));
        CK(cudaEventCreateWithFlags(&h->frame_ev[k], cudaEventDisableTiming));
      }
    }
    // the slot's previous copy has been waited for by the caller or is
    // ordered before this one on the copy stream
    CK(cudaEventRecord(h->frame_ready, h->stream));
    CK(cudaStreamWaitEvent(h->copy_stream, h->frame_ready, 0));
    CK(cudaMemcpyAsync(h->frame_host[slot], h->d.q, bytes, cudaMemcpyDeviceToHost, h->copy_stream));
    CK(cudaEventRecord(h->frame_ev[slot], h->copy_stream));
    h->frame_guard = slot;
    return PDF_OK;
  });
}

int pdf_frame_wait(pdf_handle* h, int32_t slot, const double** q) {
  if (!h || slot < 0 || slot > 1 || !q) return fail(h, PDF_INVALID_ARG, "invalid handle, frame slot or output");
  if (!h->frame_host[slot]) return fail(h, PDF_INVALID_ARG, "frame slot never captured");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaEventSynchronize(h->frame_ev[slot]));
    *q = h->frame_host[slot];
    return PDF_OK;
  });
}

int pdf_get_vertices(pdf_handle* h, const int32_t* vertices, int32_t n, double* q, double* v) {
  if (!h || n < 0 || (n > 0 && !vertices)) return fail(h, PDF_INVALID_ARG, "invalid vertex list");
  for (int k = 0; k < n; ++k)
    if (vertices[k] < 0 || vertices[k] >= h->dm.N) return fail(h, PDF_INVALID_ARG, "vertex index out of range");
  if (n == 0) return PDF_OK;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    cudaStream_t st = h->stream;
    if (n > h->gather_cap) {
      if (h->gather_idx) CK(cudaFree(h->gather_idx));
      if (h->gather_out) CK(cudaFree(h->gather_out));
      h->gather_idx = nullptr;
      h->gather_out = nullptr;
      h->gather_idx = dalloc<int>(n);
      h->gather_out = dalloc<double>(6 * (size_t)n);
      h->gather_cap = n;
    }
    CK(cudaMemcpyAsync(h->gather_idx, vertices, n * sizeof(int), cudaMemcpyHostToDevice, st));
    k_gather_vertices<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(n, h->gather_idx, h->d.q, h->d.v,
                                                                          h->gather_out);
    CK(cudaGetLastError());
    h->launches_outside += 1;
    std::vector<double> out(6 * (size_t)n);
    CK(cudaMemcpyAsync(out.data(), h->gather_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (q) std::copy(out.begin(), out.begin() + 3 * (size_t)n, q);
    if (v) std::copy(out.begin() + 3 * (size_t)n, out.end(), v);
    return PDF_OK;
  });
}

int pdf_get_alart_curnier_trace(pdf_handle* h, double* out, int64_t cap, int32_t* iterations, int32_t* n_contacts,
                                int32_t* n_self) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  if (!h->d.c.ac_trace) return fail(h, PDF_INVALID_ARG, "created without trace_alart_curnier");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaStreamSynchronize(h->stream));
    int counts[3];
    CK(cudaMemcpy(&counts[0], h->d.c.n_contacts, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&counts[1], h->d.c.n_self, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&counts[2], h->d.iter, sizeof(int), cudaMemcpyDeviceToHost));
    const int C = std::min(counts[0], h->d.c.cap), S = std::min(counts[1], h->d.c.self_cap);
    const int it = std::min(counts[2], h->d.c.trace_k);
    if (iterations) *iterations = it;
    if (n_contacts) *n_contacts = C;
    if (n_self) *n_self = S;
    const int64_t need = 2 * (int64_t)it * (C + S);
    if (!out) return PDF_OK;
    if (cap < need) return fail(h, PDF_CAPACITY_EXCEEDED, "trace buffer too small");
    if (need == 0) return PDF_OK;
    const size_t row = 2 * sizeof(double) * (size_t)(C + S);
    CK(cudaMemcpy2D(out, row, h->d.c.ac_trace, 2 * sizeof(double) * (size_t)h->d.c.trace_stride, row, it,
                    cudaMemcpyDeviceToHost));
    return PDF_OK;
  });
}

int pdf_get_residual_history(pdf_handle* h, double* out, int32_t cap, int32_t* n) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  if (n) *n = (int)h->residual_hist.size();
  if (out)
    for (int i = 0; i < (int)h->residual_hist.size() && i < cap; ++i) out[i] = h->residual_hist[i];
  return PDF_OK;
}

void pdf_destroy(pdf_handle* h) { free_handle(h); }

int pdf_time_solve_parts(pdf_handle* h, int32_t reps, double* part_ms) {
  if (!h || reps <= 0 || !part_ms) return fail(h, PDF_INVALID_ARG, "invalid solve timing request");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    DeviceBuffers& d = h->d;
    const int N = h->dm.N;
    cudaStream_t st = h->stream;
    std::vector<double> vsave(3 * (size_t)N), qsave(3 * (size_t)N);
    CK(cudaMemcpy(vsave.data(), d.v, vsave.size() * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(qsave.data(), d.qk, qsave.size() * sizeof(double), cudaMemcpyDeviceToHost));
    const size_t bbytes = 3 * (size_t)N * (h->fp32 ? sizeof(float) : sizeof(double));
    void* bsave = nullptr;
    CK(cudaMalloc(&bsave, bbytes));
    void* bcur = h->fp32 ? (void*)d.b32 : (void*)d.b64;
    CK(cudaMemcpyAsync(bsave, bcur, bbytes, cudaMemcpyDeviceToDevice, st));
    cudaEvent_t ev[6];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    double acc[5] = {0, 0, 0, 0, 0};
    for (int r = 0; r < reps; ++r) {
      CK(cudaMemcpyAsync(bcur, bsave, bbytes, cudaMemcpyDeviceToDevice, st));
      CK(cudaEventRecord(ev[0], st));
      WriteBack wb{d.v, d.qk, d.q, h->prm.time_step, h->fp32 ? 1 : 0};
      if (h->fp32)
        launch_solve_sweeps<float>(st, d.plan, d.Wf32, d.Wb32, d.b32, d.y32, d.x32, N, d.sync, wb, ev + 1);
      else
        launch_solve_sweeps<double>(st, d.plan, d.Wf64, d.Wb64, d.b64, d.y64, d.x64, N, d.sync, wb, ev + 1);
      CK(cudaEventRecord(ev[5], st));
      CK(cudaEventSynchronize(ev[5]));
      for (int k = 0; k < 5; ++k) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
        acc[k] += ms;
      }
    }
    for (int k = 0; k < 5; ++k) part_ms[k] = acc[k] / reps;
    for (auto& e : ev) cudaEventDestroy(e);
    CK(cudaMemcpyAsync(bcur, bsave, bbytes, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpy(d.v, vsave.data(), vsave.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.qk, qsave.data(), qsave.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(st));
    cudaFree(bsave);
    return PDF_OK;
  });
}

int pdf_set_sweep_schedule(pdf_handle* h, int32_t chunk, int32_t cut_level, int32_t upper_mode,
                           int32_t block_shape) {
  if (!h) return fail(h, PDF_INVALID_ARG, "null handle");
  if (std::find(std::begin(kChunkCandidates), std::end(kChunkCandidates), chunk) == std::end(kChunkCandidates) ||
      cut_level < 0 || cut_level >= kCutCandidates || (upper_mode != 0 && upper_mode != 1) || block_shape < 0 ||
      block_shape >= kBlockShapes)
    return fail(h, PDF_INVALID_ARG,
                "sweep schedule outside chunk {32, 64, 128}, cut level 0-7, mode 0/1, block shape 0-4");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaStreamSynchronize(h->stream));
    build_schedule(h, chunk, cut_level, upper_mode, block_shape);
    const bool mode_ok = h->d.plan.upper_mode == upper_mode && h->d.plan.block_shape == block_shape;
    if (!mode_ok) build_schedule(h, chunk, cut_level, 0, 0);
    DeviceBuffers& d = h->d;
    if (h->fp32)
      launch_solve_prep<float>(h->stream, h->dm.N, d.x32, d.y32, d.sync);
    else
      launch_solve_prep<double>(h->stream, h->dm.N, d.x64, d.y64, d.sync);
    // a captured iteration graph holds the old schedule's launch parameters
    if (h->graph) {
      CK(cudaGraphExecDestroy(h->graph));
      h->graph = nullptr;
    }
    CK(cudaStreamSynchronize(h->stream));
    if (!mode_ok)
      return fail(h, PDF_INVALID_ARG,
                  "the scene has more upper levels than the level launch table holds, or its blocks do not fit "
                  "the launch shape");
    return PDF_OK;
  });
}

int pdf_check_wait_timeout(pdf_handle* h, int32_t max_spins) {
  if (!h || max_spins <= 0) return fail(h, PDF_INVALID_ARG, "invalid wait-timeout check");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    DeviceBuffers& d = h->d;
    const int N = h->dm.N;
    cudaStream_t st = h->stream;
    build_schedule(h, h->stats.sweep_chunk > 0 ? h->stats.sweep_chunk : kChunk, 0);
    if (d.plan.nfup == 0) return fail(h, PDF_INVALID_ARG, "the scene's sweep schedule has no dependency wait");
    // targets one solve ahead: the counters stop one solve short of them
    const unsigned long long ahead = 2ULL;
    CK(cudaMemcpy(d.sync.epoch, &ahead, sizeof(ahead), cudaMemcpyHostToDevice));
    SweepSync sy = d.sync;
    sy.max_spins = max_spins;
    if (h->fp32) {
      launch_solve_prep<float>(st, N, d.x32, d.y32, sy);
      launch_solve_with<float>(h, sy, d.b32, d.y32, d.x32, d.Wf32, d.Wb32, 1);
    } else {
      launch_solve_prep<double>(st, N, d.x64, d.y64, sy);
      launch_solve_with<double>(h, sy, d.b64, d.y64, d.x64, d.Wf64, d.Wb64, 0);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    int derr = 0;
    CK(cudaMemcpy(&derr, d.sync.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!(derr & 1)) return fail(h, PDF_INVALID_ARG, "no dependency wait gave up");
    return fail(h, PDF_DEVICE_TIMEOUT, "a supernodal sweep gave up waiting for a dependency (wait-timeout check)");
  });
}

int pdf_factor_check(const pdf_scene_desc* scene, const pdf_params* params, const double* b, double* x) {
  if (!scene || !params || !b || !x) return fail(nullptr, PDF_INVALID_ARG, "null argument");
  try {
    Model m;
    build_model(*scene, *params, m);
    Factor f;
    std::string err;
    if (!factorize(m, params->time_step, 40, f, err)) return fail(nullptr, PDF_NOT_SPD, err);
    std::vector<double> bv(b, b + 3 * (size_t)m.N), xv;
    // every schedule the autotuner can choose: cut levels 0 .. 7, chunks
    // 32 / 64 / 128; all must solve the system alike
    std::vector<double> x0;
    double scale = 0.;
    for (int cut = 0; cut < kCutCandidates; ++cut)
      for (int chunk : kChunkCandidates) {
        SweepPlan plan;
        build_sweep_plan(f, chunk, cut, plan);
        if (!emulate_sweeps(f, plan, bv, xv, err)) return fail(nullptr, PDF_INVALID_ARG, err);
        if (x0.empty()) {
          x0 = xv;
          for (double t : x0) scale = std::max(scale, std::fabs(t));
          continue;
        }
        for (size_t k = 0; k < xv.size(); ++k)
          if (!(std::fabs(xv[k] - x0[k]) <= 1e-10 * scale))
            return fail(nullptr, PDF_INVALID_ARG,
                        "sweep schedules disagree (cut level " + std::to_string(cut) + ", chunk " +
                            std::to_string(chunk) + ")");
      }
    xv = x0;
    std::copy(xv.begin(), xv.end(), x);
  } catch (const std::exception& e) {
    return fail(nullptr, PDF_INVALID_ARG, e.what());
  }
  return PDF_OK;
}

int pdf_detect_candidates(const double* positions, int32_t n_vertices, const int32_t* triangles, int32_t n_triangles,
                          double tolerance, int32_t* pairs, int32_t cap, int32_t* n, int32_t device) {
  std::string err;
  int st = PDF_OK;
  try {
    st = standalone_candidates(positions, n_vertices, triangles, n_triangles, tolerance, pairs, cap, n, device, err);
  } catch (const std::overflow_error& e) {
    err = e.what();
    st = PDF_CAPACITY_EXCEEDED;
  } catch (const std::exception& e) {
    err = e.what();
    st = PDF_CUDA_ERROR;
  }
  if (st != PDF_OK) g_error = err;
  return st;
}

int pdf_detect_self_collisions(const double* positions, int32_t n_vertices, const int32_t* triangles,
                               int32_t n_triangles, double tolerance, pdf_contact* out, int32_t cap, int32_t* n,
                               int32_t device) {
  std::string err;
  int st = PDF_OK;
  try {
    st = standalone_self(positions, n_vertices, triangles, n_triangles, tolerance, out, cap, n, device, err);
  } catch (const std::overflow_error& e) {
    err = e.what();
    st = PDF_CAPACITY_EXCEEDED;
  } catch (const std::exception& e) {
    err = e.what();
    st = PDF_CUDA_ERROR;
  }
  if (st != PDF_OK) g_error = err;
  return st;
}

// ---- learned warm start ----------------------------------------------------

int32_t pdf_mlp_param_count(void) { return kMlpParams; }

int pdf_mlp_init(float* weights, uint64_t seed) {
  if (!weights) return fail(nullptr, PDF_INVALID_ARG, "null weights");
  mlp_init_host(weights, seed);
  return PDF_OK;
}

int pdf_mlp_save(const char* path, const float* weights) {
  if (!path || !weights) return fail(nullptr, PDF_INVALID_ARG, "null path or weights");
  std::ofstream out(path, std::ios::binary);
  if (!out) return fail(nullptr, PDF_IO_ERROR, std::string("cannot write ") + path);
  const int32_t hdr[4] = {kMlpIn, kMlpHidden, kMlpOut, kMlpParams};
  out.write(kMlpMagic, 8);
  out.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
  out.write(reinterpret_cast<const char*>(weights), kMlpParams * sizeof(float));
  if (!out) return fail(nullptr, PDF_IO_ERROR, std::string("write failed: ") + path);
  return PDF_OK;
}

int pdf_mlp_load(const char* path, float* weights) {
  if (!path || !weights) return fail(nullptr, PDF_INVALID_ARG, "null path or weights");
  return guarded(nullptr, [&]() -> int {
    load_weights_file(path, weights);
    return PDF_OK;
  });
}

}  // extern "C"

namespace {
void select_device(int32_t device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw std::domain_error("no CUDA device");
  if (device < 0 || device >= ndev) throw std::invalid_argument("device ordinal out of range");
  CK(cudaSetDevice(device));
}
template <typename T>
struct HostToDevice {  // device copy of a host array, freed on scope exit
  T* p = nullptr;
  HostToDevice(const T* src, size_t n) {
    p = dalloc<T>(n);
    if (src && n) CK(cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice));
  }
  ~HostToDevice() { cudaFree(p); }
};
}  // namespace

extern "C" {

int pdf_mlp_forward(const float* weights, const float* X, int32_t n, float* Y, int32_t device) {
  if (!weights || n < 0 || (n > 0 && (!X || !Y))) return fail(nullptr, PDF_INVALID_ARG, "invalid MLP forward arguments");
  return guarded(nullptr, [&]() -> int {
    select_device(device);
    if (n == 0) return PDF_OK;
    HostToDevice<float> w(weights, kMlpParams), x(X, (size_t)n * kMlpIn), y(nullptr, (size_t)n * kMlpOut);
    mlp_forward_device(w.p, x.p, n, y.p, 0);
    CK(cudaGetLastError());
    CK(cudaMemcpy(Y, y.p, (size_t)n * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost));
    return PDF_OK;
  });
}

int pdf_mlp_gradient(const float* weights, const float* X, const float* T, int32_t n, float* grad, double* loss,
                     int32_t device) {
  if (!weights || !X || !T || !grad || n <= 0) return fail(nullptr, PDF_INVALID_ARG, "invalid MLP gradient arguments");
  return guarded(nullptr, [&]() -> int {
    select_device(device);
    HostToDevice<float> w(weights, kMlpParams), x(X, (size_t)n * kMlpIn), t(T, (size_t)n * kMlpOut),
        g(nullptr, kMlpParams);
    HostToDevice<double> l(nullptr, 1);
    CK(cudaMemset(g.p, 0, kMlpParams * sizeof(float)));
    CK(cudaMemset(l.p, 0, sizeof(double)));
    mlp_grad_device(w.p, x.p, t.p, nullptr, n, g.p, l.p, 0);
    CK(cudaGetLastError());
    CK(cudaMemcpy(grad, g.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
    double lv = 0.;
    CK(cudaMemcpy(&lv, l.p, sizeof(double), cudaMemcpyDeviceToHost));
    if (loss) *loss = lv;
    return PDF_OK;
  });
}

int pdf_mlp_fit(float* weights, const float* X, const float* T, int32_t n, int32_t epochs, int32_t batch,
                double learning_rate, uint64_t seed, int32_t device, double* train_loss, double* val_loss) {
  if (!weights || !X || !T || n < 2 || epochs <= 0 || batch <= 0 || !(learning_rate > 0.))
    return fail(nullptr, PDF_INVALID_ARG, "invalid MLP training arguments");
  return guarded(nullptr, [&]() -> int {
    select_device(device);
    HostToDevice<float> w(weights, kMlpParams), x(X, (size_t)n * kMlpIn), t(T, (size_t)n * kMlpOut);
    double vl = 0.;
    const double tl = mlp_train_device(w.p, x.p, t.p, n, epochs, batch, learning_rate, seed, &vl, 0);
    CK(cudaMemcpy(weights, w.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
    if (train_loss) *train_loss = tl;
    if (val_loss) *val_loss = vl;
    return PDF_OK;
  });
}

int pdf_mlp_set_weights(pdf_handle* h, const float* weights, int32_t count) {
  if (!h || !weights || count != kMlpParams) return fail(h, PDF_INVALID_ARG, "invalid MLP weights");
  for (int i = 0; i < kMlpParams; ++i)
    if (!std::isfinite(weights[i])) return fail(h, PDF_NAN_DETECTED, "non-finite MLP weight");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(h->mlp_w, weights, kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
    h->mlp_ready = true;
    return PDF_OK;
  });
}

int pdf_mlp_get_weights(pdf_handle* h, float* weights, int32_t count) {
  if (!h || !weights || count != kMlpParams) return fail(h, PDF_INVALID_ARG, "invalid MLP weights buffer");
  if (!h->mlp_ready) return fail(h, PDF_INVALID_ARG, "no MLP weights set");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(weights, h->mlp_w, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
    return PDF_OK;
  });
}

int pdf_mlp_log(pdf_handle* h, int32_t capacity) {
  if (!h || capacity < 0) return fail(h, PDF_INVALID_ARG, "invalid sample log capacity");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaStreamSynchronize(h->stream));
    if (h->log_cap > 0) {  // a running log is freed and restarted empty
      cudaFree(h->log_X);
      cudaFree(h->log_T);
      cudaFree(h->log_n);
      h->log_X = h->log_T = nullptr;
      h->log_n = nullptr;
      h->log_cap = 0;
    }
    if (capacity == 0) return PDF_OK;
    ensure_mlp_buffers(h);
    h->log_X = dalloc<float>((size_t)capacity * kMlpIn);
    h->log_T = dalloc<float>((size_t)capacity * kMlpOut);
    h->log_n = dalloc<int>(1);
    CK(cudaMemset(h->log_n, 0, sizeof(int)));
    h->log_cap = capacity;
    return PDF_OK;
  });
}

int pdf_mlp_samples(pdf_handle* h, float* X, float* T, int32_t cap, int32_t* n) {
  if (!h || !n || cap < 0) return fail(h, PDF_INVALID_ARG, "invalid sample read-back arguments");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaStreamSynchronize(h->stream));
    int cnt = 0;
    if (h->log_cap > 0) CK(cudaMemcpy(&cnt, h->log_n, sizeof(int), cudaMemcpyDeviceToHost));
    *n = cnt;
    const size_t m = std::min(cnt, cap);
    if (X && m) CK(cudaMemcpy(X, h->log_X, m * kMlpIn * sizeof(float), cudaMemcpyDeviceToHost));
    if (T && m) CK(cudaMemcpy(T, h->log_T, m * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost));
    if ((X || T) && cnt > cap) return fail(h, PDF_CAPACITY_EXCEEDED, "sample buffer too small");
    return PDF_OK;
  });
}

int pdf_mlp_train(pdf_handle* h, int32_t epochs, int32_t batch, double learning_rate, uint64_t seed,
                  double* train_loss, double* val_loss) {
  if (!h || epochs <= 0 || batch <= 0 || !(learning_rate > 0.))
    return fail(h, PDF_INVALID_ARG, "invalid MLP training arguments");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->prm.device));
    CK(cudaStreamSynchronize(h->stream));
    int cnt = 0;
    if (h->log_cap > 0) CK(cudaMemcpy(&cnt, h->log_n, sizeof(int), cudaMemcpyDeviceToHost));
    if (cnt < 2) return fail(h, PDF_INVALID_ARG, "fewer than 2 logged samples (pdf_mlp_log, then step)");
    double vl = 0.;
    const double tl = mlp_train_standardized(h->mlp_w, h->log_X, h->log_T, cnt, epochs, batch, learning_rate, seed,
                                             &vl, h->stream);
    h->mlp_ready = true;
    if (train_loss) *train_loss = tl;
    if (val_loss) *val_loss = vl;
    return PDF_OK;
  });
}

}  // extern "C"
