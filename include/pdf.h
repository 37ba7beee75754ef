/*
 * pdf.h — C ABI of the B200 projective-dynamics frictional-contact step loop.
 *
 * This is the drop-in boundary for the reference's step loop
 * ("Projective Dynamics with Dry Frictional Contact", SIGGRAPH 2020 code).
 * Every entry point takes plain pointers and sizes and returns an int status
 * (0 = PDF_OK).  The reference interfaces that each entry point replaces are
 * cited beside it (paths are relative to the reference project root).
 *
 * Ownership: host arrays passed in are copied during the call; the handle owns
 * all device memory, one CUDA stream and (optionally) a captured CUDA graph.
 * Threading: a handle is not thread-safe; drive one handle from one host
 * thread, exactly like the reference's single-threaded main loop
 * (src/main.cpp:86-114).
 */
#ifndef PDF_B200_H
#define PDF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum pdf_status {
  PDF_OK = 0,
  PDF_INVALID_ARG = 1,       /* bad argument or malformed scene / JSON / OBJ */
  PDF_CUDA_ERROR = 2,        /* a CUDA runtime call failed                  */
  PDF_NOT_SPD = 3,           /* the global-step matrix is not positive definite */
  PDF_CAPACITY_EXCEEDED = 4, /* a contact / candidate buffer would overflow  */
  PDF_DEVICE_TIMEOUT = 5,    /* a bounded device-side wait ran out           */
  PDF_NAN_DETECTED = 6,      /* non-finite value in inputs or state          */
  PDF_IO_ERROR = 7,          /* file could not be opened / read              */
  PDF_NO_DEVICE = 8          /* no usable CUDA device                        */
};

/* ---- obstacles (include/physics/Obstacle.hpp:64-95) -------------------- */
enum pdf_obstacle_type {
  PDF_OBSTACLE_SPHERE = 0,          /* StaticSphere   (src/physics/StaticSphere.cpp:35-47)   */
  PDF_OBSTACLE_ROTATING_SPHERE = 1, /* RotatingSphere (src/physics/RotatingSphere.cpp:71-93) */
  PDF_OBSTACLE_PLANE = 2,           /* StaticPlane    (src/physics/StaticPlane.cpp:57-73)    */
  PDF_OBSTACLE_MESH = 3,            /* StaticMesh     (src/physics/StaticMesh.cpp:33-56)     */
  PDF_OBSTACLE_BOX = 4,             /* StaticAxisAlignedBox
                                       (src/physics/StaticAxisAlignedBox.cpp:41-201) */
  PDF_OBSTACLE_MOVING_MESH = 5      /* MovingMesh     (src/physics/MovingMesh.cpp:28-264) */
};

typedef struct pdf_obstacle {
  int32_t type;                 /* pdf_obstacle_type                         */
  int32_t material;             /* row/column of the friction table          */
  double center[3];             /* spheres: centre ("Position")               */
  double radius;                /* spheres: radius                            */
  double axis[3];               /* rotating sphere: "Rotation Axe"            */
  double angular_speed;         /* rotating sphere: "Radial Speed" (rad/s)    */
  double rotation_start_time;   /* rotating sphere: "Rotation Start Time" (s) */
  double point[3];              /* plane: "Point"                             */
  double normal[3];             /* plane: "Normal"                            */
  int32_t n_vertices;           /* mesh obstacle: vertex count (of one key
                                   frame for a moving mesh)                   */
  int32_t n_triangles;          /* mesh obstacle: triangle count              */
  const double* vertices;       /* mesh obstacle: 3*n_vertices doubles; moving
                                   mesh: n_frames key frames one after the
                                   other, 3*n_vertices*n_frames doubles       */
  const int32_t* triangles;     /* mesh obstacle: 3*n_triangles indices       */
  double threshold;             /* mesh obstacle: "Threshold"; moving mesh:
                                   "Collision tolerance"                      */
  int32_t mesh;                 /* -1: acts on every dynamic mesh (the
                                   reference's behaviour); >= 0: only on that
                                   mesh (batches of independent cloths)       */
  double size[3];               /* box: "Size"; its "Position" (the corner
                                   with the smallest coordinates) is center  */
  int32_t n_frames;             /* moving mesh: "Number Frame" (>= 2)         */
  double frame_interval;        /* moving mesh: "Time Between Frame" (s); key
                                   frame f is reached at time f*interval      */
} pdf_obstacle;

/* ---- dynamic meshes (include/physics/PhysicMesh.hpp, PhysicParameters) -- */
typedef struct pdf_mesh_desc {
  int32_t vertex_offset;        /* first vertex of this mesh in the scene arrays */
  int32_t n_vertices;
  int32_t triangle_offset;      /* first triangle of this mesh                   */
  int32_t n_triangles;          /* triangle indices are scene-global             */
  double area_density;          /* "Area Density"  (kg/m^2)                      */
  double bending;               /* "Bending"       (weight of the bending rows)  */
  double stretching;            /* "Stretching"    (weight of the spring rows)   */
  int32_t material;             /* "Material Identifier"                         */
} pdf_mesh_desc;

/* ---- scene (PhysicScene, include/physics/PhysicScene.hpp:38-324) ------- */
typedef struct pdf_scene_desc {
  int32_t n_vertices;
  const double* rest_positions; /* 3N: rest state ("Obj filename")             */
  const double* positions;      /* 3N: initial state, NULL = rest state         */
  const double* velocities;     /* 3N: initial velocities, NULL = zero          */
  int32_t n_triangles;
  const int32_t* triangles;     /* 3T, scene-global vertex indices, CCW         */
  int32_t n_meshes;
  const pdf_mesh_desc* meshes;
  /* Attachment constraints (src/physics/AttachmentConstraint.cpp:31-51).
   * The reference has the constraint but no JSON key for it; the JSON reader
   * here accepts the extension key "Attachments". */
  int32_t n_pins;
  const int32_t* pin_vertices;
  const double* pin_positions;  /* 3*n_pins */
  const double* pin_weights;    /* n_pins   */
  int32_t n_obstacles;
  const pdf_obstacle* obstacles;
  int32_t n_materials;
  const double* friction;       /* n_materials^2, row-major ("Friction coefficients") */
} pdf_scene_desc;

/* ---- parameters (SimulationParameters, include/simulation_building.hpp:34-45) */
enum pdf_precision {
  PDF_FP64 = 0,          /* plain FP64 local step and triangular solves        */
  PDF_FP32_REFINE = 1    /* FP32 local step / solves + FP64-residual refinement */
};
enum pdf_warm_start {
  PDF_WARM_NONE = 0,     /* cold start: v^0 = t_n (SimulationSpeed.cpp:62-76)  */
  PDF_WARM_MLP = 1       /* learned per-contact warm start of the contact force */
};

typedef struct pdf_params {
  double time_step;                 /* "Timestep"                               */
  int32_t local_global_iterations;  /* "LocalGlobal" (cap when tolerance > 0)   */
  int32_t self_collision;           /* "Self-collision"                         */
  double self_collision_tolerance;  /* "Self-collision tolerance"               */
  double gravity[3];                /* "Gravity"                                */
  double air_damping;               /* "Air damping" (optional, default 0)      */
  int32_t precision;                /* pdf_precision                             */
  double residual_tolerance;        /* > 0: stop PD iterations once the mean
                                       Alart-Curnier residual is below it       */
  int32_t warm_start;               /* pdf_warm_start                            */
  int32_t refine_max;               /* FP32 mode: max refinement sweeps / solve */
  double refine_tolerance;          /* FP32 mode: relative FP64 residual target */
  int32_t device;                   /* CUDA device ordinal                       */
  int32_t contact_capacity;         /* 0 = automatic                             */
  int32_t use_graph;                /* capture the iteration loop in a CUDA graph */
  char mlp_weights[256];            /* PDF_WARM_MLP: weights file loaded at create
                                       ("" = set later with pdf_mlp_set_weights
                                       or pdf_mlp_train)                        */
  int32_t trace_alart_curnier;      /* 1: record every iteration's per-contact
                                       Alart-Curnier norms for
                                       pdf_get_alart_curnier_trace (the
                                       reference's PRINT_ALART_CURNIER_ERROR
                                       build option, SFE:720-752)              */
} pdf_params;

/* Fills p with the reference defaults (air damping 0, FP64, fixed iterations). */
void pdf_params_default(pdf_params* p);

/* ---- per-step report --------------------------------------------------- */
typedef struct pdf_step_report {
  int32_t n_contacts;               /* obstacle contacts of the last step       */
  int32_t n_self_contacts;          /* self contacts of the last step           */
  int32_t n_levels;                 /* self-contact Gauss-Seidel levels         */
  int32_t iterations;               /* PD iterations run in the last step       */
  double residual;                  /* mean AC norm after the last iteration    */
  double residual_max;              /* max AC norm after the last iteration     */
  double normal_residual;           /* mean |AC_N| (obstacle + self)            */
  double tangential_residual;       /* mean |AC_T| (obstacle + self)            */
  double time;                      /* simulated time after the step (s)        */
  int32_t refine_sweeps;            /* FP32 mode: refinement sweeps, last step  */
  double solve_residual;            /* FP32 mode: last relative FP64 residual   */
  double device_ms;                 /* device time of the whole pdf_step call,
                                       CUDA events on the handle's stream      */
} pdf_step_report;

typedef struct pdf_stats {
  /* cumulative device time (ms) per phase since creation, CUDA events */
  double detection_ms, self_detection_ms, ordering_ms;
  double rhs_ms, friction_ms, self_friction_ms, solve_ms, step_ms;
  int64_t steps, iterations;
  /* one-time set-up */
  double setup_ms, factor_ms;
  int64_t factor_nnz;               /* nnz(L) of the Cholesky factor            */
  int32_t n_supernodes, n_levels;   /* supernodal elimination tree              */
  int64_t lhs_nnz;                  /* nnz(M + dt^2 A^T A)                      */
  int32_t n_constraint_rows;        /* rows(A)                                  */
  int64_t kernel_launches;          /* this library's kernels launched so far   */
  int64_t factor_nnz_true;          /* structural nnz(L) without padding        */
  int32_t sweep_chunk;              /* work-item width chosen by the autotuner  */
  double sweep_chunk_ms[3];         /* solve time measured for 32, 64, 128      */
  /* subtree blocks of the solve schedule chosen by the autotuner: the
   * elimination-tree level up to which subtrees are solved by one CTA each,
   * the number of blocks, and the factor elements in blocks / above them */
  int32_t sweep_cut_level, sweep_blocks;
  int64_t sweep_block_elems, sweep_upper_elems;
  double sweep_cut_ms[8];           /* solve time measured for cut levels 0-7   */
  /* the supernodes above the blocks: 0 = dependency-driven work items in one
   * launch per sweep, 1 = one launch per elimination-tree level; the number
   * of such levels, and the solve time in mode 1 for cut levels 0-7 (0 where
   * the levels exceed the launch table) */
  int32_t sweep_upper_mode, sweep_upper_levels;
  double sweep_cut_level_ms[8];
  /* launch shape of the block kernels: 0-4 = 1 CTA of 8 warps, 2 CTAs of 8
   * warps, 3 CTAs of 4 warps, 4 CTAs of 4 warps, 1 CTA of 16 warps per SM;
   * its warps and CTAs,
   * the bulk-copy stages per warp (forward, backward), and the solve time of
   * each shape at the chosen cut level (0 where it does not fit) */
  int32_t sweep_block_shape, sweep_block_warps, sweep_block_ctas;
  int32_t sweep_ring_stages[2];
  double sweep_shape_ms[5];
} pdf_stats;

/* One contact, as the reference's CollisionInfo / SelfCollisionInfo plus
 * the iterate's local force r and AC residual (SFE:350-423, 590-652). */
typedef struct pdf_contact {
  int32_t vertex;                   /* colliding vertex                          */
  int32_t partner;                  /* self contact: paired vertex; else -1      */
  int32_t face[3];                  /* self contact: triangle; else -1           */
  double normal[3];
  double speed[3];                  /* obstacle velocity at the contact point   */
  double mu;
  double force[3];                  /* local-frame contact force r (N, T1, T2)  */
  double ac;                        /* Alart-Curnier norm of the last iteration */
} pdf_contact;

/* ---- opaque handles ---------------------------------------------------- */
typedef struct pdf_handle pdf_handle;
typedef struct pdf_scene pdf_scene;

/* Scene JSON -> scene.  Replaces getSceneFromJSONDocument
 * (include/scene_building.hpp:36-39, src/scene_building.cpp:49-75) together with
 * getJSONDocumentFromFilename (src/jsonHelper.cpp:22-40) and read_obj
 * (src/geometry/io.cpp:65-121).  OBJ coordinates pass through float like the
 * reference's tinyobj reader.  Relative OBJ paths resolve against the JSON
 * file's directory first, then the working directory.  On error *out is NULL
 * and the message is available from pdf_global_error(). */
int pdf_scene_load_json(const char* json_path, pdf_scene** out);
/* Borrowed view of a loaded scene (valid until pdf_scene_free). */
int pdf_scene_view(const pdf_scene* scene, pdf_scene_desc* out);
void pdf_scene_free(pdf_scene* scene);

/* Replaces getSimulationParametersFromJSONDocument
 * (src/simulation_building.cpp:37-78).  Also returns "Frame number" and
 * "Steps per frame" for the caller's loop (may be NULL). */
int pdf_params_load_json(const char* json_path, pdf_params* out,
                         int32_t* frame_number, int32_t* steps_per_frame);

/* Replaces getSimulation(PhysicScene&, const SimulationParameters&)
 * (src/simulation_building.cpp:80-98) and the constructors it runs
 * (SimulationFrictionEstimation SFE:31-62, SimulationSpeed.cpp:29-60,
 * SimulationBase.cpp:46-100): assembles A, the LHS M + dt^2 A^T A, its one-time
 * Cholesky factor, and uploads everything to the device. */
int pdf_create(const pdf_scene_desc* scene, const pdf_params* params,
               pdf_handle** out);

/* Replaces SimulationBase::step() (src/physics/SimulationBase.cpp:103-173),
 * called nsteps times.  report may be NULL.
 * Fixed per-vertex limits of self-collision detection (the reference's
 * vectors have none): at most 32 candidate triangles per vertex before the
 * closest-point filter, and at most 16 pairing partners per vertex; beyond
 * them, or beyond the contact buffers, the call returns
 * PDF_CAPACITY_EXCEEDED.  The steps are enqueued together and the error is
 * read after the last one, so from the first step that overflowed on, the
 * state (and every later step of the call) was computed with truncated
 * contacts: after PDF_CAPACITY_EXCEEDED restore a state saved before the
 * call (pdf_set_state) or recreate the handle. */
int pdf_step(pdf_handle* h, int32_t nsteps, pdf_step_report* report);

/* State read-back / overwrite (PhysicScene::getGeneralizedPositions/Speeds,
 * src/physics/PhysicScene.cpp:233-305).  3N doubles each, either may be NULL.
 * pdf_set_state checks the uploaded state on the device: a non-finite value
 * is rejected (PDF_NAN_DETECTED, state unchanged); the state the handle
 * already holds is a no-op; any other state also drops the learned warm
 * start's memory of the last step's contact impulses. */
int pdf_get_state(pdf_handle* h, double* q, double* v);
int pdf_set_state(pdf_handle* h, const double* q, const double* v);

/* Device-resident state (no copies): pointers to the handle's FP64 q and v
 * (3N each, vertex-major xyz) and the CUDA stream the handle launches on. */
int pdf_device_state(pdf_handle* h, double** q_dev, double** v_dev,
                     void** cuda_stream);

/* Contacts of the last step; *n receives the count; out may be NULL to query. */
int pdf_get_contacts(pdf_handle* h, pdf_contact* out, int32_t capacity,
                     int32_t* n);
int pdf_get_self_contacts(pdf_handle* h, pdf_contact* out, int32_t capacity,
                          int32_t* n);
/* Self-contact Gauss-Seidel levels (SFE:161-279): level_ptr[n_levels+1],
 * order[n_self] (indices into pdf_get_self_contacts' order). */
int pdf_get_self_levels(pdf_handle* h, int32_t* level_ptr, int32_t level_cap,
                        int32_t* order, int32_t order_cap, int32_t* n_levels);

/* Per-phase statistics.  pdf_export_stats replaces exportStats
 * (SimulationBase.cpp:474-494 inside SFE:756-771, sections written by
 * computeAndWriteStats, template/physics/io.tpp:23-63): the reference's
 * sections in its order, one sample per step (detection, self detection,
 * ordering, step) or per PD iteration (iteration, solver, full RHS, base RHS,
 * friction, self friction) in microseconds of device time.  Per-iteration
 * times come from the device clock (%globaltimer) read at the entry of the
 * iteration's kernels, since the iterations run inside a CUDA graph. */
int pdf_get_stats(pdf_handle* h, pdf_stats* out);
int pdf_export_stats(pdf_handle* h, const char* path);
/* The same text into a caller buffer: *len receives its length (without the
 * terminating NUL); at most cap - 1 characters and a NUL are written (cap 0:
 * query the length).  Lets a caller append the sections to a stream it
 * already holds, as SimulationBase::exportStats(std::ofstream&) does. */
int pdf_export_stats_text(pdf_handle* h, char* buf, int64_t cap, int64_t* len);

/* ---- frame output and per-step logs (src/main.cpp:86-114) -------------- */
/* Enqueues a copy of the current positions (3N doubles) into the handle's
 * pinned frame buffer `slot` (0 or 1) on a copy stream and returns at once;
 * the copy overlaps the following steps (the next step's write-back of q
 * waits for it).  No counterpart in the reference, whose frame writer
 * (Mesh::writeObj, src/geometry/Mesh.cpp:95-109) reads the state
 * synchronously. */
int pdf_frame_capture(pdf_handle* h, int32_t slot);
/* Waits for the copy of `slot`; *q receives its 3N positions (valid until the
 * slot is captured again or the handle is destroyed: capture a slot again
 * only once its previous positions have been consumed). */
int pdf_frame_wait(pdf_handle* h, int32_t slot, const double** q);
/* Positions and velocities (3 doubles each per listed vertex; either output
 * may be NULL) of n scene vertices: the reads of the reference's log
 * callbacks (getVertexPosition / getVertexSpeed, src/log_building.cpp:89-118),
 * gathered on the device. */
int pdf_get_vertices(pdf_handle* h, const int32_t* vertices, int32_t n,
                     double* q, double* v);
/* Per-iteration Alart-Curnier norms of every contact of the last step, when
 * the handle was created with trace_alart_curnier = 1
 * (SimulationFrictionEstimation::updateIterationData SFE:720-752).  out holds
 * iterations x (n_contacts + n_self) x 2 doubles: per iteration, the obstacle
 * contacts then the self contacts, each (tangential norm, |normal|).  out may
 * be NULL to query the sizes; PDF_CAPACITY_EXCEEDED when cap is too small. */
int pdf_get_alart_curnier_trace(pdf_handle* h, double* out, int64_t cap,
                                int32_t* iterations, int32_t* n_contacts,
                                int32_t* n_self);

/* The scene JSON's optional "log" array (getLogCallBacksFromJSONDocument,
 * src/log_building.cpp:28-129): each entry prints, after every step, the
 * positions ("position") or velocities ("velocity") of listed vertices of
 * mesh 0. */
enum pdf_log_kind { PDF_LOG_POSITION = 0, PDF_LOG_VELOCITY = 1 };
typedef struct pdf_log_entry {
  int32_t kind;               /* pdf_log_kind              */
  int32_t n_vertices;
  const int32_t* vertices;    /* "vertices", mesh-0 indices */
} pdf_log_entry;
typedef struct pdf_log pdf_log;
/* No "log" member: an empty list.  Errors as the reference's reader. */
int pdf_log_load_json(const char* json_path, pdf_log** out);
int pdf_log_view(const pdf_log* log, int32_t* n_entries,
                 const pdf_log_entry** entries);
void pdf_log_free(pdf_log* log);

/* Per-iteration mean AC residuals of the last step (n <= cap written). */
int pdf_get_residual_history(pdf_handle* h, double* out, int32_t cap,
                             int32_t* n);

/* Times one phase of the PD iteration in isolation on the handle's stream:
 * reps back-to-back launches bracketed by CUDA events, average device time per
 * repetition in *ms.  Phases: 0 = global solve (forward + backward supernodal
 * sweeps), 1 = local step (projections + right-hand side), 2 = contact
 * projection, 3 = detection (obstacles and self-collision).  The state is not
 * advanced in a meaningful way; call it before or after a measured run.
 * *bytes receives the algorithmic bytes one repetition must move (phases 0,
 * 1 and 3; 0 for phase 2). */
int pdf_time_phase(pdf_handle* h, int32_t phase, int32_t reps, double* ms,
                   double* bytes);

/* Device time (CUDA events, average of reps) of the five launches of one
 * global solve on the handle's current right-hand side: part_ms[0] block
 * forward sweep, [1] upper forward items, [2] upper backward items, [3]
 * block backward sweep with its write-back, [4] the upper columns'
 * write-back.  The state is restored afterwards (no counterpart in the
 * reference; a profiling aid). */
int pdf_time_solve_parts(pdf_handle* h, int32_t reps, double* part_ms);

/* Replaces the solve schedule the autotuner chose at create (no counterpart
 * in the reference): work-item width chunk (32, 64 or 128), subtree-block
 * cut level 0-7, the mode of the supernodes above the blocks (0 =
 * dependency-driven work items, 1 = one launch per elimination-tree level),
 * and the launch shape of the block kernels (0-4, as stats
 * sweep_block_shape).  Every schedule solves the same system; the results
 * agree to rounding.  PDF_INVALID_ARG for values outside these sets, for
 * mode 1 on a scene with more upper levels than the launch table holds
 * (stats sweep_upper_levels), or for a shape the blocks do not fit. */
int pdf_set_sweep_schedule(pdf_handle* h, int32_t chunk, int32_t cut_level,
                           int32_t upper_mode, int32_t block_shape);

/* Check of the bounded device waits (no counterpart in the reference): runs
 * one global solve whose dependency targets lie one solve ahead of the
 * completion counters, on a schedule whose blocks are only the leaves, so
 * that no wait of the supernodal sweeps can be satisfied, with each wait
 * limited to max_spins polls (about 32 ns of sleep each).  Every wait gives
 * up, the sweeps return, and the call returns PDF_DEVICE_TIMEOUT (or
 * PDF_INVALID_ARG when the scene's schedule has nothing to wait for).  The
 * GPU context stays usable; the handle does not: destroy it. */
int pdf_check_wait_timeout(pdf_handle* h, int32_t max_spins);

/* Host-only consistency check of the factorisation and of the device sweep
 * layout (no GPU needed): builds the global-step matrix of the scene, factors
 * it, and runs a sequential emulation of the two device sweeps (same subtree
 * blocks and work items, same tiled layout, every index bounds-checked) to
 * solve (M + dt^2 A^T A) x = b for three right-hand sides (3N,
 * vertex-major), for every schedule the autotuner can choose; they must
 * agree to 1e-10 relative (else PDF_INVALID_ARG). */
int pdf_factor_check(const pdf_scene_desc* scene, const pdf_params* params,
                     const double* b, double* x);

/* Last error message of this handle (never NULL). */
const char* pdf_last_error(const pdf_handle* h);
/* Last error of calls that have no handle (loading, create failures). */
const char* pdf_global_error(void);

void pdf_destroy(pdf_handle* h);

/* ---- stand-alone detection kernels (bit-exact candidate sets) ---------- */
/* Vertex-triangle candidates of one mesh: the set
 * { (v, t) : AABB(t) intersects [x_v - 1.1 tol, x_v + 1.1 tol] } (closed
 * boxes) that getMeshPotentialTriangleCollision computes with CGAL
 * box_intersection_d (src/geometry/geometry_util.cpp:284-327), found with a GPU
 * LBVH over triangles.  Output sorted by (vertex, triangle).  pairs: 2*cap
 * int32.  Returns PDF_CAPACITY_EXCEEDED (and the true count in *n) if cap is
 * too small. */
int pdf_detect_candidates(const double* positions, int32_t n_vertices,
                          const int32_t* triangles, int32_t n_triangles,
                          double tolerance, int32_t* pairs, int32_t cap,
                          int32_t* n, int32_t device);

/* Self collisions of one mesh: candidates, closest-point filter
 * (geometry_util.cpp:229-262, 506-616) and the greedy node-node pairing
 * (geometry_util.cpp:94-219) in canonical (vertex, triangle) order.
 * out: contacts with vertex, partner, face, normal filled. */
int pdf_detect_self_collisions(const double* positions, int32_t n_vertices,
                               const int32_t* triangles, int32_t n_triangles,
                               double tolerance, pdf_contact* out, int32_t cap,
                               int32_t* n, int32_t device);

/* Allocation-free variant of pdf_detect_candidates.  It has no counterpart in
 * the reference.  For callers that must not allocate device memory when they
 * detect (code inside another framework's memory pool, real-time loops with a
 * fixed memory budget, hosts whose allocator is not the CUDA runtime's): the
 * whole workspace is one fixed, file-scope device array (about 30 MB, held by
 * every GPU that loads this library until the process exits); the call makes
 * no cudaMalloc / cudaFree and no allocating library call.
 *   positions (3*n_vertices doubles), triangles (3*n_triangles) and pairs
 *   (2*cap int32) are DEVICE pointers on the current device; *n (host)
 *   receives the number of candidate pairs, written sorted by (vertex,
 *   triangle) exactly as pdf_detect_candidates returns them.
 *   Limits: n_triangles <= 65536 and at most 262144 candidate pairs; larger
 *   inputs return PDF_CAPACITY_EXCEEDED without touching pairs (when the
 *   pairs exceed cap or the limit, *n still receives their number).  A vertex
 *   whose hierarchy walk overflows its stack also gives
 *   PDF_CAPACITY_EXCEEDED.
 *   Every call looks up the array's device address on the current device
 *   (cudaGetSymbolAddress, which allocates nothing), so it stays valid after a
 *   cudaDeviceReset and from any host thread.  All calls share the one array
 *   and find it as the previous call left it: calls that overlap on the GPU
 *   (other streams, other host threads) race.  The call reads the pair count
 *   back to the host and synchronises cuda_stream (NULL = the legacy default
 *   stream), so it cannot be recorded into a CUDA graph by stream capture. */
int pdf_detect_candidates_noalloc(const double* positions, int32_t n_vertices,
                                  const int32_t* triangles, int32_t n_triangles,
                                  double tolerance, int32_t* pairs, int32_t cap,
                                  int32_t* n, void* cuda_stream);

/* ---- learned warm start (no counterpart in the reference) --------------- */
/* A per-contact MLP 10 -> 64 -> 64 -> 3 (ReLU) predicts the converged local
 * force of every obstacle contact from the predictor velocity relative to the
 * obstacle, the gap, the vertex's contact impulse of the previous step and
 * mu; under PDF_WARM_MLP the first PD iteration of a step uses the prediction
 * (projected on the friction cone) instead of the cone projection.  BF16
 * tensor-core forward and backward kernels, FP32 master weights, Adam.
 * Weights: pdf_mlp_param_count() floats, W1[64][10] b1 W2[64][64] b2 W3[3][64] b3. */
int32_t pdf_mlp_param_count(void);
/* Seeded He initialisation (host only). */
int pdf_mlp_init(float* weights, uint64_t seed);
/* Weights file: "PDFMLP01", int32 {10, 64, 3, count}, count little-endian floats. */
int pdf_mlp_save(const char* path, const float* weights);
int pdf_mlp_load(const char* path, float* weights);
/* Stand-alone kernels on host buffers (device = CUDA ordinal):
 * Y[n][3] = MLP(X[n][10]); grad = d(mean_s |MLP(x_s) - t_s|^2)/d(weights)
 * and *loss = that mean; fit = seeded shuffle, 90/10 split, Adam over
 * mini-batches, weights updated in place, losses of the last epoch and of the
 * held-out part. */
int pdf_mlp_forward(const float* weights, const float* X, int32_t n, float* Y,
                    int32_t device);
int pdf_mlp_gradient(const float* weights, const float* X, const float* T,
                     int32_t n, float* grad, double* loss, int32_t device);
int pdf_mlp_fit(float* weights, const float* X, const float* T, int32_t n,
                int32_t epochs, int32_t batch, double learning_rate,
                uint64_t seed, int32_t device, double* train_loss,
                double* val_loss);
/* Per-handle: weights used by PDF_WARM_MLP steps. */
int pdf_mlp_set_weights(pdf_handle* h, const float* weights, int32_t count);
int pdf_mlp_get_weights(pdf_handle* h, float* weights, int32_t count);
/* Sample log on the device: after every step, one (features, converged local
 * force / (m |g| dt)) sample per obstacle contact (0 for a contact that took
 * off in the last iteration), up to capacity samples.  capacity 0 stops
 * logging and frees the log; a new call restarts it empty. */
int pdf_mlp_log(pdf_handle* h, int32_t capacity);
/* Copies the logged samples out (X: n*10, T: n*3 floats; either NULL to query *n). */
int pdf_mlp_samples(pdf_handle* h, float* X, float* T, int32_t cap, int32_t* n);
/* Trains the handle's weights on its logged samples without leaving the
 * device: per-feature standardisation of inputs and targets, seeded He
 * initialisation, Adam, then the standardisation folded back into the first
 * and last layers.  The losses are those of the standardised problem
 * (1.0 = predicting the mean). */
int pdf_mlp_train(pdf_handle* h, int32_t epochs, int32_t batch,
                  double learning_rate, uint64_t seed, double* train_loss,
                  double* val_loss);

#ifdef __cplusplus
}
#endif
#endif /* PDF_B200_H */
