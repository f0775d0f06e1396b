/*
 * avbd.h - C-ABI of the B200 (sm_100a) augmented vertex block descent step.
 *
 * Drop-in boundary for SkyePhyX's `Solver` (src/physics/solver.hpp:22-94):
 * the same bodies, box colliders, joints, springs, Neo-Hookean tetrahedra and
 * StVK triangles, built through the same calls and stepped by `avbd_step`,
 * which replaces `Solver::Step()` (src/physics/solver.cpp:199-627).  All step
 * work runs in CUDA kernels; the host only stages scenes and reads results.
 *
 * Conventions: plain pointers and sizes, float32, quaternions as (w, x, y, z),
 * vectors as 3 consecutive floats; body / force / energy ids are creation
 * indices returned by the add_* calls.  Negative returns are AVBD_ERR_* codes;
 * step calls return an AVBD_STATUS_* value.  One world is not thread-safe;
 * distinct worlds are independent.
 */
#ifndef AVBD_H
#define AVBD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status and error codes ---- */
#define AVBD_STATUS_OK        0  /* step ran */
#define AVBD_STATUS_EXPLODED  1  /* a velocity component left [-500, 500] m/s (solver.cpp:182-196); the
                                    world is frozen like Solver::emergencyStop and later steps are no-ops */
#define AVBD_STATUS_NAN       2  /* a pose became NaN; frozen like EXPLODED */
#define AVBD_STATUS_CAPACITY  3  /* a device table was too small for this step; the step was not applied */
#define AVBD_STATUS_TIMEOUT   4  /* a bounded device wait gave up; the step was not applied */

#define AVBD_ERR_INVALID  (-1)   /* bad argument (unknown id, null pointer, bad size) */
#define AVBD_ERR_CUDA     (-2)   /* a CUDA runtime call failed */
#define AVBD_ERR_NOMEM    (-3)   /* device or host allocation failed */
#define AVBD_ERR_STATE    (-4)   /* call not valid in the current state */
#define AVBD_ERR_NODEVICE (-5)   /* no CUDA device: there is no CPU fallback */

/* ModelType (geometry.hpp:17-22); every body collides as a box (collision.hpp:28-31). */
#define AVBD_MODEL_CUBE    0
#define AVBD_MODEL_SPHERE  1
#define AVBD_MODEL_PYRAMID 2

/* EigenProjectionMode (math.hpp:99-104). */
#define AVBD_PROJECT_CLAMP    0
#define AVBD_PROJECT_ABSOLUTE 1
#define AVBD_PROJECT_ADAPTIVE 2

/* Public solver parameters, same names and defaults as solver.hpp:69-84. */
typedef struct AvbdParams {
    int32_t num_iterations;         /* numIterations = 10 */
    float   step_value;             /* stepValue (dt) = 1/60 s */
    float   alpha;                  /* 0.95 */
    float   beta;                   /* 100000 */
    float   gamma;                  /* 0.99 */
    float   on_penetration_penalty; /* 0 */
    int32_t post_stabilization;     /* 1 */
    int32_t projection_mode;        /* AVBD_PROJECT_ABSOLUTE */
    float   trust_region_rho;       /* 0 */
} AvbdParams;

/* Per-phase device times of the last step in ms, named after SolverTimings
 * (solver.hpp:10-19) plus the colouring phase this build adds. */
typedef struct AvbdTimings {
    float broad_phase_ms;
    float warmstart_ms;       /* narrowphase + manifold warm-start + incidence build */
    float colouring_ms;
    float prediction_ms;
    float primal_dual_ms;
    float velocity_update_ms;
    float post_stab_ms;
    float total_substep_ms;
} AvbdTimings;

typedef struct AvbdWorld AvbdWorld;
typedef struct AvbdBatch AvbdBatch;

void avbd_default_params(AvbdParams* out);
const char* avbd_status_string(int32_t code);

/* ---------------------------------------------------------------------------
 * Single scene (the plain path).  Replaces one Solver instance.
 * ------------------------------------------------------------------------- */

/* Solver::Solver / Solver::Start (solver.cpp:18-33). device = CUDA ordinal. */
int32_t avbd_world_create(const AvbdParams* params, int32_t device, AvbdWorld** out);
/* Solver::~Solver / Clear (solver.cpp:23-47). */
int32_t avbd_world_destroy(AvbdWorld* w);
int32_t avbd_world_clear(AvbdWorld* w);
int32_t avbd_set_params(AvbdWorld* w, const AvbdParams* params);
int32_t avbd_get_params(const AvbdWorld* w, AvbdParams* out);

/* Solver::AddBody (solver.cpp:50-101). Returns the body id. */
int32_t avbd_add_body(AvbdWorld* w, int32_t model_type, float density, float friction, const float pos[3],
                      const float scale[3], const float vel[3], const float quat_wxyz[4], const float omega[3],
                      int32_t is_static);
/* n calls of Solver::AddBody with one model type, from arrays (density[n],
 * friction[n], pos[3n], scale[3n], quat_wxyz[4n], is_static[n]; vel/omega
 * [3n] may be NULL for zero). Returns the id of the first body. */
int32_t avbd_add_bodies(AvbdWorld* w, int32_t n, int32_t model_type, const float* density, const float* friction,
                        const float* pos, const float* scale, const float* vel, const float* quat_wxyz,
                        const float* omega, const int32_t* is_static);
/* Solver::AddParticle (solver.cpp:119-131): a 0.1 m cube with zero inertia. */
int32_t avbd_add_particle(AvbdWorld* w, float mass, float friction, const float pos[3], const float vel[3],
                          int32_t is_static);
/* Mesh::isStatic set after creation, as levels.h:472-473 pins cloth corners. */
int32_t avbd_set_body_static(AvbdWorld* w, int32_t body, int32_t is_static);
/* Spring (force.hpp:95, spring.cpp:13-37). body_a = -1 anchors r_a in world
 * space; rest_length < 0 takes the initial distance; fracture applies to its
 * single row (levels.h:282 sets constraintPoints[0].fracture). Returns force id. */
int32_t avbd_add_spring(AvbdWorld* w, int32_t body_a, const float r_a[3], int32_t body_b, const float r_b[3],
                        float stiffness, float rest_length, int32_t is_rope, float fracture);
/* Joint (force.hpp:119-122, joint.cpp:24-66): 3 positional + 3 angular rows;
 * stiffness/fracture per row (INFINITY = hard / unbreakable). Returns force id. */
int32_t avbd_add_joint(AvbdWorld* w, int32_t body_a, const float r_a[3], int32_t body_b, const float r_b[3],
                       const float stiffness[6], const float fracture[6]);
/* NeoHookeanFEM (energy.hpp:50-52, neohookeanfem.cpp:5-37). Returns energy id. */
int32_t avbd_add_neohookean_tet(AvbdWorld* w, const int32_t v[4], float youngs_modulus, float poisson_ratio);
/* STVKFEM triangle membrane (energy.hpp:90-92, stvkfem.cpp:5-35). Returns energy id. */
int32_t avbd_add_stvk_tri(AvbdWorld* w, const int32_t v[3], float youngs_modulus, float poisson_ratio);
/* St. Venant-Kirchhoff tet (no reference counterpart: the reference has the
 * StVK triangle only, stvkfem.cpp).  Psi = mu tr(E^2) + lambda/2 tr(E)^2 with
 * E = (F^T F - I)/2, the Neo-Hookean tet's rest data, projection modes and
 * vertex-Hessian reconstruction; below 1% of its rest volume an element takes
 * STVKFEM's isotropic penalty.  Shares the tet id space. Returns the tet id. */
int32_t avbd_add_stvk_tet(AvbdWorld* w, const int32_t v[4], float youngs_modulus, float poisson_ratio);
/* makeTetVolume's particles and tets (geometry.cpp:30-94) with StVK tets. */
int32_t avbd_make_stvk_tet_volume(AvbdWorld* w, float ox, float oy, float oz, int32_t nx, int32_t ny, int32_t nz,
                                  float cell_size, float youngs_modulus, float poisson_ratio, float particle_mass,
                                  float friction, int32_t pin_min_x);
/* GeometryHelpers::makeTetVolume (geometry.cpp:30-94): nx*ny*nz particles,
 * 5 Neo-Hookean tets per hex. Returns the id of the first particle. */
int32_t avbd_make_tet_volume(AvbdWorld* w, float ox, float oy, float oz, int32_t nx, int32_t ny, int32_t nz,
                             float cell_size, float youngs_modulus, float poisson_ratio, float particle_mass,
                             float friction, int32_t pin_min_x);

/* GeometryHelpers::makeTetSphere (geometry.cpp:106-232): a centre particle
 * and N = round(res) concentric shells of 6N x 3N ring particles plus poles,
 * filled with Neo-Hookean tets (the innermost shell fanned to the centre,
 * prisms of 3 tets between shells).  Returns the id of the first particle. */
int32_t avbd_make_tet_sphere(AvbdWorld* w, float cx, float cy, float cz, float radius, float res,
                             float youngs_modulus, float poisson_ratio, float particle_mass, float friction);

/* Solver::RemoveBody (solver.hpp:49, solver.cpp:104-115) and Mesh::~Mesh (geometry.cpp:11-25):
 * the body and every force and energy on it stop taking part.  Ids stay
 * stable (the reference swap-removes and renumbers).  Valid before or after
 * the first step. */
int32_t avbd_remove_body(AvbdWorld* w, int32_t body);
/* Solver::RemoveForce (solver.hpp:47): a joint or spring by force id. */
int32_t avbd_remove_force(AvbdWorld* w, int32_t force);
/* Solver::RemoveEnergy (solver.hpp:48): a Neo-Hookean tet or StVK triangle
 * by the id its add call returned (the two kinds are numbered apart). */
int32_t avbd_remove_neohookean_tet(AvbdWorld* w, int32_t tet);
int32_t avbd_remove_stvk_tri(AvbdWorld* w, int32_t tri);

/* Solver::Step() (solver.cpp:199-627) with the world's params. */
int32_t avbd_step(AvbdWorld* w);
/* Sets stepValue/numIterations, then steps. */
int32_t avbd_step_dt(AvbdWorld* w, float dt, int32_t iterations);

int32_t avbd_num_bodies(const AvbdWorld* w);
int32_t avbd_num_dynamic_bodies(const AvbdWorld* w);
/* Solver::emergencyStop (solver.hpp:84). */
int32_t avbd_emergency_stop(const AvbdWorld* w);
/* 1 while joint/spring `force` takes part in the step; 0 once a fracture
 * disabled it (Force::Disable, force.hpp:57-66; solver.cpp:473-481) or it was
 * removed with a body.  The reference's caller sees the same by the Force
 * leaving Solver::solverForces. */
int32_t avbd_force_live(AvbdWorld* w, int32_t force);

/* Body state by id into caller-owned HOST buffers (any may be NULL):
 * pos n*3, quat n*4 (w,x,y,z), vel n*3, omega n*3; n = avbd_num_bodies().
 * A removed body (avbd_remove_body, or out of bounds, solver.cpp:521-534)
 * reads NaN. */
int32_t avbd_get_state(AvbdWorld* w, float* pos, float* quat_wxyz, float* vel, float* omega);
/* Overwrites body state (e.g. to restore a snapshot); NULL leaves a field as is. */
int32_t avbd_set_state(AvbdWorld* w, const float* pos, const float* quat_wxyz, const float* vel,
                       const float* omega);

/* Snapshot / restore of a stepped world (device-resident state, byte for
 * byte: bodies, forces, energies, both manifold tables and their contacts,
 * colour lists, counters).  No counterpart in the reference.  The buffer may
 * be host or device memory (copies use unified addressing); size it with
 * avbd_snapshot_bytes.  avbd_restore takes a snapshot of the same world, or
 * of a world built the same way, whose tables have not grown since: then the
 * next steps repeat bit for bit (deterministic replay, pre-emption).  Returns
 * AVBD_ERR_STATE before the first step or when the table sizes differ. */
int64_t avbd_snapshot_bytes(const AvbdWorld* w);
int32_t avbd_snapshot(AvbdWorld* w, void* dst, int64_t bytes);
int32_t avbd_restore(AvbdWorld* w, const void* src, int64_t bytes);

/* Mesh::color (AddBody's color argument, solver.cpp:50); default white.
 * Read only by the instance export. */
int32_t avbd_set_body_color(AvbdWorld* w, int32_t body, const float rgb[3]);

/* The renderer's GPUInstanceData (RenderEngine.hpp:43-49), 128 bytes:
 * model matrix (column-major 4x4: rotation x scale, position), normal matrix
 * (the inverse transpose of its 3x3 block, three columns padded to four
 * floats) and colour (r, g, b, 1). */
typedef struct AvbdInstance {
    float model[16];
    float normal[12];
    float color[4];
} AvbdInstance;

/* Headless pose export (RenderEngine::UpdateInstanceBuffer,
 * RenderEngine.cpp:951-1000, without a graphics API): one AvbdInstance per
 * live body, grouped by model type (cube, sphere, pyramid) and by body id
 * within a type, as the renderer packs its per-model batches.  dst is device
 * memory an external renderer can read (written in place by a kernel) or
 * host memory (copied).  first/count per model may be NULL.  Returns the
 * instances written, AVBD_ERR_INVALID when capacity is too small. */
int32_t avbd_export_instances(AvbdWorld* w, AvbdInstance* dst, int32_t capacity, int32_t first_per_model[3],
                              int32_t count_per_model[3]);

/* Live contact manifolds after the last step (parity introspection).
 * Returns the count; fills up to max entries: pairs (A,B) body ids, counts,
 * ids (8 per manifold, unused = 0xFFFFFFFF) and data (8 x 16 floats per
 * manifold: penetration, normal xyz, rA xyz, rB xyz, penalty x3, lambda x3). */
int32_t avbd_get_contacts(AvbdWorld* w, int32_t max, int32_t* pairs, int32_t* counts, uint32_t* ids,
                          float* data);
/* Colour of each body in the last step (-1 = static); returns the colour count. */
int32_t avbd_get_colours(AvbdWorld* w, int32_t* colours);
int32_t avbd_get_timings(const AvbdWorld* w, AvbdTimings* out);

/* CollisionSpace::CollisionBoxBox (collision.cpp:271-447) on two bodies as
 * they stand, on the device. Fills ids[8], data[8*13] (penetration, normal,
 * rA, rB, position); returns the contact count. Kernel-level parity check. */
int32_t avbd_collide(AvbdWorld* w, int32_t body_a, int32_t body_b, uint32_t* ids, float* data);

/* Allocation-free variant of avbd_collide for up to
 * AVBD_COLLIDE_NOALLOC_MAX_PAIRS pairs (body_a[i], body_b[i]) per call. It has
 * no counterpart in the reference. It is for callers that may not allocate
 * device memory during a call (fixed memory budgets, custom pools, hosts
 * where cudaMalloc/cudaFree would synchronise or fail): its device scratch is
 * one fixed array of about 1.9 MB that every GPU loading this library holds
 * until exit. Outputs go to caller-owned host buffers: ids[8n] (unused =
 * 0xFFFFFFFF), data[8*13*n] (as avbd_collide), counts[n]. The world must have
 * been uploaded (stepped, or avbd_collide called, once). The call copies the
 * pairs in from host memory and returns once the results are in the host
 * buffers. The first call on a device looks up the scratch address, so make
 * it before any stream capture. Calls share the scratch: calls that overlap
 * on the GPU (several threads, or several worlds on one device) race. More
 * pairs than the maximum, or an unknown body id, return AVBD_ERR_INVALID.
 * The caller's current device is left as it was. */
#define AVBD_COLLIDE_NOALLOC_MAX_PAIRS 4096
int32_t avbd_collide_noalloc(AvbdWorld* w, int32_t n, const int32_t* body_a, const int32_t* body_b, uint32_t* ids,
                             float* data, int32_t* counts);

/* ---------------------------------------------------------------------------
 * Batched: many independent scenes advanced by one persistent kernel per step
 * (no reference counterpart; each scene behaves as its own Solver).
 * ------------------------------------------------------------------------- */
int32_t avbd_batch_create(const AvbdParams* params, int32_t device, AvbdBatch** out);
int32_t avbd_batch_destroy(AvbdBatch* b);
/* Reserves the batch's device pools: capacity for `bodies` bodies, `forces`
 * joints+springs, `tets`, `tris` and `scenes` scene slots (contact and
 * incidence tables are sized from the body count). Without a reservation the
 * first step sizes the pools to the scenes added so far. */
int32_t avbd_batch_reserve(AvbdBatch* b, int64_t bodies, int64_t forces, int64_t tets, int64_t tris,
                           int32_t scenes);
/* Copies the scene staged in `w` (built with the calls above, never stepped)
 * into the batch and returns its scene id (ids of retired scenes are reused).
 * Once the pools exist (a reservation or a first step) the scene is placed and
 * uploaded at once and takes part from the next step on; AVBD_ERR_NOMEM means
 * it does not fit in the free pool space now (nothing was changed). */
int32_t avbd_batch_add_scene(AvbdBatch* b, const AvbdWorld* w);
/* Retires a scene and returns its pool space for later admissions. */
int32_t avbd_batch_remove_scene(AvbdBatch* b, int32_t scene);
/* Index of a live scene's first body in the pose buffers of avbd_batch_get_all_poses. */
int32_t avbd_batch_scene_body_offset(const AvbdBatch* b, int32_t scene);
/* Allocates the pools for the scenes added so far, chooses the launch shape
 * and stages the scenes into page-locked host buffers; the scenes are copied
 * to the device (one copy per device array) by the next batch call that
 * touches the device: usually the first avbd_batch_step.  The page-locked
 * buffers are held until avbd_batch_destroy.  Optional: the first
 * avbd_batch_step stages through pageable buffers, freed after the copy,
 * when it was not called.  No-op once the pools exist. */
int32_t avbd_batch_prepare(AvbdBatch* b);
/* Host-to-device bytes the last upload of staged scenes copied (0 before it). */
int64_t avbd_batch_uploaded_bytes(const AvbdBatch* b);
/* Page-locked host memory for the caller's pose and instance buffers
 * (asynchronous copies need it): bytes on the given device's context;
 * AVBD_ERR_NOMEM when the host cannot lock that much. */
int32_t avbd_host_alloc_pinned(int32_t device, int64_t bytes, void** out);
int32_t avbd_host_free_pinned(void* p);
/* Advances every live scene by `steps` steps (one persistent kernel launch per
 * step, replayed from a CUDA graph). Returns AVBD_STATUS_OK or an error. */
int32_t avbd_batch_step(AvbdBatch* b, int32_t steps);
/* Scenes held (live or staged). */
int32_t avbd_batch_num_scenes(const AvbdBatch* b);
int32_t avbd_batch_scene_status(AvbdBatch* b, int32_t scene);
int32_t avbd_batch_scene_bodies(const AvbdBatch* b, int32_t scene);
/* Dynamic bodies summed over live scenes (body-iterations per step =
 * this x num_iterations). */
int64_t avbd_batch_dynamic_bodies(const AvbdBatch* b);
/* Poses of one scene into host buffers (pos n*3, quat n*4). */
int32_t avbd_batch_get_state(AvbdBatch* b, int32_t scene, float* pos, float* quat_wxyz, float* vel,
                             float* omega);
/* Poses of every pool slot (pos and rotation x y z w as float4 per body) into
 * host buffers of max_bodies float4; a scene's bodies start at
 * avbd_batch_scene_body_offset(). */
int32_t avbd_batch_get_all_poses(AvbdBatch* b, float* pos, float* quat_xyzw, int64_t max_bodies);
/* The same poses, read back while the next step runs: the call snapshots them
 * on the device (so avbd_batch_step may follow at once) and returns; the copy
 * into the host buffers (page-locked for an asynchronous copy) completes by
 * avbd_batch_read_poses_wait, or before the read after next reuses the
 * snapshot.  The host buffers must stay valid until then. */
int32_t avbd_batch_read_poses(AvbdBatch* b, float* pos, float* quat_xyzw, int64_t max_bodies);
int32_t avbd_batch_read_poses_wait(AvbdBatch* b);
/* Snapshot of one live scene of a batch (no reference counterpart): every
 * device value of the scene (bodies, forces, energies, both manifold tables
 * and contacts, incidence, colours, counters).  dst may be host or device
 * memory of avbd_batch_scene_snapshot_bytes() bytes.  avbd_batch_scene_restore
 * admits a snapshot as a new scene of this batch (or of another batch of the
 * same pools layout), wherever it fits, and returns its scene id; the scene
 * then takes the steps it would have taken without the interruption, bit for
 * bit (serving pre-emption: snapshot, remove, restore later).  NOMEM when it
 * does not fit now. */
int64_t avbd_batch_scene_snapshot_bytes(AvbdBatch* b, int32_t scene);
int32_t avbd_batch_scene_snapshot(AvbdBatch* b, int32_t scene, void* dst, int64_t bytes);
int32_t avbd_batch_scene_restore(AvbdBatch* b, const void* src, int64_t bytes);
/* avbd_export_instances for one scene of a batch. */
int32_t avbd_batch_export_instances(AvbdBatch* b, int32_t scene, AvbdInstance* dst, int32_t capacity,
                                    int32_t first_per_model[3], int32_t count_per_model[3]);
/* Device bytes a scene staged in `w` needs inside a batch (admission control). */
int64_t avbd_scene_footprint_bytes(const AvbdWorld* w);
/* Per-scene counters after the last step: status, colours, candidate pairs,
 * contact points, incidence entries, steps taken (6 values). */
int32_t avbd_batch_scene_info(AvbdBatch* b, int32_t scene, int32_t out[6]);
/* Launch shape of the persistent kernel: threads per CTA (32..1024, 0 = the
 * most the kernel build serves; clamped to it) and CTAs per SM (0 = as many
 * as fit). */
int32_t avbd_batch_set_launch(AvbdBatch* b, int32_t threads_per_cta, int32_t ctas_per_sm);
int32_t avbd_batch_get_launch(const AvbdBatch* b, int32_t* threads_per_cta, int32_t* ctas_per_sm);
/* Small scenes share a CTA: a scene with at most units_per_lane (bodies +
 * tets) per lane of half a team is run by half of it while the other half
 * takes the next scene, down to a warp (or an eighth of a larger CTA).
 * 0 (the default) keeps one scene per CTA.  Autotuner knob. */
int32_t avbd_batch_set_team_work(AvbdBatch* b, int32_t units_per_lane);
/* The same threshold for scenes with tets (their per-colour finish leaves
 * most of a team idle, which a second scene on the CTA can use). Default 0. */
int32_t avbd_batch_set_fem_team_work(AvbdBatch* b, int32_t units_per_lane);
/* Thread-block clusters of cluster_size (1, 2, 4 or 8) CTAs: scenes of at
 * least min_units bodies + tets are each run by a whole cluster (ranks over
 * its CTAs, shared scalars in distributed shared memory, cluster barriers)
 * before the CTAs take the smaller scenes one team each.  A scene's results
 * do not depend on it (bitwise).  1 (the default) is a plain launch.  Before
 * the first step (autotuner knob). */
int32_t avbd_batch_set_cluster(AvbdBatch* b, int32_t cluster_size, int32_t min_units);
/* Scenes of at least min_bodies bodies find broadphase candidates with a
 * uniform grid (the same candidate set and order as the reference's all-pairs
 * loop, which smaller scenes keep); 0 = all-pairs everywhere.  Default 128. */
int32_t avbd_batch_set_grid_broadphase(AvbdBatch* b, int32_t min_bodies);
/* The persistent kernel's queue takes scenes in decreasing body_weight x
 * bodies + tets (default 1: bodies + tets; with clusters always 1), an
 * estimate of each scene's step time for the largest-first order.
 * Autotuner knob; results do not depend on it. */
int32_t avbd_batch_set_queue_weight(AvbdBatch* b, int32_t body_weight);
/* Per-scene device timing (off by default): each step stamps the GPU's
 * global timer (ns) AVBD_SCENE_STAMPS times per scene: when its team starts
 * the step, after the broadphase, the narrowphase, the joint/spring warm
 * start and incidence, the colouring, the prediction, the iterations, the
 * velocity update and removals, and at the end (post-stabilisation done).
 * avbd_batch_scene_times copies those stamps of each slot's last step, up to
 * max_slots slots, and returns the slots copied (zeros for a slot that has
 * not stepped since timing was switched on; a step that stopped early leaves
 * its later stamps from the previous step); with stamps_ns NULL it returns
 * the number of slots. */
#define AVBD_SCENE_STAMPS 9
/* Debug builds (libavbd_checks.so, compiled with AVBD_CHECKS): the first
 * failed device index check of a world / batch as (code, index, bound,
 * failures); returns 1 and fills out[4] in a debug build, 0 otherwise.  A
 * failed check skips its access and never traps. */
int32_t avbd_check_word(const AvbdWorld* w, int32_t out[4]);
int32_t avbd_batch_check_word(AvbdBatch* b, int32_t out[4]);
int32_t avbd_batch_set_scene_timing(AvbdBatch* b, int32_t on);
int32_t avbd_batch_scene_times(AvbdBatch* b, int64_t* stamps_ns, int32_t max_slots);
/* Build of the persistent kernel: 1..4 serve CTAs of up to 256 threads with
 * about 156, 128, 80 or 64 registers per thread (spills traded for resident
 * warps); 5 and 6 serve 512 threads (128 or 64 registers), 7 serves 1024
 * threads (64 registers), giving each scene more lanes. */
int32_t avbd_batch_set_kernel(AvbdBatch* b, int32_t register_variant);
/* Lanes that share one body's primal update (1, 2, 4, 8, 16 or 32), for rigid
 * scenes and for FEM scenes; before the first step (autotuner knob).
 * fem_group may also be AVBD_GROUP_FLAT: every (particle, tet) term of a colour
 * is evaluated by its own lane and each particle then sums its terms in
 * incidence order (scenes with StVK triangles use 4 lanes instead). */
#define AVBD_GROUP_FLAT 64
int32_t avbd_batch_set_groups(AvbdBatch* b, int32_t rigid_group, int32_t fem_group);
/* Same knob for a single world (0 = by scene kind); before the first step. */
int32_t avbd_set_group(AvbdWorld* w, int32_t group);
/* Device time of the last avbd_batch_step call in ms. */
float avbd_batch_last_ms(const AvbdBatch* b);

/* ---------------------------------------------------------------------------
 * Serving: continuous batching of scene-simulation requests (no reference
 * counterpart).  Each request is a staged scene and a step count.  A tick
 * admits the requests that have arrived, in arrival order, as long as their
 * scene fits the free pool space (HBM-budget admission; one that does not
 * fit waits for space), advances every resident scene one step with one
 * graph launch, and retires the scenes that took their last step, so their
 * space goes to the next admissions.  avbd_server_tick returns while the
 * step runs on the GPU: the next tick stages its newcomers meanwhile and then
 * waits for it.  Not thread-safe per server.
 * ------------------------------------------------------------------------- */
typedef struct AvbdServer AvbdServer;

#define AVBD_SERVE_KEEP_RESULT 1   /* keep the poses after the last step (avbd_server_result) */
#define AVBD_SERVE_KEEP_FIRST  2   /* keep the poses after the first step too (tolerance checks) */

typedef struct AvbdServedRequest {
    int32_t request;     /* id returned by avbd_server_submit */
    int32_t status;      /* AVBD_STATUS_* of the scene after its last step */
    int32_t steps;
    int32_t bodies;
    double arrival_s;    /* the times the caller passed: arrival, and the ticks that */
    double admitted_s;   /* admitted it and that found its last step complete */
    double finished_s;
} AvbdServedRequest;

typedef struct AvbdServerStats {
    int64_t submitted, admitted, completed, ticks;
    int64_t body_iterations;   /* dynamic bodies x iterations over the steps launched */
    int64_t uploaded_bytes;    /* host-to-device bytes of admitted scenes */
    int64_t pending, active, resident_dynamic;
    int64_t device_us;         /* device time of the steps completed, microseconds */
    int64_t wait_us;           /* host time blocked on the step in flight, microseconds */
    int64_t regrown;           /* scenes whose full tables grew (each re-ran the steps it missed) */
    int64_t catchup_us;        /* host time spent growing tables and re-running steps, microseconds */
    int64_t stage_us;          /* host time placing and staging newcomers (while a step runs) */
    int64_t retire_us;         /* host time filing readbacks and retiring scenes after a step, incl. catch-up */
    int64_t issue_us;          /* host time issuing uploads, the order list, the step and readbacks */
} AvbdServerStats;

/* Pools for `bodies` bodies (a quarter as many joints+springs and
 * triangles, two tets per body) and `max_scenes` resident scenes, reserved
 * at the first tick. */
int32_t avbd_server_create(const AvbdParams* params, int32_t device, int64_t bodies, int32_t max_scenes,
                           AvbdServer** out);
int32_t avbd_server_destroy(AvbdServer* s);
/* The server's batch, for the launch knobs (avbd_batch_set_*) before the
 * first tick; the server drives it (do not step or add scenes directly). */
AvbdBatch* avbd_server_batch(AvbdServer* s);
/* Copies the scene staged in `scene` (built, never stepped) as a request of
 * `steps` steps arriving at `arrival_s` (the caller's clock, as passed to
 * avbd_server_tick); flags: AVBD_SERVE_KEEP_*.  Returns the request id. */
int32_t avbd_server_submit(AvbdServer* s, const AvbdWorld* scene, int32_t steps, double arrival_s, int32_t flags);
/* One tick at the caller's time now_s; returns the scenes the launched step
 * advances (0 when nothing is resident). */
int32_t avbd_server_tick(AvbdServer* s, double now_s);
/* Waits for the step in flight and retires the scenes it finished. */
int32_t avbd_server_drain(AvbdServer* s, double now_s);
/* Takes the next finished request: 1 when one was written to out, 0 when none. */
int32_t avbd_server_poll(AvbdServer* s, AvbdServedRequest* out);
/* Kept poses of a finished request into host buffers (pos n*3, quat n*4
 * w x y z; any may be NULL).  Returns the body count, AVBD_ERR_STATE when
 * the request is not finished or a requested result was not kept. */
int32_t avbd_server_result(AvbdServer* s, int32_t request, float* pos, float* quat_wxyz, float* first_pos,
                           float* first_quat_wxyz);
/* Frees the kept poses of a request. */
int32_t avbd_server_release(AvbdServer* s, int32_t request);
int32_t avbd_server_stats(const AvbdServer* s, AvbdServerStats* out);

#ifdef __cplusplus
}
#endif
#endif /* AVBD_H */
