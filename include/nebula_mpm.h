/* nebula_mpm.h -- C ABI of the B200-native MPMEngine substep.
 *
 * This is the drop-in boundary for nebula's MLS-MPM path.  The reference
 * exposes it as the C++ class `MPMEngine` (src/engine/MPMEngine.h:59-186) whose
 * `step` records Vulkan dispatches; here the same parameter surface is a plain
 * C ABI (no CUDA or torch types in the signatures; streams are `void*` holding a
 * cudaStream_t) over hand-written sm_100a CUDA kernels.
 *
 * Conventions
 *   - Every call returns NEBULA_MPM_OK (0) or an error code; the message of the
 *     last failure on the calling thread is returned by nebula_mpm_last_error().
 *     No C++ exception crosses this boundary.
 *   - Particle arrays use the reference layout (MPMEngine.cpp:46-53): 8 float4
 *     per particle -- P=(x,Vp), v=(v, material id bits), F0..F2 = columns of F
 *     with the Kirchhoff stress diagonal in w, B0..B2 = APIC B columns with the
 *     stress off-diagonals (xy, xz, yz) in w (mpm_common.glsl:98-122).
 *   - The engine owns its device memory; the caller owns the stream.  Host
 *     setters copy synchronously.  nebula_mpm_step is stream-ordered and does
 *     not synchronize.
 */
#ifndef NEBULA_MPM_H
#define NEBULA_MPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define NEBULA_MPM_OK 0
#define NEBULA_MPM_ERR_INVALID 1     /* bad argument or size */
#define NEBULA_MPM_ERR_CUDA 2        /* a CUDA runtime call failed */
#define NEBULA_MPM_ERR_OOM 3         /* device allocation failed */
#define NEBULA_MPM_ERR_DEVICE 4      /* a kernel raised its error flag (bounded wait expired, non-finite state) */
#define NEBULA_MPM_ERR_UNSUPPORTED 5 /* feature outside this build (e.g. a noise force) */

/* ---------------------------------------------------------------- records */
/* MPMConfig (src/engine/MPMEngine.h:22-55): initial nx*ny*nz lattice, domain
 * size [m], cell size [m], buffer capacity (0 = nx*ny*nz), E, nu, rho0. */
typedef struct nebula_mpm_config {
  uint32_t nx, ny, nz;
  float domainSize[3];
  float cellSize;
  uint32_t maxParticles;
  float E, nu, rho0;
} nebula_mpm_config;

/* MaterialParams (src/core/MaterialParams.h:16-38), 64 bytes. model:
 * 0 ELASTIC (Hencky), 1 VON_MISES, 2 DRUCKER_PRAGER, 3 GRANULAR_POWDER,
 * 4 FLUID, 5 VISCOPLASTIC_MUD; and 6 FIXED_COROTATED, which the reference
 * names (README.md:78) but does not implement: Kirchhoff stress
 * 2 mu (F - R) F^T + lambda (J - 1) J I, R the rotation of F's polar
 * decomposition.  Other values act as ELASTIC. */
typedef struct nebula_mpm_material {
  float mu, lambda, rho0;
  uint32_t model;
  float M_friction, q_cohesion, q_max, bulkK;
  float fluidGamma, viscosity, hardening, xi;
  float pad[4];
} nebula_mpm_material;

/* ColliderPrimitive (src/core/Collider.h:19-29), 64 bytes. type: 0 plane
 * (p, n), 1 sphere (p, radius), 2 box (centre p, half extents n), 3 capsule
 * (start p, axis vector n, radius). */
typedef struct nebula_mpm_collider {
  uint32_t type;
  float px, py, pz;
  float nx, ny, nz;
  float radius;
  float vx, vy, vz;
  float restitution, friction;
  float pad[3];
} nebula_mpm_collider;

/* ForceGPU (src/core/Force.h:27-32), 32 bytes.  Supported types: 0 GRAVITY and
 * 1 CONSTANT_WIND (data[0..2] = direction, data[3] = strength; both add
 * direction*strength*dt to every grid velocity, Force.h:136-141).  affectMask 0
 * or with bit 0 set applies to MPM nodes (typeFlag 0). */
typedef struct nebula_mpm_force {
  uint16_t type, affectMask;
  float data[7];
} nebula_mpm_force;

/* The public tunables of MPMEngine (src/engine/MPMEngine.h:72-80).
 * flip_ratio: 0 PIC, -1 APIC, (0.01, 1] FLIP blend. restitution and
 * wall_friction are carried but read by no substep kernel, as in the reference. */
typedef struct nebula_mpm_params {
  float restitution;
  float wall_friction;
  int32_t numSubsteps;
  uint32_t plasticModel;
  float q_max;
  float M_friction;
  float q_cohesion;
  float flip_ratio;
} nebula_mpm_params;

/* Particle fields for upload/download/device pointers. */
typedef enum nebula_mpm_field {
  NEBULA_MPM_P = 0, NEBULA_MPM_V = 1,
  NEBULA_MPM_F0 = 2, NEBULA_MPM_F1 = 3, NEBULA_MPM_F2 = 4,
  NEBULA_MPM_B0 = 5, NEBULA_MPM_B1 = 6, NEBULA_MPM_B2 = 7
} nebula_mpm_field;

/* Engine-internal counters (for measurement and tests). */
typedef struct nebula_mpm_stats {
  uint64_t substeps;          /* substeps run since create */
  uint32_t live_particles;
  uint32_t active_bricks;     /* 4x4x4-cell grid bricks touched by the last P2G */
  uint32_t particle_bricks;   /* bricks holding particles at the last binning */
  uint32_t grid_res[3];
  uint32_t cube_res;
  uint32_t hash_cells;
  uint64_t kernel_launches;   /* kernels this engine has launched */
  uint32_t overflow_particles;/* particles whose P2G stencil left their block tile (slow path) */
  uint32_t error_flags;       /* device error bits seen at the last check */
  uint64_t graph_launches;    /* steps replayed from a CUDA graph */
} nebula_mpm_stats;

typedef struct nebula_mpm nebula_mpm;

/* ---------------------------------------------------------------- engine (MPMEngine) */
/* MPMEngine::init (MPMEngine.cpp:34-156): allocates state for
 * cfg->maxParticles (or nx*ny*nz) particles and places the default lattice. */
int nebula_mpm_create(const nebula_mpm_config* cfg, nebula_mpm** out);
/* MPMEngine::cleanup (MPMEngine.cpp:160-163). */
int nebula_mpm_destroy(nebula_mpm* e);
const char* nebula_mpm_last_error(void);

/* The public fields of MPMEngine (MPMEngine.h:72-80). */
int nebula_mpm_set_params(nebula_mpm* e, const nebula_mpm_params* p);
int nebula_mpm_get_params(const nebula_mpm* e, nebula_mpm_params* p);

/* MPMEngine::setMaterials (MPMEngine.cpp:239-243): n in [1, 16]; n == 0 is ignored. */
int nebula_mpm_set_materials(nebula_mpm* e, const nebula_mpm_material* mats, uint32_t n);
/* MPMEngine::setParticleMaterialIds (MPMEngine.cpp:245-256): overwrites v with
 * (0, 0, 0, id bits) for particles [0, n). */
int nebula_mpm_set_particle_material_ids(nebula_mpm* e, const uint32_t* ids, uint32_t n);
/* MPMEngine::setColliders / clearAnalyticColliders (MPMEngine.cpp:260-267): n <= 64. */
int nebula_mpm_set_colliders(nebula_mpm* e, const nebula_mpm_collider* c, uint32_t n);
int nebula_mpm_clear_analytic_colliders(nebula_mpm* e);
/* MPMEngine::setColliderSDF (MPMEngine.cpp:204-209): n == hashCells floats,
 * indexed by Morton code, world units, negative inside. */
int nebula_mpm_set_collider_sdf(nebula_mpm* e, const float* morton_sdf, uint64_t n);
/* MPMEngine::setColliderSphere / clearCollider (MPMEngine.cpp:180-202). */
int nebula_mpm_set_collider_sphere(nebula_mpm* e, float radius, float cx, float cy, float cz);
int nebula_mpm_clear_collider(nebula_mpm* e);
/* setColliderSDF(buildMeshSDF(tris, gridRes, hashCells, cellSize)) (MeshSDF.h:98-132):
 * the signed distance of every cell centre to a triangle mesh, built on the
 * GPU into the engine's SDF.  tris: n records of 12 host floats (normal, v0,
 * v1, v2), the binary STL order (loadBinarySTL, MeshSDF.h:22-43). */
int nebula_mpm_set_collider_mesh(nebula_mpm* e, const float* tris, uint32_t n);
/* The moving-obstacle rebuild of examples/pyro_basic.cpp:130-134,
 * setColliderSDF(buildMeshSDF(transformTriangles(tris, t, q), ...)) with
 * transformTriangles (MeshSDF.h:134-141) and the build on the device, from the
 * triangles of the last nebula_mpm_set_collider_mesh: no host transfer.
 * rotation_wxyz: unit quaternion (w, x, y, z). */
int nebula_mpm_set_collider_mesh_pose(nebula_mpm* e, const float translation[3], const float rotation_wxyz[4]);
/* Closest-point definition of the engine's mesh SDF builds, from the next
 * nebula_mpm_set_collider_mesh / _pose on: NEBULA_MPM_CLOSEST_POINT_COMPLETE
 * (default; the complete Voronoi-region test) or
 * NEBULA_MPM_CLOSEST_POINT_REFERENCE (closestPtOnTriangle of MeshSDF.h:48-78
 * step for step, without its edge-BC region, by brute force over the
 * triangles as buildMeshSDF does: the reference's SDF exactly, including its
 * wrong distances and signs where edge BC is closest). */
#define NEBULA_MPM_CLOSEST_POINT_COMPLETE 0
#define NEBULA_MPM_CLOSEST_POINT_REFERENCE 1
int nebula_mpm_set_collider_mesh_closest_point(nebula_mpm* e, int mode);
/* EngineBase::setForces / addForce / clearForces (EngineBase.cpp:22-40):
 * replaces the force table (n <= 16).  No shader is rebuilt: forces are a
 * kernel parameter table. */
int nebula_mpm_set_forces(nebula_mpm* e, const nebula_mpm_force* f, uint32_t n);
/* addForce(GravityForce) as one call (the reference removed its gravity member,
 * MPMEngine.h:57-58): every GRAVITY entry of the table is replaced by one of
 * vector (gx, gy, gz); other forces stay; (0, 0, 0) removes gravity. */
int nebula_mpm_set_gravity(nebula_mpm* e, float gx, float gy, float gz);
/* MPMEngine::appendParticles (MPMEngine.cpp:211-235): pos4=(x,Vp),
 * vel4=(v, id bits); F=I, B=0, stress=0; truncated at capacity.  *appended
 * (may be NULL) receives the count actually added. */
int nebula_mpm_append_particles(nebula_mpm* e, const float* pos4, const float* vel4, uint32_t n, uint32_t* appended);
/* Seeded particle placement of the measurement configurations (no
 * counterpart in the reference, whose init places an unjittered lattice,
 * MPMEngine.cpp:86-137): counts[0] x counts[1] x counts[2] points, x fastest,
 * then z, then y, at origin + index * spacing, each coordinate offset by
 * U(-jitter, +jitter) drawn from the counter-based SplitMix64 stream
 * (seed, stream) in that order (x, y, z of point 0, then of point 1, ...);
 * computed in double, stored as float.  P.w = particleVolume, v = vel,
 * v.w = materialId bits. */
typedef struct nebula_mpm_lattice {
  uint32_t counts[3];
  uint32_t materialId;
  double spacing;
  double origin[3];
  double jitter;
  uint64_t seed;
  uint64_t stream;
  float particleVolume;
  float vel[3];
} nebula_mpm_lattice;
/* The lattice's points on the host: pos4 and vel4 hold 4 * n floats,
 * n = counts[0] * counts[1] * counts[2]. */
int nebula_mpm_lattice_points(const nebula_mpm_lattice* L, float* pos4, float* vel4, uint64_t n);
/* nebula_mpm_append_particles of the lattice's points (truncated at capacity). */
int nebula_mpm_append_lattice(nebula_mpm* e, const nebula_mpm_lattice* L, uint32_t* appended);
/* MPMEngine::resetParticles (MPMEngine.cpp:281-287); also rewinds the emitters. */
int nebula_mpm_reset_particles(nebula_mpm* e);

/* Emitter (src/core/Emitter.h:39-224) as used by MPMEngine::emitFromEmitters
 * (MPMEngine.cpp:289-352).  shape 0 AABB: size = full edge lengths; 1 SPHERE:
 * size[0] = radius; 2 ELLIPSE: size[0] = semi-axis along x, size[1] = along
 * y, z fixed at center[2].  step_count 0 = every step, -1 = first step only,
 * >0 = that many steps.  particleVolume <= 0 takes the config's
 * (domainSize/n)^3 product, as the reference does.
 * At the start of each nebula_mpm_step every due emitter appends
 * min(particles_per_step, capacity - live) particles IN A KERNEL on the step's
 * stream (no host upload, no synchronisation), then moves its centre by
 * center_vel * dt.  Positions and velocity randomness come from a
 * counter-based hash of (seed, emission, particle): the same shapes and
 * distributions as the reference's std::mt19937 sampling, not its numbers. */
typedef struct nebula_mpm_emitter {
  uint32_t shape;
  float center[3];
  float size[3];
  float vel[3];
  float center_vel[3];
  int32_t particles_per_step;
  uint32_t particleType;      /* material id of the emitted particles */
  uint32_t emitAlongNormal;   /* 1: |vel| along the shape's outward normal */
  float velocityRandomness;   /* > 0: + U(-r, r)^3 per particle */
  int32_t step_count;
  float particleVolume;
  uint32_t pad;
} nebula_mpm_emitter;
/* MPMEngine::addEmitter / clearEmitters (MPMEngine.cpp:271-279). */
int nebula_mpm_add_emitter(nebula_mpm* e, const nebula_mpm_emitter* em, uint32_t* index);
int nebula_mpm_clear_emitters(nebula_mpm* e);
/* The emitter's current record (its centre moves with center_vel) and how many times it has emitted. */
int nebula_mpm_get_emitter(const nebula_mpm* e, uint32_t index, nebula_mpm_emitter* em, int32_t* stepsDone);
/* Replace the full state of particles [0, n) (n <= capacity; sets the live
 * count to n) from 8 host float4 arrays in the reference layout (P, v, F0..B2). */
int nebula_mpm_upload_state(nebula_mpm* e, const float* const fields[8], uint32_t n);
/* Copy field `f` of the live particles (original particle order) to host:
 * count = 4 * live floats. */
int nebula_mpm_download(nebula_mpm* e, int field, float* host, uint64_t count);
/* All 8 fields at once (P, v, F0, F1, F2, B0, B1, B2), original particle order,
 * count = 4 * live floats per field; one unpermute and one synchronisation. */
int nebula_mpm_download_state(nebula_mpm* e, float* const host[8], uint64_t count);
/* Streaming state exchange, stream-ordered on `stream` and overlapped with
 * the steps queued before it: the copies run on two engine-owned copy
 * streams through device staging buffers (2 x 128 B per particle of
 * capacity, allocated on first use), one per direction, so a loop of
 *   step(k); download_state_async(k); upload_state_async(k + 1)
 * moves step k's result to the host and step k + 1's input to the device
 * while step k computes.
 * upload_state_async: replaces the state of particles [0, n) like
 * nebula_mpm_upload_state (live count n, original particle order) at this
 * point of `stream`; the host arrays (pinned for the copy to be
 * asynchronous) must stay unchanged until the stream has passed it.
 * download_state_async: copies the state as of this point of `stream` (all 8
 * fields, original order, count = 4 * live floats per field) to the host
 * arrays; they hold it after nebula_mpm_sync, or once `stream` has passed a
 * later nebula_mpm_wait_downloads.
 * wait_downloads: makes `stream` wait for every download queued so far. */
int nebula_mpm_upload_state_async(nebula_mpm* e, const float* const fields[8], uint32_t n, void* stream);
int nebula_mpm_download_state_async(nebula_mpm* e, float* const host[8], uint64_t count, void* stream);
int nebula_mpm_wait_downloads(nebula_mpm* e, void* stream);
/* getPositionBuffer / getVelocityBuffer (MPMEngine.cpp:165-166) for any field:
 * the device array of field `f` (4 * live floats) in the original particle
 * order.  The engine reorders particles during a step, so the pointer is valid
 * until the next call that steps or changes the particles; query it again
 * after each step.  Writes through it (stream-ordered by the caller) are seen
 * by the next step. */
int nebula_mpm_device_ptr(nebula_mpm* e, int field, float** out);
/* MPMEngine::step (MPMEngine.cpp:404-474): numSubsteps substeps of dt/numSubsteps,
 * stream-ordered on `stream` (a cudaStream_t, NULL = legacy default stream).
 * The engine replays the substep loop from CUDA graphs of its own: the second
 * step in a row with the same kernel arguments (substep parameters, buffers,
 * live count, substep count, launch shape) is captured, later ones replay it;
 * a replay launches exactly what the uncaptured loop would.  Emitters and
 * setters run on the host before the loop and change the key where they
 * change an argument.  Off while phase profiling and while `stream` is being
 * captured by the caller.
 * A caller may also capture a step into a graph of its own on a non-NULL
 * stream and replay it when numSubsteps is even (the ping-pong state buffers
 * then end each step in the parity the graph was captured with), after one
 * uncaptured step, and with no emitter due and no setter called between
 * replays (those act on the host side of a step, which a replay does not run). */
int nebula_mpm_step(nebula_mpm* e, float dt, void* stream);
/* Engine-owned graph replays of nebula_mpm_step on (enable != 0, the default)
 * or off (drops the captured graphs). */
int nebula_mpm_set_graphs(nebula_mpm* e, int enable);
/* MPMEngine::liveParticleCount (MPMEngine.h:67). */
int nebula_mpm_live_count(const nebula_mpm* e, uint32_t* n);
int nebula_mpm_get_stats(nebula_mpm* e, nebula_mpm_stats* s);
/* Synchronize the engine's last stream and report device-side error flags. */
int nebula_mpm_sync(nebula_mpm* e);
/* Binning of the current positions in the reference's output format
 * (MPMHarness::buildHashGridCPU, MPMHarness.cpp:132-178): cellCount[hashCells],
 * cellOffset[hashCells] = END of each cell's range, sorted[live] = particle
 * indices, ascending inside each cell.  Host arrays. */
int nebula_mpm_export_bins(nebula_mpm* e, uint32_t* cellCount, uint32_t* cellOffset, uint32_t* sorted);
/* The grid that P2G of the current particle state produces with substep
 * length `dt` (mpm_zero_grid.comp + mpm_p2g.comp), in the reference layout:
 * mom[4*hashCells] (w = 0) and mass[hashCells].  Host arrays.  The particle
 * state is not advanced. */
int nebula_mpm_export_grid(nebula_mpm* e, float dt, float* mom, float* mass);

/* Per-phase device timing (no counterpart in the reference, which has no MPM
 * timers): when enabled, the engine brackets each kernel phase of every
 * substep with CUDA events on the launching stream.  Phases: 0 binning,
 * 1 P2G, 2 grid update, 3 G2P, 4 fused G2P+P2G, 5 other.  Reading synchronizes
 * and returns milliseconds and launch counts accumulated since the last reset. */
#define NEBULA_MPM_PHASES 6
int nebula_mpm_profile_enable(nebula_mpm* e, int enable);
int nebula_mpm_profile_read(nebula_mpm* e, double ms[NEBULA_MPM_PHASES], uint64_t launches[NEBULA_MPM_PHASES], int reset);

/* Substep pipeline (no counterpart in the reference, which always records its
 * eleven dispatches): FUSED (default) keeps particles in 4x4x4-cell brick
 * order and runs grid update, fused G2P+P2G, brick scan and permutation per
 * substep on the bricks particles touch; DENSE runs one kernel per reference
 * dispatch over the whole Morton grid.  Both compute the same substep. */
#define NEBULA_MPM_PIPELINE_DENSE 0
#define NEBULA_MPM_PIPELINE_FUSED 1
int nebula_mpm_set_pipeline(nebula_mpm* e, int pipeline);

/* Launch shape of the per-substep kernels (block and tile sizes), picked per
 * GPU and workload by the project's autotuner (nebula_b200/autotune.py, a
 * JSON cache keyed by GPU and configuration).  fused_threads: CTA size of the
 * fused G2P/P2G kernel (192 or 256; each warp takes 32 slots of the brick per
 * round; 0, the default: 192 for scenes of 65,537 to 524,287 particles, else
 * 256); fused_ctas_per_sm, grid_ctas_per_sm: persistent CTAs per SM of the
 * fused and grid-update kernels (0 = as many as fit; larger values are capped
 * at that); grid_batch: grid nodes per thread per round (2 or 4); fused_split:
 * work items per particle brick of the fused kernel (1-4; 0, the default: 2 for
 * scenes of up to 65,536 particles, else 1):
 * 1 keeps a brick in one CTA, k > 1 cuts its slots into k contiguous parts
 * handled by k CTAs (more parallel items for scenes with few bricks, one
 * staging and one tile flush per item).  Every shape
 * computes the same substep (float sums may associate differently).  No
 * counterpart in the reference (its dispatch sizes are fixed in the shaders). */
typedef struct nebula_mpm_launch_config {
  uint32_t fused_threads;
  uint32_t fused_ctas_per_sm;
  uint32_t grid_ctas_per_sm;
  uint32_t grid_batch;
  uint32_t fused_split;
} nebula_mpm_launch_config;
int nebula_mpm_set_launch_config(nebula_mpm* e, const nebula_mpm_launch_config* c);
int nebula_mpm_get_launch_config(nebula_mpm* e, nebula_mpm_launch_config* c);
/* The most CTAs per SM of each variant on the current device (occupancy):
 * fused_ctas_per_sm[fused_threads == 256], grid_ctas_per_sm[grid_batch == 4];
 * flip / batch select the fused kernel's FLIP and batched instantiations. */
int nebula_mpm_launch_limits(int flip, int batch, uint32_t fused_ctas_per_sm[2], uint32_t grid_ctas_per_sm[2]);
/* Self-test of the failure path of the kernels' waits: one warp of the brick
 * scan's decoupled look-back waits on a predecessor tile that never publishes.
 * The wait is bounded (about a second), so the kernel gives up, sets the
 * scan-timeout bit (1) in *error_bits and returns; the CUDA context stays
 * usable.  No counterpart in the reference. */
int nebula_mpm_probe_wait_expiry(uint32_t* error_bits);
/* The engine's own brick binning of the current positions (FUSED pipeline):
 * *numBricks listed bricks (brick id = cell Morton code >> 6) with the first
 * sorted slot of each (brickStarts has *numBricks + 1 entries, the last = live
 * count), and the original particle index in each sorted slot.  brickIds and
 * brickStarts hold hashCells/64 (+1) entries, sortedPids live entries.  Host arrays. */
int nebula_mpm_export_brick_bins(nebula_mpm* e, uint32_t* numBricks, uint32_t* brickIds, uint32_t* brickStarts, uint32_t* sortedPids);

/* ---------------------------------------------------------------- batched scenes
 * No counterpart in the reference (one MPMEngine holds one scene).  A batch
 * holds many independent scenes, each with the engine's parameter surface,
 * and advances all of them with one set of launches per substep: scenes share
 * one brick space and one particle array, and a step of K substeps is
 * replayed from a CUDA graph captured on first use (when `stream` is not
 * NULL).  Scenes are added before the first step; the layout is fixed after
 * it.  Substep k of a step uses collider set min(k, trackLen-1) of each
 * scene's collider track, which is how a host moves a collider every
 * substep (the reference re-uploads ColliderSet between dispatches). */
typedef struct nebula_mpm_batch nebula_mpm_batch;
typedef struct nebula_mpm_batch_config {
  uint32_t maxScenes;     /* scene table capacity (<= 65536) */
  uint32_t maxParticles;  /* particle capacity over all scenes */
} nebula_mpm_batch_config;
typedef struct nebula_mpm_scene_info {
  uint32_t grid_res[3];
  uint32_t cube_res;
  uint32_t hash_cells;
  uint32_t particles;
  uint32_t first_brick;   /* the scene's bricks in the shared brick space */
  uint32_t bricks;
} nebula_mpm_scene_info;
typedef struct nebula_mpm_batch_stats {
  uint64_t substeps;
  uint32_t scenes;
  uint32_t live_particles;
  uint32_t total_bricks;
  uint32_t active_bricks;     /* grid bricks touched by the last P2G, all scenes */
  uint32_t particle_bricks;   /* bricks holding particles at the last binning */
  uint32_t overflow_particles;
  uint64_t kernel_launches;   /* kernels launched, graph replays included */
  uint64_t graph_launches;
  uint32_t error_flags;
} nebula_mpm_batch_stats;

int nebula_mpm_batch_create(const nebula_mpm_batch_config* cfg, nebula_mpm_batch** out);
int nebula_mpm_batch_destroy(nebula_mpm_batch* b);
/* Adds a scene with domain, cell size, E, nu, rho0 from `cfg` (nx, ny, nz and
 * maxParticles are ignored) and n particles pos4=(x,Vp), vel4=(v, id bits),
 * F=I, B=0 (MPMEngine::appendParticles semantics).  *scene receives its index. */
int nebula_mpm_batch_add_scene(nebula_mpm_batch* b, const nebula_mpm_config* cfg, const float* pos4, const float* vel4, uint32_t n,
                               uint32_t* scene);
/* Per-scene forms of the engine setters above (numSubsteps is ignored: the
 * batch step takes its own count). */
int nebula_mpm_batch_set_params(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_params* p);
int nebula_mpm_batch_get_params(const nebula_mpm_batch* b, uint32_t scene, nebula_mpm_params* p);
int nebula_mpm_batch_set_materials(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_material* mats, uint32_t n);
int nebula_mpm_batch_set_particle_material_ids(nebula_mpm_batch* b, uint32_t scene, const uint32_t* ids, uint32_t n);
int nebula_mpm_batch_set_colliders(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_collider* c, uint32_t n);
/* substeps consecutive sets of perSubstep colliders (perSubstep <= 64). */
int nebula_mpm_batch_set_collider_track(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_collider* c, uint32_t perSubstep,
                                        uint32_t substeps);
int nebula_mpm_batch_set_collider_sdf(nebula_mpm_batch* b, uint32_t scene, const float* morton_sdf, uint64_t n);
int nebula_mpm_batch_clear_collider_sdf(nebula_mpm_batch* b, uint32_t scene);
int nebula_mpm_batch_set_forces(nebula_mpm_batch* b, uint32_t scene, const nebula_mpm_force* f, uint32_t n);
/* Replace the scene's full state (n must equal its particle count). */
int nebula_mpm_batch_upload_state(nebula_mpm_batch* b, uint32_t scene, const float* const fields[8], uint32_t n);
/* Field `field` of the scene's particles in their original order (count = 4 * particles). */
int nebula_mpm_batch_download(nebula_mpm_batch* b, uint32_t scene, int field, float* host, uint64_t count);
/* `substeps` substeps of dt/substeps for every scene, stream-ordered. */
int nebula_mpm_batch_step(nebula_mpm_batch* b, float dt, uint32_t substeps, void* stream);
/* Graph capture and replay of steps (default on); off launches eagerly. */
int nebula_mpm_batch_set_graphs(nebula_mpm_batch* b, int enable);
/* nebula_mpm_set_launch_config for a batch; drops its captured graphs. */
int nebula_mpm_batch_set_launch_config(nebula_mpm_batch* b, const nebula_mpm_launch_config* c);
int nebula_mpm_batch_get_launch_config(nebula_mpm_batch* b, nebula_mpm_launch_config* c);
int nebula_mpm_batch_sync(nebula_mpm_batch* b);
int nebula_mpm_batch_get_stats(nebula_mpm_batch* b, nebula_mpm_batch_stats* s);
int nebula_mpm_batch_scene_info(const nebula_mpm_batch* b, uint32_t scene, nebula_mpm_scene_info* info);

/* Collider track of the single-scene engine: substep k of each later step
 * uses collider set min(k, substeps-1) (same semantics as the batch call);
 * nebula_mpm_set_colliders resets it to one set. */
int nebula_mpm_set_collider_track(nebula_mpm* e, const nebula_mpm_collider* c, uint32_t perSubstep, uint32_t substeps);

/* ---------------------------------------------------------------- differentiable rollout
 * No counterpart in the reference (it has no adjoint).  A rollout of
 * `substeps` substeps of `dt` of an APIC, ELASTIC (Hencky) body with a
 * per-particle Young's modulus (uniform nu and rho0), gravity and the grid
 * wall band, on a dense grid of domainSize / cellSize; the loss is
 * |COM(x_T) - target|^2 with the mass-weighted centre of mass.  backward()
 * returns dL/dv0, dL/dE (and dL/dx0) by a hand-written reverse pass of G2P,
 * grid update and P2G with checkpoints every `checkpointEvery` substeps
 * (float32; the SVD and the Hencky-stress derivative in float64).  Arrays are
 * DEVICE pointers: pos4 = (x, Vp), vel4 = (v, -), E per particle, outputs of
 * the same shapes.  Forward and backward are replayed from CUDA graphs
 * captured on first use when `stream` is not NULL.  Events seen by the last
 * forward (bits: 1 J reset, 2 world clamp, 4 speed cap) make the gradient
 * one of a non-smooth map there. */
typedef struct nebula_mpm_adjoint nebula_mpm_adjoint;
typedef struct nebula_mpm_adjoint_config {
  float domainSize[3];
  float cellSize;
  uint32_t particles;
  uint32_t substeps;
  uint32_t checkpointEvery;
  float dt;
  float gravity[3];
  float nu;
  float rho0;
} nebula_mpm_adjoint_config;
int nebula_mpm_adjoint_create(const nebula_mpm_adjoint_config* cfg, nebula_mpm_adjoint** out);
int nebula_mpm_adjoint_destroy(nebula_mpm_adjoint* a);
/* dLoss (device, 1 float, may be NULL) receives the loss. */
int nebula_mpm_adjoint_forward(nebula_mpm_adjoint* a, const float* dPos4, const float* dVel4, const float* dE, const float target[3],
                               float* dLoss, void* stream);
/* Gradients of lossGrad * L for the inputs of the last forward; NULL outputs are skipped. */
int nebula_mpm_adjoint_backward(nebula_mpm_adjoint* a, float lossGrad, float* dGradVel4, float* dGradE, float* dGradPos4, void* stream);
/* Field `field` of the final state of the last forward, to host (count = 4 * particles). */
int nebula_mpm_adjoint_download(nebula_mpm_adjoint* a, int field, float* host, uint64_t count);
int nebula_mpm_adjoint_events(nebula_mpm_adjoint* a, uint32_t* events);
int nebula_mpm_adjoint_set_graphs(nebula_mpm_adjoint* a, int enable);
int nebula_mpm_adjoint_launches(nebula_mpm_adjoint* a, uint64_t* launches);

/* Domain helpers (src/core/Domain.h:14-39). */
void nebula_mpm_domain_grid_res(const float domainSize[3], float cellSize, uint32_t out[3]);
uint32_t nebula_mpm_domain_cube_res(const uint32_t res[3]);
uint32_t nebula_mpm_domain_hash_cells(const uint32_t res[3]);
uint32_t nebula_mpm_domain_n_groups(uint32_t cells);

/* buildMeshSDF (src/core/MeshSDF.h:98-132) on DEVICE buffers: dSdf[totalCells]
 * (totalCells >= cubeRes^3 of realRes) receives the Morton-ordered signed
 * distances of the cell centres (ix+0.5, iy+0.5, iz+0.5) * cellSize inside
 * realRes, 1e9 elsewhere; dTris: nTris records of 12 floats (normal, v0, v1, v2),
 * 16-byte aligned.  The closest point uses the complete Voronoi-region test
 * (the reference's closestPtOnTriangle, MeshSDF.h:48-78, omits the edge-BC
 * region). */
int nebula_mpm_mesh_sdf(const float* dTris, uint32_t nTris, const uint32_t realRes[3], uint32_t totalCells, float cellSize, float* dSdf,
                        void* stream);
/* A mesh prepared on the device for repeated SDF builds (a moving obstacle):
 * triangles sorted by the Morton code of their centroids and grouped in
 * clusters of 32 with bounding spheres, so that the build culls clusters
 * before triangles.  Same result as nebula_mpm_mesh_sdf on the same list
 * (ties in distance go to the earlier triangle of the list).  tris: n host
 * records of 12 floats (normal, v0, v1, v2).  Used by
 * nebula_mpm_set_collider_mesh / _pose. */
typedef struct nebula_mpm_mesh nebula_mpm_mesh;
int nebula_mpm_mesh_create(const float* tris, uint32_t n, nebula_mpm_mesh** out);
int nebula_mpm_mesh_destroy(nebula_mpm_mesh* m);
/* buildMeshSDF(transformTriangles(tris, translation, rotation), realRes, totalCells, cellSize)
 * into dSdf on `stream`; null translation / rotation = identity. */
int nebula_mpm_mesh_build_sdf(const nebula_mpm_mesh* m, const float translation[3], const float rotation_wxyz[4], const uint32_t realRes[3],
                              uint32_t totalCells, float cellSize, float* dSdf, void* stream);
/* The same of transformTriangles(tris, translation, rotation) (MeshSDF.h:134-141),
 * the pose applied on the device; a null translation or rotation is the identity. */
int nebula_mpm_mesh_sdf_posed(const float* dTris, uint32_t nTris, const float translation[3], const float rotation_wxyz[4],
                              const uint32_t realRes[3], uint32_t totalCells, float cellSize, float* dSdf, void* stream);
/* buildMeshSDF (MeshSDF.h:98-132) with the reference's own closest point
 * (closestPtOnTriangle, MeshSDF.h:48-78, no edge-BC region): every cell
 * visits every triangle, O(cells x triangles), since that point can lie
 * outside the triangle and no distance bound holds for it.  Same arguments
 * and output as nebula_mpm_mesh_sdf_posed (null translation / rotation =
 * identity); the _build_ form takes a prepared mesh, keeping the first-in-
 * list rule for equal distances. */
int nebula_mpm_mesh_sdf_reference(const float* dTris, uint32_t nTris, const float translation[3], const float rotation_wxyz[4],
                                  const uint32_t realRes[3], uint32_t totalCells, float cellSize, float* dSdf, void* stream);
int nebula_mpm_mesh_build_sdf_reference(const nebula_mpm_mesh* m, const float translation[3], const float rotation_wxyz[4],
                                        const uint32_t realRes[3], uint32_t totalCells, float cellSize, float* dSdf, void* stream);

/* ---------------------------------------------------------------- single passes
 * One reference dispatch each, on caller-owned DEVICE buffers in the reference
 * layout, mirroring the per-pass harness (MPMHarness::runP2G / runGridUpdate /
 * runG2P, MPMHarness.cpp:260-282).  `pass` carries the MPMSimPC scalars. */
typedef struct nebula_mpm_pass {
  float dt;
  float cellSize;
  uint32_t gridRes[3];
  uint32_t hashCells;      /* cubeRes^3 */
  float worldMin[3];
  float worldMax[3];
  float flip_ratio;
  uint32_t particleCount;
  uint32_t materialCount;  /* 0 = use the global fallbacks below */
  uint32_t colliderCount;
  uint32_t forceCount;
  float mu_lame, lambda_lame, rho0, M_friction, q_cohesion, q_max;
  uint32_t plasticModel;
} nebula_mpm_pass;

/* Particle state: 8 device float4 arrays (P, v, F0, F1, F2, B0, B1, B2). */
typedef struct nebula_mpm_particles {
  float* f[8];
} nebula_mpm_particles;

/* zero_cells + mpm_hash_count + scan + mpm_hash_sort (zero_cells.comp,
 * mpm_hash_count.comp, hash_scan_*.comp, hash_add_base.comp, mpm_hash_sort.comp):
 * cellCount[hashCells], cellOffset[hashCells] (range END), sorted[particleCount]
 * ascending inside each cell.  Uses a caller-visible workspace from
 * nebula_mpm_bin_workspace_size(). */
size_t nebula_mpm_bin_workspace_size(uint32_t hashCells, uint32_t particleCount);
int nebula_mpm_bin(const nebula_mpm_pass* pass, const float* dPos4, uint32_t* dCellCount, uint32_t* dCellOffset, uint32_t* dSorted,
                   void* dWorkspace, size_t workspaceBytes, void* stream);
/* Error word of the last nebula_mpm_bin (or nebula_hash_bin) that used this
 * workspace, read on `stream` (the call synchronizes it): *errorBits = 0 and
 * NEBULA_MPM_OK when the binning ran clean; otherwise the bits (1: a bounded
 * look-back wait of the scan expired, 8: a binning index fell outside the
 * particle range, which follows an expired wait) and NEBULA_MPM_ERR_DEVICE.
 * hashCells / particleCount are those of the binning call.  The bits stay in
 * the workspace until the next binning call clears them.  The reference
 * reports nothing from its binning dispatches (MPMEngine.cpp:423-456). */
int nebula_mpm_bin_status(const void* dWorkspace, size_t workspaceBytes, uint32_t hashCells, uint32_t particleCount, uint32_t* errorBits,
                          void* stream);
/* Self-test of that failure path on a caller workspace: one CTA of the
 * binning scan runs as tile 1 against a tile 0 that never publishes, so its
 * bounded look-back (about a second) gives up and sets bit 1 in the
 * workspace's error word, which nebula_mpm_bin_status then returns.  Reads
 * dCellCount[0, hashCells) and writes only workspace words; needs hashCells
 * >= 4096.  No counterpart in the reference. */
int nebula_mpm_bin_probe_wait_expiry(const nebula_mpm_pass* pass, const uint32_t* dCellCount, void* dWorkspace, size_t workspaceBytes,
                                     void* stream);
/* Same outputs as nebula_mpm_bin, for callers that cannot allocate device
 * memory or hand over a workspace: a foreign-function binding that holds only
 * the three output arrays, or a frame loop that must not call cudaMalloc
 * (which may synchronize the whole device) between frames.  The scratch is a
 * fixed file-scope device array inside the library, held by every GPU that
 * loads it until the process exits: hashCells <=
 * nebula_mpm_bin_noalloc_max_cells() = 2^21 (128^3) and particleCount <=
 * nebula_mpm_bin_noalloc_max_particles() = 2^18; larger sizes return
 * NEBULA_MPM_ERR_INVALID.  No device memory is allocated.  The first call in
 * each CUDA context (with its device current) looks up the array's address;
 * make it before any stream capture.  Every call clears what it needs on the
 * stream.  Calls on one device share the scratch, so calls that can overlap
 * in time race and must be ordered by the caller.  No counterpart in the
 * reference. */
size_t nebula_mpm_bin_noalloc_max_cells(void);
size_t nebula_mpm_bin_noalloc_max_particles(void);
int nebula_mpm_bin_noalloc(const nebula_mpm_pass* pass, const float* dPos4, uint32_t* dCellCount, uint32_t* dCellOffset, uint32_t* dSorted,
                           void* stream);
/* Error word of the last nebula_mpm_bin_noalloc on the current device, read
 * on `stream` (synchronized): the bits and status codes of
 * nebula_mpm_bin_status.  Allocates nothing.  No counterpart in the reference. */
int nebula_mpm_bin_noalloc_status(uint32_t* errorBits, void* stream);
/* nebula_mpm_bin_probe_wait_expiry on the library-held scratch (hashCells >=
 * 4096 and within the limits above); read the result with
 * nebula_mpm_bin_noalloc_status.  Allocates nothing.  No counterpart in the
 * reference. */
int nebula_mpm_bin_noalloc_probe_wait_expiry(const nebula_mpm_pass* pass, const uint32_t* dCellCount, void* stream);
/* mpm_zero_grid.comp + mpm_p2g.comp: writes gridMom[0, hashCells) (w = 0) and
 * gridMass; clears gridMom[hashCells, 2 hashCells). */
int nebula_mpm_p2g(const nebula_mpm_pass* pass, const nebula_mpm_particles* parts, const uint32_t* dCellCount, const uint32_t* dCellOffset,
                   const uint32_t* dSorted, const nebula_mpm_material* dMaterials, float* dGridMom, float* dGridMass, void* stream);
/* mpm_grid_update.comp (+ forces, walls, analytic colliders) and, when dSdf is
 * non-NULL, mpm_nanovdb_bc.comp, fused per node. */
int nebula_mpm_grid_update(const nebula_mpm_pass* pass, float* dGridMom, const float* dGridMass, const nebula_mpm_collider* dColliders,
                           const nebula_mpm_force* dForces, const float* dSdf, void* stream);
/* mpm_g2p.comp: gather, F update, return maps, stress, position update. */
int nebula_mpm_g2p(const nebula_mpm_pass* pass, const nebula_mpm_particles* parts, const float* dGridMom, const float* dGridMass,
                   const nebula_mpm_material* dMaterials, const float* dSdf, void* stream);

/* ---------------------------------------------------------------- PBF spatial hash
 * The same counting sort serving the PBF fluid engine's neighbour search:
 * zero_cells + hash_count + hash_scan_local/global + hash_add_base + hash_sort
 * (shaders/hash_count.comp, hash_scan_*.comp, hash_add_base.comp,
 * hash_sort.comp; dispatched by FluidEngine.cpp:445-474 and
 * tests/helpers/PBFHarness.cpp:153-180).  Cell of a particle = Morton code of
 * clamp((predP.xyz - worldMin) / cellSize, 0, gridRes - 1) truncated
 * (common.glsl:100-105).  Particles whose typeFlag is 6 (TYPE_FLAG_UNUSED,
 * empty boundary slots) are left out (hash_count.comp:9-16,
 * hash_sort.comp:14-17); dTypeFlag may be NULL (nothing left out).
 * Outputs, in the state the pbf_* shaders read them: cellCount[hashCells];
 * cellOffset[hashCells] = END of each cell's range (hash_sort consumes the
 * exclusive offsets, so readers take start = cellOffset - cellCount,
 * pbf_density.comp:50-51); sortedIdx[0, m) the m included particles, in
 * ascending index inside each cell (the shader's order is that of its
 * atomics); sortedIdx[m, particleCount) is not written.  The scan covers any
 * hashCells (hash_scan_global.comp handles at most 1,024 group sums). */
typedef struct nebula_hash_grid {
  float worldMin[3];
  float cellSize;
  uint32_t gridRes[3];
  uint32_t hashCells; /* >= cubeRes^3 of gridRes */
} nebula_hash_grid;
size_t nebula_hash_bin_workspace_size(uint32_t hashCells, uint32_t particleCount);
int nebula_hash_bin(const nebula_hash_grid* grid, const float* dPredP4, const uint32_t* dTypeFlag, uint32_t particleCount,
                    uint32_t* dCellCount, uint32_t* dCellOffset, uint32_t* dSortedIdx, void* dWorkspace, size_t workspaceBytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NEBULA_MPM_H */
