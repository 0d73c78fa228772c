/*
 * solunar_fluid.h -- C ABI of the B200 particle-fluid library.
 *
 * This is the drop-in boundary for solunar's particle fluid (`FluidWorld`, src/fluid in
 * SkuldNorniern/solunar).  The reference has no FFI of its own: its interface is the Rust
 * public API re-exported at src/lib.rs:53-57.  Every entry point below names the Rust
 * item it replaces (file:line, relative to the reference project).
 *
 * Conventions
 *  - Every call returns an int32_t status: SLF_OK or one of the SLF_ERR_* codes.  Codes 1..5
 *    are the PhysicsError variants the fluid uses (src/error.rs:5-22).
 *  - Handles are opaque.  The library owns all device memory; callers own host buffers.
 *  - Calls on one handle must not overlap (the Rust methods take `&mut self`).  Each handle
 *    issues its work on one CUDA stream of its own and returns when that work is done.
 *  - Vectors are passed as `float[3]` (x, y, z); arrays of vectors are packed xyz triples.
 *  - On error the particles are left as the last finished substep put them
 *    (src/fluid/step.rs:55-57).
 *  - There is no host job dispatcher: the `&dyn JobDispatch` argument of the Rust methods
 *    (src/dispatch.rs:1-7) has no counterpart, the GPU is the dispatcher.
 */
#ifndef SOLUNAR_FLUID_H
#define SOLUNAR_FLUID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
enum {
    SLF_OK = 0,
    SLF_ERR_INVALID_SETTINGS = 1,    /* PhysicsError::InvalidSettings (src/error.rs:11) */
    SLF_ERR_NON_FINITE = 2,          /* PhysicsError::NonFinite(_) (src/error.rs:9) */
    SLF_ERR_OUT_OF_RANGE = 3,        /* PhysicsError::OutOfRange (src/error.rs:14) */
    SLF_ERR_FLUID_FULL = 4,          /* PhysicsError::FluidFull (src/error.rs:21) */
    SLF_ERR_DISPATCH_INCOMPLETE = 5, /* PhysicsError::DispatchIncomplete (src/error.rs:15) */
    SLF_ERR_UNSUPPORTED = 6,         /* a combination not built: FAST arithmetic with terrain or bodies,
                                      * cell-relative positions with EXACT arithmetic, a tape with
                                      * dynamic bodies or with bodies and checkpoints, terrain
                                      * added while a tape records, shallow water */
    SLF_ERR_CUDA = 7,                /* a CUDA call failed; see slf_last_error() */
    SLF_ERR_TIMEOUT = 8,             /* a bounded device loop gave up */
    SLF_ERR_INVALID_ARGUMENT = 9,    /* null pointer or wrong buffer size */
    SLF_ERR_SNAPSHOT = 10,           /* SnapshotError (src/snapshot/mod.rs:56-63); see slf_last_error() */
    SLF_ERR_INVALID_SHAPE = 11       /* PhysicsError::InvalidShape (src/error.rs:10) */
};

/* FluidSolver (src/fluid/mod.rs:43-53). */
enum { SLF_SOLVER_WCSPH = 0, SLF_SOLVER_DFSPH = 1 };

/* How particle positions are held on the device.  ABSOLUTE follows the reference's f32
 * arithmetic; CELL_RELATIVE keeps each position as an offset from the origin of its grid
 * cell, so neighbour offsets do not lose bits to the magnitude of the coordinates. */
enum { SLF_POSITIONS_ABSOLUTE = 0, SLF_POSITIONS_CELL_RELATIVE = 1 };

/* EXACT rounds every operation as the reference's scalar f32 code does (no fused
 * multiply-add, IEEE division and square root), so results match the CPU restatement bit
 * for bit.  FAST lets the compiler fuse and uses reciprocal forms inside the pair loops. */
enum { SLF_ARITHMETIC_EXACT = 0, SLF_ARITHMETIC_FAST = 1 };

/* FluidSettings (src/fluid/mod.rs:55-78) followed by this library's own fields.  Defaults
 * come from slf_settings_default() and equal FluidSettings::default (mod.rs:80-95) and the
 * DFSPH constants (src/fluid/dfsph.rs:8-16). */
typedef struct slf_settings {
    int32_t solver;          /* SLF_SOLVER_* */
    float spacing;           /* m between particles at rest */
    float rest_density;      /* kg/m^3 */
    float support;           /* kernel reach as a multiple of spacing, 1.5..4.0 */
    uint64_t max_particles;
    float sound_speed;       /* m/s */
    float viscosity;
    float gravity[3];        /* m/s^2 */
    float courant;           /* share of the kernel radius a particle may move a substep */
    uint32_t max_substeps;
    /* library fields (the reference hard-codes these) */
    int32_t positions;             /* SLF_POSITIONS_*, default ABSOLUTE */
    int32_t arithmetic;            /* SLF_ARITHMETIC_*, default EXACT */
    int32_t warm_start;            /* 1: each DFSPH solve starts with one push at half the stiffness
                                    * impulse (sum of kappa dt) the particle's solve of the same kind
                                    * applied the substep before (dfsph.rs cold-starts: 0, the
                                    * default).  Snapshots do not carry it: a loaded world starts
                                    * cold.  Not with slf_tape_begin. */
    float divergence_tolerance;    /* dfsph.rs:11, 1e-3 */
    float density_tolerance;       /* dfsph.rs:9, 5e-4 */
    uint32_t min_iterations;       /* dfsph.rs:12, 2 */
    uint32_t max_iterations;       /* dfsph.rs:13, 100 */
    int32_t device;                /* CUDA device ordinal of the world, 0 */
} slf_settings;

/* FluidReport (src/fluid/step.rs:27-49). */
typedef struct slf_report {
    uint32_t substeps;
    int32_t capped;
    float max_compression;
    float max_speed;
    uint32_t held_back;
    uint32_t iterations;
    uint32_t emitted;
    uint32_t drained;
    uint32_t lost;
    float sound_speed;
} slf_report;

typedef struct slf_world slf_world;

/* ---- settings and lifetime --------------------------------------------------------- */

/* FluidSettings::default (src/fluid/mod.rs:80-95). */
int32_t slf_settings_default(slf_settings* out);

/* FluidWorld::new (src/fluid/mod.rs:344); FluidSettings::validate (mod.rs:98-117).  Fails
 * with SLF_ERR_INVALID_SETTINGS on settings out of range, SLF_ERR_CUDA without a device. */
int32_t slf_create(const slf_settings* settings, slf_world** out);

/* Drop of FluidWorld.  Null is ignored. */
void slf_destroy(slf_world* world);

/* FluidWorld::settings (mod.rs:372). */
int32_t slf_get_settings(const slf_world* world, slf_settings* out);

/* FluidWorld::particle_mass (mod.rs:380). */
int32_t slf_particle_mass(const slf_world* world, float* out);

/* FluidWorld::kernel (mod.rs:376): the Wendland C2 kernel's radius and scale (mod.rs:125-138). */
int32_t slf_kernel(const slf_world* world, float* radius, float* scale);

/* FluidWorld::len (mod.rs:384). */
int32_t slf_len(const slf_world* world, uint64_t* out);

/* ---- particles, walls, domain ------------------------------------------------------ */

/* FluidWorld::add_particle (mod.rs:412-426). */
int32_t slf_add_particle(slf_world* world, const float position[3], const float velocity[3],
                         uint32_t* id_out);

/* n calls of FluidWorld::add_particle, all or none: every value is checked first.  ids_out
 * may be null. */
int32_t slf_add_particles(slf_world* world, uint64_t n, const float* positions,
                          const float* velocities, uint32_t* ids_out);

/* FluidWorld::fill_box (mod.rs:493-524). */
int32_t slf_fill_box(slf_world* world, const float low[3], const float high[3],
                     uint64_t* count_out);

/* FluidWorld::set_domain (mod.rs:433-444).  low == high == NULL clears the domain. */
int32_t slf_set_domain(slf_world* world, const float* low, const float* high);

/* FluidWorld::add_box_container (src/fluid/boundary.rs:41-68). */
int32_t slf_add_box_container(slf_world* world, const float low[3], const float high[3],
                              uint32_t* boundary_out);

/* FluidWorld::add_wall (boundary.rs:74-91). */
int32_t slf_add_wall(slf_world* world, const float low[3], const float high[3],
                     uint32_t* boundary_out);

/* FluidWorld::remove_boundary (boundary.rs:94-115).  *removed = 0 for an unknown id. */
int32_t slf_remove_boundary(slf_world* world, uint32_t boundary, int32_t* removed);

/* FluidWorld::save_snapshot (src/fluid/save.rs:18-73): the SLFL version 3 bytes of the world.
 * *size receives the byte count; out = NULL asks for the size only, else capacity >= *size. */
int32_t slf_save_snapshot(slf_world* world, uint8_t* out, uint64_t capacity, uint64_t* size);
/* FluidWorld::load_snapshot (save.rs:79-181): a new world from untrusted snapshot bytes
 * (versions 1-3).  The library's own settings fields (positions, arithmetic, solver limits,
 * device) come from `library`, or the defaults when it is NULL.  Bad bytes return
 * SLF_ERR_SNAPSHOT with the reference's message in slf_last_error().  Coupled bodies come back
 * with their points and probes (couple.rs:58-75). */
int32_t slf_load_snapshot(const uint8_t* data, uint64_t size, const slf_settings* library, slf_world** out);

/* ---- coupled bodies (src/fluid/couple.rs, lift.rs) ---------------------------------------
 * The caller owns the rigid bodies.  A body is named by the reference's BodyHandle::to_raw()
 * pair (index, generation) as index << 32 | generation, which orders bodies as the reference
 * does.  Each step the caller gives every coupled body's pose and gets back what the water did to
 * it, to apply to its body as force and torque (impulse / dt) over the rigid step that follows. */
enum { SLF_SHAPE_CUBOID = 0, SLF_SHAPE_SPHERE = 1, SLF_SHAPE_CAPSULE = 2 };

/* SubstepPose (src/substep.rs) as FluidWorld::step_with_bodies reads it (couple.rs:418-426). */
typedef struct slf_body_pose {
    uint64_t body;
    double position[3];          /* the rigid world's f64 position; the water uses it as f32 */
    float rotation[4];           /* unit quaternion x, y, z, w */
    float linear_velocity[3];
    float angular_velocity[3];
    int32_t dynamic;             /* 1: the body takes pushes (apply_force succeeds in the reference) */
} slf_body_pose;

/* What the water did to one coupled body over a step. */
typedef struct slf_body_push {
    uint64_t body;
    float lift[3];               /* lift.rs: buoyancy, drag and wave damping, impulse over the step */
    float lift_angular[3];       /* its angular impulse about the body's centre */
    float damping[3];            /* couple.rs:375-416: the body points' damping, impulse */
    float damping_angular[3];
    int32_t lifted;              /* 1: the body is dynamic and the water lost the lift's momentum */
} slf_body_push;

/* FluidWorld::couple (couple.rs:165-200): shape SLF_SHAPE_CUBOID with dims = half extents,
 * SPHERE with dims[0] = radius, CAPSULE with dims[0] = radius and dims[1] = half height.  A
 * body coupled again takes the new shape.  SLF_ERR_INVALID_SHAPE for a bad shape or one too
 * small to hold a point, SLF_ERR_FLUID_FULL past max_particles points. */
int32_t slf_couple(slf_world* world, uint64_t body, int32_t shape, const float dims[3]);
/* FluidWorld::uncouple (couple.rs:203-207): *removed = 0 for a body that was not coupled. */
int32_t slf_uncouple(slf_world* world, uint64_t body, int32_t* removed);
/* The coupled bodies in body order with their point and probe counts; *count receives how many
 * there are, arrays (any may be NULL) hold at most `capacity`. */
int32_t slf_coupled(const slf_world* world, uint64_t* bodies, uint32_t* points, uint32_t* probes,
                    uint64_t capacity, uint64_t* count);
/* FluidWorld::step_with_bodies (couple.rs:219-248) with the rigid world left to the caller: the
 * coupled bodies stand where `poses` puts them (a coupled body without a pose is uncoupled, as
 * the reference drops bodies gone from the world) and sweep on at their velocities through the
 * substeps; `pushes` (room for `capacity`) receives one entry per coupled body, in body order,
 * and *count how many.  A dynamic body's lift is taken out of the water it was read from.  WCSPH
 * only (SLF_ERR_INVALID_SETTINGS for DFSPH with coupled bodies) and EXACT arithmetic only
 * (SLF_ERR_UNSUPPORTED for FAST). */
int32_t slf_step_with_bodies(slf_world* world, float dt, const slf_body_pose* poses, uint64_t npose,
                             slf_report* out, slf_body_push* pushes, uint64_t capacity, uint64_t* count);

/* The node lattice of a terrain region over [low, high] (terrain.rs:275-283): nodes[a] nodes along
 * axis a, spacing / 2 apart from `low`.  SLF_ERR_FLUID_FULL above 2^24 nodes. */
int32_t slf_terrain_nodes(const slf_world* world, const float low[3], const float high[3], uint64_t nodes[3]);
/* FluidWorld::add_terrain (terrain.rs:262-302): ground under a signed distance field (positive in
 * the open) inside the box.  The reference samples an SDF volume at the nodes; here the caller
 * passes those samples: distances[(y * nodes[2] + z) * nodes[0] + x] at low + (x, y, z) spacing/2,
 * count = the number of nodes.  WCSPH worlds with EXACT arithmetic; a DFSPH step with terrain
 * fails with SLF_ERR_INVALID_SETTINGS, as in the reference.  Removed by slf_remove_boundary. */
int32_t slf_add_terrain(slf_world* world, const float low[3], const float high[3], const float* distances,
                        uint64_t count, uint32_t* boundary_out);

/* FluidWorld::add_emitter (flow.rs:86-99): after each step every lattice slot of the box with
 * no water within 0.9 spacing of its centre gets a particle moving at `velocity`.  Boxes of more
 * than 2^30 slots are refused when the step runs them (SLF_ERR_OUT_OF_RANGE). */
int32_t slf_add_emitter(slf_world* world, const float low[3], const float high[3], const float velocity[3],
                        uint32_t* flow_out);
/* FluidWorld::add_drain (flow.rs:104-106): after each step the water in the box is taken out. */
int32_t slf_add_drain(slf_world* world, const float low[3], const float high[3], uint32_t* flow_out);
/* FluidWorld::remove_flow (flow.rs:109-113): *removed = 0 for an id that is not there. */
int32_t slf_remove_flow(slf_world* world, uint32_t flow, int32_t* removed);

/* FluidWorld::wall_positions (boundary.rs:118-120): count, then xyz triples in wall order. */
int32_t slf_wall_count(const slf_world* world, uint64_t* out);
int32_t slf_read_wall_positions(const slf_world* world, float* out, uint64_t n);

/* ---- the step ------------------------------------------------------------------------ */

/* FluidWorld::step (src/fluid/step.rs:58-90): as many WCSPH substeps as the flow needs
 * (step.rs:102-224) or DFSPH substeps (src/fluid/dfsph.rs:46-103). */
int32_t slf_step(slf_world* world, float dt, slf_report* out);

/* FluidWorld::update_neighbors (mod.rs:540-608): sorts particles by cell then id. */
int32_t slf_update_neighbors(slf_world* world);

/* FluidWorld::compute_densities (mod.rs:621-675).  SLF_ERR_OUT_OF_RANGE when particles were
 * added since the last slf_update_neighbors. */
int32_t slf_compute_densities(slf_world* world);

/* ---- read-outs (arrays in the current particle order) ------------------------------ */

/* FluidWorld::ids (mod.rs:393), positions (:397), velocities (:401), densities (:406).
 * n must equal slf_len(). */
int32_t slf_read_ids(const slf_world* world, uint32_t* out, uint64_t n);
int32_t slf_read_positions(const slf_world* world, float* out, uint64_t n);
int32_t slf_read_velocities(const slf_world* world, float* out, uint64_t n);
/* Positions and velocities together (xyz triples each), with one wait for the device. */
int32_t slf_read_state(const slf_world* world, float* positions, float* velocities, uint64_t n);
int32_t slf_read_densities(const slf_world* world, float* out, uint64_t n);

/* FluidWorld::neighbors_of (mod.rs:612-614) for every particle at once, as the lists the
 * last slf_update_neighbors would build (mod.rs:279-308): start[n+1] and items.  Call with
 * items == NULL to learn *items_len.  start may be NULL. */
int32_t slf_neighbor_lists(slf_world* world, uint32_t* start, uint64_t start_len,
                           uint32_t* items, uint64_t items_capacity, uint64_t* items_len);

/* The wall lists of the same pass (`wall_neighbors`, mod.rs:327), indexes into the wall
 * order of slf_read_wall_positions. */
int32_t slf_wall_neighbor_lists(slf_world* world, uint32_t* start, uint64_t start_len,
                                uint32_t* items, uint64_t items_capacity, uint64_t* items_len);

/* FluidWorld::state_hash (mod.rs:677-691), FNV-1a (src/snapshot/bytes.rs:6-13). */
int32_t slf_state_hash(const slf_world* world, uint64_t* out);

/* Overwrites the positions and velocities of the current particles, in the current order (the
 * arrays FluidWorld::positions / velocities expose, mod.rs:397-403).  n must equal slf_len().
 * A host that owns the particle arrays uploads them with this before a step.  A non finite
 * value (found on the device as the arrays unpack) returns SLF_ERR_NON_FINITE and leaves the
 * world's state as it was. */
int32_t slf_write_state(slf_world* world, const float* positions, const float* velocities,
                        uint64_t n);

/* The CUDA stream (a cudaStream_t) the world issues its work on, for callers that order their
 * own work or events after a step. */
int32_t slf_get_stream(const slf_world* world, void** stream);

/* Message of the last failed call on any handle of this thread ("" if none). */
const char* slf_last_error(void);

/* ---- the adjoint (no counterpart in the reference, which has no gradients) -------------- */

/* Gradients of a loss with respect to the settings, accumulated over the taped steps. */
typedef struct slf_param_grads {
    double viscosity;    /* dL / d settings.viscosity */
    double sound_speed;  /* dL / d settings.sound_speed: Tait stiffness and both viscosities */
    double gravity[3];   /* dL / d settings.gravity */
} slf_param_grads;

/* Starts recording the steps that follow for slf_step_backward.  The number of particles must not
 * change while recording.
 *
 * checkpoint_every = k > 0 (segment checkpointing): the current state is the first checkpoint and
 * the state before every k-th substep is kept too, 36 bytes per particle each (44 with warm
 * starts: the two solver impulses).  The backward pass runs each segment of k substeps forward
 * again from its checkpoint, recording it, so it holds one segment's records at a time however
 * many substeps the flow makes a step take.  When a segment's worth fits in half the device's
 * free memory, its records also keep each substep's neighbour lists, so the backward does not run
 * the substep a third time: WCSPH about 16 bytes per particle per list slot, reserved by this
 * call; DFSPH 48 with the EXACT kept gradients (about 3.2 GB a substep at a million particles),
 * taken by the first backward that keeps, which it does on tapes of at least 32 segments or
 * with solve graphs off (slf_solver_graphs 0).  Otherwise the backward runs each of the
 * segment's substeps (DFSPH: its sort and densities) once more before its adjoint.
 *
 * checkpoint_every = 0: every substep keeps the state before it and its solver record (the rates
 * and velocities of each DFSPH iteration), about 68 + 20 x iterations bytes per particle per
 * substep (8 more with warm starts); the backward pass redoes only each substep's sort and
 * densities.
 *
 * Taken: WCSPH and DFSPH, absolute or cell-relative positions (cell-relative checkpoints and
 * records add the 16-byte cell of each particle); WCSPH with terrain (its density, push, damping
 * and contact; terrain added while recording is UNSUPPORTED); WCSPH with coupled bodies on the
 * caller's paths, checkpoint_every 0 only (each substep's forward is kept as it runs, since the
 * body points' order follows their history); DFSPH with warm_start (checkpoints and records keep
 * each particle's two impulses, 8 bytes, and the backward pass carries their adjoint from substep
 * to substep).  UNSUPPORTED: dynamic bodies (whose lift gives momentum back to the water), bodies
 * with checkpoints. */
int32_t slf_tape_begin(slf_world* world, uint32_t checkpoint_every);
/* Stops recording.  The tape's device buffers (substep records, checkpoints) stay with the world
 * and are reused by the next tape, so the rounds of an optimisation loop record without
 * allocating; slf_destroy frees them. */
int32_t slf_tape_end(slf_world* world);
/* Reverse pass over every step recorded since slf_tape_begin.  dpositions, dvelocities: dL/d of
 * the current positions and velocities (xyz triples, current order, n = slf_len()).  Writes
 * dL/d of the positions and velocities at slf_tape_begin, in the order they had then, and the
 * parameter gradients.  Neighbour lists are the forward's, fixed within each substep; substep
 * lengths and DFSPH solver iteration counts are those the forward took.  The world's state is
 * left as it was. */
int32_t slf_step_backward(slf_world* world, const float* dpositions, const float* dvelocities, uint64_t n,
                          float* dpositions0, float* dvelocities0, slf_param_grads* out);

/* ---- sorting without allocation ---------------------------------------------------------- */

/* No counterpart in the reference: the cell sort of slf_update_neighbors for callers that
 * cannot allocate device memory (an engine that hands out all GPU memory from its own pool, a
 * plugin that only receives buffers from its host).  It allocates nothing: its scratch is one
 * fixed array in device memory, about 7.4 MB, that every GPU which loads this library holds
 * until the process exits.
 *
 * positions: n packed xyz float triples and ids: n ids, both in device memory; radius: the
 * cell size (the kernel radius, spacing * support).  order (device, n entries) receives, for
 * each place k of the (cell, id) order of update_neighbors (src/fluid/mod.rs:541-550), the
 * input index of the particle found there.  At most 262,144 particles whose bounding box spans
 * at most 1,048,576 cells: larger calls fail with SLF_ERR_OUT_OF_RANGE, and so do particles whose
 * cells saturate the i32 range (positions far beyond radius * 2^31).  Ids should be distinct, as
 * a world's are; repeated ids still give a permutation, in no particular order among themselves.
 * Ranking within a cell compares each particle with the cell's others, so a cell holding k
 * particles costs k^2 work: a call whose particles crowd into a few cells (a radius far larger
 * than their spacing) runs long, up to seconds at the particle limit.  The call runs on
 * `stream` (a cudaStream_t; NULL for the default stream) and waits for it before returning.
 * The first call on a device looks up the scratch array's address there, so make that first
 * call before any stream capture.  All calls share the one array and it keeps the last call's
 * contents (the call clears what must start at zero); calls whose work overlaps on the GPU
 * race on it. */
int32_t slf_sort_by_cell_noalloc(const float* positions, const uint32_t* ids, uint64_t n, float radius,
                                 uint32_t* order, void* stream);

/* ---- diagnostics and testing ------------------------------------------------------------ */

/* Per-kernel device time.  While profiling is on, every launch of the world is bracketed by
 * CUDA events on its stream; entries accumulate launches, milliseconds and the algorithmic
 * bytes each launch must move (one read or write of each particle field it touches). */
typedef struct slf_profile_entry {
    char name[32];
    uint64_t launches;
    double milliseconds;
    double algorithmic_bytes;
} slf_profile_entry;

int32_t slf_profile_enable(slf_world* world, int32_t on);
/* Copies up to `capacity` entries; *count receives how many exist.  Resets nothing. */
int32_t slf_profile_read(slf_world* world, slf_profile_entry* out, uint32_t capacity,
                         uint32_t* count);
int32_t slf_profile_reset(slf_world* world);

/* Kernels this process has run through the library so far (a solve run as a CUDA graph counts
 * the kernels its loop ran). */
int32_t slf_kernel_launches(uint64_t* out);

/* How a step without recorded solves or a profile launches its work.  mode = 2 (the default):
 * each substep is one CUDA graph launch (sort and density; DFSPH: both solves with loops the
 * device ends, viscosity, advance; WCSPH: the force and advance pass), recorded when its launches
 * first occur and cached (once recorded graphs go unused, as when the particle count changes every
 * tick, only launches that recur are recorded); substeps with terrain or coupled bodies, and those
 * the cache does not hold, run as in mode 1.  mode = 1: each DFSPH solve is one graph launch, the
 * rest is launched eagerly.  mode = 0: the solves' launches are queued in batches with a host
 * check between them.  In every mode the host waits once a substep and the results are the same
 * bit for bit; the profiler and recorded solves take the batched launches.  Other modes:
 * SLF_ERR_INVALID_SETTINGS. */
int32_t slf_solver_graphs(slf_world* world, int32_t mode);

/* Substeps this world has run as one whole-substep graph launch (mode 2). */
int32_t slf_graph_substeps(const slf_world* world, uint64_t* out);

/* DFSPH solver iterations of the last substep: divergence and density (the per-solve split of
 * FluidReport::iterations, src/fluid/dfsph.rs:89,100). */
int32_t slf_last_iterations(const slf_world* world, uint32_t* divergence, uint32_t* density);

/* Fault injection, the counterpart of the reference's `SkipsJobs` test dispatcher
 * (src/dispatch.rs:50-65): the next sort leaves the 512-particle job `job` undone, which the
 * completeness check reports as SLF_ERR_DISPATCH_INCOMPLETE with the particles untouched. */
int32_t slf_debug_skip_job(slf_world* world, int64_t job);

/* Test hook: sets the neighbour lists' room to `room` entries a particle (rounded down to a
 * multiple of 8, at least 8), so that the next substep's lists outgrow it and the substep is run
 * again with room for its longest list, from the committed state.  Invalidates the lists. */
int32_t slf_debug_list_room(slf_world* world, uint32_t room);

#ifdef __cplusplus
}
#endif

#endif /* SOLUNAR_FLUID_H */
