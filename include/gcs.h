/*
 * gcs.h - C ABI of the B200 Barnes-Hut engine ("gcs" = galaxy collision
 * simulator).
 *
 * This is the boundary a foreign caller binds (ctypes, cgo, JNI ...).  The
 * reference exposes its GPU engine as C++ functions over file-scope globals
 * (cuda_engine.h:5-32 of lakshya076/Galaxy-Collision-Simulator); those exact
 * C++ signatures are kept in include/cuda_engine.h as thin wrappers over the
 * context API below.  Everything here is extern "C", takes plain pointers and
 * sizes, and reports failure through an int status (GCS_OK == 0).
 *
 * One context owns one device's state: the particle arrays of one or more
 * segments (independent scenarios laid out back to back), the tree, the sort
 * buffers and the per-step scratch.  All work is queued on the context's
 * stream; calls that return host data synchronise that stream.
 *
 * Per step, for every segment, the engine runs the reference's pipeline
 * (cuda_engine.cu:379-451): bounds -> 63-bit Morton encode -> stable radix
 * sort with index tie-break -> gather -> Karras build -> bottom-up
 * aggregation -> tree walk -> kick+drift (+ colour) -> optional pack.
 */
#ifndef GCS_H
#define GCS_H

#include <stddef.h>
#include <stdint.h>
#include "gcs_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GCS_OK            0
#define GCS_ERR_ARG      -1  /* bad argument (null, size out of range, ...) */
#define GCS_ERR_CUDA     -2  /* a CUDA runtime call failed */
#define GCS_ERR_NOMEM    -3  /* device or host allocation failed */
#define GCS_ERR_CAPACITY -4  /* more particles/segments than the context holds */
#define GCS_ERR_DEVICE   -5  /* a kernel raised a bit of the device status word */
#define GCS_ERR_STATE    -6  /* call not valid in the context's current state */
#define GCS_ERR_NO_DEVICE -7 /* no CUDA device, or not an sm_100 device */

/* Bits of the device status word (gcs_device_status).  Kernels never trap:
 * a bounded wait that runs out, or a capacity that would be exceeded, sets a
 * bit, skips the offending access and returns. */
#define GCS_DEV_SORT_LOOKBACK_TIMEOUT 0x1u /* radix-sort decoupled look-back gave up */
#define GCS_DEV_WALK_STACK_OVERFLOW   0x2u /* a walk stack would have overflowed */
#define GCS_DEV_NONFINITE_POSITION    0x4u /* NaN/Inf position met in bounds/encode */
#define GCS_DEV_BUILD_RANGE           0x8u /* Karras build produced an out-of-range child */
#define GCS_DEV_TREE_MALFORMED        0x10u /* a walk or climb exceeded the bound a valid tree obeys */

/* ---- step parameters --------------------------------------------------- */
#define GCS_BOUNDS_CALLER 0 /* use global_min/global_max for every segment (reference API) */
#define GCS_BOUNDS_DEVICE 1 /* per-segment min/max reduced on the device */

typedef struct gcs_params {
    float G;            /* gravitational constant (reference passes 1) */
    float epsilon_sq;   /* Plummer softening eps^2, added to every d^2 */
    float theta;        /* opening angle: a node is used as a monopole when
                           width^2 < theta^2 * (d^2 + eps^2); the reference's
                           GPU walk is theta = 1 (cuda_engine.cu:143) */
    float dt;           /* kick+drift step */
    int32_t leaf_size;  /* L >= 1: an opened node holding <= L particles is
                           summed particle by particle (reference: 1) */
    int32_t bounds_mode;/* GCS_BOUNDS_CALLER or GCS_BOUNDS_DEVICE */
    float global_min;   /* Morton cube, used with GCS_BOUNDS_CALLER */
    float global_max;
    int32_t recolor;    /* 1: the reference's speed colour map for types 0/2 */
    int32_t com_fp64;   /* 1: node centres of mass from FP64 sums;
                           0: the reference's FP32 pairwise formula */
    int32_t walk_batch; /* nodes fetched per stack pop, 1..64 (0 = default 32) */
    int32_t walk_blocks_per_sm; /* persistent walk occupancy (0 = default) */
    int32_t with_potential; /* 1: the walk also sums potentials (ACCEL .w) */
    int32_t tune_leaf_min;  /* gcs_autotune: smallest leaf size it may pick (0 = 1) */
    int32_t reserved[2];
} gcs_params;

/* The reference's fixed settings: G=1, eps^2=10, theta=1, dt=0.01, L=1,
 * caller bounds [-1e4, 1e4] (main.cpp:111-112,197,461-462), FP32 COM,
 * recolouring on. */
void gcs_params_reference(gcs_params* p);

/* ---- context lifecycle -------------------------------------------------- */
typedef struct gcs_ctx gcs_ctx;

/* Allocates device state for up to `capacity` particles in up to
 * `max_segments` segments on `device`.  The context starts with one segment
 * of `capacity` particles. */
int gcs_create(gcs_ctx** out, int64_t capacity, int32_t max_segments, int32_t device);
void gcs_destroy(gcs_ctx* ctx);
/* Queue all further work on `stream` (a cudaStream_t; NULL = the legacy
 * default stream).  The caller keeps the stream alive. */
int gcs_set_stream(gcs_ctx* ctx, void* stream);
void* gcs_get_stream(const gcs_ctx* ctx);
const char* gcs_status_string(int status);
/* Text of the last failure on this context ("" if none). */
const char* gcs_last_error(const gcs_ctx* ctx);

/* ---- layout --------------------------------------------------------------
 * Segments are independent scenarios packed back to back: segment s holds
 * particles [off_s, off_s + counts[s]).  Changing the layout invalidates the
 * particle data. */
int gcs_set_segments(gcs_ctx* ctx, int32_t num_segments, const int64_t* counts);
/* Change the layout keeping the particles of some segments: new segment s
 * takes over old segment src_segment[s] (same count) or, with -1, starts
 * empty (upload its Stars afterwards at gcs_segment_offset).  Kept segments
 * are copied on the device; their state is unchanged. */
int gcs_relayout(gcs_ctx* ctx, int32_t num_segments, const int64_t* counts, const int32_t* src_segment);
/* First particle of `segment` (segment == number of segments gives N). */
int64_t gcs_segment_offset(const gcs_ctx* ctx, int32_t segment);
int64_t gcs_num_particles(const gcs_ctx* ctx);
int32_t gcs_num_segments(const gcs_ctx* ctx);

/* Targets per walk group (8..64, default 32): the walk's warps each take a
 * run of this many consecutive sorted particles of one segment (above 32, two
 * targets per lane).  Results do not depend on it (each target's terms are
 * its own walk's); speed does. */
int gcs_set_group_width(gcs_ctx* ctx, int32_t width);
int32_t gcs_group_width(const gcs_ctx* ctx);
/* Walk frontiers (enable = 1, the default; no counterpart in the reference,
 * whose walk starts every target at the root, cuda_engine.cu:100-107): before
 * the walk, one pass per super-group of about 256 consecutive targets decides
 * the top of the tree against the super-group's bounding box - nodes every
 * one of its targets accepts, nodes every one opens - and each walk group
 * evaluates the accepted nodes for all its targets and starts its own walk
 * at the undecided nodes.  With enable = 0 every group walks from its
 * segment's root.  Both give every target exactly its own walk's terms; only
 * the order of the FP32 sums differs. */
int gcs_set_walk_frontier(gcs_ctx* ctx, int32_t enable);

/* ---- one scenario across devices -----------------------------------------
 * Every rank of a multi-GPU job holds the whole scenario and runs the same
 * bounds, sort, build and aggregation, which give the same sorted order and
 * tree everywhere; each rank then walks and kicks/drifts only its slice of
 * the sorted particles, and an all-gather of the slices of the position and
 * velocity arrays (gcs_device_array) completes the step.  The result is the
 * single-device step, bit for bit.  (The reference steps one scenario on one
 * device; this has no counterpart there.) */
/* Restrict the walk and the kick/drift (gcs_step, the walk and integrate
 * stages, gcs_kick) to the sorted particles [first, first + count); count < 0
 * restores every particle.  Both bounds must be the first particle of a walk
 * group (a multiple of the group width within its segment) or the particle
 * count.  A layout change resets the range. */
int gcs_set_step_range(gcs_ctx* ctx, int64_t first, int64_t count);
/* Device address of the context's current arrays: which = GCS_BUF_POS or
 * GCS_BUF_VEL (float4 per particle, the state after the last step) or
 * GCS_BUF_ACCEL; NULL otherwise.  Steps alternate between two position and
 * velocity arrays, so ask again after every step. */
void* gcs_device_array(gcs_ctx* ctx, int32_t which);

/* ---- particle data ------------------------------------------------------ */
/* Copy host Stars into particles [offset, offset+n) (host may be pageable or
 * pinned); the reference's cuda_upload_initial_stars (cuda_engine.cu:342-352). */
int gcs_upload_stars(gcs_ctx* ctx, const Star* host, int64_t offset, int64_t n);
/* Pack particles [offset, offset+n) as Stars and copy them to host; synchronises. */
int gcs_download_stars(gcs_ctx* ctx, Star* host, int64_t offset, int64_t n);
/* Pack particles [offset, offset+n) as simulation.bin records and copy to
 * host; synchronises. */
int gcs_download_playback(gcs_ctx* ctx, PlaybackStar* host, int64_t offset, int64_t n);

/* ---- stepping ----------------------------------------------------------- */
/* One full step of every segment, queued on the context stream. */
int gcs_step(gcs_ctx* ctx, const gcs_params* p);
/* With graphs on, gcs_step launches the whole step as one CUDA graph
 * (captured on first use, one graph per ping-pong parity of the particle
 * arrays) and recaptures only when the parameters, the segment layout, the
 * group width or the stream change.  Needs a non-default stream. */
int gcs_set_graphs(gcs_ctx* ctx, int32_t enable);
/* Timing hooks: `start` and `end` (cudaEvent_t of the context's device, or
 * NULL) are recorded on the context stream right before and after the walk
 * stage of every gcs_step and gcs_run_stages from now on (not in the host
 * steps, gcs_step_host and gcs_step_host_io), in eager steps and inside
 * graph-captured steps alike (there they are
 * event-record nodes; a gcs_step after a change of events points those nodes
 * at the new events before it launches, so each step can be timed with its
 * own pair).  Setting or clearing an event recaptures the graphs at the next
 * gcs_step; replacing one by another does not.  No counterpart in the
 * reference. */
int gcs_set_walk_events(gcs_ctx* ctx, void* start, void* end);
/* How many times the step graphs have been captured on this context. */
int32_t gcs_graph_builds(const gcs_ctx* ctx);
/* One step with every particle's stepped Star (sorted order) written to
 * `host`, synchronised on return: the reference's cuda_physics_step with
 * use_interop=false (cuda_engine.cu:379-451).  Without a step range the
 * transfer overlaps the walk: the walk's epilogue applies the kick/drift and
 * writes the Star records group by group.  When `host` is pinned host memory
 * mapped into the device (cudaMallocHost, cudaHostAlloc, registered memory;
 * all n records inside one allocation, 16-byte aligned), the records are
 * written straight into it over PCIe; otherwise each finished chunk of groups
 * is copied from device staging while later groups are still being walked
 * (up to 64 chunks a step: large ones over the groups handed out early,
 * small ones over the last groups, which finish together at the end).  The
 * Stars and the device state are the same bits as
 * gcs_run_stages(bounds..integrate) followed by gcs_download_stars. */
int gcs_step_host(gcs_ctx* ctx, const gcs_params* p, Star* host);
/* One step from host Stars to host Stars: the same result as
 * gcs_upload_stars(ctx, in, 0, n) followed by gcs_step_host(ctx, p, out)
 * (`out` may be `in`), with the upload in up to 8 chunks on a copy stream,
 * each chunk unpacked and reduced into the device bounds as soon as it lands,
 * and no host synchronisation between the upload and the step (the
 * reference uploads its Stars once, cuda_engine.cu:283-296, and copies them
 * back after every step, cuda_engine.cu:442-448). */
int gcs_step_host_io(gcs_ctx* ctx, const gcs_params* p, const Star* in, Star* out);
/* Accelerations at the current positions (bounds..walk, no kick/drift).
 * Afterwards the particle arrays are in this step's Morton order and the
 * acceleration buffer matches them. */
int gcs_compute_accels(gcs_ctx* ctx, const gcs_params* p);
/* v += a * dt with the last computed accelerations (a half-kick for
 * kick-drift-kick open/close). */
int gcs_kick(gcs_ctx* ctx, float dt);

/* Pipeline stages, for stage-by-stage checking.  gcs_run_stages runs
 * stages first..last inclusive with the given parameters. */
#define GCS_STAGE_BOUNDS    0
#define GCS_STAGE_ENCODE    1
#define GCS_STAGE_SORT      2
#define GCS_STAGE_GATHER    3
#define GCS_STAGE_BUILD     4
#define GCS_STAGE_AGGREGATE 5
#define GCS_STAGE_WALK      6
#define GCS_STAGE_INTEGRATE 7
int gcs_run_stages(gcs_ctx* ctx, const gcs_params* p, int32_t first, int32_t last);

/* Wait for the context stream; returns GCS_ERR_DEVICE if the device status
 * word is non-zero (read it with gcs_device_status). */
int gcs_synchronize(gcs_ctx* ctx);
/* Device status word (GCS_DEV_* bits), synchronising; `clear` resets it. */
int gcs_device_status(gcs_ctx* ctx, uint32_t* status, int32_t clear);

/* ---- introspection (synchronises) ----------------------------------------
 * Copy `count` elements starting at element `first` of an internal buffer to
 * host.  Element types: KEYS u64, INDEX u32 (sorted position -> position
 * before this step's sort), NODES BvhNodeTraverse, BUILD BvhNodeBuild,
 * LEAF_PARENT i32, ACCEL float4 (ax,ay,az,potential), POS float4 (x,y,z,m),
 * VEL float4 (vx,vy,vz, bits of type|r|g|b), BOUNDS float2 per segment,
 * KEYS_UNSORTED u64 (encode output; valid until the sort stage runs, which
 * uses that buffer for its passes). */
#define GCS_BUF_KEYS          0
#define GCS_BUF_INDEX         1
#define GCS_BUF_NODES         2
#define GCS_BUF_BUILD         3
#define GCS_BUF_LEAF_PARENT   4
#define GCS_BUF_ACCEL         5
#define GCS_BUF_POS           6
#define GCS_BUF_VEL           7
#define GCS_BUF_BOUNDS        8
#define GCS_BUF_KEYS_UNSORTED 9
int gcs_read_buffer(gcs_ctx* ctx, int32_t which, void* host, int64_t first, int64_t count);
/* Number of internal tree nodes (sum over segments of count-1). */
int64_t gcs_num_internal_nodes(const gcs_ctx* ctx);

/* ---- initial conditions -------------------------------------------------
 * Seeded two-galaxy collision: each galaxy is a Miyamoto-Nagai disc, a
 * Hernquist bulge and a Hernquist dark-matter halo (the reference's
 * generator.cpp:3-196 components), with the recipe's masses, scale lengths,
 * truncations and orbit given here.  Deterministic for a given spec. */
typedef struct gcs_galaxy_spec {
    int64_t n_disc, n_bulge, n_halo;
    float disc_mass, disc_a, disc_b, disc_rmax, disc_zmax;
    float bulge_mass, bulge_a, bulge_rmax;
    float halo_mass, halo_a, halo_rmax;
    float pos[3], vel[3];
    float incline_deg;   /* rotation of the whole galaxy about the x axis */
    uint8_t type;        /* 0 = galaxy A colours, 2 = galaxy B colours */
} gcs_galaxy_spec;

typedef struct gcs_collision_spec {
    gcs_galaxy_spec galaxy[2];
    uint64_t seed;
    float G;
    float disc_dispersion; /* disc velocity noise, fraction of v_c */
} gcs_collision_spec;

/* Equal galaxies (the recipe of the 45,056- and 1,048,576-particle cases):
 * disc a=3, b=0.3, M=1 (R<=15, |z|<=3); bulge a=0.5, M=0.33 (r<=5); halo
 * a=10, M=5.8 (r<=30); galaxy A at (-20,-5,0) moving (+0.4,0,0), galaxy B at
 * (+20,+5,0) moving (-0.4,0,0) with its disc inclined 30 deg about x.
 * Per-galaxy counts are given (16384/4096/2048 and 384000/96000/44288 in
 * the two cases). */
int gcs_collision_spec_equal(gcs_collision_spec* spec, int64_t n_disc, int64_t n_bulge,
                             int64_t n_halo, uint64_t seed);
/* Unequal pair: galaxy B is the equal-case galaxy, galaxy A is it scaled to
 * mass ratio q = M_A/M_B in (0,1] (lengths by q^(1/3)); impact parameter b
 * along y, relative speed v along x, 40 length units apart in x, centre of
 * mass at rest at the origin; galaxy B inclined by incline_deg.  Particle
 * counts are proportional to mass (equal particle masses across galaxies),
 * split disc:bulge:halo as 384000:96000:44288. */
int gcs_collision_spec_pair(gcs_collision_spec* spec, int64_t n_total, float q,
                            float impact, float rel_speed, float incline_deg,
                            uint64_t seed);
int64_t gcs_collision_count(const gcs_collision_spec* spec);
int gcs_generate_collision(const gcs_collision_spec* spec, Star* out, int64_t n);

/* ---- diagnostics --------------------------------------------------------
 * FP64 reductions over one segment's current state: out = {kinetic energy,
 * px, py, pz, total mass, potential energy}.  The potential energy is
 * 0.5 * sum m_i phi_i over the potentials of the last walk, which must have
 * run with with_potential = 1 at the current positions (else it is 0). */
int gcs_diagnostics(gcs_ctx* ctx, int32_t segment, double out[6]);
/* The same with every velocity taken as v + a * kick (FP64) from the last
 * computed accelerations: after gcs_compute_accels at step n of the
 * leapfrog (whose stored velocities are the half-step ones, v_{n-1/2}),
 * kick = dt/2 gives the energy and momentum at the synchronised v_n. */
int gcs_diagnostics_kicked(gcs_ctx* ctx, int32_t segment, double kick, double out[6]);
/* Interaction counts of one walk at the current state: runs bounds..walk
 * with the counting walk and returns {monopole terms, particle terms}
 * summed over all targets (the unit of interactions/s; 20 FP32 flops each),
 * then the warp-wide {node evaluations, particle-source evaluations} (each
 * serves up to 32 targets; terms / (32 * evaluations) is the lane
 * utilisation of the group walk), then {stack pop rounds, stack spills to
 * global memory}, then {node evaluations opened by every active lane, node
 * evaluations accepted by every active lane}. */
int gcs_count_interactions(gcs_ctx* ctx, const gcs_params* p, uint64_t out[8]);
/* Deepest walk stack of the last gcs_count_interactions, in entries (one
 * node and its target masks each), over every warp: out[0]; out[1] the
 * entries of the global-memory bottom each walk warp may spill to (32-target
 * groups; the shared-memory top holds a few hundred more).  Synchronises the
 * context stream.  No counterpart in the reference, whose walk keeps a fixed
 * 256-entry local stack per thread (cuda_engine.cu:106). */
int gcs_walk_stack_peak(gcs_ctx* ctx, int64_t out[2]);
/* Lane use of the last gcs_count_interactions.  The walk evaluates rows: one
 * node or particle source for every target slot of a walk warp at once (32
 * slots, 64 for groups wider than 32), each target keeping or discarding its
 * term.  out[0..3]: rows of the super-group take lists, of take nodes holding
 * every live target, of other take nodes, of mixed nodes (each target
 * decides); out[4]: targets in the masks of the other take nodes; out[5]:
 * targets in the masks of mixed nodes; out[6]: of those, the targets that
 * accepted the node as a monopole; out[7]: targets in the masks of particle
 * sources (their rows are gcs_count_interactions' out[3]).  Synchronises the context stream.  No counterpart in the
 * reference, whose walk gives each target its own thread. */
int gcs_walk_lane_use(gcs_ctx* ctx, uint64_t out[8]);
/* Autotuner: times the walk on the current state for leaf sizes
 * {1,2,4,8,16,32} from p->tune_leaf_min up to p->leaf_size (the caller's
 * "leaf <= L"; leaf size 2 gives exactly the reference's terms, sizes >= 3
 * replace monopoles inside small opened nodes by exact sums), pop
 * batches {16,32,64}, group widths {32,16} and two occupancies, then writes the
 * fastest leaf_size / walk_batch / walk_blocks_per_sm into *p and keeps the
 * fastest group width on the context.  It runs bounds..aggregate once (the
 * particle arrays end in this step's Morton order, values unchanged) and
 * the walk repeatedly; best_walk_ms (may be NULL) receives the best time. */
int gcs_autotune(gcs_ctx* ctx, gcs_params* p, double* best_walk_ms);
/* Allocation-free sort (no counterpart in the reference): a stable sort of
 * n <= 1,048,576 (u64 key, u32 value) pairs by the whole key, for callers
 * that cannot allocate device memory where they sort (a real-time loop or
 * host callback that must not trigger an allocation's implicit device
 * synchronisation, or a plug-in whose host application owns the device
 * memory budget).  All pointers are device memory owned by the caller:
 * keys/vals hold the pairs and receive the sorted pairs; keys_alt/vals_alt
 * are the same length and are overwritten by the passes; status (a device
 * word) receives GCS_DEV_SORT_LOOKBACK_TIMEOUT if a pass gave up and the
 * call only queues work on `stream`.  With status == NULL the call waits for
 * `stream` and returns GCS_ERR_DEVICE if a pass gave up.  The
 * histograms and look-back state live in one static device array of about
 * 2.1 MB that every GPU loading this library keeps until exit; no call
 * allocates.  Each call clears that array on `stream` (a cudaStream_t, NULL
 * = legacy default) before using it, so calls ordered on the GPU are
 * independent, but calls that overlap on the GPU race on it.  The first
 * call on a device looks up the array's device address (with that device
 * current) - make it before any stream capture.  Larger n returns
 * GCS_ERR_CAPACITY. */
int gcs_sort_pairs_static(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                          int64_t n, uint32_t* status, void* stream);
/* FP64 direct-sum accelerations (excluding only i == j) at `n_targets`
 * sorted positions `targets` of one segment; result as double[3*n_targets].
 * Reads the current positions; eps^2 and G from p. */
int gcs_direct_accels_fp64(gcs_ctx* ctx, const gcs_params* p, int32_t segment,
                           const int64_t* targets, int64_t n_targets, double* out);
/* Device bytes the context holds. */
int64_t gcs_device_bytes(const gcs_ctx* ctx);
/* Device bytes gcs_create(capacity, max_segments, device) would allocate
 * (nothing is allocated); a negative status on bad arguments or device. */
int64_t gcs_context_bytes(int64_t capacity, int32_t max_segments, int32_t device);

/* ---- bake --------------------------------------------------------------------
 * `frames` steps of every segment, each followed by one simulation.bin frame
 * (n PlaybackStar records of the stepped state in that step's order, the
 * records gcs_download_playback returns) appended to `path` (created, or
 * appended to with append = 1): the reference's Bake loop (main.cpp:119-297).
 * Frames are packed on the device, copied into two pinned buffers on a
 * second stream while the next step computes, and written by a writer
 * thread in order (the pinned buffers and the stream are created at the
 * first call and kept by the context).  Returns when every frame has been
 * written; seconds (may be NULL) receives the wall time. */
int gcs_bake(gcs_ctx* ctx, const gcs_params* p, int32_t frames, const char* path, int32_t append,
             double* seconds);

/* ---- playback ----------------------------------------------------------------
 * Reading a simulation.bin file back frame by frame: the reference's Playback
 * mode (main.cpp:299-453) without its window.  Host only; no GPU is needed.
 * particles > 0: records per frame; the file must hold a whole number of
 * frames of that size.  particles = 0: the reference's inference, particles =
 * file size / frames_hint / 16 (the reference hard-codes 2000 frames,
 * main.cpp:309), and only whole frames are kept.  Errors: GCS_ERR_ARG (no
 * such file, an empty file, a size that is not a whole number of frames,
 * bad arguments), GCS_ERR_NOMEM. */
typedef struct gcs_playback gcs_playback;
int gcs_playback_open(const char* path, int64_t particles, int64_t frames_hint, gcs_playback** out);
int64_t gcs_playback_frames(const gcs_playback* pb);
int64_t gcs_playback_particles(const gcs_playback* pb);
/* The frame the next gcs_playback_next returns. */
int64_t gcs_playback_position(const gcs_playback* pb);
/* Read the next frame into `host` (particles records); after the last frame
 * playback loops to the first (main.cpp:413-419). */
int gcs_playback_next(gcs_playback* pb, PlaybackStar* host);
/* Step back: the frame before the one last read, or the last frame when that
 * is before the first (main.cpp:397-410); reading goes on forward from it. */
int gcs_playback_prev(gcs_playback* pb, PlaybackStar* host);
/* Move so that the next read returns `frame` (taken modulo the frame count). */
int gcs_playback_seek(gcs_playback* pb, int64_t frame);
/* The camera target of a frame: the mean position in FP64, rounded to float
 * (main.cpp:435-441). */
int gcs_playback_centre(const PlaybackStar* frame, int64_t n, float centre[3]);
void gcs_playback_close(gcs_playback* pb);

/* ---- headless point-splat renderer ------------------------------------------
 * The reference draws every Star as one GL point (renderer.cpp:97-148,
 * vertex attributes 226-233): the
 * vertex shader transforms it by view and projection and sizes it by its
 * view-space distance d (dark matter, type 1: clamp(2500/d, 1, 6) pixels;
 * stars: clamp(1000/d, 1, 3)); the fragment shader gives each pixel of the
 * point's square whose centre lies at normalised radius r <= 1 an alpha of
 * exp(-3 r^2), times 0.03 with colour (0.4, 0, 0.8) for dark matter and
 * times 0.15 with the Star's own rgb/255 otherwise; fragments are added to
 * the framebuffer with glBlendFunc(GL_SRC_ALPHA, GL_ONE) (renderer.cpp:
 * 202-204) over the clear colour (0.01, 0.01, 0.02, 1) (renderer.cpp:248).
 * There is no graphics stack here, so the same arithmetic runs as a CUDA
 * splat: fragments are summed in 64-bit fixed point (2^-24 units per channel,
 * so a frame does not depend on fragment order) and resolved once to RGBA8
 * (round to nearest, clamped), row 0 at the bottom as in GL's default
 * framebuffer.  Points whose centre lies outside the clip volume are culled;
 * fragments outside the viewport are dropped. */
typedef struct gcs_camera {
    float pos[3];       /* eye (renderer.cpp:9) */
    float front[3];     /* looks at pos + front (renderer.cpp:10, 262) */
    float up[3];        /* renderer.cpp:11 */
    float fovy_deg;     /* vertical field of view, degrees (renderer.cpp:263: 45) */
    float z_near;       /* renderer.cpp:263: 0.1 */
    float z_far;        /* renderer.cpp:263: 5000 */
} gcs_camera;
/* The reference's start-up camera: eye (0, 150, 600), front (0, -0.2, -1),
 * up (0, 1, 0), 45 degrees, near 0.1, far 5000. */
void gcs_camera_reference(gcs_camera* cam);
/* Point the camera at `target` from where it stands: front = normalize(target -
 * pos), as the reference does every frame while the camera is locked on the
 * centre of mass or, in Playback mode, the frame's mean position
 * (renderer.cpp:255-256; the target from gcs_playback_centre or
 * cuda_get_center_of_mass).  The direction is formed as d * (1 / |d|); the
 * reference's glm::normalize multiplies by an inverse square root, so the two
 * agree up to the last bit of rounding.  The reference also re-derives its
 * mouse-look yaw and pitch from the new front (renderer.cpp:257-258); that
 * interactive state has no counterpart here (a caller that keeps one uses
 * pitch = asin(front.y), yaw = atan2(front.z, front.x)).  GCS_ERR_ARG when
 * target is the eye. */
int gcs_camera_look_at(gcs_camera* cam, const float target[3]);
/* The 4x4 view and projection matrices (row-major, applied to column
 * vectors) the renderer uses for cam at width x height: glm::lookAt(pos,
 * pos + front, up) and glm::perspective(fovy, width/height, near, far). */
int gcs_camera_matrices(const gcs_camera* cam, int32_t width, int32_t height, float view[16],
                        float proj[16]);
/* Render the context's current particles of `segment` (-1: every segment)
 * into rgba (width*height*4 bytes; host memory when rgba_on_host, else
 * device memory), on the context's stream.  The context keeps a fixed-point
 * accumulator of width*height*24 bytes, allocated at the first call and
 * grown when a larger frame is asked for.  A host target synchronises the
 * stream; a device target does not. */
int gcs_render_frame(gcs_ctx* ctx, const gcs_camera* cam, int32_t segment, int32_t width,
                     int32_t height, uint8_t* rgba, int32_t rgba_on_host);
/* Render n device Stars (for example gcs_dropin_device_stars()) on `stream`
 * (NULL: the default stream), asynchronously: fragments are added to the
 * caller's device accumulator accum (width*height*3 uint64, 2^-24 units per
 * channel, pixel-major r, g, b; zero it before a new frame) and, unless rgba
 * is NULL, the frame is resolved into the device buffer rgba.  stars must be
 * 16-byte aligned, accum 8-byte and rgba 4-byte aligned. */
int gcs_render_stars(const Star* stars, int64_t n, const gcs_camera* cam, int32_t width,
                     int32_t height, uint64_t* accum, uint8_t* rgba, void* stream);
/* As gcs_render_stars for n device PlaybackStar records (a simulation.bin
 * frame copied to the device): the reference's Playback mode draws a frame's
 * records as Stars with the same position, colour and type (main.cpp:423-433),
 * so a frame renders exactly as the Stars it was written from.  frame must
 * be 16-byte aligned. */
int gcs_render_playback(const PlaybackStar* frame, int64_t n, const gcs_camera* cam, int32_t width,
                        int32_t height, uint64_t* accum, uint8_t* rgba, void* stream);

/* ---- serving ---------------------------------------------------------------
 * Continuous batching of independent collision scenarios on one device (no
 * counterpart in the reference, whose engine holds one simulation in
 * file-scope globals, cuda_engine.cu:16-44).  Requests are queued by
 * gcs_server_submit; every gcs_server_tick admits queued scenarios in
 * arrival order while segment slots and particle capacity allow, lays the
 * resident scenarios out as segments of one context (kept scenarios stay
 * on the device; the step graph is captured again only after a membership
 * change), advances all of them by one step with one launch per stage, and
 * retires those that reached their step count.  Each scenario's final
 * Stars are byte-identical to stepping it alone with the same parameters.
 * Not thread-safe: one host thread drives a server. */
typedef struct gcs_server gcs_server;
typedef struct gcs_server_result {
    uint64_t id;
    int64_t n;
    int32_t steps;
    int32_t status;    /* GCS_OK, or GCS_ERR_DEVICE if a status bit was raised */
    double queued_ms;  /* submit -> admission */
    double latency_ms; /* submit -> final Stars on the host */
} gcs_server_result;
/* A server on `device` holding up to max_segments scenarios and
 * max_particles particles, shrunk so that its whole device footprint stays
 * within hbm_budget_bytes (gcs_server_capacity gives the result). */
int gcs_server_create(gcs_server** out, int32_t device, int64_t max_particles,
                      int32_t max_segments, double hbm_budget_bytes, const gcs_params* p);
void gcs_server_destroy(gcs_server* srv);
/* The context underneath (for diagnostics; do not change its layout). */
gcs_ctx* gcs_server_context(gcs_server* srv);
int64_t gcs_server_capacity(const gcs_server* srv);
const char* gcs_server_last_error(const gcs_server* srv);
/* With dir set, scenario <id> writes <dir>/<id>.bin in the simulation.bin
 * format (frames of n PlaybackStar records, main.cpp:264-272): a frame every
 * frame_every steps (0: none) and always its final frame. */
int gcs_server_set_output(gcs_server* srv, const char* dir, int32_t frame_every);
/* Queue a scenario (Stars are copied); GCS_ERR_CAPACITY if n exceeds the
 * server's particle capacity. */
int gcs_server_submit(gcs_server* srv, uint64_t id, const Star* stars, int64_t n, int32_t steps);
/* One scheduling round; out (may be NULL) = {resident scenarios, resident
 * particles, admitted this round, retired this round}.  At most two steps
 * are in flight on the device when it returns. */
int gcs_server_tick(gcs_server* srv, int64_t out[4]);
/* out = {queued, resident, finished and not yet popped}. */
int gcs_server_counts(const gcs_server* srv, int64_t out[3]);
/* Progress since creation: out[0] particle-steps advanced (the resident
 * particles of every tick's step, queued steps included), out[1] steps
 * (ticks that stepped), out[2] peak resident scenarios, out[3] peak resident
 * particles. */
int gcs_server_progress(const gcs_server* srv, int64_t out[4]);
/* Pop the oldest finished scenario: returns 1 and fills info (and host, if
 * not NULL, with its n final Stars), 0 if none has finished. */
int gcs_server_pop(gcs_server* srv, gcs_server_result* info, Star* host, int64_t host_capacity);

#ifdef __cplusplus
}
#endif

#endif /* GCS_H */
