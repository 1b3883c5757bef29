/*
 * firex.h — C ABI of the B200-native Fire-X simulation step.
 *
 * The library owns all device memory; host buffers always belong to the caller.
 * Every call returns an int status (FIREX_OK or a negative FIREX_ERR_*); the text of
 * the most recent failure on a handle is available from firex_last_error().
 * One simulation handle is not thread-safe: serialise calls on it (the reference
 * engine serialises resource mutations on a promise queue, FireXEngine.ts:1882-1889).
 *
 * Reference interface replaced by this ABI (taesiri/Fire):
 *   SimulationEngine          src/sim/types.ts:34-63
 *   FireXEngine               src/sim/firex/FireXEngine.ts:370
 * Each entry point below names the reference member it stands in for.
 */
#ifndef FIREX_H
#define FIREX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FIREX_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------------- */
#define FIREX_OK 0
#define FIREX_ERR_BAD_ARG (-1)     /* invalid argument (reference: thrown Error / RangeError) */
#define FIREX_ERR_OOM (-2)         /* device allocation failed; previous state kept */
#define FIREX_ERR_BUDGET (-3)      /* admission refused by the memory budget / preflight */
#define FIREX_ERR_CUDA (-4)        /* CUDA runtime error; the handle is poisoned */
#define FIREX_ERR_TIMEOUT (-5)     /* a bounded device wait gave up */
#define FIREX_ERR_UNSUPPORTED (-6) /* option combination not implemented */
#define FIREX_ERR_STATE (-7)       /* handle disposed or poisoned (reference: device lost) */

/* ---- options ---------------------------------------------------------------------- */
/* Storage precision of the step. F32 mirrors the reference's f32 storage buffers;
 * MIXED stores the transported species (fuel, O2, products, vapor) in FP16 (RNE) and keeps
 * velocity and temperature (one 16-byte record), divergence and reaction in FP32; all
 * arithmetic is FP32 and norms are FP64. Pressure storage follows the pressure branch
 * (FP16 only in branch B). Against the FP64 oracle, FP32 arithmetic itself leaves the
 * post-projection divergence 4e-5 .. 9e-5 of the pre-projection norm away; FP16 species
 * move that by under 1e-6, FP16 pressure (branch B) raises it to 4e-3 .. 8e-3. */
#define FIREX_PRECISION_F32 0
#define FIREX_PRECISION_MIXED 1

/* Pressure branch (FireXEngine.ts:2175-2274). AUTO applies the reference rule: below
 * FIREX_HEAVY_GRID_CELL_THRESHOLD cells the warm-started f32 global solve (branch A),
 * at or above it the f16-storage tiled solve (branch B). */
#define FIREX_PRESSURE_AUTO 0
#define FIREX_PRESSURE_WARM_F32 1 /* branch A: f32, primary pressure warm-starts across steps */
#define FIREX_PRESSURE_F16 2      /* branch B: f16 storage, f32 math, warm start */
#define FIREX_PRESSURE_COLD_F32 3 /* branch C: f32, both solves cold-start in two shared buffers */

#define FIREX_HEAVY_GRID_CELL_THRESHOLD (64LL * 1024 * 1024) /* gridConfiguration.ts:105 */

/* Emitter model. BURNER is the reference's analytic elliptical burner
 * (shaders.ts:101-133). SPHERES replaces it with a list of spheres in cell units:
 * a cell is inside when |c + 0.5 - center|^2 <= radius^2 (float arithmetic, fixed
 * order), and inside cells receive fuel = max(fuel, f*j), T = max(T, T_amb + (T_e -
 * T_amb)*j) and the burner's swirl/lift with source = 1, where j is the per-step
 * emission jitter. SPHERES is an extension (no reference counterpart). */
#define FIREX_EMITTER_BURNER 0
#define FIREX_EMITTER_SPHERES 1
#define FIREX_MAX_SPHERES 8

typedef struct firex_sphere {
    float center[3];   /* cell units, x y z */
    float radius;      /* cell units */
    float fuel;        /* injected fuel concentration */
    float temperature; /* injected temperature, K */
} firex_sphere;

typedef struct firex_options {
    int32_t precision;             /* FIREX_PRECISION_* */
    int32_t pressure_mode;         /* FIREX_PRESSURE_* */
    int32_t pressure_iterations;   /* P, primary Jacobi sweeps per step */
    int32_t correction_iterations; /* R, residual Jacobi sweeps per step */
    int32_t emitter_mode;          /* FIREX_EMITTER_* */
    int32_t num_spheres;           /* 0..FIREX_MAX_SPHERES */
    firex_sphere spheres[FIREX_MAX_SPHERES];
    uint64_t seed;                 /* seeds velocity noise and emission jitter */
    float velocity_noise;          /* initial velocity: uniform in [-a, a] per component */
    float emission_jitter;         /* per-step emission factor uniform in [1-a, 1+a] */
    int32_t cinematic;             /* mixing.z; offline tiers force 1 (FireXEngine.ts:2097,2819) */
    int32_t jacobi_block;          /* 2: two Jacobi sweeps per launch (FUSED, see firex_set_jacobi); 0/1: AUTO */
    uint64_t memory_budget_bytes;  /* 0 = no budget; else create fails with FIREX_ERR_BUDGET */
    int32_t jacobi_zchunk;         /* z planes per CTA of a fused Jacobi launch; 0 = auto */
    int32_t particle_count;        /* SPH droplets (FIREX_QUALITY particleCount, FireXEngine.ts:187-277);
                                      they run while waterEnabled and waterFlow > 0.001 */
    int32_t reserved[6];
} firex_options;

/* Fills *opt with the defaults: F32, AUTO pressure, P = R = 64 (offline HD tier,
 * FireXEngine.ts:240-252), burner emitter, seed 0, no noise, no jitter, cinematic 1. */
void firex_default_options(firex_options* opt);

/* ---- fields ----------------------------------------------------------------------- */
/* Field ids for firex_read_field / firex_write_field. Layout is always the
 * reference's: cell index = x + X*(y + Y*z) (shaders.ts:47-51), and the element types
 * below, whatever the internal storage precision. */
#define FIREX_FIELD_FLOW 0             /* float4 per cell: u v w T   (flow[0], canonical) */
#define FIREX_FIELD_SPECIES 1          /* float4 per cell: fuel O2 products vapor (current) */
#define FIREX_FIELD_PRESSURE 2         /* float per cell: current primary pressure */
#define FIREX_FIELD_DIVERGENCE 3       /* float per cell: the divergence buffer */
#define FIREX_FIELD_REACTION 4         /* float per cell: instantaneous reaction rate */
#define FIREX_FIELD_LIQUID 5           /* uint32 per cell: deposited liquid, fixed point x4096 */
#define FIREX_FIELD_EMITTER_MASK 6     /* uint8 per cell, read only: sphere emitter mask */
#define FIREX_FIELD_CORRECTION 7       /* float per cell: last residual-pressure result */
#define FIREX_FIELD_FINAL_DIVERGENCE 8 /* float per cell, read only: divergence of FLOW */
/* The three render volumes (storePackedFields, qualityShaders.ts:37-75), read only: 4 FP16
 * values per cell (round to nearest even), as the reference's rgba16float textures hold. */
#define FIREX_FIELD_RENDER_FLOW 9      /* u, v, w, clamp((T - 300) / 2600, 0, 1) */
#define FIREX_FIELD_RENDER_CHEMISTRY 10 /* max(species, 0) */
#define FIREX_FIELD_RENDER_MEDIA 11    /* reaction, soot, liquid, display value (view 7: divergence) */
#define FIREX_FIELD_COUNT 12

/* Element size in bytes of a field (16, 4 or 1), or 0 for an unknown id. */
size_t firex_field_element_size(int32_t field);

/* ---- engine state ----------------------------------------------------------------- */
typedef struct firex_state {
    double simulation_time;  /* FireXEngine.simulationTime */
    int64_t frame_index;     /* FireXEngine.frameIndex */
    int32_t species_index;   /* FireXEngine.speciesIndex (0/1) */
    int32_t pressure_index;  /* FireXEngine.pressureIndex (0/1) */
} firex_state;

#define FIREX_UNIFORM_FLOATS 44  /* FireXEngine.ts:163 */

typedef struct firex_sim firex_sim;
typedef struct firex_batch firex_batch;

/* Allocates the solver bundle for a dims[0] x dims[1] x dims[2] grid and resets it.
 * Axes must be positive multiples of 4 (gridConfiguration.ts:98, preflight :306-317).
 * Replaces FireXEngine.initialize + createResourceSet (FireXEngine.ts:506-547,1536-1880).
 * On failure *out is NULL; the message is available from firex_last_error(NULL). */
int firex_create(const int32_t dims[3], const firex_options* opt, firex_sim** out);

/* Releases every device allocation. Replaces FireXEngine.dispose (FireXEngine.ts:1034). */
int firex_destroy(firex_sim* sim);

/* Text of the last failure on sim (or, when sim is NULL, of the last failed firex_create
 * or firex_divergence_norm_noalloc on the calling thread). */
const char* firex_last_error(const firex_sim* sim);

/* Named engine parameter with the reference's clamps and fallbacks
 * (FireXEngine.setParameter, FireXEngine.ts:937-1032). kind 0 passes a number, kind 1
 * a boolean (value != 0). Unknown names are ignored, as in the reference. */
#define FIREX_VALUE_NUMBER 0
#define FIREX_VALUE_BOOLEAN 1
int firex_set_parameter(firex_sim* sim, const char* name, int32_t kind, double value);
int firex_get_parameter(const firex_sim* sim, const char* name, double* value);

/* Every parameter at once from a 44-float block in the layout of the reference's uniform
 * buffer (Parameters, shaders.ts:2-14, as FireXEngine.writeUniforms fills it,
 * FireXEngine.ts:2043-2113; firex_get_uniforms returns the same layout). Each parameter slot
 * goes through the rules of firex_set_parameter (clamps, rounding, thresholds, booleans; the
 * spray angle is read in radians). The grid slots 0-2 must equal the handle's dimensions,
 * else FIREX_ERR_BAD_ARG and nothing changes. The time slots (dt, simulation time, frame),
 * the fixed ambient temperature, the canvas and particle slots and the cinematic flag are the
 * handle's own (firex_step, firex_set_state, the creation options) and are not read. */
int firex_set_params(firex_sim* sim, const float params[FIREX_UNIFORM_FLOATS]);

/* Re-initialises every field and the counters (FireXEngine.reset, FireXEngine.ts:843-852,
 * initializeFields :1933-1974). */
int firex_reset(firex_sim* sim);

/* Advances nsteps fixed steps of dt seconds each (one encodeSimulationStep per step,
 * FireXEngine.ts:2115-2276; simulationTime += dt and frameIndex += 1 per step as in
 * renderOfflineFrameInternal, :669-682). dt is a double like the reference's JS number:
 * simulationTime accumulates in double and the uniform block holds its f32 rounding.
 * Asynchronous: returns once the work is queued. */
int firex_step(firex_sim* sim, int32_t nsteps, double dt);

/* Blocks until queued work has finished (FireXEngine: queue.onSubmittedWorkDone, :692). */
int firex_sync(firex_sim* sim);

/* Copies a whole field to / from caller memory in the reference layout. bytes must equal
 * cells * firex_field_element_size(field). Synchronous. (No reference counterpart: the
 * reference never reads fields back; this is the field-readback half of the drop-in.) */
int firex_read_field(firex_sim* sim, int32_t field, void* host, size_t bytes);
int firex_write_field(firex_sim* sim, int32_t field, const void* host, size_t bytes);

/* Overlapped readback of a field (no reference counterpart: the reference reads no field
 * back). The field as it stands after the steps enqueued so far is copied in stream order
 * into a device staging buffer, then to `host` on a separate copy stream, so the copy
 * overlaps the steps enqueued after this call. `host` must stay valid (and should be
 * pinned, or the copy does not overlap) until firex_sync (or firex_batch_sync); a second
 * call waits on the device for the first copy to leave the staging buffer. Fields whose
 * host form needs a conversion (FP16 storage, emitter mask, final divergence) are
 * refused with FIREX_ERR_UNSUPPORTED: use firex_read_field. The first call allocates the
 * staging buffer (16 B/cell) and the copy stream. */
int firex_read_field_async(firex_sim* sim, int32_t field, void* host, size_t bytes);

/* Render volumes. Replaces packFields / copyAndPackBeautyFields (qualityShaders.ts:65-87),
 * whose rgba16float textures become three device buffers of 4 x FP16 per cell (cell index
 * x + X*(y + Y*z)) in the order of FIREX_FIELD_RENDER_FLOW, _CHEMISTRY, _MEDIA. With
 * packing on, every step ends by packing them from the canonical state; reading a render
 * field packs them on demand either way. firex_render_volumes gives their device
 * addresses (NULL until first allocated) for a renderer on the same device. */
int firex_set_render_packing(firex_sim* sim, int32_t on);
int firex_render_volumes(const firex_sim* sim, void* out[3]);

/* SPH droplets (particleBuffers, FireXEngine.ts:1598-1603): particle_count records of
 * two float4 each, (x, y, z, age) in domain units [0,1] and (vx, vy, vz, mass), as the
 * droplets stand after the steps so far. bytes must equal particle_count * 32. A write
 * replaces the current droplet state (the next step reads it); it does not change
 * whether the spray is on: that follows waterEnabled and waterFlow at every step. */
int firex_read_particles(firex_sim* sim, void* host, size_t bytes);
int firex_write_particles(firex_sim* sim, const void* host, size_t bytes);

/* Post-projection divergence of FLOW over interior cells (the one-cell outer shell is
 * excluded, qualityShaders.ts:47-57), reduced in FP64: out[0] = L2 norm, out[1] = max
 * abs, out[2] = number of interior cells. (Presentation diagnostic, FireXEngine.ts:2588-2596.) */
int firex_divergence_norm(firex_sim* sim, double out[3]);

/* The same norm for a flow field the caller owns, with no device allocation: for hosts
 * whose device memory belongs to their own pool or budget, or whose frame or serving loop
 * must not stall on cudaMalloc/cudaFree (both may synchronise the device), and which
 * therefore cannot let the library allocate or create a handle just for a norm.
 * No counterpart in the reference (its divergence view is a presentation pass).
 *
 * flow: device pointer, 16-byte aligned, dims[0]*dims[1]*dims[2] float4 records (u v w T)
 * with cell index x + X*(y + Y*z) (the layout of FIREX_FIELD_FLOW); metric: grid/domain
 * per axis as FP32 (shaders.ts:39-41); stream: cudaStream_t as void* (NULL: the legacy
 * default stream) on the device that owns flow. out[0] = L2, out[1] = max abs, out[2] =
 * interior cell count, as firex_divergence_norm. Returns after the result reached out.
 *
 * Scratch is a 32 KiB array in the library's device image (held on every GPU that loads
 * the library until exit), one slot pair per interior z plane: Z - 2 above
 * FIREX_NOALLOC_MAX_PLANES is rejected with FIREX_ERR_BAD_ARG. The first call on a device
 * looks up that array's device address; make it before any stream capture. Calls share
 * the array, so calls that overlap on a GPU race: serialise them. */
#define FIREX_NOALLOC_MAX_PLANES 2048
int firex_divergence_norm_noalloc(const void* flow, const int32_t dims[3], const float metric[3], void* stream,
                                  double out[3]);

/* Bounded device waits. The resident Jacobi's CTAs wait on their neighbours' flags; a wait
 * gives up after `polls` polls (0: the library's limit, well over a second), sets the
 * simulation's error word and returns, and the next firex_sync / firex_batch_sync answers
 * FIREX_ERR_TIMEOUT and poisons the handle (the reference's device-lost state,
 * FireXEngine.ts:538-542,2887-2897: later calls fail with FIREX_ERR_STATE). */
int firex_set_wait_limit(firex_sim* sim, uint32_t polls);

/* Test hook for the error path above (no reference counterpart): from the next step on, box
 * `box` of the resident Jacobi stops publishing its faces from sweep `sweep` on (in either
 * phase), a flag that nothing sets, so its neighbours' bounded waits expire. box < 0 clears it. */
int firex_test_hold_face(firex_sim* sim, int32_t box, int32_t sweep);

/* Counters that decide ping-pong parity and time (FireXEngine.ts:396-409). */
int firex_get_state(const firex_sim* sim, firex_state* st);
int firex_set_state(firex_sim* sim, const firex_state* st);

/* The 44-float uniform block the next step will use for time dt (writeUniforms,
 * FireXEngine.ts:2043-2113). */
int firex_get_uniforms(const firex_sim* sim, double dt, float out[FIREX_UNIFORM_FLOATS]);

/* Grid dimensions and options the handle was created with. */
int firex_get_info(const firex_sim* sim, int32_t dims[3], firex_options* opt);

/* Device bytes held by the handle (actual allocation, not the reference's model). */
int firex_device_bytes(const firex_sim* sim, uint64_t* bytes);

/* The reference's persistent-memory model (estimateFireXGridMemory,
 * gridConfiguration.ts:272-291): 116 B/cell below the heavy threshold, 108 B/cell at
 * or above, + 80 B/particle + the 64^3 RGBA8 detail texture. */
uint64_t firex_reference_memory_estimate(const int32_t dims[3], int64_t particle_count);

/* Grid preflight (preflightFireXGrid, gridConfiguration.ts:297-350): the reference's
 * checks and issue codes, one bit per code, evaluated on the host before any device
 * memory is touched. The estimate is the reference's model (as above) for
 * opt->particle_count droplets; the budget check compares it with
 * opt->memory_budget_bytes (0 = no budget check). limits NULL takes this library's own:
 * at most 2048 cells per axis and fewer than 2^31 cells (16-byte vector fields up to
 * (2^31 - 1) * 16 bytes). firex_create refuses a grid with any of the first five issues
 * (FIREX_ERR_BAD_ARG) and answers the budget with FIREX_ERR_BUDGET against its own
 * planned residency; its error text names the issue codes. */
#define FIREX_ISSUE_INVALID_DIMENSION 0x01u       /* "invalid-dimension" */
#define FIREX_ISSUE_UNALIGNED_DIMENSION 0x02u     /* "unaligned-dimension" */
#define FIREX_ISSUE_TEXTURE_DIMENSION_LIMIT 0x04u /* "texture-dimension-limit" */
#define FIREX_ISSUE_STORAGE_BINDING_LIMIT 0x08u   /* "storage-binding-limit" */
#define FIREX_ISSUE_BUFFER_SIZE_LIMIT 0x10u       /* "buffer-size-limit" */
#define FIREX_ISSUE_MEMORY_BUDGET 0x20u           /* "memory-budget" */

typedef struct firex_device_limits {
    uint64_t max_texture_dimension_3d;        /* cells per axis */
    uint64_t max_storage_buffer_binding_size; /* bytes */
    uint64_t max_buffer_size;                 /* bytes */
} firex_device_limits;

typedef struct firex_preflight_result {
    uint32_t issues;      /* FIREX_ISSUE_* bits; 0 = ok */
    uint32_t issue_count; /* issues found, one per axis for the per-axis codes */
    uint64_t cell_count, grid_bytes, particle_bytes, fixed_bytes, total_bytes, largest_storage_buffer_bytes;
    uint64_t planned_device_bytes; /* this library's residency for the grid (0 if the grid is refused) */
    char message[1024];            /* "code: message" of each issue in the reference's order, '; '-separated */
} firex_preflight_result;

int firex_preflight(const int32_t dims[3], const firex_options* opt, const firex_device_limits* limits,
                    firex_preflight_result* out);

/* CUDA stream the handle runs on (cudaStream_t as void*), for callers that order their
 * own work after a step. */
void* firex_stream(const firex_sim* sim);

/* ---- profiling (reference: per-pass encoder labels and CPU phase timers,
 * FireXEngine.ts:712-797; here CUDA events on the handle's stream) ------------------- */
#define FIREX_PASS_SIMULATE 0   /* advect/react (simulate) */
#define FIREX_PASS_DIVERGENCE 1 /* both divergence passes */
#define FIREX_PASS_JACOBI 2     /* every primary and residual Jacobi launch */
#define FIREX_PASS_PROJECT 3    /* both projections */
#define FIREX_PASS_OTHER 4      /* parameter upload and buffer clears */
#define FIREX_PASS_PARTICLES 5  /* droplet pass: liquid clear, density, integrate, deposit */
#define FIREX_PASS_COUNT 6

/* Turns per-pass event recording on (1) or off (0) for subsequent steps. */
int firex_set_profiling(firex_sim* sim, int32_t on);

/* Waits for the stream, then returns and clears the accumulated device milliseconds per
 * pass (ms[FIREX_PASS_COUNT]) and the number of kernel launches per pass
 * (launches[FIREX_PASS_COUNT]) since the previous call. Either pointer may be NULL. */
int firex_pass_times(firex_sim* sim, double* ms, int64_t* launches);

/* Device bytes firex_create would allocate for this grid and options (admission). */
uint64_t firex_planned_device_bytes(const int32_t dims[3], const firex_options* opt);

/* Replays each step from a captured CUDA graph (1, the default) or launches the passes
 * directly (0). Results are identical; graphs remove per-launch host overhead. */
int firex_set_graphs(firex_sim* sim, int32_t on);

/* Jacobi kernel choice. Every kernel computes each sweep's update with the same FP32
 * operations; they differ in how data reaches the SMs:
 *   UNBLOCKED — one thread per 4 cells, neighbours through L1 (best for small grids);
 *   ZMARCH    — x-y tiles marching z through a cp.async shared-memory ring (one read of
 *               each value per sweep: best once the grid outgrows L2);
 *   FUSED     — two sweeps per launch (`block` 2): z-marching tiles with a one-cell ring,
 *               one read of pressure and divergence per two sweeps (AUTO's choice at 8 Mi
 *               cells and above). The fused sweeps give the same results as single sweeps
 *               (with FP16 pressure storage the first sweep is rounded as a stored one). A
 *               phase falls back to single sweeps when the fused launches would leave its
 *               result in the other buffer of the pair (half its sweep count, rounded down,
 *               is odd).
 * `zchunk`: z planes per CTA for ZMARCH and FUSED (0 = auto). AUTO takes RESIDENT when the
 * batch fits on chip, else by its cell count: UNBLOCKED below 8 Mi cells, FUSED with block 2
 * and 16-plane chunks below 16 Mi, FUSED with block 2 and 64-plane chunks from 16 Mi. */
#define FIREX_JACOBI_AUTO 0
#define FIREX_JACOBI_UNBLOCKED 1
#define FIREX_JACOBI_ZMARCH 2
#define FIREX_JACOBI_FUSED 3
/* Every sweep of a phase in one cooperative launch with the pressure held in shared
 * memory (only box faces cross L2 between sweeps); used by AUTO whenever the batch fits
 * on chip, else the single-sweep default runs. With RESIDENT, `block` 1-5 restricts the
 * box plan to variant block - 1 (0 columns, 1 faces first, 2 faces first for small
 * boxes, 3 faces first with interior columns, 4 variant 3 with a copy warp that brings
 * the halo rows in by bulk asynchronous copies: FP32 pressure only); 0 lets the planner
 * choose. */
#define FIREX_JACOBI_RESIDENT 4
int firex_set_jacobi(firex_sim* sim, int32_t kernel, int32_t block, int32_t zchunk);
int firex_batch_set_jacobi(firex_batch* batch, int32_t kernel, int32_t block, int32_t zchunk);

/* How the two-sweep pass (FUSED, block 2) brings its pressure and divergence planes into
 * shared memory. TMA (FP32 pressure only): one elected thread per CTA issues tiled tensor
 * loads (cp.async.bulk.tensor) completing on per-slot mbarriers. CPASYNC: per-thread cp.async
 * copies. Both give the same results bit for bit. AUTO (the default) = CPASYNC, measured
 * faster on B200; FP16 pressure (branch B) always uses CPASYNC. A batch's own setting overrides
 * its members' (AUTO: the first member's). No reference counterpart (the reference's tiled
 * solve stages through workgroup memory, shaders.ts:405-459). */
#define FIREX_STAGING_AUTO 0
#define FIREX_STAGING_CPASYNC 1
#define FIREX_STAGING_TMA 2
int firex_set_staging(firex_sim* sim, int32_t staging);
int firex_batch_set_staging(firex_batch* batch, int32_t staging);

/* Launch shapes of the passes around the Jacobi. simulate_by: the source pass (simulate,
 * shaders.ts:151-342) runs one thread per cell of a 32 x simulate_by x (8 / simulate_by) brick,
 * simulate_by = 2, 4 (the default) or 8; 0 restores the default. project: the primary
 * projection and the divergence of its result (the residual's right-hand side,
 * FireXEngine.ts:2256-2257) run as one fused pass (FUSED) or as two (SEPARATE); AUTO fuses
 * them below 8 Mi cells per batch (the recomputed neighbours then come from L2). Unless
 * SEPARATE, a residual phase run by the resident Jacobi's variant 4 also projects the flow
 * as its epilogue (no separate projection launch; firex_diagnostics.project_resident).
 * Every choice gives identical results; fire_b200/autotune.py times them. A batch's own
 * setting overrides its members' (0 / AUTO: the first member's). */
#define FIREX_PROJECT_AUTO 0
#define FIREX_PROJECT_FUSED 1
#define FIREX_PROJECT_SEPARATE 2
int firex_set_tiles(firex_sim* sim, int32_t simulate_by, int32_t project);
int firex_batch_set_tiles(firex_batch* batch, int32_t simulate_by, int32_t project);

/* What the engine chose for the most recent step of the simulation (or its batch). */
typedef struct firex_diagnostics {
    int32_t fast_division;    /* 1: the Jacobi division uses the checked constant-divisor path */
    int32_t jacobi_block;     /* sweeps fused per Jacobi launch (1: one sweep per launch) */
    int32_t jacobi_zchunk;    /* z planes per CTA of the Jacobi launches */
    int32_t graph;            /* 1: steps replay a captured CUDA graph */
    int32_t launches_per_step;
    int32_t jacobi_kernel;    /* FIREX_JACOBI_* kernel the last step ran */
    int32_t jacobi_variant;   /* RESIDENT: the box variant (0-4) it ran; else -1 */
    int32_t jacobi_staging;   /* two-sweep pass: FIREX_STAGING_TMA or _CPASYNC it ran; else -1 */
    int32_t simulate_by;      /* source-pass bricks of 32 x simulate_by x (8 / simulate_by) cells */
    int32_t project_fused;    /* 1: the primary projection and the residual divergence ran as one pass */
    int32_t project_resident; /* 1: the residual projection ran inside the resident Jacobi's launch */
    int32_t reserved[5];
} firex_diagnostics;
int firex_get_diagnostics(const firex_sim* sim, firex_diagnostics* out);

/* ---- batches: many simulations stepped by the same launches -------------------------
 * No reference counterpart (the reference runs one simulation per WebGPU device). A batch
 * steps its members together: each pass is one persistent launch over the bricks of all
 * members, whatever their grid sizes, and the step is replayed from a CUDA graph. Members
 * must share the storage precision and the pressure storage type; their iteration counts
 * may differ. While a member, a simulation is stepped only through its batch; its field,
 * parameter and state calls stay valid and are ordered with the batch's work. */
int firex_batch_create(firex_batch** out);
int firex_batch_destroy(firex_batch* batch); /* members are detached, not destroyed */
int firex_batch_add(firex_batch* batch, firex_sim* sim);
int firex_batch_remove(firex_batch* batch, firex_sim* sim);
int firex_batch_size(const firex_batch* batch, int32_t* members);
int firex_batch_step(firex_batch* batch, int32_t nsteps, double dt);
int firex_batch_sync(firex_batch* batch);
const char* firex_batch_last_error(const firex_batch* batch);
void* firex_batch_stream(const firex_batch* batch);

#ifdef __cplusplus
}
#endif

#endif /* FIREX_H */
