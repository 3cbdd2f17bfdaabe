/*
 * dmph.h — C ABI of the B200 DEM-MPH explicit-timestep library (libdmph.so).
 *
 * The reference solver (Ryo1011gd/DEM_MPH) has no plugin or FFI layer: its
 * physics are file-static functions over file-scope globals in
 * source/DEM-MPH.cpp, called from main (source/DEM-MPH.cpp:350-617), and its
 * external contract is the process CLI plus the text formats dem.data, .grid
 * and .prof.  This header is the boundary that replaces that path: a host
 * driver (the `dem_mph` executable built from dem_mph_b200/host/, or any
 * caller over ctypes / cgo / JNI) reads the same files and calls the GPU only
 * through these entry points.  Each function below cites the reference code
 * it stands in for.
 *
 * Conventions
 *   - All arrays are caller-owned host memory, copied in or out; device
 *     buffers are owned by the context.
 *   - Vectors are interleaved x,y,z per particle (the reference's
 *     double[N][3] layout).
 *   - Every function returns 0 on success or a negative DMPH_E* code; the
 *     message is available from dmph_last_error().
 *   - One host thread per context.  Contexts are independent (re-entrant
 *     across contexts), each with its own CUDA stream.
 */
#ifndef DMPH_H_INCLUDED
#define DMPH_H_INCLUDED

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DMPH_ABI_VERSION 1
#define DMPH_TYPE_COUNT 6 /* source/DEM-MPH.cpp:46 */

/* particle classes by type (source/DEM-MPH.cpp:46-52) */
#define DMPH_FLUID_BEGIN 0
#define DMPH_FLUID_END 2
#define DMPH_SOLID_BEGIN 2
#define DMPH_SOLID_END 4
#define DMPH_WALL_BEGIN 4
#define DMPH_WALL_END 6

/* error codes */
#define DMPH_OK 0
#define DMPH_EINVAL (-1)   /* bad argument or inconsistent parameters */
#define DMPH_ECUDA (-2)    /* CUDA runtime error */
#define DMPH_ENOMEM (-3)   /* device allocation failed */
#define DMPH_EIO (-4)      /* file could not be read or written */
#define DMPH_ENAN (-5)     /* non-finite state detected */
#define DMPH_ETIMEOUT (-6) /* a bounded device wait ran out */
#define DMPH_ERANGE (-7)   /* a size limit was exceeded */

/* precision of the pair kernels */
#define DMPH_PRECISION_FP64 0       /* parity build: FP64 everywhere */
#define DMPH_PRECISION_FP32_SPLIT 1 /* FP32 pair math on cell-relative positions */

/* flags */
#define DMPH_FLAG_SURFACE_TENSION_AUTO 0u /* default: on iff an InteractionRatio != 0 */
#define DMPH_FLAG_SURFACE_TENSION_ON (1u << 0)
#define DMPH_FLAG_SURFACE_TENSION_OFF (1u << 1)
#define DMPH_FLAG_WALL_DEM_COEFFS (1u << 2) /* also compute the (output-only) DEM constants of wall particles */
#define DMPH_FLAG_RIGID_CLUMPS (1u << 3)    /* debris bodies move as rigid clumps (no reference counterpart) */
#define DMPH_FLAG_ALL_NEIGHBOR_COUNTS (1u << 4) /* keep NeighborCount for every particle (VTK "neighbor") */
/* FP32 split build, Verlet lists: keep the lists across the reference's
 * rebuild triggers while they stay valid (no reference counterpart; see
 * dmph_get_rebuild_stats) */
#define DMPH_FLAG_LIST_REUSE (1u << 5)

/*
 * Simulation parameters: the keywords of dem.data
 * (readDataFile, source/DEM-MPH.cpp:621-679) plus the grid header
 * (readGridFile, source/DEM-MPH.cpp:689-702).  RadiusRatioG is forced equal
 * to RadiusRatioA as in the reference (source/DEM-MPH.cpp:1009).
 */
typedef struct dmph_params {
    int32_t dim;       /* 2: the reference's TWO_DIMENSIONAL build (source/DEM-MPH.cpp:39); 3: the 3D branches */
    int32_t precision; /* DMPH_PRECISION_* */
    uint32_t flags;    /* DMPH_FLAG_* */
    int32_t reserved0;
    double dt;
    double dem_dt;
    double output_interval;
    double vtk_output_interval;
    double end_time;
    double radius_ratio_a;
    double radius_ratio_p;
    double radius_ratio_v;
    double density[DMPH_TYPE_COUNT];
    double bulk_modulus[DMPH_TYPE_COUNT];
    double bulk_viscosity[DMPH_TYPE_COUNT];
    double shear_viscosity[DMPH_TYPE_COUNT];
    double surface_tension[DMPH_TYPE_COUNT];
    double interaction_ratio[DMPH_TYPE_COUNT][DMPH_TYPE_COUNT];
    double gravity[3];
    double young_modulus[DMPH_TYPE_COUNT];
    double poisson_ratio[DMPH_TYPE_COUNT];
    double restitution_coefficient[DMPH_TYPE_COUNT];
    double viscous_friction_coefficient[DMPH_TYPE_COUNT];
    double wall_center[DMPH_TYPE_COUNT][3];
    double wall_velocity[DMPH_TYPE_COUNT][3];
    double wall_omega[DMPH_TYPE_COUNT][3];
    /* grid-file header */
    double time;
    double particle_spacing;
    double domain_min[3];
    double domain_max[3];
} dmph_params;

typedef struct dmph_ctx dmph_ctx;

/* ---------------------------------------------------------------- host I/O */

/* Fill defaults (the reference's static initialisers, source/DEM-MPH.cpp:61-75,
 * 159, 238-250) into *p: dt = dem_dt = 1e100, everything else 0, dim = 3. */
void dmph_params_default(dmph_params *p);

/* Parse a dem.data keyword file into *p (readDataFile, source/DEM-MPH.cpp:621-679).
 * '#' lines are comments; unknown lines are reported through
 * dmph_io_last_message() and ignored, like the reference. */
int dmph_read_data_file(const char *path, dmph_params *p);

/* Read a .grid / .prof file (readGridFile, source/DEM-MPH.cpp:681-851).
 * First call with type == NULL to get *n; then call again with arrays of n
 * (type) and 3n (x3, v3) elements.  The header fills p->time,
 * p->particle_spacing, p->domain_min/max. */
int dmph_read_grid_file(const char *path, dmph_params *p, int *n, int *type, double *x3, double *v3);

/* Write a .prof file (writeProfFile, source/DEM-MPH.cpp:853-877): same
 * header and "%d %e %e %e  %e %e %e" rows, particles in the solver's current
 * (sorted) order. */
int dmph_write_prof_file(const char *path, const dmph_params *p, int n, const int *type, const double *x3,
                         const double *v3);

/* Write a VTK file (writeVtkFile, source/DEM-MPH.cpp:879-1005): legacy ASCII
 * unstructured grid, point data label, the four DEM constants, neighbor,
 * volumef, drag, velocity, VolStrainP, VirialPressureAtParticle in the
 * reference's order and formats; arrays in the solver's current order. */
int dmph_write_vtk_file(const char *path, int n, const int *type, const double *x3, const double *v3,
                        const double *kn, const double *cn, const double *kt, const double *ct,
                        const int *neighbor_count, const double *alpha, const double *drag,
                        const double *vol_strain, const double *virial_pressure);

/* Last informational message of the I/O layer (invalid data-file lines). */
const char *dmph_io_last_message(void);

/* ------------------------------------------------------------ solver context */

/*
 * Create a solver on the current CUDA device and upload the particles.
 * Replaces the initialisation of main (source/DEM-MPH.cpp:370-426):
 * initializeWeight :1007, initializeFluid :1128, initializeWall :1166,
 * initializeDomain :1207, then the first cell sort, neighbour build and
 * density evaluation (:419-425).
 */
int dmph_create(const dmph_params *p, int n, const int *type, const double *x3, const double *v3, dmph_ctx **out);

/* Advance nsteps explicit steps: one iteration of the reference main loop
 * (source/DEM-MPH.cpp:450-579) each, without file output.
 * Failure detection (no counterpart in the reference, which runs on with NaN):
 * every step's drift also checks every position and velocity; a non-finite
 * one sets a device flag, from then on no neighbour rebuild runs (so no
 * non-finite position ever becomes a cell index), and the call returns
 * DMPH_ENAN (checked every 256 steps and at the end of the call).  Later
 * calls return DMPH_ENAN at once until dmph_set_state replaces the state. */
int dmph_step(dmph_ctx *ctx, int nsteps);

/* Same as dmph_step, and report the device time of the nsteps as measured by
 * CUDA events recorded on the context's stream. */
int dmph_step_timed(dmph_ctx *ctx, int nsteps, float *device_ms);

/* One step split at the rebuild decision, for drivers that decide it over
 * several contexts (a domain split into slabs, one context per rank: the
 * reference's trigger, source/DEM-MPH.cpp:1264-1286, is a maximum over all
 * particles, so the ranks combine their maxima and rebuild together).
 * dmph_step_begin runs the drift, wall motion, periodic wrap and force reset
 * of one step (:1860, :2846, :3153, :1894) and reports the largest squared
 * displacement since the last rebuild (+inf when a position or velocity is
 * not finite); dmph_step_finish(rebuild) completes the step: the neighbour
 * rebuild when rebuild != 0 (never on a non-finite state: DMPH_ENAN), the
 * passes, the fluid update and the DEM substeps.  No graph replay.  On a
 * context that has not stepped yet, dmph_step_finish(ctx, 0) alone completes
 * the step whose drift was applied to the state it was created from (its
 * creation sorted the particles and built the lists: that step's rebuild). */
int dmph_step_begin(dmph_ctx *ctx, double *max_shift2);
int dmph_step_finish(dmph_ctx *ctx, int rebuild);

/* Positions and velocities (3 per row, either pointer may be NULL) of the
 * given input-grid rows (orig_id), read or overwritten; a write takes effect
 * at the next step (the ghost particles of a slab decomposition are refreshed
 * this way from the ranks that own them). */
int dmph_get_rows(dmph_ctx *ctx, int count, const int *rows, double *x3, double *v3);
int dmph_set_rows(dmph_ctx *ctx, int count, const int *rows, const double *x3, const double *v3);

/* Copy the particle state to host arrays in the solver's current (sorted)
 * order.  Any pointer may be NULL.  orig_id is the reference's ParticleIndex
 * (source/DEM-MPH.cpp:82): the row of the particle in the input grid. */
int dmph_get_state(dmph_ctx *ctx, int *type, double *x3, double *v3, int *orig_id);

/* Overwrite positions and velocities (current order, 3n each).  Used by
 * host-driven coupling loops; takes effect at the next step, and clears the
 * non-finite flag of dmph_step (the next step checks the new state). */
int dmph_set_state(dmph_ctx *ctx, const double *x3, const double *v3);

/* Checkpoint for an exact resume.  The reference restarts from a .prof file
 * (source/DEM-MPH.cpp:433, :690, :853-877) and so loses what the file does not
 * hold: the positions of the last neighbour rebuild (the trigger's
 * NeighborCalculatedPosition), the sorted order and the neighbour lists of
 * that rebuild, the DEM constants, the wall centres and the body states; a
 * run resumed from it follows another trajectory.  dmph_checkpoint_write
 * saves all of the context's device state and its clock (time, step and
 * rebuild counts, wall centres, launch settings) to one binary file, with
 * the parameters, the particle types and rows and the rigid-body membership,
 * plus up to DMPH_CHECKPOINT_USER_MAX bytes of the caller's own (e.g. its
 * output schedule).  dmph_checkpoint_open creates a context on the current
 * device from such a file; stepping it gives the same bits as stepping the
 * context that wrote the file.  The file is native (little-endian, this
 * library's structure layouts) and about as large as the context's device
 * memory.  Not saved: a surrogate (dmph_surrogate_enable), profiling and
 * graph settings.  Write fails with DMPH_ENAN on a state dmph_step has
 * flagged non-finite and with DMPH_EINVAL between dmph_step_begin and
 * dmph_step_finish; open fails with DMPH_EIO on a truncated or foreign file
 * and with DMPH_EINVAL when user_capacity is smaller than the saved bytes. */
#define DMPH_CHECKPOINT_USER_MAX 4096
int dmph_checkpoint_write(dmph_ctx *ctx, const char *path, const void *user, int user_bytes);
int dmph_checkpoint_open(const char *path, dmph_ctx **out, void *user, int user_capacity, int *user_bytes);

/* Per-particle fields, current order; `out` holds n (scalars) or 3n (vectors)
 * values of the type given beside each id. */
enum dmph_field {
    DMPH_FIELD_FORCE = 0,               /* double[3n]  Force :87 */
    DMPH_FIELD_VOL_STRAIN_P = 1,        /* double[n]   VolStrainP :141 */
    DMPH_FIELD_DIVERGENCE_P = 2,        /* double[n]   DivergenceP :142 */
    DMPH_FIELD_PRESSURE_P = 3,          /* double[n]   PressureP :143 */
    DMPH_FIELD_DENSITY_A = 4,           /* double[n]   DensityA :138 */
    DMPH_FIELD_GRAVITY_CENTER = 5,      /* double[3n]  GravityCenter :139 */
    DMPH_FIELD_PRESSURE_A = 6,          /* double[n]   PressureA :140 */
    DMPH_FIELD_NORMAL_SPRING = 7,       /* double[n]   NormalSpringConstant :190 */
    DMPH_FIELD_NORMAL_DAMPING = 8,      /* double[n]   NormalViscousDampingConstant :192 */
    DMPH_FIELD_TANGENTIAL_SPRING = 9,   /* double[n]   TangentialSpringConstant :191 */
    DMPH_FIELD_TANGENTIAL_DAMPING = 10, /* double[n]   TangentialViscousDampingConstant :193 */
    DMPH_FIELD_ALPHA = 11,              /* double[n]   alpha (solid volume fraction) :194 */
    DMPH_FIELD_DRAG_C = 12,             /* double[n]   DragC :195 */
    DMPH_FIELD_NEIGHBOR_COUNT = 13,     /* int32[n]    NeighborCount :88 (rebuild time) */
    DMPH_FIELD_SOLID_NEIGHBOR_COUNT = 14, /* int32[n]  SolidNeighborCount :94 (rebuild time) */
    DMPH_FIELD_CELL_INDEX = 15,         /* int32[n]    sorted cell key CellIndex :121 */
    DMPH_FIELD_MASS = 16,               /* double[n]   Mass :84 */
    DMPH_FIELD_VIRIAL_PRESSURE = 17,    /* double[n]   VirialPressureAtParticle :147, computed on request
                                           from the current state (calculateVirialStressAtParticle :2904) */
    DMPH_FIELD_COUNT_ = 18
};
int dmph_get_field(dmph_ctx *ctx, int field_id, void *out);

/* Scalars of the context. */
typedef struct dmph_info {
    int32_t n;                 /* ParticleCount */
    int32_t n_fluid, n_solid, n_wall;
    int32_t cell_count[3];     /* CellCount :116 */
    int32_t total_cell_count;  /* TotalCellCount :117 */
    int32_t power_count;       /* PowerParticleCount :113 */
    int32_t dem_substeps;      /* (int)(Dt/DEMDt) :434 */
    int64_t steps;             /* steps advanced since create */
    int64_t rebuilds;          /* neighbour rebuilds since create (the initial one excluded) */
    double time;               /* Time :69 */
    double cell_width[3];      /* CellWidth :115 */
    double n0a, n0p, r2g;      /* :248-250 */
    double max_radius;         /* MaxRadius :238 */
    int32_t num_bodies;        /* rigid clumps (0 unless DMPH_FLAG_RIGID_CLUMPS) */
    int32_t surface_tension;   /* 1 if the surface-tension passes run */
    int64_t kernel_launches;   /* kernels this library launched in dmph_step calls since create */
} dmph_info;
int dmph_get_info(dmph_ctx *ctx, dmph_info *info);

/* The parameters the context was created with, `time` set to its current
 * Time (a context opened from a checkpoint gives those of the context that
 * wrote it). */
int dmph_get_params(dmph_ctx *ctx, dmph_params *out);

/*
 * Neighbour list in the reference's CSR form (calculateNeighbor,
 * source/DEM-MPH.cpp:1521-1851): for every particle, all particles within
 * MaxRadius+MARGIN at the last rebuild, fluid then solid then wall cells of
 * the periodic 3x3(x3) stencil; ptr has n+1 entries.  Call first with
 * ind == NULL to get the total count in *ptr[n].  This CSR copy is made on
 * demand, so the neighbour sets can be checked against the reference; the
 * timestep keeps its own per-particle lists (dmph_set_pair_mode).
 */
int dmph_get_neighbor_list(dmph_ctx *ctx, int64_t *ptr, int32_t *ind, int64_t capacity);

/*
 * Global sums over the fluid and debris particles (no counterpart in the
 * reference): total mass, momentum, kinetic energy 0.5 m |v|^2 and the
 * potential energy of gravity -m g.x, in FP64 on the GPU with a fixed-order
 * reduction (the same bits on every call for the same state).  In the FP32
 * build the fluid's positions and velocities are widened from the FP32
 * state, the debris use their FP64 master state.  Debris masses are their
 * body's density times the particle volume in rigid-body mode.
 */
enum {
    DMPH_SUM_MASS = 0,
    DMPH_SUM_MOMENTUM_X = 1,
    DMPH_SUM_MOMENTUM_Y = 2,
    DMPH_SUM_MOMENTUM_Z = 3,
    DMPH_SUM_KINETIC = 4,
    DMPH_SUM_POTENTIAL = 5,
    DMPH_SUM_COUNT = 6
};
int dmph_get_global_sums(dmph_ctx *ctx, double sums[DMPH_SUM_COUNT]);

/*
 * Size of the pair work of the current Verlet lists (no counterpart in the
 * reference): the entries pass A walks (all particles with a list) and those
 * pass B walks (fluid and debris).  In the FP32 build, lists made with the
 * walls at rest hold no wall-wall pairs.  *overflowed = 1 when a list of the
 * last rebuild outgrew its capacity (the steps then walk the stencil until
 * the next rebuild, and the counts are those of the truncated lists).  Any
 * pointer may be NULL; all read 0 in stencil mode.
 */
int dmph_get_list_stats(dmph_ctx *ctx, int64_t *entries_pass_a, int64_t *entries_pass_b, int32_t *overflowed);

/*
 * List reuse (DMPH_FLAG_LIST_REUSE, FP32 split build with Verlet lists, walls
 * at rest, debris as rigid bodies or none, without
 * DMPH_FLAG_ALL_NEIGHBOR_COUNTS; otherwise the flag only widens the cells).  The reference rebuilds at every
 * trigger of its displacement test (neighborCalculation :1264-1286): cell
 * sort, NeighborInd, and the neighbour counts the drag terms read.  With the
 * flag, the cells are MaxRadius + 0.4 dx wide (instead of MaxRadius + MARGIN)
 * and each list is
 * built with a skin S of 0.1 or 0.4 dx past MaxRadius (chosen on the device
 * from how many steps lay between the last two triggers: the wide skin when
 * they come at most four steps apart).  Every trigger still resets the
 * trigger positions and recounts NeighborCount and SolidNeighborCount within
 * MaxRadius + MARGIN (from the lists, on the FP64 positions); the cell sort
 * and the lists are remade only when some particle has moved more than
 * S/2 - MARGIN/2 since the lists were built, so that until the next trigger
 * (which comes before any particle moves MARGIN/2 further) every pair within
 * MaxRadius + MARGIN is in the lists.  The physics is the reference's; the
 * order of a cell's particles, and so the order of the neighbour sums, is
 * that of the last sort.  *triggers counts the reference's rebuilds (as
 * dmph_info.rebuilds), *list_builds the cell sorts and list builds among them.
 */
int dmph_get_rebuild_stats(dmph_ctx *ctx, int64_t *triggers, int64_t *list_builds);

/*
 * Rigid debris bodies (no counterpart in the reference, whose debris particles
 * move individually, source/DEM-MPH.cpp:1872-1891).  body_of_row[r] is the body
 * of input-grid row r (-1: none); every solid particle must belong to a body.
 * body_density[b] replaces the type density for the particles of body b.
 * Mass, centre of mass, inertia tensor, velocity and angular momentum of each
 * body are computed from its particles' current state (FP64); from the next
 * step on, DEM substeps move each body rigidly (translation + quaternion
 * rotation in FP64) under the sum of its particles' fluid and contact forces.
 * Call once, before the first dmph_step.
 */
int dmph_set_bodies(dmph_ctx *ctx, int nbodies, const int *body_of_row, const double *body_density);

/*
 * Rigid bodies at the drop-in boundary (no counterpart in the reference,
 * whose .grid rows carry no body and whose two solid types are its only
 * densities, generator/generator.cpp:97, 211-214).  A body sidecar file beside
 * the .grid gives each body's density and each grid row's body:
 *     DMPH_BODIES 1
 *     <nbodies> <nrows>
 *     <density of body b>        nbodies lines
 *     <body of grid row r>       nrows lines, -1 for no body
 * dmph_read_bodies_file: call with body_of_row == NULL to get the counts;
 * then with arrays of *nrows and *nbodies entries (their sizes passed in
 * *nrows and *nbodies).  dmph_bodies_from_contacts: without a sidecar, the
 * bodies are the connected components of the solid rows under contact at
 * 1.01 dx (periodic minimum image), numbered by their first row, each with
 * the density of its first row's type; body_of_row has n entries,
 * body_density (optional) density_capacity.  Messages of the three calls:
 * dmph_bodies_last_message().
 */
int dmph_write_bodies_file(const char *path, int nbodies, int nrows, const int *body_of_row,
                           const double *body_density);
int dmph_read_bodies_file(const char *path, int *nbodies, int *nrows, int *body_of_row, double *body_density);
int dmph_bodies_from_contacts(const dmph_params *p, int n, const int *type, const double *x3, int *body_of_row,
                              int *nbodies, double *body_density, int density_capacity);
const char *dmph_bodies_last_message(void);

/* Body state, each pointer optional: X,V,L 3 per body (centre of mass,
 * velocity, angular momentum), q 4 per body (w,x,y,z), mass 1 per body,
 * F,T 3 per body (total force and torque of the last substep). */
int dmph_get_bodies(dmph_ctx *ctx, double *X, double *V, double *q, double *L, double *mass, double *F, double *T);

/* How pass A and pass B find their pairs:
 *  DMPH_PAIRS_VERLET_LIST (default): at every rebuild each particle records
 *    the particles within the reference's list radius MaxRadius + MARGIN
 *    (calculateNeighbor, source/DEM-MPH.cpp:1521-1851) in ascending order, at
 *    most 192 (3D) or 64 (2D) (in the FP64 build exactly the reference's
 *    NeighborInd); the passes then walk the lists (FP32: one thread per
 *    particle).  A list that would overflow makes the step fall back to the
 *    stencil kernels until the next rebuild.  Results are bit-identical to
 *    the stencil walk in the FP64 build.
 *  DMPH_PAIRS_STENCIL: every pass walks the 27 (9) cells of the stencil. */
#define DMPH_PAIRS_STENCIL 0
#define DMPH_PAIRS_VERLET_LIST 1
int dmph_set_pair_mode(dmph_ctx *ctx, int mode);

/* Record a step as one CUDA graph and replay it (enable != 0): the rebuild
 * decision is taken on the device and the neighbour rebuild runs as the body
 * of a conditional graph node, so steps need no host synchronisation.  Steps
 * that cannot use the recorded graph (Time <= 0, the moving-wall window
 * 0.2 <= Time <= 0.4 of calculateWall :2857, or profiling on) fall back to
 * individual launches.  Results are identical either way. */
int dmph_set_graph(dmph_ctx *ctx, int enable);

/* Autotuner of the FP32 pair passes: times every launch variant (warps per
 * block x resident blocks per SM requested from the register allocator) of
 * pass A and pass B on the current state and keeps the fastest for the
 * following steps.  Reports the chosen variants and, when ms_a/ms_b are
 * non-NULL, the time of each of DMPH_PASS_VARIANTS variants.  In Verlet-list
 * mode (dmph_set_pair_mode) the variants are those of the list passes
 * (entries loaded per batch x resident blocks, DMPH_LIST_VARIANTS of them)
 * and dmph_set_variants sets those.  The passes only read the state, so
 * tuning changes no result.  FP32 split build only. */
#define DMPH_LIST_VARIANTS 4
#define DMPH_PASS_VARIANTS 5
int dmph_autotune(dmph_ctx *ctx, int *variant_a, int *variant_b, float *ms_a, float *ms_b);
int dmph_set_variants(dmph_ctx *ctx, int variant_a, int variant_b);

/* Autotuner of the FP32 list build (Verlet-list mode): advances
 * steps_per_variant steps with each of DMPH_BUILD_VARIANTS launch variants of
 * the list build (warps per block x resident blocks per SM) and the phase
 * timer on, and keeps the variant whose rebuilds' list build was fastest.
 * All variants build the same lists, so the steps are ordinary steps; ms[v]
 * (optional) gets variant v's mean list-build time, -1 when its steps had no
 * rebuild.  Runs without graph replay; the setting of dmph_set_graph holds
 * again afterwards. */
#define DMPH_BUILD_VARIANTS 3
int dmph_autotune_list_build(dmph_ctx *ctx, int steps_per_variant, int *variant, float *ms);

/* Ensemble of independent scenes (no counterpart in the reference, which runs
 * one scene per process).  Every scene keeps its own context, parameters,
 * cell grid and state; an ensemble step advances all of them by one step:
 * each scene's drift and rebuild decision (with its own conditional rebuild),
 * then pass A and pass B of ALL scenes as one persistent launch each over the
 * concatenated chunk lists, then each scene's DEM substeps or rigid bodies.
 * With graph replay on (the default) a whole ensemble step is one CUDA graph.
 * Results are bit-identical to stepping each scene alone.  Scenes must be FP32
 * split contexts on one device, at most 256, each in at most one ensemble;
 * set their bodies before creating the ensemble and step them only through it
 * while it exists. */
typedef struct dmph_ensemble dmph_ensemble;
int dmph_ensemble_create(dmph_ctx *const *scenes, int nscenes, dmph_ensemble **out);
int dmph_ensemble_step(dmph_ensemble *e, int nsteps);
int dmph_ensemble_step_timed(dmph_ensemble *e, int nsteps, float *device_ms);
int dmph_ensemble_autotune(dmph_ensemble *e, int *variant_a, int *variant_b, float *ms_a, float *ms_b);
int dmph_ensemble_set_graph(dmph_ensemble *e, int enable);
int dmph_ensemble_info(dmph_ensemble *e, int64_t *kernel_launches, int64_t *steps);
/* Per-phase device timing of the ensemble's shared launches (no graph replay
 * while on): phase 2 = pass A of all scenes, 3 = pass B of all scenes, in the
 * indexing of dmph_get_phase_times; other phases read 0. */
int dmph_ensemble_set_profiling(dmph_ensemble *e, int enable);
int dmph_ensemble_get_phase_times(dmph_ensemble *e, double *ms, int64_t *launches, int n);
const char *dmph_ensemble_last_error(dmph_ensemble *e);
int dmph_ensemble_destroy(dmph_ensemble *e); /* NULL: nothing to do, returns 0 */

/* Learned surrogate of K solver steps (no counterpart in the reference).
 * FP32 split build only.  A surrogate call evaluates pass A and pass B at the
 * current state, computes 52 cell-list aggregated features per fluid and
 * debris particle, runs a 64-128-128-128-16 MLP (BF16 on the tensor cores,
 * FP32 accumulation) predicting the K-step velocity increment dv of each
 * fluid particle (outputs 0-2: (dv / (K dt) - a0) / (|g| / 16), a0 its
 * acceleration at the block start; outputs 3-15 unused), and applies it to
 * the fluid with the displacement K dt v0 + (K - 1) dt dv / 2; debris advance
 * by the solver's own DEM or rigid-body substeps with the fluid force of the
 * block start held; walls stay.  The network is
 * trained (Adam, FP32 master weights) on samples the solver generates:
 * dmph_surrogate_collect runs plain K-step blocks and records (features,
 * increments) of a sampled subset of particles into a pool.
 * dmph_surrogate_advance(ctx, n) advances n blocks of K steps: surrogate
 * calls, except that every check_interval calls one block runs on the plain
 * solver as the judge; if the relative L2 error of the predicted velocity
 * increments of that block (each particle weighted by 1 + 20 |v0|^2 / vs^2,
 * vs = c0 / 10, so that the fast particles of the surge front count) exceeds
 * `tolerance`, the next fallback_blocks
 * blocks run plain (collecting and training with train_iters_per_block Adam
 * steps each).  Blocks at Time <= 0, and blocks that reach into the
 * moving-wall window while a wall type actually moves, run plain too. */
typedef struct dmph_surrogate_params {
    int substeps;              /* K (8) */
    int check_interval;        /* surrogate calls between two judged blocks (50) */
    double tolerance;          /* judged velocity-increment error that triggers the fallback (0.02) */
    int fallback_blocks;       /* plain blocks after a fallback (50) */
    int train_iters_per_block; /* Adam steps per plain block during a fallback (4) */
    int batch;                 /* training batch, a multiple of 8192 (65536) */
    int pool_rows;             /* sample pool capacity, >= batch (4,194,304) */
    float learning_rate;       /* Adam (1e-3) */
    unsigned long long seed;   /* initial weights */
    int residual;              /* 1: learn dv - K dt a0 (a0 = acceleration at the block start), 0: dv (1) */
    /* surge-front judge (0: off, the default): fall back when the estimated
     * deviation of the surge front (the x below which 99% of the fluid lies)
     * exceeds this fraction of the front's travel since the first call.  At
     * every judged block the network's prediction of that block is compared
     * with the plain solver's: the front's position, and the x-velocity of
     * the fluid in the front's 1%, whose error persists into the calls that
     * follow; each of the n calls since the previous judged block is taken
     * to have made the position error plus the velocity error times
     * n K Dt / 2, and the estimate adds them up (reset at a fallback).
     * tolerance <= 0 switches the velocity-increment judge off. */
    double front_tolerance;
} dmph_surrogate_params;

typedef struct dmph_surrogate_stats {
    int64_t calls;        /* surrogate calls (blocks advanced by the network) */
    int64_t plain_blocks; /* blocks advanced by the plain solver (collect, judge, fallback) */
    int64_t judged;       /* judged blocks */
    int64_t fallbacks;    /* fallbacks triggered */
    int64_t samples;      /* samples ever appended to the pool */
    int64_t train_iters;  /* Adam steps */
    int64_t pool_rows;    /* samples currently in the pool */
    int in_fallback;      /* 1 while plain blocks of a fallback remain */
    double last_error;    /* last judged relative L2 error of the displacements */
    double last_error_v;  /* same for the velocity increments (the fallback criterion) */
    double last_loss;     /* mean squared error of the last training batch */
    double last_front_dev;   /* surge-front deviation of the last judged block (m) */
    double front_estimate;   /* the front judge's estimate, as a fraction of the front's travel */
} dmph_surrogate_stats;

int dmph_surrogate_params_default(dmph_surrogate_params *p);
int dmph_surrogate_enable(dmph_ctx *ctx, const dmph_surrogate_params *p);
int dmph_surrogate_collect(dmph_ctx *ctx, int nblocks);
int dmph_surrogate_train(dmph_ctx *ctx, int iters, float *loss);
/* The training pool as host rows, and rows added to it (a corpus recorded on
 * other scenes, dem_mph_b200/corpus.py): X capacity x 64 FP32 (features,
 * BF16 in the pool), T capacity x 16 FP32 (targets, the first 6 meaningful);
 * get copies min(pool rows, capacity) rows, oldest first, into *rows; add
 * appends n rows to the pool's ring (the last pool_rows of them stay). */
int dmph_surrogate_get_samples(dmph_ctx *ctx, float *X, float *T, int capacity, int *rows);
int dmph_surrogate_add_samples(dmph_ctx *ctx, const float *X, const float *T, int n);
int dmph_surrogate_advance(dmph_ctx *ctx, int nblocks);
int dmph_surrogate_get_stats(dmph_ctx *ctx, dmph_surrogate_stats *out);
/* parameters: weights [out][in] then biases of each layer, FP32; with w NULL
 * returns the parameter count */
int dmph_surrogate_get_weights(dmph_ctx *ctx, float *w, int count);
int dmph_surrogate_set_weights(dmph_ctx *ctx, const float *w, int count);
/* the network on host rows: X n x 64 (FP32, rounded to BF16 on upload),
 * Y n x 16 FP32 (first 6 meaningful); n <= particle count.  The fused
 * forward kernel of the surrogate calls (weights resident in shared memory,
 * TMA-fed feature tiles, activations kept on chip); _layers runs the same
 * network through one GEMM launch per layer, as training does. */
int dmph_mlp_forward(dmph_ctx *ctx, const float *X, int n, float *Y);
int dmph_mlp_forward_layers(dmph_ctx *ctx, const float *X, int n, float *Y);
/* device milliseconds of one forward pass over the first n rows of the
 * features the surrogate holds, averaged over reps (layers: the per-layer
 * GEMMs instead of the fused kernel) */
int dmph_mlp_forward_timed(dmph_ctx *ctx, int n, int reps, int layers, float *ms);
/* mean squared error over the first 6 outputs and the parameter gradient of
 * one batch of host rows (n = the training batch) */
int dmph_mlp_gradient(dmph_ctx *ctx, const float *X, const float *T, int n, float *grad, float *loss);
/* features of the current state for the fluid and debris slots, rows x 52 */
int dmph_surrogate_features(dmph_ctx *ctx, float *F, int *rows);

/* Per-phase device timing.  With enable != 0, every following step records
 * CUDA events on the context's stream around each phase (this adds event
 * overhead, so time throughput with it off); dmph_get_phase_times returns the
 * accumulated milliseconds and launch counts per phase since it was enabled:
 * index 0 drift, 1 rebuild, 2 pass A, 3 pass B, 4 DEM substeps, 5 rigid
 * bodies, 6 the neighbour-list build alone (list mode; part of 1). */
#define DMPH_PHASE_COUNT 7
int dmph_set_profiling(dmph_ctx *ctx, int enable);
int dmph_get_phase_times(dmph_ctx *ctx, double *ms, int64_t *launches, int n);

/*
 * Allocation-free cell sort.  No counterpart in the reference: it serves
 * callers that cannot call cudaMalloc (work recorded while a stream is being
 * captured into a CUDA graph, hosts whose framework owns every device
 * allocation, real-time loops that must not enter the allocator).  It runs the
 * neighbour-rebuild sort of calculateCellParticle (cell key with class offset
 * and the reference's bitonic network) on the caller's stream and allocates
 * nothing: its scratch space is a file-scope device array of
 * DMPH_NOALLOC_MAX_WORDS 64-bit words (4 MiB) that every GPU loading the
 * library keeps until the process exits, so n must stay below
 * DMPH_NOALLOC_MAX_WORDS (n <= 524287).
 *   pos_planes  device, 3n doubles: x[0..n), y[0..n), z[0..n)
 *   type        device, n ints
 *   sorted_key  device, n ints out: the sorted keys (CellIndex)
 *   perm        device, n ints out: input row of each sorted slot
 *   stream      cudaStream_t (NULL = legacy default stream)
 * Set-up: the first call on a device, and the first call after that
 * device's CUDA context was replaced (cudaDeviceReset, a primary context
 * released and made again), looks up the scratch array's device address
 * (cudaGetSymbolAddress) with that device current and caches it with the
 * context's id; make that first call before any stream capture.  All calls
 * share the one array and it keeps the last call's contents, so calls whose
 * work overlaps on the GPU (other streams, other host threads) race;
 * serialise them.  Returns DMPH_ERANGE when n is too large, and DMPH_ECUDA
 * without running anything when a CUDA error of earlier work is pending on
 * the calling thread (that error is left for its owner to read).  On any
 * failure dmph_last_error(NULL), on the calling thread, gives the reason.
 */
#define DMPH_NOALLOC_MAX_WORDS (1 << 19)
int dmph_cell_sort_noalloc(const dmph_params *p, int n, const double *pos_planes, const int *type,
                           int32_t *sorted_key, int32_t *perm, void *stream);

/* Release the context and its device memory (NULL: nothing to do, returns 0). */
int dmph_destroy(dmph_ctx *ctx);

/* Message of the last failing call on ctx (or of the last failing
 * dmph_create when ctx is NULL).  Never NULL. */
const char *dmph_last_error(dmph_ctx *ctx);

/* Library build string (compiler, arch), never NULL. */
const char *dmph_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DMPH_H_INCLUDED */
