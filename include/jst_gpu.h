/*
 * jst_gpu.h — C ABI of the B200 (sm_100a) implementation of PurineCFD's
 * explicit JST + Spalart-Allmaras RANS loop (the jst-rs `Solver`).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns a jst_status.  Each handle is single-threaded (like the reference's
 * `&mut Solver`); separate handles may be used from separate threads.  All
 * cell arrays crossing the boundary are the interior NI x NJ cells, i-major /
 * j-minor (the order of the reference's golden data and `result.csv`), where
 * i is the radial ring index (0 = wall) and j the circumferential index.
 *
 * Citations are file:line in the reference's jst-rs crate; each entry point
 * names the Rust interface it replaces.
 */
#ifndef JST_GPU_H
#define JST_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct jst_solver jst_solver;

/* Status codes.  The JST_ERR_MESH_* values map one-to-one onto the
 * reference's MeshError variants (mesh.rs:17-44); JST_ERR_CONFIG is its
 * io::Error(InvalidData) from Config::from_str (config.rs:165-170);
 * JST_ERR_NONPHYSICAL is NonPhysical (state.rs:242-257). */
typedef enum {
    JST_OK = 0,
    JST_ERR_MESH_IO = 1,
    JST_ERR_MESH_BAD_HEADER = 2,
    JST_ERR_MESH_EMPTY = 3,
    JST_ERR_MESH_COUNT_MISMATCH = 4,
    JST_ERR_MESH_BAD_POINT = 5,
    JST_ERR_MESH_TOO_SMALL = 6,
    JST_ERR_CONFIG = 7,
    JST_ERR_NONPHYSICAL = 8,
    JST_ERR_CUDA = 9,
    JST_ERR_TIMEOUT = 10,
    JST_ERR_OOM = 11,
    JST_ERR_ARG = 12
} jst_status;

/* Arithmetic of the stage kernels. */
typedef enum {
    JST_PREC_FP64 = 0,      /* everything in FP64 (the reference's arithmetic) */
    JST_PREC_FP32_SPLIT = 1 /* FP32 fluxes/dissipation/gradients/SA; FP64 metrics,
                               wall distance, U_n accumulator, reductions */
} jst_precision;

/* Time step used by the RK update. */
typedef enum {
    JST_DT_GLOBAL = 0, /* every cell advances with the global minimum step (solver.rs:110-116) */
    JST_DT_LOCAL = 1   /* each cell advances with its own CFL step (steady-state acceleration) */
} jst_dt_mode;

/* How the marching-strip stage kernels stage each row's inputs in shared
 * memory (no counterpart in the reference).  Both give the same results. */
typedef enum {
    JST_STAGING_AUTO = 0,     /* the autotuner's choice (per-lane copies when the tile is given) */
    JST_STAGING_PER_LANE = 1, /* one cp.async per lane and field */
    JST_STAGING_BULK = 2      /* one cp.async.bulk (TMA) copy per field's row segment, completed on an
                                 mbarrier with a bounded wait (rings whose width is not a multiple of
                                 16 bytes, or under 36 columns, fall back to per-lane copies) */
} jst_staging;

/* Which kernels run a stage. */
typedef enum {
    JST_PATH_FUSED = 0, /* one stage kernel per RK stage (production): warp-marching
                           strips or shared-memory tiles, chosen by the autotuner */
    JST_PATH_PASSES = 1 /* one kernel per reference pass, strict FP64 (parity mode) */
} jst_kernel_path;

typedef struct {
    int precision;   /* jst_precision */
    int dt_mode;     /* jst_dt_mode */
    int kernel_path; /* jst_kernel_path */
    int device;      /* CUDA device ordinal */
    int tile_i;      /* fused path: tile rows, or maximum strip height when tile_j == 26 */
    int tile_j;      /* fused path: tile columns; 26 selects the marching strips (0, 0 = autotuned) */
    int use_graph;   /* capture each RK step as a CUDA graph (fused path) */
    double nut_inf_ratio; /* free-stream nu-tilde / nu; <= 0 uses the config value or 0.1 */
    int block_threads;    /* fused path threads per block (0 = default for the tile) */
    int staging;          /* jst_staging of the marching strips */
} jst_opts;

/* Fills opts with the defaults: FP64, global dt, fused path, device 0,
 * autotuned tiles, graphs on, nu-tilde ratio from the config. */
void jst_default_opts(jst_opts* opts);

/* Solver::from_paths (solver.rs:64-68): read config.json and an O-mesh text
 * file, build geometry, initialise the free stream and apply the boundary
 * conditions (Solver::new, solver.rs:47-62). */
jst_status jst_create_from_paths(const char* config_path, const char* mesh_path, const jst_opts* opts,
                                 jst_solver** out);

/* Solver::new (solver.rs:47-62) from a config.json text and a node array
 * (n_rings x n_theta nodes, (x, y) interleaved, ring-major, counter-clockwise;
 * a closing duplicate point per ring is trimmed as in mesh.rs:169-189). */
jst_status jst_create(const char* config_json, const double* xy, int n_rings, int n_theta, const jst_opts* opts,
                      jst_solver** out);

/* Releases the handle and its device memory. */
void jst_destroy(jst_solver* s);

/* Message of the last error on this handle (or of the last failed create
 * when s is NULL). */
const char* jst_last_error(const jst_solver* s);

/* Mesh sizes: NI = n_rings - 1 radial cells, NJ circumferential cells. */
int jst_ni(const jst_solver* s);
int jst_nj(const jst_solver* s);

/* The NonPhysical error of state.rs:242-257. */
typedef struct {
    int64_t i, j;
    double rho, p;
} jst_nonphysical;

/* Solver::advance (solver.rs:97-120): one 5-stage RK step.  On
 * JST_ERR_NONPHYSICAL the first offending cell (row-major order within the
 * first failing stage) is written to *bad (may be NULL). */
jst_status jst_advance(jst_solver* s, jst_nonphysical* bad);

/* RunReport (solver.rs:36-43). */
typedef struct {
    int64_t steps;
    double residual;
    double totaltime;
    int converged;
} jst_run_report;

typedef void (*jst_step_cb)(void* user, uint64_t step, double residual);

/* Solver::run (solver.rs:203-226): advance until max_steps (< 0: the config's
 * solver.iteration) or until the residual drops below solver.targetres.  The
 * callback (may be NULL) runs on the caller's thread after each step with the
 * step's residual (solver.rs:190-200). */
jst_status jst_run(jst_solver* s, int64_t max_steps, jst_step_cb cb, void* user, jst_run_report* report,
                   jst_nonphysical* bad);

/* Solver::residual_terms (solver.rs:86-94): boundary conditions plus the
 * residual terms Fc, Fv, Fd, S of the current state, without an update
 * (golden/bench use).  Also computes the per-cell local time step first
 * when *dt is non-NULL (timestep::compute, timestep.rs:24-47), returning the
 * global minimum in *dt. */
jst_status jst_residual_terms(jst_solver* s, double* dt);

/* The residual the RK update applies (solver.rs:128-133), R = Fc - Fv - Fd
 * with S subtracted from component 4, of every interior cell of the current
 * state: Solver::residual_terms (solver.rs:86-94) after timestep::compute
 * (timestep.rs:24-47), combined per cell.  On the fused path R comes from
 * the stage kernel this solver runs its RK stages with (the autotuned
 * marching-strip or tile kernel, in the solver's precision; stage 0 run
 * without its update); on the passes path from the separate terms.  out
 * receives 5 planes of NI*NJ doubles (component-major, i-major / j-minor);
 * n >= 5*NI*NJ.  The conserved state is not changed. */
jst_status jst_stage_residual(jst_solver* s, double* out, size_t n);

/* timestep::compute (timestep.rs:24-57) on the current state. */
jst_status jst_timestep(jst_solver* s, double* dt);

/* Solver::residual (solver.rs:190-200) of the last completed step. */
jst_status jst_residual(jst_solver* s, double* out);

/* Solver public fields `totaltime` and `step` (solver.rs:25-34). */
jst_status jst_totaltime(const jst_solver* s, double* out);
jst_status jst_step_count(const jst_solver* s, int64_t* out);

/* Cell fields readable with jst_get_field. */
typedef enum {
    JST_F_RHO = 0, JST_F_P, JST_F_T, JST_F_U, JST_F_V, JST_F_E, JST_F_H, JST_F_C, JST_F_NUT,
    JST_F_U0, JST_F_U1, JST_F_U2, JST_F_U3, JST_F_U4,
    JST_F_FC0, JST_F_FC1, JST_F_FC2, JST_F_FC3, JST_F_FC4,
    JST_F_FV0, JST_F_FV1, JST_F_FV2, JST_F_FV3, JST_F_FV4,
    JST_F_FD0, JST_F_FD1, JST_F_FD2, JST_F_FD3, JST_F_FD4,
    JST_F_S,
    JST_F_DUDX, JST_F_DUDY, JST_F_DVDX, JST_F_DVDY, JST_F_DTDX, JST_F_DTDY, JST_F_DNUTDX, JST_F_DNUTDY,
    JST_F_SA_CHI, JST_F_SA_FV1,
    JST_F_LOCALDT,
    JST_F_VOL, JST_F_CX, JST_F_CY, JST_F_WALL_DIST,
    JST_F_COUNT
} jst_field;

/* Copies an interior cell field into out[n] (n >= NI*NJ).  Primitive and
 * conserved fields are available on both paths; the separate residual terms,
 * gradients and chi/fv1 after jst_residual_terms on the passes path. */
jst_status jst_get_field(jst_solver* s, int field, double* out, size_t n);

/* Face geometry: which = 0 for tau faces ((NI+1) x NJ), 1 for n faces
 * (NI x NJ); out receives (nx, ny, mx, my) per face, i-major (geometry.rs:25-34). */
jst_status jst_get_faces(jst_solver* s, int which, double* out, size_t n);

/* Overwrites the conserved state U (5 planes of NI*NJ, component-major) and
 * re-derives the primitives (solver.rs:151-185); fails with
 * JST_ERR_NONPHYSICAL exactly where unpack would. */
jst_status jst_set_conserved(jst_solver* s, const double* u5, size_t n, jst_nonphysical* bad);

/* Checkpoint dump (no counterpart in the reference, whose Solver keeps no
 * dump): writes U (5 planes, FP64), the completed step count, the physical
 * time and the last residual to a binary file; loading it into a solver
 * built from the same mesh continues the run where it stopped (the next
 * step's time step is re-derived from U, as every step of the reference
 * derives it).  File: "JSTCKPT1", int32 NI, int32 NJ, int64 step, double
 * totaltime, double residual, 5*NI*NJ doubles, native byte order.
 * Load fails with JST_ERR_ARG on a size mismatch or a damaged file and with
 * JST_ERR_NONPHYSICAL like jst_set_conserved. */
jst_status jst_checkpoint_save(jst_solver* s, const char* path);
jst_status jst_checkpoint_load(jst_solver* s, const char* path, jst_nonphysical* bad);

/* Lift and drag coefficients of the current state (no counterpart in the
 * reference): wall pressure and viscous face fluxes integrated over ring 0,
 * rotated by the angle of attack and divided by 0.5*rho_inf*V_inf^2*chord,
 * chord = x-extent of the wall ring.  Runs jst_residual_terms' boundary and
 * viscous passes on the current state first. */
jst_status jst_forces(jst_solver* s, double* cl, double* cd);

/* Solver::write_csv (solver.rs:229-255): `i,j,x,y,rho,p,T,u,v,miubl`,
 * 1-based indices, values in Rust `{:.8e}` format. */
jst_status jst_write_csv(jst_solver* s, const char* path);

/* Device timing (no counterpart in the reference; used by benchmarks):
 * enqueues nsteps RK steps with the convergence test disabled and returns
 * their device time in *ms, measured with CUDA events on the solver's own
 * stream.  When stage_ms is non-NULL ten further steps run back to back from
 * one graph with a CUDA event recorded before, between and after each step's
 * five stage launches, and stage_ms[0..4] receive the stage kernels' mean
 * times over those steps. */
jst_status jst_time_steps(jst_solver* s, int nsteps, double* ms, double* stage_ms);

/* ------------------------------------------------------------------------
 * Batched solving and serving (no counterpart in the reference, which solves
 * one case per process): many independent solves of different meshes and
 * flow conditions share one persistent stage kernel over a table of
 * (instance, tile) work items, with each RK step replayed from a CUDA graph.
 * Instances are admitted as HBM and slots allow, stay device-resident, and
 * retire individually on convergence, on NonPhysical, or at their step limit.
 * ------------------------------------------------------------------------ */
typedef struct jst_batch jst_batch;

typedef struct {
    int precision;        /* jst_precision of every instance */
    int dt_mode;          /* jst_dt_mode of every instance */
    int device;
    int tile_i, tile_j;   /* 0 = default tile */
    int max_instances;    /* slots */
    int steps_per_poll;   /* RK steps per graph replay between convergence polls */
    double hbm_budget_gb; /* device memory the batch may hold for instances */
    int keep_fields;      /* copy U of retired instances to host memory */
    int block_threads;    /* threads per block (0 = default for the tile) */
    int staging;          /* jst_staging of the marching strips */
} jst_batch_opts;

void jst_batch_default_opts(jst_batch_opts* o);
jst_status jst_batch_create(const jst_batch_opts* o, jst_batch** out);
void jst_batch_destroy(jst_batch* b);

/* Queue one solve.  max_steps < 0 uses the config's solver.iteration;
 * residual_drop > 0 retires the instance once its residual falls below
 * residual_drop times its first-step residual (the config's targetres also
 * applies); cl_tol > 0 retires it once |CL(n) - CL(n-100)| < cl_tol.  The
 * instance is admitted at the next jst_batch_step when a slot and memory are
 * free.  *id receives its id. */
jst_status jst_batch_submit(jst_batch* b, const char* config_json, const double* xy, int n_rings, int n_theta,
                            int64_t max_steps, double residual_drop, double cl_tol, int64_t* id);

/* Admit queued instances, advance every active instance by up to nsteps RK
 * steps (in graph replays of steps_per_poll), retire finished ones.  Returns
 * after nsteps or when nothing is active or queued. */
jst_status jst_batch_step(jst_batch* b, int nsteps);

/* (tile_i, tile_j, block_threads) the batch's stage kernel runs with: set by
 * the options or, when those are 0, by the autotuner at the first
 * jst_batch_step (tile_j == 26: marching strips of at most tile_i rows). */
jst_status jst_batch_kernel_config(const jst_batch* b, int* tile_i, int* tile_j, int* block_threads);

/* jst_staging the batch's stage kernel runs with (0 when it is not a
 * marching strip).  A bounded row-copy wait that runs out makes
 * jst_batch_step fail with JST_ERR_TIMEOUT. */
jst_status jst_batch_kernel_staging(const jst_batch* b, int* staging);

/* Counts of active and queued instances and device bytes in use. */
jst_status jst_batch_stats(jst_batch* b, int* active, int* queued, double* bytes_in_use);

/* Ids retired since the last poll (up to cap); *n receives the count. */
jst_status jst_batch_poll(jst_batch* b, int64_t* ids, int cap, int* n);

typedef struct {
    int64_t id;
    int status;        /* JST_OK, JST_ERR_NONPHYSICAL, or JST_ERR_TIMEOUT (step limit) */
    int64_t steps;
    double residual, residual_first, totaltime;
    double cl, cd;
    double t_submit, t_admit, t_done; /* seconds since the batch was created */
    int ni, nj;
    jst_nonphysical bad;
} jst_batch_result;

/* Result of a retired instance; with keep_fields, fields (5*NI*NJ doubles,
 * may be NULL) receives its final conserved state. */
jst_status jst_batch_result_get(jst_batch* b, int64_t id, jst_batch_result* r, double* fields, size_t n);

/* The density residual of solver.rs:190-200, sqrt(sum((rho - rho_prev)^2) / NI / NJ),
 * for callers that cannot allocate device memory (no counterpart in the
 * reference, whose Solver owns its fields).  Plugin hosts that own every
 * device allocation through their own pool, and monitoring loops that must
 * not call cudaMalloc (it synchronises the device), pass device pointers to
 * their own NI*NJ density fields and to one double for the result; the call
 * enqueues two kernels on `stream` (a cudaStream_t, NULL for the default
 * stream) and returns without synchronising or allocating.  Its scratch is a
 * fixed file-scope device array of 8192 partial sums, so NI*NJ may not exceed
 * 16,777,216 cells (larger sizes fail with JST_ERR_ARG before any launch).
 * The kernels run on the calling thread's current device (cudaSetDevice),
 * whatever device the pointers belong to, so make the fields' device current
 * first.  The first call in each CUDA context on a device looks up that
 * array's address (again after cudaDeviceReset, which creates a new
 * context); make it before any stream capture.  All calls share the array:
 * calls whose kernels overlap on the GPU race, so serialise them (one
 * stream, or events). */
jst_status jst_residual_noalloc(const double* rho, const double* rho_prev, int ni, int nj, double* out,
                                void* stream);

/* Tile shape and block size the fused path runs with (chosen by the
 * autotuner when jst_opts.tile_i/tile_j are 0); zeros on the passes path. */
jst_status jst_kernel_config(const jst_solver* s, int* tile_i, int* tile_j, int* block_threads);

/* jst_staging of the fused path's marching strips (0 for tiles and the
 * passes path).  With JST_STAGING_BULK, a row-copy wait that runs out (about
 * 0.1 s) makes jst_advance / jst_run return JST_ERR_TIMEOUT. */
jst_status jst_kernel_staging(const jst_solver* s, int* staging);

/* Version string of this library. */
const char* jst_version(void);

#ifdef __cplusplus
}
#endif

#endif /* JST_GPU_H */
