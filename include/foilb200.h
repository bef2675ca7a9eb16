/*
 * foilb200.h - C ABI of libfoilb200.so, the B200 (sm_100a) Stable Fluids step.
 *
 * The library owns device-resident solver state (MAC face velocities, solid mask,
 * pressure and Krylov work arrays, transform tables) and runs the step as
 * hand-written CUDA. Every entry point takes plain pointers and sizes, is
 * synchronous from the caller's view, returns an fb_status code, and never
 * reports failure through a device trap. Host buffers are caller-owned.
 *
 * Reference interfaces replaced (paths relative to the FoilBench project root,
 * PY = implementations/python/src/foilbench_py):
 *   fb_solver_create/fb_initialize  <- StableFluidsSolver.__init__/initialize  PY/solvers/stable_fluids.py:129,195
 *   fb_restart                      <- StableFluidsSolver.restart              PY/solvers/stable_fluids.py:218
 *   fb_advance                      <- StableFluidsSolver.advance              PY/solvers/stable_fluids.py:332
 *   fb_export_velocity              <- StableFluidsSolver.export_state/cell_velocity PY/solvers/stable_fluids.py:605-634
 *   fb_import_velocity              <- StableFluidsSolver.import_state         PY/solvers/stable_fluids.py:636
 *   fb_sample_velocity              <- StableFluidsSolver.sample_velocity      PY/solvers/stable_fluids.py:609
 *   fb_diagnostics                  <- StableFluidsSolver.diagnostics          PY/solvers/stable_fluids.py:708
 *   fb_compute_mask                 <- NacaFoil.mask                           PY/core/geometry.py:157
 *   fb_naca_signed_distance         <- NacaFoil.signed_distance                PY/core/geometry.py:92
 *   fb_op_advect_velocity           <- advect_velocity                         PY/core/grid.py:506
 *   fb_op_implicit_diffuse          <- implicit_diffuse                        PY/core/grid.py:183
 *   fb_op_solve_masked_poisson      <- solve_masked_poisson                    PY/core/_scipy_adapter.py:16
 *   fb_op_project_faces             <- project_faces                           PY/core/grid.py:134
 */
#ifndef FOILB200_H
#define FOILB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FB_ABI_VERSION 1

/* Return codes. FB_ERR_NUMERICAL means a classified numerical failure whose
 * reason/stage/evidence are in the fb_report passed to the call; solver state
 * is then exactly what it was before the call (transactional). */
typedef enum fb_status {
    FB_OK = 0,
    FB_ERR_INVALID_ARGUMENT = 1,
    FB_ERR_CUDA = 2,
    FB_ERR_OUT_OF_MEMORY = 3,
    FB_ERR_NOT_INITIALIZED = 4,
    FB_ERR_NUMERICAL = 5,
    FB_ERR_DEVICE_TIMEOUT = 6,
    FB_ERR_BUDGET = 7
} fb_status;

/* Failure vocabulary (PY/core/models.py:14-44). */
typedef enum fb_reason {
    FB_REASON_NONE = 0,
    FB_REASON_EXCESSIVE_VELOCITY = 1,
    FB_REASON_STABILITY_LIMIT = 2,
    FB_REASON_NONFINITE_STATE = 3,
    FB_REASON_CONVERGENCE_FAILURE = 4,
    FB_REASON_PROJECTION_FAILURE = 5,
    FB_REASON_POSTCONDITION_FAILURE = 6,
    FB_REASON_TIME_CONTRACT_FAILURE = 7
} fb_reason;

typedef enum fb_stage {
    FB_STAGE_NONE = 0,
    FB_STAGE_ADVECTION = 1,
    FB_STAGE_VISCOSITY = 2,
    FB_STAGE_PROJECTION = 3,
    FB_STAGE_BOUNDARY = 4,
    FB_STAGE_POSTCONDITION = 5,
    FB_STAGE_CANONICAL_IMPORT = 6,
    FB_STAGE_TIME_MAPPING = 7
} fb_stage;

typedef enum fb_precision { FB_FLOAT32 = 0, FB_FLOAT64 = 1 } fb_precision;

/* Pressure solve scheme. REFERENCE: DST-I preconditioned CG in FP64, the
 * reference's iteration and stopping rule. MIXED: the same preconditioned CG run
 * in FP32 inside an FP64 defect-correction loop that recomputes r = b - A x in
 * FP64 until the reference tolerance is met. */
typedef enum fb_pressure_scheme { FB_PRESSURE_REFERENCE = 0, FB_PRESSURE_MIXED = 1 } fb_pressure_scheme;

/* Transport of the velocity (stable_advection; PY/core/grid.py:306-503 for the face and skew
 * forms). SKEW_RK2 always works on the faces. */
typedef enum fb_advection {
    FB_ADVECT_SEMI_LAGRANGIAN = 0, FB_ADVECT_MACCORMACK = 1, FB_ADVECT_SKEW_RK2 = 2
} fb_advection;

/* Row DST-I of the pressure preconditioner (no reference counterpart: the reference calls
 * scipy.fft.dstn, _scipy_adapter.py:76-96). FFT: Bluestein FFT in the Krylov precision (the
 * REFERENCE scheme always uses it). TENSOR: TF32 tcgen05 GEMMs with FP32 accumulation (MIXED
 * scheme only; the FP32 inner CG's FP64 defect correction keeps the projection's accuracy).
 * AUTO: TENSOR for the MIXED scheme on grids with at least 64 work units of 128 rows x 128
 * wavenumbers per parity (2 * ceil(ny/128) * ceil(ceil(nx/2)/128) >= 64), else FFT. */
typedef enum fb_row_transform {
    FB_ROW_TRANSFORM_AUTO = 0, FB_ROW_TRANSFORM_FFT = 1, FB_ROW_TRANSFORM_TENSOR = 2
} fb_row_transform;

typedef enum fb_initial_condition {
    FB_IC_FREESTREAM = 0, FB_IC_TAYLOR_GREEN = 1, FB_IC_POISEUILLE = 2
} fb_initial_condition;

/* Scenario as the device needs it (PY/core/models.py:50-224 resolved to numbers). */
typedef struct fb_scenario_desc {
    int32_t nx, ny;                    /* cells along x, y (DomainSpec.resolution) */
    double x0, x1, y0, y1;             /* DomainSpec.bounds */
    int32_t periodic_x, periodic_y;    /* DomainSpec.periodic_axes */
    int32_t channel_walls;             /* no-slip y walls (Poiseuille initial condition) */
    double freestream_x, freestream_y;
    char naca[4];                      /* four NACA digits, e.g. '2','4','1','2' */
    double chord, pivot_x, pivot_y;
    int32_t precision;                 /* fb_precision of the velocity fields */
    int32_t pressure_scheme;           /* fb_pressure_scheme */
    int32_t advection;                 /* fb_advection */
    int32_t initial_condition;         /* fb_initial_condition */
    double reference_speed;            /* Scenario.reference_speed */
    double cfl;                        /* solver_options.stable_cfl (default 0.7) */
    double pressure_tolerance;         /* solver_options.pressure_tolerance (default 1e-5) */
    int32_t pressure_max_iterations;   /* solver_options.pressure_max_iterations (default 640) */
    int32_t pressure_fixed_iterations; /* > 0: exactly this many CG iterations per solve, accepted whatever the residual */
    double mixed_inner_rtol;           /* MIXED: inner FP32 relative-residual floor (<= 0: default 3e-6) */
    double divergence_limit;           /* mac_maximum_divergence_linf (+inf when absent) */
    double leakage_limit;              /* mac_maximum_solid_leakage (+inf when absent) */
    int32_t passive_scalar;            /* carry a cell scalar advected by the same trace */
    int32_t face_advection;            /* stable_face_advection: transport the faces themselves */
    int32_t row_transform;             /* fb_row_transform of the pressure preconditioner */
    int32_t reserved[5];
} fb_scenario_desc;

/* Outcome of a call that steps or projects (StepReport evidence, PY/solvers/stable_fluids.py:576-603). */
typedef struct fb_report {
    int32_t status;                 /* fb_status */
    int32_t reason;                 /* fb_reason */
    int32_t stage;                  /* fb_stage */
    int32_t substeps;
    int32_t stability_retries;
    int32_t pressure_iterations;    /* CG iterations of the last projection (inner iterations when MIXED) */
    int32_t pressure_outer_iterations; /* MIXED: FP64 residual recomputations of the last projection */
    int32_t pressure_converged;
    int32_t viscosity_iterations;
    int32_t viscosity_converged;
    int32_t total_pressure_iterations; /* summed over the substeps of the call */
    int32_t reserved_i[5];
    double max_speed;               /* max |cell velocity| of the final state */
    double wall_speed;
    double accepted_measure;        /* dt * advective rate of the accepted attempt */
    double advective_rate;
    double boundary_sweep;
    double pressure_relative_residual;
    double viscosity_final_residual;
    double divergence_linf;
    double solid_leakage;
    double required_substeps;       /* evidence on stability_limit */
    double evidence[6];             /* reason-specific evidence, see fb_report_evidence_names */
    double device_ms;               /* device time of the call's kernels (CUDA events) */
    int32_t kernel_launches;        /* kernels this call launched */
    int32_t reserved_j[3];
} fb_report;

typedef struct fb_ctx fb_ctx;
typedef struct fb_solver fb_solver;

/* ---- library / context ---------------------------------------------------------------- */
int32_t fb_abi_version(void);
/* sizeof(fb_scenario_desc) and sizeof(fb_report), for bindings to check their layouts. */
int32_t fb_abi_struct_sizes(uint64_t *desc_bytes, uint64_t *report_bytes);
/* Message for the last failing call on this host thread (empty when none). */
const char *fb_last_error(void);
int32_t fb_device_count(int32_t *count);
/* A context binds one CUDA device and an HBM budget (bytes, 0 = no limit) that
 * solver creation is admitted against. */
int32_t fb_ctx_create(int32_t device, uint64_t hbm_budget, fb_ctx **out);
int32_t fb_ctx_destroy(fb_ctx *ctx);
int32_t fb_ctx_bytes_in_use(fb_ctx *ctx, uint64_t *bytes);
/* Page-locked host buffers for exports (no counterpart in the reference). Freed blocks are
 * kept per size and handed out again, so repeated exports of a state neither pin nor fault
 * pages; device-to-host copies into them run at full link speed. At most
 * FB_HOST_POOL_BYTES are held (in use plus cached); past that fb_host_alloc returns
 * FB_ERR_BUDGET and the caller uses ordinary memory. */
#define FB_HOST_POOL_BYTES (4ull << 30)
int32_t fb_host_alloc(uint64_t bytes, void **out);
int32_t fb_host_free(void *p);

/* ---- solver lifecycle (FlowSolver) ---------------------------------------------------- */
/* Grid widths up to 8192 columns (with a double-precision pressure CG, rows over 4096 columns
 * run the preconditioner's convolution in two halves); wider grids return
 * FB_ERR_INVALID_ARGUMENT naming the shared memory they need. */
int32_t fb_solver_create(fb_ctx *ctx, const fb_scenario_desc *desc, fb_solver **out);
int32_t fb_solver_destroy(fb_solver *s);
/* Device bytes the solver holds (state, work arrays, tables). */
int32_t fb_solver_bytes(const fb_scenario_desc *desc, uint64_t *bytes);
/* Initial field, mask at angle0, initial projection with dt = project_dt. */
int32_t fb_initialize(fb_solver *s, double angle0_degrees, double reynolds, double project_dt, fb_report *out);
/* Second half of restart (the caller runs fb_initialize first, as the reference restart
 * calls initialize): move to the restart pose and Reynolds number, rebuild the initial
 * field with solid cells set to the wall velocity, and re-project. */
int32_t fb_restart(fb_solver *s, double time, double angle_degrees, double reynolds, double project_dt,
                   fb_report *out);
int32_t fb_set_viscosity(fb_solver *s, double viscosity);
/* Options the reference re-reads at every advance (stable_cfl, pressure tolerance and
 * budgets, MAC postcondition limits, transport, mixed-scheme floor): copies those fields of
 * desc. Grid, precision, pressure scheme and the passive-scalar flag stay as created. */
int32_t fb_update_options(fb_solver *s, const fb_scenario_desc *desc);
/* One output interval: substep planning, substeps, retries, postconditions, rollback. */
int32_t fb_advance(fb_solver *s, double control_time, double control_angle_degrees,
                   double control_angular_velocity_degrees, double target_dt, fb_report *out);
/* Canonical cell velocity (ny, nx, 2) in the solver precision; solids zeroed when zero_solids. */
int32_t fb_export_velocity(fb_solver *s, void *host, size_t bytes, int32_t zero_solids);
/* export_state (PY/solvers/stable_fluids.py:613-634): the canonical cell velocity with solids
 * zeroed, plus the number of non-finite values in it, counted on the device as they are
 * written, so that the caller need not scan the array again for the canonical state's
 * finiteness invariant (PY/core/models.py CanonicalFlowState). */
int32_t fb_export_state(fb_solver *s, void *host, size_t bytes, int64_t *nonfinite);
/* MAC faces: u (ny, nx+1) and v (ny+1, nx) in the solver precision. */
int32_t fb_export_faces(fb_solver *s, void *host_u, size_t bytes_u, void *host_v, size_t bytes_v);
/* Last pressure field (ny, nx) float64. */
int32_t fb_export_pressure(fb_solver *s, double *host, size_t bytes);
/* Current solid mask (ny, nx) as bytes 0/1. */
int32_t fb_export_mask(fb_solver *s, uint8_t *host, size_t bytes);
/* Passive scalar (ny, nx) in the solver precision (only when desc.passive_scalar). */
int32_t fb_export_scalar(fb_solver *s, void *host, size_t bytes);
int32_t fb_import_scalar(fb_solver *s, const void *host, size_t bytes);
/* Canonical import: cell velocity (ny, nx, 2) in the solver precision; solid cells take
 * the wall velocity; faces re-projected with dt = project_dt. Transactional. */
int32_t fb_import_velocity(fb_solver *s, const void *host, size_t bytes, double time, double angle_degrees,
                           double angular_velocity_degrees, double project_dt, fb_report *out);
/* Bilinear sample of the cell velocity at n points (x, y) float64 -> (n, 2) float64. */
int32_t fb_sample_velocity(fb_solver *s, const double *points, int64_t n, double *out);
/* Diagnostics in the order kinetic_energy, enstrophy, divergence_l2, divergence_linf,
 * solid_leakage, wake_width, recirculation_area. */
int32_t fb_diagnostics(fb_solver *s, double *values, int32_t count);
/* Solver time/pose held by the device side. */
int32_t fb_get_pose(fb_solver *s, double *time, double *angle_degrees, double *angular_velocity_degrees);

/* ---- tracing ------------------------------------------------------------------------------ */
/* Phase trace of the step kernel: CTA 0 stamps %globaltimer (ns) after every grid barrier
 * with a phase tag; entries are (tag << 56) | (ns & (2^56 - 1)). capacity 0 disables.
 * fb_trace_read copies up to `capacity` entries, reports how many were recorded and clears. */
int32_t fb_trace_enable(fb_solver *s, int32_t capacity);
int32_t fb_trace_read(fb_solver *s, uint64_t *host, int64_t capacity, int64_t *count);

/* ---- autotuner ------------------------------------------------------------------------------
 * No counterpart in the reference (its solver runs on the host). Chooses the step kernel's
 * launch shapes and the mixed scheme's sweep schedule by measurement: one substep of this
 * solver's current state, planned as fb_advance would plan it for target_dt, runs `reps`
 * times per candidate (state restored after every trial; median device time), first with the
 * built-in heuristic, then in a coordinate search over the CTA count (the co-resident maximum,
 * fractions of the SM count, and the count that gives the row transforms whole rounds), the
 * tridiagonal column tile width (16, 8, 4, 2 columns, as shared memory allows) and, for the
 * mixed scheme without a caller-set mixed_inner_rtol, the inner FP32 CG's relative stop floor
 * (1e-6, 3e-6, 1e-5, 3e-5). The fastest choice (by at least 0.5 %) is applied to this solver
 * and cached for the process under (grid, precision, scheme, transport, periodic axes,
 * device); solvers created later with that key start from it. out[0..7] (n values at most):
 * column tile width, CTA count, inner floor, heuristic ms, tuned ms, trials, heuristic column
 * tile width, heuristic CTA count. */
int32_t fb_autotune(fb_solver *s, double target_dt, int32_t reps, double *out, int32_t n);
/* Set the step kernel's launch shape by hand: ctas in [1, co-resident maximum] and column_tile
 * a power of two in [2, the widest that fits] (0 keeps either). Results stay within the
 * solver's tolerances for any shape; reduction order, and so the last bits, follow the CTA
 * count. Used to time a solve on the CTAs it would get in a batched launch. */
int32_t fb_set_launch_shape(fb_solver *s, int32_t ctas, int32_t column_tile);
/* The launch shape in use and the mixed scheme's inner stop floor (any pointer may be NULL). */
int32_t fb_get_launch_shape(fb_solver *s, int32_t *ctas, int32_t *column_tile, double *inner_rtol);

/* ---- failure detection test hook -----------------------------------------------------------
 * No counterpart in the reference (its solver runs on the host and has no device waits). Every
 * grid-barrier wait of the step kernel is bounded by a time limit, after which the kernel
 * raises an abort flag, every CTA returns, and the call reports FB_ERR_DEVICE_TIMEOUT with the
 * state rolled back. This hook makes that path testable without a device fault: with
 * withhold_barrier = k > 0, CTA 0 of each later launch does not arrive at its k-th barrier, so
 * that barrier's waits run out after limit_ns (0 restores the default 2 s limit). k = 0 turns
 * the hook off. No bulk copy is in flight at any grid barrier, so an abort there leaves none. */
int32_t fb_debug_barrier_timeout(fb_solver *s, int32_t withhold_barrier, uint64_t limit_ns);

/* ---- geometry ---------------------------------------------------------------------------- */
/* Surface forces on the foil (no counterpart in the reference, which computes none): from the
 * current state's faces and last pressure, in FP64. values[8] = pressure force x, y; viscous
 * force x, y; total force x, y; drag and lift coefficients (force along / across the
 * freestream divided by 0.5 |U|^2 chord). Faces between fluid and solid cells carry the fluid
 * cell's kinematic pressure and the shear nu (u_fluid - u_wall) / (h / 2). Lift is positive
 * toward +90 deg from the freestream; the reference's angle turns the section counter-clockwise
 * (trailing edge up), so positive angles in a +x stream give negative lift. */
int32_t fb_forces(fb_solver *s, double *values, int32_t count);
/* Solid mask of a NACA section for a domain at an angle, bytes 0/1 (ny, nx). */
int32_t fb_compute_mask(fb_ctx *ctx, const fb_scenario_desc *desc, double angle_degrees, uint8_t *host_mask,
                        size_t bytes);
/* Signed distance (NacaFoil.signed_distance) at n points (x, y) float64. */
int32_t fb_naca_signed_distance(fb_ctx *ctx, const char naca[4], double chord, double pivot_x, double pivot_y,
                                const double *points, int64_t n, double angle_degrees, double *out);

/* ---- operator-level entry points (the same device code, on caller data) --------------------
 * Each creates transient device state for the grid in desc, runs the requested stage and
 * copies the result back. Arrays are row-major with x fastest, in desc->precision unless noted. */
/* cell velocity (ny, nx, 2) -> advected (ny, nx, 2); maccormack selects the limited corrector. */
int32_t fb_op_advect_velocity(fb_ctx *ctx, const fb_scenario_desc *desc, const void *vel_in, void *vel_out,
                              double dt, int32_t maccormack);
/* Jacobi backward-Euler viscosity of a cell velocity; iterations/residual/converged out. */
int32_t fb_op_implicit_diffuse(fb_ctx *ctx, const fb_scenario_desc *desc, const void *vel_in, void *vel_out,
                               double viscosity, double dt, double tolerance, int32_t max_iterations,
                               fb_report *out);
/* Masked Poisson solve: rhs (ny, nx) float64, fluid (ny, nx) bytes -> pressure float64.
 * report.pressure_iterations / pressure_relative_residual / pressure_converged (info == 0). */
int32_t fb_op_solve_masked_poisson(fb_ctx *ctx, const fb_scenario_desc *desc, const double *rhs,
                                   const uint8_t *fluid, double *pressure, fb_report *out);
/* Face projection with solid mask and rigid wall rotation omega (deg/s) about the pivot:
 * u (ny, nx+1), v (ny+1, nx) in/out, solid (ny, nx) bytes. */
int32_t fb_op_project_faces(fb_ctx *ctx, const fb_scenario_desc *desc, void *u, void *v, const uint8_t *solid,
                            double omega_degrees, double dt, fb_report *out);

/* ---- batched solves --------------------------------------------------------------------------
 * Many scenarios advance together in ONE cooperative launch per attempt: every member owns a
 * contiguous group of CTAs (in proportion to its expected work: cells x substeps x CG effort)
 * with its own barrier, reductions and report, and runs all its planned substeps in it, so
 * members never wait for each other; only members that must retry run again. Each member
 * advances exactly as fb_advance would (substep plan, retries, postconditions, rollback on
 * failure); the reference has no batched counterpart (its runner advances one solver at a
 * time, PY/benchmark/runner.py:240-273). Members: initialized float32 solvers with the mixed
 * pressure scheme, non-periodic, nx a multiple of 16 with 129..2048 columns, no tracing; at
 * most one member per CTA the device can hold. */
typedef struct fb_batch fb_batch;
int32_t fb_batch_create(fb_ctx *ctx, fb_solver *const *solvers, int32_t count, fb_batch **out);
int32_t fb_batch_destroy(fb_batch *batch);
/* CTAs each member had in the latest batched launch (0: it did not run); count entries. */
int32_t fb_batch_ctas(const fb_batch *batch, int32_t *ctas, int32_t count);
/* Advance member i by target_dt[i] toward its control (time, angle, angular velocity). Per
 * member: reports[i] and status[i] (FB_OK or the failure, state unchanged). Returns FB_OK when
 * every member advanced, FB_ERR_NUMERICAL when some did not. reports[i].device_ms is the
 * batch's device time. */
int32_t fb_batch_advance(fb_batch *batch, const double *control_time, const double *control_angle_degrees,
                         const double *control_angular_velocity_degrees, const double *target_dt, fb_report *reports,
                         int32_t *status);

/* ---- allocation-free viscosity ---------------------------------------------------------------
 * No counterpart in the reference. For callers that cannot let this library allocate device
 * memory: a simulation or viewer loop that owns every device byte through its own pool, sized
 * once at start-up, and forbids driver allocations while it runs (a cudaMalloc there would
 * break its memory budget or stall the loop on the driver's implicit synchronisation). Same
 * Jacobi viscosity as fb_op_implicit_diffuse, on the caller's device buffers: vx_in, vy_in,
 * vx_out, vy_out are (ny, nx) component planes in desc->precision; stream is a cudaStream_t
 * (NULL for the default stream). The working set lives in one file-scope device array of
 * FB_NOALLOC_SCRATCH_BYTES on each device that loads the library (held until the process
 * exits): four planes rounded up to 256 bytes plus a 393,728-byte header, so at most 2,084,832
 * cells in float64 and 4,169,664 in float32; larger grids are rejected with
 * FB_ERR_INVALID_ARGUMENT and a message naming the limit. The first call on a device looks up
 * the array's device address (with that device current), so make that call before any stream
 * capture. All calls share the array and it keeps the last call's contents (the call clears
 * its barrier and report words itself): calls that overlap on the GPU race. The call makes
 * `device` current and restores the caller's current device before it returns; it returns
 * after its kernel has finished (it waits on the stream and reads the report back), with the
 * same statuses and report fields as fb_op_implicit_diffuse. It never allocates or frees
 * device memory. */
#define FB_NOALLOC_SCRATCH_BYTES (64ull << 20)
int32_t fb_op_implicit_diffuse_noalloc(int32_t device, const fb_scenario_desc *desc, const void *vx_in,
                                       const void *vy_in, void *vx_out, void *vy_out, double viscosity, double dt,
                                       double tolerance, int32_t max_iterations, void *stream, fb_report *out);

#ifdef __cplusplus
}
#endif

#endif /* FOILB200_H */
