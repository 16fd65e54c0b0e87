/*
 * cp_simple.h - C ABI of the B200-native SIMPLE solver (libcoldplate.so).
 *
 * Drop-in boundary for the reference's 2-D staggered-grid SIMPLE iteration
 * (Carloossgg/coldplate-solver).  All state lives on the GPU inside a
 * cp_ctx; host arrays cross this interface only as plain pointers with
 * explicit (rows, cols, row_stride, col_stride) in elements, so Eigen's
 * column-major MatrixXf/MatrixXd (row_stride 1, col_stride rows) and numpy's
 * row-major arrays both pass without copies on the caller's side.
 *
 * Index conventions are the reference's: physical cells Ny x Nx,
 * M = Ny + 1, N = Nx + 1 (SIMPLE.cpp:53-54); u is (M+1) x N, v is M x (N+1),
 * p is (M+1) x (N+1) (SIMPLE.cpp:252-273).
 *
 * Every call returns a cp_status; cp_last_error_string() describes the last
 * failure of the calling thread.  Contexts are independent: one per host
 * thread (or stream) may run concurrently.
 */
#ifndef CP_SIMPLE_H
#define CP_SIMPLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cp_status {
    CP_OK = 0,
    CP_ERR_BAD_PARAM = 1,    /* invalid argument or parameter value          */
    CP_ERR_UNSUPPORTED = 2,  /* a reference option this build does not run  */
    CP_ERR_NONFINITE = 3,    /* NaN/Inf in inputs or produced by the solve   */
    /* 4 is not used: the reference iteration has no divergence rule, and a
     * solve that blows up stops with CP_ERR_NONFINITE */
    CP_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up           */
    CP_ERR_CUDA = 6,         /* a CUDA runtime call failed                   */
    CP_ERR_STATE = 7         /* call not valid in the context's state        */
} cp_status;

/* Arithmetic of the inner solves.  CP_PREC_FP64: everything in double (the
 * reference algorithm re-typed).  CP_PREC_MIXED: momentum Jacobi sweeps and
 * the PCG matvec/preconditioner in float on corrections of double state;
 * residuals, global dot products, the mass imbalance and all fields stay
 * double, so the converged fixed point is the FP64 one. */
typedef enum cp_precision { CP_PREC_FP64 = 0, CP_PREC_MIXED = 1 } cp_precision;

typedef enum cp_stop_reason {
    CP_RUNNING = 0,
    CP_STOP_RESIDUAL = 1,    /* error <= epsilon (SIMPLE.cpp:378)            */
    CP_STOP_MAX_ITER = 2,    /* maxIterations reached                        */
    CP_STOP_DP_WINDOW = 3,   /* pressure-drop window (SIMPLE.cpp:449-491)    */
    CP_STOP_ERROR = 4        /* a device-side error stopped the loop         */
} cp_stop_reason;

typedef enum cp_field {
    CP_FIELD_U = 0, CP_FIELD_V, CP_FIELD_P, CP_FIELD_USTAR, CP_FIELD_VSTAR, CP_FIELD_PSTAR,
    CP_FIELD_DE, CP_FIELD_DN, CP_FIELD_GAMMA, CP_FIELD_ALPHA, CP_FIELD_CELLTYPE
} cp_field;

/*
 * Parameter set: the public knobs of class SIMPLE (SIMPLE.h:68-448) with the
 * same names and defaults (floats widened to double, bools as int), plus the
 * inputs the reference reads from ExportFiles/fluid_params.txt
 * (SIMPLE.cpp:41-59).  cp_params_default() fills the SIMPLE.h defaults.
 * Options that this build does not run must keep their default "off" value;
 * cp_create() returns CP_ERR_UNSUPPORTED otherwise.
 */
typedef struct cp_params {
    /* fluid_params.txt: "Ny Nx hy hx U N_in N_out [Ht]" */
    int Ny, Nx;                    /* physical cells (file order: rows, cols) */
    double hy, hx;                 /* cell size [m]                            */
    double targetVel;              /* inlet velocity U [m/s]                   */
    int N_in_buffer, N_out_buffer; /* thermal crop buffers (bookkeeping only)  */
    double Ht_channel;             /* out-of-plane height [m] (optional)       */

    /* convergence control (SIMPLE.h:68-69) */
    double epsilon;
    int maxIterations;
    /* output / restart (SIMPLE.h:77-78); host-side only */
    int saveStateInterval;
    int reuseInitialFields;
    /* sampling planes (SIMPLE.h:88-89) */
    double xPlaneCoreInlet, xPlaneCoreOutlet;
    /* pressure-drop convergence (SIMPLE.h:98-103) */
    int usePressureDropConvergence;
    int dpConvergenceWindow;
    double dpConvergencePercent;
    int usePressureDropSlopeGate;
    int dpSlopeWindowIters;
    double dpSlopeMaxDelta;
    /* OpenMP threads of the CPU code (SIMPLE.h:111); ignored */
    int numThreads;
    /* pressure solver (SIMPLE.h:145-156): type 1 runs the reference's
     * Jacobi-preconditioned CG (pressure_solver.cpp:121-184); types 2 and 4
     * (AMGCL AMG-CG in the reference; 4 is its default) run CG preconditioned
     * by a multigrid V-cycle: smoothed aggregation for 4, 2 x 2 aggregation
     * for 2 (and for every field of a batch); 0 (SOR) and 3 (LDLT) are
     * CP_ERR_UNSUPPORTED */
    int pressureSolverType;
    int parallelizeDirectSolver;
    int maxPressureIter;
    double pTol;
    double sorOmega;
    /* momentum solver (SIMPLE.h:172-183): only type 1 (implicit Jacobi) */
    int momentumSolverType;
    double momentumTol;
    int maxMomentumIter;
    double momentumSorOmega;        /* printed by the reference, never used */
    /* convection (SIMPLE.h:193): 0 FOU, 1 SOU deferred correction */
    int convectionScheme;
    /* 2.5-D model (SIMPLE.h:205-208) */
    int enableTwoPointFiveD;
    double twoPointFiveDConvectionFactor;
    double twoPointFiveDSinkMultiplier;
    /* Brinkman penalisation (SIMPLE.h:242-244); alpha_max = eta / K_min */
    double brinkmanKMin;
    double brinkmanQ;
    /* pseudo-transient continuation (SIMPLE.h:260-345): must stay off */
    double timeStepMultiplier;
    int enablePseudoTimeStepping;
    double pseudoCFL;
    double minPseudoSpeed;
    int useLocalPseudoTime;
    int pseudoControllerMode;
    int enableSER;
    int enableLineSearch;
    int enableCflRamp;
    /* fluid properties (SIMPLE.h:374-375) */
    double rho, eta;
    /* inlet ramp (SIMPLE.h:385-386) */
    int enableInletRamp;
    int rampSteps;
    /* under-relaxation (SIMPLE.h:397-398) */
    double uvAlpha, pAlpha;
    /* residual artificial viscosity (SIMPLE.h:406-411): must stay off */
    int enableResidualViscosity;
    /* residual reporting (SIMPLE.h:424, 447-448) */
    int enableNormalizedResiduals;
    double residNormFloorVel, residNormFloorMass;

    /* ---- additions of this implementation ---- */
    int precision;                  /* cp_precision                           */
    int historyCapacity;            /* rows of per-iteration history kept     */
    int chunk;                      /* outer iterations between host polls    */
    int adjointModel;               /* cp_adjoint_model of cp_adjoint_dp_dgamma */
} cp_params;

/* Per-iteration record (one row of the history, see cp_get_history). */
typedef struct cp_iter_report {
    int iter;                 /* completed outer iterations                   */
    int done;                 /* 1 once the loop stopped                      */
    int stop_reason;          /* cp_stop_reason                               */
    int pressureIterations;   /* PCG iterations of the last outer iteration   */
    int momentumItersU, momentumItersV;
    double error;             /* max(residU, residV, residMass) as reported   */
    double residU, residV, residMass;          /* reported (raw or normalised) */
    double residU_RMS, residV_RMS, residMass_RMS;
    double residU_max, residV_max, residMass_max;
    double coreTotalDrop, fullTotalDrop;       /* total-pressure drop [Pa]     */
    double coreStaticDrop, fullStaticDrop;
    double inletMassFlux, outletMassFlux;      /* [kg/s per m depth]           */
    double device_ms;         /* device time of the call (CUDA events)         */
} cp_iter_report;

typedef struct cp_ctx cp_ctx;

/* Fills the SIMPLE.h defaults (pressureSolverType 4, maxPressureIter 30, ...). */
void cp_params_default(cp_params* p);

/* Reads "Ny Nx hy hx U N_in N_out [Ht]" like SIMPLE::loadParameters
 * (SIMPLE.cpp:31-66) into the grid fields of *p. */
cp_status cp_read_fluid_params(const char* path, cp_params* p);

/* Allocates the device state for p (validated first). Fields start at zero
 * and gamma at 1 (all fluid), like SIMPLE::initializeMemory. */
cp_status cp_create(const cp_params* p, cp_ctx** out);
cp_status cp_destroy(cp_ctx* ctx);

/* Geometry.  cellType: Ny x Nx, 0 fluid .. 1 solid (geometry_fluid.txt,
 * SIMPLE.cpp:633-690, converted as SIMPLE.cpp:695-777).  gamma: Ny x Nx
 * density, 1 fluid .. 0 solid (set directly, e.g. by an optimiser).  A
 * non-finite entry returns CP_ERR_NONFINITE and leaves the geometry as it
 * was.  The first call allocates a pinned (M x N doubles) staging array that
 * the context keeps for later calls and frees in cp_destroy. */
cp_status cp_set_cell_type(cp_ctx* ctx, const double* cellType, long rows, long cols,
                           long row_stride, long col_stride);
cp_status cp_set_gamma(cp_ctx* ctx, const double* gamma, long rows, long cols,
                       long row_stride, long col_stride);
cp_status cp_read_geometry(cp_ctx* ctx, const char* path);

/* Field transfer in the reference shapes (see cp_field). */
cp_status cp_get_field(cp_ctx* ctx, cp_field which, double* host, long rows, long cols,
                       long row_stride, long col_stride);
cp_status cp_set_field(cp_ctx* ctx, cp_field which, const double* host, long rows, long cols,
                       long row_stride, long col_stride);

/* Whole outer iterations: SIMPLE::calculateStep (iterations.cpp:82) plus the
 * pressure sampling and stop rules of SIMPLE::runIterations
 * (SIMPLE.cpp:378-491).  cp_step runs at most n_outer iterations (fewer if the
 * loop stops); cp_run runs until a stop rule fires.  `out` (may be NULL)
 * receives the last iteration's record. */
cp_status cp_step(cp_ctx* ctx, int n_outer, cp_iter_report* out);
cp_status cp_run(cp_ctx* ctx, cp_iter_report* out);
/* Clears the stop state so that cp_step/cp_run continue from the fields. */
cp_status cp_reset_loop(cp_ctx* ctx);
/* Back to the state after construction: u, v, p, u*, v*, p', dE, dN zero,
 * loop state and history cleared; geometry and parameters kept.  No
 * allocation, so repeated solves of one geometry reuse the device buffers. */
cp_status cp_reset(cp_ctx* ctx);

/* Solver-dispatch boundary of the reference (SIMPLE.h:876-880, 546):
 *   cp_momentum_u  ~ int solveUMomentumImplicit(SIMPLE&, float& residU)
 *   cp_momentum_v  ~ int solveVMomentumImplicit(SIMPLE&, float& residV)
 *   cp_pressure    ~ bool SIMPLE::solvePressureSystem(int&, float&)
 * They act on the device-resident u, v, p (cp_set_field) and write uStar /
 * vStar, dE / dN and pStar like the reference; *iters gets the Jacobi or PCG
 * iteration count, *resid the max |u* - u| and *residMass the max mass
 * imbalance. */
cp_status cp_momentum_u(cp_ctx* ctx, double* resid, int* iters);
cp_status cp_momentum_v(cp_ctx* ctx, double* resid, int* iters);
cp_status cp_pressure(cp_ctx* ctx, int* iters, double* residMass);

/* Pressure-correction solve that allocates no device memory.  No
 * counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc, e.g. a plugin inside a host application that has already
 * committed the whole device-memory budget to its own pool, or a
 * latency-bound control loop that must not stall in the allocator.  It runs
 * the same Jacobi-PCG as cp_pressure with pressureSolverType 1 and returns
 * the same p', iteration count and max mass imbalance.
 *
 * Inputs and output are device pointers the caller owns, row-major doubles
 * with one common row pitch `pitch` (elements, >= Nx + 2) in the reference
 * shapes: dE and uStar (Ny+2) x (Nx+1), dN and vStar (Ny+1) x (Nx+2), pStar
 * (Ny+2) x (Nx+2).  Only p->Ny, Nx, hx, hy, rho, pTol, maxPressureIter and
 * pressureSolverType (must be 1) are read.  `stream` is a cudaStream_t (or
 * NULL); the call returns after the solve has finished on it.
 *
 * Working memory: one fixed device array inside the library, which every GPU
 * that loads the library holds until the process exits.  It bounds the grid:
 * (Ny + 3) * pitch must not exceed 131072 (e.g. Ny 254 with Nx up to 509 at
 * pitch 512); larger grids return CP_ERR_BAD_PARAM.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before capturing any stream.
 * The address is kept with the context it was found in and looked up again
 * when the current context differs (after cudaDeviceReset, say), so such a
 * later call is again a first call.
 * All calls share the array, so calls that overlap on the GPU (other streams
 * or other threads) race and must be serialised by the caller. */
cp_status cp_pressure_noalloc(const cp_params* p, const double* dE, const double* dN, const double* uStar,
                              const double* vStar, long pitch, double* pStar, int* iters, double* residMass,
                              void* stream);

/* Discrete adjoint of the full-system total-pressure drop J (fullTotalDrop,
 * SIMPLE.cpp:432) with respect to the density field gamma, at the context's
 * current state (run the forward solve to convergence first).  New: the
 * reference has no flow adjoint.  grad receives dJ/dgamma for the Ny x Nx
 * cells (strides in elements).  The adjoint equations J_X^T lambda = dJ/dX
 * are solved by restarted flexible GMRES(30) with a transposed-SIMPLE
 * preconditioner; iteration stops when ||dJ/dX - J_X^T lambda|| <= tol
 * ||dJ/dX|| or after max_iter.  cp_params.adjointModel selects what is
 * differentiated (cp_adjoint_model); the report says which model ran. */
typedef enum cp_adjoint_model {
    CP_ADJ_AUTO = 0,         /* FIXED_POINT where the state is a fixed point of the
                                iteration with velocities on the clamp, else
                                EQUATIONS                                          */
    CP_ADJ_EQUATIONS = 1,    /* the discretisation R(X) = 0: exact with no velocity
                                on the clamp (R = 0 holds there at a fixed point)  */
    CP_ADJ_FIXED_POINT = 2   /* the iteration's fixed point with the Jacobi sweep
                                count and the clamped unknowns frozen: the momentum
                                rows are s Jacobi sweeps from u (their result must
                                equal u), clamped unknowns stay at +-maxVel        */
} cp_adjoint_model;
typedef struct cp_adjoint_report {
    int iterations;        /* FGMRES iterations run                     */
    int converged;         /* 1 if the relative residual reached tol    */
    double residual;       /* final relative residual                   */
    double J;              /* pressure drop evaluated at the state [Pa] */
    double device_ms;      /* device time of the adjoint (CUDA events)  */
    int model;             /* cp_adjoint_model used (EQUATIONS or FIXED_POINT) */
    int clampedUnknowns;   /* velocity unknowns the scatter clamps at the state */
} cp_adjoint_report;
cp_status cp_adjoint_dp_dgamma(cp_ctx* ctx, double* grad, long rows, long cols, long row_stride,
                               long col_stride, int max_iter, double tol, cp_adjoint_report* rep);

/* Verification of the adjoint (tests): at the current state and with the
 * model cp_adjoint_dp_dgamma would use, op 0 writes y = J_X^T x, op 1
 * y = dJ/dX and op 2 the adjoint solution lambda (FGMRES with max_iter /
 * tol as above; rep filled).  x and y hold cp_adjoint_probe_len(ctx)
 * doubles: the U, V and continuity (pressure) blocks, each in the solver's
 * padded layout (row pitch info[3], element (i, j) of the staggered field at
 * i * pitch + j); entries outside the unknowns are zero in y and ignored in
 * x.  info[0..2] = model, U and V Jacobi sweep counts of the state. */
size_t cp_adjoint_probe_len(const cp_ctx* ctx);
cp_status cp_adjoint_probe(cp_ctx* ctx, int op, const double* x, double* y, int max_iter, double tol, int* info,
                           cp_adjoint_report* rep);

/* Per-iteration history rows (cp_iter_report layout without device_ms, as
 * doubles: see cp_history_columns()).  Returns the number of rows copied. */
int cp_history_columns(void);
cp_status cp_get_history(cp_ctx* ctx, double* rows, int max_rows, int* n_rows);

/* Per-kernel device time (CUDA events around each launch) over n_outer
 * iterations run without graph capture; the native counterpart of the
 * reference's GlobalTimer / ScopedTimer phases (Utilities/Timer.h:12-82).
 * Kernel kinds: see cp_kernel_kind.  The iterations advance the solution
 * like cp_step. */
typedef enum cp_kernel_kind {
    CP_K_BC = 0, CP_K_ASSEMBLE, CP_K_JACOBI, CP_K_MASS, CP_K_PCG, CP_K_CORRECT, CP_K_FINALIZE,
    CP_K_COUNT
} cp_kernel_kind;
typedef struct cp_kernel_timing {
    double ms[CP_K_COUNT];      /* summed device time per kind            */
    int launches[CP_K_COUNT];   /* launches per kind                      */
    long long jacobiSweeps;     /* sweeps (U + V) run by the Jacobi kernel */
    long long pcgIterations;    /* PCG iterations run                      */
    int iterations;             /* outer iterations timed                  */
} cp_kernel_timing;
cp_status cp_kernel_times(cp_ctx* ctx, int n_outer, cp_kernel_timing* out);

/* ---------------------------------------------------------------- batches
 * New (the reference runs one field per process, run_solvers.py:248): many
 * fields, each its own context with its own grid size, geometry and
 * parameters, advanced together by one persistent cooperative kernel per
 * launch.  Two schedules:
 *   - teams (every field pressureSolverType 4): the grid is cut into teams
 *     of consecutive CTAs; each team takes the next field from a queue
 *     (largest first) and runs its outer iterations with the single-field
 *     device code (smoothed-aggregation PCG included) on its own barrier;
 *     the autotuner picks the team size;
 *   - cell tiles (otherwise; pressureSolverType 2 or 4, every field on the
 *     2 x 2 aggregation cycle): every phase covers the rows x cols cell
 *     tiles of all fields still iterating; the autotuner picks the tile.
 * Each field keeps its own stop rules (Jacobi, CG and outer loop), history
 * and status, so cp_get_field, cp_get_history and cp_adjoint_dp_dgamma work
 * on a field's context after a batch run as after cp_step.  Requirements:
 * pressureSolverType 2 or 4, the same precision for every field, contexts on
 * one device.  The contexts must outlive the batch and must not be stepped
 * while a batch call runs. */
typedef struct cp_batch cp_batch;
typedef struct cp_batch_report {
    int outerIterations;   /* largest completed outer iteration count     */
    int fieldsDone;        /* fields whose loop has stopped               */
    int launches;          /* persistent-kernel launches (64 iterations each at most) */
    int tileRows, tileCols;/* cell tile used (0 in team mode)             */
    double device_ms;      /* device time of the call (CUDA events)       */
    int teamCtas;          /* CTAs per team (0 in cell-tile mode)         */
} cp_batch_report;
cp_status cp_batch_create(cp_ctx* const* fields, int n, cp_batch** out);
cp_status cp_batch_destroy(cp_batch* batch);
/* rows x cols in [256, 4096]; the default is 16 x 64 (cell-tile mode) */
cp_status cp_batch_set_tile(cp_batch* batch, int rows, int cols);
/* CTAs per team in [1, SMs]; the default is 4; CP_ERR_UNSUPPORTED in
 * cell-tile mode */
cp_status cp_batch_set_team(cp_batch* batch, int ctas);
/* Runs until every field has stopped or max_outer iterations, in launches of
 * up to 64 outer iterations replayed from a captured CUDA graph. */
cp_status cp_batch_run(cp_batch* batch, int max_outer, cp_batch_report* rep);
/* Times trial_outer iterations from the initial state for each candidate tile
 * shape (team mode: team size), keeps the fastest, and resets every field
 * (cp_reset) afterwards. */
cp_status cp_batch_autotune(cp_batch* batch, int trial_outer, cp_batch_report* best);

/* Self-test of the bounded device waits.  The persistent kernels wait on
 * grid barriers (kind 0) and the TMA pipelines on mbarriers (kind 1); each
 * wait gives up after a time limit and records CP_ERR_TIMEOUT instead of
 * holding the GPU.  This call runs one wait of the given kind on an event
 * that never comes (a second block that does not exist, an mbarrier phase
 * nobody arrives on) with a limit of limit_seconds (at most 10), and writes
 * the status word the kernel left into *device_status: CP_ERR_TIMEOUT when
 * the give-up path works.  Returns CP_OK when the launch itself succeeded.
 * No counterpart in the reference. */
cp_status cp_selftest_bounded_wait(int kind, double limit_seconds, int* device_status);

const char* cp_status_string(cp_status s);
const char* cp_last_error_string(void);

#ifdef __cplusplus
}
#endif

#endif /* CP_SIMPLE_H */
