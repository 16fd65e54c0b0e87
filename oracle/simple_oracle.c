/*
 * CPU restatement of the reference's 2-D staggered-grid SIMPLE iteration
 * (Carloossgg/coldplate-solver), single threaded and deterministic.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the parity tests check the
 * CUDA path against; the product never links, loads or calls it.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * The file is compiled twice: -DORC_REAL=float (the reference as shipped,
 * float32 storage, SIMPLE.h:479-525) and -DORC_REAL=double (the reference
 * re-typed to double, the FP64 parity oracle).  Every exported symbol gets a
 * _f32 / _f64 suffix.  With -ffp-contract=off the float build reproduces the
 * reference compiled the same way bit for bit (pinned by tests against
 * oracle/_ref/ref_f32_pin and ref_f64_pin): the arithmetic below keeps the
 * reference's operation order wherever rounding depends on it, while the
 * data layout is its own (row-major arrays, matrix-free stencils instead of
 * the reference's CSR, no DOF maps).
 *
 * Index conventions follow the reference: M = Ny + 1, N = Nx + 1
 * (SIMPLE.cpp:53-54); u is (M+1) x N, v is M x (N+1), p is (M+1) x (N+1),
 * cell fields (gamma, alpha, cellType) are M x N (SIMPLE.cpp:252-273).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL real;

#define ORC_IS_FLOAT (sizeof(real) == 4)
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#ifdef ORC_FLOAT
#define ORC(name) CAT(name, _f32)
#define RL(x) CAT(x, f) /* literal with the float suffix, as in the sources */
#define RSQRT sqrtf
#define RABS fabsf
#define RFLOOR floorf
#define SCAN_FMT "%f"
#else
#define ORC(name) CAT(name, _f64)
#define RL(x) x
#define RSQRT sqrt
#define RABS fabs
#define RFLOOR floor
#define SCAN_FMT "%lf"
#endif

/* std::max / std::min / std::clamp semantics (first argument wins ties). */
static inline real rmax(real a, real b) { return (a < b) ? b : a; }
static inline real rmin(real a, real b) { return (b < a) ? b : a; }
static inline real rclamp(real x, real lo, real hi) { return (x < lo) ? lo : ((hi < x) ? hi : x); }

/* ------------------------------------------------------------------------ */
/* Parameters: the SIMPLE.h knobs that reach the hot path (SIMPLE.h:68-411). */
/* Passed in double by the caller and narrowed to `real` like the reference  */
/* narrows its literals.                                                      */
typedef struct {
    double epsilon;
    int maxIterations;
    int maxPressureIter;
    double pTol;
    int pressureSolverType;
    int momentumSolverType;
    double momentumTol;
    int maxMomentumIter;
    int convectionScheme;
    int enableTwoPointFiveD;
    double twoPointFiveDConvectionFactor;
    double twoPointFiveDSinkMultiplier;
    double brinkmanKMin;
    double brinkmanQ;
    double rho;
    double eta;
    double uvAlpha;
    double pAlpha;
    double xPlaneCoreInlet;
    double xPlaneCoreOutlet;
    int enableInletRamp;
    int rampSteps;
    int enableNormalizedResiduals;
    double residNormFloorVel;
    double residNormFloorMass;
} orc_params;

typedef struct {
    int M, N;
    real hx, hy, targetVel, inletVelocity, Ht;
    /* narrowed parameters */
    real epsilon, pTol, momentumTol, convFactor, sinkMult, KMin, q, rho, eta;
    real uvAlpha, pAlpha, xCoreIn, xCoreOut, alphaMax, velFloor, massFloor;
    int maxIterations, maxPressureIter, maxMomentumIter, convectionScheme, twoPointFiveD;
    int pressureSolverType, momentumSolverType, enableInletRamp, rampSteps, normalized;
    /* fields */
    real *u, *v, *p, *uStar, *vStar, *pStar, *uOld, *vOld, *dE, *dN;
    real *cellType, *gamma, *alpha;
    /* momentum scratch: coefficients of the last assembled system (U or V) */
    real *cP, *cE, *cW, *cN, *cS, *cB, *x0, *x1;
    /* pressure scratch */
    real *pr, *pz, *pp, *pAp, *pdiag, *pb, *px;
    /* scalars (SIMPLE.h:426-448) */
    real residU, residV, residMass, residU_max, residV_max, residMass_max;
    real residU_RMS, residV_RMS, residMass_RMS, residU_RMS0, residV_RMS0, residMass_RMS0;
    int rmsU0set, rmsV0set, rmsM0set;
    int lastMomItersU, lastMomItersV, lastPressureIters, iter;
    double lastError;   /* error of the last completed iteration (1 before any) */
} orc_state;

#define UI(s, i, j) ((size_t)(i) * (size_t)(s)->N + (size_t)(j))        /* u, dE: (M+1) x N */
#define VI(s, i, j) ((size_t)(i) * (size_t)((s)->N + 1) + (size_t)(j))  /* v, dN: M x (N+1) */
#define PI_(s, i, j) ((size_t)(i) * (size_t)((s)->N + 1) + (size_t)(j)) /* p: (M+1) x (N+1) */
#define CI(s, i, j) ((size_t)(i) * (size_t)(s)->N + (size_t)(j))        /* cells: M x N */

static real* alloc0(size_t n) { return (real*)calloc(n ? n : 1, sizeof(real)); }

/* ------------------------------------------------------------------------ */
/* Set-up: SIMPLE::loadParameters / loadTopology / loadDensityField /         */
/* buildAlphaFromDensity (SIMPLE.cpp:31-101, 633-777).                        */

static void apply_params(orc_state* s, const orc_params* prm) {
    s->epsilon = (real)prm->epsilon;
    s->maxIterations = prm->maxIterations;
    s->maxPressureIter = prm->maxPressureIter;
    s->pTol = (real)prm->pTol;
    s->pressureSolverType = prm->pressureSolverType;
    s->momentumSolverType = prm->momentumSolverType;
    s->momentumTol = (real)prm->momentumTol;
    s->maxMomentumIter = prm->maxMomentumIter;
    s->convectionScheme = prm->convectionScheme;
    s->twoPointFiveD = prm->enableTwoPointFiveD;
    s->convFactor = (real)prm->twoPointFiveDConvectionFactor;
    s->sinkMult = (real)prm->twoPointFiveDSinkMultiplier;
    s->KMin = (real)prm->brinkmanKMin;
    s->q = (real)prm->brinkmanQ;
    s->rho = (real)prm->rho;
    s->eta = (real)prm->eta;
    s->uvAlpha = (real)prm->uvAlpha;
    s->pAlpha = (real)prm->pAlpha;
    s->xCoreIn = (real)prm->xPlaneCoreInlet;
    s->xCoreOut = (real)prm->xPlaneCoreOutlet;
    s->enableInletRamp = prm->enableInletRamp;
    s->rampSteps = prm->rampSteps;
    s->normalized = prm->enableNormalizedResiduals;
    s->velFloor = (real)prm->residNormFloorVel;
    s->massFloor = (real)prm->residNormFloorMass;
    /* 2.5-D needs a positive height (SIMPLE.cpp:67-73). */
    if (s->twoPointFiveD && s->Ht <= RL(0.0)) s->twoPointFiveD = 0;
    /* alpha_max = mu / K_min (SIMPLE.cpp:78-79) */
    s->alphaMax = s->eta / rmax(s->KMin, RL(1e-20));
}

/* gamma = 1 - clamp(cellType, 0, 1) with the padded row/column copied
 * (SIMPLE.cpp:667-676, 707-729); alpha by RAMP (SIMPLE.cpp:766-772). */
static void build_density(orc_state* s) {
    const int M = s->M, N = s->N, pr = M - 1, pc = N - 1;
    for (int i = 0; i < pr; ++i) s->cellType[CI(s, i, pc)] = s->cellType[CI(s, i, pc - 1)];
    for (int j = 0; j < N; ++j) {
        int src = j < pc - 1 ? j : pc - 1;
        s->cellType[CI(s, pr, j)] = s->cellType[CI(s, pr - 1, src)];
    }
    for (size_t k = 0; k < (size_t)M * N; ++k) s->gamma[k] = RL(1.0);
    for (int i = 0; i < pr; ++i)
        for (int j = 0; j < pc; ++j) {
            real val = s->cellType[CI(s, i, j)];
            real vc = rmax(RL(0.0), rmin(RL(1.0), val));
            s->gamma[CI(s, i, j)] = RL(1.0) - vc;
        }
    for (int i = 0; i < pr; ++i) s->gamma[CI(s, i, pc)] = s->gamma[CI(s, i, pc - 1)];
    for (int j = 0; j < N; ++j) {
        int src = j < pc - 1 ? j : pc - 1;
        s->gamma[CI(s, pr, j)] = s->gamma[CI(s, pr - 1, src)];
    }
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < N; ++j) {
            real g = s->gamma[CI(s, i, j)];
            s->alpha[CI(s, i, j)] = s->alphaMax * (RL(1.0) - g) / (RL(1.0) + s->q * g + RL(1e-10));
        }
}

static orc_state* state_alloc(int Ny, int Nx) {
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    s->M = Ny + 1;
    s->N = Nx + 1;
    const size_t M = (size_t)s->M, N = (size_t)s->N;
    const size_t nu = (M + 1) * N, nv = M * (N + 1), np = (M + 1) * (N + 1), nc = M * N;
    s->u = alloc0(nu); s->uStar = alloc0(nu); s->uOld = alloc0(nu); s->dE = alloc0(nu);
    s->v = alloc0(nv); s->vStar = alloc0(nv); s->vOld = alloc0(nv); s->dN = alloc0(nv);
    s->p = alloc0(np); s->pStar = alloc0(np);
    s->cellType = alloc0(nc); s->gamma = alloc0(nc); s->alpha = alloc0(nc);
    const size_t nm = (M + 1) * (N + 1);
    s->cP = alloc0(nm); s->cE = alloc0(nm); s->cW = alloc0(nm); s->cN = alloc0(nm);
    s->cS = alloc0(nm); s->cB = alloc0(nm); s->x0 = alloc0(nm); s->x1 = alloc0(nm);
    s->pr = alloc0(nm); s->pz = alloc0(nm); s->pp = alloc0(nm); s->pAp = alloc0(nm);
    s->pdiag = alloc0(nm); s->pb = alloc0(nm); s->px = alloc0(nm);
    s->residU = s->residV = s->residMass = RL(1.0);
    s->residU_max = s->residV_max = s->residMass_max = RL(1.0);
    s->lastError = 1.0;
    return s;
}

/* Create from arrays: cellType is Ny x Nx row-major (0 fluid, 1 solid). */
orc_state* ORC(orc_create)(const orc_params* prm, int Ny, int Nx, double hy, double hx,
                           double targetVel, double Ht, const double* cellType) {
    if (Ny < 2 || Nx < 3) return NULL;
    orc_state* s = state_alloc(Ny, Nx);
    s->hy = (real)hy; s->hx = (real)hx; s->targetVel = (real)targetVel; s->Ht = (real)Ht;
    s->inletVelocity = RL(0.0);
    apply_params(s, prm);
    for (int i = 0; i < Ny; ++i)
        for (int j = 0; j < Nx; ++j) s->cellType[CI(s, i, j)] = (real)cellType[(size_t)i * Nx + j];
    build_density(s);
    return s;
}

/* Create from a reference case directory: ExportFiles/fluid_params.txt
 * ("Ny Nx hy hx U N_in N_out [Ht]", SIMPLE.cpp:41-59) and
 * ExportFiles/geometry_fluid.txt (Ny rows x Nx values, SIMPLE.cpp:653-662),
 * parsed in the working precision like the reference's stream reads. */
orc_state* ORC(orc_create_from_case)(const orc_params* prm, const char* caseDir) {
    char path[4096];
    snprintf(path, sizeof path, "%s/ExportFiles/fluid_params.txt", caseDir);
    FILE* f = fopen(path, "r");
    if (!f) return NULL;
    int Ny = 0, Nx = 0, nin = 0, nout = 0;
    real hy = 0, hx = 0, U = 0, Ht = 0;
    if (fscanf(f, "%d %d " SCAN_FMT " " SCAN_FMT " " SCAN_FMT " %d %d", &Ny, &Nx, &hy, &hx, &U, &nin, &nout) != 7) {
        fclose(f);
        return NULL;
    }
    if (fscanf(f, " " SCAN_FMT, &Ht) != 1) Ht = 0;
    fclose(f);
    if (Ny < 2 || Nx < 3) return NULL;
    orc_state* s = state_alloc(Ny, Nx);
    s->hy = hy; s->hx = hx; s->targetVel = U; s->Ht = Ht;
    apply_params(s, prm);
    snprintf(path, sizeof path, "%s/ExportFiles/geometry_fluid.txt", caseDir);
    f = fopen(path, "r");
    if (f) {
        int done = 0;
        for (int i = 0; i < Ny && !done; ++i)
            for (int j = 0; j < Nx; ++j) {
                real val;
                if (fscanf(f, " " SCAN_FMT, &val) != 1) { done = 1; break; }
                s->cellType[CI(s, i, j)] = val;
            }
        fclose(f);
    }
    build_density(s);
    return s;
}

void ORC(orc_destroy)(orc_state* s) {
    if (!s) return;
    real* arrs[] = {s->u, s->v, s->p, s->uStar, s->vStar, s->pStar, s->uOld, s->vOld, s->dE, s->dN,
                    s->cellType, s->gamma, s->alpha, s->cP, s->cE, s->cW, s->cN, s->cS, s->cB,
                    s->x0, s->x1, s->pr, s->pz, s->pp, s->pAp, s->pdiag, s->pb, s->px};
    for (size_t k = 0; k < sizeof arrs / sizeof arrs[0]; ++k) free(arrs[k]);
    free(s);
}

/* ------------------------------------------------------------------------ */
/* Boundary conditions (boundaries.cpp:50-146)                                */

/* inlet mask: gamma(cellRow, 0) > 0.5 with the corner rows mapped to the
 * nearest physical row (boundaries.cpp:82-96) */
static int inlet_fluid(const orc_state* s, int uRow) {
    const int M = s->M;
    int cellRow = uRow <= 0 ? 0 : (uRow >= M ? (M - 2 > 0 ? M - 2 : 0) : uRow - 1);
    if (cellRow < 0) cellRow = 0;
    if (cellRow > M - 1) cellRow = M - 1;
    return s->gamma[CI(s, cellRow, 0)] > RL(0.5);
}

void ORC(orc_velocity_bc)(orc_state* s, real* u, real* v) {
    const int M = s->M, N = s->N;
    const real Uin = s->inletVelocity;
    for (int j = 0; j < N; ++j) u[UI(s, 0, j)] = RL(0.0);
    for (int j = 0; j < N + 1; ++j) v[VI(s, 0, j)] = RL(0.0);
    for (int j = 0; j < N; ++j) u[UI(s, M, j)] = RL(0.0);
    for (int j = 0; j < N + 1; ++j) v[VI(s, M - 1, j)] = RL(0.0);
    for (int i = 0; i <= M; ++i) u[UI(s, i, 0)] = inlet_fluid(s, i) ? Uin : RL(0.0);
    for (int i = 0; i < M; ++i) v[VI(s, i, 0)] = RL(0.0);
    for (int i = 0; i < M + 1; ++i) u[UI(s, i, N - 1)] = u[UI(s, i, N - 2)];
    for (int i = 0; i < M; ++i) v[VI(s, i, N)] = v[VI(s, i, N - 1)];
}

void ORC(orc_pressure_bc)(orc_state* s, real* p) {
    const int M = s->M, N = s->N;
    for (int j = 1; j < N; ++j) {
        p[PI_(s, 0, j)] = p[PI_(s, 1, j)];
        p[PI_(s, M, j)] = p[PI_(s, M - 1, j)];
    }
    for (int i = 1; i < M; ++i) p[PI_(s, i, 0)] = p[PI_(s, i, 1)];
    for (int i = 1; i < M; ++i) p[PI_(s, i, N)] = RL(0.0);
}

/* ------------------------------------------------------------------------ */
/* Face interpolation of cell fields (SIMPLE.h:642-686, 740-778)              */

static real alpha_at_u(const orc_state* s, int i, int j) {
    if (i < 1 || i >= s->M || j < 1 || j >= s->N - 1) return RL(0.0);
    return RL(0.5) * (s->alpha[CI(s, i - 1, j - 1)] + s->alpha[CI(s, i - 1, j)]);
}
static real alpha_at_v(const orc_state* s, int i, int j) {
    if (i < 1 || i >= s->M - 1 || j < 1 || j >= s->N) return RL(0.0);
    return RL(0.5) * (s->alpha[CI(s, i - 1, j - 1)] + s->alpha[CI(s, i, j - 1)]);
}
static real gamma_at_u(const orc_state* s, int i, int j) {
    if (i < 1 || i >= s->M || j < 1 || j >= s->N - 1) return RL(1.0);
    return RL(0.5) * (s->gamma[CI(s, i - 1, j - 1)] + s->gamma[CI(s, i - 1, j)]);
}
static real gamma_at_v(const orc_state* s, int i, int j) {
    if (i < 1 || i >= s->M - 1 || j < 1 || j >= s->N) return RL(1.0);
    return RL(0.5) * (s->gamma[CI(s, i - 1, j - 1)] + s->gamma[CI(s, i, j - 1)]);
}

/* Face-local half-cell wall flags (boundaries.cpp:148-206); fluidTol 0.999. */
static int wall_south_u(const orc_state* s, int i, int j) {
    if (i - 1 != 0) return 0;
    if (j < 1 || j > s->N - 2) return 0;
    if (gamma_at_u(s, i, j) < RL(0.999)) return 0;
    const real tol = RL(1e-8);
    int uz = RABS(s->u[UI(s, 0, j)]) <= tol;
    int vz = RABS(s->v[VI(s, 0, j)]) <= tol && RABS(s->v[VI(s, 0, j + 1)]) <= tol;
    return uz && vz;
}
static int wall_north_u(const orc_state* s, int i, int j) {
    if (i + 1 != s->M) return 0;
    if (j < 1 || j > s->N - 2) return 0;
    if (gamma_at_u(s, i, j) < RL(0.999)) return 0;
    const real tol = RL(1e-8);
    int uz = RABS(s->u[UI(s, s->M, j)]) <= tol;
    int vz = RABS(s->v[VI(s, s->M - 1, j)]) <= tol && RABS(s->v[VI(s, s->M - 1, j + 1)]) <= tol;
    return uz && vz;
}
static int wall_west_v(const orc_state* s, int i, int j) {
    if (j - 1 != 0) return 0;
    if (i < 1 || i > s->M - 2) return 0;
    if (gamma_at_v(s, i, j) < RL(0.999)) return 0;
    const real tol = RL(1e-8);
    if (RABS(s->targetVel) > tol) return 0;
    int vz = RABS(s->v[VI(s, i, 0)]) <= tol;
    int uz = RABS(s->u[UI(s, i, 0)]) <= tol && RABS(s->u[UI(s, i + 1, 0)]) <= tol;
    return vz && uz;
}
static int wall_east_v(const orc_state* s, int i, int j) {
    if (j + 1 != s->N) return 0;
    if (i < 1 || i > s->M - 2) return 0;
    if (gamma_at_v(s, i, j) < RL(0.999)) return 0;
    const real tol = RL(1e-8);
    if (RABS(s->p[PI_(s, i, s->N)]) <= tol) return 0;
    int vz = RABS(s->v[VI(s, i, s->N)]) <= tol;
    int uz = RABS(s->u[UI(s, i, s->N - 1)]) <= tol && RABS(s->u[UI(s, i + 1, s->N - 1)]) <= tol;
    return vz && uz;
}

/* Mask export for bit-exact mask tests: per DOF flags, bit0 S/W, bit1 N/E. */
void ORC(orc_wall_flags)(const orc_state* s, int isU, unsigned char* out) {
    const int M = s->M, N = s->N;
    if (isU) {
        for (int i = 1; i < M; ++i)
            for (int j = 1; j < N - 1; ++j)
                out[(size_t)(i - 1) * (N - 2) + (j - 1)] =
                    (unsigned char)(wall_south_u(s, i, j) | (wall_north_u(s, i, j) << 1));
    } else {
        for (int i = 1; i < M - 1; ++i)
            for (int j = 1; j < N; ++j)
                out[(size_t)(i - 1) * (N - 1) + (j - 1)] =
                    (unsigned char)(wall_west_v(s, i, j) | (wall_east_v(s, i, j) << 1));
    }
}

/* ------------------------------------------------------------------------ */
/* SOU deferred correction (convection.cpp:53-186)                            */

static real sou_u(const orc_state* s, int i, int j, real Fe, real Fw, real Fn, real Fs) {
    const int M = s->M, N = s->N;
    const real* u = s->u;
#define U_(a, b) u[UI(s, (a), (b))]
    real S = RL(0.0);
    if (Fe >= RL(0.0)) {
        if (j >= 2) S -= Fe * ((RL(1.5) * U_(i, j) - RL(0.5) * U_(i, j - 1)) - U_(i, j));
    } else {
        if (j + 2 < N) S -= Fe * ((RL(1.5) * U_(i, j + 1) - RL(0.5) * U_(i, j + 2)) - U_(i, j + 1));
    }
    if (Fw >= RL(0.0)) {
        if (j >= 2) S += Fw * ((RL(1.5) * U_(i, j - 1) - RL(0.5) * U_(i, j - 2)) - U_(i, j - 1));
    } else {
        if (j + 1 < N) S += Fw * ((RL(1.5) * U_(i, j) - RL(0.5) * U_(i, j + 1)) - U_(i, j));
    }
    if (Fn >= RL(0.0)) {
        if (i >= 1) S -= Fn * ((RL(1.5) * U_(i, j) - RL(0.5) * U_(i - 1, j)) - U_(i, j));
    } else {
        if (i + 2 <= M) S -= Fn * ((RL(1.5) * U_(i + 1, j) - RL(0.5) * U_(i + 2, j)) - U_(i + 1, j));
    }
    if (Fs >= RL(0.0)) {
        if (i >= 2) S += Fs * ((RL(1.5) * U_(i - 1, j) - RL(0.5) * U_(i - 2, j)) - U_(i - 1, j));
    } else {
        if (i + 1 <= M) S += Fs * ((RL(1.5) * U_(i, j) - RL(0.5) * U_(i + 1, j)) - U_(i, j));
    }
#undef U_
    return S;
}

static real sou_v(const orc_state* s, int i, int j, real Fe, real Fw, real Fn, real Fs) {
    const int M = s->M, N = s->N;
    const real* v = s->v;
#define V_(a, b) v[VI(s, (a), (b))]
    real S = RL(0.0);
    if (Fe >= RL(0.0)) {
        if (j >= 2) S -= Fe * ((RL(1.5) * V_(i, j) - RL(0.5) * V_(i, j - 1)) - V_(i, j));
    } else {
        if (j + 2 <= N) S -= Fe * ((RL(1.5) * V_(i, j + 1) - RL(0.5) * V_(i, j + 2)) - V_(i, j + 1));
    }
    if (Fw >= RL(0.0)) {
        if (j >= 2) S += Fw * ((RL(1.5) * V_(i, j - 1) - RL(0.5) * V_(i, j - 2)) - V_(i, j - 1));
    } else {
        if (j + 1 <= N) S += Fw * ((RL(1.5) * V_(i, j) - RL(0.5) * V_(i, j + 1)) - V_(i, j));
    }
    if (Fn >= RL(0.0)) {
        if (i >= 1) S -= Fn * ((RL(1.5) * V_(i, j) - RL(0.5) * V_(i - 1, j)) - V_(i, j));
    } else {
        if (i + 2 < M) S -= Fn * ((RL(1.5) * V_(i + 1, j) - RL(0.5) * V_(i + 2, j)) - V_(i + 1, j));
    }
    if (Fs >= RL(0.0)) {
        if (i >= 2) S += Fs * ((RL(1.5) * V_(i - 1, j) - RL(0.5) * V_(i - 2, j)) - V_(i - 1, j));
    } else {
        if (i + 1 < M) S += Fs * ((RL(1.5) * V_(i, j) - RL(0.5) * V_(i + 1, j)) - V_(i, j));
    }
#undef V_
    return S;
}

/* ------------------------------------------------------------------------ */
/* Momentum: assembly (momentum_solver.cpp:197-314), Jacobi                   */
/* (jacobi_solver.cpp:20-75), scatter + clamp + max change (:335-351).        */
/* The system of one component is kept matrix-free in cP..cS (0 where the     */
/* neighbour is not an unknown) and cB, indexed like the component's field.   */

static real max_vel(const orc_state* s) { return RL(3.0) * rmax(RABS(s->inletVelocity), RL(0.1)); }

void ORC(orc_assemble)(orc_state* s, int isU) {
    const int M = s->M, N = s->N;
    const real hx = s->hx, hy = s->hy, vol = hx * hy, rho = s->rho, eta = s->eta;
    const real maxVel = max_vel(s);
    const real sinkCoeff = (s->twoPointFiveD && s->Ht > RL(0.0))
                               ? s->sinkMult * (RL(12.0) * eta / (s->Ht * s->Ht)) : RL(0.0);
    const real sinkDiag = sinkCoeff * vol;
    const real DeScale = hy / hx, DnScale = hx / hy;
    const real convScale = s->twoPointFiveD ? s->convFactor : RL(1.0);
    const int i0 = 1, i1 = isU ? M - 1 : M - 2, j0 = 1, j1 = isU ? N - 2 : N - 1;
    const real* u = s->u;
    const real* v = s->v;
    const real* p = s->p;
    for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j) {
            const size_t k = isU ? UI(s, i, j) : VI(s, i, j);
            real alphaLocal = isU ? alpha_at_u(s, i, j) : alpha_at_v(s, i, j);
            real ue, uw, vn, vs;
            if (isU) {
                ue = rclamp(RL(0.5) * (u[UI(s, i, j)] + u[UI(s, i, j + 1)]), -maxVel, maxVel);
                uw = rclamp(RL(0.5) * (u[UI(s, i, j - 1)] + u[UI(s, i, j)]), -maxVel, maxVel);
                vn = rclamp(RL(0.5) * (v[VI(s, i, j)] + v[VI(s, i, j + 1)]), -maxVel, maxVel);
                vs = rclamp(RL(0.5) * (v[VI(s, i - 1, j)] + v[VI(s, i - 1, j + 1)]), -maxVel, maxVel);
            } else {
                ue = rclamp(RL(0.5) * (u[UI(s, i, j)] + u[UI(s, i + 1, j)]), -maxVel, maxVel);
                uw = rclamp(RL(0.5) * (u[UI(s, i, j - 1)] + u[UI(s, i + 1, j - 1)]), -maxVel, maxVel);
                vn = rclamp(RL(0.5) * (v[VI(s, i, j)] + v[VI(s, i + 1, j)]), -maxVel, maxVel);
                vs = rclamp(RL(0.5) * (v[VI(s, i - 1, j)] + v[VI(s, i, j)]), -maxVel, maxVel);
            }
            real Fe = convScale * rho * hy * ue, Fw = convScale * rho * hy * uw;
            real Fn = convScale * rho * hx * vn, Fs = convScale * rho * hx * vs;
            real De = eta * DeScale, Dn = eta * DnScale;
            real aE = De + rmax(RL(0.0), -Fe);
            real aW = De + rmax(RL(0.0), Fw);
            real aN = Dn + rmax(RL(0.0), -Fn);
            real aS = Dn + rmax(RL(0.0), Fs);
            if (isU) {
                if (wall_south_u(s, i, j)) aS += Dn;
                if (wall_north_u(s, i, j)) aN += Dn;
            } else {
                if (wall_west_v(s, i, j)) aW += De;
                if (wall_east_v(s, i, j)) aE += De;
            }
            real sumA = aE + aW + aN + aS;
            real transCoeff = RL(0.0);
            real brinkmanDrag = alphaLocal * vol;
            real aP0 = sumA + (Fe - Fw + Fn - Fs) + transCoeff + sinkDiag + brinkmanDrag;
            aP0 = rmax(aP0, RL(1e-10));
            real aP = aP0 / s->uvAlpha;
            real Sp, velOld, velCur;
            if (isU) {
                Sp = (p[PI_(s, i, j)] - p[PI_(s, i, j + 1)]) * hy;
                velOld = s->uOld[UI(s, i, j)]; velCur = u[UI(s, i, j)];
            } else {
                Sp = (p[PI_(s, i, j)] - p[PI_(s, i + 1, j)]) * hx;
                velOld = s->vOld[VI(s, i, j)]; velCur = v[VI(s, i, j)];
            }
            Sp += transCoeff * velOld;
            Sp += (RL(1.0) - s->uvAlpha) / s->uvAlpha * aP0 * velCur;
            if (s->convectionScheme == 1) Sp += isU ? sou_u(s, i, j, Fe, Fw, Fn, Fs) : sou_v(s, i, j, Fe, Fw, Fn, Fs);
            if (isU) s->dE[k] = hy / aP0; else s->dN[k] = hx / aP0;
            /* neighbours that are not unknowns move to the right-hand side
             * with their current value, in the order E, W, N, S (:300-311) */
            const real* f = isU ? u : v;
            const int eIn = j + 1 <= j1, wIn = j - 1 >= j0, nIn = i + 1 <= i1, sIn = i - 1 >= i0;
            const size_t kE = isU ? UI(s, i, j + 1) : VI(s, i, j + 1);
            const size_t kW = isU ? UI(s, i, j - 1) : VI(s, i, j - 1);
            const size_t kN = isU ? UI(s, i + 1, j) : VI(s, i + 1, j);
            const size_t kS = isU ? UI(s, i - 1, j) : VI(s, i - 1, j);
            s->cP[k] = aP;
            if (eIn) s->cE[k] = aE; else { s->cE[k] = RL(0.0); Sp += aE * f[kE]; }
            if (wIn) s->cW[k] = aW; else { s->cW[k] = RL(0.0); Sp += aW * f[kW]; }
            if (nIn) s->cN[k] = aN; else { s->cN[k] = RL(0.0); Sp += aN * f[kN]; }
            if (sIn) s->cS[k] = aS; else { s->cS[k] = RL(0.0); Sp += aS * f[kS]; }
            s->x0[k] = f[k];
            s->cB[k] = Sp;
        }
}

/* Jacobi sweeps on the assembled component.  The reference sums a CSR row in
 * column order S, W, P, E, N with -a for off-diagonals; absent neighbours
 * have no entry at all (so they are skipped, not multiplied by zero). */
int ORC(orc_jacobi)(orc_state* s, int isU, real* resid_sq_out) {
    const int M = s->M, N = s->N;
    const int i1 = isU ? M - 1 : M - 2, j1 = isU ? N - 2 : N - 1;
    const int n = i1 * j1;
    const int stride = isU ? N : N + 1;
    if (n == 0) return 0;
    real* xc = s->x0;
    real* xn = s->x1;
    const real tol_sq = s->momentumTol * s->momentumTol;
    int iter = 0;
    real total = RL(0.0);
    for (; iter < s->maxMomentumIter; ++iter) {
        total = RL(0.0);
        for (int i = 1; i <= i1; ++i)
            for (int j = 1; j <= j1; ++j) {
                const size_t k = (size_t)i * stride + j;
                real Ax = RL(0.0);
                if (i > 1) Ax += (-s->cS[k]) * xc[k - stride];
                if (j > 1) Ax += (-s->cW[k]) * xc[k - 1];
                Ax += s->cP[k] * xc[k];
                if (j < j1) Ax += (-s->cE[k]) * xc[k + 1];
                if (i < i1) Ax += (-s->cN[k]) * xc[k + stride];
                real r = s->cB[k] - Ax;
                total += r * r;
                xn[k] = xc[k] + r / s->cP[k];
            }
        real* t = xc; xc = xn; xn = t;
        if (total < tol_sq * (real)n) { iter++; break; }
    }
    if (xc != s->x0) memcpy(s->x0, xc, sizeof(real) * (size_t)(i1 + 2) * stride);
    if (resid_sq_out) *resid_sq_out = total;
    return iter;
}

/* solveUMomentumImplicit / solveVMomentumImplicit: returns the Jacobi
 * iteration count and the max |u* - u| in *resid. */
int ORC(orc_momentum)(orc_state* s, int isU, real* resid) {
    ORC(orc_assemble)(s, isU);
    int it = ORC(orc_jacobi)(s, isU, NULL);
    const int M = s->M, N = s->N;
    const int i1 = isU ? M - 1 : M - 2, j1 = isU ? N - 2 : N - 1;
    const real maxVel = max_vel(s);
    real r = RL(0.0);
    for (int i = 1; i <= i1; ++i)
        for (int j = 1; j <= j1; ++j) {
            const size_t k = isU ? UI(s, i, j) : VI(s, i, j);
            real nv = rclamp(s->x0[k], -maxVel, maxVel);
            if (isU) { r = rmax(r, RABS(nv - s->u[k])); s->uStar[k] = nv; }
            else { r = rmax(r, RABS(nv - s->v[k])); s->vStar[k] = nv; }
        }
    *resid = r;
    if (isU) s->lastMomItersU = it; else s->lastMomItersV = it;
    return it;
}

/* ------------------------------------------------------------------------ */
/* Pressure correction (pressure_solver.cpp:462-816, PCG 121-184)             */
/* Unknowns: i in [1, M-1], j in [1, N-2]; p'(:, N-1) = 0 (Dirichlet).        */

static void pcg_matvec(const orc_state* s, const real* x, real* y) {
    const int M = s->M, N = s->N, st = N + 1;
    const real rho = s->rho, hx = s->hx, hy = s->hy;
    for (int i = 1; i < M; ++i)
        for (int j = 1; j < N - 1; ++j) {
            const size_t k = PI_(s, i, j);
            real aE = (j < N - 1) ? rho * s->dE[UI(s, i, j)] * hy : RL(0.0);
            real aW = (j > 1) ? rho * s->dE[UI(s, i, j - 1)] * hy : RL(0.0);
            real aN = (i < M - 1) ? rho * s->dN[VI(s, i, j)] * hx : RL(0.0);
            real aS = (i > 1) ? rho * s->dN[VI(s, i - 1, j)] * hx : RL(0.0);
            real aP = aE + aW + aN + aS;
            if (aP < RL(1e-20)) aP = RL(1.0);
            /* CSR order S, W, P, E, N; E exists only for j + 1 <= N - 2 */
            real sum = RL(0.0);
            if (i > 1) sum += (-aS) * x[k - st];
            if (j > 1) sum += (-aW) * x[k - 1];
            sum += aP * x[k];
            if (j + 1 < N - 1) sum += (-aE) * x[k + 1];
            if (i < M - 1) sum += (-aN) * x[k + st];
            y[k] = sum;
        }
}

static int pcg_solve(orc_state* s) {
    const int M = s->M, N = s->N;
    const real rho = s->rho, hx = s->hx, hy = s->hy;
    if ((M - 1) * (N - 2) == 0) return 0;
    for (int i = 1; i < M; ++i)
        for (int j = 1; j < N - 1; ++j) {
            real aE = (j < N - 1) ? rho * s->dE[UI(s, i, j)] * hy : RL(0.0);
            real aW = (j > 1) ? rho * s->dE[UI(s, i, j - 1)] * hy : RL(0.0);
            real aN = (i < M - 1) ? rho * s->dN[VI(s, i, j)] * hx : RL(0.0);
            real aS = (i > 1) ? rho * s->dN[VI(s, i - 1, j)] * hx : RL(0.0);
            real aP = aE + aW + aN + aS;
            if (aP < RL(1e-20)) aP = RL(1.0);
            s->pdiag[PI_(s, i, j)] = aP;
        }
#define FOR_DOF for (int i = 1; i < M; ++i) for (int j = 1; j < N - 1; ++j)
    pcg_matvec(s, s->px, s->pAp);
    FOR_DOF { size_t k = PI_(s, i, j); s->pr[k] = s->pb[k] - s->pAp[k]; }
#define APPLY_JAC FOR_DOF { size_t k = PI_(s, i, j); real d = s->pdiag[k]; \
        s->pz[k] = (RABS(d) > RL(1e-20)) ? s->pr[k] / d : s->pr[k]; }
    APPLY_JAC
    FOR_DOF { size_t k = PI_(s, i, j); s->pp[k] = s->pz[k]; }
    real rz = RL(0.0);
    FOR_DOF { size_t k = PI_(s, i, j); rz += s->pr[k] * s->pz[k]; }
    int iter = 0;
    for (; iter < s->maxPressureIter; ++iter) {
        pcg_matvec(s, s->pp, s->pAp);
        real pAp = RL(0.0);
        FOR_DOF { size_t k = PI_(s, i, j); pAp += s->pp[k] * s->pAp[k]; }
        if (RABS(pAp) < RL(1e-20)) break;
        real alpha = rz / pAp;
        FOR_DOF { size_t k = PI_(s, i, j); s->px[k] += alpha * s->pp[k]; s->pr[k] -= alpha * s->pAp[k]; }
        real err = RL(0.0);
        FOR_DOF { size_t k = PI_(s, i, j); err += s->pr[k] * s->pr[k]; }
        if (RSQRT(err) < s->pTol) break;
        APPLY_JAC
        real rz_prev = rz;
        rz = RL(0.0);
        FOR_DOF { size_t k = PI_(s, i, j); rz += s->pr[k] * s->pz[k]; }
        real beta = rz / rz_prev;
        FOR_DOF { size_t k = PI_(s, i, j); s->pp[k] = s->pz[k] + beta * s->pp[k]; }
    }
#undef APPLY_JAC
#undef FOR_DOF
    return iter;
}

/* mass imbalance of one cell, massW - massE + massS - massN (:478-482) */
static real mass_imbalance(const orc_state* s, int i, int j) {
    const real rho = s->rho, hx = s->hx, hy = s->hy;
    real massE = rho * s->uStar[UI(s, i, j)] * hy;
    real massW = rho * s->uStar[UI(s, i, j - 1)] * hy;
    real massN = rho * s->vStar[VI(s, i, j)] * hx;
    real massS = rho * s->vStar[VI(s, i - 1, j)] * hx;
    return massW - massE + massS - massN;
}

int ORC(orc_pressure)(orc_state* s, real* localResidMass) {
    const int M = s->M, N = s->N;
    memset(s->pStar, 0, sizeof(real) * (size_t)(M + 1) * (N + 1));
    real rmaxv = RL(0.0);
    double sumSq = 0.0;
    long long count = 0;
    for (int i = 1; i < M; ++i)
        for (int j = 1; j < N; ++j) {
            real b = RABS(mass_imbalance(s, i, j));
            if (b > rmaxv) rmaxv = b;
            sumSq += (double)b * (double)b;
            count++;
        }
    *localResidMass = rmaxv;
    s->residMass_max = rmaxv;
    s->residMass_RMS = count > 0 ? (real)sqrt(sumSq / (double)count) : RL(0.0);
    s->residMass = rmaxv;
    int iters = 0;
    if (s->pressureSolverType == 1 && (M - 1) * (N - 2) > 0) {
        for (int i = 1; i < M; ++i)
            for (int j = 1; j < N - 1; ++j) {
                size_t k = PI_(s, i, j);
                s->pb[k] = mass_imbalance(s, i, j);
                s->px[k] = s->pStar[k];
            }
        iters = pcg_solve(s);
        for (int i = 1; i < M; ++i)
            for (int j = 1; j < N - 1; ++j) s->pStar[PI_(s, i, j)] = s->px[PI_(s, i, j)];
        for (int i = 1; i < M; ++i) s->pStar[PI_(s, i, N - 1)] = RL(0.0);
    }
    s->lastPressureIters = iters;
    return iters;
}

/* ------------------------------------------------------------------------ */
/* One outer iteration: SIMPLE::calculateStep (iterations.cpp:82-659) with    */
/* momentumSolverType = 1, pseudo-time and residual viscosity off.            */

double ORC(orc_step)(orc_state* s, int* pressureIterations) {
    const int M = s->M, N = s->N;
    const real maxVel = max_vel(s);
    real localResidU = RL(0.0), localResidV = RL(0.0), localResidMass = RL(0.0);
    ORC(orc_velocity_bc)(s, s->u, s->v);
    ORC(orc_pressure_bc)(s, s->p);
    memcpy(s->uOld, s->u, sizeof(real) * (size_t)(M + 1) * N);
    memcpy(s->vOld, s->v, sizeof(real) * (size_t)M * (N + 1));
    ORC(orc_momentum)(s, 1, &localResidU);
    ORC(orc_momentum)(s, 0, &localResidV);
    s->residU = localResidU;
    s->residV = localResidV;
    ORC(orc_velocity_bc)(s, s->uStar, s->vStar);
    s->residU_max = s->residU;
    s->residV_max = s->residV;
    {
        double sumU = 0.0, sumV = 0.0;
        long long cU = 0, cV = 0;
        for (int i = 1; i < M; ++i)
            for (int j = 1; j < N - 1; ++j) {
                real d = s->uStar[UI(s, i, j)] - s->uOld[UI(s, i, j)];
                sumU += (double)d * (double)d;
                cU++;
            }
        for (int i = 1; i < M - 1; ++i)
            for (int j = 1; j < N; ++j) {
                real d = s->vStar[VI(s, i, j)] - s->vOld[VI(s, i, j)];
                sumV += (double)d * (double)d;
                cV++;
            }
        s->residU_RMS = cU > 0 ? (real)sqrt(sumU / (double)cU) : RL(0.0);
        s->residV_RMS = cV > 0 ? (real)sqrt(sumV / (double)cV) : RL(0.0);
    }
    int pit = ORC(orc_pressure)(s, &localResidMass);
    if (pressureIterations) *pressureIterations = pit;
    s->residMass = localResidMass;
    for (int i = 1; i < M; ++i)
        for (int j = 1; j < N; ++j) s->p[PI_(s, i, j)] += s->pAlpha * s->pStar[PI_(s, i, j)];
    ORC(orc_pressure_bc)(s, s->p);
    for (int i = 1; i < M; ++i)
        for (int j = 1; j < N - 1; ++j) {
            real du = s->dE[UI(s, i, j)] * (s->pStar[PI_(s, i, j)] - s->pStar[PI_(s, i, j + 1)]);
            du = rmax(-maxVel, rmin(maxVel, du));
            real nu = s->uStar[UI(s, i, j)] + du;
            s->u[UI(s, i, j)] = rmax(-maxVel, rmin(maxVel, nu));
        }
    for (int i = 1; i < M - 1; ++i)
        for (int j = 1; j < N; ++j) {
            real dv = s->dN[VI(s, i, j)] * (s->pStar[PI_(s, i, j)] - s->pStar[PI_(s, i + 1, j)]);
            dv = rmax(-maxVel, rmin(maxVel, dv));
            real nv = s->vStar[VI(s, i, j)] + dv;
            s->v[VI(s, i, j)] = rmax(-maxVel, rmin(maxVel, nv));
        }
    ORC(orc_velocity_bc)(s, s->u, s->v);
    /* residual normalisation bookkeeping (iterations.cpp:628-656) */
    const real velFloor = rmax(s->velFloor, RL(1e-30));
    const real massFloor = rmax(s->massFloor, RL(1e-30));
    if (!s->rmsU0set && s->residU_RMS > velFloor) { s->residU_RMS0 = s->residU_RMS; s->rmsU0set = 1; }
    if (!s->rmsV0set && s->residV_RMS > velFloor) { s->residV_RMS0 = s->residV_RMS; s->rmsV0set = 1; }
    if (!s->rmsM0set && s->residMass_RMS > massFloor) { s->residMass_RMS0 = s->residMass_RMS; s->rmsM0set = 1; }
    if (!s->rmsU0set) s->residU_RMS0 = velFloor;
    if (!s->rmsV0set) s->residV_RMS0 = velFloor;
    if (!s->rmsM0set) s->residMass_RMS0 = massFloor;
    if (s->normalized) {
        s->residU = s->residU_RMS / s->residU_RMS0;
        s->residV = s->residV_RMS / s->residV_RMS0;
        s->residMass = s->residMass_RMS / s->residMass_RMS0;
    } else {
        s->residU = s->residU_RMS;
        s->residV = s->residV_RMS;
        s->residMass = s->residMass_RMS;
    }
    return (double)rmax(rmax(s->residU, s->residV), s->residMass);
}

/* ------------------------------------------------------------------------ */
/* Pressure-drop sampling (postprocessing.cpp:53-327)                         */
/* metrics[5] = flowArea, massFlux, avgStatic, avgDynamic, avgTotal           */

static void finish_metrics(real area, real fluxSum, real st, real dy, real tw, double* m) {
    real avgS = RL(0.0), avgD = RL(0.0), avgT = RL(0.0);
    if (area > RL(0.0)) { avgS = st / area; avgD = dy / area; }
    if (fluxSum > RL(0.0)) avgT = tw / fluxSum;
    else if (area > RL(0.0)) avgT = avgS + avgD;
    m[0] = area; m[1] = fluxSum; m[2] = avgS; m[3] = avgD; m[4] = avgT;
}

void ORC(orc_sample_plane)(const orc_state* s, double xPhysical, double* out) {
    const int M = s->M, N = s->N, MC = M - 1, NC = N - 1;
    const real hx = s->hx, hy = s->hy, rho = s->rho;
    const real xp = (real)xPhysical;
    for (int k = 0; k < 5; ++k) out[k] = 0.0;
    if (MC <= 0 || NC <= 0 || hx <= RL(0.0) || hy <= RL(0.0)) return;
    int cl, cr;
    real t;
    if (NC <= 1) { cl = 0; cr = 0; t = RL(0.0); }
    else {
        real xMin = RL(0.5) * hx, xMax = ((real)NC - RL(0.5)) * hx;
        real xc = rmax(xMin, rmin(xp, xMax));
        real jf = xc / hx - RL(0.5);
        cl = (int)RFLOOR(jf);
        if (cl > NC - 2) cl = NC - 2;
        if (cl < 0) cl = 0;
        cr = cl + 1;
        real xl = ((real)cl + RL(0.5)) * hx, xr = ((real)cr + RL(0.5)) * hx;
        if (RABS(xr - xl) < RL(1e-12)) t = RL(0.0);
        else t = (xc - xl) / (xr - xl);
        t = rmax(RL(0.0), rmin(RL(1.0), t));
    }
    real st = 0, dy = 0, tw = 0, area = 0, fs = 0;
    for (int i = 1; i < M; ++i) {
        const int cellRow = i - 1;
        if (cellRow < 0 || cellRow >= MC) continue;
        if (cl < 0 || cl >= NC || cr < 0 || cr >= NC) continue;
        const real tolf = RL(1e-6);
        if (s->gamma[CI(s, cellRow, cl)] < RL(1.0) - tolf || s->gamma[CI(s, cellRow, cr)] < RL(1.0) - tolf) continue;
        const real fa = hy;
        area += fa;
        int pl = cl + 1, prr = cr + 1;
        if (pl > N) pl = N;
        if (prr > N) prr = N;
        real staticP = (RL(1.0) - t) * s->p[PI_(s, i, pl)] + t * s->p[PI_(s, i, prr)];
        int ul = cl < N - 1 ? cl : N - 1, ur = cr < N - 1 ? cr : N - 1;
        real un = (RL(1.0) - t) * s->u[UI(s, i, ul)] + t * s->u[UI(s, i, ur)];
        int vl = cl < N ? cl : N, vr = cr < N ? cr : N;
        int vt = i - 1 < M - 1 ? i - 1 : M - 1, vb = i < M - 1 ? i : M - 1;
        if (vt < 0) vt = 0;
        real vTop = (RL(1.0) - t) * s->v[VI(s, vt, vl)] + t * s->v[VI(s, vt, vr)];
        real vBot = (RL(1.0) - t) * s->v[VI(s, vb, vl)] + t * s->v[VI(s, vb, vr)];
        real vtan = RL(0.5) * (vTop + vBot);
        real vm = RSQRT(un * un + vtan * vtan);
        real dynP = RL(0.5) * rho * vm * vm;
        real tot = staticP + dynP;
        st += staticP * fa;
        dy += dynP * fa;
        real flux = rho * un * fa;
        real fabs_ = RABS(flux);
        if (fabs_ > RL(0.0)) { fs += fabs_; tw += tot * fabs_; }
    }
    finish_metrics(area, fs, st, dy, tw, out);
}

void ORC(orc_sample_patch)(const orc_state* s, int inlet, double* out) {
    const int M = s->M, N = s->N, MC = M - 1, NC = N - 1;
    const real hy = s->hy, rho = s->rho;
    for (int k = 0; k < 5; ++k) out[k] = 0.0;
    if (MC <= 0 || NC <= 0 || hy <= RL(0.0)) return;
    const int uCol = inlet ? 0 : N - 1, pCol = inlet ? 0 : N, vCol = inlet ? 0 : N;
    const int adj = inlet ? 0 : NC - 1;
    real st = 0, dy = 0, tw = 0, area = 0, fs = 0;
    for (int i = 1; i < M; ++i) {
        const int cellRow = i - 1;
        if (cellRow < 0 || cellRow >= MC) continue;
        if (adj < 0 || adj >= NC) continue;
        if (s->gamma[CI(s, cellRow, adj)] < RL(1.0) - RL(1e-6)) continue;
        const real fa = hy;
        area += fa;
        int vt = i - 1 < M - 1 ? i - 1 : M - 1, vb = i < M - 1 ? i : M - 1;
        if (vt < 0) vt = 0;
        real staticP = s->p[PI_(s, i, pCol)];
        real un = s->u[UI(s, i, uCol)];
        real vtan = RL(0.5) * (s->v[VI(s, vt, vCol)] + s->v[VI(s, vb, vCol)]);
        real vm = RSQRT(un * un + vtan * vtan);
        real dynP = RL(0.5) * rho * vm * vm;
        real tot = staticP + dynP;
        st += staticP * fa;
        dy += dynP * fa;
        real fabs_ = RABS(rho * un * fa);
        if (fabs_ > RL(0.0)) { fs += fabs_; tw += tot * fabs_; }
    }
    finish_metrics(area, fs, st, dy, tw, out);
}

/* ------------------------------------------------------------------------ */
/* Outer loop (SIMPLE.cpp:378-521 without logging); history rows as the      */
/* reference harness writes them:                                             */
/*  iter error residU_RMS residV_RMS residMass_RMS residU_max residV_max      */
/*  residMass_max pIters coreTotal fullTotal coreStatic fullStatic            */
/*  inMassFlux outMassFlux                                                    */
#define ORC_HIST_COLS 15

int ORC(orc_run)(orc_state* s, int maxIter, double* hist, int histCap) {
    double error = s->lastError;
    int n = 0;
    while (n < maxIter && s->iter < s->maxIterations && error > (double)s->epsilon) {
        if (s->enableInletRamp && s->rampSteps > 0 && s->iter < s->rampSteps)
            s->inletVelocity = ((real)(s->iter + 1) / (real)s->rampSteps) * s->targetVel;
        else
            s->inletVelocity = s->targetVel;
        int pit = 0;
        real e = (real)ORC(orc_step)(s, &pit);
        error = (double)e;
        s->lastError = error;
        double ci[5], co[5], fi[5], fo[5];
        ORC(orc_sample_plane)(s, (double)s->xCoreIn, ci);
        ORC(orc_sample_plane)(s, (double)s->xCoreOut, co);
        ORC(orc_sample_patch)(s, 1, fi);
        ORC(orc_sample_patch)(s, 0, fo);
        if (hist && n < histCap) {
            double* h = hist + (size_t)n * ORC_HIST_COLS;
            h[0] = s->iter; h[1] = error; h[2] = s->residU_RMS; h[3] = s->residV_RMS;
            h[4] = s->residMass_RMS; h[5] = s->residU_max; h[6] = s->residV_max; h[7] = s->residMass_max;
            h[8] = pit;
            h[9] = (double)((real)ci[4] - (real)co[4]);
            h[10] = (double)((real)fi[4] - (real)fo[4]);
            h[11] = (double)((real)ci[2] - (real)co[2]);
            h[12] = (double)((real)fi[2] - (real)fo[2]);
            h[13] = fi[1]; h[14] = fo[1];
        }
        n++;
        s->iter++;
    }
    return n;
}

/* ------------------------------------------------------------------------ */
/* Field access by name (row-major, full staggered shape), as double.         */

static real* field_ptr(orc_state* s, const char* name, int* rows, int* cols) {
    const int M = s->M, N = s->N;
    struct { const char* n; real* p; int r, c; } t[] = {
        {"u", s->u, M + 1, N}, {"v", s->v, M, N + 1}, {"p", s->p, M + 1, N + 1},
        {"uStar", s->uStar, M + 1, N}, {"vStar", s->vStar, M, N + 1}, {"pStar", s->pStar, M + 1, N + 1},
        {"uOld", s->uOld, M + 1, N}, {"vOld", s->vOld, M, N + 1},
        {"dE", s->dE, M + 1, N}, {"dN", s->dN, M, N + 1},
        {"gamma", s->gamma, M, N}, {"alpha", s->alpha, M, N}, {"cellType", s->cellType, M, N},
        {"cP", s->cP, M + 1, N + 1}, {"cE", s->cE, M + 1, N + 1}, {"cW", s->cW, M + 1, N + 1},
        {"cN", s->cN, M + 1, N + 1}, {"cS", s->cS, M + 1, N + 1}, {"cB", s->cB, M + 1, N + 1},
        {"x0", s->x0, M + 1, N + 1},
    };
    for (size_t k = 0; k < sizeof t / sizeof t[0]; ++k)
        if (strcmp(t[k].n, name) == 0) { *rows = t[k].r; *cols = t[k].c; return t[k].p; }
    return NULL;
}

/* Copies `name` into out (rows*cols doubles).  The momentum coefficient
 * arrays use the component's own row stride (N for U, N+1 for V) inside a
 * (M+1) x (N+1) buffer; they are returned raw. Returns element count or -1. */
int ORC(orc_get)(orc_state* s, const char* name, double* out) {
    int r, c;
    real* p = field_ptr(s, name, &r, &c);
    if (!p) return -1;
    for (size_t k = 0; k < (size_t)r * c; ++k) out[k] = (double)p[k];
    return r * c;
}

int ORC(orc_set)(orc_state* s, const char* name, const double* in) {
    int r, c;
    real* p = field_ptr(s, name, &r, &c);
    if (!p) return -1;
    for (size_t k = 0; k < (size_t)r * c; ++k) p[k] = (real)in[k];
    return r * c;
}

void ORC(orc_set_inlet_velocity)(orc_state* s, double v) { s->inletVelocity = (real)v; }

int ORC(orc_dims)(const orc_state* s, int* M, int* N) { *M = s->M; *N = s->N; return 0; }

/* scalars: residU residV residMass residU_max residV_max residMass_max
 *          residU_RMS residV_RMS residMass_RMS itersU itersV itersP */
void ORC(orc_scalars)(const orc_state* s, double* out) {
    out[0] = s->residU; out[1] = s->residV; out[2] = s->residMass;
    out[3] = s->residU_max; out[4] = s->residV_max; out[5] = s->residMass_max;
    out[6] = s->residU_RMS; out[7] = s->residV_RMS; out[8] = s->residMass_RMS;
    out[9] = s->lastMomItersU; out[10] = s->lastMomItersV; out[11] = s->lastPressureIters;
}
