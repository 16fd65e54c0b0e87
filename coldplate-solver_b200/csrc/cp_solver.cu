// Host driver of the B200-native SIMPLE solver and the C ABI declared in
// include/cp_simple.h.
//
// A cp_ctx owns every device buffer of one field for its lifetime (the
// reference's GPU backends instead copy the whole CSR system host->device on
// every call, momentum_solver.cu:156-171, pressure_solver.cu:136-146).  One
// outer iteration is a fixed sequence of launches on the context's stream;
// it is captured once into a CUDA graph and replayed in chunks, and the host
// only reads the device status word between chunks.  The stop rules run on
// the device (k_finalize), so replaying past convergence does no work.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cp_kernels.cuh"
#include "cp_mg.cuh"
#include "cp_sa.cuh"
#include "cp_adjoint.cuh"
#include "cp_batch.cuh"

using namespace cp;

namespace {

thread_local std::string g_err;

cp_status fail(cp_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

}  // namespace

// The error string of the other translation units (cp_thermal.cu).
__attribute__((visibility("hidden"))) cp_status cp_internal_set_error(cp_status s, const char* msg) {
    g_err = msg;
    return s;
}

namespace {

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(CP_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),       \
                        __FILE__, __LINE__);                                                       \
    } while (0)

constexpr int kThreads = 256;

}  // namespace

struct cp_ctx {
    cp_params prm{};
    KParams k{};
    Dims d{};
    int dev = 0, numSMs = 0;
    cudaStream_t stream = nullptr;
    size_t nElem = 0;
    int es = 8;  // bytes of the inner-system type
    // fields (double)
    double *u = nullptr, *v = nullptr, *p = nullptr, *uStar = nullptr, *vStar = nullptr, *pStar = nullptr;
    double *dE = nullptr, *dN = nullptr, *gamma = nullptr, *alpha = nullptr;
    std::vector<double> cellTypeHost;  // M x N padded, as the reference keeps it
    double* gammaStage = nullptr;      // pinned M x N staging of gamma (first set_cell_type / set_gamma)
    // inner systems (double or float)
    void* mom[12] = {};
    void* xb[4] = {};
    void* pcg[9] = {};
    double *partJ = nullptr, *partM = nullptr, *partP = nullptr;
    unsigned *barJ = nullptr, *barP = nullptr;
    Status* st = nullptr;
    Status* stHost = nullptr;
    double* hist = nullptr;
    int histCap = 0;
    double* dpWin = nullptr;
    int gJac = 0, gPcg = 0, gElem = 0, nbMass = 0;
    // multigrid hierarchy (pressureSolverType 2 / 4)
    bool useMg = false;
    int mgL = 0, mgLg = 0, gMg = 0;
    int mgNI[kMgMaxLevels] = {}, mgNJ[kMgMaxLevels] = {}, mgP[kMgMaxLevels] = {};
    void* mgArr[kMgMaxLevels][7] = {};   // fE fN d dx x y b
    void* mgDense = nullptr;
    // Jacobi damping of the V-cycle smoother: with the 1.8 coarse scale,
    // 0.9 reaches pTol 1e-6 in 29 CG iterations at 2048 x 1024 against 32 at
    // 0.8 and 38 at 0.7 (measured)
    double mgOmega = 0.9;
    // Scaling of the coarse-grid correction.  Piecewise-constant aggregation
    // under-corrects smooth error; an over-correction s in (0, 2) keeps the
    // V-cycle symmetric positive definite.  On the 2048 x 1024 density
    // workload, s = 1.8 lowers the mean CG iterations per outer iteration
    // (fewer solves reach the 30-iteration cap) and the time to converge by
    // about a quarter, with the same converged pressure drop.
    double mgScale = 1.8;
    unsigned long long* mgProf = nullptr;   // per-phase timers when CP_MG_PROFILE is set
    // smoothed-aggregation hierarchy (pressureSolverType 4); the 2 x 2 one
    // above stays for type 2 and for batches
    bool useSa = false;
    int saL = 0, saLg = 0;
    int saNI[kSaMaxLevels] = {}, saNJ[kSaMaxLevels] = {}, saP[kSaMaxLevels] = {};
    // per level: c[0..8] x y b t pw[0..3] (level 0: x y b t and pw[0..2];
    // pw only on levels that run grid-wide and have a coarser one)
    void* saArr[kSaMaxLevels][17] = {};
    void* saDinv0 = nullptr;                 // level-0 inverse diagonal
    size_t saSmem = 0;                       // k_pcg_sa's dynamic shared memory (bytes)
    void* saY[9] = {};
    void* saDense = nullptr;
    double saOmega = 0.9, saW0 = 2.0 / 3.0, saWc = 0.8;
    unsigned long long* saProf = nullptr;    // per-phase timers when CP_SA_PROFILE is set
    int saReuse = 4;                         // outer iterations between coarse-operator rebuilds
    int* saDirty = nullptr;                  // device flag: rebuild the coarse operators on the next solve
    int* saDirtyAdj = nullptr;               // the same flag for the adjoint's pressure-like solves
    MgMaps mgMaps;                           // TMA tensor maps of the level-0 tile phases
    // adjoint buffers (allocated on first use, double)
    double* adj[40] = {};
    // forward Jacobi iterates x_1..x_s of the adjoint's frozen sweeps (U, V),
    // allocated as the sweep counts need them
    std::vector<double*> adjXU, adjXV;
    void* adjMom[12] = {};
    Status* adjSt = nullptr;
    double* adjPart = nullptr;
    unsigned* adjBar = nullptr;
    // flexible GMRES of the adjoint: basis V_0..V_m, preconditioned
    // directions Z_0..Z_m-1, the work vector W and lambda, each 3 * nElem
    double* adjKry = nullptr;
    double* adjKryPart = nullptr;
    double* adjH = nullptr;
    int adjRestart = 30;     // m
    int adjSweeps = 6;       // equations model: transposed momentum Jacobi sweeps per preconditioner application
    int adjPIters = 6;       // multigrid-PCG iterations per preconditioner application
    cudaGraphExec_t graph = nullptr;
    bool graphTried = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<void*> allocs;
};

namespace {

template <typename T>
cp_status dalloc(cp_ctx* c, T** ptr, size_t count) {
    void* q = nullptr;
    CK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
    CK(cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), c->stream));
    c->allocs.push_back(q);
    *ptr = static_cast<T*>(q);
    return CP_OK;
}

cp_status dalloc_bytes(cp_ctx* c, void** ptr, size_t bytes) {
    CK(cudaMalloc(ptr, std::max<size_t>(bytes, 1)));
    CK(cudaMemsetAsync(*ptr, 0, std::max<size_t>(bytes, 1), c->stream));
    c->allocs.push_back(*ptr);
    return CP_OK;
}

bool finite(double x) { return std::isfinite(x); }

cp_status validate(const cp_params* p) {
    if (!p) return fail(CP_ERR_BAD_PARAM, "params is NULL");
    if (p->Ny < 2 || p->Nx < 3) return fail(CP_ERR_BAD_PARAM, "grid %d x %d too small (need Ny >= 2, Nx >= 3)", p->Ny, p->Nx);
    if ((long long)(p->Ny + 3) * (long long)(p->Nx + 33) > (1ll << 31))
        return fail(CP_ERR_BAD_PARAM, "grid %d x %d exceeds the 2^31-element index range", p->Ny, p->Nx);
    const double pos[] = {p->hy, p->hx, p->rho, p->eta, p->uvAlpha, p->pAlpha};
    const char* posn[] = {"hy", "hx", "rho", "eta", "uvAlpha", "pAlpha"};
    for (int q = 0; q < 6; ++q)
        if (!finite(pos[q]) || pos[q] <= 0.0) return fail(CP_ERR_BAD_PARAM, "%s must be finite and > 0", posn[q]);
    const double fin[] = {p->targetVel, p->epsilon, p->pTol, p->momentumTol, p->brinkmanKMin, p->brinkmanQ,
                          p->Ht_channel, p->twoPointFiveDConvectionFactor, p->twoPointFiveDSinkMultiplier,
                          p->xPlaneCoreInlet, p->xPlaneCoreOutlet};
    for (double x : fin)
        if (!finite(x)) return fail(CP_ERR_NONFINITE, "non-finite parameter");
    if (p->maxIterations < 0 || p->maxPressureIter < 0 || p->maxMomentumIter < 0)
        return fail(CP_ERR_BAD_PARAM, "iteration limits must be >= 0");
    if (p->pressureSolverType != 1 && p->pressureSolverType != 2 && p->pressureSolverType != 4)
        return fail(CP_ERR_UNSUPPORTED,
                    "pressureSolverType %d not available: 1 (Jacobi-PCG) and 2 / 4 (multigrid-PCG) run natively",
                    p->pressureSolverType);
    if (p->momentumSolverType != 1)
        return fail(CP_ERR_UNSUPPORTED, "momentumSolverType %d not available: only 1 (implicit Jacobi)",
                    p->momentumSolverType);
    if (p->enablePseudoTimeStepping || p->enableSER || p->enableLineSearch || p->enableCflRamp)
        return fail(CP_ERR_UNSUPPORTED, "pseudo-transient continuation is not available");
    if (p->enableResidualViscosity) return fail(CP_ERR_UNSUPPORTED, "residual artificial viscosity is not available");
    if (p->usePressureDropSlopeGate) return fail(CP_ERR_UNSUPPORTED, "pressure-drop slope gate is not available");
    if (p->convectionScheme != 0 && p->convectionScheme != 1)
        return fail(CP_ERR_BAD_PARAM, "convectionScheme must be 0 (FOU) or 1 (SOU)");
    if (p->precision != CP_PREC_FP64 && p->precision != CP_PREC_MIXED)
        return fail(CP_ERR_BAD_PARAM, "precision must be CP_PREC_FP64 or CP_PREC_MIXED");
    if (p->usePressureDropConvergence && p->dpConvergenceWindow <= 0)
        return fail(CP_ERR_BAD_PARAM, "dpConvergenceWindow must be > 0");
    return CP_OK;
}

void fill_kparams(cp_ctx* c) {
    const cp_params& p = c->prm;
    KParams& k = c->k;
    k.d = c->d;
    k.hx = p.hx; k.hy = p.hy; k.rho = p.rho; k.eta = p.eta;
    k.uvAlpha = p.uvAlpha; k.pAlpha = p.pAlpha;
    k.targetVel = p.targetVel;
    k.rampOn = p.enableInletRamp; k.rampSteps = p.rampSteps;
    // 2.5-D needs Ht > 0 (SIMPLE.cpp:67-73); sink 12 mu / Ht^2 (momentum_solver.cpp:187-189)
    const bool twoD5 = p.enableTwoPointFiveD && p.Ht_channel > 0.0;
    k.convScale = twoD5 ? p.twoPointFiveDConvectionFactor : 1.0;
    const double sink = twoD5 ? p.twoPointFiveDSinkMultiplier * (12.0 * p.eta / (p.Ht_channel * p.Ht_channel)) : 0.0;
    k.sinkDiag = sink * (p.hx * p.hy);
    k.sou = p.convectionScheme == 1;
    k.pTol = p.pTol; k.momTol = p.momentumTol;
    k.maxP = p.maxPressureIter; k.maxMom = p.maxMomentumIter;
    k.xCoreIn = p.xPlaneCoreInlet; k.xCoreOut = p.xPlaneCoreOutlet;
    k.eps = p.epsilon; k.maxIterations = p.maxIterations;
    k.normalized = p.enableNormalizedResiduals;
    k.velFloor = p.residNormFloorVel; k.massFloor = p.residNormFloorMass;
    k.dpConv = p.usePressureDropConvergence; k.dpWindow = p.dpConvergenceWindow; k.dpRampSteps = p.rampSteps;
    k.dpPercent = p.dpConvergencePercent;
    const int M = c->d.M, N = c->d.N;
    k.nU = (M - 1) * (N - 2);
    k.nV = (M - 2) * (N - 1);
    k.nP = (M - 1) * (N - 2);
}

// density -> gamma (1 - clamp(cellType)) with the padded row/column copied,
// alpha by RAMP (SIMPLE.cpp:667-676, 707-729, 766-772); all M x N, double.
void build_density(const cp_ctx* c, const std::vector<double>& cellTypePadded, double* gamma) {
    const int M = c->d.M, N = c->d.N, pr = M - 1, pc = N - 1;
    for (int i = 0; i < pr; ++i)
        for (int j = 0; j < pc; ++j) {
            const double val = cellTypePadded[(size_t)i * N + j];
            const double vc = std::max(0.0, std::min(1.0, val));
            gamma[(size_t)i * N + j] = 1.0 - vc;
        }
    for (int i = 0; i < pr; ++i) gamma[(size_t)i * N + pc] = gamma[(size_t)i * N + pc - 1];
    for (int j = 0; j < N; ++j) gamma[(size_t)pr * N + j] = gamma[(size_t)(pr - 1) * N + std::min(j, pc - 1)];
}

// RAMP interpolation alpha = alpha_max (1 - gamma) / (1 + q gamma + 1e-10)
// (SIMPLE.cpp:770) over the M x N cells, rounded step by step as the host
// formula (no fused multiply-add)
__global__ void k_alpha(const double* gamma, double* alpha, int M, int N, int P, double amax, double q) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < M * N; t += gridDim.x * blockDim.x) {
        const int i = t / N, j = t - i * N;
        const double g = gamma[(size_t)i * P + j];
        alpha[(size_t)i * P + j] = __ddiv_rn(__dmul_rn(amax, 1.0 - g), __dadd_rn(__dadd_rn(1.0, __dmul_rn(q, g)), 1e-10));
    }
}

// the smoothed-aggregation coarse operators are rebuilt by the next solve
// (after a change of geometry or state from the host, or a dispatch call)
cp_status mark_sa_stale(cp_ctx* c) {
    if (!c->saDirty) return CP_OK;
    static const int one = 1;
    CK(cudaMemcpyAsync(c->saDirty, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    return CP_OK;
}

// gamma (M x N, host) to the device, alpha from it; returns after the copy
cp_status upload_cells(cp_ctx* c, const double* g) {
    const int M = c->d.M, N = c->d.N;
    CK(cudaMemcpy2DAsync(c->gamma, (size_t)c->d.P * 8, g, (size_t)N * 8, (size_t)N * 8, M,
                         cudaMemcpyHostToDevice, c->stream));
    const double amax = c->prm.eta / std::max(c->prm.brinkmanKMin, 1e-20);
    k_alpha<<<c->gElem, kThreads, 0, c->stream>>>(c->gamma, c->alpha, M, N, c->d.P, amax, c->prm.brinkmanQ);
    CK(cudaGetLastError());
    cp_status s = mark_sa_stale(c);
    if (s != CP_OK) return s;
    CK(cudaStreamSynchronize(c->stream));
    return CP_OK;
}

bool field_shape(const cp_ctx* c, cp_field f, double** dptr, int* rows, int* cols) {
    const int M = c->d.M, N = c->d.N;
    switch (f) {
        case CP_FIELD_U: *dptr = c->u; *rows = M + 1; *cols = N; return true;
        case CP_FIELD_V: *dptr = c->v; *rows = M; *cols = N + 1; return true;
        case CP_FIELD_P: *dptr = c->p; *rows = M + 1; *cols = N + 1; return true;
        case CP_FIELD_USTAR: *dptr = c->uStar; *rows = M + 1; *cols = N; return true;
        case CP_FIELD_VSTAR: *dptr = c->vStar; *rows = M; *cols = N + 1; return true;
        case CP_FIELD_PSTAR: *dptr = c->pStar; *rows = M + 1; *cols = N + 1; return true;
        case CP_FIELD_DE: *dptr = c->dE; *rows = M + 1; *cols = N; return true;
        case CP_FIELD_DN: *dptr = c->dN; *rows = M; *cols = N + 1; return true;
        case CP_FIELD_GAMMA: *dptr = c->gamma; *rows = M; *cols = N; return true;
        case CP_FIELD_ALPHA: *dptr = c->alpha; *rows = M; *cols = N; return true;
        case CP_FIELD_CELLTYPE: *dptr = nullptr; *rows = M; *cols = N; return true;
    }
    return false;
}

// ---------------------------------------------------------------- launches
// Optional CUDA-event bracket around each launch (cp_kernel_times).
struct EvRec {
    static constexpr int kMax = 24;
    cudaEvent_t ev[2 * kMax] = {};
    int kind[kMax] = {};
    int n = 0;
    void begin(cudaStream_t s, int k) {
        if (n < kMax) { kind[n] = k; cudaEventRecord(ev[2 * n], s); }
    }
    void end(cudaStream_t s) {
        if (n < kMax) { cudaEventRecord(ev[2 * n + 1], s); ++n; }
    }
};
#define REC_BEGIN(r, k) do { if (r) (r)->begin(c->stream, (k)); } while (0)
#define REC_END(r) do { if (r) (r)->end(c->stream); } while (0)

template <typename Kern, typename... Args>
cudaError_t launch_coop(Kern kern, int grid, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <typename TC>
MomSys<TC> mom_sys(cp_ctx* c, int comp) {
    MomSys<TC> s;
    TC** a = reinterpret_cast<TC**>(c->mom + comp * 6);
    s.aP = a[0]; s.aE = a[1]; s.aW = a[2]; s.aN = a[3]; s.aS = a[4]; s.b = a[5];
    return s;
}

template <typename TV>
PcgBufs<TV> pcg_bufs(cp_ctx* c) {
    PcgBufs<TV> b;
    TV** a = reinterpret_cast<TV**>(c->pcg);
    b.fE = a[0]; b.fN = a[1]; b.d = a[2]; b.x = a[3]; b.r = a[4]; b.pa = a[5]; b.pb = a[6]; b.Ap = a[7];
    b.rhs = a[8];
    return b;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

cp_status encode_map(CUtensorMap* m, void* base, int elemBytes, int pitch, int rows, int boxW, int boxR) {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !f)
            return fail(CP_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<EncodeTiledFn>(f);
    }
    // tile origins are multiples of 32 elements and the boxes' inner extents
    // multiples of 16 bytes; the pitch must keep every row 16-byte aligned
    if (((size_t)pitch * elemBytes) % 16 != 0 || ((size_t)boxW * elemBytes) % 16 != 0 ||
        (reinterpret_cast<uintptr_t>(base) & 15) != 0)
        return fail(CP_ERR_CUDA, "tensor map alignment");
    const cuuint64_t dims[2] = {(cuuint64_t)pitch, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch * elemBytes};
    const cuuint32_t box[2] = {(cuuint32_t)boxW, (cuuint32_t)boxR};
    const cuuint32_t es[2] = {1, 1};
    CUresult r = fn(m, elemBytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base,
                    dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(CP_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return CP_OK;
}

template <typename TV>
MgHier<TV> mg_hier(cp_ctx* c) {
    MgHier<TV> H;
    memset(&H, 0, sizeof(H));
    H.L = c->mgL;
    H.Lg = c->mgLg;
    H.omega = c->mgOmega;
    H.scale = c->mgScale;
    H.dense = (TV*)c->mgDense;
    H.prof = c->mgProf;
    for (int l = 0; l < c->mgL; ++l) {
        MgLevel<TV>& v = H.lv[l];
        v.nI = c->mgNI[l]; v.nJ = c->mgNJ[l]; v.P = c->mgP[l];
        TV** a = reinterpret_cast<TV**>(c->mgArr[l]);
        v.fE = a[0]; v.fN = a[1]; v.d = a[2]; v.dx = a[3]; v.x = a[4]; v.y = a[5]; v.b = a[6];
    }
    return H;
}

constexpr int kMgThreads = 512;
// dynamic shared memory: the dense set-up workspace and, afterwards, the two
// TMA tile stages (sized for double; the float kernel uses less of it)
constexpr size_t kMgDenseSmem = sizeof(double) * (size_t)(kMgDense * 2 * kMgDense + kMgDense);
constexpr size_t kMgTileSmem = (size_t)TileSmem<double>::kBytes > (size_t)TileSmem<float>::kBytes
                                   ? (size_t)TileSmem<double>::kBytes
                                   : (size_t)TileSmem<float>::kBytes;
constexpr size_t kMgDynSmem = kMgDenseSmem > kMgTileSmem ? kMgDenseSmem : kMgTileSmem;
static_assert(kMgDynSmem + 4096 <= 227 * 1024, "k_pcg_mg's dynamic shared memory exceeds a block's limit");

// Level sizes: halve (rounding up) until at most kMgDense unknowns; levels
// above kMgCtaCells unknowns (and always level 0) run grid-wide.
cp_status mg_build(cp_ctx* c) {
    int nI = c->d.M - 1, nJ = c->d.N - 2;
    int L = 0;
    for (;;) {
        if (L >= kMgMaxLevels) return fail(CP_ERR_BAD_PARAM, "multigrid hierarchy too deep");
        c->mgNI[L] = nI; c->mgNJ[L] = nJ;
        ++L;
        if ((long long)nI * nJ <= kMgDense && L >= 2) break;
        nI = (nI + 1) / 2; nJ = (nJ + 1) / 2;
    }
    c->mgL = L;
    int Lg = 1;
    long long ctaCells = kMgCtaCells;
    if (const char* e = getenv("CP_MG_CTA_CELLS")) ctaCells = std::max(atoll(e), 1LL);
    while (Lg < L && (long long)c->mgNI[Lg] * c->mgNJ[Lg] > ctaCells) ++Lg;
    c->mgLg = Lg;
    // level 0 shares the field layout and the PCG face / diagonal arrays
    c->mgP[0] = c->d.P;
    c->mgArr[0][0] = c->pcg[0];
    c->mgArr[0][1] = c->pcg[1];
    c->mgArr[0][2] = c->pcg[2];
    // level 0: dx, y and x of its own (x holds the pre-smoothed iterate
    // omega r / d); its rhs is the CG residual r
    for (int q = 3; q < 6; ++q) {
        cp_status s = dalloc_bytes(c, &c->mgArr[0][q], c->nElem * c->es);
        if (s != CP_OK) return s;
    }
    c->mgArr[0][6] = c->pcg[4];
    for (int l = 1; l < L; ++l) {
        c->mgP[l] = ((c->mgNJ[l] + 2 + 31) / 32) * 32;
        const size_t ne = (size_t)(c->mgNI[l] + 2) * c->mgP[l];
        for (int q = 0; q < 7; ++q) {
            cp_status s = dalloc_bytes(c, &c->mgArr[l][q], ne * c->es);
            if (s != CP_OK) return s;
        }
    }
    cp_status s = dalloc_bytes(c, &c->mgDense, (size_t)kMgDense * kMgDense * c->es);
    if (s != CP_OK) return s;
    // tensor maps of the level-0 tile phases: z (level-0 y), p_a, p_b, r, d,
    // fE, fN on the field layout; the level-1 corrected iterate for the
    // prolongation (y of a grid-wide level 1, x of a CTA level)
    {
        const int R0 = c->d.M + 2, P0 = c->d.P, es = c->es;
        // the box shapes of the kernel instance for this element size
        const int kBoxR = es == 4 ? TileGeom<float>::BoxR : TileGeom<double>::BoxR;
        const int kBoxW = es == 4 ? TileGeom<float>::BoxW : TileGeom<double>::BoxW;
        const int kCBoxR = es == 4 ? TileGeom<float>::CBoxR : TileGeom<double>::CBoxR;
        const int kCBoxW = es == 4 ? TileGeom<float>::CBoxW : TileGeom<double>::CBoxW;
        void* a0[7] = {c->mgArr[0][5], c->pcg[5], c->pcg[6], c->pcg[4], c->pcg[2], c->pcg[0], c->pcg[1]};
        CUtensorMap* m0[7] = {&c->mgMaps.z, &c->mgMaps.pa, &c->mgMaps.pb, &c->mgMaps.r, &c->mgMaps.d,
                              &c->mgMaps.fE, &c->mgMaps.fN};
        for (int q = 0; q < 7; ++q)
            if ((s = encode_map(m0[q], a0[q], es, P0, R0, kBoxW, kBoxR)) != CP_OK) return s;
        if ((s = encode_map(&c->mgMaps.x0, c->mgArr[0][4], es, P0, R0, kBoxW, kBoxR)) != CP_OK) return s;
        void* e1 = (Lg > 1) ? c->mgArr[1][5] : c->mgArr[1][4];
        if ((s = encode_map(&c->mgMaps.e1, e1, es, c->mgP[1], c->mgNI[1] + 2, kCBoxW, kCBoxR)) != CP_OK) return s;
    }
    const char* om = getenv("CP_MG_OMEGA");
    if (om) c->mgOmega = atof(om);
    const char* sc = getenv("CP_MG_SCALE");
    if (sc) c->mgScale = atof(sc);
    if (getenv("CP_MG_PROFILE")) {
        cp_status s2 = dalloc(c, &c->mgProf, (size_t)kMgProfSlots);
        if (s2 != CP_OK) return s2;
    }
    // one CTA per SM (the dense set-up needs kMgDynSmem of shared memory)
    int nb = 0;
    if (c->prm.precision == CP_PREC_MIXED) {
        cudaFuncSetAttribute(k_pcg_mg<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMgDynSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pcg_mg<float>, kMgThreads, kMgDynSmem);
    } else {
        cudaFuncSetAttribute(k_pcg_mg<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMgDynSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pcg_mg<double>, kMgThreads, kMgDynSmem);
    }
    if (nb < 1) return fail(CP_ERR_CUDA, "multigrid PCG kernel does not fit on an SM");
    c->gMg = c->numSMs;
    return CP_OK;
}

template <typename TV>
SaHier<TV> sa_hier(cp_ctx* c) {
    SaHier<TV> H;
    memset(&H, 0, sizeof(H));
    H.L = c->saL;
    H.Lg = c->saLg;
    H.omega = c->saOmega;
    H.w0 = c->saW0;
    H.wc = c->saWc;
    H.dense = (TV*)c->saDense;
    H.prof = c->saProf;
    H.r2 = (TV*)c->saArr[0][11];
    H.dinv0 = (TV*)c->saDinv0;
    H.reuse = c->saReuse;
    H.dirty = c->saDirty;
    for (int q = 0; q < 9; ++q) H.Y[q] = (TV*)c->saY[q];
    for (int l = 0; l < c->saL; ++l) {
        SaLevel<TV>& v = H.lv[l];
        v.nI = c->saNI[l]; v.nJ = c->saNJ[l]; v.P = c->saP[l];
        TV** a = reinterpret_cast<TV**>(c->saArr[l]);
        for (int q = 0; q < 9; ++q) v.c[q] = a[q];
        v.x = a[9]; v.y = a[10]; v.b = a[11]; v.t = a[12];
        for (int q = 0; q < 4; ++q) v.pw[q] = a[13 + q];
    }
    return H;
}

// dynamic shared memory of k_pcg_sa: the dense set-up workspace, then CTA
// 0's staged levels (at most kSaSmemBudget bytes)
constexpr size_t kSaDynSmem = sizeof(double) * (size_t)(kSaDense * 2 * kSaDense + kSaDense);
constexpr size_t kSaSmemMax = kSaDynSmem > kSaSmemBudget ? kSaDynSmem : kSaSmemBudget;
static_assert(kSaSmemMax + 4096 <= 227 * 1024, "k_pcg_sa's dynamic shared memory exceeds a block's limit");

// Level sizes of the smoothed aggregation: 3 x 3 aggregates (rounding up)
// until at most kSaDense unknowns.  Level 0 and the levels above kSaCtaCells
// unknowns run grid-wide, and so do further levels until the rest fits CTA
// 0's shared-memory budget.
cp_status sa_build(cp_ctx* c) {
    int nI = c->d.M - 1, nJ = c->d.N - 2;
    int L = 0;
    for (;;) {
        if (L >= kSaMaxLevels) return fail(CP_ERR_BAD_PARAM, "smoothed-aggregation hierarchy too deep");
        c->saNI[L] = nI; c->saNJ[L] = nJ;
        ++L;
        if ((long long)nI * nJ <= kSaDense && L >= 2) break;
        nI = sa_coarse(nI); nJ = sa_coarse(nJ);
    }
    c->saL = L;
    size_t budget = kSaSmemBudget;
    if (const char* e = getenv("CP_SA_SMEM_KB")) budget = std::min(budget, (size_t)std::max(atoi(e), 1) * 1024);
    int Lg = 1;
    while (Lg < L - 1 && ((long long)c->saNI[Lg] * c->saNJ[Lg] > kSaCtaCells ||
                          sa_cta_elems(c->saNI, c->saNJ, Lg, L) * c->es > budget))
        ++Lg;
    c->saLg = Lg;
    c->saSmem = std::max(kSaDynSmem, sa_cta_elems(c->saNI, c->saNJ, Lg, L) * c->es);
    if (c->saSmem > kSaSmemMax) return fail(CP_ERR_BAD_PARAM, "smoothed-aggregation coarsest level too large");
    c->saP[0] = c->d.P;
    cp_status s;
    // level 0: pre-smoothed iterate, corrected iterate, the second CG
    // residual buffer (its rhs is the CG residual), scratch
    for (int q = 9; q <= 15; ++q)
        if ((s = dalloc_bytes(c, &c->saArr[0][q], c->nElem * c->es)) != CP_OK) return s;
    if ((s = dalloc_bytes(c, &c->saDinv0, c->nElem * c->es)) != CP_OK) return s;
    if ((s = dalloc(c, &c->saDirty, 1)) != CP_OK) return s;
    if ((s = dalloc(c, &c->saDirtyAdj, 1)) != CP_OK) return s;
    const int one = 1;
    CK(cudaMemcpyAsync(c->saDirty, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int l = 1; l < L; ++l) {
        c->saP[l] = ((c->saNJ[l] + 2 + 31) / 32) * 32;
        const size_t ne = (size_t)(c->saNI[l] + 2) * c->saP[l];
        const int nq = (l < Lg && l < L - 1) ? 17 : 13;
        for (int q = 0; q < nq; ++q)
            if ((s = dalloc_bytes(c, &c->saArr[l][q], ne * c->es)) != CP_OK) return s;
    }
    for (int q = 0; q < 9; ++q)
        if ((s = dalloc_bytes(c, &c->saY[q], c->nElem * c->es)) != CP_OK) return s;
    if ((s = dalloc_bytes(c, &c->saDense, (size_t)kSaDense * kSaDense * c->es)) != CP_OK) return s;
    if (const char* e = getenv("CP_SA_OMEGA")) c->saOmega = atof(e);
    if (const char* e = getenv("CP_SA_W0")) c->saW0 = atof(e);
    if (const char* e = getenv("CP_SA_WC")) c->saWc = atof(e);
    if (const char* e = getenv("CP_SA_REUSE")) c->saReuse = std::max(atoi(e), 1);
    if (getenv("CP_SA_PROFILE") && (s = dalloc(c, &c->saProf, (size_t)SA_P_COUNT)) != CP_OK) return s;
    int nb = 0;
    if (c->prm.precision == CP_PREC_MIXED) {
        cudaFuncSetAttribute(k_pcg_sa<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSaSmemMax);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pcg_sa<float>, kMgThreads, c->saSmem);
    } else {
        cudaFuncSetAttribute(k_pcg_sa<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSaSmemMax);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pcg_sa<double>, kMgThreads, c->saSmem);
    }
    if (nb < 1) return fail(CP_ERR_CUDA, "smoothed-aggregation PCG kernel does not fit on an SM");
    return CP_OK;
}

template <typename Kern, typename... Args>
cudaError_t launch_coop_cfg(Kern kern, int grid, int threads, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <typename TC, bool Mixed>
cp_status enqueue_momentum(cp_ctx* c, int doU, int doV, int applyBC, EvRec* rec = nullptr) {
    Fields f{c->u, c->v, c->p, c->alpha, c->gamma};
    MomSys<TC> U = mom_sys<TC>(c, 0), V = mom_sys<TC>(c, 1);
    REC_BEGIN(rec, CP_K_ASSEMBLE);
    k_assemble<TC, Mixed><<<c->gElem, kThreads, 0, c->stream>>>(c->k, c->st, f, U, V, c->dE, c->dN, doU, doV);
    REC_END(rec);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(c->barJ, 0, sizeof(unsigned), c->stream));
    JacobiOut out{c->uStar, c->vStar};
    REC_BEGIN(rec, CP_K_JACOBI);
    CK(launch_coop(k_jacobi<TC, Mixed>, c->gJac, c->stream, c->k, c->st, U, V, (const double*)c->u,
                   (const double*)c->v, (TC*)c->xb[0], (TC*)c->xb[1], (TC*)c->xb[2], (TC*)c->xb[3], out,
                   (const double*)c->gamma, c->partJ, c->barJ, doU, doV, applyBC));
    REC_END(rec);
    return CP_OK;
}

template <typename TV>
cp_status enqueue_pressure(cp_ctx* c, EvRec* rec = nullptr) {
    PcgBufs<TV> B = pcg_bufs<TV>(c);
    REC_BEGIN(rec, CP_K_MASS);
    k_mass<TV><<<c->nbMass, kThreads, 0, c->stream>>>(c->k, c->st, c->u, c->v, c->uStar, c->vStar, B.rhs, c->partM);
    REC_END(rec);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(c->barP, 0, sizeof(unsigned), c->stream));
    REC_BEGIN(rec, CP_K_PCG);
    if (c->useSa) {
        SaHier<TV> H = sa_hier<TV>(c);
        CK(launch_coop_cfg(k_pcg_sa<TV>, c->gMg, kMgThreads, c->saSmem, c->stream, c->k, c->st,
                           (const double*)c->dE, (const double*)c->dN, B, H, c->pStar, c->partP, c->barP));
    } else if (c->useMg) {
        MgHier<TV> H = mg_hier<TV>(c);
        CK(launch_coop_cfg(k_pcg_mg<TV>, c->gMg, kMgThreads, kMgDynSmem, c->stream, c->k, c->st,
                           (const double*)c->dE, (const double*)c->dN, B, H, c->pStar, c->partP, c->barP, c->mgMaps));
    } else {
        CK(launch_coop(k_pcg<TV>, c->gPcg, c->stream, c->k, c->st, (const double*)c->dE, (const double*)c->dN, B,
                       c->pStar, c->partP, c->barP));
    }
    REC_END(rec);
    return CP_OK;
}

template <typename TC, bool Mixed>
cp_status enqueue_iteration(cp_ctx* c, EvRec* rec = nullptr) {
    REC_BEGIN(rec, CP_K_BC);
    k_bc<<<c->gElem, kThreads, 0, c->stream>>>(c->k, c->st, c->u, c->v, c->p, c->gamma, 1);
    REC_END(rec);
    CK(cudaGetLastError());
    cp_status s = enqueue_momentum<TC, Mixed>(c, 1, 1, 1, rec);
    if (s != CP_OK) return s;
    s = enqueue_pressure<TC>(c, rec);
    if (s != CP_OK) return s;
    REC_BEGIN(rec, CP_K_CORRECT);
    k_correct<<<c->gElem, kThreads, 0, c->stream>>>(c->k, c->st, c->u, c->v, c->p, c->uStar, c->vStar, c->pStar,
                                                    c->dE, c->dN);
    REC_END(rec);
    CK(cudaGetLastError());
    REC_BEGIN(rec, CP_K_BC);
    k_bc<<<c->gElem, kThreads, 0, c->stream>>>(c->k, c->st, c->u, c->v, c->p, c->gamma, 0);
    REC_END(rec);
    CK(cudaGetLastError());
    FinalizeArgs fa{c->u, c->v, c->p, c->gamma, c->partM, c->nbMass, c->hist, c->histCap, c->dpWin};
    REC_BEGIN(rec, CP_K_FINALIZE);
    k_finalize<<<1, 1024, 0, c->stream>>>(c->k, c->st, fa);
    REC_END(rec);
    CK(cudaGetLastError());
    return CP_OK;
}

cp_status enqueue_iteration_any(cp_ctx* c, EvRec* rec = nullptr) {
    return c->prm.precision == CP_PREC_MIXED ? enqueue_iteration<float, true>(c, rec)
                                             : enqueue_iteration<double, false>(c, rec);
}

cp_status build_graph(cp_ctx* c) {
    c->graphTried = true;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return CP_OK;
    }
    cp_status s = enqueue_iteration_any(c);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (s != CP_OK || e != cudaSuccess || !g) {
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        g_err.clear();
        return CP_OK;  // fall back to direct launches
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return CP_OK;
    }
    c->graph = ex;
    return CP_OK;
}

cp_status read_status(cp_ctx* c) {
    CK(cudaMemcpyAsync(c->stHost, c->st, sizeof(Status), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CP_OK;
}

void fill_report(cp_ctx* c, cp_iter_report* out) {
    if (!out) return;
    memset(out, 0, sizeof(*out));
    const Status& s = *c->stHost;
    out->iter = s.iter;
    out->done = s.done;
    out->stop_reason = s.reason;
    const int last = s.iter - 1;
    if (last >= 0 && last < c->histCap) {
        double row[kHistCols];
        if (cudaMemcpy(row, c->hist + (size_t)last * kHistCols, sizeof row, cudaMemcpyDeviceToHost) == cudaSuccess) {
            out->error = row[H_ERROR];
            out->residU_RMS = row[H_RMS_U]; out->residV_RMS = row[H_RMS_V]; out->residMass_RMS = row[H_RMS_MASS];
            out->residU_max = row[H_MAX_U]; out->residV_max = row[H_MAX_V]; out->residMass_max = row[H_MAX_MASS];
            out->pressureIterations = (int)row[H_ITERS_P];
            out->momentumItersU = (int)row[H_ITERS_U]; out->momentumItersV = (int)row[H_ITERS_V];
            out->coreTotalDrop = row[H_CORE_TOTAL]; out->fullTotalDrop = row[H_FULL_TOTAL];
            out->coreStaticDrop = row[H_CORE_STATIC]; out->fullStaticDrop = row[H_FULL_STATIC];
            out->inletMassFlux = row[H_IN_FLUX]; out->outletMassFlux = row[H_OUT_FLUX];
            out->residU = row[H_RES_U]; out->residV = row[H_RES_V]; out->residMass = row[H_RES_MASS];
        }
    }
}

cp_status device_error(cp_ctx* c) {
    if (c->stHost->err != 0)
        return fail((cp_status)c->stHost->err, "device reported %s at iteration %d",
                    cp_status_string((cp_status)c->stHost->err), c->stHost->iter);
    return CP_OK;
}

cp_status run_iterations(cp_ctx* c, long long n, bool untilDone, cp_iter_report* out) {
    if (!c->graphTried) {
        cp_status s = build_graph(c);
        if (s != CP_OK) return s;
    }
    CK(cudaEventRecord(c->ev0, c->stream));
    long long done = 0;
    const int chunk = std::max(1, c->prm.chunk);
    for (;;) {
        const long long todo = untilDone ? chunk : std::min<long long>(chunk, n - done);
        if (todo <= 0) break;
        for (long long q = 0; q < todo; ++q) {
            if (c->graph) CK(cudaGraphLaunch(c->graph, c->stream));
            else {
                cp_status s = enqueue_iteration_any(c);
                if (s != CP_OK) return s;
            }
        }
        done += todo;
        cp_status s = read_status(c);
        if (s != CP_OK) return s;
        if (c->stHost->done) break;
        if (!untilDone && done >= n) break;
    }
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    fill_report(c, out);
    if (out) out->device_ms = ms;
    return device_error(c);
}

cp_status strided_to_dense(const double* host, long rows, long cols, long rs, long cs, int R, int C,
                           std::vector<double>& dense) {
    if (!host) return fail(CP_ERR_BAD_PARAM, "host pointer is NULL");
    if (rows != R || cols != C) return fail(CP_ERR_BAD_PARAM, "shape %ld x %ld, expected %d x %d", rows, cols, R, C);
    dense.resize((size_t)R * C);
    for (long i = 0; i < rows; ++i)
        for (long j = 0; j < cols; ++j) {
            const double x = host[i * rs + j * cs];
            if (!std::isfinite(x)) return fail(CP_ERR_NONFINITE, "non-finite input at (%ld, %ld)", i, j);
            dense[(size_t)i * C + j] = x;
        }
    return CP_OK;
}

}  // namespace

// ======================================================================== C ABI
extern "C" {

const char* cp_status_string(cp_status s) {
    switch (s) {
        case CP_OK: return "CP_OK";
        case CP_ERR_BAD_PARAM: return "CP_ERR_BAD_PARAM";
        case CP_ERR_UNSUPPORTED: return "CP_ERR_UNSUPPORTED";
        case CP_ERR_NONFINITE: return "CP_ERR_NONFINITE";
        case CP_ERR_TIMEOUT: return "CP_ERR_TIMEOUT";
        case CP_ERR_CUDA: return "CP_ERR_CUDA";
        case CP_ERR_STATE: return "CP_ERR_STATE";
    }
    return "CP_ERR_UNKNOWN";
}

const char* cp_last_error_string(void) { return g_err.c_str(); }

void cp_params_default(cp_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->epsilon = 1e-7;
    p->maxIterations = 1000;
    p->saveStateInterval = 1000;
    p->reuseInitialFields = 0;
    p->xPlaneCoreInlet = 0.01;
    p->xPlaneCoreOutlet = 0.05;
    p->usePressureDropConvergence = 1;
    p->dpConvergenceWindow = 500;
    p->dpConvergencePercent = 1.0;
    p->usePressureDropSlopeGate = 0;
    p->dpSlopeWindowIters = 1000;
    p->dpSlopeMaxDelta = 10.0;
    p->numThreads = 8;
    p->pressureSolverType = 4;
    p->parallelizeDirectSolver = 1;
    p->maxPressureIter = 30;
    p->pTol = 1e-6;
    p->sorOmega = 0.0;
    p->momentumSolverType = 1;
    p->momentumTol = 1e-6;
    p->maxMomentumIter = 400;
    p->momentumSorOmega = 1.0;
    p->convectionScheme = 0;
    p->enableTwoPointFiveD = 0;
    p->twoPointFiveDConvectionFactor = 1.2;
    p->twoPointFiveDSinkMultiplier = 1.0;
    p->Ht_channel = 0.0;
    p->brinkmanKMin = 1e-14;
    p->brinkmanQ = 1.0;
    p->timeStepMultiplier = 0.01;
    p->enablePseudoTimeStepping = 0;
    p->pseudoCFL = 0.1;
    p->minPseudoSpeed = 0.05;
    p->useLocalPseudoTime = 1;
    p->pseudoControllerMode = 2;
    p->enableSER = 0;
    p->enableLineSearch = 0;
    p->enableCflRamp = 0;
    p->rho = 997.0;
    p->eta = 0.00089;
    p->targetVel = 0.0;
    p->enableInletRamp = 0;
    p->rampSteps = 1000;
    p->uvAlpha = 0.7;
    p->pAlpha = 0.3;
    p->enableResidualViscosity = 0;
    p->enableNormalizedResiduals = 0;
    p->residNormFloorVel = 1e-6;
    p->residNormFloorMass = 1e-12;
    p->precision = CP_PREC_FP64;
    p->historyCapacity = 0;   // 0: maxIterations rows
    p->chunk = 32;
    p->adjointModel = CP_ADJ_AUTO;
}

cp_status cp_read_fluid_params(const char* path, cp_params* p) {
    if (!path || !p) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    FILE* f = fopen(path, "r");
    if (!f) return fail(CP_ERR_BAD_PARAM, "cannot open %s", path);
    int Ny = 0, Nx = 0, nin = 0, nout = 0;
    double hy = 0, hx = 0, U = 0, Ht = 0;
    const int got = fscanf(f, "%d %d %lf %lf %lf %d %d", &Ny, &Nx, &hy, &hx, &U, &nin, &nout);
    if (got != 7) {
        fclose(f);
        return fail(CP_ERR_BAD_PARAM, "%s: expected 'Ny Nx hy hx U N_in N_out [Ht]'", path);
    }
    if (fscanf(f, "%lf", &Ht) != 1) Ht = p->Ht_channel;
    fclose(f);
    if (Ny <= 0 || Nx <= 0 || hy <= 0 || hx <= 0)
        return fail(CP_ERR_BAD_PARAM, "%s: non-positive grid size or spacing", path);
    p->Ny = Ny; p->Nx = Nx; p->hy = hy; p->hx = hx; p->targetVel = U;
    p->N_in_buffer = nin; p->N_out_buffer = nout; p->Ht_channel = Ht;
    return CP_OK;
}

cp_status cp_create(const cp_params* prm, cp_ctx** out) {
    if (!out) return fail(CP_ERR_BAD_PARAM, "out is NULL");
    *out = nullptr;
    cp_status s = validate(prm);
    if (s != CP_OK) return s;
    cp_ctx* c = new cp_ctx();
    c->prm = *prm;
    if (c->prm.enableTwoPointFiveD && c->prm.Ht_channel <= 0.0) c->prm.enableTwoPointFiveD = 0;
    const int M = prm->Ny + 1, N = prm->Nx + 1;
    c->d.M = M;
    c->d.N = N;
    c->d.P = ((N + 1 + 31) / 32) * 32;
    c->nElem = (size_t)(M + 2) * c->d.P;
    c->es = prm->precision == CP_PREC_MIXED ? 4 : 8;
    auto bail = [&](cp_status e) { cp_destroy(c); return e; };
    if (cudaGetDevice(&c->dev) != cudaSuccess) return bail(fail(CP_ERR_CUDA, "no CUDA device"));
    if (cudaDeviceGetAttribute(&c->numSMs, cudaDevAttrMultiProcessorCount, c->dev) != cudaSuccess)
        return bail(fail(CP_ERR_CUDA, "cudaDeviceGetAttribute failed"));
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(CP_ERR_CUDA, "cudaStreamCreate failed"));
    if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess)
        return bail(fail(CP_ERR_CUDA, "cudaEventCreate failed"));
    fill_kparams(c);
    double** fields[] = {&c->u, &c->v, &c->p, &c->uStar, &c->vStar, &c->pStar, &c->dE, &c->dN, &c->gamma, &c->alpha};
    for (double** f : fields)
        if ((s = dalloc(c, f, c->nElem)) != CP_OK) return bail(s);
    for (auto& m : c->mom)
        if ((s = dalloc_bytes(c, &m, c->nElem * c->es)) != CP_OK) return bail(s);
    for (auto& x : c->xb)
        if ((s = dalloc_bytes(c, &x, c->nElem * c->es)) != CP_OK) return bail(s);
    for (auto& x : c->pcg)
        if ((s = dalloc_bytes(c, &x, c->nElem * c->es)) != CP_OK) return bail(s);
    // cooperative grids: every block must be resident
    int nbJ = 0, nbP = 0;
    if (c->prm.precision == CP_PREC_MIXED) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbJ, k_jacobi<float, true>, kThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbP, k_pcg<float>, kThreads, 0);
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbJ, k_jacobi<double, false>, kThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbP, k_pcg<double>, kThreads, 0);
    }
    if (nbJ < 1 || nbP < 1) return bail(fail(CP_ERR_CUDA, "cooperative kernels do not fit on an SM"));
    // as many Jacobi CTAs per SM as fit (float: 3 of 256 threads, 12 % faster
    // sweeps at 2048 x 1024 than 2; double: 2), at most 4; CP_JACOBI_CTAS
    // caps it lower
    int jacCtas = 4;
    if (const char* e = getenv("CP_JACOBI_CTAS")) jacCtas = std::max(atoi(e), 1);
    c->gJac = c->numSMs * std::min(nbJ, jacCtas);
    c->gPcg = c->numSMs * std::min(nbP, 4);
    c->gElem = c->numSMs * 4;
    c->nbMass = c->numSMs * 4;
    if (c->gJac > kMaxBlocks || c->gPcg > kMaxBlocks || c->nbMass > kMaxBlocks)
        return bail(fail(CP_ERR_CUDA, "too many SMs for the partial-sum buffers"));
    c->useMg = (prm->pressureSolverType == 2 || prm->pressureSolverType == 4);
    if (c->useMg && (s = mg_build(c)) != CP_OK) return bail(s);
    // type 4 (AMGCL's AMG-CG in the reference) runs the smoothed-aggregation
    // cycle; CP_PRESSURE_CYCLE=pairs selects the 2 x 2 aggregation of type 2
    const char* cyc = getenv("CP_PRESSURE_CYCLE");
    c->useSa = prm->pressureSolverType == 4 && !(cyc && strcmp(cyc, "pairs") == 0);
    if (c->useSa && (s = sa_build(c)) != CP_OK) return bail(s);
    if ((s = dalloc(c, &c->partJ, (size_t)4 * c->gJac)) != CP_OK) return bail(s);
    if ((s = dalloc(c, &c->partM, (size_t)4 * c->nbMass)) != CP_OK) return bail(s);
    if ((s = dalloc(c, &c->partP, (size_t)3 * std::max(c->gPcg, c->gMg))) != CP_OK) return bail(s);
    if ((s = dalloc(c, &c->barJ, 1)) != CP_OK) return bail(s);
    if ((s = dalloc(c, &c->barP, 1)) != CP_OK) return bail(s);
    if ((s = dalloc(c, &c->st, 1)) != CP_OK) return bail(s);
    c->histCap = prm->historyCapacity > 0 ? prm->historyCapacity : std::max(prm->maxIterations, 1);
    if ((s = dalloc(c, &c->hist, (size_t)c->histCap * kHistCols)) != CP_OK) return bail(s);
    if ((s = dalloc(c, &c->dpWin, (size_t)std::max(prm->dpConvergenceWindow, 1))) != CP_OK) return bail(s);
    if (cudaMallocHost(&c->stHost, sizeof(Status)) != cudaSuccess) return bail(fail(CP_ERR_CUDA, "cudaMallocHost failed"));
    memset(c->stHost, 0, sizeof(Status));
    // all fluid until a geometry is set (SIMPLE.cpp:267-269)
    c->cellTypeHost.assign((size_t)M * N, 0.0);
    std::vector<double> g((size_t)M * N);
    build_density(c, c->cellTypeHost, g.data());
    if ((s = upload_cells(c, g.data())) != CP_OK) return bail(s);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(CP_ERR_CUDA, "initialisation failed"));
    *out = c;
    return CP_OK;
}

cp_status cp_destroy(cp_ctx* c) {
    if (!c) return CP_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->saProf) {
        // CP_SA_PROFILE: device time per phase of the smoothed-aggregation PCG,
        // summed over the context's life (block 0's clock after each barrier)
        unsigned long long t[SA_P_COUNT];
        if (cudaMemcpy(t, c->saProf, sizeof t, cudaMemcpyDeviceToHost) == cudaSuccess) {
            fprintf(stderr, "CP_SA_PROFILE ms: setup %.3f galerkin %.3f matvec %.3f update %.3f cta %.3f", t[SA_P_SETUP] * 1e-6,
                    t[SA_P_GALERKIN] * 1e-6, t[SA_P_MATVEC] * 1e-6, t[SA_P_UPDATE] * 1e-6, t[SA_P_CTA] * 1e-6);
            for (int l = 0; l < c->saLg; ++l) fprintf(stderr, " down%d %.3f", l, t[SA_P_DOWN + l] * 1e-6);
            for (int l = 0; l < c->saLg; ++l) fprintf(stderr, " up%d %.3f", l, t[SA_P_UP + l] * 1e-6);
            fprintf(stderr, " levels %d grid %d\n", c->saL, c->saLg);
        }
    }
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (void* q : c->allocs) cudaFree(q);
    if (c->stHost) cudaFreeHost(c->stHost);
    if (c->gammaStage) cudaFreeHost(c->gammaStage);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return CP_OK;
}

// The padded cell types (the extra row and column copied, SIMPLE.cpp:667-676)
// from a strided host array of cell types or, with fromGamma, of densities
// (cellType = 1 - gamma), checked for non-finite values before anything
// changes; then the density field on the device.
static cp_status set_cells(cp_ctx* c, const double* src, long rows, long cols, long rs, long cs, bool fromGamma) {
    if (!c) return fail(CP_ERR_BAD_PARAM, "ctx is NULL");
    if (!src) return fail(CP_ERR_BAD_PARAM, "host pointer is NULL");
    const int M = c->d.M, N = c->d.N, pr = M - 1, pc = N - 1;
    if (rows != pr || cols != pc) return fail(CP_ERR_BAD_PARAM, "shape %ld x %ld, expected %d x %d", rows, cols, pr, pc);
    // checked first, so that a rejected input leaves the geometry as it was
    for (long i = 0; i < rows; ++i)
        for (long j = 0; j < cols; ++j)
            if (!std::isfinite(src[i * rs + j * cs])) return fail(CP_ERR_NONFINITE, "non-finite input at (%ld, %ld)", i, j);
    // gamma goes up from a pinned staging array the context keeps (DMA; no
    // fresh host pages per call)
    if (!c->gammaStage && cudaMallocHost(&c->gammaStage, (size_t)M * N * sizeof(double)) != cudaSuccess) {
        c->gammaStage = nullptr;
        cudaGetLastError();
        return fail(CP_ERR_CUDA, "cudaMallocHost of the gamma staging array failed");
    }
    std::vector<double>& P = c->cellTypeHost;   // M x N padded; every entry is rewritten
    for (long i = 0; i < rows; ++i) {
        const double* row = src + i * rs;
        double* out = P.data() + (size_t)i * N;
        for (long j = 0; j < cols; ++j) out[j] = fromGamma ? 1.0 - row[j * cs] : row[j * cs];
    }
    for (int i = 0; i < pr; ++i) P[(size_t)i * N + pc] = P[(size_t)i * N + pc - 1];
    for (int j = 0; j < N; ++j) P[(size_t)pr * N + j] = P[(size_t)(pr - 1) * N + std::min(j, pc - 1)];
    build_density(c, P, c->gammaStage);
    return upload_cells(c, c->gammaStage);
}

cp_status cp_set_cell_type(cp_ctx* c, const double* ct, long rows, long cols, long rs, long cs) {
    return set_cells(c, ct, rows, cols, rs, cs, false);
}

cp_status cp_set_gamma(cp_ctx* c, const double* gm, long rows, long cols, long rs, long cs) {
    return set_cells(c, gm, rows, cols, rs, cs, true);
}

cp_status cp_read_geometry(cp_ctx* c, const char* path) {
    if (!c || !path) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    const int pr = c->d.M - 1, pc = c->d.N - 1;
    std::vector<double> ct((size_t)pr * pc, 0.0);
    FILE* f = fopen(path, "r");
    if (f) {  // missing file: all fluid (SIMPLE.cpp:645-649); short file: rest fluid
        for (size_t q = 0; q < ct.size(); ++q)
            if (fscanf(f, "%lf", &ct[q]) != 1) break;
        fclose(f);
    }
    return cp_set_cell_type(c, ct.data(), pr, pc, pc, 1);
}

cp_status cp_get_field(cp_ctx* c, cp_field which, double* host, long rows, long cols, long rs, long cs) {
    if (!c || !host) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    double* dp = nullptr;
    int R = 0, C = 0;
    if (!field_shape(c, which, &dp, &R, &C)) return fail(CP_ERR_BAD_PARAM, "unknown field %d", (int)which);
    if (rows != R || cols != C) return fail(CP_ERR_BAD_PARAM, "shape %ld x %ld, expected %d x %d", rows, cols, R, C);
    if (which != CP_FIELD_CELLTYPE && cs == 1 && rs >= C) {
        // rows of the caller's array directly (pinned memory goes by DMA)
        CK(cudaMemcpy2DAsync(host, (size_t)rs * 8, dp, (size_t)c->d.P * 8, (size_t)C * 8, R, cudaMemcpyDeviceToHost,
                             c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return CP_OK;
    }
    std::vector<double> dense((size_t)R * C);
    if (which == CP_FIELD_CELLTYPE) {
        dense = c->cellTypeHost;
    } else {
        CK(cudaMemcpy2DAsync(dense.data(), (size_t)C * 8, dp, (size_t)c->d.P * 8, (size_t)C * 8, R,
                             cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    for (long i = 0; i < rows; ++i)
        for (long j = 0; j < cols; ++j) host[i * rs + j * cs] = dense[(size_t)i * C + j];
    return CP_OK;
}

cp_status cp_set_field(cp_ctx* c, cp_field which, const double* host, long rows, long cols, long rs, long cs) {
    if (!c) return fail(CP_ERR_BAD_PARAM, "ctx is NULL");
    if (which == CP_FIELD_GAMMA || which == CP_FIELD_ALPHA || which == CP_FIELD_CELLTYPE)
        return fail(CP_ERR_BAD_PARAM, "use cp_set_cell_type / cp_set_gamma for the geometry");
    double* dp = nullptr;
    int R = 0, C = 0;
    if (!field_shape(c, which, &dp, &R, &C)) return fail(CP_ERR_BAD_PARAM, "unknown field %d", (int)which);
    std::vector<double> dense;
    cp_status s = strided_to_dense(host, rows, cols, rs, cs, R, C, dense);
    if (s != CP_OK) return s;
    CK(cudaMemcpy2DAsync(dp, (size_t)c->d.P * 8, dense.data(), (size_t)C * 8, (size_t)C * 8, R,
                         cudaMemcpyHostToDevice, c->stream));
    if (mark_sa_stale(c) != CP_OK) return CP_ERR_CUDA;
    CK(cudaStreamSynchronize(c->stream));
    return CP_OK;
}

cp_status cp_step(cp_ctx* c, int n_outer, cp_iter_report* out) {
    if (!c) return fail(CP_ERR_BAD_PARAM, "ctx is NULL");
    if (n_outer < 0) return fail(CP_ERR_BAD_PARAM, "n_outer < 0");
    cp_status s = read_status(c);
    if (s != CP_OK) return s;
    if (c->stHost->done) {
        fill_report(c, out);
        return c->stHost->err ? device_error(c) : CP_OK;
    }
    return run_iterations(c, n_outer, false, out);
}

cp_status cp_run(cp_ctx* c, cp_iter_report* out) {
    if (!c) return fail(CP_ERR_BAD_PARAM, "ctx is NULL");
    cp_status s = read_status(c);
    if (s != CP_OK) return s;
    if (c->stHost->done) {
        fill_report(c, out);
        return c->stHost->err ? device_error(c) : CP_OK;
    }
    return run_iterations(c, 0, true, out);
}

cp_status cp_reset_loop(cp_ctx* c) {
    if (!c) return fail(CP_ERR_BAD_PARAM, "ctx is NULL");
    CK(cudaMemsetAsync(c->st, 0, sizeof(Status), c->stream));
    CK(cudaMemsetAsync(c->dpWin, 0, sizeof(double) * std::max(c->prm.dpConvergenceWindow, 1), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CP_OK;
}

cp_status cp_reset(cp_ctx* c) {
    if (!c) return fail(CP_ERR_BAD_PARAM, "ctx is NULL");
    double* f[] = {c->u, c->v, c->p, c->uStar, c->vStar, c->pStar, c->dE, c->dN};
    for (double* q : f) CK(cudaMemsetAsync(q, 0, c->nElem * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->hist, 0, (size_t)c->histCap * kHistCols * sizeof(double), c->stream));
    return cp_reset_loop(c);
}

cp_status cp_kernel_times(cp_ctx* c, int n_outer, cp_kernel_timing* out) {
    if (!c || !out) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    memset(out, 0, sizeof(*out));
    EvRec rec;
    for (auto& e : rec.ev) CK(cudaEventCreate(&e));
    cp_status s = CP_OK;
    for (int it = 0; it < n_outer && s == CP_OK; ++it) {
        if ((s = read_status(c)) != CP_OK) break;
        if (c->stHost->done) break;
        rec.n = 0;
        if ((s = enqueue_iteration_any(c, &rec)) != CP_OK) break;
        if ((s = read_status(c)) != CP_OK) break;
        for (int q = 0; q < rec.n; ++q) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, rec.ev[2 * q], rec.ev[2 * q + 1]) == cudaSuccess) {
                out->ms[rec.kind[q]] += ms;
                out->launches[rec.kind[q]] += 1;
            }
        }
        out->jacobiSweeps += c->stHost->itersU + c->stHost->itersV;
        out->pcgIterations += c->stHost->itersP;
        out->iterations += 1;
        if ((s = device_error(c)) != CP_OK) break;
    }
    for (auto& e : rec.ev) cudaEventDestroy(e);
    if (c->mgProf && out->iterations > 0) {
        unsigned long long pr[kMgProfSlots];
        if (cudaMemcpy(pr, c->mgProf, sizeof pr, cudaMemcpyDeviceToHost) == cudaSuccess) {
            const char* names[MG_P_COUNT] = {"setup", "cg_A", "cg_B", "vdown", "vcta", "vup"};
            fprintf(stderr, "[cp mg profile] per outer iteration (us):");
            for (int q = 0; q < MG_P_COUNT; ++q) fprintf(stderr, " %s %.1f", names[q], pr[q] * 1e-3 / out->iterations);
            fprintf(stderr, "\n[cp mg profile] restriction out of level l:");
            for (int l = 0; l < c->mgLg; ++l) fprintf(stderr, " %d:%.1f", l, pr[MG_P_COUNT + l] * 1e-3 / out->iterations);
            fprintf(stderr, "\n[cp mg profile] prolongation into level l:");
            for (int l = 0; l < c->mgLg; ++l)
                fprintf(stderr, " %d:%.1f", l, pr[MG_P_COUNT + kMgMaxLevels + l] * 1e-3 / out->iterations);
            fprintf(stderr, "\n");
        }
        cudaMemset(c->mgProf, 0, sizeof pr);
    }
    return s;
}

static cp_status momentum_one(cp_ctx* c, int isU, double* resid, int* iters) {
    if (!c) return fail(CP_ERR_BAD_PARAM, "ctx is NULL");
    cp_status s = read_status(c);
    if (s != CP_OK) return s;
    if (c->stHost->done) return fail(CP_ERR_STATE, "loop already stopped; call cp_reset_loop first");
    // reset the max-change accumulators, then assemble + solve one component
    CK(cudaMemsetAsync(&c->st->maxDU, 0, 2 * sizeof(unsigned long long), c->stream));
    s = c->prm.precision == CP_PREC_MIXED ? enqueue_momentum<float, true>(c, isU, !isU, 0)
                                          : enqueue_momentum<double, false>(c, isU, !isU, 0);
    if (s != CP_OK) return s;
    if ((s = read_status(c)) != CP_OK) return s;
    const unsigned long long bits = isU ? c->stHost->maxDU : c->stHost->maxDV;
    double r;
    memcpy(&r, &bits, sizeof r);
    if (resid) *resid = r;
    if (iters) *iters = isU ? c->stHost->itersU : c->stHost->itersV;
    return device_error(c);
}

cp_status cp_momentum_u(cp_ctx* c, double* resid, int* iters) { return momentum_one(c, 1, resid, iters); }
cp_status cp_momentum_v(cp_ctx* c, double* resid, int* iters) { return momentum_one(c, 0, resid, iters); }

cp_status cp_pressure(cp_ctx* c, int* iters, double* residMass) {
    if (!c) return fail(CP_ERR_BAD_PARAM, "ctx is NULL");
    cp_status s = read_status(c);
    if (s != CP_OK) return s;
    if (c->stHost->done) return fail(CP_ERR_STATE, "loop already stopped; call cp_reset_loop first");
    CK(cudaMemsetAsync(c->pStar, 0, c->nElem * sizeof(double), c->stream));
    if ((s = mark_sa_stale(c)) != CP_OK) return s;
    s = c->prm.precision == CP_PREC_MIXED ? enqueue_pressure<float>(c) : enqueue_pressure<double>(c);
    if (s != CP_OK) return s;
    std::vector<double> part((size_t)4 * c->nbMass);
    CK(cudaMemcpyAsync(part.data(), c->partM, part.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    if ((s = read_status(c)) != CP_OK) return s;
    double mx = 0.0;
    for (int b = 0; b < c->nbMass; ++b) mx = std::max(mx, part[(size_t)b * 4 + 3]);
    if (residMass) *residMass = mx;
    if (iters) *iters = c->stHost->itersP;
    return device_error(c);
}

int cp_history_columns(void) { return kHistCols; }

cp_status cp_get_history(cp_ctx* c, double* rows, int max_rows, int* n_rows) {
    if (!c || !rows) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    cp_status s = read_status(c);
    if (s != CP_OK) return s;
    const int n = std::min(std::min(c->stHost->iter, c->histCap), std::max(max_rows, 0));
    if (n > 0)
        CK(cudaMemcpy(rows, c->hist, (size_t)n * kHistCols * sizeof(double), cudaMemcpyDeviceToHost));
    if (n_rows) *n_rows = n;
    return CP_OK;
}

}  // extern "C"

// ======================================================================== adjoint
namespace {

cp_status adjoint_alloc(cp_ctx* c) {
    if (c->adjSt) return CP_OK;
    for (auto& a : c->adj) {
        cp_status s = dalloc(c, &a, c->nElem);
        if (s != CP_OK) return s;
    }
    for (auto& m : c->adjMom) {
        cp_status s = dalloc_bytes(c, &m, c->nElem * sizeof(double));
        if (s != CP_OK) return s;
    }
    cp_status s;
    if ((s = dalloc(c, &c->adjSt, 1)) != CP_OK) return s;
    if ((s = dalloc(c, &c->adjPart, (size_t)4 * kMaxBlocks)) != CP_OK) return s;
    if ((s = dalloc(c, &c->adjBar, 1)) != CP_OK) return s;
    if (const char* e = getenv("CP_ADJ_RESTART")) c->adjRestart = std::min(std::max(atoi(e), 1), kKryMaxDots - 1);
    if (const char* e = getenv("CP_ADJ_PITERS")) c->adjPIters = std::max(atoi(e), 1);
    if (const char* e = getenv("CP_ADJ_SWEEPS")) c->adjSweeps = std::max(atoi(e), 1);
    if (!c->useMg) c->adjPIters = std::max(c->adjPIters, 100);
    const size_t L = 3 * c->nElem;
    if ((s = dalloc(c, &c->adjKry, (size_t)(2 * c->adjRestart + 3) * L)) != CP_OK) return s;
    if ((s = dalloc(c, &c->adjKryPart, (size_t)kKryMaxDots * kMaxBlocks)) != CP_OK) return s;
    if ((s = dalloc(c, &c->adjH, (size_t)3 * kKryMaxDots)) != CP_OK) return s;
    return CP_OK;
}

template <typename TV>
cp_status adjoint_pcg(cp_ctx* c, const KParams& k, const double* dE, const double* dN, double* out) {
    PcgBufs<TV> B = pcg_bufs<TV>(c);
    CK(cudaMemsetAsync(c->adjBar, 0, sizeof(unsigned), c->stream));
    if (c->useSa) {
        SaHier<TV> H = sa_hier<TV>(c);
        // the adjoint's operator is fixed over one adjoint solve: built by its
        // first pressure-like solve, reused by the rest (the caller marks both
        // flags stale at the start)
        H.dirty = c->saDirtyAdj;
        H.reuse = 0;
        CK(launch_coop_cfg(k_pcg_sa<TV>, c->gMg, kMgThreads, c->saSmem, c->stream, k, c->adjSt, dE, dN, B, H, out,
                           c->adjPart, c->adjBar));
    } else if (c->useMg) {
        MgHier<TV> H = mg_hier<TV>(c);
        CK(launch_coop_cfg(k_pcg_mg<TV>, c->gMg, kMgThreads, kMgDynSmem, c->stream, k, c->adjSt, dE, dN, B, H, out,
                           c->adjPart, c->adjBar, c->mgMaps));
    } else {
        CK(launch_coop(k_pcg<TV>, c->gPcg, c->stream, k, c->adjSt, dE, dN, B, out, c->adjPart, c->adjBar));
    }
    return CP_OK;
}

// x_{j+1} buffer of the frozen sweeps (allocated on first use)
cp_status adjoint_xbuf(cp_ctx* c, std::vector<double*>& xs, size_t j, double** out) {
    while (xs.size() <= j) {
        double* q = nullptr;
        cp_status s = dalloc(c, &q, c->nElem);
        if (s != CP_OK) return s;
        CK(cudaMemsetAsync(q, 0, c->nElem * sizeof(double), c->stream));
        xs.push_back(q);
    }
    *out = xs[j];
    return CP_OK;
}

// The forward Jacobi sweeps of one component at the converged state, in
// FP64 and with the reference's stop rule (sum of r^2 of the pre-update
// residual below momentumTol^2 n, at most maxMomentumIter sweeps); the
// iterates are kept for the reverse sweeps.  Returns the sweep count.
template <bool IsU>
cp_status adjoint_sweeps(cp_ctx* c, const KParams& k, const MomSys<double>& S, const double* field,
                         std::vector<double*>& xs, int* count) {
    int i1, j1;
    mom_range<IsU>(c->d, i1, j1);
    const double lim = k.momTol * k.momTol * (double)i1 * (double)j1;
    const int nb = c->gElem;
    std::vector<double> part(nb);
    const double* x = nullptr;
    int its = 0;
    for (int q = 0; q < std::max(k.maxMom, 1); ++q) {
        double* xn = nullptr;
        cp_status s = adjoint_xbuf(c, xs, (size_t)q, &xn);
        if (s != CP_OK) return s;
        k_adj_sweep<IsU><<<nb, kThreads, 0, c->stream>>>(k, S, field, x, xn, c->adjPart);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(part.data(), c->adjPart, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        double tot = 0.0;
        for (int b = 0; b < nb; ++b) tot += part[b];
        x = xn;
        its = q + 1;
        if (!std::isfinite(tot)) return fail(CP_ERR_NONFINITE, "adjoint: momentum sweep residual is not finite");
        if (tot < lim) break;
    }
    *count = its;
    return CP_OK;
}

template <typename TV>
cp_status adjoint_prhs(cp_ctx* c, const KParams& k, const double* du, const double* dv, const double* rp) {
    PcgBufs<TV> B = pcg_bufs<TV>(c);
    k_adj_prhs<TV><<<c->gElem, kThreads, 0, c->stream>>>(k, du, dv, rp, B.rhs);
    CK(cudaGetLastError());
    return CP_OK;
}

}  // namespace

// The adjoint solve; probeOp >= 0 selects a verification output instead of
// the gradient (cp_adjoint_probe): 0 y = J_X^T x, 1 y = dJ/dX, 2 y = lambda.
static cp_status adjoint_impl(cp_ctx* c, double* grad, long rows, long cols, long rs, long cs, int max_iter, double tol,
                              cp_adjoint_report* rep, int probeOp, const double* px, double* py, int* info) {
    const int M = c->d.M, N = c->d.N;
    cp_status s = adjoint_alloc(c);
    if (s != CP_OK) return s;
    // the adjoint's pressure-like solves store their own coarse operators:
    // built once for this solve, and the forward's rebuilt after it
    if (c->saDirtyAdj) {
        static const int one = 1;
        CK(cudaMemcpyAsync(c->saDirtyAdj, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
        if ((s = mark_sa_stale(c)) != CP_OK) return s;
    }
    CK(cudaEventRecord(c->ev0, c->stream));
    // vectors
    double** A = c->adj;
    AdjVecs V;
    V.lu = A[0]; V.lv = A[1]; V.lc = A[2]; V.yu = A[3]; V.yv = A[4]; V.yp = A[5];
    V.gu = A[6]; V.gv = A[7]; V.gp = A[8]; V.du = A[9]; V.dv = A[10]; V.eu = A[11]; V.ev = A[12];
    double *dc = A[16], *Jd = A[17];
    double *clampU = A[13], *clampV = A[14], *dEp = A[15], *dNp = A[19];
    double* ybU[2] = {A[32], A[33]};
    double* ybV[2] = {A[34], A[35]};
    const size_t bytes = c->nElem * sizeof(double);
    for (int q = 0; q < 40; ++q) CK(cudaMemsetAsync(A[q], 0, bytes, c->stream));
    CK(cudaMemsetAsync(c->adjSt, 0, sizeof(Status), c->stream));
    // the converged state's iteration count fixes the inlet velocity (ramp)
    CK(cudaMemcpyAsync(c->stHost, c->st, sizeof(Status), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const int iterState = std::max(c->stHost->iter - 1, 0);
    KParams k = c->k;
    // Picard coefficients of the converged state (double), dE / dN
    MomSys<double> Us, Vs;
    {
        double** m = reinterpret_cast<double**>(c->adjMom);
        Us.aP = m[0]; Us.aE = m[1]; Us.aW = m[2]; Us.aN = m[3]; Us.aS = m[4]; Us.b = m[5];
        Vs.aP = m[6]; Vs.aE = m[7]; Vs.aW = m[8]; Vs.aN = m[9]; Vs.aS = m[10]; Vs.b = m[11];
    }
    // the assembly reads Status::iter for the inlet velocity
    CK(cudaMemcpyAsync(&c->adjSt->iter, &iterState, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    Fields f{c->u, c->v, c->p, c->alpha, c->gamma};
    k_assemble<double, false><<<c->gElem, kThreads, 0, c->stream>>>(k, c->adjSt, f, Us, Vs, c->dE, c->dN, 1, 1);
    CK(cudaGetLastError());
    AdjCtx ac;
    ac.k = k;
    ac.u = c->u; ac.v = c->v; ac.p = c->p; ac.alpha = c->alpha; ac.gamma = c->gamma;
    ac.maxVel = max_vel(inlet_velocity(k, iterState));
    // the frozen sweeps: the reference's Jacobi iterates from x_0 = u (v) at
    // the converged state, their count and the clamped unknowns
    int sU = 0, sV = 0;
    if ((s = adjoint_sweeps<true>(c, k, Us, c->u, c->adjXU, &sU)) != CP_OK) return s;
    if ((s = adjoint_sweeps<false>(c, k, Vs, c->v, c->adjXV, &sV)) != CP_OK) return s;
    const int nb = c->gElem;
    k_adj_clampmask<true><<<nb, kThreads, 0, c->stream>>>(k, c->adjXU[sU - 1], ac.maxVel, clampU);
    k_adj_clampmask<false><<<nb, kThreads, 0, c->stream>>>(k, c->adjXV[sV - 1], ac.maxVel, clampV);
    CK(cudaGetLastError());
    AdjSweep UsA{Us.aP, Us.aE, Us.aW, Us.aN, Us.aS, clampU, A[20], A[21], A[22], A[23], A[24], A[25]};
    AdjSweep VsA{Vs.aP, Vs.aE, Vs.aW, Vs.aN, Vs.aS, clampV, A[26], A[27], A[28], A[29], A[30], A[31]};
    // which model: the fixed point of the frozen iteration where the state is
    // one (every unclamped sweep result equals the state to 1e-7 maxVel) and
    // velocities sit on the clamp; the equations R = 0 otherwise (exact
    // without clamped velocities, and the only meaningful linearisation away
    // from a fixed point)
    int nClamped = 0;
    double fpRes = 0.0;
    {
        k_adj_fixedpoint<<<nb, kThreads, 0, c->stream>>>(k, c->adjXU[sU - 1], c->u, clampU, c->adjXV[sV - 1], c->v,
                                                          clampV, c->adjPart);
        CK(cudaGetLastError());
        std::vector<double> pf((size_t)2 * nb);
        CK(cudaMemcpyAsync(pf.data(), c->adjPart, pf.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        double cnt = 0.0;
        for (int b = 0; b < nb; ++b) { cnt += pf[2 * b]; fpRes = std::max(fpRes, pf[2 * b + 1]); }
        nClamped = (int)cnt;
    }
    int model = c->prm.adjointModel;
    if (model != CP_ADJ_EQUATIONS && model != CP_ADJ_FIXED_POINT)
        model = (nClamped > 0 && fpRes <= 1e-7 * ac.maxVel) ? CP_ADJ_FIXED_POINT : CP_ADJ_EQUATIONS;
    const bool fixedPoint = model == CP_ADJ_FIXED_POINT;
    if (fixedPoint) {
        k_adj_prec_faces<<<nb, kThreads, 0, c->stream>>>(k, c->dE, c->dN, UsA, VsA, dEp, dNp);
        CK(cudaGetLastError());
    }
    // right-hand side dJ/dX and J
    k_adj_g<<<1, 1024, 0, c->stream>>>(ac, V, Jd);
    CK(cudaGetLastError());
    // pressure-like solves: fixed iteration count, no early stop
    KParams kp = k;
    kp.pTol = 0.0;
    kp.maxP = c->adjPIters;
    const int m = c->adjRestart;
    const size_t L = 3 * c->nElem;
    double* kry = c->adjKry;
    auto Vq = [&](int q) { return kry + (size_t)q * L; };             // q = 0..m
    auto Zq = [&](int q) { return kry + (size_t)(m + 1 + q) * L; };   // q = 0..m-1
    double* W = kry + (size_t)(2 * m + 1) * L;
    double* LAM = kry + (size_t)(2 * m + 2) * L;
    CK(cudaMemsetAsync(kry, 0, (size_t)(2 * m + 3) * L * sizeof(double), c->stream));
    V.lu = LAM; V.lv = LAM + c->nElem; V.lc = LAM + 2 * c->nElem;
    std::vector<double> part((size_t)2 * nb);

    // the reverse sweeps of both components for the adjoint vector x: the
    // adjoints of r0 and of the coefficients into UsA / VsA
    auto reverse = [&](const double* x) -> cp_status {
        for (int q = 20; q < 32; ++q) CK(cudaMemsetAsync(A[q], 0, bytes, c->stream));
        const double* yu = x;
        const double* yv = x + c->nElem;
        int pu = 0, pv = 0;
        for (int j = std::max(sU, sV) - 1; j >= 0; --j) {
            const int doU = j < sU, doV = j < sV;
            const double* xUj = j == 0 ? c->u : c->adjXU[j - 1];
            const double* xVj = j == 0 ? c->v : c->adjXV[j - 1];
            const double* xUj1 = c->adjXU[std::min(j, sU - 1)];
            const double* xVj1 = c->adjXV[std::min(j, sV - 1)];
            k_adj_rev<<<nb, kThreads, 0, c->stream>>>(k, UsA, VsA, c->u, c->v, xUj, xUj1, xVj, xVj1, yu, yv,
                                                      ybU[pu], ybV[pv], doU, doV, j == sU - 1, j == sV - 1);
            CK(cudaGetLastError());
            if (doU) { yu = ybU[pu]; pu ^= 1; }
            if (doV) { yv = ybV[pv]; pv ^= 1; }
        }
        return CP_OK;
    };
    // y = J^T x (x a Krylov vector); out = gs g - ys y on the unknowns; returns
    // (|out|^2, |g|^2) through the block partials
    auto product = [&](const double* x, double gs, double ys, double* out, double* rr, double* gg) -> cp_status {
        AdjVecs Vx = V;
        Vx.lu = const_cast<double*>(x); Vx.lv = Vx.lu + c->nElem; Vx.lc = Vx.lu + 2 * c->nElem;
        if (fixedPoint) {
            cp_status s1 = reverse(x);
            if (s1 != CP_OK) return s1;
        }
        for (double* y : {V.yu, V.yv, V.yp}) CK(cudaMemsetAsync(y, 0, bytes, c->stream));
        if (fixedPoint) k_adj_jt<<<nb, kThreads, 0, c->stream>>>(ac, Vx, UsA, VsA);
        else k_adj_jt_eq<<<nb, kThreads, 0, c->stream>>>(ac, Vx, nullptr, nullptr, nullptr);
        CK(cudaGetLastError());
        k_adj_defect<<<nb, kThreads, 0, c->stream>>>(k, V, gs, ys, out, out + c->nElem, out + 2 * c->nElem,
                                                     c->adjPart);
        CK(cudaGetLastError());
        if (rr) {
            CK(cudaMemcpyAsync(part.data(), c->adjPart, part.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream));
            CK(cudaStreamSynchronize(c->stream));
            double a0 = 0.0, a1 = 0.0;
            for (int b = 0; b < nb; ++b) { a0 += part[2 * b]; a1 += part[2 * b + 1]; }
            *rr = a0;
            if (gg) *gg = a1;
        }
        return CP_OK;
    };
    // z = P^-1 r: the momentum part, then the pressure-like correction
    // the equations model: Jacobi sweeps on the transposed Picard momentum
    // system, then the pressure-like correction with the forward matrix
    auto precondition_eq = [&](const double* r, double* z) -> cp_status {
        const double *ru = r, *rv = r + c->nElem, *rp = r + 2 * c->nElem;
        double *xu = V.du, *xv = V.dv;
        double *yu = V.eu, *yv = V.ev;
        for (int q = 0; q < c->adjSweeps; ++q) {
            k_adj_jacobi_t<<<nb, kThreads, 0, c->stream>>>(k, Us, Vs, ru, rv, xu, xv, yu, yv, q == 0);
            CK(cudaGetLastError());
            std::swap(xu, yu);
            std::swap(xv, yv);
        }
        cp_status s2 = c->prm.precision == CP_PREC_MIXED ? adjoint_prhs<float>(c, kp, xu, xv, rp)
                                                         : adjoint_prhs<double>(c, kp, xu, xv, rp);
        if (s2 != CP_OK) return s2;
        CK(cudaMemsetAsync(c->adjSt, 0, sizeof(Status), c->stream));
        s2 = c->prm.precision == CP_PREC_MIXED ? adjoint_pcg<float>(c, kp, c->dE, c->dN, dc)
                                               : adjoint_pcg<double>(c, kp, c->dE, c->dN, dc);
        if (s2 != CP_OK) return s2;
        k_adj_update_eq<<<nb, kThreads, 0, c->stream>>>(k, xu, xv, dc, c->dE, c->dN, c->prm.pAlpha, z,
                                                        z + c->nElem, z + 2 * c->nElem);
        CK(cudaGetLastError());
        return CP_OK;
    };
    auto precondition = [&](const double* r, double* z) -> cp_status {
        if (!fixedPoint) return precondition_eq(r, z);
        const double *ru = r, *rv = r + c->nElem, *rp = r + 2 * c->nElem;
        k_adj_prec_mom<<<nb, kThreads, 0, c->stream>>>(k, ru, rv, UsA, VsA, V.du, V.dv, V.eu, V.ev);
        CK(cudaGetLastError());
        cp_status s2 = c->prm.precision == CP_PREC_MIXED ? adjoint_prhs<float>(c, kp, V.eu, V.ev, rp)
                                                         : adjoint_prhs<double>(c, kp, V.eu, V.ev, rp);
        if (s2 != CP_OK) return s2;
        CK(cudaMemsetAsync(c->adjSt, 0, sizeof(Status), c->stream));
        s2 = c->prm.precision == CP_PREC_MIXED ? adjoint_pcg<float>(c, kp, dEp, dNp, dc)
                                               : adjoint_pcg<double>(c, kp, dEp, dNp, dc);
        if (s2 != CP_OK) return s2;
        k_adj_update<<<nb, kThreads, 0, c->stream>>>(k, V.du, V.dv, dc, UsA, VsA, z, z + c->nElem, z + 2 * c->nElem);
        CK(cudaGetLastError());
        return CP_OK;
    };
    // h[0..nv) = <w, B_0..B_nv-1> into dst (device)
    auto mdot = [&](const double* w, const double* B, int nv, double* dst) -> cp_status {
        k_kry_mdot<<<nb, 256, 0, c->stream>>>(w, B, L, nv, c->adjKryPart);
        CK(cudaGetLastError());
        k_kry_sum<<<1, 1024, 0, c->stream>>>(c->adjKryPart, nb, nv, dst);
        CK(cudaGetLastError());
        return CP_OK;
    };

    if (info) {
        info[0] = model;
        info[1] = sU;
        info[2] = sV;
        info[3] = c->d.P;
    }
    if (probeOp == 0 || probeOp == 1) {
        // y = J^T x (x copied into the work vector W) or y = dJ/dX (x = 0)
        CK(cudaMemsetAsync(W, 0, L * sizeof(double), c->stream));
        if (probeOp == 0) CK(cudaMemcpyAsync(W, px, L * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if ((s = product(W, probeOp == 1 ? 1.0 : 0.0, probeOp == 1 ? 0.0 : -1.0, Vq(0), nullptr, nullptr)) != CP_OK)
            return s;
        CK(cudaMemcpyAsync(py, Vq(0), L * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return CP_OK;
    }
    double res = 1.0, gnorm = 0.0, rr = 0.0, gg = 0.0;
    int it = 0;
    bool conv = false;
    std::vector<double> H((size_t)(m + 1) * m), gc(m), gs(m), gv(m + 1), y(m), hh(3 * kKryMaxDots);
    auto Hij = [&](int i, int j) -> double& { return H[(size_t)i * m + j]; };
    // initial residual: lambda = 0, r0 = g
    if ((s = product(LAM, 1.0, 1.0, Vq(0), &rr, &gg)) != CP_OK) return s;
    gnorm = std::sqrt(gg);
    double beta = std::sqrt(rr);
    res = gnorm > 0.0 ? beta / gnorm : 0.0;
    while (true) {
        if (!std::isfinite(res)) return fail(CP_ERR_NONFINITE, "adjoint residual is not finite at iteration %d", it);
        if (res <= tol) { conv = true; break; }
        if (it >= max_iter) break;
        // restart cycle: V_0 = r / beta
        k_kry_scale<<<nb, kThreads, 0, c->stream>>>(Vq(0), Vq(0), L, 1.0 / beta);
        CK(cudaGetLastError());
        std::fill(gv.begin(), gv.end(), 0.0);
        gv[0] = beta;
        int jn = 0;
        for (int j = 0; j < m && it < max_iter; ++j) {
            if ((s = precondition(Vq(j), Zq(j))) != CP_OK) return s;
            if ((s = product(Zq(j), 0.0, -1.0, W, nullptr, nullptr)) != CP_OK) return s;
            // classical Gram-Schmidt, twice
            double* h1 = c->adjH;
            double* h2 = c->adjH + kKryMaxDots;
            double* nr = c->adjH + 2 * kKryMaxDots;
            // (each projection fused with the dot products that follow it)
            if ((s = mdot(W, Vq(0), j + 1, h1)) != CP_OK) return s;
            k_kry_axpy_mdot<<<nb, 256, 0, c->stream>>>(W, Vq(0), L, j + 1, h1, -1.0, j + 1, 0, c->adjKryPart);
            CK(cudaGetLastError());
            k_kry_sum<<<1, 1024, 0, c->stream>>>(c->adjKryPart, nb, j + 1, h2);
            CK(cudaGetLastError());
            k_kry_axpy_mdot<<<nb, 256, 0, c->stream>>>(W, Vq(0), L, j + 1, h2, -1.0, 1, 1, c->adjKryPart);
            CK(cudaGetLastError());
            k_kry_sum<<<1, 1024, 0, c->stream>>>(c->adjKryPart, nb, 1, nr);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(hh.data(), c->adjH, hh.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            for (int i = 0; i <= j; ++i) Hij(i, j) = hh[i] + hh[kKryMaxDots + i];
            const double hn = std::sqrt(std::max(hh[2 * kKryMaxDots], 0.0));
            Hij(j + 1, j) = hn;
            if (!std::isfinite(hn)) return fail(CP_ERR_NONFINITE, "adjoint Krylov basis is not finite");
            if (hn > 0.0) {
                k_kry_scale<<<nb, kThreads, 0, c->stream>>>(Vq(j + 1), W, L, 1.0 / hn);
                CK(cudaGetLastError());
            }
            // Givens rotations of the new column; the residual estimate is |gv[j+1]|
            for (int i = 0; i < j; ++i) {
                const double a0 = Hij(i, j), a1 = Hij(i + 1, j);
                Hij(i, j) = gc[i] * a0 + gs[i] * a1;
                Hij(i + 1, j) = -gs[i] * a0 + gc[i] * a1;
            }
            const double a0 = Hij(j, j), a1 = Hij(j + 1, j);
            const double rnorm = std::hypot(a0, a1);
            gc[j] = rnorm > 0.0 ? a0 / rnorm : 1.0;
            gs[j] = rnorm > 0.0 ? a1 / rnorm : 0.0;
            Hij(j, j) = rnorm;
            Hij(j + 1, j) = 0.0;
            gv[j + 1] = -gs[j] * gv[j];
            gv[j] = gc[j] * gv[j];
            ++it;
            jn = j + 1;
            const double est = gnorm > 0.0 ? std::fabs(gv[j + 1]) / gnorm : 0.0;
            if (est <= tol || hn == 0.0) break;
        }
        // y = R^-1 g; lambda += Z y
        for (int i = jn - 1; i >= 0; --i) {
            double a = gv[i];
            for (int q = i + 1; q < jn; ++q) a -= Hij(i, q) * y[q];
            y[i] = Hij(i, i) != 0.0 ? a / Hij(i, i) : 0.0;
        }
        CK(cudaMemcpyAsync(c->adjH, y.data(), jn * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        k_kry_axpy<<<nb, 256, 0, c->stream>>>(LAM, Zq(0), L, jn, c->adjH, 1.0);
        CK(cudaGetLastError());
        // true residual for the stop test and the next cycle
        if ((s = product(LAM, 1.0, 1.0, Vq(0), &rr, nullptr)) != CP_OK) return s;
        beta = std::sqrt(rr);
        res = gnorm > 0.0 ? beta / gnorm : 0.0;
    }
    if (probeOp == 2) {
        CK(cudaMemcpyAsync(py, LAM, L * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (rep) {
            rep->iterations = it;
            rep->converged = conv ? 1 : 0;
            rep->residual = res;
            rep->model = model;
            rep->clampedUnknowns = nClamped;
        }
        return CP_OK;
    }
    // gradient on the Ny x Nx cells (fixed point: from the reverse sweeps of
    // lambda)
    double* gd = A[18];
    const double amax = c->prm.eta / std::max(c->prm.brinkmanKMin, 1e-20);
    if (fixedPoint) {
        if ((s = reverse(LAM)) != CP_OK) return s;
        k_adj_grad<<<nb, kThreads, 0, c->stream>>>(ac, UsA, VsA, amax, c->prm.brinkmanQ, gd);
    } else {
        k_adj_grad_eq<<<nb, kThreads, 0, c->stream>>>(ac, V, amax, c->prm.brinkmanQ, gd);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, c->stream));
    std::vector<double> g((size_t)(M - 1) * (N - 1));
    double Jh = 0.0;
    CK(cudaMemcpyAsync(g.data(), gd, g.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&Jh, Jd, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    Status hs;
    CK(cudaMemcpy(&hs, c->adjSt, sizeof(Status), cudaMemcpyDeviceToHost));
    if (hs.err) return fail((cp_status)hs.err, "device reported %s in the adjoint", cp_status_string((cp_status)hs.err));
    for (long i = 0; i < rows; ++i)
        for (long j = 0; j < cols; ++j) grad[i * rs + j * cs] = g[(size_t)i * (N - 1) + j];
    if (rep) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        rep->iterations = it;
        rep->converged = conv ? 1 : 0;
        rep->residual = res;
        rep->J = Jh;
        rep->device_ms = ms;
        rep->model = model;
        rep->clampedUnknowns = nClamped;
    }
    return CP_OK;
}

extern "C" cp_status cp_adjoint_dp_dgamma(cp_ctx* c, double* grad, long rows, long cols, long rs, long cs,
                                          int max_iter, double tol, cp_adjoint_report* rep) {
    if (!c || !grad) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    const int M = c->d.M, N = c->d.N;
    if (rows != M - 1 || cols != N - 1) return fail(CP_ERR_BAD_PARAM, "grad shape %ld x %ld, expected %d x %d",
                                                    rows, cols, M - 1, N - 1);
    if (max_iter < 1 || !(tol > 0.0)) return fail(CP_ERR_BAD_PARAM, "max_iter >= 1 and tol > 0 required");
    return adjoint_impl(c, grad, rows, cols, rs, cs, max_iter, tol, rep, -1, nullptr, nullptr, nullptr);
}

extern "C" size_t cp_adjoint_probe_len(const cp_ctx* c) { return c ? 3 * c->nElem : 0; }

extern "C" cp_status cp_adjoint_probe(cp_ctx* c, int op, const double* x, double* y, int max_iter, double tol,
                                      int* info, cp_adjoint_report* rep) {
    if (!c || !y || !info) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    if (op < 0 || op > 2) return fail(CP_ERR_BAD_PARAM, "probe op %d (0, 1 or 2)", op);
    if (op == 0 && !x) return fail(CP_ERR_BAD_PARAM, "probe op 0 needs x");
    if (op == 2 && (max_iter < 1 || !(tol > 0.0))) return fail(CP_ERR_BAD_PARAM, "max_iter >= 1 and tol > 0 required");
    return adjoint_impl(c, nullptr, c->d.M - 1, c->d.N - 1, 0, 0, max_iter, tol, rep, op, x, y, info);
}

// ======================================================================== no-allocation entry point
// cp_pressure_noalloc: the Jacobi-PCG pressure-correction solve (k_mass +
// k_pcg<double>, the kernels behind cp_pressure for pressureSolverType 1)
// for callers that cannot allocate device memory.  All of its working
// memory lives in one file-scope device array of fixed size, below; the
// caller provides only the inputs and the output.
namespace {

// Largest pressure grid the array serves: (Ny + 3) * pitch elements per
// working array, where pitch is the row pitch (in doubles) the caller uses.
constexpr size_t kNoAllocCells = 131072;
constexpr size_t kNoAllocArrays = 9;                  // fE fN d x r pa pb Ap rhs
constexpr size_t kNoAllocHead = 256 + 256 + 8 * 4 * kMaxBlocks + 8 * 3 * kMaxBlocks;
constexpr size_t kNoAllocBytes = kNoAllocHead + kNoAllocArrays * 8 * kNoAllocCells;

// Every GPU that loads the library holds these bytes until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};
void* g_noalloc_ctx[kNoAllocMaxDevices] = {};   // the context the cached address belongs to

// cuCtxGetCurrent through the runtime's driver entry point (no libcuda link)
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

cp_status current_context(void** ctx) {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !f)
            return fail(CP_ERR_CUDA, "cuCtxGetCurrent is not available");
        fn = reinterpret_cast<CtxGetCurrentFn>(f);
    }
    CUcontext c = nullptr;
    if (fn(&c) != CUDA_SUCCESS) return fail(CP_ERR_CUDA, "cuCtxGetCurrent failed");
    *ctx = c;
    return CP_OK;
}

// Device address of the array for the current device.  It is looked up
// (with that device current) on the first call and again whenever the
// device's context has changed since, e.g. after cudaDeviceReset, which
// unloads the module and may place the array elsewhere.
cp_status noalloc_scratch(unsigned char** out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(CP_ERR_CUDA, "device ordinal %d out of range", dev);
    void* ctx = nullptr;
    cp_status st = current_context(&ctx);
    if (st != CP_OK) return st;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!ctx || !g_noalloc_ptr[dev] || g_noalloc_ctx[dev] != ctx) {
        // the lookup also creates the device's primary context if none is current
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        if ((st = current_context(&ctx)) != CP_OK) return st;
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
        g_noalloc_ctx[dev] = ctx;
    }
    *out = g_noalloc_ptr[dev];
    return CP_OK;
}

// max |mass imbalance| of the k_mass partials into st->lastError
__global__ void k_noalloc_massmax(const double* partM, int nb, Status* st) {
    double m = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) m = dmax(m, partM[b * 4 + 3]);
    m = warp_max(m);
    __shared__ double sm[32];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int q = 0; q < (int)((blockDim.x + 31) >> 5); ++q) r = dmax(r, sm[q]);
        st->lastError = r;
    }
}

}  // namespace

extern "C" cp_status cp_pressure_noalloc(const cp_params* p, const double* dE, const double* dN,
                                         const double* uStar, const double* vStar, long pitch, double* pStar,
                                         int* iters, double* residMass, void* stream) {
    if (!p || !dE || !dN || !uStar || !vStar || !pStar) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    if (p->Ny < 2 || p->Nx < 3) return fail(CP_ERR_BAD_PARAM, "grid %d x %d too small", p->Ny, p->Nx);
    if (p->pressureSolverType != 1)
        return fail(CP_ERR_UNSUPPORTED, "cp_pressure_noalloc runs the Jacobi-PCG (pressureSolverType 1) only");
    if (!(p->rho > 0.0) || !(p->hx > 0.0) || !(p->hy > 0.0) || !std::isfinite(p->pTol) || p->maxPressureIter < 0)
        return fail(CP_ERR_BAD_PARAM, "rho, hx, hy must be > 0, pTol finite, maxPressureIter >= 0");
    const int M = p->Ny + 1, N = p->Nx + 1;
    if (pitch < N + 1) return fail(CP_ERR_BAD_PARAM, "pitch %ld < Nx + 2 = %d", pitch, N + 1);
    const size_t cells = (size_t)(M + 2) * (size_t)pitch;
    if (cells > kNoAllocCells)
        return fail(CP_ERR_BAD_PARAM,
                    "grid too large for cp_pressure_noalloc: (Ny + 3) * pitch = %zu exceeds %zu; use cp_pressure",
                    cells, kNoAllocCells);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    cp_status st = noalloc_scratch(&base);
    if (st != CP_OK) return st;
    int dev = 0, sms = 0, nbP = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbP, k_pcg<double>, kThreads, 0));
    if (nbP < 1) return fail(CP_ERR_CUDA, "PCG kernel does not fit on an SM");
    const int gPcg = sms * std::min(nbP, 4), nbMass = sms * 4;
    if (gPcg > kMaxBlocks || nbMass > kMaxBlocks) return fail(CP_ERR_CUDA, "too many SMs");
    // carve the array: status, barrier counter, partial sums, nine working arrays
    Status* dst = reinterpret_cast<Status*>(base);
    unsigned* bar = reinterpret_cast<unsigned*>(base + 256);
    double* partM = reinterpret_cast<double*>(base + 512);
    double* partP = partM + 4 * kMaxBlocks;
    double* arr = reinterpret_cast<double*>(base + kNoAllocHead);
    PcgBufs<double> B;
    double* a[kNoAllocArrays];
    for (size_t q = 0; q < kNoAllocArrays; ++q) a[q] = arr + q * cells;
    B.fE = a[0]; B.fN = a[1]; B.d = a[2]; B.x = a[3]; B.r = a[4]; B.pa = a[5]; B.pb = a[6]; B.Ap = a[7];
    B.rhs = a[8];
    // the array keeps the previous call's contents: clear everything this
    // call relies on being zero (status, counter, partials, the frames of
    // the working arrays), and the output like the reference's pStar.setZero()
    CK(cudaMemsetAsync(base, 0, kNoAllocHead + kNoAllocArrays * 8 * cells, s));
    CK(cudaMemset2DAsync(pStar, (size_t)pitch * 8, 0, (size_t)(N + 1) * 8, (size_t)(M + 1), s));
    KParams k{};
    k.d.M = M; k.d.N = N; k.d.P = (int)pitch;
    k.hx = p->hx; k.hy = p->hy; k.rho = p->rho;
    k.pTol = p->pTol; k.maxP = p->maxPressureIter;
    k.nU = (M - 1) * (N - 2); k.nV = (M - 2) * (N - 1); k.nP = (M - 1) * (N - 2);
    // the RMS columns of k_mass are not reported here; u*/v* stand in for u/v
    k_mass<double><<<nbMass, kThreads, 0, s>>>(k, dst, uStar, vStar, uStar, vStar, B.rhs, partM);
    CK(cudaGetLastError());
    CK(launch_coop(k_pcg<double>, gPcg, s, k, dst, dE, dN, B, pStar, partP, bar));
    k_noalloc_massmax<<<1, 256, 0, s>>>(partM, nbMass, dst);
    CK(cudaGetLastError());
    Status hs;
    CK(cudaMemcpyAsync(&hs, dst, sizeof(Status), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (hs.err != 0) return fail((cp_status)hs.err, "device reported %s", cp_status_string((cp_status)hs.err));
    if (iters) *iters = hs.itersP;
    if (residMass) *residMass = hs.lastError;
    return CP_OK;
}

// ======================================================================== bounded-wait self-test
// The persistent kernels wait on grid barriers and the TMA pipelines on
// mbarriers; every such wait gives up after a time limit and records
// CP_ERR_TIMEOUT in the status word, so a wait that cannot end returns an
// error instead of holding the GPU.  This self-test runs each kind of wait
// on something that never happens (a second block that does not exist, an
// mbarrier phase nobody arrives on) with a short limit, so that the give-up
// path is exercised without any fault.
namespace {

__global__ void k_selftest_wait(int kind, unsigned long long limitNs, unsigned* counter, int* err) {
    if (kind == 0) {
        // one block waits for two arrivals
        grid_barrier(counter, 2u, err, limitNs);
    } else {
        __shared__ __align__(8) uint64_t bar;
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (threadIdx.x == 0) mbar_wait(&bar, 0u, err, limitNs);   // phase 0 never completes
        __syncthreads();
    }
}

}  // namespace

extern "C" cp_status cp_selftest_bounded_wait(int kind, double limit_seconds, int* device_status) {
    if (kind != 0 && kind != 1) return fail(CP_ERR_BAD_PARAM, "kind must be 0 (grid barrier) or 1 (mbarrier)");
    if (!(limit_seconds > 0.0) || limit_seconds > 10.0) return fail(CP_ERR_BAD_PARAM, "limit must be in (0, 10] s");
    if (!device_status) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    void* buf = nullptr;
    CK(cudaMalloc(&buf, 256));
    struct Free { void* p; ~Free() { cudaFree(p); } } guard{buf};
    CK(cudaMemset(buf, 0, 256));
    unsigned* counter = static_cast<unsigned*>(buf);
    int* err = reinterpret_cast<int*>(static_cast<char*>(buf) + 128);
    k_selftest_wait<<<1, 32>>>(kind, (unsigned long long)(limit_seconds * 1e9), counter, err);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(device_status, err, sizeof(int), cudaMemcpyDeviceToHost));
    return CP_OK;
}

// ======================================================================== batched solves
// cp_batch: the fields of several contexts advanced by one persistent
// cooperative kernel (k_batch).  The batch keeps only the per-field
// descriptors, the tile tables and the scratch of the shared reductions;
// every field's buffers stay in its own context.
struct cp_batch {
    std::vector<cp_ctx*> f;
    int dev = 0, numSMs = 0, grid = 0;
    bool mixed = false;
    int R = 16, C = 64;
    int maxLg = 1, maxMom = 0, maxP = 0;
    size_t partCap = 0;          // tiles of level 0 the partial array holds
    void* dF = nullptr;          // BField<TC>[n]
    int* dToff = nullptr;
    BState* dBs = nullptr;
    double* dPart = nullptr;
    unsigned* dBar = nullptr;
    int* dErr = nullptr;
    int* dAllDone = nullptr;
    unsigned long long* dProf = nullptr;   // per-phase timers when CP_BATCH_PROFILE is set
    // team mode (every field runs smoothed aggregation): k_batch_team
    bool teamMode = false;
    int team = 4, nTeams = 0;    // CTAs per team, teams
    size_t teamSmem = 0;         // dynamic shared memory (the largest field's k_pcg_sa staging)
    int* dOrder = nullptr;       // queue order, largest field first
    unsigned* dTbar = nullptr;   // [grid * kTeamStride] team barrier counters
    int* dQueue = nullptr;       // [1 + 2 grid]
    int* dRunning = nullptr;     // fields still running after a launch
    int* hFlags = nullptr;       // pinned: allDone (team mode: fields running), err
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graphOuter = 0;
    std::vector<void*> allocs;
};

namespace {

constexpr int kBatchChunk = 64;   // outer iterations per launch
// tile shapes the autotuner tries (rows x columns)
constexpr int kBatchTiles[][2] = {{16, 64}, {8, 128}, {32, 32}, {4, 256}, {8, 64}, {16, 32},
                                  {16, 128}, {32, 64}, {8, 256}};
constexpr size_t kBatchDynSmem = kMgDenseSmem;
// team sizes the autotuner tries in team mode (CTAs per team)
constexpr int kBatchTeams[] = {2, 3, 4, 6, 8, 12, 16};
constexpr int kBatchTeamDefault = 4;

size_t batch_tiles0(const cp_batch* b, int R, int C) {
    size_t t = 0;
    for (cp_ctx* c : b->f)
        t += (size_t)((c->d.M - 1 + R - 1) / R) * (size_t)((c->d.N - 1 + C - 1) / C);
    return t;
}

// first tile of every field per level: level 0 tiles the (M-1) x (N-1)
// cells, level l >= 1 its nI x nJ unknowns where the field runs level l
// grid-wide or restricts into it (l <= Lg)
std::vector<int> batch_toff(const cp_batch* b, int R, int C) {
    const int n = (int)b->f.size();
    std::vector<int> t((size_t)(b->maxLg + 1) * (n + 1), 0);
    for (int l = 0; l <= b->maxLg; ++l) {
        int acc = 0;
        for (int q = 0; q < n; ++q) {
            const cp_ctx* c = b->f[q];
            t[(size_t)l * (n + 1) + q] = acc;
            int nI = 0, nJ = 0;
            if (l == 0) { nI = c->d.M - 1; nJ = c->d.N - 1; }
            else if (l <= c->mgLg && l < c->mgL) { nI = c->mgNI[l]; nJ = c->mgNJ[l]; }
            acc += ((nI + R - 1) / R) * ((nJ + C - 1) / C);
        }
        t[(size_t)l * (n + 1) + n] = acc;
    }
    return t;
}

template <typename TC>
BField<TC> batch_field(cp_ctx* c) {
    BField<TC> bf;
    memset(&bf, 0, sizeof(bf));
    bf.k = c->k;
    bf.st = c->st;
    bf.u = c->u; bf.v = c->v; bf.p = c->p; bf.uStar = c->uStar; bf.vStar = c->vStar; bf.pStar = c->pStar;
    bf.dE = c->dE; bf.dN = c->dN; bf.alpha = c->alpha; bf.gamma = c->gamma;
    bf.U = mom_sys<TC>(c, 0);
    bf.V = mom_sys<TC>(c, 1);
    bf.xU0 = (TC*)c->xb[0]; bf.xU1 = (TC*)c->xb[1]; bf.xV0 = (TC*)c->xb[2]; bf.xV1 = (TC*)c->xb[3];
    bf.B = pcg_bufs<TC>(c);
    bf.H = mg_hier<TC>(c);
    bf.H.prof = nullptr;
    bf.hist = c->hist; bf.histCap = c->histCap; bf.dpWin = c->dpWin;
    return bf;
}

template <typename TC>
BFieldSa<TC> batch_field_sa(cp_ctx* c) {
    BFieldSa<TC> bf;
    memset(&bf, 0, sizeof(bf));
    bf.k = c->k;
    bf.st = c->st;
    bf.u = c->u; bf.v = c->v; bf.p = c->p; bf.uStar = c->uStar; bf.vStar = c->vStar; bf.pStar = c->pStar;
    bf.dE = c->dE; bf.dN = c->dN; bf.alpha = c->alpha; bf.gamma = c->gamma;
    bf.U = mom_sys<TC>(c, 0);
    bf.V = mom_sys<TC>(c, 1);
    bf.xU0 = (TC*)c->xb[0]; bf.xU1 = (TC*)c->xb[1]; bf.xV0 = (TC*)c->xb[2]; bf.xV1 = (TC*)c->xb[3];
    bf.B = pcg_bufs<TC>(c);
    bf.H = sa_hier<TC>(c);
    bf.H.prof = nullptr;
    bf.partJ = c->partJ; bf.partM = c->partM; bf.partP = c->partP;
    bf.hist = c->hist; bf.histCap = c->histCap; bf.dpWin = c->dpWin;
    return bf;
}

cp_status batch_set_team(cp_batch* b, int ctas) {
    if (ctas < 1 || ctas > b->grid) return fail(CP_ERR_BAD_PARAM, "team of %d CTAs (1..%d)", ctas, b->grid);
    b->team = ctas;
    b->nTeams = b->grid / ctas;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    return CP_OK;
}

template <typename TC, bool Mixed>
cp_status batch_launch_team(cp_batch* b, int nOuter) {
    TeamArgs a{};
    a.nf = (int)b->f.size();
    a.team = b->team;
    a.nTeams = b->nTeams;
    a.nOuter = nOuter;
    a.order = b->dOrder;
    a.tbar = b->dTbar;
    a.queue = b->dQueue;
    a.err = b->dErr;
    a.running = b->dRunning;
    CK(cudaMemsetAsync(b->dTbar, 0, (size_t)b->grid * kTeamStride * sizeof(unsigned), b->stream));
    CK(cudaMemsetAsync(b->dQueue, 0, (size_t)(1 + 2 * b->grid) * sizeof(int), b->stream));
    CK(cudaMemsetAsync(b->dRunning, 0, sizeof(int), b->stream));
    CK(launch_coop_cfg(k_batch_team<TC, Mixed>, b->grid, kBatchThreads, b->teamSmem, b->stream, a,
                       (const BFieldSa<TC>*)b->dF));
    return CP_OK;
}

cp_status batch_balloc(cp_batch* b, void** p, size_t bytes) {
    CK(cudaMalloc(p, std::max<size_t>(bytes, 1)));
    b->allocs.push_back(*p);
    CK(cudaMemsetAsync(*p, 0, std::max<size_t>(bytes, 1), b->stream));
    return CP_OK;
}

cp_status batch_set_tile(cp_batch* b, int R, int C) {
    if (R < 1 || C < 1 || R * C < 256 || R * C > 4096)
        return fail(CP_ERR_BAD_PARAM, "tile %d x %d: rows x cols must lie in [256, 4096]", R, C);
    if (batch_tiles0(b, R, C) > b->partCap)
        return fail(CP_ERR_BAD_PARAM, "tile %d x %d: more tiles than the batch was sized for", R, C);
    std::vector<int> t = batch_toff(b, R, C);
    CK(cudaMemcpyAsync(b->dToff, t.data(), t.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    b->R = R;
    b->C = C;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    return CP_OK;
}

template <typename TC, bool Mixed>
cp_status batch_launch(cp_batch* b, int nOuter) {
    BatchArgs a{};
    a.nf = (int)b->f.size();
    a.R = b->R; a.C = b->C;
    a.maxLg = b->maxLg; a.maxMom = b->maxMom; a.maxP = b->maxP;
    a.nOuter = nOuter;
    a.toff = b->dToff; a.bs = b->dBs; a.ipart = b->dPart; a.bar = b->dBar; a.err = b->dErr;
    a.allDone = b->dAllDone;
    a.prof = b->dProf;
    CK(cudaMemsetAsync(b->dBar, 0, sizeof(unsigned), b->stream));
    CK(launch_coop_cfg(k_batch<TC, Mixed>, b->grid, kBatchThreads, kBatchDynSmem, b->stream, a,
                       (const BField<TC>*)b->dF));
    return CP_OK;
}

cp_status batch_launch_any(cp_batch* b, int nOuter) {
    if (b->teamMode)
        return b->mixed ? batch_launch_team<float, true>(b, nOuter) : batch_launch_team<double, false>(b, nOuter);
    return b->mixed ? batch_launch<float, true>(b, nOuter) : batch_launch<double, false>(b, nOuter);
}

// one graph of [barrier reset, k_batch(nOuter)], replayed per chunk
cp_status batch_graph(cp_batch* b, int nOuter) {
    if (b->graph && b->graphOuter == nOuter) return CP_OK;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return CP_OK;
    }
    cp_status s = batch_launch_any(b, nOuter);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (s != CP_OK || e != cudaSuccess || !g) {
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        g_err.clear();
        return CP_OK;   // launched directly instead
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return CP_OK;
    }
    b->graph = ex;
    b->graphOuter = nOuter;
    return CP_OK;
}

template <typename TC>
cp_status batch_upload_fields(cp_batch* b) {
    if (b->teamMode) {
        std::vector<BFieldSa<TC>> h;
        for (cp_ctx* c : b->f) h.push_back(batch_field_sa<TC>(c));
        CK(cudaMemcpyAsync(b->dF, h.data(), h.size() * sizeof(BFieldSa<TC>), cudaMemcpyHostToDevice, b->stream));
        // queue order: largest field first (cells), so the last fields a team
        // takes are the short ones
        std::vector<int> order(b->f.size());
        for (size_t q = 0; q < order.size(); ++q) order[q] = (int)q;
        auto cells = [&](int q) { return (long long)(b->f[q]->d.M - 1) * (b->f[q]->d.N - 1); };
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cells(x) > cells(y); });
        CK(cudaMemcpyAsync(b->dOrder, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    } else {
        std::vector<BField<TC>> h;
        for (cp_ctx* c : b->f) h.push_back(batch_field<TC>(c));
        CK(cudaMemcpyAsync(b->dF, h.data(), h.size() * sizeof(BField<TC>), cudaMemcpyHostToDevice, b->stream));
    }
    CK(cudaStreamSynchronize(b->stream));
    return CP_OK;
}

cp_status batch_sync_fields(cp_batch* b) {
    for (cp_ctx* c : b->f) CK(cudaStreamSynchronize(c->stream));
    return CP_OK;
}

// run up to max_outer outer iterations (every field stops on its own rules
// before that); rep gets the totals
cp_status batch_run(cp_batch* b, int max_outer, cp_batch_report* rep, bool useGraph) {
    cp_status s = batch_sync_fields(b);
    if (s != CP_OK) return s;
    CK(cudaMemsetAsync(b->dErr, 0, sizeof(int), b->stream));
    CK(cudaMemsetAsync(b->dAllDone, 0, sizeof(int), b->stream));
    CK(cudaEventRecord(b->ev0, b->stream));
    int done = 0, launches = 0;
    bool all = false;
    while (done < max_outer && !all) {
        const int n = std::min(kBatchChunk, max_outer - done);
        if (useGraph && n == kBatchChunk) {
            if ((s = batch_graph(b, n)) != CP_OK) return s;
        }
        if (useGraph && b->graph && b->graphOuter == n) CK(cudaGraphLaunch(b->graph, b->stream));
        else if ((s = batch_launch_any(b, n)) != CP_OK) return s;
        ++launches;
        done += n;
        CK(cudaMemcpyAsync(b->hFlags, b->teamMode ? b->dRunning : b->dAllDone, sizeof(int),
                           cudaMemcpyDeviceToHost, b->stream));
        CK(cudaMemcpyAsync(b->hFlags + 1, b->dErr, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
        CK(cudaStreamSynchronize(b->stream));
        if (b->hFlags[1] != 0)
            return fail((cp_status)b->hFlags[1], "device reported %s in the batch",
                        cp_status_string((cp_status)b->hFlags[1]));
        all = b->teamMode ? b->hFlags[0] == 0 : b->hFlags[0] != 0;
    }
    CK(cudaEventRecord(b->ev1, b->stream));
    CK(cudaEventSynchronize(b->ev1));
    if (rep) {
        memset(rep, 0, sizeof(*rep));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        rep->device_ms = ms;
        rep->launches = launches;
        rep->tileRows = b->teamMode ? 0 : b->R;
        rep->tileCols = b->teamMode ? 0 : b->C;
        rep->teamCtas = b->teamMode ? b->team : 0;
        int maxIt = 0, nd = 0;
        for (cp_ctx* c : b->f) {
            CK(cudaMemcpy(c->stHost, c->st, sizeof(Status), cudaMemcpyDeviceToHost));
            maxIt = std::max(maxIt, c->stHost->iter);
            nd += c->stHost->done ? 1 : 0;
        }
        rep->outerIterations = maxIt;
        rep->fieldsDone = nd;
    }
    if (b->dProf) {
        // CP_BATCH_PROFILE: device time per phase since the batch was made
        static const char* names[BP_COUNT] = {"bc", "assemble", "jacobi", "jacobi_sum", "scatter", "bc_star",
                                              "mass", "mass_sum", "coarsen", "coarsen_cta", "restrict",
                                              "cycle_cta", "prolong", "cycle_sum", "matvec", "matvec_sum",
                                              "update", "update_sum", "p_star", "correct", "bc_end", "finalize"};
        unsigned long long t[BP_COUNT];
        CK(cudaMemcpy(t, b->dProf, sizeof(t), cudaMemcpyDeviceToHost));
        fprintf(stderr, "CP_BATCH_PROFILE ms:");
        for (int q = 0; q < BP_COUNT; ++q) fprintf(stderr, " %s %.3f", names[q], t[q] * 1e-6);
        fprintf(stderr, "\n");
    }
    return CP_OK;
}

}  // namespace

extern "C" {

cp_status cp_batch_create(cp_ctx* const* fields, int n, cp_batch** out) {
    if (!fields || !out) return fail(CP_ERR_BAD_PARAM, "NULL argument");
    *out = nullptr;
    if (n < 1 || n > kBatchMaxFields) return fail(CP_ERR_BAD_PARAM, "batch of %d fields (1..%d)", n, kBatchMaxFields);
    for (int q = 0; q < n; ++q) {
        cp_ctx* c = fields[q];
        if (!c) return fail(CP_ERR_BAD_PARAM, "field %d is NULL", q);
        for (int r = 0; r < q; ++r)
            if (fields[r] == c) return fail(CP_ERR_BAD_PARAM, "field %d repeats field %d", q, r);
        if (!c->useMg)
            return fail(CP_ERR_UNSUPPORTED, "field %d: batches run pressureSolverType 2 or 4 (multigrid-PCG)", q);
        if (c->prm.precision != fields[0]->prm.precision)
            return fail(CP_ERR_BAD_PARAM, "field %d: every field of a batch needs the same precision", q);
        if (c->dev != fields[0]->dev) return fail(CP_ERR_BAD_PARAM, "field %d is on another device", q);
        if (c->mgLg + 1 > kBatchMaxLevels) return fail(CP_ERR_BAD_PARAM, "field %d: grid too large for a batch", q);
    }
    cp_batch* b = new cp_batch();
    b->f.assign(fields, fields + n);
    b->dev = fields[0]->dev;
    b->numSMs = fields[0]->numSMs;
    b->mixed = fields[0]->prm.precision == CP_PREC_MIXED;
    for (cp_ctx* c : b->f) {
        b->maxLg = std::max(b->maxLg, c->mgLg);
        b->maxMom = std::max(b->maxMom, c->k.maxMom);
        b->maxP = std::max(b->maxP, c->k.maxP);
    }
    auto bail = [&](cp_status s) {
        std::string keep = g_err;
        cp_batch_destroy(b);
        g_err = keep;
        return s;
    };
    cp_status s = CP_OK;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaMallocHost(&b->hFlags, 2 * sizeof(int)) != cudaSuccess)
        return bail(fail(CP_ERR_CUDA, "batch stream / events / pinned flags"));
    // team mode when every field runs smoothed aggregation (CP_BATCH_TILES=1
    // keeps the tile kernel, which runs the 2 x 2 cycle for every field)
    b->teamMode = !getenv("CP_BATCH_TILES");
    for (cp_ctx* c : b->f) b->teamMode = b->teamMode && c->useSa;
    // one block per SM: the kernel must fit with its shared-memory workspace
    int nb = 0;
    if (b->teamMode) {
        for (cp_ctx* c : b->f) b->teamSmem = std::max(b->teamSmem, c->saSmem);
        if (b->mixed) {
            cudaFuncSetAttribute(k_batch_team<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)b->teamSmem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch_team<float, true>, kBatchThreads,
                                                          b->teamSmem);
        } else {
            cudaFuncSetAttribute(k_batch_team<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)b->teamSmem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch_team<double, false>, kBatchThreads,
                                                          b->teamSmem);
        }
    } else if (b->mixed) {
        cudaFuncSetAttribute(k_batch<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchDynSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch<float, true>, kBatchThreads, kBatchDynSmem);
    } else {
        cudaFuncSetAttribute(k_batch<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kBatchDynSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch<double, false>, kBatchThreads, kBatchDynSmem);
    }
    if (nb < 1) return bail(fail(CP_ERR_CUDA, "the batch kernel does not fit on an SM"));
    b->grid = b->numSMs;
    for (const auto& t : kBatchTiles) b->partCap = std::max(b->partCap, batch_tiles0(b, t[0], t[1]));
    const size_t nt = (size_t)(b->maxLg + 1) * (n + 1);
    const size_t fbytes = b->teamMode ? (b->mixed ? sizeof(BFieldSa<float>) : sizeof(BFieldSa<double>))
                                      : (b->mixed ? sizeof(BField<float>) : sizeof(BField<double>));
    if ((s = batch_balloc(b, &b->dF, fbytes * n)) != CP_OK) return bail(s);
    if ((s = batch_balloc(b, (void**)&b->dToff, nt * sizeof(int))) != CP_OK) return bail(s);
    if ((s = batch_balloc(b, (void**)&b->dBs, (size_t)n * sizeof(BState))) != CP_OK) return bail(s);
    if ((s = batch_balloc(b, (void**)&b->dPart, b->partCap * kBatchPartStride * sizeof(double))) != CP_OK)
        return bail(s);
    if ((s = batch_balloc(b, (void**)&b->dBar, sizeof(unsigned))) != CP_OK) return bail(s);
    if ((s = batch_balloc(b, (void**)&b->dErr, sizeof(int))) != CP_OK) return bail(s);
    if ((s = batch_balloc(b, (void**)&b->dAllDone, sizeof(int))) != CP_OK) return bail(s);
    if (getenv("CP_BATCH_PROFILE") &&
        (s = batch_balloc(b, (void**)&b->dProf, BP_COUNT * sizeof(unsigned long long))) != CP_OK)
        return bail(s);
    if (b->teamMode) {
        if ((s = batch_balloc(b, (void**)&b->dOrder, (size_t)n * sizeof(int))) != CP_OK) return bail(s);
        if ((s = batch_balloc(b, (void**)&b->dTbar, (size_t)b->grid * kTeamStride * sizeof(unsigned))) != CP_OK)
            return bail(s);
        if ((s = batch_balloc(b, (void**)&b->dQueue, (size_t)(1 + 2 * b->grid) * sizeof(int))) != CP_OK)
            return bail(s);
        if ((s = batch_balloc(b, (void**)&b->dRunning, sizeof(int))) != CP_OK) return bail(s);
    }
    s = b->mixed ? batch_upload_fields<float>(b) : batch_upload_fields<double>(b);
    if (s != CP_OK) return bail(s);
    if ((s = batch_set_tile(b, b->R, b->C)) != CP_OK) return bail(s);
    if (b->teamMode && (s = batch_set_team(b, std::min(kBatchTeamDefault, b->grid))) != CP_OK) return bail(s);
    *out = b;
    return CP_OK;
}

cp_status cp_batch_destroy(cp_batch* b) {
    if (!b) return CP_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (void* q : b->allocs) cudaFree(q);
    if (b->hFlags) cudaFreeHost(b->hFlags);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return CP_OK;
}

cp_status cp_batch_set_tile(cp_batch* b, int rows, int cols) {
    if (!b) return fail(CP_ERR_BAD_PARAM, "batch is NULL");
    return batch_set_tile(b, rows, cols);
}

cp_status cp_batch_set_team(cp_batch* b, int ctas) {
    if (!b) return fail(CP_ERR_BAD_PARAM, "batch is NULL");
    if (!b->teamMode) return fail(CP_ERR_UNSUPPORTED, "the batch runs cell tiles (not every field is type 4)");
    return batch_set_team(b, ctas);
}

cp_status cp_batch_run(cp_batch* b, int max_outer, cp_batch_report* rep) {
    if (!b) return fail(CP_ERR_BAD_PARAM, "batch is NULL");
    if (max_outer < 0) return fail(CP_ERR_BAD_PARAM, "max_outer < 0");
    return batch_run(b, max_outer, rep, true);
}

cp_status cp_batch_autotune(cp_batch* b, int trial_outer, cp_batch_report* best) {
    if (!b) return fail(CP_ERR_BAD_PARAM, "batch is NULL");
    if (trial_outer < 1) return fail(CP_ERR_BAD_PARAM, "trial_outer >= 1 required");
    double bestMs = -1.0;
    if (b->teamMode) {
        int bT = b->team;
        for (int t : kBatchTeams) {
            if (t > b->grid) continue;
            cp_status s = batch_set_team(b, t);
            if (s != CP_OK) return s;
            for (cp_ctx* c : b->f)
                if ((s = cp_reset(c)) != CP_OK) return s;
            cp_batch_report r;
            if ((s = batch_run(b, trial_outer, &r, false)) != CP_OK) return s;
            if (bestMs < 0.0 || r.device_ms < bestMs) { bestMs = r.device_ms; bT = t; }
        }
        cp_status s = batch_set_team(b, bT);
        if (s != CP_OK) return s;
        for (cp_ctx* c : b->f)
            if ((s = cp_reset(c)) != CP_OK) return s;
        if (best) {
            memset(best, 0, sizeof(*best));
            best->teamCtas = bT;
            best->device_ms = bestMs;
            best->outerIterations = trial_outer;
        }
        return CP_OK;
    }
    int bR = b->R, bC = b->C;
    for (const auto& t : kBatchTiles) {
        if (batch_tiles0(b, t[0], t[1]) > b->partCap) continue;
        cp_status s = batch_set_tile(b, t[0], t[1]);
        if (s != CP_OK) return s;
        for (cp_ctx* c : b->f)
            if ((s = cp_reset(c)) != CP_OK) return s;
        cp_batch_report r;
        if ((s = batch_run(b, trial_outer, &r, false)) != CP_OK) return s;
        if (bestMs < 0.0 || r.device_ms < bestMs) { bestMs = r.device_ms; bR = t[0]; bC = t[1]; }
    }
    cp_status s = batch_set_tile(b, bR, bC);
    if (s != CP_OK) return s;
    for (cp_ctx* c : b->f)
        if ((s = cp_reset(c)) != CP_OK) return s;
    if (best) {
        memset(best, 0, sizeof(*best));
        best->tileRows = bR;
        best->tileCols = bC;
        best->device_ms = bestMs;
        best->outerIterations = trial_outer;
    }
    return CP_OK;
}

}  // extern "C"
