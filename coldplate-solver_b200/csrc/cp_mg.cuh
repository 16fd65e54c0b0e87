// Multigrid-preconditioned CG for the pressure correction
// (pressureSolverType 2 / 4).
//
// The reference runs these solver types with AMGCL: smoothed-aggregation AMG
// as a CG preconditioner (pressure_solver.cu:81-163, cuda_common.cuh:44-53).
// Here the preconditioner is geometric aggregation multigrid on the
// structured pressure grid:
//   * 2 x 2 aggregation with piecewise-constant prolongation P, restriction
//     P^T and Galerkin coarse operators A_c = P^T A P, which stay 5-point:
//     a coarse face coefficient is the sum of the fine face coefficients
//     that cross it, and the Dirichlet faces of the outlet column carry over
//     to the coarse cells that contain it;
//   * V(1,1) cycle with one damped-Jacobi sweep before and after the coarse
//     correction (the same sweep both ways, so the preconditioner is
//     symmetric and CG applies);
//   * levels with more than kMgCtaCells unknowns run on the whole grid with
//     bounded grid barriers; smaller levels run on CTA 0 alone with block
//     barriers; the coarsest level (<= kMgDense unknowns) is solved with a
//     dense inverse built once per pressure solve.
// The CG recurrences and the |p.Ap| < 1e-20 exit are those of
// pressure_solver.cpp:121-184.  The convergence test is AMGCL's, since the
// reference hands pTol and maxPressureIter to AMGCL's CG for these types
// (pressure_solver.cpp:754-757, pressure_solver.cu:114-116): stop once
// ||r|| <= pTol ||b|| (relative to the right-hand side, x0 = 0), and report
// the number of completed iterations.  AMGCL (github.com/ddemidov/amgcl) is
// not vendored with the reference (its directory there is empty), so this
// follows AMGCL's published CG; its version is not pinned.
#pragma once

#include "cp_kernels.cuh"
#include "cp_tma.cuh"

namespace cp {

constexpr int kMgMaxLevels = 16;
constexpr int kMgCtaCells = 1024;    // levels at or below this size run on one CTA
constexpr int kMgDense = 64;         // coarsest level size solved by a dense inverse

template <typename TV>
struct MgLevel {
    int nI, nJ, P;          // unknowns i in [1, nI], j in [1, nJ]; zero frame around them
    TV *fE, *fN, *d, *dx;   // east / north face coefficients, diagonal, extra diagonal
    TV *x, *y, *b;          // iterate (ping-pong x/y) and right-hand side
};

template <typename TV>
struct MgHier {
    int L;                  // number of levels
    int Lg;                 // levels [0, Lg) run grid-wide
    MgLevel<TV> lv[kMgMaxLevels];
    TV* dense;              // kMgDense^2 inverse of the coarsest operator
    double omega;           // Jacobi damping
    double scale;           // coarse-correction scaling (1: plain Galerkin correction)
    unsigned long long* prof;  // optional per-phase device-time accumulators (ns), or null
};

enum MgPhase { MG_P_SETUP = 0, MG_P_A, MG_P_B, MG_P_DOWN, MG_P_CTA, MG_P_UP, MG_P_COUNT };
// per-level timers follow the phase timers: restriction out of level l at
// MG_P_COUNT + l, prolongation into level l at MG_P_COUNT + kMgMaxLevels + l
constexpr int kMgProfSlots = MG_P_COUNT + 2 * kMgMaxLevels;

// ---------------------------------------------------------------- level ops
template <typename TV>
__device__ __forceinline__ size_t lidx(const MgLevel<TV>& l, int i, int j) {
    return (size_t)i * l.P + j;
}

// A x at (i, j) of a level (x is zero on the frame)
template <typename TV>
__device__ __forceinline__ TV mg_ax(const MgLevel<TV>& l, const TV* x, size_t c) {
    return l.d[c] * x[c] - l.fE[c] * x[c + 1] - l.fE[c - 1] * x[c - 1] - l.fN[c] * x[c + l.P] -
           l.fN[c - l.P] * x[c - l.P];
}

// coarse operator of level l+1 from level l (one coarse cell)
template <typename TV>
__device__ __forceinline__ void mg_coarsen_cell(const MgLevel<TV>& f, const MgLevel<TV>& c, int I, int J) {
    const int i0 = 2 * I - 1, i1 = min(2 * I, f.nI), j0 = 2 * J - 1, j1 = min(2 * J, f.nJ);
    // east face of the aggregate: fine faces at column j1 (the Dirichlet face when j1 == f.nJ)
    auto eastFace = [&](int jj) -> double {
        double s = 0.0;
        for (int i = i0; i <= i1; ++i) s += (double)f.fE[lidx(f, i, jj)];
        return s;
    };
    auto northFace = [&](int ii) -> double {
        double s = 0.0;
        for (int j = j0; j <= j1; ++j) s += (double)f.fN[lidx(f, ii, j)];
        return s;
    };
    const double fe = eastFace(j1);
    const double fn = (I < c.nI) ? northFace(i1) : 0.0;
    // west / south coarse faces recomputed from the neighbouring aggregates
    const double fw = (J > 1) ? eastFace(j0 - 1) : 0.0;
    const double fs = (I > 1) ? northFace(i0 - 1) : 0.0;
    double ex = 0.0;
    for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j) ex += (double)f.dx[lidx(f, i, j)];
    const size_t q = lidx(c, I, J);
    c.fE[q] = (TV)fe;
    c.fN[q] = (TV)fn;
    c.dx[q] = (TV)ex;
    c.d[q] = (TV)(fe + fw + fn + fs + ex);
}

// restriction of the residual of level l into b of level l+1, and the first
// (pre-)smoothing step of level l+1 from zero: x_{l+1} = omega b / d
template <typename TV>
__device__ __forceinline__ void mg_restrict_cell(const MgLevel<TV>& f, const MgLevel<TV>& c, int I, int J,
                                                 double omega) {
    const int i0 = 2 * I - 1, i1 = min(2 * I, f.nI), j0 = 2 * J - 1, j1 = min(2 * J, f.nJ);
    double s = 0.0;
    for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j) {
            const size_t q = lidx(f, i, j);
            s += (double)(f.b[q] - mg_ax(f, f.x, q));
        }
    const size_t q = lidx(c, I, J);
    c.b[q] = (TV)s;
    c.x[q] = (TV)(omega * s / (double)c.d[q]);
}

// prolongation of level l+1 into level l followed by one Jacobi sweep:
// x' = x + P e; y = x' + omega D^-1 (b - A x').  Writes y (the other buffer).
template <typename TV>
__device__ __forceinline__ TV mg_prolong_smooth_cell(const MgLevel<TV>& f, const MgLevel<TV>& c, const TV* e,
                                                     int i, int j, double omega, double c_scale) {
    // e: the coarse level's corrected iterate (its x or y buffer)
    const TV sc = (TV)c_scale;
    auto xp = [&](int ii, int jj) -> TV {
        if (ii < 1 || ii > f.nI || jj < 1 || jj > f.nJ) return (TV)0;
        return f.x[lidx(f, ii, jj)] + sc * e[lidx(c, (ii + 1) >> 1, (jj + 1) >> 1)];
    };
    const size_t q = lidx(f, i, j);
    const TV xc = xp(i, j);
    const TV ax = f.d[q] * xc - f.fE[q] * xp(i, j + 1) - f.fE[q - 1] * xp(i, j - 1) - f.fN[q] * xp(i + 1, j) -
                  f.fN[q - f.P] * xp(i - 1, j);
    const TV y = xc + (TV)omega * (f.b[q] - ax) / f.d[q];
    f.y[q] = y;
    return y;
}

// ---------------------------------------------------------------- level 0
// Level 0 keeps no iterate of its own: its right-hand side is the CG
// residual r (f.b aliases it) and the pre-smoothed iterate from zero is
// x0 = omega r / d, recomputed where needed (zero off the unknowns, where
// r and d are zero).
template <typename TV>
__device__ __forceinline__ TV l0_x(const MgLevel<TV>& f, size_t q, TV om) {
    const TV dd = f.d[q];
    return dd != (TV)0 ? om * f.b[q] / dd : (TV)0;
}

// restriction of the level-0 residual b - A x0 over one 2 x 2 aggregate;
// d x0 = omega b, so the residual is (1 - omega) b + off-diagonal terms
template <typename TV>
__device__ __forceinline__ void mg_restrict0_cell(const MgLevel<TV>& f, const MgLevel<TV>& c, int I, int J,
                                                  double omega) {
    const int i0 = 2 * I - 1, i1 = min(2 * I, f.nI), j0 = 2 * J - 1, j1 = min(2 * J, f.nJ);
    const TV om = (TV)omega;
    double s = 0.0;
    for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j) {
            const size_t q = lidx(f, i, j);
            const TV r = ((TV)1 - om) * f.b[q] + f.fE[q] * l0_x(f, q + 1, om) + f.fE[q - 1] * l0_x(f, q - 1, om) +
                         f.fN[q] * l0_x(f, q + f.P, om) + f.fN[q - f.P] * l0_x(f, q - f.P, om);
            s += (double)r;
        }
    const size_t q = lidx(c, I, J);
    c.b[q] = (TV)s;
    c.x[q] = (TV)(omega * s / (double)c.d[q]);
}

// The same two level-0 operators with the pre-smoothed iterate stored in
// f.x (omega r / d, zero off the unknowns) instead of recomputed.
template <typename TV>
__device__ __forceinline__ void mg_restrict0x_cell(const MgLevel<TV>& f, const MgLevel<TV>& c, int I, int J,
                                                   double omega) {
    const int i0 = 2 * I - 1, i1 = min(2 * I, f.nI), j0 = 2 * J - 1, j1 = min(2 * J, f.nJ);
    const TV om = (TV)omega;
    double s = 0.0;
    for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j) {
            const size_t q = lidx(f, i, j);
            const TV r = ((TV)1 - om) * f.b[q] + f.fE[q] * f.x[q + 1] + f.fE[q - 1] * f.x[q - 1] +
                         f.fN[q] * f.x[q + f.P] + f.fN[q - f.P] * f.x[q - f.P];
            s += (double)r;
        }
    const size_t q = lidx(c, I, J);
    c.b[q] = (TV)s;
    c.x[q] = (TV)(omega * s / (double)c.d[q]);
}

template <typename TV>
__device__ __forceinline__ TV mg_prolong0x_cell(const MgLevel<TV>& f, const MgLevel<TV>& c, const TV* e, int i,
                                                int j, double omega, double c_scale) {
    const TV om = (TV)omega, sc = (TV)c_scale;
    auto xp = [&](int ii, int jj) -> TV {
        if (ii < 1 || ii > f.nI || jj < 1 || jj > f.nJ) return (TV)0;
        return f.x[lidx(f, ii, jj)] + sc * e[lidx(c, (ii + 1) >> 1, (jj + 1) >> 1)];
    };
    const size_t q = lidx(f, i, j);
    const TV xc = xp(i, j);
    const TV ax = f.d[q] * xc - f.fE[q] * xp(i, j + 1) - f.fE[q - 1] * xp(i, j - 1) - f.fN[q] * xp(i + 1, j) -
                  f.fN[q - f.P] * xp(i - 1, j);
    const TV y = xc + om * (f.b[q] - ax) / f.d[q];
    f.y[q] = y;
    return y;
}

// prolongation into level 0 + one Jacobi sweep: x' = x0 + s P e, y = x' + omega (b - A x') / d
template <typename TV>
__device__ __forceinline__ TV mg_prolong0_cell(const MgLevel<TV>& f, const MgLevel<TV>& c, const TV* e, int i,
                                               int j, double omega, double c_scale) {
    const TV om = (TV)omega, sc = (TV)c_scale;
    auto xp = [&](int ii, int jj) -> TV {
        if (ii < 1 || ii > f.nI || jj < 1 || jj > f.nJ) return (TV)0;
        return l0_x(f, lidx(f, ii, jj), om) + sc * e[lidx(c, (ii + 1) >> 1, (jj + 1) >> 1)];
    };
    const size_t q = lidx(f, i, j);
    const TV xc = xp(i, j);
    const TV ax = f.d[q] * xc - f.fE[q] * xp(i, j + 1) - f.fE[q - 1] * xp(i, j - 1) - f.fN[q] * xp(i + 1, j) -
                  f.fN[q - f.P] * xp(i - 1, j);
    const TV y = xc + om * (f.b[q] - ax) / f.d[q];
    f.y[q] = y;
    return y;
}

// ---------------------------------------------------------------- work splits
struct Split {
    int t0, nt;
};

template <typename F>
__device__ __forceinline__ void for_cells(Split s, int nI, int nJ, F&& fn) {
    const int n = nI * nJ;
    for (int t = s.t0; t < n; t += s.nt) fn(1 + t / nJ, 1 + t % nJ);
}

// dense inverse of the coarsest operator (Gauss-Jordan, SPD, no pivoting),
// run by one CTA; A is assembled from the level's stencil
template <typename TV>
__device__ void mg_dense_setup(const MgLevel<TV>& l, TV* inv, double* work /* smem n*2n + n */) {
    const int n = l.nI * l.nJ, w = 2 * n;
    double* fac = work + n * w;
    for (int e = threadIdx.x; e < n * w; e += blockDim.x) work[e] = 0.0;
    __syncthreads();
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        const int i = 1 + a / l.nJ, j = 1 + a % l.nJ;
        const size_t q = lidx(l, i, j);
        work[a * w + a] = (double)l.d[q];
        if (j < l.nJ) work[a * w + a + 1] = -(double)l.fE[q];
        if (j > 1) work[a * w + a - 1] = -(double)l.fE[q - 1];
        if (i < l.nI) work[a * w + a + l.nJ] = -(double)l.fN[q];
        if (i > 1) work[a * w + a - l.nJ] = -(double)l.fN[q - l.P];
        work[a * w + n + a] = 1.0;
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double piv = work[k * w + k];
        __syncthreads();
        for (int c = threadIdx.x; c < w; c += blockDim.x) work[k * w + c] /= piv;
        for (int r = threadIdx.x; r < n; r += blockDim.x) fac[r] = work[r * w + k];
        __syncthreads();
        for (int e = threadIdx.x; e < n * w; e += blockDim.x) {
            const int r = e / w, c = e % w;
            if (r != k) work[e] -= fac[r] * work[k * w + c];
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) inv[e] = (TV)work[(e / n) * w + n + e % n];
    __syncthreads();
}

template <typename TV>
__device__ void mg_dense_solve(const MgLevel<TV>& l, const TV* inv) {
    const int n = l.nI * l.nJ;
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        double s = 0.0;
        for (int b2 = 0; b2 < n; ++b2) s += (double)inv[a * n + b2] * (double)l.b[lidx(l, 1 + b2 / l.nJ, 1 + b2 % l.nJ)];
        l.x[lidx(l, 1 + a / l.nJ, 1 + a % l.nJ)] = (TV)s;
    }
    __syncthreads();
}

// single-CTA part of the V-cycle: levels [Lg, L); on entry b and x
// (= omega b / d) of level Lg are set; on exit x of level Lg holds the
// corrected iterate.
template <typename TV>
__device__ void mg_cta_cycle(const MgHier<TV>& H) {
    Split s{(int)threadIdx.x, (int)blockDim.x};
    for (int l = H.Lg; l < H.L - 1; ++l) {
        for_cells(s, H.lv[l + 1].nI, H.lv[l + 1].nJ,
                  [&](int I, int J) { mg_restrict_cell(H.lv[l], H.lv[l + 1], I, J, H.omega); });
        __syncthreads();
    }
    mg_dense_solve(H.lv[H.L - 1], H.dense);
    for (int l = H.L - 2; l >= H.Lg; --l) {
        const MgLevel<TV>& f = H.lv[l];
        for_cells(s, f.nI, f.nJ,
                  [&](int i, int j) { mg_prolong_smooth_cell(f, H.lv[l + 1], H.lv[l + 1].x, i, j, H.omega, H.scale); });
        __syncthreads();
        for_cells(s, f.nI, f.nJ, [&](int i, int j) { const size_t q = lidx(f, i, j); f.x[q] = f.y[q]; });
        __syncthreads();
    }
}

// ---------------------------------------------------------------- TMA tiles of level 0
// Tensor maps of the arrays the level-0 phases read (built per context).
struct MgMaps {
    CUtensorMap z, pa, pb, r, d, fE, fN, e1, x0;
};

// Depth of the TMA pipeline of the level-0 tile phases: up to kTmaStages
// tiles in flight per CTA.  Four stages (197 KB of shared memory for double)
// timed the same as two at 2048 x 1024 (156 vs 153 us per CG iteration,
// mixed): the phases are bound by the grid barriers, not by TMA latency.
constexpr int kTmaStages = 2;

template <typename TV>
struct TileSmem {
    typedef TileGeom<TV> G;
    static constexpr int kBox = ((G::BoxR * G::BoxW * (int)sizeof(TV) + 127) / 128) * 128;
    static constexpr int kCBox = ((G::CBoxR * G::CBoxW * (int)sizeof(TV) + 127) / 128) * 128;
    static constexpr int kStage = 6 * kBox;   // up to five fine boxes and a coarse one per stage
    static constexpr int kBytes = kTmaStages * kStage;
};

// Runs compute(tile, stage) over this CTA's tiles (tile = blockIdx.x + k G)
// with a kTmaStages-deep TMA pipeline; issue(tile, stage) is called by thread 0
// and must arm the stage's mbarrier and start the copies.  `parity` holds
// the phase bit of each stage's mbarrier (kept in step by all threads).
template <typename Issue, typename Compute>
__device__ __forceinline__ bool tile_loop(int ntiles, uint64_t* bars, unsigned& parity, int* err, Issue&& issue,
                                          Compute&& compute) {
    const int G = gridDim.x;
    if (threadIdx.x == 0) {
        fence_proxy_async_global();
        for (int s = 0; s < kTmaStages; ++s) {
            const int t = blockIdx.x + s * G;
            if (t < ntiles) issue(t, s);
        }
    }
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += G, ++k) {
        const int s = k % kTmaStages;
        if (!mbar_wait(&bars[s], (parity >> s) & 1u, err)) return false;
        parity ^= (1u << s);
        compute(t, s);
        __syncthreads();
        if (threadIdx.x == 0) {
            const int tn = t + kTmaStages * G;
            if (tn < ntiles) {
                fence_proxy_async_shared();
                issue(tn, s);
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------- the solver
// B (PcgBufs) holds level-0 faces, diagonal and the CG vectors in the field
// layout; H.lv[0] aliases them (fE, fN, d) plus its own x/y/b/dx buffers.
template <typename TV>
__global__ void __launch_bounds__(512, 1) k_pcg_mg(KParams k, Status* st, const double* dE, const double* dN,
                                                PcgBufs<TV> B, MgHier<TV> H, double* pStar, double* part,
                                                unsigned* bar, const __grid_constant__ MgMaps maps) {
    if (st->done) return;
    // dynamic shared memory: dense set-up workspace, later the TMA tile stages
    extern __shared__ __align__(128) double dsm[];
    __shared__ double sm[96];
    __shared__ __align__(8) uint64_t tbar[kTmaStages];
    unsigned tpar = 0;
    if (threadIdx.x == 0) {
        for (int q = 0; q < kTmaStages; ++q) mbar_init(&tbar[q], 1);
        mbar_fence_init();
    }
    __syncthreads();
    unsigned char* stg = reinterpret_cast<unsigned char*>(dsm);
    typedef TileSmem<TV> TS;
    auto box = [&](int stage, int q) -> TV* { return reinterpret_cast<TV*>(stg + stage * TS::kStage + q * TS::kBox); };
    const Dims d = k.d;
    const int M = d.M, N = d.N, w = N - 2;
    const int n = (M - 1) * w;
    const int G = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = G * blockDim.x;
    const Split all{tid, nth};
    const double rho = k.rho, hx = k.hx, hy = k.hy, om = H.omega;
    unsigned target = 0;
    double* partA = part;
    double* partB = part + G;
    const MgLevel<TV>& L0 = H.lv[0];
#define MG_SYNC()                                                   \
    do {                                                            \
        target += G;                                                \
        if (!grid_barrier(bar, target, &st->err)) return;           \
    } while (0)

    // ---- setup: level-0 operator (reference formulas), x = 0, r = b
    double bb[1] = {0.0};
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        const double aE = rho * dE[c] * hy;
        const double aW = (j > 1) ? rho * dE[c - 1] * hy : 0.0;
        const double aN = (i < M - 1) ? rho * dN[c] * hx : 0.0;
        const double aS = (i > 1) ? rho * dN[c - d.P] * hx : 0.0;
        double aP = aE + aW + aN + aS;
        double extra = 0.0;
        if (aP < 1e-20) { extra = 1.0 - aP; aP = 1.0; }
        B.fE[c] = (TV)aE;
        if (i < M - 1) B.fN[c] = (TV)aN;
        const TV dt = (TV)aP;
        B.d[c] = dt;
        L0.dx[c] = (TV)extra;
        B.x[c] = (TV)0;
        const TV rt = B.rhs[c];
        B.r[c] = rt;
        L0.x[c] = (TV)om * rt / dt;   // pre-smoothed level-0 iterate omega r / d
        bb[0] += (double)rt * (double)rt;
    }
    block_sum<1>(bb, sm);
    if (threadIdx.x == 0) partA[blockIdx.x] = bb[0];
    MG_SYNC();
    // partA is next written in the first CG iteration, after several grid barriers
    double bnorm2[1];
    sum_partials<1>(partA, G, 1, bnorm2, sm);
    const double rTol = k.pTol * sqrt(bnorm2[0]);
    // ---- setup: coarse operators
    for (int l = 0; l < H.L - 1; ++l) {
        const bool cta = (l + 1) >= H.Lg;
        if (!cta) {
            for_cells(all, H.lv[l + 1].nI, H.lv[l + 1].nJ,
                      [&](int I, int J) { mg_coarsen_cell(H.lv[l], H.lv[l + 1], I, J); });
            MG_SYNC();
        } else if (blockIdx.x == 0) {
            for_cells(Split{(int)threadIdx.x, (int)blockDim.x}, H.lv[l + 1].nI, H.lv[l + 1].nJ,
                      [&](int I, int J) { mg_coarsen_cell(H.lv[l], H.lv[l + 1], I, J); });
            __syncthreads();
        }
    }
    if (blockIdx.x == 0) mg_dense_setup(H.lv[H.L - 1], H.dense, dsm);
    MG_SYNC();

    auto tick = [&](int ph, unsigned long long& t0) {
        if (H.prof && blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long t = globaltimer_ns();
            atomicAdd(H.prof + ph, t - t0);
            t0 = t;
        }
    };
    unsigned long long tp = (H.prof && blockIdx.x == 0 && threadIdx.x == 0) ? globaltimer_ns() : 0ull;

    // ---- level-0 tile phases (TMA staged)
    constexpr int kTileR = TileGeom<TV>::R, kTileC = TileGeom<TV>::C, kBoxR = TileGeom<TV>::BoxR,
                  kBoxW = TileGeom<TV>::BoxW, kCBoxR = TileGeom<TV>::CBoxR, kCBoxW = TileGeom<TV>::CBoxW;
    // the restriction pairs lanes with a shuffle: every thread of the 512 takes the same passes
    static_assert((kTileR * kTileC / 2) % 512 == 0, "tile pairs must fill whole passes of 512 threads");
    static_assert(kTileR % 2 == 0 && kTileC % 16 == 0, "tile rows even, tile columns 16-byte aligned");
    const int nI0 = M - 1, nJ0 = w;
    const int tilesI = (nI0 + kTileR - 1) / kTileR, tilesJ = (nJ0 + kTileC - 1) / kTileC;
    const int ntiles = tilesI * tilesJ;
    const TV omT = (TV)om;
    const unsigned fineBox = kBoxR * kBoxW * sizeof(TV);
    const unsigned coarseBox = kCBoxR * kCBoxW * sizeof(TV);
    auto issue_fine = [&](int t, int s, const CUtensorMap* const* mp, int nb, bool withCoarse) {
        const int tI = t / tilesJ, tJ = t % tilesJ;
        mbar_expect_tx(&tbar[s], nb * fineBox + (withCoarse ? coarseBox : 0u));
        for (int q = 0; q < nb; ++q) tma_load_2d(box(s, q), mp[q], kTileC * tJ, kTileR * tI, &tbar[s]);
        if (withCoarse)
            tma_load_2d(box(s, nb), &maps.e1, (kTileC / 2) * tJ, (kTileR / 2) * tI, &tbar[s]);
    };
    // smem element (li, lj) of a fine box: array row i0 - 1 + li, column j0 - 1 + lj
#define SB(q, li, lj) (bx[q][(li) * kBoxW + (lj)])
    // The level-0 pre-smoothed iterate x0 = omega r / d is stored (L0.x) by
    // the set-up and by every CG update, and read as a box: one division per
    // unknown per CG iteration instead of one per stencil point.
    // restriction of the level-0 residual into level 1 (boxes: r, x0, fE, fN)
    auto restrict0_tiles = [&]() -> bool {
        const CUtensorMap* mp[4] = {&maps.r, &maps.x0, &maps.fE, &maps.fN};
        const MgLevel<TV>& C1 = H.lv[1];
        return tile_loop(ntiles, tbar, tpar, &st->err,
                         [&](int t, int s) { issue_fine(t, s, mp, 4, false); },
                         [&](int t, int s) {
            TV* bx[4] = {box(s, 0), box(s, 1), box(s, 2), box(s, 3)};
            const int tI = t / tilesJ, tJ = t % tilesJ;
            const int i0 = 1 + kTileR * tI, j0 = 1 + kTileC * tJ;
            for (int u = threadIdx.x; u < 2 * (kTileR / 2) * (kTileC / 2); u += blockDim.x) {
                const int cc = u >> 1, h = u & 1;
                const int cr = cc / (kTileC / 2), ccol = cc % (kTileC / 2);
                const int a = 2 * cr + h;
                double sum = 0.0;
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int b = 2 * ccol + q;
                    if (i0 + a <= nI0 && j0 + b <= nJ0) {
                        const int li = a + 1, lj = b + 1;
                        const TV r = ((TV)1 - omT) * SB(0, li, lj) + SB(2, li, lj) * SB(1, li, lj + 1) +
                                     SB(2, li, lj - 1) * SB(1, li, lj - 1) + SB(3, li, lj) * SB(1, li + 1, lj) +
                                     SB(3, li - 1, lj) * SB(1, li - 1, lj);
                        sum += (double)r;
                    }
                }
                sum += __shfl_xor_sync(0xffffffffu, sum, 1);
                const int I = 1 + (kTileR / 2) * tI + cr, J = 1 + (kTileC / 2) * tJ + ccol;
                if (h == 0 && I <= C1.nI && J <= C1.nJ) {
                    const size_t q = lidx(C1, I, J);
                    C1.b[q] = (TV)sum;
                    C1.x[q] = (TV)(om * sum / (double)C1.d[q]);
                }
            }
        });
    };
    // prolongation from level 1 + post-smoothing of level 0 (boxes: r, d,
    // fE, fN, x0 and the coarse correction); writes z = L0.y, accumulates r.z
    const TV scT = (TV)H.scale;
    auto prolong0_tiles = [&](double& rzacc) -> bool {
        const CUtensorMap* mp[5] = {&maps.r, &maps.d, &maps.fE, &maps.fN, &maps.x0};
        const MgLevel<TV>& F0 = H.lv[0];
        return tile_loop(ntiles, tbar, tpar, &st->err,
                         [&](int t, int s) { issue_fine(t, s, mp, 5, true); },
                         [&](int t, int s) {
            TV* bx[5] = {box(s, 0), box(s, 1), box(s, 2), box(s, 3), box(s, 4)};
            const TV* ce = box(s, 5);
            const int tI = t / tilesJ, tJ = t % tilesJ;
            const int i0 = 1 + kTileR * tI, j0 = 1 + kTileC * tJ;
            // x' = x0 + e(agg) on unknowns, 0 elsewhere
            auto xp = [&](int li, int lj) -> TV {
                const int ii = i0 - 1 + li, jj = j0 - 1 + lj;
                if (ii < 1 || ii > nI0 || jj < 1 || jj > nJ0) return (TV)0;
                const int cli = ((ii + 1) >> 1) - (kTileR / 2) * tI, clj = ((jj + 1) >> 1) - (kTileC / 2) * tJ;
                return SB(4, li, lj) + scT * ce[cli * kCBoxW + clj];
            };
            for (int u = threadIdx.x; u < kTileR * kTileC; u += blockDim.x) {
                const int a = u / kTileC, b = u % kTileC;
                if (i0 + a > nI0 || j0 + b > nJ0) continue;
                const int li = a + 1, lj = b + 1;
                const TV xc = xp(li, lj);
                const TV ax = SB(1, li, lj) * xc - SB(2, li, lj) * xp(li, lj + 1) - SB(2, li, lj - 1) * xp(li, lj - 1) -
                              SB(3, li, lj) * xp(li + 1, lj) - SB(3, li - 1, lj) * xp(li - 1, lj);
                const TV rb = SB(0, li, lj);
                const TV y = xc + omT * (rb - ax) / SB(1, li, lj);
                F0.y[at(d, i0 + a, j0 + b)] = y;
                rzacc += (double)rb * (double)y;
            }
        });
    };
    // CG matvec on the new direction p = z + beta p_old (boxes: z, p_old, d, fE, fN)
    auto cgA_tiles = [&](bool first, double beta, TV* pnew, const CUtensorMap* pold, double& acc) -> bool {
        const CUtensorMap* mp[5] = {&maps.z, pold, &maps.d, &maps.fE, &maps.fN};
        const TV bt = (TV)beta;
        return tile_loop(ntiles, tbar, tpar, &st->err,
                         [&](int t, int s) { issue_fine(t, s, mp, 5, false); },
                         [&](int t, int s) {
            TV* bx[5] = {box(s, 0), box(s, 1), box(s, 2), box(s, 3), box(s, 4)};
            const int tI = t / tilesJ, tJ = t % tilesJ;
            const int i0 = 1 + kTileR * tI, j0 = 1 + kTileC * tJ;
            auto dir = [&](int li, int lj) -> TV {
                return first ? SB(0, li, lj) : (TV)(SB(0, li, lj) + bt * SB(1, li, lj));
            };
            for (int u = threadIdx.x; u < kTileR * kTileC; u += blockDim.x) {
                const int a = u / kTileC, b = u % kTileC;
                if (i0 + a > nI0 || j0 + b > nJ0) continue;
                const int li = a + 1, lj = b + 1;
                const TV pc = dir(li, lj);
                const TV ap = SB(2, li, lj) * pc - SB(4, li - 1, lj) * dir(li - 1, lj) - SB(3, li, lj - 1) * dir(li, lj - 1) -
                              SB(3, li, lj) * dir(li, lj + 1) - SB(4, li, lj) * dir(li + 1, lj);
                const size_t c = at(d, i0 + a, j0 + b);
                pnew[c] = pc;
                B.Ap[c] = ap;
                acc += (double)pc * (double)ap;
            }
        });
    };

    // ---- z = M r (V-cycle).  Level 0's rhs is r (L0.b aliases B.r) and its
    // pre-smoothed iterate omega r / d is implicit.  Result z in L0.y, and
    // `rz` gets the global r.z.
    auto vcycle = [&](double& rz) -> bool {
        // down: restrict into every level up to the first CTA level
        for (int l = 0; l < H.Lg; ++l) {
            if (l == 0) {
                if (!restrict0_tiles()) return false;
            } else
                for_cells(all, H.lv[l + 1].nI, H.lv[l + 1].nJ,
                          [&](int I, int J) { mg_restrict_cell(H.lv[l], H.lv[l + 1], I, J, om); });
            target += G;
            if (!grid_barrier(bar, target, &st->err)) return false;
            tick(MG_P_COUNT + l, tp);
        }
        tick(MG_P_DOWN, tp);
        // the small levels on CTA 0
        if (blockIdx.x == 0) {
            if (H.Lg < H.L - 1) mg_cta_cycle(H);
            else mg_dense_solve(H.lv[H.L - 1], H.dense);
        }
        target += G;
        if (!grid_barrier(bar, target, &st->err)) return false;
        tick(MG_P_CTA, tp);
        // up: prolongate + post-smooth into y (the corrected iterate of a
        // grid-wide level stays in y, of a CTA level in x)
        for (int l = H.Lg - 1; l >= 0; --l) {
            const MgLevel<TV>& f = H.lv[l];
            const TV* e = (l + 1 < H.Lg) ? H.lv[l + 1].y : H.lv[l + 1].x;
            double acc[1] = {0.0};
            if (l == 0) {
                if (!prolong0_tiles(acc[0])) return false;
                block_sum<1>(acc, sm);
                if (threadIdx.x == 0) partB[2 * blockIdx.x + 1] = acc[0];
            } else {
                for_cells(all, f.nI, f.nJ, [&](int i, int j) { mg_prolong_smooth_cell(f, H.lv[l + 1], e, i, j, om, H.scale); });
            }
            target += G;
            if (!grid_barrier(bar, target, &st->err)) return false;
            tick(MG_P_COUNT + kMgMaxLevels + l, tp);
        }
        double t2[2];
        sum_partials<2>(partB, G, 2, t2, sm);
        rz = t2[1];
        tick(MG_P_UP, tp);
        return true;
    };

    tick(MG_P_SETUP, tp);
    double rz = 0.0;
    if (!vcycle(rz)) return;
    // z lives in L0.y; p_new = z + beta p_old recomputed at the neighbours
    double beta = 0.0;
    int it = 0;
    TV* pbuf[2] = {B.pa, B.pb};
    for (; it < k.maxP; ++it) {
        const bool first = (it == 0);
        TV* __restrict__ pnew = pbuf[it & 1];
        double accA[1] = {0.0};
        if (!cgA_tiles(first, beta, pnew, (it & 1) ? &maps.pa : &maps.pb, accA[0])) return;
        block_sum<1>(accA, sm);
        if (threadIdx.x == 0) partA[blockIdx.x] = accA[0];
        MG_SYNC();
        double pAp[1];
        sum_partials<1>(partA, G, 1, pAp, sm);
        tick(MG_P_A, tp);
        if (fabs(pAp[0]) < 1e-20) break;
        const double alpha = rz / pAp[0];
        const TV al = (TV)alpha;
        double accB[1] = {0.0};
        for (int t0 = tid; t0 < n; t0 += 2 * nth) {
            TV xv[2], pv[2], rv[2], av[2], dv[2];
            size_t cc[2];
            bool ok[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int t = t0 + q * nth;
                ok[q] = t < n;
                const int tt = ok[q] ? t : t0;
                const size_t c = at(d, 1 + tt / w, 1 + tt % w);
                cc[q] = c;
                xv[q] = B.x[c]; pv[q] = pnew[c]; rv[q] = B.r[c]; av[q] = B.Ap[c]; dv[q] = B.d[c];
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!ok[q]) continue;
                B.x[cc[q]] = xv[q] + al * pv[q];
                const TV r = rv[q] - al * av[q];
                B.r[cc[q]] = r;
                L0.x[cc[q]] = omT * r / dv[q];
                accB[0] += (double)r * (double)r;
            }
        }
        block_sum<1>(accB, sm);
        if (threadIdx.x == 0) partB[2 * blockIdx.x] = accB[0];
        MG_SYNC();
        double tB[2];
        sum_partials<2>(partB, G, 2, tB, sm);
        tick(MG_P_B, tp);
        if (sqrt(tB[0]) <= rTol) { ++it; break; }
        double rzn = 0.0;
        if (!vcycle(rzn)) return;
        beta = rzn / rz;
        rz = rzn;
    }
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        pStar[c] = (double)B.x[c];
        if (j == w) pStar[c + 1] = 0.0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->itersP = it;
#undef MG_SYNC
#undef SB
}

}  // namespace cp
