// Smoothed-aggregation multigrid as the CG preconditioner of the pressure
// correction (pressureSolverType 4).
//
// The reference runs type 4 with AMGCL's AMG-CG: smoothed aggregation
// (amgcl::coarsening::smoothed_aggregation) with SPAI0/Jacobi relaxation as
// the preconditioner of CG (pressure_solver.cu:81-163, cuda_common.cuh:44-53).
// AMGCL is not vendored with the reference and its version is not pinned, so
// this follows the published method on the structured pressure grid, with
// geometric aggregates:
//   * aggregates of 3 x 3 unknowns; tentative prolongation P0 piecewise
//     constant; smoothed prolongation P = (I - w D^-1 A) P0; restriction P^T;
//   * Galerkin coarse operators A_c = P^T A P.  The smoothed support of an
//     aggregate is 5 x 5 fine unknowns, so A_c is a 9-point stencil on the
//     coarse grid; it is computed exactly by nine coloured probes (the
//     aggregates of one colour (I mod 3, J mod 3) have disjoint supports):
//     Y_c = A P e_c on the fine grid, then row I of P^T Y_c is the entry of
//     coarse row I towards its colour-c neighbour;
//   * w = 4 / (3 lambda) with lambda the largest eigenvalue of D^-1 A: 2/3 on
//     the fine 5-point level (lambda near 2) and 0.8 on the 9-point coarse
//     levels (lambda 1.6-1.8 there); on the density workload these fixed
//     weights give the CG counts of power-iteration estimates (12 at
//     512 x 256, 14 at 1024 x 512, emulated in double);
//   * V(1,1) cycle with damped Jacobi (omega 0.9) before and after the
//     coarse correction, a dense inverse on the coarsest level (<= 64
//     unknowns).  The cycle is symmetric, so CG applies.
// Levels with more than kSaCtaCells unknowns (and always level 0) run on the
// whole grid between bounded grid barriers; smaller levels run on CTA 0.
// The CG recurrences, the |p.Ap| < 1e-20 exit and AMGCL's relative stop rule
// ||r|| <= pTol ||b|| are those of k_pcg_mg.
#pragma once

#include "cp_mg.cuh"

namespace cp {

constexpr int kSaMaxLevels = 12;
constexpr int kSaCtaCells = 4096;    // levels at or below this size run on one CTA
constexpr int kSaDense = 64;         // coarsest level size solved by a dense inverse

// A level: unknowns i in [1, nI], j in [1, nJ] with a zero frame, row pitch P.
// Level 0 keeps its 5-point operator as face coefficients (fE, fN, d of the
// PCG buffers); levels >= 1 hold a 9-point stencil c[k], k = (di+1)*3 + (dj+1),
// c[4] the diagonal, entries towards unknowns outside the level zero.
template <typename TV>
struct SaLevel {
    int nI, nJ, P;
    TV* c[9];
    TV *x, *y, *b, *t;      // pre-smoothed iterate, corrected iterate, rhs, scratch
};

template <typename TV>
struct SaHier {
    int L, Lg;              // levels; levels [0, Lg) run grid-wide
    SaLevel<TV> lv[kSaMaxLevels];
    const TV *fE, *fN, *d;  // level-0 operator
    TV* Y[9];               // coloured probes A P e_c (level-0 sized)
    TV* dense;              // inverse of the coarsest operator
    double omega, w0, wc;   // Jacobi damping, prolongator smoothing weights
    unsigned long long* prof;  // optional per-phase device time (ns, block 0's view), or null
};

// profile slots: set-up, Galerkin, CG matvec, CG update, CTA levels, then
// restriction out of level l at SA_P_DOWN + l and prolongation into level l
// at SA_P_UP + l
enum SaPhase { SA_P_SETUP = 0, SA_P_GALERKIN, SA_P_MATVEC, SA_P_UPDATE, SA_P_CTA, SA_P_DOWN, SA_P_UP = SA_P_DOWN + kSaMaxLevels,
               SA_P_COUNT = SA_P_UP + kSaMaxLevels };

__host__ __device__ __forceinline__ int sa_coarse(int n) { return (n + 2) / 3; }

// ---------------------------------------------------------------- stencils
// Coefficient of row (i, j) towards offset k of a level's operator, zero
// towards anything outside [1, nI] x [1, nJ].
template <typename TV>
struct Stencil5 {
    const TV *fE, *fN, *d;
    int nI, nJ, P;
    static constexpr int kN = 5;
    __device__ __forceinline__ static int k_of(int q) { return q == 0 ? 1 : (q == 1 ? 3 : (q == 2 ? 4 : (q == 3 ? 5 : 7))); }
    __device__ __forceinline__ double operator()(int i, int j, int k) const {
        const size_t q = (size_t)i * P + j;
        switch (k) {
            case 4: return (double)d[q];
            case 5: return j < nJ ? -(double)fE[q] : 0.0;
            case 3: return j > 1 ? -(double)fE[q - 1] : 0.0;
            case 7: return i < nI ? -(double)fN[q] : 0.0;
            case 1: return i > 1 ? -(double)fN[q - P] : 0.0;
            default: return 0.0;
        }
    }
};

template <typename TV>
struct Stencil9 {
    TV* const* c;
    int nI, nJ, P;
    static constexpr int kN = 9;
    __device__ __forceinline__ static int k_of(int q) { return q; }
    __device__ __forceinline__ double operator()(int i, int j, int k) const {
        return (double)c[k][(size_t)i * P + j];
    }
};

__device__ __forceinline__ int sa_di(int k) { return k / 3 - 1; }
__device__ __forceinline__ int sa_dj(int k) { return k % 3 - 1; }
// colour of the aggregate that holds unknown (i, j)
__device__ __forceinline__ int sa_colour(int i, int j) { return (((i - 1) / 3) % 3) * 3 + ((j - 1) / 3) % 3; }

struct SaSplit {
    int t0, nt;
};

template <typename F>
__device__ __forceinline__ void sa_cells(SaSplit s, int nI, int nJ, F&& fn) {
    const int n = nI * nJ;
    for (int t = s.t0; t < n; t += s.nt) fn(1 + t / nJ, 1 + t % nJ);
}

// ---------------------------------------------------------------- Galerkin set-up
// Y_c(i, j) = (A P e_c)(i, j) for the nine colours c, where e_c is 1 on the
// coarse unknowns of colour c and (P e_c)(m) = e_c(agg m) - w / d_m
// sum_n A_mn e_c(agg n).
template <typename TV, class St>
__device__ __forceinline__ void sa_probe_cell(const St& A, int P, TV* const* Y, double w, int i, int j) {
    double y[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) y[c] = 0.0;
#pragma unroll
    for (int a = 0; a < St::kN; ++a) {
        const int k = St::k_of(a);
        const int mi = i + sa_di(k), mj = j + sa_dj(k);
        if (mi < 1 || mi > A.nI || mj < 1 || mj > A.nJ) continue;
        const double akm = A(i, j, k);
        if (akm == 0.0) continue;
        const double sc = -akm * w / A(mi, mj, 4);
        const int cm = sa_colour(mi, mj);
#pragma unroll
        for (int c = 0; c < 9; ++c) y[c] += (c == cm) ? akm : 0.0;
#pragma unroll
        for (int b = 0; b < St::kN; ++b) {
            const int kk = St::k_of(b);
            const int ni = mi + sa_di(kk), nj = mj + sa_dj(kk);
            if (ni < 1 || ni > A.nI || nj < 1 || nj > A.nJ) continue;
            const double v = sc * A(mi, mj, kk);
            const int cn = sa_colour(ni, nj);
#pragma unroll
            for (int c = 0; c < 9; ++c) y[c] += (c == cn) ? v : 0.0;
        }
    }
    const size_t q = (size_t)i * P + j;
#pragma unroll
    for (int c = 0; c < 9; ++c) Y[c][q] = (TV)y[c];
}

// P_kI: the smoothed prolongator's entry of fine unknown k for aggregate I
template <class St>
__device__ __forceinline__ double sa_pk(const St& A, int i, int j, int I, int J, double w) {
    auto in_agg = [&](int ii, int jj) { return (ii - 1) / 3 + 1 == I && (jj - 1) / 3 + 1 == J; };
    double s = 0.0;
#pragma unroll
    for (int b = 0; b < St::kN; ++b) {
        const int kk = St::k_of(b);
        const int ni = i + sa_di(kk), nj = j + sa_dj(kk);
        if (ni < 1 || ni > A.nI || nj < 1 || nj > A.nJ) continue;
        if (in_agg(ni, nj)) s += A(i, j, kk);
    }
    return (in_agg(i, j) ? 1.0 : 0.0) - w * s / A(i, j, 4);
}

// coarse row (I, J) of A_c = P^T A P from the probes of the fine level
template <typename TV, class St>
__device__ __forceinline__ void sa_galerkin_cell(const St& A, int Pf, TV* const* Y, const SaLevel<TV>& C, double w,
                                                 int I, int J) {
    double ac[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) ac[c] = 0.0;
    for (int i = 3 * I - 3; i <= 3 * I + 1; ++i) {
        if (i < 1 || i > A.nI) continue;
        for (int j = 3 * J - 3; j <= 3 * J + 1; ++j) {
            if (j < 1 || j > A.nJ) continue;
            const double p = sa_pk(A, i, j, I, J, w);
            if (p == 0.0) continue;
            const size_t q = (size_t)i * Pf + j;
#pragma unroll
            for (int c = 0; c < 9; ++c) ac[c] += p * (double)Y[c][q];
        }
    }
    const size_t qc = (size_t)I * C.P + J;
    const int ai = (I - 1) % 3, aj = (J - 1) % 3;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        // the neighbour of colour c: offsets in {-1, 0, 1} with matching residues
        const int di = ((c / 3 - ai + 4) % 3) - 1, dj = ((c % 3 - aj + 4) % 3) - 1;
        const int k = (di + 1) * 3 + (dj + 1);
        const bool in = I + di >= 1 && I + di <= C.nI && J + dj >= 1 && J + dj <= C.nJ;
        double v = in ? ac[c] : 0.0;
        if (k == 4 && !(v > 0.0)) v = 1.0;   // guard: an isolated coarse unknown
        C.c[k][qc] = (TV)v;
    }
}

// ---------------------------------------------------------------- cycle pieces
// (A v)(i, j) on a level, v zero outside the unknowns (frame) and read only
// inside them
template <typename TV, class St>
__device__ __forceinline__ double sa_av(const St& A, int P, const TV* v, int i, int j) {
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < St::kN; ++a) {
        const int k = St::k_of(a);
        const int ni = i + sa_di(k), nj = j + sa_dj(k);
        if (ni < 1 || ni > A.nI || nj < 1 || nj > A.nJ) continue;
        s += A(i, j, k) * (double)v[(size_t)ni * P + nj];
    }
    return s;
}

// restriction, part 1 (fine unknown): t = r1 = b - A x (x the pre-smoothed
// iterate) and y = r1 / d
template <typename TV, class St>
__device__ __forceinline__ void sa_resid_cell(const St& A, const SaLevel<TV>& f, int i, int j) {
    const size_t q = (size_t)i * f.P + j;
    const double r1 = (double)f.b[q] - sa_av(A, f.P, f.x, i, j);
    f.t[q] = (TV)r1;
    f.y[q] = (TV)(r1 / A(i, j, 4));
}

// restriction, part 2 (coarse unknown): b_c = sum over the aggregate of
// r1 - w A D^-1 r1 (= P^T r1), and the pre-smoothed x_c = omega b_c / d_c
template <typename TV, class St>
__device__ __forceinline__ void sa_restrict_cell(const St& A, const SaLevel<TV>& f, const SaLevel<TV>& C, double w,
                                                 double omega, int I, int J) {
    double s = 0.0;
    for (int i = 3 * I - 2; i <= min(3 * I, f.nI); ++i)
        for (int j = 3 * J - 2; j <= min(3 * J, f.nJ); ++j)
            s += (double)f.t[(size_t)i * f.P + j] - w * sa_av(A, f.P, f.y, i, j);
    const size_t qc = (size_t)I * C.P + J;
    C.b[qc] = (TV)s;
    C.x[qc] = (TV)(omega * s / (double)C.c[4][qc]);
}

// prolongation, part 1 (fine unknown): t = x + P e, e the coarse corrected
// iterate: (P e)(m) = e(agg m) - w / d_m sum_n A_mn e(agg n)
template <typename TV, class St>
__device__ __forceinline__ void sa_prolong_cell(const St& A, const SaLevel<TV>& f, const TV* e, int Pc, double w,
                                                int i, int j) {
    auto e0 = [&](int ii, int jj) -> double { return (double)e[(size_t)((ii - 1) / 3 + 1) * Pc + (jj - 1) / 3 + 1]; };
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < St::kN; ++a) {
        const int k = St::k_of(a);
        const int ni = i + sa_di(k), nj = j + sa_dj(k);
        if (ni < 1 || ni > A.nI || nj < 1 || nj > A.nJ) continue;
        s += A(i, j, k) * e0(ni, nj);
    }
    const size_t q = (size_t)i * f.P + j;
    f.t[q] = (TV)((double)f.x[q] + e0(i, j) - w * s / A(i, j, 4));
}

// prolongation, part 2 (fine unknown): post-smoothing y = t + omega (b - A t) / d
template <typename TV, class St>
__device__ __forceinline__ double sa_smooth_cell(const St& A, const SaLevel<TV>& f, double omega, int i, int j) {
    const size_t q = (size_t)i * f.P + j;
    const double tc = (double)f.t[q];
    const double y = tc + omega * ((double)f.b[q] - sa_av(A, f.P, f.t, i, j)) / A(i, j, 4);
    f.y[q] = (TV)y;
    return y;
}

// dense inverse of the coarsest (9-point) operator by Gauss-Jordan (SPD, no
// pivoting), one CTA
template <typename TV>
__device__ void sa_dense_setup(const SaLevel<TV>& l, TV* inv, double* work /* smem n*2n + n */) {
    const int n = l.nI * l.nJ, w = 2 * n;
    double* fac = work + n * w;
    for (int e = threadIdx.x; e < n * w; e += blockDim.x) work[e] = 0.0;
    __syncthreads();
    Stencil9<TV> A{l.c, l.nI, l.nJ, l.P};
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        const int i = 1 + a / l.nJ, j = 1 + a % l.nJ;
        for (int k = 0; k < 9; ++k) {
            const int ni = i + sa_di(k), nj = j + sa_dj(k);
            if (ni < 1 || ni > l.nI || nj < 1 || nj > l.nJ) continue;
            work[a * w + (ni - 1) * l.nJ + (nj - 1)] = A(i, j, k);
        }
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

// coarsest level: y = A^-1 b
template <typename TV>
__device__ void sa_dense_solve(const SaLevel<TV>& l, const TV* inv) {
    const int n = l.nI * l.nJ;
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        double s = 0.0;
        for (int b2 = 0; b2 < n; ++b2)
            s += (double)inv[a * n + b2] * (double)l.b[(size_t)(1 + b2 / l.nJ) * l.P + 1 + b2 % l.nJ];
        l.y[(size_t)(1 + a / l.nJ) * l.P + 1 + a % l.nJ] = (TV)s;
    }
    __syncthreads();
}

// ---------------------------------------------------------------- the solver
template <typename TV>
__global__ void __launch_bounds__(512, 1) k_pcg_sa(KParams k, Status* st, const double* dE, const double* dN,
                                                PcgBufs<TV> B, SaHier<TV> H, double* pStar, double* part,
                                                unsigned* bar) {
    if (st->done) return;
    extern __shared__ __align__(128) double dsm[];
    __shared__ double sm[96];
    const Dims d = k.d;
    const int M = d.M, N = d.N, w = N - 2;
    const int n = (M - 1) * w;
    const int G = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = G * blockDim.x;
    const SaSplit all{tid, nth}, cta{(int)threadIdx.x, (int)blockDim.x};
    const double rho = k.rho, hx = k.hx, hy = k.hy, om = H.omega;
    unsigned target = 0;
    double* partA = part;
    double* partB = part + G;
#define SA_SYNC()                                                   \
    do {                                                            \
        target += G;                                                \
        if (!grid_barrier(bar, target, &st->err)) return;           \
    } while (0)

    SaLevel<TV> L0 = H.lv[0];
    L0.b = B.r;
    unsigned long long tp = (H.prof && blockIdx.x == 0 && threadIdx.x == 0) ? globaltimer_ns() : 0ull;
    auto tick = [&](int ph) {
        if (H.prof && blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long t = globaltimer_ns();
            atomicAdd(H.prof + ph, t - tp);
            tp = t;
        }
    };
    const Stencil5<TV> A0{B.fE, B.fN, B.d, M - 1, w, d.P};
    auto stencil = [&](int l) { return Stencil9<TV>{H.lv[l].c, H.lv[l].nI, H.lv[l].nJ, H.lv[l].P}; };
    auto lvl = [&](int l) -> const SaLevel<TV>& { return l == 0 ? L0 : H.lv[l]; };
    auto wgt = [&](int l) { return l == 0 ? H.w0 : H.wc; };

    // ---- set-up: level-0 operator (the reference's formulas), x = 0, r = b
    double bb[1] = {0.0};
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        const double aE = rho * dE[c] * hy;
        const double aW = (j > 1) ? rho * dE[c - 1] * hy : 0.0;
        const double aN = (i < M - 1) ? rho * dN[c] * hx : 0.0;
        const double aS = (i > 1) ? rho * dN[c - d.P] * hx : 0.0;
        double aP = aE + aW + aN + aS;
        if (aP < 1e-20) aP = 1.0;
        B.fE[c] = (TV)aE;
        B.fN[c] = (TV)aN;
        B.d[c] = (TV)aP;
        B.x[c] = (TV)0;
        const TV rt = B.rhs[c];
        B.r[c] = rt;
        L0.x[c] = (TV)(om * (double)rt / aP);
        bb[0] += (double)rt * (double)rt;
    }
    block_sum<1>(bb, sm);
    if (threadIdx.x == 0) partA[blockIdx.x] = bb[0];
    SA_SYNC();
    double bnorm2[1];
    sum_partials<1>(partA, G, 1, bnorm2, sm);
    const double rTol = k.pTol * sqrt(bnorm2[0]);
    tick(SA_P_SETUP);

    // ---- set-up: coarse operators by coloured probes
    for (int l = 0; l < H.L - 1; ++l) {
        const bool grid = l < H.Lg;
        if (!grid && blockIdx.x != 0) continue;
        const SaSplit sp = grid ? all : cta;
        const SaLevel<TV>& f = lvl(l);
        if (l == 0) sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_probe_cell(A0, f.P, H.Y, wgt(l), i, j); });
        else sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_probe_cell(stencil(l), f.P, H.Y, wgt(l), i, j); });
        if (grid) SA_SYNC(); else __syncthreads();
        const SaLevel<TV>& C = H.lv[l + 1];
        if (l == 0)
            sa_cells(sp, C.nI, C.nJ, [&](int I, int J) { sa_galerkin_cell(A0, f.P, H.Y, C, wgt(l), I, J); });
        else
            sa_cells(sp, C.nI, C.nJ, [&](int I, int J) { sa_galerkin_cell(stencil(l), f.P, H.Y, C, wgt(l), I, J); });
        if (grid) SA_SYNC(); else __syncthreads();
    }
    if (blockIdx.x == 0) sa_dense_setup(H.lv[H.L - 1], H.dense, dsm);
    SA_SYNC();
    tick(SA_P_GALERKIN);

    // one restriction l -> l+1 (two passes) and one prolongation l+1 -> l
    // with post-smoothing (two passes), on the grid or on CTA 0
    auto restrict_level = [&](int l, bool grid) -> bool {
        const SaSplit sp = grid ? all : cta;
        const SaLevel<TV>& f = lvl(l);
        const SaLevel<TV>& C = H.lv[l + 1];
        if (l == 0) sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_resid_cell(A0, f, i, j); });
        else sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_resid_cell(stencil(l), f, i, j); });
        if (grid) { target += G; if (!grid_barrier(bar, target, &st->err)) return false; } else __syncthreads();
        if (l == 0) sa_cells(sp, C.nI, C.nJ, [&](int I, int J) { sa_restrict_cell(A0, f, C, wgt(l), om, I, J); });
        else sa_cells(sp, C.nI, C.nJ, [&](int I, int J) { sa_restrict_cell(stencil(l), f, C, wgt(l), om, I, J); });
        if (grid) { target += G; if (!grid_barrier(bar, target, &st->err)) return false; } else __syncthreads();
        return true;
    };
    auto prolong_level = [&](int l, bool grid, double* rz) -> bool {
        const SaSplit sp = grid ? all : cta;
        const SaLevel<TV>& f = lvl(l);
        const SaLevel<TV>& C = H.lv[l + 1];
        if (l == 0) sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_prolong_cell(A0, f, C.y, C.P, wgt(l), i, j); });
        else sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_prolong_cell(stencil(l), f, C.y, C.P, wgt(l), i, j); });
        if (grid) { target += G; if (!grid_barrier(bar, target, &st->err)) return false; } else __syncthreads();
        double acc[1] = {0.0};
        if (l == 0)
            sa_cells(sp, f.nI, f.nJ, [&](int i, int j) {
                const double y = sa_smooth_cell(A0, f, om, i, j);
                acc[0] += (double)f.b[(size_t)i * f.P + j] * y;
            });
        else sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_smooth_cell(stencil(l), f, om, i, j); });
        if (rz) {
            block_sum<1>(acc, sm);
            if (threadIdx.x == 0) partB[2 * blockIdx.x + 1] = acc[0];
        }
        if (grid) { target += G; if (!grid_barrier(bar, target, &st->err)) return false; } else __syncthreads();
        return true;
    };
    // ---- z = M r (V-cycle); z in level 0's y, rz = r.z
    auto vcycle = [&](double& rz) -> bool {
        for (int l = 0; l < H.Lg; ++l) {
            if (!restrict_level(l, true)) return false;
            tick(SA_P_DOWN + l);
        }
        if (blockIdx.x == 0) {
            for (int l = H.Lg; l < H.L - 1; ++l) restrict_level(l, false);
            sa_dense_solve(H.lv[H.L - 1], H.dense);
            for (int l = H.L - 2; l >= H.Lg; --l) prolong_level(l, false, nullptr);
        }
        target += G;
        if (!grid_barrier(bar, target, &st->err)) return false;
        tick(SA_P_CTA);
        for (int l = H.Lg - 1; l >= 0; --l) {
            if (!prolong_level(l, true, l == 0 ? &rz : nullptr)) return false;
            tick(SA_P_UP + l);
        }
        double t2[2];
        sum_partials<2>(partB, G, 2, t2, sm);
        rz = t2[1];
        return true;
    };

    double rz = 0.0;
    if (!vcycle(rz)) return;
    double beta = 0.0;
    int it = 0;
    TV* pbuf[2] = {B.pa, B.pb};
    const TV* z = L0.y;
    for (; it < k.maxP; ++it) {
        TV* __restrict__ pnew = pbuf[it & 1];
        const TV* pold = pbuf[(it + 1) & 1];
        const TV bt = (TV)beta;
        const bool first = it == 0;
        auto dir = [&](size_t c) -> TV { return first ? z[c] : (TV)(z[c] + bt * pold[c]); };
        double accA[1] = {0.0};
        for (int t = tid; t < n; t += nth) {
            const int i = 1 + t / w, j = 1 + t % w;
            const size_t c = at(d, i, j);
            const TV pc = dir(c);
            TV ap = B.d[c] * pc;
            if (j < w) ap -= B.fE[c] * dir(c + 1);
            if (j > 1) ap -= B.fE[c - 1] * dir(c - 1);
            if (i < M - 1) ap -= B.fN[c] * dir(c + d.P);
            if (i > 1) ap -= B.fN[c - d.P] * dir(c - d.P);
            pnew[c] = pc;
            B.Ap[c] = ap;
            accA[0] += (double)pc * (double)ap;
        }
        block_sum<1>(accA, sm);
        if (threadIdx.x == 0) partA[blockIdx.x] = accA[0];
        SA_SYNC();
        double pAp[1];
        sum_partials<1>(partA, G, 1, pAp, sm);
        tick(SA_P_MATVEC);
        if (fabs(pAp[0]) < 1e-20) break;
        const double alpha = rz / pAp[0];
        const TV al = (TV)alpha, omT = (TV)om;
        double accB[1] = {0.0};
        for (int t = tid; t < n; t += nth) {
            const size_t c = at(d, 1 + t / w, 1 + t % w);
            B.x[c] = B.x[c] + al * pnew[c];
            const TV r = B.r[c] - al * B.Ap[c];
            B.r[c] = r;
            L0.x[c] = omT * r / B.d[c];
            accB[0] += (double)r * (double)r;
        }
        block_sum<1>(accB, sm);
        if (threadIdx.x == 0) partB[2 * blockIdx.x] = accB[0];
        SA_SYNC();
        double tB[2];
        sum_partials<2>(partB, G, 2, tB, sm);
        tick(SA_P_UPDATE);
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
#undef SA_SYNC
}

}  // namespace cp
