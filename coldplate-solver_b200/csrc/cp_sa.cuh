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
    TV* r2;                 // second CG residual buffer (the residual ping-pongs)
    int reuse;              // rebuild the coarse operators every `reuse` outer iterations
    int force;              // 1: rebuild now and leave the hierarchy marked stale
    int* dirty;             // device flag: the stored hierarchy is not the forward's
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

// ---------------------------------------------------------------- level-0 passes
// Level 0 has the 5-point operator of the face coefficients fE (east), fN
// (north) and the diagonal d.  Its arrays are zero on the frame (only the
// unknowns are ever written), and fE / fN are zero on the frame rows and
// columns, so these passes read neighbours without range checks wherever a
// zero frame value gives the right term.  Arithmetic in TV.
template <typename TV>
struct Sa0 {
    const TV *fE, *fN, *d;
    int nI, nJ, P;
};

// CG matvec on p = z + beta p_old: writes p and Ap, returns p.Ap's share
template <typename TV>
__device__ __forceinline__ double sa0_matvec(const Sa0<TV>& A, const TV* z, const TV* pold, TV bt, bool first,
                                             TV* pnew, TV* Ap, int i, int j) {
    const int c = i * A.P + j;
    auto dir = [&](int q) -> TV { return first ? z[q] : (TV)(z[q] + bt * pold[q]); };
    const TV pc = dir(c);
    const TV ap = A.d[c] * pc - A.fE[c] * dir(c + 1) - A.fE[c - 1] * dir(c - 1) - A.fN[c] * dir(c + A.P) -
                  A.fN[c - A.P] * dir(c - A.P);
    pnew[c] = pc;
    Ap[c] = ap;
    return (double)pc * (double)ap;
}

// CG update fused with the first half of the next restriction:
// x += alpha p, r' = r - alpha Ap (into rn), x0' = omega r' / d (the
// pre-smoothed level-0 iterate), and the residual of the pre-smoothing
// t = r' - A x0' = (1 - omega) r' + sum of the faces' f x0'(neighbour), with
// x0' of the neighbours recomputed from r and Ap; y = t / d.  Returns |r'|^2.
template <typename TV>
__device__ __forceinline__ double sa0_update(const Sa0<TV>& A, TV al, TV om, const TV* p, const TV* Ap, TV* x,
                                             const TV* r, TV* rn, TV* x0, TV* t, TV* y, int i, int j) {
    const int c = i * A.P + j;
    auto x0n = [&](int q) -> TV { return om * (r[q] - al * Ap[q]) / A.d[q]; };
    const TV rc = r[c] - al * Ap[c];
    x[c] = x[c] + al * p[c];
    rn[c] = rc;
    x0[c] = om * rc / A.d[c];
    TV r1 = ((TV)1 - om) * rc;
    if (j < A.nJ) r1 += A.fE[c] * x0n(c + 1);
    if (j > 1) r1 += A.fE[c - 1] * x0n(c - 1);
    if (i < A.nI) r1 += A.fN[c] * x0n(c + A.P);
    if (i > 1) r1 += A.fN[c - A.P] * x0n(c - A.P);
    t[c] = r1;
    y[c] = r1 / A.d[c];
    return (double)rc * (double)rc;
}

// the same residual half for the first cycle (x0 stored already)
template <typename TV>
__device__ __forceinline__ void sa0_resid(const Sa0<TV>& A, TV om, const TV* b, const TV* x0, TV* t, TV* y, int i,
                                          int j) {
    const int c = i * A.P + j;
    const TV r1 = ((TV)1 - om) * b[c] + A.fE[c] * x0[c + 1] + A.fE[c - 1] * x0[c - 1] + A.fN[c] * x0[c + A.P] +
                  A.fN[c - A.P] * x0[c - A.P];
    t[c] = r1;
    y[c] = r1 / A.d[c];
}

// second half of the restriction into level 1, one aggregate:
// b_c = sum over the aggregate of t - w A y, x_c = omega b_c / d_c
template <typename TV>
__device__ __forceinline__ void sa0_restrict(const Sa0<TV>& A, const TV* t, const TV* y, const SaLevel<TV>& C,
                                             TV w, double omega, int I, int J) {
    double s = 0.0;
    const int i1 = min(3 * I, A.nI), j1 = min(3 * J, A.nJ);
    for (int i = 3 * I - 2; i <= i1; ++i)
        for (int j = 3 * J - 2; j <= j1; ++j) {
            const int c = i * A.P + j;
            const TV ay = A.d[c] * y[c] - A.fE[c] * y[c + 1] - A.fE[c - 1] * y[c - 1] - A.fN[c] * y[c + A.P] -
                          A.fN[c - A.P] * y[c - A.P];
            s += (double)(t[c] - w * ay);
        }
    const int qc = I * C.P + J;
    C.b[qc] = (TV)s;
    C.x[qc] = (TV)(omega * s / (double)C.c[4][qc]);
}

// prolongation from level 1 fused with the post-smoothing of level 0:
// t = x0 + P e at the cell and its four neighbours ((P e)(m) = e(agg m) -
// w / d_m (A e0)(m)), then y = t + omega (b - A t) / d.  Returns y.
template <typename TV>
__device__ __forceinline__ TV sa0_prolong(const Sa0<TV>& A, const TV* x0, const TV* b, const TV* e, int Pc, TV w,
                                          TV om, int i, int j) {
    auto E0 = [&](int ii, int jj) -> TV {
        if (ii < 1 || ii > A.nI || jj < 1 || jj > A.nJ) return (TV)0;
        return e[((ii - 1) / 3 + 1) * Pc + (jj - 1) / 3 + 1];
    };
    auto T = [&](int ii, int jj) -> TV {
        if (ii < 1 || ii > A.nI || jj < 1 || jj > A.nJ) return (TV)0;
        const int q = ii * A.P + jj;
        const TV ec = E0(ii, jj);
        const TV ae = A.d[q] * ec - A.fE[q] * E0(ii, jj + 1) - A.fE[q - 1] * E0(ii, jj - 1) -
                      A.fN[q] * E0(ii + 1, jj) - A.fN[q - A.P] * E0(ii - 1, jj);
        return x0[q] + ec - w * ae / A.d[q];
    };
    const int c = i * A.P + j;
    const TV tc = T(i, j);
    const TV at = A.d[c] * tc - A.fE[c] * T(i, j + 1) - A.fE[c - 1] * T(i, j - 1) - A.fN[c] * T(i + 1, j) -
                  A.fN[c - A.P] * T(i - 1, j);
    return tc + om * (b[c] - at) / A.d[c];
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
    const TV omT = (TV)om, w0T = (TV)H.w0;
    unsigned target = 0;
    double* partA = part;
    double* partB = part + G;
#define SA_SYNC()                                                   \
    do {                                                            \
        target += G;                                                \
        if (!grid_barrier(bar, target, &st->err)) return;           \
    } while (0)
    // the coarse operators are rebuilt every H.reuse outer iterations (they
    // only precondition: the CG matvec always uses the current level 0), and
    // whenever the stored ones are not the forward's
    const bool rebuild = H.force || *(volatile int*)H.dirty || H.reuse <= 1 || (st->iter % H.reuse) == 0;

    SaLevel<TV> L0 = H.lv[0];
    L0.b = B.r;
    const Sa0<TV> A0f{B.fE, B.fN, B.d, M - 1, w, d.P};
    const Stencil5<TV> A0{B.fE, B.fN, B.d, M - 1, w, d.P};
    auto stencil = [&](int l) { return Stencil9<TV>{H.lv[l].c, H.lv[l].nI, H.lv[l].nJ, H.lv[l].P}; };
    auto wgt = [&](int l) { return l == 0 ? H.w0 : H.wc; };
    unsigned long long tp = (H.prof && blockIdx.x == 0 && threadIdx.x == 0) ? globaltimer_ns() : 0ull;
    auto tick = [&](int ph) {
        if (H.prof && blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long t = globaltimer_ns();
            atomicAdd(H.prof + ph, t - tp);
            tp = t;
        }
    };

    // ---- set-up: level-0 operator (the reference's formulas), x = 0, r = b,
    // x0 = omega r / d
    double bb[1] = {0.0};
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const int c = i * d.P + j;
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

    // ---- set-up: coarse operators by coloured probes (when rebuilt)
    if (rebuild) {
        for (int l = 0; l < H.L - 1; ++l) {
            const bool grid = l < H.Lg;
            if (!grid && blockIdx.x != 0) continue;
            const SaSplit sp = grid ? all : cta;
            const SaLevel<TV>& f = H.lv[l];
            if (l == 0) sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_probe_cell(A0, f.P, H.Y, wgt(l), i, j); });
            else sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_probe_cell(stencil(l), f.P, H.Y, wgt(l), i, j); });
            if (grid) SA_SYNC(); else __syncthreads();
            const SaLevel<TV>& C = H.lv[l + 1];
            if (l == 0)
                sa_cells(sp, C.nI, C.nJ, [&](int I, int J) { sa_galerkin_cell(A0, f.P, H.Y, C, wgt(l), I, J); });
            else
                sa_cells(sp, C.nI, C.nJ,
                         [&](int I, int J) { sa_galerkin_cell(stencil(l), f.P, H.Y, C, wgt(l), I, J); });
            if (grid) SA_SYNC(); else __syncthreads();
        }
        if (blockIdx.x == 0) sa_dense_setup(H.lv[H.L - 1], H.dense, dsm);
        SA_SYNC();
    }
    tick(SA_P_GALERKIN);

    // levels >= 1: restriction l -> l+1 and prolongation l+1 -> l with
    // post-smoothing, two passes each, on the grid or on CTA 0
    auto restrict_level = [&](int l, bool grid) -> bool {
        const SaSplit sp = grid ? all : cta;
        const SaLevel<TV>& f = H.lv[l];
        const SaLevel<TV>& C = H.lv[l + 1];
        sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_resid_cell(stencil(l), f, i, j); });
        if (grid) { target += G; if (!grid_barrier(bar, target, &st->err)) return false; } else __syncthreads();
        sa_cells(sp, C.nI, C.nJ, [&](int I, int J) { sa_restrict_cell(stencil(l), f, C, wgt(l), om, I, J); });
        if (grid) { target += G; if (!grid_barrier(bar, target, &st->err)) return false; } else __syncthreads();
        return true;
    };
    auto prolong_level = [&](int l, bool grid) -> bool {
        const SaSplit sp = grid ? all : cta;
        const SaLevel<TV>& f = H.lv[l];
        const SaLevel<TV>& C = H.lv[l + 1];
        sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_prolong_cell(stencil(l), f, C.y, C.P, wgt(l), i, j); });
        if (grid) { target += G; if (!grid_barrier(bar, target, &st->err)) return false; } else __syncthreads();
        sa_cells(sp, f.nI, f.nJ, [&](int i, int j) { sa_smooth_cell(stencil(l), f, om, i, j); });
        if (grid) { target += G; if (!grid_barrier(bar, target, &st->err)) return false; } else __syncthreads();
        return true;
    };
    // ---- z = M r (V-cycle) with r = L0.b; level 0's residual half (t, y)
    // is done already (by the CG update, or by `first`); z in L0.y is
    // overwritten by the prolongation; rz = r.z
    const SaLevel<TV>& C1 = H.lv[1];
    auto vcycle = [&](double& rz, bool first) -> bool {
        if (first) {
            sa_cells(all, L0.nI, L0.nJ, [&](int i, int j) { sa0_resid(A0f, omT, L0.b, L0.x, L0.t, L0.y, i, j); });
            target += G;
            if (!grid_barrier(bar, target, &st->err)) return false;
        }
        sa_cells(all, C1.nI, C1.nJ, [&](int I, int J) { sa0_restrict(A0f, L0.t, L0.y, C1, w0T, om, I, J); });
        target += G;
        if (!grid_barrier(bar, target, &st->err)) return false;
        tick(SA_P_DOWN);
        for (int l = 1; l < H.Lg; ++l) {
            if (!restrict_level(l, true)) return false;
            tick(SA_P_DOWN + l);
        }
        if (blockIdx.x == 0) {
            for (int l = H.Lg; l < H.L - 1; ++l) restrict_level(l, false);
            sa_dense_solve(H.lv[H.L - 1], H.dense);
            for (int l = H.L - 2; l >= H.Lg; --l) prolong_level(l, false);
        }
        target += G;
        if (!grid_barrier(bar, target, &st->err)) return false;
        tick(SA_P_CTA);
        for (int l = H.Lg - 1; l >= 1; --l) {
            if (!prolong_level(l, true)) return false;
            tick(SA_P_UP + l);
        }
        double acc[1] = {0.0};
        sa_cells(all, L0.nI, L0.nJ, [&](int i, int j) {
            const TV y = sa0_prolong(A0f, L0.x, L0.b, C1.y, C1.P, w0T, omT, i, j);
            const int c = i * L0.P + j;
            L0.y[c] = y;
            acc[0] += (double)L0.b[c] * (double)y;
        });
        block_sum<1>(acc, sm);
        if (threadIdx.x == 0) partB[2 * blockIdx.x + 1] = acc[0];
        target += G;
        if (!grid_barrier(bar, target, &st->err)) return false;
        double t2[2];
        sum_partials<2>(partB, G, 2, t2, sm);
        rz = t2[1];
        tick(SA_P_UP);
        return true;
    };

    double rz = 0.0;
    if (!vcycle(rz, true)) return;
    double beta = 0.0;
    int it = 0;
    TV* pbuf[2] = {B.pa, B.pb};
    TV* rbuf[2] = {B.r, H.r2};
    for (; it < k.maxP; ++it) {
        TV* __restrict__ pnew = pbuf[it & 1];
        const TV* pold = pbuf[(it + 1) & 1];
        const TV bt = (TV)beta;
        const bool first = it == 0;
        double accA[1] = {0.0};
        sa_cells(all, L0.nI, L0.nJ,
                 [&](int i, int j) { accA[0] += sa0_matvec(A0f, L0.y, pold, bt, first, pnew, B.Ap, i, j); });
        block_sum<1>(accA, sm);
        if (threadIdx.x == 0) partA[blockIdx.x] = accA[0];
        SA_SYNC();
        double pAp[1];
        sum_partials<1>(partA, G, 1, pAp, sm);
        tick(SA_P_MATVEC);
        if (fabs(pAp[0]) < 1e-20) break;
        const TV al = (TV)(rz / pAp[0]);
        const TV* rold = rbuf[it & 1];
        TV* rnew = rbuf[(it + 1) & 1];
        double accB[1] = {0.0};
        sa_cells(all, L0.nI, L0.nJ, [&](int i, int j) {
            accB[0] += sa0_update(A0f, al, omT, pnew, B.Ap, B.x, rold, rnew, L0.x, L0.t, L0.y, i, j);
        });
        L0.b = rnew;
        block_sum<1>(accB, sm);
        if (threadIdx.x == 0) partB[2 * blockIdx.x] = accB[0];
        SA_SYNC();
        double tB[2];
        sum_partials<2>(partB, G, 2, tB, sm);
        tick(SA_P_UPDATE);
        if (sqrt(tB[0]) <= rTol) { ++it; break; }
        double rzn = 0.0;
        if (!vcycle(rzn, false)) return;
        beta = rzn / rz;
        rz = rzn;
    }
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const int c = i * d.P + j;
        pStar[c] = (double)B.x[c];
        if (j == w) pStar[c + 1] = 0.0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->itersP = it;
        if (H.force) *H.dirty = 1;
        else if (rebuild) *H.dirty = 0;
    }
#undef SA_SYNC
}

}  // namespace cp
