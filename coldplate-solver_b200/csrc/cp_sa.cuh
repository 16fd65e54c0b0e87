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
// A row of P has at most four entries: the unknown's own aggregate and the
// aggregates across its horizontal, vertical and diagonal neighbours (none
// diagonal on the 5-point level 0).  Level 0 and the grid-wide coarse levels
// store these weights, so the restriction P^T t is a weighted sum over the
// 5 x 5 support and the prolongation four multiply-adds per unknown.
// Level 0 runs its CG passes on row segments: a warp takes 32 groups of 16
// bytes (4 floats or 2 doubles) of one row, with vector loads of the row and
// of its two neighbour rows and the horizontal neighbours from the adjacent
// lanes.  Levels with more than kSaCtaCells unknowns, or too many to stage,
// run on the whole grid between bounded grid barriers; the rest (and the
// dense inverse) are copied into CTA 0's shared memory once per launch and
// cycled there.  The coarse operators are rebuilt every `reuse` outer
// iterations; the CG matvec and level 0's smoother and prolongation always
// use the current operator.  The CG recurrences, the |p.Ap| < 1e-20 exit and
// AMGCL's relative stop rule ||r|| <= pTol ||b|| are those of k_pcg_mg.
#pragma once

#include "cp_mg.cuh"

namespace cp {

constexpr int kSaMaxLevels = 12;
constexpr int kSaCtaCells = 4096;    // levels at or below this size may run on one CTA
constexpr int kSaDense = 64;         // coarsest level size solved by a dense inverse
constexpr size_t kSaSmemBudget = 200 * 1024;   // CTA 0's staged levels and dense inverse

// A level: unknowns i in [1, nI], j in [1, nJ] with a zero frame, row pitch P.
// Level 0 keeps its 5-point operator as face coefficients (fE, fN, d of the
// PCG buffers); levels >= 1 hold a 9-point stencil c[k], k = (di+1)*3 + (dj+1),
// c[4] the diagonal, entries towards unknowns outside the level zero.
// pw[0..3]: the prolongation weights of each unknown towards its own,
// horizontal, vertical and diagonal aggregate (level 0 and grid-wide levels
// that have a coarser one; zero on the frame).
template <typename TV>
struct SaLevel {
    int nI, nJ, P;
    TV* c[9];
    TV *x, *y, *b, *t;      // pre-smoothed iterate, corrected iterate, rhs, scratch
    TV* pw[4];
};

template <typename TV>
struct SaHier {
    int L, Lg;              // levels; levels [0, Lg) run grid-wide, [Lg, L) on CTA 0
    SaLevel<TV> lv[kSaMaxLevels];
    TV* dinv0;              // level-0 inverse diagonal
    TV* Y[9];               // coloured probes A P e_c (level-0 sized)
    TV* dense;              // inverse of the coarsest operator
    double omega, w0, wc;   // Jacobi damping, prolongator smoothing weights
    TV* r2;                 // second CG residual buffer (the residual ping-pongs)
    int reuse;              // rebuild the coarse operators every `reuse` outer iterations (0: only when
                            // the flag says they are stale)
    int* dirty;             // device flag: the stored hierarchy is stale (cleared by a rebuild)
    unsigned long long* prof;  // optional per-phase device time (ns, block 0's view), or null
};

// profile slots: set-up, Galerkin, CG matvec, CG update, CTA levels, then
// restriction out of level l at SA_P_DOWN + l and prolongation into level l
// at SA_P_UP + l
enum SaPhase { SA_P_SETUP = 0, SA_P_GALERKIN, SA_P_MATVEC, SA_P_UPDATE, SA_P_CTA, SA_P_DOWN, SA_P_UP = SA_P_DOWN + kSaMaxLevels,
               SA_P_COUNT = SA_P_UP + kSaMaxLevels };

// shared-memory elements of levels [Lg, L) staged on CTA 0 (13 arrays of
// (nI + 2) x (nJ + 2) each) plus the dense inverse of level L - 1
__host__ __device__ inline size_t sa_cta_elems(const int* nI, const int* nJ, int Lg, int L) {
    size_t e = 0;
    for (int l = Lg; l < L; ++l) e += 13 * (size_t)(nI[l] + 2) * (nJ[l] + 2);
    const size_t n = (size_t)nI[L - 1] * nJ[L - 1];
    return e + n * n;
}

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

// cells t0, t0 + nt, ... of a level in row-major order, (i, j) stepped
// without a division per cell
template <typename F>
__device__ __forceinline__ void sa_cells(SaSplit s, int nI, int nJ, F&& fn) {
    const int n = nI * nJ;
    if (s.t0 >= n) return;
    int i = 1 + s.t0 / nJ, j = 1 + s.t0 % nJ;
    const int di = s.nt / nJ, dj = s.nt % nJ;
    for (int t = s.t0; t < n; t += s.nt) {
        fn(i, j);
        i += di;
        j += dj;
        if (j > nJ) {
            j -= nJ;
            ++i;
        }
    }
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

// coarse row (I, J) from its entries towards the coarse unknowns of each
// colour c (the colour-c neighbour sits at offsets in {-1, 0, 1} with
// matching residues)
template <typename TV>
__device__ __forceinline__ void sa_store_row(const SaLevel<TV>& C, int I, int J, const double (&ac)[9]) {
    const size_t qc = (size_t)I * C.P + J;
    const int ai = (I - 1) % 3, aj = (J - 1) % 3;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        const int di = ((c / 3 - ai + 4) % 3) - 1, dj = ((c % 3 - aj + 4) % 3) - 1;
        const int k = (di + 1) * 3 + (dj + 1);
        const bool in = I + di >= 1 && I + di <= C.nI && J + dj >= 1 && J + dj <= C.nJ;
        double v = in ? ac[c] : 0.0;
        if (k == 4 && !(v > 0.0)) v = 1.0;   // guard: an isolated coarse unknown
        C.c[k][qc] = (TV)v;
    }
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
    sa_store_row(C, I, J, ac);
}

// ---------------------------------------------------------------- prolongation weights
// Offset (-1, 0 or +1) of the aggregate across a fine unknown's horizontal
// (vertical) neighbours when it sits on the first or last column (row) of its
// aggregate; 0 in the middle one.
__device__ __forceinline__ int sa_side(int i) {
    const int r = (i - 1) % 3;
    return r == 0 ? -1 : (r == 2 ? 1 : 0);
}

// Row (i, j) of P = (I - w D^-1 A) P0: pw[0] towards the own aggregate,
// pw[1] / pw[2] / pw[3] towards the horizontal / vertical / diagonal one
// (sa_pk's entries, grouped by aggregate).
template <class St>
__device__ __forceinline__ void sa_pweights(const St& A, int i, int j, double w, double (&pw)[4]) {
    const int ri = (i - 1) % 3, rj = (j - 1) % 3;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int a = 0; a < St::kN; ++a) {
        const int k = St::k_of(a);
        const int di = sa_di(k), dj = sa_dj(k);
        const int ni = i + di, nj = j + dj;
        if (ni < 1 || ni > A.nI || nj < 1 || nj > A.nJ) continue;
        const bool oi = ri + di < 0 || ri + di > 2, oj = rj + dj < 0 || rj + dj > 2;
        s[(oi ? 2 : 0) + (oj ? 1 : 0)] += A(i, j, k);
    }
    const double sc = w / A(i, j, 4);
    pw[0] = 1.0 - sc * s[0];
    pw[1] = -sc * s[1];
    pw[2] = -sc * s[2];
    pw[3] = -sc * s[3];
}

// The same probes and Galerkin rows from the stored prolongation weights of
// the fine level f (its own, horizontal, vertical and diagonal aggregate;
// Diag false on the 5-point level 0, which has no diagonal weight):
// Y_c(i, j) = sum over the stencil of A_(ij),m P(m, agg) [colour(agg) = c],
// and row (I, J) = sum over the 5 x 5 support of P(m, (I, J)) Y_c(m).
template <typename TV, class St, bool Diag>
__device__ __forceinline__ void sa_probe_w(const St& A, const SaLevel<TV>& f, TV* const* Y, int i, int j) {
    double y[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) y[c] = 0.0;
    auto add = [&](int cc, double v) {
#pragma unroll
        for (int c = 0; c < 9; ++c) y[c] += (c == cc) ? v : 0.0;
    };
#pragma unroll
    for (int a = 0; a < St::kN; ++a) {
        const int k = St::k_of(a);
        const int mi = i + sa_di(k), mj = j + sa_dj(k);
        if (mi < 1 || mi > A.nI || mj < 1 || mj > A.nJ) continue;
        const double akm = A(i, j, k);
        if (akm == 0.0) continue;
        const size_t qm = (size_t)mi * f.P + mj;
        const int ci = (mi - 1) / 3 % 3, cj = (mj - 1) / 3 % 3;
        const int cjh = (cj + sa_side(mj) + 3) % 3, civ = (ci + sa_side(mi) + 3) % 3;
        add(ci * 3 + cj, akm * (double)f.pw[0][qm]);
        add(ci * 3 + cjh, akm * (double)f.pw[1][qm]);
        add(civ * 3 + cj, akm * (double)f.pw[2][qm]);
        if (Diag) add(civ * 3 + cjh, akm * (double)f.pw[3][qm]);
    }
    const size_t q = (size_t)i * f.P + j;
#pragma unroll
    for (int c = 0; c < 9; ++c) Y[c][q] = (TV)y[c];
}
template <typename TV, bool Corners>
__device__ __forceinline__ void sa_galerkin_w(const SaLevel<TV>& f, TV* const* Y, const SaLevel<TV>& C, int I,
                                              int J) {
    double ac[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) ac[c] = 0.0;
    const int i0 = 3 * I - 3, j0 = 3 * J - 3;
#pragma unroll
    for (int a = 0; a < 5; ++a) {
        const int ii = i0 + a;
        const int ra = (a == 0 || a == 4) ? 1 : 0;
#pragma unroll
        for (int b = 0; b < 5; ++b) {
            const int rb = (b == 0 || b == 4) ? 1 : 0;
            if (!Corners && ra && rb) continue;
            const int jj = j0 + b;
            if (ii < 1 || ii > f.nI || jj < 1 || jj > f.nJ) continue;
            const size_t q = (size_t)ii * f.P + jj;
            const double p = (double)f.pw[2 * ra + rb][q];
#pragma unroll
            for (int c = 0; c < 9; ++c) ac[c] += p * (double)Y[c][q];
        }
    }
    sa_store_row(C, I, J, ac);
}

// ---------------------------------------------------------------- cycle pieces
// (A v) at q = (i, j) of a coarse level whose c[k] and v are zero on the
// frame (the stencil towards outside the level is zero), without range checks
template <typename TV>
__device__ __forceinline__ double sa9_av(const SaLevel<TV>& f, const TV* v, size_t q) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k)
        s += (double)f.c[k][q] * (double)v[(ptrdiff_t)q + (k / 3 - 1) * (ptrdiff_t)f.P + (k % 3 - 1)];
    return s;
}

// restriction, part 1 (fine unknown of a grid-wide coarse level):
// t = r1 = b - A x (x the pre-smoothed iterate)
template <typename TV>
__device__ __forceinline__ void sa_resid_cell(const SaLevel<TV>& f, int i, int j) {
    const size_t q = (size_t)i * f.P + j;
    f.t[q] = (TV)((double)f.b[q] - sa9_av(f, f.x, q));
}

// restriction, part 2 with stored weights (coarse unknown of a 9-point
// level): b_c = (P^T t)_c over the aggregate's 5 x 5 support (the ring rows
// / columns weigh in with their vertical / horizontal / diagonal weights),
// and the pre-smoothed x_c = omega b_c / d_c
template <typename TV>
__device__ __forceinline__ void sa_restrict_w(const SaLevel<TV>& f, const SaLevel<TV>& C, double omega, int I,
                                              int J) {
    const int i0 = 3 * I - 3, j0 = 3 * J - 3;
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 5; ++a) {
        const int ii = i0 + a;
        const int ra = (a == 0 || a == 4) ? 1 : 0;
#pragma unroll
        for (int b = 0; b < 5; ++b) {
            const int rb = (b == 0 || b == 4) ? 1 : 0;
            const int jj = j0 + b;
            if (ii < 1 || ii > f.nI || jj < 1 || jj > f.nJ) continue;
            const size_t q = (size_t)ii * f.P + jj;
            s += (double)f.pw[2 * ra + rb][q] * (double)f.t[q];
        }
    }
    const size_t qc = (size_t)I * C.P + J;
    C.b[qc] = (TV)s;
    C.x[qc] = (TV)(omega * s / (double)C.c[4][qc]);
}

// prolongation, part 1 with stored weights (fine unknown): t = x + P e
template <typename TV>
__device__ __forceinline__ void sa_prolong_w(const SaLevel<TV>& f, const TV* e, int Pc, int i, int j) {
    const size_t q = (size_t)i * f.P + j;
    const int sh = sa_side(j), sv = sa_side(i) * Pc;
    const TV* er = e + (size_t)((i - 1) / 3 + 1) * Pc + (j - 1) / 3 + 1;
    const double t = (double)f.x[q] + (double)f.pw[0][q] * (double)er[0] + (double)f.pw[1][q] * (double)er[sh] +
                     (double)f.pw[2][q] * (double)er[sv] + (double)f.pw[3][q] * (double)er[sv + sh];
    f.t[q] = (TV)t;
}

// prolongation, part 2 (fine unknown of a grid-wide coarse level):
// post-smoothing y = t + omega (b - A t) / d
template <typename TV>
__device__ __forceinline__ void sa_smooth_cell(const SaLevel<TV>& f, double omega, int i, int j) {
    const size_t q = (size_t)i * f.P + j;
    const double tc = (double)f.t[q];
    f.y[q] = (TV)(tc + omega * ((double)f.b[q] - sa9_av(f, f.t, q)) / (double)f.c[4][q]);
}

// ---------------------------------------------------------------- CTA 0's levels
// A level staged in CTA 0's shared memory: 13 arrays of ne = (nI + 2) x
// (nJ + 2) elements from s (c[0..8], x, y, b, t), frames included (zero
// outside the unknowns, like the stencil towards them), pitch nJ + 2.  The
// passes run without range checks, with arithmetic in TV; P is applied
// through the operator (t - w A D^-1 t summed over the aggregate, and
// e(agg) - w D^-1 A e(agg)).
template <typename TV>
struct SaSm {
    TV* s;
    int nI, nJ, P, ne;
    __device__ __forceinline__ TV* c(int k) const { return s + k * ne; }
    __device__ __forceinline__ TV* x() const { return s + 9 * ne; }
    __device__ __forceinline__ TV* y() const { return s + 10 * ne; }
    __device__ __forceinline__ TV* b() const { return s + 11 * ne; }
    __device__ __forceinline__ TV* t() const { return s + 12 * ne; }
};

// level l of the staged levels [Lg, L) at dsm
template <typename TV>
__device__ __forceinline__ SaSm<TV> sa_sm(const SaHier<TV>& H, TV* dsm, int l) {
    int off = 0;
    for (int m = H.Lg; m < l; ++m) off += 13 * (H.lv[m].nI + 2) * (H.lv[m].nJ + 2);
    const int nI = H.lv[l].nI, nJ = H.lv[l].nJ;
    return SaSm<TV>{dsm + off, nI, nJ, nJ + 2, (nI + 2) * (nJ + 2)};
}

template <typename TV>
__device__ __forceinline__ TV sa_sm_av(const SaSm<TV>& f, const TV* v, int q) {
    TV s = (TV)0;
#pragma unroll
    for (int k = 0; k < 9; ++k) s += f.s[k * f.ne + q] * v[q + (k / 3 - 1) * f.P + (k % 3 - 1)];
    return s;
}

// restriction out of a staged level: t = b - A x, y = t / d; then
// t <- t - w A y; then per coarse unknown b_c = sum of t over the aggregate,
// x_c = omega b_c / d_c
template <typename TV>
__device__ __forceinline__ void sa_sm_resid(const SaSm<TV>& f, int i, int j) {
    const int q = i * f.P + j;
    const TV r1 = f.b()[q] - sa_sm_av(f, f.x(), q);
    f.t()[q] = r1;
    f.y()[q] = r1 / f.s[4 * f.ne + q];
}
template <typename TV>
__device__ __forceinline__ void sa_sm_smoothres(const SaSm<TV>& f, TV w, int i, int j) {
    const int q = i * f.P + j;
    f.t()[q] -= w * sa_sm_av(f, f.y(), q);
}
template <typename TV>
__device__ __forceinline__ void sa_sm_aggsum(const SaSm<TV>& f, const SaSm<TV>& C, TV omega, int I, int J) {
    TV s = (TV)0;
    const int i1 = min(3 * I, f.nI), j1 = min(3 * J, f.nJ);
    for (int i = 3 * I - 2; i <= i1; ++i)
        for (int j = 3 * J - 2; j <= j1; ++j) s += f.t()[i * f.P + j];
    const int qc = I * C.P + J;
    C.b()[qc] = s;
    C.x()[qc] = omega * s / C.s[4 * C.ne + qc];
}
// prolongation into a staged level: t = x + P e, then y = t + omega (b - A t) / d
template <typename TV>
__device__ __forceinline__ void sa_sm_prolong(const SaSm<TV>& f, const SaSm<TV>& C, TV w, int i, int j) {
    const int q = i * f.P + j;
    const TV* e = C.y();
    auto e0 = [&](int ii, int jj) -> TV { return e[((ii - 1) / 3 + 1) * C.P + (jj - 1) / 3 + 1]; };
    TV s = (TV)0;
#pragma unroll
    for (int k = 0; k < 9; ++k) s += f.s[k * f.ne + q] * e0(i + k / 3 - 1, j + k % 3 - 1);
    f.t()[q] = f.x()[q] + e0(i, j) - w * s / f.s[4 * f.ne + q];
}
template <typename TV>
__device__ __forceinline__ void sa_sm_smooth(const SaSm<TV>& f, TV omega, int i, int j) {
    const int q = i * f.P + j;
    const TV tc = f.t()[q];
    f.y()[q] = tc + omega * (f.b()[q] - sa_sm_av(f, f.t(), q)) / f.s[4 * f.ne + q];
}
// coarsest staged level: y = A^-1 b with the staged dense inverse (b is
// gathered into t first)
template <typename TV>
__device__ __forceinline__ void sa_sm_dense(const SaSm<TV>& l, const TV* inv) {
    const int n = l.nI * l.nJ;
    TV* bv = l.t();
    for (int a = threadIdx.x; a < n; a += blockDim.x) bv[a] = l.b()[(1 + a / l.nJ) * l.P + 1 + a % l.nJ];
    __syncthreads();
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        TV s = (TV)0;
        for (int b2 = 0; b2 < n; ++b2) s += inv[a * n + b2] * bv[b2];
        l.y()[(1 + a / l.nJ) * l.P + 1 + a % l.nJ] = s;
    }
    __syncthreads();
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

// ---------------------------------------------------------------- level 0
// Level 0's operator: face coefficients fE (east), fN (north), the diagonal
// d, its inverse and the prolongation weights towards the own, horizontal and
// vertical aggregate.  Every level-0 array is zero on the frame (only the
// unknowns are ever written) and fE / fN are zero on the frame rows and
// columns, so the passes read neighbours without range checks wherever a zero
// frame value gives the right term.  Arithmetic in TV.
template <typename TV>
struct Sa0 {
    const TV *fE, *fN, *d, *dinv, *pO, *pH, *pV;
    int nI, nJ, P;
};

// CG matvec on p = z + beta p_old (p_old unused when first): writes p and Ap
// on one lane group, returns the group's share of p.Ap
template <typename TV>
__device__ __forceinline__ double sa0_matvec(const Sa0<TV>& A, const TV* __restrict__ z, const TV* __restrict__ pold,
                                             TV bt, bool first, TV* __restrict__ pnew, TV* __restrict__ Ap, int i,
                                             int j0, bool act, int lane) {
    constexpr int V = Vec16<TV>::n;
    const int P = A.P, c = i * P + j0;
    auto dir = [&](int q) -> TV { return first ? z[q] : (TV)(z[q] + bt * pold[q]); };
    auto dirv = [&](int q) -> Vec16<TV> {
        Vec16<TV> a = ld16(z + q);
        if (!first) {
            const Vec16<TV> o = ld16(pold + q);
#pragma unroll
            for (int k = 0; k < V; ++k) a.v[k] = (TV)(a.v[k] + bt * o.v[k]);
        }
        return a;
    };
    Vec16<TV> pc = zero16<TV>(), pn = pc, ps = pc, d = pc, fe = pc, fn = pc, fs = pc;
    if (act) {
        pc = dirv(c);
        pn = dirv(c + P);
        ps = dirv(c - P);
        d = ld16(A.d + c);
        fe = ld16(A.fE + c);
        fn = ld16(A.fN + c);
        fs = ld16(A.fN + c - P);
    }
    TV pw = from_west(pc.v[V - 1]), pe = from_east(pc.v[0]), fw = from_west(fe.v[V - 1]);
    if (lane == 0) {
        const bool h = act && j0 > 0;
        pw = h ? dir(c - 1) : (TV)0;
        fw = h ? A.fE[c - 1] : (TV)0;
    }
    if (lane == 31) pe = act ? dir(c + V) : (TV)0;
    Vec16<TV> ap;
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const TV W = k ? pc.v[k - 1] : pw, E = k < V - 1 ? pc.v[k + 1] : pe, FW = k ? fe.v[k - 1] : fw;
        TV a = d.v[k] * pc.v[k] - fe.v[k] * E - FW * W - fn.v[k] * pn.v[k] - fs.v[k] * ps.v[k];
        if (j0 + k < 1 || j0 + k > A.nJ) a = (TV)0;
        ap.v[k] = a;
        acc += (double)pc.v[k] * (double)a;
    }
    if (act) {
        st16(pnew + c, pc);
        st16(Ap + c, ap);
    }
    return acc;
}

// CG update fused with the first half of the next restriction: x += alpha p,
// r' = r - alpha Ap (into rn), the pre-smoothed level-0 iterate
// x0' = omega r' / d, and the residual of the pre-smoothing
// t = r' - A x0' = (1 - omega) r' + sum over the faces of f x0'(neighbour),
// the neighbours' x0' recomputed from r and Ap.  Returns the group's |r'|^2.
template <typename TV>
__device__ __forceinline__ double sa0_update(const Sa0<TV>& A, TV al, TV om, const TV* __restrict__ p,
                                             const TV* __restrict__ Ap, TV* __restrict__ x, const TV* __restrict__ r,
                                             TV* __restrict__ rn, TV* __restrict__ x0, TV* __restrict__ t, int i,
                                             int j0, bool act, int lane) {
    constexpr int V = Vec16<TV>::n;
    const int P = A.P, c = i * P + j0;
    auto x0at = [&](int q) -> TV { return om * (r[q] - al * Ap[q]) * A.dinv[q]; };
    auto x0v = [&](int q) -> Vec16<TV> {
        const Vec16<TV> rr = ld16(r + q), aa = ld16(Ap + q), di = ld16(A.dinv + q);
        Vec16<TV> o;
#pragma unroll
        for (int k = 0; k < V; ++k) o.v[k] = om * (rr.v[k] - al * aa.v[k]) * di.v[k];
        return o;
    };
    Vec16<TV> rc = zero16<TV>(), xc = rc, xn = rc, xs = rc, xx = rc, pp = rc, fe = rc, fn = rc, fs = rc;
    if (act) {
        const Vec16<TV> rr = ld16(r + c), aa = ld16(Ap + c), di = ld16(A.dinv + c);
#pragma unroll
        for (int k = 0; k < V; ++k) {
            rc.v[k] = rr.v[k] - al * aa.v[k];
            xc.v[k] = om * rc.v[k] * di.v[k];
        }
        xn = x0v(c + P);
        xs = x0v(c - P);
        xx = ld16(x + c);
        pp = ld16(p + c);
        fe = ld16(A.fE + c);
        fn = ld16(A.fN + c);
        fs = ld16(A.fN + c - P);
    }
    TV xw = from_west(xc.v[V - 1]), xe = from_east(xc.v[0]), fw = from_west(fe.v[V - 1]);
    if (lane == 0) {
        const bool h = act && j0 > 0;
        xw = h ? x0at(c - 1) : (TV)0;
        fw = h ? A.fE[c - 1] : (TV)0;
    }
    if (lane == 31) xe = act ? x0at(c + V) : (TV)0;
    Vec16<TV> tt;
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const TV W = k ? xc.v[k - 1] : xw, E = k < V - 1 ? xc.v[k + 1] : xe, FW = k ? fe.v[k - 1] : fw;
        TV t1 = ((TV)1 - om) * rc.v[k] + fe.v[k] * E + FW * W + fn.v[k] * xn.v[k] + fs.v[k] * xs.v[k];
        if (j0 + k < 1 || j0 + k > A.nJ) t1 = (TV)0;
        tt.v[k] = t1;
        xx.v[k] = xx.v[k] + al * pp.v[k];
        acc += (double)rc.v[k] * (double)rc.v[k];
    }
    if (act) {
        st16(x + c, xx);
        st16(rn + c, rc);
        st16(x0 + c, xc);
        st16(t + c, tt);
    }
    return acc;
}

// the same residual half for the first cycle, x0 = omega b / d stored:
// t = (1 - omega) b + sum over the faces of f x0(neighbour)
template <typename TV>
__device__ __forceinline__ void sa0_resid(const Sa0<TV>& A, TV om, const TV* __restrict__ b,
                                          const TV* __restrict__ x0, TV* __restrict__ t, int i, int j0, bool act,
                                          int lane) {
    constexpr int V = Vec16<TV>::n;
    const int P = A.P, c = i * P + j0;
    Vec16<TV> xc = zero16<TV>(), xn = xc, xs = xc, bb = xc, fe = xc, fn = xc, fs = xc;
    if (act) {
        xc = ld16(x0 + c);
        xn = ld16(x0 + c + P);
        xs = ld16(x0 + c - P);
        bb = ld16(b + c);
        fe = ld16(A.fE + c);
        fn = ld16(A.fN + c);
        fs = ld16(A.fN + c - P);
    }
    TV xw = from_west(xc.v[V - 1]), xe = from_east(xc.v[0]), fw = from_west(fe.v[V - 1]);
    if (lane == 0) {
        const bool h = act && j0 > 0;
        xw = h ? x0[c - 1] : (TV)0;
        fw = h ? A.fE[c - 1] : (TV)0;
    }
    if (lane == 31) xe = act ? x0[c + V] : (TV)0;
    Vec16<TV> tt;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const TV W = k ? xc.v[k - 1] : xw, E = k < V - 1 ? xc.v[k + 1] : xe, FW = k ? fe.v[k - 1] : fw;
        TV t1 = ((TV)1 - om) * bb.v[k] + fe.v[k] * E + FW * W + fn.v[k] * xn.v[k] + fs.v[k] * xs.v[k];
        if (j0 + k < 1 || j0 + k > A.nJ) t1 = (TV)0;
        tt.v[k] = t1;
    }
    if (act) st16(t + c, tt);
}

// Restriction out of level 0 on aggregate-row segments: lane group g of
// aggregate row I covers fine columns [12 g, 12 g + 12) and the aggregates
// J = 4 g + 1 .. 4 g + 4 (own columns 3J-2 .. 3J, ring columns 3J-3 and
// 3J+1).  Per fine column it sums over the five rows 3I-3 .. 3I+1 the
// contribution to its own aggregate (pO on the aggregate's rows, pV on the
// two ring rows) and to its horizontal neighbour (pH); columns 12 g + 12 and
// 12 g + 13 come from the next lane group.  b_c = (P^T t)_c, x_c =
// omega b_c / d_c.  Vectors past the row's pitch and rows past the array
// read as zero; lane groups past the last aggregate (valid false) only
// supply their first columns to the group before.
template <typename TV>
__device__ __forceinline__ void sa0_restrict_seg(const Sa0<TV>& A, const TV* __restrict__ t, const SaLevel<TV>& C,
                                                 double omega, int I, int g, bool valid, int lane) {
    constexpr int V = Vec16<TV>::n, NV = 12 / V;
    const int P = A.P, j0 = 12 * g;
    TV vo[12], vh[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) vo[k] = vh[k] = (TV)0;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        const int i = 3 * I - 3 + r;
        if (i > A.nI + 2) break;
        const bool ring = r == 0 || r == 4;
        const int q0 = i * P + j0;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            if (j0 + V * v + V > P) break;
            const Vec16<TV> tv = ld16(t + q0 + V * v);
            if (ring) {
                const Vec16<TV> pv = ld16(A.pV + q0 + V * v);
#pragma unroll
                for (int k = 0; k < V; ++k) vo[V * v + k] += pv.v[k] * tv.v[k];
            } else {
                const Vec16<TV> po = ld16(A.pO + q0 + V * v), ph = ld16(A.pH + q0 + V * v);
#pragma unroll
                for (int k = 0; k < V; ++k) {
                    vo[V * v + k] += po.v[k] * tv.v[k];
                    vh[V * v + k] += ph.v[k] * tv.v[k];
                }
            }
        }
    }
    TV o12 = from_east(vo[0]), h13 = from_east(vh[1]);
    if (lane == 31) {
        o12 = (TV)0;
        h13 = (TV)0;
        for (int r = 0; r < 5; ++r) {
            const int i = 3 * I - 3 + r;
            if (i > A.nI + 2) break;
            const bool ring = r == 0 || r == 4;
            const int q = i * P + j0 + 12;
            if (j0 + 12 < P) o12 += (ring ? A.pV[q] : A.pO[q]) * t[q];
            if (!ring && j0 + 13 < P) h13 += A.pH[q + 1] * t[q + 1];
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int J = 4 * g + 1 + a;
        if (!valid || J > C.nJ) break;
        const double s = (double)vo[3 * a + 1] + (double)vo[3 * a + 2] + (double)(a == 3 ? o12 : vo[3 * a + 3]) +
                         (double)vh[3 * a] + (double)(a == 3 ? h13 : vh[3 * a + 4]);
        const size_t qc = (size_t)I * C.P + J;
        C.b[qc] = (TV)s;
        C.x[qc] = (TV)(omega * s / (double)C.c[4][qc]);
    }
}

// prolongation from level 1 and level 0's post-smoothing, two passes:
// t = x0 + P e on the lane group (P e = pO e(own) + pH e(horizontal) +
// pV e(vertical)); then, after a grid barrier,
// y = t + omega (b - A t) / d = (1 - omega) t + omega (b + sum f t(nb)) / d,
// which returns the group's share of b.y.  (One fused pass that recomputes
// t at the neighbour rows measured slower: 30.6 against 22.9 us a cycle at
// 2048 x 1024.)
template <typename TV>
__device__ __forceinline__ void sa0_prolong_t(const Sa0<TV>& A, const TV* __restrict__ x0, const TV* __restrict__ e,
                                              int Pc, TV* __restrict__ t, int i, int j0, bool act) {
    constexpr int V = Vec16<TV>::n;
    if (!act) return;
    const int c = i * A.P + j0;
    const Vec16<TV> xv = ld16(x0 + c), po = ld16(A.pO + c), ph = ld16(A.pH + c), pv = ld16(A.pV + c);
    const int I = (i - 1) / 3 + 1, sv = sa_side(i) * Pc;
    Vec16<TV> o;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const int jj = j0 + k;
        TV tk = (TV)0;
        if (jj >= 1 && jj <= A.nJ) {
            const TV* er = e + I * Pc + (jj - 1) / 3 + 1;
            tk = xv.v[k] + po.v[k] * er[0] + ph.v[k] * er[sa_side(jj)] + pv.v[k] * er[sv];
        }
        o.v[k] = tk;
    }
    st16(t + c, o);
}
template <typename TV>
__device__ __forceinline__ double sa0_smooth(const Sa0<TV>& A, TV om, const TV* __restrict__ b,
                                             const TV* __restrict__ t, TV* __restrict__ y, int i, int j0, bool act,
                                             int lane) {
    constexpr int V = Vec16<TV>::n;
    const int P = A.P, c = i * P + j0;
    Vec16<TV> tc = zero16<TV>(), tn = tc, ts = tc, bb = tc, di = tc, fe = tc, fn = tc, fs = tc;
    if (act) {
        tc = ld16(t + c);
        tn = ld16(t + c + P);
        ts = ld16(t + c - P);
        bb = ld16(b + c);
        di = ld16(A.dinv + c);
        fe = ld16(A.fE + c);
        fn = ld16(A.fN + c);
        fs = ld16(A.fN + c - P);
    }
    TV tw = from_west(tc.v[V - 1]), te = from_east(tc.v[0]), fw = from_west(fe.v[V - 1]);
    if (lane == 0) {
        const bool h = act && j0 > 0;
        tw = h ? t[c - 1] : (TV)0;
        fw = h ? A.fE[c - 1] : (TV)0;
    }
    if (lane == 31) te = act ? t[c + V] : (TV)0;
    Vec16<TV> yv;
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const TV W = k ? tc.v[k - 1] : tw, E = k < V - 1 ? tc.v[k + 1] : te, FW = k ? fe.v[k - 1] : fw;
        TV yk = ((TV)1 - om) * tc.v[k] +
                om * di.v[k] * (bb.v[k] + fe.v[k] * E + FW * W + fn.v[k] * tn.v[k] + fs.v[k] * ts.v[k]);
        if (j0 + k < 1 || j0 + k > A.nJ) yk = (TV)0;
        yv.v[k] = yk;
        acc += (double)bb.v[k] * (double)yk;
    }
    if (act) st16(y + c, yv);
    return acc;
}

// ---------------------------------------------------------------- the solver
// The PCG of one pressure-correction solve on a team of CTAs (the whole grid
// in k_pcg_sa, a group of CTAs in the batched kernel); returns false if a
// barrier gave up.  Ends without a barrier after writing p'.
template <typename TV>
__device__ __forceinline__ bool pcg_sa(const Team& T, unsigned& target, const KParams& k, Status* st,
                                       const double* dE, const double* dN, const PcgBufs<TV>& B,
                                       const SaHier<TV>& H, double* pStar, double* part) {
    extern __shared__ __align__(128) double dsm[];
    __shared__ double sm[96];
    const Dims d = k.d;
    const int M = d.M, N = d.N, w = N - 2;
    const int n = (M - 1) * w;
    const int G = T.size;
    const int tid = T.tid(), nth = T.nth();
    const bool cta0 = T.rank == 0;
    const SaSplit all{tid, nth}, cta{(int)threadIdx.x, (int)blockDim.x};
    const double rho = k.rho, hx = k.hx, hy = k.hy, om = H.omega;
    const TV omT = (TV)om;
    double* partA = part;
    double* partB = part + G;
#define SA_SYNC()                                                   \
    do {                                                            \
        if (!team_sync(T, target)) return false;                    \
    } while (0)
    // the coarse operators are rebuilt every H.reuse outer iterations (they
    // only precondition: the CG matvec and level 0's smoother and
    // prolongation always use the current operator), after a solve that
    // reached the iteration cap with them (early in a run the operator moves
    // fast), and whenever the stored ones are stale (the operator changed
    // from the host, or another solve such as the adjoint's stored its own)
    const bool rebuild = *(volatile int*)H.dirty ||
                         (H.reuse > 0 && (H.reuse == 1 || (st->iter % H.reuse) == 0 || st->itersP >= k.maxP));

    SaLevel<TV> L0 = H.lv[0];
    L0.b = B.r;
    const Sa0<TV> A0f{B.fE, B.fN, B.d, H.dinv0, L0.pw[0], L0.pw[1], L0.pw[2], M - 1, w, d.P};
    const Stencil5<TV> A0{B.fE, B.fN, B.d, M - 1, w, d.P};
    auto stencil = [&](int l) { return Stencil9<TV>{H.lv[l].c, H.lv[l].nI, H.lv[l].nJ, H.lv[l].P}; };
    auto wgt = [&](int l) { return l == 0 ? H.w0 : H.wc; };
    unsigned long long tp = (H.prof && T.lead()) ? globaltimer_ns() : 0ull;
    auto tick = [&](int ph) {
        if (H.prof && T.lead()) {
            const unsigned long long t = globaltimer_ns();
            atomicAdd(H.prof + ph, t - tp);
            tp = t;
        }
    };

    // ---- set-up: level-0 operator (the reference's formulas), its inverse
    // diagonal and prolongation weights, x = 0, r = b, x0 = omega r / d
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
        // faces towards unknowns of the own aggregate, and towards the
        // horizontal / vertical neighbour aggregate (the east face of the
        // last column is the Dirichlet outlet, with no unknown behind it)
        const int ri = (i - 1) % 3, rj = (j - 1) % 3;
        const double eIn = (j < w) ? aE : 0.0;
        const double same = (rj != 2 ? eIn : 0.0) + (rj != 0 ? aW : 0.0) + (ri != 2 ? aN : 0.0) + (ri != 0 ? aS : 0.0);
        const double fh = rj == 0 ? aW : (rj == 2 ? eIn : 0.0);
        const double fv = ri == 0 ? aS : (ri == 2 ? aN : 0.0);
        const double sc = H.w0 / aP;
        H.dinv0[c] = (TV)(1.0 / aP);
        L0.pw[0][c] = (TV)(1.0 - sc * (aP - same));
        L0.pw[1][c] = (TV)(sc * fh);
        L0.pw[2][c] = (TV)(sc * fv);
        B.x[c] = (TV)0;
        const TV rt = B.rhs[c];
        B.r[c] = rt;
        L0.x[c] = (TV)(om * (double)rt / aP);
        bb[0] += (double)rt * (double)rt;
    }
    block_sum<1>(bb, sm);
    if (threadIdx.x == 0) partA[T.rank] = bb[0];
    SA_SYNC();
    double bnorm2[1];
    sum_partials<1>(partA, G, 1, bnorm2, sm);
    const double rTol = k.pTol * sqrt(bnorm2[0]);
    tick(SA_P_SETUP);

    // ---- set-up: coarse operators by coloured probes (when rebuilt), with
    // the prolongation weights of the grid-wide coarse levels
    if (rebuild) {
        // every level grid-wide; levels with stored prolongation weights
        // (level 0 from the set-up, the grid-wide coarse levels from a pass
        // of their own) probe and contract with them
        for (int l = 0; l < H.L - 1; ++l) {
            const SaLevel<TV>& f = H.lv[l];
            const SaLevel<TV>& C = H.lv[l + 1];
            const bool wts = l < H.Lg;
            if (wts && l > 0) {
                sa_cells(all, f.nI, f.nJ, [&](int i, int j) {
                    double pw[4];
                    sa_pweights(stencil(l), i, j, wgt(l), pw);
                    const size_t q = (size_t)i * f.P + j;
#pragma unroll
                    for (int m = 0; m < 4; ++m) f.pw[m][q] = (TV)pw[m];
                });
                SA_SYNC();
            }
            if (l == 0)
                sa_cells(all, f.nI, f.nJ, [&](int i, int j) { sa_probe_w<TV, Stencil5<TV>, false>(A0, L0, H.Y, i, j); });
            else if (wts)
                sa_cells(all, f.nI, f.nJ, [&](int i, int j) { sa_probe_w<TV, Stencil9<TV>, true>(stencil(l), f, H.Y, i, j); });
            else
                sa_cells(all, f.nI, f.nJ, [&](int i, int j) { sa_probe_cell(stencil(l), f.P, H.Y, wgt(l), i, j); });
            SA_SYNC();
            if (l == 0)
                sa_cells(all, C.nI, C.nJ, [&](int I, int J) { sa_galerkin_w<TV, false>(L0, H.Y, C, I, J); });
            else if (wts)
                sa_cells(all, C.nI, C.nJ, [&](int I, int J) { sa_galerkin_w<TV, true>(f, H.Y, C, I, J); });
            else
                sa_cells(all, C.nI, C.nJ,
                         [&](int I, int J) { sa_galerkin_cell(stencil(l), f.P, H.Y, C, wgt(l), I, J); });
            SA_SYNC();
        }
        if (cta0) sa_dense_setup(H.lv[H.L - 1], H.dense, dsm);
        SA_SYNC();
    }
    tick(SA_P_GALERKIN);

    // ---- CTA 0 stages levels [Lg, L) (operators copied, vectors zeroed,
    // frames included) and the dense inverse in shared memory
    TV* const smb = reinterpret_cast<TV*>(dsm);
    TV* sInv = nullptr;
    if (cta0) {
        for (int l = H.Lg; l < H.L; ++l) {
            const SaLevel<TV>& g = H.lv[l];
            const SaSm<TV> f = sa_sm(H, smb, l);
            for (int e = threadIdx.x; e < 9 * f.ne; e += blockDim.x) {
                const int q = e / f.ne, r = e - q * f.ne, ii = r / f.P, jj = r - ii * f.P;
                f.s[e] = g.c[q][(size_t)ii * g.P + jj];
            }
            for (int e = 9 * f.ne + threadIdx.x; e < 13 * f.ne; e += blockDim.x) f.s[e] = (TV)0;
            sInv = f.s + 13 * f.ne;
        }
        const int nd = H.lv[H.L - 1].nI * H.lv[H.L - 1].nJ;
        for (int e = threadIdx.x; e < nd * nd; e += blockDim.x) sInv[e] = H.dense[e];
        __syncthreads();
    }

    // grid-wide coarse levels: restriction l -> l+1 and prolongation
    // l+1 -> l with post-smoothing, two passes each
    auto restrict_level = [&](int l) -> bool {
        const SaLevel<TV>& f = H.lv[l];
        const SaLevel<TV>& C = H.lv[l + 1];
        sa_cells(all, f.nI, f.nJ, [&](int i, int j) { sa_resid_cell(f, i, j); });
        if (!team_sync(T, target)) return false;
        sa_cells(all, C.nI, C.nJ, [&](int I, int J) { sa_restrict_w(f, C, om, I, J); });
        return team_sync(T, target);
    };
    auto prolong_level = [&](int l) -> bool {
        const SaLevel<TV>& f = H.lv[l];
        const SaLevel<TV>& C = H.lv[l + 1];
        sa_cells(all, f.nI, f.nJ, [&](int i, int j) { sa_prolong_w(f, C.y, C.P, i, j); });
        if (!team_sync(T, target)) return false;
        sa_cells(all, f.nI, f.nJ, [&](int i, int j) { sa_smooth_cell(f, om, i, j); });
        return team_sync(T, target);
    };
    // CTA 0: levels [Lg, L) in shared memory, between the copy of level Lg's
    // rhs and pre-smoothed iterate in and of its corrected iterate out
    auto cta_levels = [&]() {
        const SaLevel<TV>& Gl = H.lv[H.Lg];
        const SaSm<TV> S0 = sa_sm(H, smb, H.Lg);
        for (int a = threadIdx.x; a < Gl.nI * Gl.nJ; a += blockDim.x) {
            const int i = 1 + a / Gl.nJ, j = 1 + a % Gl.nJ;
            S0.b()[i * S0.P + j] = Gl.b[(size_t)i * Gl.P + j];
            S0.x()[i * S0.P + j] = Gl.x[(size_t)i * Gl.P + j];
        }
        __syncthreads();
        const TV wc = (TV)H.wc, omc = (TV)om;
        for (int l = H.Lg; l < H.L - 1; ++l) {
            const SaSm<TV> f = sa_sm(H, smb, l), C = sa_sm(H, smb, l + 1);
            sa_cells(cta, f.nI, f.nJ, [&](int i, int j) { sa_sm_resid(f, i, j); });
            __syncthreads();
            sa_cells(cta, f.nI, f.nJ, [&](int i, int j) { sa_sm_smoothres(f, wc, i, j); });
            __syncthreads();
            sa_cells(cta, C.nI, C.nJ, [&](int I, int J) { sa_sm_aggsum(f, C, omc, I, J); });
            __syncthreads();
        }
        sa_sm_dense(sa_sm(H, smb, H.L - 1), sInv);
        for (int l = H.L - 2; l >= H.Lg; --l) {
            const SaSm<TV> f = sa_sm(H, smb, l), C = sa_sm(H, smb, l + 1);
            sa_cells(cta, f.nI, f.nJ, [&](int i, int j) { sa_sm_prolong(f, C, wc, i, j); });
            __syncthreads();
            sa_cells(cta, f.nI, f.nJ, [&](int i, int j) { sa_sm_smooth(f, omc, i, j); });
            __syncthreads();
        }
        for (int a = threadIdx.x; a < Gl.nI * Gl.nJ; a += blockDim.x) {
            const int i = 1 + a / Gl.nJ, j = 1 + a % Gl.nJ;
            Gl.y[(size_t)i * Gl.P + j] = S0.y()[i * S0.P + j];
        }
    };
    // ---- z = M r (V-cycle) with r = L0.b; level 0's residual half t is done
    // already (by the CG update, or here when `first`); z goes to L0.y;
    // rz = r.z
    const SaLevel<TV>& C1 = H.lv[1];
    auto vcycle = [&](double& rz, bool first) __attribute__((always_inline)) -> bool {
        if (first) {
            row_segments<TV>(T, L0.nI, L0.nJ, [&](int i, int j0, bool act, int lane) {
                sa0_resid(A0f, omT, L0.b, L0.x, L0.t, i, j0, act, lane);
            });
            if (!team_sync(T, target)) return false;
        }
        {
            // aggregate-row segments of 32 lane groups, one segment per warp
            const int lane = threadIdx.x & 31;
            const int warp = (int)(tid >> 5), nw = nth >> 5;
            const int Gr = (C1.nJ + 3) / 4, S = (Gr + 31) >> 5;
            for (int sg = warp; sg < C1.nI * S; sg += nw) {
                const int I = 1 + sg / S, g = ((sg % S) << 5) + lane;
                sa0_restrict_seg(A0f, L0.t, C1, om, I, g, g < Gr, lane);
            }
        }
        if (!team_sync(T, target)) return false;
        tick(SA_P_DOWN);
        for (int l = 1; l < H.Lg; ++l) {
            if (!restrict_level(l)) return false;
            tick(SA_P_DOWN + l);
        }
        if (cta0) cta_levels();
        if (!team_sync(T, target)) return false;
        tick(SA_P_CTA);
        for (int l = H.Lg - 1; l >= 1; --l) {
            if (!prolong_level(l)) return false;
            tick(SA_P_UP + l);
        }
        double acc[1] = {0.0};
        row_segments<TV>(T, L0.nI, L0.nJ, [&](int i, int j0, bool act, int lane) {
            sa0_prolong_t(A0f, L0.x, C1.y, C1.P, L0.t, i, j0, act);
        });
        if (!team_sync(T, target)) return false;
        row_segments<TV>(T, L0.nI, L0.nJ, [&](int i, int j0, bool act, int lane) {
            acc[0] += sa0_smooth(A0f, omT, L0.b, L0.t, L0.y, i, j0, act, lane);
        });
        block_sum<1>(acc, sm);
        if (threadIdx.x == 0) partB[2 * T.rank + 1] = acc[0];
        if (!team_sync(T, target)) return false;
        double t2[2];
        sum_partials<2>(partB, G, 2, t2, sm);
        rz = t2[1];
        tick(SA_P_UP);
        return true;
    };

    double rz = 0.0;
    if (!vcycle(rz, true)) return false;
    double beta = 0.0;
    int it = 0;
    TV* pbuf[2] = {B.pa, B.pb};
    TV* rbuf[2] = {B.r, H.r2};
    for (; it < k.maxP; ++it) {
        TV* pnew = pbuf[it & 1];
        const TV* pold = pbuf[(it + 1) & 1];
        const TV bt = (TV)beta;
        const bool first = it == 0;
        double accA[1] = {0.0};
        row_segments<TV>(T, L0.nI, L0.nJ, [&](int i, int j0, bool act, int lane) {
            accA[0] += sa0_matvec(A0f, L0.y, pold, bt, first, pnew, B.Ap, i, j0, act, lane);
        });
        block_sum<1>(accA, sm);
        if (threadIdx.x == 0) partA[T.rank] = accA[0];
        SA_SYNC();
        double pAp[1];
        sum_partials<1>(partA, G, 1, pAp, sm);
        tick(SA_P_MATVEC);
        if (fabs(pAp[0]) < 1e-20) break;
        const TV al = (TV)(rz / pAp[0]);
        const TV* rold = rbuf[it & 1];
        TV* rnew = rbuf[(it + 1) & 1];
        double accB[1] = {0.0};
        row_segments<TV>(T, L0.nI, L0.nJ, [&](int i, int j0, bool act, int lane) {
            accB[0] += sa0_update(A0f, al, omT, pnew, B.Ap, B.x, rold, rnew, L0.x, L0.t, i, j0, act, lane);
        });
        L0.b = rnew;
        block_sum<1>(accB, sm);
        if (threadIdx.x == 0) partB[2 * T.rank] = accB[0];
        SA_SYNC();
        double tB[2];
        sum_partials<2>(partB, G, 2, tB, sm);
        tick(SA_P_UPDATE);
        if (sqrt(tB[0]) <= rTol) { ++it; break; }
        double rzn = 0.0;
        if (!vcycle(rzn, false)) return false;
        beta = rzn / rz;
        rz = rzn;
    }
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const int c = i * d.P + j;
        pStar[c] = (double)B.x[c];
        if (j == w) pStar[c + 1] = 0.0;
    }
    if (T.lead()) {
        st->itersP = it;
        if (rebuild) *H.dirty = 0;
    }
    return true;
#undef SA_SYNC
}

template <typename TV>
__global__ void __launch_bounds__(512, 1) k_pcg_sa(KParams k, Status* st, const double* dE, const double* dN,
                                                PcgBufs<TV> B, SaHier<TV> H, double* pStar, double* part,
                                                unsigned* bar) {
    if (st->done) return;
    unsigned target = 0;
    pcg_sa<TV>(grid_team(bar, &st->err), target, k, st, dE, dN, B, H, pStar, part);
}

}  // namespace cp
