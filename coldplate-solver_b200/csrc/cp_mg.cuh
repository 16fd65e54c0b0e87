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
// The CG recurrences, the stop rules (|p.Ap| < 1e-20, sqrt(r.r) < pTol) and
// the returned count are those of pressure_solver.cpp:121-184.
#pragma once

#include "cp_kernels.cuh"

namespace cp {

constexpr int kMgMaxLevels = 16;
constexpr int kMgCtaCells = 16384;   // levels at or below this size run on one CTA
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
};

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
                                                     int i, int j, double omega) {
    // e: the coarse level's corrected iterate (its x or y buffer)
    auto xp = [&](int ii, int jj) -> TV {
        if (ii < 1 || ii > f.nI || jj < 1 || jj > f.nJ) return (TV)0;
        return f.x[lidx(f, ii, jj)] + e[lidx(c, (ii + 1) >> 1, (jj + 1) >> 1)];
    };
    const size_t q = lidx(f, i, j);
    const TV xc = xp(i, j);
    const TV ax = f.d[q] * xc - f.fE[q] * xp(i, j + 1) - f.fE[q - 1] * xp(i, j - 1) - f.fN[q] * xp(i + 1, j) -
                  f.fN[q - f.P] * xp(i - 1, j);
    const TV y = xc + (TV)omega * (f.b[q] - ax) / f.d[q];
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
                  [&](int i, int j) { mg_prolong_smooth_cell(f, H.lv[l + 1], H.lv[l + 1].x, i, j, H.omega); });
        __syncthreads();
        for_cells(s, f.nI, f.nJ, [&](int i, int j) { const size_t q = lidx(f, i, j); f.x[q] = f.y[q]; });
        __syncthreads();
    }
}

// ---------------------------------------------------------------- the solver
// B (PcgBufs) holds level-0 faces, diagonal and the CG vectors in the field
// layout; H.lv[0] aliases them (fE, fN, d) plus its own x/y/b/dx buffers.
template <typename TV>
__global__ void __launch_bounds__(512) k_pcg_mg(KParams k, Status* st, const double* dE, const double* dN,
                                                PcgBufs<TV> B, MgHier<TV> H, double* pStar, double* part,
                                                unsigned* bar) {
    if (st->done) return;
    extern __shared__ double dsm[];   // dense setup workspace (kMgDense x 2 kMgDense)
    __shared__ double sm[96];
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
        B.d[c] = (TV)aP;
        L0.dx[c] = (TV)extra;
        B.x[c] = (TV)0;
        B.r[c] = B.rhs[c];
    }
    MG_SYNC();
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

    // ---- z = M r (V-cycle); level-0 rhs is r; result in L0.y; also r.z
    // The pre-smoothing step of level 0 (x0 = omega r / d) is written by the
    // caller phase; `rz` returns the global r.z.
    auto vcycle = [&](double& rz) -> bool {
        // down over grid-wide levels
        for (int l = 0; l < H.Lg - 1; ++l) {
            for_cells(all, H.lv[l + 1].nI, H.lv[l + 1].nJ,
                      [&](int I, int J) { mg_restrict_cell(H.lv[l], H.lv[l + 1], I, J, om); });
            target += G;
            if (!grid_barrier(bar, target, &st->err)) return false;
        }
        {
            if (blockIdx.x == 0) {
                // restrict the last grid-wide level into the first CTA level
                const int l = H.Lg - 1;
                for_cells(Split{(int)threadIdx.x, (int)blockDim.x}, H.lv[l + 1].nI, H.lv[l + 1].nJ,
                          [&](int I, int J) { mg_restrict_cell(H.lv[l], H.lv[l + 1], I, J, om); });
                __syncthreads();
                if (H.Lg < H.L - 1) {
                    mg_cta_cycle(H);
                } else {
                    mg_dense_solve(H.lv[H.L - 1], H.dense);
                }
            }
            target += G;
            if (!grid_barrier(bar, target, &st->err)) return false;
        }
        // up over grid-wide levels: prolongate + post-smooth into y (the
        // corrected iterate of a grid-wide level stays in y, of a CTA level in x)
        for (int l = H.Lg - 1; l >= 0; --l) {
            const MgLevel<TV>& f = H.lv[l];
            const TV* e = (l + 1 < H.Lg) ? H.lv[l + 1].y : H.lv[l + 1].x;
            double acc[1] = {0.0};
            for_cells(all, f.nI, f.nJ, [&](int i, int j) {
                const TV y = mg_prolong_smooth_cell(f, H.lv[l + 1], e, i, j, om);
                if (l == 0) acc[0] += (double)f.b[lidx(f, i, j)] * (double)y;
            });
            if (l == 0) {
                block_sum<1>(acc, sm);
                if (threadIdx.x == 0) partB[2 * blockIdx.x + 1] = acc[0];
            }
            target += G;
            if (!grid_barrier(bar, target, &st->err)) return false;
        }
        double t2[2];
        sum_partials<2>(partB, G, 2, t2, sm);
        rz = t2[1];
        return true;
    };

    // first preconditioning: level-0 b is r, x = omega r / d
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        L0.b[c] = B.r[c];
        L0.x[c] = (TV)(om * (double)B.r[c] / (double)B.d[c]);
    }
    MG_SYNC();
    double rz = 0.0;
    if (!vcycle(rz)) return;
    // z lives in L0.y; p_new = z + beta p_old recomputed at the neighbours
    double beta = 0.0;
    int it = 0;
    TV* pbuf[2] = {B.pa, B.pb};
    for (; it < k.maxP; ++it) {
        const bool first = (it == 0);
        const TV* pold = pbuf[(it + 1) & 1];
        TV* pnew = pbuf[it & 1];
        const TV* z = L0.y;
        auto dir = [&](size_t c) -> TV { return first ? z[c] : (TV)(z[c] + (TV)beta * pold[c]); };
        double accA[1] = {0.0};
        for (int t = tid; t < n; t += nth) {
            const int i = 1 + t / w, j = 1 + t % w;
            const size_t c = at(d, i, j);
            const TV pc = dir(c);
            const TV pS = (i > 1) ? dir(c - d.P) : (TV)0;
            const TV pW = (j > 1) ? dir(c - 1) : (TV)0;
            const TV pE = (j < w) ? dir(c + 1) : (TV)0;
            const TV pN = (i < M - 1) ? dir(c + d.P) : (TV)0;
            const TV ap = B.d[c] * pc - B.fN[c - d.P] * pS - B.fE[c - 1] * pW - B.fE[c] * pE - B.fN[c] * pN;
            pnew[c] = pc;
            B.Ap[c] = ap;
            accA[0] += (double)pc * (double)ap;
        }
        block_sum<1>(accA, sm);
        if (threadIdx.x == 0) partA[blockIdx.x] = accA[0];
        MG_SYNC();
        double pAp[1];
        sum_partials<1>(partA, G, 1, pAp, sm);
        if (fabs(pAp[0]) < 1e-20) break;
        const double alpha = rz / pAp[0];
        double accB[1] = {0.0};
        for (int t = tid; t < n; t += nth) {
            const int i = 1 + t / w, j = 1 + t % w;
            const size_t c = at(d, i, j);
            B.x[c] = B.x[c] + (TV)alpha * pnew[c];
            const TV r = B.r[c] - (TV)alpha * B.Ap[c];
            B.r[c] = r;
            accB[0] += (double)r * (double)r;
            L0.b[c] = r;
            L0.x[c] = (TV)(om * (double)r / (double)B.d[c]);
        }
        block_sum<1>(accB, sm);
        if (threadIdx.x == 0) partB[2 * blockIdx.x] = accB[0];
        MG_SYNC();
        double tB[2];
        sum_partials<2>(partB, G, 2, tB, sm);
        if (sqrt(tB[0]) < k.pTol) break;
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
}

}  // namespace cp
