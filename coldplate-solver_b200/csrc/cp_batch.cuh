// Batched SIMPLE solves: many independent fields, each with its own grid
// size, geometry and inlet velocity, advanced together by ONE persistent
// cooperative kernel.
//
// The fields are not solved one after the other, and not by fixed groups of
// SMs either: every phase of the outer iteration (boundary conditions,
// momentum assembly, the Jacobi sweeps, mass imbalance, the multigrid-PCG
// pressure solve, the correction and the pressure-drop sampling) walks the
// R x C cell tiles of ALL fields that are still iterating, strided over the
// whole grid.  The whole GPU stays busy until the last field converges, and
// the grid barriers between phases are shared by every field instead of
// being paid per field.  Each field keeps its own stop rules: it leaves the
// Jacobi sweeps, the CG iterations and the outer loop on its own criteria,
// exactly as a single-field solve does.
//
// Reductions stay deterministic: every tile writes its partial sums, and
// field f's totals are formed by block f % G (its "reducer") in tile order,
// between two grid barriers.  The coarse multigrid levels that fit one CTA
// run on the field's reducer block, so the coarse solves of different fields
// run in parallel on different SMs.
//
// The per-cell arithmetic is the single-field arithmetic (assemble_one, the
// Jacobi update in the reference's S, W, P, E, N order, the multigrid cell
// operators, finalize_block); only the order of the global sums differs.
#pragma once

#include "cp_mg.cuh"
#include "cp_sa.cuh"

namespace cp {

constexpr int kBatchMaxFields = 256;
constexpr int kBatchThreads = 512;
constexpr int kBatchMaxLevels = 10;   // tile tables for levels 0 .. maxLg
constexpr int kBatchPartStride = 5;   // partial sums per tile

// Everything one field's solve touches (device pointers of a single-field
// context plus its parameter block and multigrid hierarchy).
template <typename TC>
struct BField {
    KParams k;
    Status* st;
    double *u, *v, *p, *uStar, *vStar, *pStar, *dE, *dN;
    const double *alpha, *gamma;
    MomSys<TC> U, V;
    TC *xU0, *xU1, *xV0, *xV1;
    PcgBufs<TC> B;
    MgHier<TC> H;
    double* hist;
    int histCap;
    double* dpWin;
};

// Per-field solver state, written only by the field's reducer block between
// grid barriers and read by every block after the next barrier.
struct BState {
    int on;              // iterating in this outer iteration
    int jacU, jacV;      // Jacobi sweeps of U / V still running
    int itsU, itsV;      // sweeps done
    int cgOn;            // CG still running
    int cgIt;            // CG iterations to report
    int pad;
    double rz, alpha, beta, rTol;
    double mass[4];      // sum du^2, sum dv^2, sum b^2, max |b| (the k_mass quantities)
};

// CP_BATCH_PROFILE: device time of each phase (barrier to barrier, as seen
// by block 0), summed over the launch
enum BatchPhase { BP_BC = 0, BP_ASM, BP_JAC, BP_JACRED, BP_SCAT, BP_BCSTAR, BP_MASS, BP_MASSRED, BP_COARSE,
                  BP_COARSECTA, BP_RESTR, BP_VCTA, BP_PROL, BP_VRED, BP_MATVEC, BP_MVRED, BP_UPD, BP_UPDRED,
                  BP_PSTAR, BP_CORR, BP_BC2, BP_FIN, BP_COUNT };

struct BatchArgs {
    int nf;              // fields
    int R, C;            // cell tile: R rows x C columns
    int maxLg;           // largest number of grid-wide multigrid levels over the fields
    int maxMom, maxP;    // largest maxMomentumIter / maxPressureIter over the fields
    int nOuter;          // outer iterations this launch may run
    const int* toff;     // [(maxLg + 1) * (nf + 1)]: first tile of each field per level
    BState* bs;          // [nf]
    double* ipart;       // [tiles of level 0 * kBatchPartStride]
    unsigned* bar;       // grid barrier counter (zeroed before the launch)
    int* err;            // first device error of the batch (barrier time-out)
    int* allDone;        // 1 when every field has stopped
    unsigned long long* prof;   // [BP_COUNT] or null
};

// One Jacobi update of a momentum unknown (x+ = x + (b - A x) / aP, the
// products summed in the S, W, P, E, N order of the reference's CSR rows);
// returns r^2.  first: the iterate is the current field (FP64 form) or zero
// (the mixed form solves for a correction).
template <typename TC, bool Mixed>
__device__ __forceinline__ double jacobi_cell(const Dims& d, const MomSys<TC>& S, const double* field,
                                              const TC* xc, TC* xn, int i, int j, int i1, int j1, bool first) {
    const size_t c = at(d, i, j);
    auto X = [&](size_t q) -> TC {
        if (first) return Mixed ? (TC)0 : (TC)field[q];
        return xc[q];
    };
    const TC aP = S.aP[c], aE = S.aE[c], aW = S.aW[c], aN = S.aN[c], aS = S.aS[c], b = S.b[c];
    const TC xP = X(c);
    const TC xS = (i > 1) ? X(c - d.P) : (TC)0;
    const TC xW = (j > 1) ? X(c - 1) : (TC)0;
    const TC xE = (j < j1) ? X(c + 1) : (TC)0;
    const TC xN = (i < i1) ? X(c + d.P) : (TC)0;
    TC Ax = (TC)0;
    Ax += (-aS) * xS;
    Ax += (-aW) * xW;
    Ax += aP * xP;
    Ax += (-aE) * xE;
    Ax += (-aN) * xN;
    const TC r = b - Ax;
    xn[c] = xP + r / aP;
    return (double)r * (double)r;
}

// scatter of one momentum unknown with the clamps of momentum_solver.cpp:335-351;
// returns |u* - u|
template <typename TC, bool Mixed>
__device__ __forceinline__ double scatter_cell(const Dims& d, const double* field, const TC* xr, double* out,
                                               double maxVel, int i, int j) {
    const size_t c = at(d, i, j);
    double xv = xr ? (double)xr[c] : (Mixed ? 0.0 : field[c]);
    if (Mixed) xv += field[c];
    const double nv = dclamp(xv, -maxVel, maxVel);
    out[c] = nv;
    return fabs(nv - field[c]);
}

template <typename TC, bool Mixed>
__global__ void __launch_bounds__(kBatchThreads, 1) k_batch(BatchArgs a, const BField<TC>* __restrict__ F) {
    extern __shared__ __align__(128) double dsm[];   // dense set-up workspace of the coarsest levels
    __shared__ double sm[160];
    __shared__ int s_toff[kBatchMaxLevels * (kBatchMaxFields + 1)];
    __shared__ __align__(16) BField<TC> fs;          // the field whose tiles this block is on
    __shared__ int fsIdx;
    const int G = gridDim.x, nf = a.nf;
    for (int q = threadIdx.x; q < (a.maxLg + 1) * (nf + 1); q += blockDim.x) s_toff[q] = a.toff[q];
    if (threadIdx.x == 0) fsIdx = -1;
    __syncthreads();
    unsigned target = 0;
    unsigned long long tp = (a.prof && blockIdx.x == 0 && threadIdx.x == 0) ? globaltimer_ns() : 0ull;
    auto sync = [&](int ph) -> bool {
        target += G;
        const bool ok = grid_barrier(a.bar, target, a.err);
        if (tp) {
            const unsigned long long t = globaltimer_ns();
            a.prof[ph] += t - tp;
            tp = t;
        }
        return ok;
    };
    // make fs hold field f (block-uniform call)
    auto load_field = [&](int f) {
        if (fsIdx == f) return;
        __syncthreads();
        const int* src = reinterpret_cast<const int*>(F + f);
        int* dst = reinterpret_cast<int*>(&fs);
        for (int q = threadIdx.x; q < (int)(sizeof(BField<TC>) / sizeof(int)); q += blockDim.x) dst[q] = src[q];
        if (threadIdx.x == 0) fsIdx = f;
        __syncthreads();
    };
    auto bsv = [&](int f) -> BState& { return a.bs[f]; };
    auto ldi = [&](const int* p) -> int { return __ldcg(p); };
    auto ldd = [&](const double* p) -> double { return __ldcg(p); };
    // body(i, j) over the cells of this block's tiles of level l whose field
    // passes on(f); fin(f, g) after each tile (block-uniform).  on(f) runs
    // once per tile in every thread and may cache per-field scalars.
    auto for_tiles = [&](int l, auto&& on, auto&& body, auto&& fin) {
        const int* to = s_toff + l * (nf + 1);
        const int total = to[nf];
        int f = 0;
        for (int g = blockIdx.x; g < total; g += G) {
            while (g >= to[f + 1]) ++f;
            if (!on(f)) continue;
            load_field(f);
            int nI, nJ;
            if (l == 0) { nI = fs.k.d.M - 1; nJ = fs.k.d.N - 1; }
            else { nI = fs.H.lv[l].nI; nJ = fs.H.lv[l].nJ; }
            const int tJ = (nJ + a.C - 1) / a.C;
            const int t = g - to[f];
            const int i0 = 1 + (t / tJ) * a.R, j0 = 1 + (t % tJ) * a.C;
            for (int u = threadIdx.x; u < a.R * a.C; u += blockDim.x) {
                const int i = i0 + u / a.C, j = j0 + u % a.C;
                if (i <= nI && j <= nJ) body(i, j);
            }
            fin(f, g);
        }
    };
    // reducer loop: fn(f) for the fields this block reduces (block-uniform)
    auto for_my_fields = [&](auto&& on, auto&& fn) {
        for (int f = blockIdx.x; f < nf; f += G) {
            if (!on(f)) continue;
            load_field(f);
            fn(f);
            __syncthreads();
        }
    };
    auto tile_sum = [&](int f, double (&tot)[kBatchPartStride], int nv) {
        const int* to = s_toff;
        for (int q = 0; q < kBatchPartStride; ++q) tot[q] = 0.0;
        for (int g = to[f] + threadIdx.x; g < to[f + 1]; g += blockDim.x)
            for (int q = 0; q < nv; ++q) tot[q] += ldd(a.ipart + (size_t)g * kBatchPartStride + q);
        block_sum<kBatchPartStride>(tot, sm);
    };
    auto write_part = [&](int g, const double* v, int nv) {
        if (threadIdx.x == 0)
            for (int q = 0; q < nv; ++q) a.ipart[(size_t)g * kBatchPartStride + q] = v[q];
    };
    auto isOn = [&](int f) -> bool { return ldi(&a.bs[f].on) != 0; };
    auto cgOn = [&](int f) -> bool { return ldi(&a.bs[f].cgOn) != 0; };
    auto noFin = [&](int, int) {};
    double tVel = 0.0;   // per-tile copy of the field's velocity clamp
    auto onVel = [&](int f) -> bool {
        if (!isOn(f)) return false;
        tVel = max_vel(inlet_velocity(F[f].k, __ldcg(&F[f].st->iter)));
        return true;
    };

    for (int outer = 0; outer < a.nOuter; ++outer) {
        // ---- which fields iterate; velocity + pressure BCs (boundaries.cpp:50-146)
        for_my_fields([&](int) { return true; }, [&](int f) {
            const int on = fs.st->done ? 0 : 1;
            if (threadIdx.x == 0) {
                BState& b = bsv(f);
                b.on = on;
                b.jacU = on && fs.k.maxMom > 0;
                b.jacV = on && fs.k.maxMom > 0;
                b.itsU = b.itsV = 0;
                b.cgOn = 0;
                b.cgIt = 0;
                if (on) { fs.st->maxDU = 0ull; fs.st->maxDV = 0ull; }
            }
            if (on) apply_bc(fs.k, fs.st->iter, fs.u, fs.v, fs.p, fs.gamma, threadIdx.x, blockDim.x);
        });
        if (!sync(BP_BC)) return;
        {
            int any = 0;
            for (int f = 0; f < nf; ++f) any |= ldi(&a.bs[f].on);
            if (!any) break;
        }
        // ---- momentum assembly, U and V (momentum_solver.cpp:197-314)
        for_tiles(0, onVel, [&](int i, int j) {
            const Dims d = fs.k.d;
            const Fields fl{fs.u, fs.v, fs.p, fs.alpha, fs.gamma};
            if (i <= d.M - 1 && j <= d.N - 2) assemble_one<TC, Mixed, true>(fs.k, fl, fs.U, fs.dE, i, j, tVel);
            if (i <= d.M - 2 && j <= d.N - 1) assemble_one<TC, Mixed, false>(fs.k, fl, fs.V, fs.dN, i, j, tVel);
        }, noFin);
        if (!sync(BP_ASM)) return;
        // ---- Jacobi sweeps of U and V together; each component of each field
        // stops on its own rule (jacobi_solver.cpp:44-67)
        for (int s = 0; s < a.maxMom; ++s) {
            const bool first = (s == 0);
            double acc[2] = {0.0, 0.0};
            int tU = 0, tV = 0;
            for_tiles(0, [&](int f) {
                    tU = ldi(&a.bs[f].jacU);
                    tV = ldi(&a.bs[f].jacV);
                    return isOn(f) && (tU || tV);
                }, [&](int i, int j) {
                const Dims d = fs.k.d;
                TC* xs[4] = {fs.xU0, fs.xU1, fs.xV0, fs.xV1};
                const int cur = first ? 0 : ((s - 1) & 1), nxt = first ? 0 : 1 - cur;
                if (tU && i <= d.M - 1 && j <= d.N - 2)
                    acc[0] += jacobi_cell<TC, Mixed>(d, fs.U, fs.u, xs[cur], xs[nxt], i, j, d.M - 1, d.N - 2, first);
                if (tV && i <= d.M - 2 && j <= d.N - 1)
                    acc[1] += jacobi_cell<TC, Mixed>(d, fs.V, fs.v, xs[2 + cur], xs[2 + nxt], i, j, d.M - 2, d.N - 1,
                                                     first);
            }, [&](int, int g) {
                block_sum<2>(acc, sm);
                write_part(g, acc, 2);
                acc[0] = acc[1] = 0.0;
            });
            if (!sync(BP_JAC)) return;
            for_my_fields([&](int f) { return isOn(f) && (ldi(&a.bs[f].jacU) || ldi(&a.bs[f].jacV)); },
                          [&](int f) {
                double tot[kBatchPartStride];
                tile_sum(f, tot, 2);
                if (threadIdx.x == 0) {
                    BState& b = bsv(f);
                    const Dims d = fs.k.d;
                    const double nU = (double)((d.M - 1) * (d.N - 2)), nV = (double)((d.M - 2) * (d.N - 1));
                    const double tol2 = fs.k.momTol * fs.k.momTol;
                    if (b.jacU) {
                        b.itsU = s + 1;
                        if (tot[0] < tol2 * nU || s + 1 >= fs.k.maxMom) b.jacU = 0;
                    }
                    if (b.jacV) {
                        b.itsV = s + 1;
                        if (tot[1] < tol2 * nV || s + 1 >= fs.k.maxMom) b.jacV = 0;
                    }
                }
            });
            if (!sync(BP_JACRED)) return;
            int any = 0;
            for (int f = 0; f < nf; ++f) any |= ldi(&a.bs[f].jacU) | ldi(&a.bs[f].jacV);
            if (!any) break;
        }
        // ---- scatter with clamps and the max change (momentum_solver.cpp:335-351)
        {
            double mu = 0.0, mv = 0.0;
            int itU = 0, itV = 0;
            for_tiles(0, [&](int f) {
                    if (!onVel(f)) return false;
                    itU = ldi(&a.bs[f].itsU);
                    itV = ldi(&a.bs[f].itsV);
                    return true;
                }, [&](int i, int j) {
                const Dims d = fs.k.d;
                const TC* xu = itU == 0 ? nullptr : (((itU - 1) & 1) ? fs.xU1 : fs.xU0);
                const TC* xv = itV == 0 ? nullptr : (((itV - 1) & 1) ? fs.xV1 : fs.xV0);
                if (i <= d.M - 1 && j <= d.N - 2)
                    mu = dmax(mu, scatter_cell<TC, Mixed>(d, fs.u, xu, fs.uStar, tVel, i, j));
                if (i <= d.M - 2 && j <= d.N - 1)
                    mv = dmax(mv, scatter_cell<TC, Mixed>(d, fs.v, xv, fs.vStar, tVel, i, j));
            }, [&](int, int) {
                mu = warp_max(mu);
                mv = warp_max(mv);
                if ((threadIdx.x & 31) == 0) {
                    atomic_max_nonneg(&fs.st->maxDU, mu);
                    atomic_max_nonneg(&fs.st->maxDV, mv);
                }
                mu = mv = 0.0;
            });
        }
        if (!sync(BP_SCAT)) return;
        // ---- BCs on u*, v*; the sweep counts
        for_my_fields(isOn, [&](int f) {
            if (threadIdx.x == 0) {
                fs.st->itersU = ldi(&a.bs[f].itsU);
                fs.st->itersV = ldi(&a.bs[f].itsV);
            }
            apply_bc(fs.k, fs.st->iter, fs.uStar, fs.vStar, nullptr, fs.gamma, threadIdx.x, blockDim.x);
        });
        if (!sync(BP_BCSTAR)) return;
        // ---- mass imbalance and RMS changes (iterations.cpp:499-533,
        // pressure_solver.cpp:471-488, 733-742), fused with the level-0
        // operator of the pressure correction, x = 0, r = b
        {
            double acc[kBatchPartStride] = {0.0, 0.0, 0.0, 0.0, 0.0};   // du2 dv2 b2 max bb
            for_tiles(0, isOn, [&](int i, int j) {
                const Dims d = fs.k.d;
                const int M = d.M, N = d.N;
                const double rho = fs.k.rho, hx = fs.k.hx, hy = fs.k.hy;
                const size_t c = at(d, i, j);
                const double massE = rho * fs.uStar[c] * hy, massW = rho * fs.uStar[c - 1] * hy;
                const double massN = rho * fs.vStar[c] * hx, massS = rho * fs.vStar[c - d.P] * hx;
                const double b = massW - massE + massS - massN;
                const double ab = fabs(b);
                acc[3] = dmax(acc[3], ab);
                acc[2] += ab * ab;
                if (j <= N - 2) {
                    const double du = fs.uStar[c] - fs.u[c];
                    acc[0] += du * du;
                    const TC rb = (TC)b;
                    fs.B.rhs[c] = rb;
                    // level-0 pressure-correction operator (pressure_solver.cpp:706-730)
                    const double aE = rho * fs.dE[c] * hy;
                    const double aW = (j > 1) ? rho * fs.dE[c - 1] * hy : 0.0;
                    const double aN = (i < M - 1) ? rho * fs.dN[c] * hx : 0.0;
                    const double aS = (i > 1) ? rho * fs.dN[c - d.P] * hx : 0.0;
                    double aP = aE + aW + aN + aS;
                    double extra = 0.0;
                    if (aP < 1e-20) { extra = 1.0 - aP; aP = 1.0; }
                    fs.B.fE[c] = (TC)aE;
                    if (i < M - 1) fs.B.fN[c] = (TC)aN;
                    fs.B.d[c] = (TC)aP;
                    fs.H.lv[0].dx[c] = (TC)extra;
                    fs.B.x[c] = (TC)0;
                    fs.B.r[c] = rb;
                    fs.H.lv[0].x[c] = (TC)fs.H.omega * rb / (TC)aP;   // stored pre-smoothed iterate
                    acc[4] += (double)rb * (double)rb;
                }
                if (i <= M - 2) {
                    const double dv = fs.vStar[c] - fs.v[c];
                    acc[1] += dv * dv;
                }
            }, [&](int, int g) {
                const double mx = warp_max(acc[3]);
                double s4[4] = {acc[0], acc[1], acc[2], acc[4]};
                block_sum<4>(s4, sm);
                if ((threadIdx.x & 31) == 0) sm[128 + (threadIdx.x >> 5)] = mx;
                __syncthreads();
                if (threadIdx.x == 0) {
                    double m = 0.0;
                    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) m = dmax(m, sm[128 + q]);
                    const double v[kBatchPartStride] = {s4[0], s4[1], s4[2], m, s4[3]};
                    write_part(g, v, kBatchPartStride);
                }
                __syncthreads();
                for (int q = 0; q < kBatchPartStride; ++q) acc[q] = 0.0;
            });
        }
        if (!sync(BP_MASS)) return;
        for_my_fields(isOn, [&](int f) {
            const int* to = s_toff;
            double tot[kBatchPartStride];
            tile_sum(f, tot, kBatchPartStride);
            double mx = 0.0;
            for (int g = to[f] + threadIdx.x; g < to[f + 1]; g += blockDim.x)
                mx = dmax(mx, ldd(a.ipart + (size_t)g * kBatchPartStride + 3));
            mx = warp_max(mx);
            if ((threadIdx.x & 31) == 0) sm[128 + (threadIdx.x >> 5)] = mx;
            __syncthreads();
            if (threadIdx.x == 0) {
                double m = 0.0;
                for (int q = 0; q < (int)(blockDim.x >> 5); ++q) m = dmax(m, sm[128 + q]);
                BState& b = bsv(f);
                b.mass[0] = tot[0]; b.mass[1] = tot[1]; b.mass[2] = tot[2]; b.mass[3] = m;
                b.rTol = fs.k.pTol * sqrt(tot[4]);
                b.cgOn = fs.k.maxP > 0;
                b.cgIt = 0;
                b.beta = 0.0;
            }
        });
        if (!sync(BP_MASSRED)) return;
        // ---- coarse operators: grid-wide levels, then the CTA levels and the
        // dense inverse on the field's reducer block
        for (int l = 1; l < a.maxLg; ++l) {
            for_tiles(l, [&](int f) { return isOn(f) && l < F[f].H.Lg; }, [&](int I, int J) {
                mg_coarsen_cell(fs.H.lv[l - 1], fs.H.lv[l], I, J);
            }, noFin);
            if (!sync(BP_COARSE)) return;
        }
        for_my_fields(isOn, [&](int) {
            for (int l = fs.H.Lg - 1; l < fs.H.L - 1; ++l) {
                for_cells(Split{(int)threadIdx.x, (int)blockDim.x}, fs.H.lv[l + 1].nI, fs.H.lv[l + 1].nJ,
                          [&](int I, int J) { mg_coarsen_cell(fs.H.lv[l], fs.H.lv[l + 1], I, J); });
                __syncthreads();
            }
            mg_dense_setup(fs.H.lv[fs.H.L - 1], fs.H.dense, dsm);
        });
        if (!sync(BP_COARSECTA)) return;
        // ---- V-cycle z = M r of the fields whose CG runs; per-tile r.z partials
        auto vcycle = [&]() -> bool {
            for (int l = 0; l < a.maxLg; ++l) {
                for_tiles(l + 1, [&](int f) { return cgOn(f) && l < F[f].H.Lg; }, [&](int I, int J) {
                    if (l == 0) mg_restrict0x_cell(fs.H.lv[0], fs.H.lv[1], I, J, fs.H.omega);
                    else mg_restrict_cell(fs.H.lv[l], fs.H.lv[l + 1], I, J, fs.H.omega);
                }, noFin);
                if (!sync(BP_RESTR)) return false;
            }
            for_my_fields(cgOn, [&](int) {
                if (fs.H.Lg < fs.H.L - 1) mg_cta_cycle(fs.H);
                else mg_dense_solve(fs.H.lv[fs.H.L - 1], fs.H.dense);
            });
            if (!sync(BP_VCTA)) return false;
            for (int l = a.maxLg - 1; l >= 0; --l) {
                double acc[1] = {0.0};
                for_tiles(l, [&](int f) { return cgOn(f) && l < F[f].H.Lg; }, [&](int i, int j) {
                    const MgLevel<TC>& fl = fs.H.lv[l];
                    const MgLevel<TC>& cl = fs.H.lv[l + 1];
                    const TC* e = (l + 1 < fs.H.Lg) ? cl.y : cl.x;
                    if (l == 0) {
                        if (j > fl.nJ) return;
                        const TC y = mg_prolong0x_cell(fl, cl, e, i, j, fs.H.omega, fs.H.scale);
                        acc[0] += (double)fl.b[lidx(fl, i, j)] * (double)y;
                    } else {
                        mg_prolong_smooth_cell(fl, cl, e, i, j, fs.H.omega, fs.H.scale);
                    }
                }, [&](int, int g) {
                    if (l == 0) {
                        block_sum<1>(acc, sm);
                        write_part(g, acc, 1);
                        acc[0] = 0.0;
                    }
                });
                if (!sync(BP_PROL)) return false;
            }
            return true;
        };
        if (!vcycle()) return;
        for_my_fields(cgOn, [&](int f) {
            double tot[kBatchPartStride];
            tile_sum(f, tot, 1);
            if (threadIdx.x == 0) bsv(f).rz = tot[0];
        });
        if (!sync(BP_VRED)) return;
        // ---- CG (pressure_solver.cpp:121-184 recurrences; AMGCL's relative stop)
        for (int it = 0; it < a.maxP; ++it) {
            const bool first = (it == 0);
            {
                double acc[1] = {0.0};
                double tBeta = 0.0;
                for_tiles(0, [&](int f) {
                        tBeta = ldd(&a.bs[f].beta);
                        return cgOn(f);
                    }, [&](int i, int j) {
                    const Dims d = fs.k.d;
                    if (j > d.N - 2) return;
                    const TC bt = (TC)tBeta;
                    const TC* z = fs.H.lv[0].y;
                    TC* pnew = (it & 1) ? fs.B.pb : fs.B.pa;
                    const TC* pold = (it & 1) ? fs.B.pa : fs.B.pb;
                    auto dir = [&](size_t q) -> TC { return first ? z[q] : (TC)(z[q] + bt * pold[q]); };
                    const size_t c = at(d, i, j);
                    const TC pc = dir(c);
                    const TC pS = (i > 1) ? dir(c - d.P) : (TC)0;
                    const TC pW = (j > 1) ? dir(c - 1) : (TC)0;
                    const TC pE = (j < d.N - 2) ? dir(c + 1) : (TC)0;
                    const TC pN = (i < d.M - 1) ? dir(c + d.P) : (TC)0;
                    const TC ap = fs.B.d[c] * pc - fs.B.fN[c - d.P] * pS - fs.B.fE[c - 1] * pW - fs.B.fE[c] * pE -
                                  fs.B.fN[c] * pN;
                    pnew[c] = pc;
                    fs.B.Ap[c] = ap;
                    acc[0] += (double)pc * (double)ap;
                }, [&](int, int g) {
                    block_sum<1>(acc, sm);
                    write_part(g, acc, 1);
                    acc[0] = 0.0;
                });
            }
            if (!sync(BP_MATVEC)) return;
            for_my_fields(cgOn, [&](int f) {
                double tot[kBatchPartStride];
                tile_sum(f, tot, 1);
                if (threadIdx.x == 0) {
                    BState& b = bsv(f);
                    if (fabs(tot[0]) < 1e-20) { b.cgOn = 0; b.cgIt = it; }
                    else b.alpha = b.rz / tot[0];
                }
            });
            if (!sync(BP_MVRED)) return;
            {
                double acc[1] = {0.0};
                double tAlpha = 0.0;
                for_tiles(0, [&](int f) {
                        tAlpha = ldd(&a.bs[f].alpha);
                        return cgOn(f);
                    }, [&](int i, int j) {
                    const Dims d = fs.k.d;
                    if (j > d.N - 2) return;
                    const TC al = (TC)tAlpha;
                    const TC* pnew = (it & 1) ? fs.B.pb : fs.B.pa;
                    const size_t c = at(d, i, j);
                    fs.B.x[c] = fs.B.x[c] + al * pnew[c];
                    const TC r = fs.B.r[c] - al * fs.B.Ap[c];
                    fs.B.r[c] = r;
                    fs.H.lv[0].x[c] = (TC)fs.H.omega * r / fs.B.d[c];
                    acc[0] += (double)r * (double)r;
                }, [&](int, int g) {
                    block_sum<1>(acc, sm);
                    write_part(g, acc, 1);
                    acc[0] = 0.0;
                });
            }
            if (!sync(BP_UPD)) return;
            for_my_fields(cgOn, [&](int f) {
                double tot[kBatchPartStride];
                tile_sum(f, tot, 1);
                if (threadIdx.x == 0) {
                    BState& b = bsv(f);
                    if (sqrt(tot[0]) <= b.rTol) { b.cgOn = 0; b.cgIt = it + 1; }
                    else if (it + 1 >= fs.k.maxP) { b.cgOn = 0; b.cgIt = fs.k.maxP; }
                }
            });
            if (!sync(BP_UPDRED)) return;
            {
                int any = 0;
                for (int f = 0; f < nf; ++f) any |= ldi(&a.bs[f].cgOn);
                if (!any) break;
            }
            if (!vcycle()) return;
            for_my_fields(cgOn, [&](int f) {
                double tot[kBatchPartStride];
                tile_sum(f, tot, 1);
                if (threadIdx.x == 0) {
                    BState& b = bsv(f);
                    b.beta = tot[0] / b.rz;
                    b.rz = tot[0];
                }
            });
            if (!sync(BP_VRED)) return;
        }
        // ---- p' (pressure_solver.cpp:814: p'(:, N-1) = 0)
        for_tiles(0, isOn, [&](int i, int j) {
            const Dims d = fs.k.d;
            if (j > d.N - 2) return;
            const size_t c = at(d, i, j);
            fs.pStar[c] = (double)fs.B.x[c];
            if (j == d.N - 2) fs.pStar[c + 1] = 0.0;
        }, noFin);
        if (!sync(BP_PSTAR)) return;
        // ---- correction (iterations.cpp:556-597)
        for_tiles(0, onVel, [&](int i, int j) {
            const Dims d = fs.k.d;
            const int M = d.M, N = d.N;
            const double maxVel = tVel;
            const size_t c = at(d, i, j);
            const double ps = fs.pStar[c];
            fs.p[c] += fs.k.pAlpha * ps;
            if (j <= N - 2) {
                double du = fs.dE[c] * (ps - fs.pStar[c + 1]);
                du = dmax(-maxVel, dmin(maxVel, du));
                fs.u[c] = dmax(-maxVel, dmin(maxVel, fs.uStar[c] + du));
            }
            if (i <= M - 2) {
                double dv = fs.dN[c] * (ps - fs.pStar[c + d.P]);
                dv = dmax(-maxVel, dmin(maxVel, dv));
                fs.v[c] = dmax(-maxVel, dmin(maxVel, fs.vStar[c] + dv));
            }
        }, noFin);
        if (!sync(BP_CORR)) return;
        // ---- BCs, then sampling, history row and stop rules of each field
        for_my_fields(isOn, [&](int f) {
            apply_bc(fs.k, fs.st->iter, fs.u, fs.v, fs.p, fs.gamma, threadIdx.x, blockDim.x);
            if (threadIdx.x == 0) fs.st->itersP = ldi(&a.bs[f].cgIt);
        });
        if (!sync(BP_BC2)) return;
        for_my_fields(isOn, [&](int f) {
            FinalizeArgs fa{fs.u, fs.v, fs.p, fs.gamma, a.bs[f].mass, 1, fs.hist, fs.histCap, fs.dpWin};
            finalize_block(fs.k, fs.st, fa);
        });
        if (!sync(BP_FIN)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int all = 1;
        for (int f = 0; f < nf; ++f) all &= (__ldcg(&F[f].st->done) != 0);
        *a.allDone = all;
    }
}

// ======================================================================== teams of CTAs
// The batched kernel of smoothed-aggregation fields (pressureSolverType 4).
// The grid is cut into teams of consecutive CTAs; each team takes the next
// field from a queue (largest first) and runs that field's outer iterations
// on its own, with its own bounded barrier, through the same device code as
// the single-field kernels (k_bc, k_assemble, k_jacobi, k_mass, k_pcg_sa,
// k_correct, k_finalize): fields never wait for each other, no field idles
// the SMs of another, and a team's barriers cost what a few CTAs' arrivals
// cost.  The partial sums of a phase are per team rank, summed in rank order.

// Everything one field's solve touches (device pointers of a single-field
// context plus its parameter block and hierarchy); copied into shared
// memory by the team's CTAs when they take the field.
template <typename TC>
struct BFieldSa {
    KParams k;
    Status* st;
    double *u, *v, *p, *uStar, *vStar, *pStar, *dE, *dN;
    const double *alpha, *gamma;
    MomSys<TC> U, V;
    TC *xU0, *xU1, *xV0, *xV1;
    PcgBufs<TC> B;
    SaHier<TC> H;
    double *partJ, *partM, *partP;   // the context's partial-sum scratch (>= 4 x team size doubles)
    double* hist;
    int histCap;
    double* dpWin;
};

constexpr int kTeamStride = 32;   // unsigned words between two teams' barrier counters (128 B)

struct TeamArgs {
    int nf;              // fields
    int team;            // CTAs per team
    int nTeams;          // teams (the CTAs past nTeams x team exit at once)
    int nOuter;          // outer iterations a field may run in this launch
    const int* order;    // [nf] queue order: field indices, largest first
    unsigned* tbar;      // [nTeams * kTeamStride] team barrier counters (zeroed before the launch)
    int* queue;          // [1 + 2 nTeams]: next queue position, then each team's last two picks
    int* err;            // first device error of the batch (barrier time-out)
    int* running;        // fields left running after this launch (zeroed before the launch)
};

// One outer iteration of field f on team T: the single-field sequence
// (enqueue_iteration) with each kernel's grid replaced by the team.
template <typename TC, bool Mixed>
__device__ __forceinline__ bool team_outer(const Team& T, unsigned& target, const BFieldSa<TC>& f) {
    const KParams& k = f.k;
    Status* st = f.st;
    const int tid = T.tid(), nth = T.nth();
    const int iter = __ldcg(&st->iter);
    // ---- k_bc (boundaries.cpp:50-146), max-change counters reset
    if (T.lead()) {
        st->maxDU = 0ull;
        st->maxDV = 0ull;
    }
    apply_bc(k, iter, f.u, f.v, f.p, f.gamma, tid, nth);
    if (!team_sync(T, target)) return false;
    // ---- k_assemble (momentum_solver.cpp:197-314)
    const double maxVel = max_vel(inlet_velocity(k, iter));
    {
        const Fields fl{f.u, f.v, f.p, f.alpha, f.gamma};
        const Dims d = k.d;
        const int nU = k.nU, nV = k.nV, wU = d.N - 2, wV = d.N - 1;
        for (int t = tid; t < nU + nV; t += nth) {
            if (t < nU) assemble_one<TC, Mixed, true>(k, fl, f.U, f.dE, 1 + t / wU, 1 + t % wU, maxVel);
            else assemble_one<TC, Mixed, false>(k, fl, f.V, f.dN, 1 + (t - nU) / wV, 1 + (t - nU) % wV, maxVel);
        }
    }
    if (!team_sync(T, target)) return false;
    // ---- k_jacobi: U sweeps, V sweeps, scatter with clamps, BCs on u*, v*
    {
        int curU = -1, curV = -1, itU = 0, itV = 0;
        if (!jacobi_component<TC, Mixed, true>(k, f.U, f.u, f.xU0, f.xU1, f.partJ, T, target, curU, itU))
            return false;
        if (!jacobi_component<TC, Mixed, false>(k, f.V, f.v, f.xV0, f.xV1, f.partJ + 2 * T.size, T, target, curV,
                                                itV))
            return false;
        double mu = jacobi_scatter<TC, Mixed, true>(k, f.u, curU < 0 ? nullptr : (curU ? f.xU1 : f.xU0), f.uStar,
                                                    maxVel, tid, nth);
        double mv = jacobi_scatter<TC, Mixed, false>(k, f.v, curV < 0 ? nullptr : (curV ? f.xV1 : f.xV0), f.vStar,
                                                     maxVel, tid, nth);
        mu = warp_max(mu);
        mv = warp_max(mv);
        if ((threadIdx.x & 31) == 0) {
            atomic_max_nonneg(&st->maxDU, mu);
            atomic_max_nonneg(&st->maxDV, mv);
        }
        if (T.lead()) {
            st->itersU = itU;
            st->itersV = itV;
        }
        if (!team_sync(T, target)) return false;
        apply_bc(k, iter, f.uStar, f.vStar, nullptr, f.gamma, tid, nth);
    }
    if (!team_sync(T, target)) return false;
    // ---- k_mass, then the smoothed-aggregation PCG (k_pcg_sa)
    mass_pass<TC>(k, f.u, f.v, f.uStar, f.vStar, f.B.rhs, tid, nth, f.partM + (size_t)T.rank * 4);
    if (!team_sync(T, target)) return false;
    if (!pcg_sa<TC>(T, target, k, st, f.dE, f.dN, f.B, f.H, f.pStar, f.partP)) return false;
    if (!team_sync(T, target)) return false;
    // ---- k_correct (iterations.cpp:556-597), k_bc, k_finalize
    correct_cells(k, iter, f.u, f.v, f.p, f.uStar, f.vStar, f.pStar, f.dE, f.dN, tid, nth);
    if (!team_sync(T, target)) return false;
    apply_bc(k, iter, f.u, f.v, f.p, f.gamma, tid, nth);
    if (!team_sync(T, target)) return false;
    if (T.rank == 0) {
        const FinalizeArgs fa{f.u, f.v, f.p, f.gamma, f.partM, T.size, f.hist, f.histCap, f.dpWin};
        finalize_block(k, st, fa);
    }
    return team_sync(T, target);
}

template <typename TC, bool Mixed>
__global__ void __launch_bounds__(kBatchThreads, 1) k_batch_team(TeamArgs a, const BFieldSa<TC>* __restrict__ F) {
    __shared__ __align__(16) BFieldSa<TC> fs;
    const int team = blockIdx.x / a.team;
    if (team >= a.nTeams) return;
    const Team T{(int)blockIdx.x - team * a.team, a.team, a.tbar + (size_t)team * kTeamStride, a.err};
    int* pick = a.queue + 1 + 2 * team;
    unsigned target = 0;
    for (int n = 0;; ++n) {
        // the team's next field: drawn by its lead thread, read by every CTA
        // after the barrier (two slots, so a slow CTA still reads its pick
        // while the lead draws the next one)
        if (T.lead()) pick[n & 1] = atomicAdd(a.queue, 1);
        if (!team_sync(T, target)) return;
        const int q = __ldcg(pick + (n & 1));
        if (q >= a.nf) break;
        const BFieldSa<TC>* src = F + __ldg(a.order + q);
        {
            const int* from = reinterpret_cast<const int*>(src);
            int* to = reinterpret_cast<int*>(&fs);
            for (int e = threadIdx.x; e < (int)(sizeof(BFieldSa<TC>) / sizeof(int)); e += blockDim.x)
                to[e] = __ldg(from + e);
            __syncthreads();
        }
        int o = 0;
        for (; o < a.nOuter; ++o) {
            // st->done is written by finalize on rank 0 before the barrier that
            // ends the iteration (or by an earlier call), so every CTA reads
            // the same value
            if (__ldcg(&fs.st->done)) break;
            if (!team_outer<TC, Mixed>(T, target, fs)) return;
        }
        if (T.lead() && o == a.nOuter && !__ldcg(&fs.st->done)) atomicAdd(a.running, 1);
        __syncthreads();
    }
}

}  // namespace cp
