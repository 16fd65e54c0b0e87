// SIMPLE outer-iteration kernels for sm_100a.
//
// One outer iteration (SIMPLE::calculateStep, iterations.cpp:82-659, with
// momentumSolverType 1) runs as:
//   k_bc        velocity + pressure boundary conditions     boundaries.cpp:50-146
//   k_assemble  U and V momentum coefficients, fused:        momentum_solver.cpp:197-314
//               FOU upwinding, half-cell walls, Brinkman,    boundaries.cpp:148-206
//               2.5-D sink, relaxation, SOU correction,      convection.cpp:53-186
//               dE/dN, boundary neighbours folded into b
//   k_jacobi    persistent: Jacobi sweeps of U and V         jacobi_solver.cpp:44-67
//               together, stop rule per component, then
//               scatter/clamp/max-change and BCs on u*, v*   momentum_solver.cpp:335-351
//   k_mass      RMS of u*-u, v*-v; mass imbalance; PCG rhs   iterations.cpp:499-533,
//                                                            pressure_solver.cpp:471-488,733-742
//   k_pcg       persistent: matrix-free Jacobi-PCG on p'     pressure_solver.cpp:121-184
//   k_correct   p += pAlpha p'; u, v corrections + clamps    iterations.cpp:556-597
//   k_bc        boundary conditions again                    iterations.cpp:567,599
//   k_finalize  pressure-drop sampling, residual reporting,  postprocessing.cpp:103-327,
//               history row and the stop rules              SIMPLE.cpp:378-491
//
// All kernels return immediately once Status::done is set, so a captured
// graph of one iteration can be replayed past convergence at no cost.
//
// Precision: fields (u, v, p, u*, v*, p', dE, dN) are double.  The inner
// systems are stored in TC (double for the FP64 form, float for the mixed
// form).  In the mixed form the momentum sweeps solve for a correction
// delta of the current velocity, A delta = b - A u, whose right-hand side is
// formed in double, and the PCG runs in float on the double mass imbalance;
// all global sums are double.
#pragma once

#include "cp_device.cuh"

namespace cp {

// ------------------------------------------------------------------ systems
template <typename TC>
struct MomSys {
    TC *aP, *aE, *aW, *aN, *aS, *b;   // b: rhs (FP64 form) or b - A u (mixed form)
};

template <typename TC>
struct PcgBufs {
    TC *fE, *fN, *d;      // face coefficients rho*dE*hy (E face), rho*dN*hx (N face); diagonal
    TC *x, *r, *pa, *pb, *Ap;
    TC* rhs;              // mass imbalance per unknown (written by k_mass)
};

// ------------------------------------------------------------------ k_bc
// Velocity BCs (boundaries.cpp:50-118) on (u, v) and, when p != nullptr,
// pressure BCs (boundaries.cpp:123-146).  Every write reads only interior
// values, so the reference's sequential order is reproduced in parallel.
__device__ __forceinline__ bool inlet_fluid(const KParams& k, const double* gamma, int uRow) {
    const int M = k.d.M;
    int cellRow = uRow <= 0 ? 0 : (uRow >= M ? (M - 2 > 0 ? M - 2 : 0) : uRow - 1);
    cellRow = cellRow < 0 ? 0 : (cellRow > M - 1 ? M - 1 : cellRow);
    return gamma[at(k.d, cellRow, 0)] > 0.5;
}

__device__ __forceinline__ void apply_bc(const KParams& k, int iter, double* u, double* v, double* p,
                                         const double* gamma, int t0, int stride) {
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const double Uin = inlet_velocity(k, iter);
    const int L = (M > N ? M : N) + 1;
    for (int t = t0; t < L; t += stride) {
        if (t <= M) u[at(d, t, 0)] = inlet_fluid(k, gamma, t) ? Uin : 0.0;
        if (t >= 1 && t <= N - 1) { u[at(d, 0, t)] = 0.0; u[at(d, M, t)] = 0.0; }
        if (t >= 1 && t <= M - 1) u[at(d, t, N - 1)] = u[at(d, t, N - 2)];
        if (t <= N) { v[at(d, 0, t)] = 0.0; v[at(d, M - 1, t)] = 0.0; }
        if (t >= 1 && t <= M - 2) { v[at(d, t, 0)] = 0.0; v[at(d, t, N)] = v[at(d, t, N - 1)]; }
        if (p) {
            if (t >= 1 && t <= N - 1) { p[at(d, 0, t)] = p[at(d, 1, t)]; p[at(d, M, t)] = p[at(d, M - 1, t)]; }
            if (t >= 1 && t <= M - 1) { p[at(d, t, 0)] = p[at(d, t, 1)]; p[at(d, t, N)] = 0.0; }
        }
    }
}

__global__ void k_bc(KParams k, Status* st, double* u, double* v, double* p, const double* gamma, int resetMax) {
    if (st->done) return;
    const int iter = st->iter;
    if (resetMax && blockIdx.x == 0 && threadIdx.x == 0) {
        st->maxDU = 0ull;
        st->maxDV = 0ull;
    }
    apply_bc(k, iter, u, v, p, gamma, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ------------------------------------------------------------------ assembly
// Face averages of cell fields (SIMPLE.h:642-686, 740-778); the callers only
// pass unknowns, for which the reference's range checks always pass.
struct Fields {
    const double *u, *v, *p, *alpha, *gamma;
};

template <bool IsU>
struct AssembledRow {
    double aP0, aP, aE, aW, aN, aS, Sp;
};

// Coefficients of one momentum unknown; see momentum_solver.cpp:204-313.
template <bool IsU>
__device__ __forceinline__ void assemble_row(const KParams& k, const Fields& f, int i, int j, double maxVel,
                                             AssembledRow<IsU>& out) {
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const double* u = f.u;
    const double* v = f.v;
    const double hx = k.hx, hy = k.hy, vol = hx * hy, rho = k.rho, eta = k.eta;
    double alphaLocal, gammaFace, ue, uw, vn, vs;
    if (IsU) {
        alphaLocal = 0.5 * (f.alpha[at(d, i - 1, j - 1)] + f.alpha[at(d, i - 1, j)]);
        gammaFace = 0.5 * (f.gamma[at(d, i - 1, j - 1)] + f.gamma[at(d, i - 1, j)]);
        ue = dclamp(0.5 * (u[at(d, i, j)] + u[at(d, i, j + 1)]), -maxVel, maxVel);
        uw = dclamp(0.5 * (u[at(d, i, j - 1)] + u[at(d, i, j)]), -maxVel, maxVel);
        vn = dclamp(0.5 * (v[at(d, i, j)] + v[at(d, i, j + 1)]), -maxVel, maxVel);
        vs = dclamp(0.5 * (v[at(d, i - 1, j)] + v[at(d, i - 1, j + 1)]), -maxVel, maxVel);
    } else {
        alphaLocal = 0.5 * (f.alpha[at(d, i - 1, j - 1)] + f.alpha[at(d, i, j - 1)]);
        gammaFace = 0.5 * (f.gamma[at(d, i - 1, j - 1)] + f.gamma[at(d, i, j - 1)]);
        ue = dclamp(0.5 * (u[at(d, i, j)] + u[at(d, i + 1, j)]), -maxVel, maxVel);
        uw = dclamp(0.5 * (u[at(d, i, j - 1)] + u[at(d, i + 1, j - 1)]), -maxVel, maxVel);
        vn = dclamp(0.5 * (v[at(d, i, j)] + v[at(d, i + 1, j)]), -maxVel, maxVel);
        vs = dclamp(0.5 * (v[at(d, i - 1, j)] + v[at(d, i, j)]), -maxVel, maxVel);
    }
    const double cs = k.convScale;
    const double Fe = cs * rho * hy * ue, Fw = cs * rho * hy * uw;
    const double Fn = cs * rho * hx * vn, Fs = cs * rho * hx * vs;
    const double De = eta * (hy / hx), Dn = eta * (hx / hy);
    double aE = De + dmax(0.0, -Fe);
    double aW = De + dmax(0.0, Fw);
    double aN = Dn + dmax(0.0, -Fn);
    double aS = Dn + dmax(0.0, Fs);
    // face-local half-cell diffusion next to external no-slip walls
    const double vt = 1e-8;
    if (gammaFace >= 0.999) {
        if (IsU) {
            if (i == 1 && fabs(u[at(d, 0, j)]) <= vt && fabs(v[at(d, 0, j)]) <= vt && fabs(v[at(d, 0, j + 1)]) <= vt)
                aS += Dn;
            if (i == M - 1 && fabs(u[at(d, M, j)]) <= vt && fabs(v[at(d, M - 1, j)]) <= vt &&
                fabs(v[at(d, M - 1, j + 1)]) <= vt)
                aN += Dn;
        } else {
            if (j == 1 && !(fabs(k.targetVel) > vt) && fabs(v[at(d, i, 0)]) <= vt && fabs(u[at(d, i, 0)]) <= vt &&
                fabs(u[at(d, i + 1, 0)]) <= vt)
                aW += De;
            if (j == N - 1 && !(fabs(f.p[at(d, i, N)]) <= 1e-8) && fabs(v[at(d, i, N)]) <= vt &&
                fabs(u[at(d, i, N - 1)]) <= vt && fabs(u[at(d, i + 1, N - 1)]) <= vt)
                aE += De;
        }
    }
    const double sumA = aE + aW + aN + aS;
    double aP0 = sumA + (Fe - Fw + Fn - Fs) + k.sinkDiag + alphaLocal * vol;
    aP0 = dmax(aP0, 1e-10);
    double Sp;
    const double* w = IsU ? u : v;
    if (IsU) Sp = (f.p[at(d, i, j)] - f.p[at(d, i, j + 1)]) * hy;
    else Sp = (f.p[at(d, i, j)] - f.p[at(d, i + 1, j)]) * hx;
    Sp += (1.0 - k.uvAlpha) / k.uvAlpha * aP0 * w[at(d, i, j)];
    if (k.sou) {
        // deferred correction S = sum over faces of -/+ F (phi_SOU - phi_FOU)
        // with the reference's stencil-availability guards
        const int iMaxE = IsU ? N : N + 1;   // column count of this component
        const int iMaxR = IsU ? M + 1 : M;   // row count of this component
        double S = 0.0;
#define W_(a, b) w[at(d, (a), (b))]
        if (Fe >= 0.0) { if (j >= 2) S -= Fe * ((1.5 * W_(i, j) - 0.5 * W_(i, j - 1)) - W_(i, j)); }
        else { if (j + 2 < iMaxE) S -= Fe * ((1.5 * W_(i, j + 1) - 0.5 * W_(i, j + 2)) - W_(i, j + 1)); }
        if (Fw >= 0.0) { if (j >= 2) S += Fw * ((1.5 * W_(i, j - 1) - 0.5 * W_(i, j - 2)) - W_(i, j - 1)); }
        else { if (j + 1 < iMaxE) S += Fw * ((1.5 * W_(i, j) - 0.5 * W_(i, j + 1)) - W_(i, j)); }
        if (Fn >= 0.0) { if (i >= 1) S -= Fn * ((1.5 * W_(i, j) - 0.5 * W_(i - 1, j)) - W_(i, j)); }
        else { if (i + 2 < iMaxR) S -= Fn * ((1.5 * W_(i + 1, j) - 0.5 * W_(i + 2, j)) - W_(i + 1, j)); }
        if (Fs >= 0.0) { if (i >= 2) S += Fs * ((1.5 * W_(i - 1, j) - 0.5 * W_(i - 2, j)) - W_(i - 1, j)); }
        else { if (i + 1 < iMaxR) S += Fs * ((1.5 * W_(i, j) - 0.5 * W_(i + 1, j)) - W_(i, j)); }
#undef W_
        Sp += S;
    }
    out.aP0 = aP0;
    out.aP = aP0 / k.uvAlpha;
    out.aE = aE; out.aW = aW; out.aN = aN; out.aS = aS;
    out.Sp = Sp;
}

// Range of unknowns of one component: U i in [1, M-1], j in [1, N-2];
// V i in [1, M-2], j in [1, N-1] (momentum_solver.cpp:52-72).
template <bool IsU>
__host__ __device__ __forceinline__ void mom_range(const Dims& d, int& i1, int& j1) {
    i1 = IsU ? d.M - 1 : d.M - 2;
    j1 = IsU ? d.N - 2 : d.N - 1;
}

template <typename TC, bool Mixed, bool IsU>
__device__ __forceinline__ void assemble_one(const KParams& k, const Fields& f, MomSys<TC> sys, double* dEN,
                                             int i, int j, double maxVel) {
    const Dims d = k.d;
    int i1, j1;
    mom_range<IsU>(d, i1, j1);
    AssembledRow<IsU> a;
    assemble_row<IsU>(k, f, i, j, maxVel, a);
    const double* w = IsU ? f.u : f.v;
    const size_t c = at(d, i, j);
    // boundary neighbours go to the rhs with their current value, in the
    // order E, W, N, S (momentum_solver.cpp:300-303)
    const bool eIn = j + 1 <= j1, wIn = j >= 2, nIn = i + 1 <= i1, sIn = i >= 2;
    double Sp = a.Sp;
    if (!eIn) Sp += a.aE * w[c + 1];
    if (!wIn) Sp += a.aW * w[c - 1];
    if (!nIn) Sp += a.aN * w[c + d.P];
    if (!sIn) Sp += a.aS * w[c - d.P];
    const double cE = eIn ? a.aE : 0.0, cW = wIn ? a.aW : 0.0, cN = nIn ? a.aN : 0.0, cS = sIn ? a.aS : 0.0;
    dEN[c] = (IsU ? k.hy : k.hx) / a.aP0;
    sys.aP[c] = (TC)a.aP;
    sys.aE[c] = (TC)cE;
    sys.aW[c] = (TC)cW;
    sys.aN[c] = (TC)cN;
    sys.aS[c] = (TC)cS;
    if (Mixed) {
        // right-hand side of the correction: b - A u, formed in double
        double Au = a.aP * w[c];
        if (sIn) Au -= cS * w[c - d.P];
        if (wIn) Au -= cW * w[c - 1];
        if (eIn) Au -= cE * w[c + 1];
        if (nIn) Au -= cN * w[c + d.P];
        sys.b[c] = (TC)(Sp - Au);
    } else {
        sys.b[c] = (TC)Sp;
    }
}

template <typename TC, bool Mixed>
__global__ void __launch_bounds__(256, 4) k_assemble(KParams k, const Status* st, Fields f, MomSys<TC> U, MomSys<TC> V, double* dE,
                           double* dN, int doU, int doV) {
    if (st->done) return;
    const double maxVel = max_vel(inlet_velocity(k, st->iter));
    const Dims d = k.d;
    const int nU = doU ? k.nU : 0, nV = doV ? k.nV : 0;
    const int wU = d.N - 2, wV = d.N - 1;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV; t += gridDim.x * blockDim.x) {
        if (t < nU) {
            const int i = 1 + t / wU, j = 1 + t % wU;
            assemble_one<TC, Mixed, true>(k, f, U, dE, i, j, maxVel);
        } else {
            const int s = t - nU;
            const int i = 1 + s / wV, j = 1 + s % wV;
            assemble_one<TC, Mixed, false>(k, f, V, dN, i, j, maxVel);
        }
    }
}

// ------------------------------------------------------------------ Jacobi
// One component's sweeps.  Each thread handles two rows per loop trip with
// all loads issued before the arithmetic (memory-level parallelism); the
// sum of r^2 is reduced per sweep, one grid barrier per sweep.  Returns the
// buffer index holding the result (-1: the initial iterate) and the sweep
// count, or false if a barrier gave up.
template <typename TC, bool Mixed, bool IsU>
__device__ __forceinline__ bool jacobi_component(const KParams& k, const MomSys<TC>& S, const double* field,
                                                 TC* x0, TC* x1, double* part, const Team& T, unsigned& target,
                                                 int& cur, int& its) {
    __shared__ double sm[32];
    const Dims d = k.d;
    const int G = T.size;
    int i1, j1;
    mom_range<IsU>(d, i1, j1);
    const int n = i1 * j1;
    const double lim = k.momTol * k.momTol * (double)n;
    TC* xs[2] = {x0, x1};
    cur = -1;
    its = 0;
    for (int s = 0; s < k.maxMom; ++s) {
        const int nxt = cur < 0 ? 0 : 1 - cur;
        const TC* xc = cur < 0 ? nullptr : xs[cur];
        TC* __restrict__ xn = xs[nxt];
        const bool first = cur < 0;
        double acc[1] = {0.0};
        // row segments: a lane takes 16 bytes of a row (4 floats or 2
        // doubles); horizontal neighbours from the adjacent lanes
        constexpr int V = Vec16<TC>::n;
        row_segments<TC>(T, i1, j1, [&](int i, int j0, bool act, int lane) {
            const size_t c = at(d, i, j0);
            auto Xv = [&](size_t q) -> Vec16<TC> {
                if (first) {
                    if constexpr (Mixed) return zero16<TC>();
                    else return ld16(field + q);
                }
                return ld16(xc + q);
            };
            auto Xs = [&](size_t q) -> TC {
                if (first) return Mixed ? (TC)0 : (TC)field[q];
                return xc[q];
            };
            Vec16<TC> aP = zero16<TC>(), aE = aP, aW = aP, aN = aP, aS = aP, b = aP, xP = aP, xN = aP, xS = aP;
            if (act) {
                aP = ld16(S.aP + c);
                aE = ld16(S.aE + c);
                aW = ld16(S.aW + c);
                aN = ld16(S.aN + c);
                aS = ld16(S.aS + c);
                b = ld16(S.b + c);
                xP = Xv(c);
                if (i > 1) xS = Xv(c - d.P);
                if (i < i1) xN = Xv(c + d.P);
            }
            TC xw = from_west(xP.v[V - 1]), xe = from_east(xP.v[0]);
            if (lane == 0) xw = (act && j0 > 0) ? Xs(c - 1) : (TC)0;
            if (lane == 31) xe = act ? Xs(c + V) : (TC)0;
            Vec16<TC> o;
#pragma unroll
            for (int q = 0; q < V; ++q) {
                const int j = j0 + q;
                const bool in = act && j >= 1 && j <= j1;
                const TC W = (j > 1) ? (q ? xP.v[q - 1] : xw) : (TC)0;
                const TC E = (j < j1) ? (q < V - 1 ? xP.v[q + 1] : xe) : (TC)0;
                // S, W, P, E, N order of the reference's CSR rows
                TC Ax = (TC)0;
                Ax += (-aS.v[q]) * xS.v[q];
                Ax += (-aW.v[q]) * W;
                Ax += aP.v[q] * xP.v[q];
                Ax += (-aE.v[q]) * E;
                Ax += (-aN.v[q]) * xN.v[q];
                const TC r = b.v[q] - Ax;
                o.v[q] = in ? (TC)(xP.v[q] + r / aP.v[q]) : (TC)0;
                if (in) acc[0] += (double)r * (double)r;
            }
            if (act) st16(xn + c, o);
        });
        block_sum<1>(acc, sm);
        double* slot = part + (size_t)(s & 1) * G;
        if (threadIdx.x == 0) slot[T.rank] = acc[0];
        if (!team_sync(T, target)) return false;
        double tot[1];
        sum_partials<1>(slot, G, 1, tot, sm);
        cur = nxt;
        its = s + 1;
        if (tot[0] < lim) break;
    }
    return true;
}

// scatter with clamp and max |u* - u| (momentum_solver.cpp:335-351)
template <typename TC, bool Mixed, bool IsU>
__device__ __forceinline__ double jacobi_scatter(const KParams& k, const double* field, const TC* xr,
                                                 double* out, double maxVel, int tid, int nth) {
    const Dims d = k.d;
    int i1, j1;
    mom_range<IsU>(d, i1, j1);
    const int w = j1, n = i1 * j1;
    double m = 0.0;
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        double xv = xr ? (double)xr[c] : (Mixed ? 0.0 : field[c]);
        if (Mixed) xv += field[c];
        const double nv = dclamp(xv, -maxVel, maxVel);
        m = dmax(m, fabs(nv - field[c]));
        out[c] = nv;
    }
    return m;
}

// Jacobi sweeps x+ = x + (b - A x) / aP of the U system, then of the V
// system (they are independent: V assembles from u, v, not from u*).  Each
// component stops after the first sweep whose pre-update sum of r^2 is
// below tol^2 n, or after maxMomentumIter sweeps (jacobi_solver.cpp:44-67).
// Running the components one after the other keeps one component's system
// resident in L2.  Then the scatter with clamps and the BCs on u*, v*.
struct JacobiOut {
    double *uStar, *vStar;
};

template <typename TC, bool Mixed>
__global__ void __launch_bounds__(256) k_jacobi(KParams k, Status* st, MomSys<TC> U, MomSys<TC> V,
                                                const double* u, const double* v, TC* xU0, TC* xU1, TC* xV0,
                                                TC* xV1, JacobiOut out, const double* gamma, double* part,
                                                unsigned* bar, int doU, int doV, int applyBC) {
    if (st->done) return;
    const int G = gridDim.x;
    const int iter = st->iter;
    const double maxVel = max_vel(inlet_velocity(k, iter));
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = G * blockDim.x;
    unsigned target = 0;
    const Team T = grid_team(bar, &st->err);
    int curU = -1, curV = -1, itU = 0, itV = 0;
    if (doU && !jacobi_component<TC, Mixed, true>(k, U, u, xU0, xU1, part, T, target, curU, itU)) return;
    // V uses its own partial slots: blocks may still read U's last sums
    if (doV && !jacobi_component<TC, Mixed, false>(k, V, v, xV0, xV1, part + 2 * G, T, target, curV, itV))
        return;
    double mu = 0.0, mv = 0.0;
    if (doU) mu = jacobi_scatter<TC, Mixed, true>(k, u, curU < 0 ? nullptr : (curU ? xU1 : xU0), out.uStar, maxVel, tid, nth);
    if (doV) mv = jacobi_scatter<TC, Mixed, false>(k, v, curV < 0 ? nullptr : (curV ? xV1 : xV0), out.vStar, maxVel, tid, nth);
    mu = warp_max(mu);
    mv = warp_max(mv);
    if ((threadIdx.x & 31) == 0) {
        atomic_max_nonneg(&st->maxDU, mu);
        atomic_max_nonneg(&st->maxDV, mv);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (doU) st->itersU = itU;
        if (doV) st->itersV = itV;
    }
    if (applyBC) {
        target += G;
        if (!grid_barrier(bar, target, &st->err)) return;
        apply_bc(k, iter, out.uStar, out.vStar, nullptr, gamma, tid, nth);
    }
}

// ------------------------------------------------------------------ mass
// One pass over cells (i, j) in [1, M-1] x [1, N-1]: RMS sums of u* - u and
// v* - v over their unknowns (iterations.cpp:507-525), the mass imbalance
// max and sum of squares (pressure_solver.cpp:473-487), and the PCG rhs on
// the pressure unknowns j <= N-2 (pressure_solver.cpp:733-742).
// part[b*4 + {0,1,2,3}] = {sum du^2, sum dv^2, sum b^2, max |b|}.
template <typename TV>
__device__ __forceinline__ void mass_pass(const KParams& k, const double* u, const double* v, const double* uStar,
                                          const double* vStar, TV* rhs, int tid, int nth, double* o) {
    __shared__ double sm[128];
    const Dims d = k.d;
    const int M = d.M, N = d.N, w = N - 1;
    const double rho = k.rho, hx = k.hx, hy = k.hy;
    double acc[3] = {0.0, 0.0, 0.0};
    double mmax = 0.0;
    const int n = (M - 1) * w;
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        const double massE = rho * uStar[c] * hy, massW = rho * uStar[c - 1] * hy;
        const double massN = rho * vStar[c] * hx, massS = rho * vStar[c - d.P] * hx;
        const double b = massW - massE + massS - massN;
        const double ab = fabs(b);
        mmax = dmax(mmax, ab);
        acc[2] += ab * ab;
        if (j <= N - 2) {
            const double du = uStar[c] - u[c];
            acc[0] += du * du;
            rhs[c] = (TV)b;
        }
        if (i <= M - 2) {
            const double dv = vStar[c] - v[c];
            acc[1] += dv * dv;
        }
    }
    block_sum<3>(acc, sm);
    mmax = warp_max(mmax);
    if ((threadIdx.x & 31) == 0) sm[96 + (threadIdx.x >> 5)] = mmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int q = 0; q < (int)((blockDim.x + 31) >> 5); ++q) m = dmax(m, sm[96 + q]);
        o[0] = acc[0]; o[1] = acc[1]; o[2] = acc[2]; o[3] = m;
    }
}

template <typename TV>
__global__ void k_mass(KParams k, const Status* st, const double* u, const double* v, const double* uStar,
                       const double* vStar, TV* rhs, double* part) {
    if (st->done) return;
    mass_pass<TV>(k, u, v, uStar, vStar, rhs, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x,
                  part + (size_t)blockIdx.x * 4);
}

// ------------------------------------------------------------------ PCG
// Jacobi-preconditioned CG on the pressure correction (pressure_solver.cpp:121-184):
//   unknowns (i, j) in [1, M-1] x [1, N-2]; p'(:, N-1) = 0;
//   aE = rho dE(i,j) hy, aW = rho dE(i,j-1) hy (j > 1), aN = rho dN(i,j) hx
//   (i < M-1), aS = rho dN(i-1,j) hx (i > 1); aP = aE+aW+aN+aS (1 if < 1e-20).
// Matrix-free: fE(i,j) holds the east-face coefficient (zero at j = 0) and
// fN(i,j) the north-face one (zero at rows 0 and M-1); direction vectors are
// zero outside the unknowns, so the stencil needs no branches.
// Per iteration two grid barriers:
//   A: p_new = z + beta p_old (recomputed at the 4 neighbours from r, d,
//      p_old; written to the other buffer), Ap = A p_new, partial p.Ap
//   B: x += alpha p_new, r -= alpha Ap, partials r.r and r.z
// The reference's early exits are kept: |p.Ap| < 1e-20 and sqrt(r.r) < pTol,
// and the returned count is the loop index at exit (maxPressureIter if none).
template <typename TV>
__device__ __forceinline__ TV pcg_dir(const TV* r, const TV* dd, const TV* pold, size_t c, double beta,
                                      bool first) {
    const TV z = r[c] / dd[c];
    return first ? z : (TV)(z + (TV)beta * pold[c]);
}

template <typename TV>
__global__ void __launch_bounds__(256) k_pcg(KParams k, Status* st, const double* dE, const double* dN,
                                             PcgBufs<TV> B, double* pStar, double* part, unsigned* bar) {
    if (st->done) return;
    __shared__ double sm[96];
    const Dims d = k.d;
    const int M = d.M, N = d.N, w = N - 2;
    const int n = (M - 1) * w;
    const int G = gridDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = G * blockDim.x;
    const double rho = k.rho, hx = k.hx, hy = k.hy;
    unsigned target = 0;
    double* partA = part;           // [G]     p.Ap
    double* partB = part + G;       // [G][2]  r.r, r.z
    // init: faces, diagonal, x = 0, r = b (A 0 = 0), partial r.z
    double acc0[1] = {0.0};
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
        if (i < M - 1) B.fN[c] = (TV)aN;
        B.d[c] = (TV)aP;
        B.x[c] = (TV)0;
        const TV r = B.rhs[c];
        B.r[c] = r;
        acc0[0] += (double)r * (double)(r / (TV)aP);
    }
    block_sum<1>(acc0, sm);
    if (threadIdx.x == 0) partB[2 * blockIdx.x + 1] = acc0[0];
    target += G;
    if (!grid_barrier(bar, target, &st->err)) return;
    double tot1[1];
    {
        double t2[2];
        sum_partials<2>(partB, G, 2, t2, sm);
        tot1[0] = t2[1];
    }
    double rz = tot1[0];
    double beta = 0.0;
    int it = 0;
    TV* pbuf[2] = {B.pa, B.pb};
    for (; it < k.maxP; ++it) {
        const bool first = (it == 0);
        const TV* pold = pbuf[(it + 1) & 1];
        TV* pnew = pbuf[it & 1];
        double accA[1] = {0.0};
        for (int t = tid; t < n; t += nth) {
            const int i = 1 + t / w, j = 1 + t % w;
            const size_t c = at(d, i, j);
            const TV pc = pcg_dir(B.r, B.d, pold, c, beta, first);
            const TV pS = (i > 1) ? pcg_dir(B.r, B.d, pold, c - d.P, beta, first) : (TV)0;
            const TV pW = (j > 1) ? pcg_dir(B.r, B.d, pold, c - 1, beta, first) : (TV)0;
            const TV pE = (j < w) ? pcg_dir(B.r, B.d, pold, c + 1, beta, first) : (TV)0;
            const TV pN = (i < M - 1) ? pcg_dir(B.r, B.d, pold, c + d.P, beta, first) : (TV)0;
            TV ap = (TV)0;
            ap += (-B.fN[c - d.P]) * pS;
            ap += (-B.fE[c - 1]) * pW;
            ap += B.d[c] * pc;
            ap += (-B.fE[c]) * pE;
            ap += (-B.fN[c]) * pN;
            pnew[c] = pc;
            B.Ap[c] = ap;
            accA[0] += (double)pc * (double)ap;
        }
        block_sum<1>(accA, sm);
        if (threadIdx.x == 0) partA[blockIdx.x] = accA[0];
        target += G;
        if (!grid_barrier(bar, target, &st->err)) return;
        double pAp[1];
        sum_partials<1>(partA, G, 1, pAp, sm);
        if (fabs(pAp[0]) < 1e-20) break;
        const double alpha = rz / pAp[0];
        double accB[2] = {0.0, 0.0};
        for (int t = tid; t < n; t += nth) {
            const int i = 1 + t / w, j = 1 + t % w;
            const size_t c = at(d, i, j);
            const TV pc = pnew[c];
            B.x[c] = B.x[c] + (TV)alpha * pc;
            const TV r = B.r[c] - (TV)alpha * B.Ap[c];
            B.r[c] = r;
            accB[0] += (double)r * (double)r;
            accB[1] += (double)r * (double)(r / B.d[c]);
        }
        block_sum<2>(accB, sm);
        if (threadIdx.x == 0) { partB[2 * blockIdx.x] = accB[0]; partB[2 * blockIdx.x + 1] = accB[1]; }
        target += G;
        if (!grid_barrier(bar, target, &st->err)) return;
        double tB[2];
        sum_partials<2>(partB, G, 2, tB, sm);
        if (sqrt(tB[0]) < k.pTol) break;
        beta = tB[1] / rz;
        rz = tB[1];
    }
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        pStar[c] = (double)B.x[c];
        if (j == w) pStar[c + 1] = 0.0;  // p'(:, N-1) = 0 (pressure_solver.cpp:814)
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->itersP = it;
}

// ------------------------------------------------------------------ correction
// p += pAlpha p' on [1,M-1] x [1,N-1]; u = clamp(u* + clamp(dE (p'_ij - p'_i,j+1)))
// on U unknowns and the same for v (iterations.cpp:558-597).
__device__ __forceinline__ void correct_cells(const KParams& k, int iter, double* u, double* v, double* p,
                                              const double* uStar, const double* vStar, const double* pStar,
                                              const double* dE, const double* dN, int tid, int nth) {
    const Dims d = k.d;
    const int M = d.M, N = d.N, w = N - 1;
    const double maxVel = max_vel(inlet_velocity(k, iter));
    const int n = (M - 1) * w;
    for (int t = tid; t < n; t += nth) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        const double ps = pStar[c];
        p[c] += k.pAlpha * ps;
        if (j <= N - 2) {
            double du = dE[c] * (ps - pStar[c + 1]);
            du = dmax(-maxVel, dmin(maxVel, du));
            const double nu = uStar[c] + du;
            u[c] = dmax(-maxVel, dmin(maxVel, nu));
        }
        if (i <= M - 2) {
            double dv = dN[c] * (ps - pStar[c + d.P]);
            dv = dmax(-maxVel, dmin(maxVel, dv));
            const double nv = vStar[c] + dv;
            v[c] = dmax(-maxVel, dmin(maxVel, nv));
        }
    }
}

__global__ void k_correct(KParams k, const Status* st, double* u, double* v, double* p, const double* uStar,
                          const double* vStar, const double* pStar, const double* dE, const double* dN) {
    if (st->done) return;
    correct_cells(k, st->iter, u, v, p, uStar, vStar, pStar, dE, dN, blockIdx.x * blockDim.x + threadIdx.x,
                  gridDim.x * blockDim.x);
}

// ------------------------------------------------------------------ finalize
// Pressure sampling (postprocessing.cpp:103-327): metrics m[5] =
// {flowArea, massFlux, avgStatic, avgDynamic, avgTotal}.  Sums are double
// block reductions (the reference adds floats sequentially).
__device__ void finish_metrics(double area, double fs, double st, double dy, double tw, double* m) {
    double aS = 0.0, aD = 0.0, aT = 0.0;
    if (area > 0.0) { aS = st / area; aD = dy / area; }
    if (fs > 0.0) aT = tw / fs;
    else if (area > 0.0) aT = aS + aD;
    m[0] = area; m[1] = fs; m[2] = aS; m[3] = aD; m[4] = aT;
}

// kind 0: plane at x (interpolated), 1: inlet patch, 2: outlet patch
__device__ void sample_metric(const KParams& k, const double* u, const double* v, const double* p,
                              const double* gamma, int kind, double x, double* m, double* sm) {
    const Dims d = k.d;
    const int M = d.M, N = d.N, NC = N - 1;
    const double hx = k.hx, hy = k.hy, rho = k.rho;
    double acc[5] = {0, 0, 0, 0, 0};  // area, flux, static, dyn, totalWeighted
    int cl = 0, cr = 0;
    double t = 0.0;
    if (kind == 0 && NC > 1) {
        const double xMin = 0.5 * hx, xMax = ((double)NC - 0.5) * hx;
        const double xc = dmax(xMin, dmin(x, xMax));
        cl = (int)floor(xc / hx - 0.5);
        if (cl > NC - 2) cl = NC - 2;
        if (cl < 0) cl = 0;
        cr = cl + 1;
        const double xl = ((double)cl + 0.5) * hx, xr = ((double)cr + 0.5) * hx;
        t = (fabs(xr - xl) < 1e-12) ? 0.0 : (xc - xl) / (xr - xl);
        t = dmax(0.0, dmin(1.0, t));
    }
    for (int i = 1 + threadIdx.x; i < M; i += blockDim.x) {
        const int row = i - 1;
        const int vt = (i - 1 < M - 1) ? i - 1 : M - 1, vb = (i < M - 1) ? i : M - 1;
        double staticP, un, vtan;
        if (kind == 0) {
            if (cl < 0 || cl >= NC || cr < 0 || cr >= NC) continue;
            if (gamma[at(d, row, cl)] < 1.0 - 1e-6 || gamma[at(d, row, cr)] < 1.0 - 1e-6) continue;
            const int pl = cl + 1 < N ? cl + 1 : N, pr = cr + 1 < N ? cr + 1 : N;
            staticP = (1.0 - t) * p[at(d, i, pl)] + t * p[at(d, i, pr)];
            const int ul = cl < N - 1 ? cl : N - 1, ur = cr < N - 1 ? cr : N - 1;
            un = (1.0 - t) * u[at(d, i, ul)] + t * u[at(d, i, ur)];
            const int vl = cl < N ? cl : N, vr = cr < N ? cr : N;
            const double vTop = (1.0 - t) * v[at(d, vt, vl)] + t * v[at(d, vt, vr)];
            const double vBot = (1.0 - t) * v[at(d, vb, vl)] + t * v[at(d, vb, vr)];
            vtan = 0.5 * (vTop + vBot);
        } else {
            const bool inlet = (kind == 1);
            const int adj = inlet ? 0 : NC - 1;
            if (adj < 0 || adj >= NC) continue;
            if (gamma[at(d, row, adj)] < 1.0 - 1e-6) continue;
            const int uCol = inlet ? 0 : N - 1, pCol = inlet ? 0 : N, vCol = inlet ? 0 : N;
            staticP = p[at(d, i, pCol)];
            un = u[at(d, i, uCol)];
            vtan = 0.5 * (v[at(d, vt, vCol)] + v[at(d, vb, vCol)]);
        }
        const double vm = sqrt(un * un + vtan * vtan);
        const double dynP = 0.5 * rho * vm * vm;
        const double tot = staticP + dynP;
        acc[0] += hy;
        acc[2] += staticP * hy;
        acc[3] += dynP * hy;
        const double fa = fabs(rho * un * hy);
        if (fa > 0.0) { acc[1] += fa; acc[4] += tot * fa; }
    }
    block_sum<5>(acc, sm);
    finish_metrics(acc[0], acc[1], acc[2], acc[3], acc[4], m);
}

struct FinalizeArgs {
    const double *u, *v, *p, *gamma;
    const double* partM;   // k_mass partials
    int nbM;
    double* hist;          // [cap][kHistCols]
    int histCap;
    double* dpWin;         // [dpWindow]
};

// One block: residual norms from the k_mass partials, the four pressure
// samples, the history row and the stop rules of one field.
__device__ __forceinline__ void finalize_block(const KParams& k, Status* st, const FinalizeArgs& a) {
    __shared__ double sm[32 * 5];
    __shared__ double met[4][5];
    double sums[4];
    {
        double s4[4] = {0, 0, 0, 0};
        double mx = 0.0;
        for (int b = threadIdx.x; b < a.nbM; b += blockDim.x) {
            s4[0] += a.partM[b * 4 + 0];
            s4[1] += a.partM[b * 4 + 1];
            s4[2] += a.partM[b * 4 + 2];
            mx = dmax(mx, a.partM[b * 4 + 3]);
        }
        s4[3] = 0.0;
        double s3[3] = {s4[0], s4[1], s4[2]};
        block_sum<3>(s3, sm);
        mx = warp_max(mx);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
        __syncthreads();
        double m2 = (threadIdx.x < ((blockDim.x + 31) >> 5)) ? sm[threadIdx.x] : 0.0;
        m2 = warp_max(m2);
        __syncthreads();
        sums[0] = s3[0]; sums[1] = s3[1]; sums[2] = s3[2]; sums[3] = m2;
    }
    double m[5];
    sample_metric(k, a.u, a.v, a.p, a.gamma, 0, k.xCoreIn, m, sm);
    if (threadIdx.x == 0) for (int q = 0; q < 5; ++q) met[0][q] = m[q];
    sample_metric(k, a.u, a.v, a.p, a.gamma, 0, k.xCoreOut, m, sm);
    if (threadIdx.x == 0) for (int q = 0; q < 5; ++q) met[1][q] = m[q];
    sample_metric(k, a.u, a.v, a.p, a.gamma, 1, 0.0, m, sm);
    if (threadIdx.x == 0) for (int q = 0; q < 5; ++q) met[2][q] = m[q];
    sample_metric(k, a.u, a.v, a.p, a.gamma, 2, 0.0, m, sm);
    if (threadIdx.x == 0) for (int q = 0; q < 5; ++q) met[3][q] = m[q];
    __syncthreads();
    if (threadIdx.x != 0) return;

    const int iter = st->iter;
    const double nU = (double)k.nU, nV = (double)k.nV, nM = (double)((k.d.M - 1) * (k.d.N - 1));
    const double rmsU = nU > 0 ? sqrt(sums[0] / nU) : 0.0;
    const double rmsV = nV > 0 ? sqrt(sums[1] / nV) : 0.0;
    const double rmsM = nM > 0 ? sqrt(sums[2] / nM) : 0.0;
    const double maxM = sums[3];
    const double maxU = __longlong_as_double((long long)st->maxDU);
    const double maxV = __longlong_as_double((long long)st->maxDV);
    // residual normalisation bookkeeping (iterations.cpp:628-656)
    const double velFloor = dmax(k.velFloor, 1e-30), massFloor = dmax(k.massFloor, 1e-30);
    if (!st->rms0Uset && rmsU > velFloor) { st->rms0U = rmsU; st->rms0Uset = 1; }
    if (!st->rms0Vset && rmsV > velFloor) { st->rms0V = rmsV; st->rms0Vset = 1; }
    if (!st->rms0Mset && rmsM > massFloor) { st->rms0M = rmsM; st->rms0Mset = 1; }
    if (!st->rms0Uset) st->rms0U = velFloor;
    if (!st->rms0Vset) st->rms0V = velFloor;
    if (!st->rms0Mset) st->rms0M = massFloor;
    double rU = rmsU, rV = rmsV, rM = rmsM;
    if (k.normalized) { rU = rmsU / st->rms0U; rV = rmsV / st->rms0V; rM = rmsM / st->rms0M; }
    const double error = dmax(dmax(rU, rV), rM);
    const double coreTotal = met[0][4] - met[1][4], fullTotal = met[2][4] - met[3][4];
    const double coreStatic = met[0][2] - met[1][2], fullStatic = met[2][2] - met[3][2];
    if (iter < a.histCap) {
        double* h = a.hist + (size_t)iter * kHistCols;
        h[H_ITER] = iter; h[H_ERROR] = error; h[H_RMS_U] = rmsU; h[H_RMS_V] = rmsV; h[H_RMS_MASS] = rmsM;
        h[H_MAX_U] = maxU; h[H_MAX_V] = maxV; h[H_MAX_MASS] = maxM; h[H_ITERS_P] = st->itersP;
        h[H_CORE_TOTAL] = coreTotal; h[H_FULL_TOTAL] = fullTotal; h[H_CORE_STATIC] = coreStatic;
        h[H_FULL_STATIC] = fullStatic; h[H_IN_FLUX] = met[2][1]; h[H_OUT_FLUX] = met[3][1];
        h[H_ITERS_U] = st->itersU; h[H_ITERS_V] = st->itersV; h[H_RES_U] = rU; h[H_RES_V] = rV; h[H_RES_MASS] = rM;
    }
    st->lastError = error;
    // stop rules of the outer loop (SIMPLE.cpp:378, 449-491)
    int done = 0, reason = CP_RUNNING;
    if (!(error == error) || isinf(error) || !(coreTotal == coreTotal) || !(fullTotal == fullTotal)) {
        done = 1; reason = CP_STOP_ERROR;
        atomicCAS(&st->err, 0, (int)CP_ERR_NONFINITE);
    }
    if (st->err != 0) { done = 1; reason = CP_STOP_ERROR; }
    if (!done && k.dpConv && iter >= k.dpRampSteps && k.dpWindow > 0) {
        a.dpWin[st->dpIdx] = coreTotal;
        st->dpIdx = (st->dpIdx + 1) % k.dpWindow;
        if (st->dpIdx == 0) st->dpFilled = 1;
        if (st->dpFilled) {
            double sum = 0.0;
            for (int q = 0; q < k.dpWindow; ++q) sum += a.dpWin[q];
            const double mean = sum / (double)k.dpWindow;
            double var = 0.0;
            for (int q = 0; q < k.dpWindow; ++q) { const double df = a.dpWin[q] - mean; var += df * df; }
            const double sd = sqrt(var / (double)k.dpWindow);
            const double denom = dmax(fabs(mean), 1.0);
            const double stdPct = sd / denom * 100.0;
            const int last = (st->dpIdx - 1 + k.dpWindow) % k.dpWindow;
            const double latestPct = fabs(a.dpWin[last] - mean) / denom * 100.0;
            if (stdPct < k.dpPercent && latestPct < k.dpPercent) { done = 1; reason = CP_STOP_DP_WINDOW; }
        }
    }
    if (!done && !(error > k.eps)) { done = 1; reason = CP_STOP_RESIDUAL; }
    if (!done && iter + 1 >= k.maxIterations) { done = 1; reason = CP_STOP_MAX_ITER; }
    st->iter = iter + 1;
    if (done) { st->reason = reason; __threadfence(); st->done = 1; }
}

__global__ void __launch_bounds__(1024) k_finalize(KParams k, Status* st, FinalizeArgs a) {
    if (st->done) return;
    finalize_block(k, st, a);
}

}  // namespace cp
