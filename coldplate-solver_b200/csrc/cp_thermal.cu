// B200 3-D conjugate-heat-transfer solve (C ABI in include/cp_thermal.h).
//
// The reference (ThermalSolver/thermal_solver.cpp) assembles a 7-point
// finite-volume system on Nx x Ny x Nz cells into CSR on the host and solves
// it with AMGCL's IDR(s) preconditioned by smoothed-aggregation AMG
// (thermal_solver.cpp:417-553).  Here:
//   k_th_assemble   one thread per cell computes the reference's row in FP64
//                   (same formulas and summation order, thermal_solver.cpp:
//                   420-520) into seven coefficient arrays and b;
//   k_th_coarsen    Galerkin coarse operators P^T A P of a hierarchy that
//                   aggregates 2 x 2 columns (all z-layers kept) down to one
//                   column; P piecewise constant, so every level keeps the
//                   7-point form and the levels of A^T are the transposes;
//   k_th_lu         Thomas factors of every column's tridiagonal z-block, per
//                   level (z is the direction a column thread owns);
//   k_th_bicgstab   persistent cooperative BiCGStab right-preconditioned by
//                   one V-cycle: damped z-line Jacobi smoothing (one sweep
//                   down, one up; exact on the one-column level), residual
//                   restriction fused with the 2 x 2 sums, the prolongation
//                   formed on the fly in the two post-smoothing passes (the
//                   residual over cells, then the z-solve over columns,
//                   staged through shared memory); levels of at most
//                   kThCtaCols columns run in block 0 alone.  Bounded grid
//                   barriers, deterministic block sums, AMGCL's stop test
//                   ||r|| <= rtol ||b||.  The same kernel solves A^T x = rhs
//                   for the p-norm adjoint;
//   k_th_sens       dJ/dgamma from the adjoint field, one thread per column.
// Layout: every array is indexed k Nx Ny + j Nx + i (i contiguous), so the
// stencil loads of a warp are coalesced and a column thread walks k with
// stride Nx Ny.
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/cp_thermal.h"
#include "cp_device.cuh"

// error string of the library (cp_solver.cu)
cp_status cp_internal_set_error(cp_status s, const char* msg);

namespace {

cp_status tfail(cp_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return cp_internal_set_error(s, buf);
}

#define TCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return tfail(CP_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),      \
                         __FILE__, __LINE__);                                                      \
    } while (0)

constexpr int kThThreads = 256;
constexpr int kThZ = 16;                  // most layers (a column's sweep is kept in shared memory)
constexpr int kThMaxNz = kThZ;
#ifndef CP_TH_STAGE
#define CP_TH_STAGE 6
#endif
constexpr int kThStage = CP_TH_STAGE;     // layers per asynchronous staging chunk
constexpr int kThStageArr = 5;            // arrays staged per layer at most
constexpr size_t kThSmemBytes = (size_t)(kThZ + kThStageArr * kThStage) * kThThreads * sizeof(double);
constexpr int kThMaxLevels = 16;          // 2 x 2 aggregation from up to 2^15 columns per side
constexpr long long kThCtaCols = 64;      // levels of at most this many columns: block 0 alone
constexpr double kThOmega = 0.8;          // z-line Jacobi damping
constexpr double kThScale0 = 1.4;         // coarse-correction factor into level 0
constexpr double kThScale = 1.4;          // ... into the deeper levels (1.2 / 1.1: 95 / more iterations
                                          // at 1024 x 512 x 12, against 84)
constexpr int kThRefineRounds = 4;        // mixed precision: BiCGStab launches per solve at most

}  // namespace

namespace cp {

struct ThK {
    int Nx, Ny, Nz, nzS, nzF, mode;
    long long n, ncol;
    double dx, dy, dzS, dzF, Ht, kS, kF, rhoCp, Tin, qk;
};

// The seven coefficient arrays of a 7-point system and its right-hand side
// (T = double: the assembled system and its Galerkin levels; T = float: the
// preconditioner's copies in the mixed-precision solve)
template <typename T>
struct ThSysT {
    T *aP, *aW, *aE, *aS, *aN, *aB, *aT, *b;
};
using ThSys = ThSysT<double>;

struct ThStatus {
    int iterations, converged, err, pad;
    double residual;
};

__device__ __forceinline__ double th_dz(const ThK& k, int kk) { return kk < k.nzS ? k.dzS : k.dzF; }

// thermal_solver.cpp:271-305 (gamma clamped to [0, 1]); k_s in the base plate
__device__ __forceinline__ double th_kval(const ThK& k, const double* gamma, int i, int j, int kk) {
    if (kk < k.nzS) return k.kS;
    double g = gamma[(size_t)j * k.Nx + i];
    g = fmax(0.0, fmin(1.0, g));
    if (k.mode == 1) {
        const double num = 1.0 - g;
        const double den = 1.0 + __dmul_rn(k.qk, g);
        return k.kF + (k.kS - k.kF) * num / den;
    }
    if (k.mode == 2) return k.kS * k.kF / (__dmul_rn(1.0 - g, k.kF) + __dmul_rn(g, k.kS) + 1e-30);
    return __dmul_rn(k.kS, 1.0 - g) + __dmul_rn(k.kF, g);
}

// 1 = fluid: above the base plate with gamma > 0.01 (thermal_solver.cpp:240-244)
__device__ __forceinline__ bool th_fluid(const ThK& k, const double* gamma, int i, int j, int kk) {
    if (kk < k.nzS) return false;
    return gamma[(size_t)j * k.Nx + i] > 0.01;
}

// Poiseuille factor of a fluid layer (thermal_solver.cpp:323-327)
__device__ __forceinline__ double th_pois(const ThK& k, int kk) {
    if (kk < k.nzS) return 0.0;
    const double z = (kk - k.nzS + 0.5) * k.dzF / k.Ht;
    return 4.0 * z * (1 - z);
}

__device__ __forceinline__ double th_harm(double a, double b) { return 2 * a * b / (a + b + 1e-30); }

// One row of the reference's system, in its summation order
// (thermal_solver.cpp:420-520).  Every product that feeds a sum is rounded
// on its own (__dmul_rn) so that no multiply-add is fused and the row has the
// reference's bits.  Off-diagonal entries are the matrix values (negative);
// the reference's two entries for one neighbour (diffusion and upwind
// advection) are summed like its CSR conversion sums them.
__global__ void k_th_assemble(ThK k, const double* gamma, const double* u_xy, const double* v_xy, const double* q0,
                              ThSys S) {
    const int Nx = k.Nx, Ny = k.Ny, Nz = k.Nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < k.n;
         t += (long long)gridDim.x * blockDim.x) {
        const int kk = (int)(t / ((long long)Nx * Ny));
        const int rem = (int)(t - (long long)kk * Nx * Ny);
        const int j = rem / Nx, i = rem % Nx;
        const double dx = k.dx, dy = k.dy, rhoCp = k.rhoCp, T_in = k.Tin;
        const double dz_k = th_dz(k, kk), Ax = dy * dz_k, Ay = dx * dz_k, Az_cell = dx * dy;
        double diag = 0, bb = 0;
        const double kP = th_kval(k, gamma, i, j, kk), po = th_pois(k, kk);
        double g = (kk < k.nzS) ? 0.0 : gamma[(size_t)j * Nx + i];
        g = fmax(0.0, fmin(1.0, g));
        const double uP = (g > 0.01) ? __dmul_rn(u_xy[(size_t)j * Nx + i], po) : 0.0;
        const double vP = (g > 0.01) ? __dmul_rn(v_xy[(size_t)j * Nx + i], po) : 0.0;
        const bool regP = th_fluid(k, gamma, i, j, kk);
        double aW = 0, aE = 0, aS = 0, aN = 0, aB = 0, aT = 0;
        // x faces
        if (i > 0) {
            const double kf = th_harm(kP, th_kval(k, gamma, i - 1, j, kk)), D = kf * Ax / dx;
            diag += D;
            aW = -D;
            if (regP && th_fluid(k, gamma, i - 1, j, kk)) {
                const double uW = __dmul_rn(u_xy[(size_t)j * Nx + i - 1], po), F = rhoCp * 0.5 * (uP + uW) * Ax;
                diag += fmax(-F, 0.0);
                aW = aW + (-fmax(F, 0.0));
            }
        } else if (regP) {
            const double D_bc = 2.0 * kP * Ax / dx, F_bc = __dmul_rn(rhoCp * uP, Ax);
            diag += D_bc;
            bb += __dmul_rn(D_bc, T_in);
            if (F_bc > 0) bb += __dmul_rn(F_bc, T_in);
            else diag += -F_bc;
        }
        if (i < Nx - 1) {
            const double kf = th_harm(kP, th_kval(k, gamma, i + 1, j, kk)), D = kf * Ax / dx;
            diag += D;
            aE = -D;
            if (regP && th_fluid(k, gamma, i + 1, j, kk)) {
                const double uE = __dmul_rn(u_xy[(size_t)j * Nx + i + 1], po), F = rhoCp * 0.5 * (uP + uE) * Ax;
                diag += fmax(F, 0.0);
                aE = aE + (-fmax(-F, 0.0));
            }
        } else if (regP && uP > 0) {
            diag += __dmul_rn(rhoCp * uP, Ax);
        }
        // y faces
        if (j > 0) {
            const double kf = th_harm(kP, th_kval(k, gamma, i, j - 1, kk)), D = kf * Ay / dy;
            diag += D;
            aS = -D;
            if (regP && th_fluid(k, gamma, i, j - 1, kk)) {
                const double vS = __dmul_rn(v_xy[(size_t)(j - 1) * Nx + i], po), F = rhoCp * 0.5 * (vP + vS) * Ay;
                diag += fmax(-F, 0.0);
                aS = aS + (-fmax(F, 0.0));
            }
        }
        if (j < Ny - 1) {
            const double kf = th_harm(kP, th_kval(k, gamma, i, j + 1, kk)), D = kf * Ay / dy;
            diag += D;
            aN = -D;
            if (regP && th_fluid(k, gamma, i, j + 1, kk)) {
                const double vN = __dmul_rn(v_xy[(size_t)(j + 1) * Nx + i], po), F = rhoCp * 0.5 * (vP + vN) * Ay;
                diag += fmax(F, 0.0);
                aN = aN + (-fmax(-F, 0.0));
            }
        } else if (regP && vP > 0) {
            diag += __dmul_rn(rhoCp * vP, Ay);
        }
        // z faces (diffusion only)
        if (kk > 0) {
            const double kN = th_kval(k, gamma, i, j, kk - 1), dz_P = dz_k, dz_N = th_dz(k, kk - 1);
            const double kf = (dz_P + dz_N) / (dz_P / kP + dz_N / kN);
            const double D = kf * Az_cell / (0.5 * (dz_P + dz_N));
            diag += D;
            aB = -D;
        } else {
            bb += __dmul_rn(q0[(size_t)j * Nx + i], Az_cell);
        }
        if (kk < Nz - 1) {
            const double kN = th_kval(k, gamma, i, j, kk + 1), dz_P = dz_k, dz_N = th_dz(k, kk + 1);
            const double kf = (dz_P + dz_N) / (dz_P / kP + dz_N / kN);
            const double D = kf * Az_cell / (0.5 * (dz_P + dz_N));
            diag += D;
            aT = -D;
        }
        S.aP[t] = diag + 1e-12;
        S.aW[t] = aW; S.aE[t] = aE; S.aS[t] = aS; S.aN[t] = aN; S.aB[t] = aB; S.aT[t] = aT;
        S.b[t] = bb;
    }
}

// One level of the hierarchy (level 0: the assembled system).  x holds the
// pre-smoothed iterate, b the restricted residual and y the post-smoothed
// iterate of a coarse level.
template <typename T>
struct ThLevelT {
    int nx, ny;
    long long ncol, n;
    ThSysT<T> S;
    T *lc, *linv;
    T *b, *x, *y;
};
using ThLevel = ThLevelT<double>;

// Entries of row q of A (Tr = false) or of A^T (Tr = true) towards the
// west, east, south, north, lower and upper neighbour.  Row q of A^T holds
// column q of A: its west entry is the east coefficient of the west cell.
template <bool Tr, typename T>
__device__ __forceinline__ T th_cW(const ThSysT<T>& S, long long q) { return __ldg(Tr ? S.aE + (q - 1) : S.aW + q); }
template <bool Tr, typename T>
__device__ __forceinline__ T th_cE(const ThSysT<T>& S, long long q) { return __ldg(Tr ? S.aW + (q + 1) : S.aE + q); }
template <bool Tr, typename T>
__device__ __forceinline__ T th_cS(const ThSysT<T>& S, long long q, int nx) {
    return __ldg(Tr ? S.aN + (q - nx) : S.aS + q);
}
template <bool Tr, typename T>
__device__ __forceinline__ T th_cN(const ThSysT<T>& S, long long q, int nx) {
    return __ldg(Tr ? S.aS + (q + nx) : S.aN + q);
}
template <bool Tr, typename T>
__device__ __forceinline__ T th_sub(const ThSysT<T>& S, long long q, long long L) {
    return __ldg(Tr ? S.aT + (q - L) : S.aB + q);
}
template <bool Tr, typename T>
__device__ __forceinline__ T th_sup(const ThSysT<T>& S, long long q, long long L) {
    return __ldg(Tr ? S.aB + (q + L) : S.aT + q);
}

// (op x)_q on a level, op = A or A^T, in the level's arithmetic T (x may be
// stored narrower: the FP64 matvec of a float preconditioner output)
template <bool Tr, typename T, typename X>
__device__ __forceinline__ T th_ax(const ThLevelT<T>& F, int Nz, const X* x, long long q, int i, int j, int kk) {
    const long long L = F.ncol;
    T s = __ldg(F.S.aP + q) * T(x[q]);
    if (i > 0) s += th_cW<Tr>(F.S, q) * T(x[q - 1]);
    if (i < F.nx - 1) s += th_cE<Tr>(F.S, q) * T(x[q + 1]);
    if (j > 0) s += th_cS<Tr>(F.S, q, F.nx) * T(x[q - F.nx]);
    if (j < F.ny - 1) s += th_cN<Tr>(F.S, q, F.nx) * T(x[q + F.nx]);
    if (kk > 0) s += th_sub<Tr>(F.S, q, L) * T(x[q - L]);
    if (kk < Nz - 1) s += th_sup<Tr>(F.S, q, L) * T(x[q + L]);
    return s;
}

// Galerkin coarse operator P^T A P of 2 x 2 column aggregates, P piecewise
// constant: couplings inside an aggregate fold into the diagonal, couplings
// across an aggregate edge add up into the coarse neighbour's entry.
__global__ void k_th_coarsen(int Nz, ThLevel F, ThLevel C) {
    for (long long qc = (long long)blockIdx.x * blockDim.x + threadIdx.x; qc < C.n;
         qc += (long long)gridDim.x * blockDim.x) {
        const int kk = (int)(qc / C.ncol);
        const long long rem = qc - kk * C.ncol;
        const int I = (int)(rem % C.nx), J = (int)(rem / C.nx);
        double aP = 0, aW = 0, aE = 0, aS = 0, aN = 0, aB = 0, aT = 0;
        for (int dj = 0; dj < 2; ++dj) {
            const int j = 2 * J + dj;
            if (j >= F.ny) break;
            for (int di = 0; di < 2; ++di) {
                const int i = 2 * I + di;
                if (i >= F.nx) break;
                const long long q = kk * F.ncol + (long long)j * F.nx + i;
                aP += F.S.aP[q];
                aB += F.S.aB[q];
                aT += F.S.aT[q];
                if (di == 1) aP += F.S.aW[q]; else aW += F.S.aW[q];
                if (di == 0 && i + 1 < F.nx) aP += F.S.aE[q]; else aE += F.S.aE[q];
                if (dj == 1) aP += F.S.aS[q]; else aS += F.S.aS[q];
                if (dj == 0 && j + 1 < F.ny) aP += F.S.aN[q]; else aN += F.S.aN[q];
            }
        }
        C.S.aP[qc] = aP; C.S.aW[qc] = aW; C.S.aE[qc] = aE; C.S.aS[qc] = aS; C.S.aN[qc] = aN;
        C.S.aB[qc] = aB; C.S.aT[qc] = aT;
    }
}

// float copy of a level array (the mixed-precision preconditioner's levels)
__global__ void k_th_narrow(const double* __restrict__ src, float* __restrict__ dst, long long n) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (float)src[q];
}

// Thomas factors of each column's tridiagonal z-block of a level:
// inv_k = 1 / (d_k - sub_k c_{k-1}), c_k = sup_k inv_k
template <bool Tr>
__global__ void k_th_lu(int Nz, ThLevel F) {
    const long long L = F.ncol;
    for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < F.ncol;
         col += (long long)gridDim.x * blockDim.x) {
        double cprev = 0.0;
        for (int kk = 0; kk < Nz; ++kk) {
            const long long q = kk * L + col;
            const double den = F.S.aP[q] - (kk > 0 ? th_sub<Tr>(F.S, q, L) * cprev : 0.0);
            const double inv = 1.0 / den;
            const double c = (kk < Nz - 1 ? th_sup<Tr>(F.S, q, L) : 0.0) * inv;
            F.linv[q] = inv;
            F.lc[q] = c;
            cprev = c;
        }
    }
}

// Shared memory of the column sweeps (doubles): ys[kThZ][blockDim] holds a
// column's forward sweep, st[kThStageArr][kThStage][blockDim] the staged
// inputs of kThStage layers.  Each thread uses only its own slots, so no
// block barrier is needed around them.
struct ThSm {
    double* ys;
    double* st;
    // a slot holds one value of type S (double or float) in its first bytes
    template <typename S = double>
    __device__ __forceinline__ S& y(int kk) const {
        return *reinterpret_cast<S*>(ys + kk * blockDim.x + threadIdx.x);
    }
    template <typename S = double>
    __device__ __forceinline__ S& s(int a, int u) const {
        return *reinterpret_cast<S*>(st + (a * kThStage + u) * blockDim.x + threadIdx.x);
    }
};

template <typename S>
__device__ __forceinline__ void th_stage(S* dst, const S* src) { __pipeline_memcpy_async(dst, src, sizeof(S)); }

// Pre-smoothing from zero over the columns of a level: b = A0 + c1 A1 +
// c2 A2 (A1, A2 optional; stored to bout when set), x = omega Mz^-1 b.  The
// inputs of kThStage layers are copied to shared memory asynchronously, all
// in flight together, and the Thomas recurrence runs from shared memory.
// T is the level's type, B the type of the right-hand side's terms (double
// at level 0, where b is a Krylov vector; T on the coarse levels).
template <bool Tr, typename T, typename B>
__device__ __forceinline__ void th_presmooth(const ThLevelT<T>& F, int Nz, const B* A0, const B* A1, double c1,
                                             const B* A2, double c2, B* bout, T* x, double omega, long long t0,
                                             long long nt, const ThSm& sm) {
    const long long L = F.ncol;
    for (long long col = t0; col < F.ncol; col += nt) {
        T yprev = T(0);
        for (int k0 = 0; k0 < Nz; k0 += kThStage) {
            const int nu = min(kThStage, Nz - k0);
            for (int u = 0; u < nu; ++u) {
                const int kk = k0 + u;
                const long long q = kk * L + col;
                th_stage(&sm.s<B>(0, u), A0 + q);
                if (A1) th_stage(&sm.s<B>(1, u), A1 + q);
                if (A2) th_stage(&sm.s<B>(2, u), A2 + q);
                if (kk > 0) th_stage(&sm.s<T>(3, u), Tr ? F.S.aT + (q - L) : F.S.aB + q);
                th_stage(&sm.s<T>(4, u), F.linv + q);
            }
            __pipeline_commit();
            __pipeline_wait_prior(0);
            for (int u = 0; u < nu; ++u) {
                const int kk = k0 + u;
                B b = sm.s<B>(0, u);
                if (A1) b += c1 * sm.s<B>(1, u);
                if (A2) b += c2 * sm.s<B>(2, u);
                if (bout) bout[kk * L + col] = b;
                const T sub = kk > 0 ? sm.s<T>(3, u) : T(0);
                yprev = (T(b) - sub * yprev) * sm.s<T>(4, u);
                sm.y<T>(kk) = yprev;
            }
        }
        T xn = T(0);
        for (int k0 = ((Nz - 1) / kThStage) * kThStage; k0 >= 0; k0 -= kThStage) {
            const int nu = min(kThStage, Nz - k0);
            for (int u = 0; u < nu; ++u) {
                const int kk = k0 + u;
                if (kk < Nz - 1) th_stage(&sm.s<T>(0, u), F.lc + (kk * L + col));
            }
            __pipeline_commit();
            __pipeline_wait_prior(0);
            for (int u = nu - 1; u >= 0; --u) {
                const int kk = k0 + u;
                const T xv = sm.y<T>(kk) - (kk < Nz - 1 ? sm.s<T>(0, u) * xn : T(0));
                x[kk * L + col] = T(omega) * xv;
                xn = xv;
            }
        }
    }
}

// Residual restriction: bC = sum over the 2 x 2 aggregate of (bF - op xF).
// The four fine residuals are independent, so their loads are in flight
// together; index math in 32 bits (levels hold fewer than 2^31 cells).
template <bool Tr, typename T, typename B>
__device__ __forceinline__ void th_restrict(const ThLevelT<T>& F, const ThLevelT<T>& C, int Nz, const B* bF,
                                            const T* xF, T* bC, long long t0, long long nt) {
    const unsigned LC = (unsigned)C.ncol, cnx = (unsigned)C.nx, LF = (unsigned)F.ncol;
    for (unsigned qc = (unsigned)t0; qc < (unsigned)C.n; qc += (unsigned)nt) {
        const unsigned kk = qc / LC, rem = qc - kk * LC, J = rem / cnx, I = rem - J * cnx;
        T r[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int i = 2 * (int)I + (d & 1), j = 2 * (int)J + (d >> 1);
            r[d] = T(0);
            if (i < F.nx && j < F.ny) {
                const long long q = (long long)kk * LF + (long long)j * F.nx + i;
                r[d] = T(bF[q]) - th_ax<Tr>(F, Nz, xF, q, i, j, (int)kk);
            }
        }
        bC[qc] = ((r[0] + r[1]) + r[2]) + r[3];
    }
}

// Post-smoothing, first half (cells): out = bF - op xp with the prolonged
// iterate xp = xF + scale P xC formed on the fly at every stencil point.
// Two cells a thread per step (their loads in flight together), 32-bit
// index math.
template <bool Tr, typename T, typename B>
__device__ __forceinline__ T th_post_res1(const ThLevelT<T>& F, const ThLevelT<T>& C, int Nz, const B* bF,
                                          const T* xF, const T* xC, T scale, unsigned q) {
    const unsigned L = (unsigned)F.ncol, LC = (unsigned)C.ncol, nx = (unsigned)F.nx, cnx = (unsigned)C.nx;
    const unsigned kk = q / L, col = q - kk * L, ju = col / nx, iu = col - ju * nx;
    const int i = (int)iu, j = (int)ju;
    const unsigned kc = kk * LC, cj = (ju >> 1) * cnx;
    T ax = __ldg(F.S.aP + q) * (xF[q] + scale * xC[kc + cj + (iu >> 1)]);
    if (i > 0) ax += th_cW<Tr>(F.S, q) * (xF[q - 1] + scale * xC[kc + cj + ((iu - 1) >> 1)]);
    if (i < F.nx - 1) ax += th_cE<Tr>(F.S, q) * (xF[q + 1] + scale * xC[kc + cj + ((iu + 1) >> 1)]);
    if (j > 0) ax += th_cS<Tr>(F.S, q, F.nx) * (xF[q - nx] + scale * xC[kc + ((ju - 1) >> 1) * cnx + (iu >> 1)]);
    if (j < F.ny - 1)
        ax += th_cN<Tr>(F.S, q, F.nx) * (xF[q + nx] + scale * xC[kc + ((ju + 1) >> 1) * cnx + (iu >> 1)]);
    if (kk > 0) ax += th_sub<Tr>(F.S, q, L) * (xF[q - L] + scale * xC[kc - LC + cj + (iu >> 1)]);
    if ((int)kk < Nz - 1) ax += th_sup<Tr>(F.S, q, L) * (xF[q + L] + scale * xC[kc + LC + cj + (iu >> 1)]);
    return T(bF[q]) - ax;
}

template <bool Tr, typename T, typename B>
__device__ __forceinline__ void th_post_resid(const ThLevelT<T>& F, const ThLevelT<T>& C, int Nz, const B* bF,
                                              const T* xF, const T* xC, double scale, T* out, long long t0,
                                              long long nt) {
    const unsigned n = (unsigned)F.n, st = (unsigned)nt;
    const T sc = T(scale);
    unsigned q = (unsigned)t0;
    for (; q + st < n; q += 2 * st) {
        const T r0 = th_post_res1<Tr>(F, C, Nz, bF, xF, xC, sc, q);
        const T r1 = th_post_res1<Tr>(F, C, Nz, bF, xF, xC, sc, q + st);
        out[q] = r0;
        out[q + st] = r1;
    }
    if (q < n) out[q] = th_post_res1<Tr>(F, C, Nz, bF, xF, xC, sc, q);
}

// Post-smoothing, second half (columns): out = xp + omega Mz^-1 out, in
// place (each column reads its residual before writing the result)
template <bool Tr, typename T>
__device__ __forceinline__ void th_post_cols(const ThLevelT<T>& F, const ThLevelT<T>& C, int Nz, const T* xF,
                                             const T* xC, double scale, double omega, T* out, long long t0,
                                             long long nt, const ThSm& sm) {
    const long long L = F.ncol, LC = C.ncol;
    for (long long col = t0; col < F.ncol; col += nt) {
        const int i = (int)(col % F.nx), j = (int)(col / F.nx);
        const long long c0 = (long long)(j >> 1) * C.nx + (i >> 1);
        T yprev = T(0);
        for (int k0 = 0; k0 < Nz; k0 += kThStage) {
            const int nu = min(kThStage, Nz - k0);
            for (int u = 0; u < nu; ++u) {
                const int kk = k0 + u;
                const long long q = kk * L + col;
                th_stage(&sm.s<T>(0, u), out + q);
                if (kk > 0) th_stage(&sm.s<T>(1, u), Tr ? F.S.aT + (q - L) : F.S.aB + q);
                th_stage(&sm.s<T>(2, u), F.linv + q);
            }
            __pipeline_commit();
            __pipeline_wait_prior(0);
            for (int u = 0; u < nu; ++u) {
                const int kk = k0 + u;
                const T sub = kk > 0 ? sm.s<T>(1, u) : T(0);
                yprev = (sm.s<T>(0, u) - sub * yprev) * sm.s<T>(2, u);
                sm.y<T>(kk) = yprev;
            }
        }
        T cnext = T(0);
        for (int k0 = ((Nz - 1) / kThStage) * kThStage; k0 >= 0; k0 -= kThStage) {
            const int nu = min(kThStage, Nz - k0);
            for (int u = 0; u < nu; ++u) {
                const int kk = k0 + u;
                const long long q = kk * L + col;
                if (kk < Nz - 1) th_stage(&sm.s<T>(0, u), F.lc + q);
                th_stage(&sm.s<T>(1, u), xF + q);
                th_stage(&sm.s<T>(2, u), xC + (kk * LC + c0));
            }
            __pipeline_commit();
            __pipeline_wait_prior(0);
            for (int u = nu - 1; u >= 0; --u) {
                const int kk = k0 + u;
                const T corr = sm.y<T>(kk) - (kk < Nz - 1 ? sm.s<T>(0, u) * cnext : T(0));
                out[kk * L + col] = sm.s<T>(1, u) + T(scale) * sm.s<T>(2, u) + T(omega) * corr;
                cnext = corr;
            }
        }
    }
}

// The preconditioner's hierarchy in type T (level 0's arrays: copies of the
// assembled system when T is float)
template <typename T>
struct ThHierT {
    int L, cta;             // levels; first level run by block 0 alone (L: none)
    double omega, scale0, scale;   // coarse-correction factor into level 0, into the deeper levels
    const ThLevelT<T>* lv;  // device array of L levels
    unsigned long long* prof;  // per-phase nanoseconds (CP_TH_PROFILE), or null
};
using ThHier = ThHierT<double>;

// phase slots of the profile: the BiCGStab phases, then 16 slots per
// V-cycle phase kind indexed by level
enum ThProfSlot {
    TH_P_INIT = 0, TH_P_PRE_P = 1, TH_P_MATVEC_V = 2, TH_P_PRE_S = 3, TH_P_MATVEC_T = 4, TH_P_UPDATE = 5,
    TH_P_BLOCK0 = 6, TH_P_RESTRICT = 16, TH_P_PRESMOOTH = 32, TH_P_POSTRES = 48, TH_P_POSTCOL = 64,
    TH_P_COUNT = 80
};

// BiCGStab's vectors, FP64; the preconditioned directions ph = M^-1 p and
// sh = M^-1 s are stored in the preconditioner's type T
template <typename T>
struct ThVecsT {
    double *x, *r, *rh, *p, *v, *s, *t;
    T *ph, *sh;
};
using ThVecs = ThVecsT<double>;

// BiCGStab (van der Vorst), right-preconditioned by one V-cycle, for
// A x = rhs (Tr = false) or A^T x = rhs (Tr = true), from the x in V.x.
// F0 is the FP64 system (matvecs, residuals, dot products); the V-cycle runs
// on H in type T (T = float: the mixed-precision form; T = double: H.lv[0]
// is F0).  Dynamic shared memory: kThSmemBytes (the column sweeps' staging).
template <bool Tr, typename T>
__global__ void __launch_bounds__(kThThreads, 2) k_th_bicgstab(ThK k, ThLevel F0, ThHierT<T> H, const double* rhs,
                                                              ThVecsT<T> V, double* part, unsigned* bar, ThStatus* st,
                                                              int maxiter, double rtol) {
    __shared__ double sm[96];
    extern __shared__ double th_dyn[];
    const ThSm cs{th_dyn, th_dyn + kThZ * blockDim.x};
    const int G = gridDim.x, Nz = k.Nz;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long long)G * blockDim.x;
    unsigned target = 0;
    double* pA = part;             // [G][2]
    double* pB = part + 2 * G;     // [G][2]
    double* pC = part + 4 * G;     // [G][2]
    unsigned long long tprev = (H.prof && blockIdx.x == 0 && threadIdx.x == 0) ? globaltimer_ns() : 0ull;
    // grid barrier; with the profile on, block 0 books the time since the
    // previous barrier to the phase slot
    auto sync = [&](int slot) -> bool {
        target += G;
        const bool ok = grid_barrier(bar, target, &st->err);
        if (H.prof && blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long t = globaltimer_ns();
            H.prof[slot] += t - tprev;
            tprev = t;
        }
        return ok;
    };
    auto cells = [&](auto&& fn) {
        for (long long q = tid; q < k.n; q += nth) {
            const int kk = (int)(q / k.ncol);
            const long long rem = q - kk * k.ncol;
            fn(q, (int)(rem % k.Nx), (int)(rem / k.Nx), kk);
        }
    };
    // Two cells a thread per step: compute(q, i, j, kk) only loads and
    // computes (its loads for both cells in flight together), commit(q, v)
    // stores and accumulates; 32-bit index math.
    auto cells2 = [&](auto&& compute, auto&& commit) {
        const unsigned n = (unsigned)k.n, L = (unsigned)k.ncol, nx = (unsigned)k.Nx, stp = (unsigned)nth;
        auto at = [&](unsigned q) {
            const unsigned kk = q / L, rem = q - kk * L, j = rem / nx;
            return compute((long long)q, (int)(rem - j * nx), (int)j, (int)kk);
        };
        unsigned q = (unsigned)tid;
        for (; q + stp < n; q += 2 * stp) {
            const auto a = at(q);
            const auto b = at(q + stp);
            commit((long long)q, a);
            commit((long long)(q + stp), b);
        }
        if (q < n) commit((long long)q, at(q));
    };
    // The V-cycle after the level-0 pre-smoothing (H.lv[0].x = omega Mz^-1 b0):
    // out0 = M^-1 b0.  Ends with a grid barrier.
    auto vcycle = [&](const double* b0, T* out0) __attribute__((always_inline)) -> bool {
        const int L = H.L;
        // residual restriction from level l (its right-hand side: b0 at level 0)
        auto restrict_from = [&](int l) __attribute__((always_inline)) {
            const ThLevelT<T> &F = H.lv[l], &C = H.lv[l + 1];
            if (l == 0) th_restrict<Tr>(F, C, Nz, b0, F.x, C.b, tid, nth);
            else th_restrict<Tr>(F, C, Nz, F.b, F.x, C.b, tid, nth);
        };
        int l = 0;
        for (; l + 1 < L && l + 1 < H.cta; ++l) {
            const ThLevelT<T>& C = H.lv[l + 1];
            restrict_from(l);
            if (!sync(TH_P_RESTRICT + l)) return false;
            th_presmooth<Tr>(C, Nz, C.b, (const T*)nullptr, 0.0, (const T*)nullptr, 0.0, (T*)nullptr, C.x,
                             l + 2 == L ? 1.0 : H.omega, tid, nth, cs);
            if (!sync(TH_P_PRESMOOTH + l + 1)) return false;
        }
        if (l + 1 < L) {
            // levels l+1 .. L-1 are small: restrict to l+1 grid-wide, then block 0
            restrict_from(l);
            if (!sync(TH_P_RESTRICT + l)) return false;
            if (blockIdx.x == 0) {
                const long long bt = threadIdx.x, bn = blockDim.x;
                for (int m = l + 1;; ++m) {
                    const ThLevelT<T>& C = H.lv[m];
                    th_presmooth<Tr>(C, Nz, C.b, (const T*)nullptr, 0.0, (const T*)nullptr, 0.0, (T*)nullptr, C.x,
                                     m + 1 == L ? 1.0 : H.omega, bt, bn, cs);
                    __syncthreads();
                    if (m + 1 == L) break;
                    th_restrict<Tr>(C, H.lv[m + 1], Nz, C.b, C.x, H.lv[m + 1].b, bt, bn);
                    __syncthreads();
                }
                for (int m = L - 2; m >= l + 1; --m) {
                    const ThLevelT<T> &F = H.lv[m], &C = H.lv[m + 1];
                    const T* xc = m + 2 == L ? C.x : C.y;
                    th_post_resid<Tr>(F, C, Nz, F.b, F.x, xc, H.scale, F.y, bt, bn);
                    __syncthreads();
                    th_post_cols<Tr>(F, C, Nz, F.x, xc, H.scale, H.omega, F.y, bt, bn, cs);   // m >= 1
                    __syncthreads();
                }
            }
            if (!sync(TH_P_BLOCK0)) return false;
        } else {
            l = L - 2;   // every level grid-wide: the ascent starts above the bottom
        }
        for (int m = l; m >= 0; --m) {
            const ThLevelT<T> &F = H.lv[m], &C = H.lv[m + 1];
            const T* xc = m + 2 == L ? C.x : C.y;
            T* out = m == 0 ? out0 : F.y;
            const double sc = m == 0 ? H.scale0 : H.scale;
            if (m == 0) th_post_resid<Tr>(F, C, Nz, b0, F.x, xc, sc, out, tid, nth);
            else th_post_resid<Tr>(F, C, Nz, F.b, F.x, xc, sc, out, tid, nth);
            if (!sync(TH_P_POSTRES + m)) return false;
            th_post_cols<Tr>(F, C, Nz, F.x, xc, sc, H.omega, out, tid, nth, cs);
            if (!sync(TH_P_POSTCOL + m)) return false;
        }
        return true;
    };
    // ---- r = rhs - op x, rh = r, p = v = 0; ||rhs||^2, ||r||^2
    {
        double acc[2] = {0.0, 0.0};
        cells([&](long long q, int i, int j, int kk) {
            const double r = rhs[q] - th_ax<Tr>(F0, Nz, V.x, q, i, j, kk);
            V.r[q] = r;
            V.rh[q] = r;
            V.p[q] = 0.0;
            V.v[q] = 0.0;
            acc[0] += rhs[q] * rhs[q];
            acc[1] += r * r;
        });
        block_sum<2>(acc, sm);
        if (threadIdx.x == 0) { pC[2 * blockIdx.x] = acc[0]; pC[2 * blockIdx.x + 1] = acc[1]; }
    }
    if (!sync(TH_P_INIT)) return;
    double tot[2];
    sum_partials<2>(pC, G, 2, tot, sm);
    const double bnorm = sqrt(tot[0]) > 0.0 ? sqrt(tot[0]) : 1.0;
    double res = sqrt(tot[1]) / bnorm;
    double rho = 1.0, alpha = 1.0, omega = 1.0, rho1 = tot[1];
    int it = 0;
    bool conv = res <= rtol;
    for (; it < maxiter && !conv; ++it) {
        if (rho1 == 0.0) break;
        const double beta = (rho1 / rho) * (alpha / omega);
        // ---- p = r + beta p - beta omega v, fused with the level-0 pre-smoothing; ph = M^-1 p
        th_presmooth<Tr>(H.lv[0], Nz, (const double*)V.r, (const double*)V.p, beta, (const double*)V.v,
                         -beta * omega, V.p, H.lv[0].x, H.omega, tid, nth, cs);
        if (!sync(TH_P_PRE_P)) return;
        if (!vcycle(V.p, V.ph)) return;
        // ---- v = op ph; (rh, v)
        {
            double acc[2] = {0.0, 0.0};
            cells2([&](long long q, int i, int j, int kk) {
                return make_double2(th_ax<Tr>(F0, Nz, V.ph, q, i, j, kk), V.rh[q]);
            }, [&](long long q, double2 a) {
                V.v[q] = a.x;
                acc[0] += a.y * a.x;
            });
            block_sum<2>(acc, sm);
            if (threadIdx.x == 0) pA[2 * blockIdx.x] = acc[0];
        }
        if (!sync(TH_P_MATVEC_V)) return;
        double rv[2];
        sum_partials<2>(pA, G, 2, rv, sm);
        if (rv[0] == 0.0) break;
        alpha = rho1 / rv[0];
        // ---- s = r - alpha v, fused with the level-0 pre-smoothing; sh = M^-1 s
        th_presmooth<Tr>(H.lv[0], Nz, (const double*)V.r, (const double*)V.v, -alpha, (const double*)nullptr, 0.0,
                         V.s, H.lv[0].x, H.omega, tid, nth, cs);
        if (!sync(TH_P_PRE_S)) return;
        if (!vcycle(V.s, V.sh)) return;
        // ---- t = op sh; (t, s), (t, t)
        {
            double acc[2] = {0.0, 0.0};
            cells2([&](long long q, int i, int j, int kk) {
                return make_double2(th_ax<Tr>(F0, Nz, V.sh, q, i, j, kk), V.s[q]);
            }, [&](long long q, double2 a) {
                V.t[q] = a.x;
                acc[0] += a.x * a.y;
                acc[1] += a.x * a.x;
            });
            block_sum<2>(acc, sm);
            if (threadIdx.x == 0) { pB[2 * blockIdx.x] = acc[0]; pB[2 * blockIdx.x + 1] = acc[1]; }
        }
        if (!sync(TH_P_MATVEC_T)) return;
        double ts[2];
        sum_partials<2>(pB, G, 2, ts, sm);
        omega = ts[1] > 0.0 ? ts[0] / ts[1] : 0.0;
        // ---- x += alpha ph + omega sh; r = s - omega t; (r, r), (rh, r)
        {
            double acc[2] = {0.0, 0.0};
            cells2([&](long long q, int, int, int) {
                return make_double3(V.x[q] + alpha * double(V.ph[q]) + omega * double(V.sh[q]), V.s[q] - omega * V.t[q],
                                    V.rh[q]);
            }, [&](long long q, double3 a) {
                V.x[q] = a.x;
                V.r[q] = a.y;
                acc[0] += a.y * a.y;
                acc[1] += a.z * a.y;
            });
            block_sum<2>(acc, sm);
            if (threadIdx.x == 0) { pC[2 * blockIdx.x] = acc[0]; pC[2 * blockIdx.x + 1] = acc[1]; }
        }
        if (!sync(TH_P_UPDATE)) return;
        sum_partials<2>(pC, G, 2, tot, sm);
        res = sqrt(tot[0]) / bnorm;
        rho = rho1;
        rho1 = tot[1];
        if (!(res == res)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(&st->err, 0, (int)CP_ERR_NONFINITE);
            return;
        }
        if (res <= rtol) { conv = true; ++it; break; }
        if (omega == 0.0) { ++it; break; }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->iterations = it;
        st->converged = conv ? 1 : 0;
        st->residual = res;
    }
}

// bottom layer: partials of max T and sum T^p
__global__ void k_th_pnorm(ThK k, const double* T, double pexp, double* part) {
    __shared__ double sm[64];
    __shared__ double smx[32];
    double mx = -1e300, s[1] = {0.0};
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < k.ncol;
         q += (long long)gridDim.x * blockDim.x) {
        const double t = T[q];
        mx = fmax(mx, t);
        s[0] += pow(t, pexp);
    }
    block_sum<1>(s, sm);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) smx[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = -1e300;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, smx[w]);
        part[2 * blockIdx.x] = m;
        part[2 * blockIdx.x + 1] = s[0];
    }
}

__global__ void k_th_fill(double* x, long long n, double v) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        x[q] = v;
}

// dJ/dT of J = (mean over the bottom layer of T^p)^(1/p):
// (T / J)^(p-1) / (Nx Ny) on k = 0, zero above
__global__ void k_th_adj_rhs(ThK k, const double* T, double J, double pexp, double* rhs) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < k.n;
         q += (long long)gridDim.x * blockDim.x)
        rhs[q] = q < k.ncol ? pow(T[q] / J, pexp - 1.0) / (double)k.ncol : 0.0;
}

// dk/dgamma of a cell above the base plate at the clamped gamma; for RAMP
// the reference's dk_dgamma (thermal_solver.cpp:317-321)
__device__ __forceinline__ double th_dkdg(const ThK& k, double g) {
    g = fmax(0.0, fmin(1.0, g));
    if (k.mode == 1) {
        const double den = 1.0 + k.qk * g;
        return (k.kS - k.kF) * (-(1.0 + k.qk)) / (den * den);
    }
    if (k.mode == 2) {
        const double den = (1.0 - g) * k.kF + g * k.kS + 1e-30;
        return -k.kS * k.kF * (k.kS - k.kF) / (den * den);
    }
    return k.kF - k.kS;
}

// d harm(a, b) / da for harm = 2ab / (a + b + 1e-30)
__device__ __forceinline__ double th_dharm(double a, double b) {
    const double s = a + b + 1e-30;
    return 2.0 * b * (b + 1e-30) / (s * s);
}

// dJ/dgamma(i, j) = -lambda^T dR/dgamma(i, j) for R = A(gamma) T - b(gamma),
// one thread per column.  gamma(i, j) sets k of every cell of the column
// above the base plate, which enters the x/y face conductances (harmonic
// means), the inlet conductance 2 k Ax / dx and the z conductances
// (thickness-weighted); the velocities and the fluid/solid masks are held
// fixed (the mask is a step at gamma = 0.01 without a derivative).  A face
// of conductance D between P and N contributes (l_P - l_N)(T_P - T_N) dD.
__global__ void k_th_sens(ThK k, const double* gamma, const double* T, const double* lam, double* grad) {
    const long long L = (long long)k.Nx * k.Ny;
    const double dx = k.dx, dy = k.dy;
    for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < k.ncol;
         col += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(col % k.Nx), j = (int)(col / k.Nx);
        double acc = 0.0;
        for (int kk = k.nzS; kk < k.Nz; ++kk) {
            const long long q = kk * L + col;
            const double kP = th_kval(k, gamma, i, j, kk), dz = th_dz(k, kk);
            const double Ax = dy * dz, Ay = dx * dz, lP = lam[q], TP = T[q];
            if (i > 0)
                acc += (lP - lam[q - 1]) * (TP - T[q - 1]) * th_dharm(kP, th_kval(k, gamma, i - 1, j, kk)) * Ax / dx;
            if (i < k.Nx - 1)
                acc += (lP - lam[q + 1]) * (TP - T[q + 1]) * th_dharm(kP, th_kval(k, gamma, i + 1, j, kk)) * Ax / dx;
            if (j > 0)
                acc += (lP - lam[q - k.Nx]) * (TP - T[q - k.Nx]) * th_dharm(kP, th_kval(k, gamma, i, j - 1, kk)) *
                       Ay / dy;
            if (j < k.Ny - 1)
                acc += (lP - lam[q + k.Nx]) * (TP - T[q + k.Nx]) * th_dharm(kP, th_kval(k, gamma, i, j + 1, kk)) *
                       Ay / dy;
            if (i == 0 && th_fluid(k, gamma, i, j, kk)) acc += lP * (TP - k.Tin) * 2.0 * Ax / dx;
        }
        // z faces (kk, kk + 1) with a cell above the base plate
        for (int kk = k.nzS - 1; kk < k.Nz - 1; ++kk) {
            const long long q = kk * L + col;
            const double kL = th_kval(k, gamma, i, j, kk), kU = th_kval(k, gamma, i, j, kk + 1);
            const double dL = th_dz(k, kk), dU = th_dz(k, kk + 1), den = dL / kL + dU / kU;
            double dkf = (dL + dU) * (dU / (kU * kU)) / (den * den);
            if (kk >= k.nzS) dkf += (dL + dU) * (dL / (kL * kL)) / (den * den);
            acc += (lam[q] - lam[q + L]) * (T[q] - T[q + L]) * dkf * (dx * dy) / (0.5 * (dL + dU));
        }
        grad[col] = -th_dkdg(k, gamma[col]) * acc;
    }
}

}  // namespace cp

using namespace cp;

struct cp_thermal {
    cp_thermal_params prm{};
    ThK k{};
    int dev = 0, numSMs = 0, grid = 0, gElem = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double *gamma = nullptr, *u = nullptr, *v = nullptr, *q0 = nullptr;
    ThSys S{};
    double *lc = nullptr, *linv = nullptr, *z0 = nullptr, *lam = nullptr, *rhs = nullptr, *grad = nullptr;
    ThVecs V{};
    std::vector<ThLevel> lv;          // the hierarchy (level 0: S, lc, linv, z0)
    ThLevel* dlv = nullptr;           // its device copy
    ThHier H{};
    // CP_PREC_MIXED: float copies of every level for the V-cycle, and the
    // preconditioned directions in float
    bool mixed = false;
    std::vector<ThLevelT<float>> lvf;
    ThLevelT<float>* dlvf = nullptr;
    ThHierT<float> Hf{};
    float *phf = nullptr, *shf = nullptr;
    double* part = nullptr;
    unsigned* bar = nullptr;
    ThStatus* st = nullptr;
    bool hasInputs = false, solved = false;
    std::vector<void*> allocs;
};

namespace {

template <typename T>
cp_status th_alloc(cp_thermal* t, T** p, size_t n) {
    void* q = nullptr;
    TCK(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
    t->allocs.push_back(q);
    TCK(cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), t->stream));
    *p = static_cast<T*>(q);
    return CP_OK;
}

// float copy of a level array (mixed precision)
cp_status th_narrow(cp_thermal* t, const double* src, float* dst, long long n) {
    const int g = (int)std::min<long long>(t->gElem, (n + kThThreads - 1) / kThThreads);
    k_th_narrow<<<std::max(g, 1), kThThreads, 0, t->stream>>>(src, dst, n);
    TCK(cudaGetLastError());
    return CP_OK;
}

// The float levels of the mixed-precision V-cycle, shaped like the FP64
// hierarchy.  Level 0 needs no b (its right-hand side is a Krylov vector)
// and no y (its output is ph or sh).
cp_status th_build_float_hierarchy(cp_thermal* t) {
    const int L = (int)t->lv.size();
    t->lvf.assign(L, ThLevelT<float>{});
    for (int l = 0; l < L; ++l) {
        const ThLevel& F = t->lv[l];
        ThLevelT<float>& G = t->lvf[l];
        G.nx = F.nx;
        G.ny = F.ny;
        G.ncol = F.ncol;
        G.n = F.n;
        std::vector<float**> arr = {&G.S.aP, &G.S.aW, &G.S.aE, &G.S.aS, &G.S.aN, &G.S.aB, &G.S.aT,
                                    &G.lc,   &G.linv, &G.x};
        if (l > 0) {
            arr.push_back(&G.b);
            arr.push_back(&G.y);
        }
        for (float** q : arr) {
            cp_status s = th_alloc(t, q, (size_t)G.n);
            if (s != CP_OK) return s;
        }
    }
    void* q = nullptr;
    TCK(cudaMalloc(&q, sizeof(ThLevelT<float>) * L));
    t->allocs.push_back(q);
    t->dlvf = static_cast<ThLevelT<float>*>(q);
    TCK(cudaMemcpyAsync(t->dlvf, t->lvf.data(), sizeof(ThLevelT<float>) * L, cudaMemcpyHostToDevice, t->stream));
    t->Hf.L = t->H.L;
    t->Hf.cta = t->H.cta;
    t->Hf.omega = t->H.omega;
    t->Hf.scale0 = t->H.scale0;
    t->Hf.scale = t->H.scale;
    t->Hf.lv = t->dlvf;
    t->Hf.prof = t->H.prof;
    cp_status s = th_alloc(t, &t->phf, (size_t)t->k.n);
    if (s != CP_OK) return s;
    return th_alloc(t, &t->shf, (size_t)t->k.n);
}

// Levels of 2 x 2 column aggregates down to a single column, all z-layers
// kept; level 0 is the assembled system.  CP_TH_OMEGA, CP_TH_SCALE0,
// CP_TH_SCALE and CP_TH_CTA_COLS override the smoothing weight, the
// coarse-correction factors into level 0 and into the deeper levels, and the
// size below which block 0 runs a level alone.
cp_status th_build_hierarchy(cp_thermal* t) {
    const ThK& k = t->k;
    ThLevel f0{};
    f0.nx = k.Nx;
    f0.ny = k.Ny;
    f0.ncol = k.ncol;
    f0.n = k.n;
    f0.S = t->S;
    f0.lc = t->lc;
    f0.linv = t->linv;
    f0.x = t->z0;
    t->lv.assign(1, f0);
    while (t->lv.back().nx > 1 || t->lv.back().ny > 1) {
        if ((int)t->lv.size() == kThMaxLevels)
            return tfail(CP_ERR_BAD_PARAM, "grid %d x %d needs more than %d levels", k.Nx, k.Ny, kThMaxLevels);
        const ThLevel& F = t->lv.back();
        ThLevel C{};
        C.nx = (F.nx + 1) / 2;
        C.ny = (F.ny + 1) / 2;
        C.ncol = (long long)C.nx * C.ny;
        C.n = C.ncol * k.Nz;
        double** arr[] = {&C.S.aP, &C.S.aW, &C.S.aE, &C.S.aS, &C.S.aN, &C.S.aB, &C.S.aT,
                          &C.lc,   &C.linv, &C.b,    &C.x,    &C.y};
        for (double** q : arr) {
            cp_status s = th_alloc(t, q, (size_t)C.n);
            if (s != CP_OK) return s;
        }
        t->lv.push_back(C);
    }
    const int L = (int)t->lv.size();
    long long ctaCols = kThCtaCols;
    if (const char* e = getenv("CP_TH_CTA_COLS")) ctaCols = std::max(atoll(e), 1LL);
    int cta = L;
    for (int l = 1; l < L; ++l)
        if (t->lv[l].ncol <= ctaCols) { cta = l; break; }
    void* q = nullptr;
    TCK(cudaMalloc(&q, sizeof(ThLevel) * L));
    t->allocs.push_back(q);
    t->dlv = static_cast<ThLevel*>(q);
    TCK(cudaMemcpyAsync(t->dlv, t->lv.data(), sizeof(ThLevel) * L, cudaMemcpyHostToDevice, t->stream));
    t->H.L = L;
    t->H.cta = cta;
    t->H.omega = kThOmega;
    t->H.scale0 = kThScale0;
    t->H.scale = kThScale;
    if (const char* e = getenv("CP_TH_OMEGA")) t->H.omega = atof(e);
    if (const char* e = getenv("CP_TH_SCALE0")) t->H.scale0 = atof(e);
    if (const char* e = getenv("CP_TH_SCALE")) t->H.scale = atof(e);
    t->H.lv = t->dlv;
    t->H.prof = nullptr;
    if (getenv("CP_TH_PROFILE")) {
        TCK(cudaMalloc(&q, sizeof(unsigned long long) * TH_P_COUNT));
        t->allocs.push_back(q);
        t->H.prof = static_cast<unsigned long long*>(q);
    }
    return CP_OK;
}

// CP_TH_PROFILE: the phase times of the last solve, to stderr
void th_print_profile(cp_thermal* t, bool Tr, int iters) {
    unsigned long long h[TH_P_COUNT];
    if (cudaMemcpy(h, t->H.prof, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return;
    const double it = iters > 0 ? iters : 1;
    fprintf(stderr, "thermal %s profile, us per iteration (%d iterations):\n", Tr ? "adjoint" : "forward", iters);
    const char* top[] = {"init(total)", "update p + presmooth 0", "matvec v", "update s + presmooth 0", "matvec t",
                         "update x, r", "block-0 levels"};
    for (int i = 0; i <= TH_P_BLOCK0; ++i)
        if (h[i]) fprintf(stderr, "  %-26s %9.1f\n", top[i], h[i] * 1e-3 / (i == TH_P_INIT ? 1.0 : it));
    const char* kind[] = {"restrict from", "presmooth", "post residual", "post columns"};
    for (int kd = 0; kd < 4; ++kd)
        for (int l = 0; l < 16; ++l) {
            const unsigned long long v = h[TH_P_RESTRICT + 16 * kd + l];
            if (v) fprintf(stderr, "  %-16s level %2d %9.1f\n", kind[kd], l, v * 1e-3 / it);
        }
}

cp_status th_objective(cp_thermal* t, double p, double* Tb_max, double* Tb_pnorm) {
    k_th_pnorm<<<t->gElem, kThThreads, 0, t->stream>>>(t->k, t->V.x, p, t->part);
    TCK(cudaGetLastError());
    std::vector<double> h((size_t)2 * t->gElem);
    TCK(cudaMemcpyAsync(h.data(), t->part, h.size() * 8, cudaMemcpyDeviceToHost, t->stream));
    TCK(cudaStreamSynchronize(t->stream));
    double mx = -1e300, s = 0.0;
    for (int b = 0; b < t->gElem; ++b) {
        mx = std::max(mx, h[2 * b]);
        s += h[2 * b + 1];
    }
    if (Tb_max) *Tb_max = mx;
    if (Tb_pnorm) *Tb_pnorm = std::pow(s / (double)t->k.ncol, 1.0 / p);
    return CP_OK;
}

// Column factorisation and the persistent BiCGStab for op x = rhs, op = A or
// A^T, from V.x; records ev1 after the solve and reads the status back.
// Mixed precision: the factors are narrowed to the float levels, and the
// solve is restarted from its iterate while the FP64 residual it computes
// on entry (b - op x, not the recursive one) is above rtol, for at most
// kThRefineRounds launches in all; the iterations add up.
template <bool Tr>
cp_status th_krylov(cp_thermal* t, const double* rhs, const ThVecs& V, ThStatus* hs) {
    const ThK& k = t->k;
    for (size_t l = 0; l < t->lv.size(); ++l) {
        const ThLevel& F = t->lv[l];
        const int g = (int)std::min<long long>(t->gElem, (F.ncol + kThThreads - 1) / kThThreads);
        k_th_lu<Tr><<<g, kThThreads, 0, t->stream>>>(k.Nz, F);
        TCK(cudaGetLastError());
        if (t->mixed) {
            cp_status s = th_narrow(t, F.lc, t->lvf[l].lc, F.n);
            if (s == CP_OK) s = th_narrow(t, F.linv, t->lvf[l].linv, F.n);
            if (s != CP_OK) return s;
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(t->grid);
    cfg.blockDim = dim3(kThThreads);
    cfg.stream = t->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.dynamicSmemBytes = kThSmemBytes;
    const ThVecsT<float> Vf{V.x, V.r, V.rh, V.p, V.v, V.s, V.t, t->phf, t->shf};
    const int rounds = t->mixed ? kThRefineRounds : 1;
    int total = 0;
    for (int round = 0; round < rounds; ++round) {
        TCK(cudaMemsetAsync(t->bar, 0, sizeof(unsigned), t->stream));
        TCK(cudaMemsetAsync(t->st, 0, sizeof(ThStatus), t->stream));
        if (t->H.prof) TCK(cudaMemsetAsync(t->H.prof, 0, sizeof(unsigned long long) * TH_P_COUNT, t->stream));
        const int left = std::max(t->prm.maxiter - total, 0);
        if (t->mixed)
            TCK(cudaLaunchKernelEx(&cfg, k_th_bicgstab<Tr, float>, k, t->lv[0], t->Hf, rhs, Vf, t->part, t->bar,
                                   t->st, left, t->prm.rtol));
        else
            TCK(cudaLaunchKernelEx(&cfg, k_th_bicgstab<Tr, double>, k, t->lv[0], t->H, rhs, V, t->part, t->bar,
                                   t->st, left, t->prm.rtol));
        TCK(cudaEventRecord(t->ev1, t->stream));
        TCK(cudaMemcpyAsync(hs, t->st, sizeof *hs, cudaMemcpyDeviceToHost, t->stream));
        TCK(cudaStreamSynchronize(t->stream));
        if (hs->err)
            return tfail((cp_status)hs->err, "device reported %s in the thermal %s solve",
                         cp_status_string((cp_status)hs->err), Tr ? "adjoint" : "forward");
        if (t->H.prof) th_print_profile(t, Tr, hs->iterations);
        total += hs->iterations;
        // stop once a launch found the true residual at rtol on entry, or did not converge
        if (!hs->converged || hs->iterations == 0) break;
    }
    hs->iterations = total;
    return CP_OK;
}

void th_report(cp_thermal* t, const ThStatus& hs, cp_thermal_report* rep) {
    if (!rep) return;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t->ev0, t->ev1);
    rep->iterations = hs.iterations;
    rep->converged = hs.converged;
    rep->residual = hs.residual;
    rep->device_ms = ms;
}

}  // namespace

extern "C" {

void cp_thermal_params_default(cp_thermal_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->nz_solid = 2;
    p->nz_fluid = 7;
    p->H_b = 0.0005;
    p->H_t = 0.004;
    p->k_s = 400.0;
    p->k_f = 0.6;
    p->rho = 998.0;
    p->Cp = 4180.0;
    p->T_inlet = 30.0;
    p->rtol = 1e-6;
    p->maxiter = 1000;
    p->k_interp_mode = 1;
    p->qk = 1.0;
    p->precision = CP_PREC_FP64;
}

cp_status cp_thermal_create(const cp_thermal_params* p, cp_thermal** out) {
    if (!p || !out) return tfail(CP_ERR_BAD_PARAM, "NULL argument");
    *out = nullptr;
    if (p->Nx < 2 || p->Ny < 2 || p->nz_solid < 1 || p->nz_fluid < 1 || p->nz_solid + p->nz_fluid > kThMaxNz)
        return tfail(CP_ERR_BAD_PARAM, "grid %d x %d x (%d + %d): need Nx, Ny >= 2, nz_solid, nz_fluid >= 1 "
                     "and Nz <= %d", p->Nx, p->Ny, p->nz_solid, p->nz_fluid, kThMaxNz);
    const double pos[] = {p->dx, p->dy, p->H_b, p->H_t, p->k_s, p->k_f, p->rho, p->Cp};
    for (double x : pos)
        if (!(x > 0.0) || !std::isfinite(x)) return tfail(CP_ERR_BAD_PARAM, "dx, dy, H_b, H_t, k, rho, Cp must be > 0");
    if (!std::isfinite(p->T_inlet) || !(p->rtol >= 0.0) || p->maxiter < 0 || p->k_interp_mode < 0 ||
        p->k_interp_mode > 2 || !std::isfinite(p->qk) ||
        (p->precision != CP_PREC_FP64 && p->precision != CP_PREC_MIXED))
        return tfail(CP_ERR_BAD_PARAM, "T_inlet, rtol, maxiter, k_interp_mode, qk or precision out of range");
    cp_thermal* t = new cp_thermal();
    t->prm = *p;
    auto bail = [&](cp_status s) {
        cp_thermal_destroy(t);
        return s;
    };
    if (cudaGetDevice(&t->dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&t->numSMs, cudaDevAttrMultiProcessorCount, t->dev) != cudaSuccess) {
        cudaGetLastError();
        delete t;
        return tfail(CP_ERR_CUDA, "no CUDA device");
    }
    if (cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&t->ev0) != cudaSuccess || cudaEventCreate(&t->ev1) != cudaSuccess)
        return bail(tfail(CP_ERR_CUDA, "stream / events"));
    ThK& k = t->k;
    k.Nx = p->Nx; k.Ny = p->Ny; k.nzS = p->nz_solid; k.nzF = p->nz_fluid; k.Nz = k.nzS + k.nzF;
    k.mode = p->k_interp_mode;
    k.ncol = (long long)k.Nx * k.Ny;
    k.n = k.ncol * k.Nz;
    // the reference keeps the domain length and divides it again (thermal_solver.cpp:186-187, 729)
    k.dx = (k.Nx * p->dx) / k.Nx;
    k.dy = (k.Ny * p->dy) / k.Ny;
    k.dzS = p->H_b / p->nz_solid;
    k.dzF = p->H_t / p->nz_fluid;
    k.Ht = p->H_t; k.kS = p->k_s; k.kF = p->k_f; k.rhoCp = p->rho * p->Cp; k.Tin = p->T_inlet; k.qk = p->qk;
    if (k.n >= (1LL << 31))
        return bail(tfail(CP_ERR_BAD_PARAM, "%lld cells: the solver indexes fewer than 2^31", k.n));
    const size_t n = (size_t)k.n, nc = (size_t)k.ncol;
    cp_status s;
    double** planes[] = {&t->gamma, &t->u, &t->v, &t->q0, &t->grad};
    for (double** q : planes)
        if ((s = th_alloc(t, q, nc)) != CP_OK) return bail(s);
    double** vols[] = {&t->S.aP, &t->S.aW, &t->S.aE, &t->S.aS, &t->S.aN, &t->S.aB, &t->S.aT, &t->S.b,
                       &t->lc,   &t->linv, &t->V.x,  &t->V.r,  &t->V.rh, &t->V.p,  &t->V.v,  &t->V.s,
                       &t->V.t,  &t->V.ph, &t->V.sh, &t->lam,  &t->rhs, &t->z0};
    for (double** q : vols)
        if ((s = th_alloc(t, q, n)) != CP_OK) return bail(s);
    // the forward and the adjoint kernel run on the same grid: every block resident
    // (the forward and adjoint kernels of the solve's precision)
    t->mixed = p->precision == CP_PREC_MIXED;
    const void* kern[2] = {t->mixed ? (const void*)k_th_bicgstab<false, float> : (const void*)k_th_bicgstab<false, double>,
                           t->mixed ? (const void*)k_th_bicgstab<true, float> : (const void*)k_th_bicgstab<true, double>};
    int nb = 1 << 30;
    for (const void* f : kern) {
        int b = 0;
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kThSmemBytes) != cudaSuccess)
            return bail(tfail(CP_ERR_CUDA, "the thermal solver kernel's shared memory (%zu bytes)", kThSmemBytes));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, kThThreads, kThSmemBytes);
        nb = std::min(nb, b);
    }
    if (nb < 1) return bail(tfail(CP_ERR_CUDA, "the thermal solver kernel does not fit on an SM"));
    t->grid = t->numSMs * std::min(nb, 4);
    if ((s = th_build_hierarchy(t)) != CP_OK) return bail(s);
    if (t->mixed && (s = th_build_float_hierarchy(t)) != CP_OK) return bail(s);
    t->gElem = t->numSMs * 4;
    if ((s = th_alloc(t, &t->part, (size_t)6 * kMaxBlocks)) != CP_OK) return bail(s);
    void* q = nullptr;
    if (cudaMalloc(&q, 64) != cudaSuccess) return bail(tfail(CP_ERR_CUDA, "cudaMalloc"));
    t->allocs.push_back(q);
    t->bar = static_cast<unsigned*>(q);
    if (cudaMalloc(&q, sizeof(ThStatus)) != cudaSuccess) return bail(tfail(CP_ERR_CUDA, "cudaMalloc"));
    t->allocs.push_back(q);
    t->st = static_cast<ThStatus*>(q);
    if (cudaStreamSynchronize(t->stream) != cudaSuccess) return bail(tfail(CP_ERR_CUDA, "stream"));
    *out = t;
    return CP_OK;
}

cp_status cp_thermal_destroy(cp_thermal* t) {
    if (!t) return CP_OK;
    if (t->stream) cudaStreamSynchronize(t->stream);
    for (void* q : t->allocs) cudaFree(q);
    if (t->ev0) cudaEventDestroy(t->ev0);
    if (t->ev1) cudaEventDestroy(t->ev1);
    if (t->stream) cudaStreamDestroy(t->stream);
    delete t;
    return CP_OK;
}

cp_status cp_thermal_set_inputs(cp_thermal* t, const double* gamma, const double* u, const double* v,
                                const double* q0) {
    if (!t || !gamma || !u || !v || !q0) return tfail(CP_ERR_BAD_PARAM, "NULL argument");
    const size_t nc = (size_t)t->k.ncol;
    const double* src[] = {gamma, u, v, q0};
    for (const double* a : src)
        for (size_t q = 0; q < nc; ++q)
            if (!std::isfinite(a[q])) return tfail(CP_ERR_NONFINITE, "non-finite input at %zu", q);
    TCK(cudaMemcpyAsync(t->gamma, gamma, nc * 8, cudaMemcpyHostToDevice, t->stream));
    TCK(cudaMemcpyAsync(t->u, u, nc * 8, cudaMemcpyHostToDevice, t->stream));
    TCK(cudaMemcpyAsync(t->v, v, nc * 8, cudaMemcpyHostToDevice, t->stream));
    TCK(cudaMemcpyAsync(t->q0, q0, nc * 8, cudaMemcpyHostToDevice, t->stream));
    TCK(cudaStreamSynchronize(t->stream));
    t->hasInputs = true;
    t->solved = false;
    return CP_OK;
}

cp_status cp_thermal_solve(cp_thermal* t, cp_thermal_report* rep) {
    if (!t) return tfail(CP_ERR_BAD_PARAM, "NULL argument");
    if (!t->hasInputs) return tfail(CP_ERR_STATE, "cp_thermal_set_inputs first");
    const ThK& k = t->k;
    t->solved = false;
    TCK(cudaEventRecord(t->ev0, t->stream));
    k_th_assemble<<<t->gElem, kThThreads, 0, t->stream>>>(k, t->gamma, t->u, t->v, t->q0, t->S);
    TCK(cudaGetLastError());
    // initial guess T = T_inlet
    k_th_fill<<<t->gElem, kThThreads, 0, t->stream>>>(t->V.x, k.n, t->prm.T_inlet);
    TCK(cudaGetLastError());
    for (size_t l = 0; l + 1 < t->lv.size(); ++l) {
        const ThLevel& C = t->lv[l + 1];
        const int g = (int)std::min<long long>(t->gElem, (C.n + kThThreads - 1) / kThThreads);
        k_th_coarsen<<<g, kThThreads, 0, t->stream>>>(k.Nz, t->lv[l], C);
        TCK(cudaGetLastError());
    }
    // mixed precision: the V-cycle's float copies of every level's operator
    if (t->mixed)
        for (size_t l = 0; l < t->lv.size(); ++l) {
            const ThSys& A = t->lv[l].S;
            const ThSysT<float>& B = t->lvf[l].S;
            const double* src[7] = {A.aP, A.aW, A.aE, A.aS, A.aN, A.aB, A.aT};
            float* dst[7] = {B.aP, B.aW, B.aE, B.aS, B.aN, B.aB, B.aT};
            for (int a = 0; a < 7; ++a) {
                cp_status s = th_narrow(t, src[a], dst[a], t->lv[l].n);
                if (s != CP_OK) return s;
            }
        }
    ThStatus hs;
    cp_status s = th_krylov<false>(t, t->S.b, t->V, &hs);
    if (s != CP_OK) return s;
    t->solved = true;
    th_report(t, hs, rep);
    return CP_OK;
}

cp_status cp_thermal_get_T(cp_thermal* t, double* T) {
    if (!t || !T) return tfail(CP_ERR_BAD_PARAM, "NULL argument");
    if (!t->solved) return tfail(CP_ERR_STATE, "no solution yet (cp_thermal_solve)");
    TCK(cudaMemcpyAsync(T, t->V.x, (size_t)t->k.n * 8, cudaMemcpyDeviceToHost, t->stream));
    TCK(cudaStreamSynchronize(t->stream));
    return CP_OK;
}

cp_status cp_thermal_objective(cp_thermal* t, double p, double* Tb_max, double* Tb_pnorm) {
    if (!t) return tfail(CP_ERR_BAD_PARAM, "NULL argument");
    if (!t->solved) return tfail(CP_ERR_STATE, "no solution yet (cp_thermal_solve)");
    if (!(p > 0.0) || !std::isfinite(p)) return tfail(CP_ERR_BAD_PARAM, "p must be > 0");
    return th_objective(t, p, Tb_max, Tb_pnorm);
}

cp_status cp_thermal_pnorm_gradient(cp_thermal* t, double p, double* J, double* dJ_dgamma, cp_thermal_report* rep) {
    if (!t || !dJ_dgamma) return tfail(CP_ERR_BAD_PARAM, "NULL argument");
    if (!t->solved) return tfail(CP_ERR_STATE, "no solution yet (cp_thermal_solve)");
    if (!(p >= 1.0) || !std::isfinite(p)) return tfail(CP_ERR_BAD_PARAM, "p must be >= 1");
    const ThK& k = t->k;
    double Jv = 0.0;
    cp_status s = th_objective(t, p, nullptr, &Jv);
    if (s != CP_OK) return s;
    if (!(Jv > 0.0) || !std::isfinite(Jv))
        return tfail(CP_ERR_NONFINITE, "the p-norm of the bottom temperatures is %g", Jv);
    TCK(cudaEventRecord(t->ev0, t->stream));
    k_th_adj_rhs<<<t->gElem, kThThreads, 0, t->stream>>>(k, t->V.x, Jv, p, t->rhs);
    TCK(cudaGetLastError());
    TCK(cudaMemsetAsync(t->lam, 0, (size_t)k.n * 8, t->stream));
    ThVecs W = t->V;
    W.x = t->lam;
    ThStatus hs;
    s = th_krylov<true>(t, t->rhs, W, &hs);
    if (s != CP_OK) return s;
    k_th_sens<<<t->gElem, kThThreads, 0, t->stream>>>(k, t->gamma, t->V.x, t->lam, t->grad);
    TCK(cudaGetLastError());
    TCK(cudaEventRecord(t->ev1, t->stream));
    TCK(cudaMemcpyAsync(dJ_dgamma, t->grad, (size_t)k.ncol * 8, cudaMemcpyDeviceToHost, t->stream));
    TCK(cudaStreamSynchronize(t->stream));
    if (J) *J = Jv;
    th_report(t, hs, rep);
    return CP_OK;
}

}  // extern "C"
