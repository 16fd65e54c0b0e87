// Device-side building blocks shared by the SIMPLE kernels: field indexing,
// the per-run parameter block, the device status word, deterministic block
// reductions and a bounded grid barrier for cooperative (persistent) kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cp_simple.h"

namespace cp {

// Upper bound on blocks of any kernel that writes per-block partial sums.
constexpr int kMaxBlocks = 4096;
// Columns of one history row (see HistCol).
constexpr int kHistCols = 20;

enum HistCol {
    H_ITER = 0, H_ERROR, H_RMS_U, H_RMS_V, H_RMS_MASS, H_MAX_U, H_MAX_V, H_MAX_MASS, H_ITERS_P,
    H_CORE_TOTAL, H_FULL_TOTAL, H_CORE_STATIC, H_FULL_STATIC, H_IN_FLUX, H_OUT_FLUX,
    H_ITERS_U, H_ITERS_V, H_RES_U, H_RES_V, H_RES_MASS
};

// Geometry of the padded row-major layout.  Every staggered array (u, v, p,
// dE, dN, cell fields, coefficients) is stored with the same pitch P (a
// multiple of 32 elements) and rows 0..M+1, so (i, j) maps to i * P + j for
// all of them and a warp reads 32 consecutive j of one row.
struct Dims {
    int M, N, P;
};

__host__ __device__ __forceinline__ size_t at(const Dims& d, int i, int j) {
    return (size_t)i * (size_t)d.P + (size_t)j;
}

// Scalars every kernel needs, passed by value.
struct KParams {
    Dims d;
    double hx, hy, rho, eta, uvAlpha, pAlpha;
    double targetVel;
    int rampOn, rampSteps;
    double convScale;   // twoPointFiveDConvectionFactor when 2.5-D is on, else 1
    double sinkDiag;    // 12 mu / Ht^2 * multiplier * vol when 2.5-D is on, else 0
    int sou;            // convectionScheme == 1
    double pTol, momTol;
    int maxP, maxMom;
    double xCoreIn, xCoreOut;
    double eps;
    int maxIterations;
    int normalized;
    double velFloor, massFloor;
    int dpConv, dpWindow, dpRampSteps;
    double dpPercent;
    int nU, nV, nP;     // unknowns: U (M-1)(N-2), V (M-2)(N-1), p' (M-1)(N-2)
};

// Device status block (one per context, zeroed at creation).
struct Status {
    int done;      // 1: the outer loop has stopped; every kernel returns at once
    int reason;    // cp_stop_reason
    int err;       // cp_status code raised on the device (timeout, non-finite)
    int iter;      // completed outer iterations
    int itersU, itersV, itersP, errWhere;
    unsigned long long maxDU, maxDV;   // bit patterns of non-negative doubles (atomicMax)
    double rms0U, rms0V, rms0M;
    int rms0Uset, rms0Vset, rms0Mset, dpFilled;
    int dpIdx, dpConverged, pad0, pad1;
    double lastError;
};

__host__ __device__ __forceinline__ double inlet_velocity(const KParams& k, int iter) {
    if (k.rampOn && k.rampSteps > 0 && iter < k.rampSteps)
        return ((double)(iter + 1) / (double)k.rampSteps) * k.targetVel;
    return k.targetVel;
}

__host__ __device__ __forceinline__ double max_vel(double uin) {
    double a = uin < 0 ? -uin : uin;
    return 3.0 * (a < 0.1 ? 0.1 : a);
}

// std::clamp / std::max / std::min semantics
template <typename T>
__device__ __forceinline__ T dclamp(T x, T lo, T hi) { return (x < lo) ? lo : ((hi < x) ? hi : x); }
template <typename T>
__device__ __forceinline__ T dmax(T a, T b) { return (a < b) ? b : a; }
template <typename T>
__device__ __forceinline__ T dmin(T a, T b) { return (b < a) ? b : a; }

// ------------------------------------------------------------ reductions
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum of NV values over the block; result valid in every thread.  Fixed
// order, so the same inputs give the same bits on every run.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* >= 32*NV */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[k * 32 + wid] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = (lane < nw) ? smem[k * 32 + lane] : 0.0;
        v[k] = warp_sum(t);
    }
    __syncthreads();
}

// Sum of per-block partials part[b * stride + k], b < nb, in a fixed order;
// every thread of the block gets the totals.
template <int NV>
__device__ __forceinline__ void sum_partials(const double* part, int nb, int stride, double (&out)[NV],
                                             double* smem) {
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) out[k] += __ldcg(part + (size_t)b * stride + k);
    block_sum<NV>(out, smem);
}

// ------------------------------------------------------------ grid barrier
// Arrival counter that only grows during one launch (the host zeroes it
// before each cooperative launch).  Waiting is bounded: after kBarrierNs of
// spinning the block records CP_ERR_TIMEOUT and the caller must return.
constexpr unsigned long long kBarrierNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Returns false if the wait gave up (after limitNs of spinning) or another
// block already failed.
__device__ __forceinline__ bool grid_barrier(unsigned* counter, unsigned target, int* err,
                                             unsigned long long limitNs = kBarrierNs) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        // release pattern: the acq_rel fence orders the block's writes (made
        // before the __syncthreads above) ahead of the relaxed arrival; the
        // acquire loads below order the reads after it, and the closing
        // __syncthreads extends both to the whole block
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        asm volatile("red.relaxed.gpu.global.add.u32 [%0], 1;" ::"l"(counter) : "memory");
        unsigned long long t0 = 0;
        unsigned spins = 0;
        while (ld_acquire_u32(counter) < target) {
            if (((++spins) & 255u) == 0) {
                unsigned long long t = globaltimer_ns();
                if (t0 == 0) t0 = t;
                else if (t - t0 > limitNs || spins > (1u << 30)) {
                    atomicCAS(err, 0, (int)CP_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
            if (*(volatile int*)err != 0) { ok = 0; break; }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// A team of CTAs that runs one phase sequence together, synchronised by its
// own bounded barrier: the whole grid of a single-field launch, or a group
// of consecutive CTAs of the batched kernel that solves one field at a time.
// Partial sums are written per team rank and summed over the team's size.
struct Team {
    int rank, size;      // CTA index in the team, CTAs in the team
    unsigned* bar;       // the team's barrier counter (grows during a launch)
    int* err;            // first device error (barrier time-out)
    __device__ __forceinline__ int tid() const { return rank * (int)blockDim.x + (int)threadIdx.x; }
    __device__ __forceinline__ int nth() const { return size * (int)blockDim.x; }
    __device__ __forceinline__ bool lead() const { return rank == 0 && threadIdx.x == 0; }
};

__device__ __forceinline__ Team grid_team(unsigned* bar, int* err) {
    return Team{(int)blockIdx.x, (int)gridDim.x, bar, err};
}

__device__ __forceinline__ bool team_sync(const Team& T, unsigned& target) {
    target += (unsigned)T.size;
    return grid_barrier(T.bar, target, T.err);
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* addr, double v) {
    // non-negative IEEE doubles order like their bit patterns
    if (v > 0.0) atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// ------------------------------------------------------------ row segments
// 16 bytes of one row: 4 floats or 2 doubles
template <typename TV>
struct Vec16 {
    static constexpr int n = 16 / (int)sizeof(TV);
    TV v[n];
};
__device__ __forceinline__ Vec16<float> ld16(const float* p) {
    const float4 f = *reinterpret_cast<const float4*>(p);
    return {{f.x, f.y, f.z, f.w}};
}
__device__ __forceinline__ Vec16<double> ld16(const double* p) {
    const double2 f = *reinterpret_cast<const double2*>(p);
    return {{f.x, f.y}};
}
__device__ __forceinline__ void st16(float* p, const Vec16<float>& a) {
    *reinterpret_cast<float4*>(p) = make_float4(a.v[0], a.v[1], a.v[2], a.v[3]);
}
__device__ __forceinline__ void st16(double* p, const Vec16<double>& a) {
    *reinterpret_cast<double2*>(p) = make_double2(a.v[0], a.v[1]);
}
template <typename TV>
__device__ __forceinline__ Vec16<TV> zero16() {
    Vec16<TV> a;
#pragma unroll
    for (int k = 0; k < Vec16<TV>::n; ++k) a.v[k] = (TV)0;
    return a;
}

// Row segments of a level in the padded layout (unknowns i in [1, nI],
// j in [1, nJ], row pitch P): warp w takes segments w, w + nwarps, ... of 32
// lane groups of one row, lane group g covering columns [g V, g V + V)
// (V = 16 / sizeof(TV)); fn(i, j0, act, lane) with act false on the groups
// past the row's last unknown.  The loop is uniform over each warp, so fn
// may shuffle.  A vector of a group with g V <= nJ stays inside the row
// (the pitch is a multiple of 32 above nJ), and column g V + V, read by lane
// 31, is at most the next row's column 0.
template <typename TV, typename F>
__device__ __forceinline__ void row_segments(const Team& T, int nI, int nJ, F&& fn) {
    constexpr int V = Vec16<TV>::n;
    const int lane = threadIdx.x & 31;
    const int warp = T.tid() >> 5, nw = T.nth() >> 5;
    const int Ga = nJ / V + 1, S = (Ga + 31) >> 5;
    for (int s = warp; s < nI * S; s += nw) {
        const int i = 1 + s / S, g = ((s % S) << 5) + lane;
        fn(i, g * V, g < Ga, lane);
    }
}
template <typename TV, typename F>
__device__ __forceinline__ void row_segments(int nI, int nJ, F&& fn) {
    row_segments<TV>(Team{(int)blockIdx.x, (int)gridDim.x, nullptr, nullptr}, nI, nJ, static_cast<F&&>(fn));
}

template <typename TV>
__device__ __forceinline__ TV from_west(TV v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <typename TV>
__device__ __forceinline__ TV from_east(TV v) { return __shfl_down_sync(0xffffffffu, v, 1); }

}  // namespace cp
