// Micro-benchmarks behind the roofline notes: cost of the bounded grid
// barrier (with and without the fixed-order partial-sum reduction) versus
// blocks per SM, and streaming bandwidth for L2-resident and HBM-sized
// working sets.  Build and run on a B200:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 \
//        coldplate-solver_b200/diag/microbench.cu -o /tmp/cp_microbench && /tmp/cp_microbench
#include <cstdio>
#include <cuda_runtime.h>
#include "../csrc/cp_device.cuh"
using namespace cp;

__global__ void k_barriers(unsigned* bar, int* err, int nb) {
    unsigned target = 0;
    for (int k = 0; k < nb; ++k) {
        target += gridDim.x;
        if (!grid_barrier(bar, target, err)) return;
    }
}

// barrier + fixed-order reduction of per-block partials read by every block
__global__ void k_barrier_reduce(unsigned* bar, int* err, double* part, int nb, double* out) {
    __shared__ double sm[64];
    unsigned target = 0;
    double acc = 0;
    for (int k = 0; k < nb; ++k) {
        double v[1] = {(double)(blockIdx.x + k)};
        block_sum<1>(v, sm);
        if (threadIdx.x == 0) part[(k & 1) * gridDim.x + blockIdx.x] = v[0];
        target += gridDim.x;
        if (!grid_barrier(bar, target, err)) return;
        double t[1];
        sum_partials<1>(part + (k & 1) * gridDim.x, gridDim.x, 1, t, sm);
        acc += t[0];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *out = acc;
}

template <typename T>
__global__ void k_stream(const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ c, T* __restrict__ d, size_t n, int reps) {
    for (int r = 0; r < reps; ++r)
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
            d[i] = a[i] + b[i] * c[i] + (T)r;
}

int main() {
    int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    unsigned* bar; int* err; double* part; double* out;
    cudaMalloc(&bar, 4); cudaMalloc(&err, 4); cudaMalloc(&part, 8 * 2 * 8192); cudaMalloc(&out, 8);
    cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
    for (int threads : {256, 1024}) {
        int maxb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxb, k_barrier_reduce, threads, 0);
        for (int per : {1, 2, 4, 8}) {
            if (per > maxb) continue;
            int G = sms * per, nb = 2000;
            for (int variant = 0; variant < 2; ++variant) {
                float best = 1e9;
                for (int rep = 0; rep < 3; ++rep) {
                    cudaMemset(bar, 0, 4); cudaMemset(err, 0, 4);
                    void* args0[] = {&bar, &err, &nb};
                    void* args1[] = {&bar, &err, &part, &nb, &out};
                    cudaEventRecord(e0);
                    if (variant == 0) cudaLaunchCooperativeKernel((void*)k_barriers, G, threads, args0, 0, 0);
                    else cudaLaunchCooperativeKernel((void*)k_barrier_reduce, G, threads, args1, 0, 0);
                    cudaEventRecord(e1); cudaEventSynchronize(e1);
                    float ms; cudaEventElapsedTime(&ms, e0, e1); if (ms < best) best = ms;
                }
                int h_err; cudaMemcpy(&h_err, err, 4, cudaMemcpyDeviceToHost);
                printf("barrier%s threads=%d blocks/SM=%d G=%d: %.3f us per barrier (err %d)\n",
                       variant ? "+reduce" : "", threads, per, G, best * 1000.0 / nb, h_err);
            }
        }
    }
    // L2-resident streaming: 4 arrays of n elements
    for (size_t MB : {8, 17, 32, 64, 256}) {
        size_t n = MB * 1000000 / 8;
        double *a, *b, *c, *d;
        cudaMalloc(&a, n * 8); cudaMalloc(&b, n * 8); cudaMalloc(&c, n * 8); cudaMalloc(&d, n * 8);
        cudaMemset(a, 0, n * 8); cudaMemset(b, 0, n * 8); cudaMemset(c, 0, n * 8);
        int reps = 20;
        k_stream<<<sms * 8, 256>>>(a, b, c, d, n, 1);
        cudaEventRecord(e0);
        k_stream<<<sms * 8, 256>>>(a, b, c, d, n, reps);
        cudaEventRecord(e1); cudaEventSynchronize(e1);
        float ms; cudaEventElapsedTime(&ms, e0, e1);
        printf("stream fp64 4 arrays x %zu MB (total %zu MB): %.0f GB/s\n", MB, 4 * MB, 4.0 * n * 8 * reps / (ms * 1e-3) / 1e9);
        cudaFree(a); cudaFree(b); cudaFree(c); cudaFree(d);
    }
    printf("done %s\n", cudaGetErrorString(cudaGetLastError()));
    return 0;
}
