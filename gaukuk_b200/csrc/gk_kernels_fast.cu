// Kernels in fast mode: FMA contraction allowed, only the selected HLLC side
// evaluated, branch-free refined reciprocal / square root (gk_physics.cuh).
#define GK_NS gk_fast
#define GK_SEL 1
#define GK_FASTMATH 1
#include "gk_kernels.cuh"

namespace gk_fast {

// Error of the refined reciprocal, square root and reciprocal square root
// against CUDA's IEEE operations, in units in the last place of the IEEE
// result, over n arguments spread log-uniformly on [2^-60, 2^60].
__global__ void k_fastmath_check(int n, unsigned long long seed, double* worst) {
    double w0 = 0, w1 = 0, w2 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
        const double x = exp2(120.0 * u - 60.0);
        const double e[3] = {1.0 / x, sqrt(x), 1.0 / sqrt(x)};
        const double a[3] = {rcp_nr(x), sqrt_nr(x), rsqrt_nr(x)};
        double err[3];
        for (int k = 0; k < 3; ++k) {
            // spacing above the (positive, normal) IEEE result
            const double ulp = __longlong_as_double(__double_as_longlong(e[k]) + 1) - e[k];
            err[k] = fabs(a[k] - e[k]) / ulp;
        }
        w0 = fmax(w0, err[0]);
        w1 = fmax(w1, err[1]);
        w2 = fmax(w2, err[2]);
    }
    // reduce: non-negative doubles order like their bits
    atomicMax((unsigned long long*)&worst[0], (unsigned long long)__double_as_longlong(w0));
    atomicMax((unsigned long long*)&worst[1], (unsigned long long)__double_as_longlong(w1));
    atomicMax((unsigned long long*)&worst[2], (unsigned long long)__double_as_longlong(w2));
}

int fastmath_check(int n, unsigned long long seed, double* host_worst3) {
    double* d = nullptr;
    if (cudaMalloc(&d, 3 * sizeof(double)) != cudaSuccess) return -1;
    cudaMemset(d, 0, 3 * sizeof(double));
    k_fastmath_check<<<148 * 4, 256>>>(n, seed, d);
    cudaError_t e = cudaMemcpy(host_worst3, d, 3 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -1;
}

}  // namespace gk_fast
