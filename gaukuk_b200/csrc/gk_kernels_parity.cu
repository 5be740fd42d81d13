// Kernels in parity mode: compiled with -fmad=false, correctly rounded
// division and square root, the HLLC sides combined as the reference does
// (hllc.cpp:71-94; the unused side is skipped only where that provably gives
// the same bits).
#define GK_NS gk_parity
#define GK_SEL 2
#define GK_FASTMATH 0
#include "gk_kernels.cuh"

namespace gk_parity {

// Parity mode's quotient and root against CUDA's IEEE `/` and sqrt(): over n
// random argument pairs, counts results whose bits differ (NaN matches NaN)
// and arguments the acceptance test sent to the IEEE operation.  Arguments:
// random signs, exponents over the whole double range and significands
// (zeros, subnormals, infinities, NaNs and powers of two included), and a
// second set of quotients close to 1 (a = b*(1 + small)), where the
// candidate is most often one ulp off before its correction.
// out[0..4]: division mismatches, division fallbacks, root mismatches, root
// fallbacks, arguments tried.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double random_double(unsigned long long z) {
    const unsigned long long kind = z & 15u;
    unsigned long long bits = mix64(z + 0x9E3779B97F4A7C15ULL);
    if (kind == 0) bits &= 0x800fffffffffffffull;                      // zero or subnormal
    else if (kind == 1) bits = (bits & 0x8000000000000000ull) | 0x7ff0000000000000ull |
                               ((z >> 8) & 1 ? 0x0008000000000000ull : 0);  // inf or NaN
    else if (kind == 2) bits &= 0xfff0000000000000ull;                  // powers of two
    return __longlong_as_double((long long)bits);
}

__global__ void k_paritymath_check(long long n, unsigned long long seed, unsigned long long* out) {
    unsigned long long dmis = 0, dfb = 0, smis = 0, sfb = 0, tried = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long z = mix64(seed ^ (0xD1B54A32D192ED03ULL * (unsigned long long)(i + 1)));
        double a = random_double(z), b = random_double(mix64(z + 1));
        if ((i & 1) == 0) {
            // quotients near 1 with normal operands
            const double u = (double)(mix64(z + 2) >> 11) * (1.0 / 9007199254740992.0);
            b = __longlong_as_double((long long)(dbits(b) & 0x800fffffffffffffull) |
                                     (0x3ff0000000000000ll + ((long long)((z >> 20) & 255) - 128) * (1ll << 52)));
            a = __dmul_rn(b, 1.0 + (u - 0.5) * 1e-12);
        }
        bool ok;
        const double q = div_rn_candidate(a, b, ok);
        const double qe = a / b;
        const double qg = ok ? q : qe;
        dfb += !ok;
        dmis += !((isnan(qg) && isnan(qe)) || dbits(qg) == dbits(qe));
        const double x = fabs(a);
        const double sv = sqrt_rn_candidate(x, ok);
        const double se = sqrt(x);
        const double sg = ok ? sv : se;
        sfb += !ok;
        smis += !((isnan(sg) && isnan(se)) || dbits(sg) == dbits(se));
        ++tried;
    }
    atomicAdd(&out[0], dmis);
    atomicAdd(&out[1], dfb);
    atomicAdd(&out[2], smis);
    atomicAdd(&out[3], sfb);
    atomicAdd(&out[4], tried);
}

int paritymath_check(long long n, unsigned long long seed, unsigned long long* host_out5) {
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, 5 * sizeof(unsigned long long)) != cudaSuccess) return -1;
    cudaMemset(d, 0, 5 * sizeof(unsigned long long));
    k_paritymath_check<<<148 * 4, 256>>>(n, seed, d);
    cudaError_t e = cudaMemcpy(host_out5, d, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -1;
}

}  // namespace gk_parity
