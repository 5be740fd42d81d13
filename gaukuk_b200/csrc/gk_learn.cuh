// gk_learn.cuh -- the device pieces of the learned flux correction that the
// generic-path correction pass (gk_mlp.cu) and the fused 2D stage
// (gk_kernels.cuh, both arithmetic modes) share: the network's fragment
// loads and tensor-core products, its activation, the face features and
// detector, and the corrected flux.  Included inside a namespace, after
// <cuda_bf16.h> and gk_internal.h.
//
// The units that include it are compiled with and without FMA contraction
// (the parity unit has -fmad=false).  Every product that feeds a sum here is
// therefore written with explicit round-to-nearest intrinsics (__dmul_rn,
// __dadd_rn, __fmaf_rn, ...), and the activation, reciprocals and roots use
// the approximation instructions directly (with explicit Newton steps), so
// the same inputs give the same bits in every unit: the fused stage's
// corrections equal the correction pass's.
#pragma once

namespace gklearn {

constexpr int NI = 16, NH = 64, NO = 4;
constexpr int W1O = 0, B1O = W1O + NH * NI, W2O = B1O + NH, B2O = W2O + NH * NH;
constexpr int W3O = B2O + NH, B3O = W3O + NO * NH, NPARAM = B3O + NO;  // 5508
constexpr int XMO = NPARAM, XSO = XMO + NI, YMO = XSO + NI, YSO = YMO + NO;
constexpr int NMODEL = YSO + NO;  // parameters + normalisation = 5548 floats

constexpr float kGeluA = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float kGeluB = 0.044715f;
constexpr float kGeluE = -2.0f * 0.7978845608028654f * 1.4426950408889634f;  // -2 sqrt(2/pi) log2(e)
constexpr float kGeluEB = kGeluE * 0.044715f;

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// GELU, tanh form: 0.5 x (1 + tanh(u)), u = sqrt(2/pi) (x + 0.044715 x^3),
// evaluated as x * s with s = 0.5 (1 + tanh(u)) = 1 / (1 + exp(-2u)) (an
// identity, with no cancellation for small u), exp(-2u) = 2^(x (E + E B x^2))
// with E = -2 sqrt(2/pi) log2(e); dgelu receives the derivative
// s + 2 x s (1 - s) sqrt(2/pi) (1 + 3 * 0.044715 x^2).
__device__ __forceinline__ float gelu(float x, float* dgelu) {
    const float x2 = __fmul_rn(x, x);
    const float arg = __fmul_rn(x, __fmaf_rn(kGeluEB, x2, kGeluE));
    const float s = rcp_approx(__fadd_rn(1.f, ex2_approx(arg)));
    if (dgelu) {
        const float du = __fmul_rn(2.f * kGeluA, __fmaf_rn(3.f * kGeluB, x2, 1.f));
        *dgelu = __fmaf_rn(__fmul_rn(x, __fmul_rn(s, __fsub_rn(1.f, s))), du, s);
    }
    return __fmul_rn(x, s);
}

__device__ __forceinline__ unsigned pack(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Fragment loads from shared memory by the layouts of mma.m16n8k16 (PTX ISA):
// A rows g, g+8 and column pairs 2t, 2t+8; B row pairs 2t, 2t+8 and column
// g; g = lane / 4, t = lane % 4.  Where a register's two BF16 values are
// adjacent in S (row-major A and [n][k] B) it is one 32-bit load: S is
// 16-byte aligned and ld, k0 are even.
__device__ __forceinline__ unsigned ld_pair(const __nv_bfloat16* S, int i) {
    return *reinterpret_cast<const unsigned*>(S + i);
}
// A(m, k) = S[m0 + m][k0 + k], S row-major with leading dimension ld.
__device__ __forceinline__ void load_a(unsigned (&a)[4], const __nv_bfloat16* S, int ld, int m0, int k0) {
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    a[0] = ld_pair(S, (m0 + g) * ld + k0 + 2 * t);
    a[1] = ld_pair(S, (m0 + g + 8) * ld + k0 + 2 * t);
    a[2] = ld_pair(S, (m0 + g) * ld + k0 + 2 * t + 8);
    a[3] = ld_pair(S, (m0 + g + 8) * ld + k0 + 2 * t + 8);
}
// A(m, k) = S[k0 + k][m0 + m] (the transpose of a row-major S).
__device__ __forceinline__ void load_at(unsigned (&a)[4], const __nv_bfloat16* S, int ld, int m0, int k0) {
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    a[0] = pack(S[(k0 + 2 * t) * ld + m0 + g], S[(k0 + 2 * t + 1) * ld + m0 + g]);
    a[1] = pack(S[(k0 + 2 * t) * ld + m0 + g + 8], S[(k0 + 2 * t + 1) * ld + m0 + g + 8]);
    a[2] = pack(S[(k0 + 2 * t + 8) * ld + m0 + g], S[(k0 + 2 * t + 9) * ld + m0 + g]);
    a[3] = pack(S[(k0 + 2 * t + 8) * ld + m0 + g + 8], S[(k0 + 2 * t + 9) * ld + m0 + g + 8]);
}
// B(k, n) = S[n0 + n][k0 + k] (S row-major [n][k], e.g. weights W[out][in]).
__device__ __forceinline__ void load_b_nk(unsigned (&b)[2], const __nv_bfloat16* S, int ld, int n0, int k0) {
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    b[0] = ld_pair(S, (n0 + g) * ld + k0 + 2 * t);
    b[1] = ld_pair(S, (n0 + g) * ld + k0 + 2 * t + 8);
}
// B(k, n) = S[k0 + k][n0 + n] (S row-major [k][n]).
__device__ __forceinline__ void load_b_kn(unsigned (&b)[2], const __nv_bfloat16* S, int ld, int n0, int k0) {
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    b[0] = pack(S[(k0 + 2 * t) * ld + n0 + g], S[(k0 + 2 * t + 1) * ld + n0 + g]);
    b[1] = pack(S[(k0 + 2 * t + 8) * ld + n0 + g], S[(k0 + 2 * t + 9) * ld + n0 + g]);
}

// Weights in shared memory as BF16 (W3 padded to 16 output rows with zeros),
// biases as FP32, and the normalisation (input means and deviations, output
// means and deviations).
struct MlpWeights {
    alignas(16) __nv_bfloat16 w1[NH * NI];
    alignas(16) __nv_bfloat16 w2[NH * NH];
    alignas(16) __nv_bfloat16 w3[16 * NH];
    float b1[NH], b2[NH], b3[8];
    float norm[2 * NI + 2 * NO];
};

// Every thread of the block takes part; the caller synchronises after it.
__device__ __forceinline__ void load_weights(MlpWeights& s, const float* __restrict__ p) {
    for (int i = threadIdx.x; i < NH * NI; i += blockDim.x) s.w1[i] = __float2bfloat16_rn(p[W1O + i]);
    for (int i = threadIdx.x; i < NH * NH; i += blockDim.x) s.w2[i] = __float2bfloat16_rn(p[W2O + i]);
    for (int i = threadIdx.x; i < 16 * NH; i += blockDim.x)
        s.w3[i] = i < NO * NH ? __float2bfloat16_rn(p[W3O + i]) : __float2bfloat16_rn(0.f);
    for (int i = threadIdx.x; i < NH; i += blockDim.x) {
        s.b1[i] = p[B1O + i];
        s.b2[i] = p[B2O + i];
    }
    for (int i = threadIdx.x; i < 8; i += blockDim.x) s.b3[i] = i < NO ? p[B3O + i] : 0.f;
    for (int i = threadIdx.x; i < 2 * NI + 2 * NO; i += blockDim.x) s.norm[i] = p[XMO + i];
}

// Forward pass of MT 16-face tiles at once (one warp): x their standardised
// inputs [16 MT][NI] in shared memory.  The hidden activations never leave
// the registers: the C fragment of output columns 8j .. 8j+7 of one layer
// is, after the activation, half of the A fragment of the next layer's
// k-step j / 2 (C rows g, g+8 and columns 2t, 2t+1 are A's).  Each weight
// fragment is loaded once for the MT tiles, whose products are independent.
// Every sum has the order of a one-tile pass (bias, then k-steps in order),
// so any MT gives the same bits.  y[m] receives tile m's output C fragment:
// lane (g, t < 2) holds outputs 2t, 2t+1 of faces g (y[m][0], y[m][1]) and
// g + 8 (y[m][2], y[m][3]).
template <int MT>
__device__ __forceinline__ void forward_tiles(const MlpWeights& w, const __nv_bfloat16* x,
                                              float (&y)[MT][4]) {
    const int lane = threadIdx.x & 31, t = lane & 3;
    auto act_pair = [](float lo, float hi) {
        return pack(__float2bfloat16_rn(gelu(lo, nullptr)), __float2bfloat16_rn(gelu(hi, nullptr)));
    };
    unsigned xa[MT][4];
#pragma unroll
    for (int m = 0; m < MT; ++m) load_a(xa[m], x, NI, 16 * m, 0);
    // layer 1 -> A fragments of layer 2 (k-steps 0..3)
    unsigned h1[MT][4][4];
#pragma unroll
    for (int kb = 0; kb < 4; ++kb) {
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int j = 2 * kb + half;
            unsigned b[2];
            load_b_nk(b, w.w1, NI, 8 * j, 0);
            const float b0 = w.b1[8 * j + 2 * t], b1v = w.b1[8 * j + 2 * t + 1];
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                float z[4] = {b0, b1v, b0, b1v};
                mma(z, xa[m], b);
                h1[m][kb][2 * half] = act_pair(z[0], z[1]);
                h1[m][kb][2 * half + 1] = act_pair(z[2], z[3]);
            }
        }
    }
    // layer 2, two output blocks at a time -> A fragment of layer 3's k-step
    float acc[MT][4];
#pragma unroll
    for (int m = 0; m < MT; ++m) {
        acc[m][0] = acc[m][2] = w.b3[2 * t];
        acc[m][1] = acc[m][3] = w.b3[2 * t + 1];
    }
#pragma unroll
    for (int k3 = 0; k3 < 4; ++k3) {
        unsigned a3[MT][4];
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int j = 2 * k3 + half;
            const float b0 = w.b2[8 * j + 2 * t], b1v = w.b2[8 * j + 2 * t + 1];
            float z[MT][4];
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                z[m][0] = z[m][2] = b0;
                z[m][1] = z[m][3] = b1v;
            }
#pragma unroll
            for (int kb = 0; kb < 4; ++kb) {
                unsigned b[2];
                load_b_nk(b, w.w2, NH, 8 * j, 16 * kb);
#pragma unroll
                for (int m = 0; m < MT; ++m) mma(z[m], h1[m][kb], b);
            }
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                a3[m][2 * half] = act_pair(z[m][0], z[m][1]);
                a3[m][2 * half + 1] = act_pair(z[m][2], z[m][3]);
            }
        }
        unsigned b[2];
        load_b_nk(b, w.w3, NH, 0, 16 * k3);
#pragma unroll
        for (int m = 0; m < MT; ++m) mma(acc[m], a3[m], b);
    }
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int e = 0; e < 4; ++e) y[m][e] = acc[m][e];
}

// Reciprocal and square root of the features and bounds: the hardware
// approximations with one Newton step (relative error about 2^-44; the
// features go to BF16 and the bounds to FP32), written as explicit products
// and fused multiply-adds so every unit compiles them alike.  x > 0.
__device__ __forceinline__ double lrcp(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return fma(y, fma(-x, y, 1.0), y);
}
__device__ __forceinline__ double lsqrt(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double s = __dmul_rn(x, y);
    return fma(__dmul_rn(0.5, y), fma(-s, s, x), s);
}

// van Leer slope of the PLM reconstruction, (2ab)/(a+b) for ab > 0 else 0.
__device__ __forceinline__ double vl_slope(double a, double b) {
    const double m = __dmul_rn(a, b);
    return m <= 0.0 ? 0.0 : __dmul_rn(__dmul_rn(2.0, m), lrcp(__dadd_rn(a, b)));
}

// What the detector and the output scaling need of one face, from its
// stencil (cells -2, -1 | 0, +1): scale[0..2] = rho_ref c, rho_ref c^2,
// rho_ref c^3; gate 0 shock, 1 correct, 2 smooth; the smaller density and
// internal energy of the two cells next to the face; clip bounds of the 4
// outputs (negative: none).
struct FaceScale {
    float scale[3];
    float gate;
    float dmin, emin;
    float clip[4];
};

// Inputs (standardised, BF16) and FaceScale of one face.  r, vn, vt, p: the
// stencil's density, normal and tangential velocity and pressure.
__device__ __forceinline__ void face_inputs(const double (&r)[4], const double (&vn)[4],
                                            const double (&vt)[4], const double (&p)[4],
                                            double gamma, double gm1Rec, const gk::FluxGate& gate,
                                            const float* __restrict__ norm, __nv_bfloat16* x,
                                            FaceScale& fs) {
    const double rr = __dmul_rn(0.25, __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), r[2]), r[3]));
    const double pr = __dmul_rn(0.25, __dadd_rn(__dadd_rn(__dadd_rn(p[0], p[1]), p[2]), p[3]));
    // the features go to BF16: reciprocals of the references serve all four cells
    const double irr = lrcp(rr), ipr = lrcp(pr);
    const double cr = lsqrt(__dmul_rn(__dmul_rn(gamma, pr), irr));
    const double icr = lrcp(cr);
    float feat[NI];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        feat[4 * c + 0] = __double2float_rn(__dsub_rn(__dmul_rn(r[c], irr), 1.0));
        feat[4 * c + 1] = __double2float_rn(__dmul_rn(vn[c], icr));
        feat[4 * c + 2] = __double2float_rn(__dmul_rn(vt[c], icr));
        feat[4 * c + 3] = __double2float_rn(__dsub_rn(__dmul_rn(p[c], ipr), 1.0));
    }
    float tv = 0.f;  // total variation of the stencil's features
#pragma unroll
    for (int e = 4; e < NI; ++e) tv = __fadd_rn(tv, fabsf(__fsub_rn(feat[e], feat[e - 4])));
    double pmax = p[0], pmin = p[0];
#pragma unroll
    for (int c = 1; c < 4; ++c) {
        pmax = fmax(pmax, p[c]);
        pmin = fmin(pmin, p[c]);
    }
    const bool shock = pmax > __dmul_rn(__dadd_rn(1.0, (double)gate.shock_jump), pmin);
    const double rc = __dmul_rn(rr, cr), rc2 = __dmul_rn(rc, cr);
    fs.scale[0] = __double2float_rn(rc);
    fs.scale[1] = __double2float_rn(rc2);
    fs.scale[2] = __double2float_rn(__dmul_rn(rc2, cr));
    fs.gate = shock ? 0.f : (tv >= gate.tv_min ? 1.f : 2.f);
    fs.dmin = __double2float_rn(fmin(r[1], r[2]));
    fs.emin = __double2float_rn(__dmul_rn(fmin(p[1], p[2]), gm1Rec));
    if (gate.diss_frac >= 0.f) {
        // (1/2) max(|vn| + c) |U_R - U_L| of the van Leer PLM face states
        const double* q[4] = {r, vn, vt, p};
        double wl[4], wr[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            wl[v] = __dadd_rn(q[v][1], __dmul_rn(0.5, vl_slope(__dsub_rn(q[v][1], q[v][0]),
                                                               __dsub_rn(q[v][2], q[v][1]))));
            wr[v] = __dsub_rn(q[v][2], __dmul_rn(0.5, vl_slope(__dsub_rn(q[v][2], q[v][1]),
                                                               __dsub_rn(q[v][3], q[v][2]))));
        }
        double ul[4], ur[4], sp[2];
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const double* w = side ? wr : wl;
            double* u = side ? ur : ul;
            const double d = fmax(w[0], 1e-300), a = w[1], b = w[2];
            const double pp = fmax(w[3], 0.0);
            u[0] = d;
            u[1] = __dmul_rn(d, a);
            u[2] = __dmul_rn(d, b);
            u[3] = __dadd_rn(__dmul_rn(pp, gm1Rec),
                             __dmul_rn(__dmul_rn(0.5, d), __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b))));
            const double c2 = __dmul_rn(__dmul_rn(gamma, pp), lrcp(d));
            sp[side] = __dadd_rn(fabs(a), c2 > 0.0 ? lsqrt(c2) : 0.0);
        }
        const double sm = __dmul_rn(__dmul_rn(0.5, fmax(sp[0], sp[1])), (double)gate.diss_frac);
#pragma unroll
        for (int o = 0; o < 4; ++o) fs.clip[o] = __double2float_rn(__dmul_rn(sm, fabs(__dsub_rn(ur[o], ul[o]))));
    } else {
#pragma unroll
        for (int o = 0; o < 4; ++o) fs.clip[o] = -1.f;
    }
#pragma unroll
    for (int e = 0; e < NI; ++e)
        x[e] = __float2bfloat16_rn(__fdiv_rn(__fsub_rn(feat[e], norm[e]), norm[NI + e]));
}

// The correction of output o (0 mass, 1 normal momentum, 2 tangential
// momentum, 3 energy) from the standardised network output y: clipped to the
// training range (+-4 deviations), de-standardised, scaled, and clipped to
// the face's dissipation bound.
__device__ __forceinline__ double face_correction(float y, int o, const FaceScale& fs,
                                                  const float* __restrict__ norm) {
    const float yc = fminf(fmaxf(y, -4.f), 4.f);
    const float ys = __fmaf_rn(yc, norm[2 * NI + NO + o], norm[2 * NI + o]);
    double c = __dmul_rn((double)ys, (double)fs.scale[o == 0 ? 0 : (o == 3 ? 2 : 1)]);
    const double bound = fs.clip[o];
    if (bound >= 0.0) c = fmin(fmax(c, -bound), bound);
    return c;
}

// The positivity detector: the correction would move more than pos_frac of
// an adjacent cell's mass (c0) or internal energy (c3) in one step
// (dtdx = dt / dx along the face normal).
__device__ __forceinline__ bool face_vetoed(double c0, double c3, double dtdx, const FaceScale& fs,
                                            const gk::FluxGate& gate) {
    return fs.gate == 0.f ||
           __dmul_rn(fabs(c0), dtdx) > (double)__fmul_rn(gate.pos_frac, fs.dmin) ||
           __dmul_rn(fabs(c3), dtdx) > (double)__fmul_rn(gate.pos_frac, fs.emin);
}

}  // namespace gklearn
