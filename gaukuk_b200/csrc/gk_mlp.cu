// gk_mlp.cu -- the learned flux correction: a 16 -> 64 -> 64 -> 4 MLP (GELU)
// trained and evaluated on the tensor cores in BF16 with FP32 accumulation.
//
// Inputs: the 4-cell stencil across a face (cells -2, -1 | +0, +1), each cell
// as (rho/rho_ref - 1, vn/c_ref, vt/c_ref, p/p_ref - 1) with rho_ref, p_ref
// the stencil means and c_ref = sqrt(gamma p_ref / rho_ref); then standardised
// with the training set's means and deviations.  Outputs: the correction to
// the face's HLLC flux (mass, normal momentum, tangential momentum, energy)
// in units of rho_ref*c_ref, rho_ref*c_ref^2, rho_ref*c_ref^2, rho_ref*c_ref^3,
// standardised the same way.  The correction is added in FP64 to the face
// flux, so the update stays conservative.
//
// All matrix products are mma.sync.m16n8k16 (BF16 in, FP32 accumulate) on
// 16-sample tiles, one warp per tile; operands are gathered from shared
// memory by the fragment layouts of the PTX ISA (A: rows g, g+8 and column
// pairs 2t, 2t+8; B: row pairs 2t, 2t+8 and column g; C: rows g, g+8,
// columns 2t, 2t+1; g = lane / 4, t = lane % 4).
#include <cuda_bf16.h>

#include <cstdio>
#include <cstring>

#include "gaukuk_cuda.h"
#include "gk_internal.h"
#include "gk_learn.cuh"

namespace {

using namespace gklearn;

// Per-warp activations of one 16-sample tile (BF16, row = sample).
struct TileAct {
    alignas(16) __nv_bfloat16 x[16 * NI];
    alignas(16) __nv_bfloat16 h1[16 * NH];
    alignas(16) __nv_bfloat16 h2[16 * NH];
    alignas(16) __nv_bfloat16 dz1[16 * NH];
    alignas(16) __nv_bfloat16 dz2[16 * NH];
    alignas(16) __nv_bfloat16 dy[16 * 16];
};

// Forward pass of one tile whose inputs are in act.x.  Keeps Z1, Z2 (FP32 C
// fragments, for the backward pass) and writes H1, H2 to act; y receives the
// output C fragment (columns 0..3 valid).
__device__ __forceinline__ void forward_tile(const MlpWeights& w, TileAct& act, float (&z1)[8][4],
                                             float (&z2)[8][4], float (&y)[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    unsigned a[4], b[2];
    load_a(a, act.x, NI, 0, 0);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        z1[j][0] = z1[j][2] = w.b1[8 * j + 2 * t];
        z1[j][1] = z1[j][3] = w.b1[8 * j + 2 * t + 1];
        load_b_nk(b, w.w1, NI, 8 * j, 0);
        mma(z1[j], a, b);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * t;
        act.h1[g * NH + c] = __float2bfloat16_rn(gelu(z1[j][0], nullptr));
        act.h1[g * NH + c + 1] = __float2bfloat16_rn(gelu(z1[j][1], nullptr));
        act.h1[(g + 8) * NH + c] = __float2bfloat16_rn(gelu(z1[j][2], nullptr));
        act.h1[(g + 8) * NH + c + 1] = __float2bfloat16_rn(gelu(z1[j][3], nullptr));
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        z2[j][0] = z2[j][2] = w.b2[8 * j + 2 * t];
        z2[j][1] = z2[j][3] = w.b2[8 * j + 2 * t + 1];
    }
#pragma unroll
    for (int kb = 0; kb < 4; ++kb) {
        load_a(a, act.h1, NH, 0, 16 * kb);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            load_b_nk(b, w.w2, NH, 8 * j, 16 * kb);
            mma(z2[j], a, b);
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * t;
        act.h2[g * NH + c] = __float2bfloat16_rn(gelu(z2[j][0], nullptr));
        act.h2[g * NH + c + 1] = __float2bfloat16_rn(gelu(z2[j][1], nullptr));
        act.h2[(g + 8) * NH + c] = __float2bfloat16_rn(gelu(z2[j][2], nullptr));
        act.h2[(g + 8) * NH + c + 1] = __float2bfloat16_rn(gelu(z2[j][3], nullptr));
    }
    __syncwarp();
    y[0] = y[2] = w.b3[2 * t];
    y[1] = y[3] = w.b3[2 * t + 1];
#pragma unroll
    for (int kb = 0; kb < 4; ++kb) {
        load_a(a, act.h2, NH, 0, 16 * kb);
        load_b_nk(b, w.w3, NH, 0, 16 * kb);
        mma(y, a, b);
    }
}

// ------------------------------------------------------------ training
// One pass over a batch: forward, MSE loss on standardised targets,
// backward, and the batch-summed gradient into grad (FP32, NPARAM).  A CTA of
// 4 warps handles 4 tiles at a time; after the per-tile passes each warp
// accumulates one 16-row slice of dW2 and dW1 (and a 16-column slice of dW3)
// over the CTA's tiles in registers and adds it to grad at the end.
struct TrainShared {
    MlpWeights w;
    TileAct act[4];
};

// Sample in row r of tile `tile` of a batch: idx[tile*16 + r] when a batch
// index list is given, else the samples in order; in pair mode the in-order
// rows r and r + 8 hold the two members of a pair (2m, 2m + 1).
__device__ __forceinline__ long long batch_sample(const long long* idx, int tile, int r, bool pairs) {
    if (idx) return idx[tile * 16 + r];
    return (long long)tile * 16 + (pairs ? 2 * (r & 7) + (r >> 3) : r);
}

// Loss per sample: the squared error summed over the 4 outputs; in pair mode
// (pairs of samples that are neighbouring faces, rows g and g + 8 of a tile)
// (1 - pw) (e0^2 + e1^2) + pw (e1 - e0)^2 per output, e the errors of the two
// members: the error of their difference is what the cell between the two
// faces sees.
__global__ void __launch_bounds__(128) k_mlp_grad(const float* __restrict__ params,
                                                  const __nv_bfloat16* __restrict__ X,
                                                  const float* __restrict__ T, long long n,
                                                  const long long* __restrict__ idx, int batch,
                                                  float* __restrict__ grad, float* __restrict__ loss,
                                                  int pairs, float pw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainShared& sh = *reinterpret_cast<TrainShared*>(smem_raw);
    load_weights(sh.w, params);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    TileAct& act = sh.act[warp];
    float acc2[8][4] = {}, acc1[2][4] = {}, acc3[2][4] = {};
    float db1 = 0.f, db2 = 0.f, db3 = 0.f, lsum = 0.f;
    const int ntiles = batch / 16;
    const float scale = 2.f / (float)batch;
    for (int base = blockIdx.x * 4; base < ntiles; base += gridDim.x * 4) {
        const int tile = base + warp;
        const bool live = tile < ntiles;
        // ---- per-tile forward and backward (one warp per tile)
        if (live) {
            for (int e = lane; e < 16 * NI; e += 32) {
                const long long s = batch_sample(idx, tile, e / NI, pairs);
                act.x[e] = X[s * NI + e % NI];
            }
            __syncwarp();
            float z1[8][4], z2[8][4], y[4];
            forward_tile(sh.w, act, z1, z2, y);
            // dY = 2/B (Y - T) on columns 0..3 (rows g, g+8; columns 2t, 2t+1)
            float dy[4] = {0.f, 0.f, 0.f, 0.f};
            if (t < 2) {
                const long long s0 = batch_sample(idx, tile, g, pairs);
                const long long s8 = batch_sample(idx, tile, g + 8, pairs);
                const float r0 = y[0] - T[s0 * NO + 2 * t], r1 = y[1] - T[s0 * NO + 2 * t + 1];
                const float r2 = y[2] - T[s8 * NO + 2 * t], r3 = y[3] - T[s8 * NO + 2 * t + 1];
                if (pairs) {
                    const float d0 = r2 - r0, d1 = r3 - r1, u = 1.f - pw;
                    lsum += u * (r0 * r0 + r1 * r1 + r2 * r2 + r3 * r3) + pw * (d0 * d0 + d1 * d1);
                    dy[0] = scale * (u * r0 - pw * d0); dy[1] = scale * (u * r1 - pw * d1);
                    dy[2] = scale * (u * r2 + pw * d0); dy[3] = scale * (u * r3 + pw * d1);
                } else {
                    lsum += r0 * r0 + r1 * r1 + r2 * r2 + r3 * r3;
                    dy[0] = scale * r0; dy[1] = scale * r1; dy[2] = scale * r2; dy[3] = scale * r3;
                }
            }
            // dY as BF16 A operand [16 samples][16 outputs], columns >= 4 zero
            act.dy[g * 16 + 2 * t] = __float2bfloat16_rn(dy[0]);
            act.dy[g * 16 + 2 * t + 1] = __float2bfloat16_rn(dy[1]);
            act.dy[(g + 8) * 16 + 2 * t] = __float2bfloat16_rn(dy[2]);
            act.dy[(g + 8) * 16 + 2 * t + 1] = __float2bfloat16_rn(dy[3]);
            act.dy[g * 16 + 2 * t + 8] = __float2bfloat16_rn(0.f);
            act.dy[g * 16 + 2 * t + 9] = __float2bfloat16_rn(0.f);
            act.dy[(g + 8) * 16 + 2 * t + 8] = __float2bfloat16_rn(0.f);
            act.dy[(g + 8) * 16 + 2 * t + 9] = __float2bfloat16_rn(0.f);
            __syncwarp();
            unsigned a[4], b[2];
            // dH2 = dY W3  (K = outputs, padded to 16)
            float dh[8][4];
            load_a(a, act.dy, 16, 0, 0);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                dh[j][0] = dh[j][1] = dh[j][2] = dh[j][3] = 0.f;
                load_b_kn(b, sh.w.w3, NH, 8 * j, 0);
                mma(dh[j], a, b);
            }
            // dZ2 = dH2 * gelu'(Z2)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int c = 8 * j + 2 * t;
                float d0, d1, d2, d3;
                gelu(z2[j][0], &d0); gelu(z2[j][1], &d1); gelu(z2[j][2], &d2); gelu(z2[j][3], &d3);
                act.dz2[g * NH + c] = __float2bfloat16_rn(dh[j][0] * d0);
                act.dz2[g * NH + c + 1] = __float2bfloat16_rn(dh[j][1] * d1);
                act.dz2[(g + 8) * NH + c] = __float2bfloat16_rn(dh[j][2] * d2);
                act.dz2[(g + 8) * NH + c + 1] = __float2bfloat16_rn(dh[j][3] * d3);
            }
            __syncwarp();
            // dH1 = dZ2 W2  (K = hidden 2)
#pragma unroll
            for (int j = 0; j < 8; ++j) dh[j][0] = dh[j][1] = dh[j][2] = dh[j][3] = 0.f;
#pragma unroll
            for (int kb = 0; kb < 4; ++kb) {
                load_a(a, act.dz2, NH, 0, 16 * kb);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    load_b_kn(b, sh.w.w2, NH, 8 * j, 16 * kb);
                    mma(dh[j], a, b);
                }
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int c = 8 * j + 2 * t;
                float d0, d1, d2, d3;
                gelu(z1[j][0], &d0); gelu(z1[j][1], &d1); gelu(z1[j][2], &d2); gelu(z1[j][3], &d3);
                act.dz1[g * NH + c] = __float2bfloat16_rn(dh[j][0] * d0);
                act.dz1[g * NH + c + 1] = __float2bfloat16_rn(dh[j][1] * d1);
                act.dz1[(g + 8) * NH + c] = __float2bfloat16_rn(dh[j][2] * d2);
                act.dz1[(g + 8) * NH + c + 1] = __float2bfloat16_rn(dh[j][3] * d3);
            }
        }
        __syncthreads();
        // ---- weight gradients over the CTA's tiles: warp w owns rows
        // [16w, 16w+16) of dW2 and dW1 and columns [16w, 16w+16) of dW3
        for (int q = 0; q < 4; ++q) {
            if (base + q >= ntiles) break;
            const TileAct& at = sh.act[q];
            unsigned a[4], b[2];
            load_at(a, at.dz2, NH, 16 * warp, 0);  // A(h2, s) = dZ2[s][h2]
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                load_b_kn(b, at.h1, NH, 8 * j, 0);  // B(s, h1) = H1[s][h1]
                mma(acc2[j], a, b);
            }
            load_at(a, at.dz1, NH, 16 * warp, 0);  // A(h1, s) = dZ1[s][h1]
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                load_b_kn(b, at.x, NI, 8 * j, 0);  // B(s, i) = X[s][i]
                mma(acc1[j], a, b);
            }
            load_at(a, at.dy, 16, 0, 0);  // A(o, s) = dY[s][o]
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                load_b_kn(b, at.h2, NH, 16 * warp + 8 * j, 0);  // B(s, h2) = H2[s][h2]
                mma(acc3[j], a, b);
            }
            // bias gradients: column sums over the tile's samples
            if (lane < 16) {
                float s1 = 0.f, s2 = 0.f;
                for (int r = 0; r < 16; ++r) {
                    s1 += __bfloat162float(at.dz1[r * NH + 16 * warp + lane]);
                    s2 += __bfloat162float(at.dz2[r * NH + 16 * warp + lane]);
                }
                db1 += s1;
                db2 += s2;
            }
            if (warp == 0 && lane < NO) {
                float s3 = 0.f;
                for (int r = 0; r < 16; ++r) s3 += __bfloat162float(at.dy[r * 16 + lane]);
                db3 += s3;
            }
        }
        __syncthreads();
    }
    // ---- add this CTA's gradient to the batch gradient
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int r = 16 * warp + g, c = 8 * j + 2 * t;
        atomicAdd(&grad[W2O + r * NH + c], acc2[j][0]);
        atomicAdd(&grad[W2O + r * NH + c + 1], acc2[j][1]);
        atomicAdd(&grad[W2O + (r + 8) * NH + c], acc2[j][2]);
        atomicAdd(&grad[W2O + (r + 8) * NH + c + 1], acc2[j][3]);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int r = 16 * warp + g, c = 8 * j + 2 * t;
        atomicAdd(&grad[W1O + r * NI + c], acc1[j][0]);
        atomicAdd(&grad[W1O + r * NI + c + 1], acc1[j][1]);
        atomicAdd(&grad[W1O + (r + 8) * NI + c], acc1[j][2]);
        atomicAdd(&grad[W1O + (r + 8) * NI + c + 1], acc1[j][3]);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int c = 16 * warp + 8 * j + 2 * t;  // rows o = g (only o < 4 are outputs)
        if (g < NO) {
            atomicAdd(&grad[W3O + g * NH + c], acc3[j][0]);
            atomicAdd(&grad[W3O + g * NH + c + 1], acc3[j][1]);
        }
    }
    if (lane < 16) {
        atomicAdd(&grad[B1O + 16 * warp + lane], db1);
        atomicAdd(&grad[B2O + 16 * warp + lane], db2);
    }
    if (warp == 0 && lane < NO) atomicAdd(&grad[B3O + lane], db3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0 && loss) atomicAdd(loss, lsum);
}

// Batch of sample indices for one step: splitmix64 of (seed, step, i) mod n.
// In pair mode rows r and r + 8 of each 16-row tile draw the same pair m
// and take its members 2m and 2m + 1.
__global__ void k_batch_indices(long long* idx, int batch, long long n, unsigned long long seed,
                                long long step, int pairs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    const int r = i & 15;
    const long long key = pairs ? (long long)(i >> 4) * 8 + (r & 7) : i;
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(step * batch + key + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    idx[i] = pairs ? 2 * (long long)(z % (unsigned long long)(n / 2)) + (r >> 3)
                   : (long long)(z % (unsigned long long)n);
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; zeroes the gradient.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       float* __restrict__ grad, float lr, float b1, float b2, float eps, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAM) return;
    const float gr = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * gr;
    const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.f - powf(b1, (float)step));
    const float vh = vi / (1.f - powf(b2, (float)step));
    p[i] -= lr * mh / (sqrtf(vh) + eps);
    grad[i] = 0.f;
}

// Forward pass only, for checks: Y[n][4] (standardised outputs).
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ params,
                                                     const __nv_bfloat16* __restrict__ X,
                                                     long long n, float* __restrict__ Y) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainShared& sh = *reinterpret_cast<TrainShared*>(smem_raw);
    load_weights(sh.w, params);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    TileAct& act = sh.act[warp];
    const long long ntiles = (n + 15) / 16;
    for (long long tile = blockIdx.x * 4 + warp; tile < ntiles; tile += gridDim.x * 4) {
        for (int e = lane; e < 16 * NI; e += 32) {
            const long long s = tile * 16 + e / NI;
            act.x[e] = s < n ? X[s * NI + e % NI] : __float2bfloat16_rn(0.f);
        }
        __syncwarp();
        float z1[8][4], z2[8][4], y[4];
        forward_tile(sh.w, act, z1, z2, y);
        if (t < 2) {
            const long long s0 = tile * 16 + g, s8 = s0 + 8;
            if (s0 < n) { Y[s0 * NO + 2 * t] = y[0]; Y[s0 * NO + 2 * t + 1] = y[1]; }
            if (s8 < n) { Y[s8 * NO + 2 * t] = y[2]; Y[s8 * NO + 2 * t + 1] = y[3]; }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------ inference
// Adds the learned correction to the face fluxes of one direction of a 2D
// generic-path stage (F: FP64 face fluxes, W: FP64 primitives), after
// Flux::CalFlux formed them (cal_flux.cpp:89-121; no reference counterpart).  One warp
// per 16 faces.  The plain HLLC flux is kept where the detector fires (a
// pressure jump max(p)/min(p) > 1 + shock_jump over the stencil, or a
// correction that would move more than pos_frac of an adjacent cell's mass
// or internal energy through the face in one step) and in smooth flow (the
// stencil's total variation below tv_min); each component is clipped to
// diss_frac times the face's HLL dissipation (gk::FluxGate).  The fused 2D
// stage (gk_kernels.cuh) applies the same correction with the same
// functions (gk_learn.cuh), face by face.
struct InferShared {
    MlpWeights w;
    alignas(16) __nv_bfloat16 x[4][32 * NI];  // a warp's two tiles
    FaceScale fs[4][32];
};

__global__ void __launch_bounds__(128) k_flux_correct(const float* __restrict__ model,
                                                      const double* __restrict__ W,
                                                      double* __restrict__ F, gk::Geom g,
                                                      gk::Phys ph, const gk::DevTime* __restrict__ tm,
                                                      int dir, gk::FluxGate gate,
                                                      unsigned* __restrict__ fired) {
    if (!tm->active) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InferShared& sh = *reinterpret_cast<InferShared*>(smem_raw);
    load_weights(sh.w, model);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
    __nv_bfloat16* const x = sh.x[warp];
    const int nfx = dir == 0 ? g.nx + 1 : g.nx;       // faces per row
    const int nfy = dir == 0 ? g.ny : g.ny + 1;       // rows of faces
    const long long nfaces = (long long)nfx * nfy;
    const long long ntiles = (nfaces + 15) / 16;
    const double dtdx = tm->dt * (dir == 0 ? g.dxRec : g.dyRec);
    const int sn = dir == 0 ? gk::P_VX : gk::P_VY, st = dir == 0 ? gk::P_VY : gk::P_VX;
    const int mn = dir == 0 ? gk::S_MTX : gk::S_MTY, mt = dir == 0 ? gk::S_MTY : gk::S_MTX;
    // a warp takes two tiles at a time: lane L builds face 32 * pair + L
    const long long npairs = (ntiles + 1) / 2;
    for (long long pair = blockIdx.x * 4 + warp; pair < npairs; pair += gridDim.x * 4) {
        {
            const long long f = pair * 32 + lane;
            FaceScale& fs = sh.fs[warp][lane];
            if (f < nfaces) {
                const int fi = (int)(f % nfx), fj = (int)(f / nfx);
                const int i = g.ib + fi, j = g.jb + fj;  // face between cells (i-1|i) or (j-1|j)
                double r[4], vn[4], vt[4], p[4];
                for (int c = 0; c < 4; ++c) {
                    const int ii = dir == 0 ? i - 2 + c : i, jj = dir == 0 ? j : j - 2 + c;
                    const long long q = (long long)(g.kb - g.kofs) * g.kstride + (long long)jj * g.pitch + ii;
                    r[c] = W[gk::P_RHO * g.vstride + q];
                    vn[c] = W[sn * g.vstride + q];
                    vt[c] = W[st * g.vstride + q];
                    p[c] = W[gk::P_PRE * g.vstride + q];
                }
                face_inputs(r, vn, vt, p, ph.gamma, ph.gm1Rec, gate, sh.w.norm, x + lane * NI, fs);
            } else {
                for (int e = 0; e < NI; ++e) x[lane * NI + e] = __float2bfloat16_rn(0.f);
                fs.gate = 2.f;
            }
        }
        // tiles whose faces all keep plain HLLC (past the end, or smooth) skip the network
        const unsigned need = __ballot_sync(0xffffffffu, sh.fs[warp][lane].gate != 2.f);
        __syncwarp();
        if (!need) continue;
        float y2[2][4];
        forward_tiles<2>(sh.w, x, y2);
        for (int half16 = 0; half16 < 2; ++half16) {
            if (!((need >> (16 * half16)) & 0xffffu)) continue;
            const float (&y)[4] = y2[half16];
            // lane (gq, tq < 2) holds outputs 2tq, 2tq+1 of faces gq and gq+8;
            // its partner lane ^ 1 holds the face's other two outputs
            for (int half = 0; half < 2; ++half) {
                const int fl = 16 * half16 + gq + 8 * half;
                const long long f = pair * 32 + fl;
                const FaceScale& fs = sh.fs[warp][fl];
                const bool mine = tq < 2 && f < nfaces && fs.gate != 2.f;
                double corr[2] = {0.0, 0.0};
                if (mine)
                    for (int o2 = 0; o2 < 2; ++o2) corr[o2] = face_correction(y[2 * half + o2], 2 * tq + o2, fs, sh.w.norm);
                // lane tq = 0 holds mass (output 0), its partner energy (output 3);
                // every lane takes part in both exchanges
                const double p0 = __shfl_xor_sync(0xffffffffu, corr[0], 1);
                const double p1 = __shfl_xor_sync(0xffffffffu, corr[1], 1);
                const double c0 = tq == 0 ? corr[0] : p0;
                const double c3 = tq == 0 ? p1 : corr[1];
                const bool bad = mine && face_vetoed(c0, c3, dtdx, fs, gate);
                // one atomic per warp and half-tile for the faces left to plain HLLC
                const unsigned nbad = __ballot_sync(0xffffffffu, bad && tq == 0);
                if (lane == 0 && fired && nbad) atomicAdd(fired, (unsigned)__popc(nbad));
                if (!mine || bad) continue;
                const int fi = (int)(f % nfx), fj = (int)(f / nfx);
                const long long fc = (long long)(g.kb - g.kofs) * g.fkstride + (long long)(g.jb + fj) * g.fpitch + g.ib + fi;
                for (int o2 = 0; o2 < 2; ++o2) {
                    const int o = 2 * tq + o2;
                    const int slot = o == 0 ? gk::S_DEN : (o == 1 ? mn : (o == 2 ? mt : gk::S_ENG));
                    F[slot * g.fvstride + fc] += corr[o2];
                }
            }
        }
        __syncwarp();
    }
}

}  // namespace

// ------------------------------------------------------------ C ABI
extern "C" {

int gk_mlp_nparams(void) { return NPARAM; }
int gk_mlp_nmodel(void) { return NMODEL; }

struct gk_mlp {
    float* params = nullptr;  // FP32 master parameters + normalisation (NMODEL)
    float* m = nullptr;
    float* v = nullptr;
    float* grad = nullptr;
    float* loss = nullptr;
    long long* idx = nullptr;
    int idx_cap = 0;
    int step = 0;
    int pairs = 0;      // samples are neighbouring-face pairs (2m, 2m + 1)
    float pair_w = 0.f; // weight of the pair-difference term of the loss
    cudaStream_t stream = nullptr;
};

static size_t train_smem() { return sizeof(TrainShared); }

int gk_mlp_create(const float* model_host, gk_mlp** out) {
    if (!model_host || !out) return GK_ERR_INVALID;
    gk_mlp* M = new gk_mlp();
    cudaError_t e = cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&M->params, sizeof(float) * NMODEL);
    if (e == cudaSuccess) e = cudaMalloc(&M->m, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc(&M->v, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc(&M->grad, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc(&M->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(M->params, model_host, sizeof(float) * NMODEL, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(M->m, 0, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMemset(M->v, 0, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMemset(M->grad, 0, sizeof(float) * NPARAM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem());
    if (e != cudaSuccess) {
        std::fprintf(stderr, "gk_mlp_create: %s\n", cudaGetErrorString(e));
        gk_mlp_destroy(M);
        return GK_ERR_CUDA;
    }
    *out = M;
    return GK_OK;
}

void gk_mlp_destroy(gk_mlp* M) {
    if (!M) return;
    if (M->stream) cudaStreamSynchronize(M->stream);
    cudaFree(M->params);
    cudaFree(M->m);
    cudaFree(M->v);
    cudaFree(M->grad);
    cudaFree(M->loss);
    cudaFree(M->idx);
    if (M->stream) cudaStreamDestroy(M->stream);
    delete M;
}

int gk_mlp_get(gk_mlp* M, float* model_host) {
    if (!M || !model_host) return GK_ERR_INVALID;
    return cudaMemcpy(model_host, M->params, sizeof(float) * NMODEL, cudaMemcpyDeviceToHost) ==
                   cudaSuccess ? GK_OK : GK_ERR_CUDA;
}

// Batch gradient (sum over the batch of d(loss)/d(param), loss = mean over
// samples of the squared error summed over the 4 outputs), without
// updating; X: n x 16 BF16 device, T: n x 4 FP32 device; the first `batch`
// samples in order.  grad_host: NPARAM floats; loss_host: the summed squared
// error.
int gk_mlp_set_pair_loss(gk_mlp* M, float w) {
    if (!M || !(w <= 1.f)) return GK_ERR_INVALID;
    M->pairs = w >= 0.f;
    M->pair_w = w >= 0.f ? w : 0.f;
    return GK_OK;
}

int gk_mlp_grad(gk_mlp* M, const void* X, const float* T, long long n, int batch,
                float* grad_host, float* loss_host) {
    if (!M || !X || !T || batch <= 0 || batch % 16 || batch > n) return GK_ERR_INVALID;
    cudaMemsetAsync(M->grad, 0, sizeof(float) * NPARAM, M->stream);
    cudaMemsetAsync(M->loss, 0, sizeof(float), M->stream);
    const int ctas = (batch / 16 + 3) / 4 < 148 * 4 ? (batch / 16 + 3) / 4 : 148 * 4;
    k_mlp_grad<<<ctas, 128, train_smem(), M->stream>>>(M->params, (const __nv_bfloat16*)X, T, n,
                                                       nullptr, batch, M->grad, M->loss, M->pairs,
                                                       M->pair_w);
    if (cudaGetLastError() != cudaSuccess) return GK_ERR_CUDA;
    if (grad_host && cudaMemcpyAsync(grad_host, M->grad, sizeof(float) * NPARAM,
                                     cudaMemcpyDeviceToHost, M->stream) != cudaSuccess)
        return GK_ERR_CUDA;
    if (loss_host && cudaMemcpyAsync(loss_host, M->loss, sizeof(float), cudaMemcpyDeviceToHost,
                                     M->stream) != cudaSuccess)
        return GK_ERR_CUDA;
    cudaMemsetAsync(M->grad, 0, sizeof(float) * NPARAM, M->stream);
    return cudaStreamSynchronize(M->stream) == cudaSuccess ? GK_OK : GK_ERR_CUDA;
}

// `steps` Adam steps on batches of `batch` samples drawn with replacement
// (counter-based, seed) from X (n x 16 BF16) / T (n x 4 FP32), both on the
// device.  loss_host (may be NULL): mean squared error per sample of the last
// step.
int gk_mlp_train(gk_mlp* M, const void* X, const float* T, long long n, int batch, int steps,
                 float lr, unsigned long long seed, float* loss_host) {
    if (!M || !X || !T || batch <= 0 || batch % 16 || n <= 0 || steps < 0) return GK_ERR_INVALID;
    if (M->pairs && (n < 2 || n % 2)) return GK_ERR_INVALID;
    if (M->idx_cap < batch) {
        cudaFree(M->idx);
        if (cudaMalloc(&M->idx, sizeof(long long) * batch) != cudaSuccess) return GK_ERR_CUDA;
        M->idx_cap = batch;
    }
    const int ctas = (batch / 16 + 3) / 4 < 148 * 4 ? (batch / 16 + 3) / 4 : 148 * 4;
    for (int s = 0; s < steps; ++s) {
        ++M->step;
        k_batch_indices<<<(batch + 255) / 256, 256, 0, M->stream>>>(M->idx, batch, n, seed, M->step,
                                                                    M->pairs);
        if (s == steps - 1) cudaMemsetAsync(M->loss, 0, sizeof(float), M->stream);
        k_mlp_grad<<<ctas, 128, train_smem(), M->stream>>>(
            M->params, (const __nv_bfloat16*)X, T, n, M->idx, batch, M->grad,
            s == steps - 1 ? M->loss : nullptr, M->pairs, M->pair_w);
        k_adam<<<(NPARAM + 255) / 256, 256, 0, M->stream>>>(M->params, M->m, M->v, M->grad, lr,
                                                            0.9f, 0.999f, 1e-8f, M->step);
    }
    if (cudaGetLastError() != cudaSuccess) return GK_ERR_CUDA;
    if (loss_host) {
        float l = 0.f;
        if (cudaMemcpyAsync(&l, M->loss, sizeof(float), cudaMemcpyDeviceToHost, M->stream) != cudaSuccess)
            return GK_ERR_CUDA;
        if (cudaStreamSynchronize(M->stream) != cudaSuccess) return GK_ERR_CUDA;
        *loss_host = l / (float)batch;
    }
    return cudaStreamSynchronize(M->stream) == cudaSuccess ? GK_OK : GK_ERR_CUDA;
}

// Standardised outputs for n samples of X (device), into Y (device, n x 4).
int gk_mlp_forward(gk_mlp* M, const void* X, long long n, float* Y) {
    if (!M || !X || !Y || n <= 0) return GK_ERR_INVALID;
    const long long tiles = (n + 15) / 16;
    const int ctas = (int)((tiles + 3) / 4 < 148 * 4 ? (tiles + 3) / 4 : 148 * 4);
    k_mlp_forward<<<ctas, 128, train_smem(), M->stream>>>(M->params, (const __nv_bfloat16*)X, n, Y);
    return cudaStreamSynchronize(M->stream) == cudaSuccess ? GK_OK : GK_ERR_CUDA;
}

}  // extern "C"

// Used by gk_api.cu: the correction pass of one direction.
namespace gk {
size_t flux_correct_smem() { return sizeof(InferShared); }
void launch_flux_correct(const float* model, const double* W, double* F, const Geom& g,
                         const Phys& ph, const DevTime* tm, int dir, const FluxGate& gate,
                         unsigned* fired, cudaStream_t s) {
    static std::atomic<unsigned long long> attr{0};
    if (gk::first_on_device(attr))
        cudaFuncSetAttribute(k_flux_correct, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(InferShared));
    const long long nf = dir == 0 ? (long long)(g.nx + 1) * g.ny : (long long)g.nx * (g.ny + 1);
    const long long pairs = ((nf + 15) / 16 + 1) / 2;
    const int ctas = (int)((pairs + 3) / 4 < 148 * 8 ? (pairs + 3) / 4 : 148 * 8);
    k_flux_correct<<<ctas, 128, sizeof(InferShared), s>>>(model, W, F, g, ph, tm, dir, gate,
                                                           fired);
}
}  // namespace gk
