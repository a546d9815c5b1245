// Learned surrogate of the SNAP energy: an MLP on per-atom 2J=4 bispectra.
//
// There is no counterpart in MDP.  The network is E_i = e_mu + e_sd * y(x_i),
// x_i = (B_i - mu) * sinv (the 14 components of the 2J=4 bispectrum of atom
// i, cpuSnap4.cpp:427-592 ordering), y = w3 . silu(W2 silu(W1 x + b1) + b2) + b3
// with 64 hidden units per layer.  Forward passes use the weights rounded to
// BF16; sums are FP32.  The master weights, gradients and Adam moments are FP32.
//
// Forces: E_i depends on the positions only through U_i, so
//   dE/dr = sum_i sum_k (dE_i/dB_ik) dB_ik/dr,
// which is the linear-SNAP force with per-atom coefficients G_ik = dE_i/dB_ik:
// the inference kernel writes G, the Y kernel takes it in place of beta (its
// per-atom mode) and the dE/dr and tally kernels run unchanged at 2J=4.
#include "common.cuh"
#include "engine.h"
#include "surrogate.h"
#include "fit.h"

#include <cuda_bf16.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <vector>

namespace mdp {

// ---------------------------------------------------------------------------
// network arithmetic
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sur_sigmoid(float z) { return 1.0f / (1.0f + __expf(-z)); }
__device__ __forceinline__ float sur_silu(float z) { return z * sur_sigmoid(z); }
__device__ __forceinline__ float sur_dsilu(float z)
{
    const float s = sur_sigmoid(z);
    return s * (1.0f + z * (1.0f - s));
}

// forward of one sample: z1, a1 = silu(z1), z2 and y; W points at the
// (BF16-rounded) parameter block in shared memory
__device__ __forceinline__ float mlp_forward(const float *__restrict__ W, const float (&x)[SUR_KP], float (&z1)[SUR_H],
                                             float (&a1)[SUR_H], float (&z2)[SUR_H])
{
#pragma unroll 4
    for (int r = 0; r < SUR_H; r++) {
        float s = W[SUR_OFF_B1 + r];
#pragma unroll
        for (int k = 0; k < SUR_NK; k++) s += W[SUR_OFF_W1 + r * SUR_KP + k] * x[k];
        z1[r] = s;
        a1[r] = sur_silu(s);
    }
    float y = W[SUR_OFF_B3];
#pragma unroll 2
    for (int c = 0; c < SUR_H; c++) {
        float s = W[SUR_OFF_B2 + c];
#pragma unroll
        for (int r = 0; r < SUR_H; r++) s += W[SUR_OFF_W2 + c * SUR_H + r] * a1[r];
        z2[c] = s;
        y += W[SUR_OFF_W3 + c] * sur_silu(s);
    }
    return y;
}

// dy/dz1 given z1, z2 (g1 out), via dy/dz2 = w3 * silu'(z2)
__device__ __forceinline__ void mlp_backward_z1(const float *__restrict__ W, const float (&z1)[SUR_H],
                                                float (&z2g)[SUR_H], float (&g1)[SUR_H])
{
#pragma unroll
    for (int c = 0; c < SUR_H; c++) z2g[c] = W[SUR_OFF_W3 + c] * sur_dsilu(z2g[c]);
#pragma unroll 4
    for (int r = 0; r < SUR_H; r++) {
        float s = 0.f;
#pragma unroll
        for (int c = 0; c < SUR_H; c++) s += W[SUR_OFF_W2 + c * SUR_H + r] * z2g[c];
        g1[r] = s * sur_dsilu(z1[r]);
    }
}

// BF16 rounding of the weights used by every forward pass (biases stay FP32)
__host__ __device__ inline bool sur_is_weight(int i)
{
    return (i >= SUR_OFF_W1 && i < SUR_OFF_B1) || (i >= SUR_OFF_W2 && i < SUR_OFF_B2) ||
           (i >= SUR_OFF_W3 && i < SUR_OFF_B3);
}

__global__ void k_sur_round(const float *__restrict__ P, float *__restrict__ Pb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < SUR_NPAR) Pb[i] = sur_is_weight(i) ? __bfloat162float(__float2bfloat16_rn(P[i])) : P[i];
}

// ---------------------------------------------------------------------------
// inference on tensor cores: each warp takes 16 atoms per tile through
// mma.sync m16n8k16 (BF16 x BF16 -> FP32).  Weights are BF16 already; every
// activation operand is split into BF16 hi + lo (two MMAs), so products keep
// about 16 bits and the energy stays a smooth function of the features, in
// step with its gradient G.  A layer's FP32 accumulators (C fragments) become
// the next layer's A fragments in registers.  The backward pass uses
// transposed weight copies so every B fragment is two adjacent BF16 values.
// ---------------------------------------------------------------------------
constexpr int SUR_TC_WARPS = 4;

__device__ __forceinline__ unsigned sur_bits(__nv_bfloat162 v) { return *reinterpret_cast<unsigned *>(&v); }

// (x0, x1) -> packed BF16 hi and lo parts (x0 in the low half)
__device__ __forceinline__ void sur_split2(float x0, float x1, unsigned &h, unsigned &l)
{
    const __nv_bfloat162 hv = __floats2bfloat162_rn(x0, x1);
    const float2 hf = __bfloat1622float2(hv);
    h = sur_bits(hv);
    l = sur_bits(__floats2bfloat162_rn(x0 - hf.x, x1 - hf.y));
}

__device__ __forceinline__ void sur_mma(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A fragments (hi, lo) of k-step kk from C fragments of column tiles 2kk, 2kk+1
__device__ __forceinline__ void sur_afrag(const float (&c)[8][4], int kk, unsigned (&h)[4], unsigned (&l)[4])
{
    sur_split2(c[2 * kk][0], c[2 * kk][1], h[0], l[0]);
    sur_split2(c[2 * kk][2], c[2 * kk][3], h[1], l[1]);
    sur_split2(c[2 * kk + 1][0], c[2 * kk + 1][1], h[2], l[2]);
    sur_split2(c[2 * kk + 1][2], c[2 * kk + 1][3], h[3], l[3]);
}

__global__ void __launch_bounds__(SUR_TC_WARPS * 32)
k_sur_infer_tc(const double *__restrict__ B, long bstride, int n, const float *__restrict__ Pb, const SurNorm nrm,
               double *__restrict__ eatom, float *__restrict__ G)
{
    __shared__ __align__(16) __nv_bfloat16 W1s[SUR_H * SUR_KP], W1t[SUR_KP * SUR_H], W2s[SUR_H * SUR_H],
        W2t[SUR_H * SUR_H];
    __shared__ float sb1[SUR_H], sb2[SUR_H], sw3[SUR_H];
    for (int i = threadIdx.x; i < SUR_H * SUR_KP; i += blockDim.x) {
        const int r = i / SUR_KP, k = i % SUR_KP;
        const __nv_bfloat16 v = __float2bfloat16_rn(Pb[SUR_OFF_W1 + i]);
        W1s[i] = v;
        W1t[k * SUR_H + r] = v;
    }
    for (int i = threadIdx.x; i < SUR_H * SUR_H; i += blockDim.x) {
        const int c = i / SUR_H, r = i % SUR_H;
        const __nv_bfloat16 v = __float2bfloat16_rn(Pb[SUR_OFF_W2 + i]);
        W2s[i] = v;
        W2t[r * SUR_H + c] = v;
    }
    for (int i = threadIdx.x; i < SUR_H; i += blockDim.x) {
        sb1[i] = Pb[SUR_OFF_B1 + i]; sb2[i] = Pb[SUR_OFF_B2 + i]; sw3[i] = Pb[SUR_OFF_W3 + i];
    }
    __syncthreads();
    const float b3 = Pb[SUR_OFF_B3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, tq = lane & 3;
    const int ntile = (n + 15) / 16;
    auto wpair = [](const __nv_bfloat16 *p) { return *reinterpret_cast<const unsigned *>(p); };
    for (int tile = blockIdx.x * SUR_TC_WARPS + w; tile < ntile; tile += gridDim.x * SUR_TC_WARPS) {
        const int a0 = tile * 16 + g, a1 = a0 + 8;
        // input fragment: rows g, g+8 (atoms), columns 2tq, 2tq+1, 2tq+8, 2tq+9 (features)
        float xv[2][4];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int a = h ? a1 : a0;
            const int ks[4] = {2 * tq, 2 * tq + 1, 2 * tq + 8, 2 * tq + 9};
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int k = ks[q];
                xv[h][q] = (a < n && k < SUR_NK) ? (float)((B[(size_t)k * bstride + a] - nrm.mu[k]) * nrm.sinv[k]) : 0.f;
            }
        }
        unsigned xh[4], xl[4];
        sur_split2(xv[0][0], xv[0][1], xh[0], xl[0]);
        sur_split2(xv[1][0], xv[1][1], xh[1], xl[1]);
        sur_split2(xv[0][2], xv[0][3], xh[2], xl[2]);
        sur_split2(xv[1][2], xv[1][3], xh[3], xl[3]);
        // layer 1: z1 = x W1^T + b1
        float z1[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const int nn = 8 * nt + 2 * tq;
            z1[nt][0] = sb1[nn]; z1[nt][1] = sb1[nn + 1]; z1[nt][2] = sb1[nn]; z1[nt][3] = sb1[nn + 1];
            const unsigned b0 = wpair(&W1s[(8 * nt + g) * SUR_KP + 2 * tq]), bb1 = wpair(&W1s[(8 * nt + g) * SUR_KP + 2 * tq + 8]);
            sur_mma(z1[nt], xh, b0, bb1);
            sur_mma(z1[nt], xl, b0, bb1);
        }
        // layer 2: z2 = silu(z1) W2^T + b2
        float a1f[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) a1f[nt][q] = sur_silu(z1[nt][q]);
        float z2[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const int nn = 8 * nt + 2 * tq;
            z2[nt][0] = sb2[nn]; z2[nt][1] = sb2[nn + 1]; z2[nt][2] = sb2[nn]; z2[nt][3] = sb2[nn + 1];
        }
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            unsigned ah[4], al[4];
            sur_afrag(a1f, kk, ah, al);
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const __nv_bfloat16 *wr = &W2s[(8 * nt + g) * SUR_H + 16 * kk + 2 * tq];
                const unsigned b0 = wpair(wr), bb1 = wpair(wr + 8);
                sur_mma(z2[nt], ah, b0, bb1);
                sur_mma(z2[nt], al, b0, bb1);
            }
        }
        // output and dy/dz2 = w3 * silu'(z2)
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const int nn = 8 * nt + 2 * tq;
            y0 += sw3[nn] * sur_silu(z2[nt][0]) + sw3[nn + 1] * sur_silu(z2[nt][1]);
            y1 += sw3[nn] * sur_silu(z2[nt][2]) + sw3[nn + 1] * sur_silu(z2[nt][3]);
            z2[nt][0] = sw3[nn] * sur_dsilu(z2[nt][0]);
            z2[nt][1] = sw3[nn + 1] * sur_dsilu(z2[nt][1]);
            z2[nt][2] = sw3[nn] * sur_dsilu(z2[nt][2]);
            z2[nt][3] = sw3[nn + 1] * sur_dsilu(z2[nt][3]);
        }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1); y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1); y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        if (tq == 0 && eatom) {
            if (a0 < n) eatom[a0] = (double)nrm.e_mu + (double)nrm.e_sd * (double)(y0 + b3);
            if (a1 < n) eatom[a1] = (double)nrm.e_mu + (double)nrm.e_sd * (double)(y1 + b3);
        }
        // dy/dh1 = (dy/dz2) W2, then dy/dz1 = dy/dh1 * silu'(z1)
        float g1[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) g1[nt][q] = 0.f;
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            unsigned ah[4], al[4];
            sur_afrag(z2, kk, ah, al);
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const __nv_bfloat16 *wr = &W2t[(8 * nt + g) * SUR_H + 16 * kk + 2 * tq];
                const unsigned b0 = wpair(wr), bb1 = wpair(wr + 8);
                sur_mma(g1[nt], ah, b0, bb1);
                sur_mma(g1[nt], al, b0, bb1);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) g1[nt][q] *= sur_dsilu(z1[nt][q]);
        // dy/dx = (dy/dz1) W1
        float gx[2][4];
#pragma unroll
        for (int nt = 0; nt < 2; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) gx[nt][q] = 0.f;
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            unsigned ah[4], al[4];
            sur_afrag(g1, kk, ah, al);
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const __nv_bfloat16 *wr = &W1t[(8 * nt + g) * SUR_H + 16 * kk + 2 * tq];
                const unsigned b0 = wpair(wr), bb1 = wpair(wr + 8);
                sur_mma(gx[nt], ah, b0, bb1);
                sur_mma(gx[nt], al, b0, bb1);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 2; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int k = 8 * nt + 2 * tq + (q & 1);
                const int a = (q < 2) ? a0 : a1;
                if (k < SUR_NK && a < n) G[(size_t)k * n + a] = gx[nt][q] * (float)(nrm.sinv[k] * nrm.e_sd);
            }
    }
}

// ---------------------------------------------------------------------------
// training gradient of the energy loss L = mean_s (y_s - t_s)^2, t = (E - e_mu)/e_sd
// One sample per thread; the block's per-sample vectors go to shared memory
// and each thread then sums one output row of dW1/dW2 over the block's samples,
// so global memory sees one atomic add per parameter per block.
// ---------------------------------------------------------------------------
constexpr int SUR_TR_THREADS = 64;
constexpr size_t SUR_TR_SMEM =
    sizeof(float) * (SUR_NPAR + SUR_TR_THREADS * (SUR_KP + 1) + 4 * SUR_TR_THREADS * (SUR_H + 1) + SUR_TR_THREADS);

__global__ void __launch_bounds__(SUR_TR_THREADS)
k_sur_grad(const float *__restrict__ X, const float *__restrict__ E, const int *__restrict__ idx, int nb,
           const float *__restrict__ Pb, const SurNorm nrm, float *__restrict__ grad, float *__restrict__ loss)
{
    extern __shared__ float sur_sm[];
    float *W = sur_sm;
    typedef float RowK[SUR_KP + 1];
    typedef float RowH[SUR_H + 1];
    RowK *sx = reinterpret_cast<RowK *>(W + SUR_NPAR);
    RowH *sa1 = reinterpret_cast<RowH *>(sx + SUR_TR_THREADS);
    RowH *sg1 = sa1 + SUR_TR_THREADS;
    RowH *sa2 = sg1 + SUR_TR_THREADS;
    RowH *sg2 = sa2 + SUR_TR_THREADS;
    float *sdy = reinterpret_cast<float *>(sg2 + SUR_TR_THREADS);
    for (int i = threadIdx.x; i < SUR_NPAR; i += blockDim.x) W[i] = Pb[i];
    __syncthreads();
    const int t = threadIdx.x;
    const int s = blockIdx.x * SUR_TR_THREADS + t;
    float x[SUR_KP];
    float z1[SUR_H], a1[SUR_H], z2[SUR_H], g1[SUR_H];
    float dy = 0.f;
    if (s < nb) {
        const int row = idx[s];
#pragma unroll
        for (int k = 0; k < SUR_KP; k++) x[k] = k < SUR_NK ? (X[(size_t)row * SUR_KP + k] - nrm.mu[k]) * nrm.sinv[k] : 0.f;
        const float y = mlp_forward(W, x, z1, a1, z2);
        const float r = y - (E[row] - nrm.e_mu) / nrm.e_sd;
        dy = 2.0f * r / (float)nb;
        atomicAdd(loss, r * r / (float)nb);
#pragma unroll
        for (int c = 0; c < SUR_H; c++) sa2[t][c] = sur_silu(z2[c]);
        mlp_backward_z1(W, z1, z2, g1);   // z2 <- w3 * silu'(z2), g1 = dy/dz1 per unit dy
#pragma unroll
        for (int c = 0; c < SUR_H; c++) { sg2[t][c] = dy * z2[c]; sg1[t][c] = dy * g1[c]; sa1[t][c] = a1[c]; }
#pragma unroll
        for (int k = 0; k < SUR_KP; k++) sx[t][k] = x[k];
    } else {
#pragma unroll
        for (int c = 0; c < SUR_H; c++) { sg2[t][c] = 0.f; sg1[t][c] = 0.f; sa1[t][c] = 0.f; sa2[t][c] = 0.f; }
#pragma unroll
        for (int k = 0; k < SUR_KP; k++) sx[t][k] = 0.f;
    }
    sdy[t] = dy;
    __syncthreads();
    const int ns = min(SUR_TR_THREADS, nb - blockIdx.x * SUR_TR_THREADS);
    // row t of every weight matrix (SUR_H == SUR_TR_THREADS)
    {
        float w2[SUR_H];
#pragma unroll
        for (int r = 0; r < SUR_H; r++) w2[r] = 0.f;
        float b2 = 0.f, w3 = 0.f, b1 = 0.f, w1[SUR_KP];
#pragma unroll
        for (int k = 0; k < SUR_KP; k++) w1[k] = 0.f;
        for (int q = 0; q < ns; q++) {
            const float g2 = sg2[q][t], gg1 = sg1[q][t];
#pragma unroll
            for (int r = 0; r < SUR_H; r++) w2[r] += g2 * sa1[q][r];
            b2 += g2;
            w3 += sdy[q] * sa2[q][t];
            b1 += gg1;
#pragma unroll
            for (int k = 0; k < SUR_KP; k++) w1[k] += gg1 * sx[q][k];
        }
#pragma unroll
        for (int r = 0; r < SUR_H; r++) atomicAdd(&grad[SUR_OFF_W2 + t * SUR_H + r], w2[r]);
#pragma unroll
        for (int k = 0; k < SUR_NK; k++) atomicAdd(&grad[SUR_OFF_W1 + t * SUR_KP + k], w1[k]);
        atomicAdd(&grad[SUR_OFF_B2 + t], b2);
        atomicAdd(&grad[SUR_OFF_W3 + t], w3);
        atomicAdd(&grad[SUR_OFF_B1 + t], b1);
        if (t == 0) {
            float b3 = 0.f;
            for (int q = 0; q < ns; q++) b3 += sdy[q];
            atomicAdd(&grad[SUR_OFF_B3], b3);
        }
    }
}

// ---------------------------------------------------------------------------
// force matching.  With G_i = dE_i/dB_i, F_a = -sum_i G_i . dB_i/dx_a, and for
// the loss L_F = alpha |F - F_ref|^2 / (3 n var_F) the adjoint of G_i is
//   lambda_i = dL/dG_i = -sum_(own pairs p of i) dB_i/dr_p . (Q_j(p) - Q_i),
//   Q_a = dL/dF_a.
// Since G_ik = e_sd sinv_k dy/dx_k, the weight gradient of the force loss is
// d(grad_x y . v)/dw with v_k = lambda_ik e_sd sinv_k: forward-over-reverse
// through the network (tangent pass along v, then adjoints of both passes).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sur_d2silu(float z)
{
    const float s = sur_sigmoid(z);
    return s * (1.0f - s) * (2.0f + z * (1.0f - 2.0f * s));
}

// per atom a of the batch [a_lo, a_lo + n): predicted force, Q_a and the loss
__global__ void k_sur_fpred(int a_lo, int n, const int *__restrict__ poff, const int *__restrict__ roff,
                            const int *__restrict__ rlist, const int2 *__restrict__ pinfo,
                            const float *__restrict__ db, const float *__restrict__ G, const float *__restrict__ Fref,
                            float coef, float lw, float *__restrict__ Q, float *__restrict__ loss)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int a = a_lo + t;
    float de[3] = {0.f, 0.f, 0.f};
    for (int q = roff[a]; q < roff[a + 1]; q++) {
        const int p = rlist[q];
        const int i = pinfo[p].x - a_lo;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < SUR_NK; k++) s += G[(size_t)k * n + i] * db[((size_t)p * 3 + c) * SUR_NK + k];
            de[c] += s;
        }
    }
    for (int p = poff[a]; p < poff[a + 1]; p++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < SUR_NK; k++) s += G[(size_t)k * n + t] * db[((size_t)p * 3 + c) * SUR_NK + k];
            de[c] -= s;
        }
    float l = 0.f;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float r = -de[c] - Fref[3 * (size_t)a + c];
        Q[3 * t + c] = coef * r;
        l += r * r;
    }
    atomicAdd(loss, lw * l);
}

// lambda_i, written as the tangent v_ik = lambda_ik e_sd sinv_k ([atom][KP])
__global__ void k_sur_lambda(int a_lo, int n, const int *__restrict__ poff, const int2 *__restrict__ pinfo,
                             const float *__restrict__ db, const float *__restrict__ Q, const SurNorm nrm,
                             float *__restrict__ V)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int a = a_lo + t;
    float lam[SUR_NK];
#pragma unroll
    for (int k = 0; k < SUR_NK; k++) lam[k] = 0.f;
    const float qi0 = Q[3 * t], qi1 = Q[3 * t + 1], qi2 = Q[3 * t + 2];
    for (int p = poff[a]; p < poff[a + 1]; p++) {
        const int j = pinfo[p].y - a_lo;
        const float d0 = Q[3 * j] - qi0, d1 = Q[3 * j + 1] - qi1, d2 = Q[3 * j + 2] - qi2;
        const float *b = db + (size_t)p * 3 * SUR_NK;
#pragma unroll
        for (int k = 0; k < SUR_NK; k++) lam[k] -= b[k] * d0 + b[SUR_NK + k] * d1 + b[2 * SUR_NK + k] * d2;
    }
#pragma unroll
    for (int k = 0; k < SUR_KP; k++) V[(size_t)t * SUR_KP + k] = k < SUR_NK ? lam[k] * nrm.e_sd * nrm.sinv[k] : 0.f;
}

// energy + force gradient of the batch: one sample per thread, block-reduced
// rows of dW1 / dW2 (as k_sur_grad), with the tangent terms of the force part
constexpr int SUR_TF_THREADS = 64;
constexpr int SUR_TF_VEC = 8 * (SUR_H + 1) + 2 * (SUR_KP + 1) + 1;   // floats per sample in shared memory
constexpr size_t SUR_TF_SMEM = sizeof(float) * (SUR_NPAR + (size_t)SUR_TF_THREADS * SUR_TF_VEC);

__global__ void __launch_bounds__(SUR_TF_THREADS)
k_sur_grad_f(const double *__restrict__ B, long bstride, const float *__restrict__ E, const float *__restrict__ V,
             int n, float ew, const float *__restrict__ Pb, const SurNorm nrm, float *__restrict__ grad,
             float *__restrict__ loss)
{
    extern __shared__ float sf_sm[];
    float *W = sf_sm;
    for (int i = threadIdx.x; i < SUR_NPAR; i += blockDim.x) W[i] = Pb[i];
    float *base = W + SUR_NPAR;
    const int t = threadIdx.x, s = blockIdx.x * SUR_TF_THREADS + t;
    // per-sample vectors: 0 z2bar, 1 a1, 2 zd2bar, 3 ad1, 4 z1bar, 5 zd1bar, 6 a2, 7 ad2 (H+1 each),
    // then x, v (KP+1 each), then ybar
    auto vec = [&](int q, int who) { return base + (size_t)who * SUR_TF_VEC + q * (SUR_H + 1); };
    auto xv = [&](int q, int who) { return base + (size_t)who * SUR_TF_VEC + 8 * (SUR_H + 1) + q * (SUR_KP + 1); };
    __syncthreads();
    float *z2b = vec(0, t), *a1s = vec(1, t), *zd2b = vec(2, t), *ad1s = vec(3, t), *z1b = vec(4, t),
          *zd1b = vec(5, t), *a2s = vec(6, t), *ad2s = vec(7, t), *xs = xv(0, t), *vs = xv(1, t);
    float *ybs = base + (size_t)t * SUR_TF_VEC + 8 * (SUR_H + 1) + 2 * (SUR_KP + 1);
    if (s < n) {
        float x[SUR_KP], v[SUR_KP];
#pragma unroll
        for (int k = 0; k < SUR_KP; k++) {
            x[k] = k < SUR_NK ? (float)((B[(size_t)k * bstride + s] - nrm.mu[k]) * nrm.sinv[k]) : 0.f;
            v[k] = V[(size_t)s * SUR_KP + k];
            xs[k] = x[k];
            vs[k] = v[k];
        }
        // forward and tangent: z1 -> z1b (temporarily), zd1 -> zd1b, a1, ad1
        for (int r = 0; r < SUR_H; r++) {
            float z = W[SUR_OFF_B1 + r], zd = 0.f;
#pragma unroll
            for (int k = 0; k < SUR_NK; k++) { z += W[SUR_OFF_W1 + r * SUR_KP + k] * x[k]; zd += W[SUR_OFF_W1 + r * SUR_KP + k] * v[k]; }
            z1b[r] = z;
            zd1b[r] = zd;
            a1s[r] = sur_silu(z);
            ad1s[r] = sur_dsilu(z) * zd;
        }
        float y = W[SUR_OFF_B3];
        for (int c = 0; c < SUR_H; c++) {
            float z = W[SUR_OFF_B2 + c], zd = 0.f;
            for (int r = 0; r < SUR_H; r++) { z += W[SUR_OFF_W2 + c * SUR_H + r] * a1s[r]; zd += W[SUR_OFF_W2 + c * SUR_H + r] * ad1s[r]; }
            z2b[c] = z;      // z2 for now
            zd2b[c] = zd;    // zd2 for now
            a2s[c] = sur_silu(z);
            ad2s[c] = sur_dsilu(z) * zd;
            y += W[SUR_OFF_W3 + c] * a2s[c];
        }
        const float r = y - (E[s] - nrm.e_mu) / nrm.e_sd;
        const float yb = ew * 2.0f * r / (float)n;
        atomicAdd(loss, ew * r * r / (float)n);
        *ybs = yb;
        // adjoints of layer 2 (the force part has ydot-bar = 1)
        for (int c = 0; c < SUR_H; c++) {
            const float w3 = W[SUR_OFF_W3 + c], z = z2b[c], zd = zd2b[c];
            z2b[c] = yb * w3 * sur_dsilu(z) + w3 * sur_d2silu(z) * zd;
            zd2b[c] = w3 * sur_dsilu(z);
        }
        // adjoints of layer 1
        for (int r = 0; r < SUR_H; r++) {
            float ab = 0.f, adb = 0.f;
            for (int c = 0; c < SUR_H; c++) { ab += W[SUR_OFF_W2 + c * SUR_H + r] * z2b[c]; adb += W[SUR_OFF_W2 + c * SUR_H + r] * zd2b[c]; }
            const float z = z1b[r], zd = zd1b[r];
            z1b[r] = ab * sur_dsilu(z) + adb * sur_d2silu(z) * zd;
            zd1b[r] = adb * sur_dsilu(z);
        }
    } else {
        for (int q = 0; q < 8 * (SUR_H + 1) + 2 * (SUR_KP + 1); q++) base[(size_t)t * SUR_TF_VEC + q] = 0.f;
        *ybs = 0.f;
    }
    __syncthreads();
    const int ns = min(SUR_TF_THREADS, n - (int)blockIdx.x * SUR_TF_THREADS);
    // row t of each weight matrix over the block's samples
    float w2[SUR_H];
#pragma unroll
    for (int r = 0; r < SUR_H; r++) w2[r] = 0.f;
    float w1[SUR_KP];
#pragma unroll
    for (int k = 0; k < SUR_KP; k++) w1[k] = 0.f;
    float b2 = 0.f, b1 = 0.f, w3 = 0.f, b3 = 0.f;
    for (int q = 0; q < ns; q++) {
        const float gz2 = vec(0, q)[t], gzd2 = vec(2, q)[t], gz1 = vec(4, q)[t], gzd1 = vec(5, q)[t];
        const float *qa1 = vec(1, q), *qad1 = vec(3, q), *qx = xv(0, q), *qv = xv(1, q);
#pragma unroll
        for (int r = 0; r < SUR_H; r++) w2[r] += gz2 * qa1[r] + gzd2 * qad1[r];
#pragma unroll
        for (int k = 0; k < SUR_KP; k++) w1[k] += gz1 * qx[k] + gzd1 * qv[k];
        b2 += gz2;
        b1 += gz1;
        const float yb = base[(size_t)q * SUR_TF_VEC + 8 * (SUR_H + 1) + 2 * (SUR_KP + 1)];
        w3 += yb * vec(6, q)[t] + vec(7, q)[t];
        b3 += yb;
    }
#pragma unroll
    for (int r = 0; r < SUR_H; r++) atomicAdd(&grad[SUR_OFF_W2 + t * SUR_H + r], w2[r]);
#pragma unroll
    for (int k = 0; k < SUR_NK; k++) atomicAdd(&grad[SUR_OFF_W1 + t * SUR_KP + k], w1[k]);
    atomicAdd(&grad[SUR_OFF_B2 + t], b2);
    atomicAdd(&grad[SUR_OFF_B1 + t], b1);
    atomicAdd(&grad[SUR_OFF_W3 + t], w3);
    if (t == 0) atomicAdd(&grad[SUR_OFF_B3], b3);
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; also refreshes the
// BF16-rounded copy and clears the gradient
__global__ void k_sur_adam(float *__restrict__ P, float *__restrict__ Pb, float *__restrict__ grad,
                           float *__restrict__ m1, float *__restrict__ m2, float lr, float b1, float b2, float eps,
                           float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= SUR_NPAR) return;
    const float g = grad[i];
    const float m = b1 * m1[i] + (1.f - b1) * g;
    const float v = b2 * m2[i] + (1.f - b2) * g * g;
    m1[i] = m;
    m2[i] = v;
    const float p = P[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    P[i] = p;
    Pb[i] = sur_is_weight(i) ? __bfloat162float(__float2bfloat16_rn(p)) : p;
    grad[i] = 0.f;
}

// minibatch rows: a counter-based hash of (seed, step, slot), uniform over the
// dataset (sampling with replacement)
__device__ __forceinline__ unsigned long long sur_mix(unsigned long long z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
__global__ void k_sur_batch(int *__restrict__ idx, int nb, long n, unsigned long long seed, long long step)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nb) idx[s] = (int)(sur_mix(seed ^ sur_mix((unsigned long long)step * 0x100000001ULL + s)) % (unsigned long long)n);
}

// dataset append: B [k * bstride + atom] (double) -> X [row][SUR_KP] (float), E
__global__ void k_sur_append(const double *__restrict__ B, long bstride, const double *__restrict__ e, int n,
                             float *__restrict__ X, float *__restrict__ E, long row0)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
#pragma unroll
    for (int k = 0; k < SUR_KP; k++) X[(size_t)(row0 + a) * SUR_KP + k] = k < SUR_NK ? (float)B[(size_t)k * bstride + a] : 0.f;
    E[row0 + a] = (float)e[a];
}

// per-component sums of the dataset for the normalisation (double accumulators)
__global__ void k_sur_moments(const float *__restrict__ X, const float *__restrict__ E, long n, double *__restrict__ acc)
{
    double s[SUR_NK + 1], q[SUR_NK + 1];
#pragma unroll
    for (int k = 0; k <= SUR_NK; k++) { s[k] = 0.0; q[k] = 0.0; }
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < SUR_NK; k++) { const double v = X[r * SUR_KP + k]; s[k] += v; q[k] += v * v; }
        const double v = E[r];
        s[SUR_NK] += v; q[SUR_NK] += v * v;
    }
#pragma unroll
    for (int k = 0; k <= SUR_NK; k++) {
        double a = s[k], b = q[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) { a += __shfl_xor_sync(0xffffffffu, a, o); b += __shfl_xor_sync(0xffffffffu, b, o); }
        if ((threadIdx.x & 31) == 0) { atomicAdd(&acc[k], a); atomicAdd(&acc[SUR_NK + 1 + k], b); }
    }
}

// sum of squared force differences (for the judge) over n atoms
__global__ void k_force_sqdiff(const double4 *__restrict__ a, const double4 *__restrict__ b, int n, double *out)
{
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double4 u = a[i], v = b[i];
        const double dx = u.x - v.x, dy = u.y - v.y, dz = u.z - v.z;
        s += dx * dx + dy * dy + dz * dz;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

int force_sq_diff(const double4 *a, const double4 *b, int n, double *dev_acc, double *host_out, cudaStream_t s)
{
    MDP_CUDA_TRY(cudaMemsetAsync(dev_acc, 0, sizeof(double), s));
    k_force_sqdiff<<<std::min((n + 255) / 256, num_sms() * 8), 256, 0, s>>>(a, b, n, dev_acc);
    count_launches(1);
    MDP_CUDA_TRY(cudaMemcpyAsync(host_out, dev_acc, sizeof(double), cudaMemcpyDeviceToHost, s));
    MDP_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int launch_yi_pa_f4(const SnapModel &m, ForcePath &fp, int inum, const float *G, cudaStream_t s);
int launch_bi_tiles_f32(const float2 *Ut, int natoms, int tj, int bnorm, int bzero, double *bout, long bstride,
                        cudaStream_t s);

int sur_features(Surrogate &S, ForcePath &fp, const double4 *x, int inum, const int *nlist, const int *nnum, int nm,
                 cudaStream_t s)
{
    const SnapModel &m = S.model;
    const long ntiles = (inum + 31) / 32;
    const long pair_cap = (long)inum * nm;
    if (fp.pcount.ensure(sizeof(int) * (size_t)inum) || fp.poff.ensure(sizeof(int) * ((size_t)inum + 1)) ||
        fp.prij.ensure(sizeof(double4) * (size_t)pair_cap) || fp.pinfo.ensure(sizeof(int2) * (size_t)pair_cap) ||
        fp.pab.ensure(sizeof(double4) * (size_t)pair_cap) ||
        fp.smap.ensure(sizeof(int) * (size_t)inum * nm) || fp.dE.ensure(sizeof(double4) * (size_t)pair_cap) ||
        fp.Ut.ensure(sizeof(float2) * (size_t)ntiles * m.nu * 32) ||
        fp.Y.ensure(sizeof(float2) * (size_t)ntiles * 32 * m.nyh) ||
        fp.scan_tmp.ensure(sizeof(int) * scan_tmp_ints(inum)) || S.B.ensure(sizeof(double) * SUR_NK * (size_t)inum) ||
        S.G.ensure(sizeof(float) * SUR_NK * (size_t)inum))
        return -1;
    const int tb = 256, gb = (inum + tb - 1) / tb;
    const unsigned gw = (unsigned)(((long)inum * 32 + tb - 1) / tb);   // one warp per atom
    k_pair_count<<<gw, tb, 0, s>>>(x, nlist, nnum, inum, nm, m.geom.rcutsq, fp.pcount.as<int>());
    if (exclusive_scan(fp.pcount.as<int>(), fp.poff.as<int>(), inum, fp.scan_tmp.as<int>(), s)) return -1;
    k_pair_emit<<<gw, tb, 0, s>>>(x, nlist, nnum, inum, nm, fp.poff.as<int>(), m.geom, fp.prij.as<double4>(),
                                  fp.pinfo.as<int2>(), fp.pab.as<double4>(), fp.smap.as<int>());
    count_launches(2);
    if (launch_ui<float, 4>(m, fp, inum, s)) return -1;
    count_launches(1);
    return launch_bi_tiles_f32(fp.Ut.as<float2>(), inum, 4, m.p.bnormflag, m.p.bzeroflag, S.B.as<double>(), inum, s);
}

int sur_force(Surrogate &S, ForcePath &fp, const double4 *x, int inum, const int *nlist, const int *nnum, int nm,
              const int *roff, const long long *rlist, double *eatom, double4 *f, double *vatom, cudaStream_t s)
{
    if (!S.trained) { set_error("surrogate has no parameters"); return -1; }
    if (fp.timing && !fp.ev[0])
        for (auto &e : fp.ev) cudaEventCreate(&e);
    if (fp.timing) cudaEventRecord(fp.ev[0], s);
    if (sur_features(S, fp, x, inum, nlist, nnum, nm, s)) return -1;
    k_sur_infer_tc<<<std::min((inum + 16 * SUR_TC_WARPS - 1) / (16 * SUR_TC_WARPS), num_sms() * 16),
                     SUR_TC_WARPS * 32, 0, s>>>(S.B.as<double>(), inum, inum, S.Pb.as<float>(), S.norm, eatom,
                                                S.G.as<float>());
    if (launch_yi_pa_f4(S.model, fp, inum, S.G.as<float>(), s)) return -1;
    if (launch_fi<float, 4>(S.model, fp, inum, nm, s)) return -1;
    const int tb = 256, gb = (inum + tb - 1) / tb;
    if (fp.timing) cudaEventRecord(fp.ev[4], s);
    k_tally<<<gb, tb, 0, s>>>(fp.prij.as<double4>(), fp.dE.as<double4>(), fp.poff.as<int>(), fp.smap.as<int>(), inum,
                              roff, rlist, f, vatom, 1, 0);
    count_launches(4);
    if (fp.timing) {
        cudaEventRecord(fp.ev[5], s);
        cudaEventSynchronize(fp.ev[5]);
        float t[5], tot;
        for (int k = 0; k < 5; k++) cudaEventElapsedTime(&t[k], fp.ev[k], fp.ev[k + 1]);
        for (int k = 0; k < 5; k++) fp.stage_ms[k] += t[k];
        cudaEventElapsedTime(&tot, fp.ev[0], fp.ev[5]);
        fp.stage_ms[5] += tot;
        fp.stage_calls++;
    }
    MDP_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mdp

using namespace mdp;

extern "C" {

int mdp_sur_create(mdp_sur **h, const mdp_snap_params *p4, int device)
{
    if (!h || !p4) { set_error("null argument"); return -1; }
    *h = nullptr;
    if (p4->twojmax != 4) { set_error("the surrogate's features are the 2J=4 bispectrum (twojmax must be 4)"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(device));
    // coefficients of the feature model are all 1: the Y kernel's betaY then
    // holds the multiplicity factors that multiply the per-atom coefficients
    mdp_snap_params q = *p4;
    std::vector<double> ones(1 + SUR_NK, 1.0);
    ones[0] = 0.0;
    q.coeff = ones.data();
    q.ncoeffall = 1 + SUR_NK;
    mdp_sur *S = new mdp_sur();
    S->device = device;
    if (model_init(S->model, &q)) { delete S; return -1; }
    if (S->model.ne > 1) { set_error("the surrogate takes one element type"); delete S; return -1; }
    if (S->model.ncoeff != SUR_NK) { set_error("unexpected feature count"); delete S; return -1; }
    if (S->P.ensure(sizeof(float) * SUR_NPAR) || S->Pb.ensure(sizeof(float) * SUR_NPAR) ||
        S->grad.ensure(sizeof(float) * SUR_NPAR) || S->m1.ensure(sizeof(float) * SUR_NPAR) ||
        S->m2.ensure(sizeof(float) * SUR_NPAR) || S->scal.ensure(sizeof(double) * 64)) {
        mdp_sur_destroy(S);
        return -1;
    }
    int tr_per_sm = 0;
    if (kernel_setup((const void *)k_sur_grad, SUR_TR_THREADS, SUR_TR_SMEM, &tr_per_sm, "k_sur_grad")) {
        mdp_sur_destroy(S);
        return -1;
    }
    for (int k = 0; k < SUR_KP; k++) { S->norm.mu[k] = 0.f; S->norm.sinv[k] = 1.f; }
    S->norm.e_mu = 0.f;
    S->norm.e_sd = 1.f;
    *h = S;
    return 0;
}

void mdp_sur_destroy(mdp_sur *S)
{
    if (!S) return;
    cudaSetDevice(S->device);
    cudaDeviceSynchronize();
    DevBuf *b[] = {&S->P, &S->Pb, &S->grad, &S->m1, &S->m2, &S->X, &S->E, &S->idx, &S->scal, &S->B, &S->G};
    for (auto x : b) x->release();
    S->fp.release();
    delete S;
}

int mdp_sur_set_params(mdp_sur *S, const float *params, const float *norm)
{
    if (!S || !params) { set_error("null argument"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    MDP_CUDA_TRY(cudaMemcpy(S->P.p, params, sizeof(float) * SUR_NPAR, cudaMemcpyHostToDevice));
    k_sur_round<<<(SUR_NPAR + 255) / 256, 256>>>(S->P.as<float>(), S->Pb.as<float>());
    count_launches(1);
    MDP_CUDA_TRY(cudaMemset(S->grad.p, 0, sizeof(float) * SUR_NPAR));
    MDP_CUDA_TRY(cudaMemset(S->m1.p, 0, sizeof(float) * SUR_NPAR));
    MDP_CUDA_TRY(cudaMemset(S->m2.p, 0, sizeof(float) * SUR_NPAR));
    // the MD engine reads the rounded parameters on its own stream
    MDP_CUDA_TRY(cudaDeviceSynchronize());
    S->adam_t = 0;
    if (norm) {
        for (int k = 0; k < SUR_NK; k++) { S->norm.mu[k] = norm[k]; S->norm.sinv[k] = norm[SUR_NK + k]; }
        S->norm.e_mu = norm[2 * SUR_NK];
        S->norm.e_sd = norm[2 * SUR_NK + 1];
    }
    S->trained = true;
    MDP_CUDA_TRY(cudaDeviceSynchronize());
    return 0;
}

int mdp_sur_get_params(mdp_sur *S, float *params, float *norm)
{
    if (!S) { set_error("null handle"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    if (params) MDP_CUDA_TRY(cudaMemcpy(params, S->P.p, sizeof(float) * SUR_NPAR, cudaMemcpyDeviceToHost));
    if (norm) {
        for (int k = 0; k < SUR_NK; k++) { norm[k] = S->norm.mu[k]; norm[SUR_NK + k] = S->norm.sinv[k]; }
        norm[2 * SUR_NK] = S->norm.e_mu;
        norm[2 * SUR_NK + 1] = S->norm.e_sd;
    }
    return 0;
}

int mdp_sur_dataset_reserve(mdp_sur *S, long rows)
{
    if (!S || rows < 1) { set_error("bad arguments"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    if (S->X.ensure(sizeof(float) * SUR_KP * (size_t)rows) || S->E.ensure(sizeof(float) * (size_t)rows)) return -1;
    S->cap = rows;
    S->rows = 0;
    return 0;
}

long mdp_sur_dataset_size(mdp_sur *S) { return S ? S->rows : -1; }

int mdp_sur_dataset_add(mdp_sur *S, const double *B_dev, long bstride, const double *e_dev, int n, void *stream)
{
    if (!S || !B_dev || !e_dev || n < 1) { set_error("bad arguments"); return -1; }
    if (S->rows + n > S->cap) { set_error("dataset full (%ld of %ld rows)", S->rows, S->cap); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    k_sur_append<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(B_dev, bstride, e_dev, n, S->X.as<float>(),
                                                                  S->E.as<float>(), S->rows);
    count_launches(1);
    // the dataset is read next by training kernels on the legacy stream
    MDP_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    S->rows += n;
    return 0;
}

int mdp_sur_dataset_copy(mdp_sur *S, float *X, float *E, long row0, long nrows)
{
    if (!S || row0 < 0 || row0 + nrows > S->rows) { set_error("bad range"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    if (X) MDP_CUDA_TRY(cudaMemcpy(X, S->X.as<float>() + row0 * SUR_KP, sizeof(float) * SUR_KP * nrows, cudaMemcpyDeviceToHost));
    if (E) MDP_CUDA_TRY(cudaMemcpy(E, S->E.as<float>() + row0, sizeof(float) * nrows, cudaMemcpyDeviceToHost));
    return 0;
}

int mdp_sur_dataset_load(mdp_sur *S, const float *X, const float *E, long nrows)
{
    if (!S || !X || !E || nrows < 1) { set_error("bad arguments"); return -1; }
    if (mdp_sur_dataset_reserve(S, nrows)) return -1;
    MDP_CUDA_TRY(cudaMemcpy(S->X.p, X, sizeof(float) * SUR_KP * nrows, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(S->E.p, E, sizeof(float) * nrows, cudaMemcpyHostToDevice));
    S->rows = nrows;
    return 0;
}

// mean / standard deviation of the features and of the energy over the dataset
int mdp_sur_fit_normalization(mdp_sur *S)
{
    if (!S || S->rows < 2) { set_error("dataset too small"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    double *acc = S->scal.as<double>();
    MDP_CUDA_TRY(cudaMemset(acc, 0, sizeof(double) * 2 * (SUR_NK + 1)));
    k_sur_moments<<<num_sms() * 4, 256>>>(S->X.as<float>(), S->E.as<float>(), S->rows, acc);
    count_launches(1);
    double h[2 * (SUR_NK + 1)];
    MDP_CUDA_TRY(cudaMemcpy(h, acc, sizeof(h), cudaMemcpyDeviceToHost));
    const double n = (double)S->rows;
    for (int k = 0; k <= SUR_NK; k++) {
        const double mu = h[k] / n;
        const double var = std::max(h[SUR_NK + 1 + k] / n - mu * mu, 0.0);
        const double sd = var > 1e-24 ? sqrt(var) : 1.0;
        if (k < SUR_NK) { S->norm.mu[k] = (float)mu; S->norm.sinv[k] = (float)(1.0 / sd); }
        else { S->norm.e_mu = (float)mu; S->norm.e_sd = (float)sd; }
    }
    return 0;
}

// Adam steps on random minibatches; loss[i] = minibatch loss before step i
int mdp_sur_train(mdp_sur *S, int steps, int batch, float lr, unsigned long long seed, float *loss)
{
    if (!S || steps < 1 || batch < 1) { set_error("bad arguments"); return -1; }
    if (S->rows < 1) { set_error("empty dataset"); return -1; }
    if (!S->trained) { set_error("set initial parameters first"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    if (S->idx.ensure(sizeof(int) * (size_t)batch)) return -1;
    DevBuf lbuf;
    if (lbuf.ensure(sizeof(float) * (size_t)steps)) return -1;
    MDP_CUDA_TRY(cudaMemset(lbuf.p, 0, sizeof(float) * steps));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int it = 0; it < steps; it++) {
        S->adam_t++;
        k_sur_batch<<<(batch + 255) / 256, 256>>>(S->idx.as<int>(), batch, S->rows, seed, S->adam_t);
        k_sur_grad<<<(batch + SUR_TR_THREADS - 1) / SUR_TR_THREADS, SUR_TR_THREADS, SUR_TR_SMEM>>>(
            S->X.as<float>(), S->E.as<float>(), S->idx.as<int>(), batch, S->Pb.as<float>(), S->norm,
            S->grad.as<float>(), lbuf.as<float>() + it);
        const float c1 = 1.f - powf(b1, (float)S->adam_t), c2 = 1.f - powf(b2, (float)S->adam_t);
        k_sur_adam<<<(SUR_NPAR + 255) / 256, 256>>>(S->P.as<float>(), S->Pb.as<float>(), S->grad.as<float>(),
                                                    S->m1.as<float>(), S->m2.as<float>(), lr, b1, b2, eps, c1, c2);
        count_launches(3);
    }
    MDP_CUDA_TRY(cudaGetLastError());
    if (loss) MDP_CUDA_TRY(cudaMemcpy(loss, lbuf.p, sizeof(float) * steps, cudaMemcpyDeviceToHost));
    // the MD engine reads the parameters on its own stream
    MDP_CUDA_TRY(cudaDeviceSynchronize());
    lbuf.release();
    return 0;
}

// gradient of the minibatch loss over the given host rows (X [n][16], E [n])
// at the current parameters, without updating them
int mdp_sur_grad(mdp_sur *S, const float *X, const float *E, int n, float *grad, float *loss)
{
    if (!S || !X || !E || n < 1 || !grad) { set_error("bad arguments"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    DevBuf dx, de, di, dl;
    std::vector<int> id(n);
    for (int i = 0; i < n; i++) id[i] = i;
    if (dx.ensure(sizeof(float) * SUR_KP * (size_t)n) || de.ensure(sizeof(float) * (size_t)n) ||
        di.ensure(sizeof(int) * (size_t)n) || dl.ensure(sizeof(float)))
        return -1;
    MDP_CUDA_TRY(cudaMemcpy(dx.p, X, sizeof(float) * SUR_KP * n, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(de.p, E, sizeof(float) * n, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(di.p, id.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemset(dl.p, 0, sizeof(float)));
    MDP_CUDA_TRY(cudaMemset(S->grad.p, 0, sizeof(float) * SUR_NPAR));
    k_sur_grad<<<(n + SUR_TR_THREADS - 1) / SUR_TR_THREADS, SUR_TR_THREADS, SUR_TR_SMEM>>>(
        dx.as<float>(), de.as<float>(), di.as<int>(), n, S->Pb.as<float>(), S->norm, S->grad.as<float>(), dl.as<float>());
    count_launches(1);
    MDP_CUDA_TRY(cudaGetLastError());
    MDP_CUDA_TRY(cudaMemcpy(grad, S->grad.p, sizeof(float) * SUR_NPAR, cudaMemcpyDeviceToHost));
    if (loss) MDP_CUDA_TRY(cudaMemcpy(loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
    MDP_CUDA_TRY(cudaMemset(S->grad.p, 0, sizeof(float) * SUR_NPAR));
    dx.release(); de.release(); di.release(); dl.release();
    return 0;
}

// inference on host features B [k * n + atom] (double): energies and G [k * n + atom]
int mdp_sur_eval(mdp_sur *S, const double *B, int n, double *E, float *G)
{
    if (!S || !B || n < 1) { set_error("bad arguments"); return -1; }
    if (!S->trained) { set_error("surrogate has no parameters"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    DevBuf db, de, dg;
    if (db.ensure(sizeof(double) * SUR_NK * (size_t)n) || de.ensure(sizeof(double) * (size_t)n) ||
        dg.ensure(sizeof(float) * SUR_NK * (size_t)n))
        return -1;
    MDP_CUDA_TRY(cudaMemcpy(db.p, B, sizeof(double) * SUR_NK * n, cudaMemcpyHostToDevice));
    k_sur_infer_tc<<<(n + 16 * SUR_TC_WARPS - 1) / (16 * SUR_TC_WARPS), SUR_TC_WARPS * 32>>>(
        db.as<double>(), n, n, S->Pb.as<float>(), S->norm, de.as<double>(), dg.as<float>());
    count_launches(1);
    MDP_CUDA_TRY(cudaGetLastError());
    if (E) MDP_CUDA_TRY(cudaMemcpy(E, de.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (G) MDP_CUDA_TRY(cudaMemcpy(G, dg.p, sizeof(float) * SUR_NK * n, cudaMemcpyDeviceToHost));
    db.release(); de.release(); dg.release();
    return 0;
}

// Force-training set from a 2J=4 batch of equal-size snapshots (mdp_fit with
// the snapshots as configurations): per-pair dB/dR, features, pair structure,
// and the plain model's forces (3 per atom) and per-atom energies.
int mdp_sur_force_set(mdp_sur *S, mdp_fit *F, const double *forces, const double *energies, int per)
{
    if (!S || !F || !forces || !energies || per < 1) { set_error("bad arguments"); return -1; }
    if (F->model.p.twojmax != 4 || F->tab.ntri != SUR_NK) { set_error("the force set needs a 2J=4 batch"); return -1; }
    if (F->natoms % per != 0) { set_error("snapshots must all have %d atoms", per); return -1; }
    for (int c = 0; c < F->nconf; c++)
        if (F->h_cn[c] != per) { set_error("snapshot %d has %d atoms, not %d", c, F->h_cn[c], per); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    const long na = F->natoms, np = F->npairs;
    if (S->fB.ensure(sizeof(double) * SUR_NK * na) || S->fE.ensure(sizeof(float) * na) ||
        S->fF.ensure(sizeof(float) * 3 * na) || S->fdb.ensure(sizeof(float) * 3 * SUR_NK * std::max(np, 1L)) ||
        S->fpinfo.ensure(sizeof(int2) * std::max(np, 1L)) || S->fpoff.ensure(sizeof(int) * (na + 1)) ||
        S->froff.ensure(sizeof(int) * (na + 1)) || S->frlist.ensure(sizeof(int) * std::max(np, 1L)) ||
        S->fscal.ensure(sizeof(float) * 8))
        return -1;
    if (fit_pair_derivs(F, S->fdb.as<float>(), S->fB.as<double>())) return -1;
    MDP_CUDA_TRY(cudaMemcpy(S->fpinfo.p, F->fp.pinfo.p, sizeof(int2) * np, cudaMemcpyDeviceToDevice));
    MDP_CUDA_TRY(cudaMemcpy(S->fpoff.p, F->poff.p, sizeof(int) * (na + 1), cudaMemcpyDeviceToDevice));
    MDP_CUDA_TRY(cudaMemcpy(S->froff.p, F->roff.p, sizeof(int) * (na + 1), cudaMemcpyDeviceToDevice));
    MDP_CUDA_TRY(cudaMemcpy(S->frlist.p, F->rlist.p, sizeof(int) * np, cudaMemcpyDeviceToDevice));
    std::vector<float> hf(3 * na), he(na);
    double var = 0.0;
    for (long i = 0; i < 3 * na; i++) { hf[i] = (float)forces[i]; var += forces[i] * forces[i]; }
    for (long i = 0; i < na; i++) he[i] = (float)energies[i];
    MDP_CUDA_TRY(cudaMemcpy(S->fF.p, hf.data(), sizeof(float) * 3 * na, cudaMemcpyHostToDevice));
    MDP_CUDA_TRY(cudaMemcpy(S->fE.p, he.data(), sizeof(float) * na, cudaMemcpyHostToDevice));
    S->f_atoms = na;
    S->f_pairs = np;
    S->f_per = per;
    S->f_snaps = (int)(na / per);
    S->f_var = var / (3.0 * na) > 1e-30 ? var / (3.0 * na) : 1.0;
    return 0;
}

// Adam steps on windows of snaps_per_batch consecutive snapshots of the force
// set: loss = mean normalised per-atom energy error^2 + alpha * mean force
// error^2 / var(F).  loss_e, loss_f (may be NULL): per step.
int mdp_sur_train_forces(mdp_sur *S, int steps, int snaps_per_batch, float lr, float alpha, unsigned long long seed,
                         float *loss_e, float *loss_f)
{
    if (!S || steps < 1 || snaps_per_batch < 1) { set_error("bad arguments"); return -1; }
    if (!S->trained) { set_error("set initial parameters first"); return -1; }
    if (S->f_snaps < snaps_per_batch) { set_error("force set holds %d snapshots", S->f_snaps); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    int tf_per_sm = 0;
    if (kernel_setup((const void *)k_sur_grad_f, SUR_TF_THREADS, SUR_TF_SMEM, &tf_per_sm, "k_sur_grad_f")) return -1;
    const int n = snaps_per_batch * S->f_per;
    if (S->fG.ensure(sizeof(float) * SUR_NK * (size_t)n) || S->fQ.ensure(sizeof(float) * 3 * (size_t)n) ||
        S->fV.ensure(sizeof(float) * SUR_KP * (size_t)n))
        return -1;
    DevBuf lb;
    if (lb.ensure(sizeof(float) * 2 * (size_t)steps)) return -1;
    MDP_CUDA_TRY(cudaMemset(lb.p, 0, sizeof(float) * 2 * steps));
    const float coef = 2.0f * alpha / (float)(3.0 * n * S->f_var), lw = alpha / (float)(3.0 * n * S->f_var);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    unsigned long long st = seed * 0x9e3779b97f4a7c15ULL + 1;
    for (int it = 0; it < steps; it++) {
        st = st * 6364136223846793005ULL + 1442695040888963407ULL;
        const int s0 = (int)((st >> 33) % (unsigned long long)(S->f_snaps - snaps_per_batch + 1));
        const int a_lo = s0 * S->f_per;
        const double *Bw = S->fB.as<double>() + a_lo;
        k_sur_infer_tc<<<std::min((n + 16 * SUR_TC_WARPS - 1) / (16 * SUR_TC_WARPS), num_sms() * 16),
                         SUR_TC_WARPS * 32>>>(Bw, S->f_atoms, n, S->Pb.as<float>(), S->norm, nullptr,
                                              S->fG.as<float>());
        k_sur_fpred<<<(n + 127) / 128, 128>>>(a_lo, n, S->fpoff.as<int>(), S->froff.as<int>(), S->frlist.as<int>(),
                                              S->fpinfo.as<int2>(), S->fdb.as<float>(), S->fG.as<float>(),
                                              S->fF.as<float>(), coef, lw, S->fQ.as<float>(), lb.as<float>() + 2 * it + 1);
        k_sur_lambda<<<(n + 127) / 128, 128>>>(a_lo, n, S->fpoff.as<int>(), S->fpinfo.as<int2>(), S->fdb.as<float>(),
                                               S->fQ.as<float>(), S->norm, S->fV.as<float>());
        k_sur_grad_f<<<(n + SUR_TF_THREADS - 1) / SUR_TF_THREADS, SUR_TF_THREADS, SUR_TF_SMEM>>>(
            Bw, S->f_atoms, S->fE.as<float>() + a_lo, S->fV.as<float>(), n, 1.0f, S->Pb.as<float>(), S->norm,
            S->grad.as<float>(), lb.as<float>() + 2 * it);
        S->adam_t++;
        const float c1 = 1.f - powf(b1, (float)S->adam_t), c2 = 1.f - powf(b2, (float)S->adam_t);
        k_sur_adam<<<(SUR_NPAR + 255) / 256, 256>>>(S->P.as<float>(), S->Pb.as<float>(), S->grad.as<float>(),
                                                    S->m1.as<float>(), S->m2.as<float>(), lr, b1, b2, eps, c1, c2);
        count_launches(5);
    }
    MDP_CUDA_TRY(cudaGetLastError());
    if (loss_e || loss_f) {
        std::vector<float> h(2 * (size_t)steps);
        MDP_CUDA_TRY(cudaMemcpy(h.data(), lb.p, sizeof(float) * 2 * steps, cudaMemcpyDeviceToHost));
        for (int i = 0; i < steps; i++) {
            if (loss_e) loss_e[i] = h[2 * i];
            if (loss_f) loss_f[i] = h[2 * i + 1];
        }
    }
    // the MD engine reads the parameters on its own stream
    MDP_CUDA_TRY(cudaDeviceSynchronize());
    lb.release();
    return 0;
}

// gradient of the combined loss over one window (no update), for the oracle
// check: grad (NPAR), losses (energy, force)
int mdp_sur_force_grad(mdp_sur *S, int snap0, int snaps, float alpha, float *grad, float *losses)
{
    if (!S || !grad || snaps < 1 || snap0 < 0 || snap0 + snaps > S->f_snaps) { set_error("bad arguments"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    int tf_per_sm = 0;
    if (kernel_setup((const void *)k_sur_grad_f, SUR_TF_THREADS, SUR_TF_SMEM, &tf_per_sm, "k_sur_grad_f")) return -1;
    const int n = snaps * S->f_per, a_lo = snap0 * S->f_per;
    if (S->fG.ensure(sizeof(float) * SUR_NK * (size_t)n) || S->fQ.ensure(sizeof(float) * 3 * (size_t)n) ||
        S->fV.ensure(sizeof(float) * SUR_KP * (size_t)n))
        return -1;
    const float coef = 2.0f * alpha / (float)(3.0 * n * S->f_var), lw = alpha / (float)(3.0 * n * S->f_var);
    float *lb = S->fscal.as<float>();
    MDP_CUDA_TRY(cudaMemset(lb, 0, sizeof(float) * 2));
    MDP_CUDA_TRY(cudaMemset(S->grad.p, 0, sizeof(float) * SUR_NPAR));
    const double *Bw = S->fB.as<double>() + a_lo;
    k_sur_infer_tc<<<(n + 16 * SUR_TC_WARPS - 1) / (16 * SUR_TC_WARPS), SUR_TC_WARPS * 32>>>(
        Bw, S->f_atoms, n, S->Pb.as<float>(), S->norm, nullptr, S->fG.as<float>());
    k_sur_fpred<<<(n + 127) / 128, 128>>>(a_lo, n, S->fpoff.as<int>(), S->froff.as<int>(), S->frlist.as<int>(),
                                          S->fpinfo.as<int2>(), S->fdb.as<float>(), S->fG.as<float>(), S->fF.as<float>(),
                                          coef, lw, S->fQ.as<float>(), lb + 1);
    k_sur_lambda<<<(n + 127) / 128, 128>>>(a_lo, n, S->fpoff.as<int>(), S->fpinfo.as<int2>(), S->fdb.as<float>(),
                                           S->fQ.as<float>(), S->norm, S->fV.as<float>());
    k_sur_grad_f<<<(n + SUR_TF_THREADS - 1) / SUR_TF_THREADS, SUR_TF_THREADS, SUR_TF_SMEM>>>(
        Bw, S->f_atoms, S->fE.as<float>() + a_lo, S->fV.as<float>(), n, 1.0f, S->Pb.as<float>(), S->norm,
        S->grad.as<float>(), lb);
    count_launches(4);
    MDP_CUDA_TRY(cudaGetLastError());
    MDP_CUDA_TRY(cudaMemcpy(grad, S->grad.p, sizeof(float) * SUR_NPAR, cudaMemcpyDeviceToHost));
    if (losses) MDP_CUDA_TRY(cudaMemcpy(losses, lb, sizeof(float) * 2, cudaMemcpyDeviceToHost));
    MDP_CUDA_TRY(cudaMemset(S->grad.p, 0, sizeof(float) * SUR_NPAR));
    return 0;
}

// copy of the force set's features [k][atom] (double) and per-pair dB/dR
// [pair][3][14] (float), for the oracle check
int mdp_sur_force_set_copy(mdp_sur *S, double *B, float *db, int *pinfo, int *poff)
{
    if (!S) { set_error("null handle"); return -1; }
    MDP_CUDA_TRY(cudaSetDevice(S->device));
    if (B) MDP_CUDA_TRY(cudaMemcpy(B, S->fB.p, sizeof(double) * SUR_NK * S->f_atoms, cudaMemcpyDeviceToHost));
    if (db) MDP_CUDA_TRY(cudaMemcpy(db, S->fdb.p, sizeof(float) * 3 * SUR_NK * S->f_pairs, cudaMemcpyDeviceToHost));
    if (pinfo) MDP_CUDA_TRY(cudaMemcpy(pinfo, S->fpinfo.p, sizeof(int2) * S->f_pairs, cudaMemcpyDeviceToHost));
    if (poff) MDP_CUDA_TRY(cudaMemcpy(poff, S->fpoff.p, sizeof(int) * (S->f_atoms + 1), cudaMemcpyDeviceToHost));
    return 0;
}

long long mdp_sur_force_set_npairs(mdp_sur *S) { return S ? S->f_pairs : -1; }

int mdp_sur_nparams(void) { return SUR_NPAR; }

}  // extern "C"
