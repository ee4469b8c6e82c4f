// Learned star-pressure guess for the exact Riemann solver.
//
// The network maps the normalised left/right states of a face (6 features) to
// a correction of the analytic guess in log space, r = ln(p* / p_analytic):
//   x (6) -> Linear(6, 32) -> ReLU -> Linear(32, 32) -> ReLU -> Linear(32, 1).
// Weights and activations are BF16, accumulation FP32. Inference runs one warp
// per 32 faces on the tensor cores (mma.sync m16n8k16, BF16 in, FP32 out): the
// 32 faces are the M dimension, so the three layers are 8 + 16 + 4 MMAs whose
// FP32 outputs feed the next layer's A fragments straight from registers.
// The analytic guess stays the fallback and judge: when |r| is inside the
// network's own error band (the gate) the analytic value is used unchanged,
// and the exact solver reruns from it if the learned start hits the cap.
//
// Training (learned.cu) uses the same quantisation points in FP32 scalar code:
// x, W and the hidden activations rounded to BF16, biases and sums in FP32.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#include <cuda_bf16.h>
#endif

#include "riemann.cuh"

namespace dgpu {

constexpr int kMlpIn = 6;
constexpr int kMlpHidden = 32;
// Flat FP32 parameter vector: weights (row-major, [out][in]) and biases,
// then the input/output normalisation and the gate.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;         // 192
constexpr int kOffW2 = kOffB1 + kMlpHidden;                  // 224
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;     // 1248
constexpr int kOffW3 = kOffB2 + kMlpHidden;                  // 1280
constexpr int kOffB3 = kOffW3 + kMlpHidden;                  // 1312
constexpr int kMlpWeights = kOffB3 + 1;                      // 1313 trainable
constexpr int kOffXMean = kMlpWeights;                       // 1313
constexpr int kOffXStd = kOffXMean + kMlpIn;                 // 1319
constexpr int kOffTMean = kOffXStd + kMlpIn;                 // 1325
constexpr int kOffTStd = kOffTMean + 1;                      // 1326
constexpr int kOffGate = kOffTStd + 1;                       // 1327
constexpr int kMlpParams = kOffGate + 1;                     // 1328

// Per-lane fragment words: layer 1 B (4 n-tiles, upper k half is zero),
// layer 2 B (2 k-tiles x 4 n-tiles x 2), layer 3 B (2 k-tiles x 2).
constexpr int kFragL1 = 0, kFragL2 = 4, kFragL3 = 20, kFragWords = 24;
constexpr int kFragBias = 16;  // layer-1 then layer-2 bias pairs of the lane's C columns

// Inference image of the network in mma.sync fragment order.
struct MlpNet {
    uint32_t frag[32][kFragWords];
    float bias[32][kFragBias];
    float x_mean[kMlpIn];
    float x_inv_std[kMlpIn];
    float t_mean, t_std, gate, b3;
};

// Face features from the face-normal states: log density and pressure of each
// side relative to the geometric means, and each side's normal velocity
// relative to the mean in units of the mean sound speed. The star pressure
// over the geometric-mean pressure depends on nothing else (the exact
// Riemann problem is invariant under density and pressure scaling and
// Galilean shifts).
template <class R>
DHD void mlp_features(const Prim<R>& L, const Prim<R>& Rt, float x[kMlpIn]) {
    const float rl = (float)L.rho, rr = (float)Rt.rho, pl = (float)L.p, pr = (float)Rt.p;
    const float lr = logf(rl / rr), lp = logf(pl / pr);
    const float rbar = sqrtf(rl) * sqrtf(rr), pbar = sqrtf(pl) * sqrtf(pr);
    const float cbar = sqrtf((float)kGamma * pbar / rbar);
    const float du = (float)(Rt.vx - L.vx) / cbar;
    x[0] = 0.5f * lr;
    x[1] = 0.5f * lp;
    x[2] = -0.5f * du;
    x[3] = -0.5f * lr;
    x[4] = -0.5f * lp;
    x[5] = 0.5f * du;
}

// Guess from the network output y (normalised units) and the analytic guess.
// A non-finite output yields NaN, which the exact solver rejects.
DHD double mlp_guess_from(float y, float t_mean, float t_std, float gate, double p_analytic) {
    const float r = y * t_std + t_mean;
    if (!isfinite(r)) return NAN;
    if (fabsf(r) <= gate) return p_analytic;
    return p_analytic * exp((double)r);
}

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// D += A * B for one m16n8k16 tile, BF16 operands, FP32 accumulators.
__device__ __forceinline__ void mma_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                          uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Network output for this lane's face (normalised features xn). Warp
// collective: all 32 lanes must call it together, converged; lanes without a
// face pass any finite features and ignore the result.
//
// Fragment layout (PTX ISA, mma.m16n8k16 with .bf16): lane = 4 g + q;
// A regs hold rows g / g+8, columns 2q, 2q+1 (+8 for regs 2, 3);
// B regs hold k = 2q, 2q+1 (+8) of column g; C holds rows g / g+8,
// columns 2q, 2q+1. Faces are rows: face f sits in m-tile f / 16, row f % 16.
__device__ __forceinline__ float mlp_forward_warp(const MlpNet* __restrict__ net, const float (&xn)[kMlpIn]) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const uint32_t p0 = bf16x2(xn[0], xn[1]), p1 = bf16x2(xn[2], xn[3]), p2 = bf16x2(xn[4], xn[5]);
    // layer-1 A: [m-tile][row half]; columns 6..15 are zero
    uint32_t a1[2][2];
#pragma unroll
    for (int t = 0; t < 2; t++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int src = 16 * t + 8 * h + g;
            const uint32_t v0 = __shfl_sync(full, p0, src), v1 = __shfl_sync(full, p1, src),
                           v2 = __shfl_sync(full, p2, src);
            a1[t][h] = q == 0 ? v0 : q == 1 ? v1 : q == 2 ? v2 : 0u;
        }
    uint32_t fw[kFragWords];
    float fb[kFragBias];
    {
        const uint4* s = reinterpret_cast<const uint4*>(net->frag[lane]);
#pragma unroll
        for (int i = 0; i < kFragWords / 4; i++) {
            const uint4 v = __ldg(s + i);
            fw[4 * i] = v.x; fw[4 * i + 1] = v.y; fw[4 * i + 2] = v.z; fw[4 * i + 3] = v.w;
        }
        const float4* b = reinterpret_cast<const float4*>(net->bias[lane]);
#pragma unroll
        for (int i = 0; i < kFragBias / 4; i++) {
            const float4 v = __ldg(b + i);
            fb[4 * i] = v.x; fb[4 * i + 1] = v.y; fb[4 * i + 2] = v.z; fb[4 * i + 3] = v.w;
        }
    }
    // layer 1 (bias in the accumulator), ReLU, repack as layer-2 A fragments
    uint32_t a2[2][2][4];
#pragma unroll
    for (int t = 0; t < 2; t++) {
        float h[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            h[nt][0] = h[nt][2] = fb[2 * nt];
            h[nt][1] = h[nt][3] = fb[2 * nt + 1];
            mma_16816(h[nt], a1[t][0], a1[t][1], 0u, 0u, fw[kFragL1 + nt], 0u);
        }
#pragma unroll
        for (int kt = 0; kt < 2; kt++) {
            a2[t][kt][0] = bf16x2(fmaxf(h[2 * kt][0], 0.f), fmaxf(h[2 * kt][1], 0.f));
            a2[t][kt][1] = bf16x2(fmaxf(h[2 * kt][2], 0.f), fmaxf(h[2 * kt][3], 0.f));
            a2[t][kt][2] = bf16x2(fmaxf(h[2 * kt + 1][0], 0.f), fmaxf(h[2 * kt + 1][1], 0.f));
            a2[t][kt][3] = bf16x2(fmaxf(h[2 * kt + 1][2], 0.f), fmaxf(h[2 * kt + 1][3], 0.f));
        }
    }
    // layer 2, ReLU, repack; layer 3 into n-tile 0 (only column 0 is used)
    float yt[2][4];
#pragma unroll
    for (int t = 0; t < 2; t++) {
        float h[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            h[nt][0] = h[nt][2] = fb[8 + 2 * nt];
            h[nt][1] = h[nt][3] = fb[8 + 2 * nt + 1];
#pragma unroll
            for (int kt = 0; kt < 2; kt++)
                mma_16816(h[nt], a2[t][kt][0], a2[t][kt][1], a2[t][kt][2], a2[t][kt][3],
                          fw[kFragL2 + (kt * 4 + nt) * 2], fw[kFragL2 + (kt * 4 + nt) * 2 + 1]);
        }
        yt[t][0] = yt[t][1] = yt[t][2] = yt[t][3] = 0.f;
#pragma unroll
        for (int kt = 0; kt < 2; kt++) {
            const uint32_t c0 = bf16x2(fmaxf(h[2 * kt][0], 0.f), fmaxf(h[2 * kt][1], 0.f));
            const uint32_t c1 = bf16x2(fmaxf(h[2 * kt][2], 0.f), fmaxf(h[2 * kt][3], 0.f));
            const uint32_t c2 = bf16x2(fmaxf(h[2 * kt + 1][0], 0.f), fmaxf(h[2 * kt + 1][1], 0.f));
            const uint32_t c3 = bf16x2(fmaxf(h[2 * kt + 1][2], 0.f), fmaxf(h[2 * kt + 1][3], 0.f));
            mma_16816(yt[t], c0, c1, c2, c3, fw[kFragL3 + 2 * kt], fw[kFragL3 + 2 * kt + 1]);
        }
    }
    // row r of m-tile t: column 0 lives in lane 4 (r % 8), element 0 (r < 8) or 2
    const int t = lane >> 4, r = lane & 15, src = 4 * (r & 7);
    const float y00 = __shfl_sync(full, yt[0][0], src), y02 = __shfl_sync(full, yt[0][2], src);
    const float y10 = __shfl_sync(full, yt[1][0], src), y12 = __shfl_sync(full, yt[1][2], src);
    const float y = t == 0 ? (r < 8 ? y00 : y02) : (r < 8 ? y10 : y12);
    return y + net->b3;
}

// Newton start for this lane's face (face-normal states). Warp collective
// like mlp_forward_warp. The two-rarefaction test runs first; the network
// runs only when some lane of the warp needs Newton (a warp-uniform branch),
// and the analytic guess only on the lanes that do.
__device__ __forceinline__ LearnedGuess<double> mlp_guess_warp(const MlpNet* __restrict__ net, const Prim<double>& L,
                                                               const Prim<double>& Rt, bool valid) {
    LearnedGuess<double> g{0.0, 0.0, 1};
    const bool newton = valid && !exact_is_trrs(L, Rt);
    g.trrs = newton ? 0 : 1;
    if (!__any_sync(0xffffffffu, newton)) return g;
    float xn[kMlpIn];
    if (newton) {
        mlp_features(L, Rt, xn);
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) xn[i] = (xn[i] - net->x_mean[i]) * net->x_inv_std[i];
    } else {
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) xn[i] = 0.f;
    }
    const float y = mlp_forward_warp(net, xn);
    if (newton) {
        g.analytic = analytic_guess(L, Rt);
        g.guess = mlp_guess_from(y, net->t_mean, net->t_std, net->gate, g.analytic);
    }
    return g;
}
#endif

}  // namespace dgpu
