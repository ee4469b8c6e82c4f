// Training and inference of the learned star-pressure guess
// (include/dragon_learned.h): the training set, the forward / backward and
// optimiser kernels, the packing of the weights into tensor-core fragments,
// and a stand-alone inference kernel.
//
// Training runs in FP32 on the CUDA cores with the inference's quantisation
// points (BF16 inputs, weights and hidden activations; FP32 biases and sums),
// treating each rounding as the identity in the backward pass. A minibatch is
// spread over blocks of kTB samples; every block writes its partial gradient
// and the reduction sums the partials in block order, so a training run is
// deterministic for a given seed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/dragon_learned.h"
#include "mlp.cuh"

void dragon_gpu_set_error_message(const char* msg);

using namespace dgpu;

struct dragon_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    unsigned long long seed = 0;
    long long batches = 0;        // minibatches drawn so far (hash counter)
    long long adam_t = 0;         // optimiser steps since load
    float* P = nullptr;           // kMlpParams
    float* adam_m = nullptr;      // kMlpWeights
    float* adam_v = nullptr;      // kMlpWeights
    float* partial = nullptr;     // partial_blocks x kMlpWeights
    float* loss_part = nullptr;   // partial_blocks
    int partial_blocks = 0;
    float* out = nullptr;         // [0] loss sum, [1..kMlpWeights] gradient
    MlpNet* net = nullptr;
    bool net_dirty = true;
    float* X = nullptr;           // n x kMlpIn raw features
    float* T = nullptr;           // n targets ln(p* / p_analytic)
    long long n = 0, cap = 0;
};

namespace {

constexpr int kTB = 128;              // samples per block of the gradient kernel
constexpr int kH1 = kMlpHidden + 1;   // padded row length in shared memory
constexpr int kGradSmemFloats = 1320 + kTB * 8 + 4 * kTB * kH1 + 2 * kTB;

int fail(int code, const std::string& msg) {
    dragon_gpu_set_error_message(msg.c_str());
    return code;
}

#define CKM(x)                                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return fail(DRAGON_GPU_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_));   \
    } while (0)

__device__ __forceinline__ float q16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ Prim<double> row_state(const double* r) {
    Prim<double> w = zero_prim<double>();
    w.rho = r[0];
    w.vx = r[1];
    w.p = r[2];
    return w;
}

// Log rows -> raw features and targets ln(p* / p_analytic).
__global__ void k_mlp_prepare(const double* __restrict__ rows, long long n, float* __restrict__ X,
                              float* __restrict__ T) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const double* r = rows + s * kNewtonLogCols;
        const Prim<double> L = row_state(r), R = row_state(r + 3);
        float x[kMlpIn];
        mlp_features(L, R, x);
        for (int i = 0; i < kMlpIn; i++) X[s * kMlpIn + i] = x[i];
        T[s] = (float)log(r[6] / analytic_guess(L, R));
    }
}

// Mean and standard deviation of the features and the target over the finite
// samples (one block).
__global__ void k_mlp_stats(const float* __restrict__ X, const float* __restrict__ T, long long n, float* P) {
    __shared__ double red[2 * (kMlpIn + 1) + 1][32];
    double s[kMlpIn + 1], ss[kMlpIn + 1], cnt = 0.0;
    for (int c = 0; c <= kMlpIn; c++) s[c] = ss[c] = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        float chk = T[i];
        for (int c = 0; c < kMlpIn; c++) chk += X[i * kMlpIn + c];
        if (!isfinite(chk)) continue;
        cnt += 1.0;
        for (int c = 0; c <= kMlpIn; c++) {
            const double v = c < kMlpIn ? X[i * kMlpIn + c] : T[i];
            s[c] += v;
            ss[c] += v * v;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = 0; c <= kMlpIn; c++) {
        double a = s[c], b = ss[c];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) { red[2 * c][warp] = a; red[2 * c + 1][warp] = b; }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if (lane == 0) red[2 * (kMlpIn + 1)][warp] = cnt;
    __syncthreads();
    if (threadIdx.x <= kMlpIn) {
        const int c = threadIdx.x;
        double a = 0, b = 0, m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            a += red[2 * c][w];
            b += red[2 * c + 1][w];
            m += red[2 * (kMlpIn + 1)][w];
        }
        const double mean = m > 0 ? a / m : 0.0;
        const double var = m > 0 ? fmax(b / m - mean * mean, 0.0) : 1.0;
        const float sd = (float)fmax(sqrt(var), 1e-6);
        if (c < kMlpIn) { P[kOffXMean + c] = (float)mean; P[kOffXStd + c] = sd; }
        else { P[kOffTMean] = (float)mean; P[kOffTStd] = sd; }
    }
}

// Forward + backward of kTB samples per block; partial gradient and loss sum
// of the block. Samples are [first, first + batch) when contiguous, else drawn
// by hash from the whole set. dy carries the 1 / batch of the mean loss.
__global__ void __launch_bounds__(kTB) k_mlp_grad(const float* __restrict__ P, const float* __restrict__ X,
                                                  const float* __restrict__ T, long long N, long long first,
                                                  int contiguous, unsigned long long seed, long long draw, int batch,
                                                  float* __restrict__ partial, float* __restrict__ loss_part) {
    extern __shared__ float sm[];
    float* sW1 = sm;                  // 192
    float* sb1 = sW1 + 192;           // 32
    float* sW2 = sb1 + 32;            // 1024
    float* sb2 = sW2 + 1024;          // 32
    float* sW3 = sb2 + 32;            // 32
    float* sb3 = sW3 + 32;            // 1 (+pad)
    float* s_x = sm + 1320;           // kTB x 8
    float* s_h1 = s_x + kTB * 8;      // kTB x kH1
    float* s_dz1 = s_h1 + kTB * kH1;
    float* s_h2 = s_dz1 + kTB * kH1;
    float* s_dz2 = s_h2 + kTB * kH1;
    float* s_dy = s_dz2 + kTB * kH1;  // kTB
    float* s_red = s_dy + kTB;        // kTB
    const int t = threadIdx.x;
    for (int i = t; i < 192; i += kTB) sW1[i] = q16(P[kOffW1 + i]);
    for (int i = t; i < 1024; i += kTB) sW2[i] = q16(P[kOffW2 + i]);
    if (t < 32) {
        sb1[t] = P[kOffB1 + t];
        sb2[t] = P[kOffB2 + t];
        sW3[t] = q16(P[kOffW3 + t]);
    }
    if (t == 0) sb3[0] = P[kOffB3];
    __syncthreads();

    const long long s = (long long)blockIdx.x * kTB + t;
    bool valid = s < batch;
    float xq[kMlpIn], tn = 0.f;
    if (valid) {
        const long long idx = contiguous ? first + s
                                         : (long long)(mix64(seed ^ mix64((unsigned long long)draw) ^ (unsigned long long)s) %
                                                       (unsigned long long)N);
        float chk = T[idx];
        for (int i = 0; i < kMlpIn; i++) {
            xq[i] = q16((X[idx * kMlpIn + i] - P[kOffXMean + i]) / P[kOffXStd + i]);
            chk += xq[i];
        }
        tn = (T[idx] - P[kOffTMean]) / P[kOffTStd];
        valid = isfinite(chk);  // a malformed sample contributes nothing
    }
    if (!valid) {
        for (int i = 0; i < kMlpIn; i++) xq[i] = 0.f;
        tn = 0.f;
    }
    // forward; this sample's activations live in its shared-memory rows
    float* h1 = s_h1 + t * kH1;
    float* h2 = s_h2 + t * kH1;
    float* dz2 = s_dz2 + t * kH1;
    unsigned m1 = 0, m2 = 0;
    for (int j = 0; j < kMlpHidden; j++) {
        float z = sb1[j];
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) z += sW1[j * kMlpIn + i] * xq[i];
        if (z > 0.f) m1 |= 1u << j;
        h1[j] = q16(fmaxf(z, 0.f));
    }
    for (int k = 0; k < kMlpHidden; k++) {
        float z = sb2[k];
#pragma unroll 8
        for (int j = 0; j < kMlpHidden; j++) z += sW2[k * kMlpHidden + j] * h1[j];
        if (z > 0.f) m2 |= 1u << k;
        h2[k] = q16(fmaxf(z, 0.f));
    }
    float y = sb3[0];
    for (int k = 0; k < kMlpHidden; k++) y += sW3[k] * h2[k];
    const float e = valid ? y - tn : 0.f;
    const float dy = e / (float)batch;
    // backward
    for (int k = 0; k < kMlpHidden; k++) dz2[k] = ((m2 >> k) & 1u) ? dy * sW3[k] : 0.f;
    for (int j = 0; j < kMlpHidden; j++) {
        float dh = 0.f;
#pragma unroll 8
        for (int k = 0; k < kMlpHidden; k++) dh += sW2[k * kMlpHidden + j] * dz2[k];
        s_dz1[t * kH1 + j] = ((m1 >> j) & 1u) ? dh : 0.f;
    }
    for (int i = 0; i < kMlpIn; i++) s_x[t * 8 + i] = xq[i];
    s_dy[t] = dy;
    s_red[t] = 0.5f * e * e;
    __syncthreads();

    for (int p = t; p < kMlpWeights; p += kTB) {
        float acc = 0.f;
        if (p < kOffB1) {
            const int j = p / kMlpIn, i = p % kMlpIn;
            for (int r = 0; r < kTB; r++) acc += s_dz1[r * kH1 + j] * s_x[r * 8 + i];
        } else if (p < kOffW2) {
            const int j = p - kOffB1;
            for (int r = 0; r < kTB; r++) acc += s_dz1[r * kH1 + j];
        } else if (p < kOffB2) {
            const int k = (p - kOffW2) / kMlpHidden, j = (p - kOffW2) % kMlpHidden;
            for (int r = 0; r < kTB; r++) acc += s_dz2[r * kH1 + k] * s_h1[r * kH1 + j];
        } else if (p < kOffW3) {
            const int k = p - kOffB2;
            for (int r = 0; r < kTB; r++) acc += s_dz2[r * kH1 + k];
        } else if (p < kOffB3) {
            const int k = p - kOffW3;
            for (int r = 0; r < kTB; r++) acc += s_dy[r] * s_h2[r * kH1 + k];
        } else {
            for (int r = 0; r < kTB; r++) acc += s_dy[r];
        }
        partial[(long long)blockIdx.x * kMlpWeights + p] = acc;
    }
    for (int o = kTB / 2; o > 0; o >>= 1) {
        if (t < o) s_red[t] += s_red[t + o];
        __syncthreads();
    }
    if (t == 0) loss_part[blockIdx.x] = s_red[0];
}

// Sums the partial gradients in block order; optionally applies Adam.
__global__ void k_mlp_reduce(float* P, float* am, float* av, const float* __restrict__ partial, int nblocks,
                             const float* __restrict__ loss_part, float lr, float bc1, float bc2, float* out) {
    for (int p = threadIdx.x; p < kMlpWeights; p += blockDim.x) {
        float g = 0.f;
        for (int b = 0; b < nblocks; b++) g += partial[(long long)b * kMlpWeights + p];
        out[1 + p] = g;
        if (lr > 0.f) {
            const float m = 0.9f * am[p] + 0.1f * g;
            const float v = 0.999f * av[p] + 0.001f * g * g;
            am[p] = m;
            av[p] = v;
            P[p] -= lr * (m / bc1) / (sqrtf(v / bc2) + 1e-8f);
        }
    }
    if (threadIdx.x == 0) {
        float l = 0.f;
        for (int b = 0; b < nblocks; b++) l += loss_part[b];
        out[0] = l;
    }
}

// FP32 parameters -> per-lane BF16 fragments (layout in mlp.cuh). One warp.
__global__ void k_mlp_pack(const float* __restrict__ P, MlpNet* net) {
    const int lane = threadIdx.x, g = lane >> 2, q = lane & 3;
    auto W1 = [&](int n, int k) { return k < kMlpIn ? P[kOffW1 + n * kMlpIn + k] : 0.f; };
    auto W2 = [&](int n, int k) { return P[kOffW2 + n * kMlpHidden + k]; };
    auto W3 = [&](int k) { return g == 0 ? P[kOffW3 + k] : 0.f; };
    for (int nt = 0; nt < 4; nt++) net->frag[lane][kFragL1 + nt] = bf16x2(W1(8 * nt + g, 2 * q), W1(8 * nt + g, 2 * q + 1));
    for (int kt = 0; kt < 2; kt++)
        for (int nt = 0; nt < 4; nt++) {
            const int n = 8 * nt + g, k0 = 16 * kt + 2 * q;
            net->frag[lane][kFragL2 + (kt * 4 + nt) * 2] = bf16x2(W2(n, k0), W2(n, k0 + 1));
            net->frag[lane][kFragL2 + (kt * 4 + nt) * 2 + 1] = bf16x2(W2(n, k0 + 8), W2(n, k0 + 9));
        }
    for (int kt = 0; kt < 2; kt++) {
        const int k0 = 16 * kt + 2 * q;
        net->frag[lane][kFragL3 + 2 * kt] = bf16x2(W3(k0), W3(k0 + 1));
        net->frag[lane][kFragL3 + 2 * kt + 1] = bf16x2(W3(k0 + 8), W3(k0 + 9));
    }
    for (int nt = 0; nt < 4; nt++) {
        net->bias[lane][2 * nt] = P[kOffB1 + 8 * nt + 2 * q];
        net->bias[lane][2 * nt + 1] = P[kOffB1 + 8 * nt + 2 * q + 1];
        net->bias[lane][8 + 2 * nt] = P[kOffB2 + 8 * nt + 2 * q];
        net->bias[lane][8 + 2 * nt + 1] = P[kOffB2 + 8 * nt + 2 * q + 1];
    }
    if (lane < kMlpIn) {
        net->x_mean[lane] = P[kOffXMean + lane];
        net->x_inv_std[lane] = 1.0f / P[kOffXStd + lane];
    }
    if (lane == 0) {
        net->t_mean = P[kOffTMean];
        net->t_std = P[kOffTStd];
        net->gate = P[kOffGate];
        net->b3 = P[kOffB3];
    }
}

// Tensor-core inference over n faces; every thread of a block reaches the
// warp collective (blockDim is a multiple of 32, the tail is padded).
__global__ void k_mlp_infer(const MlpNet* __restrict__ net, const double* __restrict__ pairs, long long n,
                            double* guess, double* analytic, float* yout) {
    const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool valid = f < n;
    Prim<double> L = zero_prim<double>(), R = zero_prim<double>();
    L.rho = L.p = R.rho = R.p = 1.0;
    if (valid) {
        L = row_state(pairs + f * 6);
        R = row_state(pairs + f * 6 + 3);
    }
    float xn[kMlpIn];
    mlp_features(L, R, xn);
    for (int i = 0; i < kMlpIn; i++) xn[i] = (xn[i] - net->x_mean[i]) * net->x_inv_std[i];
    const float y = mlp_forward_warp(net, xn);
    if (!valid) return;
    const double a = analytic_guess(L, R);
    if (guess) guess[f] = mlp_guess_from(y, net->t_mean, net->t_std, net->gate, a);
    if (analytic) analytic[f] = a;
    if (yout) yout[f] = y;
}

int ensure_partial(dragon_mlp* m, int blocks) {
    if (blocks <= m->partial_blocks) return 0;
    if (m->partial) cudaFree(m->partial);
    if (m->loss_part) cudaFree(m->loss_part);
    m->partial = nullptr;
    m->loss_part = nullptr;
    m->partial_blocks = 0;
    CKM(cudaMalloc(&m->partial, sizeof(float) * (size_t)blocks * kMlpWeights));
    CKM(cudaMalloc(&m->loss_part, sizeof(float) * (size_t)blocks));
    m->partial_blocks = blocks;
    return 0;
}

// One gradient evaluation (+ optional Adam step) over batch samples.
int grad_pass(dragon_mlp* m, long long first, int contiguous, int batch, float lr) {
    const int blocks = (batch + kTB - 1) / kTB;
    int rc = ensure_partial(m, blocks);
    if (rc) return rc;
    const size_t smem = sizeof(float) * kGradSmemFloats;
    CKM(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long draw = contiguous ? 0 : m->batches++;
    k_mlp_grad<<<blocks, kTB, smem, m->stream>>>(m->P, m->X, m->T, m->n, first, contiguous, m->seed, draw, batch,
                                                 m->partial, m->loss_part);
    CKM(cudaGetLastError());
    float bc1 = 1.f, bc2 = 1.f;
    if (lr > 0.f) {
        m->adam_t++;
        bc1 = 1.f - std::pow(0.9f, (float)m->adam_t);
        bc2 = 1.f - std::pow(0.999f, (float)m->adam_t);
        m->net_dirty = true;
    }
    k_mlp_reduce<<<1, 1024, 0, m->stream>>>(m->P, m->adam_m, m->adam_v, m->partial, blocks, m->loss_part, lr, bc1, bc2,
                                            m->out);
    CKM(cudaGetLastError());
    return 0;
}

int pack_net(dragon_mlp* m) {
    if (!m->net_dirty) return 0;
    k_mlp_pack<<<1, 32, 0, m->stream>>>(m->P, m->net);
    CKM(cudaGetLastError());
    m->net_dirty = false;
    return 0;
}

}  // namespace

// Packed network of m on its device, synchronised (used by the grid runtime).
const MlpNet* dragon_mlp_packed_net(dragon_mlp* m) {
    if (!m || pack_net(m) || cudaStreamSynchronize(m->stream) != cudaSuccess) return nullptr;
    return m->net;
}

extern "C" {

int dragon_gpu_mlp_create(unsigned long long seed, dragon_mlp** out) {
    if (!out) return fail(DRAGON_GPU_EINVAL, "null argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(DRAGON_GPU_ECUDA, "no CUDA device available");
    dragon_mlp* m = new dragon_mlp();
    m->seed = seed;
    auto bad = [&](const char* what) {
        dragon_gpu_mlp_destroy(m);
        return fail(DRAGON_GPU_ECUDA, what);
    };
    cudaGetDevice(&m->device);
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return bad("cudaStreamCreate failed");
    if (cudaMalloc(&m->P, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&m->adam_m, sizeof(float) * kMlpWeights) != cudaSuccess ||
        cudaMalloc(&m->adam_v, sizeof(float) * kMlpWeights) != cudaSuccess ||
        cudaMalloc(&m->out, sizeof(float) * (kMlpWeights + 1)) != cudaSuccess ||
        cudaMalloc(&m->net, sizeof(MlpNet)) != cudaSuccess)
        return bad("cudaMalloc network failed");
    // He-uniform weights for the ReLU layers, Glorot-uniform for the output.
    std::vector<float> p(kMlpParams, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int count, double lim) {
        std::uniform_real_distribution<double> u(-lim, lim);
        for (int i = 0; i < count; i++) p[off + i] = (float)u(rng);
    };
    fill(kOffW1, kMlpHidden * kMlpIn, std::sqrt(6.0 / kMlpIn));
    fill(kOffW2, kMlpHidden * kMlpHidden, std::sqrt(6.0 / kMlpHidden));
    fill(kOffW3, kMlpHidden, std::sqrt(6.0 / (kMlpHidden + 1)));
    for (int i = 0; i < kMlpIn; i++) p[kOffXStd + i] = 1.f;
    p[kOffTStd] = 1.f;
    int rc = dragon_gpu_mlp_load(m, p.data(), kMlpParams);
    if (rc) { dragon_gpu_mlp_destroy(m); return rc; }
    *out = m;
    return 0;
}

int dragon_gpu_mlp_destroy(dragon_mlp* m) {
    if (!m) return 0;
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (void* p : {(void*)m->P, (void*)m->adam_m, (void*)m->adam_v, (void*)m->partial, (void*)m->loss_part,
                    (void*)m->out, (void*)m->net, (void*)m->X, (void*)m->T})
        if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return 0;
}

int dragon_gpu_mlp_load(dragon_mlp* m, const float* params, int n) {
    if (!m || !params || n != kMlpParams) return fail(DRAGON_GPU_EINVAL, "expected DRAGON_MLP_PARAMS floats");
    for (int i = 0; i < kMlpIn; i++)
        if (!(params[kOffXStd + i] > 0.f)) return fail(DRAGON_GPU_EINVAL, "feature standard deviations must be positive");
    if (!(params[kOffTStd] > 0.f)) return fail(DRAGON_GPU_EINVAL, "target standard deviation must be positive");
    CKM(cudaMemcpyAsync(m->P, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, m->stream));
    CKM(cudaMemsetAsync(m->adam_m, 0, sizeof(float) * kMlpWeights, m->stream));
    CKM(cudaMemsetAsync(m->adam_v, 0, sizeof(float) * kMlpWeights, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    m->adam_t = 0;
    m->net_dirty = true;
    return 0;
}

int dragon_gpu_mlp_save(dragon_mlp* m, float* params, int n) {
    if (!m || !params || n != kMlpParams) return fail(DRAGON_GPU_EINVAL, "expected DRAGON_MLP_PARAMS floats");
    CKM(cudaMemcpyAsync(params, m->P, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    return 0;
}

int dragon_gpu_mlp_add_samples(dragon_mlp* m, const double* rows, long long n, int on_device) {
    if (!m || n < 0 || (n > 0 && !rows)) return fail(DRAGON_GPU_EINVAL, "invalid samples");
    if (n == 0) return 0;
    if (m->n + n > m->cap) {
        long long cap = m->cap ? m->cap : 1 << 16;
        while (cap < m->n + n) cap *= 2;
        float *X = nullptr, *T = nullptr;
        CKM(cudaMalloc(&X, sizeof(float) * kMlpIn * cap));
        if (cudaMalloc(&T, sizeof(float) * cap) != cudaSuccess) {
            cudaFree(X);
            return fail(DRAGON_GPU_ECUDA, "cudaMalloc training set failed");
        }
        if (m->n) {
            CKM(cudaMemcpyAsync(X, m->X, sizeof(float) * kMlpIn * m->n, cudaMemcpyDeviceToDevice, m->stream));
            CKM(cudaMemcpyAsync(T, m->T, sizeof(float) * m->n, cudaMemcpyDeviceToDevice, m->stream));
        }
        CKM(cudaStreamSynchronize(m->stream));
        if (m->X) cudaFree(m->X);
        if (m->T) cudaFree(m->T);
        m->X = X;
        m->T = T;
        m->cap = cap;
    }
    const double* src = rows;
    double* tmp = nullptr;
    if (!on_device) {
        CKM(cudaMalloc(&tmp, sizeof(double) * kNewtonLogCols * n));
        CKM(cudaMemcpyAsync(tmp, rows, sizeof(double) * kNewtonLogCols * n, cudaMemcpyHostToDevice, m->stream));
        src = tmp;
    }
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    k_mlp_prepare<<<blocks, 256, 0, m->stream>>>(src, n, m->X + kMlpIn * m->n, m->T + m->n);
    cudaError_t e = cudaGetLastError();
    cudaError_t s = cudaStreamSynchronize(m->stream);
    if (tmp) cudaFree(tmp);
    if (e != cudaSuccess || s != cudaSuccess) return fail(DRAGON_GPU_ECUDA, "sample preparation failed");
    m->n += n;
    return 0;
}

long long dragon_gpu_mlp_sample_count(const dragon_mlp* m) { return m ? m->n : 0; }

int dragon_gpu_mlp_clear_samples(dragon_mlp* m) {
    if (!m) return fail(DRAGON_GPU_EINVAL, "null handle");
    m->n = 0;
    return 0;
}

int dragon_gpu_mlp_fit_normalisation(dragon_mlp* m) {
    if (!m || m->n < 2) return fail(DRAGON_GPU_EINVAL, "need at least two samples");
    k_mlp_stats<<<1, 1024, 0, m->stream>>>(m->X, m->T, m->n, m->P);
    CKM(cudaGetLastError());
    CKM(cudaStreamSynchronize(m->stream));
    m->net_dirty = true;
    return 0;
}

int dragon_gpu_mlp_features(dragon_mlp* m, long long first, long long n, float* x, float* t) {
    if (!m || first < 0 || n < 0 || first + n > m->n) return fail(DRAGON_GPU_EINVAL, "sample range out of bounds");
    if (x) CKM(cudaMemcpyAsync(x, m->X + kMlpIn * first, sizeof(float) * kMlpIn * n, cudaMemcpyDeviceToHost, m->stream));
    if (t) CKM(cudaMemcpyAsync(t, m->T + first, sizeof(float) * n, cudaMemcpyDeviceToHost, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    return 0;
}

int dragon_gpu_mlp_gradient(dragon_mlp* m, long long first, long long n, float* grad, float* loss) {
    if (!m || first < 0 || n < 1 || first + n > m->n || n > (1 << 22))
        return fail(DRAGON_GPU_EINVAL, "sample range out of bounds");
    int rc = grad_pass(m, first, 1, (int)n, 0.f);
    if (rc) return rc;
    std::vector<float> o(kMlpWeights + 1);
    CKM(cudaMemcpyAsync(o.data(), m->out, sizeof(float) * (kMlpWeights + 1), cudaMemcpyDeviceToHost, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    if (grad) std::memcpy(grad, o.data() + 1, sizeof(float) * kMlpWeights);
    if (loss) *loss = o[0] / (float)n;
    return 0;
}

int dragon_gpu_mlp_train(dragon_mlp* m, int steps, int batch, float lr, float* loss) {
    if (!m || steps < 0 || batch < 1 || batch > (1 << 22) || !(lr > 0.f)) return fail(DRAGON_GPU_EINVAL, "invalid training arguments");
    if (m->n < 1) return fail(DRAGON_GPU_EINVAL, "empty training set");
    for (int s = 0; s < steps; s++) {
        int rc = grad_pass(m, 0, 0, batch, lr);
        if (rc) return rc;
    }
    float l = 0.f;
    CKM(cudaMemcpyAsync(&l, m->out, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    if (loss) *loss = l / (float)batch;
    return 0;
}

int dragon_gpu_mlp_evaluate(dragon_mlp* m, long long first, long long n, float* rmse) {
    if (!m || first < 0 || n < 1 || first + n > m->n) return fail(DRAGON_GPU_EINVAL, "sample range out of bounds");
    double sum = 0.0;
    for (long long c = 0; c < n; c += 65536) {
        const int chunk = (int)std::min<long long>(65536, n - c);
        int rc = grad_pass(m, first + c, 1, chunk, 0.f);
        if (rc) return rc;
        float l = 0.f;
        CKM(cudaMemcpyAsync(&l, m->out, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        CKM(cudaStreamSynchronize(m->stream));
        sum += l;
    }
    float tstd = 1.f;
    CKM(cudaMemcpyAsync(&tstd, m->P + kOffTStd, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    if (rmse) *rmse = (float)(std::sqrt(2.0 * sum / (double)n) * tstd);
    return 0;
}

int dragon_gpu_mlp_set_gate(dragon_mlp* m, float gate) {
    if (!m || !(gate >= 0.f)) return fail(DRAGON_GPU_EINVAL, "gate must be non-negative");
    CKM(cudaMemcpyAsync(m->P + kOffGate, &gate, sizeof(float), cudaMemcpyHostToDevice, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    m->net_dirty = true;
    return 0;
}

int dragon_gpu_mlp_guess(dragon_mlp* m, const double* pairs, long long n, double* guess, double* analytic, float* y) {
    if (!m || n < 0 || (n > 0 && !pairs)) return fail(DRAGON_GPU_EINVAL, "invalid arguments");
    if (n == 0) return 0;
    int rc = pack_net(m);
    if (rc) return rc;
    double *dp = nullptr, *dg = nullptr, *da = nullptr;
    float* dy = nullptr;
    auto release = [&]() {
        for (void* p : {(void*)dp, (void*)dg, (void*)da, (void*)dy})
            if (p) cudaFree(p);
    };
    if (cudaMalloc(&dp, sizeof(double) * 6 * n) != cudaSuccess || cudaMalloc(&dg, sizeof(double) * n) != cudaSuccess ||
        cudaMalloc(&da, sizeof(double) * n) != cudaSuccess || cudaMalloc(&dy, sizeof(float) * n) != cudaSuccess) {
        release();
        return fail(DRAGON_GPU_ECUDA, "cudaMalloc inference buffers failed");
    }
    cudaMemcpyAsync(dp, pairs, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, m->stream);
    k_mlp_infer<<<(int)((n + 255) / 256), 256, 0, m->stream>>>(m->net, dp, n, dg, da, dy);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && guess) e = cudaMemcpyAsync(guess, dg, sizeof(double) * n, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess && analytic) e = cudaMemcpyAsync(analytic, da, sizeof(double) * n, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess && y) e = cudaMemcpyAsync(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost, m->stream);
    cudaError_t s = cudaStreamSynchronize(m->stream);
    release();
    if (e != cudaSuccess || s != cudaSuccess) return fail(DRAGON_GPU_ECUDA, "inference failed");
    return 0;
}

}  // extern "C"
