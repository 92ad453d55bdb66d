// Training and inference kernels of the learned row-bin scheduler's MLP.
//
// Network (layout shared with the inference in sched.cu):
//   x = (f - mu) / sigma                        f: NFEAT bin features
//   h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2), out = W3 h2 + b3   (MLP_H hidden, NV outputs)
// out[v] predicts log2(nanoseconds per streamed B entry) of variant v on the
// bin; the scheduler picks argmin.  Loss: masked mean squared error over the
// (bin, variant) pairs that were measured.
//
// Training runs in one persistent CTA: parameters, gradients and Adam moments
// live in shared memory; every epoch the threads stride over the samples,
// backpropagate into the shared gradient with atomic adds, and then take one
// full-batch Adam step.  Sample counts are small (hundreds to a few thousand
// bins), so one CTA is the right size; no reference counterpart.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "gk_common.cuh"
#include "gk_device.cuh"
#include "gk_sched.cuh"

namespace gk {

constexpr int P_W1 = 0;
constexpr int P_B1 = P_W1 + MLP_H * NFEAT;
constexpr int P_W2 = P_B1 + MLP_H;
constexpr int P_B2 = P_W2 + MLP_H * MLP_H;
constexpr int P_W3 = P_B2 + MLP_H;
constexpr int P_B3 = P_W3 + NV * MLP_H;
constexpr int P_MU = P_B3 + NV;
constexpr int P_SG = P_MU + NFEAT;
constexpr int NTRAIN = P_MU;  // trainable parameters (mu/sigma are set from the data)
constexpr int MLP_THREADS = 256;

__device__ void mlp_forward(const float *w, const float *f, float *x, float *h1, float *h2, float *out) {
    for (int i = 0; i < NFEAT; ++i) x[i] = (f[i] - w[P_MU + i]) / w[P_SG + i];
    for (int j = 0; j < MLP_H; ++j) {
        float a = w[P_B1 + j];
        for (int i = 0; i < NFEAT; ++i) a += w[P_W1 + j * NFEAT + i] * x[i];
        h1[j] = a > 0.f ? a : 0.f;
    }
    for (int j = 0; j < MLP_H; ++j) {
        float a = w[P_B2 + j];
        for (int i = 0; i < MLP_H; ++i) a += w[P_W2 + j * MLP_H + i] * h1[i];
        h2[j] = a > 0.f ? a : 0.f;
    }
    for (int v = 0; v < NV; ++v) {
        float a = w[P_B3 + v];
        for (int i = 0; i < MLP_H; ++i) a += w[P_W3 + v * MLP_H + i] * h2[i];
        out[v] = a;
    }
}

// The same network for one warp, outputs 0 and 1 only (the BC level shapes):
// lane j computes hidden unit j of each layer; every sum runs in the order of
// mlp_forward's (inputs of a unit in index order, each gathered from its lane),
// so the outputs are the same floats.  Call with all 32 lanes.
__device__ void mlp_forward_warp2(const float *w, const float *f, float *o0, float *o1) {
    static_assert(MLP_H == 32, "one hidden unit per lane");
    const int j = threadIdx.x & 31;
    float x[NFEAT];
#pragma unroll
    for (int i = 0; i < NFEAT; ++i) x[i] = (f[i] - w[P_MU + i]) / w[P_SG + i];
    float a = w[P_B1 + j];
#pragma unroll
    for (int i = 0; i < NFEAT; ++i) a += w[P_W1 + j * NFEAT + i] * x[i];
    const float h1 = a > 0.f ? a : 0.f;
    a = w[P_B2 + j];
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i) a += w[P_W2 + j * MLP_H + i] * __shfl_sync(0xFFFFFFFFu, h1, i);
    const float h2 = a > 0.f ? a : 0.f;
    const int v = j < 2 ? j : 0;
    a = w[P_B3 + v];
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i) a += w[P_W3 + v * MLP_H + i] * __shfl_sync(0xFFFFFFFFu, h2, i);
    *o0 = __shfl_sync(0xFFFFFFFFu, a, 0);
    *o1 = __shfl_sync(0xFFFFFFFFu, a, 1);
}

// Adds d(loss)/d(params) of one sample into g (shared memory, atomics) and
// returns the sample's squared-error sum.  scale = 1 / (number of measured pairs).
__device__ float mlp_backward(const float *w, const float *f, const float *y, const float *mask, float scale,
                              float *g) {
    float x[NFEAT], h1[MLP_H], h2[MLP_H], out[NV], dout[NV], dh2[MLP_H], dh1[MLP_H];
    mlp_forward(w, f, x, h1, h2, out);
    float se = 0.f;
    for (int v = 0; v < NV; ++v) {
        const float e = mask[v] > 0.f ? out[v] - y[v] : 0.f;
        se += e * e;
        dout[v] = 2.f * e * scale;
    }
    for (int v = 0; v < NV; ++v) {
        if (dout[v] == 0.f) continue;
        atomicAdd(g + P_B3 + v, dout[v]);
        for (int i = 0; i < MLP_H; ++i) atomicAdd(g + P_W3 + v * MLP_H + i, dout[v] * h2[i]);
    }
    for (int i = 0; i < MLP_H; ++i) {
        float a = 0.f;
        for (int v = 0; v < NV; ++v) a += w[P_W3 + v * MLP_H + i] * dout[v];
        dh2[i] = h2[i] > 0.f ? a : 0.f;
    }
    for (int j = 0; j < MLP_H; ++j) {
        if (dh2[j] == 0.f) continue;
        atomicAdd(g + P_B2 + j, dh2[j]);
        for (int i = 0; i < MLP_H; ++i) atomicAdd(g + P_W2 + j * MLP_H + i, dh2[j] * h1[i]);
    }
    for (int i = 0; i < MLP_H; ++i) {
        float a = 0.f;
        for (int j = 0; j < MLP_H; ++j) a += w[P_W2 + j * MLP_H + i] * dh2[j];
        dh1[i] = h1[i] > 0.f ? a : 0.f;
    }
    for (int j = 0; j < MLP_H; ++j) {
        if (dh1[j] == 0.f) continue;
        atomicAdd(g + P_B1 + j, dh1[j]);
        for (int i = 0; i < NFEAT; ++i) atomicAdd(g + P_W1 + j * NFEAT + i, dh1[j] * x[i]);
    }
    return se;
}

__global__ void __launch_bounds__(MLP_THREADS) k_mlp_loss_grad(const float *w_in, const float *X, const float *Y,
                                                               const float *M, int n, float inv_count, float *loss,
                                                               float *grad) {
    __shared__ float w[MLP_SIZE];
    __shared__ float g[MLP_SIZE];
    __shared__ float red[MLP_THREADS / 32];
    for (int i = threadIdx.x; i < MLP_SIZE; i += blockDim.x) {
        w[i] = w_in[i];
        g[i] = 0.f;
    }
    __syncthreads();
    float se = 0.f;
    for (int s = threadIdx.x; s < n; s += blockDim.x)
        se += mlp_backward(w, X + s * NFEAT, Y + s * NV, M + s * NV, inv_count, g);
    const float tot = block_sum(se, red);
    __syncthreads();
    for (int i = threadIdx.x; i < MLP_SIZE; i += blockDim.x) grad[i] = g[i];
    if (threadIdx.x == 0) *loss = tot * inv_count;
}

// Full-batch Adam (Kingma & Ba, ICLR 2015) for `epochs` steps, all in one CTA.
__global__ void __launch_bounds__(MLP_THREADS) k_mlp_train(float *w_io, const float *X, const float *Y, const float *M,
                                                           int n, float inv_count, int epochs, float lr,
                                                           float *loss_trace) {
    __shared__ float w[MLP_SIZE];
    __shared__ float g[MLP_SIZE];
    __shared__ float m1[NTRAIN];
    __shared__ float m2[NTRAIN];
    __shared__ float red[MLP_THREADS / 32];
    for (int i = threadIdx.x; i < MLP_SIZE; i += blockDim.x) {
        w[i] = w_io[i];
        if (i < NTRAIN) m1[i] = m2[i] = 0.f;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float b1t = 1.f, b2t = 1.f;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int i = threadIdx.x; i < MLP_SIZE; i += blockDim.x) g[i] = 0.f;
        __syncthreads();
        float se = 0.f;
        for (int s = threadIdx.x; s < n; s += blockDim.x)
            se += mlp_backward(w, X + s * NFEAT, Y + s * NV, M + s * NV, inv_count, g);
        const float tot = block_sum(se, red);
        if (threadIdx.x == 0 && loss_trace) loss_trace[ep] = tot * inv_count;
        __syncthreads();
        b1t *= b1;
        b2t *= b2;
        for (int i = threadIdx.x; i < NTRAIN; i += blockDim.x) {
            const float gi = g[i];
            m1[i] = b1 * m1[i] + (1.f - b1) * gi;
            m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
            const float mh = m1[i] / (1.f - b1t), vh = m2[i] / (1.f - b2t);
            w[i] -= lr * mh / (sqrtf(vh) + eps);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < MLP_SIZE; i += blockDim.x) w_io[i] = w[i];
}

__global__ void k_mlp_forward(const float *w, const float *X, int n, float *out) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float x[NFEAT], h1[MLP_H], h2[MLP_H], o[NV];
        mlp_forward(w, X + s * NFEAT, x, h1, h2, o);
        for (int v = 0; v < NV; ++v) out[s * NV + v] = o[v];
    }
}

struct MlpData {
    float *w, *X, *Y, *M, *out;
};

static int upload(const float *w, const float *X, const float *Y, const float *M, int n, MlpData &d, Scratch &scr,
                  cudaStream_t s) {
    GK_CHECK(scr.alloc(&d.w, MLP_SIZE));
    GK_CHECK(scr.alloc(&d.X, (size_t)n * NFEAT + 1));
    GK_CUDA(cudaMemcpyAsync(d.w, w, sizeof(float) * MLP_SIZE, cudaMemcpyHostToDevice, s));
    GK_CUDA(cudaMemcpyAsync(d.X, X, sizeof(float) * n * NFEAT, cudaMemcpyHostToDevice, s));
    if (Y) {
        GK_CHECK(scr.alloc(&d.Y, (size_t)n * NV + 1));
        GK_CHECK(scr.alloc(&d.M, (size_t)n * NV + 1));
        GK_CUDA(cudaMemcpyAsync(d.Y, Y, sizeof(float) * n * NV, cudaMemcpyHostToDevice, s));
        GK_CUDA(cudaMemcpyAsync(d.M, M, sizeof(float) * n * NV, cudaMemcpyHostToDevice, s));
    }
    return GK_OK;
}

static float inv_measured(const float *M, int n) {
    double c = 0;
    for (int i = 0; i < n * NV; ++i) c += M[i] > 0.f ? 1.0 : 0.0;
    return c > 0 ? static_cast<float>(1.0 / c) : 0.f;
}

}  // namespace gk

using namespace gk;

extern "C" {

int gk_mlp_loss_grad(const float *w, const float *X, const float *Y, const float *mask, int n, float *loss,
                     float *grad, void *stream) {
    if (!w || !X || !Y || !mask || !loss || !grad || n < 1) return fail(GK_ERR_ARG, "gk_mlp_loss_grad: bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    MlpData d;
    GK_CHECK(upload(w, X, Y, mask, n, d, scr, s));
    float *dl, *dg;
    GK_CHECK(scr.alloc(&dl, 1));
    GK_CHECK(scr.alloc(&dg, MLP_SIZE));
    k_mlp_loss_grad<<<1, MLP_THREADS, 0, s>>>(d.w, d.X, d.Y, d.M, n, inv_measured(mask, n), dl, dg);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    GK_CUDA(cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaMemcpyAsync(grad, dg, sizeof(float) * MLP_SIZE, cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

int gk_mlp_train(float *w, const float *X, const float *Y, const float *mask, int n, int epochs, float lr,
                 float *loss_trace, void *stream) {
    if (!w || !X || !Y || !mask || n < 1 || epochs < 0) return fail(GK_ERR_ARG, "gk_mlp_train: bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    MlpData d;
    GK_CHECK(upload(w, X, Y, mask, n, d, scr, s));
    float *trace = nullptr;
    if (loss_trace && epochs > 0) GK_CHECK(scr.alloc(&trace, epochs));
    k_mlp_train<<<1, MLP_THREADS, 0, s>>>(d.w, d.X, d.Y, d.M, n, inv_measured(mask, n), epochs, lr, trace);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    GK_CUDA(cudaMemcpyAsync(w, d.w, sizeof(float) * MLP_SIZE, cudaMemcpyDeviceToHost, s));
    if (trace) GK_CUDA(cudaMemcpyAsync(loss_trace, trace, sizeof(float) * epochs, cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

int gk_mlp_forward(const float *w, const float *X, int n, float *out, void *stream) {
    if (!w || !X || !out || n < 1) return fail(GK_ERR_ARG, "gk_mlp_forward: bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scr(s);
    MlpData d;
    GK_CHECK(upload(w, X, nullptr, nullptr, n, d, scr, s));
    float *dout;
    GK_CHECK(scr.alloc(&dout, (size_t)n * NV));
    k_mlp_forward<<<(n + 127) / 128, 128, 0, s>>>(d.w, d.X, n, dout);
    note_launches(1);
    GK_CUDA(cudaGetLastError());
    GK_CUDA(cudaMemcpyAsync(out, dout, sizeof(float) * n * NV, cudaMemcpyDeviceToHost, s));
    GK_CUDA(cudaStreamSynchronize(s));
    return GK_OK;
}

}  // extern "C"
