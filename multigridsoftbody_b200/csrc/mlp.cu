// The learned smoother's network: parameters, tensor-core inference, and the
// trainer (hand-written backward + Adam).  C ABI in include/mgsb.h
// (mgsb_mlp_*); no counterpart in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/mgsb.h"
#include "kernels_mlp.cuh"
#include "mlp.hpp"

using namespace mgsb;

struct mgsb_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    float *prm = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr;
    uint8_t* img = nullptr;
    int adam_t = 0;
    // growable scratch
    float *grad_part = nullptr, *loss_part = nullptr;
    int part_cap = 0;
    int32_t* idx = nullptr;
    int idx_cap = 0;
    float *X = nullptr, *T = nullptr, *Y = nullptr;
    uint8_t* tiles = nullptr;
    size_t data_cap = 0;
    int32_t* werr = nullptr;
    ~mgsb_mlp();
};

mgsb_mlp::~mgsb_mlp() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (void* p : {(void*)prm, (void*)m, (void*)v, (void*)grad, (void*)loss, (void*)img, (void*)grad_part,
                    (void*)loss_part, (void*)idx, (void*)X, (void*)T, (void*)Y, (void*)tiles, (void*)werr})
        if (p) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
}

namespace {

mgsb_status mlp_err(mgsb_mlp* h, mgsb_status s, const char* fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return s;
}

#define MLP_CUDA(h, call)                                                                              \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return mlp_err(h, MGSB_CUDA_ERROR, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define MLP_TRY(expr)                      \
    do {                                   \
        mgsb_status s_ = (expr);           \
        if (s_ != MGSB_OK) return s_;      \
    } while (0)

size_t mlp_tc_smem() { return mlp_tc_smem_bytes(); }

mgsb_status ensure_data(mgsb_mlp* h, size_t n) {
    if (n <= h->data_cap) return MGSB_OK;
    for (void* p : {(void*)h->X, (void*)h->T, (void*)h->Y, (void*)h->tiles})
        if (p) cudaFree(p);
    const size_t ntiles = (n + kMlpTile - 1) / kMlpTile;
    MLP_CUDA(h, cudaMalloc(&h->X, n * kMlpIn * sizeof(float)));
    MLP_CUDA(h, cudaMalloc(&h->T, n * kMlpOut * sizeof(float)));
    MLP_CUDA(h, cudaMalloc(&h->Y, n * sizeof(float4)));
    MLP_CUDA(h, cudaMalloc(&h->tiles, ntiles * kTileBytes));
    h->data_cap = n;
    return MGSB_OK;
}

mgsb_status ensure_parts(mgsb_mlp* h, int nblk, int nidx) {
    if (nblk > h->part_cap) {
        if (h->grad_part) cudaFree(h->grad_part);
        if (h->loss_part) cudaFree(h->loss_part);
        MLP_CUDA(h, cudaMalloc(&h->grad_part, (size_t)nblk * kMlpParams * sizeof(float)));
        MLP_CUDA(h, cudaMalloc(&h->loss_part, (size_t)nblk * sizeof(float)));
        h->part_cap = nblk;
    }
    if (nidx > h->idx_cap) {
        if (h->idx) cudaFree(h->idx);
        MLP_CUDA(h, cudaMalloc(&h->idx, (size_t)nidx * sizeof(int32_t)));
        h->idx_cap = nidx;
    }
    return MGSB_OK;
}

mgsb_status repack(mgsb_mlp* h) {
    k_mlp_pack<<<(kMlpHid * kMlpHid + 255) / 256, 256, 0, h->stream>>>(h->prm, h->img);
    MLP_CUDA(h, cudaGetLastError());
    return MGSB_OK;
}

// Gradient of the mean squared error over `nb` samples (rows idx[] of X/T, or
// rows 0..nb-1 when idx is null) into h->grad, loss into h->loss.
mgsb_status launch_grad(mgsb_mlp* h, int nb, const int32_t* idx, const float* X, const float* T) {
    const int nblk = (nb + kTrainThreads - 1) / kTrainThreads;
    MLP_TRY(ensure_parts(h, nblk, 0));
    const float inv = 1.f / (float)(nb * kMlpOut);
    k_mlp_fwd_bwd<<<nblk, kTrainThreads, kTrainSmem, h->stream>>>(nb, idx, X, T, h->prm, h->grad_part, h->loss_part, inv);
    k_mlp_reduce<<<(kMlpParams + 255) / 256, 256, 0, h->stream>>>(nblk, h->grad_part, h->loss_part, inv, h->grad, h->loss);
    MLP_CUDA(h, cudaGetLastError());
    return MGSB_OK;
}

// Deterministic initialisation (uniform +-sqrt(6/(fan_in+fan_out)), zero biases).
void init_params(uint64_t seed, std::vector<float>& p) {
    p.assign(kMlpParams, 0.f);
    uint64_t z = seed;
    auto next = [&z]() {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        x ^= x >> 31;
        return (double)(x >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int fan_out, int fan_in) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for (int i = 0; i < fan_out * fan_in; ++i) p[off + i] = (float)((2.0 * next() - 1.0) * a);
    };
    fill(kOffW1, kMlpHid, kMlpIn);
    fill(kOffW2, kMlpHid, kMlpHid);
    fill(kOffW3, kMlpOut, kMlpHid);
}

}  // namespace

namespace mgsb {
const uint8_t* mlp_device_image(const mgsb_mlp* h) { return h ? h->img : nullptr; }
int mlp_device(const mgsb_mlp* h) { return h ? h->device : -1; }
}  // namespace mgsb

extern "C" {

int32_t mgsb_mlp_num_params(void) { return kMlpParams; }

mgsb_status mgsb_mlp_create(int32_t device, uint64_t seed, mgsb_mlp** out) {
    if (!out) return MGSB_INVALID_ARG;
    *out = nullptr;
    mgsb_mlp* h = new mgsb_mlp;
    h->device = device;
    auto fail = [&](mgsb_status s) {
        delete h;
        return s;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(MGSB_CUDA_ERROR);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(MGSB_CUDA_ERROR);
    const size_t pb = kMlpParams * sizeof(float);
    if (cudaMalloc(&h->prm, pb) || cudaMalloc(&h->m, pb) || cudaMalloc(&h->v, pb) || cudaMalloc(&h->grad, pb) ||
        cudaMalloc(&h->loss, sizeof(float)) || cudaMalloc(&h->img, kImgBytes) || cudaMalloc(&h->werr, sizeof(int32_t)))
        return fail(MGSB_OUT_OF_MEMORY);
    if (cudaFuncSetAttribute(k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem) ||
        cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_tc_smem()))
        return fail(MGSB_CUDA_ERROR);
    std::vector<float> p;
    init_params(seed, p);
    if (cudaMemcpy(h->prm, p.data(), pb, cudaMemcpyHostToDevice) || cudaMemset(h->m, 0, pb) || cudaMemset(h->v, 0, pb) ||
        cudaMemset(h->werr, 0, sizeof(int32_t)))
        return fail(MGSB_CUDA_ERROR);
    if (repack(h) != MGSB_OK || cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(MGSB_CUDA_ERROR);
    *out = h;
    return MGSB_OK;
}

mgsb_status mgsb_mlp_destroy(mgsb_mlp* h) {
    delete h;
    return MGSB_OK;
}

const char* mgsb_mlp_last_error(const mgsb_mlp* h) { return h ? h->err.c_str() : "null handle"; }

mgsb_status mgsb_mlp_set_params(mgsb_mlp* h, const float* params, int32_t n) {
    if (!h || !params || n != kMlpParams) return mlp_err(h, MGSB_INVALID_ARG, "expected %d parameters", kMlpParams);
    MLP_CUDA(h, cudaSetDevice(h->device));
    MLP_CUDA(h, cudaMemcpyAsync(h->prm, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MLP_CUDA(h, cudaMemsetAsync(h->m, 0, kMlpParams * sizeof(float), h->stream));
    MLP_CUDA(h, cudaMemsetAsync(h->v, 0, kMlpParams * sizeof(float), h->stream));
    h->adam_t = 0;
    MLP_TRY(repack(h));
    MLP_CUDA(h, cudaStreamSynchronize(h->stream));
    return MGSB_OK;
}

mgsb_status mgsb_mlp_get_params(mgsb_mlp* h, float* params, int32_t n) {
    if (!h || !params || n != kMlpParams) return mlp_err(h, MGSB_INVALID_ARG, "expected %d parameters", kMlpParams);
    MLP_CUDA(h, cudaSetDevice(h->device));
    MLP_CUDA(h, cudaMemcpyAsync(params, h->prm, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MLP_CUDA(h, cudaStreamSynchronize(h->stream));
    return MGSB_OK;
}

mgsb_status mgsb_mlp_forward(mgsb_mlp* h, const float* x, int32_t n, float* y) {
    if (!h || !x || !y || n < 0) return MGSB_INVALID_ARG;
    if (n == 0) return MGSB_OK;
    MLP_CUDA(h, cudaSetDevice(h->device));
    MLP_TRY(ensure_data(h, n));
    const int ntiles = (n + kMlpTile - 1) / kMlpTile;
    MLP_CUDA(h, cudaMemcpyAsync(h->X, x, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    k_mlp_tile_features<<<(ntiles * kMlpTile * kMlpInPad + 255) / 256, 256, 0, h->stream>>>(n, ntiles, h->X, h->tiles);
    MLP_CUDA(h, cudaMemsetAsync(h->werr, 0, sizeof(int32_t), h->stream));
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
    const int grid = std::min(ntiles, 2 * dev_sms);
    k_mlp_tc<<<grid, kMlpThreads, mlp_tc_smem(), h->stream>>>(n, ntiles, h->tiles, h->img, 0,
                                                             reinterpret_cast<float4*>(h->Y), nullptr, nullptr, h->werr);
    MLP_CUDA(h, cudaGetLastError());
    std::vector<float4> tmp(n);
    int32_t werr = 0;
    MLP_CUDA(h, cudaMemcpyAsync(tmp.data(), h->Y, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost, h->stream));
    MLP_CUDA(h, cudaMemcpyAsync(&werr, h->werr, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    MLP_CUDA(h, cudaStreamSynchronize(h->stream));
    if (werr) return mlp_err(h, MGSB_TIMEOUT, "tensor-core MLP: a bounded wait ran out");
    for (int i = 0; i < n; ++i) {
        y[3 * i] = tmp[i].x;
        y[3 * i + 1] = tmp[i].y;
        y[3 * i + 2] = tmp[i].z;
    }
    return MGSB_OK;
}

mgsb_status mgsb_mlp_loss_grad(mgsb_mlp* h, const float* x, const float* t, int32_t n, float* grad, float* loss) {
    if (!h || !x || !t || n <= 0) return MGSB_INVALID_ARG;
    MLP_CUDA(h, cudaSetDevice(h->device));
    MLP_TRY(ensure_data(h, n));
    MLP_CUDA(h, cudaMemcpyAsync(h->X, x, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MLP_CUDA(h, cudaMemcpyAsync(h->T, t, (size_t)n * kMlpOut * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MLP_TRY(launch_grad(h, n, nullptr, h->X, h->T));
    if (grad)
        MLP_CUDA(h, cudaMemcpyAsync(grad, h->grad, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    if (loss) MLP_CUDA(h, cudaMemcpyAsync(loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MLP_CUDA(h, cudaStreamSynchronize(h->stream));
    return MGSB_OK;
}

mgsb_status mgsb_mlp_train(mgsb_mlp* h, const float* x, const float* t, int64_t n, int32_t steps, int32_t batch,
                           float lr, uint64_t seed, float* losses) {
    if (!h || !x || !t || n <= 0 || steps <= 0 || batch <= 0 || n > INT32_MAX) return MGSB_INVALID_ARG;
    MLP_CUDA(h, cudaSetDevice(h->device));
    MLP_TRY(ensure_data(h, (size_t)n));
    MLP_CUDA(h, cudaMemcpyAsync(h->X, x, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MLP_CUDA(h, cudaMemcpyAsync(h->T, t, (size_t)n * kMlpOut * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    MLP_TRY(ensure_parts(h, (batch + kTrainThreads - 1) / kTrainThreads, batch));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float* hist = nullptr;   // loss of every step, read back once at the end
    if (losses) MLP_CUDA(h, cudaMalloc(&hist, (size_t)steps * sizeof(float)));
    struct Free {
        float* p;
        ~Free() { if (p) cudaFree(p); }
    } free_hist{hist};
    for (int s = 0; s < steps; ++s) {
        // cosine decay of the step size to 10 %
        const float lr_s = lr * (0.55f + 0.45f * std::cos(3.14159265f * (float)s / (float)steps));
        k_sample_indices<<<(batch + 255) / 256, 256, 0, h->stream>>>(batch, (int)n, seed, (uint64_t)s, h->idx);
        MLP_TRY(launch_grad(h, batch, h->idx, h->X, h->T));
        ++h->adam_t;
        const float bc1 = 1.f - std::pow(b1, (float)h->adam_t), bc2 = 1.f - std::pow(b2, (float)h->adam_t);
        k_adam<<<(kMlpParams + 255) / 256, 256, 0, h->stream>>>(h->prm, h->grad, h->m, h->v, lr_s, b1, b2, eps, bc1, bc2);
        if (losses) MLP_CUDA(h, cudaMemcpyAsync(hist + s, h->loss, sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    }
    MLP_CUDA(h, cudaGetLastError());
    MLP_TRY(repack(h));
    if (losses)
        MLP_CUDA(h, cudaMemcpyAsync(losses, hist, (size_t)steps * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MLP_CUDA(h, cudaStreamSynchronize(h->stream));
    return MGSB_OK;
}

}  // extern "C"
