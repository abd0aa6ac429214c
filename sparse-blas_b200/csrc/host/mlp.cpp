// mlp.cpp — C ABI of the learned class selector (kernels in k_mlp.cu).
#include <cuda_runtime.h>

#include <string>

#include "../sbb_internal.h"

using namespace sbb;

static_assert(kMlpParams == SBB_MLP_PARAMS, "public and internal parameter counts differ");
static_assert(kMlpFeatures == SBB_MLP_FEATURES, "public and internal feature counts differ");

namespace {

// Device scratch of one call, freed stream-ordered when the call returns.
struct Scratch {
    cudaStream_t s;
    void *p = nullptr;
    explicit Scratch(cudaStream_t st) : s(st) {}
    bool get(size_t bytes)
    {
        if (dev_malloc_async(&p, bytes ? bytes : 16, s) != cudaSuccess) {
            set_error("selector: device allocation failed");
            p = nullptr;
            return false;
        }
        return true;
    }
    ~Scratch()
    {
        if (p) cudaFreeAsync(p, s);
    }
};

struct Acts {  // activations and error terms of N samples, carved from one block
    float *xn, *h1, *h2, *y, *dy, *dz2, *dz1, *loss;
    static size_t floats(int N)
    {
        return (size_t)N * (kMlpFeatures + 4 * kMlpHidden + 2 * kMlpClasses) + 32;
    }
    explicit Acts(float *base, int N)
    {
        float *p = base;
        xn = p, p += (size_t)N * kMlpFeatures;
        h1 = p, p += (size_t)N * kMlpHidden;
        h2 = p, p += (size_t)N * kMlpHidden;
        y = p, p += (size_t)N * kMlpClasses;
        dy = p, p += (size_t)N * kMlpClasses;
        dz2 = p, p += (size_t)N * kMlpHidden;
        dz1 = p, p += (size_t)N * kMlpHidden;
        loss = p;
    }
};

// 1 / (classes * sum of sample weights), read back once (the weights are
// fixed for a call).
int inv_norm_of(const float *d_w, int N, cudaStream_t s, float *out)
{
    double sw = N;
    if (d_w) {
        std::string err;
        float *h = new float[N];
        cudaError_t e = cudaMemcpyAsync(h, d_w, sizeof(float) * N, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            delete[] h;
            set_error(std::string("selector: weights copy: ") + cudaGetErrorString(e));
            return SBB_ERR_CUDA;
        }
        sw = 0.0;
        for (int i = 0; i < N; i++) sw += h[i];
        delete[] h;
        if (!(sw > 0.0)) {
            set_error("selector: sample weights must sum to a positive number");
            return SBB_ERR_ARG;
        }
    }
    *out = (float)(1.0 / (kMlpClasses * sw));
    return SBB_OK;
}

}  // namespace

extern "C" {

int sbb_features(int m, int n, int nnz, const int *d_rowptr, const int *d_col, float *d_feat,
                 void *stream)
{
    if (m < 0 || n < 0 || nnz < 0 || !d_rowptr || !d_feat || (nnz > 0 && !d_col)) {
        set_error("bad sbb_features arguments");
        return SBB_ERR_ARG;
    }
    auto s = static_cast<cudaStream_t>(stream);
    Scratch acc(s);
    if (!acc.get(sizeof(unsigned long long) * 8)) return SBB_ERR_NOMEM;
    launch_features(d_rowptr, d_col, m, n, nnz, static_cast<unsigned long long *>(acc.p), d_feat,
                    s);
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

int sbb_mlp_forward(const float *d_params, const float *d_x, int N, float *d_y, void *stream)
{
    if (!d_params || N < 0 || (N > 0 && (!d_x || !d_y))) {
        set_error("bad sbb_mlp_forward arguments");
        return SBB_ERR_ARG;
    }
    launch_mlp_forward(d_params, d_x, N, nullptr, nullptr, nullptr, d_y,
                       static_cast<cudaStream_t>(stream));
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

int sbb_mlp_grad(const float *d_params, const float *d_x, const float *d_t, const float *d_w,
                 int N, float *d_grad, float *d_loss, void *stream)
{
    if (!d_params || !d_grad || N <= 0 || !d_x || !d_t) {
        set_error("bad sbb_mlp_grad arguments");
        return SBB_ERR_ARG;
    }
    auto s = static_cast<cudaStream_t>(stream);
    float inv = 0.f;
    int rc = inv_norm_of(d_w, N, s, &inv);
    if (rc != SBB_OK) return rc;
    Scratch mem(s);
    if (!mem.get(sizeof(float) * Acts::floats(N))) return SBB_ERR_NOMEM;
    Acts a(static_cast<float *>(mem.p), N);
    launch_mlp_forward(d_params, d_x, N, a.xn, a.h1, a.h2, a.y, s);
    launch_mlp_backward(d_params, N, a.xn, a.h1, a.h2, a.y, d_t, d_w, inv, a.dy, a.dz2, a.dz1,
                        d_grad, d_loss, s);
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

int sbb_mlp_train(float *d_params, const float *d_x, const float *d_t, const float *d_w, int N,
                  int steps, float lr, float wd, float *d_loss_hist, void *stream)
{
    if (!d_params || N <= 0 || !d_x || !d_t || steps < 0 || !(lr > 0.f) || wd < 0.f) {
        set_error("bad sbb_mlp_train arguments");
        return SBB_ERR_ARG;
    }
    auto s = static_cast<cudaStream_t>(stream);
    float inv = 0.f;
    int rc = inv_norm_of(d_w, N, s, &inv);
    if (rc != SBB_OK) return rc;
    Scratch mem(s);
    if (!mem.get(sizeof(float) * (Acts::floats(N) + 3 * (size_t)kMlpParams))) return SBB_ERR_NOMEM;
    Acts a(static_cast<float *>(mem.p), N);
    float *g = static_cast<float *>(mem.p) + Acts::floats(N);
    float *mo = g + kMlpParams, *vo = mo + kMlpParams;
    SBB_CUDA(cudaMemsetAsync(mo, 0, sizeof(float) * 2 * kMlpParams, s));
    for (int k = 1; k <= steps; k++) {
        launch_mlp_forward(d_params, d_x, N, a.xn, a.h1, a.h2, a.y, s);
        launch_mlp_backward(d_params, N, a.xn, a.h1, a.h2, a.y, d_t, d_w, inv, a.dy, a.dz2,
                            a.dz1, g, d_loss_hist ? d_loss_hist + (k - 1) : nullptr, s);
        launch_mlp_adam(d_params, g, mo, vo, k, lr, wd, s);
    }
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

int sbb_mlp_select(const float *d_params, int m, int n, int nnz, const int *d_rowptr,
                   const int *d_col, int *cls, void *stream)
{
    if (!d_params || !cls || m < 0 || n < 0 || nnz < 0 || !d_rowptr || (nnz > 0 && !d_col)) {
        set_error("bad sbb_mlp_select arguments");
        return SBB_ERR_ARG;
    }
    auto s = static_cast<cudaStream_t>(stream);
    Scratch mem(s);
    // acc (8 words) | features (12) | scores (6) | class (1)
    if (!mem.get(64 + sizeof(float) * 32)) return SBB_ERR_NOMEM;
    auto *acc = static_cast<unsigned long long *>(mem.p);
    float *feat = reinterpret_cast<float *>(static_cast<char *>(mem.p) + 64);
    float *y = feat + kMlpFeatures;
    int *dcls = reinterpret_cast<int *>(y + 16);
    launch_features(d_rowptr, d_col, m, n, nnz, acc, feat, s);
    launch_mlp_forward(d_params, feat, 1, nullptr, nullptr, nullptr, y, s);
    launch_mlp_argmin(y, 1, dcls, s);
    SBB_CUDA(cudaMemcpyAsync(cls, dcls, sizeof(int), cudaMemcpyDeviceToHost, s));
    SBB_CUDA(cudaStreamSynchronize(s));
    return SBB_OK;
}

}  // extern "C"
