// k_mlp.cu — the learned kernel-class selector: matrix features and a small
// MLP (12 -> 64 -> 64 -> 6, ReLU, FP32) with its forward, backward and Adam
// kernels.
//
// No counterpart in the reference: its only "autotuner" is the (ngpu, q)
// sweep of test/dspmv_test.cu:314-332.  The MLP predicts, per kernel class,
// log2(t_class / t_best) of a plain launch from 12 features of the matrix;
// the selector takes the class with the smallest prediction.
//
// Determinism: the features come from integer accumulators (exact, so the
// order of the atomics does not matter), and every sum over samples in the
// backward pass runs in a fixed order, so training is bit-reproducible.
#include <math.h>
#include <stdint.h>

#include "../sbb_internal.h"

namespace sbb {

namespace {

// ---- features ---------------------------------------------------------------
// Integer accumulators over rows (index: meaning):
//   0: sum L^2   1: max L   2: empty rows   3: rows with L <= 4
//   4: rows with L > 32   5: nnz in rows with L > 128   6: sum of column spans
//   7: non-empty rows
constexpr int kAcc = 8;

__global__ void __launch_bounds__(256)
feature_acc_kernel(const int *__restrict__ rp, const int *__restrict__ col, int m,
                   unsigned long long *__restrict__ acc)
{
    unsigned long long a[kAcc] = {};
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < m;
         r += (long long)gridDim.x * blockDim.x) {
        const int lo = __ldg(rp + r), hi = __ldg(rp + r + 1);
        const unsigned long long L = hi > lo ? (unsigned long long)(hi - lo) : 0ull;
        a[0] += L * L;
        a[1] = L > a[1] ? L : a[1];
        a[2] += L == 0;
        a[3] += L <= 4;
        a[4] += L > 32;
        a[5] += L > 128 ? L : 0ull;
        if (L) {
            const int c0 = __ldg(col + lo), c1 = __ldg(col + hi - 1);
            a[6] += (unsigned long long)(c1 >= c0 ? c1 - c0 + 1 : c0 - c1 + 1);
            a[7] += 1;
        }
    }
#pragma unroll
    for (int k = 0; k < kAcc; ++k) {
        unsigned long long v = a[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
            v = k == 1 ? (u > v ? u : v) : v + u;
        }
        if ((threadIdx.x & 31) == 0) {
            if (k == 1)
                atomicMax(acc + 1, v);
            else if (v)
                atomicAdd(acc + k, v);
        }
    }
}

// The 12 features (all O(1) in magnitude before normalisation):
//   0 log2(1+m)  1 log2(1+n)  2 log2(1+nnz)  3 log2(1+mean L)
//   4 coefficient of variation of L  5 log2(1+max L)  6 log2(1+max L/mean L)
//   7 empty-row fraction  8 fraction of rows with L <= 4  9 fraction with L > 32
//   10 fraction of nnz in rows with L > 128  11 mean column span / n
__global__ void feature_final_kernel(const unsigned long long *__restrict__ acc, int m, int n,
                                     long long nnz, float *__restrict__ f)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double M = m > 0 ? m : 1, N = n > 0 ? n : 1, Z = (double)nnz;
    const double mean = Z / M;
    const double var = fmax((double)acc[0] / M - mean * mean, 0.0);
    const double mx = (double)acc[1];
    const double ne = acc[7] > 0 ? (double)acc[7] : 1.0;
    f[0] = (float)log2(1.0 + m);
    f[1] = (float)log2(1.0 + n);
    f[2] = (float)log2(1.0 + Z);
    f[3] = (float)log2(1.0 + mean);
    f[4] = (float)(mean > 0 ? sqrt(var) / mean : 0.0);
    f[5] = (float)log2(1.0 + mx);
    f[6] = (float)log2(1.0 + (mean > 0 ? mx / mean : 0.0));
    f[7] = (float)((double)acc[2] / M);
    f[8] = (float)((double)acc[3] / M);
    f[9] = (float)((double)acc[4] / M);
    f[10] = (float)(Z > 0 ? (double)acc[5] / Z : 0.0);
    f[11] = (float)((double)acc[6] / ne / N);
}

// ---- MLP --------------------------------------------------------------------
// Parameter blob (floats): mu[12], sd[12] (feature normalisation, fixed),
// W1[64][12], b1[64], W2[64][64], b2[64], W3[6][64], b3[6].
constexpr int F = kMlpFeatures, H = kMlpHidden, C = kMlpClasses;
constexpr int oMU = 0, oSD = F, oW1 = 2 * F, oB1 = oW1 + H * F, oW2 = oB1 + H, oB2 = oW2 + H * H,
              oW3 = oB2 + H, oB3 = oW3 + C * H, kParams = oB3 + C;
static_assert(kParams == kMlpParams, "parameter blob layout");

__device__ __forceinline__ float relu(float v) { return v > 0.f ? v : 0.f; }

// One thread per sample.  Stores the normalised input, both hidden layers
// (post-ReLU) and the outputs when the activation pointers are non-null.
__global__ void __launch_bounds__(128)
mlp_forward_kernel(const float *__restrict__ P, const float *__restrict__ X, int N,
                   float *__restrict__ Xn, float *__restrict__ H1, float *__restrict__ H2,
                   float *__restrict__ Y)
{
    __shared__ float s[kParams];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) s[i] = P[i];
    __syncthreads();
    const int nidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (nidx >= N) return;
    float x[F], h1[H], h2[H];
#pragma unroll
    for (int k = 0; k < F; ++k) {
        const float sd = s[oSD + k];
        x[k] = __fdiv_rn(__fsub_rn(X[nidx * F + k], s[oMU + k]), sd > 0.f ? sd : 1.f);
        if (Xn) Xn[nidx * F + k] = x[k];
    }
    for (int j = 0; j < H; ++j) {
        float z = s[oB1 + j];
#pragma unroll
        for (int k = 0; k < F; ++k) z = __fmaf_rn(s[oW1 + j * F + k], x[k], z);
        h1[j] = relu(z);
        if (H1) H1[nidx * H + j] = h1[j];
    }
    for (int j = 0; j < H; ++j) {
        float z = s[oB2 + j];
        for (int k = 0; k < H; ++k) z = __fmaf_rn(s[oW2 + j * H + k], h1[k], z);
        h2[j] = relu(z);
        if (H2) H2[nidx * H + j] = h2[j];
    }
    for (int c = 0; c < C; ++c) {
        float z = s[oB3 + c];
        for (int k = 0; k < H; ++k) z = __fmaf_rn(s[oW3 + c * H + k], h2[k], z);
        Y[nidx * C + c] = z;
    }
}

// Per-sample error terms of the loss
//   L = sum_n w_n sum_c (Y[n,c] - T[n,c])^2 / (C * sum_n w_n)
// dY = dL/dY, dZ2 = dL/d(pre-activation of layer 2), dZ1 likewise.
__global__ void __launch_bounds__(128)
mlp_delta_kernel(const float *__restrict__ P, int N, const float *__restrict__ H1,
                 const float *__restrict__ H2, const float *__restrict__ Y,
                 const float *__restrict__ T, const float *__restrict__ W, float inv_norm,
                 float *__restrict__ dY, float *__restrict__ dZ2, float *__restrict__ dZ1)
{
    __shared__ float s[kParams];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) s[i] = P[i];
    __syncthreads();
    const int nidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (nidx >= N) return;
    const float scale = __fmul_rn(2.f * inv_norm, W ? W[nidx] : 1.f);
    float dy[C], d2[H];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        dy[c] = __fmul_rn(scale, __fsub_rn(Y[nidx * C + c], T[nidx * C + c]));
        dY[nidx * C + c] = dy[c];
    }
    for (int k = 0; k < H; ++k) {
        float g = 0.f;
#pragma unroll
        for (int c = 0; c < C; ++c) g = __fmaf_rn(s[oW3 + c * H + k], dy[c], g);
        d2[k] = H2[nidx * H + k] > 0.f ? g : 0.f;
        dZ2[nidx * H + k] = d2[k];
    }
    for (int k = 0; k < H; ++k) {
        float g = 0.f;
        for (int j = 0; j < H; ++j) g = __fmaf_rn(s[oW2 + j * H + k], d2[j], g);
        dZ1[nidx * H + k] = H1[nidx * H + k] > 0.f ? g : 0.f;
    }
}

// One thread per parameter: the gradient as a sum over samples in order
// n = 0, 1, ..., N-1 (deterministic).  Normalisation entries get 0.
__global__ void __launch_bounds__(256)
mlp_wgrad_kernel(int N, const float *__restrict__ Xn, const float *__restrict__ H1,
                 const float *__restrict__ H2, const float *__restrict__ dY,
                 const float *__restrict__ dZ2, const float *__restrict__ dZ1,
                 float *__restrict__ G)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    const float *a = nullptr, *d = nullptr;
    int astride = 0, dstride = 0, ai = 0, di = 0;
    if (p < oW1) {
        G[p] = 0.f;
        return;
    } else if (p < oB1) {
        const int q = p - oW1;
        d = dZ1, dstride = H, di = q / F, a = Xn, astride = F, ai = q % F;
    } else if (p < oW2) {
        d = dZ1, dstride = H, di = p - oB1;
    } else if (p < oB2) {
        const int q = p - oW2;
        d = dZ2, dstride = H, di = q / H, a = H1, astride = H, ai = q % H;
    } else if (p < oW3) {
        d = dZ2, dstride = H, di = p - oB2;
    } else if (p < oB3) {
        const int q = p - oW3;
        d = dY, dstride = C, di = q / H, a = H2, astride = H, ai = q % H;
    } else {
        d = dY, dstride = C, di = p - oB3;
    }
    float g = 0.f;
    if (a)
        for (int n = 0; n < N; ++n) g = __fmaf_rn(d[n * dstride + di], a[n * astride + ai], g);
    else
        for (int n = 0; n < N; ++n) g = __fadd_rn(g, d[n * dstride + di]);
    G[p] = g;
}

// Loss (same normalisation as the deltas), summed in a fixed order by one
// block: thread i takes samples i, i+256, ...; then a shared-memory tree.
__global__ void __launch_bounds__(256)
mlp_loss_kernel(int N, const float *__restrict__ Y, const float *__restrict__ T,
                const float *__restrict__ W, float inv_norm, float *__restrict__ loss)
{
    __shared__ float s[256];
    float acc = 0.f;
    for (int nidx = threadIdx.x; nidx < N; nidx += 256) {
        float e = 0.f;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const float d = __fsub_rn(Y[nidx * C + c], T[nidx * C + c]);
            e = __fmaf_rn(d, d, e);
        }
        acc = __fmaf_rn(W ? W[nidx] : 1.f, e, acc);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] = __fadd_rn(s[threadIdx.x], s[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = __fmul_rn(s[0], inv_norm);
}

// Adam (bias-corrected); the normalisation entries stay fixed.
__global__ void mlp_adam_kernel(float *__restrict__ P, const float *__restrict__ G,
                                float *__restrict__ Mo, float *__restrict__ Vo, float lr,
                                float b1, float b2, float eps, float c1, float c2, float wd)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < oW1 || p >= kParams) return;
    const float g = __fmaf_rn(wd, P[p], G[p]);
    const float m = __fmaf_rn(b1, Mo[p], __fmul_rn(1.f - b1, g));
    const float v = __fmaf_rn(b2, Vo[p], __fmul_rn(__fmul_rn(1.f - b2, g), g));
    Mo[p] = m;
    Vo[p] = v;
    const float mh = __fdiv_rn(m, c1), vh = __fdiv_rn(v, c2);
    P[p] = __fsub_rn(P[p], __fdiv_rn(__fmul_rn(lr, mh), __fadd_rn(__fsqrt_rn(vh), eps)));
}

// The class with the smallest predicted score (first on ties), per sample.
__global__ void mlp_argmin_kernel(const float *__restrict__ Y, int N, int *__restrict__ cls)
{
    const int nidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (nidx >= N) return;
    int best = 0;
    for (int c = 1; c < C; ++c)
        if (Y[nidx * C + c] < Y[nidx * C + best]) best = c;
    cls[nidx] = best;
}

int blocks(long long work, int tpb) { return (int)((work + tpb - 1) / tpb); }

}  // namespace

void launch_features(const int *rp, const int *col, int m, int n, long long nnz,
                     unsigned long long *acc, float *feat, cudaStream_t s)
{
    cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * kAcc, s);
    if (m > 0) {
        int g = blocks(m, 256);
        if (g > 148 * 8) g = 148 * 8;
        feature_acc_kernel<<<g, 256, 0, s>>>(rp, col, m, acc);
    }
    feature_final_kernel<<<1, 32, 0, s>>>(acc, m, n, nnz, feat);
}

void launch_mlp_forward(const float *P, const float *X, int N, float *Xn, float *H1, float *H2,
                        float *Y, cudaStream_t s)
{
    if (N > 0) mlp_forward_kernel<<<blocks(N, 128), 128, 0, s>>>(P, X, N, Xn, H1, H2, Y);
}

void launch_mlp_backward(const float *P, int N, const float *Xn, const float *H1,
                         const float *H2, const float *Y, const float *T, const float *W,
                         float inv_norm, float *dY, float *dZ2, float *dZ1, float *G,
                         float *loss, cudaStream_t s)
{
    if (N <= 0) return;
    mlp_delta_kernel<<<blocks(N, 128), 128, 0, s>>>(P, N, H1, H2, Y, T, W, inv_norm, dY, dZ2, dZ1);
    mlp_wgrad_kernel<<<blocks(kParams, 256), 256, 0, s>>>(N, Xn, H1, H2, dY, dZ2, dZ1, G);
    if (loss) mlp_loss_kernel<<<1, 256, 0, s>>>(N, Y, T, W, inv_norm, loss);
}

void launch_mlp_adam(float *P, const float *G, float *M, float *V, int step, float lr, float wd,
                     cudaStream_t s)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    mlp_adam_kernel<<<blocks(kParams, 256), 256, 0, s>>>(P, G, M, V, lr, b1, b2, 1e-8f, c1, c2, wd);
}

void launch_mlp_argmin(const float *Y, int N, int *cls, cudaStream_t s)
{
    if (N > 0) mlp_argmin_kernel<<<blocks(N, 128), 128, 0, s>>>(Y, N, cls);
}

}  // namespace sbb
