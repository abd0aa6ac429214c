// common.cuh — device helpers shared by the SpMV kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sbb {

// Streaming (read-once) loads: evict-first, no L1 allocation, so the col/val
// streams do not push x out of L2.
__device__ __forceinline__ int ld_stream(const int *p) { return __ldcs(p); }
__device__ __forceinline__ int4 ld_stream(const int4 *p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ double2 ld_stream(const double2 *p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4 *p) { return __ldcs(p); }

// x is gathered through the read-only path and kept in L2.
template <typename T>
__device__ __forceinline__ T ld_x(const T *p) { return __ldg(p); }

// L2 cache-hint policies: x (gathered many times) is kept, streams are
// evicted first.
__device__ __forceinline__ uint64_t l2_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double ld_keep(const double *p, uint64_t pol)
{
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_keep(const float *p, uint64_t pol)
{
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
// y read and write with a streaming policy (y is touched once per SpMV).
__device__ __forceinline__ double ld_y(const double *p, uint64_t pol)
{
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_y(double *p, double v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}

// Column check: out-of-range indices read nothing, contribute 0 and raise the
// status bit (the host turns it into an error code).
template <typename T>
__device__ __forceinline__ T gather_x(const T *x, int c, int n, unsigned &bad)
{
    if ((unsigned)c < (unsigned)n) return ld_x(x + c);
    bad = 1u;
    return T(0);
}

// Per-value products for the two storage forms.
//   FP64: the product itself, rounded.
//   FP32 storage: the product of two floats taken in FP64, where it is exact
//         (24 + 24 significand bits fit in 53).
struct ProdF64 {
    using V = double;
    using P = double;
    __device__ __forceinline__ static P make(double v, double xv) { return __dmul_rn(v, xv); }
};
struct ProdF32 {
    using V = float;
    using P = double;
    __device__ __forceinline__ static P make(float v, float xv)
    {
        return __dmul_rn((double)v, (double)xv);  // exact
    }
};

// Running row-segment sums, in FP64 for both storage forms.  For FP32
// storage every product is exact, so the only rounding in a segment sum is
// that of the FP64 additions: the form is compensated by construction, to
// far below FP32's own rounding (a TwoSum-compensated FP32 sum would cost a
// chain of about ten dependent FP32 operations per nnz, and that chain, not
// the bytes, bounded the kernel's speed on B200).
struct AccF64 {
    double s;
    __device__ __forceinline__ void zero() { s = 0.0; }
    __device__ __forceinline__ void add(double p) { s = __dadd_rn(s, p); }
    // s + v*x with one rounding (the vector and tiled kernels' step)
    __device__ __forceinline__ void mac(double v, double x) { s = __fma_rn(v, x, s); }
    __device__ __forceinline__ double get() const { return s; }
};
struct AccF32 {
    double s;
    __device__ __forceinline__ void zero() { s = 0.0; }
    __device__ __forceinline__ void add(double p) { s = __dadd_rn(s, p); }
    // s + v*x with one rounding; v*x is exact in FP64, so this rounds once
    __device__ __forceinline__ void mac(float v, float x) { s = __fma_rn((double)v, (double)x, s); }
    __device__ __forceinline__ double get() const { return s; }
};
// FP32 lane sums (the tiled kernel only, sigma <= 8): a lane's run of at
// most sigma consecutive products of one row is summed by an FP32 fma chain
// and widened to FP64 once, where the warp scan, the carries and the alpha /
// beta update take over.  A run of k <= 8 terms is within k * 2^-24 of its
// exact sum relative to sum |v*x| (the chain's first step rounds the
// product, each later one the running sum); with the rounding of val and x
// to float that bounds a row's error by 10 * 2^-24 ~ 6e-7 of sum_j |a_ij x_j|.
// Per nnz: one FP32 fma instead of two float-to-double conversions and an
// FP64 fma.
struct AccF32Lane {
    float s;
    __device__ __forceinline__ void zero() { s = 0.0f; }
    __device__ __forceinline__ void mac(float v, float x) { s = __fmaf_rn(v, x, s); }
    __device__ __forceinline__ double get() const { return (double)s; }
};

// The y update alpha*sum + beta*y as fma(alpha, sum, beta*y); alpha*sum
// alone when beta == 0 (y is then not read: the cuSPARSE convention).  The
// FP64 arithmetic of every kernel is written with explicit-rounding
// intrinsics (products __dmul_rn, sums __dadd_rn, multiply-adds and this
// update __fma_rn),
// which the compiler never fuses or splits, so the same data gives the same
// bits in every kernel that runs a given reduction order (a standalone launch
// and the batched launch in particular).
__device__ __forceinline__ double y_update(double alpha, double sum, double beta, double yv)
{
    return beta == 0.0 ? __dmul_rn(alpha, sum) : __fma_rn(alpha, sum, __dmul_rn(beta, yv));
}
// Same, with y read (only when beta != 0) and written under a streaming L2
// policy.
__device__ __forceinline__ void write_y(double *yp, double alpha, double sum, double beta,
                                        uint64_t pol)
{
    st_y(yp, y_update(alpha, sum, beta, beta == 0.0 ? 0.0 : ld_y(yp, pol)), pol);
}

// Programmatic dependent launch (sm_90+): a kernel launched with the
// programmatic-serialization attribute may start before the kernel ahead of
// it in the stream has finished; grid_dependency_wait() blocks until that
// grid has completed and its memory operations are visible.
// allow_dependent_launch() lets the next such kernel be scheduled as soon as
// every block of this grid has executed it (each block's exit counts too).
__device__ __forceinline__ void grid_dependency_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void allow_dependent_launch()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace sbb
