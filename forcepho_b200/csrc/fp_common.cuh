// fp_common.cuh -- shared device/host helpers of the B200 likelihood library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/forcepho_b200.h"

// ---- error reporting (capi.cu) ------------------------------------------
int fp_set_error(int code, const char *fmt, ...);
int fp_check_cuda(cudaError_t err, const char *what);
int fp_sm_count(int *out);

// ---- constants -------------------------------------------------------------
// exp(-E/2) = 2^(c E) with c = -log2(e)/2: the exponent scale folded into the
// per-Gaussian inverse covariance so the pixel loops feed ex2 directly.
#define FP_EXP2_SCALE (-0.72134752044448170368)
// 1 / (24 c^2): turns (c vx)^2 + (c vy)^2 back into (vx^2 + vy^2) / 24.
#define FP_C24 (1.0 / (24.0 * 0.72134752044448170368 * 0.72134752044448170368))
// MAX_EXP_ARG on the scaled axis: E > 36  <=>  c E < 36 c.
#define FP_CUT_SCALED ((float)(MAX_EXP_ARG * -0.72134752044448170368))

#define FP_THREADS 256              // threads per tile CTA
#define FP_WARPS (FP_THREADS / 32)
#define FP_CHUNK 256                // Gaussians staged in shared memory at a time
#define FP_RUN 32                   // FP32 run length before flushing to FP64

// device status word bits: FP_STATUS_* in include/forcepho_b200.h

// ---- workspace layout (tiled path) -----------------------------------------
// [0, 256)                        : control block (queue counter, status)
// gauss_fwd  float4[2*n_gauss]    : (xc, yc, c fxx, c fxy), (c fyy, amp k0, amp C24, k0)
// gauss_box  float4[n_gauss]      : xmin, xmax, ymin, ymax of the E <= 36 box
// gauss_ctr  float2[n_gauss]      : xc - (float)xc, yc - (float)yc: what the FP32 centre lost
// gauss_jac  double[FP_JAC*n_gauss]
// partials   double[n_partials]
#define FP_JAC 20                   // amp, fxx, fxy, fyy, 15 Jacobian terms, pad
struct fp_control {
    unsigned long long queue;       // next work item of the persistent tile kernel
    int status;                     // FP_STATUS_* bits
    int pad[61];
};

struct fp_workspace_layout {
    size_t gauss_fwd, gauss_box, gauss_ctr, gauss_jac, partials, total;
};

static inline size_t fp_align256(size_t x) { return (x + 255) & ~(size_t)255; }

static inline fp_workspace_layout fp_layout(int64_t n_gauss, int64_t n_partials)
{
    fp_workspace_layout L;
    size_t off = fp_align256(sizeof(fp_control));
    L.gauss_fwd = off; off = fp_align256(off + (size_t)n_gauss * 2 * 16);
    L.gauss_box = off; off = fp_align256(off + (size_t)n_gauss * 16);
    L.gauss_ctr = off; off = fp_align256(off + (size_t)n_gauss * 8);
    L.gauss_jac = off; off = fp_align256(off + (size_t)n_gauss * FP_JAC * 8);
    L.partials = off;  off = fp_align256(off + (size_t)n_partials * 8);
    L.total = off;
    return L;
}

// ---- device helpers ---------------------------------------------------------
__device__ __forceinline__ float fp_ex2(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// L2 policy for data read once per evaluation (the pixel records): evict
// first, so the stream does not push the per-exposure Gaussian tables, which
// every tile of the exposure re-reads, out of L2.
__device__ __forceinline__ uint64_t fp_policy_evict_first()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// 16-byte read-only load with an L2 cache policy.
__device__ __forceinline__ float4 fp_ldg_policy(const float4 *p, uint64_t pol)
{
    float4 r;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
        : "l"(p), "l"(pol));
    return r;
}

// 2x2 matrices as {m11, m12, m21, m22}
template <typename R>
struct fp_m22 {
    R a, b, c, d;
};

template <typename R>
__host__ __device__ __forceinline__ fp_m22<R> fp_mul(const fp_m22<R> &x, const fp_m22<R> &y)
{
    return {x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d,
            x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d};
}
