// peak.cu -- in-run measurement of the two roofline denominators of this
// path: FP32 FMA throughput and SFU ex2 throughput of the current device.
//
// Each kernel keeps 8 independent dependency chains per thread so issue, not
// latency, is the limit; the grid is 8 CTAs of 256 threads per SM.  The result
// is written through a device pointer so nothing can optimise the work away.

#include "fp_common.cuh"

namespace {

constexpr int PK_THREADS = 256;
constexpr int PK_CHAINS = 8;

__global__ void __launch_bounds__(PK_THREADS) fma_peak_kernel(float seed, int iters, float *out)
{
    float a[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) a[c] = seed + 0.001f * (threadIdx.x + c);
    const float m = 0.999999f, k = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < PK_CHAINS; ++c) a[c] = fmaf(a[c], m, k);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s += a[c];
    if (s == 12345.678f) out[threadIdx.x] = s;   // practically never true; keeps the chains live
}

__global__ void __launch_bounds__(PK_THREADS) ex2_peak_kernel(float seed, int iters, float *out)
{
    float a[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) a[c] = -1.0f - 0.001f * (threadIdx.x + c) + seed;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < PK_CHAINS; ++c) a[c] = -fp_ex2(a[c]);   // stays in [-1, -0.5]
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s += a[c];
    if (s == 12345.678f) out[threadIdx.x] = s;
}

template <typename K>
int time_kernel(K kern, int iters, float *scratch, cudaStream_t st, float *ms_out, int *grid_out)
{
    int nsm = 0;
    if (int rc = fp_sm_count(&nsm)) return rc;
    const int grid = 8 * nsm;
    cudaEvent_t e0, e1;
    if (int rc = fp_check_cuda(cudaEventCreate(&e0), "cudaEventCreate")) return rc;
    if (int rc = fp_check_cuda(cudaEventCreate(&e1), "cudaEventCreate")) { cudaEventDestroy(e0); return rc; }
    kern<<<grid, PK_THREADS, 0, st>>>(0.f, iters / 8, scratch);   // warm-up
    cudaEventRecord(e0, st);
    kern<<<grid, PK_THREADS, 0, st>>>(0.f, iters, scratch);
    cudaEventRecord(e1, st);
    int rc = fp_check_cuda(cudaEventSynchronize(e1), "peak kernel");
    float ms = 0.f;
    if (!rc) rc = fp_check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms_out = ms;
    *grid_out = grid;
    return rc;
}

}  // namespace

extern "C" int fp_measure_peaks(float *d_scratch, double *fp32_tflops, double *ex2_per_s, void *stream)
{
    if (!d_scratch || !fp32_tflops || !ex2_per_s) return fp_set_error(FP_ERR_ARGUMENT, "fp_measure_peaks: NULL");
    cudaStream_t st = (cudaStream_t)stream;
    float ms = 0.f;
    int grid = 0;
    const int it_f = 4096, it_e = 1024;
    if (int rc = time_kernel(fma_peak_kernel, it_f, d_scratch, st, &ms, &grid)) return rc;
    const double fmas = (double)grid * PK_THREADS * it_f * 16 * PK_CHAINS;
    *fp32_tflops = 2.0 * fmas / (ms * 1e-3) / 1e12;
    if (int rc = time_kernel(ex2_peak_kernel, it_e, d_scratch, st, &ms, &grid)) return rc;
    const double ex2s = (double)grid * PK_THREADS * it_e * 16 * PK_CHAINS;
    *ex2_per_s = ex2s / (ms * 1e-3);
    return FP_OK;
}
