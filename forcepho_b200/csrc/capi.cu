// capi.cu -- error reporting, version and layout queries of the C ABI.

#include <stdarg.h>
#include <stdio.h>

#include "fp_common.cuh"

namespace {
thread_local char g_err[512] = "no error";
}

int fp_set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int fp_check_cuda(cudaError_t err, const char *what)
{
    if (err == cudaSuccess) return FP_OK;
    return fp_set_error(FP_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(err), cudaGetErrorName(err));
}

int fp_sm_count(int *out)
{
    int dev = 0;
    if (int rc = fp_check_cuda(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    return fp_check_cuda(cudaDeviceGetAttribute(out, cudaDevAttrMultiProcessorCount, dev),
                         "cudaDeviceGetAttribute(SM count)");
}

extern "C" const char *fp_error_string(void) { return g_err; }

extern "C" int fp_version(void) { return 100; }

extern "C" int fp_struct_sizes(int32_t out[4])
{
    if (!out) return fp_set_error(FP_ERR_ARGUMENT, "fp_struct_sizes: NULL");
    out[0] = (int32_t)sizeof(fp_patch);
    out[1] = (int32_t)sizeof(fp_source);
    out[2] = (int32_t)sizeof(fp_response);
    out[3] = (int32_t)sizeof(fp_psf_gaussian);
    return FP_OK;
}

extern "C" int fp_read_status(void *d_workspace, int32_t *status_out, void *stream)
{
    if (!d_workspace || !status_out) return fp_set_error(FP_ERR_ARGUMENT, "fp_read_status: NULL");
    fp_control *ctl = reinterpret_cast<fp_control *>(d_workspace);
    int st = 0;
    cudaStream_t s = (cudaStream_t)stream;
    if (int rc = fp_check_cuda(cudaMemcpyAsync(&st, &ctl->status, sizeof(int), cudaMemcpyDeviceToHost, s),
                               "fp_read_status copy"))
        return rc;
    if (int rc = fp_check_cuda(cudaMemsetAsync(&ctl->status, 0, sizeof(int), s), "fp_read_status clear"))
        return rc;
    if (int rc = fp_check_cuda(cudaStreamSynchronize(s), "fp_read_status sync")) return rc;
    *status_out = st;
    return FP_OK;
}

static_assert(sizeof(fp_patch) == 152, "fp_patch must match the reference Patch (152 B)");
static_assert(sizeof(fp_source) == 264, "fp_source must match the reference Source (264 B)");
static_assert(sizeof(fp_response) == 840, "fp_response must match the reference Response (840 B)");
static_assert(sizeof(fp_psf_gaussian) == 28, "fp_psf_gaussian must match PSFSourceGaussian (28 B)");
static_assert(sizeof(fp_exposure_desc) == 32, "fp_exposure_desc layout");
static_assert(sizeof(fp_tile) == 40, "fp_tile layout");
static_assert(sizeof(fp_band_desc) == 24, "fp_band_desc layout");
static_assert(sizeof(fp_control) == 256, "control block is 256 bytes");
