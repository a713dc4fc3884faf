// f64.cu -- the likelihood and its gradient in FP64 on the device.
//
// A precision reference at full size: every image Gaussian, pixel model,
// residual, chi2 term and gradient term in double precision, with the
// reference's formulas (compute_gaussians_kernel.cc:227-315,
// common_kernel.cc:57-143) and its MAX_EXP_ARG skip, over every pixel of
// every exposure (no culling).  Two launches:
//   f64_setup   one CTA per exposure: the exposure's image Gaussians
//               (fp_gauss.cuh in double) into the workspace table;
//   f64_pixels  a grid of CTAs per exposure, one pixel per thread at a time:
//               the residual over all Gaussians, the chi2 term, then per
//               source the 7 on-sky gradient sums over its Gaussians, reduced
//               per warp and CTA and added to the outputs with FP64 atomics.
// The atomics make the sums order-dependent at the 1e-16 level: exact to
// about 1e-15, not bitwise reproducible.

#include "fp_common.cuh"
#include "fp_gauss.cuh"

namespace {

constexpr int F64_THREADS = 256;
constexpr int F64_BLOCKS_PER_EXPOSURE = 32;

struct f64_ws_layout {
    size_t table, total;
};

inline f64_ws_layout f64_layout(int n_exposures, int max_gauss)
{
    f64_ws_layout L;
    size_t off = fp_align256(sizeof(fp_control));
    L.table = off;
    off = fp_align256(off + (size_t)n_exposures * (size_t)max_gauss * sizeof(fp_img_gauss<double>));
    L.total = off;
    return L;
}

// the band holding exposure e, or -1
__device__ int band_of_exposure(const fp_patch *pt, int n_bands, int e)
{
    for (int b = 0; b < n_bands; ++b)
        if (e >= pt->band_start[b] && e < pt->band_start[b] + pt->band_N[b]) return b;
    return -1;
}

__device__ __forceinline__ double warp_sum64(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(F64_THREADS)
f64_setup(const fp_patch *__restrict__ pt, const fp_source *__restrict__ srcs, int n_bands, int max_gauss,
          fp_img_gauss<double> *__restrict__ table, fp_control *ctl)
{
    const int e = blockIdx.x;
    const int b = band_of_exposure(pt, n_bands, e);
    const int ns = pt->n_sources;
    if (b < 0) return;
    if (ns > MAXSOURCES) {
        if (threadIdx.x == 0) atomicOr(&ctl->status, FP_STATUS_SOURCES);
        return;
    }
    const int n_psf = pt->n_psf_per_source[b];
    const int ng = ns * n_psf;
    if (ng > max_gauss) {
        if (threadIdx.x == 0) atomicOr(&ctl->status, FP_STATUS_GAUSS_COUNT);
        return;
    }
    for (int g = threadIdx.x; g < ng; g += blockDim.x)
        fp_make_gaussian<double>(pt, srcs, b, e, g, n_psf, table[(size_t)e * max_gauss + g]);
}

__global__ void __launch_bounds__(F64_THREADS)
f64_pixels(const fp_patch *__restrict__ pt, int n_bands, int max_gauss,
           const fp_img_gauss<double> *__restrict__ table, double *__restrict__ chi2,
           double *__restrict__ dchi2)
{
    __shared__ double s_acc[MAXSOURCES * NPARAMS];
    __shared__ double s_chi;
    const int e = blockIdx.x;
    const int b = band_of_exposure(pt, n_bands, e);
    const int ns = pt->n_sources;
    if (b < 0 || ns > MAXSOURCES) return;
    const int n_psf = pt->n_psf_per_source[b];
    const int ng = ns * n_psf;
    if (ng > max_gauss) return;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int j = tid; j < ns * NPARAMS; j += blockDim.x) s_acc[j] = 0.0;
    if (tid == 0) s_chi = 0.0;
    __syncthreads();

    const fp_img_gauss<double> *G = table + (size_t)e * max_gauss;
    const int pstart = pt->exposure_start[e], npix = pt->exposure_N[e];
    const int stride = gridDim.y * blockDim.x;
    // every lane of a warp runs the same number of iterations (warp reductions)
    const int nlim = (npix + stride - 1) / stride * stride;
    for (int p = blockIdx.y * blockDim.x + tid; p < nlim; p += stride) {
        const bool live = p < npix;
        double xp = 0.0, yp = 0.0, d = 0.0, ie = 0.0;
        if (live) {
            xp = pt->xpix[pstart + p];
            yp = pt->ypix[pstart + p];
            d = pt->data[pstart + p];
            ie = pt->ierr[pstart + p];
        }
        double r = d;
        if (live) {
            for (int i = 0; i < ng; ++i) {
                const fp_img_gauss<double> &g = G[i];
                const double dx = xp - g.xcen, dy = yp - g.ycen;
                const double vx = g.fxx * dx + g.fxy * dy;
                const double vy = g.fyy * dy + g.fxy * dx;
                const double ea = dx * vx + dy * vy;
                if (ea > MAX_EXP_ARG) continue;
                const double h = 1.0 + (vx * vx + vy * vy - g.fxx - g.fyy) / 24.0;
                r -= g.amp * exp(-0.5 * ea) * h;
            }
        }
        const double ri = r * ie, di = d * ie;
        const double c2 = warp_sum64(live ? (ri - di) * (ri + di) : 0.0);
        if (lane == 0) atomicAdd(&s_chi, c2);
        const double w = ri * ie;
        for (int s = 0; s < ns; ++s) {
            double acc[NPARAMS] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            if (live) {
                for (int i = 0; i < n_psf; ++i) {
                    const fp_img_gauss<double> &g = G[s * n_psf + i];
                    const double dx = xp - g.xcen, dy = yp - g.ycen;
                    const double vx = g.fxx * dx + g.fxy * dy;
                    const double vy = g.fyy * dy + g.fxy * dx;
                    const double ea = dx * vx + dy * vy;
                    if (ea > MAX_EXP_ARG) continue;
                    const double gp = exp(-0.5 * ea);
                    const double h = 1.0 + (vx * vx + vy * vy - g.fxx - g.fyy) / 24.0;
                    const double k = -2.0 * w * gp;
                    const double ch = k * g.amp;
                    const double dA = k * h;
                    const double cc = ch * h;
                    const double d_x = cc * vx - ch * (g.fxx * vx + g.fxy * vy) / 12.0;
                    const double d_y = cc * vy - ch * (g.fyy * vy + g.fxy * vx) / 12.0;
                    const double d_fx = -0.5 * cc * dx * dx - ch * (1.0 - 2.0 * dx * vx) / 24.0;
                    const double d_fy = -0.5 * cc * dy * dy - ch * (1.0 - 2.0 * dy * vy) / 24.0;
                    const double d_fxy = -cc * dx * dy + ch * (dy * vx + dx * vy) / 12.0;
                    acc[0] += g.dA_dflux * dA;
                    acc[1] += g.dx_dra * d_x + g.dy_dra * d_y;
                    acc[2] += g.dx_ddec * d_x + g.dy_ddec * d_y;
                    acc[3] += g.dA_dq * dA + d_fx * g.dfxx_dq + d_fxy * g.dfxy_dq + d_fy * g.dfyy_dq;
                    acc[4] += g.dA_dpa * dA + d_fx * g.dfxx_dpa + d_fxy * g.dfxy_dpa + d_fy * g.dfyy_dpa;
                    acc[5] += g.dA_dsersic * dA;
                    acc[6] += g.dA_drh * dA;
                }
            }
#pragma unroll
            for (int j = 0; j < NPARAMS; ++j) {
                const double v = warp_sum64(acc[j]);
                if (lane == 0 && v != 0.0) atomicAdd(s_acc + s * NPARAMS + j, v);
            }
        }
    }
    __syncthreads();
    if (tid == 0) atomicAdd(chi2 + b, s_chi);
    double *out = dchi2 + (size_t)b * MAXSOURCES * NPARAMS;
    for (int j = tid; j < ns * NPARAMS; j += blockDim.x)
        if (s_acc[j] != 0.0) atomicAdd(out + j, s_acc[j]);
}

}  // namespace

extern "C" int fp_f64_workspace_bytes(int n_exposures, int max_gauss_per_exposure, size_t *out)
{
    if (!out || n_exposures < 0 || max_gauss_per_exposure < 0)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_f64_workspace_bytes: bad arguments");
    *out = f64_layout(n_exposures, max_gauss_per_exposure).total;
    return FP_OK;
}

extern "C" int fp_evaluate_proposal_f64(const fp_patch *d_patch, const fp_source *d_proposal, int n_bands,
                                        int n_exposures, int max_gauss_per_exposure, double *d_chi2,
                                        double *d_dchi2, void *d_workspace, size_t workspace_bytes,
                                        void *stream)
{
    if (!d_patch || !d_proposal || !d_chi2 || !d_dchi2 || !d_workspace)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal_f64: NULL pointer");
    if (n_bands < 1 || n_bands > MAXBANDS)
        return fp_set_error(FP_ERR_LIMITS, "fp_evaluate_proposal_f64: n_bands=%d outside [1,%d]", n_bands,
                            MAXBANDS);
    if (n_exposures < 0 || max_gauss_per_exposure < 0)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal_f64: negative count");
    if (((uintptr_t)d_workspace) & 255)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal_f64: workspace must be 256-byte aligned");
    const f64_ws_layout L = f64_layout(n_exposures, max_gauss_per_exposure);
    if (workspace_bytes < L.total)
        return fp_set_error(FP_ERR_WORKSPACE, "fp_evaluate_proposal_f64: workspace %zu B < required %zu B",
                            workspace_bytes, L.total);
    cudaStream_t st = (cudaStream_t)stream;
    if (int rc = fp_check_cuda(cudaMemsetAsync(d_workspace, 0, sizeof(fp_control), st), "status clear")) return rc;
    if (int rc = fp_check_cuda(cudaMemsetAsync(d_chi2, 0, sizeof(double) * n_bands, st), "chi2 clear")) return rc;
    if (int rc = fp_check_cuda(cudaMemsetAsync(d_dchi2, 0, sizeof(double) * n_bands * MAXSOURCES * NPARAMS, st),
                               "dchi2 clear"))
        return rc;
    if (n_exposures == 0) return FP_OK;
    unsigned char *ws = reinterpret_cast<unsigned char *>(d_workspace);
    fp_control *ctl = reinterpret_cast<fp_control *>(ws);
    fp_img_gauss<double> *table = reinterpret_cast<fp_img_gauss<double> *>(ws + L.table);
    f64_setup<<<n_exposures, F64_THREADS, 0, st>>>(d_patch, d_proposal, n_bands, max_gauss_per_exposure, table,
                                                   ctl);
    if (int rc = fp_check_cuda(cudaGetLastError(), "f64_setup launch")) return rc;
    f64_pixels<<<dim3(n_exposures, F64_BLOCKS_PER_EXPOSURE), F64_THREADS, 0, st>>>(
        d_patch, n_bands, max_gauss_per_exposure, table, d_chi2, d_dchi2);
    return fp_check_cuda(cudaGetLastError(), "f64_pixels launch");
}
