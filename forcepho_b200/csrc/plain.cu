// plain.cu -- the one-patch-per-launch, port-equivalent kernel.
//
// Same decomposition as the reference's EvaluateProposal
// (forcepho/src/compute_gaussians_kernel.cu:212-312): one 1024-thread CTA per
// band; for each exposure of the band the CTA builds the band's image-Gaussian
// table in shared memory (one Gaussian per thread, FP32 like
// CreateImageGaussians, cu:45-127), then walks the exposure's pixels one per
// thread: forward residual over all Gaussians (common_kernel.cc:57-83), chi2 in
// f64, then for every source the 7 on-sky derivative sums over that source's
// Gaussians (common_kernel.cc:95-143), each reduced over the warp with shuffles
// and added to shared memory with one atomic per warp (cu:133-198).
//
// It exists as the comparator for the tiled/batched path: the arithmetic is
// FP32 with the accurate expf, exactly like the reference build.  Unlike the
// reference it opts in to the large B200 shared memory, so patches of up to
// ~2600 image Gaussians per exposure fit, and lanes past the end of an exposure
// take part in the warp reductions with zero contributions instead of leaving
// the loop (the reference relies on exposures padded to the warp size).

#include "fp_common.cuh"
#include "fp_gauss.cuh"

namespace {

struct plain_gauss {        // 84 bytes, the layout of the reference's ImageGaussian
    float amp, xcen, ycen, fxx, fyy, fxy;
    float dA_dflux, dx_dra, dy_dra, dx_ddec, dy_ddec;
    float dA_dq, dfxx_dq, dfyy_dq, dfxy_dq;
    float dA_dpa, dfxx_dpa, dfyy_dpa, dfxy_dpa;
    float dA_dsersic, dA_drh;
};

constexpr int PLAIN_THREADS = 1024;
constexpr int PLAIN_HEAD = 1024;       // bytes before the Gaussian table: chi2 + 210 floats

__device__ __forceinline__ float warp_sum(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(PLAIN_THREADS, 1)
plain_kernel(const fp_patch *__restrict__ pt, const fp_source *__restrict__ srcs,
             double *__restrict__ chi2_out, fp_response *__restrict__ resp_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double *s_chi2 = reinterpret_cast<double *>(smem);
    float *s_acc = reinterpret_cast<float *>(smem + 16);
    plain_gauss *s_g = reinterpret_cast<plain_gauss *>(smem + PLAIN_HEAD);

    const int band = blockIdx.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int ns = pt->n_sources;
    const int n_psf = pt->n_psf_per_source[band];
    const int ng = ns * n_psf;

    if (tid == 0) *s_chi2 = 0.0;
    for (int j = tid; j < MAXSOURCES * NPARAMS; j += PLAIN_THREADS) s_acc[j] = 0.f;

    const int e0 = pt->band_start[band];
    const int ne = pt->band_N[band];
    for (int ee = 0; ee < ne; ++ee) {
        const int e = e0 + ee;
        __syncthreads();   // previous exposure's pixel loop is done with the table
        for (int g = tid; g < ng; g += PLAIN_THREADS) {
            fp_img_gauss<float> G;
            fp_make_gaussian<float>(pt, srcs, band, e, g, n_psf, G);
            plain_gauss &o = s_g[g];
            o.amp = G.amp; o.xcen = G.xcen; o.ycen = G.ycen;
            o.fxx = G.fxx; o.fyy = G.fyy; o.fxy = G.fxy;
            o.dA_dflux = G.dA_dflux; o.dx_dra = G.dx_dra; o.dy_dra = G.dy_dra;
            o.dx_ddec = G.dx_ddec; o.dy_ddec = G.dy_ddec;
            o.dA_dq = G.dA_dq; o.dfxx_dq = G.dfxx_dq; o.dfyy_dq = G.dfyy_dq; o.dfxy_dq = G.dfxy_dq;
            o.dA_dpa = G.dA_dpa; o.dfxx_dpa = G.dfxx_dpa; o.dfyy_dpa = G.dfyy_dpa;
            o.dfxy_dpa = G.dfxy_dpa;
            o.dA_dsersic = G.dA_dsersic; o.dA_drh = G.dA_drh;
        }
        __syncthreads();

        const int pstart = pt->exposure_start[e];
        const int npix = pt->exposure_N[e];
        const int npad = (npix + 31) & ~31;
        for (int p = tid; p < npad; p += PLAIN_THREADS) {
            const bool live = p < npix;
            const int pix = pstart + p;
            float xp = 0.f, yp = 0.f, d = 0.f, ie = 0.f;
            if (live) { xp = pt->xpix[pix]; yp = pt->ypix[pix]; d = pt->data[pix]; ie = pt->ierr[pix]; }

            float r = d;
            if (live) {
                for (int i = 0; i < ng; ++i) {
                    const plain_gauss &g = s_g[i];
                    float dx = xp - g.xcen, dy = yp - g.ycen;
                    float vx = g.fxx * dx + g.fxy * dy;
                    float vy = g.fyy * dy + g.fxy * dx;
                    float ea = dx * vx + dy * vy;
                    if (ea > (float)MAX_EXP_ARG) continue;
                    float gp = expf(-0.5f * ea);
                    float h = 1.0f + (vx * vx + vy * vy - g.fxx - g.fyy) / 24.f;
                    r -= g.amp * gp * h;
                }
                if (pt->residual != nullptr) pt->residual[pix] = r;
            }
            float ri = r * ie, di = d * ie;
            double c2 = ((double)ri - (double)di) * ((double)ri + (double)di);
            c2 = warp_sum(c2);
            if (lane == 0) atomicAdd(s_chi2, c2);
            const float w = ri * ie;

            for (int s = 0; s < ns; ++s) {
                float acc[NPARAMS] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (live) {
                    const plain_gauss *gs = s_g + s * n_psf;
                    for (int i = 0; i < n_psf; ++i) {
                        const plain_gauss &g = gs[i];
                        float dx = xp - g.xcen, dy = yp - g.ycen;
                        float vx = g.fxx * dx + g.fxy * dy;
                        float vy = g.fyy * dy + g.fxy * dx;
                        float ea = dx * vx + dy * vy;
                        if (ea > (float)MAX_EXP_ARG) continue;
                        float gp = expf(-0.5f * ea);
                        float h = 1.0f + (vx * vx + vy * vy - g.fxx - g.fyy) * (1.0f / 24.0f);
                        float k = -2.f * w * gp;
                        float ch = k * g.amp;
                        float dA = k * h;
                        float cc = ch * h;
                        float d_x = cc * vx - ch * (g.fxx * vx + g.fxy * vy) * (1.0f / 12.0f);
                        float d_y = cc * vy - ch * (g.fyy * vy + g.fxy * vx) * (1.0f / 12.0f);
                        float d_fx = -0.5f * cc * dx * dx - ch * (1.0f - 2.0f * dx * vx) * (1.0f / 24.0f);
                        float d_fy = -0.5f * cc * dy * dy - ch * (1.0f - 2.0f * dy * vy) * (1.0f / 24.0f);
                        float d_fxy = -cc * dx * dy + ch * (dy * vx + dx * vy) * (1.0f / 12.0f);
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
                    float v = warp_sum(acc[j]);
                    if (lane == 0) atomicAdd(s_acc + s * NPARAMS + j, v);
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0) chi2_out[band] = *s_chi2;
    for (int j = tid; j < MAXSOURCES * NPARAMS; j += PLAIN_THREADS)
        resp_out[band].dchi2_dparam[j] = (j < ns * NPARAMS) ? s_acc[j] : 0.f;
}

}  // namespace

extern "C" int fp_evaluate_proposal_plain(const fp_patch *d_patch, const fp_source *d_proposal,
                                          int n_bands, int max_gauss_per_exposure,
                                          double *d_chi2, fp_response *d_response, void *stream)
{
    if (!d_patch || !d_proposal || !d_chi2 || !d_response)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal_plain: NULL pointer");
    if (n_bands < 1 || n_bands > MAXBANDS)
        return fp_set_error(FP_ERR_LIMITS, "fp_evaluate_proposal_plain: n_bands=%d outside [1,%d]",
                            n_bands, MAXBANDS);
    if (max_gauss_per_exposure < 0)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal_plain: negative Gaussian count");
    const size_t smem = PLAIN_HEAD + (size_t)max_gauss_per_exposure * sizeof(plain_gauss);
    int dev = 0, optin = 0;
    if (int rc = fp_check_cuda(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (int rc = fp_check_cuda(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
                               "cudaDeviceGetAttribute"))
        return rc;
    if (smem > (size_t)optin)
        return fp_set_error(FP_ERR_LIMITS,
                            "fp_evaluate_proposal_plain: %d image Gaussians per exposure need %zu B "
                            "of shared memory (device limit %d B)",
                            max_gauss_per_exposure, smem, optin);
    // the device's limit rather than this call's size: the attribute is per
    // function, and a smaller value set by a concurrent call must not undercut
    // a larger launch
    if (int rc = fp_check_cuda(cudaFuncSetAttribute(plain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    optin),
                               "cudaFuncSetAttribute(plain_kernel)"))
        return rc;
    plain_kernel<<<n_bands, PLAIN_THREADS, smem, (cudaStream_t)stream>>>(d_patch, d_proposal, d_chi2,
                                                                        d_response);
    return fp_check_cuda(cudaGetLastError(), "plain_kernel launch");
}
