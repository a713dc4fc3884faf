// fp_gauss.cuh -- source (x) PSF convolution into one image Gaussian plus its
// Jacobian with respect to the source's on-sky parameters.
//
// The mathematics is the reference's (forcepho/src/common_kernel.cc:175-240,
// GetGaussianAndJacobian; forcepho/src/compute_gaussians_kernel.cu:45-127,
// CreateImageGaussians):
//   T        = D R(pa) S(q),  S(q) = diag(1/q, q)
//   Sigma    = rad2[bin] T T^T + Sigma_psf,   F = Sigma^-1
//   centre   = CW (radec - crval) + crpix + psf offset
//   amp      = G a_psf sqrt(det F) / (2 pi) * flux[band] * A_bin(sersic, rhalf)
//   dF/dq    = -F (rad2 (T dT_dq^T + dT_dq T^T)) F,   likewise for pa
//   dA/dq    = amp/2 tr(Sigma dF/dq),                  likewise for pa
// with the reference's indexing quirks: the PSF Gaussian of image Gaussian
// (s, p) is psfgauss[psfgauss_start[e] + p] for every source s, and the flux
// is fluxes[band] with band the sequential band index of the patch.
#pragma once

#include "fp_common.cuh"

template <typename R>
struct fp_img_gauss {
    R amp, xcen, ycen, fxx, fyy, fxy;
    R dA_dflux, dx_dra, dy_dra, dx_ddec, dy_ddec;
    R dA_dq, dfxx_dq, dfyy_dq, dfxy_dq;
    R dA_dpa, dfxx_dpa, dfyy_dpa, dfxy_dpa;
    R dA_dsersic, dA_drh;
};

__device__ __forceinline__ void fp_sincos(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void fp_sincos(double x, double *s, double *c) { sincos(x, s, c); }
__device__ __forceinline__ float fp_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double fp_sqrt(double x) { return sqrt(x); }

// Image Gaussian `g` (source g / n_psf, PSF component g % n_psf) of exposure
// `e` in band `band`.  R = float restates the reference's FP32 setup; R = double
// is the FP64 setup of the tiled path.
template <typename R>
__device__ __forceinline__ void fp_make_gaussian(const fp_patch *pt, const fp_source *srcs,
                                                 int band, int e, int g, int n_psf,
                                                 fp_img_gauss<R> &o)
{
    const int ns = pt->n_sources;
    const int s = g / n_psf;
    const int p = g - s * n_psf;
    const fp_source *src = srcs + s;
    const int m4 = 4 * (ns * e + s), m2 = 2 * (ns * e + s);

    const fp_m22<R> D = {(R)pt->D[m4], (R)pt->D[m4 + 1], (R)pt->D[m4 + 2], (R)pt->D[m4 + 3]};
    const fp_m22<R> CW = {(R)pt->CW[m4], (R)pt->CW[m4 + 1], (R)pt->CW[m4 + 2], (R)pt->CW[m4 + 3]};

    R sn, cs;
    fp_sincos((R)src->pa, &sn, &cs);
    const R q = (R)src->q;
    const fp_m22<R> Rm = {cs, -sn, sn, cs};
    const fp_m22<R> dR = {-sn, -cs, cs, -sn};
    const fp_m22<R> Sm = {(R)1 / q, (R)0, (R)0, q};
    const fp_m22<R> dS = {(R)-1 / (q * q), (R)0, (R)0, (R)1};
    const fp_m22<R> DR = fp_mul(D, Rm);
    const fp_m22<R> T = fp_mul(DR, Sm);
    const fp_m22<R> Tq = fp_mul(DR, dS);
    const fp_m22<R> Tp = fp_mul(fp_mul(D, dR), Sm);

    const R dra = (R)src->ra - (R)pt->crval[m2];
    const R ddec = (R)src->dec - (R)pt->crval[m2 + 1];
    const R xs = CW.a * dra + CW.b * ddec + (R)pt->crpix[m2];
    const R ys = CW.c * dra + CW.d * ddec + (R)pt->crpix[m2 + 1];

    const fp_psf_gaussian pg = pt->psfgauss[pt->psfgauss_start[e] + p];
    const int bin = pg.sersic_radius_bin;
    const R r2 = (R)pt->rad2[bin];
    const R a_s = (R)src->mixture_amplitudes[bin];
    const R flux = (R)src->fluxes[band];

    // Sigma = r2 T T^T + Sigma_psf ; F = Sigma^-1
    const R sxx = r2 * (T.a * T.a + T.b * T.b) + (R)pg.Cxx;
    const R sxy = r2 * (T.a * T.c + T.b * T.d) + (R)pg.Cxy;
    const R syy = r2 * (T.c * T.c + T.d * T.d) + (R)pg.Cyy;
    const R idet = (R)1 / (sxx * syy - sxy * sxy);
    const R fxx = syy * idet, fyy = sxx * idet, fxy = -sxy * idet;
    const R detF = fxx * fyy - fxy * fxy;

    const R norm = (R)pt->G[e] * (R)pg.amp * fp_sqrt(detF) * ((R)1 / ((R)2 * (R)3.14159265358979323846));
    o.amp = norm * flux * a_s;
    o.xcen = xs + (R)pg.xcen;
    o.ycen = ys + (R)pg.ycen;
    o.fxx = fxx; o.fyy = fyy; o.fxy = fxy;

    // dSigma/dq and dSigma/dpa (symmetric): r2 (T dT^T + dT T^T)
    const R qxx = r2 * (R)2 * (T.a * Tq.a + T.b * Tq.b);
    const R qxy = r2 * (T.a * Tq.c + T.b * Tq.d + T.c * Tq.a + T.d * Tq.b);
    const R qyy = r2 * (R)2 * (T.c * Tq.c + T.d * Tq.d);
    const R pxx = r2 * (R)2 * (T.a * Tp.a + T.b * Tp.b);
    const R pxy = r2 * (T.a * Tp.c + T.b * Tp.d + T.c * Tp.a + T.d * Tp.b);
    const R pyy = r2 * (R)2 * (T.c * Tp.c + T.d * Tp.d);

    // dF = -F dSigma F for symmetric F, dSigma
    const R Fq_xx = -(fxx * (fxx * qxx + fxy * qxy) + fxy * (fxx * qxy + fxy * qyy));
    const R Fq_xy = -(fxx * (fxy * qxx + fyy * qxy) + fxy * (fxy * qxy + fyy * qyy));
    const R Fq_yy = -(fxy * (fxy * qxx + fyy * qxy) + fyy * (fxy * qxy + fyy * qyy));
    const R Fp_xx = -(fxx * (fxx * pxx + fxy * pxy) + fxy * (fxx * pxy + fxy * pyy));
    const R Fp_xy = -(fxx * (fxy * pxx + fyy * pxy) + fxy * (fxy * pxy + fyy * pyy));
    const R Fp_yy = -(fxy * (fxy * pxx + fyy * pxy) + fyy * (fxy * pxy + fyy * pyy));

    o.dA_dq = (R)0.5 * o.amp * (sxx * Fq_xx + (R)2 * sxy * Fq_xy + syy * Fq_yy);
    o.dA_dpa = (R)0.5 * o.amp * (sxx * Fp_xx + (R)2 * sxy * Fp_xy + syy * Fp_yy);
    o.dfxx_dq = Fq_xx; o.dfyy_dq = Fq_yy; o.dfxy_dq = Fq_xy;
    o.dfxx_dpa = Fp_xx; o.dfyy_dpa = Fp_yy; o.dfxy_dpa = Fp_xy;

    o.dA_dflux = norm * a_s;
    o.dA_dsersic = norm * flux * (R)src->damplitude_dnsersic[bin];
    o.dA_drh = norm * flux * (R)src->damplitude_drh[bin];
    o.dx_dra = CW.a; o.dy_dra = CW.c;
    o.dx_ddec = CW.b; o.dy_ddec = CW.d;
}
