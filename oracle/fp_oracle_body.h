/* fp_oracle_body.h -- precision-generic body of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY: included twice by fp_oracle.c, once with
 * REAL=float (restating the reference CPU kernel's FP32 arithmetic) and once
 * with REAL=double (every operation in FP64 on the same f32 inputs).
 *
 * Required macros: REAL, SFX (name suffix), EXPR (exp function for REAL),
 * SQRTR, SINR, COSR, and GRADT (type of the gradient output).
 */

typedef struct {
    REAL amp, xcen, ycen, fxx, fyy, fxy;
    /* d(image params)/d(on-sky params), 15 entries */
    REAL dA_dflux, dx_dra, dy_dra, dx_ddec, dy_ddec;
    REAL dA_dq, dfxx_dq, dfyy_dq, dfxy_dq;
    REAL dA_dpa, dfxx_dpa, dfyy_dpa, dfxy_dpa;
    REAL dA_dsersic, dA_drh;
} CAT(img_gauss_, SFX);

/* 2x2 helpers on row-major arrays m[4] = {m11, m12, m21, m22}. */
static inline void CAT(mul22_, SFX)(const REAL *a, const REAL *b, REAL *out)
{
    REAL r0 = a[0] * b[0] + a[1] * b[2];
    REAL r1 = a[0] * b[1] + a[1] * b[3];
    REAL r2 = a[2] * b[0] + a[3] * b[2];
    REAL r3 = a[2] * b[1] + a[3] * b[3];
    out[0] = r0; out[1] = r1; out[2] = r2; out[3] = r3;
}

/* Convolve every (source, PSF component) of exposure `e` into image Gaussians.
 * Follows forcepho/src/compute_gaussians_kernel.cc:45-114 (ConvolveOneSource)
 * and forcepho/src/common_kernel.cc:175-240 (GetGaussianAndJacobian). */
static void CAT(make_gaussians_, SFX)(const fp_patch *pt, const fp_source *src, int band,
                                        int e, CAT(img_gauss_, SFX) *out)
{
    const int ns = pt->n_sources;
    const int npsf = pt->n_psf_per_source[band];
    const int pstart = pt->psfgauss_start[e];
    const REAL Gcal = (REAL)pt->G[e];
    const REAL inv2pi = (REAL)1 / ((REAL)2 * (REAL)M_PI);

    for (int s = 0; s < ns; ++s) {
        const fp_source *g = src + s;
        const float *Dp = pt->D + 4 * (ns * e + s);
        const float *CWp = pt->CW + 4 * (ns * e + s);
        const float *crp = pt->crpix + 2 * (ns * e + s);
        const float *crv = pt->crval + 2 * (ns * e + s);
        REAL D[4] = {Dp[0], Dp[1], Dp[2], Dp[3]};
        REAL CW[4] = {CWp[0], CWp[1], CWp[2], CWp[3]};

        REAL q = g->q, pa = g->pa;
        REAL c = COSR(pa), sn = SINR(pa);
        REAL R[4] = {c, -sn, sn, c};
        REAL dR[4] = {-sn, -c, c, -sn};
        REAL S[4] = {(REAL)1 / q, 0, 0, q};
        REAL dS[4] = {(REAL)-1 / (q * q), 0, 0, 1};

        REAL DR[4], T[4], dT_dq[4], DdR[4], dT_dpa[4];
        CAT(mul22_, SFX)(D, R, DR);
        CAT(mul22_, SFX)(DR, S, T);
        CAT(mul22_, SFX)(DR, dS, dT_dq);
        CAT(mul22_, SFX)(D, dR, DdR);
        CAT(mul22_, SFX)(DdR, S, dT_dpa);

        /* source centre in pixels: CW (sky offset from crval) + crpix */
        REAL dra = (REAL)g->ra - (REAL)crv[0];
        REAL ddec = (REAL)g->dec - (REAL)crv[1];
        REAL xc = CW[0] * dra + CW[1] * ddec + (REAL)crp[0];
        REAL yc = CW[2] * dra + CW[3] * ddec + (REAL)crp[1];

        /* T T^T and the symmetric products T dT^T + dT T^T */
        REAL TT[3] = {T[0] * T[0] + T[1] * T[1], T[0] * T[2] + T[1] * T[3],
                      T[2] * T[2] + T[3] * T[3]};
        REAL sq[3] = {2 * (T[0] * dT_dq[0] + T[1] * dT_dq[1]),
                      T[0] * dT_dq[2] + T[1] * dT_dq[3] + T[2] * dT_dq[0] + T[3] * dT_dq[1],
                      2 * (T[2] * dT_dq[2] + T[3] * dT_dq[3])};
        REAL sp[3] = {2 * (T[0] * dT_dpa[0] + T[1] * dT_dpa[1]),
                      T[0] * dT_dpa[2] + T[1] * dT_dpa[3] + T[2] * dT_dpa[0] + T[3] * dT_dpa[1],
                      2 * (T[2] * dT_dpa[2] + T[3] * dT_dpa[3])};

        for (int p = 0; p < npsf; ++p) {
            /* every source reads the exposure's first PSF block: the reference
             * indexes psfgauss_start[e] + p without a per-source offset */
            const fp_psf_gaussian *pg = pt->psfgauss + pstart + p;
            int bin = pg->sersic_radius_bin;
            REAL r2 = pt->rad2[bin];
            REAL a_s = g->mixture_amplitudes[bin];
            REAL da_dn = g->damplitude_dnsersic[bin];
            REAL da_dr = g->damplitude_drh[bin];
            REAL flux = g->fluxes[band];

            /* convolved covariance Sigma = r2 T T^T + Sigma_psf, and F = Sigma^-1 */
            REAL sxx = r2 * TT[0] + (REAL)pg->Cxx;
            REAL sxy = r2 * TT[1] + (REAL)pg->Cxy;
            REAL syy = r2 * TT[2] + (REAL)pg->Cyy;
            REAL idet = (REAL)1 / (sxx * syy - sxy * sxy);
            REAL fxx = syy * idet, fyy = sxx * idet, fxy = -sxy * idet;
            REAL detF = fxx * fyy - fxy * fxy;

            CAT(img_gauss_, SFX) *o = out + s * npsf + p;
            o->fxx = fxx; o->fyy = fyy; o->fxy = fxy;
            o->xcen = xc + (REAL)pg->xcen;
            o->ycen = yc + (REAL)pg->ycen;
            REAL norm = Gcal * (REAL)pg->amp * SQRTR(detF) * inv2pi;
            o->amp = norm * flux * a_s;

            /* dF/dtheta = -F (dSigma/dtheta) F for theta in (q, pa) */
            REAL dq[3] = {r2 * sq[0], r2 * sq[1], r2 * sq[2]};
            REAL dp[3] = {r2 * sp[0], r2 * sp[1], r2 * sp[2]};
            REAL Fm[4] = {fxx, fxy, fxy, fyy};
            REAL DQ[4] = {dq[0], dq[1], dq[1], dq[2]};
            REAL DP[4] = {dp[0], dp[1], dp[1], dp[2]};
            REAL t1[4], dFq[4], dFp[4];
            CAT(mul22_, SFX)(Fm, DQ, t1);
            CAT(mul22_, SFX)(t1, Fm, dFq);
            CAT(mul22_, SFX)(Fm, DP, t1);
            CAT(mul22_, SFX)(t1, Fm, dFp);
            for (int k = 0; k < 4; ++k) { dFq[k] = -dFq[k]; dFp[k] = -dFp[k]; }

            /* dA/dtheta = A/2 trace(Sigma dF/dtheta) */
            REAL trq = sxx * dFq[0] + sxy * dFq[2] + sxy * dFq[1] + syy * dFq[3];
            REAL trp = sxx * dFp[0] + sxy * dFp[2] + sxy * dFp[1] + syy * dFp[3];
            o->dA_dq = (REAL)0.5 * o->amp * trq;
            o->dA_dpa = (REAL)0.5 * o->amp * trp;
            o->dA_dflux = norm * a_s;
            o->dA_dsersic = norm * flux * da_dn;
            o->dA_drh = norm * flux * da_dr;
            o->dx_dra = CW[0]; o->dy_dra = CW[2];
            o->dx_ddec = CW[1]; o->dy_ddec = CW[3];
            o->dfxx_dq = dFq[0]; o->dfyy_dq = dFq[3]; o->dfxy_dq = dFq[2];
            o->dfxx_dpa = dFp[0]; o->dfyy_dpa = dFp[3]; o->dfxy_dpa = dFp[2];
        }
    }
}

/* Residual of one pixel: data minus each Gaussian's counts in turn;
 * common_kernel.cc:57-83. */
static inline REAL CAT(pixel_residual_, SFX)(REAL xp, REAL yp, REAL d,
                                               const CAT(img_gauss_, SFX) *g, int n)
{
    REAL m = d;
    for (int i = 0; i < n; ++i, ++g) {
        REAL dx = xp - g->xcen, dy = yp - g->ycen;
        REAL vx = g->fxx * dx + g->fxy * dy;
        REAL vy = g->fyy * dy + g->fxy * dx;
        REAL ea = dx * vx + dy * vy;
        if (ea > (REAL)MAX_EXP_ARG) continue;
        REAL gp = EXPR((REAL)-0.5 * ea);
        REAL h = (REAL)1 + (vx * vx + vy * vy - g->fxx - g->fyy) / (REAL)24;
        m -= g->amp * gp * h;
    }
    return m;
}

/* Add one pixel's contribution to the 7 on-sky gradients of one source;
 * common_kernel.cc:95-143.  w = residual * ierr^2. */
static inline void CAT(pixel_grad_, SFX)(REAL xp, REAL yp, REAL w, const CAT(img_gauss_, SFX) *g,
                                           int n, REAL *acc)
{
    for (int i = 0; i < n; ++i, ++g) {
        REAL dx = xp - g->xcen, dy = yp - g->ycen;
        REAL vx = g->fxx * dx + g->fxy * dy;
        REAL vy = g->fyy * dy + g->fxy * dx;
        REAL ea = dx * vx + dy * vy;
        if (ea > (REAL)MAX_EXP_ARG) continue;
        REAL gp = EXPR((REAL)-0.5 * ea);
        REAL h = (REAL)1 + (vx * vx + vy * vy - g->fxx - g->fyy) * ((REAL)1 / (REAL)24);
        REAL k = (REAL)-2 * w * gp;        /* d chi2 / d counts, times the Gaussian shape */
        REAL ch = k * g->amp;              /* counts derivative before the H factor */
        REAL dA = k * h;
        REAL cc = ch * h;
        REAL d_x = cc * vx - ch * (g->fxx * vx + g->fxy * vy) * ((REAL)1 / (REAL)12);
        REAL d_y = cc * vy - ch * (g->fyy * vy + g->fxy * vx) * ((REAL)1 / (REAL)12);
        REAL d_fx = (REAL)-0.5 * cc * dx * dx - ch * ((REAL)1 - (REAL)2 * dx * vx) * ((REAL)1 / (REAL)24);
        REAL d_fy = (REAL)-0.5 * cc * dy * dy - ch * ((REAL)1 - (REAL)2 * dy * vy) * ((REAL)1 / (REAL)24);
        REAL d_fxy = -cc * dx * dy + ch * (dy * vx + dx * vy) * ((REAL)1 / (REAL)12);

        acc[0] += g->dA_dflux * dA;
        acc[1] += g->dx_dra * d_x + g->dy_dra * d_y;
        acc[2] += g->dx_ddec * d_x + g->dy_ddec * d_y;
        acc[3] += g->dA_dq * dA + d_fx * g->dfxx_dq + d_fxy * g->dfxy_dq + d_fy * g->dfyy_dq;
        acc[4] += g->dA_dpa * dA + d_fx * g->dfxx_dpa + d_fxy * g->dfxy_dpa + d_fy * g->dfyy_dpa;
        acc[5] += g->dA_dsersic * dA;
        acc[6] += g->dA_drh * dA;
    }
}

/* chi2 and gradient of one band; compute_gaussians_kernel.cc:227-315.
 * `resid` (may be NULL) receives the residual of every pixel of the band.
 * With nthreads > 1 the pixels of each exposure are split into nthreads
 * contiguous ranges whose partial sums are combined in range order. */
static int CAT(evaluate_band_, SFX)(const fp_patch *pt, const fp_source *src, int band,
                                      double *chi2_out, GRADT *grad_out, REAL *resid,
                                      int nthreads)
{
    const int ns = pt->n_sources;
    const int npsf = pt->n_psf_per_source[band];
    const int ng = ns * npsf;
    if (ns < 0 || ns > MAXSOURCES || npsf <= 0) return -1;
    if (nthreads < 1) nthreads = 1;

    CAT(img_gauss_, SFX) *gs = (CAT(img_gauss_, SFX) *)malloc(sizeof(*gs) * (size_t)(ng > 0 ? ng : 1));
    REAL *part = (REAL *)calloc((size_t)nthreads * MAXSOURCES * NPARAMS, sizeof(REAL));
    double *pchi = (double *)calloc((size_t)nthreads, sizeof(double));
    if (!gs || !part || !pchi) { free(gs); free(part); free(pchi); return -2; }

    const int e0 = pt->band_start[band];
    const int ne = pt->band_N[band];
    for (int ee = 0; ee < ne; ++ee) {
        const int e = e0 + ee;
        CAT(make_gaussians_, SFX)(pt, src, band, e, gs);
        const int pstart = pt->exposure_start[e];
        const int npix = pt->exposure_N[e];
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
#endif
        for (int t = 0; t < nthreads; ++t) {
            int lo = (int)((long long)npix * t / nthreads);
            int hi = (int)((long long)npix * (t + 1) / nthreads);
            REAL *acc_t = part + (size_t)t * MAXSOURCES * NPARAMS;
            double chi_t = 0;
            for (int i = lo; i < hi; ++i) {
                const int pix = pstart + i;
                REAL xp = pt->xpix[pix], yp = pt->ypix[pix];
                REAL d = pt->data[pix], ie = pt->ierr[pix];
                REAL r = CAT(pixel_residual_, SFX)(xp, yp, d, gs, ng);
                if (resid) resid[pix] = r;
                REAL ri = r * ie, di = d * ie;
                chi_t += ((double)ri - (double)di) * ((double)ri + (double)di);
                REAL w = ri * ie;
                for (int s = 0; s < ns; ++s) {
                    REAL one[NPARAMS] = {0, 0, 0, 0, 0, 0, 0};
                    CAT(pixel_grad_, SFX)(xp, yp, w, gs + s * npsf, npsf, one);
                    for (int j = 0; j < NPARAMS; ++j) acc_t[s * NPARAMS + j] += one[j];
                }
            }
            pchi[t] += chi_t;
        }
    }

    double chi = 0;
    for (int j = 0; j < MAXSOURCES * NPARAMS; ++j) grad_out[j] = 0;
    for (int t = 0; t < nthreads; ++t) {
        chi += pchi[t];
        for (int j = 0; j < ns * NPARAMS; ++j)
            grad_out[j] += (GRADT)part[(size_t)t * MAXSOURCES * NPARAMS + j];
    }
    *chi2_out = chi;
    free(gs); free(part); free(pchi);
    return 0;
}

/* Image Gaussians of one exposure, flattened to 21 values each in the order
 * amp, xcen, ycen, fxx, fyy, fxy, then the 15 Jacobian terms. */
static int CAT(image_gaussians_, SFX)(const fp_patch *pt, const fp_source *src, int band, int e,
                                        double *out)
{
    const int ng = pt->n_sources * pt->n_psf_per_source[band];
    CAT(img_gauss_, SFX) *gs = (CAT(img_gauss_, SFX) *)malloc(sizeof(*gs) * (size_t)(ng > 0 ? ng : 1));
    if (!gs) return -2;
    CAT(make_gaussians_, SFX)(pt, src, band, e, gs);
    for (int i = 0; i < ng; ++i) {
        const REAL *f = &gs[i].amp;
        for (int k = 0; k < 21; ++k) out[21 * i + k] = (double)f[k];
    }
    free(gs);
    return 0;
}
