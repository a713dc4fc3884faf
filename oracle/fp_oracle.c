/* fp_oracle.c -- CPU oracle of forcepho's EvaluateProposal.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 * It is never on the product path.
 *
 * It restates the reference CPU kernel (forcepho/src/compute_gaussians_kernel.cc:45-315
 * with forcepho/src/common_kernel.cc:57-240 and forcepho/src/matrix22.cc:32-200)
 * in two precisions from one body (fp_oracle_body.h):
 *   *_f32  FP32 arithmetic like the reference (expf, f32 accumulation of
 *          gradients, f64 accumulation of chi2);
 *   *_f64  every operation in FP64 on the same f32 inputs -- the precision
 *          yardstick.
 * Both keep the reference's semantics: the MAX_EXP_ARG skip, chi2 as
 * sum (r^2 - d^2) ierr^2, every source reading its exposure's first PSF block,
 * and fluxes indexed by the sequential band number.
 */
#define _USE_MATH_DEFINES
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/forcepho_b200.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)

/* ---- FP32 instance ---- */
#define REAL float
#define SFX f32
#define EXPR expf
#define SQRTR sqrtf
#define SINR sinf
#define COSR cosf
#define GRADT float
#include "fp_oracle_body.h"
#undef REAL
#undef SFX
#undef EXPR
#undef SQRTR
#undef SINR
#undef COSR
#undef GRADT

/* ---- FP64 instance ---- */
#define REAL double
#define SFX f64
#define EXPR exp
#define SQRTR sqrt
#define SINR sin
#define COSR cos
#define GRADT double
#include "fp_oracle_body.h"
#undef REAL
#undef SFX
#undef EXPR
#undef SQRTR
#undef SINR
#undef COSR
#undef GRADT

/* Band `band` of the patch in FP32.  Writes chi2, dchi2[MAXSOURCES*NPARAMS]
 * (rows >= n_sources zeroed), and the residual into patch->residual when that
 * pointer is not NULL (as the reference does). */
int fpo_evaluate_band_f32(const fp_patch *patch, const fp_source *sources, int band,
                          double *chi2, float *dchi2, int nthreads)
{
    return evaluate_band_f32(patch, sources, band, chi2, dchi2, patch->residual, nthreads);
}

/* Band `band` of the patch entirely in FP64.  `residual` (may be NULL) is an
 * f64 array of the patch's full pixel length. */
int fpo_evaluate_band_f64(const fp_patch *patch, const fp_source *sources, int band,
                          double *chi2, double *dchi2, double *residual, int nthreads)
{
    return evaluate_band_f64(patch, sources, band, chi2, dchi2, residual, nthreads);
}

/* The image Gaussians of exposure `e` (in band `band`): 21 doubles each. */
int fpo_image_gaussians(const fp_patch *patch, const fp_source *sources, int band, int e,
                        int use_f64, double *out)
{
    return use_f64 ? image_gaussians_f64(patch, sources, band, e, out)
                   : image_gaussians_f32(patch, sources, band, e, out);
}

/* Counts of (pixel, Gaussian) pairs of band `band`: all pairs, and those
 * with exponent argument <= MAX_EXP_ARG in FP64 (the ones that do work). */
int fpo_count_pairs(const fp_patch *patch, const fp_source *sources, int band,
                    long long *n_pairs, long long *n_active)
{
    const int ns = patch->n_sources, npsf = patch->n_psf_per_source[band];
    const int ng = ns * npsf;
    img_gauss_f64 *gs = (img_gauss_f64 *)malloc(sizeof(*gs) * (size_t)(ng > 0 ? ng : 1));
    if (!gs) return -2;
    long long tot = 0, act = 0;
    for (int ee = 0; ee < patch->band_N[band]; ++ee) {
        int e = patch->band_start[band] + ee;
        make_gaussians_f64(patch, sources, band, e, gs);
        int p0 = patch->exposure_start[e], np = patch->exposure_N[e];
        tot += (long long)np * ng;
        for (int i = 0; i < np; ++i) {
            double xp = patch->xpix[p0 + i], yp = patch->ypix[p0 + i];
            for (int g = 0; g < ng; ++g) {
                double dx = xp - gs[g].xcen, dy = yp - gs[g].ycen;
                double ea = dx * (gs[g].fxx * dx + gs[g].fxy * dy) + dy * (gs[g].fyy * dy + gs[g].fxy * dx);
                act += (ea <= MAX_EXP_ARG);
            }
        }
    }
    free(gs);
    *n_pairs = tot;
    *n_active = act;
    return 0;
}
