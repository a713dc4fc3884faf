/* forcepho_b200_limits.h -- compile-time limits shared by the CUDA kernels,
 * the C-ABI and the Python host code (which parses the #defines below).
 *
 * The values fix the byte layout of the Source and Response records that cross
 * the boundary, so they must equal the reference's (forcepho/src/kernel_limits.h:5-26);
 * a proposal array packed by the reference's Python code is then valid input here.
 */
#ifndef FORCEPHO_B200_LIMITS_H
#define FORCEPHO_B200_LIMITS_H

/* Maximum number of bands in one patch (Source.fluxes length). */
#define MAXBANDS 30

/* Maximum number of active sources in one patch (Response rows). */
#define MAXSOURCES 30

/* On-sky parameters per source per band that receive a gradient:
 * flux, ra, dec, q, pa, sersic, rhalf. */
#define NPARAMS 7

/* A (pixel, Gaussian) pair with exponent argument dx^T F dx above this value
 * contributes nothing (neither to the model nor to the gradient). */
#define MAX_EXP_ARG 36.0

/* Maximum number of Sersic mixture radii (Source amplitude array lengths). */
#define MAXRADII 10

#endif
