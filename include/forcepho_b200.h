/* forcepho_b200.h -- C ABI of the B200 likelihood library (libforcepho_b200.so).
 *
 * The library evaluates forcepho's per-patch likelihood hot path: every active
 * source's Sersic-as-Gaussian-mixture, convolved with each exposure's PSF
 * mixture, is rendered into model pixels; the ierr-weighted residuals give
 *     chi2[band]            = sum_pix (r*ierr - d*ierr) * (r*ierr + d*ierr)   (f64)
 *     dchi2_dparam[band][s] = d chi2[band] / d(flux, ra, dec, q, pa, sersic, rhalf)_s (f32)
 * exactly as the reference's EvaluateProposal does
 * (forcepho/src/compute_gaussians_kernel.cu:212-312, forcepho/src/compute_gaussians_kernel.cc:227-315).
 *
 * Conventions
 *   - All pointers named d_* are device pointers; h_* are host pointers.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *   - Every entry point returns 0 on success, or a negative FP_ERR_* code; nothing is
 *     printed.  fp_error_string() gives a one-line description of the last error.
 *   - Entry points never allocate device memory: buffers are owned by the caller
 *     (the reference's Python patch objects own theirs, forcepho/patches/device_patch.py:265-297).
 *     The one exception is fp_evaluate_proposal, the reference's own kernel ABI,
 *     which keeps a library-owned work plan per patch (fp_evaluate_proposal_release).
 *   - Launches are asynchronous on `stream` and contain no host synchronisation, so a
 *     sequence of them can be captured into a CUDA graph.  The one exception is
 *     fp_evaluate_proposal, which reads the patch struct back before its launch.
 */
#ifndef FORCEPHO_B200_H
#define FORCEPHO_B200_H

#include <stddef.h>
#include <stdint.h>

#include "forcepho_b200_limits.h"

/* Entry points are the only symbols the shared library exports. */
#if defined(__GNUC__)
#define FP_API __attribute__((visibility("default")))
#else
#define FP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------- */
/* Boundary records: bit-identical to the reference's structs.               */
/* ------------------------------------------------------------------------- */

/* One PSF Gaussian, already assigned to a Sersic radius bin: 28 bytes.
 * Mirrors PSFSourceGaussian (forcepho/src/patch.cc:103-119) and
 * PSF_DTYPE (forcepho/patches/storage.py:27-28). */
typedef struct fp_psf_gaussian {
    float amp;
    float xcen, ycen;
    float Cxx, Cyy, Cxy;
    int32_t sersic_radius_bin;
} fp_psf_gaussian;

/* Pointers to all pixel and metadata arrays of one patch: 152 bytes.
 * Mirrors class Patch (forcepho/src/patch.cc:23-100) and PatchBase.pdt
 * (forcepho/patches/patch.py:45-73).  Array shapes:
 *   data, ierr, xpix, ypix, residual  f32[n_pix]  (residual may be NULL)
 *   exposure_start, exposure_N         i32[n_exp]
 *   band_start, band_N                 i16[n_bands]
 *   rad2                               f32[n_radii]
 *   D, CW                              f32[n_exp][n_sources][2][2]
 *   crpix, crval                       f32[n_exp][n_sources][2]
 *   G                                  f32[n_exp]
 *   n_psf_per_source                   i32[n_bands]
 *   psfgauss                           fp_psf_gaussian[sum_e n_sources*n_psf_per_source[band(e)]]
 *   psfgauss_start                     i32[n_exp]                                            */
typedef struct fp_patch {
    float *data;
    float *ierr;
    float *xpix;
    float *ypix;
    float *residual;
    int32_t *exposure_start;
    int32_t *exposure_N;
    int16_t *band_start;
    int16_t *band_N;
    int32_t n_sources;
    int32_t n_radii;
    float *rad2;
    float *D;
    float *crpix;
    float *crval;
    float *CW;
    float *G;
    int32_t *n_psf_per_source;
    fp_psf_gaussian *psfgauss;
    int32_t *psfgauss_start;
} fp_patch;

/* On-sky parameters of one Sersic source: 264 bytes.
 * Mirrors class Source (forcepho/src/proposal.cu:13-27) and
 * source_struct_dtype (forcepho/proposal.py:229-240). */
typedef struct fp_source {
    float ra, dec;
    float q, pa;
    float nsersic, rh;
    float fluxes[MAXBANDS];
    float mixture_amplitudes[MAXRADII];
    float damplitude_drh[MAXRADII];
    float damplitude_dnsersic[MAXRADII];
} fp_source;

/* Gradient of one band's chi2: 840 bytes, source-major
 * (dflux, dra, ddec, dq, dpa, dsersic, drh) per source.
 * Mirrors class Response (forcepho/src/proposal.cu:33-39) and
 * response_struct_dtype (forcepho/proposal.py:243-244). */
typedef struct fp_response {
    float dchi2_dparam[MAXSOURCES * NPARAMS];
} fp_response;

/* ------------------------------------------------------------------------- */
/* Error handling                                                            */
/* ------------------------------------------------------------------------- */

#define FP_OK               0
#define FP_ERR_ARGUMENT    -1   /* bad argument (NULL, out-of-range count, misalignment) */
#define FP_ERR_LIMITS      -2   /* a count exceeds MAXSOURCES/MAXBANDS/shared memory */
#define FP_ERR_CUDA        -3   /* a CUDA runtime call failed */
#define FP_ERR_WORKSPACE   -4   /* workspace smaller than required */
#define FP_ERR_DEVICE      -5   /* a kernel reported an inconsistency in its status word */

/* Bits of the device status word of the batched kernels (fp_read_status).  A
 * tile or exposure that sets one contributes nothing to the results: a
 * rejected exposure renders a zero model with a zero gradient, a rejected
 * tile adds zero partial sums. */
#define FP_STATUS_TILE_SIZE   1 /* a tile larger than the launch's tile size */
#define FP_STATUS_GAUSS_COUNT 2 /* an exposure with more image Gaussians than the plan's maximum */
#define FP_STATUS_SOURCES     4 /* the patch struct's n_sources differs from the plan's, or exceeds MAXSOURCES */

/* One-line description of the most recent error on the calling thread. */
FP_API const char *fp_error_string(void);

/* Library version as an integer (major*10000 + minor*100 + patch). */
FP_API int fp_version(void);

/* Size checks a binding can run at load time: returns sizeof of the four
 * boundary records in out[0..3] (patch, source, response, psf gaussian). */
FP_API int fp_struct_sizes(int32_t out[4]);

/* ------------------------------------------------------------------------- */
/* Plain path: one patch per launch, port-equivalent decomposition.          */
/* ------------------------------------------------------------------------- */

/* Evaluate one proposal on one patch with the reference's decomposition:
 * one 1024-thread CTA per band, the band's image-Gaussian table in shared
 * memory, one pixel per thread, warp-shuffle + shared-atomic accumulation.
 * This is the comparator for the batched path.
 *
 * Replaces the pycuda launch in GPUProposer.evaluate_proposal
 * (forcepho/proposal.py:133-136) of EvaluateProposal
 * (forcepho/src/compute_gaussians_kernel.cu:212-312).
 *
 *   d_patch                device fp_patch
 *   d_proposal             device fp_source[n_sources]
 *   n_bands                grid size (number of bands in the patch)
 *   max_gauss_per_exposure n_sources * max_b n_psf_per_source[b]; sizes shared memory
 *   d_chi2                 device f64[n_bands]
 *   d_response             device fp_response[n_bands]
 */
FP_API int fp_evaluate_proposal_plain(const fp_patch *d_patch, const fp_source *d_proposal,
                               int n_bands, int max_gauss_per_exposure,
                               double *d_chi2, fp_response *d_response, void *stream);

/* The same evaluation in FP64 on the device: image Gaussians, pixel models,
 * residuals, chi2 and every gradient term in double precision, with the
 * reference's formulas (compute_gaussians_kernel.cc:227-315) and its
 * MAX_EXP_ARG skip.  A precision reference at full size: the FP32 paths are
 * compared against it on whole workloads, where the CPU oracle would take
 * hours.  Sums use FP64 atomics, so results are exact to about 1e-15 but not
 * bitwise reproducible.
 *
 *   d_patch, d_proposal      as fp_evaluate_proposal_plain
 *   n_bands, n_exposures     the patch's counts
 *   max_gauss_per_exposure   n_sources * max_b n_psf_per_source[b]
 *   d_chi2                   device f64[n_bands]
 *   d_dchi2                  device f64[n_bands][MAXSOURCES * NPARAMS], source-major like
 *                            fp_response (entries past n_sources are zero)
 *   d_workspace              device buffer of fp_f64_workspace_bytes bytes, 256-byte aligned
 * Queued on `stream`; an exposure with more Gaussians than max_gauss_per_exposure
 * sets FP_STATUS_GAUSS_COUNT in the workspace's status word (fp_read_status on
 * d_workspace) and contributes nothing. */
FP_API int fp_f64_workspace_bytes(int n_exposures, int max_gauss_per_exposure, size_t *out);
FP_API int fp_evaluate_proposal_f64(const fp_patch *d_patch, const fp_source *d_proposal, int n_bands,
                                    int n_exposures, int max_gauss_per_exposure, double *d_chi2,
                                    double *d_dchi2, void *d_workspace, size_t workspace_bytes,
                                    void *stream);

/* One proposal on one patch with the kernel ABI of the reference's
 * EvaluateProposal (forcepho/src/compute_gaussians_kernel.cu:212-214, launched
 * by GPUProposer.evaluate_proposal, forcepho/proposal.py:96-152): device patch
 * struct, device sources[n_sources], outputs chi2[n_bands] (f64) and
 * Response[n_bands], evaluated by the tiled B200 kernels (the path of
 * fp_evaluate_batch, not the plain comparator).
 *
 * The tiled kernels need a work plan of the patch.  The library keeps one per
 * device patch struct (and device), made on first use from the patch's own
 * device arrays and kept while the struct's xpix/ypix/index-array pointers,
 * n_sources and the index arrays' contents stay the same; otherwise it is
 * made anew.  Each call therefore reads the 152-byte struct and the index
 * arrays back to the host (two waits on `stream`; a new plan adds one for the
 * coordinates), then queues three launches that produce the results
 * asynchronously on `stream`.  Tile bounding boxes are recomputed every call,
 * so coordinates rewritten in place stay exact.  Plans (tables and workspace:
 * about 216 B per image Gaussian plus 40 B per pixel tile) are device memory
 * owned by the library, at most 64 of them (least recently used first out),
 * until fp_evaluate_proposal_release.  Calls on one patch must not overlap on
 * the GPU: they share its plan's workspace.  n_sources must equal the struct's
 * n_sources (FP_ERR_ARGUMENT otherwise). */
FP_API int fp_evaluate_proposal(const fp_patch *d_patch, const fp_source *d_sources, int n_sources,
                                int n_bands, double *d_chi2, fp_response *d_response, void *stream);

/* Free every plan fp_evaluate_proposal keeps (waits for the device first).
 * No counterpart in the reference (its kernel keeps no state). */
FP_API int fp_evaluate_proposal_release(void);

/* ------------------------------------------------------------------------- */
/* Tiled / batched path.                                                     */
/* ------------------------------------------------------------------------- */
/* A "plan" covers one or many patches whose pixel layout is fixed.  It splits
 * every exposure into spatially compact pixel tiles (the work items of one
 * persistent launch: square cells of the image plane, see fp_plan_count) and
 * lays out the workspace.  Planning runs on the host from the host copies of
 * each patch's index arrays and pixel coordinates; the caller copies the host
 * tables the plan fills to device memory and passes them, as fp_plan_tables,
 * to fp_evaluate_batch. */

/* Host-side shape of one patch (pointers are host copies of the index arrays). */
typedef struct fp_patch_shape {
    int32_t n_bands;
    int32_t n_exposures;
    int32_t n_sources;
    int32_t n_pix;                      /* total (padded) pixels */
    const int32_t *exposure_start;      /* [n_exposures] */
    const int32_t *exposure_N;          /* [n_exposures] */
    const int16_t *band_start;          /* [n_bands] */
    const int16_t *band_N;              /* [n_bands] */
    const int32_t *n_psf_per_source;    /* [n_bands] */
    const float *xpix;                  /* [n_pix] or NULL (then tiles are runs of consecutive pixels) */
    const float *ypix;                  /* [n_pix] or NULL */
} fp_patch_shape;

/* Device descriptor of one exposure of one patch (planner output). */
typedef struct fp_exposure_desc {
    int64_t gauss_offset;   /* first image Gaussian of this exposure in the Gaussian table */
    int32_t patch;          /* patch index in the plan */
    int32_t exposure;       /* exposure index within the patch */
    int32_t band;           /* band index within the patch */
    int32_t n_gauss;        /* n_sources * n_psf_per_source[band] */
    int32_t n_psf;          /* n_psf_per_source[band] */
    int32_t n_sources;
} fp_exposure_desc;        /* 32 bytes */

/* Device work item: one tile of pixels of one exposure. */
typedef struct fp_tile {
    int64_t partial_offset; /* first double of this tile's partials in the workspace */
    int32_t expo;           /* index into the plan's fp_exposure_desc table */
    int32_t perm_start;     /* first entry of this tile in the plan's pixel order */
    int32_t n_pix;          /* pixels in the tile (<= tile_pixels) */
    int32_t tile_pixels;    /* the tile's size class (256, 512 or 1024): 1, 2 or 4 pixels per thread */
    float bbox[4];          /* xmin, xmax, ymin, ymax of the tile's pixels (device-filled) */
} fp_tile;                 /* 40 bytes */

/* Device descriptor of one (patch, band) output. */
typedef struct fp_band_desc {
    int32_t patch;          /* patch index in the plan */
    int32_t band;           /* band index within the patch */
    int32_t tile_begin;     /* tiles [tile_begin, tile_end) in canonical order hold this band */
    int32_t tile_end;
    int32_t n_sources;
    int32_t pad;
} fp_band_desc;            /* 24 bytes */

/* Sizes of a plan (filled by fp_plan_count). */
typedef struct fp_plan_sizes {
    int64_t n_exposures;    /* fp_exposure_desc entries */
    int64_t n_tiles;        /* fp_tile entries */
    int64_t n_band_outputs; /* fp_band_desc entries */
    int64_t n_gauss;        /* image Gaussians per evaluation, all exposures */
    int64_t n_pairs;        /* (pixel, image Gaussian) pairs per evaluation */
    int64_t n_partials;     /* doubles of per-tile partial sums */
    int64_t max_gauss;      /* largest image-Gaussian count of one exposure */
    int64_t workspace_bytes;/* device workspace fp_evaluate_batch needs */
    int64_t n_perm;         /* entries of the plan's pixel order (sum of exposure_N) */
} fp_plan_sizes;

/* The device copies of a plan's tables (a host struct of device pointers). */
typedef struct fp_plan_tables {
    const fp_exposure_desc *expos;  /* [n_exposures] */
    fp_tile *tiles;                 /* [n_tiles], canonical order (patch, band, exposure, cell) */
    const int32_t *order;           /* [n_tiles] execution order, most work first */
    const fp_band_desc *bands;      /* [n_band_outputs] */
    const int32_t *perm;            /* [n_perm] index within its patch of every tile pixel, tile after tile */
    const float *pix;               /* [n_perm][4] (x, y, data, ierr) of every tile pixel in the same order,
                                       16-byte aligned (fp_plan_pack), or NULL: the tile kernel then reads
                                       the patch arrays through perm */
} fp_plan_tables;

/* Count the plan of `n_patches` patches split into tiles of at most
 * `tile_pixels` pixels (a multiple of 32, at most 4096).  With pixel
 * coordinates, each exposure's pixels are grouped into cells of the image
 * plane (32x32 pixels for 1024-pixel tiles, 32x16 for 512, 16x16 for 256),
 * cells taken row by row and pixels within a cell in their input order; a cell
 * with more pixels than a tile is split. */
FP_API int fp_plan_count(const fp_patch_shape *h_shapes, int n_patches, int tile_pixels,
                  fp_plan_sizes *out);

/* Tile size by exposure size: a plan may hold tiles of several size classes,
 * all evaluated in the same persistent launch.  An exposure of n pixels takes
 * the first class c with n <= max_exposure_pixels[c] (the last class takes
 * every larger one) and is split into tiles of tile_pixels[c] pixels (cells of
 * the image plane as for fp_plan_count).  With more than one class each
 * class's size must be one the kernels run (256, 512 or 1024; FP_ERR_ARGUMENT
 * otherwise); the launch's tile_pixels must be the largest class of the plan. */
#define FP_MAX_TILE_CLASSES 4
typedef struct fp_tile_rule {
    int32_t n_classes;                               /* 1 .. FP_MAX_TILE_CLASSES */
    int32_t max_exposure_pixels[FP_MAX_TILE_CLASSES];  /* ascending; ignored for the last class */
    int32_t tile_pixels[FP_MAX_TILE_CLASSES];
} fp_tile_rule;

/* fp_plan_count and fp_plan_fill with a tile rule instead of one tile size. */
FP_API int fp_plan_count_rule(const fp_patch_shape *h_shapes, int n_patches, const fp_tile_rule *rule,
                              fp_plan_sizes *out);
FP_API int fp_plan_fill_rule(const fp_patch_shape *h_shapes, int n_patches, const fp_tile_rule *rule,
                             fp_exposure_desc *h_expos, fp_tile *h_tiles, fp_band_desc *h_bands,
                             int32_t *h_order, int32_t *h_perm);

/* Fill the host tables of a plan (sizes from fp_plan_count).  Tiles are emitted
 * in canonical order (patch, band, exposure, cell); h_order receives an
 * execution order (largest estimated work first) of length n_tiles, h_perm the
 * plan's pixel order (n_perm entries). */
FP_API int fp_plan_fill(const fp_patch_shape *h_shapes, int n_patches, int tile_pixels,
                 fp_exposure_desc *h_expos, fp_tile *h_tiles, fp_band_desc *h_bands,
                 int32_t *h_order, int32_t *h_perm);

/* One-time device pass after the tables are uploaded: computes each tile's
 * pixel bounding box (into tables->tiles) from the patch's xpix/ypix.
 * d_patches: device array of n_patches device fp_patch pointers. */
FP_API int fp_plan_bbox(const fp_patch *const *d_patches, const fp_plan_sizes *sizes,
                        const fp_plan_tables *tables, void *stream);

/* Fill d_pix[n_perm][4] with the (x, y, data, ierr) records of every tile
 * pixel in the plan's pixel order (gathered through tables->perm) and
 * recompute the tile boxes.  With tables->pix = d_pix, fp_evaluate_batch then
 * reads each pixel as one contiguous 16-byte record instead of four gathers
 * through the index array.  The records are a copy: run this again whenever
 * any patch's data, ierr, xpix or ypix values or pointers change (for example
 * after a data/residual swap), before the next evaluation on that stream.
 * No reference counterpart (the reference kernel reads the SoA arrays). */
FP_API int fp_plan_pack(const fp_patch *const *d_patches, const fp_plan_sizes *sizes,
                        const fp_plan_tables *tables, float *d_pix, void *stream);

/* Launch parameters of the batched evaluation (chosen by the autotuner). */
typedef struct fp_launch {
    int32_t tile_pixels;    /* pixels per tile: 256, 512 or 1024; the plan's largest tile class */
    int32_t ctas_per_sm;    /* persistent CTAs per SM (grid = ctas_per_sm * SM count) */
    int32_t flags;          /* FP_FLAG_* */
    int32_t phases;         /* FP_PHASE_* bits to run; 0 = all three */
} fp_launch;

#define FP_FLAG_NO_CULL     1   /* evaluate every (tile, Gaussian) pair (no bounding-box culling) */
#define FP_FLAG_STATIC      2   /* static round-robin tile assignment instead of an atomic queue */
#define FP_FLAG_FORWARD_ONLY 4  /* model, residual and chi2 only: the adjoint pass is skipped and the
                                   Response records are zero (renders, fixed-source subtraction) */

#define FP_PHASE_SETUP      1   /* image-Gaussian tables (must precede the tile phase) */
#define FP_PHASE_TILES      2   /* the persistent tile kernel */
#define FP_PHASE_REDUCE     4   /* fixed-order reduction into chi2 / response */

/* Shared memory one tile CTA needs for a tile size and largest exposure
 * Gaussian count (for occupancy planning). */
FP_API int fp_tile_smem_bytes(int tile_pixels, int64_t max_gauss, int64_t *out);

/* Evaluate one proposal per patch for every patch of a plan in one pass
 * (Gaussian setup, one persistent tile launch, fixed-order reduction).
 *   d_patches     device array [n_patches] of device fp_patch pointers
 *   sizes         the plan's sizes (host struct from fp_plan_count)
 *   tables        the plan's device tables (tiles after fp_plan_bbox)
 *   d_proposals   device fp_source[n_patches][MAXSOURCES] (rows >= n_sources unused)
 *   d_chi2        device f64[n_patches][MAXBANDS]        (bands >= n_bands untouched)
 *   d_response    device fp_response[n_patches][MAXBANDS]
 *   d_workspace   device buffer of at least sizes->workspace_bytes, 256-byte aligned
 * Replaces, for many patches at once, the per-patch GPUProposer.evaluate_proposal
 * launch (forcepho/proposal.py:96-152).  Results are bitwise reproducible for
 * fixed inputs and launch parameters. */
FP_API int fp_evaluate_batch(const fp_patch *const *d_patches, int n_patches, const fp_plan_sizes *sizes,
                      const fp_plan_tables *tables,
                      const fp_source *d_proposals, double *d_chi2, fp_response *d_response,
                      void *d_workspace, size_t workspace_bytes, const fp_launch *launch,
                      void *stream);

/* Pair census of a plan (diagnostic; needs the Gaussian tables of a prior
 * fp_evaluate_batch in the same workspace).  Adds to d_counts[0..2] (zero them
 * first): [0] (pixel, Gaussian) pairs the culled tile kernel evaluates,
 * [1] pairs within the MAX_EXP_ARG cutoff, [2] within-cutoff pairs of Gaussians
 * the cull dropped (0 unless culling is wrong).  No reference counterpart. */
FP_API int fp_count_pairs(const fp_patch *const *d_patches, const fp_plan_sizes *sizes,
                          const fp_plan_tables *tables,
                          const void *d_workspace, size_t workspace_bytes,
                          unsigned long long *d_counts, void *stream);

/* Measure FP32 FMA throughput (TFLOP/s, FMA = 2 flops) and SFU ex2
 * throughput (results/s) of the current device with two short kernels; the
 * roofline denominators of this path.  d_scratch: 256 floats.  Synchronises
 * `stream`.  No reference counterpart (measurement utility). */
FP_API int fp_measure_peaks(float *d_scratch, double *fp32_tflops, double *ex2_per_s, void *stream);

/* ------------------------------------------------------------------------- */
/* Device-resident HMC around the batched likelihood.                        */
/* ------------------------------------------------------------------------- */
/* The host-side steps the reference runs per likelihood call -- the sigmoid
 * parameter transform (forcepho/model.py:596-637), the proposal with spline
 * amplitudes (forcepho/sources.py:607-681), lnp and stack_grad
 * (forcepho/model.py:302-387) -- as device launches, plus fixed-length HMC
 * leapfrog / Metropolis updates standing in for the NUTS sampler of
 * forcepho/fitting.py:254-341.  All scalars live in device memory, so the
 * launches of a trajectory can be captured into one CUDA graph. */

/* Tensor-product B-spline tables of the Sersic mixture amplitudes
 * A_r(sersic, rhalf), r < n_radii (scipy RectBivariateSpline knots and
 * coefficients; x = sersic, y = rhalf).  Pointers are device pointers. */
typedef struct fp_spline_table {
    int32_t n_radii;
    int32_t nx, ny;          /* knot counts */
    int32_t kx, ky;          /* degrees */
    int32_t pad;
    const double *tx;        /* [nx] */
    const double *ty;        /* [ny] */
    const double *coef;      /* [n_radii][(nx-kx-1)*(ny-ky-1)], x-major */
} fp_spline_table;

/* Parameter layout of one patch: per active source
 * [flux_1..flux_nb, ra, dec, q, pa, sersic, rhalf] (forcepho/sources.py:559-605). */
typedef struct fp_hmc_patch {
    int64_t param_offset;    /* first parameter of the patch in the flat state vectors */
    int32_t n_sources;
    int32_t n_bands;
} fp_hmc_patch;              /* 16 bytes */

/* theta = lower + (upper - lower) sigmoid(z) (theta = z when d_lower is NULL),
 * the proposal records d_proposals[n_patches][MAXSOURCES] from theta (spline
 * amplitudes and their sersic / rhalf derivatives evaluated on the device), and
 * the transform's diagonal Jacobian d_jac = dtheta/dz. */
FP_API int fp_hmc_prepare(const fp_hmc_patch *d_hp, int n_patches, const double *d_z,
                          const double *d_lower, const double *d_upper, const fp_spline_table *tab,
                          fp_source *d_proposals, double *d_theta, double *d_jac, void *stream);

/* lnp[p] = -1/2 sum_b chi2[p][b] (+ log|dtheta/dz| when transformed && sampling)
 * and grad = dlnp/dz = (-1/2 stack_grad(dchi2)) dtheta/dz (+ 1 - 2 sigmoid(z)),
 * from the outputs of fp_evaluate_batch. */
FP_API int fp_hmc_lnprob(const fp_hmc_patch *d_hp, int n_patches, const double *d_z, const double *d_jac,
                         const double *d_chi2, const fp_response *d_response, int transformed,
                         int sampling, double *d_lnp, double *d_grad, void *stream);

/* State of HMC over all patches (device pointers). */
typedef struct fp_hmc_state {
    int64_t n_params;        /* parameters over all patches */
    double *z, *p, *grad;    /* [n_params] position (unconstrained), momentum, dlnp/dz */
    double *z0, *grad0;      /* [n_params] saved at the start of a trajectory */
    const double *inv_mass;  /* [n_params] diagonal inverse mass matrix */
    const double *eps;       /* [n_patches] leapfrog step sizes */
    double *lnp, *lnp0, *h0; /* [n_patches] current / saved lnp, initial energy */
    double *energy_error;    /* [n_patches] H0 - H1 of the last trajectory */
    int32_t *accepted;       /* [n_patches] accepted trajectories */
    const double *normals;   /* [n_traj][n_params] standard normal draws */
    const double *uniforms;  /* [n_traj][n_patches] uniform draws */
    int64_t *traj;           /* current trajectory index (advanced by FP_HMC_END) */
    int64_t n_traj;          /* rows of normals/uniforms; trajectory t uses row t % n_traj */
} fp_hmc_state;

#define FP_HMC_BEGIN 0   /* draw momentum, save state, half kick, drift */
#define FP_HMC_STEP  1   /* full kick, drift (between two gradient evaluations) */
#define FP_HMC_END   2   /* half kick, Metropolis accept/restore, advance traj */

/* One stage of a leapfrog trajectory (see FP_HMC_*). */
FP_API int fp_hmc_leapfrog(const fp_hmc_patch *d_hp, int n_patches, const fp_hmc_state *state, int stage,
                           void *stream);

/* Size of the fixed device scratch array of fp_evaluate_batch_noalloc (32 MiB). */
#define FP_NOALLOC_WORKSPACE_BYTES (32u << 20)

/* fp_evaluate_batch without a workspace argument, for callers that cannot
 * allocate device memory: a host-language binding that only holds raw device
 * pointers given to it by another runtime and has no CUDA allocator of its
 * own, or a process whose device memory is all reserved by another
 * allocator's pool, where an extra cudaMalloc would fail or fragment it.
 * No counterpart in the reference (its kernel needs no scratch memory).
 *
 * The scratch is a file-scope device array of FP_NOALLOC_WORKSPACE_BYTES that
 * every GPU loading the library holds until the process exits.  Plans whose
 * sizes->workspace_bytes exceed it are rejected with FP_ERR_WORKSPACE (a
 * single patch of 30 sources x 8 bands x 4 exposures of 256x256 pixels needs
 * about 15 MB; a 512-patch batch does not fit).  The caller still passes all
 * inputs and outputs; nothing is allocated or freed.  Arguments are checked
 * before anything is queued, so a rejected call leaves the array and the
 * stream untouched.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current and keeps it, so
 * make that first call before any stream capture; the kept address belongs to
 * the device's primary context, so a process that calls cudaDeviceReset on a
 * device must not use this entry point on it afterwards.  All calls share the
 * array and it keeps the previous call's contents (each call clears the part
 * that must start at zero, including the status word): calls that overlap on
 * the GPU, on different streams or from different threads, race and corrupt
 * each other's results. */
FP_API int fp_evaluate_batch_noalloc(const fp_patch *const *d_patches, int n_patches,
                                     const fp_plan_sizes *sizes, const fp_plan_tables *tables,
                                     const fp_source *d_proposals,
                                     double *d_chi2, fp_response *d_response, const fp_launch *launch,
                                     void *stream);

/* Read and clear the device status word written by the batched kernels
 * (0 = no inconsistency seen; FP_STATUS_* bits otherwise).  Synchronises
 * `stream`. */
FP_API int fp_read_status(void *d_workspace, int32_t *status_out, void *stream);

/* fp_read_status for the fixed array of fp_evaluate_batch_noalloc: the
 * FP_STATUS_* bits of the last fp_evaluate_batch_noalloc call on the current
 * device (each call clears them at its start), then cleared.  Call it on the
 * stream of that call; it synchronises `stream`.  A call whose patch no longer
 * matches its plan reports FP_STATUS_SOURCES here and returns a zero model
 * (chi2 0, gradient 0) for the exposures concerned.  No counterpart in the
 * reference; it allocates nothing either. */
FP_API int fp_read_status_noalloc(int32_t *status_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FORCEPHO_B200_H */
