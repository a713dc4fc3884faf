/* A C host of the library's ABI, as a cgo / JNI / FFI binding would use it:
 * plain C99, only include/forcepho_b200.h.  Runs without a GPU: it checks the
 * record sizes, plans a two-exposure patch on the host (fp_plan_count /
 * fp_plan_fill) and prints the plan's sizes, then calls an evaluation entry
 * point with a NULL argument and prints the library's error code and message.
 *
 *   gcc -std=c99 -I include tests/c/abi_example.c -L forcepho_b200/lib -lforcepho_b200 -o abi_example
 */
#include <stdio.h>
#include <stdlib.h>

#include "forcepho_b200.h"

int main(void)
{
    int32_t sizes[4];
    if (fp_struct_sizes(sizes) != FP_OK) return 1;
    printf("version %d sizes %d %d %d %d\n", fp_version(), sizes[0], sizes[1], sizes[2], sizes[3]);

    /* one band, two exposures of a 40x24 raster */
    enum { W = 40, H = 24, N = W * H };
    static float xpix[2 * N], ypix[2 * N];
    for (int e = 0; e < 2; ++e)
        for (int i = 0; i < N; ++i) {
            xpix[e * N + i] = (float)(i % W);
            ypix[e * N + i] = (float)(i / W);
        }
    int32_t exposure_start[2] = {0, N}, exposure_N[2] = {N, N}, n_psf[1] = {9};
    int16_t band_start[1] = {0}, band_N[1] = {2};
    fp_patch_shape shape = {1, 2, 3, 2 * N, exposure_start, exposure_N, band_start, band_N, n_psf, xpix, ypix};

    fp_plan_sizes z;
    int rc = fp_plan_count(&shape, 1, 256, &z);
    if (rc != FP_OK) {
        printf("fp_plan_count failed: %s\n", fp_error_string());
        return 1;
    }
    fp_exposure_desc *expos = calloc((size_t)z.n_exposures, sizeof(*expos));
    fp_tile *tiles = calloc((size_t)z.n_tiles, sizeof(*tiles));
    fp_band_desc *bands = calloc((size_t)z.n_band_outputs, sizeof(*bands));
    int32_t *order = calloc((size_t)z.n_tiles, sizeof(*order));
    int32_t *perm = calloc((size_t)z.n_perm, sizeof(*perm));
    rc = fp_plan_fill(&shape, 1, 256, expos, tiles, bands, order, perm);
    if (rc != FP_OK) {
        printf("fp_plan_fill failed: %s\n", fp_error_string());
        return 1;
    }
    long long seen = 0;
    for (long long t = 0; t < z.n_tiles; ++t) seen += tiles[t].n_pix;
    printf("plan tiles %lld gauss %lld pairs %lld perm %lld pixels_in_tiles %lld workspace %lld\n",
           (long long)z.n_tiles, (long long)z.n_gauss, (long long)z.n_pairs, (long long)z.n_perm, seen,
           (long long)z.workspace_bytes);

    rc = fp_evaluate_proposal(NULL, NULL, 3, 1, NULL, NULL, NULL);
    printf("null call rc %d: %s\n", rc, fp_error_string());
    free(expos); free(tiles); free(bands); free(order); free(perm);
    return rc == FP_ERR_ARGUMENT ? 0 : 1;
}
