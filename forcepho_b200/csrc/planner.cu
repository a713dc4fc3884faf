// planner.cpp -- host-side work planning of the tiled/batched path.
//
// A plan splits every exposure of every patch into tiles of at most
// `tile_pixels` consecutive pixels (the work items of one persistent launch),
// numbers the image Gaussians of every exposure, and lays out the per-tile
// partial sums.  It depends only on each patch's index arrays (pixel layout),
// never on the proposal, so it is built once per set of patches.

#include <algorithm>
#include <numeric>
#include <vector>

#include "fp_common.cuh"

namespace {

int check_shape(const fp_patch_shape &s, int p)
{
    if (s.n_bands < 1 || s.n_bands > MAXBANDS)
        return fp_set_error(FP_ERR_LIMITS, "patch %d: n_bands=%d outside [1,%d]", p, s.n_bands, MAXBANDS);
    if (s.n_sources < 0 || s.n_sources > MAXSOURCES)
        return fp_set_error(FP_ERR_LIMITS, "patch %d: n_sources=%d outside [0,%d]", p, s.n_sources,
                            MAXSOURCES);
    if (s.n_exposures < 0 || !s.exposure_start || !s.exposure_N || !s.band_start || !s.band_N ||
        !s.n_psf_per_source)
        return fp_set_error(FP_ERR_ARGUMENT, "patch %d: missing index array", p);
    int64_t next = 0;
    for (int b = 0; b < s.n_bands; ++b) {
        if (s.band_start[b] != next || s.band_N[b] < 0)
            return fp_set_error(FP_ERR_ARGUMENT, "patch %d: band_start/band_N do not tile the exposures", p);
        next += s.band_N[b];
        if (s.n_psf_per_source[b] <= 0)
            return fp_set_error(FP_ERR_ARGUMENT, "patch %d: n_psf_per_source[%d]=%d", p, b,
                                s.n_psf_per_source[b]);
        if ((int64_t)s.n_psf_per_source[b] * s.n_sources > 65535)
            return fp_set_error(FP_ERR_LIMITS, "patch %d band %d: more than 65535 image Gaussians", p, b);
    }
    if (next != s.n_exposures)
        return fp_set_error(FP_ERR_ARGUMENT, "patch %d: bands hold %lld exposures, n_exposures=%d", p,
                            (long long)next, s.n_exposures);
    for (int e = 0; e < s.n_exposures; ++e) {
        if (s.exposure_start[e] < 0 || s.exposure_N[e] < 0 ||
            (int64_t)s.exposure_start[e] + s.exposure_N[e] > s.n_pix)
            return fp_set_error(FP_ERR_ARGUMENT, "patch %d exposure %d: pixels [%d, +%d) outside [0, %d)", p,
                                e, s.exposure_start[e], s.exposure_N[e], s.n_pix);
    }
    return FP_OK;
}

int check_tile_pixels(int tile_pixels)
{
    if (tile_pixels < 32 || tile_pixels > 4096 || tile_pixels % 32)
        return fp_set_error(FP_ERR_ARGUMENT, "tile_pixels=%d must be a multiple of 32 in [32, 4096]",
                            tile_pixels);
    return FP_OK;
}

}  // namespace

extern "C" int fp_plan_count(const fp_patch_shape *h_shapes, int n_patches, int tile_pixels,
                             fp_plan_sizes *out)
{
    if (!h_shapes || !out || n_patches < 1) return fp_set_error(FP_ERR_ARGUMENT, "fp_plan_count: bad arguments");
    if (int rc = check_tile_pixels(tile_pixels)) return rc;
    fp_plan_sizes z = {};
    for (int p = 0; p < n_patches; ++p) {
        const fp_patch_shape &s = h_shapes[p];
        if (int rc = check_shape(s, p)) return rc;
        for (int b = 0; b < s.n_bands; ++b) {
            const int64_t ng = (int64_t)s.n_sources * s.n_psf_per_source[b];
            for (int e = s.band_start[b]; e < s.band_start[b] + s.band_N[b]; ++e) {
                const int64_t nt = (s.exposure_N[e] + tile_pixels - 1) / tile_pixels;
                z.n_exposures += 1;
                z.n_tiles += nt;
                z.n_gauss += ng;
                z.n_pairs += ng * s.exposure_N[e];
                z.n_partials += nt * (1 + (int64_t)NPARAMS * s.n_sources);
                z.max_gauss = std::max(z.max_gauss, ng);
            }
            z.n_band_outputs += 1;
        }
    }
    if (z.n_tiles > INT32_MAX) return fp_set_error(FP_ERR_LIMITS, "plan has more than 2^31 tiles");
    z.workspace_bytes = (int64_t)fp_layout(z.n_gauss, z.n_partials).total;
    *out = z;
    return FP_OK;
}

extern "C" int fp_plan_fill(const fp_patch_shape *h_shapes, int n_patches, int tile_pixels,
                            fp_exposure_desc *h_expos, fp_tile *h_tiles, fp_band_desc *h_bands,
                            int32_t *h_order)
{
    fp_plan_sizes z;
    if (int rc = fp_plan_count(h_shapes, n_patches, tile_pixels, &z)) return rc;
    if (!h_expos || !h_tiles || !h_bands || !h_order)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_plan_fill: NULL output table");

    int64_t ie = 0, it = 0, ib = 0, goff = 0, poff = 0;
    std::vector<int64_t> work((size_t)z.n_tiles);
    for (int p = 0; p < n_patches; ++p) {
        const fp_patch_shape &s = h_shapes[p];
        const int64_t stride = 1 + (int64_t)NPARAMS * s.n_sources;
        for (int b = 0; b < s.n_bands; ++b) {
            fp_band_desc &bd = h_bands[ib++];
            bd.patch = p;
            bd.band = b;
            bd.tile_begin = (int32_t)it;
            bd.n_sources = s.n_sources;
            bd.pad = 0;
            const int n_psf = s.n_psf_per_source[b];
            const int ng = s.n_sources * n_psf;
            for (int e = s.band_start[b]; e < s.band_start[b] + s.band_N[b]; ++e) {
                fp_exposure_desc &ed = h_expos[ie];
                ed.gauss_offset = goff;
                ed.patch = p;
                ed.exposure = e;
                ed.band = b;
                ed.n_gauss = ng;
                ed.n_psf = n_psf;
                ed.n_sources = s.n_sources;
                const int N = s.exposure_N[e];
                for (int k = 0; k * tile_pixels < N; ++k) {
                    fp_tile &t = h_tiles[it];
                    t.partial_offset = poff;
                    t.expo = (int32_t)ie;
                    t.pix_start = s.exposure_start[e] + k * tile_pixels;
                    t.n_pix = std::min(tile_pixels, N - k * tile_pixels);
                    t.pad = 0;
                    t.bbox[0] = t.bbox[1] = t.bbox[2] = t.bbox[3] = 0.f;
                    work[(size_t)it] = (int64_t)t.n_pix * ng;
                    poff += stride;
                    ++it;
                }
                goff += ng;
                ++ie;
            }
            bd.tile_end = (int32_t)it;
        }
    }
    // execution order: most work first (stable), so the persistent queue ends on small items
    std::vector<int32_t> ord((size_t)z.n_tiles);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) { return work[a] > work[b]; });
    std::copy(ord.begin(), ord.end(), h_order);
    return FP_OK;
}
