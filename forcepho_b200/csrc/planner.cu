// planner.cu -- host-side work planning of the tiled/batched path.
//
// A plan splits every exposure of every patch into tiles (the work items of
// one persistent launch), numbers the image Gaussians of every exposure, and
// lays out the per-tile partial sums.  It depends only on each patch's pixel
// layout (index arrays and pixel coordinates), never on the proposal, so it is
// built once per set of patches.
//
// Tiles are spatially compact: each exposure's pixels are grouped into square
// cells of the image plane (32x32 pixels for 1024-pixel tiles, 32x16 for 512,
// 16x16 for 256), cells ordered row by row, pixels within a cell kept in their
// input order.  The tile size may differ between exposures (a tile rule of up
// to FP_MAX_TILE_CLASSES classes by exposure pixel count); each tile records
// its class, and one persistent launch evaluates tiles of every class.  The plan's pixel order (`perm`) lists, tile after tile, the
// index of every pixel within its patch.  A compact tile has a small bounding
// box, so the per-tile culling of image Gaussians keeps few that do not reach
// its pixels.  Without coordinates (xpix == NULL) tiles are runs of
// consecutive pixels.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>
#include <thread>
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
    if (s.n_exposures < 0 || s.n_pix < 0 || !s.exposure_start || !s.exposure_N || !s.band_start || !s.band_N ||
        !s.n_psf_per_source)
        return fp_set_error(FP_ERR_ARGUMENT, "patch %d: missing index array", p);
    if ((s.xpix == nullptr) != (s.ypix == nullptr))
        return fp_set_error(FP_ERR_ARGUMENT, "patch %d: give both xpix and ypix, or neither", p);
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

int check_rule(const fp_tile_rule *r)
{
    if (!r || r->n_classes < 1 || r->n_classes > FP_MAX_TILE_CLASSES)
        return fp_set_error(FP_ERR_ARGUMENT, "tile rule: n_classes must be in [1, %d]", FP_MAX_TILE_CLASSES);
    for (int c = 0; c < r->n_classes; ++c) {
        const int tp = r->tile_pixels[c];
        // a launch covers every class of its plan, so each must be a size the tile kernel runs
        if (r->n_classes > 1 && tp != 256 && tp != 512 && tp != 1024)
            return fp_set_error(FP_ERR_ARGUMENT, "tile rule: class %d has tile_pixels=%d (supported: 256, 512, 1024)",
                                c, tp);
        if (int rc = check_tile_pixels(tp)) return rc;
        if (c > 0 && c < r->n_classes - 1 && r->max_exposure_pixels[c] < r->max_exposure_pixels[c - 1])
            return fp_set_error(FP_ERR_ARGUMENT, "tile rule: class bounds must ascend");
    }
    return FP_OK;
}

fp_tile_rule single_class(int tile_pixels)
{
    fp_tile_rule r = {};
    r.n_classes = 1;
    r.max_exposure_pixels[0] = INT32_MAX;
    r.tile_pixels[0] = tile_pixels;
    return r;
}

// Tile size of an exposure of n pixels: the first class whose bound holds it.
int rule_tile(const fp_tile_rule &r, int n)
{
    for (int c = 0; c < r.n_classes - 1; ++c)
        if (n <= r.max_exposure_pixels[c]) return r.tile_pixels[c];
    return r.tile_pixels[r.n_classes - 1];
}

// cell width x height (pixels) of a tile size: the squarest power-of-two
// rectangle of tile_pixels pixels, wider than tall
void cell_dims(int tile_pixels, int *cw, int *ch)
{
    int w = 1, h = 1;
    while (w * h * 2 <= tile_pixels) {
        if (w <= h) w *= 2; else h *= 2;
    }
    *cw = w;
    *ch = h;
}

// Pixel order of one exposure (local indices 0..N-1) and its tile sizes.
// order == nullptr: only count the tiles.
void exposure_tiles(const fp_patch_shape &s, int e, int tile_pixels, std::vector<int32_t> *order,
                    std::vector<int32_t> &tile_n)
{
    const int N = s.exposure_N[e];
    const int start = s.exposure_start[e];
    tile_n.clear();
    if (order) order->clear();
    if (N == 0) return;
    if (s.xpix == nullptr) {   // consecutive runs
        for (int k = 0; k < N; k += tile_pixels) tile_n.push_back(std::min(tile_pixels, N - k));
        if (order) {
            order->resize(N);
            std::iota(order->begin(), order->end(), 0);
        }
        return;
    }
    int cw, ch;
    cell_dims(tile_pixels, &cw, &ch);
    const float *x = s.xpix + start, *y = s.ypix + start;
    float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
    for (int i = 0; i < N; ++i) {
        const float xi = x[i], yi = y[i];
        if (std::isfinite(xi) && std::isfinite(yi)) {
            x0 = std::min(x0, xi); x1 = std::max(x1, xi);
            y0 = std::min(y0, yi); y1 = std::max(y1, yi);
        }
    }
    // at most 2^30 cells per axis, so cell keys fit in int64 whatever the
    // (finite) coordinates; beyond that the outermost cells are wider
    const double max_cells = (double)(1 << 30);
    int64_t ncx = 1, ncy = 1;
    if (x1 >= x0) {
        ncx = (int64_t)std::min(((double)x1 - x0) / cw, max_cells - 1) + 1;
        ncy = (int64_t)std::min(((double)y1 - y0) / ch, max_cells - 1) + 1;
    }
    const int64_t ncell = ncx * ncy;           // key ncell: non-finite coordinates
    static thread_local std::vector<int64_t> key;
    static thread_local std::vector<int32_t> cnt;
    key.resize((size_t)N);
    const double icw = 1.0 / cw, ich = 1.0 / ch;
    for (int i = 0; i < N; ++i) {
        const float xi = x[i], yi = y[i];
        if (std::isfinite(xi) && std::isfinite(yi)) {
            // offsets are >= 0, so truncation is floor
            const int64_t cx = (int64_t)std::min(((double)xi - x0) * icw, (double)(ncx - 1));
            const int64_t cy = (int64_t)std::min(((double)yi - y0) * ich, (double)(ncy - 1));
            key[i] = cy * ncx + cx;
        } else {
            key[i] = ncell;
        }
    }
    std::vector<int32_t> ord((size_t)N);
    std::vector<int32_t> bucket_n;
    if (ncell <= 4 * (int64_t)N + 1024) {   // dense grid: stable counting sort
        cnt.assign((size_t)ncell + 2, 0);
        for (int i = 0; i < N; ++i) cnt[(size_t)key[i] + 1]++;
        for (int64_t c = 0; c <= ncell; ++c)
            if (cnt[(size_t)c + 1]) bucket_n.push_back(cnt[(size_t)c + 1]);
        if (order) {
            for (int64_t c = 1; c <= ncell + 1; ++c) cnt[(size_t)c] += cnt[(size_t)c - 1];
            for (int i = 0; i < N; ++i) ord[(size_t)cnt[(size_t)key[i]]++] = i;
        }
    } else {                                // sparse coordinates: stable sort by key
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
        for (int i = 0; i < N;) {
            int j = i;
            while (j < N && key[ord[j]] == key[ord[i]]) ++j;
            bucket_n.push_back(j - i);
            i = j;
        }
    }
    for (int32_t c : bucket_n)
        for (int k = 0; k < c; k += tile_pixels) tile_n.push_back(std::min(tile_pixels, c - k));
    if (order) order->swap(ord);
}

// Per-patch planning result (phase 1, independent per patch).
struct patch_plan {
    std::vector<int32_t> tile_n;      // tile sizes, canonical order
    std::vector<int32_t> tile_expo;   // exposure (within the patch) of each tile
    std::vector<int32_t> tile_cls;    // size class (tile_pixels) of each tile
    std::vector<int32_t> perm;        // pixel order (indices within the patch)
    int rc = FP_OK;
};

void plan_one(const fp_patch_shape &s, int p, const fp_tile_rule &rule, bool want_order, patch_plan &out)
{
    out.rc = check_shape(s, p);
    if (out.rc) return;
    std::vector<int32_t> order, tile_n;
    for (int b = 0; b < s.n_bands; ++b)
        for (int e = s.band_start[b]; e < s.band_start[b] + s.band_N[b]; ++e) {
            const int tp = rule_tile(rule, s.exposure_N[e]);
            exposure_tiles(s, e, tp, want_order ? &order : nullptr, tile_n);
            out.tile_n.insert(out.tile_n.end(), tile_n.begin(), tile_n.end());
            out.tile_expo.insert(out.tile_expo.end(), tile_n.size(), e);
            out.tile_cls.insert(out.tile_cls.end(), tile_n.size(), tp);
            if (want_order)
                for (int32_t k : order) out.perm.push_back(s.exposure_start[e] + k);
        }
}

// Phase 1 over all patches on the host's cores.
int plan_all(const fp_patch_shape *h_shapes, int n_patches, const fp_tile_rule &rule, bool want_order,
             std::vector<patch_plan> &plans)
{
    plans.assign((size_t)n_patches, patch_plan());
    unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    nt = std::min<unsigned>(nt, (unsigned)n_patches);
    std::atomic<int> next(0);
    auto work = [&]() {
        for (int p = next++; p < n_patches; p = next++) plan_one(h_shapes[p], p, rule, want_order, plans[p]);
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    for (int p = 0; p < n_patches; ++p)
        if (plans[p].rc) {   // re-run the check to report the first failing patch's message
            return check_shape(h_shapes[p], p);
        }
    return FP_OK;
}

int count_from(const fp_patch_shape *h_shapes, int n_patches, const std::vector<patch_plan> &plans,
               fp_plan_sizes *out)
{
    fp_plan_sizes z = {};
    for (int p = 0; p < n_patches; ++p) {
        const fp_patch_shape &s = h_shapes[p];
        for (int b = 0; b < s.n_bands; ++b) {
            const int64_t ng = (int64_t)s.n_sources * s.n_psf_per_source[b];
            for (int e = s.band_start[b]; e < s.band_start[b] + s.band_N[b]; ++e) {
                z.n_exposures += 1;
                z.n_gauss += ng;
                z.n_pairs += ng * s.exposure_N[e];
                z.n_perm += s.exposure_N[e];
                z.max_gauss = std::max(z.max_gauss, ng);
            }
            z.n_band_outputs += 1;
        }
        const int64_t nt = (int64_t)plans[p].tile_n.size();
        z.n_tiles += nt;
        z.n_partials += nt * (1 + (int64_t)NPARAMS * s.n_sources);
    }
    if (z.n_tiles > INT32_MAX || z.n_perm > INT32_MAX)
        return fp_set_error(FP_ERR_LIMITS, "plan has more than 2^31 tiles or pixels");
    z.workspace_bytes = (int64_t)fp_layout(z.n_gauss, z.n_partials).total;
    *out = z;
    return FP_OK;
}

}  // namespace

extern "C" int fp_plan_count_rule(const fp_patch_shape *h_shapes, int n_patches, const fp_tile_rule *rule,
                                  fp_plan_sizes *out)
{
    if (!h_shapes || !out || n_patches < 1) return fp_set_error(FP_ERR_ARGUMENT, "fp_plan_count: bad arguments");
    if (int rc = check_rule(rule)) return rc;
    std::vector<patch_plan> plans;
    if (int rc = plan_all(h_shapes, n_patches, *rule, false, plans)) return rc;
    return count_from(h_shapes, n_patches, plans, out);
}

extern "C" int fp_plan_count(const fp_patch_shape *h_shapes, int n_patches, int tile_pixels,
                             fp_plan_sizes *out)
{
    if (int rc = check_tile_pixels(tile_pixels)) return rc;
    const fp_tile_rule r = single_class(tile_pixels);
    return fp_plan_count_rule(h_shapes, n_patches, &r, out);
}

extern "C" int fp_plan_fill(const fp_patch_shape *h_shapes, int n_patches, int tile_pixels,
                            fp_exposure_desc *h_expos, fp_tile *h_tiles, fp_band_desc *h_bands,
                            int32_t *h_order, int32_t *h_perm)
{
    if (int rc = check_tile_pixels(tile_pixels)) return rc;
    const fp_tile_rule r = single_class(tile_pixels);
    return fp_plan_fill_rule(h_shapes, n_patches, &r, h_expos, h_tiles, h_bands, h_order, h_perm);
}

extern "C" int fp_plan_fill_rule(const fp_patch_shape *h_shapes, int n_patches, const fp_tile_rule *rule,
                                 fp_exposure_desc *h_expos, fp_tile *h_tiles, fp_band_desc *h_bands,
                                 int32_t *h_order, int32_t *h_perm)
{
    if (!h_shapes || n_patches < 1) return fp_set_error(FP_ERR_ARGUMENT, "fp_plan_fill: bad arguments");
    if (int rc = check_rule(rule)) return rc;
    if (!h_expos || !h_tiles || !h_bands || !h_order || !h_perm)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_plan_fill: NULL output table");
    std::vector<patch_plan> plans;
    if (int rc = plan_all(h_shapes, n_patches, *rule, true, plans)) return rc;
    fp_plan_sizes z;
    if (int rc = count_from(h_shapes, n_patches, plans, &z)) return rc;

    int64_t ie = 0, it = 0, ib = 0, goff = 0, poff = 0, pp = 0;
    std::vector<int64_t> work((size_t)z.n_tiles);
    for (int p = 0; p < n_patches; ++p) {
        const fp_patch_shape &s = h_shapes[p];
        const patch_plan &pl = plans[p];
        const int64_t stride = 1 + (int64_t)NPARAMS * s.n_sources;
        std::copy(pl.perm.begin(), pl.perm.end(), h_perm + pp);
        size_t kt = 0;        // next tile of this patch
        int64_t q = pp;
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
                for (; kt < pl.tile_n.size() && pl.tile_expo[kt] == e; ++kt) {
                    const int32_t n = pl.tile_n[kt];
                    fp_tile &t = h_tiles[it];
                    t.partial_offset = poff;
                    t.expo = (int32_t)ie;
                    t.perm_start = (int32_t)q;
                    t.n_pix = n;
                    t.tile_pixels = pl.tile_cls[kt];
                    t.bbox[0] = t.bbox[1] = t.bbox[2] = t.bbox[3] = 0.f;
                    work[(size_t)it] = (int64_t)n * ng;
                    poff += stride;
                    q += n;
                    ++it;
                }
                goff += ng;
                ++ie;
            }
            bd.tile_end = (int32_t)it;
        }
        pp += (int64_t)pl.perm.size();
    }
    // execution order: most work first (stable), so the persistent queue ends on small items
    std::vector<int32_t> ord((size_t)z.n_tiles);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) { return work[a] > work[b]; });
    std::copy(ord.begin(), ord.end(), h_order);
    return FP_OK;
}
