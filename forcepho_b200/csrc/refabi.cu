// refabi.cu -- the reference's kernel ABI on the tiled B200 kernels.
//
// fp_evaluate_proposal takes exactly what the reference's pycuda launch of
// EvaluateProposal takes (forcepho/src/compute_gaussians_kernel.cu:212-214,
// launched by GPUProposer.evaluate_proposal, forcepho/proposal.py:96-152): a
// device Patch struct, device Source records, and the chi2 / Response outputs.
// The tiled kernels need a work plan of the patch (pixel tiles, exposure and
// band tables, a workspace), which depends only on the patch's pixel layout.
// This file keeps one plan per device patch struct in a library-owned cache:
//
//   * every call reads the 152-byte struct and the small index arrays
//     (band_start/N, n_psf_per_source, exposure_start/N) back to the host (two
//     waits on the stream) and compares them, and the xpix/ypix pointers, with
//     the cached plan's; any difference makes a new plan from the device
//     coordinates (one more read-back);
//   * the tile bounding boxes are recomputed on the device at every call, so a
//     plan stays exact even when the coordinates are rewritten in place at the
//     same addresses (the pixel order then only loses compactness);
//   * the plan's tables and workspace are device memory owned by the library,
//     released by fp_evaluate_proposal_release() or at process exit.
//
// Calls on one patch must not overlap on the GPU (they share its workspace),
// which the reference's synchronous pycuda call never does either.

#include <algorithm>
#include <mutex>
#include <vector>

#include "fp_common.cuh"

namespace {

struct ref_plan {
    int device = -1;
    const fp_patch *d_patch = nullptr;
    fp_patch key;                         // the struct the plan was made for (data/residual ignored)
    std::vector<int16_t> band_start, band_N;
    std::vector<int32_t> n_psf, exposure_start, exposure_N;
    fp_plan_sizes sizes;
    fp_plan_tables tables;
    fp_launch launch;
    void *d_mem = nullptr;                // tables, the patch-pointer array and the workspace
    void *d_workspace = nullptr;
    size_t workspace_bytes = 0;
    const fp_patch **d_patches = nullptr;
    unsigned long long last_use = 0;
};

std::mutex g_mu;
std::vector<ref_plan> g_plans;
unsigned long long g_clock = 0;
constexpr size_t MAX_PLANS = 64;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

bool same_layout(const fp_patch &a, const fp_patch &b)
{
    return a.xpix == b.xpix && a.ypix == b.ypix && a.exposure_start == b.exposure_start &&
           a.exposure_N == b.exposure_N && a.band_start == b.band_start && a.band_N == b.band_N &&
           a.n_sources == b.n_sources && a.n_psf_per_source == b.n_psf_per_source;
}

void free_plan(ref_plan &p)
{
    if (p.d_mem) {
        int cur = 0;
        cudaGetDevice(&cur);
        if (cur != p.device) cudaSetDevice(p.device);
        cudaDeviceSynchronize();     // kernels queued on any stream may still read the plan
        cudaFree(p.d_mem);
        if (cur != p.device) cudaSetDevice(cur);
    }
    p.d_mem = nullptr;
}

// The largest tile that still gives every SM at least 4 tiles (256 below that).
int default_tile_pixels(int64_t n_pix, int n_sm)
{
    for (int tp : {1024, 512})
        if (n_pix / tp >= 4 * (int64_t)n_sm) return tp;
    return 256;
}

template <typename T>
int read_back(std::vector<T> &dst, const T *src, size_t n, cudaStream_t st, const char *what)
{
    dst.assign(n, T());
    if (n == 0) return FP_OK;
    if (!src) return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal: patch without %s", what);
    return fp_check_cuda(cudaMemcpyAsync(dst.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, st), what);
}

int make_plan(ref_plan &pl, const fp_patch &hp, int n_bands, cudaStream_t st)
{
    // pixel count from the exposure layout, coordinates for compact tiles
    int64_t n_pix = 0;
    for (size_t e = 0; e < pl.exposure_start.size(); ++e)
        n_pix = std::max<int64_t>(n_pix, (int64_t)pl.exposure_start[e] + pl.exposure_N[e]);
    if (n_pix > INT32_MAX) return fp_set_error(FP_ERR_LIMITS, "fp_evaluate_proposal: too many pixels");
    std::vector<float> xp, yp;
    if (int rc = read_back(xp, hp.xpix, (size_t)n_pix, st, "xpix")) return rc;
    if (int rc = read_back(yp, hp.ypix, (size_t)n_pix, st, "ypix")) return rc;
    if (int rc = fp_check_cuda(cudaStreamSynchronize(st), "fp_evaluate_proposal: read coordinates")) return rc;

    fp_patch_shape sh;
    sh.n_bands = n_bands;
    sh.n_exposures = (int32_t)pl.exposure_start.size();
    sh.n_sources = hp.n_sources;
    sh.n_pix = (int32_t)n_pix;
    sh.exposure_start = pl.exposure_start.data();
    sh.exposure_N = pl.exposure_N.data();
    sh.band_start = pl.band_start.data();
    sh.band_N = pl.band_N.data();
    sh.n_psf_per_source = pl.n_psf.data();
    sh.xpix = n_pix ? xp.data() : nullptr;
    sh.ypix = n_pix ? yp.data() : nullptr;
    int n_sm = 0;
    if (int rc = fp_sm_count(&n_sm)) return rc;
    const int tp = default_tile_pixels(n_pix, n_sm);
    fp_plan_sizes z;
    if (int rc = fp_plan_count(&sh, 1, tp, &z)) return rc;
    std::vector<fp_exposure_desc> expos((size_t)z.n_exposures);
    std::vector<fp_tile> tiles((size_t)z.n_tiles);
    std::vector<fp_band_desc> bands((size_t)z.n_band_outputs);
    std::vector<int32_t> order((size_t)z.n_tiles), perm((size_t)z.n_perm);
    if (int rc = fp_plan_fill(&sh, 1, tp, expos.data(), tiles.data(), bands.data(), order.data(), perm.data()))
        return rc;

    // one device allocation: [patch pointer | expos | tiles | bands | order | perm | workspace]
    size_t off = 0;
    const size_t o_ptr = off; off = align256(off + sizeof(void *));
    const size_t o_expos = off; off = align256(off + expos.size() * sizeof(fp_exposure_desc));
    const size_t o_tiles = off; off = align256(off + tiles.size() * sizeof(fp_tile));
    const size_t o_bands = off; off = align256(off + bands.size() * sizeof(fp_band_desc));
    const size_t o_order = off; off = align256(off + order.size() * sizeof(int32_t));
    const size_t o_perm = off; off = align256(off + perm.size() * sizeof(int32_t));
    const size_t o_ws = off; off = align256(off + (size_t)std::max<int64_t>(z.workspace_bytes, 256));
    void *mem = nullptr;
    if (int rc = fp_check_cuda(cudaMalloc(&mem, off), "fp_evaluate_proposal: plan memory")) return rc;
    unsigned char *base = static_cast<unsigned char *>(mem);
    const fp_patch *pptr = pl.d_patch;
    int rc = FP_OK;
    auto put = [&](size_t o, const void *src, size_t n) {
        if (rc == FP_OK && n)
            rc = fp_check_cuda(cudaMemcpyAsync(base + o, src, n, cudaMemcpyHostToDevice, st), "plan upload");
    };
    put(o_ptr, &pptr, sizeof(void *));
    put(o_expos, expos.data(), expos.size() * sizeof(fp_exposure_desc));
    put(o_tiles, tiles.data(), tiles.size() * sizeof(fp_tile));
    put(o_bands, bands.data(), bands.size() * sizeof(fp_band_desc));
    put(o_order, order.data(), order.size() * sizeof(int32_t));
    put(o_perm, perm.data(), perm.size() * sizeof(int32_t));
    if (rc == FP_OK) rc = fp_check_cuda(cudaMemsetAsync(base + o_ws, 0, sizeof(fp_control), st), "plan workspace");
    if (rc == FP_OK) rc = fp_check_cuda(cudaStreamSynchronize(st), "plan upload");   // host tables go out of scope
    if (rc) {
        cudaFree(mem);
        return rc;
    }
    pl.d_mem = mem;
    pl.sizes = z;
    pl.d_patches = reinterpret_cast<const fp_patch **>(base + o_ptr);
    pl.tables.expos = reinterpret_cast<const fp_exposure_desc *>(base + o_expos);
    pl.tables.tiles = reinterpret_cast<fp_tile *>(base + o_tiles);
    pl.tables.order = reinterpret_cast<const int32_t *>(base + o_order);
    pl.tables.bands = reinterpret_cast<const fp_band_desc *>(base + o_bands);
    pl.tables.perm = reinterpret_cast<const int32_t *>(base + o_perm);
    pl.tables.pix = nullptr;     // the caller's data may change between calls: gather through perm
    pl.d_workspace = base + o_ws;
    pl.workspace_bytes = off - o_ws;
    pl.launch.tile_pixels = tp;
    pl.launch.ctas_per_sm = 4;
    pl.launch.flags = 0;
    pl.launch.phases = 0;
    pl.key = hp;
    return FP_OK;
}

}  // namespace

extern "C" int fp_evaluate_proposal(const fp_patch *d_patch, const fp_source *d_sources, int n_sources,
                                    int n_bands, double *d_chi2, fp_response *d_response, void *stream)
{
    if (!d_patch || !d_sources || !d_chi2 || !d_response)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal: NULL pointer");
    if (n_bands < 1 || n_bands > MAXBANDS)
        return fp_set_error(FP_ERR_LIMITS, "fp_evaluate_proposal: n_bands=%d outside [1,%d]", n_bands, MAXBANDS);
    if (n_sources < 0 || n_sources > MAXSOURCES)
        return fp_set_error(FP_ERR_LIMITS, "fp_evaluate_proposal: n_sources=%d outside [0,%d]", n_sources,
                            MAXSOURCES);
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (int rc = fp_check_cuda(cudaGetDevice(&dev), "cudaGetDevice")) return rc;

    // 1. the struct
    fp_patch hp;
    if (int rc = fp_check_cuda(cudaMemcpyAsync(&hp, d_patch, sizeof(fp_patch), cudaMemcpyDeviceToHost, st),
                               "fp_evaluate_proposal: read patch struct"))
        return rc;
    if (int rc = fp_check_cuda(cudaStreamSynchronize(st), "fp_evaluate_proposal: stream")) return rc;
    if (hp.n_sources != n_sources)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal: n_sources=%d but the patch has %d", n_sources,
                            hp.n_sources);

    std::lock_guard<std::mutex> lock(g_mu);
    ref_plan *hit = nullptr;
    for (ref_plan &p : g_plans)
        if (p.device == dev && p.d_patch == d_patch) hit = &p;

    // 2. the index arrays (the exposure arrays sized from band_N, known from
    // the cached plan when the layout has not changed)
    ref_plan cur;
    cur.device = dev;
    cur.d_patch = d_patch;
    if (int rc = read_back(cur.band_start, hp.band_start, (size_t)n_bands, st, "band_start")) return rc;
    if (int rc = read_back(cur.band_N, hp.band_N, (size_t)n_bands, st, "band_N")) return rc;
    if (int rc = read_back(cur.n_psf, hp.n_psf_per_source, (size_t)n_bands, st, "n_psf_per_source")) return rc;
    size_t n_exp_guess = (hit && same_layout(hit->key, hp)) ? hit->exposure_start.size() : 0;
    if (n_exp_guess) {
        if (int rc = read_back(cur.exposure_start, hp.exposure_start, n_exp_guess, st, "exposure_start")) return rc;
        if (int rc = read_back(cur.exposure_N, hp.exposure_N, n_exp_guess, st, "exposure_N")) return rc;
    }
    if (int rc = fp_check_cuda(cudaStreamSynchronize(st), "fp_evaluate_proposal: read index arrays")) return rc;
    int64_t n_exp = 0;
    for (int b = 0; b < n_bands; ++b) {
        if (cur.band_N[b] < 0 || cur.band_start[b] != n_exp)
            return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_proposal: band_start/band_N do not tile the exposures");
        n_exp += cur.band_N[b];
    }
    if ((size_t)n_exp != n_exp_guess) {
        if (int rc = read_back(cur.exposure_start, hp.exposure_start, (size_t)n_exp, st, "exposure_start")) return rc;
        if (int rc = read_back(cur.exposure_N, hp.exposure_N, (size_t)n_exp, st, "exposure_N")) return rc;
        if (int rc = fp_check_cuda(cudaStreamSynchronize(st), "fp_evaluate_proposal: read exposures")) return rc;
    }

    // 3. the cached plan, or a new one
    const bool same = hit && same_layout(hit->key, hp) && hit->band_start == cur.band_start &&
                      hit->band_N == cur.band_N && hit->n_psf == cur.n_psf &&
                      hit->exposure_start == cur.exposure_start && hit->exposure_N == cur.exposure_N;
    if (!same) {
        if (int rc = make_plan(cur, hp, n_bands, st)) return rc;
        if (hit) {
            free_plan(*hit);
            *hit = cur;
        } else {
            if (g_plans.size() >= MAX_PLANS) {   // the least recently used plan makes room
                auto lru = std::min_element(g_plans.begin(), g_plans.end(),
                                            [](const ref_plan &a, const ref_plan &b) { return a.last_use < b.last_use; });
                free_plan(*lru);
                g_plans.erase(lru);
            }
            g_plans.push_back(cur);
            hit = &g_plans.back();
        }
    }
    hit->last_use = ++g_clock;

    // 4. boxes (always: the coordinates may have been rewritten in place), then
    // the evaluation into the caller's chi2[n_bands] and Response[n_bands]
    // (one patch, so the batched output rows are the caller's arrays)
    if (int rc = fp_plan_bbox(hit->d_patches, &hit->sizes, &hit->tables, stream)) return rc;
    if (hit->sizes.n_tiles == 0 && hit->sizes.n_band_outputs == 0) return FP_OK;
    return fp_evaluate_batch(hit->d_patches, 1, &hit->sizes, &hit->tables, d_sources, d_chi2, d_response,
                             hit->d_workspace, hit->workspace_bytes, &hit->launch, stream);
}

extern "C" int fp_evaluate_proposal_release(void)
{
    std::lock_guard<std::mutex> lock(g_mu);
    for (ref_plan &p : g_plans) free_plan(p);
    g_plans.clear();
    return FP_OK;
}
