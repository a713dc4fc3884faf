// tiled.cu -- the B200 path: image-Gaussian setup in FP64, one persistent
// launch over (patch, exposure, pixel-tile) work items, fixed-order reduction.
//
// Per evaluation (all on one stream, no host synchronisation):
//   setup_kernel   one CTA per exposure: every image Gaussian of the exposure in
//                  FP64 (fp_gauss.cuh), stored as FP32 pixel-loop parameters with
//                  the ex2 scale folded in, the FP32 centre's rounding residual,
//                  an FP32 bounding box of its E = dx^T F dx <= MAX_EXP_ARG
//                  region, and the FP64 Jacobian.
//   tile_kernel    persistent CTAs pop tiles (largest first).  A tile takes
//                  its pixel coordinates relative to the integer centre of its
//                  box and rebuilds each Gaussian's centre there from the FP32
//                  centre and its rounding residual, so FP32 offsets x - xc
//                  do not lose the precision of large pixel coordinates.
//                  Per tile:
//                  1. cull: keep the Gaussians whose box, and then whose
//                     E <= MAX_EXP_ARG ellipse (FP64), meets the tile's pixel
//                     box; every other Gaussian has E > MAX_EXP_ARG at every
//                     pixel of the tile and contributes exactly nothing;
//                  2. forward, pixel-parallel: P pixels per thread, Gaussians
//                     staged in shared memory; per run of 32 Gaussians one box
//                     test per lane and a warp ballot, the warp visiting only
//                     the hits; y terms once per row of pixels; SFU ex2; FP32
//                     runs flushed into per-pixel FP64 sums; residual, chi2
//                     term in f64, w = r ierr^2;
//                  3. adjoint, Gaussian-parallel: one Gaussian per lane, the
//                     tile's nonzero-weight pixels broadcast from shared memory
//                     (a chunk's last, partial group of v Gaussians is
//                     replicated over the idle lanes, each replica taking every
//                     k-th pixel, and the replicas summed by shuffles);
//                     each lane accumulates 12 moments (FP32 runs -> FP64) from
//                     which the 6 image-space partials follow exactly; the FP64
//                     Jacobian maps them to the 7 on-sky partials once per
//                     (Gaussian, segment), not once per pixel;
//                  4. per-source sums inside each warp (a segmented shuffle
//                     tree), one fixed-order sum over the warps per tile ->
//                     per-tile partials.
//   reduce_kernel  per (patch, band): partials summed over the band's tiles in
//                  canonical order (FP64) -> chi2 (f64) and Response (f32).
// No atomics touch the results, so they are bitwise reproducible.

#include <atomic>

#include "fp_common.cuh"
#include "fp_gauss.cuh"

namespace {

#ifdef FP_PHASE_TIMERS
// Diagnostic build only (libforcepho_b200_phases.so): thread 0 of each CTA
// reads clock64 at the barriers between the tile kernel's phases, and the
// per-tile differences are summed here: [1] cull, [2] forward + residual,
// [3] adjoint, [4] per-tile partials, [5] tiles, [7] all.  The normal build
// has none of this.
__device__ unsigned long long g_phase[8];
#define FP_PHASE_MARK(v) const long long v = clock64()
#else
#define FP_PHASE_MARK(v)
#endif

static_assert(FP_RUN == 32, "the forward pass sums runs of one 32-Gaussian ballot word");

// Compensated FP32 addition (Kahan): s - c tracks the exact running sum to
// about one FP32 rounding, whatever the number of terms.  Used by the FP32 +
// Kahan precision variant (FP_KAHAN); the normal build flushes FP32 runs into
// FP64 instead.
#ifdef FP_KAHAN
__device__ __forceinline__ void kahan_add(float &s, float &c, float x)
{
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}
#endif

// A chunk's last group of v < 32 Gaussians is replicated min(8, 32 / v) times
// across the warp's lanes in the adjoint, each replica taking every k-th pixel;
// 8 replicas read 8 consecutive float4 (128 B) per step.
constexpr int FP_MAX_REPLICAS = 8;


// ---------------------------------------------------------------------------
// setup
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
setup_kernel(const fp_patch *const *__restrict__ patches, const fp_exposure_desc *__restrict__ expos,
             const fp_source *__restrict__ proposals, float4 *__restrict__ gfwd,
             float4 *__restrict__ gbox, float2 *__restrict__ gctr, double *__restrict__ gjac, fp_control *ctl)
{
    const fp_exposure_desc ed = expos[blockIdx.x];
    const fp_patch *pt = patches[ed.patch];
    if (ed.n_sources > MAXSOURCES || pt->n_sources != ed.n_sources) {
        // the patch no longer matches the plan: report it, and make every
        // Gaussian of the exposure inert (zero amplitude and Jacobian, a box
        // that meets no pixel), so that whatever an earlier evaluation left in
        // the tables cannot reach this one's results
        if (threadIdx.x == 0) atomicOr(&ctl->status, FP_STATUS_SOURCES);
        for (int g = threadIdx.x; g < ed.n_gauss; g += blockDim.x) {
            const int64_t i = ed.gauss_offset + g;
            gfwd[2 * i] = make_float4(0.f, 0.f, 0.f, 0.f);
            gfwd[2 * i + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
            gbox[i] = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
            gctr[i] = make_float2(0.f, 0.f);
            double *J = gjac + (size_t)FP_JAC * i;
            for (int k = 0; k < FP_JAC; ++k) J[k] = 0.0;
        }
        return;
    }
    const fp_source *srcs = proposals + (size_t)ed.patch * MAXSOURCES;
    const double c = FP_EXP2_SCALE;
    for (int g = threadIdx.x; g < ed.n_gauss; g += blockDim.x) {
        fp_img_gauss<double> G;
        fp_make_gaussian<double>(pt, srcs, ed.band, ed.exposure, g, ed.n_psf, G);
        const int64_t i = ed.gauss_offset + g;
        const float xc = (float)G.xcen, yc = (float)G.ycen;
        const float fxs = (float)(c * G.fxx), fys = (float)(c * G.fyy), fxys = (float)(c * G.fxy);
        const double k0 = 1.0 - (G.fxx + G.fyy) / 24.0;
        gfwd[2 * i] = make_float4(xc, yc, fxs, fxys);
        gfwd[2 * i + 1] = make_float4(fys, (float)(G.amp * k0), (float)(G.amp * FP_C24), (float)k0);
        // what rounding the centre to FP32 lost (up to 6e-8 of the pixel
        // coordinates): the tiles add it back to the centre relative to their
        // own origin
        const float xlo = (float)(G.xcen - (double)xc), ylo = (float)(G.ycen - (double)yc);
        gctr[i] = make_float2(xlo, ylo);

        // box of {E <= MAX_EXP_ARG} for the FP32 parameters the pixel loops use,
        // widened by 1% in E and 1e-3 px so FP32 rounding of E cannot reach past it
        const double Fxx = (double)fxs / c, Fyy = (double)fys / c, Fxy = (double)fxys / c;
        const double det = Fxx * Fyy - Fxy * Fxy;
        float4 box = make_float4(-INFINITY, INFINITY, -INFINITY, INFINITY);   // never culled
        if (isfinite(xc) && isfinite(yc) && isfinite(det) && det > 0.0 && Fxx > 0.0 && Fyy > 0.0) {
            const double lim = MAX_EXP_ARG * 1.01;
            const double hx = sqrt(lim * Fyy / det) + 1e-3 + fabs((double)xlo);
            const double hy = sqrt(lim * Fxx / det) + 1e-3 + fabs((double)ylo);
            box = make_float4(__double2float_rd((double)xc - hx), __double2float_ru((double)xc + hx),
                              __double2float_rd((double)yc - hy), __double2float_ru((double)yc + hy));
        }
        gbox[i] = box;

        double *J = gjac + (size_t)FP_JAC * i;
        J[0] = G.amp; J[1] = G.fxx; J[2] = G.fxy; J[3] = G.fyy;
        J[4] = G.dA_dflux; J[5] = G.dx_dra; J[6] = G.dy_dra; J[7] = G.dx_ddec; J[8] = G.dy_ddec;
        J[9] = G.dA_dq; J[10] = G.dfxx_dq; J[11] = G.dfyy_dq; J[12] = G.dfxy_dq;
        J[13] = G.dA_dpa; J[14] = G.dfxx_dpa; J[15] = G.dfyy_dpa; J[16] = G.dfxy_dpa;
        J[17] = G.dA_dsersic; J[18] = G.dA_drh; J[19] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// tile bounding boxes (one-time, per plan)
// ---------------------------------------------------------------------------
__global__ void bbox_kernel(const fp_patch *const *__restrict__ patches,
                            const fp_exposure_desc *__restrict__ expos, fp_tile *tiles,
                            const int32_t *__restrict__ perm, int64_t n_tiles)
{
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (t >= n_tiles) return;
    const int lane = threadIdx.x & 31;
    const fp_tile tl = tiles[t];
    const fp_patch *pt = patches[expos[tl.expo].patch];
    float x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
    for (int i = lane; i < tl.n_pix; i += 32) {
        const int32_t ix = perm[tl.perm_start + i];
        const float x = pt->xpix[ix], y = pt->ypix[ix];
        x0 = fminf(x0, x); x1 = fmaxf(x1, x);
        y0 = fminf(y0, y); y1 = fmaxf(y1, y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        x0 = fminf(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        x1 = fmaxf(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        y0 = fminf(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        y1 = fmaxf(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if (lane == 0) {
        tiles[t].bbox[0] = x0; tiles[t].bbox[1] = x1;
        tiles[t].bbox[2] = y0; tiles[t].bbox[3] = y1;
    }
}

// ---------------------------------------------------------------------------
// pixel records in plan order (after a change of the patches' pixel values)
// ---------------------------------------------------------------------------
// One warp per tile: the tile's (x, y, data, ierr) gathered through the plan's
// pixel order into contiguous 16-byte records, which the tile kernel then
// reads with one coalesced vector load per pixel and no index array; the tile
// boxes are recomputed on the way.
__global__ void pack_kernel(const fp_patch *const *__restrict__ patches,
                            const fp_exposure_desc *__restrict__ expos, fp_tile *tiles,
                            const int32_t *__restrict__ perm, float4 *__restrict__ pix, int64_t n_tiles)
{
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (t >= n_tiles) return;
    const int lane = threadIdx.x & 31;
    const fp_tile tl = tiles[t];
    const fp_patch *pt = patches[expos[tl.expo].patch];
    float x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
    for (int i = lane; i < tl.n_pix; i += 32) {
        const int32_t ix = perm[tl.perm_start + i];
        const float x = pt->xpix[ix], y = pt->ypix[ix];
        pix[tl.perm_start + i] = make_float4(x, y, pt->data[ix], pt->ierr[ix]);
        x0 = fminf(x0, x); x1 = fmaxf(x1, x);
        y0 = fminf(y0, y); y1 = fmaxf(y1, y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        x0 = fminf(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        x1 = fmaxf(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        y0 = fminf(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        y1 = fmaxf(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if (lane == 0) {
        tiles[t].bbox[0] = x0; tiles[t].bbox[1] = x1;
        tiles[t].bbox[2] = y0; tiles[t].bbox[3] = y1;
    }
}

// The first pixel-loop parameter float4 of Gaussian gi, (xc, yc, c Fxx, c Fxy),
// with its centre taken relative to a tile origin (ox, oy): the FP32 centre
// minus the origin (exact for a Gaussian near the tile), plus what rounding
// the centre to FP32 lost.  Pixel coordinates are taken relative to the same
// origin, so dx = x - xc carries the rounding of |xc - ox|, not of |xc|: the
// pixel coordinates of a large image (thousands of pixels, ulp 1e-4 px) no
// longer limit the model's precision.
__device__ __forceinline__ float4 stage_gauss(const float4 *__restrict__ gfwd, const float2 *__restrict__ gctr,
                                              int64_t gi, float ox, float oy)
{
    float4 A = gfwd[2 * gi];
    const float2 lo = gctr[gi];
    A.x = (A.x - ox) + lo.x;
    A.y = (A.y - oy) + lo.y;
    return A;
}

// The origin of a tile's relative coordinates: its box centre, rounded to an
// integer so that integer pixel coordinates stay exact; 0 for a box that is
// not finite.
__device__ __forceinline__ float2 tile_origin(const fp_tile &tl)
{
    const float ox = rintf(0.5f * (tl.bbox[0] + tl.bbox[1])), oy = rintf(0.5f * (tl.bbox[2] + tl.bbox[3]));
    return make_float2(isfinite(ox) ? ox : 0.f, isfinite(oy) ? oy : 0.f);
}

// Forward pass of one tile, P pixels per thread (the tile holds at most
// 256 P pixels): the model of each pixel over the tile's kept Gaussians, the
// residual (written out when the patch has a residual array), the chi2 terms
// reduced into s_red[FP_WARPS], and the nonzero-weight pixels (x, y, w) compacted
// into s_pix in ascending order.  Returns their count (the same on every thread).
// Pixel coordinates and Gaussian centres are taken relative to the tile's
// origin (ox, oy) (stage_gauss); the boxes stay absolute.
template <int P>
__device__ __forceinline__ int forward_tile(const fp_tile &tl, const fp_exposure_desc &ed, const fp_patch *pt,
                                            const int32_t *__restrict__ perm, const float4 *__restrict__ pix,
                                            const float4 *__restrict__ gfwd, const float4 *__restrict__ gbox,
                                            const float2 *__restrict__ gctr, const float ox, const float oy,
                                            const bool nocull, const int gc, const uint16_t *s_idx, float4 *s_ga,
                                            float4 *s_gb, float4 *s_gbox, float4 *s_pix, int *s_int, double *s_red)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int npix = tl.n_pix;

    // the tile's pixels are listed in the plan's pixel order (compact cells)
    const int j0 = tid * P;
    const int nval = npix - j0;
    const int32_t *tperm = perm + tl.perm_start + j0;
    int idx[P];
    float xs[P], ys[P], ds[P], es[P];
    if (pix != nullptr) {
        // contiguous (x, y, data, ierr) records in plan order: one 16-byte
        // load per pixel; the patch index only where a residual is written
        const float4 *rec = pix + tl.perm_start + j0;
        const bool want_idx = pt->residual != nullptr;
        const uint64_t pol = fp_policy_evict_first();
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const float4 r = (k < nval) ? fp_ldg_policy(rec + k, pol) : make_float4(0.f, 0.f, 0.f, 0.f);
            xs[k] = r.x; ys[k] = r.y; ds[k] = r.z; es[k] = r.w;
            idx[k] = (k < nval && want_idx) ? __ldg(tperm + k) : -1;
        }
    } else {
#pragma unroll
        for (int k = 0; k < P; ++k) {
            idx[k] = (k < nval) ? __ldg(tperm + k) : -1;
            const bool ok = idx[k] >= 0;
            xs[k] = ok ? __ldg(pt->xpix + idx[k]) : 0.f;
            ys[k] = ok ? __ldg(pt->ypix + idx[k]) : 0.f;
            ds[k] = ok ? __ldg(pt->data + idx[k]) : 0.f;
            es[k] = ok ? __ldg(pt->ierr + idx[k]) : 0.f;
        }
    }
    // this warp's pixel box: Gaussians whose box misses it are skipped by
    // the whole warp (they have E > MAX_EXP_ARG at all of its pixels)
    float wx0 = INFINITY, wx1 = -INFINITY, wy0 = INFINITY, wy1 = -INFINITY;
#pragma unroll
    for (int k = 0; k < P; ++k)
        if (k < nval) {
            wx0 = fminf(wx0, xs[k]); wx1 = fmaxf(wx1, xs[k]);
            wy0 = fminf(wy0, ys[k]); wy1 = fmaxf(wy1, ys[k]);
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        wx0 = fminf(wx0, __shfl_xor_sync(0xffffffffu, wx0, o));
        wx1 = fmaxf(wx1, __shfl_xor_sync(0xffffffffu, wx1, o));
        wy0 = fminf(wy0, __shfl_xor_sync(0xffffffffu, wy0, o));
        wy1 = fmaxf(wy1, __shfl_xor_sync(0xffffffffu, wy1, o));
    }
    if (nocull) { wx0 = wy0 = -INFINITY; wx1 = wy1 = INFINITY; }
#pragma unroll
    for (int k = 0; k < P; ++k) {
        xs[k] -= ox;
        ys[k] -= oy;
    }
    // one row: every thread's pixels share their y (cell rows in row order),
    // so the y-dependent products of a Gaussian are formed once per thread
    bool same_y = true;
#pragma unroll
    for (int k = 1; k < P; ++k) same_y = same_y && (k >= nval || ys[k] == ys[0]);
    const bool rowwise = __all_sync(0xffffffffu, same_y);
#ifdef FP_KAHAN
    float KS[P], KC[P];     // per-pixel compensated FP32 model sums
#pragma unroll
    for (int k = 0; k < P; ++k) KS[k] = KC[k] = 0.f;
#else
    double M[P];
#pragma unroll
    for (int k = 0; k < P; ++k) M[k] = 0.0;
#endif

    for (int c0 = 0; c0 < gc; c0 += FP_CHUNK) {
        const int cn = min(FP_CHUNK, gc - c0);
        __syncthreads();
        for (int i = tid; i < cn; i += FP_THREADS) {
            const int64_t gi = ed.gauss_offset + s_idx[c0 + i];
            s_ga[i] = stage_gauss(gfwd, gctr, gi, ox, oy);
            s_gb[i] = gfwd[2 * gi + 1];
            s_gbox[i] = gbox[gi];
        }
        __syncthreads();
        {
            // runs of 32 Gaussians: lane l tests Gaussian r0 + l against the
            // warp's pixel box, and the warp visits the hits of the run in
            // ascending order; each run is summed in FP32, then added in FP64.
            // Every lane takes part in the ballot, including lanes without
            // pixels (their sums are never used).
            for (int r0 = 0; r0 < cn; r0 += 32) {
                const int il = r0 + lane;
                bool hit = false;
                if (il < cn) {
                    const float4 bx = s_gbox[il];
                    hit = !(bx.y < wx0 || bx.x > wx1 || bx.w < wy0 || bx.z > wy1);
                }
                unsigned word = __ballot_sync(0xffffffffu, hit);
                float m[P];
#pragma unroll
                for (int k = 0; k < P; ++k) m[k] = 0.f;
                if (rowwise) {
                    while (word) {
                        const int i = r0 + __ffs(word) - 1;
                        word &= word - 1u;
                        const float4 A = s_ga[i], B = s_gb[i];
                        const float dy = ys[0] - A.y;
                        const float ty = A.w * dy, uy = B.x * dy;     // c Fxy dy, c Fyy dy
#pragma unroll
                        for (int k = 0; k < P; ++k) {
                            const float dx = xs[k] - A.x;
                            const float vx = fmaf(A.z, dx, ty);
                            const float vy = fmaf(A.w, dx, uy);
                            const float e = fmaf(dy, vy, dx * vx);
                            const float g = fp_ex2(e);
                            const float h = fmaf(B.z, fmaf(vx, vx, vy * vy), B.y);
#ifdef FP_KAHAN
                            kahan_add(KS[k], KC[k], (e < FP_CUT_SCALED) ? 0.f : g * h);
#else
                            m[k] = (e < FP_CUT_SCALED) ? m[k] : fmaf(g, h, m[k]);
#endif
                        }
                    }
                } else {
                    while (word) {
                        const int i = r0 + __ffs(word) - 1;
                        word &= word - 1u;
                        const float4 A = s_ga[i], B = s_gb[i];
#pragma unroll
                        for (int k = 0; k < P; ++k) {
                            const float dx = xs[k] - A.x, dy = ys[k] - A.y;
                            const float vx = fmaf(A.z, dx, A.w * dy);
                            const float vy = fmaf(B.x, dy, A.w * dx);
                            const float e = fmaf(dy, vy, dx * vx);
                            const float g = fp_ex2(e);
                            const float h = fmaf(B.z, fmaf(vx, vx, vy * vy), B.y);
#ifdef FP_KAHAN
                            kahan_add(KS[k], KC[k], (e < FP_CUT_SCALED) ? 0.f : g * h);
#else
                            m[k] = (e < FP_CUT_SCALED) ? m[k] : fmaf(g, h, m[k]);
#endif
                        }
                    }
                }
#ifndef FP_KAHAN
#pragma unroll
                for (int k = 0; k < P; ++k) M[k] += (double)m[k];
#endif
            }
        }
    }

    // residual, chi2 term (f64, the reference's (r^2 - d^2) ierr^2 form), weight
    float rs[P], ws[P];
    double chi = 0.0;
    int nz = 0;
#ifdef FP_KAHAN
    float chi_s = 0.f, chi_c = 0.f;     // this thread's chi2 terms, compensated FP32
#endif
#pragma unroll
    for (int k = 0; k < P; ++k) {
        const bool live = k < nval;
#ifdef FP_KAHAN
        const float r = ds[k] - (KS[k] - KC[k]);
        rs[k] = r;
        const float rif = r * es[k], dif = ds[k] * es[k];
        kahan_add(chi_s, chi_c, live ? (rif - dif) * (rif + dif) : 0.f);
        if (k == P - 1) chi = (double)chi_s - (double)chi_c;
#else
        const double rd = (double)ds[k] - M[k];
        const float r = (float)rd;
        rs[k] = r;
        // chi2 term (r ierr - d ierr)(r ierr + d ierr) from the FP64 residual
        const double rid = rd * (double)es[k], did = (double)ds[k] * (double)es[k];
        chi += live ? (rid - did) * (rid + did) : 0.0;
#endif
        ws[k] = live ? -2.f * ((r * es[k]) * es[k]) : 0.f;
        nz += (ws[k] != 0.f) ? 1 : 0;
    }
    if (pt->residual != nullptr) {
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (idx[k] >= 0) pt->residual[idx[k]] = rs[k];
    }

    // compact nonzero-weight pixels (ascending) into s_pix; reduce chi2 (fixed tree)
    int incl = nz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) chi += __shfl_down_sync(0xffffffffu, chi, o);
    if (lane == 31) s_int[8 + warp] = incl;
    if (lane == 0) s_red[warp] = chi;
    __syncthreads();
    int off = incl - nz, nzt = 0;
#pragma unroll
    for (int w = 0; w < FP_WARPS; ++w) {
        const int cnt = s_int[8 + w];
        off += (w < warp) ? cnt : 0;
        nzt += cnt;
    }
#pragma unroll
    for (int k = 0; k < P; ++k)
        if (ws[k] != 0.f) s_pix[off++] = make_float4(xs[k], ys[k], ws[k], 0.f);
    if (tid == 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < FP_WARPS; ++w) t += s_red[w];
        s_red[FP_WARPS] = t;
    }
    return nzt;
}

// ---------------------------------------------------------------------------
// tile kernel helpers
// ---------------------------------------------------------------------------
// Adjoint moments of one Gaussian (params A, B) over pixels p0, p0 + k, ... < p1
// of the tile's nonzero-weight list (k = 1 unless STRIDED).  With K = w' 2^(cE) (w' = -2 r ierr^2, zero past
// the cutoff), H the pixel-integral factor and v' = c F dx:
//   m0 K, m1 KH, m2 KH vx', m3 KH vy', m4 K vx', m5 K vy', m6 KH dx^2,
//   m7 KH dy^2, m8 KH dx dy, m9 K dx vx', m10 K dy vy', m11 K (dx vy' + dy vx')
#ifdef FP_KAHAN
// The FP32 + Kahan variant of the moments below (diagnostic build
// libforcepho_b200_kahan.so): every moment summed over the whole pixel range
// in FP32 with a compensation term, converted to FP64 once at the end.
template <bool STRIDED>
__device__ __forceinline__ void adjoint_moments(const float4 A, const float4 B,
                                                const float4 *__restrict__ s_pix, int p0, int p1, int k,
                                                double (&m)[12])
{
    const float xc = A.x, yc = A.y, fxs = A.z, fxys = A.w, fys = B.x, k0 = B.w;
    const float c24 = (float)FP_C24;
    const int step = STRIDED ? k : 1;
    float a[12], c[12];
#pragma unroll
    for (int j = 0; j < 12; ++j) a[j] = c[j] = 0.f;
    for (int p = p0; p < p1; p += step) {
        const float4 q = s_pix[p];
        const float dx = q.x - xc, dy = q.y - yc;
        const float vx = fmaf(fxs, dx, fxys * dy);
        const float vy = fmaf(fys, dy, fxys * dx);
        const float pp = dx * vx;
        const float e = fmaf(dy, vy, pp);
        const float g = fp_ex2(e);
        const float K = (e < FP_CUT_SCALED) ? 0.f : q.z * g;
        const float s2 = fmaf(vx, vx, vy * vy);
        const float KH = K * fmaf(s2, c24, k0);
        kahan_add(a[0], c[0], K);
        kahan_add(a[1], c[1], KH);
        kahan_add(a[2], c[2], KH * vx);
        kahan_add(a[3], c[3], KH * vy);
        kahan_add(a[4], c[4], K * vx);
        kahan_add(a[5], c[5], K * vy);
        kahan_add(a[6], c[6], KH * dx * dx);
        kahan_add(a[7], c[7], KH * dy * dy);
        kahan_add(a[8], c[8], KH * dx * dy);
        kahan_add(a[9], c[9], K * pp);
        kahan_add(a[10], c[10], K * (e - pp));
        kahan_add(a[11], c[11], K * fmaf(dx, vy, dy * vx));
    }
#pragma unroll
    for (int j = 0; j < 12; ++j) m[j] += (double)a[j] - (double)c[j];
}
#else
template <bool STRIDED>
__device__ __forceinline__ void adjoint_moments(const float4 A, const float4 B,
                                                const float4 *__restrict__ s_pix, int p0, int p1, int k,
                                                double (&m)[12])
{
    const float xc = A.x, yc = A.y, fxs = A.z, fxys = A.w, fys = B.x, k0 = B.w;
    const float c24 = (float)FP_C24;
    const int step = STRIDED ? k : 1;
    for (int r0 = p0; r0 < p1; r0 += FP_RUN * step) {
        const int r1 = min(p1, r0 + FP_RUN * step);
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, a4 = 0.f, a5 = 0.f;
        float a6 = 0.f, a7 = 0.f, a8 = 0.f, a9 = 0.f, a10 = 0.f, a11 = 0.f;
#pragma unroll 4
        for (int p = r0; p < r1; p += step) {
            const float4 q = s_pix[p];
            const float dx = q.x - xc, dy = q.y - yc;
            const float vx = fmaf(fxs, dx, fxys * dy);
            const float vy = fmaf(fys, dy, fxys * dx);
            const float pp = dx * vx;
            const float e = fmaf(dy, vy, pp);
            const float g = fp_ex2(e);
            const float K = (e < FP_CUT_SCALED) ? 0.f : q.z * g;
            const float s = fmaf(vx, vx, vy * vy);
            const float KH = K * fmaf(s, c24, k0);
            a0 += K;
            a1 += KH;
            a2 = fmaf(KH, vx, a2);
            a3 = fmaf(KH, vy, a3);
            a4 = fmaf(K, vx, a4);
            a5 = fmaf(K, vy, a5);
            const float hx = KH * dx;
            a6 = fmaf(hx, dx, a6);
            a8 = fmaf(hx, dy, a8);
            a7 = fmaf(KH * dy, dy, a7);
            a9 = fmaf(K, pp, a9);
            a10 = fmaf(K, e - pp, a10);
            a11 = fmaf(K, fmaf(dx, vy, dy * vx), a11);
        }
        m[0] += a0; m[1] += a1; m[2] += a2; m[3] += a3; m[4] += a4; m[5] += a5;
        m[6] += a6; m[7] += a7; m[8] += a8; m[9] += a9; m[10] += a10; m[11] += a11;
    }
}
#endif

// Image-space partials from the moments (the reference's dC/d{A,x,y,Fxx,Fyy,Fxy}
// summed over pixels, common_kernel.cc:118-132), then the Jacobian to the 7
// on-sky partials (common_kernel.cc:135-141), all in FP64.
__device__ __forceinline__ void moments_to_grad(const double *__restrict__ J, const double (&m)[12],
                                                double (&g)[NPARAMS])
{
    const double amp = J[0], fxx = J[1], fxy = J[2], fyy = J[3];
    const double ic = 1.0 / FP_EXP2_SCALE;
    const double SA = m[1];
    const double Sx = amp * ic * (m[2] - (fxx * m[4] + fxy * m[5]) * (1.0 / 12.0));
    const double Sy = amp * ic * (m[3] - (fyy * m[5] + fxy * m[4]) * (1.0 / 12.0));
    const double Sfx = amp * (-0.5 * m[6] - m[0] * (1.0 / 24.0) + ic * m[9] * (1.0 / 12.0));
    const double Sfy = amp * (-0.5 * m[7] - m[0] * (1.0 / 24.0) + ic * m[10] * (1.0 / 12.0));
    const double Sfxy = amp * (-m[8] + ic * m[11] * (1.0 / 12.0));
    g[0] = J[4] * SA;
    g[1] = J[5] * Sx + J[6] * Sy;
    g[2] = J[7] * Sx + J[8] * Sy;
    g[3] = J[9] * SA + J[10] * Sfx + J[12] * Sfxy + J[11] * Sfy;
    g[4] = J[13] * SA + J[14] * Sfx + J[16] * Sfxy + J[15] * Sfy;
    g[5] = J[17] * SA;
    g[6] = J[18] * SA;
}

// Whether the region {E = dx^T F dx <= MAX_EXP_ARG (1% margin)} of a Gaussian
// (FP32 pixel-loop parameters A = (xc, yc, c Fxx, c Fxy), fys = c Fyy) meets
// the rectangle [x0,x1] x [y0,y1]: the minimum of the convex quadratic over the
// rectangle is at the centre if it lies inside, else on an edge, where it is a
// clamped 1-D minimum.  FP32: near the threshold the centre lies within the
// Gaussian's cutoff radius of the rectangle, so the offsets x0 - cx, ... are
// exact wherever the coordinates exceed that radius (Sterbenz: within a factor
// 2 of each other); where they do not, the coordinates are small and an offset
// error d moves E by only about 12 d / sigma.  The quadratic form's rounding
// error (~1e-4 of E) is far inside the 1% margin (0.36) as well.  No
// Gaussian with a pixel of the rectangle within the cutoff is dropped; the
// pair census checks exactly that.  Non-finite results keep the Gaussian.
__device__ __forceinline__ bool ellipse_meets_rect(const float4 A, float fys, float x0, float x1, float y0,
                                                   float y1)
{
    const float ic = (float)(1.0 / FP_EXP2_SCALE);
    const float cx = A.x, cy = A.y, fxx = A.z * ic, fxy = A.w * ic, fyy = fys * ic;
    if (cx >= x0 && cx <= x1 && cy >= y0 && cy <= y1) return true;
    const float rxx = __frcp_rn(fxx), ryy = __frcp_rn(fyy);
    float best = INFINITY;
    const float lx = x0 - cx, hx = x1 - cx, ly = y0 - cy, hy = y1 - cy;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float dx = k ? hx : lx;
        const float dy = fminf(fmaxf(-fxy * dx * ryy, ly), hy);
        best = fminf(best, fmaf(fxx * dx, dx, fmaf(2.f * fxy * dx, dy, fyy * dy * dy)));
        const float ey = k ? hy : ly;
        const float ex = fminf(fmaxf(-fxy * ey * rxx, lx), hx);
        best = fminf(best, fmaf(fxx * ex, ex, fmaf(2.f * fxy * ex, ey, fyy * ey * ey)));
    }
    return !(best > (float)(MAX_EXP_ARG * 1.01));
}

struct tile_smem {
    size_t ga, gb, box, pix, wsrc, red, ints, keepw, idx, total;
};

__host__ __device__ inline tile_smem tile_smem_layout(int tile_pixels, int max_gauss)
{
    tile_smem L;
    size_t o = 0;
    L.ga = o;   o += (size_t)FP_CHUNK * 16;
    L.gb = o;   o += (size_t)FP_CHUNK * 16;
    L.box = o;  o += (size_t)FP_CHUNK * 16;
    L.pix = o;  o += (size_t)tile_pixels * 16;
    L.wsrc = o; o += (size_t)FP_WARPS * MAXSOURCES * NPARAMS * 8;
    L.red = o;  o += 16 * 8;
    L.ints = o; o += 32 * 4;
    L.keepw = o; o += (((size_t)max_gauss + 31) / 32 * 4 + 15) & ~(size_t)15;
    L.idx = o;  o += ((size_t)max_gauss * 2 + 15) & ~(size_t)15;
    L.total = o;
    return L;
}

// ---------------------------------------------------------------------------
// tile kernel
// ---------------------------------------------------------------------------
// P: pixels per thread of the plan's largest tile class (shared memory holds
// 256 P pixels); each tile runs the forward pass of its own class.
template <int P>
__global__ void __launch_bounds__(FP_THREADS, 4)
tile_kernel(const fp_patch *const *__restrict__ patches, const fp_exposure_desc *__restrict__ expos,
            const fp_tile *__restrict__ tiles, const int32_t *__restrict__ order,
            const int32_t *__restrict__ perm, const float4 *__restrict__ pix, int64_t n_tiles,
            const float4 *__restrict__ gfwd, const float4 *__restrict__ gbox, const float2 *__restrict__ gctr,
            const double *__restrict__ gjac, double *__restrict__ partials, fp_control *ctl,
            int max_gauss, int flags)
{
    constexpr int T = FP_THREADS * P;
    extern __shared__ __align__(16) unsigned char smem[];
    const tile_smem L = tile_smem_layout(T, max_gauss);
    float4 *s_ga = reinterpret_cast<float4 *>(smem + L.ga);
    float4 *s_gb = reinterpret_cast<float4 *>(smem + L.gb);
    float4 *s_gbox = reinterpret_cast<float4 *>(smem + L.box);
    float4 *s_pix = reinterpret_cast<float4 *>(smem + L.pix);
    // per-warp source gradients [warp][source][param]: each warp adds its own
    // results into its own row, in its own program order
    double *s_wsrc = reinterpret_cast<double *>(smem + L.wsrc);
    double *s_red = reinterpret_cast<double *>(smem + L.red);
    int *s_int = reinterpret_cast<int *>(smem + L.ints);          // [0] item, [8..16) warp counts
    uint16_t *s_idx = reinterpret_cast<uint16_t *>(smem + L.idx);
    unsigned *s_keepw = reinterpret_cast<unsigned *>(smem + L.keepw); // cull ballot words

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool nocull = (flags & FP_FLAG_NO_CULL) != 0;
    const bool forward_only = (flags & FP_FLAG_FORWARD_ONLY) != 0;

    for (int64_t iter = 0;; ++iter) {
        if (tid == 0) {
            const unsigned long long it = (flags & FP_FLAG_STATIC)
                                              ? (unsigned long long)(blockIdx.x + iter * gridDim.x)
                                              : atomicAdd(&ctl->queue, 1ULL);
            s_int[0] = (it < (unsigned long long)n_tiles) ? order[it] : -1;
        }
        __syncthreads();
        const int ti = s_int[0];
        if (ti < 0) break;
        FP_PHASE_MARK(ph0);

        const fp_tile tl = tiles[ti];
        const fp_exposure_desc ed = expos[tl.expo];
        const fp_patch *pt = patches[ed.patch];
        const int ng = ed.n_gauss, ns = ed.n_sources, n_psf = ed.n_psf;
        const float2 org = tile_origin(tl);
        const float ox = org.x, oy = org.y;
        const int npix = tl.n_pix;
        double *out = partials + tl.partial_offset;
        const int tp = tl.tile_pixels;
        const bool bad_tile = npix > tp || tp > T || (tp != 256 && tp != 512 && tp != 1024);
        if (bad_tile || ng > max_gauss || ns > MAXSOURCES) {
            if (tid == 0)
                atomicOr(&ctl->status, bad_tile ? FP_STATUS_TILE_SIZE
                                                : (ng > max_gauss ? FP_STATUS_GAUSS_COUNT : FP_STATUS_SOURCES));
            for (int t = tid; t < 1 + ns * NPARAMS && t < 1 + MAXSOURCES * NPARAMS; t += FP_THREADS)
                out[t] = 0.0;
            __syncthreads();
            continue;
        }

        // ---- 1. cull (ascending-order compaction of surviving Gaussians) ----
        // Each warp tests a contiguous share of the exposure's Gaussians, 32 at
        // a time, and keeps the ballot words; after one barrier every warp
        // writes its kept indices at its offset (the warps' shares ascend).
        const float bx0 = tl.bbox[0], bx1 = tl.bbox[1], by0 = tl.bbox[2], by1 = tl.bbox[3];
        const int nwords = (ng + 31) >> 5;
        const int per_warp = (nwords + FP_WARPS - 1) / FP_WARPS;
        const int wbeg = min(nwords, warp * per_warp), wend = min(nwords, wbeg + per_warp);
        int mine = 0;
        for (int wd = wbeg; wd < wend; ++wd) {
            const int g = wd * 32 + lane;
            bool keep = false;
            if (g < ng) {
                if (nocull) {
                    keep = true;
                } else {
                    const float4 b = gbox[ed.gauss_offset + g];
                    keep = (b.y >= bx0) && (b.x <= bx1) && (b.w >= by0) && (b.z <= by1);
                    if (keep && isfinite(b.x))
                        keep = ellipse_meets_rect(gfwd[2 * (ed.gauss_offset + g)],
                                                  gfwd[2 * (ed.gauss_offset + g) + 1].x, bx0, bx1, by0, by1);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) s_keepw[wd] = m;
            mine += __popc(m);
        }
        if (lane == 0) s_int[8 + warp] = mine;
        __syncthreads();
        int gc = 0, koff = 0;
#pragma unroll
        for (int w = 0; w < FP_WARPS; ++w) {
            const int cnt = s_int[8 + w];
            koff += (w < warp) ? cnt : 0;
            gc += cnt;
        }
        for (int wd = wbeg; wd < wend; ++wd) {
            const unsigned m = s_keepw[wd];
            if (m & (1u << lane)) s_idx[koff + __popc(m & ((1u << lane) - 1u))] = (uint16_t)(wd * 32 + lane);
            koff += __popc(m);
        }
        __syncthreads();

        FP_PHASE_MARK(ph1);
        // ---- 2. forward: the tile's pixel class sets the pixels per thread ----
        int nzt;
        if (tl.tile_pixels == 1024)
            nzt = forward_tile<4>(tl, ed, pt, perm, pix, gfwd, gbox, gctr, ox, oy, nocull, gc, s_idx, s_ga,
                                  s_gb, s_gbox, s_pix, s_int, s_red);
        else if (tl.tile_pixels == 512)
            nzt = forward_tile<2>(tl, ed, pt, perm, pix, gfwd, gbox, gctr, ox, oy, nocull, gc, s_idx, s_ga,
                                  s_gb, s_gbox, s_pix, s_int, s_red);
        else
            nzt = forward_tile<1>(tl, ed, pt, perm, pix, gfwd, gbox, gctr, ox, oy, nocull, gc, s_idx, s_ga,
                                  s_gb, s_gbox, s_pix, s_int, s_red);
        for (int t = tid; t < FP_WARPS * MAXSOURCES * NPARAMS; t += FP_THREADS) s_wsrc[t] = 0.0;

        FP_PHASE_MARK(ph2);
        // ---- 3. adjoint: one Gaussian per lane, pixels broadcast ----
        for (int c0 = 0; c0 < (forward_only ? 0 : gc); c0 += FP_CHUNK) {
            const int cn = min(FP_CHUNK, gc - c0);
            __syncthreads();
            if (gc > FP_CHUNK) {
                for (int i = tid; i < cn; i += FP_THREADS) {
                    const int64_t gi = ed.gauss_offset + s_idx[c0 + i];
                    s_ga[i] = stage_gauss(gfwd, gctr, gi, ox, oy);
                    s_gb[i] = gfwd[2 * gi + 1];
                }
            }
            // the (group of 32 Gaussians) x (pixel) plane, split evenly over the warps
            __syncthreads();
            const int ngrp = (cn + 31) >> 5;
            const int vlast = cn - ((ngrp - 1) << 5);             // Gaussians in the last group
            const int krep = min(FP_MAX_REPLICAS, 32 / vlast);   // its replicas
            const int ulast = (nzt + krep - 1) / krep;            // its units of krep pixels
            // units of the (group, pixel) plane: at most 8 groups x 1024 pixels
            const int ufull = (ngrp - 1) * nzt;
            const int W = ufull + ulast;
            int u = W * warp / FP_WARPS;
            const int u1 = W * (warp + 1) / FP_WARPS;
            while (u < u1) {
                int grp, q0, qn;
                if (u < ufull) {
                    grp = u / nzt;
                    q0 = u - grp * nzt;
                    qn = nzt;
                } else {
                    grp = ngrp - 1;
                    q0 = u - ufull;
                    qn = ulast;
                }
                const int q1 = min(qn, q0 + (u1 - u));
                const int kr = (grp == ngrp - 1) ? krep : 1;      // warp-uniform
                const int vg = (grp == ngrp - 1) ? vlast : 32;
                const int rep = lane / vg;
                const int gl = grp * 32 + lane - rep * vg;
                const bool valid = rep < kr && gl < cn;
                const float4 A = valid ? s_ga[gl] : make_float4(0.f, 0.f, 0.f, 0.f);
                const float4 B = valid ? s_gb[gl] : make_float4(0.f, 0.f, 0.f, 0.f);
                double mom[12];
#pragma unroll
                for (int k = 0; k < 12; ++k) mom[k] = 0.0;
                if (kr == 1) {
                    adjoint_moments<false>(A, B, s_pix, q0, q1, 1, mom);
                } else {
                    // replica rep takes pixels q*kr + rep of units [q0, q1): the
                    // warp reads kr consecutive pixels per step
                    const int pe = min(nzt, q1 * kr);
                    adjoint_moments<true>(A, B, s_pix, valid ? q0 * kr + rep : pe, pe, kr, mom);
                    // sum the replicas into replica 0 (lanes 0 .. vg-1), fixed tree
                    for (int o = 1; o < kr; o <<= 1) {
                        const bool take = (rep & (2 * o - 1)) == 0 && rep + o < kr;
#pragma unroll
                        for (int k = 0; k < 12; ++k) {
                            const double t = __shfl_down_sync(0xffffffffu, mom[k], o * vg);
                            if (take) mom[k] += t;
                        }
                    }
                }
                double g7[NPARAMS];
                int src = -1;
                if (valid && rep == 0) {
                    const int gidx = s_idx[c0 + gl];
                    moments_to_grad(gjac + (size_t)FP_JAC * (ed.gauss_offset + gidx), mom, g7);
                    src = gidx / n_psf;               // Gaussian g belongs to source g / n_psf
                } else {
#pragma unroll
                    for (int k = 0; k < NPARAMS; ++k) g7[k] = 0.0;
                }
                // segmented sum over the lanes of each source: the chunk's Gaussians
                // ascend, so a source's lanes are contiguous; after the fixed
                // shuffle tree the first lane of each source holds its sum
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int so = __shfl_down_sync(0xffffffffu, src, o);
                    const bool same = (lane + o < 32) && (so == src);
#pragma unroll
                    for (int k = 0; k < NPARAMS; ++k) {
                        const double v = __shfl_down_sync(0xffffffffu, g7[k], o);
                        if (same) g7[k] += v;
                    }
                }
                const int sprev = __shfl_up_sync(0xffffffffu, src, 1);
                if (src >= 0 && (lane == 0 || sprev != src)) {
                    double *row = s_wsrc + ((size_t)warp * MAXSOURCES + src) * NPARAMS;
#pragma unroll
                    for (int k = 0; k < NPARAMS; ++k) row[k] += g7[k];
                }
                __syncwarp();   // another lane may update the same row in the next segment
                u += q1 - q0;
            }
        }
        __syncthreads();

        FP_PHASE_MARK(ph3);
        // ---- 4. per-tile partials ----
        if (tid == 0) out[0] = s_red[FP_WARPS];
        for (int t = tid; t < ns * NPARAMS; t += FP_THREADS) {
            double acc = 0.0;
#pragma unroll
            for (int w = 0; w < FP_WARPS; ++w) acc += s_wsrc[(size_t)w * MAXSOURCES * NPARAMS + t];
            out[1 + t] = acc;
        }
        // the next iteration's first barrier orders these reads before any reuse
#ifdef FP_PHASE_TIMERS
        __syncthreads();
        if (tid == 0) {
            const long long ph4 = clock64();
            atomicAdd(&g_phase[1], (unsigned long long)(ph1 - ph0));
            atomicAdd(&g_phase[2], (unsigned long long)(ph2 - ph1));
            atomicAdd(&g_phase[3], (unsigned long long)(ph3 - ph2));
            atomicAdd(&g_phase[4], (unsigned long long)(ph4 - ph3));
            atomicAdd(&g_phase[5], 1ULL);
            atomicAdd(&g_phase[7], (unsigned long long)(ph4 - ph0));
        }
#endif
    }
}

// ---------------------------------------------------------------------------
// reduction over tiles
// ---------------------------------------------------------------------------
constexpr int REDUCE_THREADS = 224;

__global__ void __launch_bounds__(REDUCE_THREADS)
reduce_kernel(const fp_band_desc *__restrict__ bands, const fp_tile *__restrict__ tiles,
              const double *__restrict__ partials, double *__restrict__ chi2_out,
              fp_response *__restrict__ resp_out)
{
    const fp_band_desc bd = bands[blockIdx.x];
    const int ns = bd.n_sources;
    const int stride = 1 + NPARAMS * ns;
    const int64_t base = (bd.tile_end > bd.tile_begin) ? tiles[bd.tile_begin].partial_offset : 0;
    const int64_t out = (int64_t)bd.patch * MAXBANDS + bd.band;
    for (int t = threadIdx.x; t < 1 + MAXSOURCES * NPARAMS; t += REDUCE_THREADS) {
        double acc = 0.0;
        if (t < stride)
            for (int i = 0; i < bd.tile_end - bd.tile_begin; ++i) acc += partials[base + (int64_t)i * stride + t];
        if (t == 0) chi2_out[out] = acc;
        else resp_out[out].dchi2_dparam[t - 1] = (float)acc;
    }
}

// ---------------------------------------------------------------------------
// pair census (diagnostic): how many (pixel, Gaussian) pairs the culled tile
// kernel evaluates, how many lie within the MAX_EXP_ARG cutoff (the pairs that
// change the result), and how many within-cutoff pairs belong to a Gaussian
// the cull dropped (must be zero).  Same FP32 exponent as the pixel loops, in
// the same tile-relative coordinates.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
count_kernel(const fp_patch *const *__restrict__ patches, const fp_exposure_desc *__restrict__ expos,
             const fp_tile *__restrict__ tiles, const int32_t *__restrict__ perm,
             const float4 *__restrict__ gfwd, const float4 *__restrict__ gbox, const float2 *__restrict__ gctr,
             unsigned long long *counts)
{
    extern __shared__ unsigned char s_keep[];   // [n_gauss]: the tile kernel's cull decision
    const fp_tile tl = tiles[blockIdx.x];
    const float2 org = tile_origin(tl);
    const fp_exposure_desc ed = expos[tl.expo];
    const fp_patch *pt = patches[ed.patch];
    const float bx0 = tl.bbox[0], bx1 = tl.bbox[1], by0 = tl.bbox[2], by1 = tl.bbox[3];
    for (int g = threadIdx.x; g < ed.n_gauss; g += blockDim.x) {
        const int64_t gi = ed.gauss_offset + g;
        const float4 b = gbox[gi];
        bool keep = (b.y >= bx0) && (b.x <= bx1) && (b.w >= by0) && (b.z <= by1);
        if (keep && isfinite(b.x)) keep = ellipse_meets_rect(gfwd[2 * gi], gfwd[2 * gi + 1].x, bx0, bx1, by0, by1);
        s_keep[g] = keep ? 1 : 0;
    }
    __syncthreads();
    unsigned long long inbox = 0, active = 0, bad = 0;
    for (int j = threadIdx.x; j < tl.n_pix; j += blockDim.x) {
        const int32_t ix = perm[tl.perm_start + j];
        const float x = pt->xpix[ix] - org.x, y = pt->ypix[ix] - org.y;
        for (int g = 0; g < ed.n_gauss; ++g) {
            const int64_t gi = ed.gauss_offset + g;
            const bool keep = s_keep[g] != 0;
            const float4 A = stage_gauss(gfwd, gctr, gi, org.x, org.y), B = gfwd[2 * gi + 1];
            const float dx = x - A.x, dy = y - A.y;
            const float vx = fmaf(A.z, dx, A.w * dy);
            const float vy = fmaf(B.x, dy, A.w * dx);
            const float e = fmaf(dy, vy, dx * vx);
            const bool act = !(e < FP_CUT_SCALED);
            inbox += keep ? 1 : 0;
            active += act ? 1 : 0;
            bad += (act && !keep) ? 1 : 0;
        }
    }
    __shared__ unsigned long long s[3][8];
    for (int o = 16; o > 0; o >>= 1) {
        inbox += __shfl_down_sync(0xffffffffu, inbox, o);
        active += __shfl_down_sync(0xffffffffu, active, o);
        bad += __shfl_down_sync(0xffffffffu, bad, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { s[0][w] = inbox; s[1][w] = active; s[2][w] = bad; }
    __syncthreads();
    if (threadIdx.x < 3) {
        unsigned long long t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += s[threadIdx.x][i];
        atomicAdd(counts + threadIdx.x, t);
    }
}

// Whether tile_kernel<P> (index 0, 1, 2 for P = 1, 2, 4) has had its dynamic
// shared-memory limit raised on a device.  Devices past the table set it on
// every launch (the call is idempotent).
constexpr int ATTR_MAX_DEVICES = 64;
std::atomic<bool> g_attr_set[ATTR_MAX_DEVICES][3];

template <int P>
int launch_tiles(int grid, size_t smem, cudaStream_t st, const fp_patch *const *d_patches,
                 const fp_plan_tables &tb, int64_t n_tiles, const float4 *gfwd, const float4 *gbox, const float2 *gctr,
                 const double *gjac, double *partials, fp_control *ctl, int max_gauss, int flags)
{
    int dev = 0;
    if (int rc = fp_check_cuda(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    const int pi = P == 1 ? 0 : (P == 2 ? 1 : 2);
    if (dev < 0 || dev >= ATTR_MAX_DEVICES || !g_attr_set[dev][pi].load()) {
        int optin = 0;
        if (int rc = fp_check_cuda(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
                                   "cudaDeviceGetAttribute"))
            return rc;
        if (int rc = fp_check_cuda(cudaFuncSetAttribute(tile_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        optin),
                                   "cudaFuncSetAttribute(tile_kernel)"))
            return rc;
        if (dev >= 0 && dev < ATTR_MAX_DEVICES) g_attr_set[dev][pi].store(true);
    }
    tile_kernel<P><<<grid, FP_THREADS, smem, st>>>(d_patches, tb.expos, tb.tiles, tb.order, tb.perm,
                                                    reinterpret_cast<const float4 *>(tb.pix), n_tiles,
                                                    gfwd, gbox, gctr, gjac, partials, ctl, max_gauss, flags);
    return fp_check_cuda(cudaGetLastError(), "tile_kernel launch");
}

}  // namespace

static int check_tables(const fp_plan_tables *tb, const char *who)
{
    if (!tb || !tb->expos || !tb->tiles || !tb->order || !tb->bands || !tb->perm)
        return fp_set_error(FP_ERR_ARGUMENT, "%s: NULL plan table", who);
    return FP_OK;
}

extern "C" int fp_plan_bbox(const fp_patch *const *d_patches, const fp_plan_sizes *sizes,
                            const fp_plan_tables *tables, void *stream)
{
    if (!d_patches || !sizes || sizes->n_tiles < 0) return fp_set_error(FP_ERR_ARGUMENT, "fp_plan_bbox: bad arguments");
    if (int rc = check_tables(tables, "fp_plan_bbox")) return rc;
    if (sizes->n_tiles == 0) return FP_OK;
    const int per_block = 8;
    const int64_t grid = (sizes->n_tiles + per_block - 1) / per_block;
    bbox_kernel<<<(unsigned)grid, 32 * per_block, 0, (cudaStream_t)stream>>>(d_patches, tables->expos, tables->tiles,
                                                                          tables->perm, sizes->n_tiles);
    return fp_check_cuda(cudaGetLastError(), "bbox_kernel launch");
}

extern "C" int fp_plan_pack(const fp_patch *const *d_patches, const fp_plan_sizes *sizes,
                            const fp_plan_tables *tables, float *d_pix, void *stream)
{
    if (!d_patches || !sizes || sizes->n_tiles < 0 || !d_pix)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_plan_pack: bad arguments");
    if (((uintptr_t)d_pix) & 15) return fp_set_error(FP_ERR_ARGUMENT, "fp_plan_pack: records must be 16-byte aligned");
    if (int rc = check_tables(tables, "fp_plan_pack")) return rc;
    if (sizes->n_tiles == 0) return FP_OK;
    const int per_block = 8;
    const int64_t grid = (sizes->n_tiles + per_block - 1) / per_block;
    pack_kernel<<<(unsigned)grid, 32 * per_block, 0, (cudaStream_t)stream>>>(
        d_patches, tables->expos, tables->tiles, tables->perm, reinterpret_cast<float4 *>(d_pix), sizes->n_tiles);
    return fp_check_cuda(cudaGetLastError(), "pack_kernel launch");
}

extern "C" int fp_tile_smem_bytes(int tile_pixels, int64_t max_gauss, int64_t *out)
{
    if (!out) return fp_set_error(FP_ERR_ARGUMENT, "fp_tile_smem_bytes: NULL");
    *out = (int64_t)tile_smem_layout(tile_pixels, (int)max_gauss).total;
    return FP_OK;
}

extern "C" int fp_count_pairs(const fp_patch *const *d_patches, const fp_plan_sizes *sizes,
                              const fp_plan_tables *tables, const void *d_workspace, size_t workspace_bytes,
                              unsigned long long *d_counts, void *stream)
{
    if (!d_patches || !sizes || !d_workspace || !d_counts)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_count_pairs: NULL argument");
    if (int rc = check_tables(tables, "fp_count_pairs")) return rc;
    const fp_workspace_layout L = fp_layout(sizes->n_gauss, sizes->n_partials);
    if (workspace_bytes < L.total) return fp_set_error(FP_ERR_WORKSPACE, "fp_count_pairs: workspace too small");
    if (sizes->n_tiles <= 0) return FP_OK;
    if (sizes->n_tiles > INT32_MAX) return fp_set_error(FP_ERR_LIMITS, "fp_count_pairs: too many tiles");
    const unsigned char *ws = reinterpret_cast<const unsigned char *>(d_workspace);
    const size_t keep_bytes = (size_t)(sizes->max_gauss > 0 ? sizes->max_gauss : 1);
    if (keep_bytes > 48 * 1024)
        if (int rc = fp_check_cuda(cudaFuncSetAttribute(count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        (int)keep_bytes),
                                   "cudaFuncSetAttribute(count_kernel)"))
            return rc;
    count_kernel<<<(unsigned)sizes->n_tiles, 256, keep_bytes, (cudaStream_t)stream>>>(
        d_patches, tables->expos, tables->tiles, tables->perm, reinterpret_cast<const float4 *>(ws + L.gauss_fwd),
        reinterpret_cast<const float4 *>(ws + L.gauss_box), reinterpret_cast<const float2 *>(ws + L.gauss_ctr),
        d_counts);
    return fp_check_cuda(cudaGetLastError(), "count_kernel launch");
}

namespace {

// What a validated batched evaluation needs to launch.
struct batch_launch {
    fp_workspace_layout L;
    int tile_pixels;
    size_t smem;
    int n_sm;
};

// Argument checks shared by fp_evaluate_batch and fp_evaluate_batch_noalloc:
// everything but the workspace pointer, so that a rejected call has no side
// effects (no launch, no write to any buffer).
int check_batch(const fp_patch *const *d_patches, int n_patches, const fp_plan_sizes *sizes,
                const fp_plan_tables *tables, const fp_source *d_proposals, const double *d_chi2,
                const fp_response *d_response, size_t workspace_bytes, const fp_launch *launch, const char *who,
                batch_launch *out)
{
    if (!d_patches || n_patches < 1 || !sizes || !d_proposals || !d_chi2 || !d_response || !launch)
        return fp_set_error(FP_ERR_ARGUMENT, "%s: NULL argument", who);
    if (int rc = check_tables(tables, who)) return rc;
    if (((uintptr_t)tables->pix) & 15) return fp_set_error(FP_ERR_ARGUMENT, "%s: pixel records must be 16-byte aligned", who);
    const fp_workspace_layout L = fp_layout(sizes->n_gauss, sizes->n_partials);
    if (workspace_bytes < L.total)
        return fp_set_error(FP_ERR_WORKSPACE, "%s: workspace %zu B < required %zu B", who, workspace_bytes,
                            L.total);
    const int T = launch->tile_pixels;
    if (T != 256 && T != 512 && T != 1024)
        return fp_set_error(FP_ERR_ARGUMENT, "%s: tile_pixels=%d (supported: 256, 512, 1024)", who, T);
    if (sizes->max_gauss > 65535)
        return fp_set_error(FP_ERR_LIMITS, "%s: %lld image Gaussians in one exposure (max 65535)", who,
                            (long long)sizes->max_gauss);
    if (sizes->n_exposures > INT32_MAX) return fp_set_error(FP_ERR_LIMITS, "%s: too many exposures", who);
    const size_t smem = tile_smem_layout(T, (int)sizes->max_gauss).total;
    int dev = 0, optin = 0, nsm = 0;
    if (int rc = fp_check_cuda(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (int rc = fp_check_cuda(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
                               "cudaDeviceGetAttribute"))
        return rc;
    if (smem > (size_t)optin)
        return fp_set_error(FP_ERR_LIMITS, "%s: tile needs %zu B shared memory (limit %d B)", who, smem, optin);
    if (int rc = fp_sm_count(&nsm)) return rc;
    out->L = L;
    out->tile_pixels = T;
    out->smem = smem;
    out->n_sm = nsm;
    return FP_OK;
}

// The three launches of an evaluation (arguments already checked).
int run_batch(const batch_launch &a, const fp_patch *const *d_patches, const fp_plan_sizes *sizes,
              const fp_plan_tables &tb, const fp_source *d_proposals, double *d_chi2, fp_response *d_response,
              unsigned char *ws, const fp_launch *launch, cudaStream_t st)
{
    const fp_workspace_layout &L = a.L;
    const int T = a.tile_pixels;
    fp_control *ctl = reinterpret_cast<fp_control *>(ws);
    float4 *gfwd = reinterpret_cast<float4 *>(ws + L.gauss_fwd);
    float4 *gbox = reinterpret_cast<float4 *>(ws + L.gauss_box);
    float2 *gctr = reinterpret_cast<float2 *>(ws + L.gauss_ctr);
    double *gjac = reinterpret_cast<double *>(ws + L.gauss_jac);
    double *partials = reinterpret_cast<double *>(ws + L.partials);

    const int phases = launch->phases ? launch->phases : (FP_PHASE_SETUP | FP_PHASE_TILES | FP_PHASE_REDUCE);
    if ((phases & FP_PHASE_SETUP) && sizes->n_exposures > 0) {
        setup_kernel<<<(unsigned)sizes->n_exposures, 256, 0, st>>>(d_patches, tb.expos, d_proposals, gfwd, gbox,
                                                                   gctr, gjac, ctl);
        if (int rc = fp_check_cuda(cudaGetLastError(), "setup_kernel launch")) return rc;
    }
    if ((phases & FP_PHASE_TILES) && sizes->n_tiles > 0) {
        const int cps = launch->ctas_per_sm > 0 ? launch->ctas_per_sm : 2;
        const int64_t want = (int64_t)cps * a.n_sm;
        const int grid = (int)(want < sizes->n_tiles ? want : sizes->n_tiles);
        // the persistent CTAs pop tiles from this counter
        if (int rc = fp_check_cuda(cudaMemsetAsync(&ctl->queue, 0, sizeof(ctl->queue), st), "queue reset"))
            return rc;
        int rc;
        const int mg = (int)sizes->max_gauss;
        if (T == 256)
            rc = launch_tiles<1>(grid, a.smem, st, d_patches, tb, sizes->n_tiles, gfwd, gbox, gctr, gjac, partials,
                                 ctl, mg, launch->flags);
        else if (T == 512)
            rc = launch_tiles<2>(grid, a.smem, st, d_patches, tb, sizes->n_tiles, gfwd, gbox, gctr, gjac, partials,
                                 ctl, mg, launch->flags);
        else
            rc = launch_tiles<4>(grid, a.smem, st, d_patches, tb, sizes->n_tiles, gfwd, gbox, gctr, gjac, partials,
                                 ctl, mg, launch->flags);
        if (rc) return rc;
    }
    if ((phases & FP_PHASE_REDUCE) && sizes->n_band_outputs > 0) {
        reduce_kernel<<<(unsigned)sizes->n_band_outputs, REDUCE_THREADS, 0, st>>>(tb.bands, tb.tiles, partials,
                                                                                  d_chi2, d_response);
        if (int rc = fp_check_cuda(cudaGetLastError(), "reduce_kernel launch")) return rc;
    }
    return FP_OK;
}

}  // namespace

extern "C" int fp_evaluate_batch(const fp_patch *const *d_patches, int n_patches, const fp_plan_sizes *sizes,
                                 const fp_plan_tables *tables, const fp_source *d_proposals, double *d_chi2,
                                 fp_response *d_response, void *d_workspace, size_t workspace_bytes,
                                 const fp_launch *launch, void *stream)
{
    if (!d_workspace) return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_batch: NULL workspace");
    if (((uintptr_t)d_workspace) & 255)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_evaluate_batch: workspace must be 256-byte aligned");
    batch_launch a;
    if (int rc = check_batch(d_patches, n_patches, sizes, tables, d_proposals, d_chi2, d_response, workspace_bytes,
                             launch, "fp_evaluate_batch", &a))
        return rc;
    return run_batch(a, d_patches, sizes, *tables, d_proposals, d_chi2, d_response,
                     reinterpret_cast<unsigned char *>(d_workspace), launch, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// fp_evaluate_batch_noalloc: the same evaluation with a fixed scratch array
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory: a host-language binding that only
// holds raw device pointers handed to it by another runtime (no CUDA allocator
// on its side), or a process whose device memory is entirely reserved by
// another allocator's pool, where an extra cudaMalloc fails or fragments it.
// For them the workspace is this file-scope device array: every GPU that loads
// the library holds it until the process exits.  All calls share it, and it
// keeps the previous call's contents.
static __device__ __align__(256) unsigned char g_noalloc_ws[FP_NOALLOC_WORKSPACE_BYTES];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::atomic<void *> g_noalloc_addr[NOALLOC_MAX_DEVICES];

// The array's device address on the current device.  Its name in host code is
// only a host-side stand-in, so the address is looked up (cudaGetSymbolAddress,
// with the device current) on the first call on each device and kept.  The
// kept address belongs to the device's primary context at that time:
// cudaDeviceReset destroys that context, and a process that resets a device
// must not call these entry points on it afterwards.
int noalloc_address(const char *who, void **out)
{
    int dev = 0;
    if (int rc = fp_check_cuda(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return fp_set_error(FP_ERR_ARGUMENT, "%s: device %d beyond %d", who, dev, NOALLOC_MAX_DEVICES);
    void *ws = g_noalloc_addr[dev].load();
    if (ws == nullptr) {
        if (int rc = fp_check_cuda(cudaGetSymbolAddress(&ws, g_noalloc_ws), "cudaGetSymbolAddress(noalloc workspace)"))
            return rc;
        g_noalloc_addr[dev].store(ws);
    }
    *out = ws;
    return FP_OK;
}
}  // namespace

extern "C" int fp_evaluate_batch_noalloc(const fp_patch *const *d_patches, int n_patches,
                                         const fp_plan_sizes *sizes, const fp_plan_tables *tables,
                                         const fp_source *d_proposals, double *d_chi2, fp_response *d_response,
                                         const fp_launch *launch, void *stream)
{
    const char *who = "fp_evaluate_batch_noalloc";
    if (!sizes) return fp_set_error(FP_ERR_ARGUMENT, "%s: NULL sizes", who);
    if (sizes->workspace_bytes < 0 || (uint64_t)sizes->workspace_bytes > (uint64_t)FP_NOALLOC_WORKSPACE_BYTES)
        return fp_set_error(FP_ERR_WORKSPACE,
                            "%s: the plan needs %lld B of workspace, more than the fixed %llu B array; use "
                            "fp_evaluate_batch with a caller-allocated workspace",
                            who, (long long)sizes->workspace_bytes, (unsigned long long)FP_NOALLOC_WORKSPACE_BYTES);
    // every check first: a rejected call touches neither the array nor the stream
    batch_launch a;
    if (int rc = check_batch(d_patches, n_patches, sizes, tables, d_proposals, d_chi2, d_response,
                             (size_t)FP_NOALLOC_WORKSPACE_BYTES, launch, who, &a))
        return rc;
    void *ws = nullptr;
    if (int rc = noalloc_address(who, &ws)) return rc;
    // the control block (work-queue counter, status word) must start at zero;
    // the status word then describes this call alone (fp_read_status_noalloc)
    if (int rc = fp_check_cuda(cudaMemsetAsync(ws, 0, sizeof(fp_control), (cudaStream_t)stream),
                               "fp_evaluate_batch_noalloc: clear control block"))
        return rc;
    return run_batch(a, d_patches, sizes, *tables, d_proposals, d_chi2, d_response,
                     reinterpret_cast<unsigned char *>(ws), launch, (cudaStream_t)stream);
}

extern "C" int fp_read_status_noalloc(int32_t *status_out, void *stream)
{
    if (!status_out) return fp_set_error(FP_ERR_ARGUMENT, "fp_read_status_noalloc: NULL");
    void *ws = nullptr;
    if (int rc = noalloc_address("fp_read_status_noalloc", &ws)) return rc;
    return fp_read_status(ws, status_out, stream);
}

#ifdef FP_PHASE_TIMERS
// Diagnostic build only: copy the summed phase clocks out (and zero them).
extern "C" FP_API int fp_debug_phases(unsigned long long out[8], int reset)
{
    if (!out) return fp_set_error(FP_ERR_ARGUMENT, "fp_debug_phases: NULL");
    if (int rc = fp_check_cuda(cudaDeviceSynchronize(), "fp_debug_phases sync")) return rc;
    if (int rc = fp_check_cuda(cudaMemcpyFromSymbol(out, g_phase, sizeof(unsigned long long) * 8),
                               "fp_debug_phases copy"))
        return rc;
    if (reset) {
        const unsigned long long z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (int rc = fp_check_cuda(cudaMemcpyToSymbol(g_phase, z, sizeof(z)), "fp_debug_phases reset")) return rc;
    }
    return FP_OK;
}
#endif
