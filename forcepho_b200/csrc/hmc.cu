// hmc.cu -- device-resident pieces around the likelihood for HMC sampling of
// many patches at once: the scene-parameter transform, proposal construction
// with on-device spline amplitudes, lnp and its gradient, and the leapfrog /
// Metropolis updates.  Every launch is asynchronous on the caller's stream and
// reads its scalars from device memory, so a whole trajectory (16 leapfrog
// steps = ~100 launches) is captured once into a CUDA graph and replayed.
//
// Host-side counterparts in the reference: Galaxy.proposal with scipy
// RectBivariateSpline amplitudes (forcepho/sources.py:607-681),
// FastPosterior.evaluate / stack_grad (forcepho/model.py:302-387),
// BoundedTransform (forcepho/model.py:596-637); the sampler itself is
// littlemcmc's NUTS driven by fitting.run_lmc (forcepho/fitting.py:254-341),
// replaced here by fixed-length HMC with a diagonal mass matrix.

#include <math.h>

#include "fp_common.cuh"

namespace {

constexpr int HMC_THREADS = 128;
constexpr int MAXDEG = 5;

// Nonzero B-spline basis functions of degree k at x, and their derivatives,
// on the knot vector t of n coefficients (len(t) = n + k + 1).  x is clamped to
// [t[k], t[n]] first, as FITPACK's bispev/parder do (so does scipy).
// Cox-de Boor recurrence (de Boor, "A Practical Guide to Splines", ch. X);
// returns the index of the first nonzero basis function.
__device__ int bspline_basis(const double *__restrict__ t, int n, int k, double x, double *N, double *dN)
{
    const double lo = t[k], hi = t[n];
    x = fmin(fmax(x, lo), hi);
    // span l: t[l] <= x < t[l+1], k <= l <= n-1 (x == hi falls in the last span)
    int a = k, b = n - 1;
    while (a < b) {
        const int m = (a + b + 1) >> 1;
        if (t[m] <= x) a = m; else b = m - 1;
    }
    const int l = a;
    double left[MAXDEG + 1], right[MAXDEG + 1], lower[MAXDEG + 1];
    N[0] = 1.0;
    for (int j = 1; j <= k; ++j) {
        left[j] = x - t[l + 1 - j];
        right[j] = t[l + j] - x;
        double saved = 0.0;
        for (int r = 0; r < j; ++r) {
            const double tmp = N[r] / (right[r + 1] + left[j - r]);
            N[r] = saved + right[r + 1] * tmp;
            saved = left[j - r] * tmp;
        }
        N[j] = saved;
        if (j == k - 1)
            for (int r = 0; r <= j; ++r) lower[r] = N[r];
    }
    // d/dx N_{i,k} = k (N_{i,k-1} / (t_{i+k} - t_i) - N_{i+1,k-1} / (t_{i+k+1} - t_{i+1}))
    // with N_{i,k-1} for i = l-k+1 .. l held in lower[0..k-1]
    for (int r = 0; r <= k; ++r) {
        const int i = l - k + r;
        double d = 0.0;
        if (r >= 1) {
            const double den = t[i + k] - t[i];
            if (den > 0.0) d += lower[r - 1] / den;
        }
        if (r <= k - 1) {
            const double den = t[i + k + 1] - t[i + 1];
            if (den > 0.0) d -= lower[r] / den;
        }
        dN[r] = k * d;
    }
    return l - k;
}

__device__ __forceinline__ double sigm(double z) { return 1.0 / (1.0 + exp(-z)); }

// --------------------------------------------------------------------------
// transform + proposal: one thread per (patch, source)
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(HMC_THREADS)
prepare_kernel(const fp_hmc_patch *__restrict__ hp, int n_patches, const double *__restrict__ z,
               const double *__restrict__ lower, const double *__restrict__ upper, fp_spline_table tab,
               fp_source *__restrict__ props, double *__restrict__ theta, double *__restrict__ jac)
{
    const int p = blockIdx.x;
    const fp_hmc_patch P = hp[p];
    const int nper = P.n_bands + NPARAMS - 1;
    for (int s = threadIdx.x; s < MAXSOURCES; s += blockDim.x) {
        fp_source *src = props + (size_t)p * MAXSOURCES + s;
        if (s >= P.n_sources) continue;
        double th[MAXBANDS + NPARAMS - 1];
        for (int k = 0; k < nper; ++k) {
            const int64_t j = P.param_offset + (int64_t)s * nper + k;
            const double zz = z[j];
            double q = zz, J = 1.0;
            if (lower != nullptr) {
                const double rng = upper[j] - lower[j];
                const double sg = sigm(zz);
                q = lower[j] + rng * sg;
                J = rng * sg * (1.0 - sg);
            }
            th[k] = q;
            theta[j] = q;
            jac[j] = J;
        }
        const int nb = P.n_bands;
        for (int b = 0; b < MAXBANDS; ++b) src->fluxes[b] = (b < nb) ? (float)th[b] : 0.f;
        src->ra = (float)th[nb];
        src->dec = (float)th[nb + 1];
        src->q = (float)th[nb + 2];
        src->pa = (float)th[nb + 3];
        src->nsersic = (float)th[nb + 4];
        src->rh = (float)th[nb + 5];
        // A_r(sersic, rhalf) and its partial derivatives from the tensor-product spline
        double Nx[MAXDEG + 1], dNx[MAXDEG + 1], Ny[MAXDEG + 1], dNy[MAXDEG + 1];
        const int ncx = tab.nx - tab.kx - 1, ncy = tab.ny - tab.ky - 1;
        const int ix = bspline_basis(tab.tx, ncx, tab.kx, th[nb + 4], Nx, dNx);
        const int iy = bspline_basis(tab.ty, ncy, tab.ky, th[nb + 5], Ny, dNy);
        for (int r = 0; r < MAXRADII; ++r) {
            double a = 0.0, an = 0.0, ar = 0.0;
            if (r < tab.n_radii) {
                const double *c = tab.coef + (size_t)r * ncx * ncy;
                for (int u = 0; u <= tab.kx; ++u) {
                    const double *row = c + (size_t)(ix + u) * ncy + iy;
                    double sv = 0.0, sd = 0.0;
                    for (int v = 0; v <= tab.ky; ++v) {
                        sv += row[v] * Ny[v];
                        sd += row[v] * dNy[v];
                    }
                    a += Nx[u] * sv;
                    an += dNx[u] * sv;
                    ar += Nx[u] * sd;
                }
            }
            src->mixture_amplitudes[r] = (float)a;
            src->damplitude_dnsersic[r] = (float)an;
            src->damplitude_drh[r] = (float)ar;
        }
    }
}

// --------------------------------------------------------------------------
// lnp and dlnp/dz: one CTA per patch
// --------------------------------------------------------------------------
__device__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
    return t;   // valid in thread 0
}

__global__ void __launch_bounds__(HMC_THREADS)
lnprob_kernel(const fp_hmc_patch *__restrict__ hp, const double *__restrict__ z, const double *__restrict__ jac,
              const double *__restrict__ chi2, const fp_response *__restrict__ resp, int transformed, int sampling,
              double *__restrict__ lnp, double *__restrict__ grad)
{
    __shared__ double sh[HMC_THREADS / 32];
    const int p = blockIdx.x;
    const fp_hmc_patch P = hp[p];
    const int nb = P.n_bands, nper = nb + NPARAMS - 1;
    const int n = P.n_sources * nper;
    const fp_response *R = resp + (size_t)p * MAXBANDS;
    double logj = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int s = j / nper, k = j - s * nper;
        double g;
        if (k < nb) {
            g = (double)R[k].dchi2_dparam[s * NPARAMS];
        } else {
            g = 0.0;
            for (int b = 0; b < nb; ++b) g += (double)R[b].dchi2_dparam[s * NPARAMS + 1 + (k - nb)];
        }
        const int64_t jj = P.param_offset + j;
        double gz = -0.5 * g * jac[jj];
        if (transformed && sampling) {
            gz += 1.0 - 2.0 * sigm(z[jj]);
            logj += log(fabs(jac[jj]));
        }
        grad[jj] = gz;
    }
    const double lj = block_sum(logj, sh);
    if (threadIdx.x == 0) {
        double c = 0.0;
        for (int b = 0; b < nb; ++b) c += chi2[(size_t)p * MAXBANDS + b];
        lnp[p] = -0.5 * c + lj;
    }
}

// --------------------------------------------------------------------------
// leapfrog and Metropolis: one CTA per patch; scalars from device memory
// --------------------------------------------------------------------------
// start of a trajectory: momentum from the pre-drawn normals, save (z, grad, lnp),
// H0 = -lnp + p^T M^-1 p / 2, then the first half kick and drift
__global__ void __launch_bounds__(HMC_THREADS)
begin_kernel(const fp_hmc_patch *__restrict__ hp, const fp_hmc_state st)
{
    __shared__ double sh[HMC_THREADS / 32];
    const int p = blockIdx.x;
    const fp_hmc_patch P = hp[p];
    const int n = P.n_sources * (P.n_bands + NPARAMS - 1);
    const int64_t traj = *st.traj % st.n_traj;
    const double eps = st.eps[p];
    double kin = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t jj = P.param_offset + j;
        const double im = st.inv_mass[jj];
        const double mom = st.normals[traj * st.n_params + jj] / sqrt(im);
        kin += mom * mom * im;
        st.z0[jj] = st.z[jj];
        st.grad0[jj] = st.grad[jj];
        const double ph = mom + 0.5 * eps * st.grad[jj];
        st.p[jj] = ph;
        st.z[jj] += eps * im * ph;
    }
    const double k = block_sum(kin, sh);
    if (threadIdx.x == 0) {
        st.lnp0[p] = st.lnp[p];
        st.h0[p] = -st.lnp[p] + 0.5 * k;
    }
}

// between two gradient evaluations: full kick then drift
__global__ void __launch_bounds__(HMC_THREADS)
step_kernel(const fp_hmc_patch *__restrict__ hp, const fp_hmc_state st)
{
    const int p = blockIdx.x;
    const fp_hmc_patch P = hp[p];
    const int n = P.n_sources * (P.n_bands + NPARAMS - 1);
    const double eps = st.eps[p];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t jj = P.param_offset + j;
        const double ph = st.p[jj] + eps * st.grad[jj];
        st.p[jj] = ph;
        st.z[jj] += eps * st.inv_mass[jj] * ph;
    }
}

// end of a trajectory: last half kick, H1, accept with prob min(1, exp(H0 - H1))
// using the pre-drawn uniform, otherwise restore (z, grad, lnp)
__global__ void __launch_bounds__(HMC_THREADS)
end_kernel(const fp_hmc_patch *__restrict__ hp, int n_patches, const fp_hmc_state st)
{
    __shared__ double sh[HMC_THREADS / 32];
    __shared__ int s_acc;
    const int p = blockIdx.x;
    const fp_hmc_patch P = hp[p];
    const int n = P.n_sources * (P.n_bands + NPARAMS - 1);
    const int64_t traj = *st.traj % st.n_traj;
    const double eps = st.eps[p];
    double kin = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t jj = P.param_offset + j;
        const double ph = st.p[jj] + 0.5 * eps * st.grad[jj];
        st.p[jj] = ph;
        kin += ph * ph * st.inv_mass[jj];
    }
    const double k = block_sum(kin, sh);
    if (threadIdx.x == 0) {
        const double h1 = -st.lnp[p] + 0.5 * k;
        const double du = st.uniforms[traj * n_patches + p];
        const double dh = st.h0[p] - h1;
        const int acc = isfinite(h1) && (log(du) < dh);
        s_acc = acc;
        st.accepted[p] += acc;
        st.energy_error[p] = dh;
        if (!acc) st.lnp[p] = st.lnp0[p];
    }
    __syncthreads();
    if (!s_acc) {
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int64_t jj = P.param_offset + j;
            st.z[jj] = st.z0[jj];
            st.grad[jj] = st.grad0[jj];
        }
    }
}

// advances the trajectory counter after end_kernel (a separate launch, so every
// CTA of end_kernel has read the current value)
__global__ void bump_kernel(int64_t *traj) { *traj += 1; }

}  // namespace

extern "C" int fp_hmc_prepare(const fp_hmc_patch *d_hp, int n_patches, const double *d_z, const double *d_lower,
                              const double *d_upper, const fp_spline_table *tab, fp_source *d_proposals,
                              double *d_theta, double *d_jac, void *stream)
{
    if (!d_hp || n_patches < 1 || !d_z || !tab || !d_proposals || !d_theta || !d_jac || (!d_lower != !d_upper))
        return fp_set_error(FP_ERR_ARGUMENT, "fp_hmc_prepare: bad arguments");
    if (tab->n_radii < 1 || tab->n_radii > MAXRADII || tab->kx < 1 || tab->kx > MAXDEG || tab->ky < 1 ||
        tab->ky > MAXDEG || tab->nx < 2 * tab->kx + 2 || tab->ny < 2 * tab->ky + 2 || !tab->tx || !tab->ty ||
        !tab->coef)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_hmc_prepare: bad spline table");
    prepare_kernel<<<n_patches, 32, 0, (cudaStream_t)stream>>>(d_hp, n_patches, d_z, d_lower, d_upper, *tab,
                                                               d_proposals, d_theta, d_jac);
    return fp_check_cuda(cudaGetLastError(), "prepare_kernel launch");
}

extern "C" int fp_hmc_lnprob(const fp_hmc_patch *d_hp, int n_patches, const double *d_z, const double *d_jac,
                             const double *d_chi2, const fp_response *d_response, int transformed, int sampling,
                             double *d_lnp, double *d_grad, void *stream)
{
    if (!d_hp || n_patches < 1 || !d_z || !d_jac || !d_chi2 || !d_response || !d_lnp || !d_grad)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_hmc_lnprob: bad arguments");
    lnprob_kernel<<<n_patches, HMC_THREADS, 0, (cudaStream_t)stream>>>(d_hp, d_z, d_jac, d_chi2, d_response,
                                                                       transformed, sampling, d_lnp, d_grad);
    return fp_check_cuda(cudaGetLastError(), "lnprob_kernel launch");
}

extern "C" int fp_hmc_leapfrog(const fp_hmc_patch *d_hp, int n_patches, const fp_hmc_state *state, int stage,
                               void *stream)
{
    if (!d_hp || n_patches < 1 || !state || state->n_traj < 1)
        return fp_set_error(FP_ERR_ARGUMENT, "fp_hmc_leapfrog: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    if (stage == FP_HMC_BEGIN) {
        begin_kernel<<<n_patches, HMC_THREADS, 0, st>>>(d_hp, *state);
    } else if (stage == FP_HMC_STEP) {
        step_kernel<<<n_patches, HMC_THREADS, 0, st>>>(d_hp, *state);
    } else if (stage == FP_HMC_END) {
        end_kernel<<<n_patches, HMC_THREADS, 0, st>>>(d_hp, n_patches, *state);
        if (int rc = fp_check_cuda(cudaGetLastError(), "end_kernel launch")) return rc;
        bump_kernel<<<1, 1, 0, st>>>(state->traj);
    } else {
        return fp_set_error(FP_ERR_ARGUMENT, "fp_hmc_leapfrog: unknown stage %d", stage);
    }
    return fp_check_cuda(cudaGetLastError(), "leapfrog launch");
}
