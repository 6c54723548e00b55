// fpho_model.cu -- proposals built on the device from a parameter vector.
//
// The reference builds each proposal on the host: Scene.set_all_source_params
// and Galaxy.proposal (forcepho/sources.py:46-97, 607-621), where the Sersic
// mixture amplitudes and their derivatives w.r.t. sersic index and half-light
// radius come from one scipy RectBivariateSpline per mixture radius
// (Galaxy.amplitudes / damplitude_dsersic / damplitude_drh,
// forcepho/sources.py:623-694).  Here the same bicubic B-splines (scipy's knots
// and coefficients, FITPACK's clamping of arguments to the knot range) are
// evaluated on the device in double precision, so a sampler step needs no host
// round trip and can be captured in a CUDA graph.
#include <cuda_runtime.h>

#include <cstring>
#include <new>

#include "fpho.h"
#include "fpho_internal.h"

namespace fpho {
namespace {

constexpr int SPL_MAX_KNOTS = 512;

// The four cubic B-splines that are non-zero at x (on knot interval l with
// t[l] <= x < t[l+1], l clamped to [3, n-5] and x to [t[3], t[n-4]]), and
// their first derivatives: de Boor's recursion to degree 2, one more step to
// degree 3, and B'_{i,3} = 3 (B_{i,2}/(t_{i+3}-t_i) - B_{i+1,2}/(t_{i+4}-t_{i+1})).
__device__ void cubic_basis(const double *t, int n, double x, int &l, double B[4], double dB[4]) {
    const double lo = t[3], hi = t[n - 4];
    x = fmin(fmax(x, lo), hi);
    int a = 3, b = n - 5;  // largest l in [3, n-5] with t[l] <= x
    while (a < b) {
        const int m = (a + b + 1) >> 1;
        if (t[m] <= x) a = m; else b = m - 1;
    }
    l = a;
    // degree-2 basis on interval l: N2[0..2] = B_{l-2,2}, B_{l-1,2}, B_{l,2}
    double left[4], right[4], N[4];
    N[0] = 1.0;
    for (int j = 1; j <= 2; ++j) {
        left[j] = x - t[l + 1 - j];
        right[j] = t[l + j] - x;
        double saved = 0.0;
        for (int r = 0; r < j; ++r) {
            const double den = right[r + 1] + left[j - r];
            const double tmp = den != 0.0 ? N[r] / den : 0.0;
            N[r] = saved + right[r + 1] * tmp;
            saved = left[j - r] * tmp;
        }
        N[j] = saved;
    }
    const double N2[3] = {N[0], N[1], N[2]};
    // degree 3
    left[3] = x - t[l - 2];
    right[3] = t[l + 3] - x;
    {
        double saved = 0.0;
        for (int r = 0; r < 3; ++r) {
            const double den = right[r + 1] + left[3 - r];
            const double tmp = den != 0.0 ? N[r] / den : 0.0;
            N[r] = saved + right[r + 1] * tmp;
            saved = left[3 - r] * tmp;
        }
        N[3] = saved;
    }
    for (int r = 0; r < 4; ++r) B[r] = N[r];
    // derivatives: basis index i = l-3+r; B_{i,2} is N2[r-1] (0 outside)
    for (int r = 0; r < 4; ++r) {
        const int i = l - 3 + r;
        const double b0 = (r >= 1) ? N2[r - 1] : 0.0;
        const double b1 = (r <= 2) ? N2[r] : 0.0;
        const double d0 = t[i + 3] - t[i], d1 = t[i + 4] - t[i + 1];
        dB[r] = 3.0 * ((d0 != 0.0 ? b0 / d0 : 0.0) - (d1 != 0.0 ? b1 / d1 : 0.0));
    }
}

struct SplineView {
    const double *tx, *ty, *coef, *radii;
    int ntx, nty, n_radii;
    double sersic_min;
};

// The B-spline bases at (x, y), shared by every radius's spline (all the
// mixture radii's splines have the same knots).
struct SplineBasis {
    int lx, ly;
    double Bx[4], dBx[4], By[4], dBy[4];
};
__device__ void spline_basis(const SplineView &S, double x, double y, SplineBasis &b) {
    cubic_basis(S.tx, S.ntx, x, b.lx, b.Bx, b.dBx);
    cubic_basis(S.ty, S.nty, y, b.ly, b.By, b.dBy);
}

// value, d/dx (sersic), d/dy (rh) of spline `k` from the bases at (x, y)
__device__ void spline_combine(const SplineView &S, int k, const SplineBasis &sb,
                               double out[3]) {
    const int lx = sb.lx, ly = sb.ly;
    const double *Bx = sb.Bx, *dBx = sb.dBx, *By = sb.By, *dBy = sb.dBy;
    const int ncy = S.nty - 4;
    const double *c = S.coef + (size_t)k * (S.ntx - 4) * ncy;
    double v = 0.0, vx = 0.0, vy = 0.0;
    for (int a = 0; a < 4; ++a) {
        const double *row = c + (size_t)(lx - 3 + a) * ncy + (ly - 3);
        double s = 0.0, sy = 0.0;
        for (int b = 0; b < 4; ++b) {
            s += row[b] * By[b];
            sy += row[b] * dBy[b];
        }
        v += Bx[a] * s;
        vx += dBx[a] * s;
        vy += Bx[a] * sy;
    }
    out[0] = v;
    out[1] = vx;
    out[2] = vy;
}

// value, d/dx (sersic), d/dy (rh) of spline `k` at (x, y)
__device__ void spline_eval(const SplineView &S, int k, double x, double y, double out[3]) {
    SplineBasis sb;
    spline_basis(S, x, y, sb);
    spline_combine(S, k, sb, out);
}

// One thread per source: parameters in the reference's Scene order
// [flux_1..flux_B, ra, dec, q, pa, sersic, rhalf] -> fpho_source.
// With `src_bands` / `src_off` (batched form) source s has src_bands[s] bands
// and its parameters start at theta[src_off[s]]; otherwise every source has
// `n_bands` bands and a stride of n_bands + 6.
// The knot vectors in shared memory: the binary searches of the bases then
// wait on shared-memory loads instead of dependent global ones.  Every thread
// of the block calls it (a barrier).
__device__ __forceinline__ SplineView knots_to_shared(const SplineView &S, double *s_tx,
                                                      double *s_ty) {
    for (int i = threadIdx.x; i < S.ntx; i += blockDim.x) s_tx[i] = S.tx[i];
    for (int i = threadIdx.x; i < S.nty; i += blockDim.x) s_ty[i] = S.ty[i];
    __syncthreads();
    SplineView L = S;
    L.tx = s_tx;
    L.ty = s_ty;
    return L;
}

// sigmoid in double, as torch.sigmoid evaluates it
__device__ __forceinline__ double sigmoid_d(double z) { return 1.0 / (1.0 + exp(-z)); }

// One warp per source: parameters in the reference's Scene order
// [flux_1..flux_B, ra, dec, q, pa, sersic, rhalf] -> fpho_source.  Lane i
// holds parameters i and i + 32 (with BOUNDED, mapped from unconstrained z
// through q = lower + range * sigmoid(z), BoundedTransform.transform,
// forcepho/model.py:596-637, and stored to q_out when given) and writes the
// fields they fill; lane k < n_radii evaluates mixture radius k's spline
// (value, d/dsersic, d/drh) with the reference's branches for sersic below
// the table and rh < 0 (forcepho/sources.py:656-663); every other field is
// zero.  Each field is rounded to float exactly as a per-source loop would.
// With `src_bands` / `src_off` (batched form) source s has src_bands[s]
// bands and its parameters start at par[src_off[s]]; otherwise every source
// has `n_bands` bands and a stride of n_bands + 6.
constexpr int PROP_THREADS = 128;
template <bool BOUNDED>
__global__ void __launch_bounds__(PROP_THREADS) proposal_kernel(
    SplineView S, const double *par, const double *lower, const double *range, int n_src,
    int n_bands, const int *src_bands, const long long *src_off, double *q_out,
    fpho_source *out) {
    __shared__ double s_tx[SPL_MAX_KNOTS], s_ty[SPL_MAX_KNOTS];
    const SplineView L = knots_to_shared(S, s_tx, s_ty);
    const int lane = threadIdx.x & 31;
    const int s = blockIdx.x * (PROP_THREADS / 32) + (threadIdx.x >> 5);
    if (s >= n_src) return;  // whole warps
    const int nb = src_bands ? src_bands[s] : n_bands;
    const size_t o = src_off ? (size_t)src_off[s] : (size_t)s * (nb + 6);
    const int np = nb + 6;
    float *f = reinterpret_cast<float *>(out + s);
    // field offsets (floats) in fpho_source
    constexpr int F_SHAPE = 0, F_FLUX = 6, F_AMP = F_FLUX + FPHO_MAXBANDS;
    constexpr int F_DRH = F_AMP + FPHO_MAXRADII, F_DN = F_DRH + FPHO_MAXRADII;
    double v[2] = {0.0, 0.0};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        if (i >= np) continue;
        double x = par[o + i];
        if (BOUNDED) {
            x = lower[o + i] + range[o + i] * sigmoid_d(x);
            if (q_out) q_out[o + i] = x;
        }
        v[h] = x;
        f[i < nb ? F_FLUX + i : F_SHAPE + (i - nb)] = (float)x;
    }
    if (lane >= nb && lane < FPHO_MAXBANDS) f[F_FLUX + lane] = 0.0f;
    const int in = nb + 4, ir = nb + 5;
    const double nser = __shfl_sync(0xffffffffu, in < 32 ? v[0] : v[1], in & 31);
    const double rh = __shfl_sync(0xffffffffu, ir < 32 ? v[0] : v[1], ir & 31);
    if (lane >= FPHO_MAXRADII) return;
    const int k = lane;
    float amp = 0.0f, dn = 0.0f, drh = 0.0f;
    if (nser < L.sersic_min) {  // all weight on the radius nearest rh
        int best = 0;
        double bd = fabs(rh - L.radii[0]);
        for (int j = 1; j < L.n_radii; ++j) {
            const double d = fabs(rh - L.radii[j]);
            if (d < bd) { bd = d; best = j; }
        }
        amp = (k == best) ? 1.0f : 0.0f;
    } else if (rh < 0.0) {
        amp = (k == 0) ? 1.0f : 0.0f;
    } else if (k < L.n_radii) {
        double w[3];
        spline_eval(L, k, nser, rh, w);
        amp = (float)w[0];
        dn = (float)w[1];
        drh = (float)w[2];
    }
    f[F_AMP + k] = amp;
    f[F_DRH + k] = drh;
    f[F_DN + k] = dn;
}

// lnp(z) = -chi2/2 + sum_i log jac_i and its gradient w.r.t. z, with
// jac_i = range_i s_i (1 - s_i), s_i = sigmoid(z_i) (FastPosterior.evaluate
// and BoundedTransform, forcepho/model.py:323-387, 596-637):
//   grad_i = -jac_i / 2 * sum_{k in map[i]} dchi2[k] + (1 - 2 s_i),
// the map of parameter i listing its dchi2 entries (a flux: one band; a shape
// parameter: every band of its patch, in band order), summed in double.  Each
// block writes the sum of its log jac terms; the last block to finish (a
// counter, reset for the next call) adds the partials and the chi2 in order.
constexpr int LNP_THREADS = 256;
__global__ void __launch_bounds__(LNP_THREADS) bounded_lnp_grad_kernel(
    int n, const double *z, const double *lower, const double *range, const float *dchi2,
    const int *map_off, const long long *map_idx, const double *chi2, int n_chi2, double *grad,
    double *lnp, double *partial, unsigned *counter) {
    __shared__ double red[LNP_THREADS];
    __shared__ bool last;
    const int i = blockIdx.x * LNP_THREADS + threadIdx.x;
    double lj = 0.0;
    if (i < n) {
        double gq = 0.0;
        for (int k = map_off[i]; k < map_off[i + 1]; ++k) gq += (double)dchi2[map_idx[k]];
        const double sg = sigmoid_d(z[i]);
        const double jac = range[i] * sg * (1.0 - sg);
        grad[i] = gq * (-0.5 * jac) + (1.0 - 2.0 * sg);
        lj = log(jac);
    }
    red[threadIdx.x] = lj;
    __syncthreads();
    for (int w = LNP_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = red[0];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block: -chi2/2 + the partials, each thread a strided share in
    // order, then the same tree as above
    __threadfence();
    double c = 0.0, l = 0.0;
    for (int b = threadIdx.x; b < n_chi2; b += LNP_THREADS) c += chi2[b];
    for (int b = threadIdx.x; b < (int)gridDim.x; b += LNP_THREADS)
        l += ((volatile double *)partial)[b];
    red[threadIdx.x] = -0.5 * c + l;
    __syncthreads();
    for (int w = LNP_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *lnp = red[0];
        *counter = 0u;
    }
}

// Spline values and derivatives at arbitrary points (for validation).
__global__ void spline_points_kernel(SplineView S, const double *x, const double *y, int m,
                                     double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * S.n_radii) return;
    const int pnt = i / S.n_radii, k = i - pnt * S.n_radii;
    double v[3];
    spline_eval(S, k, x[pnt], y[pnt], v);
    out[3 * i] = v[0];
    out[3 * i + 1] = v[1];
    out[3 * i + 2] = v[2];
}

}  // namespace
}  // namespace fpho

using namespace fpho;

struct fpho_spline {
    SplineView view;
    double *d_tx = nullptr, *d_ty = nullptr, *d_coef = nullptr, *d_radii = nullptr;
};

static void spline_destroy(fpho_spline *s) {
    if (!s) return;
    if (s->d_tx) cudaFree(s->d_tx);
    if (s->d_ty) cudaFree(s->d_ty);
    if (s->d_coef) cudaFree(s->d_coef);
    if (s->d_radii) cudaFree(s->d_radii);
    delete s;
}

extern "C" int fpho_spline_create(const double *tx, int ntx, const double *ty, int nty,
                                  const double *coeffs, int n_radii, const double *radii,
                                  double sersic_min, void *stream, fpho_spline **out) {
    clear_error();
    if (!tx || !ty || !coeffs || !radii || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (ntx < 8 || nty < 8 || ntx > SPL_MAX_KNOTS || nty > SPL_MAX_KNOTS)
        return set_error(FPHO_ERR_LIMIT, "knot counts (%d, %d) outside [8, %d]", ntx, nty,
                         SPL_MAX_KNOTS);
    if (n_radii < 1 || n_radii > FPHO_MAXRADII)
        return set_error(FPHO_ERR_LIMIT, "n_radii=%d outside [1, %d]", n_radii, FPHO_MAXRADII);
    for (int i = 1; i < ntx; ++i)
        if (tx[i] < tx[i - 1]) return set_error(FPHO_ERR_INVALID, "x knots not sorted");
    for (int i = 1; i < nty; ++i)
        if (ty[i] < ty[i - 1]) return set_error(FPHO_ERR_INVALID, "y knots not sorted");
    fpho_spline *s = new (std::nothrow) fpho_spline();
    if (!s) return set_error(FPHO_ERR_NOMEM, "host allocation failed");
    const size_t nc = (size_t)n_radii * (ntx - 4) * (nty - 4);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMalloc(&s->d_tx, sizeof(double) * ntx);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_ty, sizeof(double) * nty);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_coef, sizeof(double) * nc);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_radii, sizeof(double) * n_radii);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_tx, tx, sizeof(double) * ntx, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_ty, ty, sizeof(double) * nty, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_coef, coeffs, sizeof(double) * nc, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_radii, radii, sizeof(double) * n_radii, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        spline_destroy(s);
        return set_error(FPHO_ERR_CUDA, "spline upload: %s", cudaGetErrorString(e));
    }
    s->view.tx = s->d_tx;
    s->view.ty = s->d_ty;
    s->view.coef = s->d_coef;
    s->view.radii = s->d_radii;
    s->view.ntx = ntx;
    s->view.nty = nty;
    s->view.n_radii = n_radii;
    s->view.sersic_min = sersic_min;
    *out = s;
    return FPHO_OK;
}

extern "C" int fpho_spline_free(fpho_spline *s) {
    clear_error();
    spline_destroy(s);
    return FPHO_OK;
}

extern "C" int fpho_build_proposal(const fpho_spline *s, const double *theta, int n_sources,
                                   int n_bands, fpho_source *out, void *stream) {
    clear_error();
    if (!s || !theta || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (n_sources < 1 || n_sources > FPHO_MAX_ACTIVE_SOURCES)
        return set_error(FPHO_ERR_LIMIT, "n_sources=%d outside [1, %d]", n_sources,
                         FPHO_MAX_ACTIVE_SOURCES);
    if (n_bands < 1 || n_bands > FPHO_MAXBANDS)
        return set_error(FPHO_ERR_LIMIT, "n_bands=%d outside [1, %d]", n_bands, FPHO_MAXBANDS);
    proposal_kernel<false><<<(n_sources + 3) / 4, PROP_THREADS, 0, (cudaStream_t)stream>>>(
        s->view, theta, nullptr, nullptr, n_sources, n_bands, nullptr, nullptr, nullptr, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FPHO_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return FPHO_OK;
}

extern "C" int fpho_spline_points(const fpho_spline *s, const double *x, const double *y, int m,
                                  double *out, void *stream) {
    clear_error();
    if (!s || !x || !y || !out || m < 0) return set_error(FPHO_ERR_INVALID, "bad argument");
    const int n = m * s->view.n_radii;
    if (n > 0)
        spline_points_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(s->view, x, y, m,
                                                                               out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FPHO_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return FPHO_OK;
}

extern "C" int fpho_build_proposal_bounded(const fpho_spline *s, const double *z,
                                           const double *lower, const double *range,
                                           int n_sources, int n_bands, const int *src_bands,
                                           const long long *src_offset, double *q_out,
                                           fpho_source *out, void *stream) {
    clear_error();
    if (!s || !z || !lower || !range || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (n_sources < 1) return set_error(FPHO_ERR_INVALID, "n_sources=%d < 1", n_sources);
    if (!src_bands != !src_offset)
        return set_error(FPHO_ERR_INVALID, "src_bands and src_offset go together");
    if (!src_bands && (n_bands < 1 || n_bands > FPHO_MAXBANDS))
        return set_error(FPHO_ERR_LIMIT, "n_bands=%d outside [1, %d]", n_bands, FPHO_MAXBANDS);
    proposal_kernel<true><<<(n_sources + 3) / 4, PROP_THREADS, 0, (cudaStream_t)stream>>>(
        s->view, z, lower, range, n_sources, n_bands, src_bands, src_offset, q_out, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FPHO_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return FPHO_OK;
}

extern "C" int fpho_bounded_lnp_grad(int n_params, const double *z, const double *lower,
                                     const double *range, const float *dchi2,
                                     const int *map_offset, const long long *map_index,
                                     const double *chi2, int n_chi2, double *grad_out,
                                     double *lnp_out, double *work, int n_work,
                                     unsigned *counter, void *stream) {
    clear_error();
    if (n_params < 1 || n_chi2 < 0) return set_error(FPHO_ERR_INVALID, "bad sizes");
    if (!z || !lower || !range || !dchi2 || !map_offset || !map_index || (n_chi2 && !chi2) ||
        !grad_out || !lnp_out || !work || !counter)
        return set_error(FPHO_ERR_INVALID, "NULL argument");
    const int blocks = (n_params + LNP_THREADS - 1) / LNP_THREADS;
    if (n_work < blocks)
        return set_error(FPHO_ERR_LIMIT, "work holds %d partials, %d needed", n_work, blocks);
    bounded_lnp_grad_kernel<<<blocks, LNP_THREADS, 0, (cudaStream_t)stream>>>(
        n_params, z, lower, range, dchi2, map_offset, map_index, chi2, n_chi2, grad_out, lnp_out,
        work, counter);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FPHO_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return FPHO_OK;
}

extern "C" int fpho_build_proposal_batch(const fpho_spline *s, const double *theta, int n_sources,
                                         const int *src_bands, const long long *src_offset,
                                         fpho_source *out, void *stream) {
    clear_error();
    if (!s || !theta || !src_bands || !src_offset || !out)
        return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (n_sources < 1) return set_error(FPHO_ERR_INVALID, "n_sources=%d < 1", n_sources);
    proposal_kernel<false><<<(n_sources + 3) / 4, PROP_THREADS, 0, (cudaStream_t)stream>>>(
        s->view, theta, nullptr, nullptr, n_sources, 0, src_bands, src_offset, nullptr, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FPHO_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return FPHO_OK;
}
