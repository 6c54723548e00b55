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

// value, d/dx (sersic), d/dy (rh) of spline `k` at (x, y)
__device__ void spline_eval(const SplineView &S, int k, double x, double y, double out[3]) {
    int lx, ly;
    double Bx[4], dBx[4], By[4], dBy[4];
    cubic_basis(S.tx, S.ntx, x, lx, Bx, dBx);
    cubic_basis(S.ty, S.nty, y, ly, By, dBy);
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

// One thread per source: parameters in the reference's Scene order
// [flux_1..flux_B, ra, dec, q, pa, sersic, rhalf] -> fpho_source.
// With `src_bands` / `src_off` (batched form) source s has src_bands[s] bands
// and its parameters start at theta[src_off[s]]; otherwise every source has
// `n_bands` bands and a stride of n_bands + 6.
__global__ void build_proposal_kernel(SplineView S, const double *theta, int n_src, int n_bands,
                                      const int *src_bands, const long long *src_off,
                                      fpho_source *out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_src) return;
    if (src_bands) n_bands = src_bands[s];
    const double *p = theta + (src_off ? (size_t)src_off[s] : (size_t)s * (n_bands + 6));
    fpho_source src;
    memset(&src, 0, sizeof(src));
    for (int b = 0; b < n_bands; ++b) src.fluxes[b] = (float)p[b];
    src.ra = (float)p[n_bands];
    src.dec = (float)p[n_bands + 1];
    src.q = (float)p[n_bands + 2];
    src.pa = (float)p[n_bands + 3];
    const double nser = p[n_bands + 4], rh = p[n_bands + 5];
    src.nsersic = (float)nser;
    src.rh = (float)rh;
    if (nser < S.sersic_min) {  // sources.py:656-660: all weight on the radius nearest rh
        int best = 0;
        double bd = fabs(rh - S.radii[0]);
        for (int k = 1; k < S.n_radii; ++k) {
            const double d = fabs(rh - S.radii[k]);
            if (d < bd) { bd = d; best = k; }
        }
        src.mixture_amplitudes[best] = 1.0f;
    } else if (rh < 0.0) {      // sources.py:661-663
        src.mixture_amplitudes[0] = 1.0f;
    } else {
        for (int k = 0; k < S.n_radii; ++k) {
            double v[3];
            spline_eval(S, k, nser, rh, v);
            src.mixture_amplitudes[k] = (float)v[0];
            src.damplitude_dnsersic[k] = (float)v[1];
            src.damplitude_drh[k] = (float)v[2];
        }
    }
    out[s] = src;
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
    build_proposal_kernel<<<(n_sources + 63) / 64, 64, 0, (cudaStream_t)stream>>>(
        s->view, theta, n_sources, n_bands, nullptr, nullptr, out);
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

extern "C" int fpho_build_proposal_batch(const fpho_spline *s, const double *theta, int n_sources,
                                         const int *src_bands, const long long *src_offset,
                                         fpho_source *out, void *stream) {
    clear_error();
    if (!s || !theta || !src_bands || !src_offset || !out)
        return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (n_sources < 1) return set_error(FPHO_ERR_INVALID, "n_sources=%d < 1", n_sources);
    build_proposal_kernel<<<(n_sources + 63) / 64, 64, 0, (cudaStream_t)stream>>>(
        s->view, theta, n_sources, 0, src_bands, src_offset, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FPHO_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return FPHO_OK;
}
