// fpho_store.cu -- exposures resident in GPU memory, and the selection and
// packing of a patch's pixels from them.
//
// forcepho packs a patch on the host: for every exposure that overlaps the
// patch region it reads the whole super-pixel array from the HDF5 pixel store,
// tests the corners of every super-pixel against the region, and concatenates
// the selected super-pixels' fluxes, inverse errors and pixel coordinates
// (forcepho/patches/pixel_patch.py:124-198, 307-342; region tests
// forcepho/region.py:91-116 and 168-192).  Here the super-pixel arrays of all
// exposures stay in HBM (one 2048x2048 exposure is 32 MiB, so a B200 holds
// thousands), and three kernels do the selection and the packing:
//
//   store_count   one CTA per (chunk of 1024 super-pixels, exposure): the
//                 region test of every super-pixel, and the chunk's count;
//   store_scan    one CTA per exposure: exclusive prefix sum of its chunks'
//                 counts, and the exposure's total;
//   store_gather  one CTA per (chunk, exposure): the same test, the rank of
//                 each selected super-pixel within the chunk, then a copy of
//                 the chunk's selected super-pixels to their place in the
//                 patch arrays -- consecutive output addresses across the
//                 CTA, 256-byte runs of input per super-pixel of 8x8 --
//                 with the background offset and the signal-to-noise cap of
//                 forcepho/patches/pixel_patch.py:176-205 applied on the way.
//
// Output order is the reference's: exposures in the order given, super-pixels
// in row-major (x super-pixel, y super-pixel) order (numpy.where over the
// (nsx, nsy) selection), pixels in super-pixel order.  The circle test is the
// reference's arithmetic in double with every operation rounded separately
// (no contraction), so the selection is bit-identical; the rectangle test maps
// corners to the sky with the TAN projection in double, whose library
// sin/cos/atan2 may differ from the host's in the last unit, so a corner lying
// within ~1e-13 deg of the box edge can be decided differently.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "fpho_internal.h"

using fpho::set_error;
using fpho::clear_error;

#define CUDA_TRY(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return set_error(FPHO_ERR_CUDA, "%s failed: %s (%s:%d)", #call,             \
                             cudaGetErrorString(e_), __FILE__, __LINE__);               \
    } while (0)

struct fpho_store {
    int nsx = 0, nsy = 0, s = 0, s2 = 0;
    int cap = 0, n = 0;
    size_t exp_floats = 0;            // nsx * nsy * 2 s^2
    float *d_pix = nullptr;           // [cap][nsx][nsy][2 s^2]
    // per-call scratch, grown on demand
    int scratch_exp = 0;
    int *d_chunk = nullptr;           // [scratch_exp][n_chunks]
    int *d_total = nullptr;           // [scratch_exp]
    int *d_exps = nullptr;            // [scratch_exp]
    long long *d_start = nullptr;     // [scratch_exp] first output pixel
    float *d_bg = nullptr;            // [scratch_exp]
    fpho_region *d_regions = nullptr; // [scratch_exp]
    int n_chunks() const { return (nsx * nsy + kChunk - 1) / kChunk; }
    static constexpr int kChunk = 1024;
};

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = fpho_store::kChunk / kThreads;  // 4 consecutive super-pixels
constexpr double kD2R = 0.017453292519943295;              // pi / 180
constexpr double kR2D = 57.29577951308232;                 // 180 / pi

// Corner test of super-pixel (sx, sy); corners (0,0), (1,0), (1,1), (0,1)
// times (s - 1) from its first pixel (forcepho/patches/storage.py:117-139).
__device__ bool superpixel_selected(const fpho_region &R, int sx, int sy, int s) {
    const double x0 = (double)(sx * s), x1 = (double)(sx * s + s - 1);
    const double y0 = (double)(sy * s), y1 = (double)(sy * s + s - 1);
    const double cx[4] = {x0, x1, x1, x0};
    const double cy[4] = {y0, y0, y1, y1};
    if (R.kind == FPHO_REGION_CIRCLE) {
        const double xc = R.p[0], yc = R.p[1], r2 = R.p[2];
        bool in = false;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double dx = __dsub_rn(xc, cx[c]), dy = __dsub_rn(yc, cy[c]);
            in |= __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) < r2;
        }
        return in;
    }
    // rectangle: ra_min, ra_max, dec_min, dec_max, crpix1, crpix2 (1-based),
    // cd11, cd12, cd21, cd22, crval1, crval2, lonpole
    const double *p = R.p;
    const double a0 = p[10] * kD2R, d0 = p[11] * kD2R;
    double sd0, cd0;
    sincos(d0, &sd0, &cd0);
    bool in = false;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double u = __dsub_rn(__dadd_rn(cx[c], 1.0), p[4]);
        const double v = __dsub_rn(__dadd_rn(cy[c], 1.0), p[5]);
        const double xi = __dadd_rn(__dmul_rn(p[6], u), __dmul_rn(p[7], v));
        const double eta = __dadd_rn(__dmul_rn(p[8], u), __dmul_rn(p[9], v));
        const double r = hypot(xi, eta);
        const double phi = atan2(xi, -eta);
        const double theta = atan2(kR2D, r);
        const double dphi = __dsub_rn(phi, __dmul_rn(p[12], kD2R));
        double st, ct, sp, cp;
        sincos(theta, &st, &ct);
        sincos(dphi, &sp, &cp);
        const double X = __dsub_rn(__dmul_rn(st, cd0), __dmul_rn(__dmul_rn(ct, sd0), cp));
        const double Y = -__dmul_rn(ct, sp);
        const double Z = __dadd_rn(__dmul_rn(st, sd0), __dmul_rn(__dmul_rn(ct, cd0), cp));
        double ra = fmod(__dmul_rn(__dadd_rn(a0, atan2(Y, X)), kR2D), 360.0);
        if (ra < 0.0) ra += 360.0;
        const double dec = __dmul_rn(atan2(Z, hypot(X, Y)), kR2D);
        in |= (ra > p[0]) && (ra < p[1]) && (dec > p[2]) && (dec < p[3]);
    }
    return in;
}

// Flags of this thread's 4 consecutive super-pixels of the chunk (bit j set
// if super-pixel chunk*1024 + 4*tid + j is selected).
__device__ unsigned thread_flags(const fpho_region &R, int chunk, int nsx, int nsy, int s) {
    const int n = nsx * nsy;
    const int base = chunk * fpho_store::kChunk + threadIdx.x * kPerThread;
    unsigned f = 0;
#pragma unroll
    for (int j = 0; j < kPerThread; ++j) {
        const int sp = base + j;
        if (sp < n && superpixel_selected(R, sp / nsy, sp % nsy, s)) f |= 1u << j;
    }
    return f;
}

// Exclusive prefix sum of `v` over the CTA; *total receives the sum.
__device__ int block_exclusive_scan(int v, int *total) {
    __shared__ int warp_sum[kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < kThreads / 32 ? warp_sum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kThreads / 32) warp_sum[lane] = t;  // inclusive warp totals
    }
    __syncthreads();
    const int before = (w > 0 ? warp_sum[w - 1] : 0) + x - v;
    *total = warp_sum[kThreads / 32 - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(kThreads)
store_count(const fpho_region *regions, int nsx, int nsy, int s, int n_chunks, int *chunk_count) {
    const int e = blockIdx.y, chunk = blockIdx.x;
    const unsigned f = thread_flags(regions[e], chunk, nsx, nsy, s);
    const int c = __syncthreads_count(f & 1u) + __syncthreads_count(f & 2u) +
                  __syncthreads_count(f & 4u) + __syncthreads_count(f & 8u);
    if (threadIdx.x == 0) chunk_count[(size_t)e * n_chunks + chunk] = c;
}

// In place: counts -> exclusive offsets within the exposure; total per exposure.
__global__ void __launch_bounds__(kThreads)
store_scan(int n_chunks, int *chunk_count, int *total) {
    int *c = chunk_count + (size_t)blockIdx.x * n_chunks;
    int carry = 0;
    for (int i0 = 0; i0 < n_chunks; i0 += kThreads) {
        const int i = i0 + threadIdx.x;
        const int v = i < n_chunks ? c[i] : 0;
        int t;
        const int ex = block_exclusive_scan(v, &t);
        if (i < n_chunks) c[i] = carry + ex;
        carry += t;
    }
    if (threadIdx.x == 0) total[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(kThreads)
store_gather(const float *__restrict__ pix, size_t exp_floats, const int *exps,
             const fpho_region *regions, const int *chunk_off, const long long *exp_start,
             const float *bg, float max_snr, int nsx, int nsy, int s, int n_chunks,
             float *__restrict__ data, float *__restrict__ ierr, float *__restrict__ xpix,
             float *__restrict__ ypix) {
    __shared__ int sel[fpho_store::kChunk];
    const int e = blockIdx.y, chunk = blockIdx.x;
    const unsigned f = thread_flags(regions[e], chunk, nsx, nsy, s);
    int n_sel;
    int r = block_exclusive_scan(__popc(f), &n_sel);
    const int base = chunk * fpho_store::kChunk + threadIdx.x * kPerThread;
#pragma unroll
    for (int j = 0; j < kPerThread; ++j)
        if (f & (1u << j)) sel[r++] = base + j;
    __syncthreads();
    if (n_sel == 0) return;
    const int s2 = s * s;
    const long long out0 = exp_start[e] + (long long)chunk_off[(size_t)e * n_chunks + chunk] * s2;
    const float *src_e = pix + (size_t)exps[e] * exp_floats;
    const float b = bg ? bg[e] : 0.f;
    const int n = n_sel * s2;
    for (int i = threadIdx.x; i < n; i += kThreads) {
        const int sp = sel[i / s2], k = i % s2;
        const float *src = src_e + (size_t)sp * 2 * s2;
        float d = src[k], ie = src[s2 + k];
        if (bg) d = __fsub_rn(d, b);
        if (max_snr > 0.f && ie > 0.f && __fmul_rn(d, ie) > max_snr) ie = __fdiv_rn(max_snr, d);
        const long long o = out0 + i;
        data[o] = d;
        ierr[o] = ie;
        xpix[o] = (float)((sp / nsy) * s + k / s);
        ypix[o] = (float)((sp % nsy) * s + k % s);
    }
}

template <typename T>
int dalloc(T **p, size_t n) {
    *p = nullptr;
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_error(FPHO_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T),
                         cudaGetErrorString(e));
    }
    return FPHO_OK;
}
template <typename T>
void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

int ensure_scratch(fpho_store *st, int n_exp) {
    if (n_exp <= st->scratch_exp) return FPHO_OK;
    dfree(st->d_chunk); dfree(st->d_total); dfree(st->d_exps); dfree(st->d_start);
    dfree(st->d_bg); dfree(st->d_regions);
    st->scratch_exp = 0;
    int rc;
    if ((rc = dalloc(&st->d_chunk, (size_t)n_exp * st->n_chunks()))) return rc;
    if ((rc = dalloc(&st->d_total, (size_t)n_exp))) return rc;
    if ((rc = dalloc(&st->d_exps, (size_t)n_exp))) return rc;
    if ((rc = dalloc(&st->d_start, (size_t)n_exp))) return rc;
    if ((rc = dalloc(&st->d_bg, (size_t)n_exp))) return rc;
    if ((rc = dalloc(&st->d_regions, (size_t)n_exp))) return rc;
    st->scratch_exp = n_exp;
    return FPHO_OK;
}

// Validate the call's exposure list and regions, upload them, and run the
// count and scan kernels; `totals` receives super-pixels per exposure.
int count_pass(fpho_store *st, int n_exp, const int32_t *exposures, const fpho_region *regions,
               std::vector<int> &totals, cudaStream_t s) {
    if (!st || !exposures || !regions) return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (n_exp < 1 || n_exp > 65535)
        return set_error(FPHO_ERR_INVALID, "n_exp=%d outside [1, 65535]", n_exp);
    for (int e = 0; e < n_exp; ++e) {
        if (exposures[e] < 0 || exposures[e] >= st->n)
            return set_error(FPHO_ERR_INVALID, "exposure index %d outside [0, %d)", exposures[e],
                             st->n);
        if (regions[e].kind != FPHO_REGION_CIRCLE && regions[e].kind != FPHO_REGION_RECT)
            return set_error(FPHO_ERR_INVALID, "region %d: unknown kind %d", e, regions[e].kind);
    }
    int rc = ensure_scratch(st, n_exp);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(st->d_exps, exposures, sizeof(int) * n_exp, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(st->d_regions, regions, sizeof(fpho_region) * n_exp,
                             cudaMemcpyHostToDevice, s));
    const int nc = st->n_chunks();
    store_count<<<dim3(nc, n_exp), kThreads, 0, s>>>(st->d_regions, st->nsx, st->nsy, st->s, nc,
                                                     st->d_chunk);
    CUDA_TRY(cudaGetLastError());
    store_scan<<<n_exp, kThreads, 0, s>>>(nc, st->d_chunk, st->d_total);
    CUDA_TRY(cudaGetLastError());
    totals.assign(n_exp, 0);
    CUDA_TRY(cudaMemcpyAsync(totals.data(), st->d_total, sizeof(int) * n_exp,
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return FPHO_OK;
}

}  // namespace

extern "C" int fpho_store_create(int nside_x, int nside_y, int super_pixel_size, int max_exposures,
                                 fpho_store **out) {
    clear_error();
    if (!out) return set_error(FPHO_ERR_INVALID, "out is NULL");
    *out = nullptr;
    const int s = super_pixel_size;
    if (s < 1 || s > 64) return set_error(FPHO_ERR_INVALID, "super_pixel_size=%d outside [1, 64]", s);
    if (nside_x < s || nside_y < s || nside_x % s || nside_y % s)
        return set_error(FPHO_ERR_INVALID,
                         "image sides %d x %d are not positive multiples of the super-pixel "
                         "size %d", nside_x, nside_y, s);
    if (nside_x > 32767 || nside_y > 32767)  // pixel coordinates are int16 in the reference
        return set_error(FPHO_ERR_LIMIT, "image sides above 32767");
    if (max_exposures < 1) return set_error(FPHO_ERR_INVALID, "max_exposures=%d", max_exposures);
    fpho_store *st = new (std::nothrow) fpho_store();
    if (!st) return set_error(FPHO_ERR_NOMEM, "host allocation failed");
    st->nsx = nside_x / s;
    st->nsy = nside_y / s;
    st->s = s;
    st->s2 = s * s;
    st->cap = max_exposures;
    st->exp_floats = (size_t)st->nsx * st->nsy * 2 * st->s2;
    if (int rc = dalloc(&st->d_pix, st->exp_floats * (size_t)max_exposures)) {
        delete st;
        return rc;
    }
    *out = st;
    return FPHO_OK;
}

extern "C" int fpho_store_add_exposure(fpho_store *st, const float *superpixels, int on_device,
                                       void *stream, int *index) {
    clear_error();
    if (!st || !superpixels) return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (st->n >= st->cap)
        return set_error(FPHO_ERR_LIMIT, "the store is full (%d exposures)", st->cap);
    cudaStream_t s = (cudaStream_t)stream;
    CUDA_TRY(cudaMemcpyAsync(st->d_pix + (size_t)st->n * st->exp_floats, superpixels,
                             st->exp_floats * sizeof(float),
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    if (index) *index = st->n;
    st->n++;
    return FPHO_OK;
}

extern "C" int fpho_store_info(const fpho_store *st, int64_t out[6]) {
    clear_error();
    if (!st || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    out[0] = st->nsx;
    out[1] = st->nsy;
    out[2] = st->s;
    out[3] = st->n;
    out[4] = st->cap;
    out[5] = (int64_t)(st->exp_floats * sizeof(float));
    return FPHO_OK;
}

extern "C" int fpho_store_count(fpho_store *st, int n_exp, const int32_t *exposures,
                                const fpho_region *regions, int32_t *n_superpixels, void *stream) {
    clear_error();
    if (!n_superpixels) return set_error(FPHO_ERR_INVALID, "n_superpixels is NULL");
    std::vector<int> totals;
    int rc = count_pass(st, n_exp, exposures, regions, totals, (cudaStream_t)stream);
    if (rc) return rc;
    std::copy(totals.begin(), totals.end(), n_superpixels);
    return FPHO_OK;
}

extern "C" int fpho_store_gather(fpho_store *st, int n_exp, const int32_t *exposures,
                                 const fpho_region *regions, const float *background,
                                 float max_snr, float *data, float *ierr, float *xpix,
                                 float *ypix, int64_t npix_capacity, int32_t *exposure_start,
                                 int32_t *exposure_N, void *stream) {
    clear_error();
    if (!exposure_start || !exposure_N)
        return set_error(FPHO_ERR_INVALID, "exposure_start/exposure_N is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<int> totals;
    int rc = count_pass(st, n_exp, exposures, regions, totals, s);
    if (rc) return rc;
    std::vector<long long> start(n_exp);
    long long npix = 0;
    for (int e = 0; e < n_exp; ++e) {
        start[e] = npix;
        exposure_start[e] = (int32_t)std::min<long long>(npix, INT32_MAX);
        exposure_N[e] = totals[e] * st->s2;
        npix += (long long)totals[e] * st->s2;
    }
    if (npix > INT32_MAX) return set_error(FPHO_ERR_LIMIT, "the patch would have %lld pixels", npix);
    if (npix > npix_capacity)
        return set_error(FPHO_ERR_LIMIT, "the patch has %lld pixels; the output holds %lld", npix,
                         (long long)npix_capacity);
    if (npix == 0) return FPHO_OK;
    if (!data || !ierr || !xpix || !ypix)
        return set_error(FPHO_ERR_INVALID, "an output pixel array is NULL");
    CUDA_TRY(cudaMemcpyAsync(st->d_start, start.data(), sizeof(long long) * n_exp,
                             cudaMemcpyHostToDevice, s));
    if (background)
        CUDA_TRY(cudaMemcpyAsync(st->d_bg, background, sizeof(float) * n_exp,
                                 cudaMemcpyHostToDevice, s));
    const int nc = st->n_chunks();
    store_gather<<<dim3(nc, n_exp), kThreads, 0, s>>>(
        st->d_pix, st->exp_floats, st->d_exps, st->d_regions, st->d_chunk, st->d_start,
        background ? st->d_bg : nullptr, max_snr, st->nsx, st->nsy, st->s, nc, data, ierr, xpix,
        ypix);
    CUDA_TRY(cudaGetLastError());
    // the host vectors above die on return; the stream must be done with them
    CUDA_TRY(cudaStreamSynchronize(s));
    return FPHO_OK;
}

extern "C" int fpho_store_free(fpho_store *st) {
    clear_error();
    if (!st) return FPHO_OK;
    dfree(st->d_pix);
    dfree(st->d_chunk); dfree(st->d_total); dfree(st->d_exps); dfree(st->d_start);
    dfree(st->d_bg); dfree(st->d_regions);
    delete st;
    return FPHO_OK;
}
