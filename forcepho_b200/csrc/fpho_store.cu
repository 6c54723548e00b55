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
// thousands), and four kernels do the selection and the packing:
//
//   store_count    one CTA per (chunk of 1024 super-pixels, exposure): the
//                  region test of every super-pixel of the exposure's box
//                  (the rows and columns a circle can reach, computed on the
//                  host; the whole image for a rectangle), and the chunk's
//                  count;
//   store_scan     one CTA per exposure: exclusive prefix sum of its chunks'
//                  counts, and the exposure's total (read back by the host,
//                  which sizes the patch from it);
//   store_compact  one CTA per (chunk, exposure): the same test and the rank
//                  of each selected super-pixel, which goes to its place in a
//                  list of the selected super-pixels in output order;
//   store_copy     one thread per 4 output pixels of the list (float4 loads
//                  and stores when the super-pixel side is even and the
//                  outputs are 16-byte aligned), so every CTA moves data and
//                  the stores are consecutive across each warp: fluxes minus
//                  the background offset, inverse errors with the
//                  signal-to-noise cap of forcepho/patches/pixel_patch.py:
//                  176-205, and the pixel coordinates.
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
#include <cmath>
#include <cstdint>
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
    int *d_spbase = nullptr;          // [scratch_exp] selected super-pixels before exposure e
    int *d_box = nullptr;             // [scratch_exp][4] super-pixel box of each exposure
    int grid_chunks = 1;              // chunks per exposure of the last count pass
    int *d_list_sp = nullptr;         // [list_cap] selected super-pixels in output order
    int *d_list_exp = nullptr;        // [list_cap] their position in the exposure list
    size_t list_cap = 0;
    float *d_bg = nullptr;            // [scratch_exp]
    fpho_region *d_regions = nullptr; // [scratch_exp]
    // optional CUDA-event timing of the gather kernel
    bool time_gather = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_gather_ms = 0.f;
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

// The super-pixels a region can select in one exposure: rows x0..x0+nx-1,
// columns y0..y0+ny-1 (a conservative box computed on the host; the whole
// image when no box is known).  Visited in row-major order, which is the
// order of the whole image restricted to the box.
struct SpBox {
    int x0, y0, nx, ny;
};

// Flags of this thread's 4 consecutive super-pixels of the chunk of the box
// (bit j set if box position chunk*1024 + 4*tid + j is selected).
__device__ unsigned thread_flags(const fpho_region &R, const SpBox &B, int chunk, int s) {
    const int n = B.nx * B.ny;
    const int base = chunk * fpho_store::kChunk + threadIdx.x * kPerThread;
    unsigned f = 0;
#pragma unroll
    for (int j = 0; j < kPerThread; ++j) {
        const int b = base + j;
        if (b < n && superpixel_selected(R, B.x0 + b / B.ny, B.y0 + b % B.ny, s)) f |= 1u << j;
    }
    return f;
}

__device__ __forceinline__ int box_chunks(const SpBox &B) {
    return (B.nx * B.ny + fpho_store::kChunk - 1) / fpho_store::kChunk;
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
store_count(const fpho_region *regions, const SpBox *boxes, int s, int n_chunks,
            int *chunk_count) {
    const int e = blockIdx.y, chunk = blockIdx.x;
    const SpBox B = boxes[e];
    if (chunk >= box_chunks(B)) {
        if (threadIdx.x == 0) chunk_count[(size_t)e * n_chunks + chunk] = 0;
        return;
    }
    const unsigned f = thread_flags(regions[e], B, chunk, s);
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
store_compact(const fpho_region *regions, const SpBox *boxes, const int *chunk_off,
              const int *spbase, int nsy, int s, int n_chunks, int *list_sp, int *list_exp) {
    const int e = blockIdx.y, chunk = blockIdx.x;
    const SpBox B = boxes[e];
    if (chunk >= box_chunks(B)) return;
    const unsigned f = thread_flags(regions[e], B, chunk, s);
    int n_sel;
    const int r = block_exclusive_scan(__popc(f), &n_sel);
    if (n_sel == 0) return;
    const long long o = (long long)spbase[e] + chunk_off[(size_t)e * n_chunks + chunk] + r;
    const int base = chunk * fpho_store::kChunk + threadIdx.x * kPerThread;
    int q = 0;
#pragma unroll
    for (int j = 0; j < kPerThread; ++j)
        if (f & (1u << j)) {
            const int b = base + j;
            list_sp[o + q] = (B.x0 + b / B.ny) * nsy + (B.y0 + b % B.ny);
            list_exp[o + q] = e;
            ++q;
        }
}

__device__ __forceinline__ void pack_pixel(float &d, float &ie, float b, bool has_bg,
                                           float max_snr) {
    if (has_bg) d = __fsub_rn(d, b);
    if (max_snr > 0.f && ie > 0.f && __fmul_rn(d, ie) > max_snr) ie = __fdiv_rn(max_snr, d);
}

// VEC: 4 consecutive output pixels per thread (s^2 % 4 == 0, outputs 16-byte
// aligned); otherwise one.  Output pixel p belongs to list entry p / s^2.
template <bool VEC>
__global__ void __launch_bounds__(kThreads)
store_copy(const float *__restrict__ pix, size_t exp_floats, const int *__restrict__ exps,
           const int *__restrict__ list_sp, const int *__restrict__ list_exp, long long n_items,
           const float *__restrict__ bg, float max_snr, int nsy, int s,
           float *__restrict__ data, float *__restrict__ ierr, float *__restrict__ xpix,
           float *__restrict__ ypix) {
    const long long g = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (g >= n_items) return;
    const int s2 = s * s;
    const long long p = VEC ? g * 4 : g;
    const long long j = p / s2;
    const int k = (int)(p - j * s2);
    const int e = list_exp[j], sp = list_sp[j];
    const float *src = pix + (size_t)exps[e] * exp_floats + (size_t)sp * 2 * s2;
    const float b = bg ? bg[e] : 0.f;
    const int x0 = (sp / nsy) * s, y0 = (sp % nsy) * s;
    if (VEC) {
        float4 d = *reinterpret_cast<const float4 *>(src + k);
        float4 ie = *reinterpret_cast<const float4 *>(src + s2 + k);
        pack_pixel(d.x, ie.x, b, bg != nullptr, max_snr);
        pack_pixel(d.y, ie.y, b, bg != nullptr, max_snr);
        pack_pixel(d.z, ie.z, b, bg != nullptr, max_snr);
        pack_pixel(d.w, ie.w, b, bg != nullptr, max_snr);
        *reinterpret_cast<float4 *>(data + p) = d;
        *reinterpret_cast<float4 *>(ierr + p) = ie;
        *reinterpret_cast<float4 *>(xpix + p) =
            make_float4((float)(x0 + k / s), (float)(x0 + (k + 1) / s), (float)(x0 + (k + 2) / s),
                        (float)(x0 + (k + 3) / s));
        *reinterpret_cast<float4 *>(ypix + p) =
            make_float4((float)(y0 + k % s), (float)(y0 + (k + 1) % s), (float)(y0 + (k + 2) % s),
                        (float)(y0 + (k + 3) % s));
    } else {
        float d = src[k], ie = src[s2 + k];
        pack_pixel(d, ie, b, bg != nullptr, max_snr);
        data[p] = d;
        ierr[p] = ie;
        xpix[p] = (float)(x0 + k / s);
        ypix[p] = (float)(y0 + k % s);
    }
}

// Scratch comes from the handle memory pool (fpho_internal.h); the exposure
// array itself is one plain cudaMalloc at creation.
template <typename T>
int dalloc(T **p, size_t n) {
    *p = nullptr;
    cudaError_t e = fpho::pool_malloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_error(FPHO_ERR_NOMEM, "device allocation of %zu bytes failed: %s",
                         n * sizeof(T), cudaGetErrorString(e));
    }
    return FPHO_OK;
}
template <typename T>
void dfree(T *&p) {
    fpho::pool_free((void *)p);
    p = nullptr;
}

int ensure_scratch(fpho_store *st, int n_exp) {
    if (n_exp <= st->scratch_exp) return FPHO_OK;
    dfree(st->d_chunk); dfree(st->d_total); dfree(st->d_exps); dfree(st->d_spbase);
    dfree(st->d_bg); dfree(st->d_regions); dfree(st->d_box);
    st->scratch_exp = 0;
    int rc;
    if ((rc = dalloc(&st->d_chunk, (size_t)n_exp * st->n_chunks()))) return rc;
    if ((rc = dalloc(&st->d_total, (size_t)n_exp))) return rc;
    if ((rc = dalloc(&st->d_exps, (size_t)n_exp))) return rc;
    if ((rc = dalloc(&st->d_spbase, (size_t)n_exp))) return rc;
    if ((rc = dalloc(&st->d_box, (size_t)n_exp * 4))) return rc;
    if ((rc = dalloc(&st->d_bg, (size_t)n_exp))) return rc;
    if ((rc = dalloc(&st->d_regions, (size_t)n_exp))) return rc;
    st->scratch_exp = n_exp;
    return FPHO_OK;
}

// The super-pixels a region can select (rows x0.., columns y0.., counts nx,
// ny).  For a circle: super-pixels whose corner pixels all lie at least
// r + 1 pixel from the centre along x (or along y) cannot pass the test
// (xc - x)^2 + (yc - y)^2 < r2, whatever the rounding, so the box keeps the
// rows and columns within that reach.  A circle with r2 <= 0 selects
// nothing; other regions, and circles with non-finite parameters, get the
// whole image (the exact test decides).
void region_box(const fpho_region &R, int nsx, int nsy, int s, int box[4]) {
    box[0] = 0; box[1] = 0; box[2] = nsx; box[3] = nsy;
    if (R.kind != FPHO_REGION_CIRCLE) return;
    const double xc = R.p[0], yc = R.p[1], r2 = R.p[2];
    if (!std::isfinite(xc) || !std::isfinite(yc) || !std::isfinite(r2)) return;
    if (!(r2 > 0.0)) {
        box[2] = box[3] = 0;
        return;
    }
    const double reach = std::sqrt(r2) + 1.0;
    auto range = [&](double c, int n, int &lo, int &cnt) {
        // super-pixel i can pass only if [i s, i s + s - 1] meets (c - reach, c + reach)
        const double a = std::floor((c - reach - (s - 1)) / s), b = std::floor((c + reach) / s);
        const double a2 = std::max(a, 0.0), b2 = std::min(b, (double)(n - 1));
        if (a2 > b2) {
            lo = 0;
            cnt = 0;
        } else {
            lo = (int)a2;
            cnt = (int)(b2 - a2) + 1;
        }
    };
    range(xc, nsx, box[0], box[2]);
    range(yc, nsy, box[1], box[3]);
    if (box[2] == 0 || box[3] == 0) box[2] = box[3] = 0;
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
    std::vector<int> boxes(4 * (size_t)n_exp);
    int nc = 1;
    for (int e = 0; e < n_exp; ++e) {
        region_box(regions[e], st->nsx, st->nsy, st->s, &boxes[4 * (size_t)e]);
        const long long n = (long long)boxes[4 * e + 2] * boxes[4 * e + 3];
        nc = std::max(nc, (int)((n + fpho_store::kChunk - 1) / fpho_store::kChunk));
    }
    st->grid_chunks = nc;
    CUDA_TRY(cudaMemcpyAsync(st->d_box, boxes.data(), sizeof(int) * boxes.size(),
                             cudaMemcpyHostToDevice, s));
    store_count<<<dim3(nc, n_exp), kThreads, 0, s>>>(
        st->d_regions, reinterpret_cast<const SpBox *>(st->d_box), st->s, nc, st->d_chunk);
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
    const size_t bytes = st->exp_floats * (size_t)max_exposures * sizeof(float);
    if (cudaMalloc((void **)&st->d_pix, bytes) != cudaSuccess) {
        st->d_pix = nullptr;
        delete st;
        return set_error(FPHO_ERR_NOMEM, "cudaMalloc of %zu bytes for %d exposures failed",
                         bytes, max_exposures);
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
    std::vector<int> spbase(n_exp);
    long long npix = 0, nsp = 0;
    for (int e = 0; e < n_exp; ++e) {
        spbase[e] = (int)std::min<long long>(nsp, INT32_MAX);
        exposure_start[e] = (int32_t)std::min<long long>(npix, INT32_MAX);
        exposure_N[e] = totals[e] * st->s2;
        npix += (long long)totals[e] * st->s2;
        nsp += totals[e];
    }
    if (npix > INT32_MAX) return set_error(FPHO_ERR_LIMIT, "the patch would have %lld pixels", npix);
    if (npix > npix_capacity)
        return set_error(FPHO_ERR_LIMIT, "the patch has %lld pixels; the output holds %lld", npix,
                         (long long)npix_capacity);
    if (npix == 0) return FPHO_OK;
    if (!data || !ierr || !xpix || !ypix)
        return set_error(FPHO_ERR_INVALID, "an output pixel array is NULL");
    if ((size_t)nsp > st->list_cap) {
        dfree(st->d_list_sp);
        dfree(st->d_list_exp);
        st->list_cap = 0;
        if ((rc = dalloc(&st->d_list_sp, (size_t)nsp))) return rc;
        if ((rc = dalloc(&st->d_list_exp, (size_t)nsp))) return rc;
        st->list_cap = (size_t)nsp;
    }
    CUDA_TRY(cudaMemcpyAsync(st->d_spbase, spbase.data(), sizeof(int) * n_exp,
                             cudaMemcpyHostToDevice, s));
    if (background)
        CUDA_TRY(cudaMemcpyAsync(st->d_bg, background, sizeof(float) * n_exp,
                                 cudaMemcpyHostToDevice, s));
    const int nc = st->grid_chunks;
    const bool vec = (st->s2 % 4 == 0) &&
                     ((((uintptr_t)data) | ((uintptr_t)ierr) | ((uintptr_t)xpix) |
                       ((uintptr_t)ypix)) % 16 == 0);
    const long long n_items = vec ? npix / 4 : npix;
    const unsigned blocks = (unsigned)((n_items + kThreads - 1) / kThreads);
    if (st->time_gather) CUDA_TRY(cudaEventRecord(st->ev0, s));
    store_compact<<<dim3(nc, n_exp), kThreads, 0, s>>>(
        st->d_regions, reinterpret_cast<const SpBox *>(st->d_box), st->d_chunk, st->d_spbase,
        st->nsy, st->s, nc, st->d_list_sp, st->d_list_exp);
    CUDA_TRY(cudaGetLastError());
    const float *bgp = background ? st->d_bg : nullptr;
    if (vec)
        store_copy<true><<<blocks, kThreads, 0, s>>>(st->d_pix, st->exp_floats, st->d_exps,
                                                     st->d_list_sp, st->d_list_exp, n_items, bgp,
                                                     max_snr, st->nsy, st->s, data, ierr, xpix,
                                                     ypix);
    else
        store_copy<false><<<blocks, kThreads, 0, s>>>(st->d_pix, st->exp_floats, st->d_exps,
                                                      st->d_list_sp, st->d_list_exp, n_items, bgp,
                                                      max_snr, st->nsy, st->s, data, ierr, xpix,
                                                      ypix);
    CUDA_TRY(cudaGetLastError());
    if (st->time_gather) CUDA_TRY(cudaEventRecord(st->ev1, s));
    // the host vectors above die on return; the stream must be done with them
    CUDA_TRY(cudaStreamSynchronize(s));
    if (st->time_gather) CUDA_TRY(cudaEventElapsedTime(&st->last_gather_ms, st->ev0, st->ev1));
    return FPHO_OK;
}

extern "C" int fpho_store_time_gather(fpho_store *st, int enable) {
    clear_error();
    if (!st) return set_error(FPHO_ERR_INVALID, "NULL store");
    if (enable && !st->ev0) {
        CUDA_TRY(cudaEventCreate(&st->ev0));
        CUDA_TRY(cudaEventCreate(&st->ev1));
    }
    st->time_gather = enable != 0;
    return FPHO_OK;
}

extern "C" int fpho_store_last_gather_ms(const fpho_store *st, float *ms) {
    clear_error();
    if (!st || !ms) return set_error(FPHO_ERR_INVALID, "NULL argument");
    *ms = st->last_gather_ms;
    return FPHO_OK;
}

extern "C" int fpho_store_free(fpho_store *st) {
    clear_error();
    if (!st) return FPHO_OK;
    if (st->ev0) cudaEventDestroy(st->ev0);
    if (st->ev1) cudaEventDestroy(st->ev1);
    if (st->d_pix) cudaFree(st->d_pix);
    st->d_pix = nullptr;
    dfree(st->d_chunk); dfree(st->d_total); dfree(st->d_exps); dfree(st->d_spbase);
    dfree(st->d_bg); dfree(st->d_regions);
    dfree(st->d_list_sp); dfree(st->d_list_exp); dfree(st->d_box);
    delete st;
    return FPHO_OK;
}
