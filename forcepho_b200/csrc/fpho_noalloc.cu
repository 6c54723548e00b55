// fpho_noalloc.cu -- evaluation of a proposal without allocating memory.
//
// fpho_evaluate_proposal_noalloc runs the same kernels as the handle-based
// path, but takes every patch array as a device pointer from the caller and
// keeps all of its scratch (tile plan, image-Gaussian records and culling
// boxes, per-tile partial sums) in one file-scope device array of
// FPHO_NOALLOC_SCRATCH_BYTES.  It is meant for callers that cannot call
// cudaMalloc: plugins whose host framework owns every device allocation (its
// allocator alone may take device memory, so that its accounting and limits
// hold), and long-running services that must not grow or fragment device
// memory after start-up.
//
// Semantics a caller must know:
//   * The array exists once per device, in every process that loads the
//     library, until the process exits (FPHO_NOALLOC_SCRATCH_BYTES of device
//     memory per device used).
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) and raises the tile kernel's shared-memory limit
//     to the device's ceiling, so that no later call changes a kernel
//     attribute; make that first call before any stream capture.  The address
//     is kept for the life of the process: a device reset
//     (cudaDeviceReset, or a reset of the primary context) is not supported.
//   * Every call shares the array and it keeps the last call's contents; each
//     call rebuilds what it needs (the plan and the error word are written by
//     the first kernel of the call).  Calls whose kernels overlap on the GPU
//     (on different streams, or from different threads) race on the array and
//     give wrong results: serialize them.
//   * The patch arrays are not validated on the host (they are device memory);
//     index inconsistencies found on the device are reported in *dev_status,
//     and any error makes every dev_chi2 entry NaN, so that a failed call
//     never looks like a result, whether or not dev_status is given.
#include <cuda_runtime.h>

#include <mutex>

#include "fpho_impl.cuh"
#include "fpho_internal.h"
#include "fpho_kernels.cuh"
#include "fpho_tile.cuh"

namespace fpho {

static __device__ __align__(256) unsigned char g_noalloc_scratch[FPHO_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int NA_THREADS = 128;   // tile kernel: 128 threads x 4 pixels
constexpr int NA_K = 4;
constexpr int NA_TILE = NA_THREADS * NA_K;
constexpr int NA_LIVE_CAP = 256;

// device status / error word bits (bit 0, a bounded bulk-copy wait that gave
// up, is set by the tile kernel itself)
constexpr int NA_ERR_INDEX = 2;   // inconsistent band / exposure index arrays
constexpr int NA_ERR_BOUND = 4;    // the caller's size bounds were exceeded
constexpr int NA_ERR_PSF = 8;      // a PSF Gaussian's radius bin outside [0, n_radii)

struct Header {
    int n_tiles;
    int n_gauss;
    int err;
    int pad[61];
};

struct Layout {
    size_t hdr, exp_band, exp_npsf, gauss_start, tile_band_start, tiles, tbox_all, tbox_w,
        gtab, gbox, pchi2, pgrad, total;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

Layout make_layout(int n_bands, int n_exp, long long n_tiles_max, long long n_gauss_max,
                   int nsrc) {
    Layout L;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o = align256(o + bytes);
        return at;
    };
    L.hdr = take(sizeof(Header));
    L.exp_band = take(sizeof(int) * (size_t)n_exp);
    L.exp_npsf = take(sizeof(int) * (size_t)n_exp);
    L.gauss_start = take(sizeof(int) * ((size_t)n_exp + 1));
    L.tile_band_start = take(sizeof(int) * ((size_t)n_bands + 1));
    L.tiles = take(sizeof(TileDesc) * (size_t)n_tiles_max);
    L.tbox_all = take(sizeof(float4) * (size_t)n_tiles_max);
    L.tbox_w = take(sizeof(float4) * (size_t)n_tiles_max);
    L.gtab = take(sizeof(float) * GREC * (size_t)n_gauss_max);
    L.gbox = take(sizeof(float4) * (size_t)n_gauss_max);
    L.pchi2 = take(sizeof(double) * (size_t)n_tiles_max);
    L.pgrad = take(sizeof(float) * 7 * (size_t)nsrc * (size_t)n_tiles_max);
    L.total = o;
    return L;
}

// One thread builds the plan: band of each exposure, image-Gaussian offsets,
// tile list.  Clears the error word first.
// Every exposure's pixel run [exposure_start, exposure_start + exposure_N) must
// lie inside the caller's pixel arrays of total_pixels entries, and every
// exposure with PSF components needs psfgauss_start >= 0; otherwise the plan
// is empty and NA_ERR_INDEX is set, before any pixel is read.
__global__ void noalloc_plan(const int16_t *band_start, const int16_t *band_N,
                             const int *exposure_start, const int *exposure_N,
                             const int *n_psf_per_source, const int *psfgauss_start,
                             long long total_pixels, int n_bands, int n_exp, int nsrc,
                             int max_npsf, int n_tiles_max, int n_gauss_max, Header *hdr,
                             int *exp_band, int *exp_npsf, int *gauss_start,
                             int *tile_band_start, TileDesc *tiles) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int err = 0;
    for (int e = 0; e < n_exp; ++e) exp_band[e] = -1;
    for (int b = 0; b < n_bands; ++b) {
        const int s = band_start[b], n = band_N[b];
        if (s < 0 || n < 0 || s + n > n_exp) {
            err |= NA_ERR_INDEX;
            continue;
        }
        for (int e = s; e < s + n; ++e) {
            if (exp_band[e] != -1) err |= NA_ERR_INDEX;
            exp_band[e] = b;
        }
    }
    long long acc = 0;
    for (int e = 0; e < n_exp; ++e) {
        const int b = exp_band[e];
        int npsf = (b >= 0) ? n_psf_per_source[b] : 0;
        if (npsf < 0 || npsf > max_npsf) {
            err |= NA_ERR_BOUND;
            npsf = 0;
        }
        if (npsf > 0 && psfgauss_start[e] < 0) err |= NA_ERR_INDEX;
        exp_npsf[e] = npsf;
        gauss_start[e] = (int)(acc < n_gauss_max ? acc : n_gauss_max);
        acc += (long long)nsrc * npsf;
    }
    if (acc > n_gauss_max) err |= NA_ERR_BOUND;
    gauss_start[n_exp] = (int)(acc < n_gauss_max ? acc : n_gauss_max);
    long long nt = 0;
    for (int b = 0; b < n_bands; ++b) {
        tile_band_start[b] = (int)(nt < n_tiles_max ? nt : n_tiles_max);
        const int s = band_start[b], n = band_N[b];
        if (s < 0 || n < 0 || s + n > n_exp) continue;
        for (int e = s; e < s + n; ++e) {
            const int N = exposure_N[e], p0 = exposure_start[e];
            if (N < 0 || p0 < 0 || (long long)p0 + N > total_pixels) {
                err |= NA_ERR_INDEX;
                continue;
            }
            for (int off = 0; off < N; off += NA_TILE) {
                if (nt < n_tiles_max) {
                    TileDesc t;
                    t.exposure = e;
                    t.band = b;
                    t.pix_begin = p0 + off;
                    t.count = (N - off < NA_TILE) ? N - off : NA_TILE;
                    tiles[nt] = t;
                }
                ++nt;
            }
        }
    }
    tile_band_start[n_bands] = (int)(nt < n_tiles_max ? nt : n_tiles_max);
    if (nt > n_tiles_max) err |= NA_ERR_BOUND;
    if (err) {  // nothing downstream may run on an inconsistent plan
        for (int b = 0; b <= n_bands; ++b) tile_band_start[b] = 0;
        for (int e = 0; e <= n_exp; ++e) gauss_start[e] = 0;
        nt = 0;
        acc = 0;
    }
    hdr->n_tiles = (int)nt;
    hdr->n_gauss = (int)acc;
    hdr->err = err;
}

// Image Gaussians, skipping everything when the plan failed and rejecting
// radius bins outside [0, n_radii) (a rejected Gaussian gets a box that culls it).
__global__ void noalloc_gaussians(PatchView pv, const fpho_source *src, float *gtab,
                                  float4 *gbox, Header *hdr) {
    if (hdr->err) return;
    const int e = blockIdx.y;
    const int g0 = pv.gauss_start[e];
    const int n = pv.gauss_start[e + 1] - g0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int npsf = pv.exp_npsf[e];
    const int s = i / npsf, p = i - s * npsf;
    const int k = pv.psfgauss[pv.psfgauss_start[e] + p].sersic_radius_bin;
    if (k < 0 || k >= pv.n_radii) {
        atomicOr(&hdr->err, NA_ERR_PSF);
        float *rec = gtab + (size_t)(g0 + i) * GREC;
        for (int f = 0; f < GREC; ++f) rec[f] = 0.0f;
        gbox[g0 + i] = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
        return;
    }
    build_one_gaussian(pv, src, e, s, p, gtab + (size_t)(g0 + i) * GREC, gbox + g0 + i);
}

__global__ void __launch_bounds__(NA_THREADS) noalloc_tiles(TileArgs A, const Header *hdr) {
    if ((int)blockIdx.x >= hdr->n_tiles) return;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    tile_body<NA_THREADS, NA_K>(A, blockIdx.x, smem, &mbar, phase);
}

// Last kernel of a call: the status word, and NaN in every chi2 entry when
// any kernel of the call reported an error (a plan that failed leaves the
// band sums at zero, which would otherwise read as a valid chi2).
__global__ void noalloc_finish(const Header *hdr, int *dev_status, double *chi2, int n_bands) {
    const int err = hdr->err;
    if (threadIdx.x == 0 && dev_status) *dev_status = err;
    if (err)
        for (int b = threadIdx.x; b < n_bands; b += blockDim.x)
            chi2[b] = __longlong_as_double(0x7ff8000000000000ll);  // quiet NaN
}

std::mutex g_setup_mu;
void *g_scratch_ptr[64];  // device address of the scratch array, per device
int g_max_dyn_smem[64];   // dynamic shared memory the tile kernel was allowed, per device

}  // namespace
}  // namespace fpho

using namespace fpho;

extern "C" int fpho_evaluate_proposal_noalloc(const fpho_patch_struct *patch, int n_bands,
                                              int n_exp, int64_t total_pixels,
                                              int max_psf_per_source,
                                              const fpho_source *dev_proposal, double *dev_chi2,
                                              float *dev_dchi2, int dchi2_stride,
                                              int *dev_status, void *stream) {
    clear_error();
    if (!patch || !dev_proposal || !dev_chi2 || !dev_dchi2)
        return set_error(FPHO_ERR_INVALID, "NULL argument");
    const fpho_patch_struct &h = *patch;
    if (!h.data || !h.ierr || !h.xpix || !h.ypix || !h.exposure_start || !h.exposure_N ||
        !h.band_start || !h.band_N || !h.rad2 || !h.D || !h.crpix || !h.crval || !h.CW || !h.G ||
        !h.n_psf_per_source || !h.psfgauss || !h.psfgauss_start)
        return set_error(FPHO_ERR_INVALID, "a device array pointer of the patch is NULL");
    const int nsrc = h.n_sources;
    if (n_bands < 1 || n_bands > FPHO_MAXBANDS)
        return set_error(FPHO_ERR_LIMIT, "n_bands=%d outside [1, %d]", n_bands, FPHO_MAXBANDS);
    if (n_exp < 1 || n_exp > 65535)
        return set_error(FPHO_ERR_LIMIT, "n_exp=%d outside [1, 65535]", n_exp);
    if (nsrc < 1 || nsrc > FPHO_MAX_ACTIVE_SOURCES)
        return set_error(FPHO_ERR_LIMIT, "n_sources=%d outside [1, %d]", nsrc,
                         FPHO_MAX_ACTIVE_SOURCES);
    if (h.n_radii < 1 || h.n_radii > FPHO_MAXRADII)
        return set_error(FPHO_ERR_LIMIT, "n_radii=%d outside [1, %d]", h.n_radii, FPHO_MAXRADII);
    if (max_psf_per_source < 1 || max_psf_per_source > FPHO_MAX_PSF_PER_SOURCE)
        return set_error(FPHO_ERR_LIMIT, "max_psf_per_source=%d outside [1, %d]",
                         max_psf_per_source, FPHO_MAX_PSF_PER_SOURCE);
    if (total_pixels < 0 || total_pixels > (int64_t)INT32_MAX)
        return set_error(FPHO_ERR_LIMIT, "total_pixels=%lld outside [0, 2^31)",
                         (long long)total_pixels);
    if (dchi2_stride < 7 * nsrc)
        return set_error(FPHO_ERR_INVALID, "dchi2_stride=%d < 7*n_sources=%d", dchi2_stride,
                         7 * nsrc);

    const long long n_tiles_max = (total_pixels + NA_TILE - 1) / NA_TILE + n_exp;
    const long long n_gauss_max = (long long)n_exp * nsrc * max_psf_per_source;
    const Layout L = make_layout(n_bands, n_exp, n_tiles_max, n_gauss_max, nsrc);
    if (L.total > (size_t)FPHO_NOALLOC_SCRATCH_BYTES || n_gauss_max > (long long)INT32_MAX / 2)
        return set_error(FPHO_ERR_LIMIT,
                         "patch needs %zu bytes of scratch (%lld tiles, %lld image Gaussians); "
                         "the no-allocation entry point has %u",
                         L.total, n_tiles_max, n_gauss_max, (unsigned)FPHO_NOALLOC_SCRATCH_BYTES);
    const int stride = 7 * nsrc;
    const int idx_cap = nsrc * max_psf_per_source;
    const size_t smem = tile_smem_layout_bytes(NA_THREADS / 32, NA_LIVE_CAP, idx_cap, stride);
    if (smem > 227 * 1024)
        return set_error(FPHO_ERR_LIMIT, "shared memory %zu for %d image Gaussians per exposure "
                         "exceeds 227 KB", smem, idx_cap);

    // once per device (the device current for this call): the array's device
    // address, and the tile kernel's dynamic shared-memory limit raised to the
    // device's ceiling at once, so that later calls never touch kernel attributes
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return set_error(FPHO_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(ce));
    if (dev < 0 || dev >= 64) return set_error(FPHO_ERR_LIMIT, "device index %d >= 64", dev);
    unsigned char *base;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_ptr[dev]) {
            // the ceiling: the device's opt-in shared memory per block less
            // the kernel's static shared memory
            int optin = 0;
            cudaFuncAttributes fa;
            ce = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            if (ce == cudaSuccess) ce = cudaFuncGetAttributes(&fa, (const void *)noalloc_tiles);
            if (ce != cudaSuccess)
                return set_error(FPHO_ERR_CUDA, "shared-memory limits: %s", cudaGetErrorString(ce));
            const int max_dyn = optin - (int)fa.sharedSizeBytes;
            ce = cudaFuncSetAttribute((const void *)noalloc_tiles,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn);
            if (ce != cudaSuccess)
                return set_error(FPHO_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(ce));
            g_max_dyn_smem[dev] = max_dyn;
            void *ptr = nullptr;
            ce = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (ce != cudaSuccess || !ptr)
                return set_error(FPHO_ERR_CUDA, "cudaGetSymbolAddress of the scratch array: %s",
                                 cudaGetErrorString(ce));
            g_scratch_ptr[dev] = ptr;
        }
        base = (unsigned char *)g_scratch_ptr[dev];
        if (smem > (size_t)g_max_dyn_smem[dev])
            return set_error(FPHO_ERR_LIMIT, "shared memory %zu for %d image Gaussians per "
                             "exposure exceeds the %d bytes a block may use", smem, idx_cap,
                             g_max_dyn_smem[dev]);
    }
    Header *hdr = (Header *)(base + L.hdr);
    int *exp_band = (int *)(base + L.exp_band);
    int *exp_npsf = (int *)(base + L.exp_npsf);
    int *gauss_start = (int *)(base + L.gauss_start);
    int *tile_band_start = (int *)(base + L.tile_band_start);
    TileDesc *tiles = (TileDesc *)(base + L.tiles);
    float4 *tbox_all = (float4 *)(base + L.tbox_all);
    float4 *tbox_w = (float4 *)(base + L.tbox_w);
    float *gtab = (float *)(base + L.gtab);
    float4 *gbox = (float4 *)(base + L.gbox);
    double *pchi2 = (double *)(base + L.pchi2);
    float *pgrad = (float *)(base + L.pgrad);

    cudaStream_t s = (cudaStream_t)stream;
    noalloc_plan<<<1, 32, 0, s>>>(h.band_start, h.band_N, h.exposure_start, h.exposure_N,
                                  h.n_psf_per_source, h.psfgauss_start, (long long)total_pixels,
                                  n_bands, n_exp, nsrc, max_psf_per_source,
                                  (int)n_tiles_max, (int)n_gauss_max, hdr, exp_band, exp_npsf,
                                  gauss_start, tile_band_start, tiles);
    PatchView pv;
    pv.data = h.data; pv.ierr = h.ierr; pv.xpix = h.xpix; pv.ypix = h.ypix;
    pv.residual = h.residual;
    pv.rad2 = h.rad2; pv.D = h.D; pv.crpix = h.crpix; pv.crval = h.crval; pv.CW = h.CW;
    pv.G = h.G; pv.psfgauss = h.psfgauss; pv.psfgauss_start = h.psfgauss_start;
    pv.exp_band = exp_band; pv.exp_npsf = exp_npsf; pv.gauss_start = gauss_start;
    pv.n_sources = nsrc; pv.n_exp = n_exp; pv.n_bands = n_bands; pv.n_radii = h.n_radii;
    const int per_exp = nsrc * max_psf_per_source;
    noalloc_gaussians<<<dim3((per_exp + 127) / 128, n_exp), 128, 0, s>>>(pv, dev_proposal, gtab,
                                                                         gbox, hdr);
    tile_bboxes<<<(unsigned)n_tiles_max, 128, 0, s>>>(pv, tiles, tbox_all, tbox_w,
                                                      &hdr->n_tiles);
    TileArgs A;
    A.pv = pv;
    A.tiles = tiles;
    A.tbox_all = tbox_all;
    A.tbox_w = tbox_w;
    A.gtab = gtab;
    A.gbox = gbox;
    A.pchi2 = pchi2;
    A.pgrad = pgrad;
    A.pgrad_stride = stride;
    A.want_residual = h.residual != nullptr;
    A.live_cap = NA_LIVE_CAP;
    A.idx_cap = idx_cap;
    A.err = &hdr->err;
    A.pairs = nullptr;
    noalloc_tiles<<<(unsigned)n_tiles_max, NA_THREADS, smem, s>>>(A, hdr);
    reduce_bands<<<dim3(n_bands, (dchi2_stride + REDUCE_WARPS - 1) / REDUCE_WARPS),
                   32 * REDUCE_WARPS, 0, s>>>(
        tile_band_start, pchi2, pgrad, stride, dev_chi2, dev_dchi2, dchi2_stride);
    noalloc_finish<<<1, 32, 0, s>>>(hdr, dev_status, dev_chi2, n_bands);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return set_error(FPHO_ERR_CUDA, "launch: %s", cudaGetErrorString(ce));
    return FPHO_OK;
}
