// fpho_eval.cu -- patch handles and single-patch evaluation behind the C ABI
// of include/fpho.h.
//
// Per evaluation, three kernels run on the caller's stream:
//   build_image_gaussians  one thread per image Gaussian (exposure, source, PSF
//                          component): record + culling box into the workspace;
//   tile_kernel<NT,K>      one CTA per pixel tile (fpho_tile.cuh);
//   reduce_bands           FP64 sum of the tile partials of each band.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "fpho_impl.cuh"
#include "fpho_handle.h"
#include "fpho_internal.h"
#include "fpho_kernels.cuh"
#include "fpho_tile.cuh"

using namespace fpho;

// ======================================================================= errors
namespace fpho {
static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}
void clear_error() { g_last_error.clear(); }
}  // namespace fpho

#define CUDA_TRY(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return set_error(FPHO_ERR_CUDA, "%s failed: %s (%s:%d)", #call,             \
                             cudaGetErrorString(e_), __FILE__, __LINE__);               \
    } while (0)

extern "C" const char *fpho_last_error(void) { return fpho::g_last_error.c_str(); }
extern "C" int fpho_abi_version(void) { return (1 << 16) | 0; }
extern "C" int fpho_sizeof(int which) {
    switch (which) {
        case 0: return (int)sizeof(fpho_patch_struct);
        case 1: return (int)sizeof(fpho_source);
        case 2: return (int)sizeof(fpho_psfgauss);
        case 3: return (int)sizeof(fpho_response);
        default: return -1;
    }
}

// ======================================================================= kernels
namespace fpho {

template <int NT, int K, bool GRAD, bool EXACT = false>
__global__ void __launch_bounds__(NT) tile_kernel(TileArgs A) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    tile_body<NT, K, GRAD, EXACT>(A, blockIdx.x, smem, &mbar, phase);
}

// Persistent form: each CTA takes tiles from `order` through an atomic counter
// (reset with the ordering, order_tiles_body) until the list is exhausted, so
// the most expensive tiles start first and the cheap ones fill the gaps at
// the end.  The counter
// only hands out indices; no CTA waits on another.
template <int NT, int K, bool GRAD, bool EXACT = false>
__global__ void __launch_bounds__(NT) tile_kernel_dyn(TileArgs A, const int *order, int n_tiles,
                                                      int *counter) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar;
    __shared__ int s_item;
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_tiles) break;
        tile_body<NT, K, GRAD, EXACT>(A, order[item], smem, &mbar, phase);
        __syncthreads();
    }
}

// Unit-flux model rows of the design matrix, one CTA per tile.
template <int NT, int K>
__global__ void __launch_bounds__(NT) design_kernel(TileArgs A, float *X, long long npix) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    design_body<NT, K>(A, blockIdx.x, smem, &mbar, phase, X, npix);
}

// Split tiles (tile_body_split): NW warps share each tile's Gaussians, K
// pixels per thread, 32 K pixels per tile.  MINB asks the compiler for at
// least MINB resident CTAs per SM, a register cap of 64K / (32 NW MINB); the
// default, 16 / NW, caps at 128 registers a thread (left free, the compiler
// takes up to 180 and halves the resident warps).
template <int NW, int K, bool GRAD, int MINB = 16 / NW>
__global__ void __launch_bounds__(32 * NW, MINB) split_kernel(TileArgs A) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    tile_body_split<NW, K, GRAD>(A, blockIdx.x, smem, &mbar, phase);
}

template <int NW, int K, bool GRAD, int MINB = 16 / NW>
__global__ void __launch_bounds__(32 * NW, MINB) split_kernel_dyn(TileArgs A, const int *order,
                                                                  int n_tiles, int *counter) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar;
    __shared__ int s_item;
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_tiles) break;
        tile_body_split<NW, K, GRAD>(A, order[item], smem, &mbar, phase);
        __syncthreads();
    }
}

// ------------------------------------------------------------ variants
// Kernel kinds of a variant: chi2 only, chi2 + gradient, and chi2 + gradient
// with the residual pass in the reference's float arithmetic (the
// exact-residual mode; compiled for the default 64x4 tile only).
enum { KIND_CHI2 = 0, KIND_GRAD = 1, KIND_EXACT = 2, N_KINDS = 3 };
struct Variant {
    int nt;                    // threads per CTA
    int tile;                  // pixels per tile
    int split;                 // 0: tile_body (every thread its own pixels); NW: tile_body_split
    const void *fn[N_KINDS];   // one CTA per tile, by kind (nullptr: not compiled)
    const void *dyn[N_KINDS];  // persistent forms of the same
    const void *design;        // design-matrix rows over tiles of the same size
    int design_nt;             // its threads per CTA
};
#define FPHO_VARIANT(NT, K)                                                                      \
    {NT, NT * K, 0,                                                                              \
     {(const void *)tile_kernel<NT, K, false>, (const void *)tile_kernel<NT, K, true>, nullptr}, \
     {(const void *)tile_kernel_dyn<NT, K, false>, (const void *)tile_kernel_dyn<NT, K, true>,  \
      nullptr},                                                                                  \
     (const void *)design_kernel<NT, K>, NT}
#define FPHO_VARIANT_EXACT(NT, K)                                                                \
    {NT, NT * K, 0,                                                                              \
     {(const void *)tile_kernel<NT, K, false>, (const void *)tile_kernel<NT, K, true>,           \
      (const void *)tile_kernel<NT, K, true, true>},                                             \
     {(const void *)tile_kernel_dyn<NT, K, false>, (const void *)tile_kernel_dyn<NT, K, true>,  \
      (const void *)tile_kernel_dyn<NT, K, true, true>},                                         \
     (const void *)design_kernel<NT, K>, NT}
// DNT x DK: the design kernel's shape over the same 32 K pixel tiles
#define FPHO_SPLIT(NW, K, DNT, DK)                                                               \
    {32 * NW, 32 * K, NW,                                                                        \
     {(const void *)split_kernel<NW, K, false>, (const void *)split_kernel<NW, K, true>,         \
      nullptr},                                                                                  \
     {(const void *)split_kernel_dyn<NW, K, false>, (const void *)split_kernel_dyn<NW, K, true>, \
      nullptr},                                                                                  \
     (const void *)design_kernel<DNT, DK>, DNT}
#define FPHO_SPLIT_MINB(NW, K, MINB, DNT, DK)                                                    \
    {32 * NW, 32 * K, NW,                                                                        \
     {(const void *)split_kernel<NW, K, false, MINB>, (const void *)split_kernel<NW, K, true, MINB>, \
      nullptr},                                                                                  \
     {(const void *)split_kernel_dyn<NW, K, false, MINB>,                                        \
      (const void *)split_kernel_dyn<NW, K, true, MINB>, nullptr},                               \
     (const void *)design_kernel<DNT, DK>, DNT}
// Indices are part of the tuning interface (fpho_patch_set_config): new
// shapes are appended.
static const Variant kVariants[] = {
    FPHO_VARIANT(128, 4), FPHO_VARIANT(128, 2), FPHO_VARIANT(256, 2), FPHO_VARIANT_EXACT(64, 4),
    FPHO_VARIANT(256, 4), FPHO_VARIANT(128, 8), FPHO_VARIANT(64, 8), FPHO_VARIANT(32, 8),
    FPHO_SPLIT(4, 8, 64, 4), FPHO_SPLIT(2, 8, 64, 4), FPHO_SPLIT(8, 8, 64, 4),
    FPHO_SPLIT(4, 4, 32, 4), FPHO_SPLIT_MINB(4, 8, 5, 64, 4),
    FPHO_SPLIT_MINB(4, 6, 5, 32, 6),  // 192-pixel tiles, 95 registers: 5 CTAs per SM
};
#undef FPHO_VARIANT
#undef FPHO_VARIANT_EXACT
#undef FPHO_SPLIT
#undef FPHO_SPLIT_MINB
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

int variant_count() { return kNumVariants; }
bool variant_has_exact(int v) { return kVariants[v].fn[KIND_EXACT] != nullptr; }
int variant_tile_pixels(int v) { return kVariants[v].tile; }
int variant_threads(int v) { return kVariants[v].nt; }
int variant_split(int v) { return kVariants[v].split; }

static std::mutex g_attr_mu;
// per device, variant, kernel kind, form: the dynamic shared memory the
// attribute allows, and for the persistent form the resident CTAs per SM and
// the SM count at that size
static size_t g_attr_set[64][kNumVariants][N_KINDS][2];
static int g_occ[64][kNumVariants][N_KINDS], g_sms[64];
static size_t g_occ_smem[64][kNumVariants][N_KINDS];

static int prepare_fn(const void *fn, int dev, int variant, int kind, int form, size_t smem) {
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (dev < 64 && g_attr_set[dev][variant][kind][form] < smem) {
        CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        g_attr_set[dev][variant][kind][form] = smem;
    }
    return FPHO_OK;
}

int device_sms() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (!g_sms[dev] &&
        cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 148;
    return g_sms[dev];
}

int launch_tile_kernel(int variant, const TileArgs &A, int n_tiles, cudaStream_t stream,
                       bool grad, const int *order, int *counter, bool exact) {
    if (n_tiles <= 0) return FPHO_OK;
    const Variant &V = kVariants[variant];
    const bool dyn = order && counter;
    const int kind = exact ? KIND_EXACT : (grad ? KIND_GRAD : KIND_CHI2);
    const void *fn = dyn ? V.dyn[kind] : V.fn[kind];
    if (!fn)
        return set_error(FPHO_ERR_STATE, "the exact-residual kernel is not compiled for the "
                         "%d-thread, %d-pixel tile", V.nt, V.tile);
    const size_t smem = tile_smem_bytes(variant, A.live_cap, A.idx_cap, A.pgrad_stride);
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64) return set_error(FPHO_ERR_LIMIT, "device ordinal %d >= 64", dev);
    int rc = prepare_fn(fn, dev, variant, kind, dyn ? 1 : 0, smem);
    if (rc) return rc;
    if (!dyn) {
        void *args[] = {(void *)&A};
        CUDA_TRY(cudaLaunchKernel(fn, dim3(n_tiles), dim3(V.nt), args, smem, stream));
        return FPHO_OK;
    }
    int occ = 0, sms = 0;
    {
        std::lock_guard<std::mutex> lk(g_attr_mu);
        if (g_occ_smem[dev][variant][kind] != smem || g_occ[dev][variant][kind] == 0) {
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_occ[dev][variant][kind], fn,
                                                                   V.nt, smem));
            g_occ_smem[dev][variant][kind] = smem;
            if (!g_sms[dev])
                CUDA_TRY(cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev));
        }
        occ = g_occ[dev][variant][kind];
        sms = g_sms[dev];
    }
    if (occ < 1) return set_error(FPHO_ERR_LIMIT, "tile kernel cannot be resident (smem %zu)", smem);
    const int grid = std::min(n_tiles, occ * sms);
    void *args[] = {(void *)&A, (void *)&order, (void *)&n_tiles, (void *)&counter};
    CUDA_TRY(cudaLaunchKernel(fn, dim3(grid), dim3(V.nt), args, smem, stream));
    return FPHO_OK;
}

static std::mutex g_design_mu;
static size_t g_design_set[64][kNumVariants];

int launch_design_kernel(int variant, const TileArgs &A_in, int n_tiles, float *X, long long npix,
                         cudaStream_t stream) {
    if (n_tiles <= 0) return FPHO_OK;
    const Variant &V = kVariants[variant];
    TileArgs A = A_in;
    A.live_cap = std::min(A.live_cap, DESIGN_LIVE_CAP);
    const size_t smem =
        tile_smem_layout_bytes(V.design_nt / 32, A.live_cap, A.idx_cap, A.pgrad_stride);
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64) return set_error(FPHO_ERR_LIMIT, "device ordinal %d >= 64", dev);
    {
        std::lock_guard<std::mutex> lk(g_design_mu);
        if (g_design_set[dev][variant] < smem) {
            CUDA_TRY(cudaFuncSetAttribute(V.design, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
            g_design_set[dev][variant] = smem;
        }
    }
    void *args[] = {(void *)&A, (void *)&X, (void *)&npix};
    CUDA_TRY(cudaLaunchKernel(V.design, dim3(n_tiles), dim3(V.design_nt), args, smem, stream));
    return FPHO_OK;
}

size_t tile_smem_bytes(int variant, int live_cap, int idx_cap, int stride) {
    const Variant &V = kVariants[variant];
    if (V.split)
        return split_smem_layout_bytes(V.split, V.tile / 32, live_cap, idx_cap, stride);
    return tile_smem_layout_bytes(V.nt / 32, live_cap, idx_cap, stride);
}

}  // namespace fpho

// ======================================================================= handle
// struct fpho_patch is defined in fpho_handle.h

static void destroy_patch(fpho_patch *p);

namespace {

template <typename T>
int dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = fpho::pool_malloc((void **)p, n * sizeof(T));
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
template <typename T>
int dupload(T **dst, const T *src, size_t n, cudaStream_t s,
            cudaMemcpyKind kind = cudaMemcpyHostToDevice) {
    int rc = dalloc(dst, n);
    if (rc) return rc;
    if (n) CUDA_TRY(cudaMemcpyAsync(*dst, src, n * sizeof(T), kind, s));
    return FPHO_OK;
}

void free_meta(fpho_patch *p) {
    dfree(p->d_rad2); dfree(p->d_D); dfree(p->d_crpix); dfree(p->d_crval); dfree(p->d_CW);
    dfree(p->d_G); dfree(p->d_npsf); dfree(p->d_psfgauss_start); dfree(p->d_psfgauss);
    dfree(p->d_exp_band); dfree(p->d_exp_npsf); dfree(p->d_gauss_start);
    dfree(p->d_gtab); dfree(p->d_gbox); dfree(p->d_prop);
}
void free_plan(fpho_patch *p) {
    dfree(p->d_tiles); dfree(p->d_tbox_all); dfree(p->d_tbox_w); dfree(p->d_tile_band_start);
    dfree(p->d_pchi2); dfree(p->d_pgrad);
    dfree(p->d_tile_cost); dfree(p->d_tile_order); dfree(p->d_tile_counter);
}

// Validate the index arrays of a host patch description and fill host copies.
int read_pixel_index(fpho_patch *p, const fpho_patch_struct *h, int n_bands) {
    if (!h) return set_error(FPHO_ERR_INVALID, "patch description is NULL");
    if (n_bands < 1 || n_bands > FPHO_MAXBANDS)
        return set_error(FPHO_ERR_LIMIT, "n_bands=%d outside [1, %d]", n_bands, FPHO_MAXBANDS);
    if (!h->data || !h->ierr || !h->xpix || !h->ypix || !h->exposure_start || !h->exposure_N ||
        !h->band_start || !h->band_N)
        return set_error(FPHO_ERR_INVALID, "a pixel or index array pointer is NULL");
    p->n_bands = n_bands;
    p->band_start.assign(h->band_start, h->band_start + n_bands);
    p->band_N.assign(h->band_N, h->band_N + n_bands);
    int n_exp = 0;
    for (int b = 0; b < n_bands; ++b) {
        if (p->band_start[b] < 0 || p->band_N[b] < 0)
            return set_error(FPHO_ERR_INVALID, "band %d: negative band_start/band_N", b);
        n_exp = std::max(n_exp, (int)p->band_start[b] + (int)p->band_N[b]);
    }
    if (n_exp < 1) return set_error(FPHO_ERR_INVALID, "patch has no exposures");
    if (n_exp > 65535)  // exposures index gridDim.y of the image-Gaussian kernel
        return set_error(FPHO_ERR_LIMIT, "n_exp=%d exceeds 65535", n_exp);
    p->n_exp = n_exp;
    p->exposure_start.assign(h->exposure_start, h->exposure_start + n_exp);
    p->exposure_N.assign(h->exposure_N, h->exposure_N + n_exp);
    p->exp_band.assign(n_exp, -1);
    for (int b = 0; b < n_bands; ++b)
        for (int e = p->band_start[b]; e < p->band_start[b] + p->band_N[b]; ++e) {
            if (p->exp_band[e] != -1)
                return set_error(FPHO_ERR_INVALID, "exposure %d belongs to bands %d and %d", e,
                                 p->exp_band[e], b);
            p->exp_band[e] = b;
        }
    int64_t npix = 0;
    for (int e = 0; e < n_exp; ++e) {
        if (p->exposure_start[e] < 0 || p->exposure_N[e] < 0)
            return set_error(FPHO_ERR_INVALID, "exposure %d: negative exposure_start/N", e);
        npix = std::max<int64_t>(npix, (int64_t)p->exposure_start[e] + p->exposure_N[e]);
    }
    if (npix > (int64_t)INT32_MAX) return set_error(FPHO_ERR_LIMIT, "npix exceeds 2^31-1");
    p->npix = npix;
    return FPHO_OK;
}

// Validate and upload the per-scene metadata; derive the image-Gaussian index.
int upload_meta(fpho_patch *p, const fpho_patch_struct *h, cudaStream_t s,
                bool validate_only = false) {
    if (!h->rad2 || !h->D || !h->crpix || !h->crval || !h->CW || !h->G || !h->n_psf_per_source ||
        !h->psfgauss || !h->psfgauss_start)
        return set_error(FPHO_ERR_INVALID, "a metadata array pointer is NULL");
    const int nsrc = h->n_sources, nrad = h->n_radii;
    if (nsrc < 1 || nsrc > FPHO_MAX_ACTIVE_SOURCES)
        return set_error(FPHO_ERR_LIMIT, "n_sources=%d outside [1, %d]", nsrc,
                         FPHO_MAX_ACTIVE_SOURCES);
    if (nrad < 1 || nrad > FPHO_MAXRADII)
        return set_error(FPHO_ERR_LIMIT, "n_radii=%d outside [1, %d]", nrad, FPHO_MAXRADII);
    const int nb = p->n_bands, ne = p->n_exp;
    std::vector<int> npsf(h->n_psf_per_source, h->n_psf_per_source + nb);
    for (int b = 0; b < nb; ++b)
        if (npsf[b] < 0 || npsf[b] > FPHO_MAX_PSF_PER_SOURCE)
            return set_error(FPHO_ERR_LIMIT, "band %d: n_psf_per_source=%d outside [0, %d]", b,
                             npsf[b], FPHO_MAX_PSF_PER_SOURCE);
    std::vector<int> pstart(h->psfgauss_start, h->psfgauss_start + ne);
    std::vector<int> exp_npsf(ne, 0), gstart(ne + 1, 0);
    int64_t nrows = 0, ng = 0;
    for (int e = 0; e < ne; ++e) {
        const int b = p->exp_band[e];
        exp_npsf[e] = (b >= 0) ? npsf[b] : 0;
        if (exp_npsf[e] > 0) {
            if (pstart[e] < 0) return set_error(FPHO_ERR_INVALID, "psfgauss_start[%d] < 0", e);
            nrows = std::max<int64_t>(nrows, (int64_t)pstart[e] + exp_npsf[e]);
        }
        gstart[e] = (int)ng;
        ng += (int64_t)nsrc * exp_npsf[e];
        if (ng > (int64_t)INT32_MAX / 2)
            return set_error(FPHO_ERR_LIMIT, "too many image Gaussians");
    }
    gstart[ne] = (int)ng;
    for (int e = 0; e < ne; ++e)
        for (int q = 0; q < exp_npsf[e]; ++q) {
            const int k = h->psfgauss[pstart[e] + q].sersic_radius_bin;
            if (k < 0 || k >= nrad)
                return set_error(FPHO_ERR_INVALID,
                                 "psfgauss[%d].sersic_radius_bin=%d outside [0, n_radii=%d)",
                                 pstart[e] + q, k, nrad);
        }
    {
        int mg = 0;
        for (int e = 0; e < ne; ++e) mg = std::max(mg, gstart[e + 1] - gstart[e]);
        const size_t need = tile_smem_bytes(p->variant, p->live_cap, std::max(mg, 1), 7 * nsrc);
        if (need > 227 * 1024)
            return set_error(FPHO_ERR_LIMIT,
                             "%d image Gaussians per exposure and %d sources need %zu bytes of "
                             "shared memory (max 227 KB)", mg, nsrc, need);
    }
    if (validate_only) return FPHO_OK;
    free_meta(p);
    p->n_sources = nsrc;
    p->n_radii = nrad;
    p->n_psf_per_source = npsf;
    p->psfgauss_start = pstart;
    p->exp_npsf = exp_npsf;
    p->gauss_start = gstart;
    p->n_gauss = (int)ng;
    p->max_g = 0;
    for (int e = 0; e < ne; ++e) p->max_g = std::max(p->max_g, gstart[e + 1] - gstart[e]);
    p->n_psfrows = nrows;
    const size_t es = (size_t)ne * nsrc;
    int rc;
    if ((rc = dupload(&p->d_rad2, h->rad2, nrad, s))) return rc;
    if ((rc = dupload(&p->d_D, h->D, es * 4, s))) return rc;
    if ((rc = dupload(&p->d_CW, h->CW, es * 4, s))) return rc;
    if ((rc = dupload(&p->d_crpix, h->crpix, es * 2, s))) return rc;
    if ((rc = dupload(&p->d_crval, h->crval, es * 2, s))) return rc;
    if ((rc = dupload(&p->d_G, h->G, (size_t)ne, s))) return rc;
    if ((rc = dupload(&p->d_npsf, npsf.data(), (size_t)nb, s))) return rc;
    if ((rc = dupload(&p->d_psfgauss_start, pstart.data(), (size_t)ne, s))) return rc;
    if ((rc = dupload(&p->d_psfgauss, h->psfgauss, (size_t)nrows, s))) return rc;
    if ((rc = dupload(&p->d_exp_band, p->exp_band.data(), (size_t)ne, s))) return rc;
    if ((rc = dupload(&p->d_exp_npsf, exp_npsf.data(), (size_t)ne, s))) return rc;
    if ((rc = dupload(&p->d_gauss_start, gstart.data(), (size_t)ne + 1, s))) return rc;
    if ((rc = dalloc(&p->d_gtab, (size_t)ng * GREC))) return rc;
    if ((rc = dalloc(&p->d_gbox, (size_t)ng))) return rc;
    if ((rc = dalloc(&p->d_prop, (size_t)nsrc))) return rc;
    // metadata arrays are read from host memory by the async copies above
    CUDA_TRY(cudaStreamSynchronize(s));
    return FPHO_OK;
}

int build_plan(fpho_patch *p, cudaStream_t s);

int refresh_struct(fpho_patch *p, cudaStream_t s) {
    fpho_patch_struct hs;
    memset(&hs, 0, sizeof(hs));
    hs.data = p->d_data; hs.ierr = p->d_ierr; hs.xpix = p->d_xpix; hs.ypix = p->d_ypix;
    hs.residual = p->d_residual;
    hs.exposure_start = p->d_exposure_start; hs.exposure_N = p->d_exposure_N;
    hs.band_start = p->d_band_start; hs.band_N = p->d_band_N;
    hs.n_sources = p->n_sources; hs.n_radii = p->n_radii;
    hs.rad2 = p->d_rad2; hs.D = p->d_D; hs.crpix = p->d_crpix; hs.crval = p->d_crval;
    hs.CW = p->d_CW; hs.G = p->d_G; hs.n_psf_per_source = p->d_npsf;
    hs.psfgauss = p->d_psfgauss; hs.psfgauss_start = p->d_psfgauss_start;
    if (!p->d_struct) {
        int rc = dalloc(&p->d_struct, 1);
        if (rc) return rc;
    }
    CUDA_TRY(cudaMemcpyAsync(p->d_struct, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return FPHO_OK;
}

}  // namespace

namespace fpho {

cudaError_t pool_malloc(void **p, size_t bytes) {
    static std::once_flag once[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64)
        std::call_once(once[dev], [dev] {
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t keep = UINT64_MAX;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
        });
    e = cudaMallocAsync(p, bytes, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    return e;
}

void pool_free(void *p) {
    if (!p) return;
    cudaDeviceSynchronize();
    cudaFreeAsync(p, 0);
}

PatchView make_view(const fpho_patch *p) {
    PatchView v;
    v.data = p->d_data; v.ierr = p->d_ierr; v.xpix = p->d_xpix; v.ypix = p->d_ypix;
    v.residual = p->d_residual;
    v.rad2 = p->d_rad2; v.D = p->d_D; v.crpix = p->d_crpix; v.crval = p->d_crval;
    v.CW = p->d_CW; v.G = p->d_G;
    v.psfgauss = p->d_psfgauss; v.psfgauss_start = p->d_psfgauss_start;
    v.exp_band = p->d_exp_band; v.exp_npsf = p->d_exp_npsf; v.gauss_start = p->d_gauss_start;
    v.n_sources = p->n_sources; v.n_exp = p->n_exp; v.n_bands = p->n_bands;
    v.n_radii = p->n_radii;
    return v;
}

}  // namespace fpho

namespace {

int build_plan(fpho_patch *p, cudaStream_t s) {
    free_plan(p);
    const int tp = variant_tile_pixels(p->variant);
    std::vector<TileDesc> tiles;
    p->tile_band_start.assign(p->n_bands + 1, 0);
    for (int b = 0; b < p->n_bands; ++b) {
        p->tile_band_start[b] = (int)tiles.size();
        for (int e = p->band_start[b]; e < p->band_start[b] + p->band_N[b]; ++e) {
            const int n = p->exposure_N[e];
            for (int off = 0; off < n; off += tp)
                tiles.push_back({e, b, p->exposure_start[e] + off, std::min(tp, n - off)});
        }
    }
    p->tile_band_start[p->n_bands] = (int)tiles.size();
    p->n_tiles = (int)tiles.size();
    p->h_tiles = tiles;
    int rc;
    if ((rc = dupload(&p->d_tiles, tiles.data(), tiles.size(), s))) return rc;
    if ((rc = dupload(&p->d_tile_band_start, p->tile_band_start.data(),
                      p->tile_band_start.size(), s)))
        return rc;
    if ((rc = dalloc(&p->d_tbox_all, tiles.size()))) return rc;
    if ((rc = dalloc(&p->d_tbox_w, tiles.size()))) return rc;
    if ((rc = dalloc(&p->d_pchi2, tiles.size()))) return rc;
    if ((rc = dalloc(&p->d_pgrad, tiles.size() * (size_t)7 * p->n_sources))) return rc;
    if ((rc = dalloc(&p->d_tile_cost, tiles.size()))) return rc;
    if ((rc = dalloc(&p->d_tile_order, tiles.size()))) return rc;
    if ((rc = dalloc(&p->d_tile_counter, 1))) return rc;
    CUDA_TRY(cudaMemsetAsync(p->d_tile_cost, 0, sizeof(int) * std::max<size_t>(tiles.size(), 1), s));
    if (p->n_tiles > 0) {
        tile_bboxes<<<p->n_tiles, 128, 0, s>>>(make_view(p), p->d_tiles, p->d_tbox_all,
                                              p->d_tbox_w, nullptr);
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    return FPHO_OK;
}

}  // namespace

// ======================================================================= C ABI
// `pixel_kind`: where host->data, ierr, xpix and ypix live (host or device).
static int create_patch(const fpho_patch_struct *host, int n_bands, int return_residual,
                        void *stream, fpho_patch **out, cudaMemcpyKind pixel_kind) {
    clear_error();
    if (!out) return set_error(FPHO_ERR_INVALID, "out is NULL");
    *out = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    fpho_patch *p = new (std::nothrow) fpho_patch();
    if (!p) return set_error(FPHO_ERR_NOMEM, "host allocation failed");
    int rc = read_pixel_index(p, host, n_bands);
    // every host-side check happens before the first CUDA call
    if (!rc) rc = upload_meta(p, host, s, /*validate_only=*/true);
    if (!rc) {
        const size_t np = (size_t)p->npix;
        if (!rc) rc = dupload(&p->d_data, host->data, np, s, pixel_kind);
        if (!rc) rc = dupload(&p->d_ierr, host->ierr, np, s, pixel_kind);
        if (!rc) rc = dupload(&p->d_xpix, host->xpix, np, s, pixel_kind);
        if (!rc) rc = dupload(&p->d_ypix, host->ypix, np, s, pixel_kind);
        if (!rc) rc = dupload(&p->d_exposure_start, p->exposure_start.data(), (size_t)p->n_exp, s);
        if (!rc) rc = dupload(&p->d_exposure_N, p->exposure_N.data(), (size_t)p->n_exp, s);
        if (!rc) rc = dupload(&p->d_band_start, p->band_start.data(), (size_t)p->n_bands, s);
        if (!rc) rc = dupload(&p->d_band_N, p->band_N.data(), (size_t)p->n_bands, s);
        if (!rc && return_residual) {
            rc = dalloc(&p->d_residual, np);
            if (!rc && cudaMemsetAsync(p->d_residual, 0, np * sizeof(float), s) != cudaSuccess)
                rc = set_error(FPHO_ERR_CUDA, "cudaMemsetAsync failed");
            p->has_residual = true;
        }
    }
    if (!rc) rc = upload_meta(p, host, s);
    if (!rc) rc = dalloc(&p->d_err, 1);
    if (!rc && cudaMemsetAsync(p->d_err, 0, sizeof(int), s) != cudaSuccess)
        rc = set_error(FPHO_ERR_CUDA, "cudaMemsetAsync failed");
    if (!rc) rc = dalloc(&p->d_pairs, 1);
    if (!rc) rc = build_plan(p, s);
    if (!rc) rc = refresh_struct(p, s);
    if (rc) {
        destroy_patch(p);
        return rc;
    }
    *out = p;
    return FPHO_OK;
}

extern "C" int fpho_patch_create(const fpho_patch_struct *host, int n_bands, int return_residual,
                                 void *stream, fpho_patch **out) {
    return create_patch(host, n_bands, return_residual, stream, out, cudaMemcpyHostToDevice);
}

extern "C" int fpho_patch_create_device_pixels(const fpho_patch_struct *desc, int n_bands,
                                               int return_residual, void *stream,
                                               fpho_patch **out) {
    return create_patch(desc, n_bands, return_residual, stream, out, cudaMemcpyDeviceToDevice);
}

extern "C" int fpho_patch_replace_meta(fpho_patch *p, const fpho_patch_struct *host, void *stream) {
    clear_error();
    if (!p || !host) return set_error(FPHO_ERR_INVALID, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int old_nsrc = p->n_sources;
    int rc = upload_meta(p, host, s);
    if (rc) return rc;
    if (p->n_sources != old_nsrc) {
        dfree(p->d_pgrad);
        if ((rc = dalloc(&p->d_pgrad, (size_t)std::max(p->n_tiles, 1) * 7 * p->n_sources)))
            return rc;
    }
    return refresh_struct(p, s);
}

extern "C" int fpho_patch_swap_data_residual(fpho_patch *p, void *stream) {
    clear_error();
    if (!p) return set_error(FPHO_ERR_INVALID, "NULL patch");
    if (!p->has_residual)
        return set_error(FPHO_ERR_STATE, "patch was created without a residual array");
    std::swap(p->d_data, p->d_residual);
    return refresh_struct(p, (cudaStream_t)stream);
}

extern "C" int fpho_patch_retrieve(fpho_patch *p, int which, float *host_out, void *stream) {
    clear_error();
    if (!p || !host_out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    const float *src = nullptr;
    switch (which) {
        case 0: src = p->d_data; break;
        case 1: src = p->d_residual; break;
        case 2: src = p->d_ierr; break;
        case 3: src = p->d_xpix; break;
        case 4: src = p->d_ypix; break;
        default: return set_error(FPHO_ERR_INVALID, "which=%d not in 0..4", which);
    }
    if (!src) return set_error(FPHO_ERR_STATE, "array %d is not allocated", which);
    cudaStream_t s = (cudaStream_t)stream;
    CUDA_TRY(cudaMemcpyAsync(host_out, src, (size_t)p->npix * sizeof(float),
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return FPHO_OK;
}

extern "C" int fpho_patch_device_struct(fpho_patch *p, const void **dev_struct) {
    clear_error();
    if (!p || !dev_struct) return set_error(FPHO_ERR_INVALID, "NULL argument");
    *dev_struct = p->d_struct;
    return FPHO_OK;
}

extern "C" int fpho_patch_info(const fpho_patch *p, int64_t out[7]) {
    clear_error();
    if (!p || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    out[0] = p->n_bands; out[1] = p->n_exp; out[2] = p->npix; out[3] = p->n_sources;
    out[4] = p->n_radii; out[5] = p->n_tiles; out[6] = p->n_gauss;
    return FPHO_OK;
}

static void destroy_patch(fpho_patch *p) {
    free_meta(p);
    free_plan(p);
    dfree(p->d_data); dfree(p->d_ierr); dfree(p->d_xpix); dfree(p->d_ypix); dfree(p->d_residual);
    dfree(p->d_exposure_start); dfree(p->d_exposure_N); dfree(p->d_band_start);
    dfree(p->d_band_N); dfree(p->d_struct); dfree(p->d_io);
    if (p->h_io) cudaFreeHost(p->h_io);
    dfree(p->d_err); dfree(p->d_pairs); dfree(p->d_pnorm); dfree(p->d_atb);
    if (p->ev_tile0) cudaEventDestroy(p->ev_tile0);
    if (p->ev_tile1) cudaEventDestroy(p->ev_tile1);
    delete p;
}

extern "C" int fpho_patch_free(fpho_patch *p) {
    clear_error();
    if (p) destroy_patch(p);
    return FPHO_OK;
}

// ------------------------------------------------------------ tuning hooks
extern "C" int fpho_patch_set_config(fpho_patch *p, int variant, int live_cap, void *stream) {
    clear_error();
    if (!p) return set_error(FPHO_ERR_INVALID, "NULL patch");
    if (variant < 0 || variant >= variant_count())
        return set_error(FPHO_ERR_INVALID, "variant %d not in [0, %d)", variant, variant_count());
    const int nt = variant_threads(variant);
    (void)nt;
    if (live_cap < 32 || live_cap > 4096)
        return set_error(FPHO_ERR_INVALID, "live_cap %d outside [32, 4096]", live_cap);
    if (tile_smem_bytes(variant, live_cap, p->max_g, 7 * p->n_sources) > 227 * 1024)
        return set_error(FPHO_ERR_LIMIT, "shared memory for live_cap %d exceeds 227 KB",
                         live_cap);
    if (p->exact_residual && !variant_has_exact(variant))
        return set_error(FPHO_ERR_STATE, "variant %d has no exact-residual kernel; turn the "
                         "exact-residual mode off first", variant);
    const bool replan = variant_tile_pixels(variant) != variant_tile_pixels(p->variant);
    p->variant = variant;
    p->live_cap = live_cap;
    if (replan) return build_plan(p, (cudaStream_t)stream);
    return FPHO_OK;
}

extern "C" int fpho_patch_set_test_stall(fpho_patch *p, int on) {
    clear_error();
    if (!p) return set_error(FPHO_ERR_INVALID, "NULL patch");
    // one staging per tile only: after a wait that gave up, a second staging
    // on the same barrier could run ahead of its copies
    if (on && p->max_g > p->live_cap)
        return set_error(FPHO_ERR_STATE,
                         "the test stall needs every exposure's %d image Gaussians to fit one "
                         "stage of %d records", p->max_g, p->live_cap);
    if (on && p->schedule == 1 && p->n_tiles > 4 * device_sms())
        return set_error(FPHO_ERR_STATE, "the test stall needs one CTA per tile (schedule 0)");
    p->test_extra_tx = on ? 16 : 0;
    return FPHO_OK;
}

extern "C" int fpho_patch_set_exact_residual(fpho_patch *p, int on) {
    clear_error();
    if (!p) return set_error(FPHO_ERR_INVALID, "NULL patch");
    if (on && !variant_has_exact(p->variant))
        return set_error(FPHO_ERR_STATE, "the exact-residual mode needs a tile variant that "
                         "compiles it (variant 3, 64 threads x 4 pixels); this patch uses %d",
                         p->variant);
    p->exact_residual = on ? 1 : 0;
    return FPHO_OK;
}

extern "C" int fpho_patch_set_schedule(fpho_patch *p, int schedule) {
    clear_error();
    if (!p) return set_error(FPHO_ERR_INVALID, "NULL patch");
    if (schedule != 0 && schedule != 1)
        return set_error(FPHO_ERR_INVALID, "schedule %d is neither 0 nor 1", schedule);
    p->schedule = schedule;
    return FPHO_OK;
}

extern "C" int fpho_variant_info(int variant, int out[2]) {
    clear_error();
    if (variant < 0 || variant >= variant_count() || !out)
        return set_error(FPHO_ERR_INVALID, "bad variant");
    out[0] = variant_threads(variant);
    out[1] = variant_tile_pixels(variant) / variant_threads(variant);
    return variant_count();
}

extern "C" int fpho_variant_shape(int variant, int out[3]) {
    clear_error();
    if (variant < 0 || variant >= variant_count() || !out)
        return set_error(FPHO_ERR_INVALID, "bad variant");
    out[0] = variant_threads(variant);
    out[1] = variant_tile_pixels(variant);
    out[2] = variant_split(variant);
    return variant_count();
}

extern "C" int fpho_patch_count_pairs(fpho_patch *p, int enable, long long *last_count) {
    clear_error();
    if (!p) return set_error(FPHO_ERR_INVALID, "NULL patch");
    p->count_pairs = enable;
    if (last_count) {
        long long v = 0;
        CUDA_TRY(cudaMemcpy(&v, p->d_pairs, sizeof(v), cudaMemcpyDeviceToHost));
        *last_count = v;
    }
    return FPHO_OK;
}

namespace fpho {

// Enqueue one evaluation with device-resident proposal and outputs.
int enqueue_evaluate(fpho_patch *p, const fpho_source *d_prop, double *d_chi2, float *d_dchi2,
                     int out_stride, bool want_residual, cudaStream_t s, bool grad,
                     int *d_err_out = nullptr) {
    if (want_residual && !p->d_residual)
        return set_error(FPHO_ERR_STATE,
                         "residual requested but the patch was created without one");
    if (p->count_pairs) CUDA_TRY(cudaMemsetAsync(p->d_pairs, 0, sizeof(long long), s));
    const PatchView pv = make_view(p);
    // the order only matters when the tiles outnumber what runs at once
    const bool ordered = p->schedule == 1 && p->n_tiles > 4 * device_sms();
    {
        // image Gaussians, the tile order and the error word in one launch
        dim3 grid(std::max((p->max_g + PREP_THREADS - 1) / PREP_THREADS, 1),
                  std::max(p->n_exp + (ordered ? 1 : 0), 1));
        prepare_evaluation<<<grid, PREP_THREADS, 0, s>>>(pv, d_prop, p->d_gtab, p->d_gbox,
                                                p->d_tile_cost, p->n_tiles,
                                                ordered ? p->d_tile_order : nullptr,
                                                p->d_tile_counter, p->d_err);
        CUDA_TRY(cudaGetLastError());
    }
    TileArgs A;
    A.pv = pv;
    A.tiles = p->d_tiles;
    A.tbox_all = p->d_tbox_all;
    A.tbox_w = p->d_tbox_w;
    A.gtab = p->d_gtab;
    A.gbox = p->d_gbox;
    A.pchi2 = p->d_pchi2;
    A.pgrad = p->d_pgrad;
    A.pgrad_stride = 7 * p->n_sources;
    A.want_residual = want_residual ? 1 : 0;
    A.live_cap = p->live_cap;
    A.idx_cap = std::max(p->max_g, 1);
    A.err = p->d_err;
    A.pairs = p->count_pairs ? p->d_pairs : nullptr;
    A.test_extra_tx = p->test_extra_tx;
    if (p->ev_tile0) CUDA_TRY(cudaEventRecord(p->ev_tile0, s));
    int rc;
    if (ordered) {
        A.tile_cost = p->d_tile_cost;
        rc = launch_tile_kernel(p->variant, A, p->n_tiles, s, grad, p->d_tile_order,
                                p->d_tile_counter, p->exact_residual != 0);
    } else {
        rc = launch_tile_kernel(p->variant, A, p->n_tiles, s, grad, nullptr, nullptr,
                                p->exact_residual != 0);
    }
    if (rc) return rc;
    if (p->ev_tile1) CUDA_TRY(cudaEventRecord(p->ev_tile1, s));
    dim3 rg(p->n_bands, grad ? (out_stride + REDUCE_WARPS - 1) / REDUCE_WARPS : 1);
    reduce_bands<<<rg, 32 * REDUCE_WARPS, 0, s>>>(p->d_tile_band_start, p->d_pchi2, p->d_pgrad,
                                    7 * p->n_sources, d_chi2, grad ? d_dchi2 : nullptr,
                                    out_stride, p->d_err, d_err_out);
    CUDA_TRY(cudaGetLastError());
    return FPHO_OK;
}

}  // namespace fpho

extern "C" int fpho_evaluate_proposal(fpho_patch *p, const fpho_source *proposal, int n_sources,
                                      double *chi2, float *dchi2, int dchi2_stride,
                                      unsigned flags, void *stream) {
    clear_error();
    const bool grad = (flags & FPHO_CHI2_ONLY) == 0;
    if (!p || !proposal || !chi2 || (grad && !dchi2))
        return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (!grad) dchi2_stride = 7 * n_sources;
    if (n_sources != p->n_sources)
        return set_error(FPHO_ERR_INVALID, "n_sources=%d but the patch has %d", n_sources,
                         p->n_sources);
    if (dchi2_stride < 7 * n_sources)
        return set_error(FPHO_ERR_INVALID, "dchi2_stride=%d < 7*n_sources=%d", dchi2_stride,
                         7 * n_sources);
    cudaStream_t s = (cudaStream_t)stream;
    const bool host_io = (flags & FPHO_IO_HOST) != 0;
    const bool want_res = (flags & FPHO_WANT_RESIDUAL) != 0;
    if (!host_io)
        return enqueue_evaluate(p, proposal, chi2, dchi2, dchi2_stride, want_res, s, grad);

    // [chi2 (n_bands doubles)][error word, 8 bytes][dchi2]
    const size_t gfloats = (size_t)p->n_bands * dchi2_stride;
    const size_t chi2_bytes = sizeof(double) * p->n_bands;
    const size_t head_bytes = chi2_bytes + 8;
    const size_t io_bytes = head_bytes + sizeof(float) * gfloats;
    if (p->d_io_cap < io_bytes) {
        dfree(p->d_io);
        p->d_io_cap = 0;
        int rc = dalloc(&p->d_io, io_bytes);
        if (rc) return rc;
        p->d_io_cap = io_bytes;
    }
    if (p->h_io_cap < io_bytes) {
        if (p->h_io) cudaFreeHost(p->h_io);
        p->h_io = nullptr;
        p->h_io_cap = 0;
        CUDA_TRY(cudaHostAlloc((void **)&p->h_io, io_bytes, cudaHostAllocDefault));
        p->h_io_cap = io_bytes;
    }
    double *d_chi2 = reinterpret_cast<double *>(p->d_io);
    int *d_err_out = reinterpret_cast<int *>(p->d_io + chi2_bytes);
    float *d_dchi2 = reinterpret_cast<float *>(p->d_io + head_bytes);
    CUDA_TRY(cudaMemcpyAsync(p->d_prop, proposal, sizeof(fpho_source) * n_sources,
                             cudaMemcpyHostToDevice, s));
    int rc = enqueue_evaluate(p, p->d_prop, d_chi2, d_dchi2, dchi2_stride, want_res, s, grad,
                              d_err_out);
    if (rc) return rc;
    // results and error word in one transfer into pinned memory
    CUDA_TRY(cudaMemcpyAsync(p->h_io, p->d_io, grad ? io_bytes : head_bytes,
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    std::memcpy(chi2, p->h_io, chi2_bytes);
    if (grad) std::memcpy(dchi2, p->h_io + head_bytes, sizeof(float) * gfloats);
    int err = 0;
    std::memcpy(&err, p->h_io + chi2_bytes, sizeof(int));
    if (err) return set_error(FPHO_ERR_KERNEL, "tile kernel reported error word 0x%x", err);
    return FPHO_OK;
}

extern "C" int fpho_EvaluateProposal(fpho_patch *p, const void *dev_patch_struct,
                                     const void *dev_proposal, void *pchi2, void *pdchi2_dp,
                                     void *stream) {
    clear_error();
    if (!p || !dev_proposal || !pchi2 || !pdchi2_dp)
        return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (dev_patch_struct != (const void *)p->d_struct)
        return set_error(FPHO_ERR_INVALID,
                         "dev_patch_struct is not the device struct of this patch handle");
    if (p->n_sources > FPHO_MAXSOURCES)
        return set_error(FPHO_ERR_LIMIT,
                         "the Response layout holds %d sources; use fpho_evaluate_proposal",
                         FPHO_MAXSOURCES);
    return enqueue_evaluate(p, (const fpho_source *)dev_proposal, (double *)pchi2,
                            (float *)pdchi2_dp, FPHO_MAXSOURCES * FPHO_NPARAMS,
                            p->d_residual != nullptr, (cudaStream_t)stream, true);
}

extern "C" int fpho_patch_design_matrix(fpho_patch *p, const void *dev_proposal,
                                        int n_sources, float *dev_X, void *stream) {
    clear_error();
    if (!p || !dev_proposal || !dev_X) return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (n_sources != p->n_sources)
        return set_error(FPHO_ERR_INVALID, "n_sources=%d but the patch has %d", n_sources,
                         p->n_sources);
    cudaStream_t s = (cudaStream_t)stream;
    CUDA_TRY(cudaMemsetAsync(dev_X, 0, sizeof(float) * (size_t)n_sources * p->npix, s));
    CUDA_TRY(cudaMemsetAsync(p->d_err, 0, sizeof(int), s));
    const PatchView pv = make_view(p);
    if (p->max_g > 0) {
        dim3 grid((p->max_g + 127) / 128, p->n_exp);
        build_image_gaussians<<<grid, 128, 0, s>>>(
            pv, static_cast<const fpho_source *>(dev_proposal), p->d_gtab, p->d_gbox);
        CUDA_TRY(cudaGetLastError());
    }
    TileArgs A;
    A.pv = pv;
    A.tiles = p->d_tiles;
    A.tbox_all = p->d_tbox_all;
    A.tbox_w = p->d_tbox_w;
    A.gtab = p->d_gtab;
    A.gbox = p->d_gbox;
    A.pchi2 = p->d_pchi2;
    A.pgrad = p->d_pgrad;
    A.pgrad_stride = 7 * p->n_sources;
    A.want_residual = 1;
    A.live_cap = p->live_cap;
    A.idx_cap = std::max(p->max_g, 1);
    A.err = p->d_err;
    A.pairs = nullptr;
    return launch_design_kernel(p->variant, A, p->n_tiles, dev_X, (long long)p->npix, s);
}

extern "C" int fpho_patch_image_gaussians(fpho_patch *p, int exposure, float *host_out,
                                          int max_records, int *n_out) {
    clear_error();
    if (!p || !host_out || !n_out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (exposure < 0 || exposure >= p->n_exp)
        return set_error(FPHO_ERR_INVALID, "exposure %d not in [0, %d)", exposure, p->n_exp);
    const int g0 = p->gauss_start[exposure], n = p->gauss_start[exposure + 1] - g0;
    if (n > max_records) return set_error(FPHO_ERR_LIMIT, "exposure has %d records", n);
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(cudaMemcpy(host_out, p->d_gtab + (size_t)g0 * GREC, (size_t)n * GREC * sizeof(float),
                        cudaMemcpyDeviceToHost));
    *n_out = n;
    return FPHO_OK;
}

extern "C" int fpho_patch_time_tiles(fpho_patch *p, int enable) {
    clear_error();
    if (!p) return set_error(FPHO_ERR_INVALID, "NULL patch");
    if (enable && !p->ev_tile0) {
        CUDA_TRY(cudaEventCreate(&p->ev_tile0));
        CUDA_TRY(cudaEventCreate(&p->ev_tile1));
    } else if (!enable && p->ev_tile0) {
        cudaEventDestroy(p->ev_tile0);
        cudaEventDestroy(p->ev_tile1);
        p->ev_tile0 = p->ev_tile1 = nullptr;
    }
    return FPHO_OK;
}

extern "C" int fpho_patch_last_tile_ms(fpho_patch *p, float *ms) {
    clear_error();
    if (!p || !ms) return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (!p->ev_tile0) return set_error(FPHO_ERR_STATE, "tile timing is not enabled");
    CUDA_TRY(cudaEventSynchronize(p->ev_tile1));
    CUDA_TRY(cudaEventElapsedTime(ms, p->ev_tile0, p->ev_tile1));
    return FPHO_OK;
}

extern "C" int fpho_patch_error_word(fpho_patch *p, int *out) {
    clear_error();
    if (!p || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    CUDA_TRY(cudaMemcpy(out, p->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    return FPHO_OK;
}
