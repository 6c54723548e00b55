// fpho_flux.cu -- the linear flux solve of fixed-shape sources on the device.
//
// forcepho's optimize_fluxes (forcepho/fitting.py:573-627) takes the design
// matrix X (n_sources x n_pix per band: each source's model at unit flux,
// forcepho/patches/device_patch.py:185-238) and the data y, and solves the
// weighted normal equations per band:
//     ATA = (X w)(X w)^T,  ATb = (X w)(y w),  fluxes = ATA^-1 ATb,
// returning ATA as the flux precision matrix.  Here the normal equations are
// formed without writing X anywhere:
//   normal_tiles   one CTA per pixel tile builds the unit-flux model of every
//                  source at the tile's pixels into shared memory (the design
//                  kernel's scan, staging and exponential), then forms the
//                  tile's FP64 partial sums of ATA (upper triangle) and ATb;
//   normal_reduce  sums the partials of each band's tiles in tile order (FP64)
//                  into ATA (both triangles) and ATb;
//   normal_solve   one CTA per band: FP64 Cholesky factorisation and the two
//                  triangular solves; a band whose ATA is not positive definite
//                  gets NaN fluxes and a status of 1.
// The data y are the patch's device data (after fpho_patch_swap_data_residual
// of subtract_fixed, the data with the fixed sources subtracted).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "fpho_handle.h"
#include "fpho_impl.cuh"
#include "fpho_internal.h"
#include "fpho_kernels.cuh"
#include "fpho_tile.cuh"

namespace fpho {
namespace {

// Shared memory of normal_tiles: [records live_cap x 128 B][kept idx_cap x 4 B]
// [unit-flux rows ns x (tile + 1) floats][w, y: 2 x tile floats].  Rows are
// padded by one float so that threads reading different rows at the same
// pixel hit different banks.
__host__ __device__ inline size_t normal_smem_bytes(int tile, int live_cap, int idx_cap, int ns) {
    return (size_t)live_cap * GSTAGE * 4 + (size_t)idx_cap * 4 + (size_t)ns * (tile + 1) * 4 +
           (size_t)2 * tile * 4;
}

// the (s, t) pair, s <= t, of upper-triangle index p of an ns x ns matrix
__device__ __forceinline__ void upper_pair(int p, int ns, int &s, int &t) {
    s = 0;
    while (p >= ns - s) {
        p -= ns - s;
        ++s;
    }
    t = s + p;
}

// A tile's partial normal equations from its unit-flux rows (ns rows of
// TP + 1 floats), weights ws and data ys: the upper triangle of
// sum w^2 X_s X_t, then sum w^2 X_s y, each term summed in FP64 over the
// tile's pixels in order.  Every thread of the CTA takes terms.
template <int NT, int TP>
__device__ __forceinline__ void tile_normal_partials(const float *rows, const float *ws,
                                                     const float *ys, int ns, int count,
                                                     int n_terms, double *out) {
    const int n_pairs = ns * (ns + 1) / 2;
    for (int p = threadIdx.x; p < n_terms; p += NT) {
        int s, t;
        const float *other;
        if (p < n_pairs) {
            upper_pair(p, ns, s, t);
            other = rows + (size_t)t * (TP + 1);
        } else {
            s = p - n_pairs;
            other = ys;
        }
        const float *xs_ = rows + (size_t)s * (TP + 1);
        double acc = 0.0;
        for (int li = 0; li < count; ++li) {
            const double w = (double)ws[li];
            acc = fma(w * w * (double)xs_[li], (double)other[li], acc);
        }
        out[p] = acc;
    }
}

template <int NT, int K>
__global__ void __launch_bounds__(NT) normal_tiles(TileArgs A, double *pnorm, int n_terms) {
    static_assert(K % 2 == 0, "pixels per thread must be even (packed pairs)");
    constexpr int KP = K / 2;
    constexpr int TP = NT * K;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar;
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    uint32_t phase = 0;
    const int tile = blockIdx.x;
    const int cap = A.live_cap;
    const int ns = A.pv.n_sources;
    float *recs = reinterpret_cast<float *>(smem);
    int *kept = reinterpret_cast<int *>(smem + (size_t)cap * GSTAGE * 4);
    float *rows = reinterpret_cast<float *>(kept + A.idx_cap);  // [ns][TP + 1]
    float *ws = rows + (size_t)ns * (TP + 1);
    float *ys = ws + TP;

    const TileDesc td = A.tiles[tile];
    const float4 bb = A.tbox_all[tile];
    const int g0 = A.pv.gauss_start[td.exposure];
    const int g1 = A.pv.gauss_start[td.exposure + 1];
    const int npsf = A.pv.exp_npsf[td.exposure];
    for (int j = tid; j < ns * (TP + 1); j += NT) rows[j] = 0.0f;
    for (int li = tid; li < TP; li += NT) {
        const bool ok = li < td.count;
        ws[li] = ok ? A.pv.ierr[td.pix_begin + li] : 0.0f;
        ys[li] = ok ? A.pv.data[td.pix_begin + li] : 0.0f;
    }
    __syncthreads();  // barrier initialised, rows cleared

    const float xmid = 0.5f * (bb.x + bb.y), ymid = 0.5f * (bb.z + bb.w);
    v2 Xp[KP], Yp[KP], M[KP];
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        float xs[2], yv[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int li = tid + (2 * j + h) * NT;
            const bool ok = li < td.count;
            const int pix = td.pix_begin + (ok ? li : 0);
            xs[h] = ok ? A.pv.xpix[pix] : xmid;
            yv[h] = ok ? A.pv.ypix[pix] : ymid;
        }
        Xp[j] = pk(xs[0], xs[1]);
        Yp[j] = pk(yv[0], yv[1]);
        M[j] = 0ull;
    }
    const int n_live = scan_tile<NT>(A, bb, g0, g1, npsf, kept);
    const v2 KEXP2 = pk1(KEXP), KEXPLO2 = pk1(KEXP_LO), CM24 = pk1(-1.0f / 24.0f);
    for (int c0 = 0; c0 < n_live; c0 += cap) {
        const int n = min(cap, n_live - c0);
        if (c0 > 0) __syncthreads();
        stage_records<NT>(recs, A.gtab + (size_t)g0 * GREC, kept, c0, n, 0, &mbar, phase, A.err);
        for (int i = 0; i < n; ++i) {
            const float *r = recs + (size_t)i * GSTAGE;
            int flag = kept[c0 + i];
            if (!(flag & FLAG_LAST_SRC) && i + 1 < n) {
                // two Gaussians of the same source: their exponentials interleave
                design_pairs2<KP>(Xp, Yp, M, r, r + GSTAGE, CM24, KEXP2, KEXPLO2);
                ++i;
                r += GSTAGE;
                flag = kept[c0 + i];
            } else {
                design_one<KP>(Xp, Yp, M, r, flag, CM24, KEXP2, KEXPLO2);
            }
            if ((flag & FLAG_LAST_SRC) || i == n - 1) {
                // a source's Gaussians are contiguous in the kept list; one
                // that spans two chunks is flushed twice and added
                const int src = min((unsigned)__float_as_int(r[R_SRC]), (unsigned)(ns - 1));
                float *row = rows + (size_t)src * (TP + 1);
#pragma unroll
                for (int j = 0; j < KP; ++j) {
                    float m0, m1;
                    unpk(M[j], m0, m1);  // accumulated -model
                    row[tid + 2 * j * NT] -= m0;
                    row[tid + (2 * j + 1) * NT] -= m1;
                    M[j] = 0ull;
                }
            }
        }
    }
    __syncthreads();
    tile_normal_partials<NT, TP>(rows, ws, ys, ns, td.count, n_terms,
                                 pnorm + (size_t)tile * n_terms);
}

// grid (n_bands, ceil(n_terms / 128)): ATA[b] (both triangles) and ATb[b]
__global__ void normal_reduce(const int *tile_band_start, const double *pnorm, int n_terms, int ns,
                              double *ata, double *atb) {
    const int b = blockIdx.x;
    const int p = blockIdx.y * blockDim.x + threadIdx.x;
    if (p >= n_terms) return;
    const int t0 = tile_band_start[b], t1 = tile_band_start[b + 1];
    double acc = 0.0;
    for (int t = t0; t < t1; ++t) acc += pnorm[(size_t)t * n_terms + p];
    const int n_pairs = ns * (ns + 1) / 2;
    if (p < n_pairs) {
        int s, t;
        upper_pair(p, ns, s, t);
        ata[((size_t)b * ns + s) * ns + t] = acc;
        ata[((size_t)b * ns + t) * ns + s] = acc;
    } else if (atb) {
        atb[(size_t)b * ns + (p - n_pairs)] = acc;
    }
}

// One CTA of 64 threads per band: Cholesky ATA = L L^T in shared memory
// (FP64), then L z = ATb and L^T x = z.  ns <= 64.
__global__ void __launch_bounds__(64) normal_solve(const double *ata, const double *atb, int ns,
                                                   double *flux, int *status) {
    __shared__ double L[64 * 64];
    __shared__ double z[64];
    __shared__ int bad;
    const int b = blockIdx.x, tid = threadIdx.x;
    const double *Ab = ata + (size_t)b * ns * ns;
    for (int i = tid; i < ns * ns; i += blockDim.x) L[i] = Ab[i];
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int k = 0; k < ns; ++k) {
        if (tid == 0) {
            const double d = L[k * ns + k];
            if (!(d > 0.0)) bad = 1;
            L[k * ns + k] = d > 0.0 ? sqrt(d) : 1.0;
        }
        __syncthreads();
        const double dk = L[k * ns + k];
        for (int i = k + 1 + tid; i < ns; i += blockDim.x) L[i * ns + k] /= dk;
        __syncthreads();
        // trailing update of the lower triangle, column by column per thread
        for (int j = k + 1 + tid; j < ns; j += blockDim.x) {
            const double ljk = L[j * ns + k];
            for (int i = j; i < ns; ++i) L[i * ns + j] -= L[i * ns + k] * ljk;
        }
        __syncthreads();
    }
    if (tid == 0) {
        const double *bb = atb + (size_t)b * ns;
        for (int i = 0; i < ns; ++i) {  // L z = ATb
            double v = bb[i];
            for (int j = 0; j < i; ++j) v -= L[i * ns + j] * z[j];
            z[i] = v / L[i * ns + i];
        }
        for (int i = ns - 1; i >= 0; --i) {  // L^T x = z
            double v = z[i];
            for (int j = i + 1; j < ns; ++j) v -= L[j * ns + i] * z[j];
            z[i] = v / L[i * ns + i];
        }
        if (status) status[b] = bad;
    }
    __syncthreads();
    for (int i = tid; i < ns; i += blockDim.x)
        flux[(size_t)b * ns + i] = bad ? __longlong_as_double(0x7ff8000000000000ll) : z[i];
}

// the normal-equation kernel for a plan's tile size: four pixels per thread
// (two pixel pairs, two Gaussians interleaved: four independent exponential
// chains); whole warps, so the 192-pixel tile takes six pixels per thread.
// (A form with 4 warps of 8 pixels per thread sharing each 256-pixel tile's
// Gaussians, as the split tile kernels do, measured no faster: 0.430 against
// 0.427 ms for the 20-source patch.)
struct NormalShape {
    int tile, nt;
    const void *fn;
};
const NormalShape kNormalShapes[] = {
    {128, 32, (const void *)normal_tiles<32, 4>},
    {192, 32, (const void *)normal_tiles<32, 6>},
    {256, 64, (const void *)normal_tiles<64, 4>},
    {512, 128, (const void *)normal_tiles<128, 4>},
    {1024, 256, (const void *)normal_tiles<256, 4>},
};


std::mutex g_norm_mu;
size_t g_norm_attr[64][8];

}  // namespace
}  // namespace fpho

using namespace fpho;

#define CUDA_TRY(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return set_error(FPHO_ERR_CUDA, "%s failed: %s (%s:%d)", #call,             \
                             cudaGetErrorString(e_), __FILE__, __LINE__);               \
    } while (0)

// Enqueue normal_tiles + normal_reduce; ATA into d_ata, ATb into d_atb.
static int enqueue_normal(fpho_patch *p, const fpho_source *d_prop, double *d_ata, double *d_atb,
                          cudaStream_t s) {
    const int ns = p->n_sources;
    const int n_terms = ns * (ns + 1) / 2 + ns;
    const int tile = variant_tile_pixels(p->variant);
    constexpr int n_shapes = sizeof(kNormalShapes) / sizeof(kNormalShapes[0]);
    int shape = -1;
    for (int i = 0; i < n_shapes; ++i)
        if (kNormalShapes[i].tile == tile) shape = i;
    if (shape < 0)
        return set_error(FPHO_ERR_STATE, "no normal-equation kernel for %d-pixel tiles", tile);
    const NormalShape &S = kNormalShapes[shape];
    const int idx_cap = std::max(p->max_g, 1);
    const int live_cap = std::min(p->live_cap, DESIGN_LIVE_CAP);
    const size_t smem = normal_smem_bytes(tile, live_cap, idx_cap, ns);
    if (smem > 227 * 1024)
        return set_error(FPHO_ERR_LIMIT, "the normal equations of %d sources over %d-pixel tiles "
                         "need %zu bytes of shared memory (max 227 KB)", ns, tile, smem);
    const size_t need = (size_t)std::max(p->n_tiles, 1) * n_terms;
    if (p->d_pnorm_cap < need) {
        pool_free(p->d_pnorm);
        p->d_pnorm = nullptr;
        p->d_pnorm_cap = 0;
        CUDA_TRY(pool_malloc((void **)&p->d_pnorm, need * sizeof(double)));
        p->d_pnorm_cap = need;
    }
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64) return set_error(FPHO_ERR_LIMIT, "device ordinal %d >= 64", dev);
    {
        std::lock_guard<std::mutex> lk(g_norm_mu);
        if (g_norm_attr[dev][shape] < smem) {
            CUDA_TRY(cudaFuncSetAttribute(S.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
            g_norm_attr[dev][shape] = smem;
        }
    }
    CUDA_TRY(cudaMemsetAsync(p->d_err, 0, sizeof(int), s));
    const PatchView pv = make_view(p);
    if (p->max_g > 0) {
        dim3 grid((p->max_g + 127) / 128, p->n_exp);
        build_image_gaussians<<<grid, 128, 0, s>>>(pv, d_prop, p->d_gtab, p->d_gbox);
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
    A.pgrad_stride = 7 * ns;
    A.want_residual = 1;
    A.live_cap = live_cap;
    A.idx_cap = idx_cap;
    A.err = p->d_err;
    A.pairs = nullptr;
    if (p->n_tiles > 0) {
        double *pn = p->d_pnorm;
        int nt = n_terms;
        void *args[] = {(void *)&A, (void *)&pn, (void *)&nt};
        CUDA_TRY(cudaLaunchKernel(S.fn, dim3(p->n_tiles), dim3(S.nt), args, smem, s));
    }
    normal_reduce<<<dim3(p->n_bands, (n_terms + 127) / 128), 128, 0, s>>>(
        p->d_tile_band_start, p->d_pnorm, n_terms, ns, d_ata, d_atb);
    CUDA_TRY(cudaGetLastError());
    return FPHO_OK;
}

extern "C" int fpho_patch_flux_normal_equations(fpho_patch *p, const void *dev_proposal,
                                                int n_sources, double *dev_ata, double *dev_atb,
                                                void *stream) {
    clear_error();
    if (!p || !dev_proposal || !dev_ata || !dev_atb)
        return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (n_sources != p->n_sources)
        return set_error(FPHO_ERR_INVALID, "n_sources=%d but the patch has %d", n_sources,
                         p->n_sources);
    return enqueue_normal(p, (const fpho_source *)dev_proposal, dev_ata, dev_atb,
                          (cudaStream_t)stream);
}

extern "C" int fpho_patch_optimize_fluxes(fpho_patch *p, const void *dev_proposal, int n_sources,
                                          double *dev_flux, double *dev_precision,
                                          int *dev_status, void *stream) {
    clear_error();
    if (!p || !dev_proposal || !dev_flux || !dev_precision)
        return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (n_sources != p->n_sources)
        return set_error(FPHO_ERR_INVALID, "n_sources=%d but the patch has %d", n_sources,
                         p->n_sources);
    if (n_sources > 64)
        return set_error(FPHO_ERR_LIMIT, "the device flux solve takes at most 64 sources (%d)",
                         n_sources);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nb = (size_t)p->n_bands * n_sources;
    if (p->d_atb_cap < nb) {
        pool_free(p->d_atb);
        p->d_atb = nullptr;
        p->d_atb_cap = 0;
        CUDA_TRY(pool_malloc((void **)&p->d_atb, nb * sizeof(double)));
        p->d_atb_cap = nb;
    }
    int rc = enqueue_normal(p, (const fpho_source *)dev_proposal, dev_precision, p->d_atb, s);
    if (rc) return rc;
    normal_solve<<<p->n_bands, 64, 0, s>>>(dev_precision, p->d_atb, n_sources, dev_flux,
                                           dev_status);
    CUDA_TRY(cudaGetLastError());
    return FPHO_OK;
}
