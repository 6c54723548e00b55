// fpho_batch.cu -- many patches evaluated by one persistent launch.
//
// A batch is a list of patch handles evaluated together:
//   batch_gaussians  one launch builds the image Gaussians of every exposure
//                    of every patch (grid y = (patch, exposure) pairs);
//   batch_tiles      one persistent launch: each CTA takes (patch, tile) items
//                    from a work list sorted by decreasing cost (pixels x image
//                    Gaussians of the tile's exposure), through an atomic
//                    counter, until the list is exhausted -- patches of 1..30
//                    sources and 32^2..200^2 pixels balance across the SMs;
//   batch_reduce     one launch sums the tile partials of every (patch, band)
//                    in double and resets the work counter for the next call.
// No kernel waits on another CTA: the counter only hands out indices.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <vector>

#include "fpho_handle.h"
#include "fpho_internal.h"
#include "fpho_kernels.cuh"
#include "fpho_tile.cuh"

namespace fpho {
namespace {


struct BatchPatch {
    PatchView pv;
    float *gtab;
    float4 *gbox;
    int prop_off;  // first source of this patch in the concatenated proposal
};

struct BandJob {
    int t0, t1;         // tile range of the band in the patch's partials
    int stride;         // 7 * n_sources of the patch
    int chi2_index;     // output index into the concatenated chi2
    long long dchi2_off;  // output offset into the concatenated dchi2
    const double *pchi2;
    const float *pgrad;
};

__global__ void batch_gaussians(const BatchPatch *bps, const int2 *expmap,
                                const fpho_source *props) {
    const int2 pe = expmap[blockIdx.y];
    const BatchPatch &bp = bps[pe.x];
    const int e = pe.y;
    const int g0 = bp.pv.gauss_start[e];
    const int n = bp.pv.gauss_start[e + 1] - g0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int npsf = bp.pv.exp_npsf[e];
    const int s = i / npsf, p = i - s * npsf;
    build_one_gaussian(bp.pv, props + bp.prop_off, e, s, p, bp.gtab + (size_t)(g0 + i) * GREC,
                       bp.gbox + g0 + i);
}

// SPLIT = 0: tile_body with NT threads x K pixels per tile; SPLIT = NW:
// tile_body_split with NW warps (NT = 32 NW) and K pixels per thread.  MINB:
// the minimum resident CTAs per SM asked of the compiler (a register cap).
template <int NT, int K, int SPLIT, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) batch_tiles(const TileArgs *args, const int2 *work,
                                                        int n_work, int *counter) {
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
        const int it = s_item;
        __syncthreads();  // all threads hold `it` before s_item is rewritten
        if (it >= n_work) break;
        const int2 w = work[it];
        if constexpr (SPLIT > 0)
            tile_body_split<SPLIT, K>(args[w.x], w.y, smem, &mbar, phase);
        else
            tile_body<NT, K>(args[w.x], w.y, smem, &mbar, phase);
        __syncthreads();  // shared memory of this tile fully consumed
    }
}

// grid (n_jobs, ceil(max_stride / REDUCE_WARPS)), block 32 REDUCE_WARPS: the
// same per-component warp sums as reduce_bands, so a patch's batched result
// equals its single-patch one bit for bit
__global__ void batch_reduce(const BandJob *jobs, double *chi2, float *dchi2, int *counter) {
    const BandJob jb = jobs[blockIdx.x];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int j = blockIdx.y * REDUCE_WARPS + w;
    if (j < jb.stride) {
        const double acc = warp_column_sum(jb.pgrad + j, jb.stride, jb.t0, jb.t1, lane);
        if (lane == 0) dchi2[jb.dchi2_off + j] = (float)acc;
    }
    if (blockIdx.y == 0 && w == 0) {
        const double c = warp_column_sum(jb.pchi2, 1, jb.t0, jb.t1, lane);
        if (lane == 0) chi2[jb.chi2_index] = c;
    }
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *counter = 0;
}

// The tile shapes compiled for batches: (threads, pixels per tile, warps
// sharing a tile's Gaussians) and the kernel; each runs the patches planned
// with the patch variant of the same shape.
struct BatchShape {
    int nt, tile, split;
    const void *fn;
};
const BatchShape kBatchShapes[] = {
    // registers capped at 128 a thread (MINB = 65536 / (128 NT))
    {64, 512, 0, (const void *)batch_tiles<64, 8, 0, 8>},    // default: 64 threads x 8 pixels
    {64, 256, 0, (const void *)batch_tiles<64, 4, 0, 8>},
    {128, 512, 0, (const void *)batch_tiles<128, 4, 0, 4>},
    // split tiles with the registers capped at 128 (left free, the compiler
    // takes 156 and fewer CTAs fit), and at 96 for 5 CTAs per SM
    {128, 256, 4, (const void *)batch_tiles<128, 8, 4, 4>},  // 4 warps share 256-pixel tiles
    {64, 256, 2, (const void *)batch_tiles<64, 8, 2, 8>},    // 2 warps share 256-pixel tiles
    {128, 256, 4, (const void *)batch_tiles<128, 8, 4, 5>},  // 4 warps, 5 CTAs per SM
};
constexpr int kNumBatchShapes = sizeof(kBatchShapes) / sizeof(kBatchShapes[0]);

// the patch variant planned like batch shape `i` (the k-th shape of a given
// (threads, tile, split) maps to the k-th patch variant of it: the register
// cap is the only difference between such shapes), or -1 if none is compiled
int shape_variant(int i) {
    const BatchShape &B = kBatchShapes[i];
    int rank = 0;
    for (int j = 0; j < i; ++j)
        rank += kBatchShapes[j].nt == B.nt && kBatchShapes[j].tile == B.tile &&
                kBatchShapes[j].split == B.split;
    for (int v = 0; v < variant_count(); ++v)
        if (variant_threads(v) == B.nt && variant_tile_pixels(v) == B.tile &&
            variant_split(v) == B.split && rank-- == 0)
            return v;
    return -1;
}

std::mutex g_attr_mu;
size_t g_attr_set[64][kNumBatchShapes];

}  // namespace
}  // namespace fpho

using namespace fpho;

struct fpho_batch {
    std::vector<fpho_patch *> patches;
    int live_cap = 256;
    int shape = 0;         // index into kBatchShapes
    int variant = -1;      // the patches' tile variant
    int ctas_per_sm = 0;   // cap on resident CTAs per SM of the persistent grid (0: none)
    int n_work = 0, n_exp_total = 0, max_g = 0, n_jobs = 0, max_stride = 0;
    int n_src_total = 0, n_band_total = 0;
    long long n_dchi2 = 0;
    size_t smem = 0;
    int grid = 0;
    BatchPatch *d_bps = nullptr;
    int2 *d_expmap = nullptr;
    TileArgs *d_args = nullptr;
    int2 *d_work = nullptr;
    BandJob *d_jobs = nullptr;
    int *d_counter = nullptr;
    int *d_err = nullptr;
    long long *d_pairs = nullptr;
    int count_pairs = 0;
    // staging for host I/O
    fpho_source *d_props = nullptr;
    double *d_chi2 = nullptr;
    float *d_dchi2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<TileArgs> h_args;
};

#define CUDA_TRY(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return set_error(FPHO_ERR_CUDA, "%s failed: %s (%s:%d)", #call,             \
                             cudaGetErrorString(e_), __FILE__, __LINE__);               \
    } while (0)

namespace {

template <typename T>
int balloc(T **p, size_t n) {
    *p = nullptr;
    cudaError_t e = fpho::pool_malloc((void **)p, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_error(FPHO_ERR_NOMEM, "device allocation failed: %s", cudaGetErrorString(e));
    }
    return FPHO_OK;
}
template <typename T>
void bfree(T *&p) {
    fpho::pool_free((void *)p);
    p = nullptr;
}

void destroy_batch(fpho_batch *b) {
    bfree(b->d_bps); bfree(b->d_expmap); bfree(b->d_args); bfree(b->d_work); bfree(b->d_jobs);
    bfree(b->d_counter); bfree(b->d_err); bfree(b->d_pairs); bfree(b->d_props);
    bfree(b->d_chi2); bfree(b->d_dchi2);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    delete b;
}

}  // namespace

extern "C" int fpho_batch_variants(int *out, int cap) {
    clear_error();
    for (int i = 0; i < kNumBatchShapes && out && i < cap; ++i) out[i] = shape_variant(i);
    return kNumBatchShapes;
}

extern "C" int fpho_batch_create_config(fpho_patch *const *patches, int n, int variant,
                                        int live_cap, int ctas_per_sm, void *stream,
                                        fpho_batch **out) {
    clear_error();
    if (!patches || !out || n < 1) return set_error(FPHO_ERR_INVALID, "bad batch arguments");
    *out = nullptr;
    if (live_cap < 32 || live_cap > 4096)
        return set_error(FPHO_ERR_INVALID, "live_cap %d outside [32, 4096]", live_cap);
    if (ctas_per_sm < 0 || ctas_per_sm > 32)
        return set_error(FPHO_ERR_INVALID, "ctas_per_sm %d outside [0, 32]", ctas_per_sm);
    int shape = -1;
    for (int i = 0; i < kNumBatchShapes; ++i)
        if (shape_variant(i) >= 0 && (variant < 0 ? i == 0 : shape_variant(i) == variant)) {
            shape = i;
            break;
        }
    if (shape < 0)
        return set_error(FPHO_ERR_INVALID, "no batched tile kernel is compiled for variant %d",
                         variant);
    variant = shape_variant(shape);
    for (int i = 0; i < n; ++i) {
        if (!patches[i]) return set_error(FPHO_ERR_INVALID, "patch %d is NULL", i);
        int rc = fpho_patch_set_config(patches[i], variant, live_cap, stream);
        if (rc) return rc;
    }
    fpho_batch *b = new (std::nothrow) fpho_batch();
    if (!b) return set_error(FPHO_ERR_NOMEM, "host allocation failed");
    b->patches.assign(patches, patches + n);
    b->live_cap = live_cap;
    b->shape = shape;
    b->variant = variant;
    b->ctas_per_sm = ctas_per_sm;
    std::vector<BatchPatch> bps(n);
    std::vector<int2> expmap;
    std::vector<std::pair<double, int2>> items;
    std::vector<BandJob> jobs;
    int rc = FPHO_OK;
    if (!rc) rc = balloc(&b->d_err, 1);
    if (!rc && cudaMemsetAsync(b->d_err, 0, sizeof(int), (cudaStream_t)stream) != cudaSuccess)
        rc = set_error(FPHO_ERR_CUDA, "cudaMemsetAsync failed");
    if (!rc) rc = balloc(&b->d_pairs, 1);
    long long dchi2_off = 0;
    int src_off = 0, band_off = 0;
    for (int i = 0; i < n && !rc; ++i) {
        fpho_patch *p = patches[i];
        bps[i].pv = make_view(p);
        bps[i].gtab = p->d_gtab;
        bps[i].gbox = p->d_gbox;
        bps[i].prop_off = src_off;
        for (int e = 0; e < p->n_exp; ++e) {
            const int ng = p->gauss_start[e + 1] - p->gauss_start[e];
            if (ng > 0) expmap.push_back(make_int2(i, e));
            b->max_g = std::max(b->max_g, ng);
        }
        TileArgs A;
        A.pv = bps[i].pv;
        A.tiles = p->d_tiles;
        A.tbox_all = p->d_tbox_all;
        A.tbox_w = p->d_tbox_w;
        A.gtab = p->d_gtab;
        A.gbox = p->d_gbox;
        A.pchi2 = p->d_pchi2;
        A.pgrad = p->d_pgrad;
        A.pgrad_stride = 7 * p->n_sources;
        A.want_residual = 0;
        A.live_cap = live_cap;
        A.idx_cap = std::max(p->max_g, 1);
        A.err = b->d_err;
        A.pairs = nullptr;
        b->h_args.push_back(A);
        b->max_stride = std::max(b->max_stride, 7 * p->n_sources);
        for (int t = 0; t < p->n_tiles; ++t) {
            const TileDesc &td = p->h_tiles[t];
            const int ng = p->gauss_start[td.exposure + 1] - p->gauss_start[td.exposure];
            items.push_back({(double)td.count * ng, make_int2(i, t)});
        }
        for (int bnd = 0; bnd < p->n_bands; ++bnd) {
            BandJob j;
            j.t0 = p->tile_band_start[bnd];
            j.t1 = p->tile_band_start[bnd + 1];
            j.stride = 7 * p->n_sources;
            j.chi2_index = band_off + bnd;
            j.dchi2_off = dchi2_off + (long long)bnd * j.stride;
            j.pchi2 = p->d_pchi2;
            j.pgrad = p->d_pgrad;
            jobs.push_back(j);
        }
        src_off += p->n_sources;
        band_off += p->n_bands;
        dchi2_off += (long long)p->n_bands * 7 * p->n_sources;
    }
    if (!rc && (int)expmap.size() > 65535)
        rc = set_error(FPHO_ERR_LIMIT, "batch has %zu exposures (max 65535)", expmap.size());
    // longest tiles first
    std::stable_sort(items.begin(), items.end(),
                     [](const std::pair<double, int2> &a, const std::pair<double, int2> &c) {
                         return a.first > c.first;
                     });
    std::vector<int2> work(items.size());
    for (size_t k = 0; k < items.size(); ++k) work[k] = items[k].second;
    b->n_work = (int)work.size();
    b->n_exp_total = (int)expmap.size();
    b->n_jobs = (int)jobs.size();
    b->n_src_total = src_off;
    b->n_band_total = band_off;
    b->n_dchi2 = dchi2_off;
    cudaStream_t s = (cudaStream_t)stream;
    auto up = [&](auto **dst, const auto &vec) -> int {
        int r = balloc(dst, vec.size());
        if (r) return r;
        if (!vec.empty())
            CUDA_TRY(cudaMemcpyAsync(*dst, vec.data(), vec.size() * sizeof(vec[0]),
                                     cudaMemcpyHostToDevice, s));
        return FPHO_OK;
    };
    if (!rc) rc = up(&b->d_bps, bps);
    if (!rc) rc = up(&b->d_expmap, expmap);
    if (!rc) rc = up(&b->d_args, b->h_args);
    if (!rc) rc = up(&b->d_work, work);
    if (!rc) rc = up(&b->d_jobs, jobs);
    if (!rc) rc = balloc(&b->d_counter, 1);
    if (!rc && cudaMemsetAsync(b->d_counter, 0, sizeof(int), s) != cudaSuccess)
        rc = set_error(FPHO_ERR_CUDA, "cudaMemsetAsync failed");
    if (!rc) {
        b->smem = tile_smem_bytes(b->variant, live_cap, std::max(b->max_g, 1), b->max_stride);
        if (b->smem > 227 * 1024)
            rc = set_error(FPHO_ERR_LIMIT, "shared memory %zu exceeds 227 KB", b->smem);
    }
    if (!rc) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const BatchShape &B = kBatchShapes[b->shape];
        if (e == cudaSuccess) {
            std::lock_guard<std::mutex> lk(g_attr_mu);
            if (dev < 64 && g_attr_set[dev][b->shape] < b->smem) {
                e = cudaFuncSetAttribute(B.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)b->smem);
                if (e == cudaSuccess) g_attr_set[dev][b->shape] = b->smem;
            }
        }
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, B.fn, B.nt, b->smem);
        if (e != cudaSuccess)
            rc = set_error(FPHO_ERR_CUDA, "batch launch setup: %s", cudaGetErrorString(e));
        else if (per_sm < 1)
            rc = set_error(FPHO_ERR_LIMIT, "the batched tile kernel cannot be resident with "
                           "%zu bytes of shared memory", b->smem);
        else {
            if (b->ctas_per_sm > 0) per_sm = std::min(per_sm, b->ctas_per_sm);
            b->grid = std::max(1, std::min(b->n_work, sms * per_sm));
        }
    }
    if (!rc && cudaStreamSynchronize(s) != cudaSuccess)
        rc = set_error(FPHO_ERR_CUDA, "cudaStreamSynchronize failed");
    if (rc) {
        destroy_batch(b);
        return rc;
    }
    *out = b;
    return FPHO_OK;
}

extern "C" int fpho_batch_create(fpho_patch *const *patches, int n, int live_cap, void *stream,
                                 fpho_batch **out) {
    return fpho_batch_create_config(patches, n, -1, live_cap, 0, stream, out);
}

extern "C" int fpho_batch_config(const fpho_batch *b, int out[4]) {
    clear_error();
    if (!b || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    out[0] = b->variant;
    out[1] = b->live_cap;
    out[2] = b->ctas_per_sm;
    out[3] = b->grid;
    return FPHO_OK;
}

extern "C" int fpho_batch_info(const fpho_batch *b, int64_t out[7]) {
    clear_error();
    if (!b || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    out[0] = (int64_t)b->patches.size();
    out[1] = b->n_src_total;
    out[2] = b->n_band_total;
    out[3] = b->n_dchi2;
    out[4] = b->n_work;
    out[5] = b->grid;
    out[6] = b->n_exp_total;
    return FPHO_OK;
}

extern "C" int fpho_batch_count_pairs(fpho_batch *b, int enable, long long *last_count) {
    clear_error();
    if (!b) return set_error(FPHO_ERR_INVALID, "NULL batch");
    if (enable != b->count_pairs) {
        for (auto &A : b->h_args) A.pairs = enable ? b->d_pairs : nullptr;
        CUDA_TRY(cudaMemcpy(b->d_args, b->h_args.data(), b->h_args.size() * sizeof(TileArgs),
                            cudaMemcpyHostToDevice));
        b->count_pairs = enable;
    }
    if (last_count) {
        long long v = 0;
        CUDA_TRY(cudaMemcpy(&v, b->d_pairs, sizeof(v), cudaMemcpyDeviceToHost));
        *last_count = v;
    }
    return FPHO_OK;
}

extern "C" int fpho_batch_time_tiles(fpho_batch *b, int enable) {
    clear_error();
    if (!b) return set_error(FPHO_ERR_INVALID, "NULL batch");
    if (enable && !b->ev0) {
        CUDA_TRY(cudaEventCreate(&b->ev0));
        CUDA_TRY(cudaEventCreate(&b->ev1));
    } else if (!enable && b->ev0) {
        cudaEventDestroy(b->ev0);
        cudaEventDestroy(b->ev1);
        b->ev0 = b->ev1 = nullptr;
    }
    return FPHO_OK;
}

extern "C" int fpho_batch_last_tile_ms(fpho_batch *b, float *ms) {
    clear_error();
    if (!b || !ms) return set_error(FPHO_ERR_INVALID, "NULL argument");
    if (!b->ev0) return set_error(FPHO_ERR_STATE, "tile timing is not enabled");
    CUDA_TRY(cudaEventSynchronize(b->ev1));
    CUDA_TRY(cudaEventElapsedTime(ms, b->ev0, b->ev1));
    return FPHO_OK;
}

static int batch_enqueue(fpho_batch *b, const fpho_source *d_props, double *d_chi2,
                         float *d_dchi2, cudaStream_t s) {
    CUDA_TRY(cudaMemsetAsync(b->d_err, 0, sizeof(int), s));
    if (b->count_pairs) CUDA_TRY(cudaMemsetAsync(b->d_pairs, 0, sizeof(long long), s));
    if (b->n_exp_total > 0 && b->max_g > 0) {
        batch_gaussians<<<dim3((b->max_g + 127) / 128, b->n_exp_total), 128, 0, s>>>(
            b->d_bps, b->d_expmap, d_props);
        CUDA_TRY(cudaGetLastError());
    }
    if (b->ev0) CUDA_TRY(cudaEventRecord(b->ev0, s));
    if (b->n_work > 0) {
        const BatchShape &B = kBatchShapes[b->shape];
        const TileArgs *args = b->d_args;
        const int2 *work = b->d_work;
        int n_work = b->n_work;
        int *counter = b->d_counter;
        void *kargs[] = {(void *)&args, (void *)&work, (void *)&n_work, (void *)&counter};
        CUDA_TRY(cudaLaunchKernel(B.fn, dim3(b->grid), dim3(B.nt), kargs, b->smem, s));
    }
    if (b->ev1) CUDA_TRY(cudaEventRecord(b->ev1, s));
    if (b->n_jobs > 0) {
        batch_reduce<<<dim3(b->n_jobs, (b->max_stride + REDUCE_WARPS - 1) / REDUCE_WARPS),
                       32 * REDUCE_WARPS, 0, s>>>(
            b->d_jobs, d_chi2, d_dchi2, b->d_counter);
        CUDA_TRY(cudaGetLastError());
    }
    return FPHO_OK;
}

extern "C" int fpho_batch_evaluate(fpho_batch *b, const fpho_source *proposals, double *chi2,
                                   float *dchi2, unsigned flags, void *stream) {
    clear_error();
    if (!b || !proposals || !chi2 || !dchi2) return set_error(FPHO_ERR_INVALID, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (!(flags & FPHO_IO_HOST)) return batch_enqueue(b, proposals, chi2, dchi2, s);
    if (!b->d_props) {
        int rc;
        if ((rc = balloc(&b->d_props, (size_t)b->n_src_total))) return rc;
        if ((rc = balloc(&b->d_chi2, (size_t)b->n_band_total))) return rc;
        if ((rc = balloc(&b->d_dchi2, (size_t)b->n_dchi2))) return rc;
    }
    CUDA_TRY(cudaMemcpyAsync(b->d_props, proposals, sizeof(fpho_source) * b->n_src_total,
                             cudaMemcpyHostToDevice, s));
    int rc = batch_enqueue(b, b->d_props, b->d_chi2, b->d_dchi2, s);
    if (rc) return rc;
    int err = 0;
    CUDA_TRY(cudaMemcpyAsync(chi2, b->d_chi2, sizeof(double) * b->n_band_total,
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(dchi2, b->d_dchi2, sizeof(float) * b->n_dchi2,
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (err) return set_error(FPHO_ERR_KERNEL, "batched tile kernel reported error word 0x%x", err);
    return FPHO_OK;
}

extern "C" int fpho_batch_error_word(fpho_batch *b, int *out) {
    clear_error();
    if (!b || !out) return set_error(FPHO_ERR_INVALID, "NULL argument");
    CUDA_TRY(cudaMemcpy(out, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    return FPHO_OK;
}

extern "C" int fpho_batch_free(fpho_batch *b) {
    clear_error();
    if (b) destroy_batch(b);
    return FPHO_OK;
}
