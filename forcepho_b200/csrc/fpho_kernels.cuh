// fpho_kernels.cuh -- small kernels around the tile kernel, included (with
// internal linkage) by every translation unit that launches them.
#pragma once

#include "fpho_impl.cuh"

namespace fpho {

// One thread per image Gaussian of exposure blockIdx.y: record + culling box.
static __global__ void build_image_gaussians(PatchView pv, const fpho_source *src, float *gtab,
                                             float4 *gbox) {
    const int e = blockIdx.y;
    const int g0 = pv.gauss_start[e];
    const int n = pv.gauss_start[e + 1] - g0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int npsf = pv.exp_npsf[e];
    const int s = i / npsf, p = i - s * npsf;
    build_one_gaussian(pv, src, e, s, p, gtab + (size_t)(g0 + i) * GREC, gbox + g0 + i);
}

// Bounding boxes of every tile: over all pixels and over pixels with
// ierr != 0.  If n_tiles_dev is given, blocks at or beyond *n_tiles_dev exit.
static __global__ void tile_bboxes(PatchView pv, const TileDesc *tiles, float4 *tbox_all,
                                   float4 *tbox_w, const int *n_tiles_dev) {
    if (n_tiles_dev && (int)blockIdx.x >= *n_tiles_dev) return;
    const TileDesc td = tiles[blockIdx.x];
    float ax0 = INFINITY, ax1 = -INFINITY, ay0 = INFINITY, ay1 = -INFINITY;
    float wx0 = INFINITY, wx1 = -INFINITY, wy0 = INFINITY, wy1 = -INFINITY;
    for (int i = threadIdx.x; i < td.count; i += blockDim.x) {
        const int pix = td.pix_begin + i;
        const float x = pv.xpix[pix], y = pv.ypix[pix];
        ax0 = fminf(ax0, x); ax1 = fmaxf(ax1, x);
        ay0 = fminf(ay0, y); ay1 = fmaxf(ay1, y);
        if (pv.ierr[pix] != 0.0f) {
            wx0 = fminf(wx0, x); wx1 = fmaxf(wx1, x);
            wy0 = fminf(wy0, y); wy1 = fmaxf(wy1, y);
        }
    }
    __shared__ float red[8][32];
    float v[8] = {ax0, -ax1, ay0, -ay1, wx0, -wx1, wy0, -wy1};
#pragma unroll
    for (int k = 0; k < 8; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 8; ++k) red[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x / 32;
        for (int k = 0; k < 8; ++k)
            for (int w = 1; w < nw; ++w) red[k][0] = fminf(red[k][0], red[k][w]);
        tbox_all[blockIdx.x] = make_float4(red[0][0], -red[1][0], red[2][0], -red[3][0]);
        tbox_w[blockIdx.x] = make_float4(red[4][0], -red[5][0], red[6][0], -red[7][0]);
    }
}

// Work order for the persistent tile kernel: tiles by decreasing cost in the
// previous evaluation (kept image Gaussians x pixels, written by the tile
// body), approximately -- a counting sort into 64 equal-width buckets of
// [0, max cost]; within a bucket the order is whatever the shared-memory
// atomics give.  The result does not depend on the order, since every tile
// writes its own partials and reduce_bands sums them in tile-index order.
// One CTA (at least 64 threads).  Also resets the work counter.
__device__ __forceinline__ void order_tiles_body(const int *cost, int n_tiles, int *order,
                                                 int *counter) {
    constexpr int NB = 64;
    __shared__ int hist[NB];
    __shared__ int smax;
    const int tid = threadIdx.x;
    if (tid < NB) hist[tid] = 0;
    if (tid == 0) {
        smax = 0;
        *counter = 0;
    }
    __syncthreads();
    int m = 0;
    for (int i = tid; i < n_tiles; i += blockDim.x) m = max(m, cost[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0) atomicMax(&smax, m);
    __syncthreads();
    const long long span = (long long)smax + 1;
    for (int i = tid; i < n_tiles; i += blockDim.x)
        atomicAdd(&hist[NB - 1 - (int)((long long)cost[i] * NB / span)], 1);
    __syncthreads();
    if (tid == 0) {
        int acc = 0;
        for (int b = 0; b < NB; ++b) {
            const int h = hist[b];
            hist[b] = acc;
            acc += h;
        }
    }
    __syncthreads();
    for (int i = tid; i < n_tiles; i += blockDim.x)
        order[atomicAdd(&hist[NB - 1 - (int)((long long)cost[i] * NB / span)], 1)] = i;
}

// The launch before the tile kernel of an evaluation: blocks (x, e < n_exp)
// build exposure e's image Gaussians (as build_image_gaussians); with
// `order`, the block (0, n_exp) orders the tiles by the previous
// evaluation's costs (as order_tiles) at the same time; and block (0, 0)
// clears the error word.  One launch instead of a memset and two kernels.
// Launched with PREP_THREADS threads per block: the ordering block is then
// as wide as a standalone sort would be (its passes over the costs are
// latency-bound), and one block covers an exposure's image Gaussians.
constexpr int PREP_THREADS = 1024;
static __global__ void __launch_bounds__(PREP_THREADS) prepare_evaluation(
    PatchView pv, const fpho_source *src, float *gtab, float4 *gbox, const int *cost, int n_tiles,
    int *order, int *counter, int *err) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *err = 0;
    const int e = blockIdx.y;
    if (e == pv.n_exp) {
        if (blockIdx.x == 0 && order) order_tiles_body(cost, n_tiles, order, counter);
        return;
    }
    const int g0 = pv.gauss_start[e];
    const int n = pv.gauss_start[e + 1] - g0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int npsf = pv.exp_npsf[e];
    const int s = i / npsf, p = i - s * npsf;
    build_one_gaussian(pv, src, e, s, p, gtab + (size_t)(g0 + i) * GREC, gbox + g0 + i);
}

// Sum of a tile range [t0, t1) of one column (FP64): lane l adds tiles
// t0 + l, t0 + l + 32, ... in order, then the lanes combine by a fixed
// butterfly -- deterministic, and 32 loads in flight instead of one chain.
template <typename T>
__device__ __forceinline__ double warp_column_sum(const T *col, size_t step, int t0, int t1,
                                                  int lane) {
    double acc = 0.0;
    for (int t = t0 + lane; t < t1; t += 32) acc += (double)col[(size_t)t * step];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// Warps per block of reduce_bands and batch_reduce: one gradient component each.
constexpr int REDUCE_WARPS = 4;

// Sum tile partials per band in double.  grid (n_bands, ceil(out_stride /
// REDUCE_WARPS)), block 32 REDUCE_WARPS: warp w of block y sums component
// y REDUCE_WARPS + w; block y = 0, warp 0 also sums chi2.
// With err_out, block (0, 0) also copies the evaluation's error word there
// (beside the results, so that one transfer brings both to the host).
static __global__ void reduce_bands(const int *tile_band_start, const double *pchi2,
                                    const float *pgrad, int stride, double *chi2_out,
                                    float *dchi2_out, int out_stride, const int *err = nullptr,
                                    int *err_out = nullptr) {
    const int b = blockIdx.x;
    if (err_out && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *err_out = *err;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int t0 = tile_band_start[b], t1 = tile_band_start[b + 1];
    const int j = blockIdx.y * REDUCE_WARPS + w;
    if (dchi2_out && j < out_stride) {
        const double acc = j < stride ? warp_column_sum(pgrad + j, stride, t0, t1, lane) : 0.0;
        if (lane == 0) dchi2_out[(size_t)b * out_stride + j] = (float)acc;
    }
    if (blockIdx.y == 0 && w == 0) {
        const double c = warp_column_sum(pchi2, 1, t0, t1, lane);
        if (lane == 0) chi2_out[b] = c;
    }
}

}  // namespace fpho
