// fpho_tile.cuh -- the pixel-tile kernel body shared by the single-patch and
// the batched evaluation.
//
// One CTA evaluates one tile of up to NT*K pixels of one exposure:
//   1. cull: keep the exposure's image Gaussians whose exp-argument <= 36 box
//      overlaps the tile's pixel bounding box (provably equivalent to the
//      reference's per-pixel `exparg > 36` skip, which is still applied to
//      every Gaussian that can cross the threshold inside the tile);
//   2. stage the kept 128-byte records into shared memory with cp.async.bulk
//      (one bulk copy per record, issued by every thread of the CTA,
//      completion on an mbarrier);
//   3. residual pass: r = data - sum_g amp G H over kept Gaussians, in the
//      reference's Gaussian order (ComputeResidualImage, common_kernel.cc:57-83);
//   4. chi2 per pixel in double, exactly as compute_gaussians_kernel.cc:286-293;
//   5. gradient pass: for each kept Gaussian, each thread accumulates the
//      derivatives of its pixels' model w.r.t. the Gaussian's image-space
//      parameters (A, x, y, fxx, fyy, fxy), then applies the Gaussian's
//      Jacobian once (ComputeGaussianDerivative, common_kernel.cc:95-143, with
//      the per-pixel Jacobian product moved out of the pixel loop);
//   6. per-source sums are reduced across the warp and the CTA in a fixed
//      order and written as this tile's partial; chi2 partials stay double.
// Pixel pairs are processed as packed .f32x2 operands (two pixels per
// instruction).
#pragma once

#include "fpho_impl.cuh"

namespace fpho {

struct TileArgs {
    PatchView pv;
    const TileDesc *tiles;
    const float4 *tbox_all;   // per tile bounding box of all pixels (x0, x1, y0, y1)
    const float4 *tbox_w;     // per tile bounding box of pixels with ierr != 0
    const float *gtab;        // image-Gaussian records
    const float4 *gbox;       // culling boxes
    double *pchi2;            // [n_tiles] chi2 partial per tile
    float *pgrad;             // [n_tiles][pgrad_stride] gradient partial per tile
    int pgrad_stride;         // 7 * n_sources
    int want_residual;
    int live_cap;             // records that fit in the shared-memory stage (>= 1)
    int idx_cap;              // most image Gaussians of any exposure (kept-list capacity)
    int *err;                 // error word (bit 0: bulk-copy wait gave up)
    long long *pairs;         // optional: evaluated (pixel, Gaussian) pairs, or nullptr
    int *tile_cost = nullptr; // optional: [n_tiles] kept Gaussians x pixels, written per tile
    int test_extra_tx = 0;    // test of the error path only: bytes the staging wait
                              // expects beyond those copied, so that it runs out
};

// ------------------------------------------------------------ mbarrier + bulk copy
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait on an mbarrier phase.  Gives up after `limit` polls, records
// bit 0 in the error word and returns false; never spins forever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err) {
    const int limit = 1 << 22;
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(err, 1);
    return false;
}

// ------------------------------------------------------------ warp helpers
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Reduce 7 per-lane values across the warp; afterwards lane k (k < 7) holds
// the warp total of value k.  Uses 4+2+1+1+1 shuffles instead of 7*5.
__device__ __forceinline__ float warp_reduce7(float v[8], int lane) {
    // exchange 1: lanes < 16 keep 0..3, lanes >= 16 keep 4..7
    {
        const bool up = lane & 16;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float send = up ? v[i] : v[i + 4];
            const float keep = up ? v[i + 4] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
    }
    {
        const bool up = lane & 8;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const float send = up ? v[i] : v[i + 2];
            const float keep = up ? v[i + 2] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
        }
    }
    {
        const bool up = lane & 4;
        const float send = up ? v[0] : v[1];
        const float keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
    // value index held by this lane group: bits (16 -> 4, 8 -> 2, 4 -> 1)
    return v[0];
}
__device__ __forceinline__ int reduce7_index(int lane) {
    return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}

// ------------------------------------------------------------ shared layout
// Dynamic shared memory of the tile kernel:
//   [records live_cap x 128 B][kept indices idx_cap x 4 B][kept flags idx_cap x 4 B]
//   [per-warp source sums NW x stride x 4 B]
// Shared memory of one tile CTA: `live_cap` staged image-Gaussian records of
// GSTAGE floats, the kept list (one int per Gaussian of the exposure: local
// index << 2 | flags) and per-warp gradient sums.  (Reading the Jacobian half
// of the records from global memory instead halves the stage, but the
// exposure's records then miss L1 in the gradient epilogue; measured slower.)
constexpr int GSTAGE = GREC;
__host__ __device__ inline size_t tile_smem_layout_bytes(int nw, int live_cap, int idx_cap,
                                                         int stride) {
    return (size_t)live_cap * GSTAGE * 4 + (size_t)idx_cap * 4 + (size_t)nw * stride * 4;
}

// Stage the records of kept entries [c0, c0 + n) of an exposure (first record
// `gexp`) into `recs`, in list order, and wait for them.  Every thread of the
// CTA issues the bulk copies of its records (one 128-byte copy each); issued
// by one warp, the copies of a stage queued behind each other and the CTA
// spent about a fifth of each tile waiting for them.  Callers have finished
// reading `recs` (a barrier) before the call.
template <int NT>
__device__ __forceinline__ void stage_records(float *recs, const float *gexp, const int *kept,
                                              int c0, int n, int extra_tx, uint64_t *mbar,
                                              uint32_t &phase, int *err) {
    fence_proxy_async_smem();
    if (threadIdx.x == 0)
        mbar_arrive_expect_tx(mbar, (uint32_t)(n * GSTAGE * 4 + extra_tx));
    __syncthreads();  // the expected bytes are set before any copy can complete
    for (int i = threadIdx.x; i < n; i += NT)
        bulk_g2s(recs + (size_t)i * GSTAGE, gexp + (size_t)(kept[c0 + i] >> 2) * GREC,
                 GSTAGE * 4, mbar);
    mbar_wait_bounded(mbar, phase, err);
    phase ^= 1u;
}

// ------------------------------------------------------------ culling
// Minimum over the rectangle [x0,x1] x [y0,y1] of the exp-argument
// q(p) = (p-c)^T F (p-c): 0 if the centre is inside, else the smallest of the
// four edge minima (q is convex, so its minimum over the rectangle lies on the
// boundary; on an edge it is a clamped 1-D quadratic minimum).
__device__ __forceinline__ float rect_min_q(float4 bb, float xc, float yc, float fxx, float fxy,
                                            float fyy) {
    if (xc >= bb.x && xc <= bb.y && yc >= bb.z && yc <= bb.w) return 0.0f;
    float best = INFINITY;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const float dx = (e ? bb.y : bb.x) - xc;
        const float dy = fminf(fmaxf(-fxy * dx / fyy, bb.z - yc), bb.w - yc);
        best = fminf(best, dx * (fxx * dx + fxy * dy) + dy * (fyy * dy + fxy * dx));
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const float dy = (e ? bb.w : bb.z) - yc;
        const float dx = fminf(fmaxf(-fxy * dy / fxx, bb.x - xc), bb.y - xc);
        best = fminf(best, dx * (fxx * dx + fxy * dy) + dy * (fyy * dy + fxy * dx));
    }
    return best;
}

// Is an image Gaussian possibly within exp-argument 36 of some point of the
// tile box?  Conservative: cull only when the exact minimum, less a 2e-3
// relative + 2e-3 margin for float rounding, exceeds 36.  `a` and `b` are the
// record's first two float4 (-xc -xc -yc -yc, fxx fxx fxy fxy).
__device__ __forceinline__ bool keeps_tile(float4 a, float4 b, float fyy, float4 bb) {
    const float fxx = b.x, fxy = b.z;
    if (!(fxx > 0.0f && fyy > 0.0f)) return true;
    const float q = rect_min_q(bb, -a.x, -a.z, fxx, fxy, fyy);
    return !(q * (1.0f - 2.0e-3f) - 2.0e-3f > FPHO_MAX_EXP_ARG);
}

// ------------------------------------------------------------ per-Gaussian helpers
// Two packed operands from one 16-byte shared-memory load.
__device__ __forceinline__ void ld2(const float *p, v2 &a, v2 &b) {
    const ulonglong2 t = *reinterpret_cast<const ulonglong2 *>(p);
    a = t.x;
    b = t.y;
}

// Pass 1 for one Gaussian over the thread's KP pixel pairs: R -= amp G H.
template <int KP, bool CUT>
__device__ __forceinline__ void residual_pairs(const v2 (&X)[KP], const v2 (&Y)[KP], v2 (&R)[KP],
                                               v2 NXC, v2 NYC, v2 FXX, v2 FXY, v2 FYY, v2 HA,
                                               v2 HB, v2 KEXP2, v2 KEXPLO2) {
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const v2 DX = add2(X[j], NXC), DY = add2(Y[j], NYC);
        const v2 VX = fma2(FXY, DY, mul2(FXX, DX));
        const v2 VY = fma2(FXY, DX, mul2(FYY, DY));
        const v2 Q = fma2(DY, VY, mul2(DX, VX));
        // the residual needs an unbiased exponential (see exp_neg_half)
        v2 Gp = exp_neg_half(Q, KEXP2, KEXPLO2);
        if (CUT) {
            float g0, g1, q0, q1;
            unpk(Gp, g0, g1);
            unpk(Q, q0, q1);
            Gp = pk(q0 > FPHO_MAX_EXP_ARG ? 0.0f : g0, q1 > FPHO_MAX_EXP_ARG ? 0.0f : g1);
        }
        const v2 S = fma2(VY, VY, mul2(VX, VX));
        R[j] = fma2(fma2(S, HA, HB), Gp, R[j]);  // fma(S, -amp/24, -amp c0) = -amp H
    }
}

// Pass 1 for two consecutive kept Gaussians a, b at once: their exponentials
// are independent and interleave, and R is updated with a's term and then
// b's, exactly as two calls of residual_pairs in order would.  The
// exp-argument cut is applied to both; for a Gaussian without FLAG_CUT no
// weighted pixel of the tile reaches 36 (and with a residual output every
// pixel is in the tile box), so the cut changes nothing there.  (Skipping the
// cut for pairs without FLAG_CUT, as a compile-time branch, measured slower:
// it raised the split kernel's registers from 128 to 180.)
template <int KP>
__device__ __forceinline__ void residual_pairs2(const v2 (&X)[KP], const v2 (&Y)[KP], v2 (&R)[KP],
                                                const float *ra, const float *rb, v2 CM24,
                                                v2 KEXP2, v2 KEXPLO2) {
    v2 NXa, NYa, FXXa, FXYa, FYYa, AMPa, HBa, C0a;
    v2 NXb, NYb, FXXb, FXYb, FYYb, AMPb, HBb, C0b;
    ld2(ra + R_NXC, NXa, NYa);
    ld2(ra + R_FXX, FXXa, FXYa);
    ld2(ra + R_FYY, FYYa, AMPa);
    ld2(ra + R_HB, HBa, C0a);
    ld2(rb + R_NXC, NXb, NYb);
    ld2(rb + R_FXX, FXXb, FXYb);
    ld2(rb + R_FYY, FYYb, AMPb);
    ld2(rb + R_HB, HBb, C0b);
    const v2 HAa = mul2(AMPa, CM24), HAb = mul2(AMPb, CM24);
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const v2 DXa = add2(X[j], NXa), DYa = add2(Y[j], NYa);
        const v2 DXb = add2(X[j], NXb), DYb = add2(Y[j], NYb);
        const v2 VXa = fma2(FXYa, DYa, mul2(FXXa, DXa));
        const v2 VXb = fma2(FXYb, DYb, mul2(FXXb, DXb));
        const v2 VYa = fma2(FXYa, DXa, mul2(FYYa, DYa));
        const v2 VYb = fma2(FXYb, DXb, mul2(FYYb, DYb));
        const v2 Qa = fma2(DYa, VYa, mul2(DXa, VXa));
        const v2 Qb = fma2(DYb, VYb, mul2(DXb, VXb));
        v2 Ga = exp_neg_half(Qa, KEXP2, KEXPLO2);
        v2 Gb = exp_neg_half(Qb, KEXP2, KEXPLO2);
        {
            float g0, g1, q0, q1;
            unpk(Ga, g0, g1);
            unpk(Qa, q0, q1);
            Ga = pk(q0 > FPHO_MAX_EXP_ARG ? 0.0f : g0, q1 > FPHO_MAX_EXP_ARG ? 0.0f : g1);
            unpk(Gb, g0, g1);
            unpk(Qb, q0, q1);
            Gb = pk(q0 > FPHO_MAX_EXP_ARG ? 0.0f : g0, q1 > FPHO_MAX_EXP_ARG ? 0.0f : g1);
        }
        const v2 Sa = fma2(VYa, VYa, mul2(VXa, VXa));
        const v2 Sb = fma2(VYb, VYb, mul2(VXb, VXb));
        R[j] = fma2(fma2(Sa, HAa, HBa), Ga, R[j]);
        R[j] = fma2(fma2(Sb, HAb, HBb), Gb, R[j]);
    }
}

// Pass 1 in the reference's float arithmetic, for the exact-residual mode:
// ComputeResidualImage (forcepho/src/common_kernel.cc:57-83) operation by
// operation, each rounded once (no multiply-add contraction), the
// exp-argument test before the exponential, H with its division by 24, and
// exp evaluated in double and rounded once to float -- the correctly rounded
// float exp wherever double exp's error does not straddle a float rounding
// boundary.  Pixels of the pair are taken one at a time.
template <int KP>
__device__ __forceinline__ void residual_exact(const v2 (&X)[KP], const v2 (&Y)[KP], v2 (&R)[KP],
                                               const float *rec) {
    const float nxc = rec[R_NXC], nyc = rec[R_NYC];
    const float fxx = rec[R_FXX], fxy = rec[R_FXY], fyy = rec[R_FYY], amp = rec[R_AMP];
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        float xs[2], ys[2], rs[2];
        unpk(X[j], xs[0], xs[1]);
        unpk(Y[j], ys[0], ys[1]);
        unpk(R[j], rs[0], rs[1]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float dx = __fadd_rn(xs[h], nxc);  // xp - xcen (nxc = -xcen exactly)
            const float dy = __fadd_rn(ys[h], nyc);
            const float vx = __fadd_rn(__fmul_rn(fxx, dx), __fmul_rn(fxy, dy));
            const float vy = __fadd_rn(__fmul_rn(fyy, dy), __fmul_rn(fxy, dx));
            const float ea = __fadd_rn(__fmul_rn(dx, vx), __fmul_rn(dy, vy));
            if (ea > FPHO_MAX_EXP_ARG) continue;
            const float gp = (float)exp((double)__fmul_rn(-0.5f, ea));
            const float t = __fsub_rn(__fsub_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)),
                                                fxx), fyy);
            const float H = __fadd_rn(1.0f, __fdiv_rn(t, 24.0f));
            rs[h] = __fsub_rn(rs[h], __fmul_rn(__fmul_rn(amp, gp), H));
        }
        R[j] = pk(rs[0], rs[1]);
    }
}

// Pass 2 for one Gaussian over the thread's KP pixel pairs: the twelve sums
// from which the model's derivatives w.r.t. (A, x, y, fxx, fyy, fxy) follow
// (W = -2 r ie^2 G, H the pixel-integral correction, d = pixel - centre,
// v = F d): sum W H, sum W H v, sum W v, sum W H d d^T, sum W, and sum W d d^T.
// The epilogue forms sum W d.v terms from sum W d d^T and F once per
// Gaussian (d_x v_x = fxx dx^2 + fxy dx dy, and so on), which is one packed
// instruction per pixel pair cheaper than summing them per pixel; the
// products dx^2, dx dy, dy^2 are formed once and weighted by both W H and W.
struct GradSums {
    v2 A, HVx, HVy, Vx, Vy, HXX, HXY, HYY, W, WXX, WXY, WYY;
};
template <int KP, bool CUT>
__device__ __forceinline__ void gradient_pairs(const v2 (&X)[KP], const v2 (&Y)[KP],
                                               const v2 (&R2)[KP], v2 NXC, v2 NYC, v2 FXX,
                                               v2 FXY, v2 FYY, v2 C0, v2 C24, v2 KEXP2,
                                               GradSums &s) {
    s = GradSums{0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const v2 DX = add2(X[j], NXC), DY = add2(Y[j], NYC);
        const v2 VX = fma2(FXY, DY, mul2(FXX, DX));
        const v2 VY = fma2(FXY, DX, mul2(FYY, DY));
        const v2 T1 = mul2(DX, VX);
        const v2 Q = fma2(DY, VY, T1);
        float e0, e1;
        unpk(mul2(Q, KEXP2), e0, e1);
        float g0 = ex2f(e0), g1 = ex2f(e1);
        if (CUT) {
            float q0, q1;
            unpk(Q, q0, q1);
            g0 = q0 > FPHO_MAX_EXP_ARG ? 0.0f : g0;
            g1 = q1 > FPHO_MAX_EXP_ARG ? 0.0f : g1;
        }
        const v2 S = fma2(VY, VY, mul2(VX, VX));
        const v2 H = fma2(S, C24, C0);
        const v2 W = mul2(R2[j], pk(g0, g1));
        const v2 WH = mul2(W, H);
        s.A = add2(s.A, WH);
        s.HVx = fma2(WH, VX, s.HVx);
        s.HVy = fma2(WH, VY, s.HVy);
        s.Vx = fma2(W, VX, s.Vx);
        s.Vy = fma2(W, VY, s.Vy);
        const v2 DXX = mul2(DX, DX), DXY = mul2(DX, DY), DYY = mul2(DY, DY);
        s.HXX = fma2(WH, DXX, s.HXX);
        s.HXY = fma2(WH, DXY, s.HXY);
        s.HYY = fma2(WH, DYY, s.HYY);
        s.W = add2(s.W, W);
        s.WXX = fma2(W, DXX, s.WXX);
        s.WXY = fma2(W, DXY, s.WXY);
        s.WYY = fma2(W, DYY, s.WYY);
    }
}

// Pass 2 for two consecutive kept Gaussians a, b at once (independent
// exponentials interleave); each set of sums is formed in the same order as
// by gradient_pairs, and the cut is applied to both (see residual_pairs2).
template <int KP>
__device__ __forceinline__ void gradient_pairs2(const v2 (&X)[KP], const v2 (&Y)[KP],
                                                const v2 (&R2)[KP], const float *ra,
                                                const float *rb, v2 C24, v2 KEXP2, GradSums &sa,
                                                GradSums &sb) {
    v2 NXa, NYa, FXXa, FXYa, FYYa, AMPa, HBa, C0a;
    v2 NXb, NYb, FXXb, FXYb, FYYb, AMPb, HBb, C0b;
    ld2(ra + R_NXC, NXa, NYa);
    ld2(ra + R_FXX, FXXa, FXYa);
    ld2(ra + R_FYY, FYYa, AMPa);
    ld2(ra + R_HB, HBa, C0a);
    ld2(rb + R_NXC, NXb, NYb);
    ld2(rb + R_FXX, FXXb, FXYb);
    ld2(rb + R_FYY, FYYb, AMPb);
    ld2(rb + R_HB, HBb, C0b);
    sa = GradSums{0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
    sb = sa;
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const v2 DXa = add2(X[j], NXa), DYa = add2(Y[j], NYa);
        const v2 DXb = add2(X[j], NXb), DYb = add2(Y[j], NYb);
        const v2 VXa = fma2(FXYa, DYa, mul2(FXXa, DXa));
        const v2 VXb = fma2(FXYb, DYb, mul2(FXXb, DXb));
        const v2 VYa = fma2(FXYa, DXa, mul2(FYYa, DYa));
        const v2 VYb = fma2(FXYb, DXb, mul2(FYYb, DYb));
        const v2 T1a = mul2(DXa, VXa), T1b = mul2(DXb, VXb);
        const v2 Qa = fma2(DYa, VYa, T1a), Qb = fma2(DYb, VYb, T1b);
        float ea0, ea1, eb0, eb1, qa0, qa1, qb0, qb1;
        unpk(mul2(Qa, KEXP2), ea0, ea1);
        unpk(mul2(Qb, KEXP2), eb0, eb1);
        unpk(Qa, qa0, qa1);
        unpk(Qb, qb0, qb1);
        const float ga0 = qa0 > FPHO_MAX_EXP_ARG ? 0.0f : ex2f(ea0);
        const float ga1 = qa1 > FPHO_MAX_EXP_ARG ? 0.0f : ex2f(ea1);
        const float gb0 = qb0 > FPHO_MAX_EXP_ARG ? 0.0f : ex2f(eb0);
        const float gb1 = qb1 > FPHO_MAX_EXP_ARG ? 0.0f : ex2f(eb1);
        const v2 Sa = fma2(VYa, VYa, mul2(VXa, VXa)), Sb = fma2(VYb, VYb, mul2(VXb, VXb));
        const v2 Ha = fma2(Sa, C24, C0a), Hb = fma2(Sb, C24, C0b);
        const v2 Wa = mul2(R2[j], pk(ga0, ga1)), Wb = mul2(R2[j], pk(gb0, gb1));
        const v2 WHa = mul2(Wa, Ha), WHb = mul2(Wb, Hb);
        sa.A = add2(sa.A, WHa);
        sb.A = add2(sb.A, WHb);
        sa.HVx = fma2(WHa, VXa, sa.HVx);
        sb.HVx = fma2(WHb, VXb, sb.HVx);
        sa.HVy = fma2(WHa, VYa, sa.HVy);
        sb.HVy = fma2(WHb, VYb, sb.HVy);
        sa.Vx = fma2(Wa, VXa, sa.Vx);
        sb.Vx = fma2(Wb, VXb, sb.Vx);
        sa.Vy = fma2(Wa, VYa, sa.Vy);
        sb.Vy = fma2(Wb, VYb, sb.Vy);
        const v2 DXXa = mul2(DXa, DXa), DXYa = mul2(DXa, DYa), DYYa = mul2(DYa, DYa);
        const v2 DXXb = mul2(DXb, DXb), DXYb = mul2(DXb, DYb), DYYb = mul2(DYb, DYb);
        sa.HXX = fma2(WHa, DXXa, sa.HXX);
        sb.HXX = fma2(WHb, DXXb, sb.HXX);
        sa.HXY = fma2(WHa, DXYa, sa.HXY);
        sb.HXY = fma2(WHb, DXYb, sb.HXY);
        sa.HYY = fma2(WHa, DYYa, sa.HYY);
        sb.HYY = fma2(WHb, DYYb, sb.HYY);
        sa.W = add2(sa.W, Wa);
        sb.W = add2(sb.W, Wb);
        sa.WXX = fma2(Wa, DXXa, sa.WXX);
        sb.WXX = fma2(Wb, DXXb, sb.WXX);
        sa.WXY = fma2(Wa, DXYa, sa.WXY);
        sb.WXY = fma2(Wb, DXYb, sb.WXY);
        sa.WYY = fma2(Wa, DYYa, sa.WYY);
        sb.WYY = fma2(Wb, DYYb, sb.WYY);
    }
}

__device__ __forceinline__ float lanesum(v2 v) {
    float a, b;
    unpk(v, a, b);
    return a + b;
}

// kept-list flag bits (the low two bits of each entry)
constexpr int FLAG_CUT = 1;        // the exp-argument can exceed 36 inside the tile
constexpr int FLAG_LAST_SRC = 2;   // last kept Gaussian of its source in the chunk

// ------------------------------------------------------------ tile scan
// One scan of the exposure's image Gaussians [g0, g1): the ordered list of
// those that can reach the tile (box overlap, then the exact minimum of the
// exp-argument over the tile box `bb`), each entry (local index << 2 | flags)
// with FLAG_CUT when the exp-argument can exceed 36 inside the tile (its
// maximum over the box is at a corner) and FLAG_LAST_SRC on the last kept
// Gaussian of each source.  Returns the number kept; ends with the list
// visible to the whole CTA.
template <int NT>
__device__ __forceinline__ int scan_tile(const TileArgs &A, float4 bb, int g0, int g1, int npsf,
                                         int *kept) {
    constexpr int NW = NT / 32;
    __shared__ int s_cnt[NW];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int n_live = 0;
    for (int base = g0; base < g1; base += NT) {
        const int idx = base + tid;
        bool live = false;
        int flag = 0;
        if (idx < g1) {
            const float4 gb = A.gbox[idx];
            live = !(gb.y < bb.x || gb.x > bb.y || gb.w < bb.z || gb.z > bb.w);
            if (live) {
                const float *r = A.gtab + (size_t)idx * GREC;
                const float4 ra = *reinterpret_cast<const float4 *>(r);
                const float4 rb = *reinterpret_cast<const float4 *>(r + 4);
                live = keeps_tile(ra, rb, r[R_FYY], bb);
                const float nxc = r[R_NXC], nyc = r[R_NYC];
                const float fxx = r[R_FXX], fxy = r[R_FXY], fyy = r[R_FYY];
                float qmax = 0.0f;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float dx = ((c & 1) ? bb.y : bb.x) + nxc;
                    const float dy = ((c & 2) ? bb.w : bb.z) + nyc;
                    qmax = fmaxf(qmax, dx * (fxx * dx + fxy * dy) + dy * (fyy * dy + fxy * dx));
                }
                flag = (qmax * (1.0f + CULL_REL) + CULL_ABS >= FPHO_MAX_EXP_ARG) ? FLAG_CUT : 0;
            }
        }
        const unsigned ball = __ballot_sync(0xffffffffu, live);
        if (lane == 0) s_cnt[warp] = __popc(ball);
        __syncthreads();
        int off = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            off += (w < warp) ? s_cnt[w] : 0;
            tot += s_cnt[w];
        }
        if (live) {
            const int at = n_live + off + __popc(ball & ((1u << lane) - 1u));
            kept[at] = ((idx - g0) << 2) | flag;
        }
        n_live += tot;
        __syncthreads();
    }
    // last kept Gaussian of each source (sources are contiguous in the list)
    for (int i = tid; i < n_live; i += NT) {
        const int src = (kept[i] >> 2) / npsf;
        const int nxt = (i + 1 < n_live) ? (kept[i + 1] >> 2) / npsf : -1;
        if (nxt != src) kept[i] |= FLAG_LAST_SRC;
    }
    __syncthreads();
    return n_live;
}

// ------------------------------------------------------------ the tile body
// GRAD = false runs the residual pass and chi2 only (no gradient pass, no
// gradient partials written).  EXACT = true runs the residual pass in the
// reference's float arithmetic (residual_exact) instead of the packed pass.
template <int NT, int K, bool GRAD = true, bool EXACT = false>
__device__ __forceinline__ void tile_body(const TileArgs &A, int tile, unsigned char *smem,
                                          uint64_t *mbar, uint32_t &phase) {
    static_assert(K % 2 == 0, "pixels per thread must be even (packed pairs)");
    constexpr int NW = NT / 32;
    constexpr int KP = K / 2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cap = A.live_cap;
    const int stride = A.pgrad_stride;

    float *recs = reinterpret_cast<float *>(smem);
    // kept list: exposure-local Gaussian index << 2 | FLAG_* bits
    int *kept = reinterpret_cast<int *>(smem + (size_t)cap * GSTAGE * 4);
    float *wacc = reinterpret_cast<float *>(kept + A.idx_cap);

    __shared__ double s_chi2[NW];
    __shared__ int s_any_weight;

    const TileDesc td = A.tiles[tile];
    const float4 bb = A.want_residual ? A.tbox_all[tile] : A.tbox_w[tile];
    const int g0 = A.pv.gauss_start[td.exposure];
    const int g1 = A.pv.gauss_start[td.exposure + 1];
    const int npsf = A.pv.exp_npsf[td.exposure];

    for (int j = tid; j < NW * stride; j += NT) wacc[j] = 0.0f;

    // ---- this thread's pixels: pair j holds local pixels tid + 2j*NT and tid + (2j+1)*NT
    const float xmid = 0.5f * (bb.x + bb.y), ymid = 0.5f * (bb.z + bb.w);
    v2 X[KP], Y[KP], R[KP], R2[KP];
    float D[K], IE[K];
    int any_w = 0;
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        float xs[2], ys[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int li = tid + (2 * j + h) * NT;
            const bool ok = li < td.count;
            const int pix = td.pix_begin + (ok ? li : 0);
            xs[h] = ok ? A.pv.xpix[pix] : xmid;
            ys[h] = ok ? A.pv.ypix[pix] : ymid;
            D[2 * j + h] = ok ? A.pv.data[pix] : 0.0f;
            IE[2 * j + h] = ok ? A.pv.ierr[pix] : 0.0f;
            any_w |= (IE[2 * j + h] != 0.0f);
        }
        X[j] = pk(xs[0], xs[1]);
        Y[j] = pk(ys[0], ys[1]);
        R[j] = pk(D[2 * j], D[2 * j + 1]);
    }
    if (tid == 0) s_any_weight = 0;

    // ---- the ordered list of kept image Gaussians
    const int n_live = scan_tile<NT>(A, bb, g0, g1, npsf, kept);
    if (any_w) s_any_weight = 1;
    __syncthreads();
    const bool tile_has_weight = s_any_weight != 0;

    // ---- stage kept records [c0, c0 + n) into shared memory with bulk copies
    auto stage = [&](int c0, int n) {
        stage_records<NT>(recs, A.gtab + (size_t)g0 * GREC, kept, c0, n, A.test_extra_tx, mbar,
                          phase, A.err);
    };

    const v2 KEXP2 = pk1(KEXP), KEXPLO2 = pk1(KEXP_LO);
    const v2 CM24 = pk1(-1.0f / 24.0f), C24 = pk1(1.0f / 24.0f);
    const int n_chunks = (n_live + cap - 1) / cap;

    // ------------------------------------------------------------ pass 1
    for (int c = 0; c < n_chunks; ++c) {
        const int c0 = c * cap, n = min(cap, n_live - c0);
        if (c > 0) __syncthreads();  // previous chunk fully consumed
        stage(c0, n);
        if (EXACT) {
            for (int i = 0; i < n; ++i) residual_exact<KP>(X, Y, R, recs + (size_t)i * GSTAGE);
            continue;
        }
        int i = 0;
        for (; i + 1 < n; i += 2)
            residual_pairs2<KP>(X, Y, R, recs + (size_t)i * GSTAGE, recs + (size_t)(i + 1) * GSTAGE,
                                CM24, KEXP2, KEXPLO2);
        for (; i < n; ++i) {
            const float *r = recs + (size_t)i * GSTAGE;
            v2 NXC, NYC, FXX, FXY, FYY, AMP, HB, C0;
            ld2(r + R_NXC, NXC, NYC);
            ld2(r + R_FXX, FXX, FXY);
            ld2(r + R_FYY, FYY, AMP);
            ld2(r + R_HB, HB, C0);
            const v2 HA = mul2(AMP, CM24);
            if (kept[c0 + i] & FLAG_CUT)
                residual_pairs<KP, true>(X, Y, R, NXC, NYC, FXX, FXY, FYY, HA, HB, KEXP2, KEXPLO2);
            else
                residual_pairs<KP, false>(X, Y, R, NXC, NYC, FXX, FXY, FYY, HA, HB, KEXP2, KEXPLO2);
        }
    }

    // ---- residual store, chi2 (double) and the per-pixel adjoint -2 r ie^2
    double chi2 = 0.0;
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        float r[2];
        unpk(R[j], r[0], r[1]);
        float r2v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = 2 * j + h;
            const int li = tid + k * NT;
            if (A.want_residual && li < td.count) A.pv.residual[td.pix_begin + li] = r[h];
            const float ie = IE[k];
            const float rie = r[h] * ie;
            const float die = D[k] * ie;
            double c = ((double)rie - (double)die);
            c *= ((double)rie + (double)die);
            chi2 += (ie != 0.0f) ? c : 0.0;
            r2v[h] = (ie != 0.0f) ? -2.0f * (rie * ie) : 0.0f;
        }
        R2[j] = pk(r2v[0], r2v[1]);
    }
    chi2 = warp_sum_d(chi2);
    if (lane == 0) s_chi2[warp] = chi2;

    // ------------------------------------------------------------ pass 2
    // Chunks in reverse order: the last chunk of pass 1 is still staged.
    if (GRAD && tile_has_weight) {
        float P[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int c = n_chunks - 1; c >= 0; --c) {
            const int c0 = c * cap, n = min(cap, n_live - c0);
            if (c != n_chunks - 1) {
                __syncthreads();
                stage(c0, n);
            }
            // the Jacobian epilogue of one Gaussian, in list order
            auto epilogue = [&](const float *r, int flag, const GradSums &s, bool last) {
                const float4 *rj = reinterpret_cast<const float4 *>(r + R_JA_FLUX);
                // image-space gradient of this Gaussian over the thread's pixels
                // (amp factors are folded into the Jacobian rows), in scalars
                const float fxx = r[R_FXX], fxy = r[R_FXY], fyy = r[R_FYY];
                const float sVx = lanesum(s.Vx), sVy = lanesum(s.Vy), sW = lanesum(s.W);
                const float gA = lanesum(s.A);
                const float gx = lanesum(s.HVx) - (fxx * sVx + fxy * sVy) * (1.0f / 12.0f);
                const float gy = lanesum(s.HVy) - (fxy * sVx + fyy * sVy) * (1.0f / 12.0f);
                // sum W d.v terms from sum W d d^T: dx vx, dy vy, dx vy + dy vx
                const float wxx = lanesum(s.WXX), wxy = lanesum(s.WXY), wyy = lanesum(s.WYY);
                const float t1 = fxx * wxx + fxy * wxy;
                const float t2 = fyy * wyy + fxy * wxy;
                const float t3 = fxy * (wxx + wyy) + (fxx + fyy) * wxy;
                const float gfxx = t1 * (1.0f / 12.0f) - 0.5f * lanesum(s.HXX) -
                                   sW * (1.0f / 24.0f);
                const float gfyy = t2 * (1.0f / 12.0f) - 0.5f * lanesum(s.HYY) -
                                   sW * (1.0f / 24.0f);
                const float gfxy = t3 * (1.0f / 12.0f) - lanesum(s.HXY);
                const float4 j0 = rj[0], j1 = rj[1], j2 = rj[2], j3 = rj[3];
                P[0] = fmaf(j0.x, gA, P[0]);
                P[1] = fmaf(j1.z, gy, fmaf(j1.y, gx, P[1]));
                P[2] = fmaf(j2.x, gy, fmaf(j1.w, gx, P[2]));
                P[3] = fmaf(j2.w, gfyy, fmaf(j2.z, gfxy, fmaf(j2.y, gfxx, fmaf(j0.y, gA, P[3]))));
                P[4] = fmaf(j3.z, gfyy, fmaf(j3.y, gfxy, fmaf(j3.x, gfxx, fmaf(j0.z, gA, P[4]))));
                P[5] = fmaf(j0.w, gA, P[5]);
                P[6] = fmaf(j1.x, gA, P[6]);
                // flush at a source boundary or at the end of the chunk
                if ((flag & FLAG_LAST_SRC) || last) {
                    // the index comes from the staged record: bounded, so that
                    // a stage a timed-out wait left stale cannot write outside
                    // the sums (the error word already marks the evaluation)
                    const int src = min((unsigned)__float_as_int(j3.w),
                                        (unsigned)(A.pv.n_sources - 1));
                    float v[8] = {P[0], P[1], P[2], P[3], P[4], P[5], P[6], 0.0f};
#pragma unroll
                    for (int k = 0; k < 7; ++k) P[k] = 0.0f;
                    const float tot = warp_reduce7(v, lane);
                    const int k = reduce7_index(lane);
                    if ((lane & 3) == 0 && k < 7) wacc[warp * stride + src * 7 + k] += tot;
                }
            };
            int i = 0;
            for (; i + 1 < n; i += 2) {
                const float *ra = recs + (size_t)i * GSTAGE, *rb = ra + GSTAGE;
                GradSums sa, sb;
                gradient_pairs2<KP>(X, Y, R2, ra, rb, C24, KEXP2, sa, sb);
                epilogue(ra, kept[c0 + i], sa, false);
                epilogue(rb, kept[c0 + i + 1], sb, i + 1 == n - 1);
            }
            for (; i < n; ++i) {
                const float *r = recs + (size_t)i * GSTAGE;
                v2 NXC, NYC, FXX, FXY, FYY, AMP, HB, C0;
                ld2(r + R_NXC, NXC, NYC);
                ld2(r + R_FXX, FXX, FXY);
                ld2(r + R_FYY, FYY, AMP);
                ld2(r + R_HB, HB, C0);
                const int flag = kept[c0 + i];
                GradSums s;
                if (flag & FLAG_CUT)
                    gradient_pairs<KP, true>(X, Y, R2, NXC, NYC, FXX, FXY, FYY, C0, C24, KEXP2, s);
                else
                    gradient_pairs<KP, false>(X, Y, R2, NXC, NYC, FXX, FXY, FYY, C0, C24, KEXP2, s);
                epilogue(r, flag, s, i == n - 1);
            }
        }
    }
    __syncthreads();

    // ---- tile partials (fixed-order sums)
    if (tid == 0) {
        double c = 0.0;
#pragma unroll
        for (int w = 0; w < NW; ++w) c += s_chi2[w];
        A.pchi2[tile] = c;
    }
    for (int j = tid; GRAD && j < stride; j += NT) {
        float v = 0.0f;
#pragma unroll
        for (int w = 0; w < NW; ++w) v += wacc[w * stride + j];
        A.pgrad[(size_t)tile * stride + j] = v;
    }
    if (A.tile_cost && tid == 0) A.tile_cost[tile] = n_live * td.count;
    if (A.pairs && tid == 0) atomicAdd(reinterpret_cast<unsigned long long *>(A.pairs),
                                       (unsigned long long)((long long)n_live * td.count));
}

// ------------------------------------------------------------ split tile body
// A tile of 32*K pixels evaluated by NW warps that share the tile's kept
// Gaussians: every warp holds all of the tile's pixels (lane l holds pixels
// l, l+32, ..., K per thread, as K/2 packed pairs) and takes a contiguous
// 1/NW of each staged chunk of kept Gaussians.
//   pass 1: each warp sums -model over its Gaussians; the NW partial models
//           are added to the data in warp order through shared memory, so
//           every warp holds the same residual bit for bit;
//   chi2:   warp 0, in double, as tile_body;
//   pass 2: each warp forms the gradient of its Gaussians (12 packed sums per
//           Gaussian, Jacobian applied once per Gaussian per thread) and
//           flushes per-source sums into its own shared-memory row; the rows
//           are added in warp order at the end.
// Against tile_body with NT = 32 NW threads and K' = K / NW pixels per thread
// on the same tile, each thread does the per-Gaussian work (record loads,
// exp-argument set-up, Jacobian epilogue) for NW times as many pixels, and a
// CTA slot takes NW times fewer pixels per Gaussian, so tiles stay small (good
// culling) while a launch has more tiles per resident CTA (a shorter tail).
// Results are deterministic; the residual is summed in a different order from
// tile_body's, so the two agree to rounding, not bit for bit.
__host__ __device__ inline size_t split_smem_layout_bytes(int nw, int k, int live_cap, int idx_cap,
                                                         int stride) {
    return (size_t)live_cap * GSTAGE * 4 + (size_t)idx_cap * 4 + (size_t)nw * stride * 4 +
           (size_t)nw * 32 * k * 4;
}

template <int NW, int K, bool GRAD = true>
__device__ __forceinline__ void tile_body_split(const TileArgs &A, int tile, unsigned char *smem,
                                                uint64_t *mbar, uint32_t &phase) {
    static_assert(K % 2 == 0, "pixels per thread must be even (packed pairs)");
    constexpr int NT = 32 * NW;
    constexpr int KP = K / 2;
    constexpr int TP = 32 * K;  // pixels per tile
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cap = A.live_cap;
    const int stride = A.pgrad_stride;

    float *recs = reinterpret_cast<float *>(smem);
    int *kept = reinterpret_cast<int *>(smem + (size_t)cap * GSTAGE * 4);
    float *wacc = reinterpret_cast<float *>(kept + A.idx_cap);
    float *part = wacc + (size_t)NW * stride;  // [NW][TP] partial models

    __shared__ double s_chi2;
    __shared__ int s_any_weight;

    const TileDesc td = A.tiles[tile];
    const float4 bb = A.want_residual ? A.tbox_all[tile] : A.tbox_w[tile];
    const int g0 = A.pv.gauss_start[td.exposure];
    const int g1 = A.pv.gauss_start[td.exposure + 1];
    const int npsf = A.pv.exp_npsf[td.exposure];

    for (int j = tid; j < NW * stride; j += NT) wacc[j] = 0.0f;

    // ---- the tile's pixels, in every warp: pair j holds pixels lane + 64j, lane + 64j + 32
    const float xmid = 0.5f * (bb.x + bb.y), ymid = 0.5f * (bb.z + bb.w);
    v2 X[KP], Y[KP], R[KP];
    int any_w = 0;
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        float xs[2], ys[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int li = lane + (2 * j + h) * 32;
            const bool ok = li < td.count;
            const int pix = td.pix_begin + (ok ? li : 0);
            xs[h] = ok ? A.pv.xpix[pix] : xmid;
            ys[h] = ok ? A.pv.ypix[pix] : ymid;
            any_w |= ok && (A.pv.ierr[pix] != 0.0f);
        }
        X[j] = pk(xs[0], xs[1]);
        Y[j] = pk(ys[0], ys[1]);
        R[j] = 0ull;  // -model of this warp's Gaussians
    }
    if (tid == 0) s_any_weight = 0;

    const int n_live = scan_tile<NT>(A, bb, g0, g1, npsf, kept);
    if (any_w) s_any_weight = 1;
    __syncthreads();
    const bool tile_has_weight = s_any_weight != 0;

    auto stage = [&](int c0, int n) {
        stage_records<NT>(recs, A.gtab + (size_t)g0 * GREC, kept, c0, n, A.test_extra_tx, mbar,
                          phase, A.err);
    };
    // this warp's share [i0, i1) of a chunk of n records: contiguous, even
    // lengths (two Gaussians per step)
    auto share = [&](int n, int &i0, int &i1) {
        const int per = 2 * ((n + 2 * NW - 1) / (2 * NW));
        i0 = min(n, warp * per);
        i1 = min(n, i0 + per);
    };

    const v2 KEXP2 = pk1(KEXP), KEXPLO2 = pk1(KEXP_LO);
    const v2 CM24 = pk1(-1.0f / 24.0f), C24 = pk1(1.0f / 24.0f);
    const int n_chunks = (n_live + cap - 1) / cap;

    // ------------------------------------------------------------ pass 1
    for (int c = 0; c < n_chunks; ++c) {
        const int c0 = c * cap, n = min(cap, n_live - c0);
        if (c > 0) __syncthreads();
        stage(c0, n);
        int i0, i1;
        share(n, i0, i1);
        int i = i0;
        for (; i + 1 < i1; i += 2)
            residual_pairs2<KP>(X, Y, R, recs + (size_t)i * GSTAGE, recs + (size_t)(i + 1) * GSTAGE,
                                CM24, KEXP2, KEXPLO2);
        for (; i < i1; ++i) {
            const float *r = recs + (size_t)i * GSTAGE;
            v2 NXC, NYC, FXX, FXY, FYY, AMP, HB, C0;
            ld2(r + R_NXC, NXC, NYC);
            ld2(r + R_FXX, FXX, FXY);
            ld2(r + R_FYY, FYY, AMP);
            ld2(r + R_HB, HB, C0);
            const v2 HA = mul2(AMP, CM24);
            if (kept[c0 + i] & FLAG_CUT)
                residual_pairs<KP, true>(X, Y, R, NXC, NYC, FXX, FXY, FYY, HA, HB, KEXP2, KEXPLO2);
            else
                residual_pairs<KP, false>(X, Y, R, NXC, NYC, FXX, FXY, FYY, HA, HB, KEXP2, KEXPLO2);
        }
    }

    // ---- the residual: data plus the warps' partial (negative) models, in warp order
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        float m0, m1;
        unpk(R[j], m0, m1);
        part[warp * TP + lane + 64 * j] = m0;
        part[warp * TP + lane + 64 * j + 32] = m1;
    }
    __syncthreads();
    v2 R2[KP];
    double chi2 = 0.0;
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        float r2v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int li = lane + (2 * j + h) * 32;
            const bool ok = li < td.count;
            const int pix = td.pix_begin + (ok ? li : 0);
            const float d = ok ? A.pv.data[pix] : 0.0f;
            const float ie = ok ? A.pv.ierr[pix] : 0.0f;
            float r = d;
#pragma unroll
            for (int w = 0; w < NW; ++w) r += part[w * TP + li];
            if (warp == 0) {
                if (A.want_residual && ok) A.pv.residual[pix] = r;
                const float rie = r * ie, die = d * ie;
                double c = ((double)rie - (double)die);
                c *= ((double)rie + (double)die);
                chi2 += (ie != 0.0f) ? c : 0.0;
            }
            r2v[h] = (ie != 0.0f) ? -2.0f * ((r * ie) * ie) : 0.0f;
        }
        R2[j] = pk(r2v[0], r2v[1]);
    }
    if (warp == 0) {
        chi2 = warp_sum_d(chi2);
        if (lane == 0) s_chi2 = chi2;
    }

    // ------------------------------------------------------------ pass 2
    if (GRAD && tile_has_weight) {
        float P[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int c = n_chunks - 1; c >= 0; --c) {
            const int c0 = c * cap, n = min(cap, n_live - c0);
            if (c != n_chunks - 1) {
                __syncthreads();
                stage(c0, n);
            }
            int i0, i1;
            share(n, i0, i1);
            auto epilogue = [&](const float *r, int flag, const GradSums &s, bool last) {
                const float4 *rj = reinterpret_cast<const float4 *>(r + R_JA_FLUX);
                const float fxx = r[R_FXX], fxy = r[R_FXY], fyy = r[R_FYY];
                const float sVx = lanesum(s.Vx), sVy = lanesum(s.Vy), sW = lanesum(s.W);
                const float gA = lanesum(s.A);
                const float gx = lanesum(s.HVx) - (fxx * sVx + fxy * sVy) * (1.0f / 12.0f);
                const float gy = lanesum(s.HVy) - (fxy * sVx + fyy * sVy) * (1.0f / 12.0f);
                // sum W d.v terms from sum W d d^T: dx vx, dy vy, dx vy + dy vx
                const float wxx = lanesum(s.WXX), wxy = lanesum(s.WXY), wyy = lanesum(s.WYY);
                const float t1 = fxx * wxx + fxy * wxy;
                const float t2 = fyy * wyy + fxy * wxy;
                const float t3 = fxy * (wxx + wyy) + (fxx + fyy) * wxy;
                const float gfxx = t1 * (1.0f / 12.0f) - 0.5f * lanesum(s.HXX) -
                                   sW * (1.0f / 24.0f);
                const float gfyy = t2 * (1.0f / 12.0f) - 0.5f * lanesum(s.HYY) -
                                   sW * (1.0f / 24.0f);
                const float gfxy = t3 * (1.0f / 12.0f) - lanesum(s.HXY);
                const float4 j0 = rj[0], j1 = rj[1], j2 = rj[2], j3 = rj[3];
                P[0] = fmaf(j0.x, gA, P[0]);
                P[1] = fmaf(j1.z, gy, fmaf(j1.y, gx, P[1]));
                P[2] = fmaf(j2.x, gy, fmaf(j1.w, gx, P[2]));
                P[3] = fmaf(j2.w, gfyy, fmaf(j2.z, gfxy, fmaf(j2.y, gfxx, fmaf(j0.y, gA, P[3]))));
                P[4] = fmaf(j3.z, gfyy, fmaf(j3.y, gfxy, fmaf(j3.x, gfxx, fmaf(j0.z, gA, P[4]))));
                P[5] = fmaf(j0.w, gA, P[5]);
                P[6] = fmaf(j1.x, gA, P[6]);
                if ((flag & FLAG_LAST_SRC) || last) {
                    // the index comes from the staged record: bounded, so that
                    // a stage a timed-out wait left stale cannot write outside
                    // the sums (the error word already marks the evaluation)
                    const int src = min((unsigned)__float_as_int(j3.w),
                                        (unsigned)(A.pv.n_sources - 1));
                    float v[8] = {P[0], P[1], P[2], P[3], P[4], P[5], P[6], 0.0f};
#pragma unroll
                    for (int k = 0; k < 7; ++k) P[k] = 0.0f;
                    const float tot = warp_reduce7(v, lane);
                    const int k = reduce7_index(lane);
                    if ((lane & 3) == 0 && k < 7) wacc[warp * stride + src * 7 + k] += tot;
                }
            };
            int i = i0;
            for (; i + 1 < i1; i += 2) {
                const float *ra = recs + (size_t)i * GSTAGE, *rb = ra + GSTAGE;
                GradSums sa, sb;
                gradient_pairs2<KP>(X, Y, R2, ra, rb, C24, KEXP2, sa, sb);
                epilogue(ra, kept[c0 + i], sa, false);
                epilogue(rb, kept[c0 + i + 1], sb, i + 1 == i1 - 1);
            }
            for (; i < i1; ++i) {
                const float *r = recs + (size_t)i * GSTAGE;
                v2 NXC, NYC, FXX, FXY, FYY, AMP, HB, C0;
                ld2(r + R_NXC, NXC, NYC);
                ld2(r + R_FXX, FXX, FXY);
                ld2(r + R_FYY, FYY, AMP);
                ld2(r + R_HB, HB, C0);
                const int flag = kept[c0 + i];
                GradSums s;
                if (flag & FLAG_CUT)
                    gradient_pairs<KP, true>(X, Y, R2, NXC, NYC, FXX, FXY, FYY, C0, C24, KEXP2, s);
                else
                    gradient_pairs<KP, false>(X, Y, R2, NXC, NYC, FXX, FXY, FYY, C0, C24, KEXP2, s);
                epilogue(r, flag, s, i == i1 - 1);
            }
        }
    }
    __syncthreads();

    // ---- tile partials (fixed-order sums)
    if (tid == 0) A.pchi2[tile] = s_chi2;
    for (int j = tid; GRAD && j < stride; j += NT) {
        float v = 0.0f;
#pragma unroll
        for (int w = 0; w < NW; ++w) v += wacc[w * stride + j];
        A.pgrad[(size_t)tile * stride + j] = v;
    }
    if (A.tile_cost && tid == 0) A.tile_cost[tile] = n_live * td.count;
    if (A.pairs && tid == 0) atomicAdd(reinterpret_cast<unsigned long long *>(A.pairs),
                                       (unsigned long long)((long long)n_live * td.count));
}

// ------------------------------------------------------------ design rows
// Records per shared-memory stage of the design passes (the design matrix and
// the flux solve's normal equations): each chunk is staged once, so a small
// stage costs little and lets more CTAs reside.  Both passes use it, so their
// unit-flux rows -- flushed at source boundaries and chunk ends -- are the
// same floats.
constexpr int DESIGN_LIVE_CAP = 64;
// The unit-flux model of one Gaussian (dA/dflux in place of the amplitude)
// accumulated, negated, into M, as residual_pairs does for the model.
template <int KP>
__device__ __forceinline__ void design_one(const v2 (&Xp)[KP], const v2 (&Yp)[KP], v2 (&M)[KP],
                                           const float *r, int flag, v2 CM24, v2 KEXP2,
                                           v2 KEXPLO2) {
    v2 NXC, NYC, FXX, FXY, FYY, AMP, HB, C0;
    ld2(r + R_NXC, NXC, NYC);
    ld2(r + R_FXX, FXX, FXY);
    ld2(r + R_FYY, FYY, AMP);
    ld2(r + R_HB, HB, C0);
    const v2 UA = pk1(r[R_JA_FLUX]);
    const v2 HA = mul2(UA, CM24);
    const v2 UB = mul2(pk1(-1.0f), mul2(UA, C0));
    if (flag & FLAG_CUT)
        residual_pairs<KP, true>(Xp, Yp, M, NXC, NYC, FXX, FXY, FYY, HA, UB, KEXP2, KEXPLO2);
    else
        residual_pairs<KP, false>(Xp, Yp, M, NXC, NYC, FXX, FXY, FYY, HA, UB, KEXP2, KEXPLO2);
}

// The same for two consecutive Gaussians a, b of one source at once (their
// exponentials interleave), M updated with a's term and then b's, the cut
// applied to both (see residual_pairs2).
template <int KP>
__device__ __forceinline__ void design_pairs2(const v2 (&Xp)[KP], const v2 (&Yp)[KP],
                                              v2 (&M)[KP], const float *ra, const float *rb,
                                              v2 CM24, v2 KEXP2, v2 KEXPLO2) {
    v2 NXa, NYa, FXXa, FXYa, FYYa, AMPa, HBa, C0a;
    v2 NXb, NYb, FXXb, FXYb, FYYb, AMPb, HBb, C0b;
    ld2(ra + R_NXC, NXa, NYa);
    ld2(ra + R_FXX, FXXa, FXYa);
    ld2(ra + R_FYY, FYYa, AMPa);
    ld2(ra + R_HB, HBa, C0a);
    ld2(rb + R_NXC, NXb, NYb);
    ld2(rb + R_FXX, FXXb, FXYb);
    ld2(rb + R_FYY, FYYb, AMPb);
    ld2(rb + R_HB, HBb, C0b);
    const v2 UAa = pk1(ra[R_JA_FLUX]), UAb = pk1(rb[R_JA_FLUX]);
    const v2 HAa = mul2(UAa, CM24), HAb = mul2(UAb, CM24);
    const v2 UBa = mul2(pk1(-1.0f), mul2(UAa, C0a)), UBb = mul2(pk1(-1.0f), mul2(UAb, C0b));
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const v2 DXa = add2(Xp[j], NXa), DYa = add2(Yp[j], NYa);
        const v2 DXb = add2(Xp[j], NXb), DYb = add2(Yp[j], NYb);
        const v2 VXa = fma2(FXYa, DYa, mul2(FXXa, DXa));
        const v2 VXb = fma2(FXYb, DYb, mul2(FXXb, DXb));
        const v2 VYa = fma2(FXYa, DXa, mul2(FYYa, DYa));
        const v2 VYb = fma2(FXYb, DXb, mul2(FYYb, DYb));
        const v2 Qa = fma2(DYa, VYa, mul2(DXa, VXa));
        const v2 Qb = fma2(DYb, VYb, mul2(DXb, VXb));
        v2 Ga = exp_neg_half(Qa, KEXP2, KEXPLO2);
        v2 Gb = exp_neg_half(Qb, KEXP2, KEXPLO2);
        {
            float g0, g1, q0, q1;
            unpk(Ga, g0, g1);
            unpk(Qa, q0, q1);
            Ga = pk(q0 > FPHO_MAX_EXP_ARG ? 0.0f : g0, q1 > FPHO_MAX_EXP_ARG ? 0.0f : g1);
            unpk(Gb, g0, g1);
            unpk(Qb, q0, q1);
            Gb = pk(q0 > FPHO_MAX_EXP_ARG ? 0.0f : g0, q1 > FPHO_MAX_EXP_ARG ? 0.0f : g1);
        }
        const v2 Sa = fma2(VYa, VYa, mul2(VXa, VXa));
        const v2 Sb = fma2(VYb, VYb, mul2(VXb, VXb));
        M[j] = fma2(fma2(Sa, HAa, UBa), Ga, M[j]);
        M[j] = fma2(fma2(Sb, HAb, UBb), Gb, M[j]);
    }
}
// The unit-flux model of every source at every pixel of the tile:
// X[src][pix] = sum over the source's image Gaussians of dA/dflux * G * H
// (dA/dflux = the record's R_JA_FLUX; with the source's flux this is its model
// divided by the flux, as the reference's design matrix,
// forcepho/patches/device_patch.py:198-238).  Same scan, staging and
// exponential as the residual pass; X must be zero on entry, and every
// (src, pixel) is written by one thread only.
template <int NT, int K>
__device__ __forceinline__ void design_body(const TileArgs &A, int tile, unsigned char *smem,
                                            uint64_t *mbar, uint32_t &phase, float *X,
                                            long long npix) {
    static_assert(K % 2 == 0, "pixels per thread must be even (packed pairs)");
    constexpr int KP = K / 2;
    const int tid = threadIdx.x;
    const int cap = A.live_cap;
    float *recs = reinterpret_cast<float *>(smem);
    int *kept = reinterpret_cast<int *>(smem + (size_t)cap * GSTAGE * 4);

    const TileDesc td = A.tiles[tile];
    const float4 bb = A.tbox_all[tile];
    const int g0 = A.pv.gauss_start[td.exposure];
    const int g1 = A.pv.gauss_start[td.exposure + 1];
    const int npsf = A.pv.exp_npsf[td.exposure];
    const float xmid = 0.5f * (bb.x + bb.y), ymid = 0.5f * (bb.z + bb.w);
    v2 Xp[KP], Yp[KP], M[KP];
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        float xs[2], ys[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int li = tid + (2 * j + h) * NT;
            const bool ok = li < td.count;
            const int pix = td.pix_begin + (ok ? li : 0);
            xs[h] = ok ? A.pv.xpix[pix] : xmid;
            ys[h] = ok ? A.pv.ypix[pix] : ymid;
        }
        Xp[j] = pk(xs[0], xs[1]);
        Yp[j] = pk(ys[0], ys[1]);
        M[j] = 0ull;
    }
    const int n_live = scan_tile<NT>(A, bb, g0, g1, npsf, kept);
    const v2 KEXP2 = pk1(KEXP), KEXPLO2 = pk1(KEXP_LO), CM24 = pk1(-1.0f / 24.0f);
    for (int c0 = 0; c0 < n_live; c0 += cap) {
        const int n = min(cap, n_live - c0);
        if (c0 > 0) __syncthreads();
        stage_records<NT>(recs, A.gtab + (size_t)g0 * GREC, kept, c0, n, 0, mbar, phase, A.err);
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
                const int src = min((unsigned)__float_as_int(r[R_SRC]),
                                    (unsigned)(A.pv.n_sources - 1));
                float *row = X + (size_t)src * npix + td.pix_begin;
#pragma unroll
                for (int j = 0; j < KP; ++j) {
                    float m0, m1;
                    unpk(M[j], m0, m1);  // accumulated -model
                    const int l0 = tid + 2 * j * NT, l1 = l0 + NT;
                    if (l0 < td.count) row[l0] -= m0;
                    if (l1 < td.count) row[l1] -= m1;
                    M[j] = 0ull;
                }
            }
        }
    }
}

}  // namespace fpho
