// fpho_impl.cuh -- internals shared by the forcepho_b200 CUDA translation units.
//
// Device-side layout (all per evaluation, owned by a patch handle):
//   gtab  float[n_gauss][32]  one 128-byte record per image Gaussian
//                             (exposure-major, then source, then PSF component),
//                             written by build_image_gaussians and staged into
//                             shared memory per tile by bulk copies;
//   gbox  float4[n_gauss]     axis-aligned box enclosing the Gaussian's
//                             exp-argument <= 36 ellipse (plus a safety margin),
//                             used to cull Gaussians per pixel tile.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fpho.h"

namespace fpho {

// ---------------------------------------------------------------- records
constexpr int GREC = 32;  // floats per image-Gaussian record
// Floats 0..15 hold the eight per-pixel-loop parameters, each stored twice so
// that one 16-byte shared-memory load yields two packed f32x2 operands (both
// lanes of a pair of pixels use the same Gaussian).  Floats 16..30 hold the
// Jacobian of (A, x, y, fxx, fyy, fxy) w.r.t. (flux, ra, dec, q, pa, n, rh) as
// scalars; the rows acting on x, y and F are pre-multiplied by amp.
enum RecField : int {
    R_NXC = 0,    // -xcen (x2)
    R_NYC = 2,    // -ycen (x2)
    R_FXX = 4,    // F11 (x2)
    R_FXY = 6,    // F21 (x2)
    R_FYY = 8,    // F22 (x2)
    R_AMP = 10,   // amp (x2)
    R_HB = 12,    // -amp * c0 (x2)
    R_C0 = 14,    // c0 (x2)
    R_JA_FLUX = 16, R_JA_Q = 17, R_JA_PA = 18, R_JA_N = 19,
    R_JA_RH = 20, R_JX_RA = 21, R_JY_RA = 22, R_JX_DEC = 23,
    R_JY_DEC = 24, R_JFXX_Q = 25, R_JFXY_Q = 26, R_JFYY_Q = 27,
    R_JFXX_PA = 28, R_JFXY_PA = 29, R_JFYY_PA = 30,
    R_SRC = 31,   // source index (int bits)
};
// c0 = 1 - (fxx + fyy)/24, so that H = 1 + (|v|^2 - fxx - fyy)/24 = |v|^2/24 + c0.

// Culling margin on the half-widths of the exp-argument <= 36 ellipse.  The
// per-pixel exp-argument is computed in float from F; its error relative to the
// exact quadratic form is a few ulp times the condition number of F (< 1e-4
// here), so a 1e-3 relative plus 1e-3 pixel widening keeps the box conservative.
constexpr float CULL_REL = 1.0e-3f;
constexpr float CULL_ABS = 1.0e-3f;

// ---------------------------------------------------------------- views
// Device pointers of one patch, passed to kernels by value.
struct PatchView {
    const float *data, *ierr, *xpix, *ypix;
    float *residual;
    const float *rad2, *D, *crpix, *crval, *CW, *G;
    const fpho_psfgauss *psfgauss;
    const int *psfgauss_start;
    const int *exp_band;     // [n_exp] band of each exposure (-1: none)
    const int *exp_npsf;     // [n_exp] PSF components per source in that band
    const int *gauss_start;  // [n_exp + 1] first image Gaussian of each exposure
    int n_sources, n_exp, n_bands, n_radii;
};

// One pixel tile: a contiguous run of at most TILE pixels of one exposure.
struct TileDesc {
    int exposure;
    int band;
    int pix_begin;  // index into the patch pixel arrays
    int count;      // valid pixels (<= tile size)
};

// ---------------------------------------------------------------- 2x2 algebra
// Row-major 2x2 matrix (a b / c d) and the operations of
// forcepho/src/matrix22.cc, written with round-to-nearest intrinsics so that no
// multiply-add is contracted: the image-Gaussian parameters then equal, bit for
// bit, the ones the reference CPU kernel builds (compiled without FMA).
struct M22 {
    float a, b, c, d;
};
__device__ __forceinline__ float fm(float x, float y) { return __fmul_rn(x, y); }
__device__ __forceinline__ float fa(float x, float y) { return __fadd_rn(x, y); }
__device__ __forceinline__ float fs(float x, float y) { return __fsub_rn(x, y); }
// x*y + z*w without contraction
__device__ __forceinline__ float dot2(float x, float y, float z, float w) {
    return fa(fm(x, y), fm(z, w));
}
__device__ __forceinline__ M22 mmul(M22 A, M22 B) {       // matrix22.cc:136-139
    return {dot2(A.a, B.a, A.b, B.c), dot2(A.a, B.b, A.b, B.d), dot2(A.c, B.a, A.d, B.c),
            dot2(A.c, B.b, A.d, B.d)};
}
__device__ __forceinline__ M22 mscal(float s, M22 A) {    // matrix22.cc:120-125
    return {fm(s, A.a), fm(s, A.b), fm(s, A.c), fm(s, A.d)};
}
__device__ __forceinline__ M22 symabt(M22 A, M22 B) {     // matrix22.cc:164-167
    const float t = fa(fa(fa(fm(A.a, B.c), fm(A.b, B.d)), fm(A.c, B.a)), fm(A.d, B.b));
    return {fm(2.0f, dot2(A.a, B.a, A.b, B.b)), t, t, fm(2.0f, dot2(A.c, B.c, A.d, B.d))};
}
__device__ __forceinline__ M22 aba(M22 A, M22 B) {        // matrix22.cc:144-150
    M22 r;
    r.a = fa(fa(fa(fm(fm(A.a, A.a), B.a), fm(fm(A.a, A.c), B.b)), fm(fm(A.a, A.b), B.c)),
             fm(fm(A.b, A.c), B.d));
    r.b = fa(fa(fa(fm(fm(A.a, A.b), B.a), fm(fm(A.a, A.d), B.b)), fm(fm(A.b, A.b), B.c)),
             fm(fm(A.b, A.d), B.d));
    r.c = fa(fa(fa(fm(fm(A.a, A.c), B.a), fm(fm(A.c, A.c), B.b)), fm(fm(A.a, A.d), B.c)),
             fm(fm(A.c, A.d), B.d));
    r.d = fa(fa(fa(fm(fm(A.b, A.c), B.a), fm(fm(A.c, A.d), B.b)), fm(fm(A.b, A.d), B.c)),
             fm(fm(A.d, A.d), B.d));
    return r;
}

// Build image Gaussian (exposure e, source s, PSF component p): sky Gaussian of
// radius bin k convolved with PSF Gaussian p, with its Jacobian.
// Follows GetGaussianAndJacobian (forcepho/src/common_kernel.cc:175-240) and
// ConvolveOneSource (forcepho/src/compute_gaussians_kernel.cc:45-114) in the
// same operation order, including the PSF row index
// psfgauss[psfgauss_start[e] + p] used for every source.  cos/sin of the
// position angle are evaluated in double and rounded once.  Writes one record
// and one culling box.
__device__ __forceinline__ void build_one_gaussian(const PatchView &pv, const fpho_source *src,
                                                   int e, int s, int p, float *rec, float4 *box) {
    const int band = pv.exp_band[e];
    const fpho_source &gal = src[s];
    const fpho_psfgauss pg = pv.psfgauss[pv.psfgauss_start[e] + p];
    const int k = pg.sersic_radius_bin;
    const int dcw = 4 * (pv.n_sources * e + s);
    const int cr = 2 * (pv.n_sources * e + s);

    const float G = pv.G[e];
    const float q = gal.q;
    double sd, cd;
    sincos((double)gal.pa, &sd, &cd);
    const float sn = (float)sd, cs = (float)cd;
    const M22 D = {pv.D[dcw], pv.D[dcw + 1], pv.D[dcw + 2], pv.D[dcw + 3]};
    const M22 R = {cs, -sn, sn, cs};
    const M22 S = {__fdiv_rn(1.0f, q), 0.0f, 0.0f, q};
    const M22 dS = {__fdiv_rn(-1.0f, fm(q, q)), 0.0f, 0.0f, 1.0f};
    const M22 dR = {-sn, -cs, cs, -sn};
    const M22 DR = mmul(D, R);
    const M22 T = mmul(DR, S);
    const M22 dTq = mmul(DR, dS);
    const M22 dTpa = mmul(mmul(D, dR), S);
    const M22 CW = {pv.CW[dcw], pv.CW[dcw + 1], pv.CW[dcw + 2], pv.CW[dcw + 3]};
    const float s0 = fs(gal.ra, pv.crval[cr]);
    const float s1 = fs(gal.dec, pv.crval[cr + 1]);
    const float xs = fa(dot2(CW.a, s0, CW.b, s1), pv.crpix[cr]);
    const float ys = fa(dot2(CW.c, s0, CW.d, s1), pv.crpix[cr + 1]);

    const float r2 = pv.rad2[k];
    const float samp = gal.mixture_amplitudes[k];
    const float flux = gal.fluxes[band];

    // Sigma = r2 T T^t + C_psf ; F = Sigma^-1
    const float t12 = dot2(T.a, T.c, T.b, T.d);
    const M22 TTt = {dot2(T.a, T.a, T.b, T.b), t12, t12, dot2(T.c, T.c, T.d, T.d)};
    const M22 sc = mscal(r2, TTt);
    const M22 Sig = {fa(sc.a, pg.Cxx), fa(sc.b, pg.Cxy), fa(sc.c, pg.Cxy), fa(sc.d, pg.Cyy)};
    const float idet = __fdiv_rn(1.0f, fs(fm(Sig.a, Sig.d), fm(Sig.b, Sig.c)));
    const M22 F = {fm(Sig.d, idet), fm(-Sig.b, idet), fm(-Sig.c, idet), fm(Sig.a, idet)};
    const float detF = fs(fm(F.a, F.d), fm(F.b, F.c));
    const float tmp = fm(fm(fm(G, pg.amp), __fsqrt_rn(detF)),
                         (1.0f / (2.0f * 3.14159265358979323846f)));
    const float amp = fm(fm(tmp, flux), samp);

    // dSigma/dq = r2 symABt(T, dT); dF = -F dSigma F; dA = amp/2 tr(Sigma dF)
    float jF[2][3], jA[2];
    {
        const M22 dTs[2] = {dTq, dTpa};
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            const M22 dSig = mscal(r2, symabt(T, dTs[w]));
            const M22 dF = mscal(-1.0f, aba(F, dSig));
            const M22 M = mmul(Sig, dF);
            jA[w] = fm(fm(0.5f, amp), fa(M.a, M.d));
            jF[w][0] = dF.a;  // fxx
            jF[w][1] = dF.c;  // fxy
            jF[w][2] = dF.d;  // fyy
        }
    }

    const float xc = fa(xs, pg.xcen);
    const float yc = fa(ys, pg.ycen);
    const float c0 = 1.0f - (F.a + F.d) * (1.0f / 24.0f);
    const float tf = fm(tmp, flux);

    float4 *r4 = reinterpret_cast<float4 *>(rec);
    r4[0] = make_float4(-xc, -xc, -yc, -yc);
    r4[1] = make_float4(F.a, F.a, F.c, F.c);
    r4[2] = make_float4(F.d, F.d, amp, amp);
    r4[3] = make_float4(-amp * c0, -amp * c0, c0, c0);
    r4[4] = make_float4(fm(tmp, samp), jA[0], jA[1], fm(tf, gal.damplitude_dnsersic[k]));
    r4[5] = make_float4(fm(tf, gal.damplitude_drh[k]), amp * CW.a, amp * CW.c, amp * CW.b);
    r4[6] = make_float4(amp * CW.d, amp * jF[0][0], amp * jF[0][1], amp * jF[0][2]);
    r4[7] = make_float4(amp * jF[1][0], amp * jF[1][1], amp * jF[1][2], __int_as_float(s));

    // exp-argument <= 36 ellipse: half-widths 6 sqrt(Sigma11), 6 sqrt(Sigma22)
    const float wx = 6.0f * sqrtf(fmaxf(Sig.a, 0.0f)) * (1.0f + CULL_REL) + CULL_ABS;
    const float wy = 6.0f * sqrtf(fmaxf(Sig.d, 0.0f)) * (1.0f + CULL_REL) + CULL_ABS;
    *box = make_float4(xc - wx, xc + wx, yc - wy, yc + wy);
}

// ---------------------------------------------------------------- packed f32x2
// Two pixels per register pair: sm_100 executes add/mul/fma on .f32x2 operands
// as one instruction.  Values are carried as 64-bit integers holding {lo, hi}.
typedef unsigned long long v2;

__device__ __forceinline__ v2 pk(float lo, float hi) {
    v2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ v2 pk1(float x) { return pk(x, x); }
__device__ __forceinline__ float lo(v2 v) {
    return __uint_as_float(static_cast<unsigned int>(v & 0xffffffffull));
}
__device__ __forceinline__ float hi(v2 v) {
    return __uint_as_float(static_cast<unsigned int>(v >> 32));
}
__device__ __forceinline__ void unpk(v2 v, float &a, float &b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ v2 add2(v2 a, v2 b) {
    v2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ v2 mul2(v2 a, v2 b) {
    v2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ v2 fma2(v2 a, v2 b, v2 c) {
    v2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// 2^x on the SFU (MUFU.EX2), flush-to-zero: inputs below -126 give 0.
__device__ __forceinline__ float ex2f(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// -0.5 * log2(e): exp(-Q/2) = 2^(Q * KEXP).  KEXP_LO carries the rounding of
// KEXP (relative 1.3e-8), so that Q * KEXP + Q * KEXP_LO is the exponent
// without the systematic error a rounded constant would add.
constexpr float KEXP = -0.72134752044448170368f;
constexpr float KEXP_LO = -9.629815167500055e-09f;

// Unbiased exp(-Q/2) for packed exp-arguments Q in [0, 174].
//
// MUFU.EX2 (ex2.approx) is accurate to a few 1e-7 but its error has a mean of
// about -3e-8 over the exponents seen here.  In the residual r = data - model
// that bias does not average out: the gradient of chi2 near a fit measures a
// ~1% parameter offset, and a relative model bias b shows up in it amplified
// ~1e3 times.  So the residual pass evaluates 2^E, E = Q * (KEXP + KEXP_LO),
// with Cody and Waite's range reduction E = n + f:
//   n = rint(Q * KEXP), the rounding done by one FMA with 1.5*2^23, whose
//       low mantissa bits then hold n;
//   f = (Q * KEXP - n) + Q * KEXP_LO, two FMAs, the first forming the product
//       exactly, so that f (|f| <= 1/2 + 4e-7) carries one rounding of a
//       number below 1/2 rather than the rounding of E itself (up to 1e-6
//       absolute at E = -26);
// then a degree-6 polynomial for 2^f (coefficients fitted here by relative
// least squares with the constant term pinned to 1: mean relative error
// 6e-10, max 8e-8 in float) and scaling by 2^n through the exponent field.
// Arguments above 174 give garbage that callers discard (they select 0 for
// exp-arguments above the cutoff, and never use the value at pixels outside
// the culling box).
__device__ __forceinline__ v2 exp_neg_half(v2 Q, v2 KEXP2, v2 KEXPLO2) {
    const float MAGIC = 12582912.0f;  // 1.5 * 2^23
    const v2 t = fma2(Q, KEXP2, pk1(MAGIC));
    // MAGIC - t (one FMA, no sign-bit operation) is -n exactly
    const v2 f = fma2(Q, KEXPLO2, fma2(Q, KEXP2, fma2(t, pk1(-1.0f), pk1(MAGIC))));
    v2 p = pk1(1.5370704932138324e-04f);
    p = fma2(p, f, pk1(1.3399848248809576e-03f));
    p = fma2(p, f, pk1(9.618373587727547e-03f));
    p = fma2(p, f, pk1(5.550329014658928e-02f));
    p = fma2(p, f, pk1(2.4022647738456726e-01f));
    p = fma2(p, f, pk1(6.931471824645996e-01f));
    p = fma2(p, f, pk1(1.0f));
    // t's low mantissa bits hold n (two's complement); (bits(t) << 23) adds n
    // to the exponent of p, since bits(1.5*2^23) << 23 vanishes mod 2^32.
    uint32_t t0, t1, p0, p1;
    asm("mov.b64 {%0, %1}, %2;" : "=r"(t0), "=r"(t1) : "l"(t));
    asm("mov.b64 {%0, %1}, %2;" : "=r"(p0), "=r"(p1) : "l"(p));
    p0 += t0 << 23;
    p1 += t1 << 23;
    v2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(p0), "r"(p1));
    return r;
}

}  // namespace fpho
