/*
 * fpho_oracle.c -- CPU oracle for the proposal-evaluation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the forcepho_b200 product links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py use it, and only as the checker.
 *
 * It restates, in plain C, the reference's single-band CPU evaluation
 * (forcepho/src/compute_gaussians_kernel.cc:227-315) together with the shared
 * math it calls (forcepho/src/common_kernel.cc:57-240 and the 2x2 helpers of
 * forcepho/src/matrix22.cc:32-200).  Two variants are provided:
 *
 *   fpo_evaluate_band_f32  float arithmetic in the reference's operation order,
 *                          so that, compiled without FMA contraction, its
 *                          output is bit-identical to the reference CPU kernel
 *                          (pinned by tests/test_oracle.py against the
 *                          reference kernel built from its own sources and
 *                          against committed golden vectors).
 *   fpo_evaluate_band_f64  every operation in double precision, with the
 *                          exp-argument cutoff and the second-order pixel
 *                          correction switchable, so that it can be pinned to
 *                          the reference's FP64 python path (forcepho/slow).
 *
 * The struct layouts below are the reference's device ABI
 * (forcepho/src/patch.cc:23-119, forcepho/src/proposal.cu:13-39) and must stay
 * byte-compatible with it.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define FPO_MAXBANDS 30
#define FPO_NPARAMS 7
#define FPO_MAXRADII 10
#define FPO_MAX_EXP_ARG 36.0

typedef struct {
    float amp, xcen, ycen, Cxx, Cyy, Cxy;
    int sersic_radius_bin;
} fpo_psfgauss;

typedef struct {
    float *data, *ierr, *xpix, *ypix, *residual;
    int *exposure_start, *exposure_N;
    int16_t *band_start, *band_N;
    int n_sources, n_radii;
    float *rad2, *D, *crpix, *crval, *CW, *G;
    int *n_psf_per_source;
    fpo_psfgauss *psfgauss;
    int *psfgauss_start;
} fpo_patch;

typedef struct {
    float ra, dec, q, pa, nsersic, rh;
    float fluxes[FPO_MAXBANDS];
    float mixture_amplitudes[FPO_MAXRADII];
    float damplitude_drh[FPO_MAXRADII];
    float damplitude_dnsersic[FPO_MAXRADII];
} fpo_source;

int fpo_sizeof_patch(void) { return (int)sizeof(fpo_patch); }
int fpo_sizeof_source(void) { return (int)sizeof(fpo_source); }
int fpo_sizeof_psfgauss(void) { return (int)sizeof(fpo_psfgauss); }

/* ------------------------------------------------------------------------
 * float restatement
 * ------------------------------------------------------------------------ */

/* 2x2 matrix, row-major (v11 v12 / v21 v22), as matrix22.cc:32-60 */
typedef struct { float a, b, c, d; } m22f;

static m22f m22f_mul(m22f A, m22f B) {           /* matrix22.cc:136-139 */
    m22f r = {A.a * B.a + A.b * B.c, A.a * B.b + A.b * B.d,
              A.c * B.a + A.d * B.c, A.c * B.b + A.d * B.d};
    return r;
}
static m22f m22f_scal(float s, m22f A) {          /* matrix22.cc:120-125 */
    m22f r = {s * A.a, s * A.b, s * A.c, s * A.d};
    return r;
}
static m22f m22f_add(m22f A, m22f B) {            /* matrix22.cc:128-130 */
    m22f r = {A.a + B.a, A.b + B.b, A.c + B.c, A.d + B.d};
    return r;
}
static float m22f_det(m22f A) { return A.a * A.d - A.b * A.c; }   /* :98 */
static m22f m22f_inv(m22f A) {                     /* matrix22.cc:104-107 */
    float idet = 1.0f / m22f_det(A);
    m22f r = {A.d * idet, -A.b * idet, -A.c * idet, A.a * idet};
    return r;
}
static m22f m22f_aat(m22f A) {                     /* matrix22.cc:153-156 */
    float t = A.a * A.c + A.b * A.d;
    m22f r = {A.a * A.a + A.b * A.b, t, t, A.c * A.c + A.d * A.d};
    return r;
}
static m22f m22f_symabt(m22f A, m22f B) {          /* matrix22.cc:164-167 */
    float t = A.a * B.c + A.b * B.d + A.c * B.a + A.d * B.b;
    m22f r = {2.0f * (A.a * B.a + A.b * B.b), t, t, 2.0f * (A.c * B.c + A.d * B.d)};
    return r;
}
static m22f m22f_aba(m22f A, m22f B) {             /* matrix22.cc:144-150 */
    m22f r;
    r.a = A.a * A.a * B.a + A.a * A.c * B.b + A.a * A.b * B.c + A.b * A.c * B.d;
    r.b = A.a * A.b * B.a + A.a * A.d * B.b + A.b * A.b * B.c + A.b * A.d * B.d;
    r.c = A.a * A.c * B.a + A.c * A.c * B.b + A.a * A.d * B.c + A.c * A.d * B.d;
    r.d = A.b * A.c * B.a + A.c * A.d * B.b + A.b * A.d * B.c + A.d * A.d * B.d;
    return r;
}

/* ImageGaussian, common_kernel.cc:20-46: 6 parameters + 15 Jacobian terms */
typedef struct {
    float amp, xcen, ycen, fxx, fyy, fxy;
    float dA_dFlux, dx_dAlpha, dy_dAlpha, dx_dDelta, dy_dDelta;
    float dA_dQ, dFxx_dQ, dFyy_dQ, dFxy_dQ;
    float dA_dPA, dFxx_dPA, dFyy_dPA, dFxy_dPA;
    float dA_dSersic, dA_drh;
} fpo_imgauss;

/* ConvolveOneSource + GetGaussianAndJacobian, compute_gaussians_kernel.cc:45-114
 * and common_kernel.cc:175-240.  Note the PSF row index: the reference reads
 * psfgauss[psfgauss_start[e] + p] for every source (the per-source rows packed
 * by patch.py are not indexed by source), and so does this restatement. */
/* With the file-scope switch g_rounded_trig set, cos and sin of the position
 * angle are evaluated in double and rounded once to float (the correctly
 * rounded values) instead of by the C library's cosf/sinf, as the residual
 * oracle fpo_residual_band_f32_dexp does; every other caller leaves it 0. */
static int g_rounded_trig = 0;

static void convolve_source_f32(int band, int e, int g, int npsf,
                                const fpo_patch *P, const fpo_source *S,
                                fpo_imgauss *out) {
    const fpo_source *gal = S + g;
    int pstart = P->psfgauss_start[e];
    float G = P->G[e];
    int dcw = 4 * (P->n_sources * e + g);
    int cr = 2 * (P->n_sources * e + g);
    float crpix0 = P->crpix[cr], crpix1 = P->crpix[cr + 1];
    float crval0 = P->crval[cr], crval1 = P->crval[cr + 1];
    float sm0 = gal->ra - crval0, sm1 = gal->dec - crval1;

    m22f D = {P->D[dcw], P->D[dcw + 1], P->D[dcw + 2], P->D[dcw + 3]};
    float c = cosf(gal->pa), s = sinf(gal->pa);
    if (g_rounded_trig) {
        c = (float)cos((double)gal->pa);
        s = (float)sin((double)gal->pa);
    }
    m22f R = {c, -s, s, c};
    m22f Sc = {1.0f / gal->q, 0.0f, 0.0f, gal->q};
    m22f dS = {-1.0f / (gal->q * gal->q), 0.0f, 0.0f, 1.0f};
    m22f dR = {-s, -c, c, -s};
    m22f DR = m22f_mul(D, R);
    m22f T = m22f_mul(DR, Sc);
    m22f dT_dq = m22f_mul(DR, dS);
    m22f dT_dpa = m22f_mul(m22f_mul(D, dR), Sc);
    m22f CW = {P->CW[dcw], P->CW[dcw + 1], P->CW[dcw + 2], P->CW[dcw + 3]};
    float v1 = sm0, v2 = sm1;
    sm0 = CW.a * v1 + CW.b * v2;
    sm1 = CW.c * v1 + CW.d * v2;
    float xcen = sm0 + crpix0, ycen = sm1 + crpix1;
    float flux = gal->fluxes[band];
    m22f TTt = m22f_aat(T);
    m22f sym_q = m22f_symabt(T, dT_dq);
    m22f sym_pa = m22f_symabt(T, dT_dpa);

    for (int p = 0; p < npsf; p++) {
        const fpo_psfgauss *pg = P->psfgauss + pstart + p;
        fpo_imgauss *ig = out + g * npsf + p;
        int k = pg->sersic_radius_bin;
        float covar = P->rad2[k];
        float samp = gal->mixture_amplitudes[k];
        float da_dn = gal->damplitude_dnsersic[k];
        float da_dr = gal->damplitude_drh[k];

        m22f scov = m22f_scal(covar, TTt);
        m22f pc = {pg->Cxx, pg->Cxy, pg->Cxy, pg->Cyy};
        m22f Sig = m22f_add(scov, pc);
        m22f F = m22f_inv(Sig);
        float detF = m22f_det(F);
        ig->fxx = F.a;
        ig->fxy = F.c;
        ig->fyy = F.d;
        ig->xcen = xcen + pg->xcen;
        ig->ycen = ycen + pg->ycen;
        float tmp = G * pg->amp * sqrtf(detF) * (1.0f / (2.0f * (float)M_PI));
        ig->amp = tmp * flux * samp;
        m22f dSig_q = m22f_scal(covar, sym_q);
        m22f dSig_pa = m22f_scal(covar, sym_pa);
        m22f dF_q = m22f_scal(-1.0f, m22f_aba(F, dSig_q));
        m22f dF_pa = m22f_scal(-1.0f, m22f_aba(F, dSig_pa));
        m22f Mq = m22f_mul(Sig, dF_q);
        m22f Mpa = m22f_mul(Sig, dF_pa);
        ig->dA_dQ = 0.5f * ig->amp * (Mq.a + Mq.d);
        ig->dA_dPA = 0.5f * ig->amp * (Mpa.a + Mpa.d);
        ig->dA_dFlux = tmp * samp;
        ig->dA_dSersic = tmp * flux * da_dn;
        ig->dA_drh = tmp * flux * da_dr;
        ig->dx_dAlpha = CW.a;
        ig->dy_dAlpha = CW.c;
        ig->dx_dDelta = CW.b;
        ig->dy_dDelta = CW.d;
        ig->dFxx_dQ = dF_q.a;
        ig->dFyy_dQ = dF_q.d;
        ig->dFxy_dQ = dF_q.c;
        ig->dFxx_dPA = dF_pa.a;
        ig->dFyy_dPA = dF_pa.d;
        ig->dFxy_dPA = dF_pa.c;
    }
}

/* ComputeResidualImage, common_kernel.cc:57-83 */
static float residual_f32(float xp, float yp, float data, const fpo_imgauss *g, int n) {
    float r = data;
    for (int i = 0; i < n; i++, g++) {
        float dx = xp - g->xcen;
        float dy = yp - g->ycen;
        float vx = g->fxx * dx + g->fxy * dy;
        float vy = g->fyy * dy + g->fxy * dx;
        float ea = dx * vx + dy * vy;
        if (ea > (float)FPO_MAX_EXP_ARG) continue;
        float Gp = expf(-0.5f * ea);
        float H = 1.0f + (vx * vx + vy * vy - g->fxx - g->fyy) / 24.f;
        float C = g->amp * Gp * H;
        r -= C;
    }
    return r;
}

/* residual_f32 with the exponential evaluated in double and rounded once to
 * float (the correctly rounded float exp, up to double exp's own rounding)
 * in place of the C library's expf, which is not correctly rounded on a
 * small fraction of arguments.  Everything else is the reference's float
 * arithmetic, in its order. */
static float residual_f32_dexp(float xp, float yp, float data, const fpo_imgauss *g, int n) {
    float r = data;
    for (int i = 0; i < n; i++, g++) {
        float dx = xp - g->xcen;
        float dy = yp - g->ycen;
        float vx = g->fxx * dx + g->fxy * dy;
        float vy = g->fyy * dy + g->fxy * dx;
        float ea = dx * vx + dy * vy;
        if (ea > (float)FPO_MAX_EXP_ARG) continue;
        float Gp = (float)exp((double)(-0.5f * ea));
        float H = 1.0f + (vx * vx + vy * vy - g->fxx - g->fyy) / 24.f;
        float C = g->amp * Gp * H;
        r -= C;
    }
    return r;
}

/* ComputeGaussianDerivative, common_kernel.cc:95-143 */
static void derivative_f32(float xp, float yp, float rie2, const fpo_imgauss *g,
                           float *dp, int n) {
    for (int i = 0; i < n; i++, g++) {
        float dx = xp - g->xcen;
        float dy = yp - g->ycen;
        float vx = g->fxx * dx + g->fxy * dy;
        float vy = g->fyy * dy + g->fxy * dx;
        float ea = dx * vx + dy * vy;
        if (ea > (float)FPO_MAX_EXP_ARG) continue;
        float Gp = expf(-0.5f * ea);
        float H = 1.0f + (vx * vx + vy * vy - g->fxx - g->fyy) * (1.0f / 24.0f);
        float dC_dA = -2.f * rie2 * Gp;
        float c_h = dC_dA * g->amp;
        dC_dA *= H;
        float C = c_h * H;
        float dC_dx = C * vx;
        float dC_dy = C * vy;
        float dC_dfx = -0.5f * C * dx * dx;
        float dC_dfy = -0.5f * C * dy * dy;
        float dC_dfxy = -1.0f * C * dx * dy;
        dC_dx -= c_h * (g->fxx * vx + g->fxy * vy) * (1.0f / 12.0f);
        dC_dy -= c_h * (g->fyy * vy + g->fxy * vx) * (1.0f / 12.0f);
        dC_dfx -= c_h * (1.0f - 2.0f * dx * vx) * (1.0f / 24.0f);
        dC_dfy -= c_h * (1.0f - 2.0f * dy * vy) * (1.0f / 24.0f);
        dC_dfxy += c_h * (dy * vx + dx * vy) * (1.0f / 12.0f);
        dp[0] += g->dA_dFlux * dC_dA;
        dp[1] += g->dx_dAlpha * dC_dx + g->dy_dAlpha * dC_dy;
        dp[2] += g->dx_dDelta * dC_dx + g->dy_dDelta * dC_dy;
        dp[3] += g->dA_dQ * dC_dA + dC_dfx * g->dFxx_dQ + dC_dfxy * g->dFxy_dQ + dC_dfy * g->dFyy_dQ;
        dp[4] += g->dA_dPA * dC_dA + dC_dfx * g->dFxx_dPA + dC_dfxy * g->dFxy_dPA + dC_dfy * g->dFyy_dPA;
        dp[5] += g->dA_dSersic * dC_dA;
        dp[6] += g->dA_drh * dC_dA;
    }
}

/* EvaluateProposal (CPU), compute_gaussians_kernel.cc:227-315, for one band.
 * dchi2 receives n_sources*7 floats (no MAXSOURCES cap).  If residual_out is
 * non-NULL the residual of every pixel of the band is written there (indexed
 * like the patch pixel arrays), as the reference does when patch->residual is
 * set.  Returns 0, or -1 if the Gaussian scratch could not be allocated. */
int fpo_evaluate_band_f32(int band, const fpo_patch *P, const fpo_source *S,
                          double *chi2_out, float *dchi2, float *residual_out) {
    int nsrc = P->n_sources;
    int npsf = P->n_psf_per_source[band];
    int bN = P->band_N[band], b0 = P->band_start[band];
    int ntot = nsrc * npsf;
    fpo_imgauss *ig = (fpo_imgauss *)malloc(sizeof(fpo_imgauss) * (size_t)(ntot > 0 ? ntot : 1));
    if (!ig) return -1;
    for (int i = 0; i < nsrc * FPO_NPARAMS; i++) dchi2[i] = 0.0f;
    double chi2 = 0.0;
    float dp[FPO_NPARAMS];
    for (int ee = 0; ee < bN; ee++) {
        int e = b0 + ee;
        int npix = P->exposure_N[e];
        for (int g = 0; g < nsrc; g++) convolve_source_f32(band, e, g, npsf, P, S, ig);
        for (int p = 0; p < npix; p++) {
            int pix = P->exposure_start[e] + p;
            float xp = P->xpix[pix], yp = P->ypix[pix];
            float data = P->data[pix], ierr = P->ierr[pix];
            float r = residual_f32(xp, yp, data, ig, ntot);
            if (residual_out) residual_out[pix] = r;
            r *= ierr;
            data *= ierr;
            double c2 = ((double)r - (double)data);
            c2 *= ((double)r + (double)data);
            chi2 += c2;
            r *= ierr;
            for (int gal = 0; gal < nsrc; gal++) {
                for (int j = 0; j < FPO_NPARAMS; j++) dp[j] = 0.0f;
                derivative_f32(xp, yp, r, ig + gal * npsf, dp, npsf);
                for (int j = 0; j < FPO_NPARAMS; j++) dchi2[gal * FPO_NPARAMS + j] += dp[j];
            }
        }
    }
    free(ig);
    *chi2_out = chi2;
    return 0;
}

/* The reference's own float per-pixel gradient contributions, summed exactly.
 * Identical to fpo_evaluate_band_f32 (float image Gaussians, float residual,
 * float per-pixel and per-source terms dp[] in the reference's operation
 * order), except that the per-pixel terms are accumulated into double
 * dchi2[n_sources*7] instead of the reference's running float sums
 * (compute_gaussians_kernel.cc:300-305).  The difference between the
 * reference's result and this one is therefore exactly the rounding of the
 * reference's sequential float accumulation over the band's pixels. */
int fpo_evaluate_band_f32_dsum(int band, const fpo_patch *P, const fpo_source *S,
                               double *chi2_out, double *dchi2) {
    int nsrc = P->n_sources;
    int npsf = P->n_psf_per_source[band];
    int bN = P->band_N[band], b0 = P->band_start[band];
    int ntot = nsrc * npsf;
    fpo_imgauss *ig = (fpo_imgauss *)malloc(sizeof(fpo_imgauss) * (size_t)(ntot > 0 ? ntot : 1));
    if (!ig) return -1;
    for (int i = 0; i < nsrc * FPO_NPARAMS; i++) dchi2[i] = 0.0;
    double chi2 = 0.0;
    float dp[FPO_NPARAMS];
    for (int ee = 0; ee < bN; ee++) {
        int e = b0 + ee;
        int npix = P->exposure_N[e];
        for (int g = 0; g < nsrc; g++) convolve_source_f32(band, e, g, npsf, P, S, ig);
        for (int p = 0; p < npix; p++) {
            int pix = P->exposure_start[e] + p;
            float xp = P->xpix[pix], yp = P->ypix[pix];
            float data = P->data[pix], ierr = P->ierr[pix];
            float r = residual_f32(xp, yp, data, ig, ntot);
            r *= ierr;
            data *= ierr;
            double c2 = ((double)r - (double)data);
            c2 *= ((double)r + (double)data);
            chi2 += c2;
            r *= ierr;
            for (int gal = 0; gal < nsrc; gal++) {
                for (int j = 0; j < FPO_NPARAMS; j++) dp[j] = 0.0f;
                derivative_f32(xp, yp, r, ig + gal * npsf, dp, npsf);
                for (int j = 0; j < FPO_NPARAMS; j++) dchi2[gal * FPO_NPARAMS + j] += (double)dp[j];
            }
        }
    }
    free(ig);
    *chi2_out = chi2;
    return 0;
}

/* The residual of every pixel of one band as the reference CPU kernel forms
 * it, with the correctly rounded exponential of residual_f32_dexp and, when
 * rounded_trig is non-zero, correctly rounded cos and sin of the position
 * angle (the C library's cosf/sinf are not correctly rounded for about 2.6%
 * of angles). */
int fpo_residual_band_f32_dexp(int band, const fpo_patch *P, const fpo_source *S,
                               float *residual_out, int rounded_trig) {
    int nsrc = P->n_sources;
    int npsf = P->n_psf_per_source[band];
    int bN = P->band_N[band], b0 = P->band_start[band];
    int ntot = nsrc * npsf;
    fpo_imgauss *ig = (fpo_imgauss *)malloc(sizeof(fpo_imgauss) * (size_t)(ntot > 0 ? ntot : 1));
    if (!ig) return -1;
    g_rounded_trig = rounded_trig != 0;
    for (int ee = 0; ee < bN; ee++) {
        int e = b0 + ee;
        for (int g = 0; g < nsrc; g++) convolve_source_f32(band, e, g, npsf, P, S, ig);
        for (int p = 0; p < P->exposure_N[e]; p++) {
            int pix = P->exposure_start[e] + p;
            residual_out[pix] = residual_f32_dexp(P->xpix[pix], P->ypix[pix], P->data[pix], ig,
                                                  ntot);
        }
    }
    g_rounded_trig = 0;
    free(ig);
    return 0;
}

/* Image Gaussians of one exposure in float, exactly as the reference builds
 * them (21 floats per Gaussian, source-major, PSF-minor). */
int fpo_image_gaussians_f32(int band, int e, const fpo_patch *P, const fpo_source *S,
                            float *out21) {
    int npsf = P->n_psf_per_source[band];
    for (int g = 0; g < P->n_sources; g++)
        convolve_source_f32(band, e, g, npsf, P, S, (fpo_imgauss *)out21);
    return P->n_sources * npsf;
}

/* Mixed precision: the reference's float image Gaussians (bit-identical to
 * what its CPU kernel builds), then per-pixel model, chi2 and gradient in
 * double with per-Gaussian image-space gradients contracted with the float
 * Jacobian in double.  Errors of a float kernel against this isolate its
 * per-pixel arithmetic and accumulation from the rounding of the image
 * Gaussian parameters (centres near x ~ 100 px carry ~4e-6 px of float
 * rounding, which every float implementation shares). */
int fpo_evaluate_band_mixed(int band, const fpo_patch *P, const fpo_source *S,
                            int use_cutoff, double *chi2_out, double *dchi2,
                            double *residual_out) {
    int nsrc = P->n_sources;
    int npsf = P->n_psf_per_source[band];
    int bN = P->band_N[band], b0 = P->band_start[band];
    int ntot = nsrc * npsf;
    fpo_imgauss *ig = (fpo_imgauss *)malloc(sizeof(fpo_imgauss) * (size_t)(ntot > 0 ? ntot : 1));
    double *gimg = (double *)malloc(sizeof(double) * 6 * (size_t)(ntot > 0 ? ntot : 1));
    if (!ig || !gimg) { free(ig); free(gimg); return -1; }
    for (int i = 0; i < nsrc * FPO_NPARAMS; i++) dchi2[i] = 0.0;
    double chi2 = 0.0;
    for (int ee = 0; ee < bN; ee++) {
        int e = b0 + ee;
        for (int g = 0; g < nsrc; g++) convolve_source_f32(band, e, g, npsf, P, S, ig);
        memset(gimg, 0, sizeof(double) * 6 * (size_t)ntot);
        int npix = P->exposure_N[e];
        for (int p = 0; p < npix; p++) {
            int pix = P->exposure_start[e] + p;
            double xp = P->xpix[pix], yp = P->ypix[pix];
            double d = P->data[pix], ie = P->ierr[pix];
            double r = d;
            for (int i = 0; i < ntot; i++) {
                const fpo_imgauss *g = ig + i;
                double dx = xp - g->xcen, dy = yp - g->ycen;
                double fxx = g->fxx, fxy = g->fxy, fyy = g->fyy;
                double vx = fxx * dx + fxy * dy, vy = fyy * dy + fxy * dx;
                double ea = dx * vx + dy * vy;
                if (use_cutoff && ea > FPO_MAX_EXP_ARG) continue;
                double H = 1.0 + (vx * vx + vy * vy - fxx - fyy) / 24.0;
                r -= (double)g->amp * exp(-0.5 * ea) * H;
            }
            if (residual_out) residual_out[pix] = r;
            chi2 += (r * ie - d * ie) * (r * ie + d * ie);
            double rie2 = r * ie * ie;
            if (rie2 == 0.0) continue;
            for (int i = 0; i < ntot; i++) {
                const fpo_imgauss *g = ig + i;
                double dx = xp - g->xcen, dy = yp - g->ycen;
                double fxx = g->fxx, fxy = g->fxy, fyy = g->fyy, amp = g->amp;
                double vx = fxx * dx + fxy * dy, vy = fyy * dy + fxy * dx;
                double ea = dx * vx + dy * vy;
                if (use_cutoff && ea > FPO_MAX_EXP_ARG) continue;
                double Gp = exp(-0.5 * ea);
                double H = 1.0 + (vx * vx + vy * vy - fxx - fyy) / 24.0;
                double w = -2.0 * rie2;
                double C = amp * Gp * H, c_h = amp * Gp;
                double *gi = gimg + 6 * i;
                gi[0] += w * Gp * H;
                gi[1] += w * (C * vx - c_h * (fxx * vx + fxy * vy) / 12.0);
                gi[2] += w * (C * vy - c_h * (fyy * vy + fxy * vx) / 12.0);
                gi[3] += w * (-0.5 * C * dx * dx - c_h * (1.0 - 2.0 * dx * vx) / 24.0);
                gi[4] += w * (-0.5 * C * dy * dy - c_h * (1.0 - 2.0 * dy * vy) / 24.0);
                gi[5] += w * (-C * dx * dy + c_h * (dy * vx + dx * vy) / 12.0);
            }
        }
        for (int i = 0; i < ntot; i++) {
            const fpo_imgauss *g = ig + i;
            const double *gi = gimg + 6 * i;
            double *dp = dchi2 + (i / npsf) * FPO_NPARAMS;
            dp[0] += g->dA_dFlux * gi[0];
            dp[1] += g->dx_dAlpha * gi[1] + (double)g->dy_dAlpha * gi[2];
            dp[2] += g->dx_dDelta * gi[1] + (double)g->dy_dDelta * gi[2];
            dp[3] += g->dA_dQ * gi[0] + (double)g->dFxx_dQ * gi[3] + (double)g->dFyy_dQ * gi[4] +
                     (double)g->dFxy_dQ * gi[5];
            dp[4] += g->dA_dPA * gi[0] + (double)g->dFxx_dPA * gi[3] +
                     (double)g->dFyy_dPA * gi[4] + (double)g->dFxy_dPA * gi[5];
            dp[5] += g->dA_dSersic * gi[0];
            dp[6] += g->dA_drh * gi[0];
        }
    }
    free(ig);
    free(gimg);
    *chi2_out = chi2;
    return 0;
}

/* ------------------------------------------------------------------------
 * double restatement
 * ------------------------------------------------------------------------ */
typedef struct { double a, b, c, d; } m22d;
static m22d m22d_mul(m22d A, m22d B) {
    m22d r = {A.a * B.a + A.b * B.c, A.a * B.b + A.b * B.d,
              A.c * B.a + A.d * B.c, A.c * B.b + A.d * B.d};
    return r;
}

typedef struct {
    double amp, xcen, ycen, fxx, fyy, fxy;
    double jac[7][6];   /* d(A,x,y,fxx,fyy,fxy)/d(flux,ra,dec,q,pa,n,rh) */
} fpo_imgauss_d;

/* Optional double-precision mixture amplitudes, [n_sources][FPO_MAXRADII],
 * used instead of the proposal's float ones while set (finite differences
 * in sersic and rh without the float rounding of the amplitudes). */
static const double *g_amp_f64 = NULL;

static void convolve_source_f64(int band, int e, int g, int npsf,
                                const fpo_patch *P, const fpo_source *S,
                                fpo_imgauss_d *out) {
    const fpo_source *gal = S + g;
    int pstart = P->psfgauss_start[e];
    double G = P->G[e];
    int dcw = 4 * (P->n_sources * e + g);
    int cr = 2 * (P->n_sources * e + g);
    double q = gal->q, pa = gal->pa;
    m22d D = {P->D[dcw], P->D[dcw + 1], P->D[dcw + 2], P->D[dcw + 3]};
    double c = cos(pa), s = sin(pa);
    m22d R = {c, -s, s, c};
    m22d Sc = {1.0 / q, 0, 0, q};
    m22d dS = {-1.0 / (q * q), 0, 0, 1.0};
    m22d dR = {-s, -c, c, -s};
    m22d T = m22d_mul(m22d_mul(D, R), Sc);
    m22d dTq = m22d_mul(m22d_mul(D, R), dS);
    m22d dTpa = m22d_mul(m22d_mul(D, dR), Sc);
    m22d CW = {P->CW[dcw], P->CW[dcw + 1], P->CW[dcw + 2], P->CW[dcw + 3]};
    double s0 = (double)gal->ra - (double)P->crval[cr];
    double s1 = (double)gal->dec - (double)P->crval[cr + 1];
    double xc = CW.a * s0 + CW.b * s1 + (double)P->crpix[cr];
    double yc = CW.c * s0 + CW.d * s1 + (double)P->crpix[cr + 1];
    double flux = gal->fluxes[band];
    for (int p = 0; p < npsf; p++) {
        const fpo_psfgauss *pg = P->psfgauss + pstart + p;
        fpo_imgauss_d *ig = out + g * npsf + p;
        int k = pg->sersic_radius_bin;
        double r2 = P->rad2[k];
        double am = g_amp_f64 ? g_amp_f64[g * FPO_MAXRADII + k] : gal->mixture_amplitudes[k];
        /* Sigma = r2 T T^t + Cpsf */
        double s11 = r2 * (T.a * T.a + T.b * T.b) + pg->Cxx;
        double s12 = r2 * (T.a * T.c + T.b * T.d) + pg->Cxy;
        double s22 = r2 * (T.c * T.c + T.d * T.d) + pg->Cyy;
        double det = s11 * s22 - s12 * s12;
        double f11 = s22 / det, f12 = -s12 / det, f22 = s11 / det;
        double detF = f11 * f22 - f12 * f12;
        double K = G * pg->amp * sqrt(detF) / (2.0 * M_PI);
        ig->amp = K * flux * am;
        ig->fxx = f11; ig->fxy = f12; ig->fyy = f22;
        ig->xcen = xc + pg->xcen;
        ig->ycen = yc + pg->ycen;
        memset(ig->jac, 0, sizeof(ig->jac));
        /* dSigma = r2 (T dT^t + dT T^t); dF = -F dSigma F; dA = A/2 tr(Sigma dF) */
        m22d dTs[2] = {dTq, dTpa};
        for (int w = 0; w < 2; w++) {
            m22d B = dTs[w];
            double d11 = r2 * 2.0 * (T.a * B.a + T.b * B.b);
            double d12 = r2 * (T.a * B.c + T.b * B.d + T.c * B.a + T.d * B.b);
            double d22 = r2 * 2.0 * (T.c * B.c + T.d * B.d);
            m22d F = {f11, f12, f12, f22};
            m22d dS2 = {d11, d12, d12, d22};
            m22d dF = m22d_mul(m22d_mul(F, dS2), F);
            dF.a = -dF.a; dF.b = -dF.b; dF.c = -dF.c; dF.d = -dF.d;
            m22d Sg = {s11, s12, s12, s22};
            m22d M = m22d_mul(Sg, dF);
            int row = 3 + w;
            ig->jac[row][0] = 0.5 * ig->amp * (M.a + M.d);
            ig->jac[row][3] = dF.a;
            ig->jac[row][4] = dF.d;
            ig->jac[row][5] = dF.c;
        }
        ig->jac[0][0] = K * am;
        ig->jac[1][1] = CW.a; ig->jac[1][2] = CW.c;
        ig->jac[2][1] = CW.b; ig->jac[2][2] = CW.d;
        ig->jac[5][0] = K * flux * gal->damplitude_dnsersic[k];
        ig->jac[6][0] = K * flux * gal->damplitude_drh[k];
    }
}

/* All-double evaluation of one band.  use_cutoff selects the reference
 * kernel's exp-argument cutoff (common_kernel.cc:73,108); with use_cutoff=0
 * it follows the slow FP64 path (forcepho/slow/gaussmodel.py:351-476), which
 * has none.  dchi2 is double[n_sources*7]; the chi2 returned is the offset
 * form sum((r*ie)^2 - (d*ie)^2) of compute_gaussians_kernel.cc:286-293. */
int fpo_evaluate_band_f64(int band, const fpo_patch *P, const fpo_source *S,
                          int use_cutoff, double *chi2_out, double *dchi2,
                          double *residual_out) {
    int nsrc = P->n_sources;
    int npsf = P->n_psf_per_source[band];
    int bN = P->band_N[band], b0 = P->band_start[band];
    int ntot = nsrc * npsf;
    fpo_imgauss_d *ig = (fpo_imgauss_d *)malloc(sizeof(fpo_imgauss_d) * (size_t)(ntot > 0 ? ntot : 1));
    double *gimg = (double *)malloc(sizeof(double) * 6 * (size_t)(ntot > 0 ? ntot : 1));
    if (!ig || !gimg) { free(ig); free(gimg); return -1; }
    for (int i = 0; i < nsrc * FPO_NPARAMS; i++) dchi2[i] = 0.0;
    double chi2 = 0.0;
    for (int ee = 0; ee < bN; ee++) {
        int e = b0 + ee;
        for (int g = 0; g < nsrc; g++) convolve_source_f64(band, e, g, npsf, P, S, ig);
        memset(gimg, 0, sizeof(double) * 6 * (size_t)ntot);
        int npix = P->exposure_N[e];
        for (int p = 0; p < npix; p++) {
            int pix = P->exposure_start[e] + p;
            double xp = P->xpix[pix], yp = P->ypix[pix];
            double d = P->data[pix], ie = P->ierr[pix];
            double r = d;
            for (int i = 0; i < ntot; i++) {
                const fpo_imgauss_d *g = ig + i;
                double dx = xp - g->xcen, dy = yp - g->ycen;
                double vx = g->fxx * dx + g->fxy * dy, vy = g->fyy * dy + g->fxy * dx;
                double ea = dx * vx + dy * vy;
                if (use_cutoff && ea > FPO_MAX_EXP_ARG) continue;
                double H = 1.0 + (vx * vx + vy * vy - g->fxx - g->fyy) / 24.0;
                r -= g->amp * exp(-0.5 * ea) * H;
            }
            if (residual_out) residual_out[pix] = r;
            chi2 += (r * ie - d * ie) * (r * ie + d * ie);
            double rie2 = r * ie * ie;
            if (rie2 == 0.0) continue;
            for (int i = 0; i < ntot; i++) {
                const fpo_imgauss_d *g = ig + i;
                double dx = xp - g->xcen, dy = yp - g->ycen;
                double vx = g->fxx * dx + g->fxy * dy, vy = g->fyy * dy + g->fxy * dx;
                double ea = dx * vx + dy * vy;
                if (use_cutoff && ea > FPO_MAX_EXP_ARG) continue;
                double Gp = exp(-0.5 * ea);
                double H = 1.0 + (vx * vx + vy * vy - g->fxx - g->fyy) / 24.0;
                double w = -2.0 * rie2;
                double C = g->amp * Gp * H, c_h = g->amp * Gp;
                double *gi = gimg + 6 * i;
                gi[0] += w * Gp * H;
                gi[1] += w * (C * vx - c_h * (g->fxx * vx + g->fxy * vy) / 12.0);
                gi[2] += w * (C * vy - c_h * (g->fyy * vy + g->fxy * vx) / 12.0);
                gi[3] += w * (-0.5 * C * dx * dx - c_h * (1.0 - 2.0 * dx * vx) / 24.0);
                gi[4] += w * (-0.5 * C * dy * dy - c_h * (1.0 - 2.0 * dy * vy) / 24.0);
                gi[5] += w * (-C * dx * dy + c_h * (dy * vx + dx * vy) / 12.0);
            }
        }
        for (int i = 0; i < ntot; i++) {
            int gal = i / npsf;
            for (int k = 0; k < 7; k++) {
                double acc = 0.0;
                for (int m = 0; m < 6; m++) acc += ig[i].jac[k][m] * gimg[6 * i + m];
                dchi2[gal * FPO_NPARAMS + k] += acc;
            }
        }
    }
    free(ig);
    free(gimg);
    *chi2_out = chi2;
    return 0;
}

/* fpo_evaluate_band_f64 with the mixture amplitudes taken from
 * amps[n_sources][FPO_MAXRADII] (double) instead of the proposal. */
int fpo_evaluate_band_f64_amps(int band, const fpo_patch *P, const fpo_source *S,
                               const double *amps, int use_cutoff, double *chi2_out,
                               double *dchi2) {
    g_amp_f64 = amps;
    int rc = fpo_evaluate_band_f64(band, P, S, use_cutoff, chi2_out, dchi2, NULL);
    g_amp_f64 = NULL;
    return rc;
}

/* Like fpo_evaluate_band_mixed (float image Gaussians, double pixel math),
 * but contracting with the Jacobian per pixel, so that it can also return, per
 * gradient component, the sum over pixels of the absolute value of the
 * per-pixel contribution (dchi2_abs) and, if dchi2_abs_terms is not NULL, the
 * sum over pixels and image Gaussians of the absolute value of each
 * (pixel, Gaussian) term: the condition scales against which float rounding
 * is measured (a component much smaller than them is ill-conditioned; the
 * second also counts cancellation between the Gaussians of a source within a
 * pixel, e.g. of the mixed-sign d(amplitude)/d(rh) across radii).  If
 * dchi2_res_scale is not NULL it receives, per component, the sum over pixels
 * of FLT_EPSILON * (|d| + sum |model terms|) * 2 ie^2 |d model / d theta|:
 * how far float rounding of the residual alone can move the component.
 * dchi2, dchi2_abs, dchi2_abs_terms and dchi2_res_scale are
 * double[n_sources*7]. */
int fpo_evaluate_band_mixed_abs(int band, const fpo_patch *P, const fpo_source *S,
                                int use_cutoff, double *chi2_out, double *dchi2,
                                double *dchi2_abs, double *dchi2_abs_terms,
                                double *dchi2_res_scale) {
    int nsrc = P->n_sources;
    int npsf = P->n_psf_per_source[band];
    int bN = P->band_N[band], b0 = P->band_start[band];
    int ntot = nsrc * npsf;
    fpo_imgauss *ig = (fpo_imgauss *)malloc(sizeof(fpo_imgauss) * (size_t)(ntot > 0 ? ntot : 1));
    double *pc = (double *)malloc(sizeof(double) * FPO_NPARAMS * (size_t)(nsrc > 0 ? nsrc : 1));
    if (!ig || !pc) { free(ig); free(pc); return -1; }
    for (int i = 0; i < nsrc * FPO_NPARAMS; i++) dchi2[i] = dchi2_abs[i] = 0.0;
    if (dchi2_abs_terms)
        for (int i = 0; i < nsrc * FPO_NPARAMS; i++) dchi2_abs_terms[i] = 0.0;
    if (dchi2_res_scale)
        for (int i = 0; i < nsrc * FPO_NPARAMS; i++) dchi2_res_scale[i] = 0.0;
    double chi2 = 0.0;
    for (int ee = 0; ee < bN; ee++) {
        int e = b0 + ee;
        for (int g = 0; g < nsrc; g++) convolve_source_f32(band, e, g, npsf, P, S, ig);
        int npix = P->exposure_N[e];
        for (int p = 0; p < npix; p++) {
            int pix = P->exposure_start[e] + p;
            double xp = P->xpix[pix], yp = P->ypix[pix];
            double d = P->data[pix], ie = P->ierr[pix];
            double r = d, mabs = fabs(d);
            for (int i = 0; i < ntot; i++) {
                const fpo_imgauss *g = ig + i;
                double dx = xp - g->xcen, dy = yp - g->ycen;
                double fxx = g->fxx, fxy = g->fxy, fyy = g->fyy;
                double vx = fxx * dx + fxy * dy, vy = fyy * dy + fxy * dx;
                double ea = dx * vx + dy * vy;
                if (use_cutoff && ea > FPO_MAX_EXP_ARG) continue;
                double H = 1.0 + (vx * vx + vy * vy - fxx - fyy) / 24.0;
                r -= (double)g->amp * exp(-0.5 * ea) * H;
                mabs += fabs((double)g->amp * exp(-0.5 * ea) * H);
            }
            chi2 += (r * ie - d * ie) * (r * ie + d * ie);
            double rie2 = r * ie * ie;
            if (rie2 == 0.0) continue;
            /* a float evaluation of r carries an error of order
             * FLT_EPSILON * (|d| + sum |model terms|); through the weight
             * -2 r ie^2 it moves each component by that error times
             * 2 ie^2 |d model / d theta| */
            double rerr_w = 2.0 * (double)FLT_EPSILON * mabs * ie * ie / (-2.0 * rie2);
            memset(pc, 0, sizeof(double) * FPO_NPARAMS * (size_t)nsrc);
            for (int i = 0; i < ntot; i++) {
                const fpo_imgauss *g = ig + i;
                double dx = xp - g->xcen, dy = yp - g->ycen;
                double fxx = g->fxx, fxy = g->fxy, fyy = g->fyy, amp = g->amp;
                double vx = fxx * dx + fxy * dy, vy = fyy * dy + fxy * dx;
                double ea = dx * vx + dy * vy;
                if (use_cutoff && ea > FPO_MAX_EXP_ARG) continue;
                double Gp = exp(-0.5 * ea);
                double H = 1.0 + (vx * vx + vy * vy - fxx - fyy) / 24.0;
                double w = -2.0 * rie2;
                double C = amp * Gp * H, c_h = amp * Gp;
                double gA = w * Gp * H;
                double gx = w * (C * vx - c_h * (fxx * vx + fxy * vy) / 12.0);
                double gy = w * (C * vy - c_h * (fyy * vy + fxy * vx) / 12.0);
                double gfx = w * (-0.5 * C * dx * dx - c_h * (1.0 - 2.0 * dx * vx) / 24.0);
                double gfy = w * (-0.5 * C * dy * dy - c_h * (1.0 - 2.0 * dy * vy) / 24.0);
                double gfxy = w * (-C * dx * dy + c_h * (dy * vx + dx * vy) / 12.0);
                double t[FPO_NPARAMS];
                t[0] = g->dA_dFlux * gA;
                t[1] = g->dx_dAlpha * gx + (double)g->dy_dAlpha * gy;
                t[2] = g->dx_dDelta * gx + (double)g->dy_dDelta * gy;
                t[3] = g->dA_dQ * gA + (double)g->dFxx_dQ * gfx + (double)g->dFyy_dQ * gfy +
                       (double)g->dFxy_dQ * gfxy;
                t[4] = g->dA_dPA * gA + (double)g->dFxx_dPA * gfx + (double)g->dFyy_dPA * gfy +
                       (double)g->dFxy_dPA * gfxy;
                t[5] = g->dA_dSersic * gA;
                t[6] = g->dA_drh * gA;
                double *q = pc + (i / npsf) * FPO_NPARAMS;
                for (int k = 0; k < FPO_NPARAMS; k++) {
                    q[k] += t[k];
                    if (dchi2_abs_terms) dchi2_abs_terms[(i / npsf) * FPO_NPARAMS + k] += fabs(t[k]);
                }
            }
            for (int k = 0; k < nsrc * FPO_NPARAMS; k++) {
                dchi2[k] += pc[k];
                dchi2_abs[k] += fabs(pc[k]);
                if (dchi2_res_scale) dchi2_res_scale[k] += fabs(pc[k] * rerr_w);
            }
        }
    }
    free(ig);
    free(pc);
    *chi2_out = chi2;
    return 0;
}
