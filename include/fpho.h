/*
 * fpho.h -- C ABI of forcepho_b200, a B200 (sm_100a) implementation of
 * forcepho's proposal-evaluation hot path: given a packed patch and a proposal
 * of Sersic source parameters, compute chi2 and dchi2/dtheta per band.
 *
 * Conventions
 *   - Every entry point returns an int status (FPHO_OK == 0).  Nothing aborts;
 *     the message of the last failure on the calling thread is returned by
 *     fpho_last_error().
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls are stream-ordered; a handle may be used by one host thread at a
 *     time.
 *   - Device memory is owned either by the caller (pointers passed in) or by
 *     a handle, freed by the matching *_free call.  Handle memory comes from
 *     the device's default memory pool, which keeps freed memory for reuse
 *     until the process exits; a *_free waits for the device first.
 *   - No torch, numpy or CUDA types appear in the signatures.
 *
 * Struct layouts below are the reference's device ABI and are byte-compatible
 * with it, so patches packed by the reference's python packer
 * (forcepho/patches/patch.py:43-74) can be handed over unchanged.
 */
#ifndef FPHO_H
#define FPHO_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FPHO_API __attribute__((visibility("default")))
#else
#define FPHO_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Compile-time limits of the reference ABI (forcepho/src/kernel_limits.h:5-26). */
#define FPHO_MAXBANDS 30     /* Source.fluxes length */
#define FPHO_MAXSOURCES 30   /* Response stride of the reference (sources per band) */
#define FPHO_NPARAMS 7       /* flux, ra, dec, q, pa, sersic, rh */
#define FPHO_MAXRADII 10     /* Source mixture arrays length */
#define FPHO_MAX_EXP_ARG 36.0f

/* Limits of this implementation (lifted from the reference's 30 sources and
 * 48 KB of shared memory per band). */
#define FPHO_MAX_ACTIVE_SOURCES 1024
#define FPHO_MAX_PSF_PER_SOURCE 1024

enum fpho_status {
    FPHO_OK = 0,
    FPHO_ERR_INVALID = 1,   /* bad argument or inconsistent patch description */
    FPHO_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    FPHO_ERR_NOMEM = 3,     /* host or device allocation failed */
    FPHO_ERR_LIMIT = 4,     /* a size exceeds a limit of this implementation */
    FPHO_ERR_STATE = 5,     /* call not valid in the handle's current state */
    FPHO_ERR_KERNEL = 6     /* a kernel reported an error word (bounded wait ran out, bad index) */
};

/* evaluate flags */
#define FPHO_IO_HOST 1u          /* proposal and outputs are host pointers; the call synchronizes */
#define FPHO_WANT_RESIDUAL 2u    /* write data - model to the patch's residual array */
#define FPHO_CHI2_ONLY 4u        /* residual pass and chi2 only; dchi2 is not written (may be NULL) */

/* One PSF Gaussian already matched to a Sersic radius bin:
 * forcepho/src/patch.cc:101-118 (28 bytes). */
typedef struct fpho_psfgauss {
    float amp;
    float xcen, ycen;
    float Cxx, Cyy, Cxy;
    int32_t sersic_radius_bin;
} fpho_psfgauss;

/* The patch description: forcepho/src/patch.cc:23-99 (152 bytes on LP64).
 * Pointers are host pointers when given to fpho_patch_create and device
 * pointers in the copy returned by fpho_patch_device_struct. */
typedef struct fpho_patch_struct {
    float *data, *ierr, *xpix, *ypix, *residual;
    int32_t *exposure_start;   /* [n_exp] first pixel of each exposure */
    int32_t *exposure_N;       /* [n_exp] pixels (with padding) of each exposure */
    int16_t *band_start;       /* [n_bands] first exposure of each band */
    int16_t *band_N;           /* [n_bands] exposures of each band */
    int32_t n_sources;
    int32_t n_radii;
    float *rad2;               /* [n_radii] squared Sersic radii, arcsec^2 */
    float *D;                  /* [n_exp][n_sources][2][2] pixels per arcsec */
    float *crpix;              /* [n_exp][n_sources][2] */
    float *crval;              /* [n_exp][n_sources][2] */
    float *CW;                 /* [n_exp][n_sources][2][2] d(pixel)/d(ra, dec) */
    float *G;                  /* [n_exp] flux to counts */
    int32_t *n_psf_per_source; /* [n_bands] */
    fpho_psfgauss *psfgauss;   /* [sum_e n_sources * n_psf_per_source[band(e)]] */
    int32_t *psfgauss_start;   /* [n_exp] */
} fpho_patch_struct;

/* One source of a proposal: forcepho/src/proposal.cu:13-28 (264 bytes). */
typedef struct fpho_source {
    float ra, dec;
    float q, pa;
    float nsersic, rh;
    float fluxes[FPHO_MAXBANDS];
    float mixture_amplitudes[FPHO_MAXRADII];
    float damplitude_drh[FPHO_MAXRADII];
    float damplitude_dnsersic[FPHO_MAXRADII];
} fpho_source;

/* Per-band gradient block of the reference: forcepho/src/proposal.cu:33-39. */
typedef struct fpho_response {
    float dchi2_dparam[FPHO_MAXSOURCES * FPHO_NPARAMS];
} fpho_response;

typedef struct fpho_patch fpho_patch;   /* opaque: device copy of one patch + workspace */
typedef struct fpho_batch fpho_batch;   /* opaque: many patches evaluated by one launch */

/* ---- library ---------------------------------------------------------- */

/* Message of the last failure on this thread ("" if none). */
FPHO_API const char *fpho_last_error(void);
/* ABI version: (major << 16) | minor. */
FPHO_API int fpho_abi_version(void);
/* sizeof checks for bindings: 0 patch_struct, 1 source, 2 psfgauss, 3 response. */
FPHO_API int fpho_sizeof(int which);

/* ---- patches ---------------------------------------------------------- */

/* Copy every array referenced by the host-side patch description to the
 * device and prepare the tile plan.  Replaces GPUPatchMixin.send_to_device
 * (forcepho/patches/device_patch.py:268-300).  n_bands is the number of
 * bands (the reference passes it as the grid size).  If `return_residual` is
 * non-zero a device residual array is allocated (host->residual is ignored).
 * Sizes are derived from the index arrays; they are validated on the host. */
FPHO_API int fpho_patch_create(const fpho_patch_struct *host, int n_bands, int return_residual,
                      void *stream, fpho_patch **out);

/* As fpho_patch_create, but desc->data, ierr, xpix and ypix are DEVICE
 * pointers (copied device to device; the caller keeps ownership), e.g. the
 * output of fpho_store_gather.  The index arrays and the metadata are host
 * pointers, as for fpho_patch_create.  No counterpart in the reference, whose
 * pixel arrays always start on the host (device_patch.py:268-300). */
FPHO_API int fpho_patch_create_device_pixels(const fpho_patch_struct *desc, int n_bands,
                                             int return_residual, void *stream, fpho_patch **out);

/* Replace the per-scene metadata (n_sources, rad2, D, crpix, crval, CW, G,
 * n_psf_per_source, psfgauss, psfgauss_start) with new host arrays, keeping
 * the pixel arrays.  Replaces GPUPatchMixin.replace_device_meta_ptrs
 * (device_patch.py:302-311). */
FPHO_API int fpho_patch_replace_meta(fpho_patch *p, const fpho_patch_struct *host, void *stream);

/* Swap the device data and residual arrays, so that the residual of the last
 * evaluation becomes the data.  Replaces the pointer swap of
 * GPUPatchMixin.swap_on_device (device_patch.py:346-367); call
 * fpho_patch_replace_meta before it to install the next scene's metadata. */
FPHO_API int fpho_patch_swap_data_residual(fpho_patch *p, void *stream);

/* Copy one pixel array to host memory (npix floats).  which: 0 data,
 * 1 residual, 2 ierr, 3 xpix, 4 ypix.  Replaces GPUPatchMixin.retrieve_array
 * (device_patch.py:369-375).  Synchronizes `stream`. */
FPHO_API int fpho_patch_retrieve(fpho_patch *p, int which, float *host_out, void *stream);

/* Device pointer to a fpho_patch_struct (device pointers inside) describing
 * the patch, as GPUPatchMixin.device_patch (device_patch.py:313-344). */
FPHO_API int fpho_patch_device_struct(fpho_patch *p, const void **dev_struct);

/* Sizes: out[0] n_bands, out[1] n_exp, out[2] npix, out[3] n_sources,
 * out[4] n_radii, out[5] n_tiles, out[6] total image Gaussians. */
FPHO_API int fpho_patch_info(const fpho_patch *p, int64_t out[7]);

FPHO_API int fpho_patch_free(fpho_patch *p);

/* ---- evaluation ------------------------------------------------------- */

/* Evaluate a proposal on a patch: chi2 per band and dchi2/dtheta per band
 * and source.  Replaces the launch EvaluateProposal<<<n_bands, 1024, 48000>>>
 * (forcepho/src/compute_gaussians_kernel.cu:212-312) made by
 * GPUProposer.evaluate_proposal (forcepho/proposal.py:96-152).
 *   proposal  fpho_source[n_sources]
 *   chi2      double[n_bands]: sum over the band's pixels of
 *             (r*ie - d*ie)(r*ie + d*ie), r = data - model
 *   dchi2     float[n_bands][dchi2_stride]: dchi2[b][7*s + k] for source s and
 *             parameter k in (flux, ra, dec, q, pa, sersic, rh);
 *             dchi2_stride >= 7*n_sources (210 gives the reference's
 *             fpho_response layout; entries past 7*n_sources are zeroed).
 *   flags     FPHO_IO_HOST, FPHO_WANT_RESIDUAL
 * n_sources must equal the patch's n_sources. */
FPHO_API int fpho_evaluate_proposal(fpho_patch *p, const fpho_source *proposal, int n_sources,
                           double *chi2, float *dchi2, int dchi2_stride,
                           unsigned flags, void *stream);

/* The reference kernel's exact argument list: a device fpho_patch_struct*
 * (as returned by fpho_patch_device_struct for this handle), a device
 * Source[n_sources], a device double[n_bands] and a device
 * fpho_response[n_bands].  Same computation as fpho_evaluate_proposal. */
FPHO_API int fpho_EvaluateProposal(fpho_patch *p, const void *dev_patch_struct, const void *dev_proposal,
                          void *pchi2, void *pdchi2_dp, void *stream);

/* Design matrix of the proposal's sources: X[n_sources][npix] (device,
 * float) = the unit-flux model of each source at every pixel of the patch
 * (sum over its image Gaussians of dA/dflux * G * H, the exp-argument cutoff
 * applied), in the patch's packed pixel order.  Replaces the loop of
 * one-source renders of DevicePatchMixin.design_matrix
 * (forcepho/patches/device_patch.py:198-238), which divides each source's
 * model by its flux; the flux solve on top is forcepho_b200.fitting.
 * Stream-ordered, no synchronization; check fpho_patch_error_word after. */
FPHO_API int fpho_patch_design_matrix(fpho_patch *p, const void *dev_proposal, int n_sources,
                                      float *dev_X, void *stream);

/* ---- proposals built on the device -------------------------------------- */

typedef struct fpho_spline fpho_spline;   /* opaque: Sersic amplitude splines on the device */

/* Upload the bicubic B-splines of the Sersic mixture amplitudes: one spline
 * per mixture radius over (sersic, rh), sharing knots tx[ntx], ty[nty]
 * (scipy RectBivariateSpline.get_knots()); coeffs[n_radii][ntx-4][nty-4]
 * (get_coeffs() of each); radii[n_radii] in arcsec; sersic_min = lowest
 * sersic index of the table.  Replaces Galaxy.initialize_splines
 * (forcepho/sources.py:623-645). */
FPHO_API int fpho_spline_create(const double *tx, int ntx, const double *ty, int nty,
                                const double *coeffs, int n_radii, const double *radii,
                                double sersic_min, void *stream, fpho_spline **out);
FPHO_API int fpho_spline_free(fpho_spline *s);

/* Build the device proposal fpho_source[n_sources] from device parameters
 * theta[n_sources][n_bands + 6] in Scene order (flux_1..flux_B, ra, dec, q,
 * pa, sersic, rhalf), with mixture amplitudes and their sersic / rh
 * derivatives from the splines (including the reference's branches for
 * sersic below the table and rh < 0).  Replaces Scene.get_proposal /
 * Galaxy.proposal (forcepho/sources.py:80-97, 607-694). */
FPHO_API int fpho_build_proposal(const fpho_spline *s, const double *theta, int n_sources,
                                 int n_bands, fpho_source *out, void *stream);

/* The same for the sources of many patches at once: source s has
 * src_bands[s] bands and its parameters start at theta[src_offset[s]]
 * (src_bands, src_offset and theta in device memory).  No reference
 * counterpart: it builds the proposals of a batch (fpho_batch_evaluate). */
FPHO_API int fpho_build_proposal_batch(const fpho_spline *s, const double *theta, int n_sources,
                                       const int *src_bands, const long long *src_offset,
                                       fpho_source *out, void *stream);

/* The proposal from unconstrained parameters: q = lower + range *
 * sigmoid(z) per parameter (BoundedTransform.transform,
 * forcepho/model.py:596-637), then as fpho_build_proposal (src_bands and
 * src_offset NULL: every source has n_bands bands, stride n_bands + 6) or
 * fpho_build_proposal_batch (both given; n_bands ignored).  z, lower, range
 * (= upper - lower) and the optional q_out are device arrays in the
 * parameters' Scene order.  One launch replaces the transform and the
 * proposal build of a sampler step. */
FPHO_API int fpho_build_proposal_bounded(const fpho_spline *s, const double *z,
                                         const double *lower, const double *range,
                                         int n_sources, int n_bands, const int *src_bands,
                                         const long long *src_offset, double *q_out,
                                         fpho_source *out, void *stream);

/* lnp(z) = -sum(chi2)/2 + sum_i log jac_i and d lnp / dz_i
 *   = -jac_i / 2 * sum_{k = map_offset[i]}^{map_offset[i+1]-1} dchi2[map_index[k]]
 *     + (1 - 2 s_i),
 * s_i = sigmoid(z_i), jac_i = range_i s_i (1 - s_i) (FastPosterior.evaluate
 * with BoundedTransform, forcepho/model.py:323-387, 596-637).  The map lists
 * each parameter's entries of the evaluation's dchi2 (a flux: its band; a
 * shape parameter: every band, in band order; summed in double), so that it
 * also stacks the per-band gradient as stack_grad (forcepho/model.py:387-405)
 * does.  work[n_work] holds one partial per 256 parameters; *counter
 * (device, zero before the first call) is reset by every call.  The lnp sum
 * is in a fixed order.  One launch, in place of the transform's and the
 * stacking's elementwise steps. */
FPHO_API int fpho_bounded_lnp_grad(int n_params, const double *z, const double *lower,
                                   const double *range, const float *dchi2,
                                   const int *map_offset, const long long *map_index,
                                   const double *chi2, int n_chi2, double *grad_out,
                                   double *lnp_out, double *work, int n_work,
                                   unsigned *counter, void *stream);

/* Spline values and derivatives at m device points (x = sersic, y = rh):
 * out[m][n_radii][3] = (value, d/dsersic, d/drh). */
FPHO_API int fpho_spline_points(const fpho_spline *s, const double *x, const double *y, int m,
                                double *out, void *stream);

/* ---- batched evaluation ------------------------------------------------ */

/* Build a batch of patches evaluated together by one persistent launch (the
 * reference evaluates one patch per launch, forcepho/proposal.py:133-136, one
 * patch per MPI child, forcepho/dispatcher.py).  Every patch is switched to
 * the default batched tile shape (64 threads x 8 pixels) with `live_cap`;
 * rebuild the batch after fpho_patch_replace_meta or fpho_patch_set_config on
 * a member.  The patch handles must outlive the batch.  Equivalent to
 * fpho_batch_create_config(patches, n, -1, live_cap, 0, stream, out). */
FPHO_API int fpho_batch_create(fpho_patch *const *patches, int n, int live_cap, void *stream,
                               fpho_batch **out);

/* As fpho_batch_create with the launch configuration chosen by the caller
 * (the batch autotuner; no reference counterpart, whose launch shape is
 * thread_block, shared_size and max_registers, forcepho/proposal.py:62-65,88-89):
 *   variant      the patches' tile variant, one of fpho_batch_variants
 *                (-1: the default, 64 threads x 8 pixels);
 *   live_cap     image-Gaussian records per shared-memory stage;
 *   ctas_per_sm  cap on resident CTAs per SM of the persistent grid, 0 for
 *                as many as fit.
 * FPHO_ERR_INVALID for a variant without a batched kernel. */
FPHO_API int fpho_batch_create_config(fpho_patch *const *patches, int n, int variant,
                                      int live_cap, int ctas_per_sm, void *stream,
                                      fpho_batch **out);

/* The tile variants that have a batched kernel: fills out[0..cap) and
 * returns how many there are (an entry is -1 if its patch variant is not
 * compiled). */
FPHO_API int fpho_batch_variants(int *out, int cap);

/* The configuration of a batch: out = (variant, live_cap, ctas_per_sm cap,
 * persistent grid size). */
FPHO_API int fpho_batch_config(const fpho_batch *b, int out[4]);

/* out[0] patches, out[1] total sources, out[2] total bands, out[3] total dchi2
 * floats, out[4] work items (tiles), out[5] persistent grid, out[6] exposures. */
FPHO_API int fpho_batch_info(const fpho_batch *b, int64_t out[7]);

/* Evaluate one proposal per patch.
 *   proposals  fpho_source[sum n_sources], patch i's sources after patch i-1's
 *   chi2       double[sum n_bands], patch by patch
 *   dchi2      float[sum n_bands * n_sources * 7], patch by patch, each
 *              [n_bands][n_sources][7]
 *   flags      FPHO_IO_HOST (host buffers; the call synchronizes)
 * A batch is used by one stream at a time. */
FPHO_API int fpho_batch_evaluate(fpho_batch *b, const fpho_source *proposals, double *chi2,
                                 float *dchi2, unsigned flags, void *stream);

/* As the patch versions: evaluated-pair counting and timing of the tile kernel. */
FPHO_API int fpho_batch_count_pairs(fpho_batch *b, int enable, long long *last_count);
FPHO_API int fpho_batch_time_tiles(fpho_batch *b, int enable);
FPHO_API int fpho_batch_last_tile_ms(fpho_batch *b, float *ms);
/* The batch's error word (0 = no kernel reported an error) of the last
 * evaluation; device-buffer evaluations (without FPHO_IO_HOST) do not check
 * it.  Synchronizes the device.  No reference counterpart. */
FPHO_API int fpho_batch_error_word(fpho_batch *b, int *out);
FPHO_API int fpho_batch_free(fpho_batch *b);

/* ---- evaluation without allocation (no counterpart in the reference) ---- */

/* Size of the device array that holds all scratch of
 * fpho_evaluate_proposal_noalloc (one per device, alive until process exit). */
#define FPHO_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)

/* Same computation as fpho_evaluate_proposal, for callers that cannot
 * allocate device memory: plugins whose host framework owns every device
 * allocation (its allocator alone may take device memory, so that its
 * accounting and limits hold), and services that must not grow or fragment
 * device memory after start-up.  It calls no
 * cudaMalloc/cudaFree and no allocating library routine; its scratch (tile
 * plan, image Gaussians, per-tile partial sums) lives in a file-scope device
 * array of FPHO_NOALLOC_SCRATCH_BYTES.
 *   patch         host struct whose array pointers are DEVICE pointers
 *                 (residual may be NULL; if set, data - model is written there)
 *   n_bands, n_exp  band and exposure counts of the index arrays
 *   total_pixels  length of the pixel arrays (data, ierr, xpix, ypix and
 *                 residual); every exposure's run [exposure_start,
 *                 exposure_start + exposure_N) must lie inside it
 *   max_psf_per_source  upper bound on n_psf_per_source[]
 *   dev_proposal, dev_chi2, dev_dchi2  device fpho_source[n_sources],
 *                 double[n_bands], float[n_bands][dchi2_stride]
 *   dev_status    optional device int: 0, or error bits (1 a bounded wait gave
 *                 up, 2 inconsistent index arrays -- bands overlapping, an
 *                 exposure's pixels outside total_pixels, a negative
 *                 psfgauss_start --, 4 a size bound was exceeded, 8 a PSF
 *                 radius bin out of range).  On any error every dev_chi2
 *                 entry is NaN, with or without dev_status.
 * The psfgauss rows the exposures index (psfgauss_start[e] + component) must
 * exist: the device array's length is not passed, so it cannot be checked.
 * Sizes whose scratch exceeds FPHO_NOALLOC_SCRATCH_BYTES are rejected with
 * FPHO_ERR_LIMIT.  The first call on a device looks up the array's address
 * and sets a kernel attribute (once, to the shared-memory ceiling): make it
 * before any stream capture.  The address is kept until the process exits, so
 * a device reset is not supported.  All calls
 * share the array, which keeps the last call's contents; calls that overlap
 * on the GPU race and must be serialized.  The call is asynchronous. */
FPHO_API int fpho_evaluate_proposal_noalloc(const fpho_patch_struct *patch, int n_bands,
                                            int n_exp, int64_t total_pixels,
                                            int max_psf_per_source,
                                            const fpho_source *dev_proposal, double *dev_chi2,
                                            float *dev_dchi2, int dchi2_stride, int *dev_status,
                                            void *stream);

/* Read (and keep) the error word of the last evaluation: bit 0 set when a
 * bounded wait on a bulk copy gave up.  Synchronizes the device. */
FPHO_API int fpho_patch_error_word(fpho_patch *p, int *out);

/* ---- tuning (no counterpart in the reference) --------------------------- */

/* Number of compiled tile-kernel variants; out[0] threads per CTA and out[1]
 * tile pixels per thread of `variant`. */
FPHO_API int fpho_variant_info(int variant, int out[2]);

/* Number of compiled tile-kernel variants; out[0] threads per CTA, out[1]
 * pixels per tile, out[2] warps that share each tile's image Gaussians (0:
 * every thread evaluates its own pixels over all of them; NW > 0: NW warps
 * each hold all of the tile's pixels and take 1/NW of its Gaussians). */
FPHO_API int fpho_variant_shape(int variant, int out[3]);

/* Select the tile-kernel variant and the shared-memory stage size (image
 * Gaussians per chunk) used by this patch; re-plans the tiles if the tile
 * size changes.  Default: variant 8 (128 threads: 4 warps sharing each
 * 256-pixel tile's Gaussians, 8 pixels per thread), live_cap 256. */
FPHO_API int fpho_patch_set_config(fpho_patch *p, int variant, int live_cap, void *stream);

/* Tile scheduling of this patch: 0 = one CTA per tile; 1 (default) = as many
 * persistent CTAs as fit on the GPU, taking tiles in decreasing order of
 * their cost in the previous evaluation (kept image Gaussians x pixels);
 * patches of at most 4 tiles per SM always run one CTA per tile.
 * Results are identical either way.  No reference counterpart (the
 * reference launches one block per band). */
FPHO_API int fpho_patch_set_schedule(fpho_patch *p, int schedule);

/* Exact-residual mode (a parity diagnostic; no reference counterpart).  With
 * `on` non-zero the residual pass of this patch's evaluations follows the
 * reference's ComputeResidualImage (forcepho/src/common_kernel.cc:57-83) in
 * float operation by operation, each operation rounded once, with exp
 * evaluated in double and rounded once to float; the gradient pass is
 * unchanged.  Residuals then equal the reference CPU kernel's wherever its
 * float exp is correctly rounded.  Slower than the default pass; compiled for
 * variant 3 (64 threads x 4 pixels) only: FPHO_ERR_STATE for other variants. */
FPHO_API int fpho_patch_set_exact_residual(fpho_patch *p, int on);

/* For tests of the error path only (no reference counterpart): with `on`
 * non-zero, every staging wait of this patch's tile kernel expects 16 bytes
 * that no copy delivers, so each wait gives up after its bounded spin (about
 * 2^22 polls), sets the error word and the evaluation returns
 * FPHO_ERR_KERNEL (host I/O) or leaves the word for fpho_patch_error_word.
 * Nothing hangs or faults, and the results of such an evaluation are
 * meaningless.  Switch it off to evaluate normally again.  Refused
 * (FPHO_ERR_STATE) unless every tile is staged at most once and runs in its
 * own CTA: more image Gaussians per exposure than the stage holds, or a
 * persistent schedule over many tiles. */
FPHO_API int fpho_patch_set_test_stall(fpho_patch *p, int on);

/* Enable counting of evaluated (pixel, image Gaussian) pairs, i.e. pairs that
 * survive the per-tile culling; *last_count receives the count of the last
 * evaluation (synchronizes).  last_count may be NULL. */
FPHO_API int fpho_patch_count_pairs(fpho_patch *p, int enable, long long *last_count);

/* ---- linear flux solve ------------------------------------------------- */

/* The weighted normal equations of the flux fit of the patch's sources at
 * the shapes of `dev_proposal` (device fpho_source[n_sources]), per band:
 * dev_ata[n_bands][n_sources][n_sources] = sum_pix ierr^2 X_s X_t and
 * dev_atb[n_bands][n_sources] = sum_pix ierr^2 X_s data, where X_s is source
 * s's model at unit flux and data the patch's device data.  Replaces the
 * reference's design matrix and normal-equation products
 * (forcepho/patches/device_patch.py:185-238, forcepho/fitting.py:573-594);
 * X is never stored: each tile forms FP64 partial sums, reduced per band in
 * a fixed order.  Asynchronous on `stream`. */
FPHO_API int fpho_patch_flux_normal_equations(fpho_patch *p, const void *dev_proposal,
                                              int n_sources, double *dev_ata, double *dev_atb,
                                              void *stream);

/* forcepho's optimize_fluxes (forcepho/fitting.py:597-627) on the device:
 * the normal equations above, then per band an FP64 Cholesky solve.
 * dev_flux[n_bands][n_sources] = ATA^-1 ATb (the maximum-likelihood fluxes
 * given the shapes), dev_precision[n_bands][n_sources][n_sources] = ATA (the
 * flux precision matrix), dev_status[n_bands] (optional): 0, or 1 where ATA
 * is not positive definite (that band's fluxes are NaN; the reference
 * raises LinAlgError).  At most 64 sources.  Asynchronous on `stream`. */
FPHO_API int fpho_patch_optimize_fluxes(fpho_patch *p, const void *dev_proposal, int n_sources,
                                        double *dev_flux, double *dev_precision,
                                        int *dev_status, void *stream);

/* Copy the image-Gaussian records that the last evaluation built for one
 * exposure to host memory (32 floats each: -xcen, -ycen, fxx, fxy, fyy, amp,
 * -amp*c0 and c0 = 1 - (fxx+fyy)/24, each stored twice, in floats 0..15; the
 * 15-term Jacobian in floats 16..30; the source index as int bits in float
 * 31); *n_out receives the number of records.  Synchronizes the device. */
FPHO_API int fpho_patch_image_gaussians(fpho_patch *p, int exposure, float *host_out,
                                        int max_records, int *n_out);

/* Enable (1) or disable (0) CUDA events recorded immediately before and after
 * the pixel-tile kernel of every following evaluation, on its stream, so the
 * dominant kernel can be timed on its own. */
FPHO_API int fpho_patch_time_tiles(fpho_patch *p, int enable);
/* Milliseconds of the tile kernel of the last evaluation (waits for it). */
FPHO_API int fpho_patch_last_tile_ms(fpho_patch *p, float *ms);

/* Throughput probes for roofline denominators: which 0 = packed FP32 FMA
 * chains (flops = blocks*threads*iters*32), 1 = MUFU.EX2 chains
 * (ops = blocks*threads*iters*8).  dev_out: device float[blocks] scratch. */
FPHO_API int fpho_probe_launch(int which, int blocks, int threads, int iters, float *dev_out,
                               void *stream);

/* ---- exposure store: super-pixel exposures resident in GPU memory ------ */

/* Replaces the host packing of StorePatch (forcepho/patches/pixel_patch.py:
 * 124-198 pack_pix, 297-342 find_exposures/find_pixels): the exposures of a
 * pixel store are uploaded once, in the pixel store's layout -- per exposure
 * (nside_x/s, nside_y/s, 2 s^2) floats, each super-pixel's s x s fluxes in
 * row-major order then their inverse errors (forcepho/patches/storage.py:
 * 62-96, 245-276) -- and a patch's pixels are selected and packed on the
 * device. */
typedef struct fpho_store fpho_store;

#define FPHO_REGION_CIRCLE 1
#define FPHO_REGION_RECT 2

/* The region test of one exposure, in that exposure's pixels.  A super-pixel
 * is selected if one of its corner pixels -- (0,0), (1,0), (1,1), (0,1) times
 * (s-1) from its first pixel -- passes:
 *   FPHO_REGION_CIRCLE  p = {xc, yc, r2}: (xc-x)^2 + (yc-y)^2 < r2 in double
 *                       (CircularRegion.contains, forcepho/region.py:91-116);
 *   FPHO_REGION_RECT    p = {ra_min, ra_max, dec_min, dec_max, crpix1, crpix2
 *                       (1-based), cd11, cd12, cd21, cd22, crval1, crval2,
 *                       lonpole}: the corner's TAN sky position strictly inside
 *                       the box (RectangularRegion.contains, region.py:168-192). */
typedef struct fpho_region {
    int32_t kind;
    int32_t reserved;
    double p[14];
} fpho_region;

/* A store for up to max_exposures exposures of nside_x x nside_y pixels in
 * super-pixels of super_pixel_size (all memory is allocated here). */
FPHO_API int fpho_store_create(int nside_x, int nside_y, int super_pixel_size, int max_exposures,
                               fpho_store **out);
/* Append one exposure's super-pixel array (host memory, or device memory if
 * on_device); *index receives its store index. */
FPHO_API int fpho_store_add_exposure(fpho_store *st, const float *superpixels, int on_device,
                                     void *stream, int *index);
/* out: nsx, nsy, super_pixel_size, exposures, capacity, bytes per exposure. */
FPHO_API int fpho_store_info(const fpho_store *st, int64_t out[6]);
/* Selected super-pixels of each listed exposure (host n_superpixels[n_exp]);
 * synchronizes.  StorePatch.find_exposures keeps exposures with at least one. */
FPHO_API int fpho_store_count(fpho_store *st, int n_exp, const int32_t *exposures,
                              const fpho_region *regions, int32_t *n_superpixels, void *stream);
/* Pack the selected pixels of the listed exposures, in that order, into the
 * device arrays data, ierr, xpix, ypix (npix_capacity floats each; LIMIT if
 * the patch is larger).  background (host, n_exp, nullable) is subtracted from
 * the fluxes in float; max_snr > 0 caps ierr at max_snr / flux where
 * flux * ierr > max_snr (PixelPatch._cap_snr).  exposure_start/exposure_N
 * (host, n_exp) receive the pixel index of each exposure.  Synchronizes. */
FPHO_API int fpho_store_gather(fpho_store *st, int n_exp, const int32_t *exposures,
                               const fpho_region *regions, const float *background, float max_snr,
                               float *data, float *ierr, float *xpix, float *ypix,
                               int64_t npix_capacity, int32_t *exposure_start,
                               int32_t *exposure_N, void *stream);
/* Enable (1) or disable (0) CUDA events around the gather kernel of every
 * following fpho_store_gather; fpho_store_last_gather_ms gives the last one's
 * milliseconds (the gather synchronizes, so it is ready on return). */
FPHO_API int fpho_store_time_gather(fpho_store *st, int enable);
FPHO_API int fpho_store_last_gather_ms(const fpho_store *st, float *ms);
FPHO_API int fpho_store_free(fpho_store *st);

#ifdef __cplusplus
}
#endif
#endif /* FPHO_H */
