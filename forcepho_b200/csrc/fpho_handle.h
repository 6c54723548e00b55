// fpho_handle.h -- the patch handle behind the opaque fpho_patch of the C ABI,
// shared by the translation units that evaluate patches.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "fpho.h"
#include "fpho_impl.cuh"

struct fpho_patch {
    // host copies of the index arrays
    int n_bands = 0, n_exp = 0, n_sources = 0, n_radii = 0;
    int64_t npix = 0;
    std::vector<int16_t> band_start, band_N;
    std::vector<int> exposure_start, exposure_N, n_psf_per_source, psfgauss_start;
    std::vector<int> exp_band, exp_npsf, gauss_start;
    int n_gauss = 0;
    int max_g = 0;  // most image Gaussians of any exposure
    int64_t n_psfrows = 0;
    bool has_residual = false;
    // device pixel + index arrays
    float *d_data = nullptr, *d_ierr = nullptr, *d_xpix = nullptr, *d_ypix = nullptr,
          *d_residual = nullptr;
    int *d_exposure_start = nullptr, *d_exposure_N = nullptr;
    int16_t *d_band_start = nullptr, *d_band_N = nullptr;
    // device metadata
    float *d_rad2 = nullptr, *d_D = nullptr, *d_crpix = nullptr, *d_crval = nullptr,
          *d_CW = nullptr, *d_G = nullptr;
    int *d_npsf = nullptr, *d_psfgauss_start = nullptr;
    fpho_psfgauss *d_psfgauss = nullptr;
    int *d_exp_band = nullptr, *d_exp_npsf = nullptr, *d_gauss_start = nullptr;
    fpho_patch_struct *d_struct = nullptr;
    // tile plan (host copy of the tile list kept for batching); the default
    // configuration is variant 8 (4 warps sharing each 256-pixel tile's
    // Gaussians, 8 pixels per thread, 4 CTAs per SM), 256 records per
    // shared-memory stage, persistent schedule -- the fastest measured on the
    // 20-source, 8-band x 4-exposure, 128x128 px patch
    int variant = 8, live_cap = 256, n_tiles = 0;
    std::vector<fpho::TileDesc> h_tiles;
    std::vector<int> tile_band_start;
    fpho::TileDesc *d_tiles = nullptr;
    float4 *d_tbox_all = nullptr, *d_tbox_w = nullptr;
    int *d_tile_band_start = nullptr;
    // tile scheduling: 0 = one CTA per tile (hardware order), 1 = persistent
    // CTAs taking tiles by decreasing cost of the previous evaluation
    int schedule = 1;
    // 1: the residual pass in the reference's float arithmetic (see
    // fpho_patch_set_exact_residual)
    int exact_residual = 0;
    int test_extra_tx = 0;  // see fpho_patch_set_test_stall
    int *d_tile_cost = nullptr, *d_tile_order = nullptr, *d_tile_counter = nullptr;
    // workspace
    float *d_gtab = nullptr;
    float4 *d_gbox = nullptr;
    double *d_pchi2 = nullptr;
    float *d_pgrad = nullptr;
    fpho_source *d_prop = nullptr;
    // host-I/O evaluations: the results on the device, [chi2 (n_bands
    // doubles)][error word, 8 bytes][dchi2], copied back in one transfer into
    // a pinned staging buffer and from there to the caller's arrays
    unsigned char *d_io = nullptr;
    size_t d_io_cap = 0;
    unsigned char *h_io = nullptr;
    size_t h_io_cap = 0;
    int *d_err = nullptr;
    long long *d_pairs = nullptr;
    // flux solve (fpho_flux.cu): per-tile normal-equation partials and ATb
    double *d_pnorm = nullptr, *d_atb = nullptr;
    size_t d_pnorm_cap = 0, d_atb_cap = 0;
    int count_pairs = 0;
    // optional events recorded around the tile kernel (timing of the dominant kernel)
    cudaEvent_t ev_tile0 = nullptr, ev_tile1 = nullptr;
};

