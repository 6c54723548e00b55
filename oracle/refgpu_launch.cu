// refgpu_launch.cu -- host launcher for the reference's own CUDA kernel.
// TEST AND BENCHMARK INFRASTRUCTURE ONLY: the forcepho_b200 product never
// loads this library.
//
// The reference launches `EvaluateProposal` from Python through pycuda
// (forcepho/proposal.py:62-93 compile options -std=c++11 -maxrregcount=64;
// proposal.py:133-136 launch: grid = n_bands, block = 1024 threads, dynamic
// shared memory = shared_size).  pycuda is not available here, so this file
// compiles the reference's kernel source unchanged, where it lies
// (forcepho/src/compute_gaussians_kernel.cu, which includes header.hh,
// patch.cc, proposal.cu and common_kernel.cc), and adds a C launcher.  The
// kernel keeps its image Gaussians and accumulator in dynamic shared memory
// without bounds checks, so the launcher computes the size the kernel needs
// (NUMACCUMS accumulators + n_sources * n_psf_per_source ImageGaussians of
// the largest band) and refuses patches that need more than the 227 KB a
// B200 CTA can have, or more than MAXSOURCES sources.
#include "compute_gaussians_kernel.cu"

extern "C" int refgpu_shared_bytes(int n_gauss_total) {
    return (int)(NUMACCUMS * sizeof(Accumulator) + (size_t)n_gauss_total * sizeof(ImageGaussian));
}

extern "C" int refgpu_max_sources(void) { return MAXSOURCES; }

// Returns 0, or a cudaError_t value, or -1 for an argument the kernel cannot take.
extern "C" int refgpu_launch(void *dev_patch, void *dev_proposal, void *dev_chi2,
                             void *dev_response, int n_bands, int n_sources, int max_gauss_band,
                             int threads, void *stream) {
    if (n_sources < 1 || n_sources > MAXSOURCES || n_bands < 1 || max_gauss_band < 1) return -1;
    const int smem = refgpu_shared_bytes(max_gauss_band);
    if (smem > 227 * 1024 || threads < 32 || threads > 1024) return -1;
    cudaError_t e = cudaFuncSetAttribute(EvaluateProposal,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return (int)e;
    EvaluateProposal<<<n_bands, threads, smem, (cudaStream_t)stream>>>(dev_patch, dev_proposal,
                                                                        dev_chi2, dev_response);
    return (int)cudaGetLastError();
}
