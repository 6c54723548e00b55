// fpho_probe.cu -- throughput probes used as roofline denominators.
//
// The pixel kernels are bound by the FP32 pipe (FFMA) with the SFU (MUFU.EX2)
// as the secondary limit; neither figure is in the measured-peaks file, so the
// benchmark measures them live on the same GPU with these two kernels:
//   probe_ffma2  8 independent packed f32x2 FMA chains per thread
//                (flops = threads * iters * 8 chains * 2 lanes * 2);
//   probe_ex2    8 independent MUFU.EX2 chains per thread
//                (ex2 ops = threads * iters * 8).
#include <cuda_runtime.h>

#include "fpho_impl.cuh"
#include "fpho_internal.h"

namespace fpho {

__global__ void probe_ffma2(int iters, float *out) {
    v2 a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = pk(threadIdx.x * 1e-3f + j, blockIdx.x * 1e-3f - j);
    const v2 b = pk(0.999999f, 1.000001f), c = pk(1e-6f, -1e-6f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fma2(a[j], b, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += lo(a[j]) + hi(a[j]);
    if (s == 1234.5678f) out[blockIdx.x] = s;  // keeps the chains live
}

__global__ void probe_ex2(int iters, float *out) {
    float a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = -(threadIdx.x & 7) * 0.01f - j * 0.1f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = -ex2f(a[j]);
    }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += a[j];
    if (s == 1234.5678f) out[blockIdx.x] = s;
}

}  // namespace fpho

// which: 0 FFMA2 probe, 1 EX2 probe.  Launches `blocks` x `threads`.
extern "C" FPHO_API int fpho_probe_launch(int which, int blocks, int threads, int iters,
                                          float *dev_out, void *stream) {
    fpho::clear_error();
    if (blocks < 1 || threads < 32 || threads > 1024 || iters < 1 || !dev_out)
        return fpho::set_error(FPHO_ERR_INVALID, "bad probe launch arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (which == 0)
        fpho::probe_ffma2<<<blocks, threads, 0, s>>>(iters, dev_out);
    else if (which == 1)
        fpho::probe_ex2<<<blocks, threads, 0, s>>>(iters, dev_out);
    else
        return fpho::set_error(FPHO_ERR_INVALID, "probe %d unknown", which);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fpho::set_error(FPHO_ERR_CUDA, "probe launch: %s", cudaGetErrorString(e));
    return FPHO_OK;
}
