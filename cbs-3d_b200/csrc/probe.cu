// Measurement probes used to state the rooflines of the solver kernels: the
// copy bandwidth of a buffer pair that fits in L2 (or not), timed with CUDA
// events on the probe's own stream.
#include "cbs3d_gpu.h"
#include "pcg.cuh"

#include <cuda_runtime.h>

namespace cbs3d {
namespace {

// dst = src: four independent 16-byte loads per thread per step (all issued
// before the stores), grid-stride, so the copy is bandwidth- rather than
// latency-bound
__global__ void __launch_bounds__(512) k_copy_probe(const double2* __restrict__ src, double2* __restrict__ dst, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {
        double2 a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) a[u] = __ldcg(src + i + u * stride);
#pragma unroll
        for (int u = 0; u < 4; ++u) dst[i + u * stride] = a[u];
    }
    for (; i < n; i += stride) dst[i] = __ldcg(src + i);
}

}  // namespace

cbs3d_status copy_bandwidth_probe(int device, long long bytes, int reps, double* gbs)
{
    if (bytes < 4096 || reps < 1 || !gbs) return CBS3D_INVALID_INPUT;
    if (cudaSetDevice(device) != cudaSuccess) return CBS3D_CUDA_ERROR;
    const long long n = bytes / 16;
    double2 *a = nullptr, *b = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cbs3d_status rc = CBS3D_OK;
    int sms = 0;
    float ms = 0.0f;
    if (cudaMalloc(&a, n * 16) != cudaSuccess || cudaMalloc(&b, n * 16) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaMemsetAsync(a, 0, n * 16, st) != cudaSuccess) {
        rc = CBS3D_CUDA_ERROR;
    } else {
        const unsigned grid = static_cast<unsigned>(sms) * 4;
        for (int w = 0; w < 3; ++w) k_copy_probe<<<grid, 512, 0, st>>>(a, b, n);   // warm-up (and warm L2)
        cudaEventRecord(e0, st);
        for (int r = 0; r < reps; ++r) k_copy_probe<<<grid, 512, 0, st>>>(a, b, n);
        cudaEventRecord(e1, st);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.0f)
            rc = CBS3D_CUDA_ERROR;
        else
            *gbs = 2.0 * 16.0 * static_cast<double>(n) * reps / (ms * 1.0e-3) / 1.0e9;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    return rc;
}

}  // namespace cbs3d

extern "C" cbs3d_status cbs3d_probe_copy_bandwidth(int device, long long bytes, int reps, double* gbs)
{
    return cbs3d::copy_bandwidth_probe(device, bytes, reps, gbs);
}

extern "C" cbs3d_status cbs3d_probe_allreduce(int device, int iters, double* us_per_allreduce)
{
    try {
        return cbs3d::allreduce_probe(device, iters, us_per_allreduce);
    } catch (const cbs3d::Error& e) {
        return e.code;
    } catch (...) {
        return CBS3D_INTERNAL;
    }
}
