// Measurement probes used to state the rooflines of the solver kernels: the
// bandwidth of reading (or copying) a device buffer that fits in L2 (or not),
// `passes` passes inside ONE launch so that the launch's fixed cost (about
// 4 us on B200, as much as a whole pass over 24 MiB from L2) does not count,
// timed with CUDA events on the probe's own stream.
#include "cbs3d_gpu.h"
#include "pcg.cuh"

#include <cuda_runtime.h>

namespace cbs3d {
namespace {

// Read: every thread sums its grid-stride share of the buffer, four
// independent 16-byte loads in flight per step, `passes` times; the sum is
// stored only in a case that never happens, which keeps the loads.
__global__ void __launch_bounds__(512) k_read_probe(const double2* src, long long n, int passes, double* sink)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (int p = 0; p < passes; ++p) {
        long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        for (; i + 3 * stride < n; i += 4 * stride) {
            double2 a[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) a[u] = __ldcg(src + i + u * stride);
#pragma unroll
            for (int u = 0; u < 4; ++u) acc += a[u].x + a[u].y;
        }
        for (; i < n; i += stride) acc += __ldcg(src + i).x;
    }
    if (acc == 1.0e300) sink[0] = acc;
}

// Copy: dst = src, `passes` times (the buffers may alias as far as the
// compiler knows, so no pass is folded into another).
__global__ void __launch_bounds__(512) k_copy_probe(const double2* src, double2* dst, long long n, int passes)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int p = 0; p < passes; ++p) {
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
}

}  // namespace

cbs3d_status bandwidth_probe(int device, long long bytes, int passes, int mode, double* gbs)
{
    if (bytes < 4096 || passes < 1 || (mode != 0 && mode != 1) || !gbs) return CBS3D_INVALID_INPUT;
    if (cudaSetDevice(device) != cudaSuccess) return CBS3D_CUDA_ERROR;
    const long long n = bytes / 16;
    double2 *a = nullptr, *b = nullptr;
    double* sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cbs3d_status rc = CBS3D_OK;
    int sms = 0;
    float ms = 0.0f;
    if (cudaMalloc(&a, n * 16) != cudaSuccess || (mode == 1 && cudaMalloc(&b, n * 16) != cudaSuccess) ||
        cudaMalloc(&sink, sizeof(double)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaMemsetAsync(a, 0, n * 16, st) != cudaSuccess) {
        rc = CBS3D_CUDA_ERROR;
    } else {
        const unsigned grid = static_cast<unsigned>(sms) * 4;
        auto run = [&](int np) {
            if (mode == 0) k_read_probe<<<grid, 512, 0, st>>>(a, n, np, sink);
            else k_copy_probe<<<grid, 512, 0, st>>>(a, b, n, np);
        };
        run(1);   // warm-up (and warm L2)
        cudaEventRecord(e0, st);
        run(passes);
        cudaEventRecord(e1, st);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.0f)
            rc = CBS3D_CUDA_ERROR;
        else
            *gbs = (mode == 1 ? 2.0 : 1.0) * 16.0 * static_cast<double>(n) * passes / (ms * 1.0e-3) / 1.0e9;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    if (sink) cudaFree(sink);
    return rc;
}

}  // namespace cbs3d

extern "C" cbs3d_status cbs3d_probe_bandwidth(int device, long long bytes, int passes, int mode, double* gbs)
{
    return cbs3d::bandwidth_probe(device, bytes, passes, mode, gbs);
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
