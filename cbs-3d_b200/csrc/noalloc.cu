// Convergence norms for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc: code that runs
// under a memory manager owning every device allocation (a framework's
// caching allocator, a pool handed out by an embedding application), or a
// process that has budgeted its device memory up front and may not grow it
// mid-run.  cbs3d_convergence_norms_static serves them: it evaluates the
// Convergence::evaluate measures from device arrays the caller already
// holds, and its only scratch -- the per-block partial sums of the two-pass
// reduction -- lives in the file-scope array below, which every GPU that
// loads this library keeps until the process exits.
//
// Limits and sharing: the array holds NA_MAX_BLOCKS block partials, so npoin
// may not exceed NA_MAX_BLOCKS * NA_THREADS = 2,097,152 nodes (1 MiB of
// scratch per device).  All calls on a device share the array; each call
// writes every partial it later reads, so a call needs nothing zeroed, but two
// calls whose kernels overlap on the GPU race on it.
//
// Ordering: the kernels run on the legacy default stream and the call
// returns after a blocking copy of the result, so it holds the host until
// then and is ordered after blocking streams only.  The caller must finish
// (or synchronise) every stream that writes the inputs -- in particular any
// cudaStreamNonBlocking stream, such as this library's own context streams --
// before the call.
#include "cbs3d_gpu.h"

#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_MAX_BLOCKS = 8192;
constexpr int NA_MAX_DEVICES = 64;

// partials [block][16] (15 measures + the block's count of orphan nodes)
// followed by the 15 finished measures and the total orphan count
static __device__ __align__(256) double g_norm_scratch[NA_MAX_BLOCKS * 16 + 16];

// Host-side copy of each device's address of g_norm_scratch, looked up once
// per device.  In host code the symbol name is only a host stand-in, never a
// device address.  A cudaDeviceReset reloads the module and may move the
// array, so calls after a reset of that device are not supported.
double* g_scratch_addr[NA_MAX_DEVICES] = {};
std::mutex g_scratch_mutex;

// Same per-node sums and fixed block-reduction order as the engine's
// Convergence::evaluate kernels (src/solver/Convergence.cpp:276-349).  A node
// that touches no element (flags & 3 == 0) is counted instead: the reference
// rejects such a mesh (Convergence.cpp:157-161), and so does the host.
__global__ void k_norms_partial(const double* unkno, const double* unkn1, const double* pres,
                                const double* pres1, const double* temp, const double* temp1,
                                const double* elcoe2, const double* elcoe2p, const unsigned char* flags,
                                int npoin, int temp_calc, double* scratch)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = 0.0;
    if (i < npoin) {
        const unsigned char f = flags[i];
        const bool tf = f & 1, ts = f & 2;
        if (!tf && !ts) v[15] = 1.0;
        if (tf && !ts) {
            const double m = elcoe2[i];
            const double w = (fabs(m) <= 1.0e-300 || !isfinite(m)) ? 1.0 : 1.0 / m;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double nw = unkno[3 * i + d];
                const double dl = nw - unkn1[3 * i + d];
                v[3 * d] = dl * dl;
                v[3 * d + 1] = nw * nw;
                const double rs = dl * w;
                v[3 * d + 2] = rs * rs;
            }
        }
        if (tf) {
            const double dl = pres[i] - pres1[i];
            v[9] = dl * dl;
            v[10] = pres[i] * pres[i];
            v[11] = dl * dl;
        }
        if (temp_calc > 0 && (tf || ts)) {
            const double dl = temp[i] - temp1[i];
            v[12] = dl * dl;
            v[13] = temp[i] * temp[i];
            const double m = elcoe2p[i];
            const double w = (fabs(m) <= 1.0e-300 || !isfinite(m)) ? 1.0 : 1.0 / m;
            const double rs = dl * w;
            v[14] = rs * rs;
        }
    }
    __shared__ double sm[16][NA_THREADS / 32];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) sm[q][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 16) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sm[threadIdx.x][w];
        scratch[(size_t)blockIdx.x * 16 + threadIdx.x] = s;
    }
}

__global__ void k_norms_finish(double* scratch, int nblocks, int temp_calc)
{
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ double hb[16];
    if (q < 16) {
        double s = 0.0;
        for (int b = lane; b < nblocks; b += 32) s += scratch[(size_t)b * 16 + q];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) hb[q] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double h[15];
        for (int k = 0; k < 15; ++k) h[k] = hb[k];
        for (int b = 0; b < 9; b += 3) {
            h[b] = sqrt(h[b] / (h[b + 1] + 1.0e-30));
            h[b + 1] = sqrt(h[b + 1]);
            h[b + 2] = sqrt(h[b + 2]);
        }
        h[9] = sqrt(h[9] / (h[10] + 1.0e-30));
        h[10] = sqrt(h[10]);
        h[11] = sqrt(h[11]);
        if (temp_calc > 0) {
            h[12] = sqrt(h[12] / (h[13] + 1.0e-30));
            h[13] = sqrt(h[13]);
            h[14] = sqrt(h[14]);
        } else {
            h[12] = h[13] = h[14] = 0.0;
        }
        for (int k = 0; k < 15; ++k) scratch[(size_t)NA_MAX_BLOCKS * 16 + k] = h[k];
        scratch[(size_t)NA_MAX_BLOCKS * 16 + 15] = hb[15];
    }
}

// Device address of g_norm_scratch on `device` (which must be current);
// looked up once per device.
cudaError_t scratch_address(int device, double** out)
{
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[device]) {
        double* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_norm_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = p;
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" cbs3d_status cbs3d_convergence_norms_static(int device, const double* unkno, const double* unkn1,
                                                       const double* pres, const double* pres1,
                                                       const double* temperature, const double* temperature1,
                                                       const double* elcoe2, const double* elcoe2p,
                                                       const unsigned char* node_flags, int npoin, int temp_calc,
                                                       double hb[15])
{
    if (device < 0 || device >= NA_MAX_DEVICES || npoin < 1 || !hb || !unkno || !unkn1 || !pres || !pres1 ||
        !elcoe2 || !node_flags || (temp_calc > 0 && (!temperature || !temperature1 || !elcoe2p)))
        return CBS3D_INVALID_INPUT;
    const int nblocks = (npoin + NA_THREADS - 1) / NA_THREADS;
    if (nblocks > NA_MAX_BLOCKS) return CBS3D_INVALID_INPUT;   // npoin > 2,097,152
    // the caller's current device is restored on every return path
    int caller_device = -1;
    if (cudaGetDevice(&caller_device) != cudaSuccess) return CBS3D_CUDA_ERROR;
    const auto done = [caller_device](cbs3d_status st) -> cbs3d_status {
        if (cudaSetDevice(caller_device) != cudaSuccess && st == CBS3D_OK) return CBS3D_CUDA_ERROR;
        return st;
    };
    if (cudaSetDevice(device) != cudaSuccess) return done(CBS3D_CUDA_ERROR);
    double* scratch = nullptr;
    if (scratch_address(device, &scratch) != cudaSuccess) return done(CBS3D_CUDA_ERROR);
    k_norms_partial<<<nblocks, NA_THREADS>>>(unkno, unkn1, pres, pres1, temperature, temperature1, elcoe2,
                                             elcoe2p, node_flags, npoin, temp_calc, scratch);
    k_norms_finish<<<1, 16 * 32>>>(scratch, nblocks, temp_calc);
    if (cudaGetLastError() != cudaSuccess) return done(CBS3D_CUDA_ERROR);
    double out[16];
    if (cudaMemcpy(out, scratch + (size_t)NA_MAX_BLOCKS * 16, sizeof(out), cudaMemcpyDeviceToHost) != cudaSuccess)
        return done(CBS3D_CUDA_ERROR);
    if (out[15] != 0.0) return done(CBS3D_INVALID_INPUT);   // a node touches no element
    for (int k = 0; k < 15; ++k) hb[k] = out[k];
    return done(CBS3D_OK);
}
