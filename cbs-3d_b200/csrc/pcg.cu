// Pressure PCG on sm_100a.
//
// Operator.  The reference applies the pressure operator element by element,
// colour by colour (src/linalg/MatrixVectorCalc.cpp:125-205).  Here the six
// per-element coefficients gstif = gstifE*dt_e are summed once per step into
// one coefficient per node pair (contributions added in ascending element
// order), stored as SELL-32: slices of 32 consecutive rows, each slice padded
// to its longest row and laid out column-major so a warp reads 32 rows'
// k-th entries in one coalesced 256-byte (FP64) load.  For the Kuhn meshes
// this halves the bytes per matvec against the element-by-element form
// (14 pair entries of 12 B per node instead of ~5.7 tets of 64 B).
//
// Solver.  One persistent cooperative kernel runs the whole Jacobi-PCG of
// ConjugateGradient::solvePressure (src/linalg/ConjugateGradient.cpp:584-869):
// the same masks, constraints, checks, convergence tests and iteration
// count semantics, with two grid-wide barriers per iteration.  The search
// direction update p = z + beta*p of the next iteration is folded into the
// matvec (double-buffered p; neighbours' new p formed on the fly from z and
// the previous p), and every CTA reduces the per-CTA partials in the same
// fixed order, so alpha, beta and the stopping decision are identical in all
// CTAs and reproducible run to run.
#include "pcg.cuh"

#include <cstdio>
#include <cstring>

namespace cbs3d {

namespace {

constexpr int PCG_THREADS = 256;
constexpr int PCG_WARPS = PCG_THREADS / 32;

#define CUDA_OK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) throw Error(CBS3D_CUDA_ERROR, std::string(#x) + ": " + cudaGetErrorString(e_)); } while (0)

template <typename T>
T* dalloc(size_t n)
{
    T* p = nullptr;
    if (n == 0) n = 1;
    CUDA_OK(cudaMalloc(&p, n * sizeof(T)));
    return p;
}

// ------------------------------------------------------- ELL assembly
__global__ void k_ell_from_state(DevState S, const long long* cptr, const int* cent, double* val,
                                 float* val32, long long nslots)
{
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int E = S.P.E;
    double v = 0.0;
    for (long long c = cptr[s]; c < cptr[s + 1]; ++c) {
        const int ent = cent[c];
        const int e = ent >> 3, g = ent & 7;
        v += S.gstifE[(size_t)g * E + e] * S.delte[e];
    }
    val[s] = v;
    if (val32) val32[s] = (float)v;
}

__global__ void k_ell_from_gstif(const double* gstif, const long long* cptr, const int* cent,
                                 double* val, float* val32, long long nslots)
{
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    double v = 0.0;
    for (long long c = cptr[s]; c < cptr[s + 1]; ++c) {
        const int ent = cent[c];
        v += gstif[(size_t)(ent >> 3) * 6 + (ent & 7)];
    }
    val[s] = v;
    if (val32) val32[s] = (float)v;
}

// impose_pressure_constraints (src/linalg/ConjugateGradient.cpp:188-214)
__global__ void k_impose(PcgDev D)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.N) return;
    const uint8_t f = D.nflag[i];
    if (!(f & 1)) {
        D.pres[i] = 0.0; D.rhs1[i] = 0.0; D.pdiag[i] = 0.0;
    } else if (f & 4) {
        D.pres[i] = D.pfix[i]; D.rhs1[i] = D.pfix[i]; D.pdiag[i] = 1.0;
    }
}

// y = A x on the assembled operator; identity rows on fixed nodes
__global__ void k_ell_multiply(PcgDev D, const double* x, double* y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.N) return;
    const int s = i >> 5, lane = i & 31;
    const long long base = D.slice_off[s] + lane;
    const int w = D.slice_w[s];
    double off = 0.0;
    for (int k = 0; k < w; ++k) off = fma(D.val[base + 32LL * k], x[D.col[base + 32LL * k]], off);
    double v = fma(D.pdiag[i], x[i], off);
    if (D.nflag[i] & 4) v = x[i];
    y[i] = v;
}

// ------------------------------------------------- deterministic reductions
struct Acc4 {
    double a, b, mx, flag;
};

// Block partial of (sum a, sum b, max mx, max flag), written by thread 0 in
// a fixed warp order.
__device__ __forceinline__ void block_partial(Acc4 v, double* out)
{
    __shared__ double sm[PCG_WARPS][4];
    for (int o = 16; o > 0; o >>= 1) {
        v.a += __shfl_down_sync(0xffffffffu, v.a, o);
        v.b += __shfl_down_sync(0xffffffffu, v.b, o);
        v.mx = fmax(v.mx, __shfl_down_sync(0xffffffffu, v.mx, o));
        v.flag = fmax(v.flag, __shfl_down_sync(0xffffffffu, v.flag, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sm[w][0] = v.a; sm[w][1] = v.b; sm[w][2] = v.mx; sm[w][3] = v.flag; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, mx = 0.0, fl = 0.0;
        for (int k = 0; k < PCG_WARPS; ++k) { a += sm[k][0]; b += sm[k][1]; mx = fmax(mx, sm[k][2]); fl = fmax(fl, sm[k][3]); }
        out[0] = a; out[1] = b; out[2] = mx; out[3] = fl;
        __threadfence();
    }
}

// Grid total of the block partials, summed in the same fixed tree by every
// CTA (lane l takes partials l, l+32, ... then a shuffle tree), so every CTA
// obtains bit-identical totals.
__device__ __forceinline__ Acc4 grid_total(const double* part, int G)
{
    __shared__ double tot[4];
    if (threadIdx.x < 32) {
        double a = 0.0, b = 0.0, mx = 0.0, fl = 0.0;
        for (int k = threadIdx.x; k < G; k += 32) {
            const double* p = part + (size_t)k * 8;
            a += __ldcg(p); b += __ldcg(p + 1); mx = fmax(mx, __ldcg(p + 2)); fl = fmax(fl, __ldcg(p + 3));
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
            mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
            fl = fmax(fl, __shfl_down_sync(0xffffffffu, fl, o));
        }
        if (threadIdx.x == 0) { tot[0] = a; tot[1] = b; tot[2] = mx; tot[3] = fl; }
    }
    __syncthreads();
    Acc4 r{tot[0], tot[1], tot[2], tot[3]};
    __syncthreads();
    return r;
}

__device__ __forceinline__ bool cg_converged(int test, double rel, double mx, double rtol, double atol)
{
    if (test == 1) return mx <= atol;
    if (test == 2) return rel <= rtol;
    return mx <= atol || rel <= rtol;
}

__device__ __forceinline__ void cg_finish(const PcgDev& D, int it, int conv, double init, double fin,
                                          double rel, double mx)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        D.out->iterations = it;
        D.out->converged = conv;
        D.out->initial_l2 = init;
        D.out->final_l2 = fin;
        D.out->rel = rel;
        D.out->max_abs = mx;
    }
}

// ---------------------------------------------------- persistent FP64 PCG
__global__ void __launch_bounds__(PCG_THREADS) k_pcg64(PcgDev D)
{
    const int G = gridDim.x, b = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s_beg = (int)((long long)b * D.nslices / G);
    const int s_end = (int)((long long)(b + 1) * D.nslices / G);
    unsigned* cnt = D.bar;
    unsigned* gen = D.bar + 1;
    int phase = 0;
    const int N = D.N;

    // ---- r0 = b - A p0, z0, d0 = z0, (r,r), (r,z), max|r|
    Acc4 acc{0.0, 0.0, 0.0, 0.0};
    for (int s = s_beg + warp; s < s_end; s += PCG_WARPS) {
        const int i = s * 32 + lane;
        if (i >= N) continue;
        const long long base = D.slice_off[s] + lane;
        const int w = D.slice_w[s];
        double off = 0.0;
        for (int k = 0; k < w; ++k) off = fma(D.val[base + 32LL * k], D.pres[D.col[base + 32LL * k]], off);
        const uint8_t f = D.nflag[i];
        const bool active = f & 1, freen = (f & 1) && !(f & 4);
        const double y = fma(D.pdiag[i], D.pres[i], off);
        double ri = active ? D.rhs1[i] - y : 0.0;
        if (!freen) ri = 0.0;
        double zi = 0.0;
        if (freen) {
            if (D.precond) {
                const double dg = D.pdiag[i];
                if (!(isfinite(dg) && dg > 1.0e-30)) acc.flag = fmax(acc.flag, 1.0);
                else zi = ri / dg;
            } else {
                zi = ri;
            }
            if (!isfinite(ri)) acc.flag = fmax(acc.flag, 2.0);
            acc.a = fma(ri, ri, acc.a);
            acc.b = fma(ri, zi, acc.b);
            acc.mx = fmax(acc.mx, fabs(ri));
        }
        D.r[i] = ri;
        D.z[i] = zi;
        D.pA[i] = zi;
    }
    block_partial(acc, D.part + ((size_t)(phase & 1) * G + b) * 8);
    if (!grid_barrier(cnt, gen, G, D.status, ST_PCG)) return;
    Acc4 t = grid_total(D.part + (size_t)(phase & 1) * G * 8, G);
    ++phase;
    const double init = sqrt(t.a);
    if (init <= 1.0e-300) { cg_finish(D, 0, 1, init, init, 0.0, t.mx); return; }
    if (cg_converged(D.conv_test, 1.0, t.mx, D.rel_tol, D.abs_tol)) { cg_finish(D, 0, 1, init, init, 1.0, t.mx); return; }
    if (t.flag >= 2.0) { if (b == 0 && threadIdx.x == 0) set_status(D.status, 4, ST_PCG, 0, R_PCG_RESID); return; }
    if (t.flag >= 1.0) { if (b == 0 && threadIdx.x == 0) set_status(D.status, 1, ST_PCG, 0, R_PCG_DIAG); return; }
    double rz = t.b;
    if (rz <= 1.0e-300 || !isfinite(rz)) { if (b == 0 && threadIdx.x == 0) set_status(D.status, 3, ST_PCG, 0, R_PCG_RZ0); return; }

    double* pc = D.pA;   // current direction
    double* pp = D.pB;   // previous direction (unused at it=1)
    double beta = 0.0, fin = init, rel = 1.0, mx = t.mx;
    int it = 0, conv = 0;
    for (it = 1; it <= D.max_iter; ++it) {
        // ---- q = A p (p formed here from z and the previous p), (p, q)
        Acc4 pa{0.0, 0.0, 0.0, 0.0};
        const bool upd = it > 1;
        for (int s = s_beg + warp; s < s_end; s += PCG_WARPS) {
            const int i = s * 32 + lane;
            if (i >= N) continue;
            const long long base = D.slice_off[s] + lane;
            const int w = D.slice_w[s];
            const uint8_t f = D.nflag[i];
            const bool freen = (f & 1) && !(f & 4);
            double off = 0.0, pci;
            if (upd) {
                for (int k = 0; k < w; ++k) {
                    const int j = D.col[base + 32LL * k];
                    off = fma(D.val[base + 32LL * k], fma(beta, __ldcg(pp + j), __ldcg(D.z + j)), off);
                }
                pci = freen ? fma(beta, pp[i], D.z[i]) : 0.0;
                pc[i] = pci;
            } else {
                for (int k = 0; k < w; ++k) off = fma(D.val[base + 32LL * k], __ldcg(pc + D.col[base + 32LL * k]), off);
                pci = pc[i];
            }
            const double qi = freen ? fma(D.pdiag[i], pci, off) : 0.0;
            D.q[i] = qi;
            if (freen) pa.a = fma(pci, qi, pa.a);
        }
        block_partial(pa, D.part + ((size_t)(phase & 1) * G + b) * 8);
        if (!grid_barrier(cnt, gen, G, D.status, ST_PCG)) return;
        t = grid_total(D.part + (size_t)(phase & 1) * G * 8, G);
        ++phase;
        const double pAp = t.a;
        if (fabs(pAp) <= 1.0e-300 || !isfinite(pAp)) { if (b == 0 && threadIdx.x == 0) set_status(D.status, 3, ST_PCG, it, R_PCG_PAP); return; }
        const double alpha = rz / pAp;

        // ---- p += alpha d, r -= alpha q, z = M^-1 r, (r,r), (r,z), max|r|
        Acc4 rr{0.0, 0.0, 0.0, 0.0};
        for (int s = s_beg + warp; s < s_end; s += PCG_WARPS) {
            const int i = s * 32 + lane;
            if (i >= N) continue;
            const uint8_t f = D.nflag[i];
            if (!((f & 1) && !(f & 4))) continue;
            D.pres[i] = fma(alpha, pc[i], D.pres[i]);
            const double ri = fma(-alpha, D.q[i], D.r[i]);
            D.r[i] = ri;
            const double zi = D.precond ? ri / D.pdiag[i] : ri;
            D.z[i] = zi;
            if (!isfinite(ri)) rr.flag = 1.0;
            rr.a = fma(ri, ri, rr.a);
            rr.b = fma(ri, zi, rr.b);
            rr.mx = fmax(rr.mx, fabs(ri));
        }
        block_partial(rr, D.part + ((size_t)(phase & 1) * G + b) * 8);
        if (!grid_barrier(cnt, gen, G, D.status, ST_PCG)) return;
        t = grid_total(D.part + (size_t)(phase & 1) * G * 8, G);
        ++phase;
        fin = sqrt(t.a);
        mx = t.mx;
        rel = fin / init;
        if (cg_converged(D.conv_test, rel, mx, D.rel_tol, D.abs_tol)) { conv = 1; break; }
        if (t.flag > 0.0) { if (b == 0 && threadIdx.x == 0) set_status(D.status, 4, ST_PCG, it, R_PCG_RESID); return; }
        const double rzn = t.b;
        if (rzn <= 1.0e-300 || !isfinite(rzn)) { if (b == 0 && threadIdx.x == 0) set_status(D.status, 3, ST_PCG, it, R_PCG_RZ); return; }
        beta = rzn / rz;
        rz = rzn;
        double* tmp = pp; pp = pc; pc = tmp;
    }
    if (it > D.max_iter) it = D.max_iter;
    cg_finish(D, it, conv, init, fin, rel, mx);
    if (!conv && b == 0 && threadIdx.x == 0) set_status(D.status, 2, ST_PCG, it, R_PCG_MAXIT);
}

// Self-test of the bounded device wait: CTA 0 leaves without arriving, so the
// other CTAs' barrier waits can only end by running out of their spin limit.
__global__ void k_barrier_selftest(unsigned* bar, DevStatus* st)
{
    if (blockIdx.x == 0) return;
    grid_barrier(bar, bar + 1, gridDim.x, st, ST_PCG);
}

}  // namespace

cbs3d_status selftest_wait_timeout(int device, int* observed)
{
    CUDA_OK(cudaSetDevice(device));
    unsigned* bar = dalloc<unsigned>(2);
    DevStatus* st = dalloc<DevStatus>(1);
    CUDA_OK(cudaMemset(bar, 0, 2 * sizeof(unsigned)));
    CUDA_OK(cudaMemset(st, 0, sizeof(DevStatus)));
    k_barrier_selftest<<<4, 32>>>(bar, st);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaDeviceSynchronize());
    DevStatus h{};
    CUDA_OK(cudaMemcpy(&h, st, sizeof h, cudaMemcpyDeviceToHost));
    cudaFree(bar);
    cudaFree(st);
    if (observed) *observed = h.code;
    return CBS3D_OK;
}

// ============================================================ PcgEngine
void PcgEngine::init(const HostModel& m, const uint8_t* nflag, const double* pfix, DevStatus* status,
                     int device, int blocks_override, bool mixed_mode)
{
    N = m.N;
    E = m.E;
    mixed = mixed_mode;
    const PressurePattern& P = m.pat;
    nslices = P.nslices;
    nslots = P.nslots;
    ncontrib = static_cast<long long>(P.cent.size());
    nnz_offdiag = 0;
    for (size_t q = 0; q + 1 < P.cptr.size(); ++q) nnz_offdiag += (P.cptr[q + 1] > P.cptr[q]) ? 1 : 0;
    d_slice_off = dalloc<long long>(P.slice_off.size());
    d_slice_w = dalloc<int>(P.slice_w.size());
    d_col = dalloc<int>(static_cast<size_t>(nslots));
    d_cptr = dalloc<long long>(P.cptr.size());
    d_cent = dalloc<int>(static_cast<size_t>(ncontrib));
    d_val = dalloc<double>(static_cast<size_t>(nslots));
    CUDA_OK(cudaMemcpy(d_slice_off, P.slice_off.data(), P.slice_off.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_slice_w, P.slice_w.data(), P.slice_w.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (nslots) CUDA_OK(cudaMemcpy(d_col, P.col.data(), static_cast<size_t>(nslots) * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_cptr, P.cptr.data(), P.cptr.size() * sizeof(long long), cudaMemcpyHostToDevice));
    if (ncontrib) CUDA_OK(cudaMemcpy(d_cent, P.cent.data(), static_cast<size_t>(ncontrib) * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemset(d_val, 0, static_cast<size_t>(nslots ? nslots : 1) * sizeof(double)));
    const size_t n = static_cast<size_t>(N);
    d_r = dalloc<double>(n); d_z = dalloc<double>(n); d_pA = dalloc<double>(n);
    d_pB = dalloc<double>(n); d_q = dalloc<double>(n);
    CUDA_OK(cudaMemset(d_pB, 0, n * sizeof(double)));
    if (mixed) {
        d_val32 = dalloc<float>(static_cast<size_t>(nslots));
        d_f32 = dalloc<float>(7 * n);
        CUDA_OK(cudaMemset(d_f32, 0, 7 * n * sizeof(float)));
    }
    d_nflag = nflag;
    d_pfix = pfix;
    d_status = status;

    int sms = 0, per_sm = 0;
    CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg64, PCG_THREADS, 0));
    int g = sms * (per_sm < 2 ? per_sm : 2);
    if (blocks_override > 0 && blocks_override < g) g = blocks_override;
    // never more CTAs than slices
    if (g > nslices) g = nslices > 0 ? nslices : 1;
    nblocks = g;
    d_part = dalloc<double>(static_cast<size_t>(2 * nblocks * 8));
    d_bar = dalloc<unsigned>(4);
    d_out = dalloc<CgOut>(1);
    CUDA_OK(cudaMemset(d_bar, 0, 4 * sizeof(unsigned)));

    dev = PcgDev{};
    dev.N = N; dev.E = E; dev.nslices = nslices; dev.nblocks = nblocks;
    dev.slice_off = d_slice_off; dev.slice_w = d_slice_w; dev.col = d_col; dev.val = d_val;
    dev.val32 = d_val32; dev.cptr = d_cptr; dev.cent = d_cent;
    dev.nflag = d_nflag; dev.pfix = d_pfix;
    dev.r = d_r; dev.z = d_z; dev.pA = d_pA; dev.pB = d_pB; dev.q = d_q;
    if (mixed) {
        dev.r32 = d_f32; dev.z32 = d_f32 + n; dev.pA32 = d_f32 + 2 * n; dev.pB32 = d_f32 + 3 * n;
        dev.q32 = d_f32 + 4 * n; dev.x32 = d_f32 + 5 * n; dev.dinv32 = d_f32 + 6 * n;
    }
    dev.part = d_part; dev.bar = d_bar; dev.status = d_status; dev.out = d_out;
}

void PcgEngine::release()
{
    void* ptrs[] = {d_slice_off, d_slice_w, d_col, d_cptr, d_cent, d_val, d_val32, d_r, d_z, d_pA,
                    d_pB, d_q, d_f32, d_part, d_bar, d_out};
    for (void* p : ptrs) if (p) cudaFree(p);
    d_slice_off = nullptr; d_slice_w = nullptr; d_col = nullptr; d_cptr = nullptr; d_cent = nullptr;
    d_val = nullptr; d_val32 = nullptr; d_r = d_z = d_pA = d_pB = d_q = nullptr; d_f32 = nullptr;
    d_part = nullptr; d_bar = nullptr; d_out = nullptr;
}

void PcgEngine::assemble_from_state(const DevState& S, cudaStream_t st)
{
    if (!nslots) return;
    const int T = 256;
    k_ell_from_state<<<static_cast<unsigned>((nslots + T - 1) / T), T, 0, st>>>(S, d_cptr, d_cent, d_val, d_val32, nslots);
}

void PcgEngine::assemble_from_gstif(const double* gstif, cudaStream_t st)
{
    if (!nslots) return;
    const int T = 256;
    k_ell_from_gstif<<<static_cast<unsigned>((nslots + T - 1) / T), T, 0, st>>>(gstif, d_cptr, d_cent, d_val, d_val32, nslots);
}

void PcgEngine::multiply(const double* pdiag, const double* x, double* y, cudaStream_t st)
{
    PcgDev D = dev;
    D.pdiag = const_cast<double*>(pdiag);
    k_ell_multiply<<<(N + 255) / 256, 256, 0, st>>>(D, x, y);
}

cbs3d_status PcgEngine::solve(double* pres, double* rhs1, double* pdiag, int precond, int conv_test,
                              int max_iter, double rel_tol, double abs_tol, cudaStream_t st, bool sync,
                              cudaEvent_t ev0, cudaEvent_t ev1)
{
    PcgDev D = dev;
    D.pres = pres; D.rhs1 = rhs1; D.pdiag = pdiag;
    D.precond = precond; D.conv_test = conv_test; D.max_iter = max_iter;
    D.rel_tol = rel_tol; D.abs_tol = abs_tol; D.inner_tol = inner_tol;
    k_impose<<<(N + 255) / 256, 256, 0, st>>>(D);
    CUDA_OK(cudaMemsetAsync(d_bar, 0, 2 * sizeof(unsigned), st));
    void* args[] = {&D};
    if (ev0) CUDA_OK(cudaEventRecord(ev0, st));
    CUDA_OK(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_pcg64), dim3(nblocks), dim3(PCG_THREADS), args, 0, st));
    if (ev1) CUDA_OK(cudaEventRecord(ev1, st));
    if (sync) CUDA_OK(cudaStreamSynchronize(st));
    return CBS3D_OK;
}

cbs3d_status PcgEngine::read_result(cbs3d_cg_result& r, cudaStream_t st)
{
    CgOut o{};
    CUDA_OK(cudaMemcpyAsync(&o, d_out, sizeof o, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    std::memset(&r, 0, sizeof r);
    r.iterations = o.iterations;
    r.initial_l2 = o.initial_l2;
    r.final_l2 = o.final_l2;
    r.final_relative_l2 = o.rel;
    r.final_max_abs = o.max_abs;
    r.converged = o.converged;
    r.matvec_calls = o.iterations + 1;
    r.outer_sweeps = o.outer;
    return o.converged ? CBS3D_OK : CBS3D_NOT_CONVERGED;
}

size_t PcgEngine::bytes_per_iter() const
{
    // Phase A: coefficient + column per pair entry; z and previous p of the
    // row (16 B), pdiag (8), new p written (8), q written (8), node flag (1).
    // Phase B: q, r, pres, pdiag read (32), r, pres, z written (24).
    return static_cast<size_t>(nnz_offdiag) * 12 + static_cast<size_t>(N) * 97;
}

}  // namespace cbs3d
