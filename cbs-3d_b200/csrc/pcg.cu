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
#include "mg.cuh"

#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>
#include <cstring>
#include <vector>

namespace cbs3d {

namespace {

// One 512-thread CTA per SM (128 registers per thread fill the register
// file): half the CTAs of two 256-thread CTAs per SM, so the grid-wide
// all-reduce reads half the partials.
constexpr int PCG_THREADS = 512;
constexpr int PCG_CTAS_PER_SM = 1;
constexpr int PCG_WARPS = PCG_THREADS / 32;

#define CUDA_OK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) throw Error(CBS3D_CUDA_ERROR, std::string(#x) + ": " + cudaGetErrorString(e_)); } while (0)

// The dynamic shared-memory limit is one attribute per kernel and device,
// shared by every engine and batch in the process: it only ever grows, so a
// smaller later request cannot invalidate an earlier engine's launches.
cudaError_t raise_smem_limit(const void* fn, size_t smem)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = limit[{dev, fn}];
    if (smem <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e == cudaSuccess) cur = smem;
    return e;
}

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
    if (i >= D.NN) return;
    const uint8_t f = D.nflag[i];
    if (!(f & 1)) {
        D.pres[i] = 0.0; D.rhs1[i] = 0.0; D.pdiag[i] = 0.0;
    } else if (f & 4) {
        D.pres[i] = D.pfix[i]; D.rhs1[i] = D.pfix[i]; D.pdiag[i] = 1.0;
    }
}

// Node order -> row-position order of the solver's inputs, and back for the
// pressure.  Padding positions get inactive flags and zeros.
__global__ void k_perm_in(PcgDev D, const double* pres, const double* rhs1, const double* pdiag,
                          const uint8_t* nflag, double* xp, double* bp, double* dp, uint8_t* fp)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= D.N) return;
    const int i = D.row_node[pos];
    xp[pos] = i >= 0 ? pres[i] : 0.0;
    bp[pos] = i >= 0 ? rhs1[i] : 0.0;
    dp[pos] = i >= 0 ? pdiag[i] : 0.0;
    fp[pos] = i >= 0 ? (uint8_t)(nflag[i] & 5) : (uint8_t)0;
}

__global__ void k_perm_out(PcgDev D, const double* xp, double* pres)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= D.N) return;
    const int i = D.row_node[pos];
    if (i >= 0) pres[i] = xp[pos];
}

// y = A x on the assembled operator; identity rows on fixed nodes
__global__ void k_ell_multiply(PcgDev D, const double* x, double* y)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= D.nslices * 32) return;
    const int i = D.row_node[pos];
    if (i < 0) return;
    const int s = pos >> 5, lane = pos & 31;
    const long long base = D.slice_off[s] + lane;
    const int w = D.slice_w[s];
    double off = 0.0;
    for (int k = 0; k < w; ++k) {
        const int j = D.row_node[D.col[base + 32LL * k]];
        off = fma(D.val[base + 32LL * k], j >= 0 ? x[j] : 0.0, off);
    }
    double v = fma(D.pdiag[i], x[i], off);
    if (D.nflag[i] & 4) v = x[i];
    y[i] = v;
}

// ------------------------------------------------------- solve segments
// One cooperative launch solves one system, or -- for the batched step --
// several independent systems at once: CTAs [cta0, cta0+ncta) of the grid
// then own instance k's slice range [s0, s1), and every reduction, barrier,
// status and result is per instance.  SegView is this CTA's view, with the
// solve's scalars.
struct SegView {
    int G, b;      // CTAs of this CTA's solve; this CTA's index among them
    int s0, s1;    // slice range of the solve
    int k;         // instance, -1 for a single solve
    int precond, conv_test, max_iter;
    double rel_tol, abs_tol;
};

template <bool BATCH>
__device__ __forceinline__ SegView seg_view(const PcgDev& D)
{
    if constexpr (!BATCH)
        return SegView{(int)gridDim.x, (int)blockIdx.x, 0, D.nslices, -1, D.precond, D.conv_test, D.max_iter,
                       D.rel_tol, D.abs_tol};
    else {
    const int k = D.cta_inst[blockIdx.x];
    const PcgInst& I = D.inst[k];
    return SegView{I.ncta, (int)blockIdx.x - I.cta0, I.s0, I.s1, k, I.precond, I.conv_test, I.max_iter,
                   I.rel_tol, I.abs_tol};
    }
}
__device__ __forceinline__ DevStatus* seg_status(const PcgDev& D, const SegView& g) { return g.k < 0 ? D.status : D.inst[g.k].status; }
__device__ __forceinline__ CgOut* seg_out(const PcgDev& D, const SegView& g) { return g.k < 0 ? D.out : D.inst[g.k].out; }
__device__ __forceinline__ unsigned* seg_bar(const PcgDev& D, const SegView& g) { return g.k < 0 ? D.bar : D.inst[g.k].bar; }
__device__ __forceinline__ double* seg_part(const PcgDev& D, const SegView& g) { return g.k < 0 ? D.part : D.inst[g.k].part; }

// ------------------------------------------------- deterministic reductions
struct Acc4 {
    double a, b, mx, flag;
};

// Grid-wide all-reduce of (sum a, sum b, max mx, max flag) fused with the
// grid barrier (grid_allreduce_v below).
template <int NV, int NSUM, int NT = PCG_THREADS>
__device__ __forceinline__ bool grid_allreduce_v(double (&v)[NV], const PcgDev& D, const SegView& g, int phase,
                                                 double (&out)[NV]);

__device__ __forceinline__ bool grid_allreduce(Acc4 v, const PcgDev& D, const SegView& g, int phase, Acc4& out)
{
    double a[4] = {v.a, v.b, v.mx, v.flag}, o[4];
    const bool ok = grid_allreduce_v<4, 2>(a, D, g, phase, o);
    out = Acc4{o[0], o[1], o[2], o[3]};
    return ok;
}

__device__ __forceinline__ bool cg_converged(int test, double rel, double mx, double rtol, double atol)
{
    if (test == 1) return mx <= atol;
    if (test == 2) return rel <= rtol;
    return mx <= atol || rel <= rtol;
}

__device__ __forceinline__ void cg_finish(const PcgDev& D, const SegView& g, int it, int conv, double init,
                                          double fin, double rel, double mx)
{
    if (g.b == 0 && threadIdx.x == 0) {
        CgOut* o = seg_out(D, g);
        o->iterations = it;
        o->converged = conv;
        o->initial_l2 = init;
        o->final_l2 = fin;
        o->rel = rel;
        o->max_abs = mx;
    }
}

// ---------------------------------------------------- persistent FP64 PCG
// HALO: the neighbour values of each iteration's product (z and the previous
// direction of every column of the CTA's rows) are staged in shared memory
// once per iteration, and the slots carry 16-bit indices into that halo
// (D.halo_ptr/halo_idx/lcol of this kernel's partition), so the rounds
// stream only coefficients and local columns and read neighbours from shared
// memory.  Same arithmetic in the same order as without.
template <bool HALO>
__global__ void __launch_bounds__(PCG_THREADS, PCG_CTAS_PER_SM) k_pcg64(PcgDev D)
{
    const SegView g = seg_view<false>(D);
    const int G = g.G, b = g.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s_beg = g.s0 + (int)((long long)b * (g.s1 - g.s0) / G);
    const int s_end = g.s0 + (int)((long long)(b + 1) * (g.s1 - g.s0) / G);
    int phase = 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // HALO: per halo entry (z, previous direction) -- on the first
    // iteration (0, current direction) -- one 16-byte read per neighbour
    double2* hzp = reinterpret_cast<double2*>(smem_raw);
    // HALO: the CTA's slices in KP parts (one unless a CTA's whole halo
    // would not fit), each staged and processed in turn
    const int KP = HALO ? (D.halo_parts > 0 ? D.halo_parts : 1) : 1;

    // ---- r0 = b - A p0, z0, d0 = z0, (r,r), (r,z), max|r|
    Acc4 acc{0.0, 0.0, 0.0, 0.0};
    for (int s = s_beg + warp; s < s_end; s += PCG_WARPS) {
        const int i = s * 32 + lane;
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
            if (g.precond) {
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
    Acc4 t = Acc4{0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce(acc, D, g, phase, t)) return;
    ++phase;
    const double init = sqrt(t.a);
    if (init <= 1.0e-300) { cg_finish(D, g, 0, 1, init, init, 0.0, t.mx); return; }
    if (cg_converged(g.conv_test, 1.0, t.mx, g.rel_tol, g.abs_tol)) { cg_finish(D, g, 0, 1, init, init, 1.0, t.mx); return; }
    if (t.flag >= 2.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, 0, R_PCG_RESID); return; }
    if (t.flag >= 1.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 1, ST_PCG, 0, R_PCG_DIAG); return; }
    double rz = t.b;
    if (rz <= 1.0e-300 || !isfinite(rz)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, 0, R_PCG_RZ0); return; }

    double* pc = D.pA;   // current direction
    double* pp = D.pB;   // previous direction (unused at it=1)
    double beta = 0.0, fin = init, rel = 1.0, mx = t.mx;
    int it = 0, conv = 0;
    for (it = 1; it <= g.max_iter; ++it) {
        // ---- q = A p (p formed here from z and the previous p), (p, q)
        Acc4 pa{0.0, 0.0, 0.0, 0.0};
        const bool upd = it > 1;
        for (int part = 0; part < KP; ++part) {
        const int ps0 = s_beg + (int)((long long)part * (s_end - s_beg) / KP);
        const int ps1 = s_beg + (int)((long long)(part + 1) * (s_end - s_beg) / KP);
        if constexpr (HALO) {
            // z and pp (or pc) were written before the last all-reduce
            __syncthreads();
            const int h0 = D.halo_ptr[b * KP + part], nh = D.halo_ptr[b * KP + part + 1] - h0;
            for (int k = threadIdx.x; k < nh; k += PCG_THREADS) {
                const int j = D.halo_idx[h0 + k];
                hzp[k] = make_double2(upd ? __ldcg(D.z + j) : 0.0, __ldcg((upd ? pp : pc) + j));
            }
            __syncthreads();
        }
        for (int s = ps0 + warp; s < ps1; s += PCG_WARPS) {
            const int i = s * 32 + lane;
            const long long base = D.slice_off[s] + lane;
            const int w = D.slice_w[s];
            const uint8_t f = D.nflag[i];
            const bool freen = (f & 1) && !(f & 4);
            double off = 0.0, pci;
            // Rounds of eight slots; the next round's columns and
            // coefficients (streamed from HBM on large meshes) are requested
            // before this round's neighbour gathers (mostly L2 hits), so the
            // two latencies overlap and each lane keeps more loads in flight.
            // The sum still runs over the slots in order.
            constexpr int CH = 8;
            // columns: global positions, or (HALO) indices into the staged halo
            auto colat = [&](long long t) -> int { return HALO ? (int)__ldcs(D.lcol + t) : D.col[t]; };
            const int cpad = HALO ? 0 : i;   // a valid column for the padding lanes of a round
            int cn[CH];
            double vn[CH];
#pragma unroll
            for (int u = 0; u < CH; ++u) {
                cn[u] = u < w ? colat(base + 32LL * u) : cpad;
                vn[u] = u < w ? __ldcs(D.val + base + 32LL * u) : 0.0;
            }
            for (int k0 = 0; k0 < w; k0 += CH) {
                int c[CH];
                double v[CH];
#pragma unroll
                for (int u = 0; u < CH; ++u) { c[u] = cn[u]; v[u] = vn[u]; }
#pragma unroll
                for (int u = 0; u < CH; ++u) {
                    const int k = k0 + CH + u;
                    cn[u] = k < w ? colat(base + 32LL * k) : cpad;
                    vn[u] = k < w ? __ldcs(D.val + base + 32LL * k) : 0.0;
                }
                double x[CH];
                if constexpr (HALO) {
                    if (upd) {
#pragma unroll
                        for (int u = 0; u < CH; ++u) {
                            const double2 zp = hzp[c[u]];
                            x[u] = fma(beta, zp.y, zp.x);
                        }
                    } else {
#pragma unroll
                        for (int u = 0; u < CH; ++u) x[u] = hzp[c[u]].y;
                    }
                } else if (upd) {
#pragma unroll
                    for (int u = 0; u < CH; ++u) x[u] = fma(beta, __ldcg(pp + c[u]), __ldcg(D.z + c[u]));
                } else {
#pragma unroll
                    for (int u = 0; u < CH; ++u) x[u] = __ldcg(pc + c[u]);
                }
#pragma unroll
                for (int u = 0; u < CH; ++u)
                    if (k0 + u < w) off = fma(v[u], x[u], off);
            }
            if (upd) {
                pci = freen ? fma(beta, pp[i], D.z[i]) : 0.0;
                pc[i] = pci;
            } else {
                pci = pc[i];
            }
            const double qi = freen ? fma(D.pdiag[i], pci, off) : 0.0;
            D.q[i] = qi;
            if (freen) pa.a = fma(pci, qi, pa.a);
        }
        }   // parts
        t = Acc4{0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce(pa, D, g, phase, t)) return;
        ++phase;
        const double pAp = t.a;
        if (fabs(pAp) <= 1.0e-300 || !isfinite(pAp)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_PAP); return; }
        const double alpha = rz / pAp;

        // ---- p += alpha d, r -= alpha q, z = M^-1 r, (r,r), (r,z), max|r|
        Acc4 rr{0.0, 0.0, 0.0, 0.0};
        for (int s = s_beg + warp; s < s_end; s += PCG_WARPS) {
            const int i = s * 32 + lane;
            const uint8_t f = D.nflag[i];
            if (!((f & 1) && !(f & 4))) continue;
            D.pres[i] = fma(alpha, pc[i], D.pres[i]);
            const double ri = fma(-alpha, D.q[i], D.r[i]);
            D.r[i] = ri;
            const double zi = g.precond ? ri / D.pdiag[i] : ri;
            D.z[i] = zi;
            if (!isfinite(ri)) rr.flag = 1.0;
            rr.a = fma(ri, ri, rr.a);
            rr.b = fma(ri, zi, rr.b);
            rr.mx = fmax(rr.mx, fabs(ri));
        }
        t = Acc4{0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce(rr, D, g, phase, t)) return;
        ++phase;
        fin = sqrt(t.a);
        mx = t.mx;
        rel = fin / init;
        if (cg_converged(g.conv_test, rel, mx, g.rel_tol, g.abs_tol)) { conv = 1; break; }
        if (t.flag > 0.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, it, R_PCG_RESID); return; }
        const double rzn = t.b;
        if (rzn <= 1.0e-300 || !isfinite(rzn)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_RZ); return; }
        beta = rzn / rz;
        rz = rzn;
        double* tmp = pp; pp = pc; pc = tmp;
    }
    if (it > g.max_iter) it = g.max_iter;
    cg_finish(D, g, it, conv, init, fin, rel, mx);
    if (!conv && b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 2, ST_PCG, it, R_PCG_MAXIT);
}

// ------------------------------------------- register-resident FP64 PCG
// Same algorithm as k_pcg64, for meshes where every thread owns at most RMAX
// rows (slices s_beg + warp + 8r, lane = row within the slice).  The row
// state -- residual, search direction, q, diagonal and flags -- stays in
// registers for the whole solve; each iteration writes the new direction
// (double-buffered, for the neighbours' on-the-fly update), z and the
// pressure to global memory.  Each row's pair entries are fetched eight at a time before
// the neighbour gathers are issued, so a lane keeps many loads in flight.
template <int RMAX>
__global__ void __launch_bounds__(PCG_THREADS, PCG_CTAS_PER_SM) k_pcg64r(PcgDev D)
{
    const SegView g = seg_view<false>(D);
    const int G = g.G, b = g.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s_beg = g.s0 + (int)((long long)b * (g.s1 - g.s0) / G);
    const int s_end = g.s0 + (int)((long long)(b + 1) * (g.s1 - g.s0) / G);
    int phase = 0;
    

    double r[RMAX], p[RMAX], q[RMAX], dg[RMAX];
    bool fr[RMAX];
    int row[RMAX];
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int s = s_beg + warp + PCG_WARPS * k;
        row[k] = (s < s_end) ? s * 32 + lane : -1;
        r[k] = p[k] = q[k] = dg[k] = 0.0;
        fr[k] = false;
    }

    // off[k] = sum_j A_ij v_j over row k's pair entries, v_j = beta*pp_j + zz_j
    // (v = zz when pp is null).  All of the thread's rows advance chunk by
    // chunk together, so RMAX*CH coefficient loads and then RMAX*CH gathers
    // are in flight at once; each row still accumulates in ascending k.
    constexpr int CH = (RMAX >= 8) ? 1 : (RMAX >= 4) ? 2 : 8;
    long long base[RMAX];
    int wr[RMAX];
    int wmax = 0;
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        base[k] = 0;
        wr[k] = 0;
        if (row[k] >= 0) {
            const int s = row[k] >> 5;
            base[k] = D.slice_off[s] + lane;
            wr[k] = D.slice_w[s];
            wmax = wr[k] > wmax ? wr[k] : wmax;
        }
    }
    auto offdiag_all = [&](double beta, const double* pp, const double* zz, double* off) {
#pragma unroll
        for (int k = 0; k < RMAX; ++k) off[k] = 0.0;
        for (int k0 = 0; k0 < wmax; k0 += CH) {
            int c[RMAX][CH];
            double v[RMAX][CH], g[RMAX][CH];
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < CH; ++u) {
                    const bool ok = k0 + u < wr[k];
                    c[k][u] = ok ? D.col[base[k] + 32LL * (k0 + u)] : 0;
                    v[k][u] = ok ? D.val[base[k] + 32LL * (k0 + u)] : 0.0;
                }
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < CH; ++u) {
                    const bool ok = k0 + u < wr[k];
                    g[k][u] = ok ? (pp ? fma(beta, __ldcg(pp + c[k][u]), __ldcg(zz + c[k][u])) : __ldcg(zz + c[k][u])) : 0.0;
                }
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < CH; ++u) off[k] = fma(v[k][u], g[k][u], off[k]);
        }
    };

    // ---- r0 = b - A p0, z0; direction buffer 0 cleared for iteration 1
    Acc4 acc{0.0, 0.0, 0.0, 0.0};
    double off[RMAX];
    offdiag_all(0.0, nullptr, D.pres, off);
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int i = row[k];
        if (i < 0) continue;
        const uint8_t f = D.nflag[i];
        const bool active = f & 1;
        fr[k] = (f & 1) && !(f & 4);
        dg[k] = D.pdiag[i];
        const double y = fma(dg[k], D.pres[i], off[k]);
        double ri = active ? D.rhs1[i] - y : 0.0;
        if (!fr[k]) ri = 0.0;
        double zi = 0.0;
        if (fr[k]) {
            if (g.precond) {
                if (!(isfinite(dg[k]) && dg[k] > 1.0e-30)) acc.flag = fmax(acc.flag, 1.0);
                else zi = ri / dg[k];
            } else {
                zi = ri;
            }
            if (!isfinite(ri)) acc.flag = fmax(acc.flag, 2.0);
            acc.a = fma(ri, ri, acc.a);
            acc.b = fma(ri, zi, acc.b);
            acc.mx = fmax(acc.mx, fabs(ri));
        }
        r[k] = ri;
        D.z[i] = zi;
        D.pA[i] = 0.0;
    }
    Acc4 t = Acc4{0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce(acc, D, g, phase, t)) return;
    ++phase;
    const double init = sqrt(t.a);
    if (init <= 1.0e-300) { cg_finish(D, g, 0, 1, init, init, 0.0, t.mx); return; }
    if (cg_converged(g.conv_test, 1.0, t.mx, g.rel_tol, g.abs_tol)) { cg_finish(D, g, 0, 1, init, init, 1.0, t.mx); return; }
    if (t.flag >= 2.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, 0, R_PCG_RESID); return; }
    if (t.flag >= 1.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 1, ST_PCG, 0, R_PCG_DIAG); return; }
    double rz = t.b;
    if (rz <= 1.0e-300 || !isfinite(rz)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, 0, R_PCG_RZ0); return; }

    double beta = 0.0, fin = init, rel = 1.0, mx = t.mx;
    int it = 0, conv = 0;
    for (it = 1; it <= g.max_iter; ++it) {
        const double* pprev = (it & 1) ? D.pA : D.pB;
        double* pnew = (it & 1) ? D.pB : D.pA;
        // ---- p = z + beta p (own rows), q = A p with neighbours' p formed on the fly
        Acc4 pa{0.0, 0.0, 0.0, 0.0};
        offdiag_all(beta, pprev, D.z, off);
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            p[k] = fr[k] ? fma(beta, p[k], D.z[i]) : 0.0;
            pnew[i] = p[k];
            q[k] = fr[k] ? fma(dg[k], p[k], off[k]) : 0.0;
            if (fr[k]) pa.a = fma(p[k], q[k], pa.a);
        }
        t = Acc4{0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce(pa, D, g, phase, t)) return;
        ++phase;
        const double pAp = t.a;
        if (fabs(pAp) <= 1.0e-300 || !isfinite(pAp)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_PAP); return; }
        const double alpha = rz / pAp;

        // ---- x += alpha p, r -= alpha q, z = M^-1 r
        Acc4 rr{0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0 || !fr[k]) continue;
            D.pres[i] = fma(alpha, p[k], D.pres[i]);
            r[k] = fma(-alpha, q[k], r[k]);
            const double zk = g.precond ? r[k] / dg[k] : r[k];
            D.z[i] = zk;
            if (!isfinite(r[k])) rr.flag = 1.0;
            rr.a = fma(r[k], r[k], rr.a);
            rr.b = fma(r[k], zk, rr.b);
            rr.mx = fmax(rr.mx, fabs(r[k]));
        }
        t = Acc4{0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce(rr, D, g, phase, t)) return;
        ++phase;
        fin = sqrt(t.a);
        mx = t.mx;
        rel = fin / init;
        if (cg_converged(g.conv_test, rel, mx, g.rel_tol, g.abs_tol)) { conv = 1; break; }
        if (t.flag > 0.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, it, R_PCG_RESID); return; }
        const double rzn = t.b;
        if (rzn <= 1.0e-300 || !isfinite(rzn)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_RZ); return; }
        beta = rzn / rz;
        rz = rzn;
    }
    if (it > g.max_iter) it = g.max_iter;
    cg_finish(D, g, it, conv, init, fin, rel, mx);
    if (!conv && b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 2, ST_PCG, it, R_PCG_MAXIT);
}

// ---------------------------------------- halo-staged FP64 PCG (default)
// The register-resident algorithm of k_pcg64r with the neighbour gathers
// served from shared memory.  Each persistent CTA owns a contiguous block of
// slices; the host lists, per CTA, the distinct nodes its rows reference (its
// halo, own rows included) and rewrites every pair entry's column as a 16-bit
// index into that list.  Each phase the CTA stages the values it needs
// (v = beta*p_prev + z, or the pressure in phase 0) for its halo into shared
// memory with one cooperative, mostly contiguous load, and the matvec then
// reads only the streamed coefficients from global memory.  The local column
// indices stay in shared memory for the whole solve.
template <int RMAX>
__global__ void __launch_bounds__(PCG_THREADS, PCG_CTAS_PER_SM) k_pcg64h(PcgDev D)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SegView g = seg_view<false>(D);
    const int G = g.G, b = g.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s_beg = g.s0 + (int)((long long)b * (g.s1 - g.s0) / G);
    const int s_end = g.s0 + (int)((long long)(b + 1) * (g.s1 - g.s0) / G);
    const long long S0 = D.slice_off[s_beg];
    const int nsl = (int)(D.slice_off[s_end] - S0);
    const int h0 = D.halo_ptr[blockIdx.x];
    const int nh = D.halo_ptr[blockIdx.x + 1] - h0;
    double* vh = reinterpret_cast<double*>(smem_raw);
    int* hidx = reinterpret_cast<int*>(vh + D.halo_max);
    unsigned short* lcs = reinterpret_cast<unsigned short*>(hidx + D.halo_max);
    for (int k = threadIdx.x; k < nh; k += PCG_THREADS) hidx[k] = D.halo_idx[h0 + k];
    for (int k = threadIdx.x; k < nsl; k += PCG_THREADS) lcs[k] = D.lcol[S0 + k];
    int phase = 0;
    

    double r[RMAX], p[RMAX], q[RMAX], dg[RMAX];
    bool fr[RMAX];
    int row[RMAX], lbase[RMAX], wr[RMAX];
    int wmax = 0;
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int s = s_beg + warp + PCG_WARPS * k;
        row[k] = (s < s_end) ? s * 32 + lane : -1;
        lbase[k] = 0;
        wr[k] = 0;
        if (s < s_end) {
            lbase[k] = (int)(D.slice_off[s] - S0) + lane;
            wr[k] = D.slice_w[s];
            wmax = wr[k] > wmax ? wr[k] : wmax;
        }
        r[k] = p[k] = q[k] = dg[k] = 0.0;
        fr[k] = false;
    }

    // stage v_j = beta*pp_j + zz_j (v = zz when pp is null) for the halo
    auto stage = [&](double beta, const double* pp, const double* zz) {
        __syncthreads();
        for (int k = threadIdx.x; k < nh; k += PCG_THREADS) {
            const int j = hidx[k];
            vh[k] = pp ? fma(beta, __ldcg(pp + j), __ldcg(zz + j)) : __ldcg(zz + j);
        }
        __syncthreads();
    };
    constexpr int CH = (RMAX >= 8) ? 2 : (RMAX >= 4) ? 4 : 8;
    auto offdiag_all = [&](double* off) {
#pragma unroll
        for (int k = 0; k < RMAX; ++k) off[k] = 0.0;
        for (int k0 = 0; k0 < wmax; k0 += CH) {
            double v[RMAX][CH];
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < CH; ++u)
                    v[k][u] = (k0 + u < wr[k]) ? __ldcg(D.val + S0 + lbase[k] + 32 * (k0 + u)) : 0.0;
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < CH; ++u) {
                    const double g = (k0 + u < wr[k]) ? vh[lcs[lbase[k] + 32 * (k0 + u)]] : 0.0;
                    off[k] = fma(v[k][u], g, off[k]);
                }
        }
    };

    // ---- r0 = b - A p0, z0; direction buffer 0 cleared for iteration 1
    Acc4 acc{0.0, 0.0, 0.0, 0.0};
    double off[RMAX];
    stage(0.0, nullptr, D.pres);
    offdiag_all(off);
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int i = row[k];
        if (i < 0) continue;
        const uint8_t f = D.nflag[i];
        const bool active = f & 1;
        fr[k] = (f & 1) && !(f & 4);
        dg[k] = D.pdiag[i];
        const double y = fma(dg[k], D.pres[i], off[k]);
        double ri = active ? D.rhs1[i] - y : 0.0;
        if (!fr[k]) ri = 0.0;
        double zi = 0.0;
        if (fr[k]) {
            if (g.precond) {
                if (!(isfinite(dg[k]) && dg[k] > 1.0e-30)) acc.flag = fmax(acc.flag, 1.0);
                else zi = ri / dg[k];
            } else {
                zi = ri;
            }
            if (!isfinite(ri)) acc.flag = fmax(acc.flag, 2.0);
            acc.a = fma(ri, ri, acc.a);
            acc.b = fma(ri, zi, acc.b);
            acc.mx = fmax(acc.mx, fabs(ri));
        }
        r[k] = ri;
        D.z[i] = zi;
        D.pA[i] = 0.0;
    }
    Acc4 t = Acc4{0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce(acc, D, g, phase, t)) return;
    ++phase;
    const double init = sqrt(t.a);
    if (init <= 1.0e-300) { cg_finish(D, g, 0, 1, init, init, 0.0, t.mx); return; }
    if (cg_converged(g.conv_test, 1.0, t.mx, g.rel_tol, g.abs_tol)) { cg_finish(D, g, 0, 1, init, init, 1.0, t.mx); return; }
    if (t.flag >= 2.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, 0, R_PCG_RESID); return; }
    if (t.flag >= 1.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 1, ST_PCG, 0, R_PCG_DIAG); return; }
    double rz = t.b;
    if (rz <= 1.0e-300 || !isfinite(rz)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, 0, R_PCG_RZ0); return; }

    double beta = 0.0, fin = init, rel = 1.0, mx = t.mx;
    int it = 0, conv = 0;
    for (it = 1; it <= g.max_iter; ++it) {
        const double* pprev = (it & 1) ? D.pA : D.pB;
        double* pnew = (it & 1) ? D.pB : D.pA;
        Acc4 pa{0.0, 0.0, 0.0, 0.0};
        stage(beta, pprev, D.z);
        offdiag_all(off);
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            p[k] = fr[k] ? fma(beta, p[k], D.z[i]) : 0.0;
            pnew[i] = p[k];
            q[k] = fr[k] ? fma(dg[k], p[k], off[k]) : 0.0;
            if (fr[k]) pa.a = fma(p[k], q[k], pa.a);
        }
        t = Acc4{0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce(pa, D, g, phase, t)) return;
        ++phase;
        const double pAp = t.a;
        if (fabs(pAp) <= 1.0e-300 || !isfinite(pAp)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_PAP); return; }
        const double alpha = rz / pAp;

        Acc4 rr{0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0 || !fr[k]) continue;
            D.pres[i] = fma(alpha, p[k], D.pres[i]);
            r[k] = fma(-alpha, q[k], r[k]);
            const double zk = g.precond ? r[k] / dg[k] : r[k];
            D.z[i] = zk;
            if (!isfinite(r[k])) rr.flag = 1.0;
            rr.a = fma(r[k], r[k], rr.a);
            rr.b = fma(r[k], zk, rr.b);
            rr.mx = fmax(rr.mx, fabs(r[k]));
        }
        t = Acc4{0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce(rr, D, g, phase, t)) return;
        ++phase;
        fin = sqrt(t.a);
        mx = t.mx;
        rel = fin / init;
        if (cg_converged(g.conv_test, rel, mx, g.rel_tol, g.abs_tol)) { conv = 1; break; }
        if (t.flag > 0.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, it, R_PCG_RESID); return; }
        const double rzn = t.b;
        if (rzn <= 1.0e-300 || !isfinite(rzn)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_RZ); return; }
        beta = rzn / rz;
        rz = rzn;
    }
    if (it > g.max_iter) it = g.max_iter;
    cg_finish(D, g, it, conv, init, fin, rel, mx);
    if (!conv && b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 2, ST_PCG, it, R_PCG_MAXIT);
}

// --------------------------- single-synchronisation halo PCG (default)
// Chronopoulos-Gear form of the same Jacobi-PCG: the matvec is applied to z
// (w = A z) and the direction's product s = A p follows the recurrence
// s = w + beta*s, so alpha and beta come from one grid reduction of
// (r.z, z.w, r.r, max|r|) per iteration instead of two.  Residuals, stopping
// test, iteration count and breakdown checks keep the reference's meaning
// (src/linalg/ConjugateGradient.cpp:725-853); in exact arithmetic the iterates
// equal the standard PCG's.  Neighbour values of the new z are formed while
// the halo is staged, from the previous iteration's r, w, s (double-buffered
// by iteration parity) and the diagonal, with the same operations the owner
// applies to its own rows.
struct Acc6 {
    double a, b, c, mx, flag;
};

// Grid-wide all-reduce of NV values per thread: the first NSUM summed, the
// rest max-reduced.  Every CTA publishes its partials (double-buffered by
// phase parity), arrives on a 64-bit counter that only grows, waits until
// all G CTAs of this phase have arrived, and then reduces the G partials
// itself in a fixed order (thread t takes CTAs t, t+T, ...; warp shuffles;
// warps in order).  The partials are stored value-major (value q of CTA b at
// q*G + b), so a warp reading one value of 32 CTAs touches two L2 lines.  Every CTA therefore computes bit-identical totals without
// a second round trip through a last-arriving CTA.  The caller passes the
// number of all-reduces this launch has completed as `phase`.  Returns false
// when the wait gave up (status TIMEOUT) or another CTA raised a status.
template <int NV, int NSUM, int NT>
__device__ __forceinline__ bool grid_allreduce_v(double (&v)[NV], const PcgDev& D, const SegView& g, int phase,
                                                 double (&out)[NV])
{
    static_assert(NV <= 8, "partials hold 8 doubles per CTA");
    __shared__ double sm[(NT / 32)][NV];
    __shared__ int s_ok;
    const int G = g.G;
    DevStatus* status = seg_status(D, g);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const double x = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = q < NSUM ? v[q] + x : fmax(v[q], x);
        }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sm[w][q] = v[q];
    __syncthreads();
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(seg_bar(D, g));
    double* part = seg_part(D, g) + (size_t)(phase & 1) * G * 8;
    if (threadIdx.x == 0) {
        double t[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) t[q] = 0.0;
        for (int k = 0; k < (NT / 32); ++k)
#pragma unroll
            for (int q = 0; q < NV; ++q) t[q] = q < NSUM ? t[q] + sm[k][q] : fmax(t[q], sm[k][q]);
#pragma unroll
        for (int q = 0; q < NV; ++q) __stcg(part + (q * G + g.b), t[q]);
        const unsigned long long target = (unsigned long long)(phase + 1) * (unsigned long long)G;
        unsigned long long arrived;
        asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], 1;" : "=l"(arrived) : "l"(cnt) : "memory");
        int ok = 1;
        if (arrived + 1 < target) {
            const long long t0 = clock64();
            for (;;) {
                unsigned long long c;
                asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(c) : "l"(cnt) : "memory");
                if (c >= target) break;
                if (ld_relaxed_int(&status->code) != 0) { ok = 0; break; }
                if (clock64() - t0 > (1LL << 31)) {
                    set_status(status, 5 /*CBS3D_TIMEOUT*/, ST_PCG, 0, R_PCG_BARRIER);
                    ok = 0;
                    break;
                }
            }
        }
        if (ok && ld_relaxed_int(&status->code) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    const bool ok = s_ok != 0;
    double t[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) t[q] = 0.0;
    if (ok) {
        for (int k = threadIdx.x; k < G; k += NT) {
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                const double x = __ldcg(part + (q * G + k));
                t[q] = q < NSUM ? t[q] + x : fmax(t[q], x);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const double x = __shfl_down_sync(0xffffffffu, t[q], o);
            t[q] = q < NSUM ? t[q] + x : fmax(t[q], x);
        }
    // sm was last read by thread 0 before the barrier that published s_ok,
    // so the warps' totals can overwrite it now.  Thread q folds value q
    // over the warps in warp order (the same sums as every thread folding
    // all of them) and the warps read the NV results: NV shared-memory
    // reads per warp instead of NV * warps broadcasts, which at 16 warps
    // kept the shared-memory pipe busy for ~1,300 cycles per all-reduce.
    __shared__ double so[NV];
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sm[w][q] = t[q];
    __syncthreads();
    if (threadIdx.x < NV) {
        const int q = threadIdx.x;
        double x = 0.0;
        for (int k = 0; k < (NT / 32); ++k) x = q < NSUM ? x + sm[k][q] : fmax(x, sm[k][q]);
        so[q] = x;
    }
    __syncthreads();
    // no barrier after these reads: so is rewritten only after the next
    // call's third barrier, and every thread reads it before it arrives at
    // that call's first
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = so[q];
    return ok;
}

template <int NT>
__device__ __forceinline__ bool grid_allreduce3(Acc6 v, const PcgDev& D, const SegView& g, int phase, Acc6& out)
{
    double a[5] = {v.a, v.b, v.c, v.mx, v.flag}, o[5];
    const bool ok = grid_allreduce_v<5, 3, NT>(a, D, g, phase, o);
    out = Acc6{o[0], o[1], o[2], o[3], o[4]};
    return ok;
}

// Five sums, a max and a flag (the mixed solver's refresh after a correction).
struct Acc8 {
    double a, b, c, d, e, mx, flag;
};

template <int NT>
__device__ __forceinline__ bool grid_allreduce5(Acc8 v, const PcgDev& D, const SegView& g, int phase, Acc8& out)
{
    double a[7] = {v.a, v.b, v.c, v.d, v.e, v.mx, v.flag}, o[7];
    const bool ok = grid_allreduce_v<7, 5, NT>(a, D, g, phase, o);
    out = Acc8{o[0], o[1], o[2], o[3], o[4], o[5], o[6]};
    return ok;
}

// Grid all-reduce of (sum a, sum b, sum c, max mx, max flag) that also
// gathers one per-CTA sum: every CTA's block sum of `x` lands in cvec[CTA]
// of every CTA (the aggregated vectors of the two-level preconditioner).
template <int NT>
__device__ __forceinline__ bool grid_allreduce3g(Acc6 v, double x, const PcgDev& D, const SegView& g, int phase,
                                                 Acc6& out, double* cvec)
{
    constexpr int NW = NT / 32;
    __shared__ double sm[NW][6];
    __shared__ int s_ok;
    const int G = g.G;
    DevStatus* status = seg_status(D, g);
    double vv[6] = {v.a, v.b, v.c, v.mx, v.flag, x};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const double y = __shfl_down_sync(0xffffffffu, vv[q], o);
            vv[q] = (q < 3 || q == 5) ? vv[q] + y : fmax(vv[q], y);
        }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 6; ++q) sm[w][q] = vv[q];
    __syncthreads();
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(seg_bar(D, g));
    double* part = seg_part(D, g) + (size_t)(phase & 1) * G * 8;
    if (threadIdx.x == 0) {
        double t[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < NW; ++k)
#pragma unroll
            for (int q = 0; q < 6; ++q) t[q] = (q < 3 || q == 5) ? t[q] + sm[k][q] : fmax(t[q], sm[k][q]);
#pragma unroll
        for (int q = 0; q < 6; ++q) __stcg(part + (q * G + g.b), t[q]);
        const unsigned long long target = (unsigned long long)(phase + 1) * (unsigned long long)G;
        unsigned long long arrived;
        asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], 1;" : "=l"(arrived) : "l"(cnt) : "memory");
        int ok = 1;
        if (arrived + 1 < target) {
            const long long t0 = clock64();
            for (;;) {
                unsigned long long c;
                asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(c) : "l"(cnt) : "memory");
                if (c >= target) break;
                if (ld_relaxed_int(&status->code) != 0) { ok = 0; break; }
                if (clock64() - t0 > (1LL << 31)) {
                    set_status(status, 5 /*CBS3D_TIMEOUT*/, ST_PCG, 0, R_PCG_BARRIER);
                    ok = 0;
                    break;
                }
            }
        }
        if (ok && ld_relaxed_int(&status->code) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    const bool ok = s_ok != 0;
    double t[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (ok) {
        for (int k = threadIdx.x; k < G; k += NT) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double y = __ldcg(part + (q * G + k));
                t[q] = q < 3 ? t[q] + y : fmax(t[q], y);
            }
            cvec[k] = __ldcg(part + (5 * G + k));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double y = __shfl_down_sync(0xffffffffu, t[q], o);
            t[q] = q < 3 ? t[q] + y : fmax(t[q], y);
        }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 5; ++q) sm[w][q] = t[q];
    __syncthreads();
    double o5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < NW; ++k)
#pragma unroll
        for (int q = 0; q < 5; ++q) o5[q] = q < 3 ? o5[q] + sm[k][q] : fmax(o5[q], sm[k][q]);
    out = Acc6{o5[0], o5[1], o5[2], o5[3], o5[4]};
    __syncthreads();
    return ok;
}

// ------------------------------------ global-vector single-reduction PCG
// The Chronopoulos-Gear iteration of k_pcg64c for meshes whose rows do not
// fit the register tiling: the rows' r, s, w (double-buffered by iteration
// parity), direction p and pressure stay in global memory, and every CTA
// stages, per part of its slices, the new z of its halo into shared memory
// from the previous iteration's r, w, s and the inverse diagonal -- the same
// operations the owner applies to its rows.  One grid all-reduce per
// iteration (k_pcg64 takes two) and no separate vector-update pass.  The
// search direction lives in the engine's permuted right-hand side, which is
// dead once r0 is formed.  Where the whole halo fits (one part) the inverse
// diagonal of the halo stays in shared memory for the solve.
__global__ void __launch_bounds__(PCG_THREADS, PCG_CTAS_PER_SM) k_pcg64g(PcgDev D)
{
    constexpr int NT = PCG_THREADS;
    const SegView g = seg_view<false>(D);
    const int G = g.G, b = g.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s_beg = g.s0 + (int)((long long)b * (g.s1 - g.s0) / G);
    const int s_end = g.s0 + (int)((long long)(b + 1) * (g.s1 - g.s0) / G);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int KP = D.halo_parts > 0 ? D.halo_parts : 1;
    const bool dzres = KP == 1;   // the halo's inverse diagonal resident in shared memory
    double* vh = reinterpret_cast<double*>(smem_raw);
    double* dzh = vh + D.halo_max;
    int phase = 0;
    const int N = D.N;
    double* rb[2] = {D.r, D.r + N};
    double* wb[2] = {D.q, D.q + N};
    double* sb[2] = {D.pA, D.pB};
    double* dz = D.z;     // free ? 1/diagonal : 0  (z = r * dz)
    double* pv = D.rhs1;  // search direction (after r0)

    // halo of part q: h0, nh
    auto halo_of = [&](int q, int& h0, int& nh) {
        h0 = D.halo_ptr[b * KP + q];
        nh = D.halo_ptr[b * KP + q + 1] - h0;
    };
    // off-diagonal sum of row s*32+lane over the staged halo: rounds of eight
    // slots, the next round's local columns and coefficients requested before
    // this round's shared-memory reads; the sum runs over the slots in order
    auto offdiag = [&](int s) -> double {
        const long long base = D.slice_off[s] + lane;
        const int w = D.slice_w[s];
        constexpr int CH = 8;
        double off = 0.0;
        int cn[CH];
        double vn[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            cn[u] = u < w ? (int)__ldcs(D.lcol + base + 32LL * u) : 0;
            vn[u] = u < w ? __ldcs(D.val + base + 32LL * u) : 0.0;
        }
        for (int k0 = 0; k0 < w; k0 += CH) {
            int c[CH];
            double v[CH];
#pragma unroll
            for (int u = 0; u < CH; ++u) { c[u] = cn[u]; v[u] = vn[u]; }
#pragma unroll
            for (int u = 0; u < CH; ++u) {
                const int k = k0 + CH + u;
                cn[u] = k < w ? (int)__ldcs(D.lcol + base + 32LL * k) : 0;
                vn[u] = k < w ? __ldcs(D.val + base + 32LL * k) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < CH; ++u)
                if (k0 + u < w) off = fma(v[u], vh[c[u]], off);
        }
        return off;
    };

    // ---- phase 0a: r0 = b - A x0 (constraints as the reference), dz, p = s = 0
    Acc6 acc{0.0, 0.0, 0.0, 0.0, 0.0};
    for (int part = 0; part < KP; ++part) {
        const int ps0 = s_beg + (int)((long long)part * (s_end - s_beg) / KP);
        const int ps1 = s_beg + (int)((long long)(part + 1) * (s_end - s_beg) / KP);
        int h0, nh;
        halo_of(part, h0, nh);
        __syncthreads();
        for (int k = threadIdx.x; k < nh; k += NT) vh[k] = __ldcg(D.pres + D.halo_idx[h0 + k]);
        __syncthreads();
        for (int s = ps0 + warp; s < ps1; s += PCG_WARPS) {
            const int i = s * 32 + lane;
            const double off = offdiag(s);
            const uint8_t f = D.nflag[i];
            const bool active = f & 1, fr = (f & 1) && !(f & 4);
            const double pd = D.pdiag[i];
            const double y = fma(pd, D.pres[i], off);
            double ri = active ? D.rhs1[i] - y : 0.0;
            double dd = 0.0;
            if (!fr) ri = 0.0;
            if (fr) {
                if (g.precond) {
                    if (!(isfinite(pd) && pd > 1.0e-30)) acc.flag = fmax(acc.flag, 1.0);
                    dd = 1.0 / pd;
                } else {
                    dd = 1.0;
                }
                if (!isfinite(ri)) acc.flag = fmax(acc.flag, 2.0);
                acc.c = fma(ri, ri, acc.c);
                acc.mx = fmax(acc.mx, fabs(ri));
            }
            rb[0][i] = ri;
            dz[i] = dd;
            sb[0][i] = 0.0;
        }
    }
    Acc6 t{0.0, 0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce3<NT>(acc, D, g, phase, t)) return;
    ++phase;
    const double init = sqrt(t.c);
    if (init <= 1.0e-300) { cg_finish(D, g, 0, 1, init, init, 0.0, t.mx); return; }
    if (cg_converged(g.conv_test, 1.0, t.mx, g.rel_tol, g.abs_tol)) { cg_finish(D, g, 0, 1, init, init, 1.0, t.mx); return; }
    if (t.flag >= 2.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, 0, R_PCG_RESID); return; }
    if (t.flag >= 1.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 1, ST_PCG, 0, R_PCG_DIAG); return; }

    // ---- phase 0b: z0 = M^-1 r0, w0 = A z0, gamma0 = (r0,z0), delta0 = (z0,w0);
    // the right-hand side is no longer needed: p = 0 from here
    acc = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
    for (int part = 0; part < KP; ++part) {
        const int ps0 = s_beg + (int)((long long)part * (s_end - s_beg) / KP);
        const int ps1 = s_beg + (int)((long long)(part + 1) * (s_end - s_beg) / KP);
        int h0, nh;
        halo_of(part, h0, nh);
        __syncthreads();
        for (int k = threadIdx.x; k < nh; k += NT) {
            const int j = D.halo_idx[h0 + k];
            const double dj = __ldcg(dz + j);
            if (dzres) dzh[k] = dj;
            vh[k] = __ldcg(rb[0] + j) * dj;
        }
        __syncthreads();
        for (int s = ps0 + warp; s < ps1; s += PCG_WARPS) {
            const int i = s * 32 + lane;
            const double off = offdiag(s);
            const uint8_t f = D.nflag[i];
            const bool fr = (f & 1) && !(f & 4);
            const double ri = rb[0][i];
            const double zi = ri * dz[i];
            const double wi = fr ? fma(D.pdiag[i], zi, off) : 0.0;
            wb[0][i] = wi;
            pv[i] = 0.0;
            if (fr) {
                acc.a = fma(ri, zi, acc.a);
                acc.b = fma(zi, wi, acc.b);
            }
        }
    }
    t = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce3<NT>(acc, D, g, phase, t)) return;
    ++phase;
    double gam = t.a;
    if (gam <= 1.0e-300 || !isfinite(gam)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, 0, R_PCG_RZ0); return; }
    double den = t.b;
    double beta = 0.0, fin = init, rel = 1.0, mx = 0.0, alpha = 0.0;
    int it = 0, conv = 0;
    for (it = 1; it <= g.max_iter; ++it) {
        if (fabs(den) <= 1.0e-300 || !isfinite(den)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_PAP); return; }
        alpha = gam / den;
        const int po = (it - 1) & 1, pn = it & 1;
        const double* so = sb[po];
        const double* wo = wb[po];
        const double* ro = rb[po];
        Acc6 a6{0.0, 0.0, 0.0, 0.0, 0.0};
        for (int part = 0; part < KP; ++part) {
            const int ps0 = s_beg + (int)((long long)part * (s_end - s_beg) / KP);
            const int ps1 = s_beg + (int)((long long)(part + 1) * (s_end - s_beg) / KP);
            int h0, nh;
            halo_of(part, h0, nh);
            // stage z_it of the halo: s = w_o + beta*s_o, r = r_o - alpha*s,
            // z = r * dz (SU nodes per thread per round, all loads first); the
            // all-reduce (or the previous part) ended with a barrier
            {
                constexpr int SU = 4;
                __syncthreads();
                for (int k0 = threadIdx.x; k0 < nh; k0 += SU * NT) {
                    double a[SU], c[SU], e[SU], d[SU];
#pragma unroll
                    for (int u = 0; u < SU; ++u) {
                        const int k = k0 + u * NT;
                        const int j = k < nh ? D.halo_idx[h0 + k] : 0;
                        a[u] = __ldcg(so + j);
                        c[u] = __ldcg(wo + j);
                        e[u] = __ldcg(ro + j);
                        d[u] = dzres ? 0.0 : __ldcg(dz + j);
                    }
#pragma unroll
                    for (int u = 0; u < SU; ++u) {
                        const int k = k0 + u * NT;
                        if (k < nh) {
                            const double sj = fma(beta, a[u], c[u]);
                            const double rj = fma(-alpha, sj, e[u]);
                            vh[k] = rj * (dzres ? dzh[k] : d[u]);
                        }
                    }
                }
                __syncthreads();
            }
            // own rows: p = z_o + beta*p, s = w_o + beta*s_o, x += alpha*p,
            // r = r_o - alpha*s; then w = A z, the partials
            for (int s = ps0 + warp; s < ps1; s += PCG_WARPS) {
                const int i = s * 32 + lane;
                const uint8_t f = D.nflag[i];
                const bool fr = (f & 1) && !(f & 4);
                const double r_o = ro[i], s_o = so[i], w_o = wo[i], dd = dz[i];
                const double p_o = pv[i];
                const double off = offdiag(s);
                const double zo = r_o * dd;
                const double pi = fr ? fma(beta, p_o, zo) : 0.0;
                const double si = fma(beta, s_o, w_o);
                if (fr) D.pres[i] = fma(alpha, pi, D.pres[i]);
                const double ri = fma(-alpha, si, r_o);
                pv[i] = pi;
                rb[pn][i] = ri;
                sb[pn][i] = si;
                const double zi = ri * dd;
                const double wi = fr ? fma(D.pdiag[i], zi, off) : 0.0;
                wb[pn][i] = wi;
                if (fr) {
                    if (!isfinite(ri)) a6.flag = 1.0;
                    a6.a = fma(ri, zi, a6.a);
                    a6.b = fma(zi, wi, a6.b);
                    a6.c = fma(ri, ri, a6.c);
                    a6.mx = fmax(a6.mx, fabs(ri));
                }
            }
        }
        t = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce3<NT>(a6, D, g, phase, t)) return;
        ++phase;
        fin = sqrt(t.c);
        mx = t.mx;
        rel = fin / init;
        if (cg_converged(g.conv_test, rel, mx, g.rel_tol, g.abs_tol)) { conv = 1; break; }
        if (t.flag > 0.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, it, R_PCG_RESID); return; }
        const double gn = t.a;
        if (gn <= 1.0e-300 || !isfinite(gn)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_RZ); return; }
        beta = gn / gam;
        den = t.b - beta * gn / alpha;
        gam = gn;
    }
    if (it > g.max_iter) it = g.max_iter;
    cg_finish(D, g, it, conv, init, fin, rel, mx);
    if (!conv && b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 2, ST_PCG, it, R_PCG_MAXIT);
}

// ---------------------------------------------- tensor memory as storage
// The SM's 256 KB tensor memory (TMEM: 128 lanes x 512 columns of 32 bits)
// holds, for the whole solve, coefficients that would otherwise stream from
// L2 in every iteration.  No MMA touches it: it is read with tcgen05.ld into
// registers.  With the 32x32b access shape, warp w reads and writes lanes
// 32*(w%4) .. 32*(w%4)+31, one lane per thread, so the four warps that share
// a lane quarter split the 512 columns into four ranges of 128.  One warp
// allocates all 512 columns (one CTA per SM, nothing else in this library
// uses TMEM) and frees them before the CTA exits, on every path.
__device__ __forceinline__ void tmem_alloc_all(uint32_t* slot)
{
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(slot));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(a) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free_all(uint32_t base)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(base) : "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// one double into two consecutive columns of this thread's lane (low word first)
__device__ __forceinline__ void tmem_st_f64(uint32_t addr, double v)
{
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(addr),
                 "r"(static_cast<uint32_t>(b)), "r"(static_cast<uint32_t>(b >> 32))
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// N consecutive 32-bit columns of this thread's lane; the registers are
// undefined until tmem_wait_ld, after which tmem_hold pins their uses
template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t addr, uint32_t (&r)[N]);
template <>
__device__ __forceinline__ void tmem_ld<4>(uint32_t addr, uint32_t (&r)[4])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}
template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t addr, uint32_t (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15])
                 : "r"(addr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// after tmem_wait_ld: an empty statement that "rewrites" the loaded registers,
// so no use of them can be scheduled before the wait
template <int N>
__device__ __forceinline__ void tmem_hold(uint32_t (&r)[N])
{
#pragma unroll
    for (int i = 0; i < N; ++i) asm volatile("" : "+r"(r[i]));
}

// KT > 0: the coefficients of each thread's rows KS .. KS+KT-1 live in TMEM
// for the solve (D.tm_w slots per row, zero-padded past the slice's width);
// `tm` is the CTA's TMEM base address (0 when KT = 0).
template <int RMAX, bool BATCH, int NT, int KS, int KT>
__device__ __forceinline__ void pcg64c_body(const PcgDev& D, uint32_t tm)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SegView g = seg_view<BATCH>(D);
    const int G = g.G, b = g.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s_beg = g.s0 + (int)((long long)b * (g.s1 - g.s0) / G);
    const int s_end = g.s0 + (int)((long long)(b + 1) * (g.s1 - g.s0) / G);
    const long long S0 = D.slice_off[s_beg];
    const int nsl = (int)(D.slice_off[s_end] - S0);
    const int h0 = D.halo_ptr[blockIdx.x];
    const int nh = D.halo_ptr[blockIdx.x + 1] - h0;
    double* vh = reinterpret_cast<double*>(smem_raw);
    double* dzh = vh + D.halo_max;
    int* hidx = reinterpret_cast<int*>(dzh + D.halo_max);
    unsigned short* lcs = reinterpret_cast<unsigned short*>(hidx + D.halo_max);
    // the own rows' pressure and diagonal, kept in shared memory for the
    // solve when the engine sized it so (the two-CTAs-per-SM kernel of small
    // meshes only; the other instantiations compile the global accesses alone)
    constexpr bool XS = NT == 256 && !BATCH;
    double* xs = XS && D.xs_off ? reinterpret_cast<double*>(smem_raw + D.xs_off) : nullptr;
    double* pds = xs ? xs + RMAX * NT
                : (NT == 512 && !BATCH && D.pds_off ? reinterpret_cast<double*>(smem_raw + D.pds_off) : nullptr);
    // XR: the own rows' pressure held in registers for the solve and stored
    // on every exit (the one-CTA-per-SM kernel: 12.18 -> 11.73 us per
    // iteration at 64^3; holding the diagonal there too was slower, 14.0 us)
    constexpr bool XR = NT == 512 && !BATCH;
    for (int k = threadIdx.x; k < nh; k += NT) hidx[k] = D.halo_idx[h0 + k];
    for (int k = threadIdx.x; k < nsl; k += NT) lcs[k] = D.lcol[S0 + k];
    // KS = 1: the coefficients of every warp's first row (the CTA's first
    // NT/32 slices, its leading slots) copied once into shared memory and
    // read from there in every iteration instead of from L2
    double* cvs = reinterpret_cast<double*>(smem_raw + D.coef_off);
    if constexpr (KS > 0) {
        const int sc = s_beg + (NT / 32) * KS < s_end ? s_beg + (NT / 32) * KS : s_end;
        const int c0 = (int)(D.slice_off[sc] - S0);
        for (int k = threadIdx.x; k < c0; k += NT) cvs[k] = __ldcg(D.val + S0 + k);
    }
    int phase = 0;
    const int N = D.N;
    // parity buffers: r in r/pA, w in q/pB, s in z/dz(+N)... laid out by the engine
    double* rb[2] = {D.r, D.r + N};
    double* wb[2] = {D.q, D.q + N};
    double* sb[2] = {D.pA, D.pB};
    double* dz = D.z;   // free ? 1/diagonal : 0  (z = r * dz)

    double r[RMAX], p[RMAX], s[RMAX], w[RMAX], dd[RMAX];
    double xr[RMAX];
    bool fr[RMAX];
    int row[RMAX], lbase[RMAX], wr[RMAX];
    int wmax = 0;
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int sl = s_beg + warp + (NT / 32) * k;
        row[k] = (sl < s_end) ? sl * 32 + lane : -1;
        lbase[k] = 0;
        wr[k] = 0;
        if (sl < s_end) {
            lbase[k] = (int)(D.slice_off[sl] - S0) + lane;
            wr[k] = D.slice_w[sl];
            wmax = wr[k] > wmax ? wr[k] : wmax;
        }
        r[k] = p[k] = s[k] = w[k] = 0.0;
        xr[k] = 0.0;
        dd[k] = 0.0;   // reciprocal of the Jacobi diagonal; 0 off the free rows
        fr[k] = false;
    }
    // coefficient columns loaded per round (measured: 2 rather than 4 at four
    // rows per thread takes the 64^3 iteration from 13.0 to 12.2 us)
    constexpr int CH = (RMAX >= 8) ? 2 : (RMAX >= 4) ? 2 : 8;
    static_assert(KT == 0 || KS + KT <= RMAX, "TMEM rows follow the shared-memory rows");
    // TMEM rows: row KS+q of this thread starts at column
    // 128*(warp/4) + 2*tm_w*q of lane 32*(warp%4)+lane; slot u of the row is
    // the double in columns 2u, 2u+1.  Every warp runs the same (uniform)
    // loops here, as the .sync.aligned forms require.
    uint32_t tmr[KT > 0 ? KT : 1];
    if constexpr (KT > 0) {
        const int tw = D.tm_w;
        const uint32_t wb0 = tm + (static_cast<uint32_t>(32 * (warp & 3)) << 16) + static_cast<uint32_t>(128 * (warp >> 2));
#pragma unroll
        for (int q = 0; q < KT; ++q) {
            tmr[q] = wb0 + static_cast<uint32_t>(2 * tw * q);
            const int k = KS + q;
            for (int u = 0; u < tw; ++u) {
                const double c = (u < wr[k]) ? __ldcg(D.val + S0 + lbase[k] + 32 * u) : 0.0;
                tmem_st_f64(tmr[q] + 2 * u, c);
            }
        }
        tmem_wait_st();
    }
    auto offdiag_all = [&](double* off) {
#pragma unroll
        for (int k = 0; k < RMAX; ++k) off[k] = 0.0;
        for (int k0 = 0; k0 < wmax; k0 += CH) {
            double v[RMAX][CH];
            uint32_t tv[KT > 0 ? KT : 1][2 * CH];
            if constexpr (KT > 0) {
#pragma unroll
                for (int q = 0; q < KT; ++q) tmem_ld<2 * CH>(tmr[q] + 2 * k0, tv[q]);
            }
#pragma unroll
            for (int k = 0; k < RMAX; ++k) {
                if (k >= KS && k < KS + KT) continue;
#pragma unroll
                for (int u = 0; u < CH; ++u)
                    v[k][u] = (k0 + u < wr[k]) ? (k < KS ? cvs[lbase[k] + 32 * (k0 + u)]
                                                         : __ldcg(D.val + S0 + lbase[k] + 32 * (k0 + u)))
                                               : 0.0;
            }
            if constexpr (KT > 0) {
                tmem_wait_ld();
#pragma unroll
                for (int q = 0; q < KT; ++q) {
                    tmem_hold<2 * CH>(tv[q]);
#pragma unroll
                    for (int u = 0; u < CH; ++u)
                        v[KS + q][u] = (k0 + u < wr[KS + q])
                                           ? __hiloint2double(static_cast<int>(tv[q][2 * u + 1]),
                                                              static_cast<int>(tv[q][2 * u]))
                                           : 0.0;
                }
            }
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < CH; ++u) {
                    const double g = (k0 + u < wr[k]) ? vh[lcs[lbase[k] + 32 * (k0 + u)]] : 0.0;
                    off[k] = fma(v[k][u], g, off[k]);
                }
        }
    };

    // ---- phase 0a: r0 = b - A x0 (constraints as the reference), dz
    double off[RMAX];
    __syncthreads();
    for (int k0 = threadIdx.x; k0 < nh; k0 += 4 * NT) {
        double a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * NT;
            a[u] = __ldcg(D.pres + (k < nh ? hidx[k] : 0));
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k0 + u * NT < nh) vh[k0 + u * NT] = a[u];
    }
    __syncthreads();
    offdiag_all(off);
    Acc6 acc{0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int i = row[k];
        if (i < 0) continue;
        const uint8_t f = D.nflag[i];
        const bool active = f & 1;
        fr[k] = (f & 1) && !(f & 4);
        const double pd = D.pdiag[i];
        const double xi = D.pres[i];
        if (xs) xs[k * NT + threadIdx.x] = xi;
        if (pds) pds[k * NT + threadIdx.x] = pd;
        if (XR) xr[k] = xi;
        const double y = fma(pd, xi, off[k]);
        double ri = active ? D.rhs1[i] - y : 0.0;
        if (!fr[k]) ri = 0.0;
        if (fr[k]) {
            if (g.precond) {
                if (!(isfinite(pd) && pd > 1.0e-30)) acc.flag = fmax(acc.flag, 1.0);
                dd[k] = 1.0 / pd;
            } else {
                dd[k] = 1.0;
            }
            if (!isfinite(ri)) acc.flag = fmax(acc.flag, 2.0);
            acc.c = fma(ri, ri, acc.c);
            acc.mx = fmax(acc.mx, fabs(ri));
        }
        r[k] = ri;
        rb[0][i] = ri;
        dz[i] = dd[k];
        sb[0][i] = 0.0;
    }
    // the pressure of the free own rows back to global memory
    auto store_x = [&]() {
        if (XR) {
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
                if (row[k] >= 0 && fr[k]) D.pres[row[k]] = xr[k];
            return;
        }
        if (!xs) return;
#pragma unroll
        for (int k = 0; k < RMAX; ++k)
            if (row[k] >= 0 && fr[k]) D.pres[row[k]] = xs[k * NT + threadIdx.x];
    };
    Acc6 t{0.0, 0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce3<NT>(acc, D, g, phase, t)) return;
    ++phase;
    const double init = sqrt(t.c);
    if (init <= 1.0e-300) { cg_finish(D, g, 0, 1, init, init, 0.0, t.mx); return; }
    if (cg_converged(g.conv_test, 1.0, t.mx, g.rel_tol, g.abs_tol)) { cg_finish(D, g, 0, 1, init, init, 1.0, t.mx); return; }
    if (t.flag >= 2.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, 0, R_PCG_RESID); return; }
    if (t.flag >= 1.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 1, ST_PCG, 0, R_PCG_DIAG); return; }

    // ---- phase 0b: z0 = M^-1 r0, w0 = A z0, gamma0 = (r0,z0), delta0 = (z0,w0)
    __syncthreads();
    for (int k0 = threadIdx.x; k0 < nh; k0 += 4 * NT) {
        double a[4], c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * NT;
            const int j = k < nh ? hidx[k] : 0;
            a[u] = __ldcg(dz + j);
            c[u] = __ldcg(rb[0] + j);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * NT;
            if (k < nh) { dzh[k] = a[u]; vh[k] = c[u] * a[u]; }
        }
    }
    __syncthreads();
    offdiag_all(off);
    acc = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int i = row[k];
        if (i < 0) continue;
        const double zi = r[k] * dd[k];
        w[k] = fr[k] ? fma(pds ? pds[k * NT + threadIdx.x] : D.pdiag[i], zi, off[k]) : 0.0;
        wb[0][i] = w[k];
        if (fr[k]) {
            acc.a = fma(r[k], zi, acc.a);
            acc.b = fma(zi, w[k], acc.b);
        }
    }
    t = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce3<NT>(acc, D, g, phase, t)) { store_x(); return; }
    ++phase;
    double gam = t.a;
    if (gam <= 1.0e-300 || !isfinite(gam)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, 0, R_PCG_RZ0); return; }
    double den = t.b;
    double beta = 0.0, fin = init, rel = 1.0, mx = 0.0, alpha = 0.0;
    int it = 0, conv = 0;
    for (it = 1; it <= g.max_iter; ++it) {
        if (fabs(den) <= 1.0e-300 || !isfinite(den)) { store_x(); if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_PAP); return; }
        alpha = gam / den;
        const int po = (it - 1) & 1, pn = it & 1;
        // stage z_it of the halo: s = w_o + beta*s_o, r = r_o - alpha*s, z = r / dz
        // (SU halo nodes per thread per round, all their loads issued first);
        // the all-reduce above ended with a barrier, so vh is free to write
        {
            constexpr int SU = 4;
            const double* so = sb[po];
            const double* wo = wb[po];
            const double* ro = rb[po];
            for (int k0 = threadIdx.x; k0 < nh; k0 += SU * NT) {
                double a[SU], c[SU], e[SU];
#pragma unroll
                for (int u = 0; u < SU; ++u) {
                    const int k = k0 + u * NT;
                    const int j = k < nh ? hidx[k] : 0;
                    a[u] = __ldcg(so + j);
                    c[u] = __ldcg(wo + j);
                    e[u] = __ldcg(ro + j);
                }
#pragma unroll
                for (int u = 0; u < SU; ++u) {
                    const int k = k0 + u * NT;
                    if (k < nh) {
                        const double sj = fma(beta, a[u], c[u]);
                        const double rj = fma(-alpha, sj, e[u]);
                        vh[k] = rj * dzh[k];
                    }
                }
            }
        }
        __syncthreads();
        // own rows: p = z_o + beta*p, s = w + beta*s, x += alpha*p, r -= alpha*s
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            const double zo = r[k] * dd[k];
            p[k] = fr[k] ? fma(beta, p[k], zo) : 0.0;
            s[k] = fma(beta, s[k], w[k]);
            if (fr[k]) {
                if (XR) xr[k] = fma(alpha, p[k], xr[k]);
                else if (xs) xs[k * NT + threadIdx.x] = fma(alpha, p[k], xs[k * NT + threadIdx.x]);
                else D.pres[i] = fma(alpha, p[k], D.pres[i]);
            }
            r[k] = fma(-alpha, s[k], r[k]);
            rb[pn][i] = r[k];
            sb[pn][i] = s[k];
        }
        offdiag_all(off);
        Acc6 a6{0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            const double zi = r[k] * dd[k];
            w[k] = fr[k] ? fma(pds ? pds[k * NT + threadIdx.x] : D.pdiag[i], zi, off[k]) : 0.0;
            wb[pn][i] = w[k];
            if (fr[k]) {
                if (!isfinite(r[k])) a6.flag = 1.0;
                a6.a = fma(r[k], zi, a6.a);
                a6.b = fma(zi, w[k], a6.b);
                a6.c = fma(r[k], r[k], a6.c);
                a6.mx = fmax(a6.mx, fabs(r[k]));
            }
        }
        t = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
        if constexpr (NT == 256) {
            // four values: a non-finite residual is carried as an infinite
            // max |r| (measured faster for the small-mesh kernel only)
            double a4[4] = {a6.a, a6.b, a6.c, a6.flag > 0.0 ? __longlong_as_double(0x7ff0000000000000LL) : a6.mx};
            double o4[4];
            if (!grid_allreduce_v<4, 3, NT>(a4, D, g, phase, o4)) { store_x(); return; }
            t = Acc6{o4[0], o4[1], o4[2], o4[3], isinf(o4[3]) ? 1.0 : 0.0};
        } else {
            if (!grid_allreduce3<NT>(a6, D, g, phase, t)) { store_x(); return; }
        }
        ++phase;
        fin = sqrt(t.c);
        mx = t.mx;
        rel = fin / init;
        if (cg_converged(g.conv_test, rel, mx, g.rel_tol, g.abs_tol)) { conv = 1; break; }
        if (t.flag > 0.0) { store_x(); if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, it, R_PCG_RESID); return; }
        const double gn = t.a;
        if (gn <= 1.0e-300 || !isfinite(gn)) { store_x(); if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_RZ); return; }
        beta = gn / gam;
        den = t.b - beta * gn / alpha;
        gam = gn;
    }
    store_x();
    if (it > g.max_iter) it = g.max_iter;
    cg_finish(D, g, it, conv, init, fin, rel, mx);
    if (!conv && b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 2, ST_PCG, it, R_PCG_MAXIT);
}

// The single-reduction (Chronopoulos-Gear) Jacobi-PCG with its rows in
// registers.  KT > 0 (one 512-thread CTA per SM): warp 0 takes the SM's
// tensor memory before the solve and returns it after; every exit of the
// body (converged, an error status, a timed-out wait) is CTA-uniform and
// comes back here, so the memory is freed on every path.
template <int RMAX, bool BATCH, int NT, int KS = 0, int KT = 0>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2) k_pcg64c(PcgDev D)
{
    if constexpr (KT == 0) {
        pcg64c_body<RMAX, BATCH, NT, KS, 0>(D, 0u);
    } else {
        static_assert(NT == 512 && !BATCH, "TMEM rows: one CTA per SM, single system");
        __shared__ uint32_t s_tm;
        const bool w0 = (threadIdx.x >> 5) == 0;
        if (w0) tmem_alloc_all(&s_tm);
        tmem_fence_before_sync();
        __syncthreads();
        tmem_fence_after_sync();
        const uint32_t tm = s_tm;
        pcg64c_body<RMAX, BATCH, NT, KS, KT>(D, tm);
        tmem_fence_before_sync();
        __syncthreads();
        tmem_fence_after_sync();
        if (w0) tmem_free_all(tm);
    }
}

template <int RMAX>
__global__ void __launch_bounds__(512, 1) k_pcg64d(PcgDev D, CoarseDev C)
{
    constexpr bool BATCH = false;
    constexpr int NT = 512;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SegView g = seg_view<BATCH>(D);
    const int G = g.G, b = g.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s_beg = g.s0 + (int)((long long)b * (g.s1 - g.s0) / G);
    const int s_end = g.s0 + (int)((long long)(b + 1) * (g.s1 - g.s0) / G);
    const long long S0 = D.slice_off[s_beg];
    const int nsl = (int)(D.slice_off[s_end] - S0);
    const int h0 = D.halo_ptr[blockIdx.x];
    const int nh = D.halo_ptr[blockIdx.x + 1] - h0;
    double* vh = reinterpret_cast<double*>(smem_raw);
    double* dzh = vh + D.halo_max;
    int* hidx = reinterpret_cast<int*>(dzh + D.halo_max);
    unsigned short* lcs = reinterpret_cast<unsigned short*>(hidx + D.halo_max);
    for (int k = threadIdx.x; k < nh; k += NT) hidx[k] = D.halo_idx[h0 + k];
    for (int k = threadIdx.x; k < nsl; k += NT) lcs[k] = D.lcol[S0 + k];
    // coarse space: this CTA's rows of the coarse inverse (its own and its
    // halo's owners), the coarse vectors P^T r, P^T s, P^T w, the coarse
    // correction of each neighbour and the owner of every halo entry
    const int GC = C.G;
    const int nb0 = C.nbr_ptr[blockIdx.x];
    const int nn = C.nbr_ptr[blockIdx.x + 1] - nb0;
    double* ainv = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(lcs + D.slot_max) + 15) & ~static_cast<uintptr_t>(15));
    double* cr = ainv + (size_t)C.nbr_max * GC;
    double* cs = cr + GC;
    double* cw = cs + GC;
    double* ec = cw + GC;
    unsigned char* hown = reinterpret_cast<unsigned char*>(ec + C.nbr_max);
    __shared__ int s_own;
    __shared__ double s_ecp;   // this CTA's coarse correction of the previous iteration's z
    if (threadIdx.x == 0)
        for (int j = 0; j < nn; ++j)
            if (C.nbr_ids[nb0 + j] == (int)blockIdx.x) s_own = j;
    for (int t = threadIdx.x; t < nn * GC; t += NT)
        ainv[t] = C.ainv[(size_t)C.nbr_ids[nb0 + t / GC] * GC + t % GC];
    for (int k = threadIdx.x; k < nh; k += NT) hown[k] = C.hown[h0 + k];
    for (int t = threadIdx.x; t < GC; t += NT) cs[t] = 0.0;
    // ec[j] = (A_c^-1 P^T r)[neighbour j]: one warp per neighbour, fixed order
    auto coarse_correction = [&]() {
        __syncthreads();
        for (int j = warp; j < nn; j += NT / 32) {
            double acc = 0.0;
            for (int t = lane; t < GC; t += 32) acc = fma(ainv[(size_t)j * GC + t], cr[t], acc);
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if (lane == 0) ec[j] = acc;
        }
        __syncthreads();
    };
    int phase = 0;
    const int N = D.N;
    // parity buffers: r in r/pA, w in q/pB, s in z/dz(+N)... laid out by the engine
    double* rb[2] = {D.r, D.r + N};
    double* wb[2] = {D.q, D.q + N};
    double* sb[2] = {D.pA, D.pB};
    double* dz = D.z;   // free ? 1/diagonal : 0  (z = r * dz)

    // rows of this thread: slice s_beg + warp + NW*k, lane; their slot base
    // and width are re-read where needed (registers go to the coarse state)
    double r[RMAX], p[RMAX], s[RMAX], w[RMAX], dd[RMAX];
    bool fr[RMAX];
    int wmax = 0;
    auto slice_of = [&](int k) { return s_beg + warp + (NT / 32) * k; };
    auto row_of = [&](int k) { const int sl = slice_of(k); return sl < s_end ? sl * 32 + lane : -1; };
    auto width_of = [&](int k) { const int sl = slice_of(k); return sl < s_end ? D.slice_w[sl] : 0; };
    auto base_of = [&](int k) { const int sl = slice_of(k); return sl < s_end ? (int)(D.slice_off[sl] - S0) + lane : 0; };
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int wk = width_of(k);
        wmax = wk > wmax ? wk : wmax;
        r[k] = p[k] = s[k] = w[k] = 0.0;
        dd[k] = 0.0;   // reciprocal of the Jacobi diagonal; 0 off the free rows
        fr[k] = false;
    }
    constexpr int CH = (RMAX >= 8) ? 2 : (RMAX >= 4) ? 4 : 8;
    auto offdiag_all = [&](double* off) {
        int lbase[RMAX], wr[RMAX];
#pragma unroll
        for (int k = 0; k < RMAX; ++k) { off[k] = 0.0; lbase[k] = base_of(k); wr[k] = width_of(k); }
        for (int k0 = 0; k0 < wmax; k0 += CH) {
            double v[RMAX][CH];
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < CH; ++u)
                    v[k][u] = (k0 + u < wr[k]) ? __ldcg(D.val + S0 + lbase[k] + 32 * (k0 + u)) : 0.0;
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < CH; ++u) {
                    const double g = (k0 + u < wr[k]) ? vh[lcs[lbase[k] + 32 * (k0 + u)]] : 0.0;
                    off[k] = fma(v[k][u], g, off[k]);
                }
        }
    };

    // ---- phase 0a: r0 = b - A x0 (constraints as the reference), dz
    double off[RMAX];
    __syncthreads();
    for (int k0 = threadIdx.x; k0 < nh; k0 += 4 * NT) {
        double a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * NT;
            a[u] = __ldcg(D.pres + (k < nh ? hidx[k] : 0));
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k0 + u * NT < nh) vh[k0 + u * NT] = a[u];
    }
    __syncthreads();
    offdiag_all(off);
    Acc6 acc{0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int i = row_of(k);
        if (i < 0) continue;
        const uint8_t f = D.nflag[i];
        const bool active = f & 1;
        fr[k] = (f & 1) && !(f & 4);
        const double pd = D.pdiag[i];
        const double y = fma(pd, D.pres[i], off[k]);
        double ri = active ? D.rhs1[i] - y : 0.0;
        if (!fr[k]) ri = 0.0;
        if (fr[k]) {
            if (g.precond) {
                if (!(isfinite(pd) && pd > 1.0e-30)) acc.flag = fmax(acc.flag, 1.0);
                dd[k] = 1.0 / pd;
            } else {
                dd[k] = 1.0;
            }
            if (!isfinite(ri)) acc.flag = fmax(acc.flag, 2.0);
            acc.c = fma(ri, ri, acc.c);
            acc.mx = fmax(acc.mx, fabs(ri));
        }
        r[k] = ri;
        rb[0][i] = ri;
        dz[i] = dd[k];
        sb[0][i] = 0.0;
    }
    double xs = 0.0;
#pragma unroll
    for (int k = 0; k < RMAX; ++k) xs += r[k];
    Acc6 t{0.0, 0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce3g<NT>(acc, xs, D, g, phase, t, cr)) return;
    ++phase;
    const double init = sqrt(t.c);
    if (init <= 1.0e-300) { cg_finish(D, g, 0, 1, init, init, 0.0, t.mx); return; }
    if (cg_converged(g.conv_test, 1.0, t.mx, g.rel_tol, g.abs_tol)) { cg_finish(D, g, 0, 1, init, init, 1.0, t.mx); return; }
    if (t.flag >= 2.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, 0, R_PCG_RESID); return; }
    if (t.flag >= 1.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 1, ST_PCG, 0, R_PCG_DIAG); return; }

    // ---- phase 0b: z0 = M^-1 r0, w0 = A z0, gamma0 = (r0,z0), delta0 = (z0,w0)
    coarse_correction();
    for (int k0 = threadIdx.x; k0 < nh; k0 += 4 * NT) {
        double a[4], c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * NT;
            const int j = k < nh ? hidx[k] : 0;
            a[u] = __ldcg(dz + j);
            c[u] = __ldcg(rb[0] + j);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * NT;
            if (k < nh) { dzh[k] = a[u]; vh[k] = a[u] != 0.0 ? fma(c[u], a[u], ec[hown[k]]) : 0.0; }
        }
    }
    __syncthreads();
    offdiag_all(off);
    acc = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int i = row_of(k);
        if (i < 0) continue;
        const double zi = fr[k] ? fma(r[k], dd[k], ec[s_own]) : 0.0;
        w[k] = fr[k] ? fma(D.pdiag[i], zi, off[k]) : 0.0;
        wb[0][i] = w[k];
        if (fr[k]) {
            acc.a = fma(r[k], zi, acc.a);
            acc.b = fma(zi, w[k], acc.b);
        }
    }
    xs = 0.0;
#pragma unroll
    for (int k = 0; k < RMAX; ++k) xs += w[k];
    t = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce3g<NT>(acc, xs, D, g, phase, t, cw)) return;
    ++phase;
    if (threadIdx.x == 0) s_ecp = ec[s_own];
    double gam = t.a;
    if (gam <= 1.0e-300 || !isfinite(gam)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, 0, R_PCG_RZ0); return; }
    double den = t.b;
    double beta = 0.0, fin = init, rel = 1.0, mx = 0.0, alpha = 0.0;
    int it = 0, conv = 0;
    for (it = 1; it <= g.max_iter; ++it) {
        if (fabs(den) <= 1.0e-300 || !isfinite(den)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_PAP); return; }
        alpha = gam / den;
        const int po = (it - 1) & 1, pn = it & 1;
        // P^T s = P^T w_o + beta P^T s_o, P^T r = P^T r_o - alpha P^T s (the
        // recurrences of s and r, aggregated), then the new coarse correction
        for (int c = threadIdx.x; c < GC; c += NT) {
            cs[c] = fma(beta, cs[c], cw[c]);
            cr[c] = fma(-alpha, cs[c], cr[c]);
        }
        coarse_correction();
        // stage z_it of the halo: s = w_o + beta*s_o, r = r_o - alpha*s, z = r / dz
        // (SU halo nodes per thread per round, all their loads issued first)
        __syncthreads();
        {
            constexpr int SU = 8;   // halo nodes per thread per round (measured: 8 beats 4 and 2)
            const double* so = sb[po];
            const double* wo = wb[po];
            const double* ro = rb[po];
            for (int k0 = threadIdx.x; k0 < nh; k0 += SU * NT) {
                double a[SU], c[SU], e[SU];
#pragma unroll
                for (int u = 0; u < SU; ++u) {
                    const int k = k0 + u * NT;
                    const int j = k < nh ? hidx[k] : 0;
                    a[u] = __ldcg(so + j);
                    c[u] = __ldcg(wo + j);
                    e[u] = __ldcg(ro + j);
                }
#pragma unroll
                for (int u = 0; u < SU; ++u) {
                    const int k = k0 + u * NT;
                    if (k < nh) {
                        const double sj = fma(beta, a[u], c[u]);
                        const double rj = fma(-alpha, sj, e[u]);
                        vh[k] = dzh[k] != 0.0 ? fma(rj, dzh[k], ec[hown[k]]) : 0.0;
                    }
                }
            }
        }
        __syncthreads();
        // own rows: p = z_o + beta*p, s = w + beta*s, x += alpha*p, r -= alpha*s
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row_of(k);
            if (i < 0) continue;
            const double zo = fma(r[k], dd[k], s_ecp);
            p[k] = fr[k] ? fma(beta, p[k], zo) : 0.0;
            s[k] = fma(beta, s[k], w[k]);
            if (fr[k]) D.pres[i] = fma(alpha, p[k], D.pres[i]);
            r[k] = fma(-alpha, s[k], r[k]);
            rb[pn][i] = r[k];
            sb[pn][i] = s[k];
        }
        offdiag_all(off);
        Acc6 a6{0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row_of(k);
            if (i < 0) continue;
            const double zi = fr[k] ? fma(r[k], dd[k], ec[s_own]) : 0.0;
            w[k] = fr[k] ? fma(D.pdiag[i], zi, off[k]) : 0.0;
            wb[pn][i] = w[k];
            if (fr[k]) {
                if (!isfinite(r[k])) a6.flag = 1.0;
                a6.a = fma(r[k], zi, a6.a);
                a6.b = fma(zi, w[k], a6.b);
                a6.c = fma(r[k], r[k], a6.c);
                a6.mx = fmax(a6.mx, fabs(r[k]));
            }
        }
        xs = 0.0;
#pragma unroll
        for (int k = 0; k < RMAX; ++k) xs += w[k];
        t = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce3g<NT>(a6, xs, D, g, phase, t, cw)) return;
        ++phase;
        if (threadIdx.x == 0) s_ecp = ec[s_own];
        fin = sqrt(t.c);
        mx = t.mx;
        rel = fin / init;
        if (cg_converged(g.conv_test, rel, mx, g.rel_tol, g.abs_tol)) { conv = 1; break; }
        if (t.flag > 0.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, it, R_PCG_RESID); return; }
        const double gn = t.a;
        if (gn <= 1.0e-300 || !isfinite(gn)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_RZ); return; }
        beta = gn / gam;
        den = t.b - beta * gn / alpha;
        gam = gn;
    }
    if (it > g.max_iter) it = g.max_iter;
    cg_finish(D, g, it, conv, init, fin, rel, mx);
    if (!conv && b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 2, ST_PCG, it, R_PCG_MAXIT);
}

// ------------------------------------------- mixed-precision PCG (FP32)
// The Chronopoulos-Gear iteration of k_pcg64c in FP32 -- r, z, w, s, p and
// the assembled coefficients are single precision, the coefficients and local
// column indices resident in shared memory for the whole solve -- with the
// reductions, alpha/beta and the pressure in FP64, and FP64 defect
// correction by residual replacement: whenever the recursive residual has
// fallen by the inner tolerance since the last correction, and whenever it meets the
// stopping test, the true residual r = b - A x is recomputed from the FP64
// coefficients and FP64 pressure, and w = A z, s = A p are recomputed, so the
// FP32 recurrences restart from exact data without discarding the search
// direction; the curvature of the next direction is then computed from
// fresh products rather than recurred, and a correction that finds no
// progress since the previous one also drops the direction.  The solve
// stops only when the FP64 true residual meets the reference's stopping
// test.
constexpr int RU_STALL = 256;   // iterations without a correction before one is forced

template <int RMAX, bool BATCH, int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2) k_pcg32m(PcgDev D)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SegView g = seg_view<BATCH>(D);
    const int G = g.G, b = g.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s_beg = g.s0 + (int)((long long)b * (g.s1 - g.s0) / G);
    const int s_end = g.s0 + (int)((long long)(b + 1) * (g.s1 - g.s0) / G);
    const long long S0 = D.slice_off[s_beg];
    const int nsl = (int)(D.slice_off[s_end] - S0);
    const int h0 = D.halo_ptr[blockIdx.x];
    const int nh = D.halo_ptr[blockIdx.x + 1] - h0;
    const int HM = D.halo_max;
    double* vh64 = reinterpret_cast<double*>(smem_raw);                 // HM doubles, or:
    float* vz = reinterpret_cast<float*>(smem_raw);                     //   HM floats (z)
    float* vp = vz + HM;                                                //   HM floats (p)
    float* dzh = reinterpret_cast<float*>(vh64 + HM);                   // HM
    int* hidx = reinterpret_cast<int*>(dzh + HM);                       // HM
    float* val32s = reinterpret_cast<float*>(hidx + HM);                // nsl
    unsigned short* lcs = reinterpret_cast<unsigned short*>(val32s + D.slot_max);
    for (int k = threadIdx.x; k < nh; k += NT) hidx[k] = D.halo_idx[h0 + k];
    for (int k = threadIdx.x; k < nsl; k += NT) {
        lcs[k] = D.lcol[S0 + k];
        val32s[k] = D.val32[S0 + k];
    }
    int phase = 0;
    const int N = D.N;
    float* rb[2] = {D.r32, D.r32 + N};
    float* wb[2] = {D.w32, D.w32 + N};
    float* sb[2] = {D.s32, D.s32 + N};
    float* pb = D.p32;
    float* dz = D.dz32;

    float r[RMAX], p[RMAX], sv[RMAX], w[RMAX], dd[RMAX];
    bool fr[RMAX];
    int row[RMAX], lbase[RMAX], wr[RMAX];
    int wmax = 0;
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int sl = s_beg + warp + (NT / 32) * k;
        row[k] = (sl < s_end) ? sl * 32 + lane : -1;
        lbase[k] = 0;
        wr[k] = 0;
        if (sl < s_end) {
            lbase[k] = (int)(D.slice_off[sl] - S0) + lane;
            wr[k] = D.slice_w[sl];
            wmax = wr[k] > wmax ? wr[k] : wmax;
        }
        r[k] = p[k] = sv[k] = w[k] = 0.0f;
        dd[k] = 0.0f;   // reciprocal of the Jacobi diagonal; 0 off the free rows
        fr[k] = false;
    }
    // FP64 off-diagonal sums from the streamed FP64 coefficients and vh64
    auto offdiag64 = [&](double* off) {
#pragma unroll
        for (int k = 0; k < RMAX; ++k) off[k] = 0.0;
        for (int k0 = 0; k0 < wmax; k0 += 4) {
            double v[RMAX][4];
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    v[k][u] = (k0 + u < wr[k]) ? __ldcg(D.val + S0 + lbase[k] + 32 * (k0 + u)) : 0.0;
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const double g = (k0 + u < wr[k]) ? vh64[lcs[lbase[k] + 32 * (k0 + u)]] : 0.0;
                    off[k] = fma(v[k][u], g, off[k]);
                }
        }
    };
    // FP32 off-diagonal sums from the resident coefficients and a float halo
    auto offdiag32 = [&](const float* vx, float* off) {
#pragma unroll
        for (int k = 0; k < RMAX; ++k) off[k] = 0.0f;
        for (int kk = 0; kk < wmax; ++kk) {
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
                if (kk < wr[k]) {
                    const int sl = lbase[k] + 32 * kk;
                    off[k] = fmaf(val32s[sl], vx[lcs[sl]], off[k]);
                }
        }
    };
    auto stage64 = [&](const double* x) {
        __syncthreads();
        for (int k0 = threadIdx.x; k0 < nh; k0 += 4 * NT) {
            double a[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u * NT;
                a[u] = __ldcg(x + (k < nh ? hidx[k] : 0));
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k0 + u * NT < nh) vh64[k0 + u * NT] = a[u];
        }
        __syncthreads();
    };
    // true residual of the own rows into r[], rb[buf]; returns partials
    auto true_residual = [&](int buf, Acc6& acc) {
        stage64(D.pres);
        double off[RMAX];
        offdiag64(off);
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            const double y = fma(D.pdiag[i], D.pres[i], off[k]);
            double ri = (D.nflag[i] & 1) ? D.rhs1[i] - y : 0.0;
            if (!fr[k]) ri = 0.0;
            if (fr[k]) {
                if (!isfinite(ri)) acc.flag = fmax(acc.flag, 2.0);
                acc.c = fma(ri, ri, acc.c);
                acc.mx = fmax(acc.mx, fabs(ri));
            }
            r[k] = (float)ri;
            rb[buf][i] = r[k];
            pb[i] = p[k];
        }
    };
    // w = A z and s = A p from the staged halos (p taken as zero when
    // zero_p, which restarts the direction); partials of r.z, z.w, z.s, p.w
    // and p.s, from which the step length of the next direction
    // (z + beta p).A(z + beta p) follows directly
    auto refresh_ws = [&](int buf, bool zero_p, Acc8& acc) {
        __syncthreads();
        for (int k0 = threadIdx.x; k0 < nh; k0 += 4 * NT) {
            float a[4], c[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u * NT;
                const int j = k < nh ? hidx[k] : 0;
                a[u] = __ldcg(rb[buf] + j);
                c[u] = zero_p ? 0.0f : __ldcg(pb + j);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u * NT;
                if (k < nh) { vz[k] = a[u] * dzh[k]; vp[k] = c[u]; }
            }
        }
        __syncthreads();
        float offz[RMAX], offp[RMAX];
        offdiag32(vz, offz);
        offdiag32(vp, offp);
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            if (zero_p) p[k] = 0.0f;
            const float pd = (float)D.pdiag[i];
            const float zi = r[k] * dd[k];
            w[k] = fr[k] ? fmaf(pd, zi, offz[k]) : 0.0f;
            sv[k] = fr[k] ? fmaf(pd, p[k], offp[k]) : 0.0f;
            wb[buf][i] = w[k];
            sb[buf][i] = sv[k];
            if (fr[k]) {
                const double zd = zi, pv = p[k];
                acc.a = fma((double)r[k], zd, acc.a);
                acc.b = fma(zd, (double)w[k], acc.b);
                acc.c = fma(zd, (double)sv[k], acc.c);
                acc.d = fma(pv, (double)w[k], acc.d);
                acc.e = fma(pv, (double)sv[k], acc.e);
            }
        }
    };

    // ---- phase 0a: FP64 r0 = b - A x0, its norm, dz
    Acc6 acc{0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int i = row[k];
        if (i < 0) continue;
        const uint8_t f = D.nflag[i];
        fr[k] = (f & 1) && !(f & 4);
        const double pd = D.pdiag[i];
        if (fr[k]) {
            if (g.precond && !(isfinite(pd) && pd > 1.0e-30)) acc.flag = fmax(acc.flag, 1.0);
            dd[k] = g.precond ? (float)(1.0 / pd) : 1.0f;
        }
        dz[i] = dd[k];
        sb[0][i] = 0.0f;
    }
    true_residual(0, acc);
    Acc6 t{0.0, 0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce3<NT>(acc, D, g, phase, t)) return;
    ++phase;
    const double init = sqrt(t.c);
    if (init <= 1.0e-300) { cg_finish(D, g, 0, 1, init, init, 0.0, t.mx); return; }
    if (cg_converged(g.conv_test, 1.0, t.mx, g.rel_tol, g.abs_tol)) { cg_finish(D, g, 0, 1, init, init, 1.0, t.mx); return; }
    if (t.flag >= 2.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, 0, R_PCG_RESID); return; }
    if (t.flag >= 1.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 1, ST_PCG, 0, R_PCG_DIAG); return; }
    double rr_last = t.c;

    // ---- phase 0b: z0, w0 = A z0 (p = 0, s = 0)
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += NT) dzh[k] = __ldcg(dz + hidx[k]);
    Acc8 a8{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    refresh_ws(0, true, a8);
    Acc8 t8{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (!grid_allreduce5<NT>(a8, D, g, phase, t8)) return;
    ++phase;
    double gam = t8.a;
    if (gam <= 1.0e-300 || !isfinite(gam)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, 0, R_PCG_RZ0); return; }
    double den = t8.b;
    double beta = 0.0, fin = init, rel = 1.0, mx = 0.0, alpha = 0.0;
    int it = 0, conv = 0, outer = 0, last_fix = 0;
    for (it = 1; it <= g.max_iter; ++it) {
        if (fabs(den) <= 1.0e-300 || !isfinite(den)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_PAP); return; }
        alpha = gam / den;
        const float a32 = (float)alpha, b32 = (float)beta;
        const int po = (it - 1) & 1, pn = it & 1;
        __syncthreads();
        {
            const float* so = sb[po];
            const float* wo = wb[po];
            const float* ro = rb[po];
            for (int k0 = threadIdx.x; k0 < nh; k0 += 4 * NT) {
                float a[4], c[4], e[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = k0 + u * NT;
                    const int j = k < nh ? hidx[k] : 0;
                    a[u] = __ldcg(so + j);
                    c[u] = __ldcg(wo + j);
                    e[u] = __ldcg(ro + j);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = k0 + u * NT;
                    if (k < nh) {
                        const float sj = fmaf(b32, a[u], c[u]);
                        const float rj = fmaf(-a32, sj, e[u]);
                        vz[k] = rj * dzh[k];
                    }
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            const float zo = r[k] * dd[k];
            p[k] = fr[k] ? fmaf(b32, p[k], zo) : 0.0f;
            sv[k] = fmaf(b32, sv[k], w[k]);
            if (fr[k]) D.pres[i] = fma(alpha, (double)p[k], D.pres[i]);
            r[k] = fmaf(-a32, sv[k], r[k]);
            rb[pn][i] = r[k];
            sb[pn][i] = sv[k];
        }
        float off[RMAX];
        offdiag32(vz, off);
        Acc6 a6{0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            const float zi = r[k] * dd[k];
            w[k] = fr[k] ? fmaf((float)D.pdiag[i], zi, off[k]) : 0.0f;
            wb[pn][i] = w[k];
            if (fr[k]) {
                if (!isfinite(r[k])) a6.flag = 1.0;
                a6.a = fma((double)r[k], (double)zi, a6.a);
                a6.b = fma((double)zi, (double)w[k], a6.b);
                a6.c = fma((double)r[k], (double)r[k], a6.c);
                a6.mx = fmax(a6.mx, fabs((double)r[k]));
            }
        }
        t = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
        if (!grid_allreduce3<NT>(a6, D, g, phase, t)) return;
        ++phase;
        if (t.flag > 0.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, it, R_PCG_RESID); return; }
        fin = sqrt(t.c);
        mx = t.mx;
        rel = fin / init;
        const bool candidate = cg_converged(g.conv_test, rel, mx, g.rel_tol, g.abs_tol);
        if (candidate || t.c <= D.inner_tol * D.inner_tol * rr_last || it - last_fix >= RU_STALL) {
            // residual replacement from the FP64 coefficients and pressure
            Acc6 u1{0.0, 0.0, 0.0, 0.0, 0.0};
            true_residual(pn, u1);
            t = Acc6{0.0, 0.0, 0.0, 0.0, 0.0};
            if (!grid_allreduce3<NT>(u1, D, g, phase, t)) return;
            ++phase;
            ++outer;
            last_fix = it;
            if (t.flag > 0.0) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 4, ST_PCG, it, R_PCG_RESID); return; }
            fin = sqrt(t.c);
            mx = t.mx;
            rel = fin / init;
            // no progress of the true residual since the last correction:
            // the FP32 recurrences have lost the Krylov relations, restart
            const bool restart = t.c >= rr_last;
            rr_last = t.c;
            if (cg_converged(g.conv_test, rel, mx, g.rel_tol, g.abs_tol)) { conv = 1; break; }
            Acc8 u2{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            refresh_ws(pn, restart, u2);
            t8 = Acc8{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            if (!grid_allreduce5<NT>(u2, D, g, phase, t8)) return;
            ++phase;
            const double gn = t8.a;
            if (gn <= 1.0e-300 || !isfinite(gn)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_RZ); return; }
            // next direction z + beta p with its curvature computed, not recurred
            beta = restart ? 0.0 : gn / gam;
            den = t8.b + beta * (t8.c + t8.d) + beta * beta * t8.e;
            gam = gn;
            continue;
        }
        const double gn = t.a;
        if (gn <= 1.0e-300 || !isfinite(gn)) { if (b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 3, ST_PCG, it, R_PCG_RZ); return; }
        beta = gn / gam;
        den = t.b - beta * gn / alpha;
        gam = gn;
    }
    if (it > g.max_iter) it = g.max_iter;
    cg_finish(D, g, it, conv, init, fin, rel, mx);
    if (b == 0 && threadIdx.x == 0) seg_out(D, g)->outer = outer;
    if (!conv && b == 0 && threadIdx.x == 0) set_status(seg_status(D, g), 2, ST_PCG, it, R_PCG_MAXIT);
}

// ------------------------------------------------- two-level set-up kernels
// Aggregated operator P^T A P of the free rows: one CTA per nonzero (I, J)
// block; thread t sums entries t, t+T, ... (coefficient slots, or the
// diagonal of row -e-1), then warps and the CTA reduce in a fixed order.
// The diagonal is read by row position, or through row_node when that is
// given (the node-ordered diagonal: the same values on free rows).
__global__ void __launch_bounds__(256) k_coarse_blocks(const int* pair_ptr, const int2* pair_ij, const int* ent,
                                                       const double* val, const double* pdiag, const int* row_node,
                                                       int G, double* ac)
{
    __shared__ double sm[8];
    const int q = blockIdx.x;
    double s = 0.0;
    for (int k = pair_ptr[q] + threadIdx.x; k < pair_ptr[q + 1]; k += 256) {
        const int e = ent[k];
        s += e >= 0 ? val[e] : pdiag[row_node ? row_node[-e - 1] : -e - 1];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sm[w];
        ac[(size_t)pair_ij[q].x * G + pair_ij[q].y] = t;
    }
}

// In-place Gauss-Jordan inverse of the SPD coarse operator in shared memory
// (one CTA; warps take rows, lanes columns).  An aggregate without free rows
// has an empty row and column; it gets a unit diagonal and stays decoupled.
__global__ void __launch_bounds__(512) k_coarse_invert(int G, double* ac)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* a = reinterpret_cast<double*>(smem_raw);
    double* rowk = a + (size_t)G * G;
    double* colk = rowk + G;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int t = threadIdx.x; t < G * G; t += blockDim.x) a[t] = ac[t];
    __syncthreads();
    for (int t = threadIdx.x; t < G; t += blockDim.x)
        if (a[(size_t)t * G + t] == 0.0) a[(size_t)t * G + t] = 1.0;
    for (int k = 0; k < G; ++k) {
        __syncthreads();
        const double pinv = 1.0 / a[(size_t)k * G + k];
        for (int t = threadIdx.x; t < G; t += blockDim.x) {
            rowk[t] = a[(size_t)k * G + t] * pinv;   // new row k (its pivot entry fixed below)
            colk[t] = a[(size_t)t * G + k];
        }
        __syncthreads();
        for (int i = warp; i < G; i += nw) {
            double* ai = a + (size_t)i * G;
            if (i == k) {
                for (int j = lane; j < G; j += 32) ai[j] = (j == k) ? pinv : rowk[j];
            } else {
                const double ci = colk[i];
                for (int j = lane; j < G; j += 32) ai[j] = (j == k) ? -ci * pinv : fma(-ci, rowk[j], ai[j]);
            }
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G * G; t += blockDim.x) ac[t] = a[t];
}

// The same Gauss-Jordan inverse with the matrix held in registers: thread
// (ty = warp, tx = lane) of 16 x 32 owns rows ty + 16a (a < 10) and columns
// tx + 32b (b < 5), so G <= 160.  Step k reads the old pivot row and column
// from shared memory; the owners of row and column k+1 publish their new
// values into the other half of a double buffer, so one barrier per pivot
// suffices.  Every entry goes through the operations of k_coarse_invert in
// the same order, so both give the same bits.
constexpr int CINV_RA = 10, CINV_CB = 5, CINV_MAX = 160;
__global__ void __launch_bounds__(512, 1) k_coarse_invert_reg(int G, double* ac)
{
    __shared__ double srow[2][CINV_MAX], scol[2][CINV_MAX];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double v[CINV_RA][CINV_CB];
#pragma unroll
    for (int a = 0; a < CINV_RA; ++a)
#pragma unroll
        for (int b = 0; b < CINV_CB; ++b) {
            const int i = ty + 16 * a, j = tx + 32 * b;
            double x = (i < G && j < G) ? ac[(size_t)i * G + j] : 0.0;
            if (i == j && i < G && x == 0.0) x = 1.0;
            v[a][b] = x;
        }
    for (int t = threadIdx.x; t < 2 * CINV_MAX; t += blockDim.x) {
        (&srow[0][0])[t] = 0.0;
        (&scol[0][0])[t] = 0.0;
    }
    __syncthreads();
    if (ty == 0)
#pragma unroll
        for (int b = 0; b < CINV_CB; ++b) srow[0][tx + 32 * b] = v[0][b];
    if (tx == 0)
#pragma unroll
        for (int a = 0; a < CINV_RA; ++a) scol[0][ty + 16 * a] = v[a][0];
    for (int k = 0; k < G; ++k) {
        __syncthreads();
        const int cur = k & 1, nxt = cur ^ 1;
        const double pinv = 1.0 / srow[cur][k];
        double rk[CINV_CB];
#pragma unroll
        for (int b = 0; b < CINV_CB; ++b) rk[b] = srow[cur][tx + 32 * b] * pinv;
        // elimination, with column k and row k selected in place
#pragma unroll
        for (int a = 0; a < CINV_RA; ++a) {
            const int i = ty + 16 * a;
            const double ci = scol[cur][i];
            const double cneg = -ci * pinv;
#pragma unroll
            for (int b = 0; b < CINV_CB; ++b) {
                const int j = tx + 32 * b;
                const double t = fma(-ci, rk[b], v[a][b]);
                v[a][b] = (i == k) ? ((j == k) ? pinv : rk[b]) : ((j == k) ? cneg : t);
            }
        }
        const int k1 = k + 1;
        if (k1 < G) {
            if ((k1 & 15) == ty)
#pragma unroll
                for (int a = 0; a < CINV_RA; ++a)
                    if (ty + 16 * a == k1)
#pragma unroll
                        for (int b = 0; b < CINV_CB; ++b) srow[nxt][tx + 32 * b] = v[a][b];
            if ((k1 & 31) == tx)
#pragma unroll
                for (int b = 0; b < CINV_CB; ++b)
                    if (tx + 32 * b == k1)
#pragma unroll
                        for (int a = 0; a < CINV_RA; ++a) scol[nxt][ty + 16 * a] = v[a][b];
        }
    }
#pragma unroll
    for (int a = 0; a < CINV_RA; ++a)
#pragma unroll
        for (int b = 0; b < CINV_CB; ++b) {
            const int i = ty + 16 * a, j = tx + 32 * b;
            if (i < G && j < G) ac[(size_t)i * G + j] = v[a][b];
        }
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

namespace {
// Back-to-back grid all-reduces of the single-reduction kernel's kind (five
// values per CTA, 512-thread CTAs, one per SM), each depending on the last.
__global__ void __launch_bounds__(512, 1) k_allreduce_probe(PcgDev D, int iters, double* out)
{
    const SegView g = seg_view<false>(D);
    Acc6 t{0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < iters; ++i) {
        Acc6 v{1.0 + t.a * 1.0e-300, (double)blockIdx.x, 0.0, 0.0, (double)threadIdx.x};
        if (!grid_allreduce3<512>(v, D, g, i, t)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = t.a;
}
}  // namespace

cbs3d_status allreduce_probe(int device, int iters, double* us)
{
    if (iters < 1 || !us) return CBS3D_INVALID_INPUT;
    CUDA_OK(cudaSetDevice(device));
    int sms = 0;
    CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    int per = 0;
    CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_allreduce_probe, 512, 0));
    if (per < 1) return CBS3D_CUDA_ERROR;
    PcgDev D{};
    D.nslices = sms;
    D.part = dalloc<double>(static_cast<size_t>(sms) * 16);
    D.bar = dalloc<unsigned>(4);
    D.status = dalloc<DevStatus>(1);
    double* out = dalloc<double>(1);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cbs3d_status rc = CBS3D_OK;
    float ms = 0.0f;
    CUDA_OK(cudaEventCreate(&e0));
    CUDA_OK(cudaEventCreate(&e1));
    for (int rep = 0; rep < 2 && rc == CBS3D_OK; ++rep) {   // the first launch warms up
        CUDA_OK(cudaMemset(D.bar, 0, 4 * sizeof(unsigned)));
        CUDA_OK(cudaMemset(D.status, 0, sizeof(DevStatus)));
        void* args[] = {&D, &iters, &out};
        CUDA_OK(cudaEventRecord(e0));
        CUDA_OK(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_allreduce_probe), dim3(sms), dim3(512),
                                            args, 0, nullptr));
        CUDA_OK(cudaEventRecord(e1));
        CUDA_OK(cudaEventSynchronize(e1));
        CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
        DevStatus h{};
        CUDA_OK(cudaMemcpy(&h, D.status, sizeof h, cudaMemcpyDeviceToHost));
        if (h.code != 0) rc = static_cast<cbs3d_status>(h.code);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(D.part);
    cudaFree(D.bar);
    cudaFree(D.status);
    cudaFree(out);
    if (rc == CBS3D_OK) *us = 1.0e3 * ms / iters;
    return rc;
}

cbs3d_status coarse_inverse(int device, int g, const double* a, double* ainv, int variant)
{
    if (!a || !ainv || g < 1 || (variant != 0 && variant != 1) || g > (variant == 0 ? CINV_MAX : 164))
        return CBS3D_INVALID_INPUT;
    CUDA_OK(cudaSetDevice(device));
    const size_t bytes = static_cast<size_t>(g) * g * sizeof(double);
    double* d = dalloc<double>(static_cast<size_t>(g) * g);
    cudaError_t e = cudaMemcpy(d, a, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        if (variant == 0) {
            k_coarse_invert_reg<<<1, 512>>>(g, d);
        } else {
            const size_t ismem = (static_cast<size_t>(g) * g + 2 * static_cast<size_t>(g)) * 8;
            e = raise_smem_limit(reinterpret_cast<const void*>(k_coarse_invert), ismem);
            if (e == cudaSuccess) k_coarse_invert<<<1, 512, ismem>>>(g, d);
        }
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(ainv, d, bytes, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    CUDA_OK(e);
    return CBS3D_OK;
}

// ============================================================ PcgEngine
namespace {

// Placement of one CTA's halo in shared memory.  A warp's neighbour gather
// reads 32 doubles of the halo per slot (one per row of the slice); a double
// at halo position h sits in the bank pair h mod 16, and two lanes of a half
// warp whose values share a bank pair without sharing the value cost an
// extra shared-memory wavefront.  The order of the halo changes no value and
// no sum, so within every aligned block of 32 positions the block's entries
// (32 consecutive columns) are placed greedily: entries that occur in the
// most half-warp gathers first, each at the free position of the block
// whose bank pair has the fewest entries already placed in those gathers
// (weighted quadratically).  A block keeps its 32 entries, so the staging
// loads of each warp touch the same L2 sectors as in column order (a global
// bank placement spread them over 2.5x the sectors and made the 64^3
// iteration 17% slower).  64^3 jittered cavity, 148 CTAs: half-warp
// wavefronts of the gathers 666,745 -> 485,378 per iteration (ideal
// 391,104).  lc: the slots' halo indices (column order) of slices
// sb..se-1, offset by a0; returns pos, the position of each entry.
void bank_spread_halo(int nh, const unsigned short* lc, const long long* slice_off, const int* slice_w, int sb,
                      int se, long long a0, std::vector<int>& pos)
{
    std::vector<std::vector<int>> in_grp(static_cast<size_t>(nh));
    int ng = 0;
    for (int s = sb; s < se; ++s)
        for (int u = 0; u < slice_w[s]; ++u)
            for (int hw = 0; hw < 2; ++hw, ++ng)
                for (int l = 16 * hw; l < 16 * hw + 16; ++l) {
                    auto& v = in_grp[lc[slice_off[s] - a0 + 32 * u + l]];
                    if (v.empty() || v.back() != ng) v.push_back(ng);
                }
    std::vector<unsigned char> cnt(static_cast<size_t>(ng) * 16, 0);
    pos.assign(static_cast<size_t>(nh), 0);
    for (int b0 = 0; b0 < nh; b0 += 32) {
        const int b1 = std::min(nh, b0 + 32);
        int order[32];
        bool used[32] = {};
        for (int e = b0; e < b1; ++e) order[e - b0] = e;
        std::stable_sort(order, order + (b1 - b0), [&](int x, int y) {
            return in_grp[static_cast<size_t>(x)].size() > in_grp[static_cast<size_t>(y)].size();
        });
        for (int i = 0; i < b1 - b0; ++i) {
            const int e = order[i];
            const auto& gs = in_grp[static_cast<size_t>(e)];
            int best = -1;
            long long bc = 0;
            for (int j = 0; j < b1 - b0; ++j) {
                if (used[j]) continue;
                const int bank = (b0 + j) & 15;
                long long c = 0;
                for (int q : gs) {
                    const long long k = cnt[static_cast<size_t>(q) * 16 + bank];
                    c += 4 * k * k + k;
                }
                if (best < 0 || c < bc) { bc = c; best = j; }
            }
            used[best] = true;
            pos[static_cast<size_t>(e)] = b0 + best;
            const int bank = (b0 + best) & 15;
            for (int q : gs) {
                unsigned char& k = cnt[static_cast<size_t>(q) * 16 + bank];
                if (k < 255) ++k;
            }
        }
    }
}

// Shared-memory wavefronts of the neighbour gathers of slices sb..se-1 with
// the halo entries at `pos`: per slot and half warp, the largest number of
// distinct entries sharing a bank pair (at least one).
long long gather_wavefronts(const unsigned short* lc, const long long* slice_off, const int* slice_w, int sb, int se,
                            long long a0, const std::vector<int>& pos)
{
    long long w = 0;
    for (int s = sb; s < se; ++s)
        for (int u = 0; u < slice_w[s]; ++u)
            for (int hw = 0; hw < 2; ++hw) {
                int seen[16], nseen = 0, cnt[16] = {};
                for (int l = 16 * hw; l < 16 * hw + 16; ++l) {
                    const int p = pos[lc[slice_off[s] - a0 + 32 * u + l]];
                    bool dup = false;
                    for (int q = 0; q < nseen; ++q) dup = dup || seen[q] == p;
                    if (dup) continue;
                    seen[nseen++] = p;
                    ++cnt[p & 15];
                }
                int m = 1;
                for (int b = 0; b < 16; ++b) m = std::max(m, cnt[b]);
                w += m;
            }
    return w;
}

// Instantiations of the single-reduction kernels by rows per thread, batch
// mode and CTA size.
template <bool BATCH, int NT, int KS = 0>
const void* fn_cgcg(int rmax)
{
    return rmax == 1 ? reinterpret_cast<const void*>(k_pcg64c<1, BATCH, NT, KS>)
         : rmax == 2 ? reinterpret_cast<const void*>(k_pcg64c<2, BATCH, NT, KS>)
         : rmax == 4 ? reinterpret_cast<const void*>(k_pcg64c<4, BATCH, NT, KS>)
                     : reinterpret_cast<const void*>(k_pcg64c<8, BATCH, NT, KS>);
}
template <bool BATCH, int NT>
const void* fn_mixed(int rmax)
{
    return rmax == 1 ? reinterpret_cast<const void*>(k_pcg32m<1, BATCH, NT>)
         : rmax == 2 ? reinterpret_cast<const void*>(k_pcg32m<2, BATCH, NT>)
         : rmax == 4 ? reinterpret_cast<const void*>(k_pcg32m<4, BATCH, NT>)
                     : reinterpret_cast<const void*>(k_pcg32m<8, BATCH, NT>);
}
const void* fn_twolevel(int rmax)
{
    return rmax == 1 ? reinterpret_cast<const void*>(k_pcg64d<1>)
         : rmax == 2 ? reinterpret_cast<const void*>(k_pcg64d<2>)
         : rmax == 4 ? reinterpret_cast<const void*>(k_pcg64d<4>)
                     : reinterpret_cast<const void*>(k_pcg64d<8>);
}
// rows per thread read from tensor memory by the one-CTA-per-SM kernel with
// its first row in shared memory (0: that kernel has no such form)
int cgcg_tmem_rows(int rmax) { return rmax == 2 ? 1 : rmax == 4 ? 3 : rmax == 8 ? 4 : 0; }
const void* fn_cgcg_single(int rmax, int nt, int ks = 0, bool tmem = false)
{
    // every row of the thread in tensor memory (no shared-memory copy); at
    // eight rows the first four, the rest from L2
    if (!ks && tmem && nt == 512)
        return rmax == 2 ? reinterpret_cast<const void*>(k_pcg64c<2, false, 512, 0, 2>)
             : rmax == 4 ? reinterpret_cast<const void*>(k_pcg64c<4, false, 512, 0, 4>)
                         : reinterpret_cast<const void*>(k_pcg64c<8, false, 512, 0, 4>);
    if (ks && tmem && nt == 512) {
        return rmax == 2 ? reinterpret_cast<const void*>(k_pcg64c<2, false, 512, 1, 1>)
             : rmax == 4 ? reinterpret_cast<const void*>(k_pcg64c<4, false, 512, 1, 3>)
                         : reinterpret_cast<const void*>(k_pcg64c<8, false, 512, 1, 4>);
    }
    if (ks) return nt == 256 ? fn_cgcg<false, 256, 1>(rmax) : fn_cgcg<false, 512, 1>(rmax);
    return nt == 256 ? fn_cgcg<false, 256>(rmax) : fn_cgcg<false, 512>(rmax);
}
const void* fn_mixed_single(int rmax, int nt) { return nt == 256 ? fn_mixed<false, 256>(rmax) : fn_mixed<false, 512>(rmax); }

// The batch runs 256-thread CTAs, two per SM: its instances are small and
// many, and more, smaller CTAs spread them better.
constexpr int BATCH_THREADS = 256;

}  // namespace

void coarse_invert_launch(int g, double* a, cudaStream_t st)
{
    k_coarse_invert_reg<<<1, 512, 0, st>>>(g, a);
}

cudaError_t pcg_raise_smem_limit(const void* fn, size_t smem) { return raise_smem_limit(fn, smem); }

int PcgEngine::launches_per_solve() const
{
    if (mgh) return 4 + mgh->launches_per_setup();
    return coarse ? 6 : 4;
}

void PcgEngine::build_coarse(const HostModel& m, const std::vector<int>& colp)
{
    const int G = nblocks;
    const PressurePattern& P = m.pat;
    if (G > 160) return;   // the inverse must fit one CTA's shared memory
    std::vector<int> cta_of_slice(static_cast<size_t>(nslices), 0);
    for (int b = 0; b < G; ++b) {
        const int sb = static_cast<int>(static_cast<long long>(b) * nslices / G);
        const int se = static_cast<int>(static_cast<long long>(b + 1) * nslices / G);
        for (int q = sb; q < se; ++q) cta_of_slice[static_cast<size_t>(q)] = b;
    }
    std::vector<char> fixed(static_cast<size_t>(N), 0), freep(static_cast<size_t>(NP), 0);
    for (int v : m.bc_list) fixed[static_cast<size_t>(v - 1)] = 1;
    for (int pos = 0; pos < NP; ++pos) {
        const int node = P.row_node[static_cast<size_t>(pos)];
        freep[static_cast<size_t>(pos)] = node >= 0 && m.tf[static_cast<size_t>(node)] && !fixed[static_cast<size_t>(node)];
    }
    // entries of every nonzero block (I, J) of P^T A P, ascending
    std::vector<std::vector<int>> blocks(static_cast<size_t>(G) * G);
    for (int q = 0; q < nslices; ++q) {
        const int I = cta_of_slice[static_cast<size_t>(q)];
        for (int lane = 0; lane < 32; ++lane) {
            const int pos = q * 32 + lane;
            if (!freep[static_cast<size_t>(pos)]) continue;
            blocks[static_cast<size_t>(I) * G + I].push_back(-(pos + 1));
            for (int k = 0; k < P.slice_w[static_cast<size_t>(q)]; ++k) {
                const long long t = P.slice_off[static_cast<size_t>(q)] + lane + 32LL * k;
                const int c = colp[static_cast<size_t>(t)];
                if (!freep[static_cast<size_t>(c)]) continue;
                blocks[static_cast<size_t>(I) * G + cta_of_slice[static_cast<size_t>(c / 32)]].push_back(static_cast<int>(t));
            }
        }
    }
    std::vector<int> ptr(1, 0), ent;
    std::vector<int2> ij;
    for (int I = 0; I < G; ++I)
        for (int J = 0; J < G; ++J) {
            auto& v = blocks[static_cast<size_t>(I) * G + J];
            if (v.empty()) continue;
            std::sort(v.begin(), v.end());
            ent.insert(ent.end(), v.begin(), v.end());
            ptr.push_back(static_cast<int>(ent.size()));
            ij.push_back(make_int2(I, J));
        }
    // each CTA's neighbour list: itself and the owners of its halo entries
    std::vector<int> nptr(1, 0), nids;
    std::vector<unsigned char> hown(h_hidx.size(), 0);
    int nmax = 0;
    for (int b = 0; b < G; ++b) {
        std::vector<int> l(1, b);
        for (int k = h_hptr[static_cast<size_t>(b)]; k < h_hptr[static_cast<size_t>(b) + 1]; ++k)
            l.push_back(cta_of_slice[static_cast<size_t>(h_hidx[static_cast<size_t>(k)] / 32)]);
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
        if (l.size() > 255) return;
        for (int k = h_hptr[static_cast<size_t>(b)]; k < h_hptr[static_cast<size_t>(b) + 1]; ++k) {
            const int o = cta_of_slice[static_cast<size_t>(h_hidx[static_cast<size_t>(k)] / 32)];
            hown[static_cast<size_t>(k)] = static_cast<unsigned char>(std::lower_bound(l.begin(), l.end(), o) - l.begin());
        }
        nids.insert(nids.end(), l.begin(), l.end());
        nptr.push_back(static_cast<int>(nids.size()));
        nmax = std::max(nmax, static_cast<int>(l.size()));
    }
    const size_t base = (halo_smem + 15) & ~static_cast<size_t>(15);
    const size_t smem = base + (static_cast<size_t>(nmax) * G + 3 * static_cast<size_t>(G) + nmax) * 8 +
                        static_cast<size_t>(dev_halo_max) + 16;
    const size_t ismem = (static_cast<size_t>(G) * G + 2 * static_cast<size_t>(G)) * 8;
    const void* fn = fn_twolevel(rmax);
    int per = 0;
    if (smem > 220 * 1024 || ismem > 220 * 1024 || raise_smem_limit(fn, smem) != cudaSuccess ||
        raise_smem_limit(reinterpret_cast<const void*>(k_coarse_invert), ismem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, 512, smem) != cudaSuccess || per * sms_ < G) {
        cudaGetLastError();
        return;
    }
    npairs = static_cast<int>(ij.size());
    d_pair_ptr = dalloc<int>(ptr.size());
    d_pair_ij = dalloc<int2>(ij.size());
    d_pair_ent = dalloc<int>(ent.size());
    d_ac = dalloc<double>(static_cast<size_t>(G) * G);
    d_nbr_ptr = dalloc<int>(nptr.size());
    d_nbr_ids = dalloc<int>(nids.size());
    d_hown = dalloc<unsigned char>(hown.size());
    CUDA_OK(cudaMemcpy(d_pair_ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_pair_ij, ij.data(), ij.size() * sizeof(int2), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_pair_ent, ent.data(), ent.size() * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_nbr_ptr, nptr.data(), nptr.size() * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_nbr_ids, nids.data(), nids.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!hown.empty()) CUDA_OK(cudaMemcpy(d_hown, hown.data(), hown.size(), cudaMemcpyHostToDevice));
    cdev = CoarseDev{G, nmax, d_nbr_ptr, d_nbr_ids, d_hown, d_ac};
    coarse_smem = smem;
    coarse_ismem = ismem;
    coarse = true;
}

void PcgEngine::init(const HostModel& m, const uint8_t* nflag, const double* pfix, DevStatus* status,
                     int device, int blocks_override, bool mixed_mode, int kernel_choice, bool two_level,
                     bool multigrid)
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
    NP = nslices * 32;
    d_row_node = dalloc<int>(P.row_node.size());
    CUDA_OK(cudaMemcpy(d_row_node, P.row_node.data(), P.row_node.size() * sizeof(int), cudaMemcpyHostToDevice));
    // columns as row positions: the solver works in row-position order
    std::vector<int> pos_of(static_cast<size_t>(N), 0);
    for (size_t p = 0; p < P.row_node.size(); ++p)
        if (P.row_node[p] >= 0) pos_of[static_cast<size_t>(P.row_node[p])] = static_cast<int>(p);
    std::vector<int> colp(static_cast<size_t>(nslots));
    for (size_t t = 0; t < colp.size(); ++t) colp[t] = pos_of[static_cast<size_t>(P.col[t])];
    d_slice_off = dalloc<long long>(P.slice_off.size());
    d_slice_w = dalloc<int>(P.slice_w.size());
    d_col = dalloc<int>(static_cast<size_t>(nslots));
    d_cptr = dalloc<long long>(P.cptr.size());
    d_cent = dalloc<int>(static_cast<size_t>(ncontrib));
    d_val = dalloc<double>(static_cast<size_t>(nslots));
    CUDA_OK(cudaMemcpy(d_slice_off, P.slice_off.data(), P.slice_off.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_slice_w, P.slice_w.data(), P.slice_w.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (nslots) CUDA_OK(cudaMemcpy(d_col, colp.data(), static_cast<size_t>(nslots) * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_cptr, P.cptr.data(), P.cptr.size() * sizeof(long long), cudaMemcpyHostToDevice));
    if (ncontrib) CUDA_OK(cudaMemcpy(d_cent, P.cent.data(), static_cast<size_t>(ncontrib) * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemset(d_val, 0, static_cast<size_t>(nslots ? nslots : 1) * sizeof(double)));
    const size_t n = static_cast<size_t>(NP);
    d_r = dalloc<double>(2 * n); d_z = dalloc<double>(n); d_pA = dalloc<double>(n);
    d_pB = dalloc<double>(n); d_q = dalloc<double>(2 * n);
    d_xp = dalloc<double>(n); d_bp = dalloc<double>(n); d_dp = dalloc<double>(n);
    d_fp = dalloc<uint8_t>(n);
    CUDA_OK(cudaMemset(d_pB, 0, n * sizeof(double)));
    if (mixed) {
        d_val32 = dalloc<float>(static_cast<size_t>(nslots));
        d_f32 = dalloc<float>(8 * n);
        CUDA_OK(cudaMemset(d_f32, 0, 8 * n * sizeof(float)));
    }
    d_nflag = nflag;
    d_pfix = pfix;
    d_status = status;

    int sms = 0;
    CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    sms_ = sms;
    // Register-resident kernel when every thread's rows fit its register
    // arrays; otherwise the kernel that keeps the vectors in global memory.
    auto grid_for = [&](const void* fn) {
        int per_sm = 0;
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PCG_THREADS, 0));
        int g = sms * (per_sm < 2 ? per_sm : 2);
        if (blocks_override > 0 && blocks_override < g) g = blocks_override;
        if (g > nslices) g = nslices > 0 ? nslices : 1;
        return g;
    };
    rmax = 0;
    variant = 1;
    nblocks = grid_for(reinterpret_cast<const void*>(k_pcg64<false>));
    const int rm[4] = {1, 2, 4, 8};
    if (kernel_choice == 0 || kernel_choice == 3 || kernel_choice == 4 || kernel_choice == 10 || kernel_choice == 11) {
        const void* hc3[4] = {reinterpret_cast<const void*>(k_pcg64h<1>), reinterpret_cast<const void*>(k_pcg64h<2>),
                              reinterpret_cast<const void*>(k_pcg64h<4>), reinterpret_cast<const void*>(k_pcg64h<8>)};
        const int want = kernel_choice == 3 ? 3 : 4;
        // CTA size of the single-reduction kernel: one 512-thread CTA per SM
        // once every warp of such a grid has rows (fewer partials per
        // all-reduce), two 256-thread CTAs per SM below that
        const int nt = (want == 4 && nslices < 16 * sms) ? 256 : 512;
        const int nwarps = nt / 32;
        for (int c = 0; c < 4 && variant == 1; ++c) {
            const void* fn = want == 4 ? fn_cgcg_single(rm[c], nt) : hc3[c];
            int per_sm = 0;
            CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, nt, 0));
            int g = sms * (per_sm < 2 ? per_sm : 2);
            if (blocks_override > 0 && blocks_override < g) g = blocks_override;
            if (g > nslices) g = nslices > 0 ? nslices : 1;
            const int per_cta = (nslices + g - 1) / g;
            if ((per_cta + nwarps - 1) / nwarps > rm[c]) continue;
            // halo of every CTA: distinct columns of its slot range
            std::vector<int> hptr(static_cast<size_t>(g) + 1, 0), hidx;
            std::vector<unsigned short> lcol(static_cast<size_t>(nslots), 0);
            int hmax = 0;
            long long smax = 0;
            bool fits = true;
            std::vector<int> cols, hpos, hcols;
            for (int bb = 0; bb < g && fits; ++bb) {
                const int sb = static_cast<int>(static_cast<long long>(bb) * nslices / g);
                const int se = static_cast<int>(static_cast<long long>(bb + 1) * nslices / g);
                const long long a0 = P.slice_off[static_cast<size_t>(sb)], a1 = P.slice_off[static_cast<size_t>(se)];
                cols.assign(colp.begin() + a0, colp.begin() + a1);
                std::sort(cols.begin(), cols.end());
                cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
                if (cols.size() > 65535) { fits = false; break; }
                for (long long t = a0; t < a1; ++t)
                    lcol[static_cast<size_t>(t)] = static_cast<unsigned short>(
                        std::lower_bound(cols.begin(), cols.end(), colp[static_cast<size_t>(t)]) - cols.begin());
                // the halo's order in shared memory: bank-spread
                const int nh = static_cast<int>(cols.size());
                bank_spread_halo(nh, lcol.data() + a0, P.slice_off.data(), P.slice_w.data(), sb, se, a0, hpos);
                for (long long t = a0; t < a1; ++t)
                    lcol[static_cast<size_t>(t)] = static_cast<unsigned short>(hpos[lcol[static_cast<size_t>(t)]]);
                hcols.resize(cols.size());
                for (int e = 0; e < nh; ++e) hcols[static_cast<size_t>(hpos[static_cast<size_t>(e)])] = cols[static_cast<size_t>(e)];
                hidx.insert(hidx.end(), hcols.begin(), hcols.end());
                hptr[static_cast<size_t>(bb) + 1] = static_cast<int>(hidx.size());
                hmax = std::max(hmax, static_cast<int>(cols.size()));
                smax = std::max(smax, a1 - a0);
            }
            if (!fits) continue;
            const size_t smem = static_cast<size_t>(hmax) * (want == 4 ? 20 : 12) + static_cast<size_t>(smax) * 2 + 16;
            if (smem > 200 * 1024) continue;
            CUDA_OK(raise_smem_limit(fn, smem));
            CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, nt, smem));
            if (per_sm * sms < g) continue;
            variant = want;
            nthreads = nt;
            rmax = rm[c];
            nblocks = g;
            halo_smem = smem;
            // the CG-CG kernel's own rows (pressure, diagonal) in shared
            // memory: measured faster for the two-CTAs-per-SM kernel of small
            // meshes (5.2 instead of 5.4 us per iteration at 16^3) and slower
            // for the one-CTA kernel of large ones (13.4 instead of 13.1 us at
            // 64^3, where those rows already hit in L1 and a larger shared-
            // memory carve-out leaves less L1 for the rest)
            cgcg_smem = smem;
            cgcg_xs_off = 0;
            if (want == 4 && nt == 256) {
                const size_t off = (smem + 15) & ~static_cast<size_t>(15);
                const size_t with = off + static_cast<size_t>(rm[c]) * nt * 16;
                int per2 = 0;
                if (with <= 227 * 1024 && raise_smem_limit(fn, with) == cudaSuccess &&
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, fn, nt, with) == cudaSuccess &&
                    per2 * sms >= g) {
                    cgcg_smem = with;
                    cgcg_xs_off = static_cast<int>(off);
                }
                cudaGetLastError();
            }
            // the kernel that reads every warp's first row's coefficients
            // from shared memory, where the CTAs' first slices fit beside
            // the halo
            cgcg_ks = 0;
            cgcg_coef_off = 0;
            // tensor memory (one-CTA-per-SM kernel): 128 columns = 64 doubles
            // per thread, the slots of a row padded to the widest slice of
            // the mesh.  Where all the thread's rows fit, they all live there
            // and no coefficients are copied into shared memory; otherwise
            // the rows after the shared-memory one that fit.
            cgcg_kt = 0;
            cgcg_tm_w = 0;
            int tm_tw = 0;
            if (want == 4 && nt == 512 && kernel_choice != 10) {
                int wmx = 0;
                for (int q = 0; q < nslices; ++q) wmx = std::max(wmx, P.slice_w[static_cast<size_t>(q)]);
                const int chw = rm[c] >= 4 ? 2 : 8;
                tm_tw = (wmx + chw - 1) / chw * chw;
                if (kernel_choice != 11 && (rm[c] == 2 || rm[c] == 4) && tm_tw > 0 && rm[c] * tm_tw <= 64) {
                    cgcg_kt = rm[c];
                    cgcg_tm_w = tm_tw;
                }
            }
            if (want == 4 && cgcg_kt == 0) {
                long long cmax = 0;
                for (int bb = 0; bb < g; ++bb) {
                    const int sb = static_cast<int>(static_cast<long long>(bb) * nslices / g);
                    const int se = static_cast<int>(static_cast<long long>(bb + 1) * nslices / g);
                    const int sc = std::min(sb + nwarps, se);
                    cmax = std::max(cmax, P.slice_off[static_cast<size_t>(sc)] - P.slice_off[static_cast<size_t>(sb)]);
                }
                const long long per_need = (g + sms - 1) / sms;
                const long long cap = std::min<long long>(227 * 1024, 228 * 1024 / per_need - 1024);
                const size_t off = (cgcg_smem + 15) & ~static_cast<size_t>(15);
                const size_t with = off + static_cast<size_t>(cmax) * 8;
                const void* fk = fn_cgcg_single(rm[c], nt, 1);
                int per2 = 0;
                if (static_cast<long long>(with) <= cap && raise_smem_limit(fk, with) == cudaSuccess &&
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, fk, nt, with) == cudaSuccess &&
                    per2 * sms >= g) {
                    cgcg_ks = 1;
                    cgcg_smem = with;
                    cgcg_coef_off = static_cast<int>(off);
                }
                cudaGetLastError();
            }
            // the one-CTA-per-SM kernel with its first row in shared memory
            // keeps the coefficients of its next rows in the SM's tensor
            // memory for the solve: 128 columns (64 doubles) per thread, the
            // slots of a row padded to the widest slice of the mesh
            if (cgcg_ks && tm_tw > 0 && cgcg_tmem_rows(rm[c]) * tm_tw <= 64) {
                cgcg_kt = cgcg_tmem_rows(rm[c]);
                cgcg_tm_w = tm_tw;
            }
            // eight rows per thread where the shared-memory copy did not fit:
            // the first four rows in tensor memory
            if (!cgcg_ks && cgcg_kt == 0 && rm[c] == 8 && tm_tw > 0 && 4 * tm_tw <= 64) {
                cgcg_kt = 4;
                cgcg_tm_w = tm_tw;
            }
            // the one-CTA-per-SM kernel's rows' diagonal in shared memory
            // (64^3: 12.05 -> 11.95 us per iteration; in registers it was
            // slower)
            cgcg_pds_off = 0;
            if (want == 4 && nt == 512) {
                const size_t off = (cgcg_smem + 15) & ~static_cast<size_t>(15);
                const size_t with = off + static_cast<size_t>(rm[c]) * nt * 8;
                const void* fk = fn_cgcg_single(rm[c], nt, cgcg_ks, cgcg_kt > 0);
                int per2 = 0;
                if (with <= 227 * 1024 && raise_smem_limit(fk, with) == cudaSuccess &&
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, fk, nt, with) == cudaSuccess &&
                    per2 * sms >= g) {
                    cgcg_smem = with;
                    cgcg_pds_off = static_cast<int>(off);
                }
                cudaGetLastError();
            }
            if (cgcg_kt > 0) {
                // the tensor-memory kernel must hold the whole grid resident
                // with one CTA per SM: each CTA takes all 512 columns, so a
                // second CTA on the SM would wait for the first to finish
                const void* fk = fn_cgcg_single(rm[c], nt, cgcg_ks, true);
                int per2 = 0;
                if (g > sms || !(raise_smem_limit(fk, cgcg_smem) == cudaSuccess &&
                      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, fk, nt, cgcg_smem) == cudaSuccess &&
                      per2 * sms >= g)) {
                    cgcg_kt = 0;
                    cgcg_tm_w = 0;
                }
                cudaGetLastError();
            }
            d_halo_ptr = dalloc<int>(hptr.size());
            d_halo_idx = dalloc<int>(hidx.size());
            d_lcol = dalloc<unsigned short>(lcol.size());
            CUDA_OK(cudaMemcpy(d_halo_ptr, hptr.data(), hptr.size() * sizeof(int), cudaMemcpyHostToDevice));
            CUDA_OK(cudaMemcpy(d_halo_idx, hidx.data(), hidx.size() * sizeof(int), cudaMemcpyHostToDevice));
            if (!lcol.empty()) CUDA_OK(cudaMemcpy(d_lcol, lcol.data(), lcol.size() * sizeof(unsigned short), cudaMemcpyHostToDevice));
            dev_halo_max = hmax;
            dev_slot_max = static_cast<int>(smax);
            h_hptr = hptr;
            h_hidx = hidx;
            if (mixed && want == 4) {
                const void* mc[4] = {fn_mixed_single(1, nt), fn_mixed_single(2, nt), fn_mixed_single(4, nt),
                                     fn_mixed_single(8, nt)};
                const size_t ms = static_cast<size_t>(hmax) * 16 + static_cast<size_t>(smax) * 6 + 16;
                int per = 0;
                if (ms <= 220 * 1024 &&
                    raise_smem_limit(mc[c], ms) == cudaSuccess &&
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, mc[c], nt, ms) == cudaSuccess &&
                    per * sms >= g) {
                    mixed_ok = true;
                    mixed_smem = ms;
                }
                cudaGetLastError();
            }
        }
    }
    if (variant == 1 && kernel_choice != 1 && kernel_choice != 5) {
        const void* cands[4] = {reinterpret_cast<const void*>(k_pcg64r<1>), reinterpret_cast<const void*>(k_pcg64r<2>),
                                reinterpret_cast<const void*>(k_pcg64r<4>), reinterpret_cast<const void*>(k_pcg64r<8>)};
        for (int c = 0; c < 4; ++c) {
            const int g = grid_for(cands[c]);
            const int per_cta = (nslices + g - 1) / g;
            if ((per_cta + PCG_WARPS - 1) / PCG_WARPS <= rm[c]) { rmax = rm[c]; nblocks = g; variant = 2; break; }
        }
    }
    if (variant == 1 && N > 0) {
        // the global-vector kernel with its neighbour values staged in shared
        // memory: each CTA's slices in the fewest parts (at most 8) whose
        // halos fit
        const int g = nblocks;
        std::vector<int> hptr, hidx, cols;
        std::vector<unsigned short> lcol(static_cast<size_t>(nslots), 0);
        int hmax = 0;
        bool fits = false;
        for (int kp = 1; kp <= 8 && !fits; ++kp) {
            hptr.assign(static_cast<size_t>(g) * kp + 1, 0);
            hidx.clear();
            hmax = 0;
            fits = true;
            for (int bb = 0; bb < g && fits; ++bb) {
                const int sb = static_cast<int>(static_cast<long long>(bb) * nslices / g);
                const int se = static_cast<int>(static_cast<long long>(bb + 1) * nslices / g);
                for (int q = 0; q < kp && fits; ++q) {
                    const int pb = sb + static_cast<int>(static_cast<long long>(q) * (se - sb) / kp);
                    const int pe = sb + static_cast<int>(static_cast<long long>(q + 1) * (se - sb) / kp);
                    const long long a0 = P.slice_off[static_cast<size_t>(pb)], a1 = P.slice_off[static_cast<size_t>(pe)];
                    cols.assign(colp.begin() + a0, colp.begin() + a1);
                    std::sort(cols.begin(), cols.end());
                    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
                    if (cols.size() > 65535 || cols.size() * 16 + 16 > 220 * 1024) { fits = false; break; }
                    for (long long t = a0; t < a1; ++t)
                        lcol[static_cast<size_t>(t)] = static_cast<unsigned short>(
                            std::lower_bound(cols.begin(), cols.end(), colp[static_cast<size_t>(t)]) - cols.begin());
                    hidx.insert(hidx.end(), cols.begin(), cols.end());
                    hptr[static_cast<size_t>(bb) * kp + q + 1] = static_cast<int>(hidx.size());
                    hmax = std::max(hmax, static_cast<int>(cols.size()));
                }
            }
            if (fits) global_halo_parts = kp;
        }
        // automatic and choice 5: the single-reduction kernel; choice 1:
        // the two-reduction one (bitwise the same arithmetic as choices 2, 3)
        global_cgcg = kernel_choice != 1;
        const void* fh = global_cgcg ? reinterpret_cast<const void*>(k_pcg64g) : reinterpret_cast<const void*>(k_pcg64<true>);
        const size_t smem = static_cast<size_t>(hmax) * 16 + 16;
        int per = 0;
        if (fits && raise_smem_limit(fh, smem) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fh, PCG_THREADS, smem) == cudaSuccess && per * sms >= g) {
            d_halo_ptr = dalloc<int>(hptr.size());
            d_halo_idx = dalloc<int>(hidx.size());
            d_lcol = dalloc<unsigned short>(lcol.size());
            CUDA_OK(cudaMemcpy(d_halo_ptr, hptr.data(), hptr.size() * sizeof(int), cudaMemcpyHostToDevice));
            CUDA_OK(cudaMemcpy(d_halo_idx, hidx.data(), hidx.size() * sizeof(int), cudaMemcpyHostToDevice));
            CUDA_OK(cudaMemcpy(d_lcol, lcol.data(), lcol.size() * sizeof(unsigned short), cudaMemcpyHostToDevice));
            dev_halo_max = hmax;
            global_halo = true;
            global_halo_smem = smem;
            global_halo_total = static_cast<long long>(hidx.size());
        }
        cudaGetLastError();
    }
    if (two_level && variant == 4 && nthreads == 512 && !mixed_ok) build_coarse(m, colp);
    if (multigrid && !mixed && !coarse) {
        mgh = new MgHierarchy;
        bool ok = false;
        try {
            ok = mgh->build(m, colp, nflag, d_slice_off, d_slice_w, d_col, device, sms, blocks_override);
        } catch (...) {
            mgh->release();
            delete mgh;
            mgh = nullptr;
            throw;
        }
        if (!ok) {
            // the caller asked for multigrid: say why it runs Jacobi-PCG instead
            std::fprintf(stderr, "cbs3d: multigrid preconditioner unavailable for this mesh (%s); "
                                 "Jacobi-PCG is used\n", mgh->why.c_str());
            mgh->release();
            delete mgh;
            mgh = nullptr;
        }
    }
    d_part = dalloc<double>(static_cast<size_t>(nblocks) * 16);
    d_bar = dalloc<unsigned>(4);
    d_out = dalloc<CgOut>(1);
    CUDA_OK(cudaMemset(d_bar, 0, 4 * sizeof(unsigned)));

    dev = PcgDev{};
    dev.N = NP; dev.NN = N; dev.E = E; dev.nslices = nslices; dev.nblocks = nblocks;
    dev.slice_off = d_slice_off; dev.slice_w = d_slice_w; dev.col = d_col; dev.val = d_val;
    dev.val32 = d_val32; dev.cptr = d_cptr; dev.cent = d_cent;
    dev.nflag = d_nflag; dev.pfix = d_pfix;
    dev.r = d_r; dev.z = d_z; dev.pA = d_pA; dev.pB = d_pB; dev.q = d_q;
    if (mixed) {
        dev.r32 = d_f32; dev.w32 = d_f32 + 2 * n; dev.s32 = d_f32 + 4 * n;
        dev.p32 = d_f32 + 6 * n; dev.dz32 = d_f32 + 7 * n;
    }
    dev.slot_max = dev_slot_max;
    dev.part = d_part; dev.bar = d_bar; dev.status = d_status; dev.out = d_out;
    dev.halo_ptr = d_halo_ptr; dev.halo_idx = d_halo_idx; dev.lcol = d_lcol; dev.halo_max = dev_halo_max;
    dev.xs_off = cgcg_xs_off;
    dev.coef_off = cgcg_coef_off;
    dev.pds_off = cgcg_pds_off;
    dev.tm_w = cgcg_tm_w;
    dev.halo_parts = global_halo ? global_halo_parts : 0;
    dev.row_node = d_row_node;
}

void PcgEngine::release()
{
    if (mgh) {
        mgh->release();
        delete mgh;
        mgh = nullptr;
    }
    mg_ready = false;
    void* ptrs[] = {d_slice_off, d_slice_w, d_col, d_cptr, d_cent, d_val, d_val32, d_r, d_z, d_pA,
                    d_pB, d_q, d_f32, d_part, d_bar, d_out, d_halo_ptr, d_halo_idx, d_lcol, d_row_node,
                    d_xp, d_bp, d_dp, d_fp, d_pair_ptr, d_pair_ij, d_pair_ent, d_ac, d_nbr_ptr, d_nbr_ids, d_hown};
    for (void* p : ptrs) if (p) cudaFree(p);
    d_pair_ptr = nullptr; d_pair_ij = nullptr; d_pair_ent = nullptr; d_ac = nullptr;
    d_nbr_ptr = nullptr; d_nbr_ids = nullptr; d_hown = nullptr;
    coarse = false;
    d_slice_off = nullptr; d_slice_w = nullptr; d_col = nullptr; d_cptr = nullptr; d_cent = nullptr;
    d_val = nullptr; d_val32 = nullptr; d_r = d_z = d_pA = d_pB = d_q = nullptr; d_f32 = nullptr;
    d_part = nullptr; d_bar = nullptr; d_out = nullptr;
    d_halo_ptr = nullptr; d_halo_idx = nullptr; d_lcol = nullptr; d_row_node = nullptr;
    d_xp = d_bp = d_dp = nullptr; d_fp = nullptr;
}

void PcgEngine::coarse_setup(const double* pdiag, const int* row_node, cudaStream_t st)
{
    const int G = nblocks;
    CUDA_OK(cudaMemsetAsync(d_ac, 0, static_cast<size_t>(G) * G * sizeof(double), st));
    k_coarse_blocks<<<static_cast<unsigned>(npairs), 256, 0, st>>>(d_pair_ptr, d_pair_ij, d_pair_ent, d_val, pdiag,
                                                                  row_node, G, d_ac);
    if (G <= CINV_MAX)
        k_coarse_invert_reg<<<1, 512, 0, st>>>(G, d_ac);
    else
        k_coarse_invert<<<1, 512, coarse_ismem, st>>>(G, d_ac);
}

void PcgEngine::prepare_coarse(const double* d_pdiag_node, cudaStream_t st)
{
    if (mgh) {
        mgh->setup(d_val, d_pdiag_node, d_row_node, st);
        mg_ready = true;
        return;
    }
    if (!coarse) return;
    coarse_setup(d_pdiag_node, d_row_node, st);
    coarse_ready = true;
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
    k_ell_multiply<<<(nslices * 32 + 255) / 256, 256, 0, st>>>(D, x, y);
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
    k_perm_in<<<(NP + 255) / 256, 256, 0, st>>>(D, pres, rhs1, pdiag, D.nflag, d_xp, d_bp, d_dp, d_fp);
    D.pres = d_xp; D.rhs1 = d_bp; D.pdiag = d_dp; D.nflag = d_fp;
    CUDA_OK(cudaMemsetAsync(d_bar, 0, 4 * sizeof(unsigned), st));
    CUDA_OK(cudaMemsetAsync(d_out, 0, sizeof(CgOut), st));
    void* args[] = {&D};
    const void* fn = !global_halo ? reinterpret_cast<const void*>(k_pcg64<false>)
                     : global_cgcg ? reinterpret_cast<const void*>(k_pcg64g)
                                   : reinterpret_cast<const void*>(k_pcg64<true>);
    size_t smem = global_halo ? global_halo_smem : 0;
    if (variant == 2) {
        if (rmax == 1) fn = reinterpret_cast<const void*>(k_pcg64r<1>);
        else if (rmax == 2) fn = reinterpret_cast<const void*>(k_pcg64r<2>);
        else if (rmax == 4) fn = reinterpret_cast<const void*>(k_pcg64r<4>);
        else fn = reinterpret_cast<const void*>(k_pcg64r<8>);
    } else if (variant == 3) {
        if (rmax == 1) fn = reinterpret_cast<const void*>(k_pcg64h<1>);
        else if (rmax == 2) fn = reinterpret_cast<const void*>(k_pcg64h<2>);
        else if (rmax == 4) fn = reinterpret_cast<const void*>(k_pcg64h<4>);
        else fn = reinterpret_cast<const void*>(k_pcg64h<8>);
        smem = halo_smem;
    } else if (variant == 4 && mixed_ok) {
        fn = fn_mixed_single(rmax, nthreads);
        smem = mixed_smem;
    } else if (variant == 4) {
        fn = fn_cgcg_single(rmax, nthreads, cgcg_ks, cgcg_kt > 0);
        smem = cgcg_smem;
    }
    CoarseDev C = cdev;
    void* args2[] = {&D, &C};
    if (coarse) {
        // the aggregated operator of this solve and its inverse, unless
        // prepare_coarse made them already
        if (!coarse_ready) coarse_setup(d_dp, nullptr, st);
        coarse_ready = false;
        fn = fn_twolevel(rmax);
        smem = coarse_smem;
    }
    if (mgh && precond == 1) {
        // the multigrid set-up of this solve, unless prepare_coarse made it
        if (!mg_ready) mgh->setup(d_val, d_dp, nullptr, st);
        mg_ready = false;
        if (ev0) CUDA_OK(cudaEventRecord(ev0, st));
        mgh->launch(D, st);
        if (ev1) CUDA_OK(cudaEventRecord(ev1, st));
    } else {
        mg_ready = false;
        if (ev0) CUDA_OK(cudaEventRecord(ev0, st));
        CUDA_OK(cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(nthreads), coarse ? args2 : args, smem, st));
        if (ev1) CUDA_OK(cudaEventRecord(ev1, st));
    }
    k_perm_out<<<(NP + 255) / 256, 256, 0, st>>>(D, d_xp, pres);
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
    if (mgh) {
        // level 0: three products (pre-smoothing residual, post-smoothing,
        // A p) over the coefficients; per node the pressure read and written,
        // z and q written and read back, the smoothed residual written and
        // read by the restriction; coarse levels: two products each
        size_t b = static_cast<size_t>(nnz_offdiag) * 24 + static_cast<size_t>(N) * 64;
        for (int l = 1; l < mgh->Lc; ++l)
            b += static_cast<size_t>(mgh->n[static_cast<size_t>(l)]) * (16 * mgh->W[static_cast<size_t>(l)] + 48);
        return b;
    }
    if (variant == 4 && mixed_ok) {
        // coefficients resident in shared memory; per node: r, w, s of the
        // previous iteration read once for staging (12), r, s, w written (12),
        // pressure read and written (16), pdiag read (8)
        return static_cast<size_t>(N) * 48;
    }
    if (variant == 4) {
        // coefficient per pair entry; per node: r, w, s of the previous
        // iteration read once for staging (24), r, s, w written (24), pressure
        // read and written (16), pdiag read (8)
        return static_cast<size_t>(nnz_offdiag) * 8 + static_cast<size_t>(N) * 72;
    }
    if (variant == 3) {
        // coefficient per pair entry; per node: halo staging of z and the
        // previous direction (each node is in about one CTA's halo per owner
        // plus the overlap, counted once here), z read back, new direction and
        // z written, pressure read and written
        return static_cast<size_t>(nnz_offdiag) * 8 + static_cast<size_t>(N) * 56;
    }
    if (rmax > 0) {
        // coefficient + column per pair entry; per node the z and previous
        // direction gathered once, z read back, new direction and z written,
        // pressure read and written
        return static_cast<size_t>(nnz_offdiag) * 12 + static_cast<size_t>(N) * 56;
    }
    // Phase A: coefficient + column per pair entry; z and previous p of the
    // row (16 B), pdiag (8), new p written (8), q written (8), node flag (1).
    // Phase B: q, r, pres, pdiag read (32), r, pres, z written (24).  With the
    // shared-memory halo the columns are 16-bit and every halo entry's z and
    // previous p are read once per iteration.
    if (global_halo && global_cgcg) {
        // single reduction: coefficient + 16-bit column per pair entry; per
        // node r, s, w of the previous iteration, p, pressure, inverse
        // diagonal and diagonal read (56), node flag (1), p, pressure and the
        // new r, s, w written (40); per halo entry r, s, w (24) and, with
        // several parts per CTA, the inverse diagonal (8)
        return static_cast<size_t>(nnz_offdiag) * 10 + static_cast<size_t>(N) * 97 +
               static_cast<size_t>(global_halo_total) * (global_halo_parts > 1 ? 32 : 24);
    }
    if (global_halo)
        return static_cast<size_t>(nnz_offdiag) * 10 + static_cast<size_t>(N) * 97 +
               static_cast<size_t>(global_halo_total) * 16;
    return static_cast<size_t>(nnz_offdiag) * 12 + static_cast<size_t>(N) * 97;
}

// ================================================================ batch
void PcgBatch::init(const std::vector<PcgBatchMember>& members, int dev_id, bool mixed_mode, double inner_tol)
{
    mem = members;
    device = dev_id;
    mixed = mixed_mode;
    const size_t K = mem.size();
    CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    gmax = 2 * sms;   // two BATCH_THREADS CTAs per SM
    slice0.assign(K, 0); nsl.assign(K, 0); N_k.assign(K, 0);
    slot0.assign(K, 0); nslot.assign(K, 0);
    nslices = 0; nslots = 0;
    for (size_t k = 0; k < K; ++k) {
        const PressurePattern& P = mem[k].m->pat;
        slice0[k] = nslices; nsl[k] = P.nslices; N_k[k] = mem[k].m->N;
        slot0[k] = nslots; nslot[k] = P.nslots;
        nslices += P.nslices;
        nslots += P.nslots;
    }
    NP = nslices * 32;
    // concatenated pattern: global slot offsets, widths, columns as global
    // row positions, and each position's instance-local node
    h_slice_off.assign(static_cast<size_t>(nslices) + 1, 0);
    std::vector<int> sw(static_cast<size_t>(nslices), 0), rn(static_cast<size_t>(NP), -1);
    h_col.assign(static_cast<size_t>(nslots), 0);
    for (size_t k = 0; k < K; ++k) {
        const PressurePattern& P = mem[k].m->pat;
        const int p0 = slice0[k] * 32;
        std::vector<int> pos_of(static_cast<size_t>(N_k[k]), 0);
        for (size_t p = 0; p < P.row_node.size(); ++p) {
            rn[static_cast<size_t>(p0) + p] = P.row_node[p];
            if (P.row_node[p] >= 0) pos_of[static_cast<size_t>(P.row_node[p])] = p0 + static_cast<int>(p);
        }
        for (int s = 0; s < P.nslices; ++s) {
            h_slice_off[static_cast<size_t>(slice0[k] + s)] = slot0[k] + P.slice_off[static_cast<size_t>(s)];
            sw[static_cast<size_t>(slice0[k] + s)] = P.slice_w[static_cast<size_t>(s)];
        }
        for (long long t = 0; t < P.nslots; ++t)
            h_col[static_cast<size_t>(slot0[k] + t)] = pos_of[static_cast<size_t>(P.col[static_cast<size_t>(t)])];
        long long* cp = dalloc<long long>(P.cptr.size());
        int* ce = dalloc<int>(P.cent.size());
        CUDA_OK(cudaMemcpy(cp, P.cptr.data(), P.cptr.size() * sizeof(long long), cudaMemcpyHostToDevice));
        if (!P.cent.empty()) CUDA_OK(cudaMemcpy(ce, P.cent.data(), P.cent.size() * sizeof(int), cudaMemcpyHostToDevice));
        d_cptr.push_back(cp);
        d_cent.push_back(ce);
    }
    h_slice_off[static_cast<size_t>(nslices)] = nslots;
    d_slice_off = dalloc<long long>(h_slice_off.size());
    d_slice_w = dalloc<int>(sw.size());
    d_col = dalloc<int>(h_col.size());
    d_row_node = dalloc<int>(rn.size());
    CUDA_OK(cudaMemcpy(d_slice_off, h_slice_off.data(), h_slice_off.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_slice_w, sw.data(), sw.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!h_col.empty()) CUDA_OK(cudaMemcpy(d_col, h_col.data(), h_col.size() * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_row_node, rn.data(), rn.size() * sizeof(int), cudaMemcpyHostToDevice));
    d_lcol = dalloc<unsigned short>(static_cast<size_t>(nslots));
    d_val = dalloc<double>(static_cast<size_t>(nslots));
    CUDA_OK(cudaMemset(d_val, 0, static_cast<size_t>(nslots ? nslots : 1) * sizeof(double)));
    const size_t n = static_cast<size_t>(NP);
    d_r = dalloc<double>(2 * n); d_q = dalloc<double>(2 * n);
    d_z = dalloc<double>(n); d_pA = dalloc<double>(n); d_pB = dalloc<double>(n);
    d_xp = dalloc<double>(n); d_bp = dalloc<double>(n); d_dp = dalloc<double>(n);
    d_fp = dalloc<uint8_t>(n);
    CUDA_OK(cudaMemset(d_pB, 0, n * sizeof(double)));
    if (mixed) {
        d_val32 = dalloc<float>(static_cast<size_t>(nslots));
        d_f32 = dalloc<float>(8 * n);
        CUDA_OK(cudaMemset(d_f32, 0, 8 * n * sizeof(float)));
    }
    d_part = dalloc<double>(K * static_cast<size_t>(gmax) * 16);
    d_bar = dalloc<unsigned>(4 * K);
    d_out = dalloc<CgOut>(K);
    CUDA_OK(cudaMemset(d_bar, 0, 4 * K * sizeof(unsigned)));
    CUDA_OK(cudaMemset(d_out, 0, K * sizeof(CgOut)));

    base = PcgDev{};
    base.N = NP; base.nslices = nslices; base.inner_tol = inner_tol;
    base.slice_off = d_slice_off; base.slice_w = d_slice_w; base.col = d_col; base.val = d_val;
    base.val32 = d_val32; base.row_node = d_row_node;
    base.pres = d_xp; base.rhs1 = d_bp; base.pdiag = d_dp; base.nflag = d_fp;
    base.r = d_r; base.z = d_z; base.pA = d_pA; base.pB = d_pB; base.q = d_q;
    if (mixed) {
        base.r32 = d_f32; base.w32 = d_f32 + 2 * n; base.s32 = d_f32 + 4 * n;
        base.p32 = d_f32 + 6 * n; base.dz32 = d_f32 + 7 * n;
    }
    base.lcol = d_lcol;
}

void PcgBatch::free_waves()
{
    for (Wave& w : waves) {
        void* ptrs[] = {w.d_cta_inst, w.d_inst, w.d_hptr, w.d_hidx};
        for (void* p : ptrs) if (p) cudaFree(p);
    }
    waves.clear();
}

bool PcgBatch::plan(const PcgBatchPlan& p, std::string* why)
{
    if (p.rmax != 1 && p.rmax != 2 && p.rmax != 4 && p.rmax != 8) {
        if (why) *why = "rows per thread must be 1, 2, 4 or 8";
        return false;
    }
    const int K = static_cast<int>(mem.size());
    const int cap = (BATCH_THREADS / 32) * p.rmax;   // slices one CTA holds in registers
    std::vector<int> minc(static_cast<size_t>(K));
    for (int k = 0; k < K; ++k) {
        minc[static_cast<size_t>(k)] = std::max(1, (nsl[static_cast<size_t>(k)] + cap - 1) / cap);
        if (minc[static_cast<size_t>(k)] > gmax) {
            if (why) *why = "instance " + std::to_string(k) + " needs more CTAs than one launch holds at this tiling";
            return false;
        }
    }
    // first-fit decreasing by slices into waves of at most gmax CTAs
    std::vector<int> order(static_cast<size_t>(K));
    for (int k = 0; k < K; ++k) order[static_cast<size_t>(k)] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return nsl[static_cast<size_t>(a)] > nsl[static_cast<size_t>(b)]; });
    std::vector<std::vector<int>> packs;
    std::vector<int> used;
    for (int k : order) {
        size_t w = 0;
        while (w < packs.size() && used[w] + minc[static_cast<size_t>(k)] > gmax) ++w;
        if (w == packs.size()) { packs.emplace_back(); used.push_back(0); }
        packs[w].push_back(k);
        used[w] += minc[static_cast<size_t>(k)];
    }
    const void* c64[4] = {fn_cgcg<true, BATCH_THREADS>(1), fn_cgcg<true, BATCH_THREADS>(2), fn_cgcg<true, BATCH_THREADS>(4),
                          fn_cgcg<true, BATCH_THREADS>(8)};
    const void* c32[4] = {fn_mixed<true, BATCH_THREADS>(1), fn_mixed<true, BATCH_THREADS>(2), fn_mixed<true, BATCH_THREADS>(4),
                          fn_mixed<true, BATCH_THREADS>(8)};
    const int ci = p.rmax == 1 ? 0 : p.rmax == 2 ? 1 : p.rmax == 4 ? 2 : 3;

    struct HostWave {
        int G = 0, hmax = 0;
        long long smax = 0;
        std::vector<int> cta_inst, hptr, hidx;
        std::vector<PcgInst> inst;
    };
    std::vector<HostWave> hw(packs.size());
    std::vector<unsigned short> lcol(static_cast<size_t>(nslots), 0);
    for (size_t w = 0; w < packs.size(); ++w) {
        HostWave& H = hw[w];
        const std::vector<int>& mk = packs[w];
        std::vector<int> G(mk.size());
        int tot = 0;
        for (size_t j = 0; j < mk.size(); ++j) { G[j] = minc[static_cast<size_t>(mk[j])]; tot += G[j]; }
        if (p.spread) {
            // spare CTAs, one at a time, to the instance with the most slices per CTA
            while (tot < gmax) {
                int best = -1;
                double bw = 0.0;
                for (size_t j = 0; j < mk.size(); ++j) {
                    if (G[j] >= nsl[static_cast<size_t>(mk[j])]) continue;
                    const double wpc = static_cast<double>(nsl[static_cast<size_t>(mk[j])]) / G[j];
                    if (wpc > bw) { bw = wpc; best = static_cast<int>(j); }
                }
                if (best < 0) break;
                ++G[static_cast<size_t>(best)];
                ++tot;
            }
        }
        H.G = tot;
        H.hptr.push_back(0);
        int cta = 0;
        for (size_t j = 0; j < mk.size(); ++j) {
            const int k = mk[j];
            const PressurePattern& P = mem[static_cast<size_t>(k)].m->pat;
            PcgInst I{};
            I.cta0 = cta; I.ncta = G[j];
            I.s0 = slice0[static_cast<size_t>(k)]; I.s1 = I.s0 + nsl[static_cast<size_t>(k)];
            I.precond = mem[static_cast<size_t>(k)].m->p.cg_preconditioner;
            I.conv_test = mem[static_cast<size_t>(k)].m->p.cg_conv_test;
            I.max_iter = mem[static_cast<size_t>(k)].m->p.cg_max_iter;
            I.rel_tol = mem[static_cast<size_t>(k)].m->p.relToler;
            I.abs_tol = mem[static_cast<size_t>(k)].m->p.absToler;
            I.bar = d_bar + 4 * k;
            I.part = d_part + static_cast<size_t>(k) * static_cast<size_t>(gmax) * 16;
            I.status = mem[static_cast<size_t>(k)].d_status;
            I.out = d_out + k;
            H.inst.push_back(I);
            (void)P;
            std::vector<int> cols;
            for (int b = 0; b < G[j]; ++b) {
                H.cta_inst.push_back(static_cast<int>(j));
                const int sb = I.s0 + static_cast<int>(static_cast<long long>(b) * (I.s1 - I.s0) / G[j]);
                const int se = I.s0 + static_cast<int>(static_cast<long long>(b + 1) * (I.s1 - I.s0) / G[j]);
                const long long a0 = h_slice_off[static_cast<size_t>(sb)], a1 = h_slice_off[static_cast<size_t>(se)];
                cols.assign(h_col.begin() + a0, h_col.begin() + a1);
                std::sort(cols.begin(), cols.end());
                cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
                if (cols.size() > 65535) {
                    if (why) *why = "a CTA halo exceeds 65535 columns";
                    return false;
                }
                for (long long t = a0; t < a1; ++t)
                    lcol[static_cast<size_t>(t)] = static_cast<unsigned short>(
                        std::lower_bound(cols.begin(), cols.end(), h_col[static_cast<size_t>(t)]) - cols.begin());
                H.hidx.insert(H.hidx.end(), cols.begin(), cols.end());
                H.hptr.push_back(static_cast<int>(H.hidx.size()));
                H.hmax = std::max(H.hmax, static_cast<int>(cols.size()));
                H.smax = std::max(H.smax, a1 - a0);
            }
            cta += G[j];
        }
    }
    // kernels and shared memory of every wave, before anything is replaced
    std::vector<Wave> nw(hw.size());
    for (size_t w = 0; w < hw.size(); ++w) {
        const HostWave& H = hw[w];
        Wave& W = nw[w];
        W.G = H.G; W.rmax = p.rmax;
        const size_t s64 = static_cast<size_t>(H.hmax) * 20 + static_cast<size_t>(H.smax) * 2 + 16;
        const size_t s32 = static_cast<size_t>(H.hmax) * 16 + static_cast<size_t>(H.smax) * 6 + 16;
        auto fits = [&](const void* fn, size_t smem) {
            if (smem > 220 * 1024) return false;
            if (raise_smem_limit(fn, smem) != cudaSuccess) {
                cudaGetLastError();
                return false;
            }
            int per = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, BATCH_THREADS, smem) != cudaSuccess) {
                cudaGetLastError();
                return false;
            }
            return per * sms >= H.G;
        };
        if (mixed && fits(c32[ci], s32)) { W.mixed = true; W.fn = c32[ci]; W.smem = s32; }
        else if (fits(c64[ci], s64)) { W.mixed = false; W.fn = c64[ci]; W.smem = s64; }
        else {
            if (why) *why = "a wave does not fit co-resident at this tiling";
            return false;
        }
    }
    free_waves();
    mixed_any = false;
    CUDA_OK(cudaMemcpy(d_lcol, lcol.data(), lcol.size() * sizeof(unsigned short), cudaMemcpyHostToDevice));
    for (size_t w = 0; w < hw.size(); ++w) {
        const HostWave& H = hw[w];
        Wave& W = nw[w];
        W.d_cta_inst = dalloc<int>(H.cta_inst.size());
        W.d_inst = dalloc<PcgInst>(H.inst.size());
        W.d_hptr = dalloc<int>(H.hptr.size());
        W.d_hidx = dalloc<int>(H.hidx.size());
        CUDA_OK(cudaMemcpy(W.d_cta_inst, H.cta_inst.data(), H.cta_inst.size() * sizeof(int), cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemcpy(W.d_inst, H.inst.data(), H.inst.size() * sizeof(PcgInst), cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemcpy(W.d_hptr, H.hptr.data(), H.hptr.size() * sizeof(int), cudaMemcpyHostToDevice));
        if (!H.hidx.empty()) CUDA_OK(cudaMemcpy(W.d_hidx, H.hidx.data(), H.hidx.size() * sizeof(int), cudaMemcpyHostToDevice));
        W.dev = base;
        W.dev.nblocks = W.G;
        W.dev.cta_inst = W.d_cta_inst;
        W.dev.inst = W.d_inst;
        W.dev.halo_ptr = W.d_hptr;
        W.dev.halo_idx = W.d_hidx;
        W.dev.halo_max = H.hmax;
        W.dev.slot_max = static_cast<int>(H.smax);
        mixed_any = mixed_any || W.mixed;
    }
    waves = std::move(nw);
    current = p;
    return true;
}

void PcgBatch::release()
{
    free_waves();
    for (long long* p : d_cptr) cudaFree(p);
    for (int* p : d_cent) cudaFree(p);
    d_cptr.clear();
    d_cent.clear();
    void* ptrs[] = {d_slice_off, d_slice_w, d_col, d_row_node, d_lcol, d_val, d_val32, d_r, d_z, d_pA, d_pB, d_q,
                    d_xp, d_bp, d_dp, d_fp, d_f32, d_part, d_bar, d_out};
    for (void* p : ptrs) if (p) cudaFree(p);
    d_slice_off = nullptr; d_slice_w = d_col = d_row_node = nullptr; d_lcol = nullptr; d_val = nullptr;
    d_val32 = nullptr; d_r = d_z = d_pA = d_pB = d_q = nullptr; d_xp = d_bp = d_dp = nullptr; d_fp = nullptr;
    d_f32 = nullptr; d_part = nullptr; d_bar = nullptr; d_out = nullptr;
}

void PcgBatch::prepare(int k, const DevState& S, cudaStream_t st)
{
    const size_t kk = static_cast<size_t>(k);
    const int T = 256;
    if (nslot[kk])
        k_ell_from_state<<<static_cast<unsigned>((nslot[kk] + T - 1) / T), T, 0, st>>>(
            S, d_cptr[kk], d_cent[kk], d_val + slot0[kk], d_val32 ? d_val32 + slot0[kk] : nullptr, nslot[kk]);
    PcgDev D = base;
    D.NN = N_k[kk];
    D.nflag = mem[kk].d_nflag;
    D.pfix = mem[kk].d_pfix;
    D.pres = S.pres; D.rhs1 = S.rhs1; D.pdiag = S.pdiag;
    k_impose<<<(N_k[kk] + T - 1) / T, T, 0, st>>>(D);
    const int p0 = slice0[kk] * 32, np = nsl[kk] * 32;
    D.N = np;
    D.row_node = d_row_node + p0;
    k_perm_in<<<(np + T - 1) / T, T, 0, st>>>(D, S.pres, S.rhs1, S.pdiag, mem[kk].d_nflag, d_xp + p0, d_bp + p0,
                                               d_dp + p0, d_fp + p0);
}

void PcgBatch::solve(cudaStream_t st)
{
    CUDA_OK(cudaMemsetAsync(d_bar, 0, 4 * mem.size() * sizeof(unsigned), st));
    CUDA_OK(cudaMemsetAsync(d_out, 0, mem.size() * sizeof(CgOut), st));
    for (Wave& W : waves) {
        void* args[] = {&W.dev};
        CUDA_OK(cudaLaunchCooperativeKernel(W.fn, dim3(static_cast<unsigned>(W.G)), dim3(BATCH_THREADS), args, W.smem, st));
    }
}

void PcgBatch::finish(int k, double* pres, cudaStream_t st)
{
    const size_t kk = static_cast<size_t>(k);
    const int T = 256;
    const int p0 = slice0[kk] * 32, np = nsl[kk] * 32;
    PcgDev D = base;
    D.N = np;
    D.row_node = d_row_node + p0;
    k_perm_out<<<(np + T - 1) / T, T, 0, st>>>(D, d_xp + p0, pres);
}

}  // namespace cbs3d

extern "C" cbs3d_status cbs3d_probe_halo_placement(int nh, int nslices, const long long* slice_off, const int* slice_w,
                                                   const unsigned short* lc, int* pos, long long* wavefronts)
{
    try {
        if (nh < 1 || nh > 65535 || nslices < 1 || !slice_off || !slice_w || !lc || !pos || !wavefronts)
            return CBS3D_INVALID_INPUT;
        if (slice_off[0] != 0) return CBS3D_INVALID_INPUT;
        for (int q = 0; q < nslices; ++q)
            if (slice_w[q] < 0 || slice_off[q + 1] - slice_off[q] != 32LL * slice_w[q]) return CBS3D_INVALID_INPUT;
        for (long long t = 0; t < slice_off[nslices]; ++t)
            if (lc[t] >= nh) return CBS3D_INVALID_INPUT;
        std::vector<int> id(static_cast<size_t>(nh)), pv;
        for (int e = 0; e < nh; ++e) id[static_cast<size_t>(e)] = e;
        wavefronts[0] = cbs3d::gather_wavefronts(lc, slice_off, slice_w, 0, nslices, 0, id);
        cbs3d::bank_spread_halo(nh, lc, slice_off, slice_w, 0, nslices, 0, pv);
        wavefronts[1] = cbs3d::gather_wavefronts(lc, slice_off, slice_w, 0, nslices, 0, pv);
        for (int e = 0; e < nh; ++e) pos[e] = pv[static_cast<size_t>(e)];
        return CBS3D_OK;
    } catch (...) {
        return CBS3D_INTERNAL;
    }
}
