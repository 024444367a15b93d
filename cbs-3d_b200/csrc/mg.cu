// Aggregation multigrid preconditioned CG for the pressure system: host-side
// hierarchy, per-solve Galerkin set-up kernels and the persistent solver
// kernel.  The algorithm and its invariants are described in mg.cuh.
#include "mg.cuh"

#include <algorithm>
#include <cstring>
#include <utility>
#include <vector>

namespace cbs3d {

namespace {

#define MG_CUDA_OK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) throw Error(CBS3D_CUDA_ERROR, std::string(#x) + ": " + cudaGetErrorString(e_)); } while (0)

constexpr int MG_NT = 512;                 // threads of the solver CTA
constexpr int MG_NW = MG_NT / 32;
constexpr int MG_CHUNK_SLICES = 4;         // partition and reduction unit: 4 SELL slices = 128 rows
constexpr double MG_OVER = 1.5;            // coarse over-correction
constexpr double MG_OMEGA = 0.8;           // smoother weight cap
constexpr double MG_GERSH = 1.8;           // weight bound: omega * gershgorin <= 1.8 < 2

// threads per row of coarse level l in the solver kernel (fixed per level,
// so every row's sum has the same order for any grid size)
inline int level_tpr(int l) { return l == 1 ? 2 : l == 2 ? 8 : 32; }

__device__ __forceinline__ double smoother_weight(double d, double offabs)
{
    if (!(d > 0.0) || !isfinite(d)) return 0.0;
    return fmin(MG_OMEGA, MG_GERSH * d / (d + offabs)) / d;
}

// ------------------------------------------------------------ set-up kernels
// Level-0 smoother weights from the assembled rows (free columns only).
__global__ void k_mg_weights0(const long long* slice_off, const int* slice_w, const int* colp, const double* val,
                              const double* pdiag, const int* row_node, const uint8_t* free0, int NP, double* wd0)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    if (!free0[p]) { wd0[p] = 0.0; return; }
    const double d = row_node ? pdiag[row_node[p]] : pdiag[p];
    const int s = p >> 5, lane = p & 31;
    const long long base = slice_off[s] + lane;
    const int w = slice_w[s];
    double a = 0.0;
    for (int k = 0; k < w; ++k) {
        const long long t = base + 32LL * k;
        if (free0[colp[t]]) a += fabs(val[t]);
    }
    wd0[p] = smoother_weight(d, a);
}

// Galerkin sums: output o = sum of its sources in list order; a source id
// >= 0 is an off-diagonal entry of the level below, id < 0 the diagonal of
// its row -(id+1) (level 0: pdiag, node-ordered through row_node if given).
__global__ void k_mg_galerkin(const long long* gptr, const int* gent, long long nout, const double* vsrc,
                              const double* dsrc, const int* row_node, double* vout)
{
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nout) return;
    double v = 0.0;
    for (long long c = gptr[o]; c < gptr[o + 1]; ++c) {
        const int id = gent[c];
        if (id >= 0) {
            v += vsrc[id];
        } else {
            const int i = -(id + 1);
            v += row_node ? dsrc[row_node[i]] : dsrc[i];
        }
    }
    vout[o] = v;
}

__global__ void k_mg_weights(const double* val, const int* col, int n, int W, double* wd)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n) return;
    double a = 0.0;
    for (int k = 0; k < W; ++k) {
        const long long s = mg_slot(I, k, W);
        if (col[s] >= 0) a += fabs(val[s]);
    }
    wd[I] = smoother_weight(val[mg_slots(n, W) + I], a);
}

// The coarsest operator as a dense matrix (rows without free children are
// left zero; the inverse kernel turns a zero diagonal into 1).
__global__ void k_mg_dense(const double* val, const int* col, int n, int W, double* a)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n) return;
    double* row = a + (size_t)I * n;
    for (int J = 0; J < n; ++J) row[J] = 0.0;
    row[I] = val[mg_slots(n, W) + I];
    for (int k = 0; k < W; ++k) {
        const long long s = mg_slot(I, k, W);
        if (col[s] >= 0) row[col[s]] = val[s];
    }
}

// ------------------------------------------------------------ grid sync
// Thread 0 only: arrive on the monotonic counter and wait (bounded) until
// every CTA has; false when the wait ran out or a failure was recorded.
__device__ __forceinline__ bool mg_arrive_wait(unsigned long long* cnt, unsigned long long target, DevStatus* st)
{
    unsigned long long arrived;
    asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], 1;" : "=l"(arrived) : "l"(cnt) : "memory");
    if (arrived + 1 < target) {
        const long long t0 = clock64();
        for (;;) {
            unsigned long long c;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(c) : "l"(cnt) : "memory");
            if (c >= target) break;
            if (ld_relaxed_int(&st->code) != 0) return false;
            if (clock64() - t0 > (1LL << 31)) {
                set_status(st, 5 /*CBS3D_TIMEOUT*/, ST_PCG, 0, R_PCG_BARRIER);
                return false;
            }
        }
    }
    return ld_relaxed_int(&st->code) == 0;
}

// Off-diagonal product of coarse row I over the staged halo values vl: the
// row's T threads (sub = 0..T-1) take entries sub, sub+T, ... in order, four
// loads issued at a time, then a fixed xor tree over the T lanes.  All lanes
// of the warp call it (active false: contributes nothing).
__device__ __forceinline__ double coarse_row(const MgLevelDev& Lv, int I, int sub, int T, bool active,
                                             const double* vl)
{
    double acc = 0.0;
    if (active) {
        const int W = Lv.W;
        for (int k0 = sub; k0 < W; k0 += 8 * T) {
            unsigned short lc[8];
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int k = k0 + u * T;
                const long long s = mg_slot(I, k < W ? k : 0, W);
                lc[u] = k < W ? __ldg(Lv.lcol + s) : (unsigned short)0xffffu;
                v[u] = k < W ? __ldg(Lv.val + s) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (lc[u] != 0xffffu) acc = fma(v[u], vl[lc[u]], acc);
        }
    }
    for (int m = 1; m < T; m <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
    return acc;
}

// ------------------------------------------------------------ solver kernel
template <int RMAX>
__global__ void __launch_bounds__(MG_NT, 1) k_pcg_mg(PcgDev D, MgDev M)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_sl[4][RMAX * MG_NW];   // per-slice partials
    __shared__ double s_w[4][MG_NW];            // per-warp partials of the chunk sums
    __shared__ int s_ok;
    const int G = gridDim.x, b = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c0 = (int)((long long)b * M.nchunks / G), c1 = (int)((long long)(b + 1) * M.nchunks / G);
    const int s_beg = MG_CHUNK_SLICES * c0;
    const int s_end = min(MG_CHUNK_SLICES * c1, D.nslices);
    const int NP = D.N;
    const long long pos0 = 32LL * s_beg, pos1 = 32LL * s_end;
    const long long S0 = D.slice_off[s_beg];
    const int nsl = (int)(D.slice_off[s_end] - S0);
    const int h0 = D.halo_ptr[b];
    const int nh = D.halo_ptr[b + 1] - h0;
    const int HM = D.halo_max;
    DevStatus* status = D.status;

    double* rh = reinterpret_cast<double*>(smem_raw);   // halo: CG residual
    double* ph = rh + HM;                               // halo: search direction
    double* vh = ph + HM;                               // halo: values the next product reads
    double* dbase = reinterpret_cast<double*>(smem_raw);
    int* ibase = reinterpret_cast<int*>(dbase + M.sd_xc + 2 * M.nc);
    int* hidx = ibase;
    unsigned short* lcs = reinterpret_cast<unsigned short*>(ibase + M.si_end);
    double* rc = dbase + M.sd_xc;                       // coarsest level: r
    double* xc = rc + M.nc;                             // coarsest level: x
    for (int k = threadIdx.x; k < nh; k += MG_NT) hidx[k] = D.halo_idx[h0 + k];
    for (int k = threadIdx.x; k < nsl; k += MG_NT) lcs[k] = D.lcol[S0 + k];
    for (int l = 1; l < M.Lc; ++l) {
        const MgLevelDev& Lv = M.lv[l];
        const int a0 = Lv.hptr[b], an = Lv.hptr[b + 1] - a0;
        int* jl = ibase + Lv.si;
        for (int k = threadIdx.x; k < an; k += MG_NT) jl[k] = Lv.hidx[a0 + k];
    }

    int phase = 0;
    auto sync_grid = [&]() -> bool {
        __syncthreads();
        if (threadIdx.x == 0) s_ok = mg_arrive_wait(M.bar, (unsigned long long)(phase + 1) * G, status);
        __syncthreads();
        ++phase;
        return s_ok != 0;
    };
    // All-reduce of NV values (q < NS summed, the rest max-reduced): v[q][k]
    // is this thread's value of row k.  Rows are summed per slice (fixed
    // shuffle tree), slices per chunk in order, chunks in a fixed order that
    // does not depend on the grid; every CTA computes the same result.
    auto allreduce = [&](double (&v)[4][RMAX], double* out, int NV, int NS) -> bool {
        const int nls = s_end - s_beg;
        for (int q = 0; q < NV; ++q)
#pragma unroll
            for (int k = 0; k < RMAX; ++k) {
                double x = v[q][k];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double y = __shfl_down_sync(0xffffffffu, x, o);
                    x = q < NS ? x + y : fmax(x, y);
                }
                if (lane == 0) s_sl[q][warp + MG_NW * k] = x;
            }
        __syncthreads();
        const int nck = c1 - c0;
        double* part = M.part + (size_t)(phase & 1) * 4 * M.nchunks;
        for (int t = threadIdx.x; t < nck * NV; t += MG_NT) {
            const int q = t / nck, cc = t - q * nck;
            double x = 0.0;
            for (int u = 0; u < MG_CHUNK_SLICES; ++u) {
                const int ls = cc * MG_CHUNK_SLICES + u;
                const double y = ls < nls ? s_sl[q][ls] : 0.0;
                x = q < NS ? x + y : fmax(x, y);
            }
            __stcg(part + (size_t)q * M.nchunks + c0 + cc, x);
        }
        if (!sync_grid()) return false;
        double t4[4] = {0.0, 0.0, 0.0, 0.0};
        // four chunks per round, all their loads issued before the sums
        // (each thread's chunks are still summed in ascending order)
        for (int c0 = threadIdx.x; c0 < M.nchunks; c0 += 4 * MG_NT) {
            double y[4][4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int c = c0 + u * MG_NT;
                    y[u][q] = (q < NV && c < M.nchunks) ? __ldcg(part + (size_t)q * M.nchunks + c) : 0.0;
                }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (c0 + u * MG_NT < M.nchunks)
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (q < NV) t4[q] = q < NS ? t4[q] + y[u][q] : fmax(t4[q], y[u][q]);
        }
        for (int q = 0; q < NV; ++q) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double y = __shfl_down_sync(0xffffffffu, t4[q], o);
                t4[q] = q < NS ? t4[q] + y : fmax(t4[q], y);
            }
            if (lane == 0) s_w[q][warp] = t4[q];
        }
        __syncthreads();
        for (int q = 0; q < NV; ++q) {
            double x = 0.0;
            for (int w = 0; w < MG_NW; ++w) x = q < NS ? x + s_w[q][w] : fmax(x, s_w[q][w]);
            out[q] = x;
        }
        __syncthreads();
        return true;
    };

    double r[RMAX], p[RMAX], z[RMAX], dg[RMAX], wd[RMAX];
    bool fr[RMAX];
    int row[RMAX], lbase[RMAX], wr[RMAX];
    int wmax = 0;
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        const int sl = s_beg + warp + MG_NW * k;
        row[k] = (sl < s_end) ? sl * 32 + lane : -1;
        lbase[k] = 0;
        wr[k] = 0;
        if (sl < s_end) {
            lbase[k] = (int)(D.slice_off[sl] - S0) + lane;
            wr[k] = D.slice_w[sl];
            wmax = wr[k] > wmax ? wr[k] : wmax;
        }
        r[k] = p[k] = z[k] = dg[k] = wd[k] = 0.0;
        fr[k] = false;
    }
    // off[k] = sum_j A_ij src[j] over the own rows' off-diagonal slots
    auto offdiag = [&](const double* src, double* off) {
#pragma unroll
        for (int k = 0; k < RMAX; ++k) off[k] = 0.0;
        for (int k0 = 0; k0 < wmax; k0 += 2) {
            double v[RMAX][2];
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    v[k][u] = (k0 + u < wr[k]) ? __ldcg(D.val + S0 + lbase[k] + 32 * (k0 + u)) : 0.0;
#pragma unroll
            for (int k = 0; k < RMAX; ++k)
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const double g = (k0 + u < wr[k]) ? src[lcs[lbase[k] + 32 * (k0 + u)]] : 0.0;
                    off[k] = fma(v[k][u], g, off[k]);
                }
        }
    };

    // One V(1,1) cycle on the residual r (own rows in registers, halo copy
    // in rh): z = B r.
    auto vcycle = [&]() -> bool {
        double off[RMAX];
        // level 0: pre-smoothing from zero (x = W r, halo included), residual
        // (the halo's smoother weights are read through L1: constant per solve)
        for (int k = threadIdx.x; k < nh; k += MG_NT) vh[k] = __ldg(M.wd0 + hidx[k]) * rh[k];
        __syncthreads();
        offdiag(vh, off);
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0) continue;
            const double rho = fr[k] ? r[k] - dg[k] * (wd[k] * r[k]) - off[k] : 0.0;
            __stcg(M.rho0 + i, rho);
        }
        if (!sync_grid()) return false;
        // coarse levels, downwards: restrict, pre-smooth from zero, residual
        for (int l = 1; l < M.Lc; ++l) {
            const MgLevelDev& Lv = M.lv[l];
            const double* rprev = l == 1 ? M.rho0 : M.lv[l - 1].rho;
            const long long nprev = l == 1 ? NP : M.lv[l - 1].n;
            const int a0 = Lv.hptr[b], an = Lv.hptr[b + 1] - a0;
            const int* jl = ibase + Lv.si;
            double* rl = dbase + Lv.sd;
            double* wl = rl + Lv.hmax;
            double* vl = wl + Lv.hmax;
            for (int k = threadIdx.x; k < an; k += MG_NT) {
                const long long base = 8LL * jl[k];
                double s = 0.0;
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (base + c < nprev) s += __ldcg(rprev + base + c);
                const double w = __ldg(Lv.wd + jl[k]);
                rl[k] = s;
                wl[k] = w;
                vl[k] = w * s;
            }
            __syncthreads();
            long long sc = 1;
            for (int q = 0; q < l; ++q) sc *= 8;
            const int o = (int)((pos0 + sc - 1) / sc);
            const int e = (int)min((long long)Lv.n, (pos1 + sc - 1) / sc);
            const int T = Lv.tpr, W = Lv.W, hown = Lv.hown[b];
            const int sub = threadIdx.x % T;
            for (int rb = 0; rb < e - o; rb += MG_NT / T) {
                const int ri = rb + threadIdx.x / T;
                const int I = o + ri;
                const double acc = coarse_row(Lv, I, sub, T, ri < e - o, vl);
                if (ri < e - o && sub == 0) {
                    const int hI = hown + ri;
                    const double w = wl[hI];
                    const double rho = w > 0.0 ? rl[hI] - __ldg(Lv.val + mg_slots(Lv.n, W) + I) * vl[hI] - acc : 0.0;
                    __stcg(Lv.rho + I, rho);
                }
            }
            if (!sync_grid()) return false;
        }
        // coarsest level: every CTA restricts and solves it whole
        {
            const double* rprev = M.Lc == 1 ? M.rho0 : M.lv[M.Lc - 1].rho;
            const long long nprev = M.Lc == 1 ? NP : M.lv[M.Lc - 1].n;
            for (int I = threadIdx.x; I < M.nc; I += MG_NT) {
                double s = 0.0;
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (8LL * I + c < nprev) s += __ldcg(rprev + 8LL * I + c);
                rc[I] = s;
            }
            __syncthreads();
            // four threads per row (columns sub, sub+4, ... in order, then a
            // fixed xor tree); every warp runs the same number of rounds
            for (int I0 = 0; I0 < M.nc; I0 += MG_NT / 4) {
                const int I = I0 + (threadIdx.x >> 2), sub = threadIdx.x & 3;
                double x = 0.0;
                if (I < M.nc)
                    for (int J = sub; J < M.nc; J += 4) x = fma(__ldg(M.ainv + (size_t)I * M.nc + J), rc[J], x);
                x += __shfl_xor_sync(0xffffffffu, x, 1);
                x += __shfl_xor_sync(0xffffffffu, x, 2);
                if (I < M.nc && sub == 0) xc[I] = x;
            }
            __syncthreads();
        }
        // coarse levels, upwards: interpolate, post-smooth
        for (int l = M.Lc - 1; l >= 1; --l) {
            const MgLevelDev& Lv = M.lv[l];
            const int a0 = Lv.hptr[b], an = Lv.hptr[b + 1] - a0;
            const int* jl = ibase + Lv.si;
            double* rl = dbase + Lv.sd;
            double* wl = rl + Lv.hmax;
            double* vl = wl + Lv.hmax;
            const double* xup = l + 1 < M.Lc ? M.lv[l + 1].x : nullptr;
            for (int k = threadIdx.x; k < an; k += MG_NT) {
                const int J = jl[k];
                const double xcg = xup ? __ldcg(xup + (J >> 3)) : xc[J >> 3];
                const double w = wl[k];
                vl[k] = w > 0.0 ? fma(w, rl[k], MG_OVER * xcg) : 0.0;
            }
            __syncthreads();
            long long sc = 1;
            for (int q = 0; q < l; ++q) sc *= 8;
            const int o = (int)((pos0 + sc - 1) / sc);
            const int e = (int)min((long long)Lv.n, (pos1 + sc - 1) / sc);
            const int T = Lv.tpr, W = Lv.W, hown = Lv.hown[b];
            const int sub = threadIdx.x % T;
            for (int rb = 0; rb < e - o; rb += MG_NT / T) {
                const int ri = rb + threadIdx.x / T;
                const int I = o + ri;
                const double acc = coarse_row(Lv, I, sub, T, ri < e - o, vl);
                if (ri < e - o && sub == 0) {
                    const int hI = hown + ri;
                    const double w = wl[hI];
                    const double xv = vl[hI];
                    const double xn =
                        w > 0.0 ? xv + w * (rl[hI] - __ldg(Lv.val + mg_slots(Lv.n, W) + I) * xv - acc) : 0.0;
                    __stcg(Lv.x + I, xn);
                }
            }
            if (!sync_grid()) return false;
        }
        // level 0: interpolate, post-smooth
        const double* x1 = M.Lc > 1 ? M.lv[1].x : nullptr;
        for (int k = threadIdx.x; k < nh; k += MG_NT) {
            const int pos = hidx[k];
            const double w = __ldg(M.wd0 + pos);
            const double xcg = x1 ? __ldcg(x1 + (pos >> 3)) : xc[pos >> 3];
            vh[k] = w > 0.0 ? fma(w, rh[k], MG_OVER * xcg) : 0.0;
        }
        __syncthreads();
        offdiag(vh, off);
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            z[k] = 0.0;
            if (i < 0 || !fr[k]) continue;
            const double xcg = x1 ? __ldcg(x1 + (i >> 3)) : xc[i >> 3];
            const double x0 = fma(wd[k], r[k], MG_OVER * xcg);
            z[k] = x0 + wd[k] * (r[k] - dg[k] * x0 - off[k]);
        }
        return true;
    };

    auto finish = [&](int it, int conv, double init, double fin, double rel, double mx) {
        if (b == 0 && threadIdx.x == 0) {
            D.out->iterations = it;
            D.out->converged = conv;
            D.out->initial_l2 = init;
            D.out->final_l2 = fin;
            D.out->rel = rel;
            D.out->max_abs = mx;
        }
    };
    auto fail = [&](int code, int it, int reason) {
        if (b == 0 && threadIdx.x == 0) set_status(status, code, ST_PCG, it, reason);
    };
    auto converged = [&](double rel, double mx) {
        if (D.conv_test == 1) return mx <= D.abs_tol;
        if (D.conv_test == 2) return rel <= D.rel_tol;
        return mx <= D.abs_tol || rel <= D.rel_tol;
    };

    // ---- r0 = b - A x0 with the reference's constraints and checks
    for (int k = threadIdx.x; k < nh; k += MG_NT) {
        vh[k] = __ldcg(D.pres + hidx[k]);
        ph[k] = 0.0;
    }
    __syncthreads();
    double off[RMAX];
    offdiag(vh, off);
    double v4[4][RMAX], o4[4];
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        v4[0][k] = v4[1][k] = v4[2][k] = v4[3][k] = 0.0;
        const int i = row[k];
        if (i < 0) continue;
        const uint8_t f = D.nflag[i];
        const bool active = f & 1;
        fr[k] = active && !(f & 4);
        const double pd = D.pdiag[i];
        const double y = fma(pd, D.pres[i], off[k]);
        double ri = active ? D.rhs1[i] - y : 0.0;
        if (!fr[k]) ri = 0.0;
        if (fr[k]) {
            if (!(isfinite(pd) && pd > 1.0e-30)) v4[2][k] = 1.0;
            if (!isfinite(ri)) v4[2][k] = 2.0;
            v4[0][k] = ri * ri;
            v4[1][k] = fabs(ri);
            dg[k] = pd;
            wd[k] = __ldg(M.wd0 + i);
        }
        r[k] = ri;
        __stcg(D.r + i, ri);
    }
    if (!allreduce(v4, o4, 3, 1)) return;
    const double init = sqrt(o4[0]);
    if (init <= 1.0e-300) { finish(0, 1, init, init, 0.0, o4[1]); return; }
    if (converged(1.0, o4[1])) { finish(0, 1, init, init, 1.0, o4[1]); return; }
    if (o4[2] >= 2.0) { fail(4, 0, R_PCG_RESID); return; }
    if (o4[2] >= 1.0) { fail(1, 0, R_PCG_DIAG); return; }
    for (int k = threadIdx.x; k < nh; k += MG_NT) rh[k] = __ldcg(D.r + hidx[k]);
    __syncthreads();

    // ---- z0 = B r0, p0 = z0, rz = (r0, z0)
    if (!vcycle()) return;
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
        v4[0][k] = 0.0;
        if (row[k] < 0) continue;
        __stcg(D.z + row[k], z[k]);
        if (fr[k]) v4[0][k] = r[k] * z[k];
        p[k] = z[k];
    }
    if (!allreduce(v4, o4, 1, 1)) return;
    double rz = o4[0];
    if (rz <= 1.0e-300 || !isfinite(rz)) { fail(3, 0, R_PCG_RZ0); return; }
    for (int k = threadIdx.x; k < nh; k += MG_NT) ph[k] = __ldcg(D.z + hidx[k]);
    __syncthreads();

    double fin = init, rel = 1.0, mx = o4[1];
    int it = 0, conv = 0;
    for (it = 1; it <= D.max_iter; ++it) {
        // q = A p, pAp
        offdiag(ph, off);
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            v4[0][k] = 0.0;
            const int i = row[k];
            if (i < 0) continue;
            const double q = fr[k] ? fma(dg[k], p[k], off[k]) : 0.0;
            z[k] = q;   // z holds q until the next cycle
            __stcg(D.q + i, q);
            if (fr[k]) v4[0][k] = p[k] * q;
        }
        if (!allreduce(v4, o4, 1, 1)) return;
        const double pap = o4[0];
        if (fabs(pap) <= 1.0e-300 || !isfinite(pap)) { fail(3, it, R_PCG_PAP); return; }
        const double alpha = rz / pap;
        // x += alpha p, r -= alpha q (own rows and the halo copy)
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            const int i = row[k];
            if (i < 0 || !fr[k]) continue;
            D.pres[i] = fma(alpha, p[k], D.pres[i]);
            r[k] = fma(-alpha, z[k], r[k]);
        }
        for (int k = threadIdx.x; k < nh; k += MG_NT) rh[k] = fma(-alpha, __ldcg(D.q + hidx[k]), rh[k]);
        __syncthreads();
        // z = B r; the norms of r decide convergence of this iteration
        if (!vcycle()) return;
#pragma unroll
        for (int k = 0; k < RMAX; ++k) {
            v4[0][k] = v4[1][k] = v4[2][k] = v4[3][k] = 0.0;
            const int i = row[k];
            if (i < 0) continue;
            __stcg(D.z + i, z[k]);
            if (fr[k]) {
                v4[0][k] = r[k] * z[k];
                v4[1][k] = r[k] * r[k];
                v4[2][k] = fabs(r[k]);
                v4[3][k] = isfinite(r[k]) ? 0.0 : 1.0;
            }
        }
        if (!allreduce(v4, o4, 4, 2)) return;
        fin = sqrt(o4[1]);
        mx = o4[2];
        rel = fin / init;
        if (converged(rel, mx)) { conv = 1; break; }
        if (o4[3] > 0.0) { fail(4, it, R_PCG_RESID); return; }
        const double rzn = o4[0];
        if (rzn <= 1.0e-300 || !isfinite(rzn)) { fail(3, it, R_PCG_RZ); return; }
        const double beta = rzn / rz;
        rz = rzn;
#pragma unroll
        for (int k = 0; k < RMAX; ++k) p[k] = fr[k] ? fma(beta, p[k], z[k]) : 0.0;
        for (int k = threadIdx.x; k < nh; k += MG_NT) ph[k] = fma(beta, ph[k], __ldcg(D.z + hidx[k]));
        __syncthreads();
    }
    if (it > D.max_iter) it = D.max_iter;
    finish(it, conv, init, fin, rel, mx);
    if (!conv) fail(2, it, R_PCG_MAXIT);
}

const void* fn_mg(int rmax)
{
    return rmax == 1 ? reinterpret_cast<const void*>(k_pcg_mg<1>)
         : rmax == 2 ? reinterpret_cast<const void*>(k_pcg_mg<2>)
         : rmax == 4 ? reinterpret_cast<const void*>(k_pcg_mg<4>)
                     : reinterpret_cast<const void*>(k_pcg_mg<8>);
}

// One level's rows as a CSR of (column, ordered source ids) for building
// the next level.
struct LevelPattern {
    int n = 0;
    std::vector<int> rptr, col;          // off-diagonal columns per row (sorted)
    std::vector<int> sid;                // source id of every off-diagonal entry at the next level:
                                         // its slot in the padded layout (level >= 1) or SELL slot (level 0)
    std::vector<char> freerow;
};

}  // namespace

template <typename T>
T* MgHierarchy::upload(const std::vector<T>& v)
{
    T* p = nullptr;
    MG_CUDA_OK(cudaMalloc(&p, std::max<size_t>(v.size(), 1) * sizeof(T)));
    allocs.push_back(p);
    if (!v.empty()) MG_CUDA_OK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return p;
}

template <typename T>
T* MgHierarchy::zeros(size_t count)
{
    T* p = nullptr;
    MG_CUDA_OK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    allocs.push_back(p);
    MG_CUDA_OK(cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T)));
    return p;
}

bool MgHierarchy::build(const HostModel& m, const std::vector<int>& colp, const uint8_t* d_nflag,
                        const long long* slice_off_d, const int* slice_w_d, const int* colp_d, int device, int sms,
                        int blocks_override)
{
    (void)device;
    const PressurePattern& P = m.pat;
    nslices = P.nslices;
    NP = nslices * 32;
    d_slice_off = slice_off_d;
    d_slice_w = slice_w_d;
    d_colp = colp_d;

    // ---- level sizes
    n.assign(1, NP);
    while (n.back() > MG_COARSE_MAX && static_cast<int>(n.size()) <= MG_MAX_LEVELS) n.push_back((n.back() + 7) / 8);
    if (n.back() > MG_COARSE_MAX || n.size() < 2) {
        why = n.size() < 2 ? "mesh too small for a hierarchy (at most 160 rows)"
                           : "more than 8 levels needed for a coarsest level of at most 160 rows";
        return false;
    }
    Lc = static_cast<int>(n.size()) - 1;

    // ---- partition: chunks of 4 slices, contiguous chunk ranges per CTA
    nchunks = (nslices + MG_CHUNK_SLICES - 1) / MG_CHUNK_SLICES;
    G = std::min(sms, nchunks);
    if (blocks_override > 0) G = std::min(G, blocks_override);
    if (G < 1) { why = "empty grid"; return false; }
    const int cpc = (nchunks + G - 1) / G;
    const int per_warp = (cpc * MG_CHUNK_SLICES + MG_NW - 1) / MG_NW;
    rmax = per_warp <= 1 ? 1 : per_warp <= 2 ? 2 : per_warp <= 4 ? 4 : per_warp <= 8 ? 8 : 0;
    if (!rmax) {
        why = "more than 8 slices per warp: the rows do not fit the register tiling";
        return false;
    }
    auto cta_pos = [&](int bb, long long& p0, long long& p1) {
        const int a = static_cast<int>(static_cast<long long>(bb) * nchunks / G);
        const int z = static_cast<int>(static_cast<long long>(bb + 1) * nchunks / G);
        p0 = 32LL * MG_CHUNK_SLICES * a;
        p1 = 32LL * std::min(MG_CHUNK_SLICES * z, nslices);
    };

    // ---- level-0 free rows (the solver's own node flags: bit0 fluid-connected,
    // bit2 fixed pressure) and pattern (real off-diagonal slots to free columns)
    std::vector<uint8_t> nflag(static_cast<size_t>(m.N), 0);
    MG_CUDA_OK(cudaMemcpy(nflag.data(), d_nflag, nflag.size(), cudaMemcpyDeviceToHost));
    std::vector<uint8_t> free0(static_cast<size_t>(NP), 0);
    for (int p = 0; p < NP; ++p) {
        const int node = P.row_node[static_cast<size_t>(p)];
        free0[static_cast<size_t>(p)] = node >= 0 && (nflag[static_cast<size_t>(node)] & 1) &&
                                        !(nflag[static_cast<size_t>(node)] & 4);
    }
    LevelPattern cur;
    cur.n = NP;
    cur.rptr.assign(static_cast<size_t>(NP) + 1, 0);
    cur.freerow.assign(free0.begin(), free0.end());
    nnz0 = 0;
    for (int p = 0; p < NP; ++p) {
        if (free0[static_cast<size_t>(p)]) {
            const int s = p >> 5, lane = p & 31;
            for (int k = 0; k < P.slice_w[static_cast<size_t>(s)]; ++k) {
                const long long t = P.slice_off[static_cast<size_t>(s)] + lane + 32LL * k;
                if (P.cptr[static_cast<size_t>(t) + 1] <= P.cptr[static_cast<size_t>(t)]) continue;   // padding slot
                const int c = colp[static_cast<size_t>(t)];
                if (!free0[static_cast<size_t>(c)]) continue;
                cur.col.push_back(c);
                cur.sid.push_back(static_cast<int>(t));
                ++nnz0;
            }
        }
        cur.rptr[static_cast<size_t>(p) + 1] = static_cast<int>(cur.col.size());
    }

    // ---- coarse levels: Galerkin patterns and their source lists
    W.assign(static_cast<size_t>(Lc) + 1, 0);
    h_lv.assign(MG_MAX_LEVELS, MgLevelDev{});
    std::vector<LevelPattern> pats(static_cast<size_t>(Lc) + 1);
    std::vector<std::vector<int>> lvcol(static_cast<size_t>(Lc) + 1);
    d_gptr.assign(static_cast<size_t>(Lc) + 1, nullptr);
    d_gent.assign(static_cast<size_t>(Lc) + 1, nullptr);
    gout.assign(static_cast<size_t>(Lc) + 1, 0);
    for (int l = 0; l < Lc; ++l) {
        const int nf = cur.n, nn = n[static_cast<size_t>(l) + 1];
        std::vector<std::vector<int>> ocol(static_cast<size_t>(nn));
        std::vector<std::vector<std::vector<int>>> osrc(static_cast<size_t>(nn));
        std::vector<std::vector<int>> dsrc(static_cast<size_t>(nn));
        std::vector<char> nfree(static_cast<size_t>(nn), 0);
        std::vector<std::pair<int, int>> tmp;
        for (int I = 0; I < nn; ++I) {
            tmp.clear();
            for (int i = 8 * I; i < std::min(8 * I + 8, nf); ++i) {
                if (!cur.freerow[static_cast<size_t>(i)]) continue;
                nfree[static_cast<size_t>(I)] = 1;
                dsrc[static_cast<size_t>(I)].push_back(-(i + 1));
                for (int q = cur.rptr[static_cast<size_t>(i)]; q < cur.rptr[static_cast<size_t>(i) + 1]; ++q)
                    tmp.emplace_back(cur.col[static_cast<size_t>(q)] >> 3, cur.sid[static_cast<size_t>(q)]);
            }
            std::sort(tmp.begin(), tmp.end());
            for (const auto& js : tmp) {
                if (js.first == I) {
                    dsrc[static_cast<size_t>(I)].push_back(js.second);
                    continue;
                }
                if (ocol[static_cast<size_t>(I)].empty() || ocol[static_cast<size_t>(I)].back() != js.first) {
                    ocol[static_cast<size_t>(I)].push_back(js.first);
                    osrc[static_cast<size_t>(I)].emplace_back();
                }
                osrc[static_cast<size_t>(I)].back().push_back(js.second);
            }
            std::sort(dsrc[static_cast<size_t>(I)].begin(), dsrc[static_cast<size_t>(I)].end());
        }
        int w = 0;
        for (int I = 0; I < nn; ++I) w = std::max(w, static_cast<int>(ocol[static_cast<size_t>(I)].size()));
        W[static_cast<size_t>(l) + 1] = w;
        // outputs: mg_slots(nn, w) off-diagonal slots (in slot order) then nn diagonals
        const long long ns = mg_slots(nn, w);
        std::vector<const std::vector<int>*> at(static_cast<size_t>(ns), nullptr);
        std::vector<int> colv(static_cast<size_t>(ns), -1);
        for (int I = 0; I < nn; ++I)
            for (int k = 0; k < static_cast<int>(ocol[static_cast<size_t>(I)].size()); ++k) {
                const long long s = mg_slot(I, k, w);
                colv[static_cast<size_t>(s)] = ocol[static_cast<size_t>(I)][static_cast<size_t>(k)];
                at[static_cast<size_t>(s)] = &osrc[static_cast<size_t>(I)][static_cast<size_t>(k)];
            }
        std::vector<long long> gp(static_cast<size_t>(ns) + nn + 1, 0);
        std::vector<int> ge;
        long long o = 0;
        for (; o < ns; ++o) {
            if (at[static_cast<size_t>(o)]) ge.insert(ge.end(), at[static_cast<size_t>(o)]->begin(), at[static_cast<size_t>(o)]->end());
            gp[static_cast<size_t>(o) + 1] = static_cast<long long>(ge.size());
        }
        for (int I = 0; I < nn; ++I, ++o) {
            ge.insert(ge.end(), dsrc[static_cast<size_t>(I)].begin(), dsrc[static_cast<size_t>(I)].end());
            gp[static_cast<size_t>(o) + 1] = static_cast<long long>(ge.size());
        }
        gout[static_cast<size_t>(l) + 1] = o;
        d_gptr[static_cast<size_t>(l) + 1] = upload(gp);
        d_gent[static_cast<size_t>(l) + 1] = upload(ge);
        lvcol[static_cast<size_t>(l) + 1] = colv;
        // the next level's pattern, with its entries' slots as source ids
        LevelPattern nx;
        nx.n = nn;
        nx.rptr.assign(static_cast<size_t>(nn) + 1, 0);
        nx.freerow = nfree;
        for (int I = 0; I < nn; ++I) {
            for (int k = 0; k < static_cast<int>(ocol[static_cast<size_t>(I)].size()); ++k) {
                nx.col.push_back(ocol[static_cast<size_t>(I)][static_cast<size_t>(k)]);
                nx.sid.push_back(static_cast<int>(mg_slot(I, k, w)));
            }
            nx.rptr[static_cast<size_t>(I) + 1] = static_cast<int>(nx.col.size());
        }
        pats[static_cast<size_t>(l) + 1] = nx;
        cur = std::move(nx);
    }

    // ---- level-0 halo of this partition
    std::vector<int> hptr(static_cast<size_t>(G) + 1, 0), hidx;
    std::vector<unsigned short> lcol(static_cast<size_t>(P.nslots), 0);
    int hmax0 = 0;
    long long smax = 0;
    {
        std::vector<int> cols;
        for (int bb = 0; bb < G; ++bb) {
            long long p0, p1;
            cta_pos(bb, p0, p1);
            const int sb = static_cast<int>(p0 / 32), se = static_cast<int>(p1 / 32);
            const long long a0 = P.slice_off[static_cast<size_t>(sb)], a1 = P.slice_off[static_cast<size_t>(se)];
            cols.assign(colp.begin() + a0, colp.begin() + a1);
            std::sort(cols.begin(), cols.end());
            cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
            if (cols.size() > 65535) { why = "a CTA halo exceeds 65,535 rows"; return false; }
            for (long long t = a0; t < a1; ++t)
                lcol[static_cast<size_t>(t)] = static_cast<unsigned short>(
                    std::lower_bound(cols.begin(), cols.end(), colp[static_cast<size_t>(t)]) - cols.begin());
            hidx.insert(hidx.end(), cols.begin(), cols.end());
            hptr[static_cast<size_t>(bb) + 1] = static_cast<int>(hidx.size());
            hmax0 = std::max(hmax0, static_cast<int>(cols.size()));
            smax = std::max(smax, a1 - a0);
        }
    }

    // ---- coarse levels' halos (own rows and the columns of their entries)
    std::vector<std::vector<int>> chptr(static_cast<size_t>(Lc)), chidx(static_cast<size_t>(Lc)),
        chown(static_cast<size_t>(Lc));
    std::vector<std::vector<unsigned short>> clcol(static_cast<size_t>(Lc));
    std::vector<int> chmax(static_cast<size_t>(Lc), 0);
    for (int l = 1; l < Lc; ++l) {
        const LevelPattern& pl = pats[static_cast<size_t>(l)];
        const int w = W[static_cast<size_t>(l)];
        long long sc = 1;
        for (int q = 0; q < l; ++q) sc *= 8;
        auto& hp = chptr[static_cast<size_t>(l)];
        auto& hi = chidx[static_cast<size_t>(l)];
        auto& ho = chown[static_cast<size_t>(l)];
        auto& lc = clcol[static_cast<size_t>(l)];
        hp.assign(static_cast<size_t>(G) + 1, 0);
        ho.assign(static_cast<size_t>(G), 0);
        lc.assign(static_cast<size_t>(mg_slots(pl.n, w)), 0xffff);
        std::vector<int> cols;
        for (int bb = 0; bb < G; ++bb) {
            long long p0, p1;
            cta_pos(bb, p0, p1);
            const int o = static_cast<int>((p0 + sc - 1) / sc);
            const int e = static_cast<int>(std::min<long long>(pl.n, (p1 + sc - 1) / sc));
            cols.clear();
            for (int I = o; I < e; ++I) {
                cols.push_back(I);
                for (int q = pl.rptr[static_cast<size_t>(I)]; q < pl.rptr[static_cast<size_t>(I) + 1]; ++q)
                    cols.push_back(pl.col[static_cast<size_t>(q)]);
            }
            std::sort(cols.begin(), cols.end());
            cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
            if (cols.size() > 65535) { why = "a CTA halo exceeds 65,535 rows"; return false; }
            ho[static_cast<size_t>(bb)] =
                o < e ? static_cast<int>(std::lower_bound(cols.begin(), cols.end(), o) - cols.begin()) : 0;
            for (int I = o; I < e; ++I)
                for (int k = 0; k < w; ++k) {
                    const size_t s = static_cast<size_t>(mg_slot(I, k, w));
                    const int J = lvcol[static_cast<size_t>(l)][s];
                    if (J >= 0)
                        lc[s] = static_cast<unsigned short>(std::lower_bound(cols.begin(), cols.end(), J) - cols.begin());
                }
            hi.insert(hi.end(), cols.begin(), cols.end());
            hp[static_cast<size_t>(bb) + 1] = static_cast<int>(hi.size());
            chmax[static_cast<size_t>(l)] = std::max(chmax[static_cast<size_t>(l)], static_cast<int>(cols.size()));
        }
    }

    // ---- shared memory: doubles (level 0: 3 per halo entry; coarse: 3 per
    // halo entry; coarsest r and x), then ints (halo rows), then the level-0
    // slot columns
    const int nc = n[static_cast<size_t>(Lc)];
    long long sd = 3LL * hmax0;
    for (int l = 1; l < Lc; ++l) {
        h_lv[static_cast<size_t>(l)].sd = static_cast<int>(sd);
        sd += 3LL * chmax[static_cast<size_t>(l)];
    }
    const long long sd_xc = sd;
    sd += 2LL * nc;
    long long si = hmax0;
    for (int l = 1; l < Lc; ++l) {
        h_lv[static_cast<size_t>(l)].si = static_cast<int>(si);
        si += chmax[static_cast<size_t>(l)];
    }
    smem = static_cast<size_t>(sd) * 8 + static_cast<size_t>(si) * 4 + static_cast<size_t>(smax) * 2 + 16;
    // 227 KB per CTA, less the kernel's static shared memory (< 5 KB)
    if (smem > 222 * 1024) {
        why = "shared memory " + std::to_string(smem / 1024) + " KB per CTA exceeds 222 KB";
        return false;
    }
    const void* fn = fn_mg(rmax);
    int per = 0;
    if (pcg_raise_smem_limit(fn, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, MG_NT, smem) != cudaSuccess || per * sms < G) {
        cudaGetLastError();
        why = "the solver kernel does not fit one CTA per SM with its shared memory";
        return false;
    }

    // ---- device arrays
    d_free0 = upload(free0);
    fine = PcgDev{};
    fine.halo_ptr = upload(hptr);
    fine.halo_idx = upload(hidx);
    fine.lcol = upload(lcol);
    fine.halo_max = hmax0;
    fine.slot_max = static_cast<int>(smax);
    for (int l = 1; l <= Lc; ++l) {
        MgLevelDev& L = h_lv[static_cast<size_t>(l)];
        const int nl = n[static_cast<size_t>(l)], w = W[static_cast<size_t>(l)];
        L.n = nl;
        L.W = w;
        L.tpr = level_tpr(l);
        L.col = upload(lvcol[static_cast<size_t>(l)]);
        L.val = zeros<double>(static_cast<size_t>(mg_slots(nl, w)) + nl);
        L.wd = zeros<double>(static_cast<size_t>(nl));
        L.rho = zeros<double>(static_cast<size_t>(nl));
        L.x = zeros<double>(static_cast<size_t>(nl));
        if (l < Lc) {
            L.hptr = upload(chptr[static_cast<size_t>(l)]);
            L.hidx = upload(chidx[static_cast<size_t>(l)]);
            L.hown = upload(chown[static_cast<size_t>(l)]);
            L.lcol = upload(clcol[static_cast<size_t>(l)]);
            L.hmax = chmax[static_cast<size_t>(l)];
        }
    }
    d_dense = zeros<double>(static_cast<size_t>(nc) * nc);
    dev = MgDev{};
    dev.Lc = Lc;
    dev.nchunks = nchunks;
    dev.nc = nc;
    dev.sd_xc = static_cast<int>(sd_xc);
    dev.si_end = static_cast<int>(si);
    dev.lv = upload(h_lv);
    dev.ainv = d_dense;
    dev.rho0 = zeros<double>(static_cast<size_t>(NP));
    dev.wd0 = zeros<double>(static_cast<size_t>(NP));
    dev.part = zeros<double>(static_cast<size_t>(2) * 4 * nchunks);
    dev.bar = zeros<unsigned long long>(1);
    return true;
}

void MgHierarchy::release()
{
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
}

void MgHierarchy::setup(const double* d_val, const double* pdiag, const int* row_node, cudaStream_t st)
{
    const int T = 256;
    k_mg_weights0<<<(NP + T - 1) / T, T, 0, st>>>(d_slice_off, d_slice_w, d_colp, d_val, pdiag, row_node, d_free0, NP,
                                                  dev.wd0);
    for (int l = 1; l <= Lc; ++l) {
        const MgLevelDev& L = h_lv[static_cast<size_t>(l)];
        const long long no = gout[static_cast<size_t>(l)];
        if (l == 1)
            k_mg_galerkin<<<static_cast<unsigned>((no + T - 1) / T), T, 0, st>>>(
                d_gptr[1], d_gent[1], no, d_val, pdiag, row_node, L.val);
        else {
            const MgLevelDev& Lp = h_lv[static_cast<size_t>(l) - 1];
            k_mg_galerkin<<<static_cast<unsigned>((no + T - 1) / T), T, 0, st>>>(
                d_gptr[static_cast<size_t>(l)], d_gent[static_cast<size_t>(l)], no, Lp.val,
                Lp.val + mg_slots(Lp.n, Lp.W), nullptr, L.val);
        }
        if (l < Lc) k_mg_weights<<<(L.n + T - 1) / T, T, 0, st>>>(L.val, L.col, L.n, L.W, L.wd);
    }
    const MgLevelDev& Lc_ = h_lv[static_cast<size_t>(Lc)];
    k_mg_dense<<<(Lc_.n + T - 1) / T, T, 0, st>>>(Lc_.val, Lc_.col, Lc_.n, Lc_.W, d_dense);
    coarse_invert_launch(Lc_.n, d_dense, st);
}

void MgHierarchy::launch(const PcgDev& D, cudaStream_t st)
{
    PcgDev d = D;
    d.halo_ptr = fine.halo_ptr;
    d.halo_idx = fine.halo_idx;
    d.lcol = fine.lcol;
    d.halo_max = fine.halo_max;
    d.slot_max = fine.slot_max;
    MgDev m = dev;
    MG_CUDA_OK(cudaMemsetAsync(dev.bar, 0, sizeof(unsigned long long), st));
    void* args[] = {&d, &m};
    MG_CUDA_OK(cudaLaunchCooperativeKernel(fn_mg(rmax), dim3(G), dim3(MG_NT), args, smem, st));
}

}  // namespace cbs3d
