// Tangent-linear (TLM) and adjoint of the CBS step with respect to a nodal
// body force f (extension: the reference has no body force and no
// derivatives).  With a fixed time step the pressure operator, the lumped
// diagonals and the boundary programs are constant, so one step is
//
//   Step 1   u*  = B1( u^n + m * (R(u^n) + M_f f) )      R: element residual, quadratic in u^n
//   Step 2   A p = G* u* + G1 u^n                         (free rows; fixed rows hold p_bc)
//   Step 3   u^{n+1} = B3( u* - m * Gp p )
//
// with m = elcoe2, M_f the fluid lumped mass, B the velocity boundary
// program (projections, fixed values, outlet backflow removal) and G the
// Step-2 assembly.  The TLM carries (du, dp) forward; the adjoint runs the
// transposed steps backward: element scatters of the forward become element
// gathers of nodal adjoints followed by deterministic node gathers, and the
// pressure adjoint reuses the symmetric PCG operator.  The element Jacobian of
// R comes from forward-mode dual numbers (exact for a quadratic residual).
//
// Forward states for the reverse sweep come from checkpoints of (u, p) every
// `every` steps; each segment is recomputed once into a buffer and every step
// is recomputed once more with its Step-1/Step-3 intermediates captured.
// Deterministic kernels make every recomputation bit-identical to the
// original forward run.
#include "ctx.cuh"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace {

constexpr double F1 = 1.0 / 24.0, F2 = 1.0 / 12.0, F3 = 1.0 / 6.0, F4 = 1.0 / 3.0;
constexpr double FD1 = 1.0 / 6.0, FD2 = 1.0 / 3.0;
// nodes of face f (opposite local node f), as the forward kernels use them
__constant__ int c_face[4][3] = {{2, 1, 3}, {2, 3, 0}, {0, 3, 1}, {0, 1, 2}};

__device__ __forceinline__ int nd(const int4& n, int a) { return a == 0 ? n.x : a == 1 ? n.y : a == 2 ? n.z : n.w; }
__device__ __forceinline__ int fedge(uint8_t packed, int f) { return (packed >> (2 * f)) & 3; }

// ------------------------------------------------------------ dual numbers
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.v * b.d + a.d * b.v}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual zero(Dual) { return {0.0, 0.0}; }

// Step-1 element residual of a fluid element as a function of its nodal
// u^n (the terms of k_step1_elem: Galerkin convection with its boundary
// faces, characteristic correction, diffusion), evaluated on dual numbers.
template <typename R>
__device__ void s1_residual(const DevState& S, int e, const R (&lu)[3][4], R (&lr)[3][4])
{
    const int E = S.P.E;
    const double det = S.detJ[e];
    double g[3][4];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < 4; ++a) g[d][a] = S.grad[(size_t)(d * 4 + a) * E + e];
    const uint8_t fe = S.fedge[e];
    const R z = zero(lu[0][0]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int a = 0; a < 4; ++a) lr[i][a] = z;
    // Galerkin convection
    R ls[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            R s = z;
#pragma unroll
            for (int a = 0; a < 4; ++a) s = s + lu[j][a] * lu[i][a];
            ls[i][j] = s;
        }
    const double vf = det * F1;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) lr[i][a] = lr[i][a] + ls[i][j] * (g[j][a] * vf);
    for (int is = 0; is < 4; ++is) {
        if (fedge(fe, is) == 0) continue;
        for (int j = 0; j < 3; ++j) {
            const double ff = S.annxf[(size_t)(is * 4 + j) * E + e] * F2;
            for (int fn = 0; fn < 3; ++fn) {
                const int a = c_face[is][fn];
                for (int i = 0; i < 3; ++i) {
                    const R la = lu[j][a] * lu[i][a];
                    const R lis = lu[j][is] * lu[i][is];
                    lr[i][a] = lr[i][a] - (ls[i][j] - lis + la) * ff;
                }
            }
        }
    }
    // characteristic correction
    R lsk[3][3];
    {
        R sj[3], um[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            R s = z, u = z;
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int a = 0; a < 4; ++a) s = s + (lu[j][a] * lu[i][a]) * g[j][a];
#pragma unroll
            for (int a = 0; a < 4; ++a) u = u + lu[i][a];
            sj[i] = s;
            um[i] = u / 4.0;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int k = 0; k < 3; ++k) lsk[i][k] = um[k] * sj[i];
    }
    const double dt = S.delte[e];
    const double ld = 0.5 * dt * det * F3, ld2 = 0.5 * dt * F4;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) lr[i][a] = lr[i][a] - lsk[i][k] * (g[k][a] * ld);
    for (int is = 0; is < 4; ++is) {
        if (fedge(fe, is) == 0) continue;
        for (int k = 0; k < 3; ++k) {
            const double ff = S.annxf[(size_t)(is * 4 + k) * E + e] * ld2;
            for (int fn = 0; fn < 3; ++fn) {
                const int a = c_face[is][fn];
                for (int i = 0; i < 3; ++i) lr[i][a] = lr[i][a] + lsk[i][k] * ff;
            }
        }
    }
    // diffusion
    double nu = S.P.ani;
    if (S.P.dimensional_material) nu = S.mu[e] / S.rho[e];
    R gu[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            R s = z;
#pragma unroll
            for (int a = 0; a < 4; ++a) s = s + lu[i][a] * g[j][a];
            gu[i][j] = s;
        }
    const double vd = nu * det * FD1;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int j = 0; j < 3; ++j) lr[i][a] = lr[i][a] - gu[i][j] * (g[j][a] * vd);
    const double fdf = nu * FD2;
    for (int is = 0; is < 4; ++is) {
        if (fedge(fe, is) == 0) continue;
        for (int j = 0; j < 3; ++j) {
            const double ff = S.annxf[(size_t)(is * 4 + j) * E + e] * fdf;
            for (int i = 0; i < 3; ++i)
                for (int fn = 0; fn < 3; ++fn) {
                    const int a = c_face[is][fn];
                    lr[i][a] = lr[i][a] + gu[i][j] * ff;
                }
        }
    }
}

// ------------------------------------------------- velocity boundary program
// The forward program maps the pre-BC value up to the post-BC value; these
// are its derivative (tangent) and the transpose of that derivative
// (adjoint) at up, with the outlet backflow branches taken as the forward
// takes them.
__device__ void bc_tangent(const DevState& S, int i, const double (&up)[3], double (&t)[3])
{
    const int idx = S.vbc_idx[i];
    if (idx < 0) return;
    const VelBC b = static_cast<const VelBC*>(S.vbc)[idx];
    if (b.flags & VBC_SOLID) { t[0] = t[1] = t[2] = 0.0; return; }
    double u[3] = {up[0], up[1], up[2]};
    for (int k = 0; k < b.sym_cnt; ++k) {
        const double* n = S.vbc_nrm + 3 * (b.sym_beg + k);
        const double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
        const double tn = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
        for (int d = 0; d < 3; ++d) { u[d] -= un * n[d]; t[d] -= tn * n[d]; }
    }
    if (b.flags & VBC_FIXED) {
        for (int d = 0; d < 3; ++d) { u[d] = b.fix[d]; t[d] = 0.0; }
    }
    for (int k = 0; k < b.out_cnt; ++k) {
        const double* n = S.vbc_nrm + 3 * (b.out_beg + k);
        const double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
        if (un < 0.0) {
            const double tn = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
            for (int d = 0; d < 3; ++d) { u[d] -= un * n[d]; t[d] -= tn * n[d]; }
        }
    }
}

__device__ void bc_adjoint(const DevState& S, int i, const double (&up)[3], double (&l)[3])
{
    const int idx = S.vbc_idx[i];
    if (idx < 0) return;
    const VelBC b = static_cast<const VelBC*>(S.vbc)[idx];
    if (b.flags & VBC_SOLID) { l[0] = l[1] = l[2] = 0.0; return; }
    double u[3] = {up[0], up[1], up[2]};
    for (int k = 0; k < b.sym_cnt; ++k) {
        const double* n = S.vbc_nrm + 3 * (b.sym_beg + k);
        const double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
        for (int d = 0; d < 3; ++d) u[d] -= un * n[d];
    }
    if (b.flags & VBC_FIXED)
        for (int d = 0; d < 3; ++d) u[d] = b.fix[d];
    unsigned taken = 0u;   // outlet projections the forward applies (at most 32 per node)
    for (int k = 0; k < b.out_cnt && k < 32; ++k) {
        const double* n = S.vbc_nrm + 3 * (b.out_beg + k);
        const double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
        if (un < 0.0) {
            taken |= 1u << k;
            for (int d = 0; d < 3; ++d) u[d] -= un * n[d];
        }
    }
    // transposes in reverse order; each projection I - n n^T is symmetric
    for (int k = (b.out_cnt < 32 ? b.out_cnt : 32) - 1; k >= 0; --k) {
        if (!(taken & (1u << k))) continue;
        const double* n = S.vbc_nrm + 3 * (b.out_beg + k);
        const double ln = l[0] * n[0] + l[1] * n[1] + l[2] * n[2];
        for (int d = 0; d < 3; ++d) l[d] -= ln * n[d];
    }
    if (b.flags & VBC_FIXED) { l[0] = l[1] = l[2] = 0.0; return; }
    for (int k = b.sym_cnt - 1; k >= 0; --k) {
        const double* n = S.vbc_nrm + 3 * (b.sym_beg + k);
        const double ln = l[0] * n[0] + l[1] * n[1] + l[2] * n[2];
        for (int d = 0; d < 3; ++d) l[d] -= ln * n[d];
    }
}

// --------------------------------------------------------------- kernels
// Element-node buffers are [row][E]; gathers sum a node's fluid elements in
// element order (deterministic).
__global__ void k_gather3(DevState S, const double* eb, double* out, int accumulate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r[3] = {0.0, 0.0, 0.0};
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2, a = S.n2e[k] & 3;
        if (S.mat[e] != 0) continue;
        for (int d = 0; d < 3; ++d) r[d] += eb[(size_t)(d * 4 + a) * E + e];
    }
    for (int d = 0; d < 3; ++d) out[3 * i + d] = accumulate ? out[3 * i + d] + r[d] : r[d];
}

// per element one value per component (the same for the 4 nodes)
__global__ void k_gather3_elem(DevState S, const double* eb, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r[3] = {0.0, 0.0, 0.0};
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2;
        if (S.mat[e] != 0) continue;
        for (int d = 0; d < 3; ++d) r[d] += eb[(size_t)d * E + e];
    }
    for (int d = 0; d < 3; ++d) out[3 * i + d] += r[d];
}

__global__ void k_gather1(DevState S, const double* eb, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r = 0.0;
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2, a = S.n2e[k] & 3;
        if (S.mat[e] != 0) continue;
        r += eb[(size_t)a * E + e];
    }
    out[i] = r;
}

// TLM of the Step-1 element residual at u1 in direction du1
__global__ void k_tlm_s1_elem(DevState S, const double* u1, const double* du1, double* eb)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E || S.mat[e] != 0) return;
    const int4 n = S.intma[e];
    Dual lu[3][4], lr[3][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) lu[i][a] = Dual{u1[3 * nd(n, a) + i], du1[3 * nd(n, a) + i]};
    s1_residual(S, e, lu, lr);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int a = 0; a < 4; ++a) eb[(size_t)(i * 4 + a) * E + e] = lr[i][a].d;
}

// Adjoint of the Step-1 element residual: (dR/du1)^T mu, one dual sweep per
// element input.
__global__ void k_adj_s1_elem(DevState S, const double* u1, const double* mu, double* eb)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E || S.mat[e] != 0) return;
    const int4 n = S.intma[e];
    double u[3][4], w[3][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            u[i][a] = u1[3 * nd(n, a) + i];
            w[i][a] = mu[3 * nd(n, a) + i];
        }
    for (int jb = 0; jb < 12; ++jb) {
        Dual lu[3][4], lr[3][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i) lu[i][a] = Dual{u[i][a], (i * 4 + a == jb) ? 1.0 : 0.0};
        s1_residual(S, e, lu, lr);
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int a = 0; a < 4; ++a) acc += w[i][a] * lr[i][a].d;
        eb[(size_t)jb * E + e] = acc;
    }
}

// Step-1 node TLM: du* = B1'(u*_pre) (du1 + m (dR + M_f df))
__global__ void k_tlm_s1_node(DevState S, const double* u1, const double* rhs_s1, const double* dr,
                              const double* mfl, const double* df, const double* du1, double* dstar)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const double m = S.elcoe2[i];
    double up[3], t[3];
    for (int d = 0; d < 3; ++d) {
        up[d] = u1[3 * i + d] + rhs_s1[3 * i + d] * m;
        const double f = df ? mfl[i] * df[3 * i + d] : 0.0;
        t[d] = du1[3 * i + d] + (dr[3 * i + d] + f) * m;
    }
    bc_tangent(S, i, up, t);
    for (int d = 0; d < 3; ++d) dstar[3 * i + d] = t[d];
}

// Step-3 node TLM: du = B3'(u_pre) (du* - m Gp dp), Gp dp gathered from eb[d*E+e]
__global__ void k_tlm_s3_node(DevState S, const double* ustar, const double* rhs_s3, const double* eb,
                              const double* dstar, double* du)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r[3] = {0.0, 0.0, 0.0};
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2;
        if (S.mat[e] != 0) continue;
        for (int d = 0; d < 3; ++d) r[d] -= eb[(size_t)d * E + e];
    }
    const double m = S.elcoe2[i];
    double up[3], t[3];
    for (int d = 0; d < 3; ++d) {
        up[d] = ustar[3 * i + d] + rhs_s3[3 * i + d] * m;
        t[d] = dstar[3 * i + d] + r[d] * m;
    }
    bc_tangent(S, i, up, t);
    for (int d = 0; d < 3; ++d) du[3 * i + d] = t[d];
}

// Step-3 node adjoint: l_pre = B3'^T l; l* = l_pre; mu3 = m l_pre
__global__ void k_adj_s3_node(DevState S, const double* ustar, const double* rhs_s3, const double* lam,
                              double* lstar, double* mu3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const double m = S.elcoe2[i];
    double up[3], l[3];
    for (int d = 0; d < 3; ++d) {
        up[d] = ustar[3 * i + d] + rhs_s3[3 * i + d] * m;
        l[d] = lam[3 * i + d];
    }
    bc_adjoint(S, i, up, l);
    for (int d = 0; d < 3; ++d) {
        lstar[3 * i + d] = l[d];
        mu3[3 * i + d] = m * l[d];
    }
}

// Step-3 element adjoint: lambda_p contributions -vol4 grad_a . sum_b mu3_b
__global__ void k_adj_s3_elem(DevState S, const double* mu3, double* eb)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E || S.mat[e] != 0) return;
    const int4 n = S.intma[e];
    double s[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < 4; ++a)
        for (int d = 0; d < 3; ++d) s[d] += mu3[3 * nd(n, a) + d];
    const double vol4 = S.detJ[e] * F1;
    for (int a = 0; a < 4; ++a) {
        double v = 0.0;
        for (int d = 0; d < 3; ++d) v += S.grad[(size_t)(d * 4 + a) * E + e] * s[d];
        eb[(size_t)a * E + e] = -vol4 * v;
    }
}

// Step-2 element adjoint: the u* part (one value per component, eb3) and the
// u^n boundary-face part (per element node, eb12)
__global__ void k_adj_s2_elem(DevState S, const double* lb, double* eb3, double* eb12)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    for (int r = 0; r < 12; ++r) eb12[(size_t)r * E + e] = 0.0;
    if (S.mat[e] != 0) return;
    const int4 n = S.intma[e];
    const double vol4 = S.detJ[e] * F1;
    for (int d = 0; d < 3; ++d) {
        double c = 0.0;
        for (int a = 0; a < 4; ++a) c += S.grad[(size_t)(d * 4 + a) * E + e] * lb[nd(n, a)];
        eb3[(size_t)d * E + e] = vol4 * c;
    }
    const uint8_t fe = S.fedge[e];
    for (int is = 0; is < 4; ++is) {
        if (fedge(fe, is) != 1) continue;
        double sl = 0.0;
        for (int q = 0; q < 3; ++q) sl += lb[nd(n, c_face[is][q])];
        for (int d = 0; d < 3; ++d) {
            const double nf = S.annxf[(size_t)(is * 4 + d) * E + e] * F2;
            for (int q = 0; q < 3; ++q) {
                const int a = c_face[is][q];
                eb12[(size_t)(d * 4 + a) * E + e] -= nf * (sl + lb[nd(n, a)]);
            }
        }
    }
}

// Step-1 node adjoint: l_pre = B1'^T l*; l_n += l_pre; mu1 = m l_pre; grad += M_f mu1
__global__ void k_adj_s1_node(DevState S, const double* u1, const double* rhs_s1, const double* lstar,
                              const double* mfl, double* ln, double* mu1, double* grad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const double m = S.elcoe2[i];
    double up[3], l[3];
    for (int d = 0; d < 3; ++d) {
        up[d] = u1[3 * i + d] + rhs_s1[3 * i + d] * m;
        l[d] = lstar[3 * i + d];
    }
    bc_adjoint(S, i, up, l);
    for (int d = 0; d < 3; ++d) {
        ln[3 * i + d] += l[d];
        mu1[3 * i + d] = m * l[d];
        grad[3 * i + d] += mfl[i] * m * l[d];
    }
}

// ------------------------------------------------------------------ driver
// Work space of one tangent or adjoint run on a context; the context's
// fields, step counter and physical time are restored when it ends.
class Run {
public:
    explicit Run(cbs3d_ctx& ctx) : c(ctx), N(ctx.m.N), E(ctx.m.E)
    {
        if (c.m.p.step2_check > 0)
            throw Error(CBS3D_INVALID_INPUT, "tangent/adjoint runs do not support the Step-2 time-step correction (step2_check > 0)");
        st = c.st;
        u1 = alloc(3 * N); rhs_s1 = alloc(3 * N); ustar = alloc(3 * N); rhs_s3 = alloc(3 * N);
        v0 = alloc(3 * N); v1 = alloc(3 * N); v2 = alloc(3 * N); v3 = alloc(3 * N);
        s0 = alloc(N); s1 = alloc(N); pd = alloc(N); mfl = alloc(N); zpfix = alloc(N);
        eb12 = alloc(12 * E); eb3 = alloc(3 * E);
        su = alloc(3 * N); sp = alloc(N); stt = alloc(N);
        CUDA_OK(cudaMemsetAsync(zpfix, 0, N * sizeof(double), st));
        k_mass_fluid<<<nb(static_cast<long long>(N)), T, 0, st>>>(c.S, mfl);
        // save the state
        CUDA_OK(cudaMemcpyAsync(su, c.S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaMemcpyAsync(sp, c.S.pres, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaMemcpyAsync(stt, c.S.temp, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaMemcpyAsync(&rtime0, c.S.dscal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        it0 = c.iitime;
        time_pcg0 = c.opt.time_pcg;
        c.opt.time_pcg = 0;
        c.ensure_log(1);
        c.reset_status();
    }
    ~Run()
    {
        c.opt.time_pcg = time_pcg0;
        pcg.release();
        for (void* p : ptrs) cudaFree(p);
    }
    void check_fixed_dt(int nsteps) const
    {
        for (int s = 1; s <= nsteps; ++s)
            if (!c.fixed_dt(it0 + s))
                throw Error(CBS3D_INVALID_INPUT, "tangent/adjoint runs need a fixed time step (dtfixed > 0 or ilots <= -1)");
    }
    void restore()
    {
        CUDA_OK(cudaMemcpyAsync(c.S.unkno, su, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaMemcpyAsync(c.S.pres, sp, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaMemcpyAsync(c.S.temp, stt, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaMemcpyAsync(c.S.dscal + 1, &rtime0, sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaStreamSynchronize(st));
        c.iitime = it0;
    }
    // one forward step of the context, optionally keeping the intermediates
    // the tangent and adjoint steps linearise about
    void forward(bool capture)
    {
        const int it = c.iitime + 1;
        c.enqueue_pre(it);
        if (capture) {
            CUDA_OK(cudaMemcpyAsync(u1, c.S.unkn1, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            CUDA_OK(cudaMemcpyAsync(rhs_s1, c.S.rhs, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            CUDA_OK(cudaMemcpyAsync(ustar, c.S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        }
        c.stage_solve();
        c.enqueue_post(it);
        if (capture) CUDA_OK(cudaMemcpyAsync(rhs_s3, c.S.rhs, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        c.launches += c.kernels_outside_solve(it) + 1 + c.pcg.launches_per_solve();
        c.iitime = it;
    }
    // the pressure operator solve with zero fixed values (tangent/adjoint systems)
    void solve(double* x, double* b)
    {
        if (!pcg_ready) {
            pcg.inner_tol = 1.0e-5;
            pcg.init(c.m, c.S.nflag, zpfix, c.S.status, c.opt.device, 0, false, 0);
            pcg_ready = true;
        }
        pcg.assemble_from_state(c.S, st);
        CUDA_OK(cudaMemsetAsync(x, 0, N * sizeof(double), st));
        CUDA_OK(cudaMemcpyAsync(pd, c.S.pdiag, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        const cbs3d_params& P = c.m.p;
        pcg.solve(x, b, pd, P.cg_preconditioner, P.cg_conv_test, P.cg_max_iter, P.relToler, P.absToler, st, false);
    }
    // tangent step: v0 = du^n in, du^{n+1} out (after forward(true))
    void tangent(const double* df)
    {
        const unsigned gn = nb(static_cast<long long>(N)), ge = nb(static_cast<long long>(E));
        k_tlm_s1_elem<<<ge, T, 0, st>>>(c.S, u1, v0, eb12);
        k_gather3<<<gn, T, 0, st>>>(c.S, eb12, v1, 0);
        k_tlm_s1_node<<<gn, T, 0, st>>>(c.S, u1, rhs_s1, v1, mfl, df, v0, v2);
        DevState S2 = c.S;
        S2.unkno = v2; S2.unkn1 = v0; S2.rhs1 = s0; S2.elbuf = eb12;
        k_step2_elem<<<ge, T, 0, st>>>(S2);
        k_step2_node<<<gn, T, 0, st>>>(S2);
        solve(s1, s0);
        DevState S3 = c.S;
        S3.pres = s1; S3.elbuf = eb12;
        k_step3_elem<<<ge, T, 0, st>>>(S3);
        k_tlm_s3_node<<<gn, T, 0, st>>>(c.S, ustar, rhs_s3, eb12, v2, v0);
        CUDA_OK(cudaGetLastError());
    }
    // adjoint step: v0 = adjoint of u^{n+1} in, of u^n out; grad += dJ/df part
    void adjoint(double* grad)
    {
        const unsigned gn = nb(static_cast<long long>(N)), ge = nb(static_cast<long long>(E));
        k_adj_s3_node<<<gn, T, 0, st>>>(c.S, ustar, rhs_s3, v0, v1, v2);
        k_adj_s3_elem<<<ge, T, 0, st>>>(c.S, v2, eb12);
        k_gather1<<<gn, T, 0, st>>>(c.S, eb12, s0);
        solve(s1, s0);
        k_adj_s2_elem<<<ge, T, 0, st>>>(c.S, s1, eb3, eb12);
        k_gather3_elem<<<gn, T, 0, st>>>(c.S, eb3, v1);
        k_gather3<<<gn, T, 0, st>>>(c.S, eb12, v3, 0);
        k_adj_s1_node<<<gn, T, 0, st>>>(c.S, u1, rhs_s1, v1, mfl, v3, v2, grad);
        k_adj_s1_elem<<<ge, T, 0, st>>>(c.S, u1, v2, eb12);
        k_gather3<<<gn, T, 0, st>>>(c.S, eb12, v3, 1);
        CUDA_OK(cudaMemcpyAsync(v0, v3, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaGetLastError());
    }
    // J = 1/2 sum_i w_i |u_i|^2 of the current u; optionally lambda_N = w u into v0
    double objective(const double* w, bool seed)
    {
        std::vector<double> u(3 * N);
        CUDA_OK(cudaMemcpyAsync(u.data(), c.S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        c.check_status();
        double J = 0.0;
        for (size_t i = 0; i < N; ++i)
            J += 0.5 * w[i] * (u[3 * i] * u[3 * i] + u[3 * i + 1] * u[3 * i + 1] + u[3 * i + 2] * u[3 * i + 2]);
        if (seed) {
            for (size_t i = 0; i < N; ++i)
                for (int d = 0; d < 3; ++d) u[3 * i + d] *= w[i];
            CUDA_OK(cudaMemcpyAsync(v0, u.data(), 3 * N * sizeof(double), cudaMemcpyHostToDevice, st));
            CUDA_OK(cudaStreamSynchronize(st));
        }
        return J;
    }
    double dot_w(const double* w, const double* dvec)
    {
        std::vector<double> u(3 * N), d(3 * N);
        CUDA_OK(cudaMemcpyAsync(u.data(), c.S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(d.data(), dvec, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        double s = 0.0;
        for (size_t i = 0; i < N; ++i)
            s += w[i] * (u[3 * i] * d[3 * i] + u[3 * i + 1] * d[3 * i + 1] + u[3 * i + 2] * d[3 * i + 2]);
        return s;
    }
    double* alloc(size_t n)
    {
        void* p = nullptr;
        CUDA_OK(cudaMalloc(&p, (n ? n : 1) * sizeof(double)));
        ptrs.push_back(p);
        return static_cast<double*>(p);
    }

    cbs3d_ctx& c;
    size_t N, E;
    cudaStream_t st = nullptr;
    std::vector<void*> ptrs;
    double *u1, *rhs_s1, *ustar, *rhs_s3, *v0, *v1, *v2, *v3, *s0, *s1, *pd, *mfl, *zpfix, *eb12, *eb3;
    double *su, *sp, *stt;
    double rtime0 = 0.0;
    int it0 = 0, time_pcg0 = 0;
    PcgEngine pcg;
    bool pcg_ready = false;
};

template <typename F>
cbs3d_status run_guarded(cbs3d_ctx* c, F&& f)
{
    if (!c) return CBS3D_INVALID_INPUT;
    try {
        CUDA_OK(cudaSetDevice(c->opt.device));
        f();
        c->err.clear();
        return CBS3D_OK;
    } catch (const Error& e) {
        c->err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        c->err = e.what();
        return CBS3D_INTERNAL;
    }
}

}  // namespace

extern "C" {

cbs3d_status cbs3d_set_body_force(cbs3d_ctx* c, const double* f)
{
    return run_guarded(c, [&] {
        const size_t N = c->m.N;
        if (!f) {
            c->S.bforce = nullptr;
            c->S.mfluid = nullptr;
        } else {
            if (!c->d_bforce) {
                c->d_bforce = c->buf.alloc<double>(3 * N);
                c->d_mfluid = c->buf.alloc<double>(N);
                k_mass_fluid<<<nb(static_cast<long long>(N)), T, 0, c->st>>>(c->S, c->d_mfluid);
            }
            CUDA_OK(cudaMemcpyAsync(c->d_bforce, f, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->st));
            CUDA_OK(cudaStreamSynchronize(c->st));
            c->S.bforce = c->d_bforce;
            c->S.mfluid = c->d_mfluid;
        }
        // the captured step graph holds the previous device-state view
        if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
    });
}

cbs3d_status cbs3d_objective_run(cbs3d_ctx* c, int nsteps, const double* w, double* J)
{
    return run_guarded(c, [&] {
        if (nsteps < 1 || !w || !J) throw Error(CBS3D_INVALID_INPUT, "cbs3d_objective_run - nsteps >= 1, w and J required");
        Run r(*c);
        for (int s = 0; s < nsteps; ++s) r.forward(false);
        *J = r.objective(w, false);
        r.restore();
    });
}

cbs3d_status cbs3d_tlm_run(cbs3d_ctx* c, int nsteps, const double* w, const double* df, double* J, double* dJ)
{
    return run_guarded(c, [&] {
        if (nsteps < 1 || !w || !df || !J || !dJ) throw Error(CBS3D_INVALID_INPUT, "cbs3d_tlm_run - nsteps >= 1, w, df, J and dJ required");
        Run r(*c);
        r.check_fixed_dt(nsteps);
        double* ddf = r.alloc(3 * r.N);
        CUDA_OK(cudaMemcpyAsync(ddf, df, 3 * r.N * sizeof(double), cudaMemcpyHostToDevice, r.st));
        CUDA_OK(cudaMemsetAsync(r.v0, 0, 3 * r.N * sizeof(double), r.st));
        for (int s = 0; s < nsteps; ++s) {
            r.forward(true);
            r.tangent(ddf);
        }
        *J = r.objective(w, false);
        *dJ = r.dot_w(w, r.v0);
        r.restore();
    });
}

cbs3d_status cbs3d_adjoint_run(cbs3d_ctx* c, int nsteps, int every, const double* w, double* J, double* grad)
{
    return run_guarded(c, [&] {
        if (nsteps < 1 || every < 1 || !w || !J || !grad)
            throw Error(CBS3D_INVALID_INPUT, "cbs3d_adjoint_run - nsteps >= 1, every >= 1, w, J and grad required");
        Run r(*c);
        r.check_fixed_dt(nsteps);
        const size_t N = r.N;
        const int ncp = (nsteps + every - 1) / every;
        std::vector<double*> cpu(static_cast<size_t>(ncp)), cpp(static_cast<size_t>(ncp));
        for (int k = 0; k < ncp; ++k) { cpu[static_cast<size_t>(k)] = r.alloc(3 * N); cpp[static_cast<size_t>(k)] = r.alloc(N); }
        const int seg = every < nsteps ? every : nsteps;
        std::vector<double*> sgu(static_cast<size_t>(seg)), sgp(static_cast<size_t>(seg));
        for (int k = 0; k < seg; ++k) { sgu[static_cast<size_t>(k)] = r.alloc(3 * N); sgp[static_cast<size_t>(k)] = r.alloc(N); }
        double* G = r.alloc(3 * N);
        CUDA_OK(cudaMemsetAsync(G, 0, 3 * N * sizeof(double), r.st));
        auto save = [&](double* du, double* dp) {
            CUDA_OK(cudaMemcpyAsync(du, c->S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
            CUDA_OK(cudaMemcpyAsync(dp, c->S.pres, N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
        };
        auto load = [&](const double* du, const double* dp) {
            CUDA_OK(cudaMemcpyAsync(c->S.unkno, du, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
            CUDA_OK(cudaMemcpyAsync(c->S.pres, dp, N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
        };
        // forward sweep with checkpoints of (u, p) every `every` steps
        for (int s = 0; s < nsteps; ++s) {
            if (s % every == 0) save(cpu[static_cast<size_t>(s / every)], cpp[static_cast<size_t>(s / every)]);
            r.forward(false);
        }
        *J = r.objective(w, true);   // seeds v0 = dJ/du^N
        // reverse sweep, one checkpoint segment at a time
        for (int k = ncp - 1; k >= 0; --k) {
            const int a = k * every, b = (a + every < nsteps) ? a + every : nsteps;
            load(cpu[static_cast<size_t>(k)], cpp[static_cast<size_t>(k)]);
            c->iitime = r.it0 + a;
            for (int s = a; s < b; ++s) {
                save(sgu[static_cast<size_t>(s - a)], sgp[static_cast<size_t>(s - a)]);
                r.forward(false);
            }
            for (int s = b - 1; s >= a; --s) {
                load(sgu[static_cast<size_t>(s - a)], sgp[static_cast<size_t>(s - a)]);
                c->iitime = r.it0 + s;
                r.forward(true);
                r.adjoint(G);
            }
        }
        CUDA_OK(cudaMemcpyAsync(grad, G, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, r.st));
        CUDA_OK(cudaStreamSynchronize(r.st));
        c->check_status();
        r.restore();
    });
}

}  // extern "C"
