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

// Neumaier's compensated summation (host): the objective and the directional
// derivatives are sums over every node, and a plain running sum over ~28,000
// terms rounds by several ulp of the total, differently for J(f + h d) and
// J(f - h d) -- at h = 1e-6 that rounding alone was comparable to the
// difference being measured.  Compensated, the sum is rounded about once.
struct CompSum {
    double s = 0.0, c = 0.0;
    void add(double x)
    {
        const double t = s + x;
        c += std::fabs(s) >= std::fabs(x) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    double value() const { return s + c; }
};

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


// ------------------------------------------------------------- energy step
// Step-4 element residual as T-coefficients: lr[a] = sum_d c[d][a] t_d with
// t_d = sum_b g[d][b] T_b (advection, its stabilisation, conduction; the
// volumetric source does not depend on T).
__device__ void s4_coef(const DevState& S, int e, double (&g)[3][4], double (&c)[3][4])
{
    const int E = S.P.E;
    const int4 n = S.intma[e];
    const double det = S.detJ[e], rcp = S.rho_cp[e], k = S.kc[e];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < 4; ++a) { g[d][a] = S.grad[(size_t)(d * 4 + a) * E + e]; c[d][a] = 0.0; }
    if (S.mat[e] == 0) {
        double u[3][4], sum[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) { u[d][a] = S.unkno[3 * nd(n, a) + d]; sum[d] += u[d][a]; }
        const double af = rcp * det / 120.0;
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) c[d][a] -= af * (sum[d] + u[d][a]);
        const double tau = 0.5 * S.delte[e] * rcp * (det / 6.0);
        const double ub[3] = {sum[0] / 4.0, sum[1] / 4.0, sum[2] / 4.0};
        for (int a = 0; a < 4; ++a) {
            const double ug = ub[0] * g[0][a] + ub[1] * g[1][a] + ub[2] * g[2][a];
            for (int d = 0; d < 3; ++d) c[d][a] += tau * ug * ub[d];
        }
    }
    const double kv = k * (det / 6.0);
    for (int a = 0; a < 4; ++a)
        for (int d = 0; d < 3; ++d) c[d][a] -= kv * g[d][a];
}

__global__ void k_tlm_s4_elem(DevState S, const double* dT, double* eb)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int4 n = S.intma[e];
    double g[3][4], c[3][4];
    s4_coef(S, e, g, c);
    double t[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < 4; ++b)
        for (int d = 0; d < 3; ++d) t[d] += g[d][b] * dT[nd(n, b)];
    for (int a = 0; a < 4; ++a) eb[(size_t)a * E + e] = c[0][a] * t[0] + c[1][a] * t[1] + c[2][a] * t[2];
}

// dT^{n+1} = dT^n + m_p (K dT^n + H dq) off the Dirichlet-T nodes, 0 on them
__global__ void k_tlm_s4_node(DevState S, const double* eb, const int* hf_face, const double* hf_area,
                              const double* dq, const double* dT, double* dTn)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r = 0.0;
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2, a = S.n2e[k] & 3;
        r += eb[(size_t)a * E + e];
    }
    if (dq)
        for (int k = S.hf_ptr[i]; k < S.hf_ptr[i + 1]; ++k) r += dq[hf_face[k]] * hf_area[k] / 3.0;
    dTn[i] = S.tbc_flag[i] ? 0.0 : dT[i] + r * S.elcoe2p[i];
}

__global__ void k_adj_s4_node(DevState S, const double* lam, double* lpre, double* mu)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const double l = S.tbc_flag[i] ? 0.0 : lam[i];
    lpre[i] = l;
    mu[i] = S.elcoe2p[i] * l;
}

__global__ void k_adj_s4_elem(DevState S, const double* mu, double* eb)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int4 n = S.intma[e];
    double g[3][4], c[3][4];
    s4_coef(S, e, g, c);
    double s[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < 4; ++a) {
        const double m = mu[nd(n, a)];
        for (int d = 0; d < 3; ++d) s[d] += m * c[d][a];
    }
    for (int b = 0; b < 4; ++b) eb[(size_t)b * E + e] = g[0][b] * s[0] + g[1][b] * s[1] + g[2][b] * s[2];
}

// lam^n = lpre + K^T mu (every element, element order)
__global__ void k_adj_s4_gather(DevState S, const double* eb, const double* lpre, double* lam)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r = lpre[i];
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2, a = S.n2e[k] & 3;
        r += eb[(size_t)a * E + e];
    }
    lam[i] = r;
}

// dJ/dq_f += area_f/3 * sum of mu over the face's nodes
__global__ void k_adj_qface(int nqf, const int* qf_nodes, const double* qf_area, const double* mu, double* grad)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nqf) return;
    const double s = mu[qf_nodes[3 * f]] + mu[qf_nodes[3 * f + 1]] + mu[qf_nodes[3 * f + 2]];
    grad[f] += qf_area[f] / 3.0 * s;
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
            pcg.inner_tol = 0.05;
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
    // heat-flux face data on the device (once per run)
    void heat_setup()
    {
        if (c.m.qf_area.empty())
            throw Error(CBS3D_INVALID_INPUT, "heat-flux runs need BC-532 faces and heat_flux_bc != 0 in the case");
        nqf = static_cast<int>(c.m.qf_area.size());
        hf_face = reinterpret_cast<int*>(alloc((c.m.hf_face.size() + 1) / 2 + 1));
        hf_area = alloc(c.m.hf_area.size());
        qf_nodes = reinterpret_cast<int*>(alloc((c.m.qf_nodes.size() + 1) / 2 + 1));
        qf_area = alloc(c.m.qf_area.size());
        CUDA_OK(cudaMemcpy(hf_face, c.m.hf_face.data(), c.m.hf_face.size() * sizeof(int), cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemcpy(hf_area, c.m.hf_area.data(), c.m.hf_area.size() * sizeof(double), cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemcpy(qf_nodes, c.m.qf_nodes.data(), c.m.qf_nodes.size() * sizeof(int), cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemcpy(qf_area, c.m.qf_area.data(), c.m.qf_area.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    // energy tangent step after forward(): s0 = dT^n in, dT^{n+1} out
    void heat_tangent(const double* dq)
    {
        const unsigned gn = nb(static_cast<long long>(N)), ge = nb(static_cast<long long>(E));
        k_tlm_s4_elem<<<ge, T, 0, st>>>(c.S, s0, eb12);
        k_tlm_s4_node<<<gn, T, 0, st>>>(c.S, eb12, hf_face, hf_area, dq, s0, s1);
        CUDA_OK(cudaMemcpyAsync(s0, s1, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaGetLastError());
    }
    // energy adjoint step after forward(): s0 = adjoint of T^{n+1} in, of T^n out
    void heat_adjoint(double* grad)
    {
        const unsigned gn = nb(static_cast<long long>(N)), ge = nb(static_cast<long long>(E));
        k_adj_s4_node<<<gn, T, 0, st>>>(c.S, s0, s1, pd);
        k_adj_qface<<<nb(nqf), T, 0, st>>>(nqf, qf_nodes, qf_area, pd, grad);
        k_adj_s4_elem<<<ge, T, 0, st>>>(c.S, pd, eb12);
        k_adj_s4_gather<<<gn, T, 0, st>>>(c.S, eb12, s1, s0);
        CUDA_OK(cudaGetLastError());
    }
    // J = sum_i w_i T_i; optionally its gradient w into s0
    double objective_T(const double* w, bool seed)
    {
        std::vector<double> t(N);
        CUDA_OK(cudaMemcpyAsync(t.data(), c.S.temp, N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        c.check_status();
        CompSum J;
        for (size_t i = 0; i < N; ++i) J.add(w[i] * t[i]);
        if (seed) {
            CUDA_OK(cudaMemcpyAsync(s0, w, N * sizeof(double), cudaMemcpyHostToDevice, st));
            CUDA_OK(cudaStreamSynchronize(st));
        }
        return J.value();
    }
    double dot_plain(const double* w, const double* dvec)
    {
        std::vector<double> d(N);
        CUDA_OK(cudaMemcpyAsync(d.data(), dvec, N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        CompSum s;
        for (size_t i = 0; i < N; ++i) s.add(w[i] * d[i]);
        return s.value();
    }

    // J = 1/2 sum_i w_i |u_i|^2 of the current u; optionally lambda_N = w u into v0
    double objective(const double* w, bool seed)
    {
        std::vector<double> u(3 * N);
        CUDA_OK(cudaMemcpyAsync(u.data(), c.S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        c.check_status();
        CompSum Js;
        for (size_t i = 0; i < N; ++i)
            Js.add(0.5 * w[i] * (u[3 * i] * u[3 * i] + u[3 * i + 1] * u[3 * i + 1] + u[3 * i + 2] * u[3 * i + 2]));
        const double J = Js.value();
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
        CompSum s;
        for (size_t i = 0; i < N; ++i)
            s.add(w[i] * (u[3 * i] * d[3 * i] + u[3 * i + 1] * d[3 * i + 1] + u[3 * i + 2] * d[3 * i + 2]));
        return s.value();
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
    int nqf = 0;
    int *hf_face = nullptr, *qf_nodes = nullptr;
    double *hf_area = nullptr, *qf_area = nullptr;
};

// Forward sweep with (u, p, T) checkpoints every `every` steps, then the
// reverse sweep one segment at a time: for each step in reverse the state
// before it is restored, the step is recomputed (step(true) captures what
// the adjoint step linearises about) and back(s) runs the adjoint step.
template <typename Back>
void reverse_sweep(Run& r, cbs3d_ctx* c, int nsteps, int every, Back&& back)
{
    const size_t N = r.N;
    const int ncp = (nsteps + every - 1) / every;
    const int seg = every < nsteps ? every : nsteps;
    std::vector<double*> cp(static_cast<size_t>(ncp)), sg(static_cast<size_t>(seg));
    for (auto& p : cp) p = r.alloc(5 * N);
    for (auto& p : sg) p = r.alloc(5 * N);
    auto save = [&](double* b) {
        CUDA_OK(cudaMemcpyAsync(b, c->S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
        CUDA_OK(cudaMemcpyAsync(b + 3 * N, c->S.pres, N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
        CUDA_OK(cudaMemcpyAsync(b + 4 * N, c->S.temp, N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
    };
    auto load = [&](const double* b) {
        CUDA_OK(cudaMemcpyAsync(c->S.unkno, b, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
        CUDA_OK(cudaMemcpyAsync(c->S.pres, b + 3 * N, N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
        CUDA_OK(cudaMemcpyAsync(c->S.temp, b + 4 * N, N * sizeof(double), cudaMemcpyDeviceToDevice, r.st));
    };
    for (int s = 0; s < nsteps; ++s) {
        if (s % every == 0) save(cp[static_cast<size_t>(s / every)]);
        r.forward(false);
    }
    back(-1);   // seed at the final state
    for (int k = ncp - 1; k >= 0; --k) {
        const int a = k * every, b = (a + every < nsteps) ? a + every : nsteps;
        load(cp[static_cast<size_t>(k)]);
        c->iitime = r.it0 + a;
        for (int s = a; s < b; ++s) {
            save(sg[static_cast<size_t>(s - a)]);
            r.forward(false);
        }
        for (int s = b - 1; s >= a; --s) {
            load(sg[static_cast<size_t>(s - a)]);
            c->iitime = r.it0 + s;
            r.forward(true);
            back(s);
        }
    }
}

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
        double* G = r.alloc(3 * N);
        CUDA_OK(cudaMemsetAsync(G, 0, 3 * N * sizeof(double), r.st));
        reverse_sweep(r, c, nsteps, every, [&](int s) {
            if (s < 0) *J = r.objective(w, true);   // v0 = dJ/du^N
            else r.adjoint(G);
        });
        CUDA_OK(cudaMemcpyAsync(grad, G, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, r.st));
        CUDA_OK(cudaStreamSynchronize(r.st));
        c->check_status();
        r.restore();
    });
}

cbs3d_status cbs3d_heat_flux_face_count(cbs3d_ctx* c, int* nfaces)
{
    if (!c || !nfaces) return CBS3D_INVALID_INPUT;
    *nfaces = static_cast<int>(c->m.qf_area.size());
    return CBS3D_OK;
}

cbs3d_status cbs3d_set_face_heat_flux(cbs3d_ctx* c, const double* q)
{
    return run_guarded(c, [&] {
        const HostModel& m = c->m;
        if (m.qf_area.empty())
            throw Error(CBS3D_INVALID_INPUT, "cbs3d_set_face_heat_flux - the case has no heat-flux faces (BC 532 with heat_flux_bc != 0)");
        std::vector<double> v(m.hf_val);
        if (q)
            for (size_t k = 0; k < v.size(); ++k) v[k] = q[m.hf_face[k]] * m.hf_area[k] / 3.0;
        CUDA_OK(cudaMemcpyAsync(const_cast<double*>(c->S.hf_val), v.data(), v.size() * sizeof(double),
                                cudaMemcpyHostToDevice, c->st));
        CUDA_OK(cudaStreamSynchronize(c->st));
    });
}

cbs3d_status cbs3d_heat_objective_run(cbs3d_ctx* c, int nsteps, const double* w, double* J)
{
    return run_guarded(c, [&] {
        if (nsteps < 1 || !w || !J) throw Error(CBS3D_INVALID_INPUT, "cbs3d_heat_objective_run - nsteps >= 1, w and J required");
        if (c->m.temp_calc < 1) throw Error(CBS3D_INVALID_INPUT, "cbs3d_heat_objective_run - the case does not solve the energy equation");
        Run r(*c);
        for (int s = 0; s < nsteps; ++s) r.forward(false);
        *J = r.objective_T(w, false);
        r.restore();
    });
}

cbs3d_status cbs3d_heat_tlm_run(cbs3d_ctx* c, int nsteps, const double* w, const double* dq, double* J, double* dJ)
{
    return run_guarded(c, [&] {
        if (nsteps < 1 || !w || !dq || !J || !dJ) throw Error(CBS3D_INVALID_INPUT, "cbs3d_heat_tlm_run - nsteps >= 1, w, dq, J and dJ required");
        if (c->m.temp_calc < 1) throw Error(CBS3D_INVALID_INPUT, "cbs3d_heat_tlm_run - the case does not solve the energy equation");
        Run r(*c);
        r.heat_setup();
        double* ddq = r.alloc(static_cast<size_t>(r.nqf));
        CUDA_OK(cudaMemcpyAsync(ddq, dq, static_cast<size_t>(r.nqf) * sizeof(double), cudaMemcpyHostToDevice, r.st));
        CUDA_OK(cudaMemsetAsync(r.s0, 0, r.N * sizeof(double), r.st));
        for (int s = 0; s < nsteps; ++s) {
            r.forward(false);
            r.heat_tangent(ddq);
        }
        *J = r.objective_T(w, false);
        *dJ = r.dot_plain(w, r.s0);
        r.restore();
    });
}

cbs3d_status cbs3d_heat_adjoint_run(cbs3d_ctx* c, int nsteps, int every, const double* w, double* J, double* grad)
{
    return run_guarded(c, [&] {
        if (nsteps < 1 || every < 1 || !w || !J || !grad)
            throw Error(CBS3D_INVALID_INPUT, "cbs3d_heat_adjoint_run - nsteps >= 1, every >= 1, w, J and grad required");
        if (c->m.temp_calc < 1) throw Error(CBS3D_INVALID_INPUT, "cbs3d_heat_adjoint_run - the case does not solve the energy equation");
        Run r(*c);
        r.heat_setup();
        double* G = r.alloc(static_cast<size_t>(r.nqf));
        CUDA_OK(cudaMemsetAsync(G, 0, static_cast<size_t>(r.nqf) * sizeof(double), r.st));
        reverse_sweep(r, c, nsteps, every, [&](int s) {
            if (s < 0) *J = r.objective_T(w, true);   // s0 = dJ/dT^N
            else r.heat_adjoint(G);
        });
        CUDA_OK(cudaMemcpyAsync(grad, G, static_cast<size_t>(r.nqf) * sizeof(double), cudaMemcpyDeviceToHost, r.st));
        CUDA_OK(cudaStreamSynchronize(r.st));
        c->check_status();
        r.restore();
    });
}

}  // extern "C"
