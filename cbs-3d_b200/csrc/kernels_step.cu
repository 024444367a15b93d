// Per-step CBS kernels for sm_100a (FP64 parity form).
//
// Every element kernel mirrors the reference's per-element arithmetic in the
// same association order and is compiled with -fmad=false, so each local
// contribution is bit-identical to the reference's.  Nodal assembly is
// atomic-free and deterministic: element kernels write their local vectors
// to a scratch (elbuf: node-major sector records for Step 1, structure of
// arrays for the others), and node kernels gather them
// through incidence lists sorted in the reference's summation order --
// (colour, element) for the coloured Step-1 scatter, element order for the
// serial assemblies -- so the nodal sums are bit-identical too.  The node
// kernels fuse the nodal update and the boundary program of the stage.
#include "dev_state.cuh"
#include "host_model.h"

#include <cfloat>

namespace cbs3d {

namespace {

constexpr double FCON1 = 1.0 / 24.0, FCON2 = 1.0 / 12.0, FCON3 = 1.0 / 6.0, FCON4 = 1.0 / 3.0;
constexpr double FDIF1 = 1.0 / 6.0, FDIF2 = 1.0 / 3.0;
constexpr double MASS_FACTOR = 1.0 / 24.0;

// local face f (0-based) opposite local node f: its three local nodes
__constant__ int c_ippn[4][3] = {{2, 1, 3}, {2, 3, 0}, {0, 3, 1}, {0, 1, 2}};

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max

__device__ __forceinline__ int node_of(const int4& n, int a)
{
    return a == 0 ? n.x : a == 1 ? n.y : a == 2 ? n.z : n.w;
}

__device__ __forceinline__ int fedge_of(uint8_t packed, int f) { return (packed >> (2 * f)) & 3; }

}  // namespace

// ============================================================== geometry
// Preprocess::shapeFunctionDerivatives (src/preprocess/Preprocess.cpp:390-505),
// getNormals (:601-679), elementSize (:863-905) and
// PressureAssembly::buildElementPressureTerms (src/assembly/PressureAssembly.cpp:136-178).
__global__ void k_geometry(DevState S)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int4 n = S.intma[e];
    const double* c = S.coord;
    const double x1 = c[3 * n.x], y1 = c[3 * n.x + 1], z1 = c[3 * n.x + 2];
    const double x2 = c[3 * n.y], y2 = c[3 * n.y + 1], z2 = c[3 * n.y + 2];
    const double x3 = c[3 * n.z], y3 = c[3 * n.z + 1], z3 = c[3 * n.z + 2];
    const double x4 = c[3 * n.w], y4 = c[3 * n.w + 1], z4 = c[3 * n.w + 2];
    const double j11 = x2 - x1, j21 = y2 - y1, j31 = z2 - z1;
    const double j12 = x3 - x1, j22 = y3 - y1, j32 = z3 - z1;
    const double j13 = x4 - x1, j23 = y4 - y1, j33 = z4 - z1;
    const double det = j11 * (j22 * j33 - j23 * j32) - j12 * (j21 * j33 - j23 * j31) + j13 * (j21 * j32 - j22 * j31);
    if (det <= 0.0 || !isfinite(det)) { set_status(S.status, 1, ST_GEOM, e + 1, R_DETJ); return; }
    const double inv = 1.0 / det;
    double g[3][4];
    g[0][1] = (j22 * j33 - j23 * j32) * inv;
    g[1][1] = (j13 * j32 - j12 * j33) * inv;
    g[2][1] = (j12 * j23 - j13 * j22) * inv;
    g[0][2] = (j23 * j31 - j21 * j33) * inv;
    g[1][2] = (j11 * j33 - j13 * j31) * inv;
    g[2][2] = (j13 * j21 - j11 * j23) * inv;
    g[0][3] = (j21 * j32 - j22 * j31) * inv;
    g[1][3] = (j12 * j31 - j11 * j32) * inv;
    g[2][3] = (j11 * j22 - j12 * j21) * inv;
    g[0][0] = -(g[0][1] + g[0][2] + g[0][3]);
    g[1][0] = -(g[1][1] + g[1][2] + g[1][3]);
    g[2][0] = -(g[2][1] + g[2][2] + g[2][3]);
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < 4; ++a) S.grad[(size_t)(d * 4 + a) * E + e] = g[d][a];
    S.detJ[e] = det;

    const double px[4] = {x1, x2, x3, x4}, py[4] = {y1, y2, y3, y4}, pz[4] = {z1, z2, z3, z4};
    const double three_volume = 0.5 * det;
    double hmin = DBL_MAX;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const int a1 = c_ippn[f][0], a2 = c_ippn[f][1], a3 = c_ippn[f][2];
        const double e1x = px[a2] - px[a1], e1y = py[a2] - py[a1], e1z = pz[a2] - pz[a1];
        const double e2x = px[a3] - px[a1], e2y = py[a3] - py[a1], e2z = pz[a3] - pz[a1];
        double ax = e1y * e2z - e1z * e2y;
        double ay = e1z * e2x - e1x * e2z;
        double az = e1x * e2y - e1y * e2x;
        const double amag = sqrt(ax * ax + ay * ay + az * az);
        if (amag <= 0.0 || !isfinite(amag)) { set_status(S.status, 1, ST_GEOM, e + 1, R_FACE_AREA); return; }
        const double fx = (px[a1] + px[a2] + px[a3]) / 3.0;
        const double fy = (py[a1] + py[a2] + py[a3]) / 3.0;
        const double fz = (pz[a1] + pz[a2] + pz[a3]) / 3.0;
        const double vx = px[f] - fx, vy = py[f] - fy, vz = pz[f] - fz;
        if (ax * vx + ay * vy + az * vz > 0.0) { ax = -ax; ay = -ay; az = -az; }
        const double area = 0.5 * amag;
        S.annxf[(size_t)(f * 4 + 0) * E + e] = 0.5 * ax;
        S.annxf[(size_t)(f * 4 + 1) * E + e] = 0.5 * ay;
        S.annxf[(size_t)(f * 4 + 2) * E + e] = 0.5 * az;
        S.annxf[(size_t)(f * 4 + 3) * E + e] = area;
        hmin = dmin(hmin, three_volume / area);
    }
    if (hmin <= 0.0 || !isfinite(hmin)) { set_status(S.status, 1, ST_GEOM, e + 1, R_HMIN); return; }
    S.alen_e[e] = hmin;

    if (S.mat[e] != 0) {
#pragma unroll
        for (int a = 0; a < 4; ++a) S.pdiagE[(size_t)a * E + e] = 0.0;
#pragma unroll
        for (int q = 0; q < 6; ++q) S.gstifE[(size_t)q * E + e] = 0.0;
        return;
    }
    const double vol = det / 6.0;
    auto gd = [&](int a, int b) { return g[0][a] * g[0][b] + g[1][a] * g[1][b] + g[2][a] * g[2][b]; };
#pragma unroll
    for (int a = 0; a < 4; ++a) S.pdiagE[(size_t)a * E + e] = vol * gd(a, a);
    S.gstifE[(size_t)0 * E + e] = vol * gd(0, 1);
    S.gstifE[(size_t)1 * E + e] = vol * gd(0, 2);
    S.gstifE[(size_t)2 * E + e] = vol * gd(0, 3);
    S.gstifE[(size_t)3 * E + e] = vol * gd(1, 2);
    S.gstifE[(size_t)4 * E + e] = vol * gd(1, 3);
    S.gstifE[(size_t)5 * E + e] = vol * gd(2, 3);
}

// Preprocess::massMatrix (src/preprocess/Preprocess.cpp:721-809): element-
// order nodal sums of the lumped mass and capacitance, with its checks.
__global__ void k_mass(DevState S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    double m = 0.0, t = 0.0;
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2;
        const double nm = S.detJ[e] * MASS_FACTOR;
        m += nm;
        t += S.rho_cp[e] * nm;
    }
    if (m <= 0.0 || !isfinite(m)) { set_status(S.status, 1, ST_MASS, i + 1, R_MASS); return; }
    if (t <= 0.0 || !isfinite(t)) { set_status(S.status, 1, ST_MASS, i + 1, R_CAPACITY); return; }
    S.mdiag_real[i] = m;
    S.elcoe2[i] = 1.0 / m;
    S.elcoe2p[i] = 1.0 / t;
}

// Fluid lumped mass per node (element order), for the body-force term.
__global__ void k_mass_fluid(DevState S, double* mfluid)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    double m = 0.0;
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2;
        if (S.mat[e] == 0) m += S.detJ[e] * MASS_FACTOR;
    }
    mfluid[i] = m;
}

// compute_nodal_lengths_from_elements (src/timestep/TimeStep.cpp:319-355):
// minimum altitude over the incident tetrahedra (order-independent).
__global__ void k_nodal_length(DevState S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double h = DBL_MAX;
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2, a = S.n2e[k] & 3;
        h = dmin(h, (0.5 * S.detJ[e]) / S.annxf[(size_t)(a * 4 + 3) * E + e]);
    }
    S.alen[i] = h;
}

// ============================================================= time step
__global__ void k_begin_step(DevState S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    S.unkn1[3 * i] = S.unkno[3 * i];
    S.unkn1[3 * i + 1] = S.unkno[3 * i + 1];
    S.unkn1[3 * i + 2] = S.unkno[3 * i + 2];
    S.pres1[i] = S.pres[i];
    S.temp1[i] = S.temp[i];
    if (i == 0) *S.dtmin_bits = 0x7fefffffffffffffULL;   // DBL_MAX
}

// Element stability time step: TimeStep::computeTimeStep's element loop and
// helpers (src/timestep/TimeStep.cpp:114-300, 522-529), with a block
// minimum reduced into dtmin_bits (positive doubles order like their bits).
__global__ void k_timestep(DevState S, int fixed_dt)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double dt = DBL_MAX;
    if (e < E) {
        if (fixed_dt) {
            dt = S.P.dtfix;
            S.delte[e] = dt;
        } else {
            const int4 n = S.intma[e];
            double h = S.alen_e[e];
            bool ok = true;
            if (h <= 0.0 || !isfinite(h)) { set_status(S.status, 1, ST_TIMESTEP, e + 1, R_HMIN); ok = false; }
            if (ok && S.P.htype == 2) {
                double hn = 0.0;
                bool valid = true;
                for (int a = 0; a < 4; ++a) {
                    const double al = S.alen[node_of(n, a)];
                    if (al <= 0.0 || !isfinite(al)) { valid = false; break; }
                    hn += al;
                }
                hn = valid ? hn / 4.0 : h;
                h = dmin(h, hn);
            }
            double speed;
            if (S.P.htype == 3) {
                double u = 0.0, v = 0.0, w = 0.0;
                for (int a = 0; a < 4; ++a) {
                    const int ip = node_of(n, a);
                    u += S.unkno[3 * ip]; v += S.unkno[3 * ip + 1]; w += S.unkno[3 * ip + 2];
                }
                u /= 4.0; v /= 4.0; w /= 4.0;
                speed = sqrt(u * u + v * v + w * w);
            } else {
                // max_a sqrt(|u_a|^2) as sqrt(max_a |u_a|^2): the square root
                // is correctly rounded, hence monotonic, so the two are equal
                // bit for bit (a NaN is skipped by std::max either way)
                double m = 0.0;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const int ip = node_of(n, a);
                    const double u = S.unkno[3 * ip], v = S.unkno[3 * ip + 1], w = S.unkno[3 * ip + 2];
                    m = dmax(m, u * u + v * v + w * w);
                }
                speed = sqrt(m);
            }
            double diff = S.P.ani;
            const bool fluid = S.mat[e] == 0;
            if (ok && S.P.dimensional_material) {
                const double al = S.alpha[e];
                if (al <= 0.0 || !isfinite(al)) { set_status(S.status, 1, ST_TIMESTEP, e + 1, R_ALPHA); ok = false; }
                diff = al;
                if (ok && fluid) {
                    if (S.rho[e] <= 0.0 || S.mu[e] < 0.0) { set_status(S.status, 1, ST_TIMESTEP, e + 1, R_RHOMU); ok = false; }
                    diff = dmax(diff, S.mu[e] / S.rho[e]);
                }
            }
            if (ok && (diff <= 0.0 || !isfinite(diff))) { set_status(S.status, 1, ST_TIMESTEP, e + 1, R_DIFF); ok = false; }
            if (ok) {
                const double adv = fluid ? h / dmax(speed, 1.0e-14) : DBL_MAX;
                const double dif = h * h * (0.5 / diff);
                dt = S.P.csafm * dmin(adv, dif);
                if (S.P.ilots == 2 && S.P.deltr > 0.0 && isfinite(S.P.deltr)) dt = dmin(dt, S.P.deltr);
                if (dt <= 0.0 || !isfinite(dt)) { set_status(S.status, 1, ST_TIMESTEP, e + 1, R_DT_LOCAL); dt = DBL_MAX; }
            }
            S.delte[e] = dt;
        }
    }
    // block min of positive doubles through their bit patterns
    unsigned long long b = __double_as_longlong(dt);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
        b = x < b ? x : b;
    }
    __shared__ unsigned long long sm[32];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long v = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0x7fefffffffffffffULL;
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, v, o);
            v = x < v ? x : v;
        }
        if (threadIdx.x == 0) atomicMin(S.dtmin_bits, v);
    }
}

// dtreal = min_e dt_e; optional forcing of the global minimum
// (src/timestep/TimeStep.cpp:531-582) and physical-time advance (Solver.cpp:625-628).
__global__ void k_dt_finish(DevState S, int fixed_dt)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double dtmin = fixed_dt ? S.P.dtfix : __longlong_as_double((long long)*S.dtmin_bits);
    if (dtmin <= 0.0 || !isfinite(dtmin) || dtmin == DBL_MAX) set_status(S.status, 1, ST_TIMESTEP, 0, R_DT_MIN);
    S.dscal[0] = dtmin;
    if (S.P.transient_on > 0) S.dscal[1] += dtmin;
}

__global__ void k_dt_force(DevState S)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < S.P.E) S.delte[e] = S.dscal[0];
}

// TimeStep::applyStep2PressureTimeStepCorrection (src/timestep/TimeStep.cpp:704-749)
__global__ void k_dt_correction(DevState S)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= S.P.E) return;
    const int4 n = S.intma[e];
    double dmn = S.delte[e];
    for (int a = 0; a < 4; ++a) {
        const int ip = node_of(n, a);
        const double pscale = fabs(S.pres1[ip]) + S.P.epsilon1;
        const double u = S.unkno[3 * ip], v = S.unkno[3 * ip + 1], w = S.unkno[3 * ip + 2];
        const double speed = sqrt(u * u + v * v + w * w);
        if (speed > 1.0e-14 && pscale > 0.0) {
            const double h = (S.alen[ip] > 0.0) ? S.alen[ip] : S.alen_e[e];
            const double cand = S.P.csafm2 * h * pscale / speed;
            if (cand > 0.0 && isfinite(cand)) dmn = dmin(dmn, cand);
        }
    }
    S.delte[e] = dmn;
}

// TimeStep::updateLhsDiagonal (src/timestep/TimeStep.cpp:778-954) as one
// element-ordered node gather: elcoe2, elcoe2p, pdiag, then the solid-only
// and fixed-pressure rows.  gstif = gstifE*dt is formed where it is consumed.
__global__ void k_lhs(DevState S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double s2 = 0.0, s2p = 0.0, pd = 0.0;
    // incident elements in order, their data loaded four at a time
    const int kb = S.n2e_ptr[i], ke = S.n2e_ptr[i + 1];
    int k = kb;
    for (; k + 4 <= ke; k += 4) {
        int ent[4];
        double dt[4], dj[4], rc[4], pe[4];
        bool fl[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) ent[u] = S.n2e[k + u];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = ent[u] >> 2, a = ent[u] & 3;
            dt[u] = S.delte[e];
            dj[u] = S.detJ[e];
            fl[u] = S.mat[e] == 0;
            rc[u] = S.rho_cp[e];
            pe[u] = S.pdiagE[(size_t)a * E + e];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (dt[u] <= 0.0 || !isfinite(dt[u])) { set_status(S.status, 1, ST_LHS, (ent[u] >> 2) + 1, R_LHS_DT); return; }
            const double mass = dj[u] * MASS_FACTOR;
            if (fl[u]) s2 += mass / dt[u];
            s2p += rc[u] * mass / dt[u];
            if (fl[u]) pd += pe[u] * dt[u];
        }
    }
    for (; k < ke; ++k) {
        const int e = S.n2e[k] >> 2, a = S.n2e[k] & 3;
        const double dt = S.delte[e];
        if (dt <= 0.0 || !isfinite(dt)) { set_status(S.status, 1, ST_LHS, e + 1, R_LHS_DT); return; }
        const double mass = S.detJ[e] * MASS_FACTOR;
        const bool fluid = S.mat[e] == 0;
        if (fluid) s2 += mass / dt;
        s2p += S.rho_cp[e] * mass / dt;
        if (fluid) pd += S.pdiagE[(size_t)a * E + e] * dt;
    }
    const uint8_t f = S.nflag[i];
    const bool tf = f & 1, ts = f & 2;
    if (!tf && !ts) { set_status(S.status, 1, ST_LHS, i + 1, R_ORPHAN); return; }
    if (tf) {
        if (s2 <= 0.0 || !isfinite(s2)) { set_status(S.status, 1, ST_LHS, i + 1, R_LHS_ELCOE2); return; }
        S.elcoe2[i] = 1.0 / s2;
    } else {
        S.elcoe2[i] = 0.0;
    }
    if (s2p <= 0.0 || !isfinite(s2p)) { set_status(S.status, 1, ST_LHS, i + 1, R_LHS_ELCOE2P); return; }
    S.elcoe2p[i] = 1.0 / s2p;
    if (tf) {
        if (fabs(pd) <= 1.0e-14 || !isfinite(pd)) { set_status(S.status, 1, ST_LHS, i + 1, R_LHS_PDIAG); return; }
        S.pdiag[i] = pd;
    } else {
        S.pdiag[i] = 0.0;
        S.pres[i] = 0.0;
        S.rhs1[i] = 0.0;
    }
    if (f & 4) {
        S.pdiag[i] = 1.0;
        S.pres[i] = S.pfix[i];
        S.rhs1[i] = S.pfix[i];
    }
}

// ====================================================== velocity BC program
// Net effect per node of Boundary::applySymmetry, applyVelocity,
// applyOutletBackflowControl and enforce_zero_velocity_in_solid in that order
// (src/solver/Steps.cpp:170-176), with the face-ordered projections kept.
__device__ __forceinline__ void apply_velocity_package(const DevState& S, int i, double& u, double& v, double& w)
{
    const int idx = S.vbc_idx[i];
    if (idx < 0) return;
    const VelBC b = static_cast<const VelBC*>(S.vbc)[idx];
    if (b.flags & VBC_SOLID) { u = 0.0; v = 0.0; w = 0.0; return; }
    for (int k = 0; k < b.sym_cnt; ++k) {
        const double* nn = S.vbc_nrm + 3 * (b.sym_beg + k);
        const double un = u * nn[0] + v * nn[1] + w * nn[2];
        u -= un * nn[0];
        v -= un * nn[1];
        w -= un * nn[2];
    }
    if (b.flags & VBC_FIXED) { u = b.fix[0]; v = b.fix[1]; w = b.fix[2]; }
    for (int k = 0; k < b.out_cnt; ++k) {
        const double* nn = S.vbc_nrm + 3 * (b.out_beg + k);
        const double un = u * nn[0] + v * nn[1] + w * nn[2];
        if (un < 0.0) {
            u -= un * nn[0];
            v -= un * nn[1];
            w -= un * nn[2];
        }
    }
}

// ================================================================ Step 1
// MomentumAssembly::assembleStep1Rhs per fluid element
// (src/assembly/MomentumAssembly.cpp:144-432, 496-529).
__global__ void __launch_bounds__(128) k_step1_elem(DevState S)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E || S.mat[e] != 0) return;
    const double det = S.detJ[e];
    if (det <= 0.0 || !isfinite(det)) { set_status(S.status, 1, ST_STEP1, 0, R_STEP1_DETJ); return; }
    const int4 n = S.intma[e];
    double lu[3][4], g[3][4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int ip = node_of(n, a);
#pragma unroll
        for (int i = 0; i < 3; ++i) lu[i][a] = S.unkn1[3 * ip + i];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < 4; ++a) g[d][a] = S.grad[(size_t)(d * 4 + a) * E + e];
    const uint8_t fe = S.fedge[e];
    double lr[3][4];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int a = 0; a < 4; ++a) lr[i][a] = 0.0;
#define LUNK(i, j, a) (lu[j][a] * lu[i][a])

    // ---- Galerkin convection (:144-220)
    {
        double ls[3][3];
        const double vf = det * FCON1;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
#pragma unroll
                for (int a = 0; a < 4; ++a) s += LUNK(i, j, a);
                ls[i][j] = s;
            }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) lr[i][a] += g[j][a] * vf * ls[i][j];
        if (fe) {
            for (int is = 0; is < 4; ++is) {
                if (fedge_of(fe, is) == 0) continue;
                double an[3];
#pragma unroll
                for (int j = 0; j < 3; ++j) an[j] = S.annxf[(size_t)(is * 4 + j) * E + e];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double ff = an[j] * FCON2;
#pragma unroll
                    for (int fn = 0; fn < 3; ++fn) {
                        const int a = c_ippn[is][fn];
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            double la, lis;
                            // lunk at node a and at the opposite node is
                            la = (a == 0) ? LUNK(i, j, 0) : (a == 1) ? LUNK(i, j, 1) : (a == 2) ? LUNK(i, j, 2) : LUNK(i, j, 3);
                            lis = (is == 0) ? LUNK(i, j, 0) : (is == 1) ? LUNK(i, j, 1) : (is == 2) ? LUNK(i, j, 2) : LUNK(i, j, 3);
                            const double lsf = ls[i][j] - lis;
                            const double val = (lsf + la) * ff;
                            if (a == 0) lr[i][0] -= val; else if (a == 1) lr[i][1] -= val;
                            else if (a == 2) lr[i][2] -= val; else lr[i][3] -= val;
                        }
                    }
                }
            }
        }
    }
    // ---- characteristic correction (:242-345)
    {
        double ls[3][3], lsk[3][3], um[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
#pragma unroll
                for (int a = 0; a < 4; ++a) s += g[j][a] * LUNK(i, j, a);
                ls[i][j] = s;
            }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
#pragma unroll
            for (int a = 0; a < 4; ++a) s += lu[i][a];
            um[i] = s / 4.0;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double sj = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) sj += ls[i][j];
#pragma unroll
            for (int k = 0; k < 3; ++k) lsk[i][k] = um[k] * sj;
        }
        const double dt = S.delte[e];
        if (dt <= 0.0 || !isfinite(dt)) { set_status(S.status, 1, ST_STEP1, e + 1, R_DT_LOCAL); return; }
        const double ld = 0.5 * dt * det * FCON3;
        const double ld2 = 0.5 * dt * FCON4;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int i = 0; i < 3; ++i) lr[i][a] -= g[k][a] * lsk[i][k] * ld;
        if (fe) {
            for (int is = 0; is < 4; ++is) {
                if (fedge_of(fe, is) == 0) continue;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double ff = S.annxf[(size_t)(is * 4 + k) * E + e] * ld2;
#pragma unroll
                    for (int fn = 0; fn < 3; ++fn) {
                        const int a = c_ippn[is][fn];
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const double val = lsk[i][k] * ff;
                            if (a == 0) lr[i][0] += val; else if (a == 1) lr[i][1] += val;
                            else if (a == 2) lr[i][2] += val; else lr[i][3] += val;
                        }
                    }
                }
            }
        }
    }
    // ---- diffusion (:369-432)
    {
        double nu = S.P.ani;
        if (S.P.dimensional_material) {
            if (S.rho[e] <= 0.0 || S.mu[e] < 0.0) { set_status(S.status, 1, ST_STEP1, e + 1, R_RHOMU); return; }
            nu = S.mu[e] / S.rho[e];
        }
        double gu[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
#pragma unroll
                for (int a = 0; a < 4; ++a) s += g[j][a] * lu[i][a];
                gu[i][j] = s;
            }
        const double vf = nu * det * FDIF1;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int j = 0; j < 3; ++j) lr[i][a] -= g[j][a] * gu[i][j] * vf;
        const double fdf = nu * FDIF2;
        if (fe) {
            for (int is = 0; is < 4; ++is) {
                if (fedge_of(fe, is) == 0) continue;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double ff = S.annxf[(size_t)(is * 4 + j) * E + e] * fdf;
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int fn = 0; fn < 3; ++fn) {
                            const int a = c_ippn[is][fn];
                            const double val = gu[i][j] * ff;
                            if (a == 0) lr[i][0] += val; else if (a == 1) lr[i][1] += val;
                            else if (a == 2) lr[i][2] += val; else lr[i][3] += val;
                        }
                }
            }
        }
    }
#undef LUNK
    // node-major records of 32 bytes per (element, local node): the three
    // components and a zero pad, so a node's gather reads exactly one sector
    // per incident tet and no sector is shared by two nodes
    double2* rec = reinterpret_cast<double2*>(S.elbuf) + (size_t)e * 8;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        rec[2 * a] = make_double2(lr[0][a], lr[1][a]);
        rec[2 * a + 1] = make_double2(lr[2][a], 0.0);
    }
}

// Colour-ordered nodal gather of the Step-1 residual, predictor
// u* = u^n + elcoe2*rhs and the velocity BC package
// (src/solver/Steps.cpp:132-142, 170-176, 273-284).
__global__ void k_step1_node(DevState S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    // colour order, records (one 32-byte sector per incident tet, see
    // k_step1_elem) loaded four at a time
    const double2* rec = reinterpret_cast<const double2*>(S.elbuf);
    const int kb = S.n2c_ptr[i], ke = S.n2c_ptr[i + 1];
    int k = kb;
    for (; k + 4 <= ke; k += 4) {
        double2 x01[4], x2[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const size_t q = 2 * (size_t)S.n2c[k + u];   // ent = 4e + a: the record's first double2
            x01[u] = rec[q];
            x2[u] = rec[q + 1];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            r0 += x01[u].x;
            r1 += x01[u].y;
            r2 += x2[u].x;
        }
    }
    for (; k < ke; ++k) {
        const size_t q = 2 * (size_t)S.n2c[k];
        const double2 x01 = rec[q], x2 = rec[q + 1];
        r0 += x01.x;
        r1 += x01.y;
        r2 += x2.x;
    }
    if (S.bforce) {
        const double mf = S.mfluid[i];
        r0 += mf * S.bforce[3 * i];
        r1 += mf * S.bforce[3 * i + 1];
        r2 += mf * S.bforce[3 * i + 2];
    }
    S.rhs[3 * i] = r0; S.rhs[3 * i + 1] = r1; S.rhs[3 * i + 2] = r2;
    const double m = S.elcoe2[i];
    double u = S.unkn1[3 * i] + r0 * m;
    double v = S.unkn1[3 * i + 1] + r1 * m;
    double w = S.unkn1[3 * i + 2] + r2 * m;
    apply_velocity_package(S, i, u, v, w);
    S.unkno[3 * i] = u; S.unkno[3 * i + 1] = v; S.unkno[3 * i + 2] = w;
}

// ================================================================ Step 2
// PressureAssembly::assembleStep2Rhs per fluid element (src/assembly/PressureAssembly.cpp:262-325)
__global__ void k_step2_elem(DevState S)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E || S.mat[e] != 0) return;
    const int4 n = S.intma[e];
    const double vol4 = S.detJ[e] * FCON1;
    double us0 = 0.0, us1 = 0.0, us2 = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int ip = node_of(n, a);
        us0 += S.unkno[3 * ip]; us1 += S.unkno[3 * ip + 1]; us2 += S.unkno[3 * ip + 2];
    }
    us0 *= vol4; us1 *= vol4; us2 *= vol4;
    double lr[4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
        lr[a] = S.grad[(size_t)(0 * 4 + a) * E + e] * us0 + S.grad[(size_t)(1 * 4 + a) * E + e] * us1 +
                S.grad[(size_t)(2 * 4 + a) * E + e] * us2;
    const uint8_t fe = S.fedge[e];
    if (fe) {
        for (int is = 0; is < 4; ++is) {
            if (fedge_of(fe, is) != 1) continue;
            double fs[3] = {0.0, 0.0, 0.0};
            for (int q = 0; q < 3; ++q) {
                const int ip = node_of(n, c_ippn[is][q]);
                fs[0] += S.unkn1[3 * ip]; fs[1] += S.unkn1[3 * ip + 1]; fs[2] += S.unkn1[3 * ip + 2];
            }
            for (int d = 0; d < 3; ++d) {
                const double nf = S.annxf[(size_t)(is * 4 + d) * E + e] * FCON2;
                for (int q = 0; q < 3; ++q) {
                    const int ln = c_ippn[is][q];
                    const double val = (fs[d] + S.unkn1[3 * node_of(n, ln) + d]) * nf;
                    if (ln == 0) lr[0] -= val; else if (ln == 1) lr[1] -= val;
                    else if (ln == 2) lr[2] -= val; else lr[3] -= val;
                }
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) S.elbuf[(size_t)a * E + e] = lr[a];
}

// element-ordered nodal gather of the Step-2 RHS (src/assembly/PressureAssembly.cpp:329-333)
__global__ void k_step2_node(DevState S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r = 0.0;
    const int kb = S.n2e_ptr[i], ke = S.n2e_ptr[i + 1];
    int k = kb;
    for (; k + 4 <= ke; k += 4) {
        double x[4];
        bool fl[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int ent = S.n2e[k + u];
            const int e = ent >> 2, a = ent & 3;
            fl[u] = S.mat[e] == 0;
            x[u] = S.elbuf[(size_t)a * E + e];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (fl[u]) r += x[u];
    }
    for (; k < ke; ++k) {
        const int e = S.n2e[k] >> 2, a = S.n2e[k] & 3;
        if (S.mat[e] != 0) continue;
        r += S.elbuf[(size_t)a * E + e];
    }
    S.rhs1[i] = r;
}

// ================================================================ Step 3
// Steps::step3SemiImplicit (src/solver/Steps.cpp:377-428)
__global__ void k_step3_elem(DevState S)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E || S.mat[e] != 0) return;
    const int4 n = S.intma[e];
    double gp[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < 4; ++a) s += S.grad[(size_t)(d * 4 + a) * E + e] * S.pres[node_of(n, a)];
        gp[d] = s;
    }
    const double vol4 = S.detJ[e] * FCON1;
#pragma unroll
    for (int d = 0; d < 3; ++d) S.elbuf[(size_t)d * E + e] = vol4 * gp[d];
}

__global__ void k_step3_node(DevState S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    const int kb = S.n2e_ptr[i], ke = S.n2e_ptr[i + 1];
    int k = kb;
    for (; k + 4 <= ke; k += 4) {
        double x0[4], x1[4], x2[4];
        bool fl[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = S.n2e[k + u] >> 2;
            fl[u] = S.mat[e] == 0;
            x0[u] = S.elbuf[(size_t)0 * E + e];
            x1[u] = S.elbuf[(size_t)1 * E + e];
            x2[u] = S.elbuf[(size_t)2 * E + e];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (fl[u]) {
                r0 -= x0[u];
                r1 -= x1[u];
                r2 -= x2[u];
            }
    }
    for (; k < ke; ++k) {
        const int e = S.n2e[k] >> 2;
        if (S.mat[e] != 0) continue;
        r0 -= S.elbuf[(size_t)0 * E + e];
        r1 -= S.elbuf[(size_t)1 * E + e];
        r2 -= S.elbuf[(size_t)2 * E + e];
    }
    S.rhs[3 * i] = r0; S.rhs[3 * i + 1] = r1; S.rhs[3 * i + 2] = r2;
    const double m = S.elcoe2[i];
    double u = S.unkno[3 * i] + r0 * m;
    double v = S.unkno[3 * i + 1] + r1 * m;
    double w = S.unkno[3 * i + 2] + r2 * m;
    apply_velocity_package(S, i, u, v, w);
    S.unkno[3 * i] = u; S.unkno[3 * i + 1] = v; S.unkno[3 * i + 2] = w;
}

// ================================================================ Step 4
// EnergyAssembly::assembleStep4Rhs per element (src/assembly/EnergyAssembly.cpp:118-458, 572-607)
__global__ void k_step4_elem(DevState S)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const double det = S.detJ[e];
    if (det <= 0.0 || !isfinite(det)) { set_status(S.status, 1, ST_STEP4, e + 1, R_DETJ); return; }
    const double rcp = S.rho_cp[e];
    if (rcp <= 0.0 || !isfinite(rcp)) { set_status(S.status, 1, ST_STEP4, e + 1, R_RHOCP); return; }
    if (S.kc[e] <= 0.0 || !isfinite(S.kc[e])) { set_status(S.status, 1, ST_STEP4, e + 1, R_K); return; }
    if (!isfinite(S.qvol[e])) { set_status(S.status, 1, ST_STEP4, e + 1, R_QVOL); return; }
    const int4 n = S.intma[e];
    double g[3][4];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < 4; ++a) g[d][a] = S.grad[(size_t)(d * 4 + a) * E + e];
    double tx = 0.0, ty = 0.0, tz = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const double T = S.temp1[node_of(n, a)];
        tx += g[0][a] * T; ty += g[1][a] * T; tz += g[2][a] * T;
    }
    double lr[4] = {0.0, 0.0, 0.0, 0.0};
    if (S.mat[e] == 0) {
        double ux[4], vy[4], wz[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int ip = node_of(n, a);
            ux[a] = S.unkno[3 * ip]; vy[a] = S.unkno[3 * ip + 1]; wz[a] = S.unkno[3 * ip + 2];
        }
        const double af = rcp * det / 120.0;
        double us = 0.0, vs = 0.0, ws = 0.0;
#pragma unroll
        for (int b = 0; b < 4; ++b) { us += ux[b]; vs += vy[b]; ws += wz[b]; }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double advT = (us + ux[a]) * tx + (vs + vy[a]) * ty + (ws + wz[a]) * tz;
            lr[a] -= af * advT;
        }
        const double dt = S.delte[e];
        if (dt <= 0.0 || !isfinite(dt)) { set_status(S.status, 1, ST_STEP4, e + 1, R_EN_DT); return; }
        double ub = 0.0, vb = 0.0, wb = 0.0;
#pragma unroll
        for (int a = 0; a < 4; ++a) { ub += ux[a]; vb += vy[a]; wb += wz[a]; }
        ub /= 4.0; vb /= 4.0; wb /= 4.0;
        const double advT = ub * tx + vb * ty + wb * tz;
        const double vol = det / 6.0;
        const double tau = 0.5 * dt * rcp * vol;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double ug = ub * g[0][a] + vb * g[1][a] + wb * g[2][a];
            lr[a] += tau * ug * advT;
        }
    }
    const double vol = det / 6.0;
    const double k = S.kc[e];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const double gdt = g[0][a] * tx + g[1][a] * ty + g[2][a] * tz;
        lr[a] -= k * vol * gdt;
    }
    const double q = S.qvol[e];
    if (q != 0.0) {
        const double src = q * det * MASS_FACTOR;
#pragma unroll
        for (int a = 0; a < 4; ++a) lr[a] += src;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) S.elbuf[(size_t)a * E + e] = lr[a];
}

// element-ordered gather, face-ordered heat flux, T = T1 + elcoe2p*rhs1 and
// Boundary::applyTemperature (src/solver/Steps.cpp:448-467)
__global__ void k_step4_node(DevState S)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    const int E = S.P.E;
    double r = 0.0;
    for (int k = S.n2e_ptr[i]; k < S.n2e_ptr[i + 1]; ++k) {
        const int e = S.n2e[k] >> 2, a = S.n2e[k] & 3;
        r += S.elbuf[(size_t)a * E + e];
    }
    for (int k = S.hf_ptr[i]; k < S.hf_ptr[i + 1]; ++k) r += S.hf_val[k];
    S.rhs1[i] = r;
    double T = S.temp1[i] + r * S.elcoe2p[i];
    if (S.tbc_flag[i]) T = S.tbc_val[i];
    S.temp[i] = T;
}

// ====================================================== convergence norms
// Solver::updateVelocityMagnitude (src/solver/Solver.cpp:689-699) and the
// per-node sums of Convergence::evaluate (src/solver/Convergence.cpp:276-317),
// reduced per block in a fixed order; the last block to finish sums the block
// partials (for each measure: lanes stride the blocks, then a fixed shuffle
// tree) and finalises them (:319-348).  With log != nullptr it then records
// the step: dtreal, the PCG result, hb, rtime, and tags a pending failure
// with the step counter.
__global__ void k_conv_partial(DevState S, const CgOut* cg, double* log, int* counter, int cap)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[15];
#pragma unroll
    for (int q = 0; q < 15; ++q) v[q] = 0.0;
    if (i < S.P.N) {
        const double u0 = S.unkno[3 * i], u1 = S.unkno[3 * i + 1], u2 = S.unkno[3 * i + 2];
        S.velocity[i] = sqrt(u0 * u0 + u1 * u1 + u2 * u2 + 1.0e-16);
        const uint8_t f = S.nflag[i];
        const bool tf = f & 1, ts = f & 2;
        if (tf && !ts) {
            const double m = S.elcoe2[i];
            const double w = (fabs(m) <= 1.0e-300 || !isfinite(m)) ? 1.0 : 1.0 / m;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double nw = S.unkno[3 * i + d];
                const double dl = nw - S.unkn1[3 * i + d];
                v[3 * d] = dl * dl;
                v[3 * d + 1] = nw * nw;
                const double rs = dl * w;
                v[3 * d + 2] = rs * rs;
            }
        }
        if (tf) {
            const double dl = S.pres[i] - S.pres1[i];
            v[9] = dl * dl;
            v[10] = S.pres[i] * S.pres[i];
            v[11] = dl * dl;
        }
        if (S.P.temp_calc > 0 && (tf || ts)) {   // thermal_active (Convergence.cpp:178)
            const double dl = S.temp[i] - S.temp1[i];
            v[12] = dl * dl;
            v[13] = S.temp[i] * S.temp[i];
            const double m = S.elcoe2p[i];
            const double w = (fabs(m) <= 1.0e-300 || !isfinite(m)) ? 1.0 : 1.0 / m;
            const double rs = dl * w;
            v[14] = rs * rs;
        }
    }
    __shared__ double sm[15][8];
#pragma unroll
    for (int q = 0; q < 15; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) sm[q][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 15) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sm[threadIdx.x][w];
        S.red[(size_t)blockIdx.x * 16 + threadIdx.x] = s;
        __threadfence();
    }
    __shared__ int s_last;
    __shared__ double hb[16];
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(S.conv_count, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int nblocks = (int)gridDim.x, lane = threadIdx.x & 31;
    for (int q = threadIdx.x >> 5; q < 15; q += (int)(blockDim.x >> 5)) {
        double s = 0.0;
        int b = lane;
        for (; b + 7 * 32 < nblocks; b += 8 * 32) {
            double y[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) y[u] = __ldcg(S.red + (size_t)(b + 32 * u) * 16 + q);
#pragma unroll
            for (int u = 0; u < 8; ++u) s += y[u];
        }
        for (; b < nblocks; b += 32) s += __ldcg(S.red + (size_t)b * 16 + q);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) hb[q] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    *S.conv_count = 0;   // for the next launch
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
    if (S.P.temp_calc > 0) {
        h[12] = sqrt(h[12] / (h[13] + 1.0e-30));
        h[13] = sqrt(h[13]);
        h[14] = sqrt(h[14]);
    } else {
        h[12] = h[13] = h[14] = 0.0;
    }
    for (int k = 0; k < 15; ++k) S.dscal[2 + k] = h[k];
    if (!log) return;
    const int k = *counter;
    *counter = k + 1;
    if (S.status->code != 0 && S.status->step == 0) S.status->step = k + 1;
    if (k >= cap) return;
    double* r = log + (size_t)k * LOG_FIELDS;
    r[0] = S.dscal[0];
    r[1] = cg->iterations;
    r[2] = cg->initial_l2;
    r[3] = cg->final_l2;
    r[4] = cg->rel;
    r[5] = cg->max_abs;
    r[6] = cg->converged;
    for (int q = 0; q < 15; ++q) r[7 + q] = h[q];
    r[22] = S.dscal[1];
    r[23] = cg->outer;
}


// gstif = gstifE * dt (TimeStep.cpp:873-892), materialised only on request
__global__ void k_gstif(DevState S, double* out)
{
    const int E = S.P.E;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const double dt = S.delte[e];
    for (int q = 0; q < 6; ++q) out[(size_t)e * 6 + q] = (S.mat[e] != 0) ? 0.0 : S.gstifE[(size_t)q * E + e] * dt;
}

}  // namespace cbs3d

namespace cbs3d {

// ============================================ reference-order pressure matvec
// MatrixVectorCalc::pressureMultiply (src/linalg/MatrixVectorCalc.cpp:125-205):
// one launch per colour, race-free scatter within the colour, so every nodal
// sum has the reference's operand order and rounding.
__global__ void k_matvec_color(DevState S, const int* color_elem, int beg, int end, const double* gst,
                               const double* x, double* y)
{
    const int k = beg + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= end) return;
    const int e = color_elem[k] - 1;
    if (S.mat[e] != 0) return;
    const int4 n = S.intma[e];
    const double x1 = x[n.x], x2 = x[n.y], x3 = x[n.z], x4 = x[n.w];
    const double* g = gst + (size_t)e * 6;
    const double a12 = g[0], a13 = g[1], a14 = g[2], a23 = g[3], a24 = g[4], a34 = g[5];
    y[n.x] += a12 * x2 + a13 * x3 + a14 * x4;
    y[n.y] += a12 * x1 + a23 * x3 + a24 * x4;
    y[n.z] += a13 * x1 + a23 * x2 + a34 * x4;
    y[n.w] += a14 * x1 + a24 * x2 + a34 * x3;
}

__global__ void k_matvec_diag(DevState S, const double* x, double* y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.P.N) return;
    double v = y[i] + S.pdiag[i] * x[i];
    if (S.nflag[i] & 4) v = x[i];
    y[i] = v;
}

}  // namespace cbs3d
