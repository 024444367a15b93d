/* Test infrastructure only: CPU restatement of the CBS3D++_SI step path.
 * See cbs_oracle.h.  Pinned against the reference itself through the golden
 * fixtures under tests/golden/ (made by tests/golden/make_golden.py with the
 * reference compiled by oracle/Makefile).  Every floating-point expression
 * keeps the reference's association and evaluation order.
 */
#include "cbs_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* RunConfig constants (include/cbs/core/RunConfig.hpp:296-322) */
static const double FCON1 = 1.0 / 24.0, FCON2 = 1.0 / 12.0, FCON3 = 1.0 / 6.0, FCON4 = 1.0 / 3.0;
static const double FDIF1 = 1.0 / 6.0, FDIF2 = 1.0 / 3.0;
static const double MASS_FACTOR = 1.0 / 24.0;

/* Local face f (1..4) is opposite local node f
 * (include/cbs/core/CBSStateSI.hpp:342-387). */
static const int IPPN1[5][3] = {{0, 0, 0}, {3, 2, 4}, {3, 4, 1}, {1, 4, 2}, {1, 2, 3}};

enum { BC500 = 500, BC501 = 501, BC502 = 502, BC503 = 503, BC504 = 504, BC506 = 506,
       BC507 = 507, BC508 = 508, BC510 = 510, BC511 = 511, BC520 = 520, BC530 = 530,
       BC532 = 532, BC901 = 901, BC902 = 902 };

struct orc_state {
    orc_params p;
    int E, N, NB;
    int *intma;      /* 4E 1-based */
    double *coord;   /* 3N */
    int *iside;      /* 6*NB: n1 n2 n3 localface parent bc */
    int *mat;        /* E */
    double *rho, *cp, *kc, *mu, *rho_cp, *alpha, *qvol;
    double ani, inlet_u_mf, dtreal;
    /* geometry */
    double *dNkdx;   /* 12E: (e*3 + dim)*4 + a */
    double *detJ, *annxf /* 16E: (e*4+face)*4+c */, *face_norm /* 4NB */, *alen_e;
    double *elcoe_e, *mdiag_real, *pdiagE, *gstifE;
    /* body force (extension, no reference counterpart): f[3N] and the fluid
     * lumped mass; Step 1 adds mfluid*f to the residual when has_bforce */
    double *bforce, *mfluid;
    int has_bforce;
    int *fedge;      /* 4E */
    char *tf, *ts;   /* touches fluid / solid per node */
    int npoin_wall, *wall_list;
    int bc_fixed, *bc_list; double *bc_values;
    int ncolor, *color_ptr, *color_elem;
    /* fields */
    double *unkno, *unkn1, *pres, *pres1, *temp, *temp1, *velocity;
    double *rhs, *rhs1, *delte, *alen, *elcoe2, *elcoe2p, *pdiag, *gstif;
    double hb[15];
    double cg[5];    /* iterations, initial_l2, final_l2, relative, max_abs */
    int cg_converged;
    char err[512];
};

#define GRAD(s, e, dim, a) ((s)->dNkdx[((size_t)(e) * 3 + (dim)) * 4 + (a)])
#define ANNXF(s, e, f, c) ((s)->annxf[((size_t)(e) * 4 + (f)) * 4 + (c)])
#define NODE(s, e, a) ((s)->intma[(size_t)(e) * 4 + (a)] - 1)

static int fail(orc_state* s, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(s->err, sizeof s->err, fmt, ap);
    va_end(ap);
    return 1;
}

static double dmin(double a, double b) { return (b < a) ? b : a; }   /* std::min */
static double dmax(double a, double b) { return (a < b) ? b : a; }   /* std::max */

static void* xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

/* ---------------------------------------------------------------- BC classes
 * src/preprocess/Preprocess.cpp:57-132 */
static int is_supported_bc(int bc)
{
    switch (bc) {
    case BC500: case BC501: case BC502: case BC503: case BC504: case BC506: case BC507:
    case BC508: case BC510: case BC511: case BC520: case BC530: case BC532: case BC901:
    case BC902: return 1;
    default: return 0;
    }
}
static int is_no_slip_wall_bc(int bc)
{ return bc == BC501 || bc == BC502 || bc == BC530 || bc == BC532 || bc == BC901; }
static int is_prescribed_velocity_face_bc(int bc)
{
    return bc == BC500 || bc == BC501 || bc == BC502 || bc == BC503 || bc == BC507 ||
           bc == BC508 || bc == BC510 || bc == BC511 || bc == BC530 || bc == BC532 ||
           bc == BC901;
}

static void touch_masks(orc_state* s)
{
    memset(s->tf, 0, (size_t)s->N);
    memset(s->ts, 0, (size_t)s->N);
    for (int e = 0; e < s->E; ++e)
        for (int a = 0; a < 4; ++a) {
            const int ip = NODE(s, e, a);
            if (s->mat[e] == 0) s->tf[ip] = 1; else s->ts[ip] = 1;
        }
}

/* -------------------------------------------------------------- preprocess */

/* Preprocess::shapeFunctionDerivatives, src/preprocess/Preprocess.cpp:390-505 */
static int shape_functions(orc_state* s)
{
    for (int e = 0; e < s->E; ++e) {
        const double* c1 = s->coord + 3 * (size_t)NODE(s, e, 0);
        const double* c2 = s->coord + 3 * (size_t)NODE(s, e, 1);
        const double* c3 = s->coord + 3 * (size_t)NODE(s, e, 2);
        const double* c4 = s->coord + 3 * (size_t)NODE(s, e, 3);
        const double j11 = c2[0] - c1[0], j21 = c2[1] - c1[1], j31 = c2[2] - c1[2];
        const double j12 = c3[0] - c1[0], j22 = c3[1] - c1[1], j32 = c3[2] - c1[2];
        const double j13 = c4[0] - c1[0], j23 = c4[1] - c1[1], j33 = c4[2] - c1[2];
        const double det = j11 * (j22 * j33 - j23 * j32)
                         - j12 * (j21 * j33 - j23 * j31)
                         + j13 * (j21 * j32 - j22 * j31);
        if (det <= 0.0 || !isfinite(det))
            return fail(s, "Preprocess::shapeFunctionDerivatives - non-positive tetrahedron volume at element %d", e + 1);
        const double inv = 1.0 / det;
        const double i11 = (j22 * j33 - j23 * j32) * inv;
        const double i12 = (j13 * j32 - j12 * j33) * inv;
        const double i13 = (j12 * j23 - j13 * j22) * inv;
        const double i21 = (j23 * j31 - j21 * j33) * inv;
        const double i22 = (j11 * j33 - j13 * j31) * inv;
        const double i23 = (j13 * j21 - j11 * j23) * inv;
        const double i31 = (j21 * j32 - j22 * j31) * inv;
        const double i32 = (j12 * j31 - j11 * j32) * inv;
        const double i33 = (j11 * j22 - j12 * j21) * inv;
        GRAD(s, e, 0, 1) = i11; GRAD(s, e, 1, 1) = i12; GRAD(s, e, 2, 1) = i13;
        GRAD(s, e, 0, 2) = i21; GRAD(s, e, 1, 2) = i22; GRAD(s, e, 2, 2) = i23;
        GRAD(s, e, 0, 3) = i31; GRAD(s, e, 1, 3) = i32; GRAD(s, e, 2, 3) = i33;
        GRAD(s, e, 0, 0) = -(i11 + i21 + i31);
        GRAD(s, e, 1, 0) = -(i12 + i22 + i32);
        GRAD(s, e, 2, 0) = -(i13 + i23 + i33);
        s->detJ[e] = det;
    }
    return 0;
}

static void sort3(int* v)
{
    int t;
    if (v[1] < v[0]) { t = v[0]; v[0] = v[1]; v[1] = t; }
    if (v[2] < v[1]) { t = v[1]; v[1] = v[2]; v[2] = t; }
    if (v[1] < v[0]) { t = v[0]; v[0] = v[1]; v[1] = t; }
}

/* Preprocess::assignBoundaryFaceNumbers, src/preprocess/Preprocess.cpp:523-574 */
static int assign_face_numbers(orc_state* s)
{
    for (int ib = 0; ib < s->NB; ++ib) {
        int* r = s->iside + 6 * (size_t)ib;
        const int parent = r[4];
        if (parent < 1 || parent > s->E)
            return fail(s, "Preprocess::assignBoundaryFaceNumbers - invalid parent tetrahedron at boundary face %d", ib + 1);
        int bf[3] = {r[0], r[1], r[2]};
        sort3(bf);
        int matched = 0;
        for (int is = 1; is <= 4; ++is) {
            int ef[3];
            for (int k = 0; k < 3; ++k) ef[k] = s->intma[(size_t)(parent - 1) * 4 + IPPN1[is][k] - 1];
            sort3(ef);
            if (bf[0] == ef[0] && bf[1] == ef[1] && bf[2] == ef[2]) { matched = is; break; }
        }
        if (!matched)
            return fail(s, "Preprocess::assignBoundaryFaceNumbers - boundary face %d does not match any face of parent tetrahedron %d", ib + 1, parent);
        r[3] = matched;
    }
    return 0;
}

/* Preprocess::getNormals, src/preprocess/Preprocess.cpp:601-679 */
static int get_normals(orc_state* s)
{
    for (int e = 0; e < s->E; ++e)
        for (int is = 1; is <= 4; ++is) {
            const double* p1 = s->coord + 3 * (size_t)NODE(s, e, IPPN1[is][0] - 1);
            const double* p2 = s->coord + 3 * (size_t)NODE(s, e, IPPN1[is][1] - 1);
            const double* p3 = s->coord + 3 * (size_t)NODE(s, e, IPPN1[is][2] - 1);
            const double* po = s->coord + 3 * (size_t)NODE(s, e, is - 1);
            const double e1x = p2[0] - p1[0], e1y = p2[1] - p1[1], e1z = p2[2] - p1[2];
            const double e2x = p3[0] - p1[0], e2y = p3[1] - p1[1], e2z = p3[2] - p1[2];
            double ax = e1y * e2z - e1z * e2y;
            double ay = e1z * e2x - e1x * e2z;
            double az = e1x * e2y - e1y * e2x;
            const double amag = sqrt(ax * ax + ay * ay + az * az);
            if (amag <= 0.0 || !isfinite(amag))
                return fail(s, "Preprocess::getNormals - zero-area face at element %d, face %d", e + 1, is);
            const double fx = (p1[0] + p2[0] + p3[0]) / 3.0;
            const double fy = (p1[1] + p2[1] + p3[1]) / 3.0;
            const double fz = (p1[2] + p2[2] + p3[2]) / 3.0;
            const double vx = po[0] - fx, vy = po[1] - fy, vz = po[2] - fz;
            if (ax * vx + ay * vy + az * vz > 0.0) { ax = -ax; ay = -ay; az = -az; }
            ANNXF(s, e, is - 1, 0) = 0.5 * ax;
            ANNXF(s, e, is - 1, 1) = 0.5 * ay;
            ANNXF(s, e, is - 1, 2) = 0.5 * az;
            ANNXF(s, e, is - 1, 3) = 0.5 * amag;
        }
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        for (int c = 0; c < 4; ++c) s->face_norm[4 * (size_t)ib + c] = ANNXF(s, r[4] - 1, r[3] - 1, c);
    }
    return 0;
}

/* Preprocess::massMatrix, src/preprocess/Preprocess.cpp:721-809 (the M_L-M_C
 * correction arrays it also fills are never read by the step path). */
static int mass_matrix(orc_state* s)
{
    double* thermal = xcalloc((size_t)s->N, sizeof(double));
    memset(s->mdiag_real, 0, sizeof(double) * (size_t)s->N);
    memset(s->mfluid, 0, sizeof(double) * (size_t)s->N);
    for (int e = 0; e < s->E; ++e) {
        if (s->detJ[e] <= 0.0 || !isfinite(s->detJ[e])) { free(thermal); return fail(s, "Preprocess::massMatrix - invalid detJ at element %d", e + 1); }
        if (s->rho_cp[e] <= 0.0 || !isfinite(s->rho_cp[e])) { free(thermal); return fail(s, "Preprocess::massMatrix - invalid rho*cp at element %d", e + 1); }
        const double nm = s->detJ[e] * MASS_FACTOR;
        const double nc = s->rho_cp[e] * nm;
        for (int a = 0; a < 4; ++a) {
            const int ip = NODE(s, e, a);
            s->mdiag_real[ip] += nm;
            if (s->mat[e] == 0) s->mfluid[ip] += nm;
            thermal[ip] += nc;
            s->elcoe_e[(size_t)e * 4 + a] = nm;
        }
    }
    for (int ip = 0; ip < s->N; ++ip) {
        if (s->mdiag_real[ip] <= 0.0 || !isfinite(s->mdiag_real[ip])) { free(thermal); return fail(s, "Preprocess::massMatrix - non-positive lumped mass at node %d", ip + 1); }
        if (thermal[ip] <= 0.0 || !isfinite(thermal[ip])) { free(thermal); return fail(s, "Preprocess::massMatrix - non-positive thermal capacitance at node %d", ip + 1); }
        s->elcoe2[ip] = 1.0 / s->mdiag_real[ip];
        s->elcoe2p[ip] = 1.0 / thermal[ip];
    }
    free(thermal);
    return 0;
}

/* Preprocess::classifyFaceEdges, src/preprocess/Preprocess.cpp:820-843 */
static void classify_face_edges(orc_state* s)
{
    memset(s->fedge, 0, sizeof(int) * 4 * (size_t)s->E);
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        s->fedge[(size_t)(r[4] - 1) * 4 + r[3] - 1] = is_prescribed_velocity_face_bc(r[5]) ? 1 : 2;
    }
}

/* Preprocess::elementSize, src/preprocess/Preprocess.cpp:863-905 */
static int element_size(orc_state* s)
{
    for (int e = 0; e < s->E; ++e) {
        const double three_volume = 0.5 * s->detJ[e];
        double hmin = DBL_MAX;
        for (int is = 0; is < 4; ++is) {
            const double area = ANNXF(s, e, is, 3);
            if (area <= 0.0 || !isfinite(area)) return fail(s, "Preprocess::elementSize - invalid face area at element %d, face %d", e + 1, is + 1);
            hmin = dmin(hmin, three_volume / area);
        }
        if (hmin <= 0.0 || !isfinite(hmin)) return fail(s, "Preprocess::elementSize - invalid characteristic length at element %d", e + 1);
        s->alen_e[e] = hmin;
    }
    return 0;
}

/* Preprocess::wallDetermination, src/preprocess/Preprocess.cpp:932-1031
 * (the averaged wall normals are not read by the step path). */
static int wall_determination(orc_state* s)
{
    int* mark = xcalloc((size_t)s->N, sizeof(int));
    s->npoin_wall = 0;
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        if (!is_no_slip_wall_bc(r[5])) continue;
        const double area = s->face_norm[4 * (size_t)ib + 3];
        if (area <= 0.0 || !isfinite(area)) { free(mark); return fail(s, "Preprocess::wallDetermination - invalid boundary face area"); }
        for (int k = 0; k < 3; ++k) {
            const int ip = r[k] - 1;
            if (!mark[ip]) { s->wall_list[s->npoin_wall++] = ip + 1; mark[ip] = 1; }
        }
    }
    for (int ip = 0; ip < s->N; ++ip)
        if (s->tf[ip] && s->ts[ip] && !mark[ip]) { s->wall_list[s->npoin_wall++] = ip + 1; mark[ip] = 1; }
    free(mark);
    return 0;
}

/* Preprocess::computeMassFlowInletVelocity, src/preprocess/Preprocess.cpp:1054-1112 */
static int massflow_velocity(orc_state* s)
{
    if (s->p.massflow_enabled < 1) return 0;
    if (s->p.inlet_density <= 0.0 || !isfinite(s->p.inlet_density)) return fail(s, "Preprocess::computeMassFlowInletVelocity - inlet density must be positive");
    double area = 0.0;
    int nf = 0;
    for (int ib = 0; ib < s->NB; ++ib) {
        if (s->iside[6 * (size_t)ib + 5] != BC511) continue;
        area += s->face_norm[4 * (size_t)ib + 3];
        ++nf;
    }
    if (nf < 1) return fail(s, "Preprocess::computeMassFlowInletVelocity - mass-flow inlet enabled but no BC_ID 511 faces were found");
    s->inlet_u_mf = s->p.inlet_mass_flow_rate / (s->p.inlet_density * area);
    return 0;
}

/* Preprocess::detectPressureBoundaryNodes, src/preprocess/Preprocess.cpp:1152-1242 */
static int pressure_nodes(orc_state* s)
{
    char* fixed = xcalloc((size_t)s->N, 1);
    s->bc_fixed = 0;
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        if (r[5] != BC520) continue;
        for (int k = 0; k < 3; ++k) {
            const int ip = r[k] - 1;
            if (!s->tf[ip]) { free(fixed); return fail(s, "Preprocess::detectPressureBoundaryNodes - pressure outlet node %d is not connected to any fluid element", ip + 1); }
            if (!fixed[ip]) {
                fixed[ip] = 1;
                s->bc_list[s->bc_fixed] = ip + 1;
                s->bc_values[s->bc_fixed] = s->p.outlet_pressure_gauge;
                ++s->bc_fixed;
            }
        }
    }
    free(fixed);
    if (s->bc_fixed < 1) {
        int ip = s->p.pnode;
        if (ip < 1 || ip > s->N || !s->tf[ip - 1]) {
            ip = 0;
            for (int c = 1; c <= s->N; ++c) if (s->tf[c - 1]) { ip = c; break; }
        }
        if (ip < 1) return fail(s, "Preprocess::detectPressureBoundaryNodes - no fluid-connected node available for pressure reference");
        s->bc_fixed = 1;
        s->bc_list[0] = ip;
        s->bc_values[0] = s->p.outlet_pressure_gauge;
    }
    return 0;
}

/* Coloring::build, include/cbs/parallel/Coloring.hpp:27-97 */
static void coloring(orc_state* s)
{
    const int E = s->E, N = s->N;
    int* ptr = xcalloc((size_t)N + 2, sizeof(int));
    for (int e = 0; e < E; ++e) for (int a = 0; a < 4; ++a) ++ptr[NODE(s, e, a) + 2];
    for (int i = 2; i <= N + 1; ++i) ptr[i] += ptr[i - 1];
    int* n2e = xcalloc((size_t)4 * E, sizeof(int));
    for (int e = 0; e < E; ++e) for (int a = 0; a < 4; ++a) n2e[ptr[NODE(s, e, a) + 1]++] = e;
    /* ptr[ip] .. ptr[ip+1] now spans node ip's elements in element order */
    int* color = xcalloc((size_t)E, sizeof(int));
    int cap = 64, ncolor = 0;
    int* stamp = malloc(sizeof(int) * (size_t)cap);
    for (int c = 0; c < cap; ++c) stamp[c] = -1;
    int stamp_size = 0;
    for (int e = 0; e < E; ++e) color[e] = -1;
    for (int e = 0; e < E; ++e) {
        for (int a = 0; a < 4; ++a) {
            const int ip = NODE(s, e, a);
            for (int k = ptr[ip]; k < ptr[ip + 1]; ++k) {
                const int cj = color[n2e[k]];
                if (cj >= 0) {
                    if (cj >= stamp_size) {
                        while (cj >= cap) {
                            stamp = realloc(stamp, sizeof(int) * (size_t)cap * 2);
                            for (int c = cap; c < 2 * cap; ++c) stamp[c] = -1;
                            cap *= 2;
                        }
                        stamp_size = cj + 1;
                    }
                    stamp[cj] = e;
                }
            }
        }
        int c = 0;
        while (c < stamp_size && stamp[c] == e) ++c;
        color[e] = c;
        if (c + 1 > ncolor) ncolor = c + 1;
    }
    s->ncolor = ncolor;
    s->color_ptr = xcalloc((size_t)ncolor + 1, sizeof(int));
    s->color_elem = xcalloc((size_t)E, sizeof(int));
    for (int e = 0; e < E; ++e) ++s->color_ptr[color[e] + 1];
    for (int c = 0; c < ncolor; ++c) s->color_ptr[c + 1] += s->color_ptr[c];
    int* off = xcalloc((size_t)ncolor + 1, sizeof(int));
    memcpy(off, s->color_ptr, sizeof(int) * ((size_t)ncolor + 1));
    for (int e = 0; e < E; ++e) s->color_elem[off[color[e]]++] = e + 1;
    free(off); free(color); free(stamp); free(n2e); free(ptr);
}

/* ------------------------------------------------------------ boundaries */

static void unit_normal(const orc_state* s, int ib, double* nx, double* ny, double* nz)
{
    const double* fn = s->face_norm + 4 * (size_t)ib;
    *nx = fn[0] / fn[3]; *ny = fn[1] / fn[3]; *nz = fn[2] / fn[3];
}

static void set_vel(orc_state* s, int ip, double u, double v, double w)
{ s->unkno[3 * (size_t)ip] = u; s->unkno[3 * (size_t)ip + 1] = v; s->unkno[3 * (size_t)ip + 2] = w; }

/* Boundary::applySymmetry, src/boundary/Boundary.cpp:275-310 */
static void apply_symmetry(orc_state* s)
{
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        if (r[5] != BC506) continue;
        double nx, ny, nz;
        unit_normal(s, ib, &nx, &ny, &nz);
        for (int k = 0; k < 3; ++k) {
            double* u = s->unkno + 3 * (size_t)(r[k] - 1);
            const double un = u[0] * nx + u[1] * ny + u[2] * nz;
            u[0] -= un * nx; u[1] -= un * ny; u[2] -= un * nz;
        }
    }
}

static double bfs_profile_u(double y)
{
    return 0.6624 * pow(y, 6) - 7.5547 * pow(y, 5) + 33.9 * pow(y, 4) - 75.283 * pow(y, 3)
         + 83.368 * pow(y, 2) - 37.793 * y + 2.6959;
}

/* Boundary::applyVelocity, src/boundary/Boundary.cpp:341-508 */
static void apply_velocity(orc_state* s)
{
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        const int bc = r[5];
        double nx = 0.0, ny = 0.0, nz = 0.0;
        if (bc == BC511) unit_normal(s, ib, &nx, &ny, &nz);
        for (int k = 0; k < 3; ++k) {
            const int ip = r[k] - 1;
            if (bc == BC500) set_vel(s, ip, s->p.inlet_u, s->p.inlet_v, s->p.inlet_w);
            else if (bc == BC501 || bc == BC502) set_vel(s, ip, 0.0, 0.0, 0.0);
            else if (bc == BC503) set_vel(s, ip, 1.0, 0.0, 0.0);
            else if (bc == BC504 || bc == BC520 || bc == BC506) continue;
            else if (bc == BC507) set_vel(s, ip, bfs_profile_u(s->coord[3 * (size_t)ip + 1]), 0.0, 0.0);
            else if (bc == BC508) {
                const double y = s->coord[3 * (size_t)ip + 1];
                set_vel(s, ip, 6.0 * y * (1.0 - y), 0.0, 0.0);
            }
            else if (bc == BC510) set_vel(s, ip, s->p.inlet_u, s->p.inlet_v, s->p.inlet_w);
            else if (bc == BC511) set_vel(s, ip, -s->inlet_u_mf * nx, -s->inlet_u_mf * ny, -s->inlet_u_mf * nz);
            else if (bc == BC530 || bc == BC532 || bc == BC901) set_vel(s, ip, 0.0, 0.0, 0.0);
        }
    }
    for (int iw = 0; iw < s->npoin_wall; ++iw) set_vel(s, s->wall_list[iw] - 1, 0.0, 0.0, 0.0);
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        if (r[5] != BC500) continue;
        for (int k = 0; k < 3; ++k) set_vel(s, r[k] - 1, s->p.inlet_u, s->p.inlet_v, s->p.inlet_w);
    }
    for (int ip = 0; ip < s->N; ++ip) if (s->ts[ip]) set_vel(s, ip, 0.0, 0.0, 0.0);
}

/* Boundary::applyOutletBackflowControl, src/boundary/Boundary.cpp:672-723 */
static void apply_backflow(orc_state* s)
{
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        if (r[5] != BC520) continue;
        double nx, ny, nz;
        unit_normal(s, ib, &nx, &ny, &nz);
        for (int k = 0; k < 3; ++k) {
            const int ip = r[k] - 1;
            if (s->ts[ip]) { set_vel(s, ip, 0.0, 0.0, 0.0); continue; }
            double* u = s->unkno + 3 * (size_t)ip;
            const double un = u[0] * nx + u[1] * ny + u[2] * nz;
            if (un < 0.0) { u[0] -= un * nx; u[1] -= un * ny; u[2] -= un * nz; }
        }
    }
}

/* Steps.cpp enforce_zero_velocity_in_solid, src/solver/Steps.cpp:102-121 */
static void zero_solid_velocity(orc_state* s)
{
    for (int e = 0; e < s->E; ++e) {
        if (s->mat[e] == 0) continue;
        for (int a = 0; a < 4; ++a) set_vel(s, NODE(s, e, a), 0.0, 0.0, 0.0);
    }
}

/* apply_velocity_boundary_package, src/solver/Steps.cpp:170-176 */
static void velocity_bc_package(orc_state* s)
{
    apply_symmetry(s);
    apply_velocity(s);
    apply_backflow(s);
    zero_solid_velocity(s);
}

/* Boundary::applyTemperature, src/boundary/Boundary.cpp:529-626 */
static void apply_temperature(orc_state* s)
{
    for (int ib = 0; ib < s->NB; ++ib) {
        const int* r = s->iside + 6 * (size_t)ib;
        const int bc = r[5];
        for (int k = 0; k < 3; ++k) {
            const int ip = r[k] - 1;
            if (bc == BC501) s->temp[ip] = 1.0;
            else if (bc == BC502 || bc == BC503 || bc == BC508) s->temp[ip] = 0.0;
            else if (bc == BC510 || bc == BC511) s->temp[ip] = s->p.inlet_temperature;
        }
    }
}

/* Boundary::applyPressure, src/boundary/Boundary.cpp:642-652 */
static void apply_pressure(orc_state* s)
{
    for (int i = 0; i < s->bc_fixed; ++i) s->pres[s->bc_list[i] - 1] = s->bc_values[i];
}

static void velocity_magnitude(orc_state* s)
{
    /* Solver::updateVelocityMagnitude, src/solver/Solver.cpp:689-699 */
    for (int ip = 0; ip < s->N; ++ip) {
        const double u = s->unkno[3 * (size_t)ip], v = s->unkno[3 * (size_t)ip + 1], w = s->unkno[3 * (size_t)ip + 2];
        s->velocity[ip] = sqrt(u * u + v * v + w * w + 1.0e-16);
    }
}

/* PressureAssembly::buildElementPressureTerms, src/assembly/PressureAssembly.cpp:136-178 */
static double grad_dot(const orc_state* s, int e, int a, int b)
{
    return GRAD(s, e, 0, a) * GRAD(s, e, 0, b) + GRAD(s, e, 1, a) * GRAD(s, e, 1, b) +
           GRAD(s, e, 2, a) * GRAD(s, e, 2, b);
}
static void element_pressure_terms(orc_state* s)
{
    static const int PAIR[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    memset(s->pdiagE, 0, sizeof(double) * 4 * (size_t)s->E);
    memset(s->gstifE, 0, sizeof(double) * 6 * (size_t)s->E);
    for (int e = 0; e < s->E; ++e) {
        if (s->mat[e] != 0) continue;
        const double vol = s->detJ[e] / 6.0;
        for (int a = 0; a < 4; ++a) s->pdiagE[(size_t)e * 4 + a] = vol * grad_dot(s, e, a, a);
        for (int g = 0; g < 6; ++g) s->gstifE[(size_t)e * 6 + g] = vol * grad_dot(s, e, PAIR[g][0], PAIR[g][1]);
    }
}

/* ---------------------------------------------------------------- create */

orc_state* orc_create(const orc_params* p, int nelem, int npoin, int nboun,
                      const int* intma, const double* coord, const int* bface,
                      const int* mat_elem, const double* rho, const double* cp,
                      const double* k, const double* mu, const double* qvol,
                      char* err, size_t errlen)
{
    orc_state* s = xcalloc(1, sizeof(orc_state));
    s->p = *p;
    s->E = nelem; s->N = npoin; s->NB = nboun;
    const size_t E = (size_t)nelem, N = (size_t)npoin, NB = (size_t)nboun;
    s->intma = malloc(sizeof(int) * 4 * E); memcpy(s->intma, intma, sizeof(int) * 4 * E);
    s->coord = malloc(sizeof(double) * 3 * N); memcpy(s->coord, coord, sizeof(double) * 3 * N);
    s->iside = xcalloc(6 * NB, sizeof(int));
    for (size_t ib = 0; ib < NB; ++ib) {
        s->iside[6 * ib + 0] = bface[5 * ib + 0];
        s->iside[6 * ib + 1] = bface[5 * ib + 1];
        s->iside[6 * ib + 2] = bface[5 * ib + 2];
        s->iside[6 * ib + 3] = 0;
        s->iside[6 * ib + 4] = bface[5 * ib + 3];
        s->iside[6 * ib + 5] = bface[5 * ib + 4];
    }
    s->mat = xcalloc(E, sizeof(int));
    s->rho = xcalloc(E, sizeof(double)); s->cp = xcalloc(E, sizeof(double));
    s->kc = xcalloc(E, sizeof(double)); s->mu = xcalloc(E, sizeof(double));
    s->rho_cp = xcalloc(E, sizeof(double)); s->alpha = xcalloc(E, sizeof(double));
    s->qvol = xcalloc(E, sizeof(double));
    s->dNkdx = xcalloc(12 * E, sizeof(double)); s->detJ = xcalloc(E, sizeof(double));
    s->annxf = xcalloc(16 * E, sizeof(double)); s->face_norm = xcalloc(4 * NB, sizeof(double));
    s->alen_e = xcalloc(E, sizeof(double)); s->elcoe_e = xcalloc(4 * E, sizeof(double));
    s->mdiag_real = xcalloc(N, sizeof(double));
    s->mfluid = xcalloc(N, sizeof(double)); s->bforce = xcalloc(3 * N, sizeof(double));
    s->pdiagE = xcalloc(4 * E, sizeof(double)); s->gstifE = xcalloc(6 * E, sizeof(double));
    s->fedge = xcalloc(4 * E, sizeof(int));
    s->tf = xcalloc(N, 1); s->ts = xcalloc(N, 1);
    s->wall_list = xcalloc(N, sizeof(int));
    s->bc_list = xcalloc(N, sizeof(int)); s->bc_values = xcalloc(N, sizeof(double));
    s->unkno = xcalloc(3 * N, sizeof(double)); s->unkn1 = xcalloc(3 * N, sizeof(double));
    s->pres = xcalloc(N, sizeof(double)); s->pres1 = xcalloc(N, sizeof(double));
    s->temp = xcalloc(N, sizeof(double)); s->temp1 = xcalloc(N, sizeof(double));
    s->velocity = xcalloc(N, sizeof(double));
    s->rhs = xcalloc(3 * N, sizeof(double)); s->rhs1 = xcalloc(N, sizeof(double));
    s->delte = xcalloc(E, sizeof(double)); s->alen = xcalloc(N, sizeof(double));
    s->elcoe2 = xcalloc(N, sizeof(double)); s->elcoe2p = xcalloc(N, sizeof(double));
    s->pdiag = xcalloc(N, sizeof(double)); s->gstif = xcalloc(6 * E, sizeof(double));

    int rc = 0;
    for (size_t e = 0; e < E; ++e)
        for (int a = 0; a < 4; ++a)
            if (intma[4 * e + a] < 1 || intma[4 * e + a] > npoin) { rc = fail(s, "MeshIO::readMeshFile - connectivity node out of range"); goto done; }

    /* materials: MeshIO::readMaterialPropertyFile (src/io/MeshIO.cpp:1590-1620)
     * or the flow-only defaults (src/io/MeshIO.cpp:401-423) */
    for (size_t e = 0; e < E; ++e) {
        if (p->material_enabled > 0) {
            s->mat[e] = mat_elem ? mat_elem[e] : 0;
            s->rho[e] = rho[e]; s->cp[e] = cp[e]; s->kc[e] = k[e]; s->mu[e] = mu[e]; s->qvol[e] = qvol[e];
            s->rho_cp[e] = s->rho[e] * s->cp[e];
            s->alpha[e] = s->kc[e] / s->rho_cp[e];
        } else {
            s->mat[e] = 0; s->rho[e] = 1.0; s->cp[e] = 1.0; s->rho_cp[e] = 1.0;
            s->mu[e] = 0.0; s->kc[e] = 1.0; s->alpha[e] = 1.0; s->qvol[e] = 0.0;
        }
    }

    /* MeshIO::initialiseFields, src/io/MeshIO.cpp:1627-1701 */
    for (size_t ip = 0; ip < N; ++ip) {
        s->unkno[3 * ip] = p->cinf[0]; s->unkno[3 * ip + 1] = p->cinf[1]; s->unkno[3 * ip + 2] = p->cinf[2];
        s->pres[ip] = p->cinf[3]; s->temp[ip] = p->cinf[4];
    }
    memcpy(s->unkn1, s->unkno, sizeof(double) * 3 * N);
    memcpy(s->pres1, s->pres, sizeof(double) * N);
    memcpy(s->temp1, s->temp, sizeof(double) * N);
    touch_masks(s);
    if (p->material_enabled > 0) {
        for (size_t ip = 0; ip < N; ++ip) {
            if (!s->tf[ip] && !s->ts[ip]) { rc = fail(s, "MeshIO::initialiseFields - orphan node not touched by any material element: %d", (int)ip + 1); goto done; }
            if (s->ts[ip]) for (int d = 0; d < 3; ++d) { s->unkno[3 * ip + d] = 0.0; s->unkn1[3 * ip + d] = 0.0; }
            if (s->ts[ip] && !s->tf[ip]) { s->pres[ip] = 0.0; s->pres1[ip] = 0.0; }
        }
    }
    if (p->convection_type == 1) { s->ani = p->pr; s->p.temp_calc = 1; }
    else { s->ani = 1.0 / p->re; if (p->ri > 0.0) s->p.temp_calc = 1; }
    if (p->material_enabled < 1) for (size_t e = 0; e < E; ++e) s->mu[e] = s->ani;

    /* Solver::initialise, src/solver/Solver.cpp:242-302 */
    for (size_t ib = 0; ib < NB; ++ib)
        if (!is_supported_bc(s->iside[6 * ib + 5])) { rc = fail(s, "Boundary - unsupported BC_ID %d at boundary face %d", s->iside[6 * ib + 5], (int)ib + 1); goto done; }
    if ((rc = shape_functions(s))) goto done;
    if ((rc = assign_face_numbers(s))) goto done;
    if ((rc = get_normals(s))) goto done;
    if ((rc = mass_matrix(s))) goto done;
    classify_face_edges(s);
    if ((rc = element_size(s))) goto done;
    if ((rc = wall_determination(s))) goto done;
    if ((rc = massflow_velocity(s))) goto done;
    if ((rc = pressure_nodes(s))) goto done;
    coloring(s);
    apply_temperature(s);
    apply_velocity(s);
    apply_pressure(s);
    velocity_magnitude(s);
    element_pressure_terms(s);
done:
    if (rc) {
        if (err) snprintf(err, errlen, "%s", s->err);
        orc_destroy(s);
        return NULL;
    }
    return s;
}

void orc_destroy(orc_state* s)
{
    if (!s) return;
    void* ptrs[] = {s->intma, s->coord, s->iside, s->mat, s->rho, s->cp, s->kc, s->mu, s->rho_cp,
                    s->alpha, s->qvol, s->dNkdx, s->detJ, s->annxf, s->face_norm, s->alen_e,
                    s->elcoe_e, s->mdiag_real, s->pdiagE, s->gstifE, s->fedge, s->tf, s->ts,
                    s->wall_list, s->bc_list, s->bc_values, s->color_ptr, s->color_elem,
                    s->unkno, s->unkn1, s->pres, s->pres1, s->temp, s->temp1, s->velocity,
                    s->rhs, s->rhs1, s->delte, s->alen, s->elcoe2, s->elcoe2p, s->pdiag, s->gstif,
                    s->bforce, s->mfluid};
    for (size_t i = 0; i < sizeof ptrs / sizeof ptrs[0]; ++i) free(ptrs[i]);
    free(s);
}

const char* orc_error(orc_state* s) { return s ? s->err : "null state"; }

/* ------------------------------------------------------------- time step */

static double node_speed(const orc_state* s, int ip)
{
    const double* u = s->unkno + 3 * (size_t)ip;
    return sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
}

/* compute_nodal_lengths_from_elements, src/timestep/TimeStep.cpp:319-355 */
static int nodal_lengths(orc_state* s)
{
    for (int ip = 0; ip < s->N; ++ip) s->alen[ip] = DBL_MAX;
    for (int e = 0; e < s->E; ++e) {
        if (s->detJ[e] <= 0.0 || !isfinite(s->detJ[e])) return fail(s, "TimeStep - invalid detJ in nodal length; run Preprocess first");
        const double volum = 0.5 * s->detJ[e];
        for (int a = 0; a < 4; ++a) {
            const double area = ANNXF(s, e, a, 3);
            if (area <= 0.0 || !isfinite(area)) return fail(s, "TimeStep - invalid face area in nodal length; run Preprocess::getNormals first");
            const int ip = NODE(s, e, a);
            s->alen[ip] = dmin(s->alen[ip], volum / area);
        }
    }
    return 0;
}

static int standard_length(orc_state* s, int e, double* h)
{
    *h = s->alen_e[e];
    if (*h <= 0.0 || !isfinite(*h)) return fail(s, "TimeStep - invalid alen_e at element %d. Run Preprocess::elementSize before timestep computation.", e + 1);
    return 0;
}

/* timestep_length / timestep_speed / element_diffusivity_for_timestep /
 * local_stability_dt, src/timestep/TimeStep.cpp:114-300 */
static int element_dt(orc_state* s, int e, double* dt_out)
{
    double h;
    if (standard_length(s, e, &h)) return 1;
    if (s->p.htype == 2) {
        double hn = 0.0;
        int ok = 1;
        for (int a = 0; a < 4; ++a) {
            const double al = s->alen[NODE(s, e, a)];
            if (al <= 0.0 || !isfinite(al)) { ok = 0; break; }
            hn += al;
        }
        hn = ok ? hn / 4.0 : h;
        h = dmin(h, hn);
    }
    double speed;
    if (s->p.htype == 3) {
        double u = 0.0, v = 0.0, w = 0.0;
        for (int a = 0; a < 4; ++a) {
            const double* x = s->unkno + 3 * (size_t)NODE(s, e, a);
            u += x[0]; v += x[1]; w += x[2];
        }
        u /= 4.0; v /= 4.0; w /= 4.0;
        speed = sqrt(u * u + v * v + w * w);
    } else {
        speed = 0.0;
        for (int a = 0; a < 4; ++a) speed = dmax(speed, node_speed(s, NODE(s, e, a)));
    }
    double diff = s->ani;
    if (s->p.dimensional_mode > 0 && s->p.material_enabled > 0) {
        if (s->alpha[e] <= 0.0 || !isfinite(s->alpha[e])) return fail(s, "TimeStep - invalid thermal diffusivity alpha_e at element %d", e + 1);
        diff = s->alpha[e];
        if (s->mat[e] == 0) {
            if (s->rho[e] <= 0.0 || s->mu[e] < 0.0) return fail(s, "TimeStep - invalid fluid rho/mu at element %d", e + 1);
            diff = dmax(diff, s->mu[e] / s->rho[e]);
        }
    }
    if (diff <= 0.0 || !isfinite(diff)) return fail(s, "TimeStep - invalid timestep diffusivity at element %d", e + 1);
    const double adv = (s->mat[e] == 0) ? h / dmax(speed, 1.0e-14) : DBL_MAX;
    const double dif = h * h * (0.5 / diff);
    double dt = s->p.csafm * dmin(adv, dif);
    if (s->p.ilots == 2 && s->p.deltr > 0.0 && isfinite(s->p.deltr)) dt = dmin(dt, s->p.deltr);
    if (dt <= 0.0 || !isfinite(dt)) return fail(s, "TimeStep - invalid local stability timestep at element %d", e + 1);
    *dt_out = dt;
    return 0;
}

/* TimeStep::computeTimeStep, src/timestep/TimeStep.cpp:473-583.  The nodal
 * dt/beta/unit-vector arrays it also fills are never read by a later stage
 * (only the nodal lengths are, by htype=2 and the Step-2 dt check). */
int orc_time_step(orc_state* s, int iitime)
{
    if (s->p.csafm <= 0.0 || !isfinite(s->p.csafm)) return fail(s, "TimeStep - csafm must be positive");
    if (s->p.dtfix <= 0.0 || !isfinite(s->p.dtfix)) return fail(s, "TimeStep - dtfix must be positive");
    if (s->p.htype < 1 || s->p.htype > 3) return fail(s, "TimeStep - htype must be 1, 2, or 3");
    if (s->p.cbs_scheme != 1) return fail(s, "Fully explicit CBS3D mode was requested, but explicit CBS3D step kernels are not yet ported.");
    if (s->p.ilots <= -1 || s->p.dtfixed > 0 || (s->p.dtfix_end > 0 && iitime <= s->p.dtfix_end)) {
        for (int e = 0; e < s->E; ++e) s->delte[e] = s->p.dtfix;
        s->dtreal = s->p.dtfix;
        return 0;
    }
    if (nodal_lengths(s)) return 1;
    double dt_min = DBL_MAX;
    for (int e = 0; e < s->E; ++e) {
        if (element_dt(s, e, &s->delte[e])) return 1;
        dt_min = dmin(dt_min, s->delte[e]);
    }
    if (dt_min <= 0.0 || !isfinite(dt_min)) return fail(s, "TimeStep::computeTimeStep - invalid global minimum timestep");
    if (s->p.transient_on > 0 || s->p.solver_opt > 1 || s->p.dtfixed == -1 ||
        (s->p.ilots != 1 && s->p.ilots != 2))
        for (int e = 0; e < s->E; ++e) s->delte[e] = dt_min;
    s->dtreal = dt_min;
    return 0;
}

/* TimeStep::applyStep2PressureTimeStepCorrection, src/timestep/TimeStep.cpp:704-749 */
int orc_dt_correction(orc_state* s)
{
    if (s->p.step2_check < 1) return 0;
    if (s->p.csafm2 <= 0.0 || !isfinite(s->p.csafm2)) return fail(s, "TimeStep::applyStep2PressureTimeStepCorrection - csafm2 must be positive");
    for (int e = 0; e < s->E; ++e) {
        double dmn = s->delte[e];
        for (int a = 0; a < 4; ++a) {
            const int ip = NODE(s, e, a);
            const double pscale = fabs(s->pres1[ip]) + s->p.epsilon1;
            const double speed = node_speed(s, ip);
            if (speed > 1.0e-14 && pscale > 0.0) {
                double h;
                if (s->alen[ip] > 0.0) h = s->alen[ip];
                else if (standard_length(s, e, &h)) return 1;
                const double cand = s->p.csafm2 * h * pscale / speed;
                if (cand > 0.0 && isfinite(cand)) dmn = dmin(dmn, cand);
            }
        }
        s->delte[e] = dmn;
    }
    return 0;
}

/* TimeStep::updateLhsDiagonal, src/timestep/TimeStep.cpp:778-954 */
int orc_lhs(orc_state* s)
{
    const int N = s->N, E = s->E;
    memset(s->elcoe2, 0, sizeof(double) * (size_t)N);
    memset(s->elcoe2p, 0, sizeof(double) * (size_t)N);
    memset(s->pdiag, 0, sizeof(double) * (size_t)N);
    for (int e = 0; e < E; ++e) {
        const double dt = s->delte[e];
        if (dt <= 0.0 || !isfinite(dt)) return fail(s, "TimeStep::updateLhsDiagonal - non-positive local timestep at element %d", e + 1);
        for (int a = 0; a < 4; ++a) {
            const int ip = NODE(s, e, a);
            const double mass = s->elcoe_e[(size_t)e * 4 + a];
            if (mass <= 0.0 || !isfinite(mass)) return fail(s, "TimeStep::updateLhsDiagonal - invalid element-node mass");
            if (s->mat[e] == 0) s->elcoe2[ip] += mass / dt;
            s->elcoe2p[ip] += s->rho_cp[e] * mass / dt;
        }
    }
    for (int ip = 0; ip < N; ++ip) {
        if (!s->tf[ip] && !s->ts[ip]) return fail(s, "TimeStep::updateLhsDiagonal - orphan node detected at node %d", ip + 1);
        if (s->tf[ip]) {
            if (s->elcoe2[ip] <= 0.0 || !isfinite(s->elcoe2[ip])) return fail(s, "TimeStep::updateLhsDiagonal - non-positive fluid momentum mass/time diagonal at node %d", ip + 1);
            s->elcoe2[ip] = 1.0 / s->elcoe2[ip];
        } else s->elcoe2[ip] = 0.0;
        if (s->elcoe2p[ip] <= 0.0 || !isfinite(s->elcoe2p[ip])) return fail(s, "TimeStep::updateLhsDiagonal - non-positive capacitance/time diagonal at node %d", ip + 1);
        s->elcoe2p[ip] = 1.0 / s->elcoe2p[ip];
    }
    for (int e = 0; e < E; ++e) {
        const double dt = s->delte[e];
        if (s->mat[e] != 0) { for (int g = 0; g < 6; ++g) s->gstif[(size_t)e * 6 + g] = 0.0; continue; }
        for (int g = 0; g < 6; ++g) s->gstif[(size_t)e * 6 + g] = s->gstifE[(size_t)e * 6 + g] * dt;
        for (int a = 0; a < 4; ++a) s->pdiag[NODE(s, e, a)] += s->pdiagE[(size_t)e * 4 + a] * dt;
    }
    for (int ip = 0; ip < N; ++ip) {
        if (s->tf[ip]) {
            if (fabs(s->pdiag[ip]) <= 1.0e-14 || !isfinite(s->pdiag[ip])) return fail(s, "TimeStep::updateLhsDiagonal - zero pressure diagonal on fluid-connected node %d", ip + 1);
        } else if (s->ts[ip]) { s->pdiag[ip] = 0.0; s->pres[ip] = 0.0; s->rhs1[ip] = 0.0; }
    }
    for (int i = 0; i < s->bc_fixed; ++i) {
        const int ip = s->bc_list[i] - 1;
        if (!s->tf[ip]) return fail(s, "TimeStep::updateLhsDiagonal - fixed pressure node is not connected to the fluid pressure domain, node %d", ip + 1);
        s->pdiag[ip] = 1.0; s->pres[ip] = s->bc_values[i]; s->rhs1[ip] = s->bc_values[i];
    }
    return 0;
}

/* ---------------------------------------------------------------- Step 1 */

/* step1_convective_galerkin, src/assembly/MomentumAssembly.cpp:144-220 */
static void step1_convective(const orc_state* s, int e, double lunk[3][3][4], double lrhs[3][4])
{
    double ls[3][3] = {{0}}, lsf[3][3];
    const double vf = s->detJ[e] * FCON1;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int a = 0; a < 4; ++a) ls[i][j] += lunk[i][j][a];
    for (int a = 0; a < 4; ++a) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j)
        lrhs[i][a] += GRAD(s, e, j, a) * vf * ls[i][j];
    for (int is = 0; is < 4; ++is) {
        if (s->fedge[(size_t)e * 4 + is] == 0) continue;
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) lsf[i][j] = ls[i][j] - lunk[i][j][is];
        for (int j = 0; j < 3; ++j) {
            const double ff = ANNXF(s, e, is, j) * FCON2;
            for (int fn = 0; fn < 3; ++fn) {
                const int a = IPPN1[is + 1][fn] - 1;
                for (int i = 0; i < 3; ++i) lrhs[i][a] -= (lsf[i][j] + lunk[i][j][a]) * ff;
            }
        }
    }
}

/* step1_characteristic_correction, src/assembly/MomentumAssembly.cpp:242-345 */
static int step1_characteristic(orc_state* s, int e, double lunk[3][3][4], double lu[3][4], double lrhs[3][4])
{
    double ls[3][3] = {{0}}, lsk[3][3], um[3] = {0};
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int a = 0; a < 4; ++a) ls[i][j] += GRAD(s, e, j, a) * lunk[i][j][a];
    for (int i = 0; i < 3; ++i) { for (int a = 0; a < 4; ++a) um[i] += lu[i][a]; um[i] /= 4.0; }
    for (int i = 0; i < 3; ++i) {
        double sj = 0.0;
        for (int j = 0; j < 3; ++j) sj += ls[i][j];
        for (int k = 0; k < 3; ++k) lsk[i][k] = um[k] * sj;
    }
    const double dt = s->delte[e];
    if (dt <= 0.0 || !isfinite(dt)) return fail(s, "MomentumAssembly::assembleStep1Rhs - invalid element timestep at element %d", e + 1);
    const double ld = 0.5 * dt * s->detJ[e] * FCON3;
    const double ld2 = 0.5 * dt * FCON4;
    for (int a = 0; a < 4; ++a) for (int k = 0; k < 3; ++k) for (int i = 0; i < 3; ++i)
        lrhs[i][a] -= GRAD(s, e, k, a) * lsk[i][k] * ld;
    for (int is = 0; is < 4; ++is) {
        if (s->fedge[(size_t)e * 4 + is] == 0) continue;
        for (int k = 0; k < 3; ++k) {
            const double ff = ANNXF(s, e, is, k) * ld2;
            for (int fn = 0; fn < 3; ++fn) {
                const int a = IPPN1[is + 1][fn] - 1;
                for (int i = 0; i < 3; ++i) lrhs[i][a] += lsk[i][k] * ff;
            }
        }
    }
    return 0;
}

/* step1_diffusion, src/assembly/MomentumAssembly.cpp:369-432 */
static void step1_diffusion(const orc_state* s, int e, double lu[3][4], double ani, double lrhs[3][4])
{
    double g[3][3] = {{0}};
    for (int i = 0; i < 3; ++i) for (int a = 0; a < 4; ++a) for (int j = 0; j < 3; ++j) g[i][j] += GRAD(s, e, j, a) * lu[i][a];
    const double vf = ani * s->detJ[e] * FDIF1;
    for (int i = 0; i < 3; ++i) for (int a = 0; a < 4; ++a) for (int j = 0; j < 3; ++j)
        lrhs[i][a] -= GRAD(s, e, j, a) * g[i][j] * vf;
    const double fdf = ani * FDIF2;
    for (int is = 0; is < 4; ++is) {
        if (s->fedge[(size_t)e * 4 + is] == 0) continue;
        for (int j = 0; j < 3; ++j) {
            const double ff = ANNXF(s, e, is, j) * fdf;
            for (int i = 0; i < 3; ++i) for (int fn = 0; fn < 3; ++fn) {
                const int a = IPPN1[is + 1][fn] - 1;
                lrhs[i][a] += g[i][j] * ff;
            }
        }
    }
}

/* MomentumAssembly::assembleStep1Rhs, src/assembly/MomentumAssembly.cpp:462-554,
 * then the nodal predictor and BC package, src/solver/Steps.cpp:273-284 */
int orc_step1(orc_state* s)
{
    memset(s->rhs, 0, sizeof(double) * 3 * (size_t)s->N);
    if (s->dtreal <= 0.0 || !isfinite(s->dtreal)) return fail(s, "MomentumAssembly::assembleStep1Rhs - dtreal must be positive before Step 1 assembly");
    int bad_detj = 0;
    for (int c = 0; c < s->ncolor; ++c)
        for (int k = s->color_ptr[c]; k < s->color_ptr[c + 1]; ++k) {
            const int e = s->color_elem[k] - 1;
            if (s->mat[e] != 0) continue;
            if (s->detJ[e] <= 0.0 || !isfinite(s->detJ[e])) { bad_detj = 1; continue; }
            double lu[3][4], lunk[3][3][4], lrhs[3][4] = {{0}};
            int ipn[4];
            for (int a = 0; a < 4; ++a) {
                ipn[a] = NODE(s, e, a);
                for (int i = 0; i < 3; ++i) lu[i][a] = s->unkn1[3 * (size_t)ipn[a] + i];
            }
            for (int a = 0; a < 4; ++a) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) lunk[i][j][a] = lu[j][a] * lu[i][a];
            step1_convective(s, e, lunk, lrhs);
            if (step1_characteristic(s, e, lunk, lu, lrhs)) return 1;
            double nu = s->ani;
            if (s->p.dimensional_mode > 0 && s->p.material_enabled > 0) {
                if (s->rho[e] <= 0.0 || s->mu[e] < 0.0) return fail(s, "MomentumAssembly::assembleStep1Rhs - invalid fluid rho/mu at element %d", e + 1);
                nu = s->mu[e] / s->rho[e];
            }
            step1_diffusion(s, e, lu, nu, lrhs);
            for (int a = 0; a < 4; ++a) for (int i = 0; i < 3; ++i) s->rhs[3 * (size_t)ipn[a] + i] += lrhs[i][a];
        }
    if (bad_detj) return fail(s, "MomentumAssembly::assembleStep1Rhs - invalid detJ at one or more elements");
    if (s->has_bforce)
        for (int ip = 0; ip < s->N; ++ip)
            for (int d = 0; d < 3; ++d) s->rhs[3 * (size_t)ip + d] += s->mfluid[ip] * s->bforce[3 * (size_t)ip + d];
    for (int ip = 0; ip < s->N; ++ip)
        for (int d = 0; d < 3; ++d)
            s->unkno[3 * (size_t)ip + d] = s->unkn1[3 * (size_t)ip + d] + s->rhs[3 * (size_t)ip + d] * s->elcoe2[ip];
    velocity_bc_package(s);
    return 0;
}

/* ---------------------------------------------------------------- Step 2 */

/* PressureAssembly::assembleStep2Rhs, src/assembly/PressureAssembly.cpp:236-335 */
int orc_step2_rhs(orc_state* s)
{
    if (s->dtreal <= 0.0 || !isfinite(s->dtreal)) return fail(s, "PressureAssembly::assembleStep2Rhs - dtreal must be positive before Step 2 RHS assembly");
    memset(s->rhs1, 0, sizeof(double) * (size_t)s->N);
    for (int e = 0; e < s->E; ++e) {
        if (s->mat[e] != 0) continue;
        const double vol4 = s->detJ[e] * FCON1;
        double us[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < 4; ++a) {
            const double* u = s->unkno + 3 * (size_t)NODE(s, e, a);
            us[0] += u[0]; us[1] += u[1]; us[2] += u[2];
        }
        us[0] *= vol4; us[1] *= vol4; us[2] *= vol4;
        double lr[4];
        for (int a = 0; a < 4; ++a)
            lr[a] = GRAD(s, e, 0, a) * us[0] + GRAD(s, e, 1, a) * us[1] + GRAD(s, e, 2, a) * us[2];
        for (int is = 0; is < 4; ++is) {
            if (s->fedge[(size_t)e * 4 + is] != 1) continue;
            double fs[3] = {0.0, 0.0, 0.0};
            for (int i = 0; i < 3; ++i) {
                const double* u1 = s->unkn1 + 3 * (size_t)NODE(s, e, IPPN1[is + 1][i] - 1);
                fs[0] += u1[0]; fs[1] += u1[1]; fs[2] += u1[2];
            }
            for (int d = 0; d < 3; ++d) {
                const double nf = ANNXF(s, e, is, d) * FCON2;
                for (int i = 0; i < 3; ++i) {
                    const int ln = IPPN1[is + 1][i] - 1;
                    lr[ln] -= (fs[d] + s->unkn1[3 * (size_t)NODE(s, e, ln) + d]) * nf;
                }
            }
        }
        for (int a = 0; a < 4; ++a) s->rhs1[NODE(s, e, a)] += lr[a];
    }
    return 0;
}

/* MatrixVectorCalc::pressureMultiply, src/linalg/MatrixVectorCalc.cpp:125-205 */
int orc_pressure_multiply(orc_state* s, const double* x, double* y)
{
    memset(y, 0, sizeof(double) * (size_t)s->N);
    for (int c = 0; c < s->ncolor; ++c)
        for (int k = s->color_ptr[c]; k < s->color_ptr[c + 1]; ++k) {
            const int e = s->color_elem[k] - 1;
            if (s->mat[e] != 0) continue;
            const int i1 = NODE(s, e, 0), i2 = NODE(s, e, 1), i3 = NODE(s, e, 2), i4 = NODE(s, e, 3);
            const double x1 = x[i1], x2 = x[i2], x3 = x[i3], x4 = x[i4];
            const double* g = s->gstif + (size_t)e * 6;
            y[i1] += g[0] * x2 + g[1] * x3 + g[2] * x4;
            y[i2] += g[0] * x1 + g[3] * x3 + g[4] * x4;
            y[i3] += g[1] * x1 + g[3] * x2 + g[5] * x4;
            y[i4] += g[2] * x1 + g[4] * x2 + g[5] * x3;
        }
    for (int ip = 0; ip < s->N; ++ip) y[ip] += s->pdiag[ip] * x[ip];
    for (int i = 0; i < s->bc_fixed; ++i) y[s->bc_list[i] - 1] = x[s->bc_list[i] - 1];
    return 0;
}

/* ConjugateGradient::solvePressure, src/linalg/ConjugateGradient.cpp:584-869
 * with the serial sums of a one-thread run; then Boundary::applyPressure. */
int orc_solve_pressure(orc_state* s)
{
    const int N = s->N;
    const orc_params* p = &s->p;
    if (p->cg_max_iter < 1) return fail(s, "ConjugateGradient::solvePressure - cg_max_iter must be positive");
    if (p->relToler <= 0.0 || p->absToler <= 0.0) return fail(s, "ConjugateGradient::solvePressure - relToler and absToler must be positive");
    if (p->cg_precond < 0 || p->cg_precond > 1) return fail(s, "ConjugateGradient::solvePressure - cg_preconditioner must be 0 or 1");
    if (p->cg_conv_test < 1 || p->cg_conv_test > 3) return fail(s, "ConjugateGradient::solvePressure - cg_conv_test must be 1, 2, or 3");
    char* act = xcalloc((size_t)N, 1);
    char* fix = xcalloc((size_t)N, 1);
    double* fval = xcalloc((size_t)N, sizeof(double));
    double* r = xcalloc((size_t)N, sizeof(double));
    double* z = xcalloc((size_t)N, sizeof(double));
    double* pv = xcalloc((size_t)N, sizeof(double));
    double* Ap = xcalloc((size_t)N, sizeof(double));
    int rc = 0;
#define FREE_NODE(i) (act[i] && !fix[i])
    for (int e = 0; e < s->E; ++e) if (s->mat[e] == 0) for (int a = 0; a < 4; ++a) act[NODE(s, e, a)] = 1;
    for (int i = 0; i < s->bc_fixed; ++i) {
        const int ip = s->bc_list[i] - 1;
        if (!act[ip]) { rc = fail(s, "ConjugateGradient::solvePressure - fixed pressure node is not fluid-connected: node %d", ip + 1); goto out; }
        fix[ip] = 1; fval[ip] = s->bc_values[i];
    }
    /* impose_pressure_constraints */
#define IMPOSE() for (int ip = 0; ip < N; ++ip) { \
        if (!act[ip]) { s->pres[ip] = 0.0; s->rhs1[ip] = 0.0; s->pdiag[ip] = 0.0; continue; } \
        if (fix[ip]) { s->pres[ip] = fval[ip]; s->rhs1[ip] = fval[ip]; s->pdiag[ip] = 1.0; } }
    IMPOSE();
    orc_pressure_multiply(s, s->pres, Ap);
    for (int ip = 0; ip < N; ++ip) r[ip] = act[ip] ? s->rhs1[ip] - Ap[ip] : 0.0;
    for (int ip = 0; ip < N; ++ip) if (!FREE_NODE(ip)) { r[ip] = 0.0; Ap[ip] = 0.0; }
    double sum = 0.0;
    for (int ip = 0; ip < N; ++ip) if (FREE_NODE(ip)) sum += r[ip] * r[ip];
    const double init = sqrt(sum);
    double fin = init, rel, maxabs = 0.0;
    int iters = 0, conv = 0;
#define MAXABS(v) do { double m_ = 0.0; for (int ip = 0; ip < N; ++ip) if (FREE_NODE(ip)) m_ = dmax(m_, fabs(v[ip])); maxabs = m_; } while (0)
#define CONVERGED(rl, mx) ((p->cg_conv_test == 1) ? ((mx) <= p->absToler) : (p->cg_conv_test == 2) ? ((rl) <= p->relToler) : ((mx) <= p->absToler || (rl) <= p->relToler))
    if (init <= 1.0e-300) { rel = 0.0; MAXABS(r); conv = 1; goto done; }
    rel = 1.0;
    MAXABS(r);
    if (CONVERGED(rel, maxabs)) { conv = 1; goto done; }
    /* apply_preconditioner */
#define PRECOND() for (int ip = 0; ip < N; ++ip) { \
        if (!FREE_NODE(ip)) { z[ip] = 0.0; continue; } \
        if (p->cg_precond == 0) { if (!isfinite(r[ip])) { rc = fail(s, "ConjugateGradient::solvePressure - invalid pressure residual at node %d", ip + 1); goto out; } z[ip] = r[ip]; continue; } \
        const double dg = s->pdiag[ip]; \
        if (!isfinite(dg) || dg <= 1.0e-30) { rc = fail(s, "ConjugateGradient::solvePressure - invalid Jacobi pressure diagonal at active node %d", ip + 1); goto out; } \
        if (!isfinite(r[ip])) { rc = fail(s, "ConjugateGradient::solvePressure - invalid pressure residual at node %d", ip + 1); goto out; } \
        z[ip] = r[ip] / dg; }
    PRECOND();
    for (int ip = 0; ip < N; ++ip) pv[ip] = FREE_NODE(ip) ? z[ip] : 0.0;
    double rz = 0.0;
    for (int ip = 0; ip < N; ++ip) if (FREE_NODE(ip)) rz += r[ip] * z[ip];
    if (rz <= 1.0e-300 || !isfinite(rz)) { rc = fail(s, "ConjugateGradient::solvePressure - invalid initial preconditioned residual dot product."); goto out; }
    for (int it = 1; it <= p->cg_max_iter; ++it) {
        orc_pressure_multiply(s, pv, Ap);
        for (int ip = 0; ip < N; ++ip) if (!FREE_NODE(ip)) Ap[ip] = 0.0;
        double pAp = 0.0;
        for (int ip = 0; ip < N; ++ip) if (FREE_NODE(ip)) pAp += pv[ip] * Ap[ip];
        if (fabs(pAp) <= 1.0e-300 || !isfinite(pAp)) { rc = fail(s, "ConjugateGradient::solvePressure - breakdown: invalid pAp"); goto out; }
        const double alpha = rz / pAp;
        for (int ip = 0; ip < N; ++ip) if (FREE_NODE(ip)) { s->pres[ip] += alpha * pv[ip]; r[ip] -= alpha * Ap[ip]; }
        IMPOSE();
        for (int ip = 0; ip < N; ++ip) if (!FREE_NODE(ip)) r[ip] = 0.0;
        iters = it;
        sum = 0.0;
        for (int ip = 0; ip < N; ++ip) if (FREE_NODE(ip)) sum += r[ip] * r[ip];
        fin = sqrt(sum);
        MAXABS(r);
        rel = fin / init;
        if (CONVERGED(rel, maxabs)) { conv = 1; break; }
        PRECOND();
        double rzn = 0.0;
        for (int ip = 0; ip < N; ++ip) if (FREE_NODE(ip)) rzn += r[ip] * z[ip];
        if (rzn <= 1.0e-300 || !isfinite(rzn)) { rc = fail(s, "ConjugateGradient::solvePressure - invalid updated preconditioned residual dot product."); goto out; }
        const double beta = rzn / rz;
        for (int ip = 0; ip < N; ++ip) pv[ip] = FREE_NODE(ip) ? z[ip] + beta * pv[ip] : 0.0;
        rz = rzn;
    }
done:
    s->cg[0] = iters; s->cg[1] = init; s->cg[2] = fin; s->cg[3] = rel; s->cg[4] = maxabs;
    s->cg_converged = conv;
    if (!conv) { rc = fail(s, "Steps::step2SemiImplicit - pressure solver failed to converge"); goto out; }
    apply_pressure(s);
out:
    free(act); free(fix); free(fval); free(r); free(z); free(pv); free(Ap);
    return rc;
#undef FREE_NODE
#undef IMPOSE
#undef MAXABS
#undef CONVERGED
#undef PRECOND
}

/* ---------------------------------------------------------------- Step 3 */

/* Steps::step3SemiImplicit, src/solver/Steps.cpp:377-428 */
int orc_step3(orc_state* s)
{
    memset(s->rhs, 0, sizeof(double) * 3 * (size_t)s->N);
    for (int e = 0; e < s->E; ++e) {
        if (s->mat[e] != 0) continue;
        double gp[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < 3; ++d) for (int a = 0; a < 4; ++a) gp[d] += GRAD(s, e, d, a) * s->pres[NODE(s, e, a)];
        const double vol4 = s->detJ[e] * FCON1;
        for (int a = 0; a < 4; ++a) {
            const int ip = NODE(s, e, a);
            for (int d = 0; d < 3; ++d) s->rhs[3 * (size_t)ip + d] -= vol4 * gp[d];
        }
    }
    for (int ip = 0; ip < s->N; ++ip)
        for (int d = 0; d < 3; ++d) s->unkno[3 * (size_t)ip + d] += s->rhs[3 * (size_t)ip + d] * s->elcoe2[ip];
    velocity_bc_package(s);
    return 0;
}

/* ---------------------------------------------------------------- Step 4 */

/* EnergyAssembly::assembleStep4Rhs, src/assembly/EnergyAssembly.cpp:566-611
 * (terms :118-532), then Steps::step4Energy, src/solver/Steps.cpp:448-467 */
int orc_step4(orc_state* s)
{
    if (s->p.temp_calc < 1) return 0;
    memset(s->rhs1, 0, sizeof(double) * (size_t)s->N);
    for (int e = 0; e < s->E; ++e) {
        if (s->detJ[e] <= 0.0 || !isfinite(s->detJ[e])) return fail(s, "EnergyAssembly::assembleStep4Rhs - invalid detJ at element %d", e + 1);
        if (s->rho_cp[e] <= 0.0 || !isfinite(s->rho_cp[e])) return fail(s, "EnergyAssembly::assembleStep4Rhs - invalid rho*Cp at element %d", e + 1);
        if (s->kc[e] <= 0.0 || !isfinite(s->kc[e])) return fail(s, "EnergyAssembly::assembleStep4Rhs - invalid thermal conductivity at element %d", e + 1);
        if (!isfinite(s->qvol[e])) return fail(s, "EnergyAssembly::assembleStep4Rhs - invalid volumetric source at element %d", e + 1);
        double tx = 0.0, ty = 0.0, tz = 0.0;
        for (int a = 0; a < 4; ++a) {
            const double T = s->temp1[NODE(s, e, a)];
            tx += GRAD(s, e, 0, a) * T; ty += GRAD(s, e, 1, a) * T; tz += GRAD(s, e, 2, a) * T;
        }
        double lr[4] = {0.0, 0.0, 0.0, 0.0};
        if (s->mat[e] == 0) {
            const double af = s->rho_cp[e] * s->detJ[e] / 120.0;
            double us = 0.0, vs = 0.0, ws = 0.0;
            for (int b = 0; b < 4; ++b) { const double* u = s->unkno + 3 * (size_t)NODE(s, e, b); us += u[0]; vs += u[1]; ws += u[2]; }
            for (int a = 0; a < 4; ++a) {
                const double* u = s->unkno + 3 * (size_t)NODE(s, e, a);
                const double advT = (us + u[0]) * tx + (vs + u[1]) * ty + (ws + u[2]) * tz;
                lr[a] -= af * advT;
            }
            const double dt = s->delte[e];
            if (dt <= 0.0 || !isfinite(dt)) return fail(s, "EnergyAssembly::assembleStep4Rhs - element timestep must be positive for thermal stabilisation at element %d", e + 1);
            double ub = 0.0, vb = 0.0, wb = 0.0;
            for (int a = 0; a < 4; ++a) { const double* u = s->unkno + 3 * (size_t)NODE(s, e, a); ub += u[0]; vb += u[1]; wb += u[2]; }
            ub /= 4.0; vb /= 4.0; wb /= 4.0;
            const double advT = ub * tx + vb * ty + wb * tz;
            const double vol = s->detJ[e] / 6.0;
            const double tau = 0.5 * dt * s->rho_cp[e] * vol;
            for (int a = 0; a < 4; ++a) {
                const double ug = ub * GRAD(s, e, 0, a) + vb * GRAD(s, e, 1, a) + wb * GRAD(s, e, 2, a);
                lr[a] += tau * ug * advT;
            }
        }
        const double vol = s->detJ[e] / 6.0;
        for (int a = 0; a < 4; ++a) {
            const double gdt = GRAD(s, e, 0, a) * tx + GRAD(s, e, 1, a) * ty + GRAD(s, e, 2, a) * tz;
            lr[a] -= s->kc[e] * vol * gdt;
        }
        if (s->qvol[e] != 0.0) {
            const double src = s->qvol[e] * s->detJ[e] * MASS_FACTOR;
            for (int a = 0; a < 4; ++a) lr[a] += src;
        }
        for (int a = 0; a < 4; ++a) s->rhs1[NODE(s, e, a)] += lr[a];
    }
    if (s->p.heat_flux_bc != 0.0)
        for (int ib = 0; ib < s->NB; ++ib) {
            const int* r = s->iside + 6 * (size_t)ib;
            if (r[5] != BC532) continue;
            const double area = s->face_norm[4 * (size_t)ib + 3];
            if (area <= 0.0 || !isfinite(area)) return fail(s, "EnergyAssembly::assembleStep4Rhs - invalid heat-flux boundary face area");
            const double contrib = s->p.heat_flux_bc * area / 3.0;
            for (int k = 0; k < 3; ++k) s->rhs1[r[k] - 1] += contrib;
        }
    for (int ip = 0; ip < s->N; ++ip) s->temp[ip] = s->temp1[ip] + s->rhs1[ip] * s->elcoe2p[ip];
    apply_temperature(s);
    return 0;
}

/* ----------------------------------------------------------- convergence */

static double safe_inverse_weight(double inv)
{
    if (fabs(inv) <= 1.0e-300 || !isfinite(inv)) return 1.0;
    return 1.0 / inv;
}

/* Convergence::evaluate, src/solver/Convergence.cpp:276-349 */
int orc_convergence(orc_state* s)
{
    velocity_magnitude(s);
    double* hb = s->hb;
    for (int i = 0; i < 15; ++i) hb[i] = 0.0;
    for (int ip = 0; ip < s->N; ++ip) {
        if (!s->tf[ip] && !s->ts[ip]) return fail(s, "Convergence - orphan node not touched by any material element");
        if (s->tf[ip] && !s->ts[ip])
            for (int d = 0; d < 3; ++d) {
                const double o = s->unkn1[3 * (size_t)ip + d], n = s->unkno[3 * (size_t)ip + d];
                const double dl = n - o;
                hb[3 * d] += dl * dl;
                hb[3 * d + 1] += n * n;
                const double rs = dl * safe_inverse_weight(s->elcoe2[ip]);
                hb[3 * d + 2] += rs * rs;
            }
        if (s->tf[ip]) {
            const double dl = s->pres[ip] - s->pres1[ip];
            hb[9] += dl * dl; hb[10] += s->pres[ip] * s->pres[ip]; hb[11] += dl * dl;
        }
        if (s->p.temp_calc > 0) {
            const double dl = s->temp[ip] - s->temp1[ip];
            hb[12] += dl * dl; hb[13] += s->temp[ip] * s->temp[ip];
            const double rs = dl * safe_inverse_weight(s->elcoe2p[ip]);
            hb[14] += rs * rs;
        }
    }
    for (int b = 0; b < 9; b += 3) {
        hb[b] = sqrt(hb[b] / (hb[b + 1] + 1.0e-30));
        hb[b + 1] = sqrt(hb[b + 1]);
        hb[b + 2] = sqrt(hb[b + 2]);
    }
    hb[9] = sqrt(hb[9] / (hb[10] + 1.0e-30)); hb[10] = sqrt(hb[10]); hb[11] = sqrt(hb[11]);
    if (s->p.temp_calc > 0) {
        hb[12] = sqrt(hb[12] / (hb[13] + 1.0e-30)); hb[13] = sqrt(hb[13]); hb[14] = sqrt(hb[14]);
    } else hb[12] = hb[13] = hb[14] = 0.0;
    return 0;
}

/* ------------------------------------------------------------ one step */

int orc_begin_step(orc_state* s)
{
    memcpy(s->unkn1, s->unkno, sizeof(double) * 3 * (size_t)s->N);
    memcpy(s->pres1, s->pres, sizeof(double) * (size_t)s->N);
    memcpy(s->temp1, s->temp, sizeof(double) * (size_t)s->N);
    return 0;
}

/* Solver::advanceOneStep, src/solver/Solver.cpp:609-680 */
int orc_step(orc_state* s, int iitime)
{
    orc_begin_step(s);
    if (orc_time_step(s, iitime)) return 1;
    if (orc_lhs(s)) return 1;
    if (orc_step1(s)) return 1;
    if (s->p.step2_check > 0) {
        if (orc_dt_correction(s)) return 1;
        if (orc_lhs(s)) return 1;
    }
    if (orc_step2_rhs(s)) return 1;
    if (orc_solve_pressure(s)) return 1;
    if (orc_step3(s)) return 1;
    if (orc_step4(s)) return 1;
    return orc_convergence(s);
}

/* ------------------------------------------------------------ accessors */

typedef struct { const char* name; char type; } entry;

static void* lookup(orc_state* s, const char* n, long* count, char* type)
{
    const long E = s->E, N = s->N, NB = s->NB;
#define D(nm, ptr, cnt) if (!strcmp(n, nm)) { *count = (cnt); *type = 'd'; return (void*)(ptr); }
#define I(nm, ptr, cnt) if (!strcmp(n, nm)) { *count = (cnt); *type = 'i'; return (void*)(ptr); }
    D("coord", s->coord, 3 * N) I("intma", s->intma, 4 * E) I("iside", s->iside, 6 * NB)
    I("mat_elem", s->mat, E) I("fedge", s->fedge, 4 * E)
    D("detJ", s->detJ, E) D("dNkdx", s->dNkdx, 12 * E) D("annxf", s->annxf, 16 * E)
    D("face_norm", s->face_norm, 4 * NB) D("alen_e", s->alen_e, E) D("elcoe_e", s->elcoe_e, 4 * E)
    D("Mdiag_real", s->mdiag_real, N) D("pdiagE", s->pdiagE, 4 * E) D("gstifE", s->gstifE, 6 * E)
    I("color_ptr", s->color_ptr, s->ncolor + 1) I("color_elem", s->color_elem, E)
    I("bc_list", s->bc_list, s->bc_fixed) D("bc_values", s->bc_values, s->bc_fixed)
    I("wall_node_list", s->wall_list, s->npoin_wall)
    D("bforce", s->bforce, 3 * N) D("mfluid", s->mfluid, N)
    D("unkno", s->unkno, 3 * N) D("unkn1", s->unkn1, 3 * N) D("pres", s->pres, N)
    D("pres1", s->pres1, N) D("temperature", s->temp, N) D("temperature1", s->temp1, N)
    D("velocity", s->velocity, N) D("rhs", s->rhs, 3 * N) D("rhs1", s->rhs1, N)
    D("delte", s->delte, E) D("alen", s->alen, N) D("elcoe2", s->elcoe2, N)
    D("elcoe2p", s->elcoe2p, N) D("pdiag", s->pdiag, N) D("gstif", s->gstif, 6 * E)
    D("hb", s->hb, 15) D("cg", s->cg, 5) D("dtreal", &s->dtreal, 1) D("ani", &s->ani, 1)
    D("inlet_u_from_massflow", &s->inlet_u_mf, 1)
#undef D
#undef I
    return NULL;
}

long orc_get(orc_state* s, const char* name, void* out, long cap, char* dtype)
{
    long n = 0;
    char t = 0;
    if (!strcmp(name, "ncolor")) { if (out && cap > 0) *(int*)out = s->ncolor; if (dtype) *dtype = 'i'; return 1; }
    void* p = lookup(s, name, &n, &t);
    if (!p) return -1;
    if (dtype) *dtype = t;
    if (out) {
        const long m = n < cap ? n : cap;
        memcpy(out, p, (size_t)m * (t == 'd' ? sizeof(double) : sizeof(int)));
    }
    return n;
}

int orc_set(orc_state* s, const char* name, const void* in, long count)
{
    long n = 0;
    char t = 0;
    void* p = lookup(s, name, &n, &t);
    if (!p || count != n) return 1;
    memcpy(p, in, (size_t)n * (t == 'd' ? sizeof(double) : sizeof(int)));
    if (p == (void*)s->bforce) s->has_bforce = 1;
    return 0;
}
