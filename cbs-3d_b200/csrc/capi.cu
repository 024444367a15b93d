// C ABI of the B200 CBS3D engine (include/cbs3d_gpu.h).
//
// A context owns the host model, one CUDA stream, the device state and the
// PCG engine.  One step enqueues the stage kernels in the order of
// Solver::advanceOneStep (reference src/solver/Solver.cpp:609-680) with no
// host synchronisation; the device status word is read back once per call.
#include "cbs3d_gpu.h"
#include "host_model.h"
#include "kernels.cuh"
#include "pcg.cuh"
#include "ctx.cuh"
#include "post.h"

#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <vector>

using namespace cbs3d;

std::string cbs3d::reason_text(const DevStatus& s)
{
    const std::string at = std::to_string(s.where);
    switch (s.reason) {
    case R_DETJ: return s.stage == ST_GEOM ? "Preprocess::shapeFunctionDerivatives - non-positive tetrahedron volume at element " + at + ". Tetrahedral connectivity must be consistently positively oriented."
                                           : "EnergyAssembly::assembleStep4Rhs - invalid detJ at element " + at;
    case R_FACE_AREA: return "Preprocess::getNormals - zero-area face at element " + at;
    case R_HMIN: return s.stage == ST_GEOM ? "Preprocess::elementSize - invalid characteristic length at element " + at
                                           : "TimeStep - invalid alen_e at element " + at + ". Run Preprocess::elementSize before timestep computation.";
    case R_MASS: return "Preprocess::massMatrix - non-positive lumped mass at node " + at;
    case R_CAPACITY: return "Preprocess::massMatrix - non-positive thermal capacitance at node " + at;
    case R_RHOCP: return "EnergyAssembly::assembleStep4Rhs - invalid rho*Cp at element " + at;
    case R_DT_LOCAL: return s.stage == ST_STEP1 ? "MomentumAssembly::assembleStep1Rhs - invalid element timestep at element " + at
                                                : "TimeStep - invalid local stability timestep at element " + at;
    case R_DT_MIN: return "TimeStep::computeTimeStep - invalid global minimum timestep";
    case R_DIFF: return "TimeStep - invalid timestep diffusivity at element " + at;
    case R_ALPHA: return "TimeStep - invalid thermal diffusivity alpha_e at element " + at;
    case R_RHOMU: return s.stage == ST_STEP1 ? "MomentumAssembly::assembleStep1Rhs - invalid fluid rho/mu at element " + at
                                             : "TimeStep - invalid fluid rho/mu at element " + at;
    case R_LHS_DT: return "TimeStep::updateLhsDiagonal - non-positive local timestep at element " + at;
    case R_LHS_ELCOE2: return "TimeStep::updateLhsDiagonal - non-positive fluid momentum mass/time diagonal at node " + at;
    case R_LHS_ELCOE2P: return "TimeStep::updateLhsDiagonal - non-positive capacitance/time diagonal at node " + at;
    case R_LHS_PDIAG: return "TimeStep::updateLhsDiagonal - zero pressure diagonal on fluid-connected node " + at;
    case R_ORPHAN: return "TimeStep::updateLhsDiagonal - orphan node detected at node " + at;
    case R_PCG_DIAG: return "ConjugateGradient::solvePressure - invalid Jacobi pressure diagonal at active node";
    case R_PCG_RZ0: return "ConjugateGradient::solvePressure - invalid initial preconditioned residual dot product.";
    case R_PCG_PAP: return "ConjugateGradient::solvePressure - breakdown: invalid pAp";
    case R_PCG_RZ: return "ConjugateGradient::solvePressure - invalid updated preconditioned residual dot product.";
    case R_PCG_RESID: return "ConjugateGradient::solvePressure - invalid pressure residual";
    case R_PCG_MAXIT: return "Steps::step2SemiImplicit - pressure solver failed to converge";
    case R_PCG_BARRIER: return "PCG grid barrier exceeded its spin limit (device wait timed out)";
    case R_STEP1_DETJ: return "MomentumAssembly::assembleStep1Rhs - invalid detJ at one or more elements";
    case R_K: return "EnergyAssembly::assembleStep4Rhs - invalid thermal conductivity at element " + at;
    case R_QVOL: return "EnergyAssembly::assembleStep4Rhs - invalid volumetric source at element " + at;
    case R_EN_DT: return "EnergyAssembly::assembleStep4Rhs - element timestep must be positive for thermal stabilisation at element " + at;
    default: return "device failure (stage " + std::to_string(s.stage) + ", reason " + std::to_string(s.reason) + ")";
    }
}

namespace {

}  // namespace


void cbs3d_ctx::setup(bool own_pcg)
{
    CUDA_OK(cudaSetDevice(opt.device));
    CUDA_OK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CUDA_OK(cudaEventCreate(&ev0));
    CUDA_OK(cudaEventCreate(&ev1));
    CUDA_OK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    CUDA_OK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    CUDA_OK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    CUDA_OK(cudaEventCreateWithFlags(&ev_lhs, cudaEventDisableTiming));
    own_engine = own_pcg;
    const size_t E = m.E, N = m.N;
    DevParams& P = S.P;
    P.E = m.E; P.N = m.N; P.NB = m.NB;
    P.temp_calc = m.temp_calc; P.htype = m.p.htype; P.ilots = m.p.ilots; P.transient_on = m.p.transient_on;
    P.solver_opt = m.p.solver_opt; P.dtfixed = m.p.dtfixed; P.dtfix_end = m.p.dtfix_end;
    P.dimensional_material = (m.p.dimensional_mode > 0 && m.p.material_properties_enabled > 0) ? 1 : 0;
    P.ani = m.ani; P.csafm = m.p.csafm; P.deltr = m.p.deltr; P.dtfix = m.p.dtfix;
    P.csafm2 = m.p.csafm2; P.epsilon1 = m.p.epsilon1;

    std::vector<int4> in4(E);
    std::vector<uint8_t> mat(E), fe(E, 0);
    for (size_t e = 0; e < E; ++e) {
        in4[e] = make_int4(m.intma[4 * e] - 1, m.intma[4 * e + 1] - 1, m.intma[4 * e + 2] - 1, m.intma[4 * e + 3] - 1);
        mat[e] = m.mat[e] != 0 ? 1 : 0;
        for (int f = 0; f < 4; ++f) fe[e] |= static_cast<uint8_t>((m.fedge[4 * e + f] & 3) << (2 * f));
    }
    std::vector<uint8_t> nflag(N, 0);
    std::vector<double> pfix(N, 0.0);
    for (size_t i = 0; i < N; ++i) nflag[i] = static_cast<uint8_t>((m.tf[i] ? 1 : 0) | (m.ts[i] ? 2 : 0));
    for (size_t k = 0; k < m.bc_list.size(); ++k) {
        const size_t i = static_cast<size_t>(m.bc_list[k] - 1);
        if (!m.tf[i])
            throw Error(CBS3D_INVALID_INPUT, "TimeStep::updateLhsDiagonal - fixed pressure node is not connected to the fluid pressure domain, node " + std::to_string(i + 1));
        nflag[i] |= 4;
        pfix[i] = m.bc_values[k];
    }
    S.intma = buf.upload(in4);
    S.mat = buf.upload(mat);
    S.fedge = buf.upload(fe);
    S.coord = buf.upload(m.coord);
    S.rho = buf.upload(m.rho);
    S.mu = buf.upload(m.mu);
    S.kc = buf.upload(m.kc);
    S.rho_cp = buf.upload(m.rho_cp);
    S.alpha = buf.upload(m.alpha);
    S.qvol = buf.upload(m.qvol);
    S.detJ = buf.alloc<double>(E);
    S.grad = buf.alloc<double>(12 * E);
    S.annxf = buf.alloc<double>(16 * E);
    S.alen_e = buf.alloc<double>(E);
    S.pdiagE = buf.alloc<double>(4 * E);
    S.gstifE = buf.alloc<double>(6 * E);
    S.alen = buf.alloc<double>(N);
    S.n2e_ptr = buf.upload(m.n2e_ptr);
    S.n2e = buf.upload(m.n2e);
    S.n2c_ptr = buf.upload(m.n2c_ptr);
    S.n2c = buf.upload(m.n2c);
    S.nflag = buf.upload(nflag);
    S.pfix = buf.upload(pfix);
    S.vbc_idx = buf.upload(m.vbc_idx);
    {
        VelBC* p = buf.alloc<VelBC>(m.vbc.size());
        if (!m.vbc.empty()) CUDA_OK(cudaMemcpy(p, m.vbc.data(), m.vbc.size() * sizeof(VelBC), cudaMemcpyHostToDevice));
        S.vbc = p;
    }
    S.vbc_nrm = buf.upload(m.vbc_nrm);
    S.tbc_flag = buf.upload(m.tbc_flag);
    S.tbc_val = buf.upload(m.tbc_val);
    S.hf_ptr = buf.upload(m.hf_ptr);
    S.hf_val = buf.upload(m.hf_val);
    S.unkno = buf.upload(m.unkno);
    S.unkn1 = buf.upload(m.unkno);
    S.pres = buf.upload(m.pres);
    S.pres1 = buf.upload(m.pres);
    S.temp = buf.upload(m.temp);
    S.temp1 = buf.upload(m.temp);
    S.velocity = buf.alloc<double>(N);
    S.rhs = buf.alloc<double>(3 * N);
    S.rhs1 = buf.alloc<double>(N);
    S.delte = buf.alloc<double>(E);
    S.elcoe2 = buf.alloc<double>(N);
    S.elcoe2p = buf.alloc<double>(N);
    S.pdiag = buf.alloc<double>(N);
    S.mdiag_real = buf.alloc<double>(N);
    S.elbuf = buf.alloc<double>(16 * E);   // Step 1: 4 records of 4 doubles per tet; others use 12*E
    S.dscal = buf.alloc<double>(32);
    S.dtmin_bits = buf.alloc<unsigned long long>(1);
    S.conv_count = buf.alloc<unsigned>(1);
    S.status = buf.alloc<DevStatus>(1);
    conv_blocks = static_cast<int>(nb(static_cast<long long>(N)));
    S.red = buf.alloc<double>(static_cast<size_t>(conv_blocks) * 16);
    d_color_elem = buf.upload(m.color_elem);
    d_counter = buf.alloc<int>(1);
    CUDA_OK(cudaMemset(S.rhs, 0, 3 * N * sizeof(double)));
    CUDA_OK(cudaMemset(S.rhs1, 0, N * sizeof(double)));
    CUDA_OK(cudaMemset(S.pdiag, 0, N * sizeof(double)));
    CUDA_OK(cudaMemset(S.delte, 0, E * sizeof(double)));
    CUDA_OK(cudaMemset(S.dscal, 0, 32 * sizeof(double)));
    CUDA_OK(cudaMemset(S.status, 0, sizeof(DevStatus)));
    CUDA_OK(cudaMemset(d_counter, 0, sizeof(int)));
    CUDA_OK(cudaMemset(S.conv_count, 0, sizeof(unsigned)));

    // Preprocess on the device (Solver::initialise geometry and mass).
    k_geometry<<<nb(m.E), T, 0, st>>>(S);
    k_mass<<<nb(m.N), T, 0, st>>>(S);
    if (m.p.htype == 2 || m.p.step2_check > 0) k_nodal_length<<<nb(m.N), T, 0, st>>>(S);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaStreamSynchronize(st));
    check_status();
    if (!own_pcg) return;
    pcg.inner_tol = opt.inner_tol > 0.0 ? opt.inner_tol : 0.05;
    pcg.init(m, S.nflag, S.pfix, S.status, opt.device, opt.pcg_blocks, opt.precision == CBS3D_MIXED, opt.pcg_kernel,
             opt.pcg_two_level > 0, opt.pcg_multigrid > 0);
}

void cbs3d_ctx::check_status()
{
    DevStatus s{};
    CUDA_OK(cudaMemcpyAsync(&s, S.status, sizeof s, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    if (s.code != 0) {
        throw Error(static_cast<cbs3d_status>(s.code), reason_text(s));
    }
}

void cbs3d_ctx::stage_time_step(int it)
{
    const int fx = fixed_dt(it) ? 1 : 0;
    k_timestep<<<nb(m.E), T, 0, st>>>(S, fx);
    k_dt_finish<<<1, 32, 0, st>>>(S, fx);
    if (!fx && force_global()) k_dt_force<<<nb(m.E), T, 0, st>>>(S);
}

// The pressure operator depends on delte and the LHS only, so once the last
// LHS update of a step is issued it is assembled (with the two-level set-up)
// on the side stream while Steps 1 and 2 run; stage_solve joins it.
void cbs3d_ctx::fork_assembly()
{
    if (!own_engine) return;
    CUDA_OK(cudaEventRecord(ev_fork, st));
    CUDA_OK(cudaStreamWaitEvent(side, ev_fork, 0));
    pcg.assemble_from_state(S, side);
    pcg.prepare_coarse(S.pdiag, side);
    CUDA_OK(cudaEventRecord(ev_join, side));
    assembly_forked = true;
}

void cbs3d_ctx::stage_solve()
{
    if (assembly_forked) {
        CUDA_OK(cudaStreamWaitEvent(st, ev_join, 0));
        assembly_forked = false;
    } else {
        pcg.assemble_from_state(S, st);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (opt.time_pcg) {
        while (static_cast<int>(pcg_ev.size()) < pcg_ev_used + 2) {
            cudaEvent_t e;
            CUDA_OK(cudaEventCreate(&e));
            pcg_ev.push_back(e);
        }
        e0 = pcg_ev[static_cast<size_t>(pcg_ev_used)];
        e1 = pcg_ev[static_cast<size_t>(pcg_ev_used) + 1];
        pcg_ev_used += 2;
    }
    pcg.solve(S.pres, S.rhs1, S.pdiag, m.p.cg_preconditioner, m.p.cg_conv_test, m.p.cg_max_iter,
              m.p.relToler, m.p.absToler, st, false, e0, e1);
}

void cbs3d_ctx::enqueue_pre(int it)
{
    k_begin_step<<<nb(m.N), T, 0, st>>>(S);
    stage_time_step(it);
    // The Step-1 element kernel reads none of the LHS's outputs (elcoe2,
    // elcoe2p, pdiag, the constrained rows' p and rhs1), so the LHS runs on
    // the side stream beside it, followed there by the operator assembly;
    // the Step-1 node gather, which reads elcoe2, waits for the LHS.
    const bool lhs_side = m.p.step2_check <= 0 && own_engine;
    if (lhs_side) {
        CUDA_OK(cudaEventRecord(ev_fork, st));
        CUDA_OK(cudaStreamWaitEvent(side, ev_fork, 0));
        k_lhs<<<nb(m.N), T, 0, side>>>(S);
        CUDA_OK(cudaEventRecord(ev_lhs, side));
        pcg.assemble_from_state(S, side);
        pcg.prepare_coarse(S.pdiag, side);
        CUDA_OK(cudaEventRecord(ev_join, side));
        assembly_forked = true;
    } else {
        k_lhs<<<nb(m.N), T, 0, st>>>(S);
        if (m.p.step2_check <= 0) fork_assembly();
    }
    k_step1_elem<<<nb(m.E, 128), 128, 0, st>>>(S);
    if (lhs_side) CUDA_OK(cudaStreamWaitEvent(st, ev_lhs, 0));
    k_step1_node<<<nb(m.N), T, 0, st>>>(S);
    if (m.p.step2_check > 0) {
        k_dt_correction<<<nb(m.E), T, 0, st>>>(S);
        k_lhs<<<nb(m.N), T, 0, st>>>(S);
        fork_assembly();
    }
    k_step2_elem<<<nb(m.E), T, 0, st>>>(S);
    k_step2_node<<<nb(m.N), T, 0, st>>>(S);
}

void cbs3d_ctx::enqueue_post(int it)
{
    (void)it;
    k_step3_elem<<<nb(m.E), T, 0, st>>>(S);
    k_step3_node<<<nb(m.N), T, 0, st>>>(S);
    if (m.temp_calc > 0) {
        k_step4_elem<<<nb(m.E), T, 0, st>>>(S);
        k_step4_node<<<nb(m.N), T, 0, st>>>(S);
    }
    k_conv_partial<<<static_cast<unsigned>(conv_blocks), T, 0, st>>>(S, batch_out ? batch_out : pcg.d_out, d_log,
                                                                    d_counter, log_cap);
}

int cbs3d_ctx::kernels_outside_solve(int it) const
{
    // begin, timestep, dt_finish, lhs, step1 x2, step2 x2, step3 x2,
    // convergence (with the step log): 11
    return 11 + (!fixed_dt(it) && force_global() ? 1 : 0) + (m.p.step2_check > 0 ? 2 : 0) +
           (m.temp_calc > 0 ? 2 : 0);
}

void cbs3d_ctx::enqueue_step(int it)
{
    enqueue_pre(it);
    stage_solve();
    enqueue_post(it);
    // plus the operator assembly and the pressure solve's launches
    step_kernels = kernels_outside_solve(it) + 1 + pcg.launches_per_solve();
}

void cbs3d_ctx::ensure_log(int n)
{
    if (n <= log_cap && d_log) return;
    if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
    if (d_log) cudaFree(d_log);
    d_log = nullptr;
    CUDA_OK(cudaMalloc(&d_log, static_cast<size_t>(n) * LOG_FIELDS * sizeof(double)));
    log_cap = n;
}

// ---------------------------------------------------------------- helpers
namespace {

template <typename C, typename F>
cbs3d_status guarded(C* c, F&& f)
{
    if (!c) return CBS3D_INVALID_INPUT;
    try {
        f();
        c->err.clear();
        return CBS3D_OK;
    } catch (const Error& e) {
        c->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        c->err = "host allocation failed";
        return CBS3D_INTERNAL;
    } catch (const std::exception& e) {
        c->err = e.what();
        return CBS3D_INTERNAL;
    }
}

void fill_err(char* err, size_t len, const std::string& m)
{
    if (err && len) std::snprintf(err, len, "%s", m.c_str());
}

}  // namespace

// ============================================================ public API
extern "C" {

int cbs3d_version(void) { return 10000; }

const char* cbs3d_status_string(cbs3d_status s)
{
    switch (s) {
    case CBS3D_OK: return "OK";
    case CBS3D_INVALID_INPUT: return "INVALID_INPUT";
    case CBS3D_NOT_CONVERGED: return "NOT_CONVERGED";
    case CBS3D_BREAKDOWN: return "BREAKDOWN";
    case CBS3D_NONFINITE: return "NONFINITE";
    case CBS3D_TIMEOUT: return "TIMEOUT";
    case CBS3D_CUDA_ERROR: return "CUDA_ERROR";
    case CBS3D_IO_ERROR: return "IO_ERROR";
    default: return "INTERNAL";
    }
}

void cbs3d_default_options(cbs3d_options* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->precision = CBS3D_FP64;
    o->inner_tol = 0.05;
    o->use_graph = 1;
}

void cbs3d_default_params(cbs3d_params* p)
{
    if (p) default_params(*p);
}

cbs3d_status cbs3d_read_params(const char* case_name, cbs3d_params* params, int* nelem, int* npoin,
                               int* nboun, char* err, size_t errlen)
{
    try {
        int e = 0, n = 0, b = 0;
        read_params_only(case_name, *params, e, n, b);
        if (nelem) *nelem = e;
        if (npoin) *npoin = n;
        if (nboun) *nboun = b;
        return CBS3D_OK;
    } catch (const Error& e) {
        fill_err(err, errlen, e.what());
        return e.code;
    } catch (const std::exception& e) {
        fill_err(err, errlen, e.what());
        return CBS3D_INTERNAL;
    }
}

static void fnv_bytes(unsigned long long* h, const void* data, size_t n)
{
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) { *h ^= p[i]; *h *= 1099511628211ULL; }
}
#define FNV(h, v) fnv_bytes(&(h), (v).data(), (v).size() * sizeof((v)[0]))

cbs3d_status cbs3d_case_digest(const char* case_name, int use_cache, unsigned long long* digest,
                               int* from_cache, char* err, size_t errlen)
{
    if (!case_name || !digest) return CBS3D_INVALID_INPUT;
    try {
        HostModel m;
        bool hit = false;
        if (use_cache) hit = parse_case_cached(case_name, m);
        else parse_case(case_name, m);
        unsigned long long h = 1469598103934665603ULL;
        const std::vector<int> sizes = {m.E, m.N, m.NB};
        FNV(h, sizes); FNV(h, m.intma); FNV(h, m.coord); FNV(h, m.iside); FNV(h, m.mat);
        FNV(h, m.rho); FNV(h, m.cp); FNV(h, m.kc); FNV(h, m.mu); FNV(h, m.qvol);
        fnv_bytes(&h, &m.p, sizeof m.p);
        *digest = h;
        if (from_cache) *from_cache = hit ? 1 : 0;
        return CBS3D_OK;
    } catch (const Error& e) {
        fill_err(err, errlen, e.what());
        return e.code;
    } catch (const std::exception& e) {
        fill_err(err, errlen, e.what());
        return CBS3D_INTERNAL;
    }
}

#undef FNV

static cbs3d_status create_common(std::unique_ptr<cbs3d_ctx>& c, const cbs3d_options* opt, cbs3d_ctx** out,
                                  char* err, size_t errlen)
{
    try {
        if (opt) c->opt = *opt; else cbs3d_default_options(&c->opt);
        c->setup();
        *out = c.release();
        return CBS3D_OK;
    } catch (const Error& e) {
        fill_err(err, errlen, e.what());
        return e.code;
    } catch (const std::exception& e) {
        fill_err(err, errlen, e.what());
        return CBS3D_INTERNAL;
    }
}

cbs3d_status cbs3d_create_from_case(const char* case_name, const cbs3d_options* opt, cbs3d_ctx** out,
                                    char* err, size_t errlen)
{
    if (!case_name || !out) return CBS3D_INVALID_INPUT;
    *out = nullptr;
    auto c = std::make_unique<cbs3d_ctx>();
    try {
        read_case(case_name, c->m, opt && opt->case_cache > 0);
    } catch (const Error& e) {
        fill_err(err, errlen, e.what());
        return e.code;
    } catch (const std::exception& e) {
        fill_err(err, errlen, e.what());
        return CBS3D_INTERNAL;
    }
    return create_common(c, opt, out, err, errlen);
}

cbs3d_status cbs3d_create(const cbs3d_mesh* mesh, const cbs3d_params* params, const cbs3d_options* opt,
                          cbs3d_ctx** out, char* err, size_t errlen)
{
    if (!mesh || !params || !out) return CBS3D_INVALID_INPUT;
    *out = nullptr;
    auto c = std::make_unique<cbs3d_ctx>();
    try {
        model_from_arrays(*mesh, *params, c->m);
    } catch (const Error& e) {
        fill_err(err, errlen, e.what());
        return e.code;
    } catch (const std::exception& e) {
        fill_err(err, errlen, e.what());
        return CBS3D_INTERNAL;
    }
    return create_common(c, opt, out, err, errlen);
}

void cbs3d_destroy(cbs3d_ctx* ctx) { delete ctx; }

const char* cbs3d_last_error(const cbs3d_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// After a call's steps have finished on the device: the status word, the
// per-step log (PCG iterations into the running total), and the stats.
static DevStatus collect_call(cbs3d_ctx* c, int done, int start, long long launches0, bool steady, float ms,
                              cbs3d_step_stats* stats)
{
    DevStatus s{};
    CUDA_OK(cudaMemcpy(&s, c->S.status, sizeof s, cudaMemcpyDeviceToHost));
    std::vector<double> log(static_cast<size_t>(done) * LOG_FIELDS);
    if (done) CUDA_OK(cudaMemcpy(log.data(), c->d_log, log.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int k = 0; k < done; ++k) c->cg_total += static_cast<long long>(log[static_cast<size_t>(k) * LOG_FIELDS + 1]);
    if (!stats) return s;
    stats->steps_done = done;
    stats->iitime = c->iitime;
    stats->gpu_seconds = ms * 1.0e-3;
    stats->steady_reached = steady ? 1 : 0;
    stats->cg_iterations_total = c->cg_total;
    stats->kernel_launches = c->launches - launches0;
    if (!c->batch_out) {
        stats->pcg_bytes_per_iter = static_cast<double>(c->pcg.bytes_per_iter());
        stats->pcg_kernel = c->pcg.mgh ? 7 : c->pcg.coarse ? 6 : c->pcg.variant == 4 && c->pcg.mixed_ok ? 5
                          : c->pcg.variant == 1 && c->pcg.global_halo && c->pcg.global_cgcg ? 8
                          : c->pcg.variant == 4 && c->pcg.cgcg_kt > 0 ? 9 : c->pcg.variant;
    }
    for (int k = 0; k + 1 < c->pcg_ev_used; k += 2) {
        float pm = 0.0f;
        CUDA_OK(cudaEventElapsedTime(&pm, c->pcg_ev[static_cast<size_t>(k)], c->pcg_ev[static_cast<size_t>(k) + 1]));
        stats->pcg_seconds += pm * 1.0e-3;
        ++stats->pcg_launches;
    }
    if (done) {
        const double* r = &log[static_cast<size_t>(done - 1) * LOG_FIELDS];
        stats->dtreal = r[0];
        stats->cg.iterations = static_cast<int>(r[1]);
        stats->cg.initial_l2 = r[2];
        stats->cg.final_l2 = r[3];
        stats->cg.final_relative_l2 = r[4];
        stats->cg.final_max_abs = r[5];
        stats->cg.converged = static_cast<int>(r[6]);
        stats->cg.outer_sweeps = static_cast<int>(r[23]);
        for (int q = 0; q < 15; ++q) stats->hb[q] = r[7 + q];
        stats->rtime = r[22];
    }
    if (s.code != 0) stats->failed_step = start + (s.step > 0 ? s.step : done);
    return s;
}

cbs3d_status cbs3d_step(cbs3d_ctx* c, int nsteps, int stop_on_steady, cbs3d_step_stats* stats)
{
    return guarded(c, [&] {
        if (nsteps < 0) throw Error(CBS3D_INVALID_INPUT, "cbs3d_step - nsteps must be >= 0");
        if (stats) std::memset(stats, 0, sizeof *stats);
        CUDA_OK(cudaSetDevice(c->opt.device));
        c->ensure_log(nsteps > 0 ? nsteps : 1);
        c->reset_status();
        CUDA_OK(cudaMemsetAsync(c->d_counter, 0, sizeof(int), c->st));
        const int start = c->iitime;
        const long long launches0 = c->launches;
        c->pcg_ev_used = 0;
        CUDA_OK(cudaEventRecord(c->ev0, c->st));
        int done = 0;
        bool steady = false;
        for (int s = 0; s < nsteps; ++s) {
            const int it = c->iitime + 1;
            const bool graphable = c->opt.use_graph && !c->opt.time_pcg && !c->graph_failed &&
                                   !(c->m.p.dtfix_end > 0 && it <= c->m.p.dtfix_end);
            if (graphable && !c->gexec) {
                cudaGraph_t g = nullptr;
                bool ok = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    c->enqueue_step(it);
                    ok = cudaStreamEndCapture(c->st, &g) == cudaSuccess && g;
                }
                if (ok) ok = cudaGraphInstantiate(&c->gexec, g, 0) == cudaSuccess;
                if (g) cudaGraphDestroy(g);
                if (!ok) {
                    cudaGetLastError();
                    c->graph_failed = true;
                    c->gexec = nullptr;
                }
            }
            if (graphable && c->gexec) CUDA_OK(cudaGraphLaunch(c->gexec, c->st));
            else c->enqueue_step(it);
            c->launches += c->step_kernels;
            CUDA_OK(cudaGetLastError());
            c->iitime = it;
            ++done;
            const bool check_steady = stop_on_steady &&
                ((c->m.p.transient_on < 1 && it >= c->m.p.steady_min_iterations) ||
                 (c->m.p.transient_on > 0 && c->m.p.end_rtime > 0.0));
            if (check_steady) {
                double rec[LOG_FIELDS];
                CUDA_OK(cudaMemcpyAsync(rec, c->d_log + static_cast<size_t>(s) * LOG_FIELDS, sizeof rec,
                                        cudaMemcpyDeviceToHost, c->st));
                CUDA_OK(cudaStreamSynchronize(c->st));
                const double* hb = rec + 7;
                const cbs3d_params& P = c->m.p;
                bool stop;
                if (P.transient_on > 0) {
                    stop = rec[22] >= P.end_rtime;   // Solver::transientEndTimeReached
                } else {
                    // Convergence::steadyStateReached, src/solver/Convergence.cpp:399-418
                    const double vr = std::max(hb[0], std::max(hb[3], hb[6]));
                    const bool vel_ok = P.vel_check < 1 || vr < P.l2norm_vel_tolerance;
                    const bool t_ok = P.temp_check < 1 || c->m.temp_calc < 1 || hb[12] < P.l2norm_temp_tolerance;
                    const bool p_ok = P.l2norm_pres_tolerance <= 0.0 || hb[9] < P.l2norm_pres_tolerance;
                    stop = vel_ok && t_ok && p_ok;
                }
                if (stop) { steady = true; break; }
            }
        }
        CUDA_OK(cudaEventRecord(c->ev1, c->st));
        CUDA_OK(cudaStreamSynchronize(c->st));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        c->last_start = start;
        c->last_done = done;
        const DevStatus s = collect_call(c, done, start, launches0, steady, ms, stats);
        if (s.code != 0) {
            const int fstep = start + (s.step > 0 ? s.step : done);
            throw Error(static_cast<cbs3d_status>(s.code), reason_text(s) + " (step " + std::to_string(fstep) + ")");
        }
    });
}

cbs3d_status cbs3d_upload_fields(cbs3d_ctx* c, const double* u, const double* p, const double* t)
{
    return guarded(c, [&] {
        const size_t N = c->m.N;
        if (u) CUDA_OK(cudaMemcpy(c->S.unkno, u, 3 * N * sizeof(double), cudaMemcpyHostToDevice));
        if (p) CUDA_OK(cudaMemcpy(c->S.pres, p, N * sizeof(double), cudaMemcpyHostToDevice));
        if (t) CUDA_OK(cudaMemcpy(c->S.temp, t, N * sizeof(double), cudaMemcpyHostToDevice));
    });
}

cbs3d_status cbs3d_download_fields(cbs3d_ctx* c, double* u, double* p, double* t)
{
    return guarded(c, [&] {
        const size_t N = c->m.N;
        CUDA_OK(cudaStreamSynchronize(c->st));
        if (u) CUDA_OK(cudaMemcpy(u, c->S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToHost));
        if (p) CUDA_OK(cudaMemcpy(p, c->S.pres, N * sizeof(double), cudaMemcpyDeviceToHost));
        if (t) CUDA_OK(cudaMemcpy(t, c->S.temp, N * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

namespace {

struct ArrayRef {
    void* dev = nullptr;          // device array (direct copy)
    long count = 0;
    int esize = 8;
    int soa_rows = 0;             // >0: device SoA [rows][E] -> reference element-major
    const void* host = nullptr;   // host-side array
};

ArrayRef find_array(cbs3d_ctx* c, const std::string& n)
{
    const long E = c->m.E, N = c->m.N, NB = c->m.NB;
    DevState& S = c->S;
    ArrayRef r;
    auto dv = [&](double* p, long cnt) { r.dev = p; r.count = cnt; r.esize = 8; };
    if (n == "unkno") dv(S.unkno, 3 * N);
    else if (n == "unkn1") dv(S.unkn1, 3 * N);
    else if (n == "pres") dv(S.pres, N);
    else if (n == "pres1") dv(S.pres1, N);
    else if (n == "temperature") dv(S.temp, N);
    else if (n == "temperature1") dv(S.temp1, N);
    else if (n == "velocity") dv(S.velocity, N);
    else if (n == "rhs") dv(S.rhs, 3 * N);
    else if (n == "rhs1") dv(S.rhs1, N);
    else if (n == "delte") dv(S.delte, E);
    else if (n == "elcoe2") dv(S.elcoe2, N);
    else if (n == "elcoe2p") dv(S.elcoe2p, N);
    else if (n == "pdiag") dv(S.pdiag, N);
    else if (n == "Mdiag_real") dv(S.mdiag_real, N);
    else if (n == "alen") dv(S.alen, N);
    else if (n == "detJ") dv(S.detJ, E);
    else if (n == "alen_e") dv(S.alen_e, E);
    else if (n == "dNkdx") { dv(S.grad, 12 * E); r.soa_rows = 12; }
    else if (n == "annxf") { dv(S.annxf, 16 * E); r.soa_rows = 16; }
    else if (n == "pdiagE") { dv(S.pdiagE, 4 * E); r.soa_rows = 4; }
    else if (n == "gstifE") { dv(S.gstifE, 6 * E); r.soa_rows = 6; }
    else if (n == "fedge") { r.host = c->m.fedge.data(); r.count = 4 * E; r.esize = 4; }
    else if (n == "iside") { r.host = c->m.iside.data(); r.count = 6 * NB; r.esize = 4; }
    else if (n == "color_ptr") { r.host = c->m.color_ptr.data(); r.count = static_cast<long>(c->m.color_ptr.size()); r.esize = 4; }
    else if (n == "color_elem") { r.host = c->m.color_elem.data(); r.count = E; r.esize = 4; }
    else if (n == "bc_list") { r.host = c->m.bc_list.data(); r.count = static_cast<long>(c->m.bc_list.size()); r.esize = 4; }
    else if (n == "bc_values") { r.host = c->m.bc_values.data(); r.count = static_cast<long>(c->m.bc_values.size()); r.esize = 8; }
    else if (n == "wall_node_list") { r.host = c->m.wall_list.data(); r.count = static_cast<long>(c->m.wall_list.size()); r.esize = 4; }
    else if (n == "face_norm") { r.host = c->m.face_norm.data(); r.count = 4 * NB; r.esize = 8; }
    else throw Error(CBS3D_INVALID_INPUT, "unknown array name: " + n);
    return r;
}

}  // namespace

cbs3d_status cbs3d_get_array(cbs3d_ctx* c, const char* name, void* host, long count, long* written)
{
    return guarded(c, [&] {
        const std::string n(name ? name : "");
        CUDA_OK(cudaStreamSynchronize(c->st));
        if (n == "ncolor" || n == "dtreal" || n == "hb" || n == "cg" || n == "gstif") {
            std::vector<double> v;
            if (n == "ncolor") {
                if (written) *written = 1;
                if (host && count >= 1) *static_cast<int*>(host) = c->m.ncolor;
                return;
            }
            if (n == "dtreal" || n == "hb") {
                double d[17];
                CUDA_OK(cudaMemcpy(d, c->S.dscal, sizeof d, cudaMemcpyDeviceToHost));
                if (n == "dtreal") v.assign(d, d + 1); else v.assign(d + 2, d + 17);
            } else if (n == "cg") {
                CgOut o{};
                CUDA_OK(cudaMemcpy(&o, c->pcg.d_out, sizeof o, cudaMemcpyDeviceToHost));
                v = {static_cast<double>(o.iterations), o.initial_l2, o.final_l2, o.rel, o.max_abs};
            } else {
                k_gstif<<<nb(c->m.E), T, 0, c->st>>>(c->S, c->S.elbuf);
                CUDA_OK(cudaGetLastError());
                v.resize(6 * static_cast<size_t>(c->m.E));
                CUDA_OK(cudaStreamSynchronize(c->st));
                CUDA_OK(cudaMemcpy(v.data(), c->S.elbuf, v.size() * sizeof(double), cudaMemcpyDeviceToHost));
            }
            if (written) *written = static_cast<long>(v.size());
            if (host) std::memcpy(host, v.data(), std::min<size_t>(v.size(), static_cast<size_t>(count)) * sizeof(double));
            return;
        }
        const ArrayRef r = find_array(c, n);
        if (written) *written = r.count;
        if (!host) return;
        const long m = std::min(count, r.count);
        if (r.host) { std::memcpy(host, r.host, static_cast<size_t>(m) * r.esize); return; }
        if (!r.soa_rows) {
            CUDA_OK(cudaMemcpy(host, r.dev, static_cast<size_t>(m) * r.esize, cudaMemcpyDeviceToHost));
            return;
        }
        std::vector<double> tmp(static_cast<size_t>(r.count));
        CUDA_OK(cudaMemcpy(tmp.data(), r.dev, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost));
        const long E = c->m.E, R = r.soa_rows;
        double* out = static_cast<double*>(host);
        for (long e = 0; e < E; ++e)
            for (long q = 0; q < R; ++q)
                if (e * R + q < m) out[e * R + q] = tmp[static_cast<size_t>(q * E + e)];
    });
}

cbs3d_status cbs3d_set_array(cbs3d_ctx* c, const char* name, const void* host, long count)
{
    return guarded(c, [&] {
        const std::string n(name ? name : "");
        static const char* settable[] = {"unkno", "unkn1", "pres", "pres1", "temperature", "temperature1",
                                         "rhs", "rhs1", "delte", "elcoe2", "elcoe2p", "pdiag"};
        bool ok = false;
        for (const char* s : settable) ok = ok || n == s;
        if (!ok) throw Error(CBS3D_INVALID_INPUT, "array is not settable: " + n);
        const ArrayRef r = find_array(c, n);
        if (count != r.count) throw Error(CBS3D_INVALID_INPUT, "size mismatch for array " + n);
        CUDA_OK(cudaStreamSynchronize(c->st));
        CUDA_OK(cudaMemcpy(r.dev, host, static_cast<size_t>(count) * r.esize, cudaMemcpyHostToDevice));
    });
}

cbs3d_status cbs3d_run_stage(cbs3d_ctx* c, const char* stage)
{
    return guarded(c, [&] {
        const std::string s(stage ? stage : "");
        c->reset_status();
        DevState& S = c->S;
        cudaStream_t st = c->st;
        const HostModel& m = c->m;
        if (s == "begin_step") { k_begin_step<<<nb(m.N), T, 0, st>>>(S); ++c->iitime; }
        else if (s == "time_step") c->stage_time_step(c->iitime);
        else if (s == "lhs") k_lhs<<<nb(m.N), T, 0, st>>>(S);
        else if (s == "step1") { k_step1_elem<<<nb(m.E, 128), 128, 0, st>>>(S); k_step1_node<<<nb(m.N), T, 0, st>>>(S); }
        else if (s == "dt_correction") k_dt_correction<<<nb(m.E), T, 0, st>>>(S);
        else if (s == "step2_rhs") { k_step2_elem<<<nb(m.E), T, 0, st>>>(S); k_step2_node<<<nb(m.N), T, 0, st>>>(S); }
        else if (s == "solve_pressure") c->stage_solve();
        else if (s == "step3") { k_step3_elem<<<nb(m.E), T, 0, st>>>(S); k_step3_node<<<nb(m.N), T, 0, st>>>(S); }
        else if (s == "step4") { if (m.temp_calc > 0) { k_step4_elem<<<nb(m.E), T, 0, st>>>(S); k_step4_node<<<nb(m.N), T, 0, st>>>(S); } }
        else if (s == "convergence") {
            k_conv_partial<<<static_cast<unsigned>(c->conv_blocks), T, 0, st>>>(S, nullptr, nullptr, nullptr, 0);
        } else throw Error(CBS3D_INVALID_INPUT, "unknown stage: " + s);
        CUDA_OK(cudaGetLastError());
        CUDA_OK(cudaStreamSynchronize(st));
        c->check_status();
    });
}

cbs3d_status cbs3d_solve_pressure(cbs3d_ctx* c, const double* gstif, double* pdiag, double* rhs1, double* pres,
                                  cbs3d_cg_result* result)
{
    return guarded(c, [&] {
        if (!gstif || !pdiag || !rhs1 || !pres) throw Error(CBS3D_INVALID_INPUT, "cbs3d_solve_pressure - null array");
        if (c->batch_out) throw Error(CBS3D_INVALID_INPUT, "cbs3d_solve_pressure - context belongs to a batch");
        const size_t E = c->m.E, N = c->m.N;
        const cudaStream_t st = c->st;
        double* dg = nullptr;
        CUDA_OK(cudaMalloc(&dg, 6 * E * sizeof(double)));
        struct Free { double* p; ~Free() { cudaFree(p); } } guard{dg};
        CUDA_OK(cudaMemcpyAsync(dg, gstif, 6 * E * sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(c->S.pdiag, pdiag, N * sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(c->S.rhs1, rhs1, N * sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(c->S.pres, pres, N * sizeof(double), cudaMemcpyHostToDevice, st));
        c->reset_status();
        c->pcg.assemble_from_gstif(dg, st);
        const cbs3d_params& P = c->m.p;
        c->pcg.solve(c->S.pres, c->S.rhs1, c->S.pdiag, P.cg_preconditioner, P.cg_conv_test, P.cg_max_iter,
                     P.relToler, P.absToler, st, false);
        CUDA_OK(cudaMemcpyAsync(pres, c->S.pres, N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(rhs1, c->S.rhs1, N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(pdiag, c->S.pdiag, N * sizeof(double), cudaMemcpyDeviceToHost, st));
        cbs3d_cg_result r{};
        const cbs3d_status conv = c->pcg.read_result(r, st);
        DevStatus ds{};
        CUDA_OK(cudaMemcpy(&ds, c->S.status, sizeof ds, cudaMemcpyDeviceToHost));
        if (result) *result = r;
        if (ds.code != 0 && ds.code != CBS3D_NOT_CONVERGED) throw Error(static_cast<cbs3d_status>(ds.code), reason_text(ds));
        if (conv != CBS3D_OK) throw Error(conv, "Steps::step2SemiImplicit - pressure solver failed to converge");
    });
}

cbs3d_status cbs3d_pressure_multiply(cbs3d_ctx* c, const double* x, double* y)
{
    return guarded(c, [&] {
        const size_t N = c->m.N;
        DevState& S = c->S;
        double* dx = c->pcg.d_r;
        double* dy = c->pcg.d_q;
        CUDA_OK(cudaStreamSynchronize(c->st));
        CUDA_OK(cudaMemcpy(dx, x, N * sizeof(double), cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemsetAsync(dy, 0, N * sizeof(double), c->st));
        k_gstif<<<nb(c->m.E), T, 0, c->st>>>(S, S.elbuf);
        for (int col = 0; col < c->m.ncolor; ++col) {
            const int beg = c->m.color_ptr[static_cast<size_t>(col)], end = c->m.color_ptr[static_cast<size_t>(col) + 1];
            if (end > beg) k_matvec_color<<<nb(end - beg), T, 0, c->st>>>(S, c->d_color_elem, beg, end, S.elbuf, dx, dy);
        }
        k_matvec_diag<<<nb(c->m.N), T, 0, c->st>>>(S, dx, dy);
        CUDA_OK(cudaGetLastError());
        CUDA_OK(cudaStreamSynchronize(c->st));
        CUDA_OK(cudaMemcpy(y, dy, N * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

}  // extern "C"

// ====================================================== drop-in PCG handle
struct cbs3d_pcg {
    HostModel m;          // only E, N and the operator pattern are used
    cbs3d_options opt{};
    cudaStream_t st = nullptr;
    DeviceBuffers buf;
    PcgEngine eng;
    uint8_t* d_nflag = nullptr;
    double* d_pfix = nullptr;
    DevStatus* d_status = nullptr;
    double *d_gstif = nullptr, *d_pres = nullptr, *d_rhs1 = nullptr, *d_pdiag = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    ~cbs3d_pcg()
    {
        eng.release();
        buf.release();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (st) cudaStreamDestroy(st);
    }
};

extern "C" {

cbs3d_status cbs3d_pcg_create(int nelem, int npoin, const int* intma, const int* mat_elem, int bc_fixed,
                              const int* bc_list, const double* bc_values, const cbs3d_options* opt,
                              cbs3d_pcg** out, char* err, size_t errlen)
{
    if (!out) return CBS3D_INVALID_INPUT;
    *out = nullptr;
    auto p = std::make_unique<cbs3d_pcg>();
    try {
        if (nelem < 1 || npoin < 1 || !intma || bc_fixed < 0 || (bc_fixed > 0 && (!bc_list || !bc_values)))
            throw Error(CBS3D_INVALID_INPUT, "cbs3d_pcg_create - invalid sizes or null arrays");
        if (opt) p->opt = *opt; else cbs3d_default_options(&p->opt);
        HostModel& m = p->m;
        m.E = nelem;
        m.N = npoin;
        m.intma.assign(intma, intma + 4 * static_cast<size_t>(nelem));
        m.mat.assign(static_cast<size_t>(nelem), 0);
        if (mat_elem) for (int e = 0; e < nelem; ++e) m.mat[static_cast<size_t>(e)] = mat_elem[e];
        for (int v : m.intma)
            if (v < 1 || v > npoin) throw Error(CBS3D_INVALID_INPUT, "ConjugateGradient::solvePressure - element connectivity node out of range");
        build_incidence(m.intma, npoin, m.n2e_ptr, m.n2e);
        build_pressure_pattern(m.intma, m.mat, npoin, m.n2e_ptr, m.n2e, m.pat, nullptr);
        // build_pressure_active_mask / build_fixed_pressure_mask (src/linalg/ConjugateGradient.cpp:98-177)
        std::vector<uint8_t> nflag(static_cast<size_t>(npoin), 0);
        std::vector<double> pfix(static_cast<size_t>(npoin), 0.0);
        for (int e = 0; e < nelem; ++e)
            if (m.mat[static_cast<size_t>(e)] == 0)
                for (int a = 0; a < 4; ++a) nflag[static_cast<size_t>(m.intma[4 * static_cast<size_t>(e) + a] - 1)] = 1;
        bool any = false;
        for (uint8_t f : nflag) any = any || (f & 1);
        if (!any) throw Error(CBS3D_INVALID_INPUT, "ConjugateGradient::solvePressure - no fluid-connected pressure nodes found");
        for (int k = 0; k < bc_fixed; ++k) {
            const int ip = bc_list[k];
            if (ip < 1 || ip > npoin) throw Error(CBS3D_INVALID_INPUT, "ConjugateGradient::solvePressure - fixed pressure node out of range");
            if (!(nflag[static_cast<size_t>(ip - 1)] & 1))
                throw Error(CBS3D_INVALID_INPUT, "ConjugateGradient::solvePressure - fixed pressure node is not fluid-connected: node " + std::to_string(ip));
            nflag[static_cast<size_t>(ip - 1)] |= 4;
            pfix[static_cast<size_t>(ip - 1)] = bc_values[k];
        }
        CUDA_OK(cudaSetDevice(p->opt.device));
        CUDA_OK(cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking));
        CUDA_OK(cudaEventCreate(&p->ev0));
        CUDA_OK(cudaEventCreate(&p->ev1));
        p->d_nflag = p->buf.upload(nflag);
        p->d_pfix = p->buf.upload(pfix);
        p->d_status = p->buf.alloc<DevStatus>(1);
        CUDA_OK(cudaMemset(p->d_status, 0, sizeof(DevStatus)));
        const size_t N = static_cast<size_t>(npoin);
        p->d_gstif = p->buf.alloc<double>(6 * static_cast<size_t>(nelem));
        p->d_pres = p->buf.alloc<double>(N);
        p->d_rhs1 = p->buf.alloc<double>(N);
        p->d_pdiag = p->buf.alloc<double>(N);
        p->eng.inner_tol = p->opt.inner_tol > 0.0 ? p->opt.inner_tol : 0.05;
        p->eng.init(m, p->d_nflag, p->d_pfix, p->d_status, p->opt.device, p->opt.pcg_blocks,
                    p->opt.precision == CBS3D_MIXED, p->opt.pcg_kernel, false, p->opt.pcg_multigrid > 0);
        *out = p.release();
        return CBS3D_OK;
    } catch (const Error& e) {
        fill_err(err, errlen, e.what());
        return e.code;
    } catch (const std::exception& e) {
        fill_err(err, errlen, e.what());
        return CBS3D_INTERNAL;
    }
}

cbs3d_status cbs3d_pcg_solve(cbs3d_pcg* p, int cg_preconditioner, int cg_conv_test, int cg_max_iter,
                             double relToler, double absToler, const double* gstif, double* pdiag,
                             double* rhs1, double* pres, cbs3d_cg_result* result)
{
    if (!p) return CBS3D_INVALID_INPUT;
    try {
        // validate_cg_config, src/linalg/ConjugateGradient.cpp:508-533
        if (cg_max_iter < 1) throw Error(CBS3D_INVALID_INPUT, "ConjugateGradient::solvePressure - cg_max_iter must be positive");
        if (relToler <= 0.0 || absToler <= 0.0) throw Error(CBS3D_INVALID_INPUT, "ConjugateGradient::solvePressure - relToler and absToler must be positive");
        if (cg_preconditioner < 0 || cg_preconditioner > 1) throw Error(CBS3D_INVALID_INPUT, "ConjugateGradient::solvePressure - cg_preconditioner must be 0 or 1");
        if (cg_conv_test < 1 || cg_conv_test > 3) throw Error(CBS3D_INVALID_INPUT, "ConjugateGradient::solvePressure - cg_conv_test must be 1, 2, or 3");
        if (!gstif || !pdiag || !rhs1 || !pres) throw Error(CBS3D_INVALID_INPUT, "cbs3d_pcg_solve - null array");
        const size_t N = static_cast<size_t>(p->m.N), E = static_cast<size_t>(p->m.E);
        CUDA_OK(cudaSetDevice(p->opt.device));
        CUDA_OK(cudaMemsetAsync(p->d_status, 0, sizeof(DevStatus), p->st));
        CUDA_OK(cudaMemcpyAsync(p->d_gstif, gstif, 6 * E * sizeof(double), cudaMemcpyHostToDevice, p->st));
        CUDA_OK(cudaMemcpyAsync(p->d_pdiag, pdiag, N * sizeof(double), cudaMemcpyHostToDevice, p->st));
        CUDA_OK(cudaMemcpyAsync(p->d_rhs1, rhs1, N * sizeof(double), cudaMemcpyHostToDevice, p->st));
        CUDA_OK(cudaMemcpyAsync(p->d_pres, pres, N * sizeof(double), cudaMemcpyHostToDevice, p->st));
        CUDA_OK(cudaEventRecord(p->ev0, p->st));
        p->eng.assemble_from_gstif(p->d_gstif, p->st);
        p->eng.solve(p->d_pres, p->d_rhs1, p->d_pdiag, cg_preconditioner, cg_conv_test, cg_max_iter,
                     relToler, absToler, p->st, false);
        CUDA_OK(cudaEventRecord(p->ev1, p->st));
        CUDA_OK(cudaMemcpyAsync(pres, p->d_pres, N * sizeof(double), cudaMemcpyDeviceToHost, p->st));
        CUDA_OK(cudaMemcpyAsync(rhs1, p->d_rhs1, N * sizeof(double), cudaMemcpyDeviceToHost, p->st));
        CUDA_OK(cudaMemcpyAsync(pdiag, p->d_pdiag, N * sizeof(double), cudaMemcpyDeviceToHost, p->st));
        cbs3d_cg_result r{};
        const cbs3d_status conv = p->eng.read_result(r, p->st);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, p->ev0, p->ev1);
        r.total_seconds = ms * 1.0e-3;
        if (result) *result = r;
        DevStatus s{};
        CUDA_OK(cudaMemcpy(&s, p->d_status, sizeof s, cudaMemcpyDeviceToHost));
        if (s.code != 0 && s.code != CBS3D_NOT_CONVERGED) throw Error(static_cast<cbs3d_status>(s.code), reason_text(s));
        p->err = conv == CBS3D_OK ? "" : "Steps::step2SemiImplicit - pressure solver failed to converge";
        return conv;
    } catch (const Error& e) {
        p->err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        p->err = e.what();
        return CBS3D_INTERNAL;
    }
}

void cbs3d_pcg_destroy(cbs3d_pcg* p) { delete p; }

cbs3d_status cbs3d_coarse_inverse(int device, int g, const double* a, double* ainv, int variant)
{
    try {
        return coarse_inverse(device, g, a, ainv, variant);
    } catch (const Error& e) {
        return e.code;
    } catch (const std::exception&) {
        return CBS3D_INTERNAL;
    }
}

cbs3d_status cbs3d_selftest_wait_timeout(int device, int* observed_status)
{
    try {
        return selftest_wait_timeout(device, observed_status);
    } catch (const Error& e) {
        return e.code;
    } catch (const std::exception&) {
        return CBS3D_INTERNAL;
    }
}

const char* cbs3d_pcg_last_error(const cbs3d_pcg* p) { return p ? p->err.c_str() : "null solver"; }

}  // extern "C"

// ================================================================ batch
struct cbs3d_batch {
    std::vector<std::unique_ptr<cbs3d_ctx>> inst;
    cbs3d_batch_options opt{};
    PcgBatch pcg;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork_pre = nullptr, fork_post = nullptr;
    std::vector<cudaEvent_t> done_pre, done_post;
    cudaGraphExec_t gexec = nullptr;
    bool graph_failed = false;
    bool tuned = false;
    int iitime = 0;
    long long launches = 0;
    cbs3d_batch_info info{};
    std::string err;

    ~cbs3d_batch()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        pcg.release();
        cudaEvent_t evs[] = {ev0, ev1, fork_pre, fork_post};
        for (cudaEvent_t e : evs) if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : done_pre) cudaEventDestroy(e);
        for (cudaEvent_t e : done_post) cudaEventDestroy(e);
        inst.clear();
        if (st) cudaStreamDestroy(st);
    }

    int kernels_per_step(int it) const
    {
        int n = pcg.nwaves();
        for (const auto& c : inst) n += c->kernels_outside_solve(it) + pcg.launches_per_instance();
        return n;
    }

    void enqueue_pre_all(int it)
    {
        CUDA_OK(cudaEventRecord(fork_pre, st));
        for (size_t k = 0; k < inst.size(); ++k) {
            cbs3d_ctx& c = *inst[k];
            CUDA_OK(cudaStreamWaitEvent(c.st, fork_pre, 0));
            c.enqueue_pre(it);
        }
    }
    void enqueue_prepare_all()
    {
        for (size_t k = 0; k < inst.size(); ++k) {
            cbs3d_ctx& c = *inst[k];
            pcg.prepare(static_cast<int>(k), c.S, c.st);
            CUDA_OK(cudaEventRecord(done_pre[k], c.st));
            CUDA_OK(cudaStreamWaitEvent(st, done_pre[k], 0));
        }
    }
    void enqueue_post_all(int it)
    {
        CUDA_OK(cudaEventRecord(fork_post, st));
        for (size_t k = 0; k < inst.size(); ++k) {
            cbs3d_ctx& c = *inst[k];
            CUDA_OK(cudaStreamWaitEvent(c.st, fork_post, 0));
            pcg.finish(static_cast<int>(k), c.S.pres, c.st);
            c.enqueue_post(it);
            CUDA_OK(cudaEventRecord(done_post[k], c.st));
            CUDA_OK(cudaStreamWaitEvent(st, done_post[k], 0));
        }
    }
    void enqueue_step(int it)
    {
        enqueue_pre_all(it);
        enqueue_prepare_all();
        pcg.solve(st);
        enqueue_post_all(it);
    }

    // First step with the autotuner: the stages before the solve run once;
    // every feasible tiling then solves the same systems (inputs re-staged
    // each time, the node-order pressure untouched) and is timed; the fastest
    // is kept and solves the step for real.
    void autotune_step(int it)
    {
        enqueue_pre_all(it);
        const PcgBatchPlan start = pcg.current;
        double best = 1e300;
        PcgBatchPlan best_plan = start;
        int nc = 0;
        const int rows[3] = {2, 4, 8};
        for (int spread = 1; spread >= 0; --spread) {
            for (int r : rows) {
                if (nc >= 8) break;
                PcgBatchPlan p;
                p.rmax = r;
                p.spread = spread;
                info.cand_rows[nc] = r;
                info.cand_spread[nc] = spread;
                info.cand_ms[nc] = -1.0;
                std::string why;
                if (pcg.plan(p, &why)) {
                    float ms = 1e30f;
                    for (int rep = 0; rep < 2; ++rep) {
                        enqueue_prepare_all();
                        CUDA_OK(cudaEventRecord(ev0, st));
                        pcg.solve(st);
                        CUDA_OK(cudaEventRecord(ev1, st));
                        CUDA_OK(cudaStreamSynchronize(st));
                        float m = 0.0f;
                        CUDA_OK(cudaEventElapsedTime(&m, ev0, ev1));
                        ms = std::min(ms, m);
                    }
                    info.cand_ms[nc] = ms;
                    if (ms < best) { best = ms; best_plan = p; }
                }
                ++nc;
            }
        }
        info.candidates = nc;
        std::string why;
        if (!pcg.plan(best_plan, &why)) throw Error(CBS3D_INTERNAL, "batch autotuner: " + why);
        tuned = true;
        enqueue_prepare_all();
        pcg.solve(st);
        enqueue_post_all(it);
    }
};

namespace {

void batch_fill_info(cbs3d_batch* b)
{
    b->info.instances = static_cast<int>(b->inst.size());
    b->info.waves = b->pcg.nwaves();
    b->info.rows_per_thread = b->pcg.current.rmax;
    b->info.spread = b->pcg.current.spread;
    b->info.mixed_waves = b->pcg.mixed_any ? 1 : 0;
    b->info.tuned = b->tuned ? 1 : 0;
}

}  // namespace

extern "C" {

void cbs3d_default_batch_options(cbs3d_batch_options* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    cbs3d_default_options(&o->base);
    o->autotune = 1;
    o->rows_per_thread = 4;
    o->spread = 1;
}

cbs3d_status cbs3d_batch_create(int n, const cbs3d_mesh* meshes, const cbs3d_params* params,
                                const cbs3d_batch_options* opt, cbs3d_batch** out, char* err, size_t errlen)
{
    if (n < 1 || !meshes || !params || !out) return CBS3D_INVALID_INPUT;
    *out = nullptr;
    auto b = std::make_unique<cbs3d_batch>();
    try {
        if (opt) b->opt = *opt; else cbs3d_default_batch_options(&b->opt);
        const int rpt = b->opt.rows_per_thread;
        if (rpt != 0 && rpt != 1 && rpt != 2 && rpt != 4 && rpt != 8)
            throw Error(CBS3D_INVALID_INPUT, "cbs3d_batch_create - rows_per_thread must be 1, 2, 4 or 8");
        CUDA_OK(cudaSetDevice(b->opt.base.device));
        CUDA_OK(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
        CUDA_OK(cudaEventCreate(&b->ev0));
        CUDA_OK(cudaEventCreate(&b->ev1));
        CUDA_OK(cudaEventCreateWithFlags(&b->fork_pre, cudaEventDisableTiming));
        CUDA_OK(cudaEventCreateWithFlags(&b->fork_post, cudaEventDisableTiming));
        std::vector<PcgBatchMember> mem;
        for (int i = 0; i < n; ++i) {
            auto c = std::make_unique<cbs3d_ctx>();
            try {
                model_from_arrays(meshes[i], params[i], c->m);
                c->opt = b->opt.base;
                c->opt.time_pcg = 0;
                c->setup(false);
            } catch (const Error& e) {
                throw Error(e.code, "instance " + std::to_string(i) + ": " + e.what());
            }
            mem.push_back(PcgBatchMember{&c->m, c->S.nflag, c->S.pfix, c->S.status});
            b->inst.push_back(std::move(c));
            cudaEvent_t e1, e2;
            CUDA_OK(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
            CUDA_OK(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming));
            b->done_pre.push_back(e1);
            b->done_post.push_back(e2);
        }
        const double itol = b->opt.base.inner_tol > 0.0 ? b->opt.base.inner_tol : 0.05;
        b->pcg.init(mem, b->opt.base.device, b->opt.base.precision == CBS3D_MIXED, itol);
        for (int i = 0; i < n; ++i) b->inst[static_cast<size_t>(i)]->batch_out = b->pcg.out(i);
        PcgBatchPlan p;
        p.rmax = b->opt.rows_per_thread > 0 ? b->opt.rows_per_thread : 4;
        p.spread = b->opt.spread ? 1 : 0;
        std::string why;
        if (!b->pcg.plan(p, &why)) {
            p.rmax = 8;   // the widest tiling holds the largest instances
            if (!b->pcg.plan(p, &why)) throw Error(CBS3D_INVALID_INPUT, "cbs3d_batch_create - " + why);
        }
        batch_fill_info(b.get());
        *out = b.release();
        return CBS3D_OK;
    } catch (const Error& e) {
        fill_err(err, errlen, e.what());
        return e.code;
    } catch (const std::exception& e) {
        fill_err(err, errlen, e.what());
        return CBS3D_INTERNAL;
    }
}

cbs3d_status cbs3d_batch_step(cbs3d_batch* b, int nsteps, cbs3d_step_stats* stats, double* gpu_seconds)
{
    return guarded(b, [&] {
        if (nsteps < 0) throw Error(CBS3D_INVALID_INPUT, "cbs3d_batch_step - nsteps must be >= 0");
        const size_t K = b->inst.size();
        if (stats) std::memset(stats, 0, K * sizeof *stats);
        CUDA_OK(cudaSetDevice(b->opt.base.device));
        std::vector<int> start(K);
        std::vector<long long> launches0(K);
        for (size_t k = 0; k < K; ++k) {
            cbs3d_ctx& c = *b->inst[k];
            const bool realloc = !c.d_log || nsteps > c.log_cap;
            c.ensure_log(nsteps > 0 ? nsteps : 1);
            if (realloc && b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
            c.reset_status();
            CUDA_OK(cudaMemsetAsync(c.d_counter, 0, sizeof(int), c.st));
            CUDA_OK(cudaStreamSynchronize(c.st));
            start[k] = c.iitime;
            launches0[k] = c.launches;
            c.pcg_ev_used = 0;
        }
        CUDA_OK(cudaEventRecord(b->ev0, b->st));
        int done = 0;
        for (int s = 0; s < nsteps; ++s) {
            const int it = b->iitime + 1;
            bool graphable = b->opt.base.use_graph && !b->graph_failed;
            for (const auto& c : b->inst)
                if (c->m.p.dtfix_end > 0 && it <= c->m.p.dtfix_end) graphable = false;
            if (b->opt.autotune && !b->tuned) {
                // The autotuner times candidates with the same events, so the
                // call's device time starts after the tuned step.
                b->autotune_step(it);
                if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
                CUDA_OK(cudaStreamSynchronize(b->st));
                CUDA_OK(cudaEventRecord(b->ev0, b->st));
            } else {
                if (graphable && !b->gexec) {
                    cudaGraph_t g = nullptr;
                    bool ok = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                    if (ok) {
                        try {
                            b->enqueue_step(it);
                        } catch (const Error&) {
                            ok = false;
                        }
                        cudaGraph_t gg = nullptr;
                        const bool ended = cudaStreamEndCapture(b->st, &gg) == cudaSuccess && gg;
                        g = gg;
                        ok = ok && ended;
                    }
                    if (ok) ok = cudaGraphInstantiate(&b->gexec, g, 0) == cudaSuccess;
                    if (g) cudaGraphDestroy(g);
                    if (!ok) {
                        cudaGetLastError();
                        b->graph_failed = true;
                        b->gexec = nullptr;
                    }
                }
                if (graphable && b->gexec) CUDA_OK(cudaGraphLaunch(b->gexec, b->st));
                else b->enqueue_step(it);
            }
            const int kn = b->kernels_per_step(it);
            b->launches += kn;
            for (auto& c : b->inst) {
                c->launches += c->kernels_outside_solve(it) + b->pcg.launches_per_instance();
                c->iitime = it;
            }
            CUDA_OK(cudaGetLastError());
            b->iitime = it;
            ++done;
        }
        CUDA_OK(cudaEventRecord(b->ev1, b->st));
        CUDA_OK(cudaStreamSynchronize(b->st));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        if (gpu_seconds) *gpu_seconds = ms * 1.0e-3;
        batch_fill_info(b);
        int bad = -1;
        DevStatus first{};
        for (size_t k = 0; k < K; ++k) {
            const DevStatus s = collect_call(b->inst[k].get(), done, start[k], launches0[k], false, ms,
                                             stats ? stats + k : nullptr);
            if (s.code != 0 && bad < 0) { bad = static_cast<int>(k); first = s; }
        }
        if (bad >= 0) {
            const int fstep = start[static_cast<size_t>(bad)] + (first.step > 0 ? first.step : done);
            throw Error(static_cast<cbs3d_status>(first.code),
                        "instance " + std::to_string(bad) + ": " + reason_text(first) + " (step " + std::to_string(fstep) + ")");
        }
    });
}

cbs3d_status cbs3d_batch_download_fields(cbs3d_batch* b, int instance, double* u, double* p, double* t)
{
    if (!b || instance < 0 || instance >= static_cast<int>(b->inst.size())) return CBS3D_INVALID_INPUT;
    const cbs3d_status s = cbs3d_download_fields(b->inst[static_cast<size_t>(instance)].get(), u, p, t);
    if (s != CBS3D_OK) b->err = b->inst[static_cast<size_t>(instance)]->err;
    return s;
}

cbs3d_status cbs3d_batch_get_info(const cbs3d_batch* b, cbs3d_batch_info* info)
{
    if (!b || !info) return CBS3D_INVALID_INPUT;
    *info = b->info;
    return CBS3D_OK;
}

void cbs3d_batch_destroy(cbs3d_batch* b) { delete b; }

const char* cbs3d_batch_last_error(const cbs3d_batch* b) { return b ? b->err.c_str() : "null batch"; }


// ----------------------------------------------------------------- output
cbs3d_status cbs3d_step_history(cbs3d_ctx* c, int first, int count, double* rec)
{
    return guarded(c, [&] {
        if (!rec || first < 0 || count < 0 || first + count > c->last_done)
            throw Error(CBS3D_INVALID_INPUT, "cbs3d_step_history - range outside the latest call's steps");
        if (count) CUDA_OK(cudaMemcpy(rec, c->d_log + static_cast<size_t>(first) * LOG_FIELDS,
                                      static_cast<size_t>(count) * LOG_FIELDS * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

cbs3d_status cbs3d_write_residual_rows(cbs3d_ctx* c, const char* path, int header)
{
    return guarded(c, [&] {
        if (!path) throw Error(CBS3D_INVALID_INPUT, "cbs3d_write_residual_rows - path required");
        if (c->m.p.residual_log_enabled < 1) return;
        if (header) write_residual_header(path);
        const int n = c->last_done;
        if (n < 1) return;
        std::vector<double> rec(static_cast<size_t>(n) * LOG_FIELDS);
        CUDA_OK(cudaMemcpy(rec.data(), c->d_log, rec.size() * sizeof(double), cudaMemcpyDeviceToHost));
        append_residual_rows(path, c->last_start + 1, c->m.p.residual_log_every, rec.data(), n);
    });
}

cbs3d_status cbs3d_write_vtu(cbs3d_ctx* c, const char* path)
{
    return guarded(c, [&] {
        if (!path) throw Error(CBS3D_INVALID_INPUT, "cbs3d_write_vtu - path required");
        const size_t N = c->m.N;
        std::vector<double> u(3 * N), p(N), t(N), v(N);
        CUDA_OK(cudaStreamSynchronize(c->st));
        CUDA_OK(cudaMemcpy(u.data(), c->S.unkno, 3 * N * sizeof(double), cudaMemcpyDeviceToHost));
        CUDA_OK(cudaMemcpy(p.data(), c->S.pres, N * sizeof(double), cudaMemcpyDeviceToHost));
        CUDA_OK(cudaMemcpy(t.data(), c->S.temp, N * sizeof(double), cudaMemcpyDeviceToHost));
        CUDA_OK(cudaMemcpy(v.data(), c->S.velocity, N * sizeof(double), cudaMemcpyDeviceToHost));
        // before the first step the device magnitude is not yet computed
        write_vtu(path, c->m, u.data(), p.data(), t.data(), c->iitime > 0 ? v.data() : nullptr);
    });
}

cbs3d_status cbs3d_write_vtu_async(cbs3d_ctx* c, const char* path)
{
    return guarded(c, [&] {
        if (!path) throw Error(CBS3D_INVALID_INPUT, "cbs3d_write_vtu_async - path required");
        CUDA_OK(cudaSetDevice(c->opt.device));
        if (!c->snaps) c->snaps.reset(new VtuSnapshots(c->opt.device, c->m, c->m.N));
        // before the first step the device magnitude is not yet computed
        c->snaps->enqueue(c->st, c->S.unkno, c->S.pres, c->S.temp, c->iitime > 0 ? c->S.velocity : nullptr, path);
    });
}

cbs3d_status cbs3d_vtu_flush(cbs3d_ctx* c)
{
    return guarded(c, [&] {
        if (!c->snaps) return;
        const std::string e = c->snaps->flush();
        if (!e.empty()) throw Error(CBS3D_IO_ERROR, e);
    });
}

cbs3d_status cbs3d_write_vtu_case(const char* case_name, const char* path, const double* u, const double* p,
                                  const double* t, char* err, size_t errlen)
{
    if (!case_name || !path || !u || !p || !t) return CBS3D_INVALID_INPUT;
    try {
        HostModel m;
        parse_case(case_name, m);
        write_vtu(path, m, u, p, t, nullptr);
        return CBS3D_OK;
    } catch (const Error& e) {
        fill_err(err, errlen, e.what());
        return e.code;
    } catch (const std::exception& e) {
        fill_err(err, errlen, e.what());
        return CBS3D_INTERNAL;
    }
}

cbs3d_status cbs3d_write_pvd(const char* path, int n, const char* const* files, const double* times)
{
    if (!path || n < 0 || (n > 0 && (!files || !times))) return CBS3D_INVALID_INPUT;
    try {
        std::vector<std::string> f;
        for (int i = 0; i < n; ++i) f.emplace_back(files[i]);
        write_pvd(path, f, std::vector<double>(times, times + n));
        return CBS3D_OK;
    } catch (const Error& e) {
        return e.code;
    } catch (const std::exception&) {
        return CBS3D_INTERNAL;
    }
}

}  // extern "C"
