/*
 * cbs3d_gpu.h - C ABI of the B200 CBS3D step engine.
 *
 * Plain pointers and sizes only; no exceptions cross this boundary.  Every
 * call returns a cbs3d_status; cbs3d_last_error() gives the message, worded
 * like the reference's std::runtime_error text where one exists.
 *
 * Host arrays follow the reference's storage order with the unused 1-based
 * slot removed (a reference caller passes Array.raw().data() + 1):
 *   intma[4*nelem]   element-major, 1-based node ids
 *   coord[3*npoin]   node-major x,y,z          unkno[3*npoin] node-major u,v,w
 *   gstif[6*nelem]   pair order 12,13,14,23,24,34
 *   bface[5*nboun]   n1 n2 n3 parent_element solver_bc   (1-based ids)
 *
 * One context owns one CUDA stream and its device memory; a context is not
 * thread-safe, separate contexts are independent.
 */
#ifndef CBS3D_GPU_H
#define CBS3D_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cbs3d_status {
    CBS3D_OK = 0,
    CBS3D_INVALID_INPUT = 1,   /* bad mesh/parameter/state (reference: runtime_error) */
    CBS3D_NOT_CONVERGED = 2,   /* pressure PCG hit cg_max_iter */
    CBS3D_BREAKDOWN = 3,       /* PCG pAp or r.z dot product invalid */
    CBS3D_NONFINITE = 4,       /* NaN/Inf met in a field or residual */
    CBS3D_TIMEOUT = 5,         /* a device-side wait ran out of its spin limit */
    CBS3D_CUDA_ERROR = 6,
    CBS3D_IO_ERROR = 7,        /* case file missing or malformed */
    CBS3D_INTERNAL = 8
} cbs3d_status;

typedef enum cbs3d_precision {
    CBS3D_FP64 = 0,            /* every stage in FP64 (parity form) */
    CBS3D_MIXED = 1            /* FP32 inner PCG with FP64 residual correction */
} cbs3d_precision;

/* Run configuration: the RunConfig fields read by the step path
 * (reference include/cbs/core/RunConfig.hpp:38-323), as parsed from .par. */
typedef struct cbs3d_params {
    int solver_opt, restart_opt, temp_calc;
    double cinf[5];                               /* Ux Uy Uz P T */
    int ntime, transient_on, dtfixed;
    double dtfix;
    int iwrite;
    double csafm, theta1;
    int cbs_scheme, ilots, htype, step2_check, rem_deltp, beta_opt, dtfix_end;
    double csafm2, epsilon1, deltr;
    double re, pr, ra, ri;
    int convection_type, pnode;
    int write_output;
    double write_time_output, time_output_interval, end_rtime;
    double relToler, absToler;
    int vel_check;
    double l2norm_vel_tolerance;
    int temp_check;
    double l2norm_temp_tolerance;
    int paraview_output, tecplot_output, nusselt_calc, nusselt_flag, runtime_mod;
    double alpha_sf, k_ratio, source_solid, heat_flux_bc;
    int dimensional_mode, material_properties_enabled, mass_flow_inlet_enabled;
    double p_ref, model_depth, inlet_mass_flow_rate, inlet_density, inlet_temperature,
           outlet_pressure_gauge;
    double inlet_u, inlet_v, inlet_w;
    double nusselt_Tinf, nusselt_Tref, nusselt_diameter;
    int cg_preconditioner, cg_conv_test, cg_max_iter;
    double l2norm_pres_tolerance;
    int residual_log_enabled, residual_log_every, console_log_every, live_residual_plot,
        vtu_output_enabled, vtu_output_every_iterations;
    double vtu_output_every_sim_time;
    int write_boundary_debug_arrays, steady_min_iterations, art_diff;
} cbs3d_params;

/* Mesh in the reference layout after .bco mapping.  The property arrays are
 * per element and are read only when material_properties_enabled > 0. */
typedef struct cbs3d_mesh {
    int nelem, npoin, nboun;
    const int* intma;
    const double* coord;
    const int* bface;
    const int* mat_elem;                           /* may be NULL: all fluid */
    const double *rho, *cp, *k, *mu, *qvol;        /* may be NULL */
} cbs3d_mesh;

typedef struct cbs3d_options {
    int precision;           /* cbs3d_precision */
    int device;              /* CUDA device ordinal */
    double inner_tol;        /* MIXED: the FP32 recurrences are replaced by the FP64 true residual
                                whenever the recursive residual has fallen by this factor (default 0.05) */
    int use_graph;           /* capture the per-step launch sequence in a CUDA graph */
    int pcg_blocks;          /* persistent PCG grid size; 0 = one wave of resident CTAs */
    int verbose;
    int time_pcg;            /* time every PCG launch with CUDA events (no graph capture) */
    int pcg_kernel;          /* 0 automatic; 1 vectors in global memory, 2 register-resident rows,
                                3 shared-memory halo, 4 halo + one grid sync per iteration,
                                5 vectors in global memory + one grid sync per iteration,
                                10 as 4 with no coefficients kept in tensor memory,
                                11 as 4 with the first row per thread in shared memory and the
                                next ones in tensor memory (0 and 4 keep every row in tensor
                                memory where they all fit, else as 11) */
    int case_cache;          /* cbs3d_create_from_case: keep the parsed case in <case>.cbscache
                                (keyed by every source file's size and time) and reuse it */
    int pcg_two_level;       /* extension: Jacobi plus a coarse correction on one aggregate of rows
                                per CTA (the aggregated operator is rebuilt and inverted every solve);
                                same stopping test, far fewer iterations; large meshes only */
    int pcg_multigrid;       /* extension (the counterpart of the reference's PETSc/AMG path,
                                src/linalg/PetscPressureSolver.cpp:335-360): aggregation-multigrid
                                V-cycle preconditioned CG in place of Jacobi-PCG; hierarchy fixed by
                                the mesh (aggregates of 8 Morton-ordered rows), Galerkin coarse
                                operators rebuilt every solve, same stopping test; FP64, for meshes
                                up to 655,360 row positions (else Jacobi) */
} cbs3d_options;

/* Mirrors ConjugateGradient::Result (include/cbs/linalg/ConjugateGradient.hpp:36-68).
 * Timings are GPU-event times of the solve; the reference's per-part timers
 * have no separate counterpart inside the fused kernel and stay 0. */
typedef struct cbs3d_cg_result {
    int iterations;
    double initial_l2, final_l2, final_relative_l2, final_max_abs;
    int converged;
    double total_seconds, setup_seconds, matvec_seconds, dot_seconds,
           preconditioner_seconds, vector_update_seconds, constraint_seconds;
    int matvec_calls, dot_calls, preconditioner_calls;
    int outer_sweeps;        /* MIXED: FP64 residual corrections performed */
} cbs3d_cg_result;

typedef struct cbs3d_step_stats {
    int steps_done;          /* steps completed by this call */
    int iitime;              /* global step counter after the call */
    int failed_step;         /* step at which a failure was detected, else 0 */
    double dtreal;           /* last step's global minimum time step */
    double rtime;            /* accumulated physical time (transient runs) */
    cbs3d_cg_result cg;      /* last step's pressure solve */
    long long cg_iterations_total;
    double hb[15];           /* Convergence::evaluate measures of the last step */
    double gpu_seconds;      /* device time of the steps of this call */
    int steady_reached;      /* Convergence::steadyStateReached at the last step */
    double pcg_seconds;      /* with time_pcg: summed duration of the PCG kernel launches */
    int pcg_launches;        /* with time_pcg: PCG kernel launches timed */
    long long kernel_launches; /* kernels this library launched during the call */
    double pcg_bytes_per_iter; /* bytes one PCG iteration of the selected kernel moves */
    int pcg_kernel;          /* PCG kernel in use: 1 global vectors, 2 register rows,
                                3 shared-memory halo, 4 single-reduction (CG-CG),
                                5 mixed FP32/FP64, 6 two-level (CG-CG + coarse correction),
                                7 aggregation-multigrid preconditioned CG,
                                8 global vectors, single-reduction (CG-CG),
                                9 single-reduction (CG-CG) with coefficients in tensor memory */
} cbs3d_step_stats;

typedef struct cbs3d_ctx cbs3d_ctx;
typedef struct cbs3d_pcg cbs3d_pcg;

int cbs3d_version(void);
const char* cbs3d_status_string(cbs3d_status s);
void cbs3d_default_options(cbs3d_options* opt);
void cbs3d_default_params(cbs3d_params* p);

/* Parses <case>.par/.plt/.bco[/.material/.matprop] with the grammar of
 * MeshIO::readAll (reference src/io/MeshIO.cpp:572-1701) into caller-visible
 * sizes and parameters.  Replaces MeshIO::readSizes/readParameterFile. */
cbs3d_status cbs3d_read_params(const char* case_name, cbs3d_params* params,
                               int* nelem, int* npoin, int* nboun, char* err, size_t errlen);

/* Host only (no device; no reference counterpart): parses <case> as
 * cbs3d_create_from_case does, through the binary cache when use_cache, and
 * returns a 64-bit digest of the parsed inputs and whether they came from
 * the cache. */
cbs3d_status cbs3d_case_digest(const char* case_name, int use_cache, unsigned long long* digest,
                               int* from_cache, char* err, size_t errlen);

/* Reads the case files and builds a device context: replaces MeshIO::readAll
 * + Solver::initialise + Solver::preparePressureSystem
 * (reference src/solver/Solver.cpp:242-302, 587-593). */
cbs3d_status cbs3d_create_from_case(const char* case_name, const cbs3d_options* opt,
                                    cbs3d_ctx** out, char* err, size_t errlen);

/* Same from in-memory arrays (raw side ids already mapped to solver BCs).
 * Applies MeshIO::initialiseFields (src/io/MeshIO.cpp:1627-1701). */
cbs3d_status cbs3d_create(const cbs3d_mesh* mesh, const cbs3d_params* params,
                          const cbs3d_options* opt, cbs3d_ctx** out, char* err, size_t errlen);

void cbs3d_destroy(cbs3d_ctx* ctx);
const char* cbs3d_last_error(const cbs3d_ctx* ctx);

/* Advances nsteps CBS steps, each replacing Solver::advanceOneStep
 * (reference src/solver/Solver.cpp:609-680): TimeStep::computeTimeStep,
 * updateLhsDiagonal, Steps::step1..step4, updateVelocityMagnitude and
 * Convergence::evaluate, all on the device.  Stops early with
 * stop_on_steady != 0 once Solver::steadyStateReached would stop the
 * reference loop (src/solver/Solver.cpp:197-203, 708-716). */
cbs3d_status cbs3d_step(cbs3d_ctx* ctx, int nsteps, int stop_on_steady, cbs3d_step_stats* stats);

/* Field transfer (node-major, npoin entries per scalar).  NULL skips a field. */
cbs3d_status cbs3d_upload_fields(cbs3d_ctx* ctx, const double* unkno, const double* pres,
                                 const double* temperature);
cbs3d_status cbs3d_download_fields(cbs3d_ctx* ctx, double* unkno, double* pres,
                                   double* temperature);

/* Named state access for stage-level checks (names follow CBSStateSI:
 * unkno unkn1 pres pres1 temperature temperature1 rhs rhs1 delte elcoe2
 * elcoe2p pdiag gstif detJ dNkdx annxf alen_e pdiagE gstifE velocity dtreal
 * hb ncolor color_ptr color_elem bc_list wall_node_list fedge iside).
 * count is the caller's capacity in elements; *written receives the size. */
cbs3d_status cbs3d_get_array(cbs3d_ctx* ctx, const char* name, void* host, long count, long* written);
cbs3d_status cbs3d_set_array(cbs3d_ctx* ctx, const char* name, const void* host, long count);

/* Runs one named stage of a step on the device: begin_step, time_step, lhs,
 * step1, step2_rhs, solve_pressure, step3, step4, convergence. */
cbs3d_status cbs3d_run_stage(cbs3d_ctx* ctx, const char* stage);

/* The pressure-solver drop-in on a context (solver_opt=1 semantics of
 * ConjugateGradient::solvePressure, src/linalg/ConjugateGradient.cpp:584-869,
 * with the context's cg_* parameters): host arrays gstif[6*nelem] (pair
 * order 12,13,14,23,24,34 per element), pdiag, rhs1 and pres[npoin]; pres is
 * the initial guess and the solution, rhs1 and pdiag come back with the
 * fixed and inactive rows imposed.  Returns CBS3D_NOT_CONVERGED (result
 * filled) when the stopping test is not met. */
cbs3d_status cbs3d_solve_pressure(cbs3d_ctx* ctx, const double* gstif, double* pdiag, double* rhs1, double* pres,
                                  cbs3d_cg_result* result);

/* y = A x with the context's current pressure operator
 * (MatrixVectorCalc::pressureMultiply, src/linalg/MatrixVectorCalc.cpp:125-205). */
cbs3d_status cbs3d_pressure_multiply(cbs3d_ctx* ctx, const double* x, double* y);

/* ---------------------------------------------------------------------------
 * Run output (Post::writeResidualRow / writeVTU / writePVD,
 * reference src/io/Post.cpp:525-560, 768-815, 887-1180).  Residual rows come
 * from the device step log of the latest cbs3d_step call (dtreal, the PCG
 * result, the 15 Convergence::evaluate measures, time), so no field leaves
 * the device for them.  VTU files are binary-appended with the reference's
 * arrays and cells (tets, then boundary triangles).
 * --------------------------------------------------------------------------- */
/* Records of steps [first, first+count) of the latest cbs3d_step call, 24
 * doubles each: dtreal, cg iterations, initial_l2, final_l2, relative_l2,
 * max_abs, converged, hb[15], rtime, outer sweeps. */
cbs3d_status cbs3d_step_history(cbs3d_ctx* ctx, int first, int count, double* records);
/* Appends the latest call's rows to the residual CSV (header first when
 * header != 0), honouring residual_log_enabled / residual_log_every. */
cbs3d_status cbs3d_write_residual_rows(cbs3d_ctx* ctx, const char* path, int header);
cbs3d_status cbs3d_write_vtu(cbs3d_ctx* ctx, const char* path);
/* The same file written off the step path: the fields are copied on the
 * device on the context's stream (microseconds), copied to pinned host
 * memory on a side stream and written by a host thread of the context, so
 * the call returns at once and later steps overlap the copy-out and the
 * file write.  The file holds the fields as they are when the work already
 * issued on the context has run.  Two snapshots may be in flight; a third
 * call waits for the oldest to be written.  The first call allocates the
 * two snapshot slots (6 doubles per node each, device and pinned host).
 * cbs3d_vtu_flush waits for every pending file and returns the first write
 * error since the previous flush (CBS3D_IO_ERROR); cbs3d_destroy writes
 * what is pending.  No reference counterpart for the asynchrony. */
cbs3d_status cbs3d_write_vtu_async(cbs3d_ctx* ctx, const char* path);
cbs3d_status cbs3d_vtu_flush(cbs3d_ctx* ctx);
/* Host only: the VTU of a case's mesh with caller fields (u[3N], p[N], t[N]). */
cbs3d_status cbs3d_write_vtu_case(const char* case_name, const char* path, const double* u, const double* p,
                                  const double* t, char* err, size_t errlen);
cbs3d_status cbs3d_write_pvd(const char* path, int n, const char* const* files, const double* times);

/* ---------------------------------------------------------------------------
 * Pressure-solver drop-in: a solver_opt backend with the inputs and side
 * effects of ConjugateGradient::solvePressure(CBSStateSI&)
 * (reference src/linalg/ConjugateGradient.cpp:584-869; dispatch at
 * src/solver/Steps.cpp:305-350).  Create once after preprocessing, solve
 * every step.
 * --------------------------------------------------------------------------- */
cbs3d_status cbs3d_pcg_create(int nelem, int npoin, const int* intma, const int* mat_elem,
                              int bc_fixed, const int* bc_list, const double* bc_values,
                              const cbs3d_options* opt, cbs3d_pcg** out, char* err, size_t errlen);

/* pres: initial guess in, solution out.  rhs1 and pdiag are overwritten on
 * fixed and inactive nodes exactly as impose_pressure_constraints does. */
cbs3d_status cbs3d_pcg_solve(cbs3d_pcg* pcg, int cg_preconditioner, int cg_conv_test,
                             int cg_max_iter, double relToler, double absToler,
                             const double* gstif, double* pdiag, double* rhs1, double* pres,
                             cbs3d_cg_result* result);
void cbs3d_pcg_destroy(cbs3d_pcg* pcg);
const char* cbs3d_pcg_last_error(const cbs3d_pcg* pcg);

/* Convergence measures without any device allocation (no counterpart in the
 * reference): the 15 values of Convergence::evaluate, returned in hb, from
 * device arrays the caller already holds (node-major unkno/unkn1[3*npoin],
 * pres/pres1/temperature/temperature1/elcoe2/elcoe2p[npoin];
 * node_flags[npoin]: bit0 = node touches a fluid element, bit1 = touches a
 * solid element; the temperature arrays may be NULL when temp_calc <= 0).
 * For callers that may not call cudaMalloc -- code whose device memory is
 * owned by another allocator (a framework's caching allocator, a pool handed
 * out by an embedding application) or a process that budgeted its device
 * memory up front: the only scratch is a 1 MiB file-scope device array that
 * every GPU loading this library holds until exit.  npoin above 2,097,152 is
 * rejected with CBS3D_INVALID_INPUT, and so is a node whose flags are 0
 * (touches no element), as Convergence::evaluate rejects it
 * (src/solver/Convergence.cpp:157-161).  The first call on a device looks up
 * that array's device address; make that first call before any stream
 * capture, and do not call it again after a cudaDeviceReset of that device.
 * All calls share the array: calls whose kernels overlap on the GPU race.
 * The kernels run on the legacy default stream and the call blocks the host
 * until hb is copied back, so finish or synchronise every stream that writes
 * the inputs (this library's context streams are non-blocking) before the
 * call.  The caller's current device is restored on return. */
cbs3d_status cbs3d_convergence_norms_static(int device, const double* unkno, const double* unkn1,
                                            const double* pres, const double* pres1,
                                            const double* temperature, const double* temperature1,
                                            const double* elcoe2, const double* elcoe2p,
                                            const unsigned char* node_flags, int npoin, int temp_calc,
                                            double hb[15]);

/* ---------------------------------------------------------------------------
 * Body force, tangent-linear and adjoint runs (no reference counterpart).
 * A per-node body force f[3*npoin] (node-major) adds M_f f to the Step-1
 * momentum residual (M_f: fluid lumped mass).  The objective of the runs is
 * J = 1/2 sum_i w[i] |u_i|^2 after nsteps steps from the context's current
 * state; every run restores the state (fields, step counter, time) when it
 * returns.  Tangent and adjoint runs need a fixed time step (dtfixed > 0),
 * under which the pressure operator is constant; the adjoint's pressure
 * systems reuse the context's PCG operator.
 * --------------------------------------------------------------------------- */
/* f = NULL removes the body force. */
cbs3d_status cbs3d_set_body_force(cbs3d_ctx* ctx, const double* f);
/* J only (the forward run of the other two). */
cbs3d_status cbs3d_objective_run(cbs3d_ctx* ctx, int nsteps, const double* w, double* J);
/* J and the directional derivative dJ = (dJ/df) . df of the tangent-linear model. */
cbs3d_status cbs3d_tlm_run(cbs3d_ctx* ctx, int nsteps, const double* w, const double* df, double* J, double* dJ);
/* J and grad[3*npoin] = dJ/df: forward with (u, p) checkpoints every `every`
 * steps, then the reverse sweep recomputing one segment at a time. */
cbs3d_status cbs3d_adjoint_run(cbs3d_ctx* ctx, int nsteps, int every, const double* w, double* J, double* grad);

/* Per-face heat flux (BC 532 faces in the order of the boundary-face list,
 * present when the case has heat_flux_bc != 0) and its sensitivities: the
 * objective is J = sum_i w[i] T_i after nsteps steps.  The temperature does
 * not act on the flow, so J is linear in the fluxes and these runs need no
 * fixed time step.  q = NULL restores the uniform heat_flux_bc. */
cbs3d_status cbs3d_heat_flux_face_count(cbs3d_ctx* ctx, int* nfaces);
cbs3d_status cbs3d_set_face_heat_flux(cbs3d_ctx* ctx, const double* q);
cbs3d_status cbs3d_heat_objective_run(cbs3d_ctx* ctx, int nsteps, const double* w, double* J);
cbs3d_status cbs3d_heat_tlm_run(cbs3d_ctx* ctx, int nsteps, const double* w, const double* dq, double* J, double* dJ);
/* grad[nfaces] = dJ/dq_f, checkpoints every `every` steps. */
cbs3d_status cbs3d_heat_adjoint_run(cbs3d_ctx* ctx, int nsteps, int every, const double* w, double* J, double* grad);

/* ---------------------------------------------------------------------------
 * Batched step (no reference counterpart; each instance is the reference's
 * single-case step): many independent cases of any sizes advanced together.
 * Per step, every instance's stages run on its own stream (graph branches);
 * all pressure systems are solved by one cooperative launch per wave of
 * instances, each instance with its own reductions, stopping test, status
 * and result.  The whole step is one CUDA graph when use_graph is set.
 * --------------------------------------------------------------------------- */
typedef struct cbs3d_batch cbs3d_batch;

typedef struct cbs3d_batch_options {
    cbs3d_options base;      /* precision, device, inner_tol, use_graph (pcg_kernel/pcg_blocks unused) */
    int autotune;            /* 1: on the first step time every feasible PCG tiling on the real
                                systems and keep the fastest */
    int rows_per_thread;     /* tiling without autotune: 1, 2, 4 or 8 slices of 32 rows per warp
                                (0: 4) */
    int spread;              /* 1: a wave's spare CTAs are shared out by instance size; 0: each
                                instance gets the fewest CTAs that hold its rows */
} cbs3d_batch_options;

typedef struct cbs3d_batch_info {
    int instances;
    int waves;               /* cooperative PCG launches per step */
    int rows_per_thread;     /* tiling in use */
    int spread;
    int mixed_waves;         /* 1 when a wave runs the mixed-precision kernel */
    int tuned;               /* 1 after the autotuner ran */
    int candidates;          /* tilings the autotuner timed */
    int cand_rows[8], cand_spread[8];
    double cand_ms[8];       /* one batched pressure solve per candidate, ms (-1: did not fit) */
} cbs3d_batch_info;

void cbs3d_default_batch_options(cbs3d_batch_options* opt);
/* n instances, each a mesh and parameter set as for cbs3d_create; all on opt->base.device. */
cbs3d_status cbs3d_batch_create(int n, const cbs3d_mesh* meshes, const cbs3d_params* params,
                                const cbs3d_batch_options* opt, cbs3d_batch** out, char* err, size_t errlen);
/* nsteps steps of every instance.  stats: n entries (or NULL), each as
 * cbs3d_step returns it for that instance; *gpu_seconds (or NULL): device
 * time of the whole call (after the autotuned first step, when the
 * autotuner runs in this call).  A failing instance stops the call after the step
 * in which it failed; its status and message are returned. */
cbs3d_status cbs3d_batch_step(cbs3d_batch* b, int nsteps, cbs3d_step_stats* stats, double* gpu_seconds);
cbs3d_status cbs3d_batch_download_fields(cbs3d_batch* b, int instance, double* u, double* p, double* t);
cbs3d_status cbs3d_batch_get_info(const cbs3d_batch* b, cbs3d_batch_info* info);
void cbs3d_batch_destroy(cbs3d_batch* b);
const char* cbs3d_batch_last_error(const cbs3d_batch* b);

/* Failure-detection self-test (no reference counterpart): launches a small
 * grid whose grid barrier can never complete and returns, in
 * *observed_status, the status its bounded device waits recorded --
 * CBS3D_TIMEOUT after about a second.  The device stays usable. */
cbs3d_status cbs3d_selftest_wait_timeout(int device, int* observed_status);

/* Dense inverse of a g x g row-major matrix by the device Gauss-Jordan
 * kernels that invert the two-level preconditioner's aggregated operator
 * (no reference counterpart; the coarse space is an extension).  variant 0:
 * the register-tiled kernel (g <= 160, the one solves use); 1: the
 * shared-memory kernel (g <= 164).  No pivoting: meant for SPD matrices; a
 * zero diagonal entry is replaced by 1 first, as for an empty aggregate.
 * a and ainv are host arrays of g*g doubles. */
cbs3d_status cbs3d_coarse_inverse(int device, int g, const double* a, double* ainv, int variant);

/* Measurement probes (no reference counterpart) that the benchmark uses to
 * state the solver kernels' rooflines.  cbs3d_probe_bandwidth: GB/s of
 * `passes` passes over a device buffer of `bytes` inside one launch (after a
 * one-pass warm-up launch), mode 0 reading it, mode 1 copying it to a second
 * buffer (read + write bytes counted); a buffer that fits in L2 gives the L2
 * bandwidth, a larger one the HBM bandwidth.  Back-to-back launches cost
 * about 4 us each on B200, so the passes run inside one launch.
 * cbs3d_probe_allreduce: microseconds per grid-wide all-reduce
 * of the persistent PCG kernel's kind (one 512-thread CTA per SM, five
 * values, `iters` dependent all-reduces in one cooperative launch) -- the
 * per-iteration latency floor of the single-reduction PCG.  Both allocate
 * and free their own device memory. */
cbs3d_status cbs3d_probe_bandwidth(int device, long long bytes, int passes, int mode, double* gbs);
cbs3d_status cbs3d_probe_allreduce(int device, int iters, double* us_per_allreduce);

/* Halo placement probe (no reference counterpart; host only, touches no
 * device).  For one CTA's SELL-32 slices -- slice q holds slice_w[q] slots
 * per row at slice_off[q] (nslices+1 offsets, slice_off[0] = 0 and
 * slice_off[q+1] = slice_off[q] + 32*slice_w[q]; slot u of lane l at
 * slice_off[q] + 32*u + l), lc giving each slot's halo entry 0..nh-1 in
 * column order -- returns in pos[nh] the shared-memory position the PCG
 * engine gives each halo entry (a permutation within every aligned block of
 * 32 positions, spreading the warps' gathers over the bank pairs), and in
 * wavefronts[0..1] the gathers' shared-memory wavefronts under a half-warp
 * bank-pair model with the entries in column order and as placed. */
cbs3d_status cbs3d_probe_halo_placement(int nh, int nslices, const long long* slice_off, const int* slice_w,
                                        const unsigned short* lc, int* pos, long long* wavefronts);

#ifdef __cplusplus
}
#endif
#endif
