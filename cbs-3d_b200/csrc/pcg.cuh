// Pressure PCG engine: the element-by-element pressure operator assembled per
// step into a SELL-32 row layout, and a persistent cooperative Jacobi-PCG
// kernel that runs a whole solve in one launch.
#pragma once

#include "dev_state.cuh"
#include "host_model.h"

#include <cuda_runtime.h>
#include <string>
#include <vector>

namespace cbs3d {

// One instance of a batched solve: CTAs [cta0, cta0+ncta) of the launch own
// slices [s0, s1); its own scalars, barrier counter, partials, status, result.
struct PcgInst {
    int cta0, ncta, s0, s1;
    int precond, conv_test, max_iter, pad;
    double rel_tol, abs_tol;
    unsigned* bar;               // 64-bit arrival counter (zeroed before each launch)
    double* part;                // 2 * ncta * 8 partials (double-buffered by phase)
    DevStatus* status;
    CgOut* out;
};

struct PcgDev {
    int N;                       // row positions (nslices*32); the solver's vectors use this order
    int NN;                      // nodes (the caller's arrays)
    int E, nslices;
    int nblocks;
    int precond, conv_test, max_iter;
    double rel_tol, abs_tol, inner_tol;
    const int* row_node;         // nslices*32: node of each row position (-1 padding)
    const long long* slice_off;
    const int* slice_w;
    const int* col;
    double* val;
    float* val32;
    const long long* cptr;
    const int* cent;
    const uint8_t* nflag;        // bit0 pressure-active (touches fluid), bit2 fixed (position order in kernels)
    const double* pfix;
    double *pres, *rhs1, *pdiag;
    double *r, *z, *pA, *pB, *q;
    float *r32, *w32, *s32;      // mixed: 2N each (parity buffers)
    float *p32, *dz32;           // mixed: N each
    int slot_max;                // largest CTA slot range (shared-memory sizing)
    const int* halo_ptr;         // nblocks+1: each CTA's halo node list in halo_idx
    const int* halo_idx;
    const unsigned short* lcol;  // per slot: column as an index into its CTA's halo
    int halo_max;                // largest halo (shared-memory sizing)
    double* part;                // 2 * nblocks * 8 partials (double-buffered by phase)
    unsigned* bar;               // 64-bit arrival counter
    DevStatus* status;
    CgOut* out;
    const int* cta_inst;         // batched launch: instance of each CTA (else null)
    const PcgInst* inst;         // batched launch: instance descriptors (else null)
    int xs_off;                  // CG-CG kernel: byte offset in shared memory of its rows' pressure
                                 // and diagonal (2*RMAX*threads doubles); 0: read from global memory
    int halo_parts;              // global-vector kernel with a shared-memory halo: parts per CTA, each
                                 // with its own halo (halo_ptr indexed by CTA*parts + part)
    int coef_off;                // CG-CG kernel with its warps' first rows' coefficients in shared
                                 // memory: byte offset of that copy
    int pds_off;                 // one-CTA-per-SM CG-CG kernel: byte offset in shared memory of its
                                 // rows' diagonal (RMAX*threads doubles); 0: read from global memory
    int tm_w;                    // CG-CG kernel with rows in tensor memory: slots per row there (the
                                 // widest slice, rounded up to the kernel's load width)
};

class MgHierarchy;

// Two-level preconditioner data of one launch: the coarse space is one
// aggregate per CTA (its free rows); ainv is the inverse of the aggregated
// operator P^T A P, nbr_ptr/nbr_ids each CTA's own and halo-owner CTAs, and
// hown the position of every halo entry's owner in its CTA's list.
struct CoarseDev {
    int G;
    int nbr_max;
    const int* nbr_ptr;
    const int* nbr_ids;
    const unsigned char* hown;
    const double* ainv;
};

// Owns the device copies of the pattern and the PCG work vectors.
class PcgEngine {
public:
    // kernel_choice: 0 automatic (4, else 3, else 2, else 5), 1 vectors in global memory,
    // 2 register-resident rows, 3 with the halo staged in shared memory,
    // 4 as 3 with one grid synchronisation per iteration (Chronopoulos-Gear),
    // 5 vectors in global memory with one grid synchronisation per iteration
    // two_level: Jacobi plus a coarse correction on one aggregate per CTA
    // (large meshes with the single-reduction kernel; else plain Jacobi)
    // multigrid: the aggregation-multigrid preconditioned CG (mg.cuh) for
    // Jacobi-preconditioned FP64 solves, where the mesh fits it
    void init(const HostModel& m, const uint8_t* d_nflag, const double* d_pfix, DevStatus* d_status,
              int device, int blocks_override, bool mixed, int kernel_choice = 0, bool two_level = false,
              bool multigrid = false);
    void release();
    // ELL values from gstifE*delte (step path) or from a caller's gstif[6E].
    void assemble_from_state(const DevState& S, cudaStream_t st);
    // Two-level set-up of the next solve (aggregated operator and its
    // inverse) from the assembled operator and the node-ordered diagonal,
    // on `st`; that solve then skips its own set-up.  No-op without coarse.
    void prepare_coarse(const double* d_pdiag_node, cudaStream_t st);
    void assemble_from_gstif(const double* d_gstif, cudaStream_t st);
    // Runs one solve on pres/rhs1/pdiag (device pointers), result to host.
    // ev0/ev1 (optional) are recorded around the persistent PCG launch.
    cbs3d_status solve(double* d_pres, double* d_rhs1, double* d_pdiag, int precond, int conv_test,
                       int max_iter, double rel_tol, double abs_tol, cudaStream_t st, bool sync,
                       cudaEvent_t ev0 = nullptr, cudaEvent_t ev1 = nullptr);
    // impose, permute in, solver, permute out (+ the preconditioner's set-up)
    int launches_per_solve() const;
    cbs3d_status read_result(cbs3d_cg_result& r, cudaStream_t st);
    // y = A x with the assembled operator (identity rows on fixed nodes).
    void multiply(const double* d_pdiag, const double* d_x, double* d_y, cudaStream_t st);

    bool mixed = false;
    MgHierarchy* mgh = nullptr;  // multigrid in use (else null)
    bool mg_ready = false;       // prepare_coarse set the multigrid up for the next solve
    int rmax = 0;            // rows per thread of the register-resident kernels (0: global kernel)
    int nthreads = 512;      // CTA size of the persistent kernel
    bool coarse = false;     // two-level preconditioner in use
    bool coarse_ready = false;   // prepare_coarse ran for the next solve
    size_t coarse_smem = 0, coarse_ismem = 0;
    int npairs = 0, sms_ = 0;
    int *d_pair_ptr = nullptr, *d_pair_ent = nullptr, *d_nbr_ptr = nullptr, *d_nbr_ids = nullptr;
    int2* d_pair_ij = nullptr;
    double* d_ac = nullptr;
    unsigned char* d_hown = nullptr;
    CoarseDev cdev{};
    std::vector<int> h_hptr, h_hidx;
    void build_coarse(const HostModel& m, const std::vector<int>& colp);
    void coarse_setup(const double* pdiag, const int* row_node, cudaStream_t st);
    int variant = 1;         // 1 global vectors, 2 register rows, 3 + shared-memory halo, 4 + one sync per iteration
    bool global_halo = false;     // variant 1 with its neighbour values staged in shared memory
    bool global_cgcg = false;     // ... run by the single-reduction kernel k_pcg64g
    size_t global_halo_smem = 0;
    long long global_halo_total = 0;   // halo entries over all CTAs
    int global_halo_parts = 1;         // parts per CTA, each with its own halo
    size_t halo_smem = 0;    // dynamic shared memory of the halo kernel
    size_t cgcg_smem = 0;    // ... of the CG-CG kernel (halo + its rows' pressure and diagonal)
    int cgcg_xs_off = 0;     // where those rows start (0: kept in global memory)
    int cgcg_ks = 0;         // 1: the kernel reads its warps' first rows' coefficients from shared memory
    int cgcg_coef_off = 0;   // where they start
    int cgcg_kt = 0;         // >0: that many rows per thread, after the shared-memory one, read from tensor memory
    int cgcg_tm_w = 0;       // slots per row in tensor memory
    int cgcg_pds_off = 0;    // where the rows' diagonal starts in shared memory (0: global memory)
    size_t mixed_smem = 0;   // dynamic shared memory of the mixed-precision kernel
    bool mixed_ok = false;   // mixed precision runs on the FP32 kernel (else FP64)
    int dev_slot_max = 0;
    int *d_halo_ptr = nullptr, *d_halo_idx = nullptr;
    unsigned short* d_lcol = nullptr;
    int* d_row_node = nullptr;
    double *d_xp = nullptr, *d_bp = nullptr, *d_dp = nullptr;   // pressure, rhs, diagonal by position
    uint8_t* d_fp = nullptr;
    int dev_halo_max = 0;
    double inner_tol = 0.05;      // mixed: residual-replacement factor
    int N = 0, NP = 0, E = 0, nslices = 0, nblocks = 0;
    long long nslots = 0, ncontrib = 0;
    long long *d_slice_off = nullptr, *d_cptr = nullptr;
    int *d_slice_w = nullptr, *d_col = nullptr, *d_cent = nullptr;
    double* d_val = nullptr;
    float* d_val32 = nullptr;
    double *d_r = nullptr, *d_z = nullptr, *d_pA = nullptr, *d_pB = nullptr, *d_q = nullptr;
    float *d_f32 = nullptr;
    double* d_part = nullptr;
    unsigned* d_bar = nullptr;
    CgOut* d_out = nullptr;
    const uint8_t* d_nflag = nullptr;
    const double* d_pfix = nullptr;
    DevStatus* d_status = nullptr;
    PcgDev dev{};
    // Algorithmic bytes of one PCG iteration of the implemented kernel: the
    // real (unpadded) pair coefficients and columns plus the per-node vector
    // traffic of the two phases.
    size_t bytes_per_iter() const;
    long long nnz_offdiag = 0;
};

// ----------------------------------------------------------- batched solves
// Many independent pressure systems (one per instance of a batch) solved by
// the same persistent kernels: instances are packed into waves, each wave is
// one cooperative launch in which every instance owns its own CTAs, halo,
// reductions, barrier, status and result.
struct PcgBatchMember {
    const HostModel* m;
    const uint8_t* d_nflag;      // the instance's node flags, node order
    const double* d_pfix;        // fixed-pressure values, node order
    DevStatus* d_status;         // the instance's status word
};

// A tiling of the batch: rows per thread (1, 2, 4 or 8 slices of 32 rows per
// warp) and whether the spare CTAs of a wave are shared out by instance size.
struct PcgBatchPlan {
    int rmax = 4;
    int spread = 1;
};

class PcgBatch {
public:
    void init(const std::vector<PcgBatchMember>& members, int device, bool mixed, double inner_tol);
    // Builds the waves of a plan; false (with the reason) when it cannot fit.
    bool plan(const PcgBatchPlan& p, std::string* why);
    void release();
    // Instance k, on its own stream: operator values from its state,
    // constraints, and its inputs moved to row-position order.
    void prepare(int k, const DevState& S, cudaStream_t st);
    // Every wave, in order, on one stream.
    void solve(cudaStream_t st);
    // Instance k: the pressure back to node order.
    void finish(int k, double* d_pres, cudaStream_t st);
    CgOut* out(int k) const { return d_out + k; }
    int nwaves() const { return static_cast<int>(waves.size()); }
    // launches per step: assemble, impose, permute in and out per instance; one per wave
    int launches_per_instance() const { return 4; }
    PcgBatchPlan current{};
    bool mixed_any = false;      // some wave runs the mixed-precision kernel

private:
    struct Wave {
        int G = 0, rmax = 4;
        bool mixed = false;
        size_t smem = 0;
        const void* fn = nullptr;
        PcgDev dev{};
        int* d_cta_inst = nullptr;
        PcgInst* d_inst = nullptr;
        int *d_hptr = nullptr, *d_hidx = nullptr;
    };
    void free_waves();
    std::vector<PcgBatchMember> mem;
    std::vector<int> slice0, nsl, N_k;
    std::vector<long long> slot0, nslot;
    std::vector<long long*> d_cptr;
    std::vector<int*> d_cent;
    std::vector<Wave> waves;
    int device = 0, sms = 0, gmax = 0;
    bool mixed = false;
    int nslices = 0, NP = 0;
    long long nslots = 0;
    std::vector<long long> h_slice_off;
    std::vector<int> h_col;
    long long* d_slice_off = nullptr;
    int *d_slice_w = nullptr, *d_col = nullptr, *d_row_node = nullptr;
    unsigned short* d_lcol = nullptr;
    double* d_val = nullptr;
    float* d_val32 = nullptr;
    double *d_r = nullptr, *d_z = nullptr, *d_pA = nullptr, *d_pB = nullptr, *d_q = nullptr;
    double *d_xp = nullptr, *d_bp = nullptr, *d_dp = nullptr;
    uint8_t* d_fp = nullptr;
    float* d_f32 = nullptr;
    double* d_part = nullptr;
    unsigned* d_bar = nullptr;
    CgOut* d_out = nullptr;
    PcgDev base{};
};

// Microseconds per grid all-reduce of the single-reduction kernel (one
// 512-thread CTA per SM, `iters` back-to-back all-reduces, CUDA events).
cbs3d_status allreduce_probe(int device, int iters, double* us);

// Launches a grid whose barrier can never complete and reports the status
// the bounded waits recorded (CBS3D_TIMEOUT when they ran out as designed).
cbs3d_status selftest_wait_timeout(int device, int* observed);

// Inverts a g x g host matrix with the coarse-operator Gauss-Jordan kernels
// (variant 0: registers, g <= 160; 1: shared memory, g <= 164).
cbs3d_status coarse_inverse(int device, int g, const double* a, double* ainv, int variant);

}  // namespace cbs3d
