// Device-side layout of one CBS3D case in HBM and the shared device helpers.
//
// Element arrays are structure-of-arrays over the element index e (0-based)
// so that a warp of consecutive elements reads each component coalesced:
//   grad[(dim*4 + a)*E + e]    dN_a/dx_dim           (reference dNkdx)
//   annxf[(f*4 + c)*E + e]     face f area normal c  (reference annxf(c,f,e))
//   pdiagE[a*E + e], gstifE[g*E + e]
// Node arrays are indexed by the 0-based node; vectors of 3 are node-major
// (u,v,w of a node adjacent), matching the reference's unkno(3,N).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cbs3d {

// Device status word.  The first failure wins (atomicCAS on code); `where`
// is the 1-based element/node index of the failure and `stage` the stage id.
struct DevStatus {
    int code;      // cbs3d_status
    int stage;
    int where;
    int reason;    // stage-specific reason id (maps to a reference message)
    int step;      // step counter value when the failure was first seen (0 = not yet)
};

// Result of one pressure solve, written by the PCG kernels.
struct CgOut {
    int iterations;
    int converged;
    int outer;
    int pad;
    double initial_l2, final_l2, rel, max_abs;
};

// doubles per step in the step log: dtreal, cg[6], hb[15], rtime, outer
constexpr int LOG_FIELDS = 24;

enum Stage {
    ST_GEOM = 1, ST_MASS, ST_TIMESTEP, ST_LHS, ST_STEP1, ST_STEP2RHS, ST_PCG, ST_STEP3, ST_STEP4,
    ST_CONV, ST_DTCORR
};

// reasons
enum Reason {
    R_DETJ = 1, R_FACE_AREA, R_HMIN, R_MASS, R_CAPACITY, R_RHOCP,
    R_DT_LOCAL, R_DT_MIN, R_DIFF, R_ALPHA, R_RHOMU,
    R_LHS_DT, R_LHS_ELCOE2, R_LHS_ELCOE2P, R_LHS_PDIAG, R_ORPHAN,
    R_PCG_DIAG, R_PCG_RZ0, R_PCG_PAP, R_PCG_RZ, R_PCG_RESID, R_PCG_MAXIT, R_PCG_BARRIER,
    R_STEP1_DETJ, R_K, R_QVOL, R_EN_DT
};

struct DevParams {
    int E, N, NB;
    int temp_calc, htype, ilots, transient_on, solver_opt, dtfixed, dtfix_end;
    int dimensional_material;      // dimensional_mode>0 && material_properties_enabled>0
    double ani, csafm, deltr, dtfix, csafm2, epsilon1;
};

struct DevState {
    DevParams P;
    // mesh
    const int4* intma;          // 0-based node ids
    const uint8_t* mat;         // 1 = solid (mat_elem != 0)
    const uint8_t* fedge;       // packed: bits 2f..2f+1 = fedge of face f
    const double* coord;        // 3N
    const double *rho, *mu, *kc, *rho_cp, *alpha, *qvol;   // E (material mode)
    // geometry (written once by the geometry kernel)
    double *detJ, *grad, *annxf, *alen_e, *pdiagE, *gstifE, *alen;
    // incidence
    const int *n2e_ptr, *n2e, *n2c_ptr, *n2c;
    // node flags: bit0 touches fluid, bit1 touches solid, bit2 fixed pressure
    const uint8_t* nflag;
    const double* pfix;         // N fixed pressure value
    // boundary programs
    const int* vbc_idx;
    const void* vbc;            // VelBC records
    const double* vbc_nrm;
    const int* tbc_flag;
    const double* tbc_val;
    const int* hf_ptr;
    const double* hf_val;
    // fields
    double *unkno, *unkn1, *pres, *pres1, *temp, *temp1, *velocity;
    double *rhs, *rhs1, *delte, *elcoe2, *elcoe2p, *pdiag, *mdiag_real;
    // body force (extension, no reference counterpart): f[3N] node-major and
    // the fluid lumped mass mfluid[N]; Step 1 adds mfluid*f to the momentum
    // residual.  Both null when no body force is set.
    const double* bforce;
    const double* mfluid;
    // element-local scratch (16E doubles, reused by every assembly stage):
    // Step 1 writes node-major 32-byte records [(4e + a)*4 + d] (d < 3, one
    // pad), the other stages structure-of-arrays [(d*4 + a)*E + e]
    double* elbuf;
    // scalars
    double* dscal;              // [0] dtreal (as double), [1] rtime, [2..16] hb
    unsigned long long* dtmin_bits;
    unsigned* conv_count;       // k_conv_partial blocks done (the last one resets it)
    DevStatus* status;
    double* red;                // reduction partials
};

// ------------------------------------------------------------- helpers
__device__ __forceinline__ void set_status(DevStatus* st, int code, int stage, int where, int reason)
{
    if (atomicCAS(&st->code, 0, code) == 0) {
        st->stage = stage;
        st->where = where;
        st->reason = reason;
    }
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_int(const int* p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier for a cooperatively launched grid.  Every wait is
// bounded: after ~2^31 SM cycles (about a second) the CTA records
// CBS3D_TIMEOUT in the status word and returns false; a CTA that sees any
// failure recorded by another CTA also returns false, so the whole grid
// leaves the kernel.  count/gen live in device memory zeroed before launch.
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks,
                                             DevStatus* st, int stage)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned g = ld_acquire(gen);
        __threadfence();
        const unsigned arrived = atomicAdd(count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            const long long t0 = clock64();
            while (ld_acquire(gen) == g) {
                if (ld_relaxed_int(&st->code) != 0) { ok = 0; break; }
                if (clock64() - t0 > (1LL << 31)) {
                    set_status(st, 5 /*CBS3D_TIMEOUT*/, stage, 0, R_PCG_BARRIER);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        if (ok && ld_relaxed_int(&st->code) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace cbs3d
