// Aggregation multigrid preconditioner for the pressure PCG (extension; the
// reference's counterpart is the PETSc/HYPRE path of solver_opt=3,
// src/linalg/PetscPressureSolver.cpp:335-360).
//
// Hierarchy.  Level 0 is the assembled pressure operator in row-position
// (Morton) order.  Every further level aggregates 8 consecutive rows of the
// level below (an aggregate of the Morton order is a compact 2x2x2-like
// block of nodes); rows that are not free (padding, inactive, fixed pressure)
// belong to no aggregate.  Coarse operators are Galerkin products
// A_{l+1} = P^T A_l P with the piecewise-constant P, so each coarse entry is a
// sum of fine entries, added in a fixed order from index lists built once per
// mesh.  Aggregation stops at 160 rows or fewer, whose operator is inverted
// densely every solve.  The aggregates depend on the mesh alone, never on the
// grid size or the GPU.
//
// Preconditioner.  One symmetric V(1,1) cycle: damped Jacobi smoothing with
// per-row weights min(0.8, 1.8/g_i), g_i the Gershgorin ratio
// (|a_ii| + sum_j |a_ij|)/a_ii of the row (so the smoother converges on any
// mesh), and the coarse correction scaled by 1.5 (over-correction, which
// the piecewise-constant interpolation needs).  The outer iteration is the
// reference's preconditioned CG with its stopping tests and checks.
//
// Solver.  One persistent cooperative kernel per solve.  The grid is
// partitioned into chunks of four SELL slices (128 rows), every CTA owns a
// contiguous range of chunks, and dot products are summed per chunk in a
// fixed order and then over all chunks in a fixed order: results and
// iteration counts do not depend on the number of CTAs.
#pragma once

#include "pcg.cuh"

namespace cbs3d {

constexpr int MG_MAX_LEVELS = 8;
constexpr int MG_COARSE_MAX = 160;

// Slot of entry k of row I in a coarse level's off-diagonal arrays: rows in
// groups of 32, column-major within a group, so a warp reading entry k of 32
// consecutive rows makes one coalesced 256-byte (FP64) load.
__host__ __device__ __forceinline__ long long mg_slot(int I, int k, int W)
{
    return ((long long)(I >> 5) * W + k) * 32 + (I & 31);
}
// Off-diagonal slots of a level of n rows (the diagonal values follow them).
__host__ __device__ __forceinline__ long long mg_slots(int n, int W) { return (long long)((n + 31) >> 5) * 32 * W; }

// One coarse level l >= 1 on the device.  Rows of level l are the
// aggregates of level l-1: row I holds rows 8I..8I+7 of level l-1.
struct MgLevelDev {
    int n;                       // rows
    int W;                       // off-diagonal entries per row (padded)
    int tpr;                     // threads per row in the solver kernel (fixed per level)
    int sd, si;                  // offsets of the level's halo arrays in the kernel's shared memory
                                 // (doubles: r, weight, staged values; ints: halo rows)
    const int* col;              // mg_slots(n, W) columns (-1 padding), at mg_slot(I, k, W)
    double* val;                 // mg_slots(n, W) off-diagonal values, then n diagonal values
    double* wd;                  // n: smoother weight / diagonal (0 on rows without free children)
    double* rho;                 // n: residual after pre-smoothing
    double* x;                   // n: correction after post-smoothing
    const int* hptr;             // G+1: every CTA's halo list (own rows and their columns)
    const int* hidx;
    const int* hown;             // G: index of the CTA's first own row in its halo list
    const unsigned short* lcol;  // mg_slots(n, W): halo-local index of every column (0xffff padding)
    int hmax;                    // largest halo
};

struct MgDev {
    int Lc;                      // aggregation steps; level Lc is the dense coarsest level
    int nchunks;                 // 4-slice chunks of level 0
    int nc;                      // rows of the coarsest level
    int sd_xc;                   // shared-memory offset (doubles) of the coarsest level's r and x
    int si_end;                  // shared-memory offset (ints) where the level-0 slot columns start
    const MgLevelDev* lv;        // device array, levels 1..Lc-1 used
    const double* ainv;          // nc*nc inverse of the coarsest operator
    double* rho0;                // level-0 residual after pre-smoothing (row positions)
    double* wd0;                 // level-0 smoother weight / diagonal (0 off free rows)
    double* part;                // 2 * 4 * nchunks chunk partials (double-buffered by phase)
    unsigned long long* bar;     // monotonic arrival counter
};

// Host side: built once per mesh, set up (values) once per solve.
class MgHierarchy {
public:
    // False when the mesh does not fit the register-tiled kernel or the
    // shared memory (the reason in `why`; release() frees what was allocated).
    // d_nflag: the solver's node flags on the device (bit0 fluid-connected,
    // bit2 fixed pressure), which decide the free rows.
    bool build(const HostModel& m, const std::vector<int>& colp, const uint8_t* d_nflag,
               const long long* d_slice_off, const int* d_slice_w, const int* d_colp, int device, int sms,
               int blocks_override);
    void release();
    // Coarse values, smoother weights and the coarsest inverse from the
    // assembled level-0 operator (d_val, row-position slots) and the
    // diagonal: node-ordered with row_node, or row-position-ordered when
    // row_node is null.
    void setup(const double* d_val, const double* pdiag, const int* row_node, cudaStream_t st);
    // Launches the solver kernel (D: the engine's view with its inputs in
    // row-position order).
    void launch(const PcgDev& D, cudaStream_t st);
    int launches_per_setup() const { return 2 * Lc + 2; }

    int G = 0, rmax = 0, Lc = 0, nchunks = 0;
    size_t smem = 0;
    std::string why;             // why build() declined the mesh
    std::vector<int> n;          // rows per level
    std::vector<int> W;          // off-diagonal width per level (level 0: SELL, unused)
    long long nnz0 = 0;          // real off-diagonal entries of level 0
    MgDev dev{};
    std::vector<MgLevelDev> h_lv;
    PcgDev fine{};               // the level-0 halo of this partition (halo_ptr, halo_idx, lcol, halo_max, slot_max)

private:
    std::vector<void*> allocs;
    template <typename T> T* upload(const std::vector<T>& v);
    template <typename T> T* zeros(size_t count);
    // Galerkin index lists per level l+1: for every output (mg_slots(n, W)
    // off-diagonal slots, then n diagonal entries) the ordered source entries of level l
    // (>= 0: off-diagonal slot of level l; < 0: diagonal of row -(id+1)).
    std::vector<long long*> d_gptr;
    std::vector<int*> d_gent;
    std::vector<long long> gout;
    uint8_t* d_free0 = nullptr;
    const long long* d_slice_off = nullptr;
    const int* d_slice_w = nullptr;
    const int* d_colp = nullptr;
    double* d_dense = nullptr;
    int NP = 0, nslices = 0;
};

// Helpers defined in pcg.cu: the Gauss-Jordan inverse of a g x g matrix in
// place (g <= 160), and the grow-only dynamic shared-memory limit of a kernel.
void coarse_invert_launch(int g, double* a, cudaStream_t st);
cudaError_t pcg_raise_smem_limit(const void* fn, size_t smem);

}  // namespace cbs3d
