// The per-case device context behind the C ABI: host model, stream, device
// state, PCG engine and step log.  Shared by the C-ABI file (capi.cu) and the
// tangent-linear/adjoint driver (adjoint.cu).
#pragma once

#include "cbs3d_gpu.h"
#include "host_model.h"
#include "kernels.cuh"
#include "pcg.cuh"
#include "snapshot.cuh"

#include <memory>
#include <string>
#include <vector>

#ifndef CUDA_OK
#define CUDA_OK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) throw cbs3d::Error(CBS3D_CUDA_ERROR, std::string(#x) + ": " + cudaGetErrorString(e_)); } while (0)
#endif

namespace cbs3d {

constexpr int T = 256;

inline unsigned nb(long long n, int t = T) { return static_cast<unsigned>((n + t - 1) / t); }

struct DeviceBuffers {
    std::vector<void*> ptrs;
    template <typename Tp>
    Tp* alloc(size_t n)
    {
        void* p = nullptr;
        CUDA_OK(cudaMalloc(&p, (n ? n : 1) * sizeof(Tp)));
        ptrs.push_back(p);
        return static_cast<Tp*>(p);
    }
    template <typename Tp>
    Tp* upload(const std::vector<Tp>& v)
    {
        Tp* p = alloc<Tp>(v.size());
        if (!v.empty()) CUDA_OK(cudaMemcpy(p, v.data(), v.size() * sizeof(Tp), cudaMemcpyHostToDevice));
        return p;
    }
    void release()
    {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
    }
};

// Message of a device status, worded like the reference's exceptions.
std::string reason_text(const DevStatus& s);

}  // namespace cbs3d

using namespace cbs3d;

struct cbs3d_ctx {
    HostModel m;
    cbs3d_options opt{};
    cudaStream_t st = nullptr;
    DevState S{};
    DeviceBuffers buf;
    int* d_color_elem = nullptr;
    double* d_log = nullptr;
    int* d_counter = nullptr;
    int log_cap = 0;
    int conv_blocks = 0;
    PcgEngine pcg;
    int iitime = 0;
    long long cg_total = 0;
    std::string err;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // operator assembly (and two-level set-up) of the pressure solve, forked
    // onto `side` after the last LHS update so that it overlaps Steps 1-2
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_lhs = nullptr;      // the LHS on `side`, waited for by the Step-1 node gather
    bool own_engine = false, assembly_forked = false;
    cudaGraphExec_t gexec = nullptr;
    bool graph_failed = false;
    std::vector<cudaEvent_t> pcg_ev;   // 2 per step when timing PCG launches
    int pcg_ev_used = 0;
    long long launches = 0;            // kernels enqueued (counted at enqueue time)
    int step_kernels = 0;              // kernels per enqueued step
    CgOut* batch_out = nullptr;        // member of a batch: its pressure-solve result (no own PCG engine)
    int last_start = 0, last_done = 0; // step counter before, and steps of, the latest cbs3d_step call
    double* d_bforce = nullptr;        // body force f[3N] (extension), when set
    double* d_mfluid = nullptr;        // fluid lumped mass, for the body force

    std::unique_ptr<VtuSnapshots> snaps;   // asynchronous VTU writer, made on first use

    ~cbs3d_ctx()
    {
        snaps.reset();   // pending snapshots are written before the fields go away
        for (cudaEvent_t e : pcg_ev) cudaEventDestroy(e);
        if (gexec) cudaGraphExecDestroy(gexec);
        pcg.release();
        buf.release();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (ev_lhs) cudaEventDestroy(ev_lhs);
        if (side) cudaStreamDestroy(side);
        if (st) cudaStreamDestroy(st);
    }

    bool fixed_dt(int it) const
    {
        // TimeStep::computeTimeStep fixed branch (src/timestep/TimeStep.cpp:492-509)
        return m.p.ilots <= -1 || m.p.dtfixed > 0 || (m.p.dtfix_end > 0 && it <= m.p.dtfix_end);
    }
    bool force_global() const
    {
        // src/timestep/TimeStep.cpp:544-547
        return m.p.transient_on > 0 || m.p.solver_opt > 1 || m.p.dtfixed == -1 ||
               (m.p.ilots != 1 && m.p.ilots != 2);
    }

    void setup(bool own_pcg = true);
    void check_status();
    void reset_status() { CUDA_OK(cudaMemsetAsync(S.status, 0, sizeof(DevStatus), st)); }
    void stage_time_step(int it);
    void stage_solve();
    void fork_assembly();
    // Solver::advanceOneStep in two halves around the pressure solve
    void enqueue_pre(int it);
    void enqueue_post(int it);
    void enqueue_step(int it);
    // kernels of one step outside the pressure solve
    int kernels_outside_solve(int it) const;
    void ensure_log(int n);
};
