// Asynchronous VTU snapshots (see snapshot.cuh).
#include "snapshot.cuh"

#include "post.h"

#include <exception>
#include <stdexcept>

namespace cbs3d {

namespace {
void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw Error(CBS3D_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

VtuSnapshots::VtuSnapshots(int device, const HostModel& m, size_t n) : device_(device), m_(m), n_(n)
{
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    try {
        cuda_check(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking), "snapshot stream");
        for (Slot& s : slot_) {
            cuda_check(cudaMalloc(&s.dev, 6 * n_ * sizeof(double)), "snapshot device buffer");
            cuda_check(cudaMallocHost(&s.host, 6 * n_ * sizeof(double)), "snapshot pinned buffer");
            cuda_check(cudaEventCreateWithFlags(&s.taken, cudaEventDisableTiming), "snapshot event");
            cuda_check(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming), "snapshot event");
        }
    } catch (...) {
        for (Slot& s : slot_) {
            if (s.dev) cudaFree(s.dev);
            if (s.host) cudaFreeHost(s.host);
            if (s.taken) cudaEventDestroy(s.taken);
            if (s.copied) cudaEventDestroy(s.copied);
        }
        if (side_) cudaStreamDestroy(side_);
        throw;
    }
    worker_ = std::thread([this] { run(); });
}

VtuSnapshots::~VtuSnapshots()
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    worker_.join();
    for (Slot& s : slot_) {
        cudaFree(s.dev);
        cudaFreeHost(s.host);
        cudaEventDestroy(s.taken);
        cudaEventDestroy(s.copied);
    }
    cudaStreamDestroy(side_);
}

void VtuSnapshots::enqueue(cudaStream_t st, const double* u, const double* p, const double* t, const double* vmag,
                           const std::string& path)
{
    int k = -1;
    {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !slot_[0].busy || !slot_[1].busy; });
        k = slot_[0].busy ? 1 : 0;
        slot_[k].busy = true;
    }
    Slot& s = slot_[k];
    try {
        const size_t n = n_;
        cuda_check(cudaMemcpyAsync(s.dev, u, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, st), "snapshot copy");
        cuda_check(cudaMemcpyAsync(s.dev + 3 * n, p, n * sizeof(double), cudaMemcpyDeviceToDevice, st), "snapshot copy");
        cuda_check(cudaMemcpyAsync(s.dev + 4 * n, t, n * sizeof(double), cudaMemcpyDeviceToDevice, st), "snapshot copy");
        if (vmag)
            cuda_check(cudaMemcpyAsync(s.dev + 5 * n, vmag, n * sizeof(double), cudaMemcpyDeviceToDevice, st),
                       "snapshot copy");
        cuda_check(cudaEventRecord(s.taken, st), "snapshot event");
        cuda_check(cudaStreamWaitEvent(side_, s.taken, 0), "snapshot wait");
        cuda_check(cudaMemcpyAsync(s.host, s.dev, (vmag ? 6 : 5) * n * sizeof(double), cudaMemcpyDeviceToHost, side_),
                   "snapshot copy-out");
        cuda_check(cudaEventRecord(s.copied, side_), "snapshot event");
    } catch (...) {
        std::lock_guard<std::mutex> lk(mu_);
        s.busy = false;
        cv_.notify_all();
        throw;
    }
    {
        std::lock_guard<std::mutex> lk(mu_);
        s.path = path;
        s.has_v = vmag != nullptr;
        queue_.push_back(k);
        ++pending_;
    }
    cv_.notify_all();
}

std::string VtuSnapshots::flush()
{
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return pending_ == 0; });
    std::string e;
    e.swap(err_);
    return e;
}

void VtuSnapshots::run()
{
    cudaSetDevice(device_);
    for (;;) {
        int k = -1;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
            if (queue_.empty()) return;   // stop requested and nothing left
            k = queue_.front();
            queue_.pop_front();
        }
        Slot& s = slot_[k];
        std::string e;
        try {
            cuda_check(cudaEventSynchronize(s.copied), "snapshot copy-out");
            const double* h = s.host;
            write_vtu(s.path, m_, h, h + 3 * n_, h + 4 * n_, s.has_v ? h + 5 * n_ : nullptr);
        } catch (const std::exception& x) {
            e = std::string("writeVTU ") + s.path + ": " + x.what();
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (!e.empty() && err_.empty()) err_ = e;
            s.busy = false;
            --pending_;
        }
        cv_.notify_all();
    }
}

}  // namespace cbs3d
