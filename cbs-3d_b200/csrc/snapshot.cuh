// Asynchronous VTU snapshots of a context's fields (Post::writeVTU,
// reference src/io/Post.cpp:887-1180, moved off the step stream).
//
// enqueue() copies u, p, T and |u| device-to-device on the caller's stream
// (a few microseconds at 64^3) and returns.  A side stream then copies the
// snapshot to pinned host memory, and a host thread writes the file once
// that copy has completed, so later steps run while the file is written.
// Two slots: a third snapshot waits until the oldest one is on disk.
#pragma once

#include "host_model.h"

#include <condition_variable>
#include <cuda_runtime.h>
#include <deque>
#include <mutex>
#include <string>
#include <thread>

namespace cbs3d {

class VtuSnapshots {
public:
    // m must outlive this object; n is the node count.
    VtuSnapshots(int device, const HostModel& m, size_t n);
    ~VtuSnapshots();   // writes every pending snapshot first
    VtuSnapshots(const VtuSnapshots&) = delete;
    VtuSnapshots& operator=(const VtuSnapshots&) = delete;

    // Snapshot of u[3n], p[n], t[n] and, unless null, vmag[n] as they are
    // once the work already on `st` has run; written to `path` later.
    void enqueue(cudaStream_t st, const double* u, const double* p, const double* t, const double* vmag,
                 const std::string& path);
    // Waits until every enqueued snapshot is written; returns the first
    // error met since the previous flush ("" when none) and clears it.
    std::string flush();

private:
    static constexpr int SLOTS = 2;
    struct Slot {
        double* dev = nullptr;    // 6n doubles: u, p, t, vmag
        double* host = nullptr;   // pinned copy of dev
        cudaEvent_t taken = nullptr, copied = nullptr;
        std::string path;
        bool has_v = false, busy = false;
    };
    void run();

    int device_;
    const HostModel& m_;
    size_t n_;
    cudaStream_t side_ = nullptr;
    Slot slot_[SLOTS];
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<int> queue_;
    int pending_ = 0;
    bool stop_ = false;
    std::string err_;
    std::thread worker_;
};

}  // namespace cbs3d
