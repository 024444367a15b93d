// Run output on the host: the residual history CSV, VTU snapshots and the
// PVD collection, with the columns, array names and cell layout of the
// reference's Post (src/io/Post.cpp:525-560, 768-815, 887-1180).
#pragma once

#include "host_model.h"

#include <string>
#include <vector>

namespace cbs3d {

// Columns of one step record of the device step log.
constexpr int LOG_DT = 0, LOG_CG = 1, LOG_HB = 7, LOG_RTIME = 22, LOG_OUTER = 23, LOG_WIDTH = 24;

void write_residual_header(const std::string& path);
// Appends rows for iterations first_iter, first_iter+1, ... (n records of
// LOG_WIDTH doubles), keeping every `every`-th iteration as the reference does.
void append_residual_rows(const std::string& path, int first_iter, int every, const double* rec, int n);
// Binary-appended VTU of the mesh (tets and boundary triangles) and the
// fields; vmag may be null (then |u| + 1e-16 as Solver::updateVelocityMagnitude).
void write_vtu(const std::string& path, const HostModel& m, const double* u, const double* p, const double* t,
               const double* vmag);
void write_pvd(const std::string& path, const std::vector<std::string>& files, const std::vector<double>& times);

}  // namespace cbs3d
