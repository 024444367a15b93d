// Launch declarations of the per-step kernels (kernels_step.cu).
#pragma once

#include "dev_state.cuh"

namespace cbs3d {

__global__ void k_geometry(DevState S);
__global__ void k_mass(DevState S);
__global__ void k_nodal_length(DevState S);
__global__ void k_mass_fluid(DevState S, double* mfluid);
__global__ void k_begin_step(DevState S);
__global__ void k_timestep(DevState S, int fixed_dt);
__global__ void k_dt_finish(DevState S, int fixed_dt);
__global__ void k_dt_force(DevState S);
__global__ void k_dt_correction(DevState S);
__global__ void k_lhs(DevState S);
__global__ void k_step1_elem(DevState S);
__global__ void k_step1_node(DevState S);
__global__ void k_step2_elem(DevState S);
__global__ void k_step2_node(DevState S);
__global__ void k_step3_elem(DevState S);
__global__ void k_step3_node(DevState S);
__global__ void k_step4_elem(DevState S);
__global__ void k_step4_node(DevState S);
__global__ void k_conv_partial(DevState S, const CgOut* cg, double* log, int* counter, int cap);
__global__ void k_gstif(DevState S, double* out);
__global__ void k_matvec_color(DevState S, const int* color_elem, int beg, int end, const double* gst,
                               const double* x, double* y);
__global__ void k_matvec_diag(DevState S, const double* x, double* y);

}  // namespace cbs3d
