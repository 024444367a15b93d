// Host-side model of one CBS3D case: parsed inputs, the integer
// preprocessing the reference does serially (face numbering, face classes,
// wall and pressure lists, greedy colouring), and the index structures the
// device kernels consume (incidence lists in the reference's summation order,
// per-node boundary programs, the pressure-operator pattern).
#pragma once

#include "cbs3d_gpu.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace cbs3d {

// Error carrying a status code; the message mirrors the reference's
// std::runtime_error text for the same condition.
struct Error : std::runtime_error {
    cbs3d_status code;
    Error(cbs3d_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Per-node velocity boundary program.  Built from the face-ordered passes of
// Boundary::applySymmetry / applyVelocity / applyOutletBackflowControl and
// Steps.cpp enforce_zero_velocity_in_solid (reference src/boundary/Boundary.cpp:
// 275-310, 341-508, 672-723; src/solver/Steps.cpp:102-176).
struct VelBC {
    int flags;           // VBC_FIXED | VBC_SOLID
    int sym_beg, sym_cnt;
    int out_beg, out_cnt;
    int pad;
    double fix[3];
};
enum { VBC_FIXED = 1, VBC_SOLID = 2 };

// SELL-32 pattern of the assembled pressure operator's off-diagonal part.
// Row i collects every node that shares a fluid tetrahedron with i; each slot
// keeps its element-pair contributions in ascending element order.
struct PressurePattern {
    int nslices = 0;
    long long nslots = 0;
    std::vector<int> row_node;           // nslices*32: node of each row position (-1 padding)
    std::vector<long long> slice_off;    // nslices+1, slot offsets
    std::vector<int> slice_w;            // nslices, slots per row in the slice
    std::vector<int> col;                // nslots (0-based node)
    std::vector<long long> cptr;         // nslots+1
    std::vector<int> cent;               // contributions: e*8 + pair
    int max_row = 0;
};

struct HostModel {
    cbs3d_params p{};
    int E = 0, N = 0, NB = 0;
    std::vector<int> intma;        // 4E, 1-based
    std::vector<double> coord;     // 3N
    std::vector<int> iside;        // 6*NB: n1 n2 n3 local_face parent bc
    std::vector<int> mat;          // E
    std::vector<double> rho, cp, kc, mu, rho_cp, alpha, qvol;
    double ani = 0.0, inlet_u_mf = 0.0;
    int temp_calc = 0;

    std::vector<int> fedge;        // 4E
    std::vector<double> face_norm; // 4*NB (boundary faces, same arithmetic as getNormals)
    std::vector<char> tf, ts;      // node touches fluid / solid
    std::vector<int> wall_list;    // 1-based
    std::vector<int> bc_list;      // 1-based
    std::vector<double> bc_values;
    int ncolor = 0;
    std::vector<int> color_ptr, color_elem, color_of;

    // Incidence lists, slot = e*4 + a (0-based e, local node a).
    std::vector<int> n2e_ptr, n2e;   // every element, ascending element index
    std::vector<int> n2c_ptr, n2c;   // fluid elements, (colour, element) order

    std::vector<int> vbc_idx;        // N: -1 or index into vbc
    std::vector<VelBC> vbc;
    std::vector<double> vbc_nrm;     // 3 per symmetry/outlet normal
    std::vector<int> tbc_flag;       // N
    std::vector<double> tbc_val;     // N
    std::vector<int> hf_ptr;         // N+1
    std::vector<double> hf_val;      // heat-flux face contributions, face order
    // Heat-flux faces (BC 532, present when heat_flux_bc != 0), for per-face
    // flux control: each hf_val entry's face and area, and each face's nodes.
    std::vector<int> hf_face;        // per hf_val entry: face index 0..nqf-1
    std::vector<double> hf_area;     // per hf_val entry: face area
    std::vector<int> qf_nodes;       // 3 per face, 0-based
    std::vector<double> qf_area;     // per face: area

    PressurePattern pat;

    std::vector<double> unkno, pres, temp;   // initial fields after initial BCs

    void build();   // everything after the inputs are set
};

// Parses the case files with the grammar of MeshIO::readAll.
// Parses and builds; with use_cache the parsed inputs are taken from (or
// written to) <case>.cbscache when every source file's size and time match.
void read_case(const std::string& case_name, HostModel& m, bool use_cache = false, bool* from_cache = nullptr);
// The parse alone (the model's inputs; build() not run), and the same through
// the cache (returns true when the inputs came from it).
void parse_case(const std::string& case_name, HostModel& m);
bool parse_case_cached(const std::string& case_name, HostModel& m);
void read_params_only(const std::string& case_name, cbs3d_params& p, int& nelem, int& npoin,
                      int& nboun);
// Fills the model from in-memory arrays (raw ids already mapped).
void model_from_arrays(const cbs3d_mesh& mesh, const cbs3d_params& p, HostModel& m);

void default_params(cbs3d_params& p);

// Node -> (element, local node) incidence in element order; slot = e*4 + a.
void build_incidence(const std::vector<int>& intma, int N, std::vector<int>& ptr, std::vector<int>& idx);
// coord (3N, may be NULL) orders the rows along a Morton curve for locality.
void build_pressure_pattern(const std::vector<int>& intma, const std::vector<int>& mat, int N,
                            const std::vector<int>& n2e_ptr, const std::vector<int>& n2e,
                            PressurePattern& pat, const double* coord);

}  // namespace cbs3d
