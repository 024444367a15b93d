// Case reader and host preprocessing.  See host_model.h.
#include "host_model.h"

#include <algorithm>
#include <array>
#include <cerrno>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <thread>
#include <unordered_map>

#include <sys/stat.h>

namespace cbs3d {

namespace {

[[noreturn]] void io_fail(const std::string& m) { throw Error(CBS3D_IO_ERROR, m); }
[[noreturn]] void bad(const std::string& m) { throw Error(CBS3D_INVALID_INPUT, m); }

// ------------------------------------------------------------------ lines
// read_data_line: trimmed, skipping blank lines and lines starting with # or !
// (reference src/io/MeshIO.cpp:23-64).
std::string trim(const std::string& s)
{
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

bool read_data_line(std::istream& in, std::string& out)
{
    std::string raw;
    while (std::getline(in, raw)) {
        raw = trim(raw);
        if (raw.empty() || raw[0] == '#' || raw[0] == '!') continue;
        out = raw;
        return true;
    }
    return false;
}

std::string next_data_line(std::istream& in, const std::string& file)
{
    std::string l;
    if (!read_data_line(in, l)) io_fail("Unexpected end of file: " + file);
    return l;
}

std::string slurp(const std::string& path, const std::string& who)
{
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) io_fail(who + " - cannot open file: " + path);
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::string buf(static_cast<size_t>(n), '\0');
    if (n > 0 && std::fread(&buf[0], 1, static_cast<size_t>(n), f) != static_cast<size_t>(n)) {
        std::fclose(f);
        io_fail(who + " - cannot read file: " + path);
    }
    std::fclose(f);
    return buf;
}

// Whitespace token scanner over a buffer with operator>> number semantics
// for well-formed input (strtol / correctly rounded strtod).
struct Scanner {
    const char* p;
    const char* end;
    bool next_int(int& v)
    {
        while (p < end && std::isspace(static_cast<unsigned char>(*p))) ++p;
        if (p >= end) return false;
        char* q = nullptr;
        errno = 0;
        const long x = std::strtol(p, &q, 10);
        if (q == p || errno) return false;
        p = q;
        v = static_cast<int>(x);
        return true;
    }
    bool next_double(double& v)
    {
        while (p < end && std::isspace(static_cast<unsigned char>(*p))) ++p;
        if (p >= end) return false;
        char* q = nullptr;
        v = std::strtod(p, &q);
        if (q == p) return false;
        p = q;
        return true;
    }
};

// ------------------------------------------------ parallel section parsing
// The element and node sections of a large .plt are parsed by several
// threads when the text holds exactly one record per line: each thread
// converts the numbers of a range of lines into a staging array in file
// order, and the records are then placed by their index in one sequential
// pass (a repeated index keeps the last record, as the sequential reader
// does).  Any other layout (records spread over lines, blank or comment
// lines inside a section, too few lines) makes the caller use the sequential
// scanner instead, so both readers accept and reject the same files.

// the position after n newline-terminated lines, or null if there are fewer
const char* skip_lines(const char* p, const char* end, size_t n)
{
    for (size_t i = 0; i < n; ++i) {
        const void* q = std::memchr(p, '\n', static_cast<size_t>(end - p));
        if (!q) return (i + 1 == n && p < end) ? end : nullptr;
        p = static_cast<const char*>(q) + 1;
    }
    return p;
}

// Numbers of one record per line: NI integers, then ND doubles.  Fills
// out[line * (NI + ND)] (integers stored as doubles are exact) and returns
// false if any line does not hold exactly NI + ND numbers.
template <int NI, int ND>
bool parse_lines(const char* p, const char* end, size_t nlines, double* out)
{
    constexpr int W = NI + ND;
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (nlines < 100000) nt = 1;
    // chunk boundaries on line starts
    std::vector<const char*> cut(nt + 1, p);
    cut[nt] = end;
    for (unsigned t = 1; t < nt; ++t) {
        const char* c = p + (end - p) * static_cast<long long>(t) / nt;
        if (c < cut[t - 1]) c = cut[t - 1];
        const void* q = std::memchr(c, '\n', static_cast<size_t>(end - c));
        cut[t] = q ? static_cast<const char*>(q) + 1 : end;
    }
    std::vector<size_t> first(nt + 1, 0);   // line index of each chunk's start
    for (unsigned t = 0; t < nt; ++t) {
        size_t n = 0;
        for (const char* c = cut[t]; c < cut[t + 1];) {
            const void* q = std::memchr(c, '\n', static_cast<size_t>(cut[t + 1] - c));
            ++n;
            c = q ? static_cast<const char*>(q) + 1 : cut[t + 1];
        }
        first[t + 1] = first[t] + n;
    }
    if (first[nt] != nlines) return false;
    std::vector<char> ok(nt, 1);
    auto work = [&](unsigned t) {
        const char* c = cut[t];
        const char* stop = cut[t + 1];
        double* o = out + first[t] * W;
        while (c < stop) {
            const char* eol = static_cast<const char*>(std::memchr(c, '\n', static_cast<size_t>(stop - c)));
            if (!eol) eol = stop;
            for (int k = 0; k < W; ++k) {
                while (c < eol && std::isspace(static_cast<unsigned char>(*c))) ++c;
                if (c >= eol) { ok[t] = 0; return; }
                char* q = nullptr;
                if (k < NI) {
                    errno = 0;
                    const long x = std::strtol(c, &q, 10);
                    if (q == c || errno || q > eol) { ok[t] = 0; return; }
                    o[k] = static_cast<double>(static_cast<int>(x));
                } else {
                    const double x = std::strtod(c, &q);
                    if (q == c || q > eol) { ok[t] = 0; return; }
                    o[k] = x;
                }
                c = q;
            }
            while (c < eol && std::isspace(static_cast<unsigned char>(*c))) ++c;
            if (c != eol) { ok[t] = 0; return; }
            c = eol < stop ? eol + 1 : stop;
            o += W;
        }
    };
    if (nt == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) th.emplace_back(work, t);
        for (auto& x : th) x.join();
    }
    for (char x : ok)
        if (!x) return false;
    return true;
}

// The element and node sections of a large regular .plt (see above); on
// success the records are placed with the sequential reader's checks and
// messages, in file order, and sc points past the node section.
bool parse_sections_parallel(HostModel& m, Scanner& sc)
{
    const size_t E = static_cast<size_t>(m.E), N = static_cast<size_t>(m.N);
    if (E + N < 100000) return false;
    const char* e_end = skip_lines(sc.p, sc.end, E);
    const char* n_end = e_end ? skip_lines(e_end, sc.end, N) : nullptr;
    if (!n_end) return false;
    std::vector<double> ev(E * 5), nv(N * 4);
    if (!parse_lines<5, 0>(sc.p, e_end, E, ev.data()) || !parse_lines<1, 3>(e_end, n_end, N, nv.data())) return false;
    for (size_t i = 0; i < E; ++i) {
        const double* r = &ev[5 * i];
        const int ie = static_cast<int>(r[0]);
        if (ie < 1 || ie > m.E) bad("MeshIO::readMeshFile - element index out of range");
        for (int j = 0; j < 4; ++j) {
            const int v = static_cast<int>(r[1 + j]);
            if (v < 1 || v > m.N) bad("MeshIO::readMeshFile - connectivity node out of range");
            m.intma[4 * static_cast<size_t>(ie - 1) + j] = v;
        }
    }
    for (size_t i = 0; i < N; ++i) {
        const double* r = &nv[4 * i];
        const int ip = static_cast<int>(r[0]);
        if (ip < 1 || ip > m.N) bad("MeshIO::readMeshFile - node index out of range");
        for (int j = 0; j < 3; ++j) m.coord[3 * static_cast<size_t>(ip - 1) + j] = r[1 + j];
    }
    sc.p = n_end;
    return true;
}

// skip the first data line (header) of a buffer, returning a pointer past it
const char* after_first_data_line(const std::string& buf, std::string& header)
{
    size_t pos = 0;
    while (pos < buf.size()) {
        size_t e = buf.find('\n', pos);
        if (e == std::string::npos) e = buf.size();
        const std::string line = trim(buf.substr(pos, e - pos));
        pos = e + 1;
        if (line.empty() || line[0] == '#' || line[0] == '!') continue;
        header = line;
        return buf.data() + std::min(pos, buf.size());
    }
    return nullptr;
}

bool supported_solver_bc_id(int bc)
{
    // MeshIO's .bco whitelist (src/io/MeshIO.cpp:447-469)
    switch (bc) {
    case 500: case 501: case 502: case 503: case 506: case 507: case 508: case 510:
    case 511: case 520: case 530: case 532: case 901: case 902: return true;
    default: return false;
    }
}

bool supported_bc(int bc)
{
    // Boundary's supported set (src/boundary/Boundary.cpp:31-49)
    return supported_solver_bc_id(bc) || bc == 504;
}

bool is_no_slip_wall_bc(int bc)
{ return bc == 501 || bc == 502 || bc == 530 || bc == 532 || bc == 901; }

bool is_prescribed_velocity_face_bc(int bc)
{
    return bc == 500 || bc == 501 || bc == 502 || bc == 503 || bc == 507 || bc == 508 ||
           bc == 510 || bc == 511 || bc == 530 || bc == 532 || bc == 901;
}

const int IPPN1[5][3] = {{0, 0, 0}, {3, 2, 4}, {3, 4, 1}, {1, 4, 2}, {1, 2, 3}};

// ----------------------------------------------------------------- .par
struct ParReader {
    std::istringstream in;
    std::string file;
    template <typename... T>
    void pair(const char* what, T&... v)
    {
        next_data_line(in, file);
        std::istringstream iss(next_data_line(in, file));
        if (!((iss >> ... >> v))) bad(std::string("MeshIO::readParameterFile - invalid ") + what);
    }
    template <typename... T>
    bool optional_pair(const char* what, T&... v)
    {
        std::string label, line;
        if (!read_data_line(in, label)) return false;
        if (!read_data_line(in, line)) bad(std::string("MeshIO::readParameterFile - missing ") + what + " data line");
        std::istringstream iss(line);
        if (!((iss >> ... >> v))) bad(std::string("MeshIO::readParameterFile - invalid ") + what + " line");
        return true;
    }
};

// MeshIO::readParameterFile, src/io/MeshIO.cpp:986-1437
void read_par(const std::string& path, cbs3d_params& p)
{
    ParReader r;
    r.in.str(slurp(path, "MeshIO::readParameterFile"));
    r.file = path;
    r.pair("SOLVER_OPT", p.solver_opt);
    r.pair("RESTART_OPT", p.restart_opt);
    r.pair("TEMP_CALC", p.temp_calc);
    r.pair("3D freestream line; expected Ux Uy Uz P T", p.cinf[0], p.cinf[1], p.cinf[2], p.cinf[3], p.cinf[4]);
    r.pair("timestep-control line", p.ntime, p.transient_on, p.dtfixed, p.dtfix, p.iwrite);
    r.pair("CSAFM/THETA line", p.csafm, p.theta1);
    {
        std::string label, line;
        if (!read_data_line(r.in, label)) bad("MeshIO::readParameterFile - missing CBS3D timestep-control label line");
        if (!read_data_line(r.in, line)) bad("MeshIO::readParameterFile - missing CBS3D timestep-control data line");
        std::istringstream iss(line);
        if (!(iss >> p.cbs_scheme >> p.ilots >> p.htype >> p.step2_check >> p.rem_deltp >> p.beta_opt >>
              p.dtfix_end >> p.csafm2 >> p.epsilon1 >> p.deltr))
            bad("MeshIO::readParameterFile - invalid CBS3D timestep-control line; expected cbs_scheme ilots htype step2_check rem_deltp beta_opt dtfix_end csafm2 epsilon1 deltr");
    }
    r.pair("Re/Pr/Ra/Ri line", p.re, p.pr, p.ra, p.ri);
    r.pair("CONVECTION_TYPE", p.convection_type);
    r.pair("PNODE", p.pnode);
    r.pair("output-control line", p.write_output, p.write_time_output, p.time_output_interval, p.end_rtime);
    r.pair("CG tolerance line", p.relToler, p.absToler);
    r.pair("steady-state tolerance line", p.vel_check, p.l2norm_vel_tolerance, p.temp_check, p.l2norm_temp_tolerance);
    r.pair("output-format line", p.paraview_output, p.tecplot_output, p.nusselt_calc, p.nusselt_flag);
    r.pair("RUNTIME_MOD", p.runtime_mod);
    if (r.optional_pair("alpha/source/flux", p.alpha_sf, p.k_ratio, p.source_solid, p.heat_flux_bc) &&
        r.optional_pair("dimensional-control", p.dimensional_mode, p.material_properties_enabled, p.mass_flow_inlet_enabled) &&
        r.optional_pair("reference/inlet/outlet", p.p_ref, p.model_depth, p.inlet_mass_flow_rate, p.inlet_density, p.inlet_temperature, p.outlet_pressure_gauge) &&
        r.optional_pair("prescribed inlet velocity", p.inlet_u, p.inlet_v, p.inlet_w)) {
        r.optional_pair("Nusselt reference", p.nusselt_Tinf, p.nusselt_Tref, p.nusselt_diameter);
    }
    {
        std::string label, line;
        if (!read_data_line(r.in, label)) bad("MeshIO::readParameterFile - missing pressure-CG-control label line");
        if (!read_data_line(r.in, line)) bad("MeshIO::readParameterFile - missing pressure-CG-control data line");
        std::istringstream iss(line);
        if (!(iss >> p.cg_preconditioner >> p.cg_conv_test >> p.cg_max_iter >> p.l2norm_pres_tolerance))
            bad("MeshIO::readParameterFile - invalid pressure-CG-control line; expected cg_preconditioner cg_conv_test cg_max_iter l2norm_pres_tolerance");
    }
    {
        std::string label, line;
        if (!read_data_line(r.in, label)) bad("MeshIO::readParameterFile - missing CBS3D output/monitor-control label line");
        if (!read_data_line(r.in, line)) bad("MeshIO::readParameterFile - missing CBS3D output/monitor-control data line");
        std::istringstream iss(line);
        if (!(iss >> p.residual_log_enabled >> p.residual_log_every >> p.console_log_every >>
              p.live_residual_plot >> p.vtu_output_enabled >> p.vtu_output_every_iterations >>
              p.vtu_output_every_sim_time >> p.write_boundary_debug_arrays >> p.steady_min_iterations))
            bad("MeshIO::readParameterFile - invalid CBS3D output/monitor-control line");
    }
    {
        std::string label, line;
        if (!read_data_line(r.in, label)) bad("MeshIO::readParameterFile - missing artificial-diffusion-control label line");
        if (!read_data_line(r.in, line)) bad("MeshIO::readParameterFile - missing artificial-diffusion-control data line");
        std::istringstream iss(line);
        if (!(iss >> p.art_diff)) bad("MeshIO::readParameterFile - invalid artificial-diffusion-control line; expected art_diff");
    }
}

// validation block of readParameterFile, src/io/MeshIO.cpp:1193-1433
void validate_params(const cbs3d_params& p, int npoin)
{
    auto req = [](bool ok, const char* m) { if (!ok) bad(std::string("MeshIO::readParameterFile - ") + m); };
    req(p.solver_opt >= 1 && p.solver_opt <= 3, "SOLVER_OPT must be 1, 2, or 3");
    req(p.restart_opt >= 0 && p.restart_opt <= 1, "RESTART_OPT must be 0 or 1");
    req(p.temp_calc >= 0 && p.temp_calc <= 1, "TEMP_CALC must be 0 or 1");
    req(p.ntime >= 1, "NTIME must be >= 1");
    req(p.transient_on >= 0 && p.transient_on <= 1, "TRANSIENT_ON must be 0 or 1");
    req(p.dtfixed >= -1 && p.dtfixed <= 1, "DTFIXED must be -1, 0 or 1");
    req(p.dtfix > 0.0, "DTFIX must be > 0");
    req(p.iwrite >= 1, "IWRITE must be >= 1");
    req(p.csafm > 0.0, "CSAFM must be > 0");
    req(p.theta1 >= 0.5 && p.theta1 <= 1.0, "THETA(1) must satisfy 0.5 <= theta <= 1.0");
    req(p.cbs_scheme >= 0 && p.cbs_scheme <= 1, "CBS_SCHEME must be 0 explicit or 1 semi-implicit");
    req(p.htype >= 1 && p.htype <= 3, "HTYPE must be 1, 2, or 3");
    req(p.step2_check >= 0 && p.step2_check <= 1, "STEP2_CHECK must be 0 or 1");
    req(p.rem_deltp >= 0 && p.rem_deltp <= 1, "REM_DELTP must be 0 or 1");
    req(p.beta_opt >= 0 && p.beta_opt <= 1, "BETA_OPT must be 0 or 1");
    req(p.dtfix_end >= 0, "DTFIX_END must be >= 0");
    req(p.csafm2 > 0.0, "CSAFM2 must be > 0");
    req(p.epsilon1 > 0.0, "EPSILON1 must be > 0");
    req(p.deltr > 0.0, "DELTR must be > 0");
    req(p.cg_preconditioner >= 0 && p.cg_preconditioner <= 1, "CG_PRECONDITIONER must be 0 or 1");
    req(p.cg_conv_test >= 1 && p.cg_conv_test <= 3, "CG_CONV_TEST must be 1, 2, or 3");
    req(p.cg_max_iter >= 1, "CG_MAX_ITER must be >= 1");
    req(p.l2norm_pres_tolerance >= 0.0, "L2NORM_PRES_TOLERANCE must be >= 0");
    req(p.residual_log_enabled >= 0 && p.residual_log_enabled <= 1, "RESIDUAL_LOG_ENABLED must be 0 or 1");
    req(p.residual_log_every >= 1, "RESIDUAL_LOG_EVERY must be >= 1");
    req(p.console_log_every >= 0, "CONSOLE_LOG_EVERY must be >= 0");
    req(p.live_residual_plot >= 0 && p.live_residual_plot <= 1, "LIVE_RESIDUAL_PLOT must be 0 or 1");
    req(p.vtu_output_enabled >= 0 && p.vtu_output_enabled <= 1, "VTU_OUTPUT_ENABLED must be 0 or 1");
    req(p.vtu_output_every_iterations >= 0, "VTU_OUTPUT_EVERY_ITERATIONS must be >= 0");
    req(p.vtu_output_every_sim_time >= 0.0, "VTU_OUTPUT_EVERY_SIM_TIME must be >= 0");
    req(p.write_boundary_debug_arrays >= 0 && p.write_boundary_debug_arrays <= 1, "WRITE_BOUNDARY_DEBUG_ARRAYS must be 0 or 1");
    req(p.steady_min_iterations >= 1, "STEADY_MIN_ITERATIONS must be >= 1");
    req(p.art_diff >= 0 && p.art_diff <= 1, "ART_DIFF must be 0 or 1");
    req(p.convection_type >= 0 && p.convection_type <= 1, "CONVECTION_TYPE must be 0 or 1");
    req(p.pnode >= 1 && p.pnode <= npoin, "PNODE out of range");
    req(p.model_depth > 0.0, "MODEL_DEPTH must be > 0");
    req(p.material_properties_enabled >= 0 && p.material_properties_enabled <= 1, "MATERIAL_PROPERTIES_ENABLED must be 0 or 1");
    req(p.mass_flow_inlet_enabled >= 0 && p.mass_flow_inlet_enabled <= 1, "MASS_FLOW_INLET_ENABLED must be 0 or 1");
    req(p.inlet_density > 0.0, "INLET_DENSITY must be > 0");
    req(p.nusselt_diameter > 0.0, "NUSSELT_DIAMETER must be > 0");
}

void sort3(int* v)
{
    if (v[1] < v[0]) std::swap(v[0], v[1]);
    if (v[2] < v[1]) std::swap(v[1], v[2]);
    if (v[1] < v[0]) std::swap(v[0], v[1]);
}

}  // namespace

void default_params(cbs3d_params& p)
{
    // RunConfig defaults, include/cbs/core/RunConfig.hpp:84-323
    std::memset(&p, 0, sizeof p);
    p.solver_opt = 1;
    p.ntime = 0;
    p.iwrite = 1;
    p.theta1 = 1.0;
    p.cbs_scheme = 1;
    p.htype = 1;
    p.beta_opt = 1;
    p.csafm2 = 2.0;
    p.epsilon1 = 1.0e-6;
    p.deltr = 1.0e20;
    p.pnode = 1;
    p.alpha_sf = 1.0;
    p.k_ratio = 1.0;
    p.source_solid = 1.0;
    p.p_ref = 15.5e6;
    p.model_depth = 1.0;
    p.inlet_density = 1.0;
    p.inlet_temperature = 568.15;
    p.nusselt_Tinf = 25.0;
    p.nusselt_Tref = 100.0;
    p.nusselt_diameter = 1.0;
    p.cg_preconditioner = 1;
    p.cg_conv_test = 3;
    p.cg_max_iter = 100000;
    p.residual_log_enabled = 1;
    p.residual_log_every = 1;
    p.console_log_every = 10;
    p.vtu_output_enabled = 1;
    p.vtu_output_every_iterations = 100;
    p.write_boundary_debug_arrays = 1;
    p.steady_min_iterations = 5;
}

void read_params_only(const std::string& case_name, cbs3d_params& p, int& nelem, int& npoin, int& nboun)
{
    default_params(p);
    read_par(case_name + ".par", p);
    std::ifstream in(case_name + ".plt");
    if (!in) io_fail("MeshIO::readSizes - cannot open mesh file: " + case_name + ".plt");
    std::istringstream iss(next_data_line(in, case_name + ".plt"));
    if (!(iss >> nelem >> npoin >> nboun)) bad("MeshIO::readSizes - invalid mesh header");
}

// MeshIO::readAll, src/io/MeshIO.cpp:572-609 (readSizes :613-709,
// readMeshFile :713-868, readBoundaryFile :872-982, materials :1441-1623)
namespace {

// ------------------------------------------------------------- case cache
// The parsed inputs of a case (sizes, parameters, connectivity, coordinates,
// boundary faces, material ids and properties) in one binary file beside the
// case files, keyed by the size and modification time of every source file.
// Parsing the ASCII mesh dominates set-up for large cases; the cache skips it.
constexpr char CACHE_MAGIC[16] = "CBS3D-CASE-v1";

struct SourceStamp {
    long long size = -1, mtime_ns = -1;
};

SourceStamp stamp(const std::string& path)
{
    SourceStamp s;
    struct stat st;
    if (::stat(path.c_str(), &st) == 0) {
        s.size = static_cast<long long>(st.st_size);
        s.mtime_ns = static_cast<long long>(st.st_mtim.tv_sec) * 1000000000LL + st.st_mtim.tv_nsec;
    }
    return s;
}

std::vector<SourceStamp> case_stamps(const std::string& c)
{
    return {stamp(c + ".plt"), stamp(c + ".bco"), stamp(c + ".par"), stamp(c + ".material"), stamp(c + ".matprop")};
}

template <typename T>
void put(std::ofstream& o, const std::vector<T>& v)
{
    const unsigned long long n = v.size();
    o.write(reinterpret_cast<const char*>(&n), sizeof n);
    if (n) o.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(n * sizeof(T)));
}

template <typename T>
bool get(std::ifstream& in, std::vector<T>& v, unsigned long long limit)
{
    unsigned long long n = 0;
    if (!in.read(reinterpret_cast<char*>(&n), sizeof n) || n > limit) return false;
    v.resize(static_cast<size_t>(n));
    if (n) in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(n * sizeof(T)));
    return static_cast<bool>(in);
}

bool load_cache(const std::string& case_name, HostModel& m)
{
    std::ifstream in(case_name + ".cbscache", std::ios::binary);
    if (!in) return false;
    char magic[16] = {};
    in.read(magic, sizeof magic);
    if (!in || std::memcmp(magic, CACHE_MAGIC, sizeof magic) != 0) return false;
    unsigned long long psize = 0;
    in.read(reinterpret_cast<char*>(&psize), sizeof psize);
    if (!in || psize != sizeof(cbs3d_params)) return false;
    std::vector<SourceStamp> st(5);
    in.read(reinterpret_cast<char*>(st.data()), static_cast<std::streamsize>(st.size() * sizeof(SourceStamp)));
    const std::vector<SourceStamp> now = case_stamps(case_name);
    for (size_t i = 0; i < st.size(); ++i)
        if (!in || st[i].size != now[i].size || st[i].mtime_ns != now[i].mtime_ns) return false;
    in.read(reinterpret_cast<char*>(&m.p), sizeof m.p);
    int sizes[3] = {0, 0, 0};
    in.read(reinterpret_cast<char*>(sizes), sizeof sizes);
    if (!in || sizes[0] < 1 || sizes[1] < 1 || sizes[2] < 0) return false;
    m.E = sizes[0]; m.N = sizes[1]; m.NB = sizes[2];
    const unsigned long long lim = 1ULL << 40;
    return get(in, m.intma, lim) && get(in, m.coord, lim) && get(in, m.iside, lim) && get(in, m.mat, lim) &&
           get(in, m.rho, lim) && get(in, m.cp, lim) && get(in, m.kc, lim) && get(in, m.mu, lim) &&
           get(in, m.rho_cp, lim) && get(in, m.alpha, lim) && get(in, m.qvol, lim) &&
           m.intma.size() == 4 * static_cast<size_t>(m.E) && m.coord.size() == 3 * static_cast<size_t>(m.N) &&
           m.iside.size() == 6 * static_cast<size_t>(m.NB) && m.mat.size() == static_cast<size_t>(m.E);
}

void save_cache(const std::string& case_name, const HostModel& m)
{
    const std::string path = case_name + ".cbscache";
    const std::string tmp = path + ".tmp";
    {
        std::ofstream o(tmp, std::ios::binary | std::ios::trunc);
        if (!o) return;   // read-only case directory: no cache
        o.write(CACHE_MAGIC, sizeof CACHE_MAGIC);
        const unsigned long long psize = sizeof(cbs3d_params);
        o.write(reinterpret_cast<const char*>(&psize), sizeof psize);
        const std::vector<SourceStamp> st = case_stamps(case_name);
        o.write(reinterpret_cast<const char*>(st.data()), static_cast<std::streamsize>(st.size() * sizeof(SourceStamp)));
        o.write(reinterpret_cast<const char*>(&m.p), sizeof m.p);
        const int sizes[3] = {m.E, m.N, m.NB};
        o.write(reinterpret_cast<const char*>(sizes), sizeof sizes);
        put(o, m.intma); put(o, m.coord); put(o, m.iside); put(o, m.mat);
        put(o, m.rho); put(o, m.cp); put(o, m.kc); put(o, m.mu); put(o, m.rho_cp); put(o, m.alpha); put(o, m.qvol);
        if (!o) { std::remove(tmp.c_str()); return; }
    }
    std::rename(tmp.c_str(), path.c_str());
}

}  // namespace

bool parse_case_cached(const std::string& case_name, HostModel& m)
{
    if (load_cache(case_name, m)) return true;
    parse_case(case_name, m);
    save_cache(case_name, m);
    return false;
}

void read_case(const std::string& case_name, HostModel& m, bool use_cache, bool* from_cache)
{
    bool hit = false;
    if (use_cache) hit = parse_case_cached(case_name, m);
    else parse_case(case_name, m);
    if (from_cache) *from_cache = hit;
    m.build();
}

void parse_case(const std::string& case_name, HostModel& m)
{
    cbs3d_params& p = m.p;
    default_params(p);
    // readSizes: SOLVER_OPT first
    {
        std::istringstream in(slurp(case_name + ".par", "MeshIO::readSizes"));
        next_data_line(in, case_name + ".par");
        std::istringstream iss(next_data_line(in, case_name + ".par"));
        if (!(iss >> p.solver_opt)) bad("MeshIO::readSizes - invalid SOLVER_OPT");
        if (p.solver_opt < 1 || p.solver_opt > 3) bad("MeshIO::readSizes - SOLVER_OPT must be 1, 2, or 3");
        if (p.solver_opt == 2) bad("Steps::step2SemiImplicit - banded pressure solver path is not ported for CBS3D yet");
    }
    const std::string plt = slurp(case_name + ".plt", "MeshIO::readSizes");
    std::string header;
    const char* body = after_first_data_line(plt, header);
    if (!body) io_fail("Unexpected end of file: " + case_name + ".plt");
    {
        std::istringstream iss(header);
        if (!(iss >> m.E >> m.N >> m.NB)) bad("MeshIO::readSizes - invalid mesh header");
        if (m.E < 1 || m.N < 1 || m.NB < 0) bad("MeshIO::readSizes - non-positive mesh size in .plt header");
    }
    // .bco header and map
    std::unordered_map<int, int> raw_to_bc;
    {
        std::istringstream in(slurp(case_name + ".bco", "MeshIO::readSizes"));
        const std::string f = case_name + ".bco";
        std::istringstream hs(next_data_line(in, f));
        int nflag = 0, mass_check = 0;
        if (!(hs >> nflag)) bad("MeshIO::readSizes - invalid .bco header");
        if (!(hs >> mass_check)) mass_check = 0;
        if (nflag < 1) bad("MeshIO::readSizes - .bco must contain at least one BC mapping");
        for (int i = 0; i < nflag; ++i) {
            std::istringstream iss(next_data_line(in, f));
            int raw = 0, bc = 0;
            if (!(iss >> raw >> bc)) bad("MeshIO::readBoundaryFile - cannot read boundary flag record");
            if (raw <= 0) bad("MeshIO::readBoundaryFile - raw boundary-side ID must be positive");
            if (!supported_solver_bc_id(bc))
                bad("MeshIO::readBoundaryFile - unsupported solver BC ID " + std::to_string(bc) +
                    " for raw boundary-side ID " + std::to_string(raw));
            if (!raw_to_bc.emplace(raw, bc).second) bad("MeshIO::readBoundaryFile - duplicate raw boundary-side ID in .bco");
        }
    }
    const size_t E = m.E, N = m.N, NB = m.NB;
    m.intma.assign(4 * E, 0);
    m.coord.assign(3 * N, 0.0);
    m.iside.assign(6 * NB, 0);
    Scanner sc{body, plt.data() + plt.size()};
    if (!parse_sections_parallel(m, sc)) {
        for (size_t i = 0; i < E; ++i) {
            int ie = 0;
            if (!sc.next_int(ie)) bad("MeshIO::readMeshFile - cannot read element index");
            if (ie < 1 || ie > m.E) bad("MeshIO::readMeshFile - element index out of range");
            for (int j = 0; j < 4; ++j) {
                int v = 0;
                if (!sc.next_int(v)) bad("MeshIO::readMeshFile - cannot read tetrahedral connectivity");
                if (v < 1 || v > m.N) bad("MeshIO::readMeshFile - connectivity node out of range");
                m.intma[4 * static_cast<size_t>(ie - 1) + j] = v;
            }
        }
        for (size_t i = 0; i < N; ++i) {
            int ip = 0;
            if (!sc.next_int(ip)) bad("MeshIO::readMeshFile - cannot read node index");
            if (ip < 1 || ip > m.N) bad("MeshIO::readMeshFile - node index out of range");
            for (int j = 0; j < 3; ++j)
                if (!sc.next_double(m.coord[3 * static_cast<size_t>(ip - 1) + j]))
                    bad("MeshIO::readMeshFile - cannot read 3D coordinate");
        }
    }
    for (size_t ib = 0; ib < NB; ++ib) {
        int n1, n2, n3, parent, raw;
        if (!(sc.next_int(n1) && sc.next_int(n2) && sc.next_int(n3) && sc.next_int(parent) && sc.next_int(raw)))
            bad("MeshIO::readMeshFile - cannot read boundary-face record");
        if (n1 < 1 || n1 > m.N || n2 < 1 || n2 > m.N || n3 < 1 || n3 > m.N)
            bad("MeshIO::readMeshFile - boundary-face node out of range");
        if (parent < 1 || parent > m.E) bad("MeshIO::readMeshFile - boundary-face parent element out of range");
        const auto it = raw_to_bc.find(raw);
        if (it == raw_to_bc.end())
            bad("MeshIO::readBoundaryFile - boundary-face raw ID " + std::to_string(raw) + " not found in .bco file");
        int* r = &m.iside[6 * ib];
        r[0] = n1; r[1] = n2; r[2] = n3; r[3] = 0; r[4] = parent; r[5] = it->second;
    }
    read_par(case_name + ".par", p);
    validate_params(p, m.N);

    m.mat.assign(E, 0);
    m.rho.assign(E, 1.0); m.cp.assign(E, 1.0); m.kc.assign(E, 1.0); m.mu.assign(E, 0.0);
    m.rho_cp.assign(E, 1.0); m.alpha.assign(E, 1.0); m.qvol.assign(E, 0.0);
    if (p.material_properties_enabled > 0) {
        // .material: optional NELEM header, then eid n1..n4 mat per element
        std::istringstream in(slurp(case_name + ".material", "MeshIO::readMaterialFile"));
        std::vector<std::string> lines;
        std::string l;
        while (read_data_line(in, l)) lines.push_back(l);
        if (lines.empty()) bad("MeshIO::readMaterialFile - empty material file: " + case_name + ".material");
        size_t first = 0;
        {
            std::istringstream iss(lines[0]);
            std::vector<int> vals;
            int v;
            while (iss >> v) vals.push_back(v);
            if (vals.size() == 1) {
                if (vals[0] != m.E) bad("MeshIO::readMaterialFile - material header NELEM mismatch");
                first = 1;
            }
        }
        if (lines.size() - first != E) bad("MeshIO::readMaterialFile - number of material records does not match NELEM");
        for (size_t i = 0; i < E; ++i) {
            std::istringstream iss(lines[first + i]);
            int ie, n1, n2, n3, n4, mt;
            if (!(iss >> ie >> n1 >> n2 >> n3 >> n4 >> mt))
                bad("MeshIO::readMaterialFile - invalid material record; expected eid n1 n2 n3 n4 material_id");
            if (ie < 1 || ie > m.E) bad("MeshIO::readMaterialFile - element index out of range");
            const int* c = &m.intma[4 * static_cast<size_t>(ie - 1)];
            if (c[0] != n1 || c[1] != n2 || c[2] != n3 || c[3] != n4)
                bad("MeshIO::readMaterialFile - connectivity mismatch with mesh file");
            m.mat[ie - 1] = mt;
        }
        std::istringstream pin(slurp(case_name + ".matprop", "MeshIO::readMaterialPropertyFile"));
        int nmat = 0;
        if (!(pin >> nmat)) bad("MeshIO::readMaterialPropertyFile - cannot read material count");
        if (nmat < 1) bad("MeshIO::readMaterialPropertyFile - invalid number of materials");
        std::unordered_map<int, std::array<double, 5>> props;
        for (int i = 0; i < nmat; ++i) {
            int id = -1;
            std::string name, phase;
            std::array<double, 5> d{};
            if (!(pin >> id >> name >> phase >> d[0] >> d[1] >> d[2] >> d[3] >> d[4]))
                bad("MeshIO::readMaterialPropertyFile - invalid .matprop record");
            if (d[0] <= 0.0 || d[1] <= 0.0 || d[2] <= 0.0)
                bad("MeshIO::readMaterialPropertyFile - material " + std::to_string(id) + " has non-positive rho/cp/k");
            if (d[3] < 0.0) bad("MeshIO::readMaterialPropertyFile - material " + std::to_string(id) + " has negative viscosity");
            if (!props.emplace(id, d).second) bad("MeshIO::readMaterialPropertyFile - duplicate material ID");
        }
        for (size_t e = 0; e < E; ++e) {
            const auto it = props.find(m.mat[e]);
            if (it == props.end())
                bad("MeshIO::readMaterialPropertyFile - element " + std::to_string(e + 1) + " uses material ID " +
                    std::to_string(m.mat[e]) + " missing from .matprop");
            m.rho[e] = it->second[0]; m.cp[e] = it->second[1]; m.kc[e] = it->second[2];
            m.mu[e] = it->second[3]; m.qvol[e] = it->second[4];
            m.rho_cp[e] = m.rho[e] * m.cp[e];
            m.alpha[e] = m.kc[e] / m.rho_cp[e];
        }
    }
}

void model_from_arrays(const cbs3d_mesh& mesh, const cbs3d_params& p, HostModel& m)
{
    m.p = p;
    if (mesh.nelem < 1 || mesh.npoin < 1 || mesh.nboun < 0 || !mesh.intma || !mesh.coord ||
        (mesh.nboun > 0 && !mesh.bface))
        bad("MeshIO::readSizes - non-positive mesh size in .plt header");
    m.E = mesh.nelem; m.N = mesh.npoin; m.NB = mesh.nboun;
    const size_t E = m.E, N = m.N, NB = m.NB;
    m.intma.assign(mesh.intma, mesh.intma + 4 * E);
    for (size_t i = 0; i < 4 * E; ++i)
        if (m.intma[i] < 1 || m.intma[i] > m.N) bad("MeshIO::readMeshFile - connectivity node out of range");
    m.coord.assign(mesh.coord, mesh.coord + 3 * N);
    m.iside.assign(6 * NB, 0);
    for (size_t ib = 0; ib < NB; ++ib) {
        const int* b = mesh.bface + 5 * ib;
        for (int k = 0; k < 3; ++k)
            if (b[k] < 1 || b[k] > m.N) bad("MeshIO::readMeshFile - boundary-face node out of range");
        if (b[3] < 1 || b[3] > m.E) bad("MeshIO::readMeshFile - boundary-face parent element out of range");
        int* r = &m.iside[6 * ib];
        r[0] = b[0]; r[1] = b[1]; r[2] = b[2]; r[3] = 0; r[4] = b[3]; r[5] = b[4];
    }
    validate_params(m.p, m.N);
    m.mat.assign(E, 0);
    m.rho.assign(E, 1.0); m.cp.assign(E, 1.0); m.kc.assign(E, 1.0); m.mu.assign(E, 0.0);
    m.rho_cp.assign(E, 1.0); m.alpha.assign(E, 1.0); m.qvol.assign(E, 0.0);
    if (m.p.material_properties_enabled > 0) {
        if (!mesh.rho || !mesh.cp || !mesh.k || !mesh.mu || !mesh.qvol)
            bad("MeshIO::readMaterialPropertyFile - material properties required but not provided");
        for (size_t e = 0; e < E; ++e) {
            m.mat[e] = mesh.mat_elem ? mesh.mat_elem[e] : 0;
            m.rho[e] = mesh.rho[e]; m.cp[e] = mesh.cp[e]; m.kc[e] = mesh.k[e];
            m.mu[e] = mesh.mu[e]; m.qvol[e] = mesh.qvol[e];
            if (m.rho[e] <= 0.0 || m.cp[e] <= 0.0 || m.kc[e] <= 0.0)
                bad("MeshIO::readMaterialPropertyFile - material " + std::to_string(m.mat[e]) + " has non-positive rho/cp/k");
            if (m.mu[e] < 0.0) bad("MeshIO::readMaterialPropertyFile - material " + std::to_string(m.mat[e]) + " has negative viscosity");
            m.rho_cp[e] = m.rho[e] * m.cp[e];
            m.alpha[e] = m.kc[e] / m.rho_cp[e];
        }
    }
    m.build();
}

void build_incidence(const std::vector<int>& intma, int N, std::vector<int>& ptr, std::vector<int>& idx)
{
    const size_t Ns = static_cast<size_t>(N), Es = intma.size() / 4;
    ptr.assign(Ns + 1, 0);
    for (size_t e = 0; e < Es; ++e) for (int a = 0; a < 4; ++a) ++ptr[static_cast<size_t>(intma[4 * e + a])];
    for (size_t i = 0; i < Ns; ++i) ptr[i + 1] += ptr[i];
    idx.assign(4 * Es, 0);
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (size_t e = 0; e < Es; ++e)
        for (int a = 0; a < 4; ++a) idx[static_cast<size_t>(fill[static_cast<size_t>(intma[4 * e + a] - 1)]++)] = static_cast<int>(4 * e + a);
}

// Row order of the pressure operator: nodes sorted along a Morton curve of
// their coordinates (identity without coordinates), so that the rows of one
// slice, and of one CTA's block of slices, are spatially compact and their
// neighbour sets (halos) small.  The order only groups rows; every row's
// entries and their contributions are unchanged.
std::vector<int> locality_order(const double* coord, int N)
{
    std::vector<int> ord(static_cast<size_t>(N));
    for (int i = 0; i < N; ++i) ord[static_cast<size_t>(i)] = i;
    if (!coord || N < 2) return ord;
    double lo[3] = {coord[0], coord[1], coord[2]}, hi[3] = {coord[0], coord[1], coord[2]};
    for (int i = 0; i < N; ++i)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], coord[3 * static_cast<size_t>(i) + d]);
            hi[d] = std::max(hi[d], coord[3 * static_cast<size_t>(i) + d]);
        }
    auto spread = [](unsigned long long v) {   // 21 bits -> every third bit
        v &= 0x1fffffULL;
        v = (v | v << 32) & 0x1f00000000ffffULL;
        v = (v | v << 16) & 0x1f0000ff0000ffULL;
        v = (v | v << 8) & 0x100f00f00f00f00fULL;
        v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
        v = (v | v << 2) & 0x1249249249249249ULL;
        return v;
    };
    std::vector<unsigned long long> key(static_cast<size_t>(N));
    for (int i = 0; i < N; ++i) {
        unsigned long long k = 0;
        for (int d = 0; d < 3; ++d) {
            const double span = hi[d] - lo[d];
            const double t = span > 0.0 ? (coord[3 * static_cast<size_t>(i) + d] - lo[d]) / span : 0.0;
            const unsigned long long q = static_cast<unsigned long long>(t * 2097151.0 + 0.5);
            k |= spread(q) << d;
        }
        key[static_cast<size_t>(i)] = k;
    }
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return key[static_cast<size_t>(x)] < key[static_cast<size_t>(y)]; });
    return ord;
}

// Coordinate-free locality order: breadth-first (Cuthill-McKee) levels from a
// pseudo-peripheral node of each connected component, neighbours visited in
// element order, so consecutive rows are near each other in the mesh.
std::vector<int> graph_order(const std::vector<int>& intma, const std::vector<int>& n2e_ptr,
                             const std::vector<int>& n2e, int N)
{
    const size_t Ns = static_cast<size_t>(N);
    std::vector<int> order, level(Ns, -1), q;
    order.reserve(Ns);
    auto bfs = [&](int start, std::vector<int>& out, std::vector<int>& lev) {
        out.clear();
        out.push_back(start);
        lev[static_cast<size_t>(start)] = 0;
        for (size_t h = 0; h < out.size(); ++h) {
            const int i = out[h];
            for (int k = n2e_ptr[static_cast<size_t>(i)]; k < n2e_ptr[static_cast<size_t>(i) + 1]; ++k) {
                const size_t e = static_cast<size_t>(n2e[static_cast<size_t>(k)] >> 2);
                for (int a = 0; a < 4; ++a) {
                    const int j = intma[4 * e + a] - 1;
                    if (lev[static_cast<size_t>(j)] < 0) {
                        lev[static_cast<size_t>(j)] = lev[static_cast<size_t>(i)] + 1;
                        out.push_back(j);
                    }
                }
            }
        }
    };
    std::vector<int> seen(Ns, 0), tmp_level(Ns, -1), comp;
    for (int s0 = 0; s0 < N; ++s0) {
        if (seen[static_cast<size_t>(s0)]) continue;
        // the last node reached from s0 starts the ordering sweep
        bfs(s0, comp, tmp_level);
        const int far = comp.back();
        for (int v : comp) tmp_level[static_cast<size_t>(v)] = -1;
        bfs(far, q, level);
        for (int v : q) { seen[static_cast<size_t>(v)] = 1; order.push_back(v); }
    }
    return order;
}

// Pattern of the assembled pressure operator (see PressurePattern); row
// position p holds node order[p].
void build_pressure_pattern(const std::vector<int>& intma, const std::vector<int>& mat, int N,
                            const std::vector<int>& n2e_ptr, const std::vector<int>& n2e,
                            PressurePattern& pat, const double* coord)
{
    const size_t Ns = static_cast<size_t>(N);
    static const int PAIR[4][4] = {{-1, 0, 1, 2}, {0, -1, 3, 4}, {1, 3, -1, 5}, {2, 4, 5, -1}};
    pat = PressurePattern{};
    const std::vector<int> order = coord ? locality_order(coord, N) : graph_order(intma, n2e_ptr, n2e, N);
    pat.nslices = (N + 31) / 32;
    pat.row_node.assign(static_cast<size_t>(pat.nslices) * 32, -1);
    for (size_t q = 0; q < Ns; ++q) pat.row_node[q] = order[q];
    pat.slice_off.assign(static_cast<size_t>(pat.nslices) + 1, 0);
    pat.slice_w.assign(static_cast<size_t>(pat.nslices), 0);
    std::vector<int> row_len(Ns, 0);
    std::vector<std::pair<int, int>> items;
    // (column, e*8 + pair) of node i's fluid pair entries, stable-sorted by
    // column so each column keeps ascending element order
    auto row_items = [&](size_t i, std::vector<std::pair<int, int>>& it) {
        it.clear();
        for (int k = n2e_ptr[i]; k < n2e_ptr[i + 1]; ++k) {
            const int slot = n2e[k];
            const size_t e = static_cast<size_t>(slot >> 2);
            const int a = slot & 3;
            if (mat[e] != 0) continue;
            for (int b = 0; b < 4; ++b) {
                if (b == a) continue;
                it.emplace_back(intma[4 * e + b] - 1, static_cast<int>(e * 8 + PAIR[a][b]));
            }
        }
        std::stable_sort(it.begin(), it.end(), [](const std::pair<int, int>& x, const std::pair<int, int>& y) {
            return x.first < y.first;
        });
    };
    for (size_t i = 0; i < Ns; ++i) {
        row_items(i, items);
        int len = 0;
        for (size_t q = 0; q < items.size(); ++q)
            if (q == 0 || items[q].first != items[q - 1].first) ++len;
        row_len[i] = len;
        pat.max_row = std::max(pat.max_row, len);
    }
    long long off = 0;
    for (int s = 0; s < pat.nslices; ++s) {
        int w = 0;
        for (int l = 0; l < 32; ++l) {
            const int i = pat.row_node[static_cast<size_t>(s) * 32 + l];
            if (i >= 0) w = std::max(w, row_len[static_cast<size_t>(i)]);
        }
        pat.slice_w[static_cast<size_t>(s)] = w;
        pat.slice_off[static_cast<size_t>(s)] = off;
        off += 32LL * w;
    }
    pat.slice_off[static_cast<size_t>(pat.nslices)] = off;
    pat.nslots = off;
    if (off > 0x7fffffffLL) bad("pressure operator pattern exceeds 2^31 slots");
    // padding slots point at the row's own node (coefficient 0)
    pat.col.assign(static_cast<size_t>(off), 0);
    std::vector<long long> slot_cnt(static_cast<size_t>(off), 0);
    for (int s = 0; s < pat.nslices; ++s)
        for (int l = 0; l < 32; ++l) {
            const int i = pat.row_node[static_cast<size_t>(s) * 32 + l];
            const long long base = pat.slice_off[static_cast<size_t>(s)] + l;
            int k = -1;
            if (i >= 0) {
                row_items(static_cast<size_t>(i), items);
                for (size_t q = 0; q < items.size(); ++q) {
                    if (q == 0 || items[q].first != items[q - 1].first) ++k;
                    const size_t slot = static_cast<size_t>(base + 32LL * k);
                    pat.col[slot] = items[q].first;
                    ++slot_cnt[slot];
                }
            }
            for (int kk = k + 1; kk < pat.slice_w[static_cast<size_t>(s)]; ++kk)
                pat.col[static_cast<size_t>(base + 32LL * kk)] = i >= 0 ? i : 0;
        }
    pat.cptr.assign(static_cast<size_t>(off) + 1, 0);
    for (size_t q = 0; q < static_cast<size_t>(off); ++q) pat.cptr[q + 1] = pat.cptr[q] + slot_cnt[q];
    pat.cent.assign(static_cast<size_t>(pat.cptr[static_cast<size_t>(off)]), 0);
    std::vector<long long> fillp(pat.cptr.begin(), pat.cptr.end() - 1);
    for (int s = 0; s < pat.nslices; ++s)
        for (int l = 0; l < 32; ++l) {
            const int i = pat.row_node[static_cast<size_t>(s) * 32 + l];
            if (i < 0) continue;
            const long long base = pat.slice_off[static_cast<size_t>(s)] + l;
            row_items(static_cast<size_t>(i), items);
            int k = -1;
            for (size_t q = 0; q < items.size(); ++q) {
                if (q == 0 || items[q].first != items[q - 1].first) ++k;
                const size_t slot = static_cast<size_t>(base + 32LL * k);
                pat.cent[static_cast<size_t>(fillp[slot]++)] = items[q].second;
            }
        }
}

// ----------------------------------------------------------------- build
void HostModel::build()
{
    const size_t Es = E, Ns = N, NBs = NB;
    const cbs3d_params& P = p;

    // MeshIO::initialiseFields, src/io/MeshIO.cpp:1627-1701
    unkno.assign(3 * Ns, 0.0);
    pres.assign(Ns, 0.0);
    temp.assign(Ns, 0.0);
    for (size_t i = 0; i < Ns; ++i) {
        unkno[3 * i] = P.cinf[0]; unkno[3 * i + 1] = P.cinf[1]; unkno[3 * i + 2] = P.cinf[2];
        pres[i] = P.cinf[3]; temp[i] = P.cinf[4];
    }
    tf.assign(Ns, 0);
    ts.assign(Ns, 0);
    for (size_t e = 0; e < Es; ++e)
        for (int a = 0; a < 4; ++a) {
            const int ip = intma[4 * e + a] - 1;
            if (mat[e] == 0) tf[ip] = 1; else ts[ip] = 1;
        }
    if (P.material_properties_enabled > 0)
        for (size_t i = 0; i < Ns; ++i) {
            if (!tf[i] && !ts[i])
                bad("MeshIO::initialiseFields - orphan node not touched by any material element: " + std::to_string(i + 1));
            if (ts[i]) { unkno[3 * i] = unkno[3 * i + 1] = unkno[3 * i + 2] = 0.0; }
            if (ts[i] && !tf[i]) pres[i] = 0.0;
        }
    temp_calc = P.temp_calc;
    if (P.convection_type == 1) { ani = P.pr; temp_calc = 1; }
    else { ani = 1.0 / P.re; if (P.ri > 0.0) temp_calc = 1; }
    if (P.material_properties_enabled < 1) for (size_t e = 0; e < Es; ++e) mu[e] = ani;
    if (P.cbs_scheme == 0)
        bad("Fully explicit CBS3D mode was requested, but explicit CBS3D step kernels are not yet ported.");

    // Preprocess::validateBoundaryFlags + Boundary validate_boundary_flags
    for (size_t ib = 0; ib < NBs; ++ib)
        if (!supported_bc(iside[6 * ib + 5]))
            bad("Boundary - unsupported BC_ID " + std::to_string(iside[6 * ib + 5]) + " at boundary face " +
                std::to_string(ib + 1) + ". This CBS3D boundary module supports the CBS2D++_SI BC family adapted to 3D.");

    // Preprocess::assignBoundaryFaceNumbers, src/preprocess/Preprocess.cpp:523-574
    for (size_t ib = 0; ib < NBs; ++ib) {
        int* r = &iside[6 * ib];
        const int parent = r[4];
        int bf[3] = {r[0], r[1], r[2]};
        sort3(bf);
        int matched = 0;
        for (int is = 1; is <= 4; ++is) {
            int ef[3];
            for (int k = 0; k < 3; ++k) ef[k] = intma[4 * static_cast<size_t>(parent - 1) + IPPN1[is][k] - 1];
            sort3(ef);
            if (bf[0] == ef[0] && bf[1] == ef[1] && bf[2] == ef[2]) { matched = is; break; }
        }
        if (!matched)
            bad("Preprocess::assignBoundaryFaceNumbers - boundary face " + std::to_string(ib + 1) +
                " does not match any face of parent tetrahedron " + std::to_string(parent));
        r[3] = matched;
    }

    // Boundary face normals with the arithmetic of Preprocess::getNormals
    // (src/preprocess/Preprocess.cpp:601-679), evaluated for boundary faces.
    face_norm.assign(4 * NBs, 0.0);
    for (size_t ib = 0; ib < NBs; ++ib) {
        const int* r = &iside[6 * ib];
        const size_t e = static_cast<size_t>(r[4] - 1);
        const int is = r[3];
        const double* p1 = &coord[3 * static_cast<size_t>(intma[4 * e + IPPN1[is][0] - 1] - 1)];
        const double* p2 = &coord[3 * static_cast<size_t>(intma[4 * e + IPPN1[is][1] - 1] - 1)];
        const double* p3 = &coord[3 * static_cast<size_t>(intma[4 * e + IPPN1[is][2] - 1] - 1)];
        const double* po = &coord[3 * static_cast<size_t>(intma[4 * e + is - 1] - 1)];
        const double e1x = p2[0] - p1[0], e1y = p2[1] - p1[1], e1z = p2[2] - p1[2];
        const double e2x = p3[0] - p1[0], e2y = p3[1] - p1[1], e2z = p3[2] - p1[2];
        double ax = e1y * e2z - e1z * e2y;
        double ay = e1z * e2x - e1x * e2z;
        double az = e1x * e2y - e1y * e2x;
        const double amag = std::sqrt(ax * ax + ay * ay + az * az);
        if (amag <= 0.0 || !std::isfinite(amag))
            bad("Preprocess::getNormals - zero-area face at element " + std::to_string(e + 1) + ", face " + std::to_string(is));
        const double fx = (p1[0] + p2[0] + p3[0]) / 3.0;
        const double fy = (p1[1] + p2[1] + p3[1]) / 3.0;
        const double fz = (p1[2] + p2[2] + p3[2]) / 3.0;
        const double vx = po[0] - fx, vy = po[1] - fy, vz = po[2] - fz;
        if (ax * vx + ay * vy + az * vz > 0.0) { ax = -ax; ay = -ay; az = -az; }
        face_norm[4 * ib] = 0.5 * ax;
        face_norm[4 * ib + 1] = 0.5 * ay;
        face_norm[4 * ib + 2] = 0.5 * az;
        face_norm[4 * ib + 3] = 0.5 * amag;
    }

    // Preprocess::classifyFaceEdges, src/preprocess/Preprocess.cpp:820-843
    fedge.assign(4 * Es, 0);
    for (size_t ib = 0; ib < NBs; ++ib) {
        const int* r = &iside[6 * ib];
        fedge[4 * static_cast<size_t>(r[4] - 1) + r[3] - 1] = is_prescribed_velocity_face_bc(r[5]) ? 1 : 2;
    }

    // Preprocess::wallDetermination, src/preprocess/Preprocess.cpp:932-1031
    {
        std::vector<char> mark(Ns, 0);
        wall_list.clear();
        for (size_t ib = 0; ib < NBs; ++ib) {
            const int* r = &iside[6 * ib];
            if (!is_no_slip_wall_bc(r[5])) continue;
            for (int k = 0; k < 3; ++k) {
                const int ip = r[k] - 1;
                if (!mark[ip]) { wall_list.push_back(ip + 1); mark[ip] = 1; }
            }
        }
        for (size_t i = 0; i < Ns; ++i)
            if (tf[i] && ts[i] && !mark[i]) { wall_list.push_back(static_cast<int>(i) + 1); mark[i] = 1; }
    }

    // Preprocess::computeMassFlowInletVelocity, src/preprocess/Preprocess.cpp:1054-1112
    inlet_u_mf = 0.0;
    if (P.mass_flow_inlet_enabled > 0) {
        double area = 0.0;
        int nf = 0;
        for (size_t ib = 0; ib < NBs; ++ib)
            if (iside[6 * ib + 5] == 511) { area += face_norm[4 * ib + 3]; ++nf; }
        if (nf < 1) bad("Preprocess::computeMassFlowInletVelocity - mass-flow inlet enabled but no BC_ID 511 faces were found");
        inlet_u_mf = P.inlet_mass_flow_rate / (P.inlet_density * area);
    }

    // Preprocess::detectPressureBoundaryNodes, src/preprocess/Preprocess.cpp:1152-1242
    {
        std::vector<char> fixed(Ns, 0);
        bc_list.clear();
        bc_values.clear();
        for (size_t ib = 0; ib < NBs; ++ib) {
            const int* r = &iside[6 * ib];
            if (r[5] != 520) continue;
            for (int k = 0; k < 3; ++k) {
                const int ip = r[k] - 1;
                if (!tf[ip])
                    bad("Preprocess::detectPressureBoundaryNodes - pressure outlet node " + std::to_string(ip + 1) +
                        " is not connected to any fluid element");
                if (!fixed[ip]) { fixed[ip] = 1; bc_list.push_back(ip + 1); bc_values.push_back(P.outlet_pressure_gauge); }
            }
        }
        if (bc_list.empty()) {
            int ip = P.pnode;
            if (ip < 1 || ip > N || !tf[ip - 1]) {
                ip = 0;
                for (int c = 1; c <= N; ++c) if (tf[c - 1]) { ip = c; break; }
            }
            if (ip < 1) bad("Preprocess::detectPressureBoundaryNodes - no fluid-connected node available for pressure reference");
            bc_list.push_back(ip);
            bc_values.push_back(P.outlet_pressure_gauge);
        }
    }

    // Node -> element incidence in element order (also Coloring's CSR).
    build_incidence(intma, N, n2e_ptr, n2e);

    // Coloring::build, include/cbs/parallel/Coloring.hpp:27-97: greedy
    // first-fit in element order; a colour is forbidden when any element
    // sharing a node already holds it.
    {
        color_of.assign(Es, -1);
        std::vector<int> stamp;
        ncolor = 0;
        for (size_t e = 0; e < Es; ++e) {
            for (int a = 0; a < 4; ++a) {
                const int ip = intma[4 * e + a] - 1;
                for (int k = n2e_ptr[ip]; k < n2e_ptr[ip + 1]; ++k) {
                    const int cj = color_of[static_cast<size_t>(n2e[k] >> 2)];
                    if (cj >= 0) {
                        if (cj >= static_cast<int>(stamp.size())) stamp.resize(static_cast<size_t>(cj) + 1, -1);
                        stamp[static_cast<size_t>(cj)] = static_cast<int>(e);
                    }
                }
            }
            int c = 0;
            while (c < static_cast<int>(stamp.size()) && stamp[static_cast<size_t>(c)] == static_cast<int>(e)) ++c;
            color_of[e] = c;
            if (c + 1 > ncolor) ncolor = c + 1;
        }
        color_ptr.assign(static_cast<size_t>(ncolor) + 1, 0);
        for (size_t e = 0; e < Es; ++e) ++color_ptr[static_cast<size_t>(color_of[e]) + 1];
        for (int c = 0; c < ncolor; ++c) color_ptr[static_cast<size_t>(c) + 1] += color_ptr[static_cast<size_t>(c)];
        color_elem.assign(Es, 0);
        std::vector<int> off(color_ptr.begin(), color_ptr.end());
        for (size_t e = 0; e < Es; ++e) color_elem[static_cast<size_t>(off[static_cast<size_t>(color_of[e])]++)] = static_cast<int>(e) + 1;
    }

    // Fluid incidence in (colour, element) order: the per-node summation
    // order of the colour-by-colour Step-1 scatter.
    n2c_ptr.assign(Ns + 1, 0);
    for (size_t e = 0; e < Es; ++e)
        if (mat[e] == 0) for (int a = 0; a < 4; ++a) ++n2c_ptr[intma[4 * e + a]];
    for (size_t i = 0; i < Ns; ++i) n2c_ptr[i + 1] += n2c_ptr[i];
    n2c.assign(static_cast<size_t>(n2c_ptr[Ns]), 0);
    {
        std::vector<int> fill(n2c_ptr.begin(), n2c_ptr.end() - 1);
        for (int c = 0; c < ncolor; ++c)
            for (int k = color_ptr[c]; k < color_ptr[c + 1]; ++k) {
                const size_t e = static_cast<size_t>(color_elem[k] - 1);
                if (mat[e] != 0) continue;
                for (int a = 0; a < 4; ++a) n2c[fill[intma[4 * e + a] - 1]++] = static_cast<int>(4 * e + a);
            }
    }

    // ---------------------------------------------------- velocity BC program
    {
        std::vector<int> fixed_flag(Ns, 0);
        std::vector<double> fixv(3 * Ns, 0.0);
        std::vector<std::vector<int>> sym(Ns), out(Ns);
        auto set = [&](int ip, double u, double v, double w) {
            fixed_flag[ip] = 1; fixv[3 * ip] = u; fixv[3 * ip + 1] = v; fixv[3 * ip + 2] = w;
        };
        for (size_t ib = 0; ib < NBs; ++ib) {
            const int* r = &iside[6 * ib];
            const int bc = r[5];
            double nx = 0.0, ny = 0.0, nz = 0.0;
            if (bc == 511 || bc == 506 || bc == 520) {
                const double area = face_norm[4 * ib + 3];
                nx = face_norm[4 * ib] / area; ny = face_norm[4 * ib + 1] / area; nz = face_norm[4 * ib + 2] / area;
            }
            for (int k = 0; k < 3; ++k) {
                const int ip = r[k] - 1;
                const double y = coord[3 * static_cast<size_t>(ip) + 1];
                if (bc == 506) sym[ip].push_back(static_cast<int>(ib));
                if (bc == 520) out[ip].push_back(static_cast<int>(ib));
                if (bc == 500 || bc == 510) set(ip, P.inlet_u, P.inlet_v, P.inlet_w);
                else if (bc == 501 || bc == 502 || bc == 530 || bc == 532 || bc == 901) set(ip, 0.0, 0.0, 0.0);
                else if (bc == 503) set(ip, 1.0, 0.0, 0.0);
                else if (bc == 507)
                    set(ip, 0.6624 * std::pow(y, 6) - 7.5547 * std::pow(y, 5) + 33.9 * std::pow(y, 4) -
                                75.283 * std::pow(y, 3) + 83.368 * std::pow(y, 2) - 37.793 * y + 2.6959,
                        0.0, 0.0);
                else if (bc == 508) set(ip, 6.0 * y * (1.0 - y), 0.0, 0.0);
                else if (bc == 511) set(ip, -inlet_u_mf * nx, -inlet_u_mf * ny, -inlet_u_mf * nz);
            }
        }
        for (int w : wall_list) set(w - 1, 0.0, 0.0, 0.0);
        for (size_t ib = 0; ib < NBs; ++ib) {
            const int* r = &iside[6 * ib];
            if (r[5] != 500) continue;
            for (int k = 0; k < 3; ++k) set(r[k] - 1, P.inlet_u, P.inlet_v, P.inlet_w);
        }
        vbc_idx.assign(Ns, -1);
        vbc.clear();
        vbc_nrm.clear();
        auto push_normal = [&](int ib) {
            const double area = face_norm[4 * static_cast<size_t>(ib) + 3];
            vbc_nrm.push_back(face_norm[4 * static_cast<size_t>(ib)] / area);
            vbc_nrm.push_back(face_norm[4 * static_cast<size_t>(ib) + 1] / area);
            vbc_nrm.push_back(face_norm[4 * static_cast<size_t>(ib) + 2] / area);
        };
        for (size_t i = 0; i < Ns; ++i) {
            if (!fixed_flag[i] && !ts[i] && sym[i].empty() && out[i].empty()) continue;
            VelBC b{};
            b.flags = (fixed_flag[i] ? VBC_FIXED : 0) | (ts[i] ? VBC_SOLID : 0);
            b.fix[0] = fixv[3 * i]; b.fix[1] = fixv[3 * i + 1]; b.fix[2] = fixv[3 * i + 2];
            b.sym_beg = static_cast<int>(vbc_nrm.size() / 3);
            for (int ib : sym[i]) push_normal(ib);
            b.sym_cnt = static_cast<int>(sym[i].size());
            b.out_beg = static_cast<int>(vbc_nrm.size() / 3);
            for (int ib : out[i]) push_normal(ib);
            b.out_cnt = static_cast<int>(out[i].size());
            vbc_idx[i] = static_cast<int>(vbc.size());
            vbc.push_back(b);
        }
    }

    // ------------------------------------------ temperature BC and heat flux
    // Boundary::applyTemperature (src/boundary/Boundary.cpp:529-626) and
    // add_prescribed_heat_flux (src/assembly/EnergyAssembly.cpp:484-532).
    tbc_flag.assign(Ns, 0);
    tbc_val.assign(Ns, 0.0);
    for (size_t ib = 0; ib < NBs; ++ib) {
        const int* r = &iside[6 * ib];
        const int bc = r[5];
        for (int k = 0; k < 3; ++k) {
            const int ip = r[k] - 1;
            if (bc == 501) { tbc_flag[ip] = 1; tbc_val[ip] = 1.0; }
            else if (bc == 502 || bc == 503 || bc == 508) { tbc_flag[ip] = 1; tbc_val[ip] = 0.0; }
            else if (bc == 510 || bc == 511) { tbc_flag[ip] = 1; tbc_val[ip] = P.inlet_temperature; }
        }
    }
    {
        std::vector<std::vector<double>> hf(Ns), ha(Ns);
        std::vector<std::vector<int>> hfc(Ns);
        qf_nodes.clear();
        qf_area.clear();
        if (P.heat_flux_bc != 0.0)
            for (size_t ib = 0; ib < NBs; ++ib) {
                const int* r = &iside[6 * ib];
                if (r[5] != 532) continue;
                const double area = face_norm[4 * ib + 3];
                const double contrib = P.heat_flux_bc * area / 3.0;
                const int f = static_cast<int>(qf_area.size());
                for (int k = 0; k < 3; ++k) {
                    hf[static_cast<size_t>(r[k] - 1)].push_back(contrib);
                    hfc[static_cast<size_t>(r[k] - 1)].push_back(f);
                    ha[static_cast<size_t>(r[k] - 1)].push_back(area);
                    qf_nodes.push_back(r[k] - 1);
                }
                qf_area.push_back(area);
            }
        hf_ptr.assign(Ns + 1, 0);
        hf_val.clear();
        hf_face.clear();
        hf_area.clear();
        for (size_t i = 0; i < Ns; ++i) {
            for (double v : hf[i]) hf_val.push_back(v);
            for (int f : hfc[i]) hf_face.push_back(f);
            for (double a : ha[i]) hf_area.push_back(a);
            hf_ptr[i + 1] = static_cast<int>(hf_val.size());
        }
    }

    // ------------------------------------------ pressure-operator pattern
    build_pressure_pattern(intma, mat, N, n2e_ptr, n2e, pat, coord.data());

    // Initial boundary values: Boundary::applyTemperature, applyVelocity,
    // applyPressure (src/solver/Solver.cpp:297-299).
    for (size_t i = 0; i < Ns; ++i) if (tbc_flag[i]) temp[i] = tbc_val[i];
    for (size_t i = 0; i < Ns; ++i) {
        const int idx = vbc_idx[i];
        if (idx < 0) continue;
        const VelBC& b = vbc[static_cast<size_t>(idx)];
        if (b.flags & VBC_FIXED) { unkno[3 * i] = b.fix[0]; unkno[3 * i + 1] = b.fix[1]; unkno[3 * i + 2] = b.fix[2]; }
        if (b.flags & VBC_SOLID) { unkno[3 * i] = unkno[3 * i + 1] = unkno[3 * i + 2] = 0.0; }
    }
    for (size_t k = 0; k < bc_list.size(); ++k) pres[static_cast<size_t>(bc_list[k] - 1)] = bc_values[k];
}

}  // namespace cbs3d
