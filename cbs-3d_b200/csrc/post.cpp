#include "post.h"

#include <cmath>
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <sstream>

namespace cbs3d {

namespace {

double safe(double v) { return std::isfinite(v) ? v : 0.0; }

std::ofstream open_out(const std::string& path, std::ios::openmode mode, const char* who)
{
    std::ofstream o(path, mode);
    if (!o) throw Error(CBS3D_IO_ERROR, std::string(who) + " - cannot open " + path);
    return o;
}

// appended-data block: UInt64 byte count, then the raw values
struct Appended {
    std::string data;
    template <typename T>
    size_t add(const std::vector<T>& v)
    {
        const size_t off = data.size();
        const uint64_t n = v.size() * sizeof(T);
        data.append(reinterpret_cast<const char*>(&n), sizeof n);
        data.append(reinterpret_cast<const char*>(v.data()), n);
        return off;
    }
};

}  // namespace

void write_residual_header(const std::string& path)
{
    std::ofstream o = open_out(path, std::ios::trunc, "Post::initialiseRunOutputs");
    o << "iteration,time,dt,u_rel,u_norm,u_abs,v_rel,v_norm,v_abs,w_rel,w_norm,w_abs,"
         "p_rel,p_norm,p_abs,T_rel,T_norm,T_abs,velocity_rel_max,cg_iterations,"
         "cg_initial_l2,cg_final_l2,cg_relative_l2,cg_max_abs\n";
}

void append_residual_rows(const std::string& path, int first_iter, int every, const double* rec, int n)
{
    std::ofstream o = open_out(path, std::ios::app, "Post::writeResidualRow");
    o << std::setprecision(16);
    for (int k = 0; k < n; ++k) {
        const int it = first_iter + k;
        if (every > 1 && it % every != 0) continue;
        const double* r = rec + static_cast<size_t>(k) * LOG_WIDTH;
        const double* hb = r + LOG_HB;
        o << it << ',' << safe(r[LOG_RTIME]) << ',' << safe(r[LOG_DT]);
        for (int q = 0; q < 15; ++q) o << ',' << safe(hb[q]);
        const double vmax = std::max(hb[0], std::max(hb[3], hb[6]));   // Convergence::velocityResidual
        o << ',' << safe(vmax) << ',' << static_cast<long long>(r[LOG_CG]) << ',' << safe(r[LOG_CG + 1]) << ','
          << safe(r[LOG_CG + 2]) << ',' << safe(r[LOG_CG + 3]) << ',' << safe(r[LOG_CG + 4]) << '\n';
    }
}

void write_vtu(const std::string& path, const HostModel& m, const double* u, const double* p, const double* t,
               const double* vmag)
{
    const size_t E = m.E, N = m.N, NB = m.NB;
    // node masks of the reference's writer: touches fluid / solid
    std::vector<char> tf(N, 0), ts(N, 0);
    for (size_t e = 0; e < E; ++e)
        for (int a = 0; a < 4; ++a) (m.mat[e] == 0 ? tf : ts)[static_cast<size_t>(m.intma[4 * e + a] - 1)] = 1;
    std::vector<double> pts(m.coord), pres(N), temp(N), vel(3 * N, 0.0), vm(N);
    std::vector<int32_t> kind(N), pact(N), vact(N), tact(N);
    for (size_t i = 0; i < N; ++i) {
        const bool f = tf[i], s = ts[i];
        pact[i] = f ? 1 : 0;
        vact[i] = (f && !s) ? 1 : 0;
        tact[i] = (f || s) ? 1 : 0;
        kind[i] = (f && s) ? 3 : f ? 1 : s ? 2 : 0;
        pres[i] = f ? safe(p[i]) : 0.0;
        temp[i] = safe(t[i]);
        if (vact[i]) for (int d = 0; d < 3; ++d) vel[3 * i + d] = safe(u[3 * i + d]);
        const double mag = vmag ? vmag[i]
                                : std::sqrt(u[3 * i] * u[3 * i] + u[3 * i + 1] * u[3 * i + 1] + u[3 * i + 2] * u[3 * i + 2] + 1.0e-16);
        vm[i] = vact[i] ? safe(mag) : 0.0;
    }
    std::vector<int32_t> conn, offs, ckind, cmat, cbc, cpar;
    std::vector<uint8_t> types;
    conn.reserve(4 * E + 3 * NB);
    int32_t off = 0;
    for (size_t e = 0; e < E; ++e) {
        for (int a = 0; a < 4; ++a) conn.push_back(m.intma[4 * e + a] - 1);
        offs.push_back(off += 4);
        types.push_back(10);
        ckind.push_back(1); cmat.push_back(m.mat[e]); cbc.push_back(0); cpar.push_back(static_cast<int32_t>(e + 1));
    }
    for (size_t b = 0; b < NB; ++b) {
        const int* r = &m.iside[6 * b];
        for (int k = 0; k < 3; ++k) conn.push_back(r[k] - 1);
        offs.push_back(off += 3);
        types.push_back(5);
        ckind.push_back(2); cmat.push_back(-1); cbc.push_back(r[5]); cpar.push_back(r[4]);
    }
    Appended ap;
    std::ostringstream x;
    auto arr = [&](const char* type, const char* name, int nc, size_t offset) {
        x << "        <DataArray type=\"" << type << "\"";
        if (name) x << " Name=\"" << name << "\"";
        x << " NumberOfComponents=\"" << nc << "\" format=\"appended\" offset=\"" << offset << "\"/>\n";
    };
    x << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
      << "  <UnstructuredGrid>\n"
      << "    <Piece NumberOfPoints=\"" << N << "\" NumberOfCells=\"" << E + NB << "\">\n"
      << "      <Points>\n";
    arr("Float64", nullptr, 3, ap.add(pts));
    x << "      </Points>\n      <Cells>\n";
    arr("Int32", "connectivity", 1, ap.add(conn));
    arr("Int32", "offsets", 1, ap.add(offs));
    arr("UInt8", "types", 1, ap.add(types));
    x << "      </Cells>\n      <PointData Scalars=\"temperature\" Vectors=\"velocity\">\n";
    arr("Float64", "pressure", 1, ap.add(pres));
    arr("Float64", "temperature", 1, ap.add(temp));
    arr("Float64", "velocity", 3, ap.add(vel));
    arr("Float64", "velocity_magnitude", 1, ap.add(vm));
    arr("Int32", "node_domain_kind", 1, ap.add(kind));
    arr("Int32", "pressure_active", 1, ap.add(pact));
    arr("Int32", "velocity_active", 1, ap.add(vact));
    arr("Int32", "thermal_active", 1, ap.add(tact));
    x << "      </PointData>\n      <CellData Scalars=\"mat_id\">\n";
    arr("Int32", "cell_kind", 1, ap.add(ckind));
    arr("Int32", "mat_id", 1, ap.add(cmat));
    arr("Int32", "bc_id", 1, ap.add(cbc));
    arr("Int32", "parent_element", 1, ap.add(cpar));
    x << "      </CellData>\n    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding=\"raw\">\n   _";
    std::ofstream o = open_out(path, std::ios::trunc | std::ios::binary, "Post::writeVTU");
    const std::string head = x.str();
    o.write(head.data(), static_cast<std::streamsize>(head.size()));
    o.write(ap.data.data(), static_cast<std::streamsize>(ap.data.size()));
    o << "\n  </AppendedData>\n</VTKFile>\n";
    if (!o) throw Error(CBS3D_IO_ERROR, "Post::writeVTU - write failed: " + path);
}

void write_pvd(const std::string& path, const std::vector<std::string>& files, const std::vector<double>& times)
{
    std::ofstream o = open_out(path, std::ios::trunc, "Post::writePVD");
    o << std::setprecision(16);
    o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
      << "  <Collection>\n";
    for (size_t i = 0; i < files.size(); ++i)
        o << "    <DataSet timestep=\"" << times[i] << "\" group=\"\" part=\"0\" file=\"" << files[i] << "\"/>\n";
    o << "  </Collection>\n</VTKFile>\n";
}

}  // namespace cbs3d
