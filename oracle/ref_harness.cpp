// Test infrastructure only: a driver over the reference solver's public API.
//
// Builds against the reference sources where they lie (see oracle/Makefile)
// and replays the reference's own initialisation order
// (src/solver/Solver.cpp:242-302, 587-593) and per-step order
// (src/solver/Solver.cpp:609-680) without the Post/console/VTU side effects.
// It writes raw little-endian arrays for the golden fixtures and times the
// step loop for the CPU baseline.  Nothing in the product links this file.
//
// Built with -DCBS_GPU_PRESSURE (cbs_ref_gpu_harness) the pressure solve of
// Step 2 goes through the GPU backend of gpu_pressure_solver.inc -- the
// INTEGRATION.md adapter calling cbs3d_pcg_solve -- instead of
// ConjugateGradient::solvePressure; everything else stays the reference's.
//
// usage:
//   cbs_ref_harness <case> <nsteps> <outdir> [--stage K] [--every M] [--time]
//     --stage K   dump every intermediate array of step K (1-based)
//     --every M   dump u/p/T after every M-th step
//     --time      time the step loop only and print one JSON line
//     --warmup W  with --time: run W untimed steps before the timed ones

#include "cbs/assembly/EnergyAssembly.hpp"
#include "cbs/assembly/MomentumAssembly.hpp"
#include "cbs/assembly/PressureAssembly.hpp"
#include "cbs/boundary/Boundary.hpp"
#include "cbs/core/CBSStateSI.hpp"
#include "cbs/io/MeshIO.hpp"
#include "cbs/linalg/ConjugateGradient.hpp"
#include "cbs/linalg/MatrixVectorCalc.hpp"
#include "cbs/parallel/Coloring.hpp"
#include "cbs/preprocess/Preprocess.hpp"
#include "cbs/solver/Convergence.hpp"
#include "cbs/solver/Steps.hpp"
#include "cbs/timestep/TimeStep.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

using namespace cbs;

#ifdef CBS_GPU_PRESSURE
#include "gpu_pressure_solver.inc"
#endif

namespace
{
    std::string g_out;
    std::ofstream g_index;

    template <typename T>
    void dump_raw(const std::string& name, const T* p, size_t n, const char* dtype)
    {
        const std::string path = g_out + "/" + name + ".bin";
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) { std::perror(path.c_str()); std::exit(3); }
        if (n) std::fwrite(p, sizeof(T), n, f);
        std::fclose(f);
        g_index << name << " " << dtype << " " << n << "\n";
    }

    // Arrays are 1-based with slot 0 unused: element 1 lives at raw()[1].
    void dump(const std::string& name, const Array1D<Real>& a)
    { dump_raw(name, a.raw().data() + 1, a.raw().size() - 1, "f8"); }
    void dump(const std::string& name, const Array2D<Real>& a)
    { dump_raw(name, a.raw().data() + 1, a.raw().size() - 1, "f8"); }
    void dump(const std::string& name, const Array3D<Real>& a)
    { dump_raw(name, a.raw().data() + 1, a.raw().size() - 1, "f8"); }
    void dump(const std::string& name, const Array1D<Int>& a, size_t n)
    { dump_raw(name, a.raw().data() + 1, n, "i4"); }
    void dump(const std::string& name, const Array2D<Int>& a)
    { dump_raw(name, a.raw().data() + 1, a.raw().size() - 1, "i4"); }
    void dump_vec(const std::string& name, const std::vector<Int>& v)
    { dump_raw(name, v.data(), v.size(), "i4"); }
    void dump_vec(const std::string& name, const std::vector<Real>& v)
    { dump_raw(name, v.data(), v.size(), "f8"); }

    void velocity_magnitude(CBSStateSI& s)
    {
        // src/solver/Solver.cpp:689-699
        for (Int ip = 1; ip <= s.cfg.npoin; ++ip)
        {
            const Real u = s.unkno(1, ip);
            const Real v = s.unkno(2, ip);
            const Real w = s.unkno(3, ip);
            s.velocity(ip) = std::sqrt(u * u + v * v + w * w + 1.0e-16);
        }
    }

    void initialise(CBSStateSI& s, const std::string& case_name)
    {
        // src/solver/Solver.cpp:242-302
        MeshIO::readAll(case_name, s);
        Preprocess::validateBoundaryFlags(s);
        Preprocess::shapeFunctionDerivatives(s);
        Preprocess::assignBoundaryFaceNumbers(s);
        Preprocess::getNormals(s);
        Preprocess::massMatrix(s);
        Preprocess::classifyFaceEdges(s);
        Preprocess::elementSize(s);
        Preprocess::wallDetermination(s);
        Preprocess::computeMassFlowInletVelocity(s);
        Preprocess::initialiseVelocityMagnitude(s);
        Preprocess::detectPressureBoundaryNodes(s);
        Coloring::build(s);
        Boundary::applyTemperature(s);
        Boundary::applyVelocity(s);
        Boundary::applyPressure(s);
        velocity_magnitude(s);
        // src/solver/Solver.cpp:587-593
        PressureAssembly::buildElementPressureTerms(s);
        PressureAssembly::buildGlobalPressureTerms(s);
    }

    struct StepRecord
    {
        double dtreal;
        double cg_iter, cg_init, cg_final, cg_rel, cg_max;
        double hb[15];
    };

    // One CBS step in the order of src/solver/Solver.cpp:609-680.  Step 2 is
    // expanded exactly as src/solver/Steps.cpp:305-350 so that the pressure
    // RHS can be dumped between assembly and solve.
    void advance(CBSStateSI& s, Int iitime, bool stage_dump, StepRecord& rec)
    {
        s.unkn1 = s.unkno;
        s.pres1 = s.pres;
        s.temperature1 = s.temperature;
        if (stage_dump)
        {
            dump("s0_unkno", s.unkno);
            dump("s0_pres", s.pres);
            dump("s0_temperature", s.temperature);
        }

        TimeStep::computeTimeStep(s, iitime);
        if (s.cfg.transient_on > 0) s.cfg.rtime += s.cfg.dtreal;
        if (stage_dump)
        {
            dump("s1_delte", s.delte);
            dump_vec("s1_dtreal", std::vector<Real>{s.cfg.dtreal});
            dump("s1_alen", s.alen);
        }

        TimeStep::updateLhsDiagonal(s);
        if (stage_dump)
        {
            dump("s2_elcoe2", s.elcoe2);
            dump("s2_elcoe2p", s.elcoe2p);
            dump("s2_pdiag", s.pdiag);
            dump("s2_gstif", s.gstif);
            dump("s2_pres", s.pres);
        }

        Steps::step1(s);
        if (stage_dump)
        {
            dump("s3_rhs", s.rhs);
            dump("s3_unkno", s.unkno);
        }

        if (s.cfg.step2_check > 0)
        {
            TimeStep::applyStep2PressureTimeStepCorrection(s);
            TimeStep::updateLhsDiagonal(s);
        }

        // Steps::step2SemiImplicit, expanded
        PressureAssembly::assembleStep2Rhs(s);
        if (stage_dump)
        {
            dump("s4_rhs1", s.rhs1);
            dump("s4_pres_in", s.pres);
            dump("s4_pdiag_in", s.pdiag);
            dump("s4_gstif", s.gstif);
            // reference matvec of the incoming pressure for the matvec KAT
            Array1D<Real> y;
            y.resize(s.cfg.npoin);
            MatrixVectorCalc::pressureMultiply(s, s.pres, y);
            dump("s4_Apres", y);
        }
#ifdef CBS_GPU_PRESSURE
        ConjugateGradient::Result r = GpuPressureSolver::solvePressure(s);
#else
        ConjugateGradient::Result r = ConjugateGradient::solvePressure(s);
#endif
        s.last_cg_iterations = r.iterations;
        s.last_cg_initial_l2 = r.initial_l2;
        s.last_cg_final_l2 = r.final_l2;
        s.last_cg_relative_l2 = r.final_relative_l2;
        s.last_cg_max_abs = r.final_max_abs;
        if (!r.converged)
            throw std::runtime_error("Steps::step2SemiImplicit - pressure solver failed to converge");
        Boundary::applyPressure(s);
        if (stage_dump)
        {
            dump("s5_pres", s.pres);
            dump("s5_rhs1", s.rhs1);
            dump("s5_pdiag", s.pdiag);
            dump_vec("s5_cg", std::vector<Real>{static_cast<Real>(r.iterations), r.initial_l2,
                                               r.final_l2, r.final_relative_l2, r.final_max_abs});
        }

        Steps::step3(s);
        if (stage_dump)
        {
            dump("s6_rhs", s.rhs);
            dump("s6_unkno", s.unkno);
        }

        Steps::step4(s);
        if (stage_dump && s.cfg.temp_calc > 0)
        {
            dump("s7_rhs1", s.rhs1);
            dump("s7_temperature", s.temperature);
        }

        velocity_magnitude(s);
        Convergence::evaluate(s);
        if (stage_dump)
        {
            dump("s8_velocity", s.velocity);
            dump_vec("s8_hb", std::vector<Real>(s.hb.begin(), s.hb.end()));
        }

        rec.dtreal = s.cfg.dtreal;
        rec.cg_iter = r.iterations;
        rec.cg_init = r.initial_l2;
        rec.cg_final = r.final_l2;
        rec.cg_rel = r.final_relative_l2;
        rec.cg_max = r.final_max_abs;
        for (int i = 0; i < 15; ++i) rec.hb[i] = s.hb[i];
    }
}

int main(int argc, char** argv)
{
    if (argc < 4)
    {
        std::fprintf(stderr, "usage: %s <case> <nsteps> <outdir> [--stage K] [--every M] [--time]\n", argv[0]);
        return 2;
    }
    const std::string case_name = argv[1];
    const int nsteps = std::atoi(argv[2]);
    g_out = argv[3];
    int stage = 0, every = 0, warmup = 0;
    bool timing = false;
    for (int i = 4; i < argc; ++i)
    {
        if (!std::strcmp(argv[i], "--stage") && i + 1 < argc) stage = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--every") && i + 1 < argc) every = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--time")) timing = true;
        else if (!std::strcmp(argv[i], "--warmup") && i + 1 < argc) warmup = std::atoi(argv[++i]);
    }

    try
    {
        static CBSStateSI s;
        const auto t_setup = std::chrono::steady_clock::now();
        {
            // keep the reference's preprocessing chatter off stdout in timing mode
            std::streambuf* old = nullptr;
            std::ofstream devnull;
            if (timing) { devnull.open("/dev/null"); old = std::cout.rdbuf(devnull.rdbuf()); }
            initialise(s, case_name);
            if (old) std::cout.rdbuf(old);
        }
        const double setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_setup).count();

        if (!timing)
        {
            g_index.open(g_out + "/index.txt");
            const Int E = s.cfg.nelem, N = s.cfg.npoin, NB = s.cfg.nboun;
            dump_vec("sizes", std::vector<Int>{E, N, NB, s.ncolor, s.cfg.bc_fixed, s.cfg.npoin_wall});
            dump("intma", s.intma);
            dump("coord", s.coord);
            dump("iside", s.iside);
            dump("mat_elem", s.mat_elem, static_cast<size_t>(E));
            dump("fedge", s.fedge);
            dump("detJ", s.detJ);
            dump("dNkdx", s.dNkdx);
            dump("annxf", s.annxf);
            dump("face_norm", s.face_norm);
            dump("alen_e", s.alen_e);
            dump("elcoe_e", s.elcoe_e);
            dump("Mdiag_real", s.Mdiag_real);
            dump("pdiagE", s.pdiagE);
            dump("gstifE", s.gstifE);
            dump_vec("color_ptr", s.color_ptr);
            dump_vec("color_elem", s.color_elem);
            dump("bc_list", s.bc_list, static_cast<size_t>(s.cfg.bc_fixed));
            dump_raw("bc_values", s.bc_values.raw().data() + 1, static_cast<size_t>(s.cfg.bc_fixed), "f8");
            dump("wall_node_list", s.wall_node_list, static_cast<size_t>(s.cfg.npoin_wall));
            dump("init_unkno", s.unkno);
            dump("init_pres", s.pres);
            dump("init_temperature", s.temperature);
            dump_vec("cfg_scalars", std::vector<Real>{s.cfg.ani, s.cfg.inlet_u_from_massflow,
                                                      static_cast<Real>(s.cfg.temp_calc)});
        }

        std::vector<Real> hist;
        StepRecord rec{};
        Int it0 = 1;
        if (timing)
            for (; it0 <= warmup; ++it0) advance(s, it0, false, rec);
        const auto t0 = std::chrono::steady_clock::now();
        int done = 0;
        for (Int it = it0; it < it0 + nsteps; ++it)
        {
            advance(s, it, !timing && it == stage, rec);
            ++done;
            if (!timing)
            {
                hist.push_back(rec.dtreal);
                hist.push_back(rec.cg_iter);
                hist.push_back(rec.cg_init);
                hist.push_back(rec.cg_final);
                hist.push_back(rec.cg_rel);
                hist.push_back(rec.cg_max);
                for (double v : rec.hb) hist.push_back(v);
                if (every > 0 && it % every == 0)
                {
                    dump("step" + std::to_string(it) + "_unkno", s.unkno);
                    dump("step" + std::to_string(it) + "_pres", s.pres);
                    if (s.cfg.temp_calc > 0) dump("step" + std::to_string(it) + "_temperature", s.temperature);
                }
            }
        }
        const double loop_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

        if (timing)
        {
            int threads = 1;
#ifdef _OPENMP
            threads = omp_get_max_threads();
#endif
            std::printf("{\"steps\": %d, \"seconds\": %.6f, \"steps_per_s\": %.6f, \"threads\": %d, "
                        "\"setup_seconds\": %.3f, \"last_cg_iterations\": %d}\n",
                        done, loop_s, done / loop_s, threads, setup_s, s.last_cg_iterations);
        }
        else
        {
            dump_vec("history", hist);
            dump("final_unkno", s.unkno);
            dump("final_pres", s.pres);
            dump("final_temperature", s.temperature);
            g_index.close();
        }
    }
    catch (const std::exception& e)
    {
        std::fprintf(stderr, "reference error: %s\n", e.what());
        return 1;
    }
    return 0;
}
