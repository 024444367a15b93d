// cbs3d_run: the reference's Solver::run (src/solver/Solver.cpp:138-224) over
// the B200 engine's C ABI.  Reads <case>.par/.plt/.bco[...], runs CBS steps
// on the device until ntime, the steady-state test or the transient end
// time, and writes output/<case>/<case>_residuals.csv, VTU snapshots and the
// PVD collection as the reference does.
//
//   cbs3d_run <case> [--device N] [--mixed] [--cache] [--chunk K]
#include "cbs3d_gpu.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <vector>

namespace fs = std::filesystem;

namespace {

void check(cbs3d_status s, cbs3d_ctx* c, const char* what)
{
    if (s != CBS3D_OK)
        throw std::runtime_error(std::string(what) + ": [" + cbs3d_status_string(s) + "] " +
                                 (c ? cbs3d_last_error(c) : ""));
}

std::string step_tag(int it)
{
    char b[32];
    std::snprintf(b, sizeof b, "step_%08d", it);
    return b;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <case> [--device N] [--mixed] [--cache] [--chunk K]\n", argv[0]);
        return 2;
    }
    const std::string case_path = argv[1];
    cbs3d_options opt;
    cbs3d_default_options(&opt);
    int chunk = 50;
    for (int i = 2; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--device" && i + 1 < argc) opt.device = std::atoi(argv[++i]);
        else if (a == "--mixed") opt.precision = CBS3D_MIXED;
        else if (a == "--cache") opt.case_cache = 1;
        else if (a == "--chunk" && i + 1 < argc) chunk = std::max(1, std::atoi(argv[++i]));
        else { std::fprintf(stderr, "unknown argument %s\n", a.c_str()); return 2; }
    }
    cbs3d_ctx* ctx = nullptr;
    try {
        cbs3d_params P;
        int ne = 0, np = 0, nb = 0;
        char err[1024] = {};
        check(cbs3d_read_params(case_path.c_str(), &P, &ne, &np, &nb, err, sizeof err), nullptr, err);
        const auto t0 = std::chrono::steady_clock::now();
        check(cbs3d_create_from_case(case_path.c_str(), &opt, &ctx, err, sizeof err), nullptr, err);
        const std::string name = fs::path(case_path).filename().string();
        const fs::path outdir = fs::path("output") / name;
        fs::create_directories(outdir);
        const std::string csv = (outdir / (name + "_residuals.csv")).string();
        const std::string pvd = (outdir / (name + ".pvd")).string();
        std::vector<std::string> vtus;
        std::vector<double> times;
        double rtime = 0.0;
        auto write_solution = [&](int it) {
            const std::string f = name + "_" + step_tag(it) + ".vtu";
            // taken on the device now, written by the context's writer thread
            check(cbs3d_write_vtu_async(ctx, (outdir / f).string().c_str()), ctx, "writeVTU");
            vtus.push_back(f);
            times.push_back(rtime);
            std::vector<const char*> fp;
            for (const auto& s : vtus) fp.push_back(s.c_str());
            check(cbs3d_write_pvd(pvd.c_str(), static_cast<int>(fp.size()), fp.data(), times.data()), ctx, "writePVD");
        };
        if (P.residual_log_enabled > 0) {
            // header only: the latest call has no steps yet
            check(cbs3d_write_residual_rows(ctx, csv.c_str(), 1), ctx, "residual CSV");
        }
        const bool vtu = P.vtu_output_enabled > 0;
        const int vtu_every = P.vtu_output_every_iterations;
        double next_vtu_time = P.vtu_output_every_sim_time;
        const bool by_time = vtu && P.transient_on > 0 && P.vtu_output_every_sim_time > 0.0;
        if (vtu) write_solution(0);
        int done = 0, last = 0;
        std::string reason = "maximum iteration count reached";
        double gpu_seconds = 0.0;
        cbs3d_step_stats st{};
        while (done < P.ntime) {
            int n = std::min(chunk, P.ntime - done);
            if (vtu && vtu_every > 0) n = std::min(n, vtu_every - done % vtu_every);
            if (by_time) n = 1;
            check(cbs3d_step(ctx, n, 1, &st), ctx, "cbs3d_step");
            gpu_seconds += st.gpu_seconds;
            if (P.residual_log_enabled > 0) check(cbs3d_write_residual_rows(ctx, csv.c_str(), 0), ctx, "residual CSV");
            done += st.steps_done;
            last = st.iitime;
            rtime = st.rtime;
            bool due = vtu && vtu_every > 0 && last % vtu_every == 0;
            if (by_time && rtime + 1.0e-14 >= next_vtu_time) {
                while (next_vtu_time <= rtime + 1.0e-14) next_vtu_time += P.vtu_output_every_sim_time;
                due = true;
            }
            if (due) write_solution(last);
            if (st.steady_reached) {
                reason = P.transient_on > 0 ? "transient end time reached" : "steady-state convergence reached";
                break;
            }
        }
        if (vtu && (vtus.empty() || vtus.back() != name + "_" + step_tag(last) + ".vtu")) write_solution(last);
        check(cbs3d_vtu_flush(ctx), ctx, "writeVTU");
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("%s: %d steps (%s); last PCG %d iterations, rel %.3e; %.3f s on the device, %.3f s total\n",
                    name.c_str(), last, reason.c_str(), st.cg.iterations, st.cg.final_relative_l2, gpu_seconds, wall);
        cbs3d_destroy(ctx);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "cbs3d_run: %s\n", e.what());
        if (ctx) cbs3d_destroy(ctx);
        return 1;
    }
}
