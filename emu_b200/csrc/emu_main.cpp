// emu_main.cpp -- host driver: Emu's evolve_flavor loop (Source/main.cpp:41-225)
// over the C ABI, reading the reference's inputs files.
//
//   emu_main <inputs file> [key=value ...]
//
// Same sequence as the reference: parameters (TestParams::Initialize),
// particles from InitParticles or from a restart plotfile (RecoverParticles),
// deposit, plotfile plt00000 with particles after initialisation, then RK
// steps with the post-step work on the device (wrap, Renormalize, compute_dt
// on the last stage mesh), plotfiles every write_plot_every steps (particles
// every write_plot_particles_every), and the figure of merit "particles
// advanced per microsecond" at the end (main.cpp:214-225).
//
// The step loop stays on the device between plotfiles: progress lines are
// printed when the host synchronises (at each plotfile and at the end), not
// after every step.
#include "emu_b200.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

int die(const emu_context* ctx, int code, const char* what)
{
    char buf[1024];
    emu_last_error(ctx, buf, sizeof buf);
    std::fprintf(stderr, "emu_main: %s failed (status %d): %s\n", what, code, buf);
    return 1;
}

std::string plot_name(int step)
{
    char b[32];
    std::snprintf(b, sizeof b, "plt%05d", step);
    return b;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2 || std::string(argv[1]) == "-h" || std::string(argv[1]) == "--help") {
        std::fprintf(stderr, "usage: %s <inputs file> [key=value ...]\n", argv[0]);
        return argc < 2 ? 2 : 0;
    }
    emu_params p;
    char err[1024] = {0};
    std::vector<const char*> ov(argv + 2, argv + argc);
    int r = emu_parse_inputs(argv[1], (int)ov.size(), ov.empty() ? nullptr : ov.data(), &p, err, sizeof err);
    if (r) {
        std::fprintf(stderr, "emu_main: inputs: %s\n", err);
        return 1;
    }
    std::printf("Initializing particles... ");
    std::fflush(stdout);
    std::vector<double> recs;
    int64_t n = 0;
    double t0 = 0.0;
    int step0 = 0;
    if (p.do_restart) {
        if ((r = emu_read_particles(p.restart_dir, p.nflavors, nullptr, 0, &n, nullptr, nullptr)))
            return die(nullptr, r, "restart");
        recs.resize((size_t)n * emu_nreal(p.nflavors));
        if ((r = emu_read_particles(p.restart_dir, p.nflavors, recs.data(), n, &n, &t0, &step0)))
            return die(nullptr, r, "restart");
        // (IO.cpp:61)
        std::printf("Restarting after time step: %d t = %.17g s.  ct = %.17g cm\n", step0 - 1, t0,
                    2.99792458e10 * t0);
    }
    emu_context* ctx = nullptr;
    if ((r = emu_create(&p, &ctx))) return die(nullptr, r, "emu_create");
    if (p.do_restart) {
        if ((r = emu_load_particles(ctx, recs.data(), n))) return die(ctx, r, "emu_load_particles");
    } else if ((r = emu_init_particles_device(ctx))) {   // InitParticles, on the device
        return die(ctx, r, "InitParticles");
    }
    if (!p.do_restart && (r = emu_write_plotfile(ctx, plot_name(step0).c_str(), t0, step0, 1)))
        return die(ctx, r, "WritePlotFile");
    std::printf("Done. \nStarting timestepping loop... \n");

    const int total = p.nsteps - step0;
    const auto start = std::chrono::steady_clock::now();
    double fom = 0.0;
    int done = 0;
    emu_run_info info{};
    if (total > 0) {
        if ((r = emu_evolve_begin(ctx, t0, p.end_time, total))) return die(ctx, r, "emu_evolve_begin");
        while (done < total) {
            // run to the next output step (or the end) without host round trips
            int next = total;
            const int s = step0 + done;
            if (p.write_plot_every > 0) next = std::min(next, (s / p.write_plot_every + 1) * p.write_plot_every - step0);
            if (p.write_plot_particles_every > 0)
                next = std::min(next, (s / p.write_plot_particles_every + 1) * p.write_plot_particles_every - step0);
            if ((r = emu_evolve_steps(ctx, next - done))) return die(ctx, r, "emu_evolve_steps");
            r = emu_evolve_end(ctx, &info);
            if (r & (EMU_ERR_TRACE | EMU_ERR_NEGDIAG | EMU_ERR_LENGTH | EMU_ERR_DT)) return die(ctx, r, "Renormalize");
            if (r) return die(ctx, r, "step loop");
            int64_t np = 0;
            emu_num_particles(ctx, &np);
            fom += (double)np * (info.steps_done - done);
            const bool stopped = info.steps_done < next;
            done = info.steps_done;
            const int step = step0 + done;
            std::printf("Completed time step: %d t = %.17g s.  ct = %.17g cm\n", step - 1, info.time,
                        2.99792458e10 * info.time);
            const bool plot = p.write_plot_every > 0 && step % p.write_plot_every == 0;
            const bool parts = p.write_plot_particles_every > 0 && step % p.write_plot_particles_every == 0;
            if ((plot || parts) && (r = emu_write_plotfile(ctx, plot_name(step).c_str(), info.time, step, parts)))
                return die(ctx, r, "WritePlotFile");
            if (stopped) break;   // end_time reached
        }
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    std::printf("Done. \n");
    std::printf("Run time w/o initialization (seconds) = %.3f\n", secs);
    std::printf("Average number of particles advanced per microsecond = %.3f\n", secs > 0 ? fom / secs / 1e6 : 0.0);
    emu_destroy(ctx);
    return 0;
}
