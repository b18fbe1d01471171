// `artss <file.xml>`: the command line of ARTSS src/main.cpp:51-104 on the B200
// runtime -- parse, set up, run the time loop to t_end, report the loop time.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

#include "solvers.h"

int main(int argc, char **argv) {
    if (argc <= 1) {
        std::fprintf(stderr, "XML file missing\n");
        return 1;
    }
    int device = 0;
    long steps = -1;
    for (int a = 2; a < argc; a++) {
        if (!std::strcmp(argv[a], "--device") && a + 1 < argc) device = std::atoi(argv[++a]);
        else if (!std::strcmp(argv[a], "--steps") && a + 1 < argc) steps = std::atol(argv[++a]);
    }
    try {
        artss::settings::Settings st = artss::settings::parse_settings_file(argv[1]);
        artss::Runtime rt(st, device);
        artss::SolverController sc(rt);
        artss::TimeIntegration ti(rt, sc);
        std::printf("Start calculating and timing...\n");
        artss::check(artss_ctx_sync(rt.ctx()), "set-up");
        auto t0 = std::chrono::steady_clock::now();
        const int64_t n = ti.run(steps);
        artss::check(artss_ctx_sync(rt.ctx()), "time loop");
        auto t1 = std::chrono::steady_clock::now();
        const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        std::printf("Done calculating and timing ...\n");
        std::printf("Global Time: %.0fms (%lld steps, %.3e cell-updates/s)\n", ms, (long long) n,
                    (double) rt.geometry().inner(0).size() * (double) n / (ms * 1e-3));
    } catch (const std::exception &ex) {
        std::fprintf(stderr, "%s\n", ex.what());
        return 2;
    }
    return 0;
}
