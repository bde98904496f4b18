// FDTD-B200 -- drop-in for the solver executable that AlpineEM's master.py
// launches as `./<solver> inputs.txt` (main_fdtd/master.py:438-441).
// Reads the deck named by its one argument, runs every time step on the GPU
// and writes the reference's output files next to the current directory.
// `--kmax` (or a program name containing "kmax") selects the constant-k
// periodic grammar, which the reference builds as a separate binary.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/alpineem_b200.h"

int main(int argc, char** argv) {
    int mode = std::strstr(argv[0], "kmax") ? AEM_KMAX : AEM_STANDARD;
    const char* deck = nullptr;
    for (int a = 1; a < argc; a++) {
        if (!std::strcmp(argv[a], "--kmax")) mode = AEM_KMAX;
        else deck = argv[a];
    }
    if (!deck) {
        std::fprintf(stderr, "usage: %s [--kmax] inputs.txt\n", argv[0]);
        return 2;
    }
    using clk = std::chrono::steady_clock;
    auto t0 = clk::now();
    std::printf("Reading in the inputs file and setting up the simulation...\n");
    aem_handle* h = nullptr;
    if (aem_create_from_file(deck, mode, nullptr, &h) != AEM_OK) {
        std::printf("%s\n", aem_last_error(nullptr));
        return 1;
    }
    int done = 0, total = 0;
    aem_steps(h, &done, &total);
    auto t1 = clk::now();
    std::printf("Setup is finished. Time to complete was %.3f seconds.\n", std::chrono::duration<double>(t1 - t0).count());
    std::printf("Starting main FDTD algorithm...\n");
    for (int n = 0; n < total; n += 100) {
        int k = total - n < 100 ? total - n : 100;
        if (aem_run(h, k) != AEM_OK) {
            std::printf("%s\n", aem_last_error(h));
            aem_destroy(h);
            return 1;
        }
        if (k == 100) {
            aem_synchronize(h);
            std::printf("%d of %d time steps\n", n + k, total);
        }
    }
    if (aem_synchronize(h) != AEM_OK) {
        std::printf("%s\n", aem_last_error(h));
        aem_destroy(h);
        return 1;
    }
    auto t2 = clk::now();
    double secs = std::chrono::duration<double>(t2 - t1).count();
    std::printf("Finished main FDTD algorithm. Time to complete was %.3f seconds.\n", secs);
    // the reference's own Mcells/s definition, fdtd_solver.f90:8315-8316
    int g[3];
    aem_grid(h, g);
    double cells = (double)(g[0] - 1) * (g[1] - 1) * (g[2] - 1);
    std::printf("Average of %.2f Mcells per second.\n", 1.0e-6 * cells * total / secs);
    std::printf("Post processing some data...\n");
    if (aem_write_outputs(h) != AEM_OK) {
        std::printf("%s\n", aem_last_error(h));
        aem_destroy(h);
        return 1;
    }
    std::printf("Finished post processing. Time to complete was %.3f seconds.\n",
                std::chrono::duration<double>(clk::now() - t2).count());
    aem_destroy(h);
    return 0;
}
