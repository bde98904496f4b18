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

// aem_run.json in the current directory: one JSON object with the run's
// timings (the same three phases the stdout lines report), the reference's
// Mcells/s, the algorithmic bytes moved per step and the achieved rate, the
// device memory held, host<->device transfers and kernel launches.  The
// reference prints only the stdout lines; no reference tool reads this file.
static void write_run_record(aem_handle* h, const char* deck, int mode, const int g[3], double cells, int steps,
                             double setup_s, double loop_s, double post_s) {
    long long lcells = 0, launches = 0, h2d = 0, d2h = 0;
    double bytes = 0.0;
    size_t dev = 0;
    aem_workload(h, &lcells, &bytes);
    aem_launch_count(h, &launches);
    aem_transfer_bytes(h, &h2d, &d2h);
    aem_device_bytes(h, &dev);
    FILE* f = std::fopen("aem_run.json", "w");
    if (!f) return;
    std::string dk;
    for (const char* c = deck; *c; c++) {
        if (*c == '"' || *c == '\\') dk += '\\';
        dk += *c;
    }
    std::fprintf(f,
                 "{\"solver\": \"FDTD-B200\", \"version\": %d, \"deck\": \"%s\", \"mode\": \"%s\", "
                 "\"grid\": [%d, %d, %d], \"steps\": %d, \"setup_s\": %.6f, \"loop_s\": %.6f, \"post_s\": %.6f, "
                 "\"mcells_per_s\": %.3f, \"storage_cells\": %lld, \"algorithmic_bytes_per_step\": %.0f, "
                 "\"achieved_gb_per_s\": %.3f, \"device_bytes\": %zu, \"h2d_bytes\": %lld, \"d2h_bytes\": %lld, "
                 "\"kernel_launches\": %lld}\n",
                 aem_version(), dk.c_str(), mode == AEM_KMAX ? "kmax" : "standard", g[0], g[1], g[2], steps, setup_s,
                 loop_s, post_s, loop_s > 0 ? 1.0e-6 * cells * steps / loop_s : 0.0, lcells, bytes,
                 loop_s > 0 ? bytes * steps / loop_s / 1e9 : 0.0, dev, h2d, d2h, launches);
    std::fclose(f);
}

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
    const double post = std::chrono::duration<double>(clk::now() - t2).count();
    std::printf("Finished post processing. Time to complete was %.3f seconds.\n", post);
    write_run_record(h, deck, mode, g, cells, total, std::chrono::duration<double>(t1 - t0).count(), secs, post);
    aem_destroy(h);
    return 0;
}
