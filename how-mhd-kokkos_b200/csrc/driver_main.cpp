// driver_main.cpp -- how_mhd_b200: the driver of src/main.cpp:25-248 on the
// C ABI.  Reads input.in (argv[1] or stdin), initialises the registered
// problem, and advances through the nt output intervals with the reference's
// dt clamp, logging one line per interval.  Like the reference it writes a
// dump file of the initial state and of each interval's end
// (src/main.cpp:144, 225) into output/, in the input's output_format
// ("none" skips them); each dump is written while the next interval runs.
// --dump FILE also writes the final q(0) in the reference layout as raw
// doubles.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <iterator>
#include <string>
#include <vector>

#include "how_mhd.h"

int main(int argc, char** argv) {
    how_params p;
    int rc;
    std::string dump;
    const char* input = nullptr;
    for (int a = 1; a < argc; ++a) {
        if (std::strcmp(argv[a], "--dump") == 0 && a + 1 < argc) dump = argv[++a];
        else input = argv[a];
    }
    if (input) rc = how_parse_input(input, &p);
    else {
        std::string text((std::istreambuf_iterator<char>(std::cin)), std::istreambuf_iterator<char>());
        rc = how_parse_input_string(text.c_str(), &p);
    }
    if (rc) { std::fprintf(stderr, "Error: %s\n", how_last_error()); return 1; }
    how_ctx* ctx = nullptr;
    if ((rc = how_create(&p, &ctx)) || (rc = how_init_problem(ctx))) {
        std::fprintf(stderr, "Error: %s\n", how_last_error());
        return 1;
    }
    std::printf("problem = %s  grid = %d x %d x %d  gam = %g  cour = %g  tend = %g  nt = %d\n",
                p.problem, p.nx, p.ny, p.nz, p.gam, p.cour, p.tend, p.nt);
    double time = 0.0;
    long total = 0;
    const double dtout = p.tend / (double)p.nt;
    if ((rc = how_output_async(ctx, 0, time, "output"))) {
        std::fprintf(stderr, "Error: %s\n", how_last_error());
        how_destroy(ctx);
        return 1;
    }
    std::printf("dtout = %g\noutput step = 0 time = 0\n", dtout);
    for (int out = 1; out <= p.nt; ++out) {
        // the interval is advanced one how_run step at a time, until the
        // time reaches its end (how_run clamps the last step to it,
        // src/main.cpp:170-172), so each output lands on its time
        long steps = 0;
        std::vector<double> dts(1);
        const double target = dtout * out;
        while (time < target) {
            long s = 0;
            rc = how_run(ctx, &time, 1, &s, dts.data(), 1);
            steps += s;
            if (rc) break;
            if (s == 0) break;
        }
        total += steps;
        if (rc) { std::fprintf(stderr, "Error: %s\n", how_last_error()); break; }
        if ((rc = how_output_async(ctx, out, time, "output"))) {
            std::fprintf(stderr, "Error: %s\n", how_last_error());
            break;
        }
        std::printf("output step = %d time = %.10g last_dt = %.6g hydro_steps = %ld\n", out, time,
                    dts[0], steps);
    }
    const int wrc = how_output_wait(ctx);
    if (wrc) { std::fprintf(stderr, "Error: %s\n", how_last_error()); rc = wrc; }
    if (!dump.empty()) {
        std::vector<double> qh((size_t)8 * (p.nx + 6) * (p.ny + 6) * (p.nz + 6));
        if (how_get_state(ctx, 0, qh.data()) == HOW_OK) {
            std::FILE* f = std::fopen(dump.c_str(), "wb");
            if (f) { std::fwrite(qh.data(), sizeof(double), qh.size(), f); std::fclose(f); }
        }
    }
    how_destroy(ctx);
    return rc ? 1 : 0;
}
