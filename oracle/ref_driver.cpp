// ref_driver.cpp -- oracle driver around the UNMODIFIED reference sources.
// TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Built by oracle/Makefile together with the reference's src/*.cpp (minus
// main.cpp) against the project-written Kokkos shim in
// oracle/kokkos_shim/.  It reproduces the reference driver's set-up
// (src/main.cpp:84-130) and time loop (src/main.cpp:158-223), and dumps raw
// state so the tests can compare the B200 path with the reference's own
// arithmetic.
//
// usage:
//   how_ref <input.in> <out.bin> [--steps K] [--state in.bin] [--dump-stages]
//           [--sweep x|y|z --dt DT] [--threads N] [--time-only]
//           [--output STEP TIME]
//
//   default      : main-loop semantics (tstep, dt clamp to the output time,
//                  ssprk) until tend, or until K hydro steps when --steps K.
//   --state F    : take q(0) (and face B if present) from F instead of the
//                  problem registry (used for problems the reference lacks and
//                  for randomised states).
//   --dump-stages: run ONE step with the body of ssprk (src/ssprk.cpp:1277-1329)
//                  restated here call-for-call so every stage can be dumped.
//   --sweep d    : only stage iw=1's copy/bound and ONE directional sweep with
//                  the given dt; dumps q(1) and the two CT flux arrays it fills.
//   --time-only  : no dump; prints wall seconds and zone-cycles/s as JSON.
//   --output S T : only the reference's own output(q, par, S, T)
//                  (src/output.cpp:555-572) on the initial or --state q(0):
//                  output/dumpSSSSSS.dat or .vts in the working directory, in
//                  the input's output_format.  <out.bin> is not written.
//   --piece R NZ KS : with --output, write what MPI rank R of a z-split
//                  writes for its slab: after setup_mpi_domain the local
//                  sizes and offsets its decomposition would set (nz = NZ,
//                  kstart = KS, cart_rank = R; gnz, dz stay the input's), so
//                  --state holds the slab (nx+6, ny+6, NZ+6).  The serial
//                  build names the file without the _rank suffix; its bytes
//                  are the MPI rank's (src/output.cpp:21-38 is the only
//                  USE_MPI difference in the writer).
//
// Dump format: a sequence of records
//   u32 name_len, name bytes, u32 ndim, u64 dims[ndim], f64 data[prod(dims)]
// Arrays keep the reference's layout (stage-less: var, i, j, k with k fastest).
#include <Kokkos_Core.hpp>

#include "parameters.hpp"
#include "mpi_domain.hpp"
#include "problem.hpp"
#include "tstep.hpp"
#include "ssprk.hpp"
#include "fluxct.hpp"
#include "bound.hpp"
#include "prot.hpp"
#include "output.hpp"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>
#include <omp.h>

// Non-static reference functions (src/ssprk.cpp) not declared in its headers.
struct RKCoeff { double k1, k2, k3, k4, k5; };   // identical to src/ssprk.cpp:62-64
RKCoeff get_rk_coeff(const int iw);
void copy_stage(Kokkos::View<double*****> q, const int dst, const int src, const Parameters& par);
void prepare_stage5(Kokkos::View<double*****> q, const RKCoeff c, const Parameters& par);
void x_sweep(Kokkos::View<double*****> q, int iw, const RKCoeff c, const Parameters& par, CTFluxes& ct);
void y_sweep(Kokkos::View<double*****> q, int iw, const Parameters& par, CTFluxes& ct);
void z_sweep(Kokkos::View<double*****> q, int iw, const Parameters& par, CTFluxes& ct);

namespace {

struct Writer {
    std::FILE* f = nullptr;
    explicit Writer(const std::string& path) {
        f = std::fopen(path.c_str(), "wb");
        if (!f) { std::fprintf(stderr, "cannot open %s\n", path.c_str()); std::exit(2); }
    }
    ~Writer() { if (f) std::fclose(f); }
    void rec(const std::string& name, const std::vector<uint64_t>& dims, const double* data) {
        uint32_t nl = (uint32_t)name.size();
        std::fwrite(&nl, 4, 1, f);
        std::fwrite(name.data(), 1, nl, f);
        uint32_t nd = (uint32_t)dims.size();
        std::fwrite(&nd, 4, 1, f);
        uint64_t n = 1;
        for (auto d : dims) { std::fwrite(&d, 8, 1, f); n *= d; }
        std::fwrite(data, 8, n, f);
    }
};

struct Reader {
    struct Rec { std::vector<uint64_t> dims; std::vector<double> data; };
    std::vector<std::pair<std::string, Rec>> recs;
    explicit Reader(const std::string& path) {
        std::FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) { std::fprintf(stderr, "cannot open %s\n", path.c_str()); std::exit(2); }
        uint32_t nl;
        while (std::fread(&nl, 4, 1, f) == 1) {
            std::string name(nl, '\0');
            if (std::fread(&name[0], 1, nl, f) != nl) break;
            uint32_t nd; if (std::fread(&nd, 4, 1, f) != 1) break;
            Rec r; r.dims.resize(nd);
            uint64_t n = 1;
            for (uint32_t i = 0; i < nd; ++i) { if (std::fread(&r.dims[i], 8, 1, f) != 1) break; n *= r.dims[i]; }
            r.data.resize(n);
            if (std::fread(r.data.data(), 8, n, f) != n) break;
            recs.push_back({name, std::move(r)});
        }
        std::fclose(f);
    }
    const Rec* find(const std::string& n) const {
        for (auto& p : recs) if (p.first == n) return &p.second;
        return nullptr;
    }
};

std::vector<double> stage_of(Kokkos::View<double*****> q, int stage) {
    const size_t n = q.extent(1) * q.extent(2) * q.extent(3) * q.extent(4);
    std::vector<double> out(n);
    std::memcpy(out.data(), &q(stage, 0, 0, 0, 0), n * sizeof(double));
    return out;
}

std::vector<double> bstage_of(Kokkos::View<double****> b, int stage) {
    const size_t n = b.extent(1) * b.extent(2) * b.extent(3);
    std::vector<double> out(n);
    std::memcpy(out.data(), &b(stage, 0, 0, 0), n * sizeof(double));
    return out;
}

void dump_state(Writer& w, const std::string& tag, Kokkos::View<double*****> q, int stage,
                const Parameters& par) {
    const uint64_t P0 = par.nx + 6, P1 = par.ny + 6, P2 = par.nz + 6;
    auto qs = stage_of(q, stage);
    w.rec(tag + "q", {8, P0, P1, P2}, qs.data());
    auto bx = bstage_of(bxb, stage), by = bstage_of(byb, stage), bz = bstage_of(bzb, stage);
    w.rec(tag + "bxb", {P0, P1, P2}, bx.data());
    w.rec(tag + "byb", {P0, P1, P2}, by.data());
    w.rec(tag + "bzb", {P0, P1, P2}, bz.data());
}

void dump_ct(Writer& w, const std::string& name, Kokkos::View<double***> a) {
    w.rec(name, {a.extent(0), a.extent(1), a.extent(2)}, a.data());
}

// Body of ssprk() (src/ssprk.cpp:1277-1329), restated call-for-call with the
// reference's own functions so that each stage can be dumped.
void ssprk_dump_stages(Kokkos::View<double*****> q, Parameters& par, Writer& w) {
    CTFluxes ct(par);
    for (int iw = 1; iw <= 5; ++iw) {
        zero_ct_fluxes(ct);
        RKCoeff c = get_rk_coeff(iw);
        if (iw <= 4) { copy_stage(q, iw, 0, par); copy_bfield_stage(iw, 0, par); }
        else { prepare_stage5(q, c, par); prepare_bfield_stage5(c.k1, c.k4, c.k5, par); }
        bound(q, iw - 1, par);
        if (iw == 5) bound(q, iw, par);
        par.dtdx = c.k2 * par.dt / par.dx;
        par.dtdy = c.k2 * par.dt / par.dy;
        par.dtdz = c.k2 * par.dt / par.dz;
        if (par.nx > 1) x_sweep(q, iw, c, par, ct);
        if (par.ny > 1) y_sweep(q, iw, par, ct);
        if (par.nz > 1) z_sweep(q, iw, par, ct);
        std::string tag = "stage" + std::to_string(iw) + "_";
        {
            auto qs = stage_of(q, iw);
            w.rec(tag + "presweep_q", {8, (uint64_t)par.nx + 6, (uint64_t)par.ny + 6, (uint64_t)par.nz + 6}, qs.data());
        }
        bound_bfield(iw - 1, par);
        fluxct(q, iw, c.k1, c.k3, par, ct);
        dump_ct(w, tag + "fsy", ct.fsy); dump_ct(w, tag + "fsz", ct.fsz);
        dump_ct(w, tag + "gsx", ct.gsx); dump_ct(w, tag + "gsz", ct.gsz);
        dump_ct(w, tag + "hsx", ct.hsx); dump_ct(w, tag + "hsy", ct.hsy);
        dump_ct(w, tag + "Ox", ct.Ox); dump_ct(w, tag + "Oy", ct.Oy); dump_ct(w, tag + "Oz", ct.Oz);
        prot(q, iw, par);
        bound(q, iw, par);
        bound_bfield(iw, par);
        dump_state(w, tag, q, iw, par);
    }
    copy_stage(q, 0, 5, par);
    copy_bfield_to_stage0(par);
}

} // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: how_ref <input.in> <out.bin> [options]\n");
        return 2;
    }
    std::string input = argv[1], out = argv[2];
    long max_steps = -1, warmup = 0;
    std::string state_path, sweep;
    double sweep_dt = 0.0;
    bool dump_stages = false, time_only = false, do_output = false;
    int piece_rank = -1, piece_nz = 0, piece_kstart = 0;
    int out_step = 0;
    double out_time = 0.0;
    for (int a = 3; a < argc; ++a) {
        std::string s = argv[a];
        if (s == "--steps" && a + 1 < argc) max_steps = std::atol(argv[++a]);
        else if (s == "--state" && a + 1 < argc) state_path = argv[++a];
        else if (s == "--dump-stages") dump_stages = true;
        else if (s == "--sweep" && a + 1 < argc) sweep = argv[++a];
        else if (s == "--dt" && a + 1 < argc) sweep_dt = std::atof(argv[++a]);
        else if (s == "--threads" && a + 1 < argc) omp_set_num_threads(std::atoi(argv[++a]));
        else if (s == "--time-only") time_only = true;
        else if (s == "--warmup" && a + 1 < argc) warmup = std::atol(argv[++a]);
        else if (s == "--piece" && a + 3 < argc) {
            piece_rank = std::atoi(argv[++a]);
            piece_nz = std::atoi(argv[++a]);
            piece_kstart = std::atoi(argv[++a]);
        }
        else if (s == "--output" && a + 2 < argc) {
            do_output = true;
            out_step = std::atoi(argv[++a]);
            out_time = std::atof(argv[++a]);
        }
        else { std::fprintf(stderr, "unknown option %s\n", s.c_str()); return 2; }
    }

    Kokkos::initialize(argc, argv);
    int rc = 0;
    {
        Parameters par;
        std::ifstream in(input);
        if (!in) { std::fprintf(stderr, "cannot open input %s\n", input.c_str()); return 2; }
        // src/main.cpp:84-86
        read_parameters(in, par);
        finalize_parameters_after_read(par);
        setup_mpi_domain(par);
        if (piece_rank >= 0) {
            par.nz = piece_nz;
            par.kstart = piece_kstart;
            par.cart_rank = piece_rank;
        }

        // src/main.cpp:114-120
        Kokkos::View<double*****> q("q", 6, 8, par.nx + 6, par.ny + 6, par.nz + 6);
        const size_t P0 = par.nx + 6, P1 = par.ny + 6, P2 = par.nz + 6;
        const size_t PV = P0 * P1 * P2;

        bool have_faceb = false;
        std::vector<double> fb[3];
        if (!state_path.empty()) {
            Reader r(state_path);
            const auto* rq = r.find("q");
            if (!rq || rq->data.size() != 8 * PV) {
                std::fprintf(stderr, "state file lacks a q record of 8x%zux%zux%zu\n", P0, P1, P2);
                return 2;
            }
            std::memcpy(&q(0, 0, 0, 0, 0), rq->data.data(), 8 * PV * sizeof(double));
            const char* nm[3] = {"bxb", "byb", "bzb"};
            have_faceb = true;
            for (int c = 0; c < 3; ++c) {
                const auto* rb = r.find(nm[c]);
                if (!rb || rb->data.size() != PV) { have_faceb = false; break; }
                fb[c] = rb->data;
            }
        } else {
            init_problem(q, par);   // src/main.cpp:125
        }
        bound(q, 0, par);           // src/main.cpp:127
        allocate_bfield_ct(par);    // src/main.cpp:129
        if (have_faceb) {
            std::memcpy(&bxb(0, 0, 0, 0), fb[0].data(), PV * sizeof(double));
            std::memcpy(&byb(0, 0, 0, 0), fb[1].data(), PV * sizeof(double));
            std::memcpy(&bzb(0, 0, 0, 0), fb[2].data(), PV * sizeof(double));
            bound_bfield(0, par);
        } else {
            initialize_bfield_from_q(q, par);   // src/main.cpp:130
        }

        if (do_output) {
            output(q, par, out_step, out_time);   // src/output.cpp:555-572
        } else if (!sweep.empty()) {
            Writer w(out);
            dump_state(w, "init_", q, 0, par);
            CTFluxes ct(par);
            zero_ct_fluxes(ct);
            RKCoeff c = get_rk_coeff(1);
            copy_stage(q, 1, 0, par);
            copy_bfield_stage(1, 0, par);
            bound(q, 0, par);
            par.dt = sweep_dt;
            par.dtdx = c.k2 * par.dt / par.dx;
            par.dtdy = c.k2 * par.dt / par.dy;
            par.dtdz = c.k2 * par.dt / par.dz;
            if (sweep == "x") { x_sweep(q, 1, c, par, ct); dump_ct(w, "fsy", ct.fsy); dump_ct(w, "fsz", ct.fsz); }
            else if (sweep == "y") { y_sweep(q, 1, par, ct); dump_ct(w, "gsz", ct.gsz); dump_ct(w, "gsx", ct.gsx); }
            else if (sweep == "z") { z_sweep(q, 1, par, ct); dump_ct(w, "hsx", ct.hsx); dump_ct(w, "hsy", ct.hsy); }
            else { std::fprintf(stderr, "bad --sweep %s\n", sweep.c_str()); return 2; }
            auto q1 = stage_of(q, 1);
            w.rec("q1", {8, P0, P1, P2}, q1.data());
        } else if (dump_stages) {
            Writer w(out);
            dump_state(w, "init_", q, 0, par);
            tstep(q, par);
            double dtv = par.dt;
            w.rec("dt", {1}, &dtv);
            ssprk_dump_stages(q, par, w);
            dump_state(w, "final_", q, 0, par);
        } else {
            // src/main.cpp:132-223 without output and logging.
            double time = 0.0;
            const double dtout = par.tend / static_cast<double>(par.nt);
            std::vector<double> dts;
            long steps = 0;
            bool stop = false;
            // --warmup W: W untimed steps first (same loop), then K timed
            double t0 = omp_get_wtime();
            long timed_from = 0;
            for (int out_step = 1; out_step <= par.nt && !stop; ++out_step) {
                const double target_time = dtout * static_cast<double>(out_step);
                while (time < target_time) {
                    if (max_steps >= 0 && steps >= max_steps + warmup) { stop = true; break; }
                    if (steps == warmup && timed_from == 0) { t0 = omp_get_wtime(); timed_from = steps; }
                    tstep(q, par);
                    if (time + par.dt > target_time) par.dt = target_time - time;
                    if (par.dt <= 0.0) { rc = 3; stop = true; break; }
                    ssprk(q, par);
                    time += par.dt;
                    dts.push_back(par.dt);
                    ++steps;
                    if (!std::isfinite(time)) { rc = 4; stop = true; break; }
                }
            }
            double wall = omp_get_wtime() - t0;
            const long timed = steps - timed_from;
            if (time_only) {
                const double zones = (double)par.nx * par.ny * par.nz;
                std::printf("{\"steps\": %ld, \"warmup\": %ld, \"wall_s\": %.6f, \"zone_cycles_per_s\": %.6e, "
                            "\"threads\": %d, \"time\": %.17g}\n",
                            timed, warmup, wall, timed > 0 ? zones * timed / wall : 0.0,
                            omp_get_max_threads(), time);
            } else {
                Writer w(out);
                double meta[3] = {time, (double)steps, wall};
                w.rec("meta", {3}, meta);
                if (!dts.empty()) w.rec("dt", {dts.size()}, dts.data());
                dump_state(w, "", q, 0, par);
            }
        }
        deallocate_bfield_ct();
    }
    Kokkos::finalize();
    return rc;
}
