// params.cpp -- input.in keyword parser with the reference's semantics
// (read_parameters, src/parameters.cpp:7-118; finalize_parameters_after_read,
// src/parameters.cpp:120-160), returning error codes instead of aborting.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

#include "how_mhd.h"

namespace how { void set_error(const char* fmt, ...); }

namespace {

template <class T>
bool read_value(std::istream& in, T& v) {
    in >> v;
    return !in.fail();
}

int bc_code(const std::string& s, int* out) {
    if (s == "periodic") { *out = HOW_BC_PERIODIC; return 0; }
    if (s == "open") { *out = HOW_BC_OPEN; return 0; }
    return -1;
}

int parse_stream(std::istream& in, how_params* p) {
    std::string key;
    std::string sval;
    while (in >> key) {
        if (key.empty()) continue;
        bool ok = true;
        if (key[0] == '#') {
            std::string dummy;
            std::getline(in, dummy);
        } else if (key == "nx" || key == "gnx") ok = read_value(in, p->nx);
        else if (key == "ny" || key == "gny") ok = read_value(in, p->ny);
        else if (key == "nz" || key == "gnz") ok = read_value(in, p->nz);
        else if (key == "nt") ok = read_value(in, p->nt);
        else if (key == "nstep") ok = read_value(in, p->nstep);
        else if (key == "ntime") ok = read_value(in, p->ntime);
        else if (key == "xsize") ok = read_value(in, p->xsize);
        else if (key == "ysize") ok = read_value(in, p->ysize);
        else if (key == "zsize") ok = read_value(in, p->zsize);
        else if (key == "gam") ok = read_value(in, p->gam);
        else if (key == "cour") ok = read_value(in, p->cour);
        else if (key == "tend") ok = read_value(in, p->tend);
        else if (key == "rhomin") ok = read_value(in, p->rhomin);
        else if (key == "pgmin") ok = read_value(in, p->pgmin);
        else if (key == "x1bc" || key == "x2bc" || key == "x3bc") {
            ok = read_value(in, sval);
            const int ax = key[1] - '1';
            if (ok && bc_code(sval, &p->bc[ax]) != 0) {
                how::set_error("unknown %s = %s (periodic|open)", key.c_str(), sval.c_str());
                return HOW_ERR_PARSE;
            }
        } else if (key == "problem") {
            ok = read_value(in, sval);
            if (ok) {
                if (sval.size() >= sizeof(p->problem)) {
                    how::set_error("problem name too long: %s", sval.c_str());
                    return HOW_ERR_PARSE;
                }
                std::snprintf(p->problem, sizeof(p->problem), "%s", sval.c_str());
            }
        } else if (key == "output_format") {
            ok = read_value(in, sval);
            if (ok) std::snprintf(p->output_format, sizeof(p->output_format), "%s", sval.c_str());
        } else if (key == "px") ok = read_value(in, p->px);
        else if (key == "py") ok = read_value(in, p->py);
        else if (key == "pz") ok = read_value(in, p->pz);
        // ---- keys added by this implementation
        else if (key == "precision") {
            ok = read_value(in, sval);
            if (ok) {
                if (sval == "fp64") p->precision = HOW_PREC_FP64;
                else if (sval == "mixed") p->precision = HOW_PREC_MIXED;
                else { how::set_error("unknown precision %s (fp64|mixed)", sval.c_str()); return HOW_ERR_PARSE; }
            }
        } else if (key == "router") {
            ok = read_value(in, sval);
            if (ok) {
                if (sval == "off" || sval == "0") p->router = 0;
                else if (sval == "on" || sval == "1") p->router = 1;
                else { how::set_error("unknown router %s (off|on)", sval.c_str()); return HOW_ERR_PARSE; }
            }
        } else if (key == "ct_avg") {
            int v = 0;
            ok = read_value(in, v);
            if (ok) {
                if (v != 2 && v != 4) { how::set_error("ct_avg must be 2 or 4, got %d", v); return HOW_ERR_PARSE; }
                p->ct_avg = v;
            }
        } else if (key == "seed") {
            unsigned long long s = 0;
            ok = read_value(in, s);
            p->seed = s;
        } else if (key.size() == 4 && key.compare(0, 3, "par") == 0 && key[3] >= '0' && key[3] <= '7') {
            ok = read_value(in, p->problem_par[key[3] - '0']);
        } else {
            // unknown key: warn and skip the rest of the line (src/parameters.cpp:112-116)
            std::cerr << "Warning: unknown parameter " << key << "\n";
            std::string dummy;
            std::getline(in, dummy);
        }
        if (!ok) {
            how::set_error("missing or invalid value for key %s", key.c_str());
            return HOW_ERR_PARSE;
        }
    }
    return how_finalize_params(p);
}

}  // namespace

extern "C" {

// defaults of read_parameters (src/parameters.cpp:9-33)
int how_params_default(how_params* p) {
    if (!p) return HOW_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    p->xsize = p->ysize = p->zsize = 1.0;
    p->gam = 5.0 / 3.0;
    p->cour = 0.4;
    p->rhomin = 1.0e-12;
    p->pgmin = 1.0e-12;
    p->bc[0] = p->bc[1] = p->bc[2] = HOW_BC_PERIODIC;
    std::snprintf(p->output_format, sizeof(p->output_format), "dat");
    p->precision = HOW_PREC_FP64;
    p->router = 0;
    p->ct_avg = 2;
    p->seed = 12345;
    return HOW_OK;
}

// finalize_parameters_after_read (src/parameters.cpp:120-160)
int how_finalize_params(how_params* p) {
    if (!p) return HOW_ERR_ARG;
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0) {
        how::set_error("global grid size must be positive: nx=%d ny=%d nz=%d", p->nx, p->ny, p->nz);
        return HOW_ERR_PARSE;
    }
    if (p->nt <= 0) { how::set_error("nt must be positive. nt = %d", p->nt); return HOW_ERR_PARSE; }
    if (!(p->tend > 0.0)) { how::set_error("tend must be positive. tend = %g", p->tend); return HOW_ERR_PARSE; }
    p->dx = p->xsize / (double)p->nx;
    p->dy = p->ysize / (double)p->ny;
    p->dz = p->zsize / (double)p->nz;
    return HOW_OK;
}

int how_parse_input(const char* path, how_params* p) {
    if (!path || !p) { how::set_error("null argument"); return HOW_ERR_ARG; }
    std::ifstream in(path);
    if (!in) { how::set_error("cannot open input file: %s", path); return HOW_ERR_ARG; }
    how_params_default(p);
    return parse_stream(in, p);
}

int how_parse_input_string(const char* text, how_params* p) {
    if (!text || !p) { how::set_error("null argument"); return HOW_ERR_ARG; }
    std::istringstream in(text);
    how_params_default(p);
    return parse_stream(in, p);
}

}  // extern "C"
