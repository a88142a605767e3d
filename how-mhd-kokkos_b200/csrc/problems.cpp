// problems.cpp -- problem registry (register_problem / init_problem,
// src/problem.hpp:8-22, src/problem.cpp:7-37) and the built-in initial
// conditions.  Initialisers fill one stage of q in the reference layout
// (var, i, j, k), k fastest, active cells only; they run on the host.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "how_mhd.h"

namespace how { void set_error(const char* fmt, ...); }

namespace {

struct Entry { how_problem_fn fn; void* user; };

std::mutex& reg_mutex() { static std::mutex m; return m; }
std::map<std::string, Entry>& registry() { static std::map<std::string, Entry> r; return r; }

struct Q {
    double* q;
    int P0, P1, P2;
    size_t at(int v, int i, int j, int k) const {
        return (((size_t)v * P0 + i) * P1 + j) * P2 + k;
    }
    // conserved state from primitives, as every reference problem does
    // (e.g. src/problems/orszag_tang.cpp:168-186)
    void set(int i, int j, int k, double gam, double rho, double vx, double vy, double vz,
             double Bx, double By, double Bz, double pg) {
        const double Mx = rho * vx, My = rho * vy, Mz = rho * vz;
        const double vv2 = vx * vx + vy * vy + vz * vz;
        const double BB2 = Bx * Bx + By * By + Bz * Bz;
        const double E = pg / (gam - 1.0) + 0.5 * rho * vv2 + 0.5 * BB2;
        q[at(0, i, j, k)] = rho; q[at(1, i, j, k)] = Mx; q[at(2, i, j, k)] = My;
        q[at(3, i, j, k)] = Mz; q[at(4, i, j, k)] = Bx; q[at(5, i, j, k)] = By;
        q[at(6, i, j, k)] = Bz; q[at(7, i, j, k)] = E;
    }
};

Q view(double* q, const how_params* p) { return Q{q, p->nx + 6, p->ny + 6, p->nz + 6}; }

constexpr double PI_L = 3.141592653589793238462643383279502884;

// src/problems/orszag_tang.cpp:120-191
int init_orszag_tang(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    const double pi = PI_L;
#pragma omp parallel for collapse(2)
    for (int i = 3; i < p->nx + 3; ++i)
        for (int j = 3; j < p->ny + 3; ++j)
            for (int k = 3; k < p->nz + 3; ++k) {
                const double x = (static_cast<double>(i - 3) + 0.5) * p->dx;
                const double y = (static_cast<double>(j - 3) + 0.5) * p->dy;
                const double rho = 25.0 / (36.0 * pi), pg = 5.0 / (12.0 * pi);
                const double vx = -std::sin(2.0 * pi * y), vy = std::sin(2.0 * pi * x);
                const double normB = std::sqrt(4.0 * pi);
                q.set(i, j, k, p->gam, rho, vx, vy, 0.0, -std::sin(2.0 * pi * y) / normB,
                      std::sin(4.0 * pi * x) / normB, 0.0, pg);
            }
    return 0;
}

// src/problems/blast3d.cpp:9-104 (B = (0.1, 0, 0), p_in 100, p_out 1)
int init_blast3d(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    const double xc = 0.5 * p->xsize, yc = 0.5 * p->ysize, zc = 0.5 * p->zsize;
    const double r0 = 0.10 * std::fmin(p->xsize, std::fmin(p->ysize, p->zsize));
#pragma omp parallel for collapse(2)
    for (int i = 3; i < p->nx + 3; ++i)
        for (int j = 3; j < p->ny + 3; ++j)
            for (int k = 3; k < p->nz + 3; ++k) {
                const double x = (static_cast<double>(i - 3) + 0.5) * p->dx;
                const double y = (static_cast<double>(j - 3) + 0.5) * p->dy;
                const double z = (static_cast<double>(k - 3) + 0.5) * p->dz;
                const double rx = x - xc, ry = y - yc, rz = z - zc;
                const double rr = std::sqrt(rx * rx + ry * ry + rz * rz);
                q.set(i, j, k, p->gam, 1.0, 0.0, 0.0, 0.0, 0.1, 0.0, 0.0, (rr <= r0) ? 100.0 : 1.0);
            }
    return 0;
}

// src/problems/brio_wu.cpp:6-62
int init_brio_wu(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    const double xmid = 0.5 * p->xsize;
    for (int i = 3; i < p->nx + 3; ++i)
        for (int j = 3; j < p->ny + 3; ++j)
            for (int k = 3; k < p->nz + 3; ++k) {
                const double x = (static_cast<double>(i - 3) + 0.5) * p->dx;
                if (x < xmid) q.set(i, j, k, p->gam, 1.0, 0.0, 0.0, 0.0, 0.75, 1.0, 0.0, 1.0);
                else q.set(i, j, k, p->gam, 0.125, 0.0, 0.0, 0.0, 0.75, -1.0, 0.0, 0.1);
            }
    return 0;
}

// src/problems/mhd_rotor.cpp:6-113
int init_mhd_rotor(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    const double pi = PI_L;
#pragma omp parallel for collapse(2)
    for (int i = 3; i < p->nx + 3; ++i)
        for (int j = 3; j < p->ny + 3; ++j)
            for (int k = 3; k < p->nz + 3; ++k) {
                const double x = (static_cast<double>(i - 3) + 0.5) * p->dx;
                const double y = (static_cast<double>(j - 3) + 0.5) * p->dy;
                const double dx = x - 0.5, dy = y - 0.5;
                const double r = std::sqrt(dx * dx + dy * dy);
                const double r0 = 0.10, r1 = 0.115, rin = 10.0, rout = 1.0, om = 20.0;
                double rho, vx, vy;
                if (r <= r0) { rho = rin; vx = -om * dy; vy = om * dx; }
                else if (r <= r1) {
                    const double f = (r1 - r) / (r1 - r0);
                    rho = rout + f * (rin - rout);
                    vx = f * (-om * dy);
                    vy = f * (om * dx);
                } else { rho = rout; vx = 0.0; vy = 0.0; }
                q.set(i, j, k, p->gam, rho, vx, vy, 0.0, 5.0 / std::sqrt(4.0 * pi), 0.0, 0.0, 1.0);
            }
    return 0;
}

// src/problems/uniform.cpp:6-28
int init_uniform(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    for (int i = 3; i < p->nx + 3; ++i)
        for (int j = 3; j < p->ny + 3; ++j)
            for (int k = 3; k < p->nz + 3; ++k) {
                const double v[8] = {1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0};
                for (int m = 0; m < 8; ++m) q.q[q.at(m, i, j, k)] = v[m];
            }
    return 0;
}

// src/problems/mpi_smooth3d.cpp:9-97 (serial offsets are zero)
int init_mpi_smooth3d(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    const double pi = PI_L;
    const double Lx = p->xsize, Ly = p->ysize, Lz = p->zsize;
#pragma omp parallel for collapse(2)
    for (int i = 3; i < p->nx + 3; ++i)
        for (int j = 3; j < p->ny + 3; ++j)
            for (int k = 3; k < p->nz + 3; ++k) {
                const double x = (static_cast<double>(i - 3) + 0.5) * p->dx;
                const double y = (static_cast<double>(j - 3) + 0.5) * p->dy;
                const double z = (static_cast<double>(k - 3) + 0.5) * p->dz;
                const double sx = std::sin(2.0 * pi * x / Lx), sy = std::sin(2.0 * pi * y / Ly);
                const double sz = std::sin(2.0 * pi * z / Lz);
                const double cx = std::cos(2.0 * pi * x / Lx), cy = std::cos(2.0 * pi * y / Ly);
                const double cz = std::cos(2.0 * pi * z / Lz);
                q.set(i, j, k, p->gam, 1.0 + 0.05 * sx * sy * sz, 0.10 + 0.01 * cy * cz,
                      0.05 + 0.01 * cz * cx, 0.02 + 0.01 * cx * cy, 0.10 + 0.005 * sy * sz,
                      0.08 + 0.005 * sz * sx, 0.06 + 0.005 * sx * sy, 1.0 + 0.02 * cx * cy * cz);
            }
    return 0;
}

// ---------------------------------------------------------------- new problems
double par_or(const how_params* p, int i, double dflt) {
    return p->problem_par[i] != 0.0 ? p->problem_par[i] : dflt;
}

// alfven3d: circularly polarised Alfven wave, an exact nonlinear solution of
// ideal MHD.  Wave vector k = 2 pi (1/Lx, 1/Ly, 1/Lz) over the axes with more
// than one cell (the box diagonal of the unit cube: wavelength 1/sqrt 3).
// In the frame (e1 = k/|k|, e2, e3): B = B_par e1 + A (sin phi e2 + cos phi e3),
// v = -(A / sqrt rho)(sin phi e2 + cos phi e3), phi = k.x; it travels along
// +e1 at v_A = B_par / sqrt(rho).  par0 = A (0.1), par1 = B_par (1),
// par2 = rho (1), par3 = p (0.1).
int init_alfven3d(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    const double A = par_or(p, 0, 0.1), Bpar = par_or(p, 1, 1.0);
    const double rho = par_or(p, 2, 1.0), pg = par_or(p, 3, 0.1);
    const double k[3] = {p->nx > 1 ? 2.0 * PI_L / p->xsize : 0.0, p->ny > 1 ? 2.0 * PI_L / p->ysize : 0.0,
                         p->nz > 1 ? 2.0 * PI_L / p->zsize : 0.0};
    const double kk = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    if (kk == 0.0) { how::set_error("alfven3d needs at least one axis with n > 1"); return -1; }
    double e1[3] = {k[0] / kk, k[1] / kk, k[2] / kk};
    // e2 = e1 x z_hat (or e1 x y_hat when e1 || z), normalised; e3 = e1 x e2
    double e2[3] = {e1[1], -e1[0], 0.0};
    double n2 = std::sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    if (n2 < 1e-6) { e2[0] = -e1[2]; e2[1] = 0.0; e2[2] = e1[0]; n2 = std::sqrt(e2[0] * e2[0] + e2[2] * e2[2]); }
    for (double& x : e2) x /= n2;
    const double e3[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const double sr = std::sqrt(rho);
#pragma omp parallel for collapse(2)
    for (int i = 3; i < p->nx + 3; ++i)
        for (int j = 3; j < p->ny + 3; ++j)
            for (int k3 = 3; k3 < p->nz + 3; ++k3) {
                const double x = (static_cast<double>(i - 3) + 0.5) * p->dx;
                const double y = (static_cast<double>(j - 3) + 0.5) * p->dy;
                const double z = (static_cast<double>(k3 - 3) + 0.5) * p->dz;
                const double ph = k[0] * x + k[1] * y + k[2] * z;
                const double s = std::sin(ph), c = std::cos(ph);
                double B[3], v[3];
                for (int d = 0; d < 3; ++d) {
                    const double bt = A * (s * e2[d] + c * e3[d]);
                    B[d] = Bpar * e1[d] + bt;
                    v[d] = -bt / sr;
                }
                q.set(i, j, k3, p->gam, rho, v[0], v[1], v[2], B[0], B[1], B[2], pg);
            }
    return 0;
}

// blast3d_b: the 3-D blast of the benchmark workload -- rho = par4 (1),
// p = par0 (10) inside r < par2 (0.1) of the box centre and par1 (0.1)
// outside, v = 0, uniform B = par3 (1) * (1, 1, 0) / sqrt 2.  The reference's
// blast3d (B = (0.1,0,0), p 100/1) keeps its own name.
int init_blast3d_b(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    const double pin = par_or(p, 0, 10.0), pout = par_or(p, 1, 0.1), r0 = par_or(p, 2, 0.1);
    const double Bm = par_or(p, 3, 1.0), rho = par_or(p, 4, 1.0);
    const double b = Bm / std::sqrt(2.0);
    const double xc = 0.5 * p->xsize, yc = 0.5 * p->ysize, zc = 0.5 * p->zsize;
#pragma omp parallel for collapse(2)
    for (int i = 3; i < p->nx + 3; ++i)
        for (int j = 3; j < p->ny + 3; ++j)
            for (int k = 3; k < p->nz + 3; ++k) {
                const double x = (static_cast<double>(i - 3) + 0.5) * p->dx - xc;
                const double y = (static_cast<double>(j - 3) + 0.5) * p->dy - yc;
                const double z = (static_cast<double>(k - 3) + 0.5) * p->dz - zc;
                const double r = std::sqrt(x * x + y * y + z * z);
                q.set(i, j, k, p->gam, rho, 0.0, 0.0, 0.0, b, b, 0.0, (r < r0) ? pin : pout);
            }
    return 0;
}

// splitmix64 (Steele, Lea & Flood 2014): the seeded generator of turb3d.
struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() {   // Box-Muller
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * PI_L * u2);
    }
};

// turb3d: decaying turbulence.  rho = par3 (1), p = par4 (1), B = (par5 (0.5), 0, 0);
// v = sum over integer wave vectors n (half space, kmin <= |n| <= kmax with
// kmin = par1 (1), kmax = par2 (4); n_d = 0 on axes with one cell) of
// a_n cos(2 pi n.x/L) + b_n sin(2 pi n.x/L), with a_n, b_n Gaussian vectors
// projected perpendicular to n (solenoidal), drawn from splitmix64(seed);
// rescaled to rms |v| = par0 (0.5) over the active cells.
int init_turb3d(double* qp, const how_params* p, void*) {
    Q q = view(qp, p);
    const double vrms = par_or(p, 0, 0.5), kmin = par_or(p, 1, 1.0), kmax = par_or(p, 2, 4.0);
    const double rho = par_or(p, 3, 1.0), pg = par_or(p, 4, 1.0), B0 = par_or(p, 5, 0.5);
    const int K = (int)std::floor(kmax);
    const int Kx = p->nx > 1 ? K : 0, Ky = p->ny > 1 ? K : 0, Kz = p->nz > 1 ? K : 0;
    struct Mode { int n[3]; double a[3], b[3]; };
    std::vector<Mode> modes;
    SplitMix rng{p->seed};
    for (int a = -Kx; a <= Kx; ++a)
        for (int b = -Ky; b <= Ky; ++b)
            for (int c = -Kz; c <= Kz; ++c) {
                const bool half = a > 0 || (a == 0 && b > 0) || (a == 0 && b == 0 && c > 0);
                const double kn = std::sqrt((double)(a * a + b * b + c * c));
                if (!half || kn < kmin || kn > kmax) continue;
                Mode m;
                m.n[0] = a; m.n[1] = b; m.n[2] = c;
                const double kh[3] = {a / kn, b / kn, c / kn};
                for (double* w : {m.a, m.b}) {
                    for (int d = 0; d < 3; ++d) w[d] = rng.normal();
                    const double dot = w[0] * kh[0] + w[1] * kh[1] + w[2] * kh[2];
                    for (int d = 0; d < 3; ++d) w[d] -= dot * kh[d];
                }
                modes.push_back(m);
            }
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    // per-axis phase tables: cos/sin(2 pi n x / L) for n in [-K, K]
    auto table = [&](int ncell, double d, double L, int KK, std::vector<double>& cs, std::vector<double>& sn) {
        cs.assign((size_t)(2 * K + 1) * ncell, 1.0);
        sn.assign((size_t)(2 * K + 1) * ncell, 0.0);
        for (int nn = -KK; nn <= KK; ++nn)
            for (int i = 0; i < ncell; ++i) {
                const double x = (static_cast<double>(i) + 0.5) * d;
                cs[(size_t)(nn + K) * ncell + i] = std::cos(2.0 * PI_L * nn * x / L);
                sn[(size_t)(nn + K) * ncell + i] = std::sin(2.0 * PI_L * nn * x / L);
            }
    };
    std::vector<double> cx, sx, cy, sy, cz, sz;
    table(nx, p->dx, p->xsize, Kx, cx, sx);
    table(ny, p->dy, p->ysize, Ky, cy, sy);
    table(nz, p->dz, p->zsize, Kz, cz, sz);
    const size_t ncell = (size_t)nx * ny * nz;
    std::vector<double> V(3 * ncell, 0.0);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                double v[3] = {0, 0, 0};
                for (const Mode& m : modes) {
                    const size_t ix = (size_t)(m.n[0] + K) * nx + i;
                    const size_t iy = (size_t)(m.n[1] + K) * ny + j;
                    const size_t iz = (size_t)(m.n[2] + K) * nz + k;
                    // cos/sin of the summed phase from the per-axis factors
                    const double cxy = cx[ix] * cy[iy] - sx[ix] * sy[iy];
                    const double sxy = sx[ix] * cy[iy] + cx[ix] * sy[iy];
                    const double c = cxy * cz[iz] - sxy * sz[iz];
                    const double s = sxy * cz[iz] + cxy * sz[iz];
                    for (int d = 0; d < 3; ++d) v[d] += m.a[d] * c + m.b[d] * s;
                }
                const size_t o = ((size_t)i * ny + j) * nz + k;
                V[o] = v[0]; V[ncell + o] = v[1]; V[2 * ncell + o] = v[2];
            }
    // mean square speed: per-plane partial sums in parallel, then added in a
    // fixed order, so the state is bitwise reproducible for a seed whatever
    // the thread count
    std::vector<double> part(nx, 0.0);
    const size_t plane = (size_t)ny * nz;
#pragma omp parallel for
    for (int i = 0; i < nx; ++i) {
        double s = 0.0;
        for (size_t o = (size_t)i * plane; o < (size_t)(i + 1) * plane; ++o)
            s += V[o] * V[o] + V[ncell + o] * V[ncell + o] + V[2 * ncell + o] * V[2 * ncell + o];
        part[i] = s;
    }
    double sum2 = 0.0;
    for (int i = 0; i < nx; ++i) sum2 += part[i];
    const double scale = sum2 > 0.0 ? vrms / std::sqrt(sum2 / (double)ncell) : 0.0;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                const size_t o = ((size_t)i * ny + j) * nz + k;
                q.set(i + 3, j + 3, k + 3, p->gam, rho, scale * V[o], scale * V[ncell + o],
                      scale * V[2 * ncell + o], B0, 0.0, 0.0, pg);
            }
    return 0;
}

void ensure_builtins() {
    static bool done = false;
    if (done) return;
    done = true;
    auto& r = registry();
    auto add = [&](const char* n, how_problem_fn f) { if (!r.count(n)) r[n] = Entry{f, nullptr}; };
    add("orszag_tang", init_orszag_tang);
    add("blast3d", init_blast3d);
    add("brio_wu", init_brio_wu);
    add("mhd_rotor", init_mhd_rotor);
    add("uniform", init_uniform);
    add("mpi_smooth3d", init_mpi_smooth3d);
    add("alfven3d", init_alfven3d);
    add("blast3d_b", init_blast3d_b);
    add("turb3d", init_turb3d);
}

}  // namespace

extern "C" {

int how_register_problem(const char* name, how_problem_fn fn, void* user) {
    if (!name || !fn || !name[0]) { how::set_error("register_problem: null name or function"); return HOW_ERR_ARG; }
    std::lock_guard<std::mutex> g(reg_mutex());
    ensure_builtins();
    registry()[name] = Entry{fn, user};
    return HOW_OK;
}

int how_list_problems(char* buf, size_t cap) {
    std::lock_guard<std::mutex> g(reg_mutex());
    ensure_builtins();
    std::string s;
    for (auto& kv : registry()) { s += kv.first; s += "\n"; }
    if (buf && cap > 0) std::snprintf(buf, cap, "%s", s.c_str());
    return (int)registry().size();
}

int how_problem_init_host(const how_params* p, double* q) {
    if (!p || !q) { how::set_error("null argument"); return HOW_ERR_ARG; }
    Entry e;
    {
        std::lock_guard<std::mutex> g(reg_mutex());
        ensure_builtins();
        auto it = registry().find(p->problem);
        if (it == registry().end()) {
            // init_problem lists the registered names (src/problem.cpp:24-34)
            std::string names;
            for (auto& kv : registry()) { names += " "; names += kv.first; }
            how::set_error("unknown problem = %s; available:%s", p->problem, names.c_str());
            return HOW_ERR_PROBLEM;
        }
        e = it->second;
    }
    const size_t n = (size_t)8 * (p->nx + 6) * (p->ny + 6) * (p->nz + 6);
    std::memset(q, 0, n * sizeof(double));
    const int rc = e.fn(q, p, e.user);
    if (rc != 0) {
        how::set_error("problem %s initialiser failed (%d)", p->problem, rc);
        return HOW_ERR_PROBLEM;
    }
    return HOW_OK;
}

}  // extern "C"
