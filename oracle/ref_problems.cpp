// ref_problems.cpp -- the problems the benchmark configurations need and the
// reference lacks (alfven3d, blast3d_b, turb3d), registered into the
// reference's own problem registry through its static registrar
// (src/problem.hpp:17-22), so the reference build (oracle/_ref/how_ref) makes
// their initial states itself.  TEST INFRASTRUCTURE ONLY: linked into the
// reference-side checker, never into the product.
//
// Each initialiser restates the product's definition (how-mhd-kokkos_b200/
// csrc/problems.cpp) with its default parameters -- the reference's
// Parameters has no problem parameters or seed, and its parser skips those
// keys with a warning (src/parameters.cpp:112-116) -- operation for
// operation, so the states are bit-identical (tests/test_oracle_pin.py).
// Conserved variables from primitives as every reference problem forms them
// (e.g. src/problems/orszag_tang.cpp:168-186).
#include <Kokkos_Core.hpp>

#include "parameters.hpp"
#include "problem.hpp"

#include <cmath>
#include <cstdint>
#include <vector>

namespace {

constexpr double PI_L = 3.141592653589793238462643383279502884;

void set_cell(Kokkos::View<double*****> q, int i, int j, int k, double gam, double rho, double vx, double vy,
              double vz, double Bx, double By, double Bz, double pg) {
    const double Mx = rho * vx, My = rho * vy, Mz = rho * vz;
    const double vv2 = vx * vx + vy * vy + vz * vz;
    const double BB2 = Bx * Bx + By * By + Bz * Bz;
    const double E = pg / (gam - 1.0) + 0.5 * rho * vv2 + 0.5 * BB2;
    q(0, 0, i, j, k) = rho; q(0, 1, i, j, k) = Mx; q(0, 2, i, j, k) = My; q(0, 3, i, j, k) = Mz;
    q(0, 4, i, j, k) = Bx; q(0, 5, i, j, k) = By; q(0, 6, i, j, k) = Bz; q(0, 7, i, j, k) = E;
}

// blast3d_b: rho 1, p 10 inside r < 0.1 of the box centre and 0.1 outside,
// v = 0, B = (1, 1, 0) / sqrt 2.
void init_blast3d_b(Kokkos::View<double*****> q, const Parameters& par) {
    const double pin = 10.0, pout = 0.1, r0 = 0.1, Bm = 1.0, rho = 1.0;
    const double b = Bm / std::sqrt(2.0);
    const double xc = 0.5 * par.xsize, yc = 0.5 * par.ysize, zc = 0.5 * par.zsize;
#pragma omp parallel for collapse(2)
    for (int i = 3; i < par.nx + 3; ++i)
        for (int j = 3; j < par.ny + 3; ++j)
            for (int k = 3; k < par.nz + 3; ++k) {
                const double x = (static_cast<double>(i - 3) + 0.5) * par.dx - xc;
                const double y = (static_cast<double>(j - 3) + 0.5) * par.dy - yc;
                const double z = (static_cast<double>(k - 3) + 0.5) * par.dz - zc;
                const double r = std::sqrt(x * x + y * y + z * z);
                set_cell(q, i, j, k, par.gam, rho, 0.0, 0.0, 0.0, b, b, 0.0, (r < r0) ? pin : pout);
            }
}

// alfven3d: circularly polarised Alfven wave along k = 2 pi (1/Lx, 1/Ly, 1/Lz)
// over the axes with more than one cell; amplitude 0.1, B_par 1, rho 1, p 0.1.
void init_alfven3d(Kokkos::View<double*****> q, const Parameters& par) {
    const double A = 0.1, Bpar = 1.0, rho = 1.0, pg = 0.1;
    const double k[3] = {par.nx > 1 ? 2.0 * PI_L / par.xsize : 0.0, par.ny > 1 ? 2.0 * PI_L / par.ysize : 0.0,
                         par.nz > 1 ? 2.0 * PI_L / par.zsize : 0.0};
    const double kk = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    if (kk == 0.0) return;
    double e1[3] = {k[0] / kk, k[1] / kk, k[2] / kk};
    double e2[3] = {e1[1], -e1[0], 0.0};
    double n2 = std::sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    if (n2 < 1e-6) { e2[0] = -e1[2]; e2[1] = 0.0; e2[2] = e1[0]; n2 = std::sqrt(e2[0] * e2[0] + e2[2] * e2[2]); }
    for (double& x : e2) x /= n2;
    const double e3[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const double sr = std::sqrt(rho);
#pragma omp parallel for collapse(2)
    for (int i = 3; i < par.nx + 3; ++i)
        for (int j = 3; j < par.ny + 3; ++j)
            for (int k3 = 3; k3 < par.nz + 3; ++k3) {
                const double x = (static_cast<double>(i - 3) + 0.5) * par.dx;
                const double y = (static_cast<double>(j - 3) + 0.5) * par.dy;
                const double z = (static_cast<double>(k3 - 3) + 0.5) * par.dz;
                const double ph = k[0] * x + k[1] * y + k[2] * z;
                const double s = std::sin(ph), c = std::cos(ph);
                double B[3], v[3];
                for (int d = 0; d < 3; ++d) {
                    const double bt = A * (s * e2[d] + c * e3[d]);
                    B[d] = Bpar * e1[d] + bt;
                    v[d] = -bt / sr;
                }
                set_cell(q, i, j, k3, par.gam, rho, v[0], v[1], v[2], B[0], B[1], B[2], pg);
            }
}

// splitmix64 (Steele, Lea & Flood 2014) and Box-Muller normals: the seeded
// generator of turb3d, seed 12345.
struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * PI_L * u2);
    }
};

// turb3d: rho 1, p 1, B = (0.5, 0, 0); v = a seeded sum of solenoidal Fourier
// modes with 1 <= |n| <= 4 (n integer, half space), rescaled to rms 0.5.
void init_turb3d(Kokkos::View<double*****> q, const Parameters& par) {
    const double vrms = 0.5, kmin = 1.0, kmax = 4.0, rho = 1.0, pg = 1.0, B0 = 0.5;
    const int K = (int)std::floor(kmax);
    const int Kx = par.nx > 1 ? K : 0, Ky = par.ny > 1 ? K : 0, Kz = par.nz > 1 ? K : 0;
    struct Mode { int n[3]; double a[3], b[3]; };
    std::vector<Mode> modes;
    SplitMix rng{12345ull};
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
    const int nx = par.nx, ny = par.ny, nz = par.nz;
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
    table(nx, par.dx, par.xsize, Kx, cx, sx);
    table(ny, par.dy, par.ysize, Ky, cy, sy);
    table(nz, par.dz, par.zsize, Kz, cz, sz);
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
                    const double cxy = cx[ix] * cy[iy] - sx[ix] * sy[iy];
                    const double sxy = sx[ix] * cy[iy] + cx[ix] * sy[iy];
                    const double c = cxy * cz[iz] - sxy * sz[iz];
                    const double s = sxy * cz[iz] + cxy * sz[iz];
                    for (int d = 0; d < 3; ++d) v[d] += m.a[d] * c + m.b[d] * s;
                }
                const size_t o = ((size_t)i * ny + j) * nz + k;
                V[o] = v[0]; V[ncell + o] = v[1]; V[2 * ncell + o] = v[2];
            }
    // per-plane partial sums added in a fixed order (thread-count independent)
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
                set_cell(q, i + 3, j + 3, k + 3, par.gam, rho, scale * V[o], scale * V[ncell + o],
                         scale * V[2 * ncell + o], B0, 0.0, 0.0, pg);
            }
}

RegisterProblem reg_blast3d_b("blast3d_b", init_blast3d_b);
RegisterProblem reg_alfven3d("alfven3d", init_alfven3d);
RegisterProblem reg_turb3d("turb3d", init_turb3d);

}  // namespace
