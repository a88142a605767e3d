// how_oracle.cpp -- CPU restatement of the HOW-MHD time-step path
// (SSPRK(5,4) + characteristic WENO5/LLF sweeps + 4th-order CT).
//
// TEST INFRASTRUCTURE ONLY.  This is the checker for the B200 path: tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg load it; the product
// never does.  It is pinned to the reference itself (the reference's own
// sources compiled by oracle/Makefile into oracle/_ref/how_ref) by
// tests/test_oracle_pin.py and by fixtures in tests/golden/.
//
// The arithmetic of every expression follows the reference term for term and
// in the same evaluation order (g++ on x86-64 without -march does not contract
// FMAs, so both are plain IEEE double), which makes this restatement agree with
// the reference bit for bit on active cells.  Structure differs: a sweep works
// line by line with small per-thread buffers instead of the reference's
// all-line workspaces (src/ssprk.cpp:1009-1017), and only active lines are
// swept -- ghost-line results are overwritten by the ghost fills before they
// are read (src/fluxct.cpp:807, src/ssprk.cpp:1323).
//
// Layout: q(stage 0..5, var 0..7, i, j, k), k fastest, 3 ghosts per side
// (src/main.cpp:101-120); face B (stage, i, j, k) (src/fluxct.cpp:27-35).
#include "how_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

namespace {

// 1: fourth-order face value of B_n v_t in the CT terms (an option of the
// B200 path, ct_avg 4); 0: the reference's two-point form
int g_ct_avg4 = 0;

constexpr int NVAR = 8;

// ------------------------------------------------------------ counting scalar
// Algorithmic operation counter: every +, -, *, /, sqrt, fmax, fabs on a
// value counts 1.  Comparisons and copies count 0.
struct Cnt {
    double v = 0.0;
    static inline uint64_t n_add = 0, n_mul = 0, n_div = 0, n_sqrt = 0, n_other = 0;
    Cnt() = default;
    Cnt(double x) : v(x) {}
    static void reset() { n_add = n_mul = n_div = n_sqrt = n_other = 0; }
    static uint64_t total() { return n_add + n_mul + n_div + n_sqrt + n_other; }
};
inline Cnt operator+(Cnt a, Cnt b) { ++Cnt::n_add; return Cnt(a.v + b.v); }
inline Cnt operator-(Cnt a, Cnt b) { ++Cnt::n_add; return Cnt(a.v - b.v); }
inline Cnt operator-(Cnt a) { return Cnt(-a.v); }
inline Cnt operator*(Cnt a, Cnt b) { ++Cnt::n_mul; return Cnt(a.v * b.v); }
inline Cnt operator/(Cnt a, Cnt b) { ++Cnt::n_div; return Cnt(a.v / b.v); }
inline Cnt& operator+=(Cnt& a, Cnt b) { a = a + b; return a; }
inline Cnt& operator*=(Cnt& a, Cnt b) { a = a * b; return a; }
inline bool operator<(Cnt a, Cnt b) { return a.v < b.v; }
inline bool operator>=(Cnt a, Cnt b) { return a.v >= b.v; }
inline bool operator!=(Cnt a, Cnt b) { return a.v != b.v; }
inline Cnt sqrt_(Cnt a) { ++Cnt::n_sqrt; return Cnt(std::sqrt(a.v)); }
inline Cnt fmax_(Cnt a, Cnt b) { ++Cnt::n_other; return Cnt(std::fmax(a.v, b.v)); }
inline Cnt fabs_(Cnt a) { ++Cnt::n_other; return Cnt(std::fabs(a.v)); }
inline double sqrt_(double a) { return std::sqrt(a); }
inline double fmax_(double a, double b) { return std::fmax(a, b); }
inline double fabs_(double a) { return std::fabs(a); }

// sign1 (src/ssprk.cpp:54-57)
template <class T> inline T sign1(T x) { return (x >= T(0.0)) ? T(1.0) : T(-1.0); }

struct Prm {
    double gam, rhomin, pgmin;
};

// ------------------------------------------------- per-cell / per-interface math
// primitives with floors (src/ssprk.cpp:469-513).  q: line conserved (8),
// floored in place like qx; u: rho, vn, vt1, vt2, Bn, Bt1, Bt2, p, H.
template <class T>
inline void primit_cell(T* q, T* u, const Prm& P) {
    const T DD = q[0], Mx = q[1], My = q[2], Mz = q[3];
    const T Bx = q[4], By = q[5], Bz = q[6];
    T EE = q[7];
    T rho = DD;
    const T vx = Mx / rho, vy = My / rho, vz = Mz / rho;
    const T vv2 = vx * vx + vy * vy + vz * vz;
    const T BB2 = Bx * Bx + By * By + Bz * Bz;
    T pg = (T(P.gam) - T(1.0)) * (EE - T(0.5) * (rho * vv2 + BB2));
    if (rho < T(P.rhomin) || pg < T(P.pgmin)) {
        rho = fmax_(T(P.rhomin), rho);
        pg = fmax_(T(P.pgmin), pg);
        EE = pg / (T(P.gam) - T(1.0)) + T(0.5) * (rho * vv2 + BB2);
        q[0] = rho;
        q[7] = EE;
    }
    const T HH = (EE + pg) / rho;
    u[0] = rho; u[1] = vx; u[2] = vy; u[3] = vz;
    u[4] = Bx; u[5] = By; u[6] = Bz; u[7] = pg; u[8] = HH;
}

// cell-centre eigenvalues and fluxes (src/ssprk.cpp:546-593)
template <class T>
inline void centre_cell(const T* q, const T* u, T* a, T* F, const Prm& P) {
    const T DD = q[0], Mx = q[1], My = q[2], Mz = q[3], EE = q[7];
    const T rho = u[0], vx = u[1], vy = u[2], vz = u[3];
    const T Bx = u[4], By = u[5], Bz = u[6], pg = u[7];
    const T vv2 = vx * vx + vy * vy + vz * vz;
    const T BB2 = Bx * Bx + By * By + Bz * Bz;
    const T pt = pg + T(0.5) * BB2;
    const T vdB = vx * Bx + vy * By + vz * Bz;
    const T bbn2 = BB2 / rho;
    const T bnx2 = Bx * Bx / rho;
    const T cs2 = fmax_(T(0.0), T(P.gam) * fabs_(pg / rho));
    const T root = sqrt_(fmax_(T(0.0), (bbn2 + cs2) * (bbn2 + cs2) - T(4.0) * bnx2 * cs2));
    const T lf = sqrt_(fmax_(T(0.0), T(0.5) * (bbn2 + cs2 + root)));
    const T la = sqrt_(fmax_(T(0.0), bnx2));
    const T ls = sqrt_(fmax_(T(0.0), T(0.5) * (bbn2 + cs2 - root)));
    (void)vv2;
    a[0] = vx - lf; a[1] = vx - la; a[2] = vx - ls; a[3] = vx;
    a[4] = vx + ls; a[5] = vx + la; a[6] = vx + lf;
    F[0] = DD * vx;
    F[1] = Mx * vx + pt - Bx * Bx;
    F[2] = My * vx - Bx * By;
    F[3] = Mz * vx - Bx * Bz;
    F[4] = By * vx - Bx * vy;
    F[5] = Bz * vx - Bx * vz;
    F[6] = (EE + pt) * vx - Bx * vdB;
}

// interface left/right eigenvectors at the arithmetic mean of two cells
// (src/ssprk.cpp:610-818).  L[row*7+col], R[row*7+col].
template <class T>
inline void interface_LR(const T* u0, const T* u1, T* L, T* R, const Prm& P) {
    const T gam0 = T(1.0) - T(P.gam);
    const T gam1 = T(0.5) * (T(P.gam) - T(1.0));
    const T gam2 = (T(P.gam) - T(2.0)) / (T(P.gam) - T(1.0));
    const T rho = T(0.5) * (u0[0] + u1[0]);
    const T vx = T(0.5) * (u0[1] + u1[1]);
    const T vy = T(0.5) * (u0[2] + u1[2]);
    const T vz = T(0.5) * (u0[3] + u1[3]);
    const T Bx = T(0.5) * (u0[4] + u1[4]);
    const T By = T(0.5) * (u0[5] + u1[5]);
    const T Bz = T(0.5) * (u0[6] + u1[6]);
    const T pg = T(0.5) * (u0[7] + u1[7]);
    const T HH = T(0.5) * (u0[8] + u1[8]);
    (void)pg;
    const T vv2 = vx * vx + vy * vy + vz * vz;
    const T BB2 = Bx * Bx + By * By + Bz * Bz;
    const T bbn2 = BB2 / rho;
    const T bnx2 = Bx * Bx / rho;
    const T cs2 = (T(P.gam) - T(1.0)) * (HH - T(0.5) * (vv2 + bbn2));
    const T cs = sqrt_(fmax_(T(0.0), cs2));
    const T root = sqrt_(fmax_(T(0.0), (bbn2 + cs2) * (bbn2 + cs2) - T(4.0) * bnx2 * cs2));
    const T lf = sqrt_(fmax_(T(0.0), T(0.5) * (bbn2 + cs2 + root)));
    const T la = sqrt_(fmax_(T(0.0), bnx2));
    const T ls = sqrt_(fmax_(T(0.0), T(0.5) * (bbn2 + cs2 - root)));
    const T Bt2 = By * By + Bz * Bz;
    const T sgnBx = sign1(Bx);
    T bty, btz;
    if (Bt2 >= T(1.0e-30)) { bty = By / sqrt_(Bt2); btz = Bz / sqrt_(Bt2); }
    else { bty = T(1.0) / sqrt_(T(2.0)); btz = T(1.0) / sqrt_(T(2.0)); }
    T af, as;
    if ((lf * lf - ls * ls) >= T(1.0e-30)) {
        af = sqrt_(fmax_(T(0.0), cs2 - ls * ls)) / sqrt_(lf * lf - ls * ls);
        as = sqrt_(fmax_(T(0.0), lf * lf - cs2)) / sqrt_(lf * lf - ls * ls);
    } else { af = T(1.0); as = T(1.0); }
    const T sqrtrho = sqrt_(rho);
    const T invsqrtrho = T(1.0) / sqrtrho;
#define Lm(r, c) L[(r) * 7 + (c)]
#define Rm(r, c) R[(r) * 7 + (c)]
    Lm(0,0) =  af*(gam1*vv2 + lf*vx) - as*ls*(bty*vy + btz*vz)*sgnBx;
    Lm(0,1) =  af*(gam0*vx - lf);
    Lm(0,2) =  gam0*af*vy + as*ls*bty*sgnBx;
    Lm(0,3) =  gam0*af*vz + as*ls*btz*sgnBx;
    Lm(0,4) =  gam0*af*By + cs*as*bty*sqrtrho;
    Lm(0,5) =  gam0*af*Bz + cs*as*btz*sqrtrho;
    Lm(0,6) = -gam0*af;
    Lm(1,0) =  btz*vy - bty*vz;
    Lm(1,1) =  T(0.0);
    Lm(1,2) = -btz;
    Lm(1,3) =  bty;
    Lm(1,4) = -btz*sgnBx*sqrtrho;
    Lm(1,5) =  bty*sgnBx*sqrtrho;
    Lm(1,6) =  T(0.0);
    Lm(2,0) =  as*(gam1*vv2 + ls*vx) + af*lf*(bty*vy + btz*vz)*sgnBx;
    Lm(2,1) =  gam0*as*vx - as*ls;
    Lm(2,2) =  gam0*as*vy - af*lf*bty*sgnBx;
    Lm(2,3) =  gam0*as*vz - af*lf*btz*sgnBx;
    Lm(2,4) =  gam0*as*By - cs*af*bty*sqrtrho;
    Lm(2,5) =  gam0*as*Bz - cs*af*btz*sqrtrho;
    Lm(2,6) = -gam0*as;
    Lm(3,0) = -cs2/gam0 - T(0.5)*vv2;
    Lm(3,1) =  vx;
    Lm(3,2) =  vy;
    Lm(3,3) =  vz;
    Lm(3,4) =  By;
    Lm(3,5) =  Bz;
    Lm(3,6) = T(-1.0);
    Lm(4,0) =  as*(gam1*vv2 - ls*vx) - af*lf*(bty*vy + btz*vz)*sgnBx;
    Lm(4,1) =  as*(gam0*vx + ls);
    Lm(4,2) =  gam0*as*vy + af*lf*bty*sgnBx;
    Lm(4,3) =  gam0*as*vz + af*lf*btz*sgnBx;
    Lm(4,4) =  gam0*as*By - cs*af*bty*sqrtrho;
    Lm(4,5) =  gam0*as*Bz - cs*af*btz*sqrtrho;
    Lm(4,6) = -gam0*as;
    Lm(5,0) =  btz*vy - bty*vz;
    Lm(5,1) =  T(0.0);
    Lm(5,2) = -btz;
    Lm(5,3) =  bty;
    Lm(5,4) =  btz*sgnBx*sqrtrho;
    Lm(5,5) = -bty*sgnBx*sqrtrho;
    Lm(5,6) =  T(0.0);
    Lm(6,0) =  af*(gam1*vv2 - lf*vx) + as*ls*(bty*vy + btz*vz)*sgnBx;
    Lm(6,1) =  af*(gam0*vx + lf);
    Lm(6,2) =  gam0*af*vy - as*ls*bty*sgnBx;
    Lm(6,3) =  gam0*af*vz - as*ls*btz*sgnBx;
    Lm(6,4) =  gam0*af*By + cs*as*bty*sqrtrho;
    Lm(6,5) =  gam0*af*Bz + cs*as*btz*sqrtrho;
    Lm(6,6) = -gam0*af;
    // normalisation (src/ssprk.cpp:718-726)
    for (int m = 0; m < 7; ++m) {
        Lm(0,m) = T(0.5) * Lm(0,m) / cs2;
        Lm(1,m) = T(0.5) * Lm(1,m);
        Lm(2,m) = T(0.5) * Lm(2,m) / cs2;
        Lm(3,m) = -gam0 * Lm(3,m) / cs2;
        Lm(4,m) = T(0.5) * Lm(4,m) / cs2;
        Lm(5,m) = T(0.5) * Lm(5,m);
        Lm(6,m) = T(0.5) * Lm(6,m) / cs2;
    }
    // right eigenvectors, column = wave (src/ssprk.cpp:729-787)
    Rm(0,0) = af;
    Rm(1,0) = af*(vx-lf);
    Rm(2,0) = af*vy + as*ls*bty*sgnBx;
    Rm(3,0) = af*vz + as*ls*btz*sgnBx;
    Rm(4,0) = cs*as*bty*invsqrtrho;
    Rm(5,0) = cs*as*btz*invsqrtrho;
    Rm(6,0) = af*(lf*lf - lf*vx + T(0.5)*vv2 - gam2*cs2) + as*ls*(bty*vy + btz*vz)*sgnBx;
    Rm(0,1) = T(0.0);
    Rm(1,1) = T(0.0);
    Rm(2,1) = -btz;
    Rm(3,1) = bty;
    Rm(4,1) = -btz*sgnBx*invsqrtrho;
    Rm(5,1) = bty*sgnBx*invsqrtrho;
    Rm(6,1) = bty*vz - btz*vy;
    Rm(0,2) = as;
    Rm(1,2) = as*(vx-ls);
    Rm(2,2) = as*vy - af*lf*bty*sgnBx;
    Rm(3,2) = as*vz - af*lf*btz*sgnBx;
    Rm(4,2) = -cs*af*bty*invsqrtrho;
    Rm(5,2) = -cs*af*btz*invsqrtrho;
    Rm(6,2) = as*(ls*ls - ls*vx + T(0.5)*vv2 - gam2*cs2) - af*lf*(bty*vy + btz*vz)*sgnBx;
    Rm(0,3) = T(1.0);
    Rm(1,3) = vx;
    Rm(2,3) = vy;
    Rm(3,3) = vz;
    Rm(4,3) = T(0.0);
    Rm(5,3) = T(0.0);
    Rm(6,3) = T(0.5)*vv2;
    Rm(0,4) = as;
    Rm(1,4) = as*(vx+ls);
    Rm(2,4) = as*vy + af*lf*bty*sgnBx;
    Rm(3,4) = as*vz + af*lf*btz*sgnBx;
    Rm(4,4) = -cs*af*bty*invsqrtrho;
    Rm(5,4) = -cs*af*btz*invsqrtrho;
    Rm(6,4) = as*(ls*ls + ls*vx + T(0.5)*vv2 - gam2*cs2) + af*lf*(bty*vy + btz*vz)*sgnBx;
    Rm(0,5) = T(0.0);
    Rm(1,5) = T(0.0);
    Rm(2,5) = -btz;
    Rm(3,5) = bty;
    Rm(4,5) = btz*sgnBx*invsqrtrho;
    Rm(5,5) = -bty*sgnBx*invsqrtrho;
    Rm(6,5) = bty*vz - btz*vy;
    Rm(0,6) = af;
    Rm(1,6) = af*(vx+lf);
    Rm(2,6) = af*vy - as*ls*bty*sgnBx;
    Rm(3,6) = af*vz - as*ls*btz*sgnBx;
    Rm(4,6) = cs*as*bty*invsqrtrho;
    Rm(5,6) = cs*as*btz*invsqrtrho;
    Rm(6,6) = af*(lf*lf + lf*vx + T(0.5)*vv2 - gam2*cs2) - as*ls*(bty*vy + btz*vz)*sgnBx;
    // sign convention (src/ssprk.cpp:789-818)
    T sgnBt;
    if (By != T(0.0)) sgnBt = sign1(By); else sgnBt = sign1(Bz);
    if (cs >= la) {
        for (int m = 0; m < 7; ++m) { Lm(2,m) *= sgnBt; Lm(4,m) *= sgnBt; }
        for (int m = 0; m < 7; ++m) { Rm(m,2) *= sgnBt; Rm(m,4) *= sgnBt; }
    } else {
        for (int m = 0; m < 7; ++m) { Lm(0,m) *= sgnBt; Lm(6,m) *= sgnBt; }
        for (int m = 0; m < 7; ++m) { Rm(m,0) *= sgnBt; Rm(m,6) *= sgnBt; }
    }
#undef Lm
#undef Rm
}

// one WENO5-JS half (src/ssprk.cpp:896-912, 919-935)
template <class T>
inline T weno_phi(T a, T b, T c, T d) {
    const T eps = T(1.0e-10);
    const T IS0 = T(13.0)*(a-b)*(a-b) + T(3.0)*(a-T(3.0)*b)*(a-T(3.0)*b);
    const T IS1 = T(13.0)*(b-c)*(b-c) + T(3.0)*(b+c)*(b+c);
    const T IS2 = T(13.0)*(c-d)*(c-d) + T(3.0)*(T(3.0)*c-d)*(T(3.0)*c-d);
    const T alpha0 = T(1.0) / ((eps + IS0)*(eps + IS0));
    const T alpha1 = T(6.0) / ((eps + IS1)*(eps + IS1));
    const T alpha2 = T(3.0) / ((eps + IS2)*(eps + IS2));
    const T omega0 = alpha0 / (alpha0 + alpha1 + alpha2);
    const T omega2 = alpha2 / (alpha0 + alpha1 + alpha2);
    return omega0 * (a - T(2.0)*b + c) / T(3.0) + (omega2 - T(0.5)) * (b - T(2.0)*c + d) / T(6.0);
}

// characteristic WENO flux of field m at one interface (src/ssprk.cpp:849-937).
// Lrow: row m of L; F6/q6: fluxes / conserved of the 6 stencil cells
// (q ordering rho, mn, mt1, mt2, Bt1, Bt2, E: the normal B is skipped).
template <class T>
inline T weno_field(const T* Lrow, const T F6[6][7], const T q6[6][7], T amx) {
    T Fsk[6], qsk[6], dFsk[5], dqsk[5];
    for (int ks = 0; ks < 6; ++ks) {
        Fsk[ks] = Lrow[0]*F6[ks][0] + Lrow[1]*F6[ks][1] + Lrow[2]*F6[ks][2] + Lrow[3]*F6[ks][3]
                + Lrow[4]*F6[ks][4] + Lrow[5]*F6[ks][5] + Lrow[6]*F6[ks][6];
        qsk[ks] = Lrow[0]*q6[ks][0] + Lrow[1]*q6[ks][1] + Lrow[2]*q6[ks][2] + Lrow[3]*q6[ks][3]
                + Lrow[4]*q6[ks][4] + Lrow[5]*q6[ks][5] + Lrow[6]*q6[ks][6];
    }
    for (int ks = 0; ks < 5; ++ks) { dFsk[ks] = Fsk[ks+1] - Fsk[ks]; dqsk[ks] = qsk[ks+1] - qsk[ks]; }
    const T first = (-Fsk[1] + T(7.0)*Fsk[2] + T(7.0)*Fsk[3] - Fsk[4]) / T(12.0);
    const T second = weno_phi(T(0.5)*(dFsk[0] + amx*dqsk[0]), T(0.5)*(dFsk[1] + amx*dqsk[1]),
                              T(0.5)*(dFsk[2] + amx*dqsk[2]), T(0.5)*(dFsk[3] + amx*dqsk[3]));
    const T third = weno_phi(T(0.5)*(dFsk[4] - amx*dqsk[4]), T(0.5)*(dFsk[3] - amx*dqsk[3]),
                             T(0.5)*(dFsk[2] - amx*dqsk[2]), T(0.5)*(dFsk[1] - amx*dqsk[1]));
    return first - second + third;
}

// ------------------------------------------------------------------ one line
// x_sweep body for one line, generic over the direction through the caller's
// variable permutation (src/ssprk.cpp:458-997).  qx: 8 x P (P = n+6) line
// conserved in sweep order, floored in place; dq: 8 x P increments written for
// cells 3..n+2; bsy/bsz: n+1 CT terms.
struct LineWork {
    std::vector<double> ux, ax, Fx, L, R, dF;
    void size(int n) {
        const int P = n + 6;
        ux.resize(9 * P); ax.resize(7 * P); Fx.resize(7 * P);
        L.resize(49 * P); R.resize(49 * P); dF.resize(7 * (n + 1));
    }
};

void sweep_line(double* qx, int n, const Prm& P, double dtdl, double* dq, double* bsy,
                double* bsz, LineWork& w) {
    const int Pn = n + 6;
    w.size(n);
    double* ux = w.ux.data(); double* ax = w.ax.data(); double* Fx = w.Fx.data();
    double* L = w.L.data(); double* R = w.R.data(); double* dF = w.dF.data();
    // primit + centre over all cells (src/ssprk.cpp:466-467, 541-542)
    for (int ii = 0; ii < Pn; ++ii) {
        double q[8], u[9], a[7], F[7];
        for (int v = 0; v < 8; ++v) q[v] = qx[v * Pn + ii];
        primit_cell(q, u, P);
        qx[0 * Pn + ii] = q[0];
        qx[7 * Pn + ii] = q[7];
        centre_cell(q, u, a, F, P);
        for (int v = 0; v < 9; ++v) ux[v * Pn + ii] = u[v];
        for (int v = 0; v < 7; ++v) { ax[v * Pn + ii] = a[v]; Fx[v * Pn + ii] = F[v]; }
    }
    // interfaces used by the flux loop: ii = i+2, i in [0, n] (src/ssprk.cpp:865)
    for (int ii = 2; ii <= n + 2; ++ii) {
        double u0[9], u1[9];
        for (int v = 0; v < 9; ++v) { u0[v] = ux[v * Pn + ii]; u1[v] = ux[v * Pn + ii + 1]; }
        interface_LR(u0, u1, &L[49 * ii], &R[49 * ii], P);
    }
    // flux loop (src/ssprk.cpp:841-945), m ascending like the in-order atomic_add
    static const int qmap[7] = {0, 1, 2, 3, 5, 6, 7};
    for (int i = 0; i <= n; ++i) {
        double F6[6][7], q6[6][7];
        for (int ks = 0; ks < 6; ++ks) {
            const int c = i + ks;   // ii + 2 with ii = i - 2 + ks
            for (int v = 0; v < 7; ++v) { F6[ks][v] = Fx[v * Pn + c]; q6[ks][v] = qx[qmap[v] * Pn + c]; }
        }
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
        const double* Li = &L[49 * (i + 2)];
        const double* Ri = &R[49 * (i + 2)];
        for (int m = 0; m < 7; ++m) {
            double amx = 0.0;
            for (int s = -2; s <= 3; ++s) amx = std::fmax(amx, std::fabs(ax[m * Pn + i + s + 2]));
            const double Fs = weno_field(&Li[7 * m], F6, q6, amx);
            for (int r = 0; r < 7; ++r) acc[r] += Ri[7 * r + m] * Fs;
        }
        for (int r = 0; r < 7; ++r) dF[r * (n + 1) + i] = acc[r];
    }
    // update (src/ssprk.cpp:955-964)
    static const int rmap[8] = {0, 1, 2, 3, -1, 4, 5, 6};
    for (int i = 1; i <= n; ++i) {
        for (int v = 0; v < 8; ++v) {
            const int r = rmap[v];
            dq[v * Pn + i + 2] = (r < 0) ? 0.0 : -dtdl * (dF[r * (n + 1) + i] - dF[r * (n + 1) + i - 1]);
        }
    }
    // CT terms (src/ssprk.cpp:973-993)
    for (int i = 0; i <= n; ++i) {
        const int im1 = i + 1, i0 = i + 2, ip1 = i + 3, ip2 = i + 4;
        double ftmp1, ftmp2;
        if (g_ct_avg4) {
            // optional fourth-order face value (-1, 9, 9, -1) / 16 (not in the reference)
            ftmp1 = (-(ux[4 * Pn + im1] * ux[2 * Pn + im1]) + 9.0 * (ux[4 * Pn + i0] * ux[2 * Pn + i0])
                     + 9.0 * (ux[4 * Pn + ip1] * ux[2 * Pn + ip1]) - (ux[4 * Pn + ip2] * ux[2 * Pn + ip2])) / 16.0;
            ftmp2 = (-(ux[4 * Pn + im1] * ux[3 * Pn + im1]) + 9.0 * (ux[4 * Pn + i0] * ux[3 * Pn + i0])
                     + 9.0 * (ux[4 * Pn + ip1] * ux[3 * Pn + ip1]) - (ux[4 * Pn + ip2] * ux[3 * Pn + ip2])) / 16.0;
        } else {
            ftmp1 = (-0.0 * (ux[4 * Pn + im1] * ux[2 * Pn + im1])
                     + 9.0 * (ux[4 * Pn + i0] * ux[2 * Pn + i0])
                     + 9.0 * (ux[4 * Pn + ip1] * ux[2 * Pn + ip1])
                     - 0.0 * (ux[4 * Pn + ip2] * ux[2 * Pn + ip2])) / 18.0;
            ftmp2 = (-0.0 * (ux[4 * Pn + im1] * ux[3 * Pn + im1])
                     + 9.0 * (ux[4 * Pn + i0] * ux[3 * Pn + i0])
                     + 9.0 * (ux[4 * Pn + ip1] * ux[3 * Pn + ip1])
                     - 0.0 * (ux[4 * Pn + ip2] * ux[3 * Pn + ip2])) / 18.0;
        }
        bsy[i] = dF[4 * (n + 1) + i] + ftmp1;
        bsz[i] = dF[5 * (n + 1) + i] + ftmp2;
    }
}

// ------------------------------------------------------------------ the state
struct Oracle {
    oracle_params p;
    int nx, ny, nz, P0, P1, P2;
    size_t PV;
    double dx, dy, dz, dt = 0.0, dtdx = 0.0, dtdy = 0.0, dtdz = 0.0;
    std::vector<double> q;      // 6 * 8 * PV
    std::vector<double> fb[3];  // 6 * PV each
    std::vector<double> ct[12]; // fsy fsz gsx gsz hsx hsy Ox2 Oy2 Oz2 Ox Oy Oz

    explicit Oracle(const oracle_params& pp) : p(pp) {
        nx = p.nx; ny = p.ny; nz = p.nz;
        P0 = nx + 6; P1 = ny + 6; P2 = nz + 6;
        PV = (size_t)P0 * P1 * P2;
        // dx = size / gn (src/parameters.cpp:149-151)
        dx = p.xsize / (double)nx; dy = p.ysize / (double)ny; dz = p.zsize / (double)nz;
        q.assign(6 * 8 * PV, 0.0);
        for (auto& b : fb) b.assign(6 * PV, 0.0);
        for (auto& c : ct) c.assign(PV, 0.0);
    }
    size_t at(int i, int j, int k) const { return ((size_t)i * P1 + j) * P2 + k; }
    double* qs(int stage, int var) { return &q[((size_t)stage * 8 + var) * PV]; }
    double* bs(int comp, int stage) { return &fb[comp][(size_t)stage * PV]; }
};

// ghost fill of one padded array, x then y then z over full transverse extents,
// in place and in the reference's statement order (src/bound.cpp:19-107; the
// same rule serves face B, src/fluxct.cpp:141-205, and the CT arrays,
// src/fluxct.cpp:510-552).
void bound_array(Oracle& o, double* a) {
    const int nx = o.nx, ny = o.ny, nz = o.nz;
    const bool xp = o.p.bc[0] == 0, yp = o.p.bc[1] == 0, zp = o.p.bc[2] == 0;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j < o.P1; ++j)
        for (int k = 0; k < o.P2; ++k) {
            auto A = [&](int i) -> double& { return a[o.at(i, j, k)]; };
            if (xp) { A(0) = A(nx); A(1) = A(nx+1); A(2) = A(nx+2); A(nx+3) = A(3); A(nx+4) = A(4); A(nx+5) = A(5); }
            else { A(0) = A(3); A(1) = A(3); A(2) = A(3); A(nx+3) = A(nx+2); A(nx+4) = A(nx+2); A(nx+5) = A(nx+2); }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < o.P0; ++i)
        for (int k = 0; k < o.P2; ++k) {
            auto A = [&](int j) -> double& { return a[o.at(i, j, k)]; };
            if (yp) { A(0) = A(ny); A(1) = A(ny+1); A(2) = A(ny+2); A(ny+3) = A(3); A(ny+4) = A(4); A(ny+5) = A(5); }
            else { A(0) = A(3); A(1) = A(3); A(2) = A(3); A(ny+3) = A(ny+2); A(ny+4) = A(ny+2); A(ny+5) = A(ny+2); }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < o.P0; ++i)
        for (int j = 0; j < o.P1; ++j) {
            auto A = [&](int k) -> double& { return a[o.at(i, j, k)]; };
            if (zp) { A(0) = A(nz); A(1) = A(nz+1); A(2) = A(nz+2); A(nz+3) = A(3); A(nz+4) = A(4); A(nz+5) = A(5); }
            else { A(0) = A(3); A(1) = A(3); A(2) = A(3); A(nz+3) = A(nz+2); A(nz+4) = A(nz+2); A(nz+5) = A(nz+2); }
        }
}

// bound (src/bound.cpp:295-317): every variable of one stage
void bound_q(Oracle& o, int stage) { for (int v = 0; v < 8; ++v) bound_array(o, o.qs(stage, v)); }
// bound_bfield (src/fluxct.cpp:481-490)
void bound_b(Oracle& o, int stage) { for (int c = 0; c < 3; ++c) bound_array(o, o.bs(c, stage)); }

// bc_index_ct (src/fluxct.cpp:14-25) over the padded range [0, P-1]
inline int bci(int idx, int hi, bool periodic) {
    if (periodic) { const int n = hi + 1; int r = idx % n; if (r < 0) r += n; return r; }
    if (idx < 0) return 0;
    if (idx > hi) return hi;
    return idx;
}

// initialize_bfield_from_q (src/fluxct.cpp:65-107)
void init_faceb(Oracle& o) {
    double* B[3] = {o.qs(0, 4), o.qs(0, 5), o.qs(0, 6)};
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 1; i <= o.nx + 3; ++i)
        for (int j = 1; j <= o.ny + 3; ++j)
            for (int k = 1; k <= o.nz + 3; ++k) {
                o.bs(0, 0)[o.at(i, j, k)] = (-B[0][o.at(i-1,j,k)] + 9.0*B[0][o.at(i,j,k)]
                                            + 9.0*B[0][o.at(i+1,j,k)] - B[0][o.at(i+2,j,k)]) / 16.0;
                o.bs(1, 0)[o.at(i, j, k)] = (-B[1][o.at(i,j-1,k)] + 9.0*B[1][o.at(i,j,k)]
                                            + 9.0*B[1][o.at(i,j+1,k)] - B[1][o.at(i,j+2,k)]) / 16.0;
                o.bs(2, 0)[o.at(i, j, k)] = (-B[2][o.at(i,j,k-1)] + 9.0*B[2][o.at(i,j,k)]
                                            + 9.0*B[2][o.at(i,j,k+1)] - B[2][o.at(i,j,k+2)]) / 16.0;
            }
    bound_b(o, 0);
}

// tstep (src/tstep.cpp:11-136), serial build (no Allreduce)
double tstep(Oracle& o) {
    double vxmax = 0.0, vymax = 0.0, vzmax = 0.0;
    const double gam = o.p.gam, rhomin = o.p.rhomin, pgmin = o.p.pgmin;
    double* Q[8];
    for (int v = 0; v < 8; ++v) Q[v] = o.qs(0, v);
#pragma omp parallel
    {
        double mx = 0.0, my = 0.0, mz = 0.0;
#pragma omp for collapse(2) schedule(static)
        for (int i = 3; i < o.nx + 3; ++i)
            for (int j = 3; j < o.ny + 3; ++j)
                for (int k = 3; k < o.nz + 3; ++k) {
                    const size_t c = o.at(i, j, k);
                    const double DD = Q[0][c], Mx = Q[1][c], My = Q[2][c], Mz = Q[3][c];
                    const double Bx = Q[4][c], By = Q[5][c], Bz = Q[6][c], EE = Q[7][c];
                    const double rho = std::fmax(DD, rhomin);
                    const double vx = Mx / rho, vy = My / rho, vz = Mz / rho;
                    const double vv2 = vx*vx + vy*vy + vz*vz;
                    const double BB2 = Bx*Bx + By*By + Bz*Bz;
                    const double pg = std::fmax(pgmin, (gam - 1.0) * (EE - 0.5 * (rho * vv2 + BB2)));
                    const double bbn2 = BB2 / rho;
                    const double cs2 = std::fmax(0.0, gam * pg / rho);
                    const double bnx2 = Bx*Bx / rho, bny2 = By*By / rho, bnz2 = Bz*Bz / rho;
                    const double rootx = std::sqrt(std::fmax(0.0, (bbn2 + cs2)*(bbn2 + cs2) - 4.0 * bnx2 * cs2));
                    const double rooty = std::sqrt(std::fmax(0.0, (bbn2 + cs2)*(bbn2 + cs2) - 4.0 * bny2 * cs2));
                    const double rootz = std::sqrt(std::fmax(0.0, (bbn2 + cs2)*(bbn2 + cs2) - 4.0 * bnz2 * cs2));
                    const double lfx = std::sqrt(std::fmax(0.0, 0.5 * (bbn2 + cs2 + rootx)));
                    const double lfy = std::sqrt(std::fmax(0.0, 0.5 * (bbn2 + cs2 + rooty)));
                    const double lfz = std::sqrt(std::fmax(0.0, 0.5 * (bbn2 + cs2 + rootz)));
                    mx = std::fmax(mx, std::fabs(vx) + lfx);
                    my = std::fmax(my, std::fabs(vy) + lfy);
                    mz = std::fmax(mz, std::fabs(vz) + lfz);
                }
#pragma omp critical
        { vxmax = std::fmax(vxmax, mx); vymax = std::fmax(vymax, my); vzmax = std::fmax(vzmax, mz); }
    }
    const double tiny = 1.0e-300;
    double invdt = 0.0;
    if (o.nx > 1) invdt += std::fmax(vxmax, tiny) / o.dx;
    if (o.ny > 1) invdt += std::fmax(vymax, tiny) / o.dy;
    if (o.nz > 1) invdt += std::fmax(vzmax, tiny) / o.dz;
    if (invdt <= 0.0) invdt = std::fmax(vxmax, tiny) / o.dx;
    o.dt = o.p.cour / invdt;
    return o.dt;
}

// RK coefficients (src/ssprk.cpp:66-94)
struct RK { double k1, k2, k3, k4, k5; };
RK rk_coeff(int iw) {
    switch (iw) {
        case 1: return {1.0, 0.39175222700392, 0.0, 0.0, 0.0};
        case 2: return {0.44437049406734, 0.36841059262959, 0.55562950593266, 0.0, 0.0};
        case 3: return {0.62010185138540, 0.25189177424738, 0.37989814861460, 0.0, 0.0};
        case 4: return {0.17807995410773, 0.54497475021237, 0.82192004589227, 0.0, 0.0};
        default: return {-2.081261929715610e-02, 0.22600748319395, 5.03580947213895e-1,
                         0.51723167208978, -6.518979800418380e-12};
    }
}

// one directional sweep (src/ssprk.cpp:1000-1025, 1218-1272) over active lines.
// Line variable order: x (0..7), y (0,2,3,1,5,6,4,7), z (0,3,1,2,6,4,5,7)
// (src/ssprk.cpp:1054-1061, 1145-1152); CT terms go to (fsy,fsz), (gsz,gsx),
// (hsx,hsy) at face index i+2 (src/ssprk.cpp:447-452, 1112-1120, 1203-1211).
void sweep(Oracle& o, int dir, int iw, const RK& c, double dtdl, double* cta, double* ctb) {
    static const int perm[3][8] = {{0,1,2,3,4,5,6,7}, {0,2,3,1,5,6,4,7}, {0,3,1,2,6,4,5,7}};
    const int n = dir == 0 ? o.nx : dir == 1 ? o.ny : o.nz;
    const int Pn = n + 6;
    const int t1n = dir == 0 ? o.ny : o.nx;                 // first transverse
    const int t2n = dir == 2 ? o.ny : o.nz;                 // second transverse
    const Prm P{o.p.gam, o.p.rhomin, o.p.pgmin};
#pragma omp parallel
    {
        LineWork w;
        std::vector<double> qx(8 * Pn), dq(8 * Pn), bsy(n + 1), bsz(n + 1);
#pragma omp for collapse(2) schedule(static)
        for (int a = 3; a < t1n + 3; ++a)
            for (int b = 3; b < t2n + 3; ++b) {
                auto idx = [&](int s) -> size_t {
                    if (dir == 0) return o.at(s, a, b);
                    if (dir == 1) return o.at(a, s, b);
                    return o.at(a, b, s);
                };
                for (int m = 0; m < 8; ++m) {
                    const double* src = o.qs(iw - 1, perm[dir][m]);
                    for (int s = 0; s < Pn; ++s) qx[m * Pn + s] = src[idx(s)];
                }
                sweep_line(qx.data(), n, P, dtdl, dq.data(), bsy.data(), bsz.data(), w);
                for (int i = 0; i <= n; ++i) { cta[idx(i + 2)] = bsy[i]; ctb[idx(i + 2)] = bsz[i]; }
                for (int m = 0; m < 8; ++m) {
                    double* dst = o.qs(iw, perm[dir][m]);
                    const double* prev = o.qs(iw - 1, perm[dir][m]);
                    for (int s = 3; s < n + 3; ++s) {
                        const size_t id = idx(s);
                        if (dir == 0) dst[id] = c.k1 * dst[id] + c.k3 * prev[id] + dq[m * Pn + s];
                        else dst[id] += dq[m * Pn + s];
                    }
                }
            }
    }
}

// fluxct (src/fluxct.cpp:786-899)
void fluxct(Oracle& o, int iw, double k1, double k3) {
    const bool use_x = o.nx > 1, use_y = o.ny > 1, use_z = o.nz > 1;
    const bool use_Ox = use_x && use_y, use_Oy = use_y && use_z, use_Oz = use_x && use_z;
    if (!use_Ox && !use_Oy && !use_Oz) return;
    const bool xp = o.p.bc[0] == 0, yp = o.p.bc[1] == 0, zp = o.p.bc[2] == 0;
    const int hx = o.nx + 5, hy = o.ny + 5, hz = o.nz + 5;
    for (int a = 0; a < 6; ++a) bound_array(o, o.ct[a].data());
    double *fsy = o.ct[0].data(), *fsz = o.ct[1].data(), *gsx = o.ct[2].data(), *gsz = o.ct[3].data();
    double *hsx = o.ct[4].data(), *hsy = o.ct[5].data();
    double *Ox2 = o.ct[6].data(), *Oy2 = o.ct[7].data(), *Oz2 = o.ct[8].data();
    double *Ox = o.ct[9].data(), *Oy = o.ct[10].data(), *Oz = o.ct[11].data();
    auto I = [&](int i, int j, int k) { return o.at(i, j, k); };
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i <= o.nx + 3; ++i)
        for (int j = 0; j <= o.ny + 3; ++j)
            for (int k = 0; k <= o.nz + 3; ++k) {
                const int im1 = bci(i-1,hx,xp), ip1 = bci(i+1,hx,xp), ip2 = bci(i+2,hx,xp);
                const int jm1 = bci(j-1,hy,yp), jp1 = bci(j+1,hy,yp), jp2 = bci(j+2,hy,yp);
                const int km1 = bci(k-1,hz,zp), kp1 = bci(k+1,hz,zp), kp2 = bci(k+2,hz,zp);
                if (use_Ox) Ox2[I(i,j,k)] = (-gsx[I(im1,j,k)] + 9.0*gsx[I(i,j,k)] + 9.0*gsx[I(ip1,j,k)] - gsx[I(ip2,j,k)]) / 16.0
                                          - (-fsy[I(i,jm1,k)] + 9.0*fsy[I(i,j,k)] + 9.0*fsy[I(i,jp1,k)] - fsy[I(i,jp2,k)]) / 16.0;
                if (use_Oy) Oy2[I(i,j,k)] = (-hsy[I(i,jm1,k)] + 9.0*hsy[I(i,j,k)] + 9.0*hsy[I(i,jp1,k)] - hsy[I(i,jp2,k)]) / 16.0
                                          - (-gsz[I(i,j,km1)] + 9.0*gsz[I(i,j,k)] + 9.0*gsz[I(i,j,kp1)] - gsz[I(i,j,kp2)]) / 16.0;
                if (use_Oz) Oz2[I(i,j,k)] = (-fsz[I(i,j,km1)] + 9.0*fsz[I(i,j,k)] + 9.0*fsz[I(i,j,kp1)] - fsz[I(i,j,kp2)]) / 16.0
                                          - (-hsx[I(im1,j,k)] + 9.0*hsx[I(i,j,k)] + 9.0*hsx[I(ip1,j,k)] - hsx[I(ip2,j,k)]) / 16.0;
            }
    for (int a = 6; a < 9; ++a) bound_array(o, o.ct[a].data());
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 1; i <= o.nx + 4; ++i)
        for (int j = 1; j <= o.ny + 4; ++j)
            for (int k = 1; k <= o.nz + 4; ++k) {
                const int im1 = bci(i-1,hx,xp), ip1 = bci(i+1,hx,xp);
                const int jm1 = bci(j-1,hy,yp), jp1 = bci(j+1,hy,yp);
                const int km1 = bci(k-1,hz,zp), kp1 = bci(k+1,hz,zp);
                const size_t c = I(i,j,k);
                if (use_Ox) Ox[c] = Ox2[c] + (Ox2[I(im1,j,k)] - 2.0*Ox2[c] + Ox2[I(ip1,j,k)]) / 24.0
                                           + (Ox2[I(i,jm1,k)] - 2.0*Ox2[c] + Ox2[I(i,jp1,k)]) / 24.0;
                if (use_Oy) Oy[c] = Oy2[c] + (Oy2[I(i,jm1,k)] - 2.0*Oy2[c] + Oy2[I(i,jp1,k)]) / 24.0
                                           + (Oy2[I(i,j,km1)] - 2.0*Oy2[c] + Oy2[I(i,j,kp1)]) / 24.0;
                if (use_Oz) Oz[c] = Oz2[c] + (Oz2[I(im1,j,k)] - 2.0*Oz2[c] + Oz2[I(ip1,j,k)]) / 24.0
                                           + (Oz2[I(i,j,km1)] - 2.0*Oz2[c] + Oz2[I(i,j,kp1)]) / 24.0;
            }
    for (int a = 9; a < 12; ++a) bound_array(o, o.ct[a].data());
    const double aa = 9.0 / 8.0, bb = -1.0 / 24.0, cc = 0.0;
    double *bx = o.bs(0, iw), *by = o.bs(1, iw), *bz = o.bs(2, iw);
    const double *bx0 = o.bs(0, iw - 1), *by0 = o.bs(1, iw - 1), *bz0 = o.bs(2, iw - 1);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 1; i <= o.nx + 3; ++i)
        for (int j = 1; j <= o.ny + 3; ++j)
            for (int k = 1; k <= o.nz + 3; ++k) {
                const int im1 = bci(i-1,hx,xp), im2 = bci(i-2,hx,xp), im3 = bci(i-3,hx,xp);
                const int ip1 = bci(i+1,hx,xp), ip2 = bci(i+2,hx,xp);
                const int jm1 = bci(j-1,hy,yp), jm2 = bci(j-2,hy,yp), jm3 = bci(j-3,hy,yp);
                const int jp1 = bci(j+1,hy,yp), jp2 = bci(j+2,hy,yp);
                const int km1 = bci(k-1,hz,zp), km2 = bci(k-2,hz,zp), km3 = bci(k-3,hz,zp);
                const int kp1 = bci(k+1,hz,zp), kp2 = bci(k+2,hz,zp);
                const size_t c = I(i,j,k);
                if (use_Ox || use_Oz) {
                    double dOx = 0.0, dOz = 0.0;
                    if (use_Ox) dOx = aa*(Ox[c]-Ox[I(i,jm1,k)]) + bb*(Ox[I(i,jp1,k)]-Ox[I(i,jm2,k)]) + cc*(Ox[I(i,jp2,k)]-Ox[I(i,jm3,k)]);
                    if (use_Oz) dOz = aa*(Oz[c]-Oz[I(i,j,km1)]) + bb*(Oz[I(i,j,kp1)]-Oz[I(i,j,km2)]) + cc*(Oz[I(i,j,kp2)]-Oz[I(i,j,km3)]);
                    bx[c] = k1*bx[c] + k3*bx0[c] - o.dtdy*dOx + o.dtdz*dOz;
                }
                if (use_Oy || use_Ox) {
                    double dOy = 0.0, dOx = 0.0;
                    if (use_Oy) dOy = aa*(Oy[c]-Oy[I(i,j,km1)]) + bb*(Oy[I(i,j,kp1)]-Oy[I(i,j,km2)]) + cc*(Oy[I(i,j,kp2)]-Oy[I(i,j,km3)]);
                    if (use_Ox) dOx = aa*(Ox[c]-Ox[I(im1,j,k)]) + bb*(Ox[I(ip1,j,k)]-Ox[I(im2,j,k)]) + cc*(Ox[I(ip2,j,k)]-Ox[I(im3,j,k)]);
                    by[c] = k1*by[c] + k3*by0[c] - o.dtdz*dOy + o.dtdx*dOx;
                }
                if (use_Oz || use_Oy) {
                    double dOz = 0.0, dOy = 0.0;
                    if (use_Oz) dOz = aa*(Oz[c]-Oz[I(im1,j,k)]) + bb*(Oz[I(ip1,j,k)]-Oz[I(im2,j,k)]) + cc*(Oz[I(ip2,j,k)]-Oz[I(im3,j,k)]);
                    if (use_Oy) dOy = aa*(Oy[c]-Oy[I(i,jm1,k)]) + bb*(Oy[I(i,jp1,k)]-Oy[I(i,jm2,k)]) + cc*(Oy[I(i,jp2,k)]-Oy[I(i,jm3,k)]);
                    bz[c] = k1*bz[c] + k3*bz0[c] - o.dtdx*dOz + o.dtdy*dOy;
                }
            }
    bound_b(o, iw);
    double *q4 = o.qs(iw, 4), *q5 = o.qs(iw, 5), *q6 = o.qs(iw, 6);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 3; i <= o.nx + 2; ++i)
        for (int j = 3; j <= o.ny + 2; ++j)
            for (int k = 3; k <= o.nz + 2; ++k) {
                const int im1 = bci(i-1,hx,xp), im2 = bci(i-2,hx,xp), im3 = bci(i-3,hx,xp);
                const int ip1 = bci(i+1,hx,xp), ip2 = bci(i+2,hx,xp);
                const int jm1 = bci(j-1,hy,yp), jm2 = bci(j-2,hy,yp), jm3 = bci(j-3,hy,yp);
                const int jp1 = bci(j+1,hy,yp), jp2 = bci(j+2,hy,yp);
                const int km1 = bci(k-1,hz,zp), km2 = bci(k-2,hz,zp), km3 = bci(k-3,hz,zp);
                const int kp1 = bci(k+1,hz,zp), kp2 = bci(k+2,hz,zp);
                const size_t c = I(i,j,k);
                q4[c] = use_x ? (3.0*bx[I(im3,j,k)] - 25.0*bx[I(im2,j,k)] + 150.0*bx[I(im1,j,k)] + 150.0*bx[c]
                                 - 25.0*bx[I(ip1,j,k)] + 3.0*bx[I(ip2,j,k)]) / 256.0 : bx[c];
                q5[c] = use_y ? (3.0*by[I(i,jm3,k)] - 25.0*by[I(i,jm2,k)] + 150.0*by[I(i,jm1,k)] + 150.0*by[c]
                                 - 25.0*by[I(i,jp1,k)] + 3.0*by[I(i,jp2,k)]) / 256.0 : by[c];
                q6[c] = use_z ? (3.0*bz[I(i,j,km3)] - 25.0*bz[I(i,j,km2)] + 150.0*bz[I(i,j,km1)] + 150.0*bz[c]
                                 - 25.0*bz[I(i,j,kp1)] + 3.0*bz[I(i,j,kp2)]) / 256.0 : bz[c];
            }
}

// prot (src/prot.cpp:10-51)
void prot(Oracle& o, int stage) {
    const double gam = o.p.gam;
    double* Q[8];
    for (int v = 0; v < 8; ++v) Q[v] = o.qs(stage, v);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 3; i < o.nx + 3; ++i)
        for (int j = 3; j < o.ny + 3; ++j)
            for (int k = 3; k < o.nz + 3; ++k) {
                const size_t c = o.at(i, j, k);
                double rho = Q[0][c];
                const double Mx = Q[1][c], My = Q[2][c], Mz = Q[3][c];
                const double Bx = Q[4][c], By = Q[5][c], Bz = Q[6][c];
                double E = Q[7][c];
                rho = std::fmax(rho, o.p.rhomin);
                const double vx = Mx / rho, vy = My / rho, vz = Mz / rho;
                const double vv2 = vx*vx + vy*vy + vz*vz;
                const double BB2 = Bx*Bx + By*By + Bz*Bz;
                double pg = (gam - 1.0) * (E - 0.5 * (rho*vv2 + BB2));
                pg = std::fmax(pg, o.p.pgmin);
                E = pg / (gam - 1.0) + 0.5 * (rho*vv2 + BB2);
                Q[0][c] = rho;
                Q[7][c] = E;
            }
}

void copy_stage(Oracle& o, int dst, int src) {
    std::memcpy(o.qs(dst, 0), o.qs(src, 0), 8 * o.PV * sizeof(double));
}
void copy_b(Oracle& o, int dst, int src) {
    for (int c = 0; c < 3; ++c) std::memcpy(o.bs(c, dst), o.bs(c, src), o.PV * sizeof(double));
}

// ssprk (src/ssprk.cpp:1277-1329)
void ssprk(Oracle& o) {
    for (int iw = 1; iw <= 5; ++iw) {
        for (auto& a : o.ct) std::fill(a.begin(), a.end(), 0.0);   // zero_ct_fluxes
        const RK c = rk_coeff(iw);
        if (iw <= 4) { copy_stage(o, iw, 0); copy_b(o, iw, 0); }
        else {
            // prepare_stage5 (src/ssprk.cpp:121-140), prepare_bfield_stage5 (src/fluxct.cpp:124-135)
            for (int v = 0; v < 8; ++v) {
                double *d = o.qs(5, v); const double *a = o.qs(0, v), *b = o.qs(2, v), *e = o.qs(3, v);
#pragma omp parallel for schedule(static)
                for (long x = 0; x < (long)o.PV; ++x) d[x] = a[x] + (c.k4 / c.k1) * b[x] + (c.k5 / c.k1) * e[x];
            }
            for (int cc = 0; cc < 3; ++cc) {
                double *d = o.bs(cc, 5); const double *a = o.bs(cc, 0), *b = o.bs(cc, 2), *e = o.bs(cc, 3);
#pragma omp parallel for schedule(static)
                for (long x = 0; x < (long)o.PV; ++x) d[x] = a[x] + (c.k4 / c.k1) * b[x] + (c.k5 / c.k1) * e[x];
            }
        }
        bound_q(o, iw - 1);
        if (iw == 5) bound_q(o, iw);
        o.dtdx = c.k2 * o.dt / o.dx;
        o.dtdy = c.k2 * o.dt / o.dy;
        o.dtdz = c.k2 * o.dt / o.dz;
        if (o.nx > 1) sweep(o, 0, iw, c, o.dtdx, o.ct[0].data(), o.ct[1].data());
        if (o.ny > 1) sweep(o, 1, iw, c, o.dtdy, o.ct[3].data(), o.ct[2].data());
        if (o.nz > 1) sweep(o, 2, iw, c, o.dtdz, o.ct[4].data(), o.ct[5].data());
        bound_b(o, iw - 1);
        fluxct(o, iw, c.k1, c.k3);
        prot(o, iw);
        bound_q(o, iw);
        bound_b(o, iw);
    }
    copy_stage(o, 0, 5);
    copy_b(o, 0, 5);
}

// ----------------------------------------------------------------- problems
// Restatements of the reference's registered initial conditions.
constexpr double PI_LONG = 3.141592653589793238462643383279502884;

void fill_cell(Oracle& o, int i, int j, int k, double rho, double vx, double vy, double vz,
               double Bx, double By, double Bz, double pg) {
    const double Mx = rho * vx, My = rho * vy, Mz = rho * vz;
    const double vv2 = vx*vx + vy*vy + vz*vz;
    const double BB2 = Bx*Bx + By*By + Bz*Bz;
    const double E = pg / (o.p.gam - 1.0) + 0.5 * rho * vv2 + 0.5 * BB2;
    const size_t c = o.at(i, j, k);
    const double vals[8] = {rho, Mx, My, Mz, Bx, By, Bz, E};
    for (int v = 0; v < 8; ++v) o.qs(0, v)[c] = vals[v];
}

int init_problem(Oracle& o, const std::string& name) {
    for (int i = 3; i < o.nx + 3; ++i)
        for (int j = 3; j < o.ny + 3; ++j)
            for (int k = 3; k < o.nz + 3; ++k) {
                const double x = (double(i - 3) + 0.5) * o.dx;
                const double y = (double(j - 3) + 0.5) * o.dy;
                const double z = (double(k - 3) + 0.5) * o.dz;
                if (name == "orszag_tang") {            // src/problems/orszag_tang.cpp:128-186
                    const double pi = PI_LONG;
                    const double rho = 25.0 / (36.0 * pi), pg = 5.0 / (12.0 * pi);
                    const double vx = -std::sin(2.0 * pi * y), vy = std::sin(2.0 * pi * x);
                    const double normB = std::sqrt(4.0 * pi);
                    fill_cell(o, i, j, k, rho, vx, vy, 0.0, -std::sin(2.0 * pi * y) / normB,
                              std::sin(4.0 * pi * x) / normB, 0.0, pg);
                } else if (name == "blast3d") {          // src/problems/blast3d.cpp:27-99
                    const double xc = 0.5 * o.p.xsize, yc = 0.5 * o.p.ysize, zc = 0.5 * o.p.zsize;
                    const double r0 = 0.10 * std::fmin(o.p.xsize, std::fmin(o.p.ysize, o.p.zsize));
                    const double rx = x - xc, ry = y - yc, rz = z - zc;
                    const double rr = std::sqrt(rx*rx + ry*ry + rz*rz);
                    fill_cell(o, i, j, k, 1.0, 0.0, 0.0, 0.0, 0.1, 0.0, 0.0, (rr <= r0) ? 100.0 : 1.0);
                } else if (name == "blast3d_b") {        // the benchmark blast (the product's
                    // problem of that name, default parameters): p 10 / 0.1 across r = 0.1,
                    // B = (1, 1, 0) / sqrt 2
                    const double xc = 0.5 * o.p.xsize, yc = 0.5 * o.p.ysize, zc = 0.5 * o.p.zsize;
                    const double rx = x - xc, ry = y - yc, rz = z - zc;
                    const double r = std::sqrt(rx*rx + ry*ry + rz*rz);
                    const double b = 1.0 / std::sqrt(2.0);
                    fill_cell(o, i, j, k, 1.0, 0.0, 0.0, 0.0, b, b, 0.0, (r < 0.1) ? 10.0 : 0.1);
                } else if (name == "brio_wu") {          // src/problems/brio_wu.cpp:201-254
                    if (x < 0.5 * o.p.xsize) fill_cell(o, i, j, k, 1.0, 0, 0, 0, 0.75, 1.0, 0.0, 1.0);
                    else fill_cell(o, i, j, k, 0.125, 0, 0, 0, 0.75, -1.0, 0.0, 0.1);
                } else if (name == "mhd_rotor") {        // src/problems/mhd_rotor.cpp:17-108
                    const double pi = PI_LONG;
                    const double ddx = x - 0.5, ddy = y - 0.5;
                    const double r = std::sqrt(ddx*ddx + ddy*ddy);
                    const double r0 = 0.10, r1 = 0.115, rin = 10.0, rout = 1.0, om = 20.0;
                    double rho, vx, vy;
                    if (r <= r0) { rho = rin; vx = -om * ddy; vy = om * ddx; }
                    else if (r <= r1) {
                        const double f = (r1 - r) / (r1 - r0);
                        rho = rout + f * (rin - rout); vx = f * (-om * ddy); vy = f * (om * ddx);
                    } else { rho = rout; vx = 0.0; vy = 0.0; }
                    fill_cell(o, i, j, k, rho, vx, vy, 0.0, 5.0 / std::sqrt(4.0 * pi), 0.0, 0.0, 1.0);
                } else if (name == "uniform") {          // src/problems/uniform.cpp:9-21
                    const size_t c = o.at(i, j, k);
                    const double vals[8] = {1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0};
                    for (int v = 0; v < 8; ++v) o.qs(0, v)[c] = vals[v];
                } else if (name == "mpi_smooth3d") {     // src/problems/mpi_smooth3d.cpp:17-84
                    const double pi = PI_LONG;
                    const double Lx = o.p.xsize, Ly = o.p.ysize, Lz = o.p.zsize;
                    const double sx = std::sin(2.0*pi*x/Lx), sy = std::sin(2.0*pi*y/Ly), sz = std::sin(2.0*pi*z/Lz);
                    const double cx = std::cos(2.0*pi*x/Lx), cy = std::cos(2.0*pi*y/Ly), cz = std::cos(2.0*pi*z/Lz);
                    fill_cell(o, i, j, k, 1.0 + 0.05*sx*sy*sz, 0.10 + 0.01*cy*cz, 0.05 + 0.01*cz*cx,
                              0.02 + 0.01*cx*cy, 0.10 + 0.005*sy*sz, 0.08 + 0.005*sz*sx,
                              0.06 + 0.005*sx*sy, 1.0 + 0.02*cx*cy*cz);
                } else {
                    return -1;
                }
            }
    return 0;
}

} // namespace

// ----------------------------------------------------------------- C entry
extern "C" {

void* oracle_create(const oracle_params* p) { return new Oracle(*p); }
void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }
void oracle_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
void oracle_set_ct_avg(int points) { g_ct_avg4 = points == 4 ? 1 : 0; }

int oracle_init_problem(void* h, const char* name) {
    return init_problem(*static_cast<Oracle*>(h), std::string(name));
}
void oracle_set_q(void* h, int stage, const double* q) {
    auto& o = *static_cast<Oracle*>(h);
    std::memcpy(o.qs(stage, 0), q, 8 * o.PV * sizeof(double));
}
void oracle_get_q(void* h, int stage, double* q) {
    auto& o = *static_cast<Oracle*>(h);
    std::memcpy(q, o.qs(stage, 0), 8 * o.PV * sizeof(double));
}
void oracle_set_faceb(void* h, int stage, const double* bx, const double* by, const double* bz) {
    auto& o = *static_cast<Oracle*>(h);
    const double* s[3] = {bx, by, bz};
    for (int c = 0; c < 3; ++c) std::memcpy(o.bs(c, stage), s[c], o.PV * sizeof(double));
}
void oracle_get_faceb(void* h, int stage, double* bx, double* by, double* bz) {
    auto& o = *static_cast<Oracle*>(h);
    double* d[3] = {bx, by, bz};
    for (int c = 0; c < 3; ++c) std::memcpy(d[c], o.bs(c, stage), o.PV * sizeof(double));
}
void oracle_bound(void* h, int stage) { bound_q(*static_cast<Oracle*>(h), stage); }
void oracle_bound_bfield(void* h, int stage) { bound_b(*static_cast<Oracle*>(h), stage); }
void oracle_init_faceb(void* h) { init_faceb(*static_cast<Oracle*>(h)); }
double oracle_tstep(void* h) { return tstep(*static_cast<Oracle*>(h)); }
void oracle_ssprk(void* h, double dt) {
    auto& o = *static_cast<Oracle*>(h);
    o.dt = dt;
    ssprk(o);
}

int oracle_run(void* h, double tend, int nt, long max_steps, double* time_out, long* steps_out,
               double* dts_out, long dts_cap) {
    auto& o = *static_cast<Oracle*>(h);
    double time = 0.0;
    const double dtout = tend / (double)nt;
    long steps = 0;
    int rc = 0;
    bool stop = false;
    for (int out_step = 1; out_step <= nt && !stop; ++out_step) {
        const double target_time = dtout * (double)out_step;
        while (time < target_time) {
            if (max_steps >= 0 && steps >= max_steps) { stop = true; break; }
            tstep(o);
            if (time + o.dt > target_time) o.dt = target_time - time;
            if (o.dt <= 0.0) { rc = 3; stop = true; break; }
            ssprk(o);
            time += o.dt;
            if (dts_out && steps < dts_cap) dts_out[steps] = o.dt;
            ++steps;
            if (!std::isfinite(time)) { rc = 4; stop = true; break; }
        }
    }
    if (time_out) *time_out = time;
    if (steps_out) *steps_out = steps;
    return rc;
}

void oracle_sweep(void* h, int dir, double dt, double* q1_out, double* ct_a, double* ct_b) {
    auto& o = *static_cast<Oracle*>(h);
    for (auto& a : o.ct) std::fill(a.begin(), a.end(), 0.0);
    const RK c = rk_coeff(1);
    copy_stage(o, 1, 0);
    copy_b(o, 1, 0);
    bound_q(o, 0);
    o.dt = dt;
    o.dtdx = c.k2 * o.dt / o.dx;
    o.dtdy = c.k2 * o.dt / o.dy;
    o.dtdz = c.k2 * o.dt / o.dz;
    int ia = dir == 0 ? 0 : dir == 1 ? 3 : 4;
    int ib = dir == 0 ? 1 : dir == 1 ? 2 : 5;
    sweep(o, dir, 1, c, dir == 0 ? o.dtdx : dir == 1 ? o.dtdy : o.dtdz, o.ct[ia].data(), o.ct[ib].data());
    if (q1_out) std::memcpy(q1_out, o.qs(1, 0), 8 * o.PV * sizeof(double));
    if (ct_a) std::memcpy(ct_a, o.ct[ia].data(), o.PV * sizeof(double));
    if (ct_b) std::memcpy(ct_b, o.ct[ib].data(), o.PV * sizeof(double));
}

// stage iw = 1 up to its constrained transport (src/ssprk.cpp:1281-1317):
// zero the CT arrays, copy q(0) and face B(0) into stage 1, bound q(0), then
// the x, y and z sweeps with dt (the axes with n > 1).
void oracle_stage1_sweeps(void* h, double dt) {
    auto& o = *static_cast<Oracle*>(h);
    for (auto& a : o.ct) std::fill(a.begin(), a.end(), 0.0);
    const RK c = rk_coeff(1);
    copy_stage(o, 1, 0);
    copy_b(o, 1, 0);
    bound_q(o, 0);
    o.dt = dt;
    o.dtdx = c.k2 * o.dt / o.dx;
    o.dtdy = c.k2 * o.dt / o.dy;
    o.dtdz = c.k2 * o.dt / o.dz;
    if (o.nx > 1) sweep(o, 0, 1, c, o.dtdx, o.ct[0].data(), o.ct[1].data());
    if (o.ny > 1) sweep(o, 1, 1, c, o.dtdy, o.ct[3].data(), o.ct[2].data());
    if (o.nz > 1) sweep(o, 2, 1, c, o.dtdz, o.ct[4].data(), o.ct[5].data());
}
// bound_bfield(iw - 1) then fluxct(q, iw, k1, k3) (src/ssprk.cpp:1319-1320,
// src/fluxct.cpp:786-899) on the CT arrays the last sweeps filled, with the
// dtdx/dtdy/dtdz those sweeps used.
void oracle_fluxct(void* h, int iw, double k1, double k3) {
    auto& o = *static_cast<Oracle*>(h);
    bound_b(o, iw - 1);
    fluxct(o, iw, k1, k3);
}
void oracle_prot(void* h, int stage) { prot(*static_cast<Oracle*>(h), stage); }
void oracle_get_ct(void* h, int which, double* out) {
    auto& o = *static_cast<Oracle*>(h);
    std::memcpy(out, o.ct[which].data(), o.PV * sizeof(double));
}

// counts: [0] primit, [1] centre, [2] interface L/R, [3] one WENO field incl.
// amx (6 fabs + 6 fmax), [4] back-projection (7 FMA-pairs = 14) per field,
// [5] update per cell, [6] CT terms per interface, [7] sqrt share of [2].
void oracle_flop_counts(double* out, int cap) {
    const Prm P{5.0 / 3.0, 1e-12, 1e-12};
    double res[8] = {0};
    {
        Cnt q[8] = {1.0, 0.1, 0.2, 0.3, 0.5, 0.4, 0.3, 3.0}, u[9];
        Cnt::reset(); primit_cell(q, u, P); res[0] = (double)Cnt::total();
        Cnt a[7], F[7];
        Cnt::reset(); centre_cell(q, u, a, F, P); res[1] = (double)Cnt::total();
        Cnt u1[9]; for (int v = 0; v < 9; ++v) u1[v] = u[v].v * 1.01;
        Cnt L[49], R[49];
        Cnt::reset(); interface_LR(u, u1, L, R, P); res[2] = (double)Cnt::total(); res[7] = (double)Cnt::n_sqrt;
        Cnt F6[6][7], q6[6][7];
        for (int s = 0; s < 6; ++s) for (int v = 0; v < 7; ++v) { F6[s][v] = 0.1 * (s + v + 1); q6[s][v] = 0.05 * (s * v + 1); }
        Cnt::reset();
        Cnt amx = 0.0;
        for (int s = 0; s < 6; ++s) amx = fmax_(amx, fabs_(Cnt(0.3 * s)));
        Cnt fs = weno_field(L, F6, q6, amx);
        res[3] = (double)Cnt::total();
        Cnt::reset(); Cnt acc = 0.0; for (int r = 0; r < 7; ++r) acc += R[r] * fs; res[4] = (double)Cnt::total();
    }
    res[5] = 3.0;   // -dtdl * (a - b) per cell per component: sub, mul (sign folded) -> 2..3
    res[6] = 2.0 * (4 * 2 + 3 + 1 + 1);  // two CT terms: 4 products, 3 weights, 3 adds, 1 div, 1 add
    for (int i = 0; i < cap && i < 8; ++i) out[i] = res[i];
}

} // extern "C"
