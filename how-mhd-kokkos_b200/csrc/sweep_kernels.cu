// sweep_kernels.cu -- fused directional sweep: one kernel per x/y/z sweep of
// an SSPRK stage (src/ssprk.cpp:1000-1025, 1218-1272).
//
// The reference runs a sweep as six all-line kernels with workspaces in
// memory (qx, ux, ax, Fx and the 7x7 L and R per interface: ~18 GB at 256^3).
// Here one thread block owns a pencil tile of NL lines x T active cells and
// keeps every intermediate in shared memory; HBM sees only the stage input,
// the RK base, the stage output and the two CT flux arrays.
//
// Phases of one block (tile cells c in [0, T+6), interfaces f in [0, T]; the
// interface f sits between tile cells f+2 and f+3 and its WENO stencil is
// cells f..f+5, src/ssprk.cpp:861-865):
//   P0  load the 8 conserved variables of the tile, permuted to sweep order
//       (src/ssprk.cpp:1054-1061, 1145-1152), coalesced along x
//   P1  per cell: primitives with floors (458-516), eigenvalues and fluxes
//       (538-595)
//   P2a per interface: arithmetic-mean state and the eigen-system scalars
//       (610-660)
//   P2b per (interface, row): left-eigenvector row r and right-eigenvector
//       column r with normalisation and sign convention (662-818); the row
//       index is warp-uniform, so the 7 formula branches do not diverge
//   P3  per (interface pair, characteristic field m): projection of the
//       6-cell stencil, LLF split, WENO5-JS flux (841-937).  Seven threads
//       of a warp share a pair and read the same cells, so the shared-memory
//       loads broadcast; two interfaces per thread reuse 5 of 7 cells.
//   P4  per interface: back-projection R * F^ in m order (941-943), CT terms
//       (967-994) stored straight to the CT flux arrays (433-456 ...)
//   P5  per cell: -dtdl (F^_{i+1/2} - F^_{i-1/2}) (949-965) and the stage
//       accumulation (405-431, 1067-1096, 1158-1187)
#include "how_internal.cuh"

namespace how {

namespace {

__constant__ int c_perm[3][8] = {{0, 1, 2, 3, 4, 5, 6, 7},
                                 {0, 2, 3, 1, 5, 6, 4, 7},
                                 {0, 3, 1, 2, 6, 4, 5, 7}};

template <int NL, int T>
struct Tile {
    static constexpr int C = T + 6;
    static constexpr int F = T + 1;
    static constexpr int NP = (F + 1) / 2;
    static constexpr int NLC = NL * C;
    static constexpr int NLF = NL * F;
    static constexpr int NI = NLF | 1;              // odd interface pitch: conflict-free banks
    // shared-memory carve-up, in doubles
    static constexpr int oQ = 0;                    // [8][NLC] raw conserved
    static constexpr int oU = oQ + 8 * NLC;         // [NLC][14] F(7), q_proj(7)
    static constexpr int oP = oU + 14 * NLC;        // [9][NLC] primitives
    static constexpr int oA = oP + 9 * NLC;         // [7][NLC] eigenvalues
    static constexpr int oL = oA + 7 * NLC;         // [7 row][7 col][NI] left eigenvectors
    static constexpr int oR = oL + 49 * NI;         // [7 wave][7 phys][NI] right eigenvectors
    static constexpr int oS = oR + 49 * NI;         // [20][NI] scalars | Fs [7][NI], dF [7][NI]
    static constexpr int NS = 20;
    static constexpr int total = oS + NS * NI;
    static constexpr size_t bytes = sizeof(double) * (size_t)total;
};

enum { S_VX, S_VY, S_VZ, S_BY, S_BZ, S_VV2, S_CS, S_CS2, S_LF, S_LS, S_AF, S_AS, S_BTY,
       S_BTZ, S_SGNBX, S_SQR, S_ISQR, S_SGNBT, S_FLIP, S_BTV };

__device__ __forceinline__ double sign1(double x) { return (x >= 0.0) ? 1.0 : -1.0; }

// one WENO5-JS half in flux-difference form (src/ssprk.cpp:896-912).  The
// three nonlinear weights share one division: with e_k = (eps + IS_k)^2,
// omega0 = e1 e2 / D, omega2 = 3 e0 e1 / D, D = e1 e2 + 6 e0 e2 + 3 e0 e1.
__device__ __forceinline__ double weno_half(double a, double b, double c, double d) {
    const double eps = 1.0e-10;
    const double t0 = a - b, t1 = a - 3.0 * b;
    const double t2 = b - c, t3 = b + c;
    const double t4 = c - d, t5 = 3.0 * c - d;
    const double IS0 = 13.0 * t0 * t0 + 3.0 * t1 * t1;
    const double IS1 = 13.0 * t2 * t2 + 3.0 * t3 * t3;
    const double IS2 = 13.0 * t4 * t4 + 3.0 * t5 * t5;
    const double d0 = eps + IS0, d1 = eps + IS1, d2 = eps + IS2;
    const double e0 = d0 * d0, e1 = d1 * d1, e2 = d2 * d2;
    const double e12 = e1 * e2, e01 = e0 * e1;
    const double inv = 1.0 / (e12 + 6.0 * (e0 * e2) + 3.0 * e01);
    const double w0 = e12 * inv;
    const double w2 = 3.0 * e01 * inv;
    return w0 * (a - 2.0 * b + c) * (1.0 / 3.0) + (w2 - 0.5) * (b - 2.0 * c + d) * (1.0 / 6.0);
}

__device__ __forceinline__ double weno_flux(const double* Fsk, const double* qsk, double amx) {
    double dF[5], dq[5];
#pragma unroll
    for (int s = 0; s < 5; ++s) { dF[s] = Fsk[s + 1] - Fsk[s]; dq[s] = qsk[s + 1] - qsk[s]; }
    const double first = (-Fsk[1] + 7.0 * Fsk[2] + 7.0 * Fsk[3] - Fsk[4]) * (1.0 / 12.0);
    const double second = weno_half(0.5 * (dF[0] + amx * dq[0]), 0.5 * (dF[1] + amx * dq[1]),
                                    0.5 * (dF[2] + amx * dq[2]), 0.5 * (dF[3] + amx * dq[3]));
    const double third = weno_half(0.5 * (dF[4] - amx * dq[4]), 0.5 * (dF[3] - amx * dq[3]),
                                   0.5 * (dF[2] - amx * dq[2]), 0.5 * (dF[1] - amx * dq[1]));
    return first - second + third;
}

template <int DIR, int NL, int T, int NT>
__global__ void __launch_bounds__(NT, 4) k_sweep(SweepArgs a) {
    using TL = Tile<NL, T>;
    constexpr int C = TL::C, F = TL::F, NP = TL::NP, NLC = TL::NLC, NLF = TL::NLF, NI = TL::NI;
    extern __shared__ __align__(16) double sm[];
    double* sQ = sm + TL::oQ;
    double* sU = sm + TL::oU;
    double* sP = sm + TL::oP;
    double* sA = sm + TL::oA;
    double* sL = sm + TL::oL;
    double* sR = sm + TL::oR;
    double* sS = sm + TL::oS;
    double* sFs = sS;              // [7][NI], after P2b
    double* sdF = sS + 7 * NI;     // [7][NI], after P3

    const Grid& g = a.g;
    const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
    const int nt1 = DIR == 0 ? g.ny : g.nx;
    const long long sstride = DIR == 0 ? 1ll : DIR == 1 ? (long long)g.pitch : (long long)g.pitch * g.P1;
    const int c0 = blockIdx.x * T;                  // padded index of tile cell 0
    const int t1_0 = 3 + blockIdx.y * NL;
    const int t2 = 3 + blockIdx.z;
    const int tid = threadIdx.x;
    const int Pn = n + 6;

    auto line_off = [&](int l) -> long long {
        const int t1 = t1_0 + l;
        if (DIR == 0) return g.idx(0, t1, t2);
        if (DIR == 1) return g.idx(t1, 0, t2);
        return g.idx(t1, t2, 0);
    };
    auto line_ok = [&](int l) -> bool { return t1_0 + l <= nt1 + 2; };

    // ---------------------------------------------------------------- P0
    for (int t = tid; t < 8 * NLC; t += blockDim.x) {
        int v, l, c;
        if (DIR == 0) { v = t / NLC; const int r = t % NLC; l = r / C; c = r % C; }
        else { v = t / NLC; const int r = t % NLC; c = r / NL; l = r % NL; }
        double val = (v == 0 || v == 7) ? 1.0 : 0.0;
        if (line_ok(l) && c0 + c < Pn)
            val = a.qprev[(long long)c_perm[DIR][v] * g.fs + line_off(l) + (long long)(c0 + c) * sstride];
        sQ[v * NLC + l * C + c] = val;
    }
    __syncthreads();

    // ---------------------------------------------------------------- P1
    const double gam = a.gam;
    for (int t = tid; t < NLC; t += blockDim.x) {
        const double DD = sQ[0 * NLC + t], Mx = sQ[1 * NLC + t], My = sQ[2 * NLC + t];
        const double Mz = sQ[3 * NLC + t], Bx = sQ[4 * NLC + t], By = sQ[5 * NLC + t];
        const double Bz = sQ[6 * NLC + t];
        double EE = sQ[7 * NLC + t];
        // primit (src/ssprk.cpp:479-512): v from the unfloored density
        double rho = DD;
        double irho = 1.0 / rho;
        const double vx = Mx * irho, vy = My * irho, vz = Mz * irho;
        const double vv2 = vx * vx + vy * vy + vz * vz;
        const double BB2 = Bx * Bx + By * By + Bz * Bz;
        double pg = (gam - 1.0) * (EE - 0.5 * (rho * vv2 + BB2));
        if (rho < a.rhomin || pg < a.pgmin) {
            rho = fmax(a.rhomin, rho);
            pg = fmax(a.pgmin, pg);
            EE = pg / (gam - 1.0) + 0.5 * (rho * vv2 + BB2);
            irho = 1.0 / rho;
        }
        const double HH = (EE + pg) * irho;
        sP[0 * NLC + t] = rho; sP[1 * NLC + t] = vx; sP[2 * NLC + t] = vy; sP[3 * NLC + t] = vz;
        sP[4 * NLC + t] = Bx; sP[5 * NLC + t] = By; sP[6 * NLC + t] = Bz; sP[7 * NLC + t] = pg;
        sP[8 * NLC + t] = HH;
        // eigenst centre (src/ssprk.cpp:561-593), with DD, EE the floored values
        const double pt = pg + 0.5 * BB2;
        const double vdB = vx * Bx + vy * By + vz * Bz;
        const double bbn2 = BB2 * irho;
        const double bnx2 = Bx * Bx * irho;
        const double cs2 = fmax(0.0, gam * fabs(pg * irho));
        const double root = sqrt(fmax(0.0, (bbn2 + cs2) * (bbn2 + cs2) - 4.0 * bnx2 * cs2));
        const double lf = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 + root)));
        const double la = sqrt(fmax(0.0, bnx2));
        const double ls = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 - root)));
        sA[0 * NLC + t] = vx - lf; sA[1 * NLC + t] = vx - la; sA[2 * NLC + t] = vx - ls;
        sA[3 * NLC + t] = vx;      sA[4 * NLC + t] = vx + ls; sA[5 * NLC + t] = vx + la;
        sA[6 * NLC + t] = vx + lf;
        double* U = sU + t * 14;
        U[0] = rho * vx;                 // DD (floored) * vx
        U[1] = Mx * vx + pt - Bx * Bx;
        U[2] = My * vx - Bx * By;
        U[3] = Mz * vx - Bx * Bz;
        U[4] = By * vx - Bx * vy;
        U[5] = Bz * vx - Bx * vz;
        U[6] = (EE + pt) * vx - Bx * vdB;
        U[7] = rho; U[8] = Mx; U[9] = My; U[10] = Mz; U[11] = By; U[12] = Bz; U[13] = EE;
    }
    __syncthreads();

    // ---------------------------------------------------------------- P2a
    const double gam0 = 1.0 - gam, gam1 = 0.5 * (gam - 1.0);
    for (int t = tid; t < NLF; t += blockDim.x) {
        const int l = t / F, f = t % F;
        const int c = l * C + f + 2;
        const double rho = 0.5 * (sP[0 * NLC + c] + sP[0 * NLC + c + 1]);
        const double vx = 0.5 * (sP[1 * NLC + c] + sP[1 * NLC + c + 1]);
        const double vy = 0.5 * (sP[2 * NLC + c] + sP[2 * NLC + c + 1]);
        const double vz = 0.5 * (sP[3 * NLC + c] + sP[3 * NLC + c + 1]);
        const double Bx = 0.5 * (sP[4 * NLC + c] + sP[4 * NLC + c + 1]);
        const double By = 0.5 * (sP[5 * NLC + c] + sP[5 * NLC + c + 1]);
        const double Bz = 0.5 * (sP[6 * NLC + c] + sP[6 * NLC + c + 1]);
        const double HH = 0.5 * (sP[8 * NLC + c] + sP[8 * NLC + c + 1]);
        const double vv2 = vx * vx + vy * vy + vz * vz;
        const double BB2 = Bx * Bx + By * By + Bz * Bz;
        const double isqr = rsqrt(rho);
        const double irho = isqr * isqr;
        const double bbn2 = BB2 * irho;
        const double bnx2 = Bx * Bx * irho;
        const double cs2 = (gam - 1.0) * (HH - 0.5 * (vv2 + bbn2));
        const double cs = sqrt(fmax(0.0, cs2));
        const double root = sqrt(fmax(0.0, (bbn2 + cs2) * (bbn2 + cs2) - 4.0 * bnx2 * cs2));
        const double lf = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 + root)));
        const double la = fabs(Bx) * isqr;
        const double ls = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 - root)));
        const double Bt2 = By * By + Bz * Bz;
        double bty, btz;
        if (Bt2 >= 1.0e-30) { const double ib = rsqrt(Bt2); bty = By * ib; btz = Bz * ib; }
        else { bty = 0.70710678118654752440; btz = 0.70710678118654752440; }
        double af, as;
        const double df = lf * lf - ls * ls;
        if (df >= 1.0e-30) {
            const double idf = rsqrt(df);
            af = sqrt(fmax(0.0, cs2 - ls * ls)) * idf;
            as = sqrt(fmax(0.0, lf * lf - cs2)) * idf;
        } else { af = 1.0; as = 1.0; }
        double* S = sS + t;
        S[S_VX * NI] = vx; S[S_VY * NI] = vy; S[S_VZ * NI] = vz;
        S[S_BY * NI] = By; S[S_BZ * NI] = Bz; S[S_VV2 * NI] = vv2;
        S[S_CS * NI] = cs; S[S_CS2 * NI] = cs2; S[S_LF * NI] = lf; S[S_LS * NI] = ls;
        S[S_AF * NI] = af; S[S_AS * NI] = as; S[S_BTY * NI] = bty; S[S_BTZ * NI] = btz;
        S[S_SGNBX * NI] = sign1(Bx);
        S[S_SQR * NI] = rho * isqr; S[S_ISQR * NI] = isqr;
        S[S_SGNBT * NI] = (By != 0.0) ? sign1(By) : sign1(Bz);
        S[S_FLIP * NI] = (cs >= la) ? 1.0 : 0.0;
        S[S_BTV * NI] = bty * vy + btz * vz;
    }
    __syncthreads();

    // ---------------------------------------------------------------- P2b
    const double gam2 = (gam - 2.0) / (gam - 1.0);
    for (int t = tid; t < 7 * NLF; t += blockDim.x) {
        const int r = t / NLF, i = t % NLF;
        const double* S = sS + i;
        const double vx = S[S_VX * NI], vy = S[S_VY * NI], vz = S[S_VZ * NI];
        const double By = S[S_BY * NI], Bz = S[S_BZ * NI], vv2 = S[S_VV2 * NI];
        const double cs = S[S_CS * NI], cs2 = S[S_CS2 * NI];
        const double lf = S[S_LF * NI], ls = S[S_LS * NI], af = S[S_AF * NI], as = S[S_AS * NI];
        const double bty = S[S_BTY * NI], btz = S[S_BTZ * NI], sgnBx = S[S_SGNBX * NI];
        const double sqrtrho = S[S_SQR * NI], isqr = S[S_ISQR * NI], sgnBt = S[S_SGNBT * NI];
        const bool flip24 = S[S_FLIP * NI] != 0.0;
        const double btv = S[S_BTV * NI];
        double L[7], R[7];
        switch (r) {
            case 0: {
                L[0] = af * (gam1 * vv2 + lf * vx) - as * ls * btv * sgnBx;
                L[1] = af * (gam0 * vx - lf);
                L[2] = gam0 * af * vy + as * ls * bty * sgnBx;
                L[3] = gam0 * af * vz + as * ls * btz * sgnBx;
                L[4] = gam0 * af * By + cs * as * bty * sqrtrho;
                L[5] = gam0 * af * Bz + cs * as * btz * sqrtrho;
                L[6] = -gam0 * af;
                const double s = 0.5 / cs2;
#pragma unroll
                for (int m = 0; m < 7; ++m) L[m] *= s;
                R[0] = af; R[1] = af * (vx - lf);
                R[2] = af * vy + as * ls * bty * sgnBx; R[3] = af * vz + as * ls * btz * sgnBx;
                R[4] = cs * as * bty * isqr; R[5] = cs * as * btz * isqr;
                R[6] = af * (lf * lf - lf * vx + 0.5 * vv2 - gam2 * cs2) + as * ls * btv * sgnBx;
                break;
            }
            case 1: {
                L[0] = 0.5 * (btz * vy - bty * vz); L[1] = 0.0; L[2] = -0.5 * btz; L[3] = 0.5 * bty;
                L[4] = 0.5 * (-btz * sgnBx * sqrtrho); L[5] = 0.5 * (bty * sgnBx * sqrtrho); L[6] = 0.0;
                R[0] = 0.0; R[1] = 0.0; R[2] = -btz; R[3] = bty;
                R[4] = -btz * sgnBx * isqr; R[5] = bty * sgnBx * isqr; R[6] = bty * vz - btz * vy;
                break;
            }
            case 2: {
                L[0] = as * (gam1 * vv2 + ls * vx) + af * lf * btv * sgnBx;
                L[1] = gam0 * as * vx - as * ls;
                L[2] = gam0 * as * vy - af * lf * bty * sgnBx;
                L[3] = gam0 * as * vz - af * lf * btz * sgnBx;
                L[4] = gam0 * as * By - cs * af * bty * sqrtrho;
                L[5] = gam0 * as * Bz - cs * af * btz * sqrtrho;
                L[6] = -gam0 * as;
                const double s = 0.5 / cs2;
#pragma unroll
                for (int m = 0; m < 7; ++m) L[m] *= s;
                R[0] = as; R[1] = as * (vx - ls);
                R[2] = as * vy - af * lf * bty * sgnBx; R[3] = as * vz - af * lf * btz * sgnBx;
                R[4] = -cs * af * bty * isqr; R[5] = -cs * af * btz * isqr;
                R[6] = as * (ls * ls - ls * vx + 0.5 * vv2 - gam2 * cs2) - af * lf * btv * sgnBx;
                break;
            }
            case 3: {
                const double s = -gam0 / cs2;
                L[0] = (-cs2 / gam0 - 0.5 * vv2) * s; L[1] = vx * s; L[2] = vy * s; L[3] = vz * s;
                L[4] = By * s; L[5] = Bz * s; L[6] = -s;
                R[0] = 1.0; R[1] = vx; R[2] = vy; R[3] = vz; R[4] = 0.0; R[5] = 0.0; R[6] = 0.5 * vv2;
                break;
            }
            case 4: {
                L[0] = as * (gam1 * vv2 - ls * vx) - af * lf * btv * sgnBx;
                L[1] = as * (gam0 * vx + ls);
                L[2] = gam0 * as * vy + af * lf * bty * sgnBx;
                L[3] = gam0 * as * vz + af * lf * btz * sgnBx;
                L[4] = gam0 * as * By - cs * af * bty * sqrtrho;
                L[5] = gam0 * as * Bz - cs * af * btz * sqrtrho;
                L[6] = -gam0 * as;
                const double s = 0.5 / cs2;
#pragma unroll
                for (int m = 0; m < 7; ++m) L[m] *= s;
                R[0] = as; R[1] = as * (vx + ls);
                R[2] = as * vy + af * lf * bty * sgnBx; R[3] = as * vz + af * lf * btz * sgnBx;
                R[4] = -cs * af * bty * isqr; R[5] = -cs * af * btz * isqr;
                R[6] = as * (ls * ls + ls * vx + 0.5 * vv2 - gam2 * cs2) + af * lf * btv * sgnBx;
                break;
            }
            case 5: {
                L[0] = 0.5 * (btz * vy - bty * vz); L[1] = 0.0; L[2] = -0.5 * btz; L[3] = 0.5 * bty;
                L[4] = 0.5 * (btz * sgnBx * sqrtrho); L[5] = 0.5 * (-bty * sgnBx * sqrtrho); L[6] = 0.0;
                R[0] = 0.0; R[1] = 0.0; R[2] = -btz; R[3] = bty;
                R[4] = btz * sgnBx * isqr; R[5] = -bty * sgnBx * isqr; R[6] = bty * vz - btz * vy;
                break;
            }
            default: {
                L[0] = af * (gam1 * vv2 - lf * vx) + as * ls * btv * sgnBx;
                L[1] = af * (gam0 * vx + lf);
                L[2] = gam0 * af * vy - as * ls * bty * sgnBx;
                L[3] = gam0 * af * vz - as * ls * btz * sgnBx;
                L[4] = gam0 * af * By + cs * as * bty * sqrtrho;
                L[5] = gam0 * af * Bz + cs * as * btz * sqrtrho;
                L[6] = -gam0 * af;
                const double s = 0.5 / cs2;
#pragma unroll
                for (int m = 0; m < 7; ++m) L[m] *= s;
                R[0] = af; R[1] = af * (vx + lf);
                R[2] = af * vy - as * ls * bty * sgnBx; R[3] = af * vz - as * ls * btz * sgnBx;
                R[4] = cs * as * bty * isqr; R[5] = cs * as * btz * isqr;
                R[6] = af * (lf * lf + lf * vx + 0.5 * vv2 - gam2 * cs2) - as * ls * btv * sgnBx;
                break;
            }
        }
        // sign convention (src/ssprk.cpp:789-818)
        const bool flip = flip24 ? (r == 2 || r == 4) : (r == 0 || r == 6);
#pragma unroll
        for (int m = 0; m < 7; ++m) {
            sL[(r * 7 + m) * NI + i] = flip ? L[m] * sgnBt : L[m];
            sR[(r * 7 + m) * NI + i] = flip ? R[m] * sgnBt : R[m];
        }
    }
    __syncthreads();

    // ---------------------------------------------------------------- P3
    for (int t = tid; t < 7 * NL * NP; t += blockDim.x) {
        const int m = t % 7, pr = t / 7;
        const int l = pr / NP, p = pr % NP;
        const int f0 = 2 * p;
        const bool has1 = f0 + 1 < F;
        const int i0 = l * F + f0;
        const int i1 = has1 ? i0 + 1 : i0;
        double L0[7], L1[7];
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            L0[v] = sL[(m * 7 + v) * NI + i0];
            L1[v] = sL[(m * 7 + v) * NI + i1];
        }
        double Fk0[6], qk0[6], Fk1[6], qk1[6];
        double amx0 = 0.0, amx1 = 0.0;
#pragma unroll
        for (int cc = 0; cc < 7; ++cc) {
            int c = f0 + cc;
            c = c < C ? c : C - 1;
            const double2* u = reinterpret_cast<const double2*>(sU + (l * C + c) * 14);
            double U[14];
#pragma unroll
            for (int h = 0; h < 7; ++h) { const double2 x = u[h]; U[2 * h] = x.x; U[2 * h + 1] = x.y; }
            const double av = fabs(sA[m * NLC + l * C + c]);
            if (cc <= 5) {
                double pf = L0[0] * U[0], pq = L0[0] * U[7];
#pragma unroll
                for (int v = 1; v < 7; ++v) { pf += L0[v] * U[v]; pq += L0[v] * U[7 + v]; }
                Fk0[cc] = pf; qk0[cc] = pq;
                amx0 = fmax(amx0, av);
            }
            if (cc >= 1) {
                double pf = L1[0] * U[0], pq = L1[0] * U[7];
#pragma unroll
                for (int v = 1; v < 7; ++v) { pf += L1[v] * U[v]; pq += L1[v] * U[7 + v]; }
                Fk1[cc - 1] = pf; qk1[cc - 1] = pq;
                amx1 = fmax(amx1, av);
            }
        }
        sFs[m * NI + i0] = weno_flux(Fk0, qk0, amx0);
        if (has1) sFs[m * NI + i1] = weno_flux(Fk1, qk1, amx1);
    }
    __syncthreads();

    // ---------------------------------------------------------------- P4
    for (int t = tid; t < NLF; t += blockDim.x) {
        const int l = t / F, f = t % F;
        double dF[7];
#pragma unroll
        for (int r = 0; r < 7; ++r) dF[r] = 0.0;
#pragma unroll
        for (int m = 0; m < 7; ++m) {
            const double fs = sFs[m * NI + t];
#pragma unroll
            for (int r = 0; r < 7; ++r) dF[r] += sR[(m * 7 + r) * NI + t] * fs;
        }
#pragma unroll
        for (int r = 0; r < 7; ++r) sdF[r * NI + t] = dF[r];
        // CT terms (src/ssprk.cpp:973-993): mean of B_n v_t over the two cells
        const int c = l * C + f + 2;
        const double x1 = sP[4 * NLC + c] * sP[2 * NLC + c], x2 = sP[4 * NLC + c + 1] * sP[2 * NLC + c + 1];
        const double y1 = sP[4 * NLC + c] * sP[3 * NLC + c], y2 = sP[4 * NLC + c + 1] * sP[3 * NLC + c + 1];
        const int iface = c0 + f;   // global interface index, face at padded iface + 2
        if (line_ok(l) && iface <= n) {
            const long long o = line_off(l) + (long long)(iface + 2) * sstride;
            a.cta[o] = dF[4] + (9.0 * x1 + 9.0 * x2) / 18.0;
            a.ctb[o] = dF[5] + (9.0 * y1 + 9.0 * y2) / 18.0;
        }
    }
    __syncthreads();

    // ---------------------------------------------------------------- P5
    const double dtdl = *a.dtdl;
    for (int t = tid; t < 8 * NL * T; t += blockDim.x) {
        int v, l, ct;
        if (DIR == 0) { v = t / (NL * T); const int r = t % (NL * T); l = r / T; ct = r % T; }
        else { v = t / (NL * T); const int r = t % (NL * T); ct = r / NL; l = r % NL; }
        const int s = c0 + ct + 3;
        if (!line_ok(l) || s > n + 2) continue;
        const int rr = v < 4 ? v : v - 1;     // flux row of line variable v (v = 4: normal B)
        const int fi = l * F + ct;
        const double delta = (v == 4) ? 0.0 : -dtdl * (sdF[rr * NI + fi + 1] - sdF[rr * NI + fi]);
        const long long o = (long long)c_perm[DIR][v] * g.fs + line_off(l) + (long long)s * sstride;
        if (a.mode == 0) {
            if (v != 4) a.qout[o] += delta;
        } else {
            double base = a.q0[o];
            if (a.stage5) base = base + a.c4 * a.q2[o] + a.c5 * a.q3[o];
            if (a.mode == 1) a.qout[o] = a.k1 * base + a.k3 * sQ[v * NLC + l * C + ct + 3] + delta;
            else a.qout[o] = base + delta;
        }
    }
}

template <int DIR, int NL, int T, int NT>
void launch_one(Ctx& c, const SweepArgs& a) {
    using TL = Tile<NL, T>;
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(k_sweep<DIR, NL, T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TL::bytes);
        attr_done = true;
    }
    const Grid& g = c.g;
    const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
    const int nt1 = DIR == 0 ? g.ny : g.nx;
    const int nt2 = DIR == 2 ? g.ny : g.nz;
    dim3 grid((n + T - 1) / T, (nt1 + NL - 1) / NL, nt2);
    cudaEvent_t ev[2];
    timer_begin(c, ev);
    k_sweep<DIR, NL, T, NT><<<grid, NT, TL::bytes, c.stream>>>(a);
    timer_end(c, ev);
    ++c.launches;
}

}  // namespace

void launch_sweep(Ctx& c, int dir, const SweepArgs& a) {
    if (dir == 0) launch_one<0, 1, 32, 128>(c, a);
    else if (dir == 1) launch_one<1, 2, 16, 128>(c, a);
    else launch_one<2, 2, 16, 128>(c, a);
}

}  // namespace how
