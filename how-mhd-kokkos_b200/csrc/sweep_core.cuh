// sweep_core.cuh -- the fused directional sweep kernel: one launch per x/y/z
// sweep of an SSPRK stage (src/ssprk.cpp:1000-1025, 1218-1272).  Included by
// sweep_kernels.cu (single-domain launches) and ensemble_sweep.cu (batched
// ensembles); each translation unit instantiates the shapes it launches.
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
//   P0  the 8 conserved variables of the tile (with its 3-cell halo) and the
//       update's read operand arrive by TMA tensor loads issued one tile
//       ahead: blocks are persistent and double-buffer the tiles, so the
//       HBM latency of tile n+1 hides behind the arithmetic of tile n.  The
//       variable permutation of the y/z sweeps (src/ssprk.cpp:1054-1061,
//       1145-1152) is applied when the tile is read from shared memory.
//   P1  per cell: primitives with floors (458-516), eigenvalues and fluxes
//       (538-595)
//   P1b per cell: differences dU(c) = U(c+1) - U(c) of (F, q_proj)
//   P2a per interface: arithmetic-mean state and the eigen-system scalars
//       (610-660)
//   P3  per (interface, characteristic field m): the left-eigenvector row m,
//       built in registers from the interface's scalars
//       (662-726, 789-818), projection of the stencil's 5 cell differences,
//       LLF split, WENO5-JS flux (841-937).  Seven threads of a warp share an
//       interface and read the same cells and scalars, so the shared-memory
//       loads broadcast (below five blocks per SM a thread takes two
//       interfaces and reuses 4 of their 6 differences).  The
//       central part's F_{i} share is not projected: with R L = I it is added
//       back in physical space in P4.
//   P4  per (interface, flux component r): row r of the right-eigenvector
//       matrix, built in registers from the scalars (729-818), the
//       back-projection sum_m R(r,m) F^_m in m order (941-943), CT terms
//       (967-994) stored straight to the CT flux arrays (433-456 ...)
//   The 7x7 eigenvector matrices are never stored: shared memory holds 21
//   scalars per interface instead of 98 matrix entries.
//   P5  per cell: -dtdl (F^_{i+1/2} - F^_{i-1/2}) (949-965) and the stage
//       accumulation (405-431, 1067-1096, 1158-1187)
//
// Precision: the kernel is a template on the working type R of the
// eigen-system, projection and WENO arithmetic (P2a-P4's characteristic part).
// R = double is the plain method.  R = float is the mixed-precision method:
// primitives, cell fluxes, the physical central flux F_i, the back-projected
// interface flux sum, the CT terms and the stage update stay FP64; the FP32
// part only carries the characteristic upwind corrections, computed from cell
// differences that are formed in FP64 and then rounded.
#pragma once

#include "how_internal.cuh"
#include "router.cuh"
#include "tma.cuh"

#include <type_traits>

namespace how {

namespace {

template <typename R> struct Math;
template <> struct Math<double> {
    using V2 = double2;
    static __device__ __forceinline__ double sq(double x) { return sqrt(x); }
    static __device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
};
template <> struct Math<float> {
    using V2 = float2;
    static __device__ __forceinline__ float sq(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
    static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
};

__host__ __device__ constexpr int align_up(int x, int a) { return (x + a - 1) / a * a; }

template <int DIR, int NL, int T, typename R>
struct Tile {
    static constexpr int C = T + 6;
    static constexpr int F = T + 1;
    static constexpr int NP = (F + 1) / 2;
    static constexpr int NLC = NL * C;
    static constexpr int NLF = NL * F;
    static constexpr int NI = NLF | 1;              // odd interface pitch: conflict-free banks
    // update tile: x starts one cell early so its innermost TMA coordinate is even
    static constexpr int TO = DIR == 0 ? T + 2 : T;
    static constexpr int NQ = 8 * NLC;              // raw tile, TMA box order [var][...]
    static constexpr int NO = 8 * NL * TO;          // update operand tile
    static constexpr int NS = 21;                   // eigen-system scalars per interface
    // byte offsets (base 128-byte aligned; TMA destinations on 128 B)
    static constexpr int bQ = 0;                                   // NBUF x [8][..] raw conserved, FP64
    static constexpr int NBUF = 2;                                // raw tiles in flight (this + 1 ahead)
    static constexpr int NOB = 2;                                 // update operands in flight (this + next)
    static constexpr int bO = bQ + NBUF * align_up(8 * NQ, 128);   // NOB x [8][..] update operand, FP64
    static constexpr int bFc = bO + NOB * align_up(8 * NO, 128);   // [NLC][7] cell fluxes, FP64
    static constexpr int bP = bFc + align_up(8 * 7 * NLC, 16);     // [9][NLC] primitives, FP64
    static constexpr int bA = bP + align_up(8 * 9 * NLC, 16);      // [7][NLC] eigenvalues, R
    static constexpr int bD = bA + align_up((int)sizeof(R) * 7 * NLC, 16);  // [NLC][14] dU, R
    // U = (F, q_proj) staged in FP64 from P1 to P1b; after P1b the same bytes
    // hold the characteristic fluxes Fs [7][NI] (R, P3 -> P4) and the
    // interface fluxes dF [7][NI] (FP64, P4 -> P5)
    static constexpr int bU = bD + align_up((int)sizeof(R) * 14 * NLC, 16);
    static constexpr int offdF = align_up((int)sizeof(R) * 7 * NI, 8);
    static constexpr int szU0 = 8 * 14 * NLC;
    static constexpr int szU1 = offdF + 8 * 7 * NI;
    // [NS][NI] eigen-system scalars of the interfaces (P2a -> P3, P4): the
    // left rows and right columns are rebuilt from them in registers where
    // they are used, never stored
    static constexpr int bS = bU + align_up(szU0 > szU1 ? szU0 : szU1, 16);
    static constexpr int bB = bS + align_up((int)sizeof(R) * NS * NI, 16);   // NBUF + NOB mbarriers
    static constexpr int szB = align_up(8 * (NBUF + NOB), 16);
    // routing (MODE 1-3): decision, compacted list, weight deviation and FP32
    // features of the tile's interfaces (collection), the linear flux's LF
    // speed, the cells' routing values (guard and collection)
    static constexpr int bDec = bB + szB;                         // [NLF] int
    static constexpr int bList = bDec + align_up(4 * NLF, 16);    // [NLF] int
    static constexpr int bDev = bList + align_up(4 * NLF, 16);    // [NLF] float (bits)
    static constexpr int bFlx = bDev + align_up(4 * NLF, 16);     // [NLF] float (bits): flux departure
    static constexpr int bFt = bFlx + align_up(4 * NLF, 16);      // [NLF][6] float
    static constexpr int bAmx = bFt + align_up(4 * 6 * NLF, 16);  // [NLF] R: linear-flux LF speed
    static constexpr int bCF = bAmx + align_up((int)sizeof(R) * NLF, 16);   // [5][NLC] float cell features
    static constexpr int bDecW = bCF + align_up(4 * 5 * NLC, 16);  // [NL][F+2] int: fetched decisions
    static constexpr int bEnd = bDecW + align_up(4 * NL * (F + 2), 16);
    // learned routing (MODE 1) keeps only what it uses: decisions, list, LF
    // speed, the cells' density and pressure (the guard), fetched decisions
    // (two sets: this tile's and the next tile's)
    static constexpr int lDec = bB + szB;
    static constexpr int lList = lDec + align_up(4 * NLF, 16);
    static constexpr int lAmx = lList + align_up(4 * NLF, 16);
    static constexpr int lCF = lAmx + align_up((int)sizeof(R) * NLF, 16);
    static constexpr int lDecW = lCF + align_up(4 * 2 * NLC, 16);
    static constexpr int lEnd = lDecW + 2 * align_up(4 * NL * (F + 2), 16);
    static constexpr size_t bytes_learned = (size_t)lEnd;
    static constexpr size_t bytes_plain = (size_t)bB + (NBUF + NOB) * 8;
    static constexpr size_t bytes_route = (size_t)bEnd;
    static constexpr uint32_t in_bytes = 8u * NQ;
    static constexpr uint32_t out_bytes = 8u * NO;
};

enum { S_VX, S_VY, S_VZ, S_BY, S_BZ, S_VV2, S_CS, S_CS2, S_LF, S_LS, S_AF, S_AS, S_BTY,
       S_BTZ, S_SGNBX, S_SQR, S_ISQR, S_SGNBT, S_FLIP, S_BTV, S_ICS2 };

template <typename R>
__device__ __forceinline__ R sign1(R x) { return (x >= R(0)) ? R(1) : R(-1); }

// The eigenvectors at one interface (src/ssprk.cpp:662-818), rebuilt from its
// eigen-system scalars S[k * NI] (the S_* table above) where they are used.
// Column / row m = 0..6 is the field with eigenvalue v - c_f, v - c_a,
// v - c_s, v, v + c_s, v + c_a, v + c_f.
//
// The four magnetosonic fields share one form: with sigma = -1 (m = 0, 2) or
// +1 (m = 4, 6), and for the fast fields (m = 0, 6) (a1, a2, l1, l2, tau) =
// (alpha_f, alpha_s, c_f, c_s, +1), for the slow ones (m = 2, 4)
// (alpha_s, alpha_f, c_s, c_f, -1), the reference's four row (and column)
// formulas are one expression in those symbols, so the seven lanes that
// build the seven rows of an interface take three branches, not seven.
//
// Sign convention (src/ssprk.cpp:789-818): the fast columns (m = 0, 6), or
// the slow ones (m = 2, 4) when c_s >= c_a, change sign with sgn(B_t).
template <typename R, int NI>
__device__ __forceinline__ R eig_col_sign(int m, const R* S) {
    const bool flip24 = S[S_FLIP * NI] != R(0);
    const bool flip = flip24 ? (m == 2 || m == 4) : (m == 0 || m == 6);
    return flip ? S[S_SGNBT * NI] : R(1);
}

// Left-eigenvector row m, normalised (src/ssprk.cpp:662-726).
template <typename R, int NI>
__device__ __forceinline__ void eig_left_row(int m, const R* S, R gam0, R gam1, R* L) {
    if (m == 3) {
        // row (-c^2/gam0 - v^2/2, v, B_t, -1) times s = -gam0/c^2; its first
        // entry (-c^2/gam0 - v^2/2) s = 1 - (v^2/2) s needs no division
        const R ics2 = S[S_ICS2 * NI], vv2 = S[S_VV2 * NI];
        const R s = -gam0 * ics2;
        L[0] = R(1) - R(0.5) * vv2 * s;
        L[1] = S[S_VX * NI] * s; L[2] = S[S_VY * NI] * s; L[3] = S[S_VZ * NI] * s;
        L[4] = S[S_BY * NI] * s; L[5] = S[S_BZ * NI] * s; L[6] = -s;
    } else if (m == 1 || m == 5) {
        const R rs = m == 1 ? R(-1) : R(1);
        const R bty = S[S_BTY * NI], btz = S[S_BTZ * NI], sb = S[S_SGNBX * NI] * S[S_SQR * NI];
        L[0] = R(0.5) * (btz * S[S_VY * NI] - bty * S[S_VZ * NI]);
        L[1] = R(0); L[2] = R(-0.5) * btz; L[3] = R(0.5) * bty;
        L[4] = R(0.5) * (rs * btz * sb); L[5] = R(0.5) * (-rs * bty * sb); L[6] = R(0);
    } else {
        const bool fast = m == 0 || m == 6;
        const R sig = m < 3 ? R(-1) : R(1), tau = fast ? R(1) : R(-1), ts = tau * sig;
        const R af = S[S_AF * NI], as = S[S_AS * NI], lf = S[S_LF * NI], ls = S[S_LS * NI];
        const R a1 = fast ? af : as, a2 = fast ? as : af, l1 = fast ? lf : ls, l2 = fast ? ls : lf;
        const R vx = S[S_VX * NI], sgnBx = S[S_SGNBX * NI], bty = S[S_BTY * NI], btz = S[S_BTZ * NI];
        const R a2l2 = ts * a2 * l2 * sgnBx, csa2 = tau * S[S_CS * NI] * a2 * S[S_SQR * NI];
        L[0] = a1 * (gam1 * S[S_VV2 * NI] - sig * l1 * vx) + a2l2 * S[S_BTV * NI];
        L[1] = a1 * (gam0 * vx + sig * l1);
        L[2] = gam0 * a1 * S[S_VY * NI] - a2l2 * bty;
        L[3] = gam0 * a1 * S[S_VZ * NI] - a2l2 * btz;
        L[4] = gam0 * a1 * S[S_BY * NI] + csa2 * bty;
        L[5] = gam0 * a1 * S[S_BZ * NI] + csa2 * btz;
        L[6] = -gam0 * a1;
        // normalisation and the sign convention (only magnetosonic rows flip)
        const R s = R(0.5) * S[S_ICS2 * NI] * eig_col_sign<R, NI>(m, S);
#pragma unroll
        for (int k = 0; k < 7; ++k) L[k] *= s;
    }
}

// Row r of the right-eigenvector matrix, R(r, m) for m = 0..6
// (src/ssprk.cpp:729-787): component r of every column.
template <typename R, int NI>
__device__ __forceinline__ void eig_right_row(int r, const R* S, R gam2, R* Rr) {
    const R af = S[S_AF * NI], as = S[S_AS * NI];
    switch (r) {
        case 0:
            Rr[0] = af; Rr[1] = R(0); Rr[2] = as; Rr[3] = R(1); Rr[4] = as; Rr[5] = R(0); Rr[6] = af;
            break;
        case 1: {
            const R vx = S[S_VX * NI], lf = S[S_LF * NI], ls = S[S_LS * NI];
            Rr[0] = af * (vx - lf); Rr[1] = R(0); Rr[2] = as * (vx - ls); Rr[3] = vx;
            Rr[4] = as * (vx + ls); Rr[5] = R(0); Rr[6] = af * (vx + lf);
            break;
        }
        case 2:
        case 3: {
            const R v = S[(r == 2 ? S_VY : S_VZ) * NI], bt = S[(r == 2 ? S_BTY : S_BTZ) * NI];
            const R sgnBx = S[S_SGNBX * NI];
            const R pf = as * S[S_LS * NI] * bt * sgnBx, ps = af * S[S_LF * NI] * bt * sgnBx;
            const R alf = r == 2 ? -S[S_BTZ * NI] : S[S_BTY * NI];
            Rr[0] = af * v + pf; Rr[1] = alf; Rr[2] = as * v - ps; Rr[3] = v;
            Rr[4] = as * v + ps; Rr[5] = alf; Rr[6] = af * v - pf;
            break;
        }
        case 4:
        case 5: {
            const R bt = S[(r == 4 ? S_BTY : S_BTZ) * NI], isqr = S[S_ISQR * NI];
            const R cs = S[S_CS * NI];
            const R f = cs * as * bt * isqr, sl = -cs * af * bt * isqr;
            const R alf = (r == 4 ? -S[S_BTZ * NI] : S[S_BTY * NI]) * S[S_SGNBX * NI] * isqr;
            Rr[0] = f; Rr[1] = alf; Rr[2] = sl; Rr[3] = R(0); Rr[4] = sl; Rr[5] = -alf; Rr[6] = f;
            break;
        }
        default: {
            const R vx = S[S_VX * NI], vv2 = S[S_VV2 * NI], lf = S[S_LF * NI], ls = S[S_LS * NI];
            const R h = R(0.5) * vv2 - gam2 * S[S_CS2 * NI];
            const R btv = S[S_BTV * NI] * S[S_SGNBX * NI];
            const R pf = as * ls * btv, ps = af * lf * btv;
            const R alf = S[S_BTY * NI] * S[S_VZ * NI] - S[S_BTZ * NI] * S[S_VY * NI];
            Rr[0] = af * (lf * lf - lf * vx + h) + pf; Rr[1] = alf;
            Rr[2] = as * (ls * ls - ls * vx + h) - ps; Rr[3] = R(0.5) * vv2;
            Rr[4] = as * (ls * ls + ls * vx + h) + ps; Rr[5] = alf;
            Rr[6] = af * (lf * lf + lf * vx + h) - pf;
            break;
        }
    }
    const R sgnBt = S[S_SGNBT * NI];
    if (S[S_FLIP * NI] != R(0)) { Rr[2] *= sgnBt; Rr[4] *= sgnBt; }
    else { Rr[0] *= sgnBt; Rr[6] *= sgnBt; }
}

// Characteristic WENO5-JS/LLF flux of one field (src/ssprk.cpp:883-937) from
// the projected cell differences dF_k = L.(F_{k+1} - F_k), dq_k = L.(q_{k+1} - q_k),
// k = 0..4 over the 6-cell stencil.
//
// Restated, not transcribed:
//  * the fourth-order central part (-F1 + 7F2 + 7F3 - F4)/12 equals
//    F2 + (dF1 + 6 dF2 - dF3)/12; its F2 share is added back in physical
//    space after the back-projection (R L = I), so only the correction is
//    returned;
//  * the LLF-split arguments 0.5 (dF +- amx dq) are used without the 0.5:
//    doubling a, b, c, d quadruples every smoothness indicator, so with
//    eps -> 4 eps the nonlinear weights are unchanged and the 0.5 moves onto
//    the linear combination (1/3 -> 1/6, 1/6 -> 1/12);
//  * FP64: omega0 = a0 / (a0 + a1 + a2) with a_k = c_k / (eps + IS_k)^2 is
//    e1 e2 / D with e_k = (eps + IS_k)^2 and D = e1 e2 + 6 e0 e2 + 3 e0 e1
//    (omega2 = 3 e0 e1 / D); the two halves share one division 1/(D+ D-).
//    FP32 keeps the a_k form (the products of e_k would underflow) with fast
//    reciprocals.
template <typename R>
__device__ __forceinline__ R weno_half_w(R a, R b, R c, R d, R& w0, R& w2) {
    const R eps4 = R(4.0e-10);
    const R t0 = a - b, t1 = a - R(3) * b;
    const R t2 = b - c, t3 = b + c;
    const R t4 = c - d, t5 = R(3) * c - d;
    const R d0 = eps4 + (R(13) * t0 * t0 + R(3) * t1 * t1);
    const R d1 = eps4 + (R(13) * t2 * t2 + R(3) * t3 * t3);
    const R d2 = eps4 + (R(13) * t4 * t4 + R(3) * t5 * t5);
    if constexpr (std::is_same<R, double>::value) {
        const R e0 = d0 * d0, e1 = d1 * d1, e2 = d2 * d2;
        w0 = e1 * e2;                       // numerators; the caller divides by D
        w2 = R(3) * (e0 * e1);
        return w0 + R(6) * (e0 * e2) + w2;  // D
    } else {
        const R a0 = Math<R>::rcp(d0 * d0);
        const R a1 = R(6) * Math<R>::rcp(d1 * d1);
        const R a2 = R(3) * Math<R>::rcp(d2 * d2);
        const R is = Math<R>::rcp(a0 + a1 + a2);
        w0 = a0 * is;
        w2 = a2 * is;
        return R(1);
    }
}

template <typename R, bool DEV = false>
__device__ __forceinline__ R weno_flux_d(const R* dF, const R* dq, R amx, R* dev = nullptr) {
    const R ap = dF[0] + amx * dq[0], bp = dF[1] + amx * dq[1], cp = dF[2] + amx * dq[2], dp = dF[3] + amx * dq[3];
    const R am = dF[4] - amx * dq[4], bm = dF[3] - amx * dq[3], cm = dF[2] - amx * dq[2], dm = dF[1] - amx * dq[1];
    R w0p, w2p, w0m, w2m;
    const R Dp = weno_half_w(ap, bp, cp, dp, w0p, w2p);
    const R Dm = weno_half_w(am, bm, cm, dm, w0m, w2m);
    if constexpr (std::is_same<R, double>::value) {
        double ip, im;
        const double DD = Dp * Dm;
        if (DD < 1.0e300) { const double r = 1.0 / DD; ip = Dm * r; im = Dp * r; }
        else { ip = 1.0 / Dp; im = 1.0 / Dm; }
        w0p *= ip; w2p *= ip; w0m *= im; w2m *= im;
    }
    if constexpr (DEV) {
        // largest departure of the nonlinear weights from the linear (0.1, 0.6, 0.3)
        const R w1p = R(1) - w0p - w2p, w1m = R(1) - w0m - w2m;
        R d = fabs(w0p - R(0.1));
        d = fmax(d, fabs(w1p - R(0.6))); d = fmax(d, fabs(w2p - R(0.3)));
        d = fmax(d, fabs(w0m - R(0.1))); d = fmax(d, fabs(w1m - R(0.6))); d = fmax(d, fabs(w2m - R(0.3)));
        *dev = d;
    }
    const R first = (dF[1] + R(6) * dF[2] - dF[3]) * R(1.0 / 12.0);
    const R second = w0p * (ap - R(2) * bp + cp) * R(1.0 / 6.0) + (w2p - R(0.5)) * (bp - R(2) * cp + dp) * R(1.0 / 12.0);
    const R third = w0m * (am - R(2) * bm + cm) * R(1.0 / 6.0) + (w2m - R(0.5)) * (bm - R(2) * cm + dm) * R(1.0 / 12.0);
    return first - second + third;
}

// Component-wise fifth-order upwind flux with the linear weights
// (0.1, 0.6, 0.3) and the stencil's largest |lambda| as Lax-Friedrichs speed:
// the cheap flux a router sends smooth interfaces to.  dF_k, dq_k are the physical cell
// differences of one component over the stencil; returns the correction to
// the central F_i (same form as weno_flux_d, no characteristic projection).
template <typename R>
__device__ __forceinline__ R linear_flux_d(const R* dF, const R* dq, R amx) {
    const R ap = dF[0] + amx * dq[0], bp = dF[1] + amx * dq[1], cp = dF[2] + amx * dq[2], dp = dF[3] + amx * dq[3];
    const R am = dF[4] - amx * dq[4], bm = dF[3] - amx * dq[3], cm = dF[2] - amx * dq[2], dm = dF[1] - amx * dq[1];
    const R first = (dF[1] + R(6) * dF[2] - dF[3]) * R(1.0 / 12.0);
    const R second = R(0.1) * (ap - R(2) * bp + cp) * R(1.0 / 6.0) + R(-0.2) * (bp - R(2) * cp + dp) * R(1.0 / 12.0);
    const R third = R(0.1) * (am - R(2) * bm + cm) * R(1.0 / 6.0) + R(-0.2) * (bm - R(2) * cm + dm) * R(1.0 / 12.0);
    return first - second + third;
}

__device__ __forceinline__ constexpr int perm_of(int dir, int v) {
    // line variable v -> conserved index (x: identity; y: rho,My,Mz,Mx,By,Bz,Bx,E;
    // z: rho,Mz,Mx,My,Bz,Bx,By,E)
    return dir == 0 ? v
         : dir == 1 ? (v == 1 ? 2 : v == 2 ? 3 : v == 3 ? 1 : v == 4 ? 5 : v == 5 ? 6 : v == 6 ? 4 : v)
                    : (v == 1 ? 3 : v == 2 ? 1 : v == 3 ? 2 : v == 4 ? 6 : v == 5 ? 4 : v == 6 ? 5 : v);
}

constexpr uint32_t kWaitLimit = 1u << 26;   // bounded TMA wait (~seconds), then flag and skip

// MODE 0: plain method.  1: learned routing (network + guard).  2: guard-only
// routing (the ablation).  3: plain method that also records features and
// nonlinear-weight labels of sampled tiles for training.
//
// ENS: one launch advances this sweep for every member of a batched
// ensemble; the global tile index runs over the members' tiles in order, and
// each tile reads its member's arguments from the ensemble table.
template <int DIR, int NL, int T, int NT, typename R, int MINB, int MODE, bool ENS = false>
__global__ void __launch_bounds__(NT, MINB) k_sweep(const __grid_constant__ SweepArgs a0) {
    static_assert(!ENS || MODE == 0, "ensembles run the plain method");
    constexpr bool ROUTED = MODE == 1 || MODE == 2;
    using TL = Tile<DIR, NL, T, R>;
    using V2 = typename Math<R>::V2;
    constexpr int C = TL::C, F = TL::F, NP = TL::NP, NLC = TL::NLC, NLF = TL::NLF, NI = TL::NI;
    constexpr int TO = TL::TO;
    constexpr int NBUF = TL::NBUF, NOB = TL::NOB;
    constexpr int FE = F + 2;                                  // fetched decisions per line (MODE 1)
    constexpr int DWS = align_up(4 * NL * FE, 16) / 4;         // ints per decision set
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations need 128-byte alignment: align the carve-up base
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    double* sFc = reinterpret_cast<double*>(sm + TL::bFc);
    double* sP = reinterpret_cast<double*>(sm + TL::bP);
    R* sA = reinterpret_cast<R*>(sm + TL::bA);
    R* sD = reinterpret_cast<R*>(sm + TL::bD);
    double* sUst = reinterpret_cast<double*>(sm + TL::bU);   // U staging (P1 -> P1b), FP64
    R* sFs = reinterpret_cast<R*>(sm + TL::bU);                        // [7][NI], P3 -> P4
    double* sdF = reinterpret_cast<double*>(sm + TL::bU + TL::offdF);   // [7][NI], P4 -> P5
    R* sS = reinterpret_cast<R*>(sm + TL::bS);                         // [NS][NI], P2a -> P3, P4
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + TL::bB);
    constexpr bool LM = MODE == 1;   // the learned mode's compact layout
    int* sDec = reinterpret_cast<int*>(sm + (LM ? TL::lDec : TL::bDec));       // 1: full WENO, 0: linear flux
    int* sList = reinterpret_cast<int*>(sm + (LM ? TL::lList : TL::bList));    // full-WENO interfaces
    float* sDev = reinterpret_cast<float*>(sm + TL::bDev);      // weight deviation (collect)
    float* sFlx = reinterpret_cast<float*>(sm + TL::bFlx);      // flux departure (collect)
    float* sFt = reinterpret_cast<float*>(sm + TL::bFt);        // features (collect)
    R* sAmx = reinterpret_cast<R*>(sm + (LM ? TL::lAmx : TL::bAmx));           // per interface: max |lambda_0|, |lambda_6|
    float* sCF = reinterpret_cast<float*>(sm + (LM ? TL::lCF : TL::bCF));      // per cell: rho, p, |B|, |v|, c_f
    int* sDecW = reinterpret_cast<int*>(sm + (LM ? TL::lDecW : TL::bDecW));    // MODE 1: fetched decisions
    __shared__ int s_nfull;
    __shared__ unsigned int s_cnt[2];   // full, cheap interfaces

    // Tiles: T active cells along the sweep x NL lines x one plane.  Lines of
    // the x sweep start at j = 3; lines of the y/z sweeps are consecutive i and
    // start at the even i = 2 (a masked ghost line) so the innermost TMA
    // coordinate stays 16-byte aligned.
    struct Geo { int n, nt1, ntx, nty; long long sstride; };
    auto geo_of = [](const Grid& g) -> Geo {
        Geo o;
        o.n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
        o.nt1 = DIR == 0 ? g.ny : g.nx;
        o.sstride = DIR == 0 ? 1ll : DIR == 1 ? (long long)g.pitch : (long long)g.pitch * g.P1;
        o.ntx = (o.n + T - 1) / T;
        o.nty = DIR == 0 ? (o.nt1 + NL - 1) / NL : (o.nt1 + 1 + NL - 1) / NL;
        return o;
    };
    const int line0 = DIR == 0 ? 3 : 2;
    // global tile -> member (ENS) and the member's arguments + local tile
    auto member_of = [&](long long tile) -> int {
        int lo = 0, hi = a0.ens_n - 1;   // last member whose first tile is <= tile
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a0.ens_tile_start[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        return lo;
    };
    // (a __grid_constant__ parameter may be addressed: it is not copied)
    auto args_of = [&](long long tile, long long& lt) -> const SweepArgs* {
        if constexpr (ENS) {
            const int m = member_of(tile);
            lt = tile - a0.ens_tile_start[m];
            return a0.ens_tab + ((long long)m * a0.ens_stride + a0.ens_off + a0.ens_par[m]);
        } else {
            lt = tile;
            return &a0;
        }
    };
    // tile index -> (tile along the sweep, first line, plane); a single domain
    // has fewer than 2^31 tiles, so 32-bit divisions serve
    auto tile_coords = [](long long t, int ntx, int nty, int& tx, int& ty, int& tz) {
        if constexpr (ENS) {
            tx = (int)(t % ntx);
            const long long r = t / ntx;
            ty = (int)(r % nty);
            tz = (int)(r / nty);
        } else {
            const unsigned u = (unsigned)t, r = u / (unsigned)ntx;
            tx = (int)(u - r * (unsigned)ntx);
            const unsigned z = r / (unsigned)nty;
            ty = (int)(r - z * (unsigned)nty);
            tz = (int)z;
        }
    };
    long long ntiles;
    if constexpr (ENS) {
        ntiles = a0.ens_tile_start[a0.ens_n];
    } else {
        const Geo G = geo_of(a0.g);
        const int nt2 = DIR == 2 ? a0.g.ny : a0.g.nz;
        ntiles = (long long)G.ntx * G.nty * nt2;
    }
    // the first tile at or after t (stepping by the grid) of a member that is
    // stepping; members that reached their end time are skipped whole
    auto advance = [&](long long t) -> long long {
        if constexpr (ENS) {
            while (t < ntiles) {
                const int m = member_of(t);
                if (a0.ens_active[m]) return t;
                const long long end = a0.ens_tile_start[m + 1];
                t += (end - t + gridDim.x - 1) / gridDim.x * gridDim.x;
            }
        }
        return t;
    };
    const int tid = threadIdx.x;
    // the compute threads' tile waits (a failure-detection test can make them
    // give up at once); the drain in bail() below always keeps kWaitLimit
    const uint32_t wait_limit = a0.wait_expire ? 0u : kWaitLimit;
    // the thread that issues and tracks the tile copies: the block's last,
    // whose warp has the least P1 work, so issuing does not delay P1
    const bool issuer = tid == NT - 1;

    if (issuer) {
        for (int k = 0; k < NBUF + NOB; ++k) mbar_init(&bars[k], 1);
        fence_barrier_init();
    }
    __syncthreads();

    // TMA loads (the issuer only): the raw tile of `tile` into raw buffer b
    // (which == 0) or its update operand into operand buffer b (which == 1).
    auto issue = [&](long long gtile, int which, int b) -> bool {
        long long tile;
        const SweepArgs& a = *args_of(gtile, tile);
        const Geo G = geo_of(a.g);
        const int ntx = G.ntx, nty = G.nty;
        int tx, ty, tz;
        tile_coords(tile, ntx, nty, tx, ty, tz);
        const int c0 = tx * T, t1_0 = line0 + ty * NL, t2 = 3 + tz;
        int cc[4];
        if (which == 0) {
            if (DIR == 0) { cc[0] = c0; cc[1] = t1_0; cc[2] = t2; }
            else if (DIR == 1) { cc[0] = t1_0; cc[1] = c0; cc[2] = t2; }
            else { cc[0] = t1_0; cc[1] = t2; cc[2] = c0; }
        } else {
            if (DIR == 0) { cc[0] = c0 + 2; cc[1] = t1_0; cc[2] = t2; }
            else if (DIR == 1) { cc[0] = t1_0; cc[1] = c0 + 3; cc[2] = t2; }
            else { cc[0] = t1_0; cc[1] = t2; cc[2] = c0 + 3; }
        }
        cc[3] = 0;
        if (cc[0] & 1) {   // never issue a misaligned tensor copy
            atomicOr(a.status, HOW_STATUS_TMA_ALIGN);
            return false;
        }
        fence_proxy_async_smem();
        if (which == 0) {
            mbar_arrive_expect_tx(&bars[b], TL::in_bytes);
            tma_load_4d(sm + TL::bQ + b * align_up(8 * TL::NQ, 128), &a.tm_in, &bars[b], cc[0], cc[1], cc[2], cc[3]);
        } else {
            mbar_arrive_expect_tx(&bars[NBUF + b], TL::out_bytes);
            tma_load_4d(sm + TL::bO + b * align_up(8 * TL::NO, 128), &a.tm_out, &bars[NBUF + b], cc[0], cc[1], cc[2],
                        cc[3]);
        }
        return true;
    };
    // MODE 1: the routing pass's decisions for tile t's faces and one more on
    // each side of every line (faces -1 .. F), fetched by asynchronous 4-byte
    // copies of the aligned words that hold them into decision set `slot`,
    // one tile ahead so their latency hides behind a whole tile.  Every
    // thread commits one group per call (empty past the last tile); returns
    // the byte of this thread's word, -1 for no face.
    auto fetch_dec = [&](long long t, int slot) -> int {
        int shift = -1;
        if constexpr (MODE == 1) {
            static_assert(NL * FE <= NT, "one fetched decision per thread");
            if (tid < NL * FE && t < ntiles) {
                const Geo G = geo_of(a0.g);
                int tx, ty, tz;
                tile_coords(t, G.ntx, G.nty, tx, ty, tz);
                const int l = tid / FE, f = tid % FE - 1;
                const int t1 = line0 + ty * NL + l, iface = tx * T + f;
                if (t1 >= 3 && t1 <= G.nt1 + 2 && iface >= 0 && iface <= G.n) {
                    const unsigned char* src = a0.route_next + route_line(a0.g, DIR, t1, 3 + tz) + (iface + 2);
                    shift = (int)(reinterpret_cast<uintptr_t>(src) & 3u);
                    cp_async4(&sDecW[slot * DWS + tid],
                              reinterpret_cast<const void*>(reinterpret_cast<uintptr_t>(src) & ~uintptr_t(3)));
                }
            }
            cp_async_commit();
        }
        return shift;
    };

    // a single domain's dt / d is one value for the whole launch
    const double dtdl_launch = ENS ? 0.0 : *a0.dtdl;
    long long tile = advance(blockIdx.x);
    int buf = 0;               // raw buffer of this tile
    int ob = 0;                // update operand buffer and decision set of this tile
    uint32_t par_bits = 0u;    // phase parity per barrier (bit k)
    uint32_t pend_bits = 0u;   // copies in flight per barrier (the issuer's view, bit k)
    bool issued_ok = true;
    if (issuer && tile < ntiles) {
        // this tile's raw tile and update operand, and the raw tiles of the
        // next NBUF - 1 tiles of this block
        issued_ok = issue(tile, 0, 0) && issue(tile, 1, 0);
        pend_bits = issued_ok ? (1u | (1u << NBUF)) : 0u;
        long long ahead = advance(tile + gridDim.x);
        for (int k = 1; k < NBUF - 1 && ahead < ntiles; ++k) {
            issued_ok = issue(ahead, 0, k) && issued_ok;
            pend_bits |= 1u << k;
            ahead = advance(ahead + gridDim.x);
        }
    }
    int dec_cur = fetch_dec(tile, 0);   // this tile's decision words (MODE 1)
    // On a failed wait the whole block leaves together; the issuer first waits
    // (bounded) for the copies it still has in flight.
    auto bail = [&]() {
        if (issuer) {
            atomicOr(a0.status, HOW_STATUS_TMA_TIMEOUT);
            for (int k = 0; k < NBUF + NOB; ++k)
                if ((pend_bits >> k) & 1u) mbar_wait_bounded(&bars[k], (par_bits >> k) & 1u, kWaitLimit);
        }
    };
    // optional per-phase cycle accounting of thread 0 (prof != nullptr)
    long long tprev = clock64();
    auto mark = [&](int ph) {
        if (a0.prof != nullptr && tid == 0) {
            const long long now = clock64();
            atomicAdd(a0.prof + ph, (unsigned long long)(now - tprev));
            if (ph == 10) atomicAdd(a0.prof + 11, 1ull);   // tiles
            tprev = now;
        }
    };
    for (; tile < ntiles; tile = advance(tile + gridDim.x)) {
        long long ltile;
        const SweepArgs& a = *args_of(tile, ltile);
        const Grid& g = a.g;
        const Geo G = geo_of(g);
        const int n = G.n, nt1 = G.nt1, ntx = G.ntx, nty = G.nty;
        const long long sstride = G.sstride;
        const double gam = a.gam;
        const R gamR = R(a.gam);
        const R gam0 = R(1) - gamR, gam1 = R(0.5) * (gamR - R(1));
        const R gam2 = (gamR - R(2)) / (gamR - R(1));
        int tx, ty, tz;
        tile_coords(ltile, ntx, nty, tx, ty, tz);
        const int c0 = tx * T;                       // padded index of tile cell 0
        const int t1_0 = line0 + ty * NL;
        const int t2 = 3 + tz;
        auto line_off = [&](int l) -> long long {
            const int t1 = t1_0 + l;
            if (DIR == 0) return g.idx(0, t1, t2);
            if (DIR == 1) return g.idx(t1, 0, t2);
            return g.idx(t1, t2, 0);
        };
        auto line_ok = [&](int l) -> bool { return t1_0 + l >= 3 && t1_0 + l <= nt1 + 2; };
        // the line's first byte in the router's per-face arrays (route_line)
        auto rline = [&](int l) -> long long { return route_line(g, DIR, t1_0 + l, t2); };
        const double* sQ = reinterpret_cast<const double*>(sm + TL::bQ + buf * align_up(8 * TL::NQ, 128));
        const double* sO = reinterpret_cast<const double*>(sm + TL::bO + ob * align_up(8 * TL::NO, 128));
        // raw conserved of line variable v at (line l, tile cell c); box order
        // x: [var][line][cell], y/z: [var][cell][line]
        auto qraw = [&](int v, int l, int c) -> double {
            const int gv = perm_of(DIR, v);
            return DIR == 0 ? sQ[(gv * NL + l) * C + c] : sQ[(gv * C + c) * NL + l];
        };
        auto oraw = [&](int gv, int l, int ct) -> double {
            return DIR == 0 ? sO[(gv * NL + l) * TO + ct + 1] : sO[(gv * TO + ct) * NL + l];
        };

        // ------------------------------------------------------------ P0
        {
            const bool ok = issued_ok && mbar_wait_bounded(&bars[buf], (par_bits >> buf) & 1u, wait_limit);
            if (__syncthreads_or(!ok)) { bail(); return; }   // results void; host sees the status
        }
        par_bits ^= 1u << buf;
        pend_bits &= ~(1u << buf);
        const long long next = advance(tile + gridDim.x);
        {
            // the raw tile NBUF - 1 tiles ahead, into the buffer the previous
            // tile used, and the next tile's update operand into the operand
            // buffer the previous tile used (every read of both ended with
            // that tile's last barrier)
            long long ahead = next;
            for (int k = 2; k < NBUF; ++k) ahead = advance(ahead + gridDim.x);
            const int nb = (buf + NBUF - 1) % NBUF;
            if (issuer && ahead < ntiles) {
                issued_ok = issue(ahead, 0, nb) && issued_ok;
                pend_bits |= 1u << nb;
            }
            if (issuer && next < ntiles) {
                issued_ok = issue(next, 1, ob ^ 1) && issued_ok;
                pend_bits |= 1u << (NBUF + (ob ^ 1));
            }
        }
        const int dec_next = fetch_dec(next, ob ^ 1);   // the next tile's decisions (MODE 1)
        // this stage's dt / d (per member in an ensemble), used in P5
        const double dtdl_tile = ENS ? *a.dtdl : dtdl_launch;
        mark(0);

        // P2a: eigen-system scalars of interface t from the arithmetic mean of
        // its two cells' primitives (src/ssprk.cpp:610-660)
        auto p2a_core = [&](int t, double mrho, double mvx, double mvy, double mvz, double mBx, double mBy,
                            double mBz, double mHH) {
            const R rho = R(mrho), vx = R(mvx), vy = R(mvy), vz = R(mvz);
            const R Bx = R(mBx), By = R(mBy), Bz = R(mBz), HH = R(mHH);
            const R vv2 = vx * vx + vy * vy + vz * vz;
            const R BB2 = Bx * Bx + By * By + Bz * Bz;
            const R isqr = Math<R>::rsq(rho);
            const R irho = isqr * isqr;
            const R bbn2 = BB2 * irho;
            const R bnx2 = Bx * Bx * irho;
            const R cs2 = (gamR - R(1)) * (HH - R(0.5) * (vv2 + bbn2));
            const R cs = Math<R>::sq(fmax(R(0), cs2));
            const R root = Math<R>::sq(fmax(R(0), (bbn2 + cs2) * (bbn2 + cs2) - R(4) * bnx2 * cs2));
            const R lf = Math<R>::sq(fmax(R(0), R(0.5) * (bbn2 + cs2 + root)));
            const R la = fabs(Bx) * isqr;
            const R ls = Math<R>::sq(fmax(R(0), R(0.5) * (bbn2 + cs2 - root)));
            const R Bt2 = By * By + Bz * Bz;
            R bty, btz;
            if (Bt2 >= R(1.0e-30)) { const R ib = Math<R>::rsq(Bt2); bty = By * ib; btz = Bz * ib; }
            else { bty = R(0.70710678118654752440); btz = R(0.70710678118654752440); }
            R af, as;
            const R df = lf * lf - ls * ls;
            if (df >= R(1.0e-30)) {
                const R idf = Math<R>::rsq(df);
                af = Math<R>::sq(fmax(R(0), cs2 - ls * ls)) * idf;
                as = Math<R>::sq(fmax(R(0), lf * lf - cs2)) * idf;
            } else { af = R(1); as = R(1); }
            R* S = sS + t;
            S[S_VX * NI] = vx; S[S_VY * NI] = vy; S[S_VZ * NI] = vz;
            S[S_BY * NI] = By; S[S_BZ * NI] = Bz; S[S_VV2 * NI] = vv2;
            S[S_CS * NI] = cs; S[S_CS2 * NI] = cs2; S[S_LF * NI] = lf; S[S_LS * NI] = ls;
            S[S_AF * NI] = af; S[S_AS * NI] = as; S[S_BTY * NI] = bty; S[S_BTZ * NI] = btz;
            S[S_SGNBX * NI] = sign1(Bx);
            S[S_SQR * NI] = rho * isqr; S[S_ISQR * NI] = isqr;
            S[S_SGNBT * NI] = (By != R(0)) ? sign1(By) : sign1(Bz);
            S[S_FLIP * NI] = (cs >= la) ? R(1) : R(0);
            S[S_BTV * NI] = bty * vy + btz * vz;
            S[S_ICS2 * NI] = Math<R>::rcp(cs2);
        };
        // entry k of the interface list (every interface in the plain method),
        // from the primitives P1 stored
        auto p2a_item = [&](int k) {
            const int t = ROUTED ? sList[k] : k;
            const int c = (t / F) * C + t % F + 2;
            p2a_core(t, 0.5 * (sP[0 * NLC + c] + sP[0 * NLC + c + 1]), 0.5 * (sP[1 * NLC + c] + sP[1 * NLC + c + 1]),
                     0.5 * (sP[2 * NLC + c] + sP[2 * NLC + c + 1]), 0.5 * (sP[3 * NLC + c] + sP[3 * NLC + c + 1]),
                     0.5 * (sP[4 * NLC + c] + sP[4 * NLC + c + 1]), 0.5 * (sP[5 * NLC + c] + sP[5 * NLC + c + 1]),
                     0.5 * (sP[6 * NLC + c] + sP[6 * NLC + c + 1]), 0.5 * (sP[8 * NLC + c] + sP[8 * NLC + c + 1]));
        };

        // ------------------------------------------------------------ P1
        // two threads per cell: the first forms primitives and fluxes, the
        // second the eigenvalues (both from the same primitive arithmetic)
        // primit (src/ssprk.cpp:479-512) of tile cell (l, cc): v from the
        // unfloored density, floors on rho and p with E recomputed
        struct Prim { double rho, irho, vx, vy, vz, Bx, By, Bz, EE, pg, vv2, BB2, Mx, My, Mz; };
        auto primit = [&](int l, int cc) -> Prim {
            Prim o;
            const double DD = qraw(0, l, cc);
            o.Mx = qraw(1, l, cc); o.My = qraw(2, l, cc); o.Mz = qraw(3, l, cc);
            o.Bx = qraw(4, l, cc); o.By = qraw(5, l, cc); o.Bz = qraw(6, l, cc);
            o.EE = qraw(7, l, cc);
            o.rho = DD;
            o.irho = 1.0 / o.rho;
            o.vx = o.Mx * o.irho; o.vy = o.My * o.irho; o.vz = o.Mz * o.irho;
            o.vv2 = o.vx * o.vx + o.vy * o.vy + o.vz * o.vz;
            o.BB2 = o.Bx * o.Bx + o.By * o.By + o.Bz * o.Bz;
            o.pg = (gam - 1.0) * (o.EE - 0.5 * (o.rho * o.vv2 + o.BB2));
            if (o.rho < a.rhomin || o.pg < a.pgmin) {
                o.rho = fmax(a.rhomin, o.rho);
                o.pg = fmax(a.pgmin, o.pg);
                o.EE = o.pg / (gam - 1.0) + 0.5 * (o.rho * o.vv2 + o.BB2);
                o.irho = 1.0 / o.rho;
            }
            return o;
        };
        for (int tt = tid; tt < 2 * NLC; tt += blockDim.x) {
            const bool eig = tt >= NLC;
            const int t = eig ? tt - NLC : tt;
            const int l = t / C, cc = t % C;
            const Prim u = primit(l, cc);
            const double rho = u.rho, irho = u.irho, vx = u.vx, vy = u.vy, vz = u.vz;
            const double Bx = u.Bx, By = u.By, Bz = u.Bz, EE = u.EE, pg = u.pg, vv2 = u.vv2, BB2 = u.BB2;
            const double Mx = u.Mx, My = u.My, Mz = u.Mz;
            if (!eig) {
                const double HH = (EE + pg) * irho;
                sP[0 * NLC + t] = rho; sP[1 * NLC + t] = vx; sP[2 * NLC + t] = vy; sP[3 * NLC + t] = vz;
                sP[4 * NLC + t] = Bx; sP[5 * NLC + t] = By; sP[6 * NLC + t] = Bz; sP[7 * NLC + t] = pg;
                sP[8 * NLC + t] = HH;
                // eigenst centre fluxes (src/ssprk.cpp:561-593), with DD, EE the floored values
                const double pt = pg + 0.5 * BB2;
                const double vdB = vx * Bx + vy * By + vz * Bz;
                double* U = sUst + t * 14;
                double* Fc = sFc + t * 7;
                Fc[0] = U[0] = rho * vx;                 // DD (floored) * vx
                Fc[1] = U[1] = Mx * vx + pt - Bx * Bx;
                Fc[2] = U[2] = My * vx - Bx * By;
                Fc[3] = U[3] = Mz * vx - Bx * Bz;
                Fc[4] = U[4] = By * vx - Bx * vy;
                Fc[5] = U[5] = Bz * vx - Bx * vz;
                Fc[6] = U[6] = (EE + pt) * vx - Bx * vdB;
                U[7] = rho; U[8] = Mx; U[9] = My; U[10] = Mz; U[11] = By; U[12] = Bz; U[13] = EE;
            } else {
                // eigenvalues (src/ssprk.cpp:561-593), in the working type R:
                // FP64 for the plain method, FP32 in the mixed one (where they
                // feed only the FP32 characteristic part)
                const R irR = R(irho);
                const R bbn2 = R(BB2) * irR;
                const R bnx2 = R(Bx * Bx) * irR;
                const R cs2 = fmax(R(0), gamR * fabs(R(pg) * irR));
                const R root = Math<R>::sq(fmax(R(0), (bbn2 + cs2) * (bbn2 + cs2) - R(4) * bnx2 * cs2));
                const R lf = Math<R>::sq(fmax(R(0), R(0.5) * (bbn2 + cs2 + root)));
                if constexpr (MODE != 0) {
                    // the routing features' cell values, once per cell (the
                    // guard of MODE 1 needs density and pressure only)
                    sCF[0 * NLC + t] = (float)rho;
                    sCF[1 * NLC + t] = (float)pg;
                    if constexpr (MODE != 1) {
                        sCF[2 * NLC + t] = sqrtf((float)BB2);
                        sCF[3 * NLC + t] = sqrtf((float)vv2);
                        sCF[4 * NLC + t] = (float)lf;
                    }
                }
                const R la = Math<R>::sq(fmax(R(0), bnx2));
                const R ls = Math<R>::sq(fmax(R(0), R(0.5) * (bbn2 + cs2 - root)));
                const R vxR = R(vx);
                // |lambda_m|: every reader takes the magnitude (the LLF speeds)
                sA[0 * NLC + t] = fabs(vxR - lf); sA[1 * NLC + t] = fabs(vxR - la);
                sA[2 * NLC + t] = fabs(vxR - ls); sA[3 * NLC + t] = fabs(vxR);
                sA[4 * NLC + t] = fabs(vxR + ls); sA[5 * NLC + t] = fabs(vxR + la);
                sA[6 * NLC + t] = fabs(vxR + lf);
            }
        }
        __syncthreads();
        mark(1);

        // ------------------------------------------------------------ P1b
        // cell differences of (F, q_proj) along each line, formed in FP64 and
        // stored in the working type; shared by all 7 fields
        for (int t = tid; t < NLC * 14; t += blockDim.x) {
            const int c = (t / 14) % C;
            sD[t] = (c + 1 < C) ? R(sUst[t + 14] - sUst[t]) : R(0);
        }
        if constexpr (MODE != 0) {
            if (tid < 2) s_cnt[tid] = 0u;
            if (tid == 0) s_nfull = 0;
        }
        if constexpr (MODE == 1) {
            // this tile's decision words (fetched one tile ago) have arrived:
            // keep this thread's byte
            cp_async_wait_prior();
            if (tid < NL * FE) {
                int* w = sDecW + ob * DWS + tid;
                *w = dec_cur < 0 ? 0 : (int)((((unsigned int)*w) >> (8 * dec_cur)) & 0xffu);
            }
        }
        __syncthreads();
        mark(2);

        // ------------------------------------------------------------ PR
        // routing: features of every interface, the hard guard, the network
        // (MODE 1), and the compacted list of interfaces that get full WENO
        int nfull = NLF;
        if constexpr (MODE != 0) {
            // features of interface t (tile-local), its guard and its flatness
            auto row_features = [&](int t, float* ft, bool& flat, float& prior) -> bool {
                const int l = t / F, f = t % F;
                StencilCell sc[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const int cc = l * C + f + k;
                    sc[k] = StencilCell{sCF[0 * NLC + cc], sCF[1 * NLC + cc], sCF[2 * NLC + cc], sCF[3 * NLC + cc],
                                        sCF[4 * NLC + cc]};
                }
                // the prior-stage feature is held at 0: fed back from the
                // network's own decisions it locked smooth flows at full WENO
                prior = 0.0f;
                return router_features(sc, prior, (float)a.rhomin, (float)a.pgmin, a.guard_jump, a.guard_floor, ft,
                                       &flat);
            };
            // Lax-Friedrichs speed of the linear flux: the stencil's largest |lambda|
            auto row_amx = [&](int t) {
                const int cb = (t / F) * C + t % F;
                R amx = fmax(sA[0 * NLC + cb], sA[6 * NLC + cb]);
#pragma unroll
                for (int k = 1; k < 6; ++k) amx = fmax(amx, fmax(sA[0 * NLC + cb + k], sA[6 * NLC + cb + k]));
                sAmx[t] = amx;
            };
            if constexpr (MODE == 1) {
                // decisions of the learned router, formed for the whole sweep by
                // the routing pass (route_prepass.cu) before this launch
                // a face takes full WENO when the pass flagged it or a neighbour
                // along the sweep (decisions formed once per step stay valid
                // while a feature moves by up to one cell)
                bool owned = false, full = false;
                if (tid < NLF) {
                    const int l = tid / F, f = tid % F;
                    const int* d = sDecW + ob * DWS + l * FE + f;   // faces f-1, f, f+1
                    // the hard guard on this stage's state, whatever the stage
                    // the network's decisions were formed at
                    const bool guard = router_guard_rp(sCF + l * C + f, sCF + NLC + l * C + f, (float)a.rhomin,
                                                       (float)a.pgmin, a.guard_jump, a.guard_floor);
                    full = guard || (d[0] | d[1] | d[2]);
                    sDec[tid] = full ? 1 : 0;
                    // list of full-WENO interfaces: P2a-P4 treat each entry on
                    // its own, so the order the atomic gives does not matter
                    if (full) sList[atomicAdd(&s_nfull, 1)] = tid;
                    row_amx(tid);
                    // counted once per face: a tile's last face is the next
                    // tile's first, owned by the lower tile unless it ends the line
                    const int iface = c0 + f;
                    owned = line_ok(l) && iface <= n && (f < T || iface == n);
                }
                const unsigned int mf = __ballot_sync(0xffffffffu, owned && full);
                const unsigned int mc = __ballot_sync(0xffffffffu, owned && !full);
                if ((tid & 31) == 0) {
                    if (mf) atomicAdd(&s_cnt[0], (unsigned int)__popc(mf));
                    if (mc) atomicAdd(&s_cnt[1], (unsigned int)__popc(mc));
                }
                __syncthreads();
                mark(3);
                mark(4);
            } else {
                for (int t = tid; t < NLF; t += blockDim.x) {
                    float ft[kRouterNF];
                    bool flat;
                    float prior;
                    const bool guard = row_features(t, ft, flat, prior);
                    row_amx(t);
                    if constexpr (MODE == 3) {
#pragma unroll
                        for (int k = 0; k < kRouterNF; ++k) sFt[t * 6 + k] = ft[k];
                        sDev[t] = 0.0f;
                        sFlx[t] = 0.0f;
                    }
                    sDec[t] = MODE == 3 ? 1 : (guard ? 1 : 0);
                    if constexpr (MODE == 2) {
                        if (guard) sList[atomicAdd(&s_nfull, 1)] = t;
                    }
                }
                __syncthreads();
                mark(3);
            }
            if constexpr (ROUTED) nfull = s_nfull;
        }

        mark(5);

        // A routed tile with no full-WENO interface skips P2a-P3 and their
        // barriers (nfull is the same for the whole block)
        if (!ROUTED || nfull > 0) {
        // ------------------------------------------------------------ P2a
        for (int k = tid; k < nfull; k += blockDim.x) p2a_item(k);
        __syncthreads();
        mark(6);

        // (the left rows and right columns are built where they are used: P3, P4)
        mark(7);

        // ------------------------------------------------------------ P3
        // one interface ii, field m: left row, projection of its 5 cell
        // differences, WENO flux
        auto p3_one = [&](int m, int ii) {
            const int l = ii / F, f = ii % F;
            R L0[7];
            eig_left_row<R, NI>(m, sS + ii, gam0, gam1, L0);
            R dF0[5], dq0[5];
            R amx0 = sA[m * NLC + l * C + f];
#pragma unroll
            for (int cc = 0; cc < 5; ++cc) {
                const int c = f + cc;
                const V2* u = reinterpret_cast<const V2*>(sD + (l * C + c) * 14);
                R pf = R(0), pq = R(0);
#pragma unroll
                for (int h = 0; h < 7; ++h) {
                    // the seven (F, q) pairs of the difference, one 16-byte load each
                    const V2 x = u[h];
                    const int v0 = 2 * h, v1 = 2 * h + 1;   // components of D[14] = (dF[7], dq[7])
                    if (v0 < 7) pf = (v0 == 0) ? L0[0] * x.x : pf + L0[v0] * x.x;
                    else pq = (v0 == 7) ? L0[0] * x.x : pq + L0[v0 - 7] * x.x;
                    if (v1 < 7) pf = pf + L0[v1] * x.y;
                    else pq = (v1 == 7) ? L0[0] * x.y : pq + L0[v1 - 7] * x.y;
                }
                dF0[cc] = pf; dq0[cc] = pq;
                amx0 = fmax(amx0, sA[m * NLC + l * C + c + 1]);
            }
            if constexpr (MODE == 3) {
                R d0;
                sFs[m * NI + ii] = weno_flux_d<R, true>(dF0, dq0, amx0, &d0);
                atomicMax(reinterpret_cast<int*>(&sDev[ii]), __float_as_int((float)d0));
            } else {
                sFs[m * NI + ii] = weno_flux_d<R>(dF0, dq0, amx0);
            }
        };
        // FP64 at five or more blocks per SM: one interface per thread, which
        // holds one left row and one stencil in registers instead of two
        constexpr bool P3_SINGLE = std::is_same<R, double>::value && MINB >= 5;
        if constexpr (!ROUTED && P3_SINGLE) {
            for (int t = tid; t < 7 * NLF; t += blockDim.x) p3_one(t % 7, t / 7);
        } else if constexpr (!ROUTED) {
            for (int t = tid; t < 7 * NL * NP; t += blockDim.x) {
                const int m = t % 7, pr = t / 7;
                const int l = pr / NP, p = pr % NP;
                const int f0 = 2 * p;
                const bool has1 = f0 + 1 < F;
                const int i0 = l * F + f0;
                const int i1 = has1 ? i0 + 1 : i0;
                R L0[7], L1[7];
                eig_left_row<R, NI>(m, sS + i0, gam0, gam1, L0);
                eig_left_row<R, NI>(m, sS + i1, gam0, gam1, L1);
                // interface f0 uses differences at cells f0..f0+4, f0+1 uses f0+1..f0+5
                R dF0[5], dq0[5], dF1[5], dq1[5];
                R amx0 = sA[m * NLC + l * C + f0];
                R amx1 = sA[m * NLC + l * C + (f0 + 1 < C ? f0 + 1 : C - 1)];
#pragma unroll
                for (int cc = 0; cc < 6; ++cc) {
                    int c = f0 + cc;
                    c = c < C - 1 ? c : C - 2;
                    const V2* u = reinterpret_cast<const V2*>(sD + (l * C + c) * 14);
                    R D[14];
#pragma unroll
                    for (int h = 0; h < 7; ++h) { const V2 x = u[h]; D[2 * h] = x.x; D[2 * h + 1] = x.y; }
                    const R av = sA[m * NLC + l * C + (c + 1)];
                    if (cc <= 4) {
                        R pf = L0[0] * D[0], pq = L0[0] * D[7];
#pragma unroll
                        for (int v = 1; v < 7; ++v) { pf += L0[v] * D[v]; pq += L0[v] * D[7 + v]; }
                        dF0[cc] = pf; dq0[cc] = pq;
                        amx0 = fmax(amx0, av);
                    }
                    if (cc >= 1) {
                        R pf = L1[0] * D[0], pq = L1[0] * D[7];
#pragma unroll
                        for (int v = 1; v < 7; ++v) { pf += L1[v] * D[v]; pq += L1[v] * D[7 + v]; }
                        dF1[cc - 1] = pf; dq1[cc - 1] = pq;
                        amx1 = fmax(amx1, av);
                    }
                }
                if constexpr (MODE == 3) {
                    R d0, d1;
                    sFs[m * NI + i0] = weno_flux_d<R, true>(dF0, dq0, amx0, &d0);
                    atomicMax(reinterpret_cast<int*>(&sDev[i0]), __float_as_int((float)d0));
                    if (has1) {
                        sFs[m * NI + i1] = weno_flux_d<R, true>(dF1, dq1, amx1, &d1);
                        atomicMax(reinterpret_cast<int*>(&sDev[i1]), __float_as_int((float)d1));
                    }
                } else {
                    sFs[m * NI + i0] = weno_flux_d<R>(dF0, dq0, amx0);
                    if (has1) sFs[m * NI + i1] = weno_flux_d<R>(dF1, dq1, amx1);
                }
            }
        } else {
            // routed: pairs of entries of the compacted list, each with its own stencil
            const int npair = (nfull + 1) / 2;
            for (int t = tid; t < 7 * npair; t += blockDim.x) {
                const int m = t % 7, p = t / 7;
                const bool has1 = 2 * p + 1 < nfull;
                const int i0 = sList[2 * p];
                const int i1 = has1 ? sList[2 * p + 1] : i0;
                p3_one(m, i0);
                if (has1) p3_one(m, i1);
            }
        }
        __syncthreads();
        }   // P2a-P3
        mark(8);

        // ------------------------------------------------------------ P4
        // per (interface, flux component): full WENO -> F_i + sum_m R(r,m) F^_m
        // (back-projection in m order, src/ssprk.cpp:941-943); routed-linear
        // interfaces -> the component-wise linear flux.  Components 4 and 5
        // also form the CT terms (src/ssprk.cpp:973-993).
        for (int t = tid; t < 7 * NLF; t += blockDim.x) {
            const int r = t / NLF, i = t % NLF;
            const int l = i / F, f = i % F;
            const int c = l * C + f + 2;          // left cell of the interface
            const double F2 = sFc[c * 7 + r];     // physical flux of that cell (central part)
            double dF;
            bool full = true;
            if constexpr (ROUTED) full = sDec[i] != 0;
            if (full) {
                R Rr[7];
                eig_right_row<R, NI>(r, sS + i, gam2, Rr);
                R acc = R(0);
#pragma unroll
                for (int m = 0; m < 7; ++m) acc += Rr[m] * sFs[m * NI + i];
                dF = (double)acc + F2;
                if constexpr (MODE == 3) {
                    // label collection: what routing this face to the cheap
                    // flux would change -- dt/dx |F_full - F_linear| for this
                    // component, relative to the local size of its conserved
                    // variable (density; rho (|v| + c) for momentum; sqrt(rho) c
                    // for the field; the total energy), with
                    // c^2 = (gam p + B^2) / rho at the mean state
                    R dFk[5], dqk[5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        const int cc = l * C + f + k;
                        dFk[k] = sD[cc * 14 + r];
                        dqk[k] = sD[cc * 14 + 7 + r];
                    }
                    const double lin = (double)linear_flux_d<R>(dFk, dqk, sAmx[i]);
                    const double rho = 0.5 * (sP[c] + sP[c + 1]);
                    const double vx = 0.5 * (sP[NLC + c] + sP[NLC + c + 1]);
                    const double vy = 0.5 * (sP[2 * NLC + c] + sP[2 * NLC + c + 1]);
                    const double vz = 0.5 * (sP[3 * NLC + c] + sP[3 * NLC + c + 1]);
                    const double bx = 0.5 * (sP[4 * NLC + c] + sP[4 * NLC + c + 1]);
                    const double by = 0.5 * (sP[5 * NLC + c] + sP[5 * NLC + c + 1]);
                    const double bz = 0.5 * (sP[6 * NLC + c] + sP[6 * NLC + c + 1]);
                    const double pg = 0.5 * (sP[7 * NLC + c] + sP[7 * NLC + c + 1]);
                    const double v2 = vx * vx + vy * vy + vz * vz, b2 = bx * bx + by * by + bz * bz;
                    const double cs = sqrt((gam * pg + b2) / rho);
                    const double scale = r == 0 ? rho
                                       : r < 4 ? rho * (sqrt(v2) + cs)
                                       : r < 6 ? sqrt(rho) * cs
                                       : pg / (gam - 1.0) + 0.5 * rho * v2 + 0.5 * b2;
                    const float dv = (float)(dtdl_tile * fabs((double)acc - lin) / scale);
                    if (dv > 0.0f) atomicMax(reinterpret_cast<int*>(&sFlx[i]), __float_as_int(dv));
                }
            } else {
                R dFk[5], dqk[5];
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    const int cc = l * C + f + k;
                    dFk[k] = sD[cc * 14 + r];
                    dqk[k] = sD[cc * 14 + 7 + r];
                }
                dF = (double)linear_flux_d<R>(dFk, dqk, sAmx[i]) + F2;
            }
            sdF[r * NI + i] = dF;
            const int iface = c0 + f;   // global interface index, face at padded iface + 2
            const bool valid = line_ok(l) && iface <= n;
            if (valid && (r == 4 || r == 5)) {
                // CT terms: mean of B_n v_t over the two cells
                const int vt = r == 4 ? 2 : 3;
                const double x1 = sP[4 * NLC + c] * sP[vt * NLC + c];
                const double x2 = sP[4 * NLC + c + 1] * sP[vt * NLC + c + 1];
                const long long o = line_off(l) + (long long)(iface + 2) * sstride;
                double avg;
                if (a.ct4) {
                    // fourth-order midpoint value (-1, 9, 9, -1) / 16 over cells c-1 .. c+2
                    const double x0 = sP[4 * NLC + c - 1] * sP[vt * NLC + c - 1];
                    const double x3 = sP[4 * NLC + c + 2] * sP[vt * NLC + c + 2];
                    avg = (-x0 + 9.0 * x1 + 9.0 * x2 - x3) / 16.0;
                } else {
                    // the reference's two-point form (-0, 9, 9, -0) / 18
                    avg = div_const(9.0 * x1 + 9.0 * x2, 18.0, 1.0 / 18.0);
                }
                (r == 4 ? a.cta : a.ctb)[o] = dF + avg;
            }
            if constexpr (MODE != 0) {
                // a tile's last interface is also the next tile's first: the
                // lower tile owns it unless it is the line's last face
                if (valid && r == 0 && (f < T || iface == n)) {
                    const long long o = rline(l) + (iface + 2);
                    if constexpr (MODE == 2) {
                        a.route_next[o] = (unsigned char)(full ? 1 : 0);
                        atomicAdd(&s_cnt[full ? 0 : 1], 1u);
                    }
                }
            }
        }
        __syncthreads();
        if constexpr (MODE == 3) {
            // the records of the tile's owned faces, once every component's
            // flux departure is in (sampled tiles: a hash of the tile index,
            // so the sample does not alias with the tile grid)
            const unsigned long long hs = (unsigned long long)tile * 0x9E3779B97F4A7C15ull;
            const bool sampled = (unsigned int)(hs >> 32) % a.collect_every == 0u;
            for (int i = tid; i < NLF; i += blockDim.x) {
                const int l = i / F, f = i % F, iface = c0 + f;
                if (!(line_ok(l) && iface <= n && (f < T || iface == n))) continue;
                a.route_next[rline(l) + (iface + 2)] = 0;
                if (!sampled) continue;
                const unsigned int slot = atomicAdd(a.collect_n, 1u);
                if (slot < a.collect_cap) {
                    float* rec = a.collect + 8ull * slot;
#pragma unroll
                    for (int k = 0; k < 6; ++k) rec[k] = sFt[i * 6 + k];
                    rec[6] = sDev[i];
                    rec[7] = sFlx[i];
                }
            }
        }
        if constexpr (ROUTED) {
            if (tid == 0) {
                atomicAdd(&a.route_count[0], (unsigned long long)s_cnt[0]);
                atomicAdd(&a.route_count[1], (unsigned long long)s_cnt[1]);

            }
        }
        mark(9);

        // ------------------------------------------------------------ P5
        {
            const bool ok = mbar_wait_bounded(&bars[NBUF + ob], (par_bits >> (NBUF + ob)) & 1u, wait_limit);
            if (__syncthreads_or(!ok)) { bail(); return; }
        }
        par_bits ^= 1u << (NBUF + ob);
        pend_bits &= ~(1u << (NBUF + ob));
        const double dtdl = dtdl_tile;
        for (int t = tid; t < 8 * NL * T; t += blockDim.x) {
            int v, l, ct;
            if (DIR == 0) { v = t / (NL * T); const int r = t % (NL * T); l = r / T; ct = r % T; }
            else { v = t / (NL * T); const int r = t % (NL * T); ct = r / NL; l = r % NL; }
            const int s = c0 + ct + 3;
            if (!line_ok(l) || s > n + 2) continue;
            const int rr = v < 4 ? v : v - 1;     // flux row of line variable v (v = 4: normal B)
            const int fi = l * F + ct;
            const double delta = (v == 4) ? 0.0 : -dtdl * (sdF[rr * NI + fi + 1] - sdF[rr * NI + fi]);
            const int gv = perm_of(DIR, v);
            const long long o = (long long)gv * g.fs + line_off(l) + (long long)s * sstride;
            const double cur = oraw(gv, l, ct);   // q(iw) (accumulate) or the RK base
            if (a.mode == 0) {
                if (v != 4) a.qout[o] = cur + delta;
            } else if (a.mode == 1) {
                a.qout[o] = a.k1 * cur + a.k3 * qraw(v, l, ct + 3) + delta;
            } else {
                a.qout[o] = cur + delta;
            }
        }
        __syncthreads();   // every read of the update operand / raw tile is done
        mark(10);
        buf = buf + 1 == NBUF ? 0 : buf + 1;
        ob ^= 1;
        dec_cur = dec_next;
    }   // tile loop
}

}  // namespace
}  // namespace how
