// cell_ops.cuh -- per-cell / per-column bodies of the memory-bound kernels
// (ghost fill, CFL reduction, positivity floor, stage-5 base, constrained
// transport).  The single-domain kernels (state_kernels.cu, ct_kernels.cu)
// and the batched ensemble kernels (ensemble.cu) both call these, so a
// member of an ensemble computes exactly what the same run computes alone.
#pragma once

#include "how_internal.cuh"

namespace how {

// Ghost fill along one axis of one column, in the reference's statement order
// (src/bound.cpp:19-107): periodic A(0)=A(n) A(1)=A(n+1) A(2)=A(n+2)
// A(n+3)=A(3) A(n+4)=A(4) A(n+5)=A(5); open A(0..2)=A(3), A(n+3..5)=A(n+2).
// The same rule fills face B (src/fluxct.cpp:141-205) and the CT arrays
// (src/fluxct.cpp:510-552).  (a, b): the column's transverse indices, a the
// faster one.  Returns false when a is outside the plane.  `sides` (bit 0 the
// low side, bit 1 the high side) says which ghost layers are filled here; a
// part of a decomposed domain fills only its physical sides and receives the
// others from its neighbours (an open side is filled on its own, a periodic
// axis only with both sides here).
template <int AX>
__device__ __forceinline__ void op_bound_column(const Grid& g, double* field, int a, int b, int periodic,
                                                int sides = 3) {
    int n;
    long long stride, base;
    if (AX == 0) { n = g.nx; if (a >= g.P1) return; base = g.idx(0, a, b); stride = 1; }
    else if (AX == 1) { n = g.ny; if (a >= g.P0) return; base = g.idx(a, 0, b); stride = g.pitch; }
    else { n = g.nz; if (a >= g.P0) return; base = g.idx(a, b, 0); stride = (long long)g.pitch * g.P1; }
    double* A = field + base;
    auto at = [&](int s) -> double& { return A[s * stride]; };
    if (sides != 3) {
        // one physical (open) side of a part, or none
        if (sides & 1) { const double lo = at(3); at(0) = lo; at(1) = lo; at(2) = lo; }
        if (sides & 2) { const double hi = at(n + 2); at(n + 3) = hi; at(n + 4) = hi; at(n + 5) = hi; }
        return;
    }
    if (periodic) {
        if (n >= 3) {
            // no source index is a ghost: all six loads go out together
            const double s0 = at(n), s1 = at(n + 1), s2 = at(n + 2), s3 = at(3), s4 = at(4), s5 = at(5);
            at(0) = s0; at(1) = s1; at(2) = s2;
            at(n + 3) = s3; at(n + 4) = s4; at(n + 5) = s5;
        } else {
            at(0) = at(n); at(1) = at(n + 1); at(2) = at(n + 2);
            at(n + 3) = at(3); at(n + 4) = at(4); at(n + 5) = at(5);
        }
    } else {
        const double lo = at(3), hi = at(n + 2);
        at(0) = lo; at(1) = lo; at(2) = lo;
        at(n + 3) = hi; at(n + 4) = hi; at(n + 5) = hi;
    }
}
// The padded index whose value the ghost fill above leaves at padded index s
// of an axis with n >= 2 active cells: the identity on [3, n+2], and an
// active index for every s in [1, n+4].
__host__ __device__ __forceinline__ int bc_map(int s, int n, int periodic) {
    if (s < 3) return periodic ? s + n : 3;
    if (s > n + 2) return periodic ? s - n : n + 2;
    return s;
}

// How the CT bodies below reach a neighbour of an active cell along an axis:
// on = 0, at the plain offset (the array's ghosts were filled); on = 1,
// through bc_map (they were not: the read returns what the fill would have
// put there).  p*: the periodic axes.
struct BCMap { int px, py, pz, on; };

// (stride * 5 fits an int for every grid the device memory holds)
__device__ __forceinline__ int nb_off(const BCMap& m, int s, int d, int n, int periodic, int stride) {
    return m.on ? (bc_map(s + d, n, periodic) - s) * stride : d * stride;
}

// columns of one field: (fast transverse extent, slow transverse extent)
template <int AX>
__host__ __device__ __forceinline__ void bound_plane(const Grid& g, int& ta, int& tb) {
    if (AX == 0) { ta = g.P1; tb = g.P2; }
    else if (AX == 1) { ta = g.P0; tb = g.P2; }
    else { ta = g.P0; tb = g.P1; }
}

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// tstep (src/tstep.cpp:28-83): |v_d| + c_f,d of active cell t (x fastest).
// Returns false when one of the cell's eight conserved values is not finite
// (the maxima ignore such a cell, as fmax does in the reference).
__device__ __forceinline__ bool op_tstep_cell(const Grid& g, const double* __restrict__ q, double gam,
                                              double rhomin, double pgmin, long long t, double& mx, double& my,
                                              double& mz) {
    const int i = 3 + (int)(t % g.nx);
    const long long r = t / g.nx;
    const int j = 3 + (int)(r % g.ny);
    const int k = 3 + (int)(r / g.ny);
    const long long c = g.idx(i, j, k);
    const double DD = q[c], Mx = q[g.fs + c], My = q[2 * g.fs + c], Mz = q[3 * g.fs + c];
    const double Bx = q[4 * g.fs + c], By = q[5 * g.fs + c], Bz = q[6 * g.fs + c];
    const double EE = q[7 * g.fs + c];
    const double rho = fmax(DD, rhomin);
    // the seven quotients by rho, each correctly rounded, from one division
    const double ir = 1.0 / rho;
    const double vx = div_const(Mx, rho, ir), vy = div_const(My, rho, ir), vz = div_const(Mz, rho, ir);
    const double vv2 = vx * vx + vy * vy + vz * vz;
    const double BB2 = Bx * Bx + By * By + Bz * Bz;
    const double pg = fmax(pgmin, (gam - 1.0) * (EE - 0.5 * (rho * vv2 + BB2)));
    const double bbn2 = div_const(BB2, rho, ir);
    const double cs2 = fmax(0.0, div_const(gam * pg, rho, ir));
    const double bnx2 = div_const(Bx * Bx, rho, ir), bny2 = div_const(By * By, rho, ir),
                 bnz2 = div_const(Bz * Bz, rho, ir);
    const double s = (bbn2 + cs2) * (bbn2 + cs2);
    const double rootx = sqrt(fmax(0.0, s - 4.0 * bnx2 * cs2));
    const double rooty = sqrt(fmax(0.0, s - 4.0 * bny2 * cs2));
    const double rootz = sqrt(fmax(0.0, s - 4.0 * bnz2 * cs2));
    const double lfx = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 + rootx)));
    const double lfy = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 + rooty)));
    const double lfz = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 + rootz)));
    mx = fmax(mx, fabs(vx) + lfx);
    my = fmax(my, fabs(vy) + lfy);
    mz = fmax(mz, fabs(vz) + lfz);
    const double big = 1.7976931348623157e308;
    return fabs(DD) <= big && fabs(Mx) <= big && fabs(My) <= big && fabs(Mz) <= big && fabs(Bx) <= big &&
           fabs(By) <= big && fabs(Bz) <= big && fabs(EE) <= big;
}

// Block reduction of the three maxima and one atomicMax per block on the bit
// patterns (non-negative doubles order like their bit patterns).
__device__ __forceinline__ void block_max3_to(double mx, double my, double mz, unsigned long long* bits) {
    mx = warp_max(mx); my = warp_max(my); mz = warp_max(mz);
    __shared__ double red[3][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = mx; red[1][w] = my; red[2][w] = mz; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        mx = l < nw ? red[0][l] : 0.0;
        my = l < nw ? red[1][l] : 0.0;
        mz = l < nw ? red[2][l] : 0.0;
        mx = warp_max(mx); my = warp_max(my); mz = warp_max(mz);
        if (l == 0) {
            atomicMax(&bits[0], (unsigned long long)__double_as_longlong(mx));
            atomicMax(&bits[1], (unsigned long long)__double_as_longlong(my));
            atomicMax(&bits[2], (unsigned long long)__double_as_longlong(mz));
        }
    }
}

__device__ __forceinline__ void fill_dtdl(DevScalars* sc, double dt, double dx, double dy, double dz) {
    // par.dtdx = c.k2 * par.dt / par.dx (src/ssprk.cpp:1302-1304)
    const double k2[6] = {0.0, 0.39175222700392, 0.36841059262959, 0.25189177424738,
                          0.54497475021237, 0.22600748319395};
    for (int iw = 1; iw <= 5; ++iw) {
        sc->dtdl[iw][0] = k2[iw] * dt / dx;
        sc->dtdl[iw][1] = k2[iw] * dt / dy;
        sc->dtdl[iw][2] = k2[iw] * dt / dz;
    }
}

// dt = cour / sum_d(vmax_d / d_d) (src/tstep.cpp:123-135), then the driver's
// clamp to the output time (src/main.cpp:170-172).  Resets the maxima.
__device__ __forceinline__ double op_tstep_finalize(DevScalars* sc, int gnx, int gny, int gnz, double dx,
                                                    double dy, double dz, double cour, double time, double target,
                                                    int clamp) {
    const double vx = __longlong_as_double((long long)sc->vmax_bits[0]);
    const double vy = __longlong_as_double((long long)sc->vmax_bits[1]);
    const double vz = __longlong_as_double((long long)sc->vmax_bits[2]);
    sc->vmax_bits[0] = sc->vmax_bits[1] = sc->vmax_bits[2] = 0ull;
    const double tiny = 1.0e-300;
    double invdt = 0.0;
    if (gnx > 1) invdt += fmax(vx, tiny) / dx;
    if (gny > 1) invdt += fmax(vy, tiny) / dy;
    if (gnz > 1) invdt += fmax(vz, tiny) / dz;
    if (invdt <= 0.0) invdt = fmax(vx, tiny) / dx;
    double dt = cour / invdt;
    sc->dt_raw = dt;
    if (clamp && time + dt > target) dt = target - time;
    sc->dt = dt;
    if (!isfinite(dt)) sc->status |= HOW_STATUS_NONFINITE_DT;
    fill_dtdl(sc, dt, dx, dy, dz);
    return dt;
}

// prot (src/prot.cpp:10-51) of one active cell
__device__ __forceinline__ void op_prot_cell(const Grid& g, double* __restrict__ q, double gam, double rhomin,
                                             double pgmin, int i, int j, int k) {
    const long long c = g.idx(i, j, k);
    double rho = q[c];
    const double Mx = q[g.fs + c], My = q[2 * g.fs + c], Mz = q[3 * g.fs + c];
    const double Bx = q[4 * g.fs + c], By = q[5 * g.fs + c], Bz = q[6 * g.fs + c];
    double E = q[7 * g.fs + c];
    rho = fmax(rho, rhomin);
    const double irho = 1.0 / rho, igm1 = 1.0 / (gam - 1.0);
    const double vx = div_const(Mx, rho, irho), vy = div_const(My, rho, irho), vz = div_const(Mz, rho, irho);
    const double vv2 = vx * vx + vy * vy + vz * vz;
    const double BB2 = Bx * Bx + By * By + Bz * Bz;
    double pg = (gam - 1.0) * (E - 0.5 * (rho * vv2 + BB2));
    pg = fmax(pg, pgmin);
    E = div_const(pg, gam - 1.0, igm1) + 0.5 * (rho * vv2 + BB2);
    q[c] = rho;
    q[7 * g.fs + c] = E;
}

// prepare_stage5 (src/ssprk.cpp:121-140): q5 = q0 + (k4/k1) q2 + (k5/k1) q3
__device__ __forceinline__ void op_stage5_cell(const Grid& g, const double* __restrict__ q0,
                                               const double* __restrict__ q2, const double* __restrict__ q3,
                                               double* __restrict__ q5, double c4, double c5, int i, int j, int k) {
    const long long c = g.idx(i, j, k);
    double r[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const long long o = v * g.fs + c;
        r[v] = q0[o] + c4 * q2[o] + c5 * q3[o];
    }
#pragma unroll
    for (int v = 0; v < 8; ++v) q5[v * g.fs + c] = r[v];
}

// ---------------------------------------------------------------- CT
struct CTFields {
    const double *fsy, *fsz, *gsx, *gsz, *hsx, *hsy;
    double *Ox2, *Oy2, *Oz2, *Ox, *Oy, *Oz;
};

__host__ __device__ __forceinline__ CTFields ct_fields(double* const* ct) {
    return CTFields{ct[0], ct[1], ct[2], ct[3], ct[4], ct[5], ct[6], ct[7], ct[8], ct[9], ct[10], ct[11]};
}

// fluxct_build_O2's 4-point face average (src/fluxct.cpp:809-821)
__device__ __forceinline__ double ct_avg4(double a, double b, double c, double d) {
    return (-a + 9.0 * b + 9.0 * c - d) / 16.0;
}
// fluxct_smooth_O's two 3-point corrections (src/fluxct.cpp:828-840)
__device__ __forceinline__ double ct_smooth(double o, double l1, double r1, double l2, double r2) {
    return o + div_const(l1 - 2.0 * o + r1, 24.0, 1.0 / 24.0) + div_const(l2 - 2.0 * o + r2, 24.0, 1.0 / 24.0);
}

// fluxct_build_O2 (src/fluxct.cpp:809-821)
__device__ __forceinline__ void op_emf2_cell(const Grid& g, const CTFields& f, const BCMap& m, int use_Ox,
                                             int use_Oy, int use_Oz, int i, int j, int k) {
    const long long c = g.idx(i, j, k);
    const long long sj = g.pitch, sk = (long long)g.pitch * g.P1;
    const int xm1 = nb_off(m, i, -1, g.nx, m.px, 1), xp1 = nb_off(m, i, 1, g.nx, m.px, 1),
              xp2 = nb_off(m, i, 2, g.nx, m.px, 1);
    const int ym1 = nb_off(m, j, -1, g.ny, m.py, (int)sj), yp1 = nb_off(m, j, 1, g.ny, m.py, (int)sj),
              yp2 = nb_off(m, j, 2, g.ny, m.py, (int)sj);
    const int zm1 = nb_off(m, k, -1, g.nz, m.pz, (int)sk), zp1 = nb_off(m, k, 1, g.nz, m.pz, (int)sk),
              zp2 = nb_off(m, k, 2, g.nz, m.pz, (int)sk);
    // every load before the first store (the compiler cannot rule out aliasing)
    double ox = 0.0, oy = 0.0, oz = 0.0;
    if (use_Ox)
        ox = ct_avg4(f.gsx[c + xm1], f.gsx[c], f.gsx[c + xp1], f.gsx[c + xp2])
           - ct_avg4(f.fsy[c + ym1], f.fsy[c], f.fsy[c + yp1], f.fsy[c + yp2]);
    if (use_Oy)
        oy = ct_avg4(f.hsy[c + ym1], f.hsy[c], f.hsy[c + yp1], f.hsy[c + yp2])
           - ct_avg4(f.gsz[c + zm1], f.gsz[c], f.gsz[c + zp1], f.gsz[c + zp2]);
    if (use_Oz)
        oz = ct_avg4(f.fsz[c + zm1], f.fsz[c], f.fsz[c + zp1], f.fsz[c + zp2])
           - ct_avg4(f.hsx[c + xm1], f.hsx[c], f.hsx[c + xp1], f.hsx[c + xp2]);
    if (use_Ox) f.Ox2[c] = ox;
    if (use_Oy) f.Oy2[c] = oy;
    if (use_Oz) f.Oz2[c] = oz;
}

// fluxct_smooth_O (src/fluxct.cpp:828-840)
__device__ __forceinline__ void op_emf_cell(const Grid& g, const CTFields& f, int use_Ox, int use_Oy, int use_Oz,
                                            int i, int j, int k) {
    const long long c = g.idx(i, j, k);
    const long long sj = g.pitch, sk = (long long)g.pitch * g.P1;
    double ox = 0.0, oy = 0.0, oz = 0.0;
    if (use_Ox) ox = ct_smooth(f.Ox2[c], f.Ox2[c - 1], f.Ox2[c + 1], f.Ox2[c - sj], f.Ox2[c + sj]);
    if (use_Oy) oy = ct_smooth(f.Oy2[c], f.Oy2[c - sj], f.Oy2[c + sj], f.Oy2[c - sk], f.Oy2[c + sk]);
    if (use_Oz) oz = ct_smooth(f.Oz2[c], f.Oz2[c - 1], f.Oz2[c + 1], f.Oz2[c - sk], f.Oz2[c + sk]);
    if (use_Ox) f.Ox[c] = ox;
    if (use_Oy) f.Oy[c] = oy;
    if (use_Oz) f.Oz[c] = oz;
}

struct BArgs {
    double* bout;                 // stage iw
    const double* bprev;          // stage iw-1
    const double *b0, *b2, *b3;   // RK base stages
    double k1, k3, c4, c5;
    int stage5;
    const double* dtdl;           // dtdx, dtdy, dtdz of this stage
};

__device__ __forceinline__ double bbase(const BArgs& a, long long off) {
    // copy_bfield_stage / prepare_bfield_stage5 (src/fluxct.cpp:111-135)
    if (a.stage5) return a.b0[off] + a.c4 * a.b2[off] + a.c5 * a.b3[off];
    return a.b0[off];
}

// fluxct_update_bfield (src/fluxct.cpp:848-877) of one active cell.
// Components the update does not touch keep the stage's copied/combined base.
__device__ __forceinline__ void op_update_b_cell(const Grid& g, const CTFields& f, const BArgs& a, int use_Ox,
                                                 int use_Oy, int use_Oz, int i, int j, int k) {
    const long long c = g.idx(i, j, k);
    const long long sj = g.pitch, sk = (long long)g.pitch * g.P1;
    const long long xm2 = -2, xm1 = -1, xp1 = 1;
    const long long ym2 = -2 * sj, ym1 = -sj, yp1 = sj;
    const long long zm2 = -2 * sk, zm1 = -sk, zp1 = sk;
    const double aa = 9.0 / 8.0, bb = -1.0 / 24.0;
    const double dtdx = a.dtdl[0], dtdy = a.dtdl[1], dtdz = a.dtdl[2];
    const long long fs = g.fs;
    // the three components are formed before any is stored (the compiler
    // cannot rule out aliasing, so a store would hold back later loads)
    double r[3];
    {
        const long long o = c;
        const double base = bbase(a, o);
        if (use_Ox || use_Oz) {
            double dOx = 0.0, dOz = 0.0;
            if (use_Ox) dOx = aa * (f.Ox[c] - f.Ox[c + ym1]) + bb * (f.Ox[c + yp1] - f.Ox[c + ym2]);
            if (use_Oz) dOz = aa * (f.Oz[c] - f.Oz[c + zm1]) + bb * (f.Oz[c + zp1] - f.Oz[c + zm2]);
            r[0] = a.k1 * base + a.k3 * a.bprev[o] - dtdy * dOx + dtdz * dOz;
        } else {
            r[0] = base;
        }
    }
    {
        const long long o = fs + c;
        const double base = bbase(a, o);
        if (use_Oy || use_Ox) {
            double dOy = 0.0, dOx = 0.0;
            if (use_Oy) dOy = aa * (f.Oy[c] - f.Oy[c + zm1]) + bb * (f.Oy[c + zp1] - f.Oy[c + zm2]);
            if (use_Ox) dOx = aa * (f.Ox[c] - f.Ox[c + xm1]) + bb * (f.Ox[c + xp1] - f.Ox[c + xm2]);
            r[1] = a.k1 * base + a.k3 * a.bprev[o] - dtdz * dOy + dtdx * dOx;
        } else {
            r[1] = base;
        }
    }
    {
        const long long o = 2 * fs + c;
        const double base = bbase(a, o);
        if (use_Oz || use_Oy) {
            double dOz = 0.0, dOy = 0.0;
            if (use_Oz) dOz = aa * (f.Oz[c] - f.Oz[c + xm1]) + bb * (f.Oz[c + xp1] - f.Oz[c + xm2]);
            if (use_Oy) dOy = aa * (f.Oy[c] - f.Oy[c + ym1]) + bb * (f.Oy[c + yp1] - f.Oy[c + ym2]);
            r[2] = a.k1 * base + a.k3 * a.bprev[o] - dtdx * dOz + dtdy * dOy;
        } else {
            r[2] = base;
        }
    }
    a.bout[c] = r[0];
    a.bout[fs + c] = r[1];
    a.bout[2 * fs + c] = r[2];
}

// B(iw) = base (1-D runs, where fluxct returns early, src/fluxct.cpp:793)
__device__ __forceinline__ void op_faceb_base_cell(const Grid& g, const BArgs& a, int i, int j, int k) {
    const long long c = g.idx(i, j, k);
    for (int comp = 0; comp < 3; ++comp) a.bout[comp * g.fs + c] = bbase(a, comp * g.fs + c);
}

// fluxct_interp_b_to_q (src/fluxct.cpp:882-897) fused with prot
// (src/prot.cpp:10-51), which the reference runs right after on the same cells
// inside ssprk; prot_too = false leaves the interpolation alone (the
// standalone fluxct).
__device__ __forceinline__ void op_interp_prot_cell(const Grid& g, const double* __restrict__ b,
                                                    double* __restrict__ q, int use_x, int use_y, int use_z,
                                                    double gam, double rhomin, double pgmin, int i, int j, int k,
                                                    bool prot_too = true) {
    const long long c = g.idx(i, j, k);
    const long long sj = g.pitch, sk = (long long)g.pitch * g.P1, fs = g.fs;
    const double* bx = b;
    const double* by = b + fs;
    const double* bz = b + 2 * fs;
    const double Bx = use_x ? (3.0 * bx[c - 3] - 25.0 * bx[c - 2] + 150.0 * bx[c - 1] + 150.0 * bx[c]
                               - 25.0 * bx[c + 1] + 3.0 * bx[c + 2]) / 256.0 : bx[c];
    const double By = use_y ? (3.0 * by[c - 3 * sj] - 25.0 * by[c - 2 * sj] + 150.0 * by[c - sj] + 150.0 * by[c]
                               - 25.0 * by[c + sj] + 3.0 * by[c + 2 * sj]) / 256.0 : by[c];
    const double Bz = use_z ? (3.0 * bz[c - 3 * sk] - 25.0 * bz[c - 2 * sk] + 150.0 * bz[c - sk] + 150.0 * bz[c]
                               - 25.0 * bz[c + sk] + 3.0 * bz[c + 2 * sk]) / 256.0 : bz[c];
    double rho = q[c];
    const double Mx = q[fs + c], My = q[2 * fs + c], Mz = q[3 * fs + c];
    double E = q[7 * fs + c];
    q[4 * fs + c] = Bx;
    q[5 * fs + c] = By;
    q[6 * fs + c] = Bz;
    if (!prot_too) return;
    rho = fmax(rho, rhomin);
    // the four quotients of prot, each correctly rounded, from two divisions
    const double irho = 1.0 / rho, igm1 = 1.0 / (gam - 1.0);
    const double vx = div_const(Mx, rho, irho), vy = div_const(My, rho, irho), vz = div_const(Mz, rho, irho);
    const double vv2 = vx * vx + vy * vy + vz * vz;
    const double BB2 = Bx * Bx + By * By + Bz * Bz;
    double pg = (gam - 1.0) * (E - 0.5 * (rho * vv2 + BB2));
    pg = fmax(pg, pgmin);
    E = div_const(pg, gam - 1.0, igm1) + 0.5 * (rho * vv2 + BB2);
    q[c] = rho;
    q[7 * fs + c] = E;
}

}  // namespace how
