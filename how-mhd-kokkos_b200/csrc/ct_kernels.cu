// ct_kernels.cu -- 4th-order constrained transport (src/fluxct.cpp:786-899).
//
// The reference builds O2 over [0,n+3], smooths over [1,n+4] and updates face
// B over [1,n+3], each followed by a full ghost fill that overwrites every
// index outside [3, n+2] (src/fluxct.cpp:826, 846, 880).  Only active-index
// results survive those fills, so these kernels compute active cells only and
// then run the same ghost fill.  Face B: bxb(i) is the x-face at i+1/2.
#include "how_internal.cuh"

namespace how {

namespace {

struct CTFields {
    const double *fsy, *fsz, *gsx, *gsz, *hsx, *hsy;
    double *Ox2, *Oy2, *Oz2, *Ox, *Oy, *Oz;
};

// fluxct_build_O2 (src/fluxct.cpp:809-821)
__global__ void k_emf2(Grid g, CTFields f, int use_Ox, int use_Oy, int use_Oz) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;
    if (i > g.nx + 2) return;
    const long long c = g.idx(i, j, k);
    const long long sj = g.pitch, sk = (long long)g.pitch * g.P1;
    if (use_Ox)
        f.Ox2[c] = (-f.gsx[c - 1] + 9.0 * f.gsx[c] + 9.0 * f.gsx[c + 1] - f.gsx[c + 2]) / 16.0
                 - (-f.fsy[c - sj] + 9.0 * f.fsy[c] + 9.0 * f.fsy[c + sj] - f.fsy[c + 2 * sj]) / 16.0;
    if (use_Oy)
        f.Oy2[c] = (-f.hsy[c - sj] + 9.0 * f.hsy[c] + 9.0 * f.hsy[c + sj] - f.hsy[c + 2 * sj]) / 16.0
                 - (-f.gsz[c - sk] + 9.0 * f.gsz[c] + 9.0 * f.gsz[c + sk] - f.gsz[c + 2 * sk]) / 16.0;
    if (use_Oz)
        f.Oz2[c] = (-f.fsz[c - sk] + 9.0 * f.fsz[c] + 9.0 * f.fsz[c + sk] - f.fsz[c + 2 * sk]) / 16.0
                 - (-f.hsx[c - 1] + 9.0 * f.hsx[c] + 9.0 * f.hsx[c + 1] - f.hsx[c + 2]) / 16.0;
}

// fluxct_smooth_O (src/fluxct.cpp:828-840)
__global__ void k_emf(Grid g, CTFields f, int use_Ox, int use_Oy, int use_Oz) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;
    if (i > g.nx + 2) return;
    const long long c = g.idx(i, j, k);
    const long long sj = g.pitch, sk = (long long)g.pitch * g.P1;
    if (use_Ox) {
        const double o = f.Ox2[c];
        f.Ox[c] = o + (f.Ox2[c - 1] - 2.0 * o + f.Ox2[c + 1]) / 24.0
                    + (f.Ox2[c - sj] - 2.0 * o + f.Ox2[c + sj]) / 24.0;
    }
    if (use_Oy) {
        const double o = f.Oy2[c];
        f.Oy[c] = o + (f.Oy2[c - sj] - 2.0 * o + f.Oy2[c + sj]) / 24.0
                    + (f.Oy2[c - sk] - 2.0 * o + f.Oy2[c + sk]) / 24.0;
    }
    if (use_Oz) {
        const double o = f.Oz2[c];
        f.Oz[c] = o + (f.Oz2[c - 1] - 2.0 * o + f.Oz2[c + 1]) / 24.0
                    + (f.Oz2[c - sk] - 2.0 * o + f.Oz2[c + sk]) / 24.0;
    }
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

// fluxct_update_bfield (src/fluxct.cpp:848-877) on active cells.  Components
// the update does not touch keep the stage's copied/combined base value.
__global__ void k_update_b(Grid g, CTFields f, BArgs a, int use_Ox, int use_Oy, int use_Oz) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;
    if (i > g.nx + 2) return;
    const long long c = g.idx(i, j, k);
    const long long sj = g.pitch, sk = (long long)g.pitch * g.P1;
    const double aa = 9.0 / 8.0, bb = -1.0 / 24.0;
    const double dtdx = a.dtdl[0], dtdy = a.dtdl[1], dtdz = a.dtdl[2];
    const long long fs = g.fs;
    {
        const long long o = c;
        const double base = bbase(a, o);
        if (use_Ox || use_Oz) {
            double dOx = 0.0, dOz = 0.0;
            if (use_Ox) dOx = aa * (f.Ox[c] - f.Ox[c - sj]) + bb * (f.Ox[c + sj] - f.Ox[c - 2 * sj]);
            if (use_Oz) dOz = aa * (f.Oz[c] - f.Oz[c - sk]) + bb * (f.Oz[c + sk] - f.Oz[c - 2 * sk]);
            a.bout[o] = a.k1 * base + a.k3 * a.bprev[o] - dtdy * dOx + dtdz * dOz;
        } else {
            a.bout[o] = base;
        }
    }
    {
        const long long o = fs + c;
        const double base = bbase(a, o);
        if (use_Oy || use_Ox) {
            double dOy = 0.0, dOx = 0.0;
            if (use_Oy) dOy = aa * (f.Oy[c] - f.Oy[c - sk]) + bb * (f.Oy[c + sk] - f.Oy[c - 2 * sk]);
            if (use_Ox) dOx = aa * (f.Ox[c] - f.Ox[c - 1]) + bb * (f.Ox[c + 1] - f.Ox[c - 2]);
            a.bout[o] = a.k1 * base + a.k3 * a.bprev[o] - dtdz * dOy + dtdx * dOx;
        } else {
            a.bout[o] = base;
        }
    }
    {
        const long long o = 2 * fs + c;
        const double base = bbase(a, o);
        if (use_Oz || use_Oy) {
            double dOz = 0.0, dOy = 0.0;
            if (use_Oz) dOz = aa * (f.Oz[c] - f.Oz[c - 1]) + bb * (f.Oz[c + 1] - f.Oz[c - 2]);
            if (use_Oy) dOy = aa * (f.Oy[c] - f.Oy[c - sj]) + bb * (f.Oy[c + sj] - f.Oy[c - 2 * sj]);
            a.bout[o] = a.k1 * base + a.k3 * a.bprev[o] - dtdx * dOz + dtdy * dOy;
        } else {
            a.bout[o] = base;
        }
    }
}

// B(iw) = base everywhere active (1-D runs, where fluxct returns early,
// src/fluxct.cpp:793, and B(iw) keeps the copied / combined stage).
__global__ void k_faceb_base(Grid g, BArgs a) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;
    if (i > g.nx + 2) return;
    const long long c = g.idx(i, j, k);
    for (int comp = 0; comp < 3; ++comp) a.bout[comp * g.fs + c] = bbase(a, comp * g.fs + c);
}

// fluxct_interp_b_to_q (src/fluxct.cpp:882-897) fused with prot
// (src/prot.cpp:10-51), which the reference runs right after on the same cells.
__global__ void k_interp_prot(Grid g, const double* __restrict__ b, double* __restrict__ q,
                              int use_x, int use_y, int use_z, double gam, double rhomin,
                              double pgmin) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;
    if (i > g.nx + 2) return;
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
    q[4 * fs + c] = Bx;
    q[5 * fs + c] = By;
    q[6 * fs + c] = Bz;
    double rho = q[c];
    const double Mx = q[fs + c], My = q[2 * fs + c], Mz = q[3 * fs + c];
    double E = q[7 * fs + c];
    rho = fmax(rho, rhomin);
    const double vx = Mx / rho, vy = My / rho, vz = Mz / rho;
    const double vv2 = vx * vx + vy * vy + vz * vz;
    const double BB2 = Bx * Bx + By * By + Bz * Bz;
    double pg = (gam - 1.0) * (E - 0.5 * (rho * vv2 + BB2));
    pg = fmax(pg, pgmin);
    E = pg / (gam - 1.0) + 0.5 * (rho * vv2 + BB2);
    q[c] = rho;
    q[7 * fs + c] = E;
}

}  // namespace

static BArgs make_bargs(Ctx& c, int iw, double k1, double k3, double c4, double c5, int stage5) {
    BArgs a;
    a.bout = c.b[iw]; a.bprev = c.b[iw - 1];
    a.b0 = c.b[0]; a.b2 = c.b[2]; a.b3 = c.b[3];
    a.k1 = k1; a.k3 = k3; a.c4 = c4; a.c5 = c5; a.stage5 = stage5;
    a.dtdl = &c.dsc->dtdl[iw][0];
    return a;
}

void launch_faceb_base(Ctx& c, int iw, double c4, double c5, int stage5) {
    const Grid& g = c.g;
    BArgs a = make_bargs(c, iw, 1.0, 0.0, c4, c5, stage5);
    dim3 grid((g.nx + 127) / 128, g.ny, g.nz);
    k_faceb_base<<<grid, 128, 0, c.stream>>>(g, a);
    ++c.launches;
    double* bf[3] = {c.b[iw], c.b[iw] + g.fs, c.b[iw] + 2 * g.fs};
    launch_bound(c, bf, 3);
}

// fluxct (src/fluxct.cpp:786-899) + prot for stage iw.  Requires the sweeps of
// the stage to have filled the CT flux arrays at active faces.
void launch_ct(Ctx& c, int iw, double k1, double k3, double c4, double c5, int stage5) {
    const Grid& g = c.g;
    const int use_x = g.nx > 1, use_y = g.ny > 1, use_z = g.nz > 1;
    const int use_Ox = use_x && use_y, use_Oy = use_y && use_z, use_Oz = use_x && use_z;
    CTFields f{c.ct[0], c.ct[1], c.ct[2], c.ct[3], c.ct[4], c.ct[5],
               c.ct[6], c.ct[7], c.ct[8], c.ct[9], c.ct[10], c.ct[11]};
    // bound_ct_fluxes (src/fluxct.cpp:765-772) for the arrays the EMFs read
    {
        double* fl[6];
        int n = 0;
        if (use_Ox) { fl[n++] = c.ct[2]; fl[n++] = c.ct[0]; }           // gsx, fsy
        if (use_Oy) { fl[n++] = c.ct[5]; fl[n++] = c.ct[3]; }           // hsy, gsz
        if (use_Oz) { fl[n++] = c.ct[1]; fl[n++] = c.ct[4]; }           // fsz, hsx
        launch_bound(c, fl, n);
    }
    dim3 grid((g.nx + 127) / 128, g.ny, g.nz);
    k_emf2<<<grid, 128, 0, c.stream>>>(g, f, use_Ox, use_Oy, use_Oz);
    ++c.launches;
    {
        double* fl[3];
        int n = 0;
        if (use_Ox) fl[n++] = c.ct[6];
        if (use_Oy) fl[n++] = c.ct[7];
        if (use_Oz) fl[n++] = c.ct[8];
        launch_bound(c, fl, n);
    }
    k_emf<<<grid, 128, 0, c.stream>>>(g, f, use_Ox, use_Oy, use_Oz);
    ++c.launches;
    {
        double* fl[3];
        int n = 0;
        if (use_Ox) fl[n++] = c.ct[9];
        if (use_Oy) fl[n++] = c.ct[10];
        if (use_Oz) fl[n++] = c.ct[11];
        launch_bound(c, fl, n);
    }
    BArgs a = make_bargs(c, iw, k1, k3, c4, c5, stage5);
    k_update_b<<<grid, 128, 0, c.stream>>>(g, f, a, use_Ox, use_Oy, use_Oz);
    ++c.launches;
    double* bf[3] = {c.b[iw], c.b[iw] + g.fs, c.b[iw] + 2 * g.fs};
    launch_bound(c, bf, 3);
    k_interp_prot<<<grid, 128, 0, c.stream>>>(g, c.b[iw], c.q[iw], use_x, use_y, use_z, c.p.gam,
                                              c.p.rhomin, c.p.pgmin);
    ++c.launches;
}

}  // namespace how
