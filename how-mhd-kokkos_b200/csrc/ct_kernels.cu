// ct_kernels.cu -- 4th-order constrained transport (src/fluxct.cpp:786-899).
//
// The reference builds O2 over [0,n+3], smooths over [1,n+4] and updates face
// B over [1,n+3], each followed by a full ghost fill that overwrites every
// index outside [3, n+2] (src/fluxct.cpp:826, 846, 880).  Only active-index
// results survive those fills, so these kernels compute active cells only and
// then run the same ghost fill.  Face B: bxb(i) is the x-face at i+1/2.
#include "cell_ops.cuh"

namespace how {

namespace {

#define HOW_CELL_IJK                                                   \
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;           \
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;                  \
    if (i > g.nx + 2) return

__global__ void k_emf2(Grid g, CTFields f, int use_Ox, int use_Oy, int use_Oz) {
    HOW_CELL_IJK;
    op_emf2_cell(g, f, use_Ox, use_Oy, use_Oz, i, j, k);
}

__global__ void k_emf(Grid g, CTFields f, int use_Ox, int use_Oy, int use_Oz) {
    HOW_CELL_IJK;
    op_emf_cell(g, f, use_Ox, use_Oy, use_Oz, i, j, k);
}

__global__ void k_update_b(Grid g, CTFields f, BArgs a, int use_Ox, int use_Oy, int use_Oz) {
    HOW_CELL_IJK;
    op_update_b_cell(g, f, a, use_Ox, use_Oy, use_Oz, i, j, k);
}

__global__ void k_faceb_base(Grid g, BArgs a) {
    HOW_CELL_IJK;
    op_faceb_base_cell(g, a, i, j, k);
}

__global__ void k_interp_prot(Grid g, const double* __restrict__ b, double* __restrict__ q,
                              int use_x, int use_y, int use_z, double gam, double rhomin,
                              double pgmin) {
    HOW_CELL_IJK;
    op_interp_prot_cell(g, b, q, use_x, use_y, use_z, gam, rhomin, pgmin, i, j, k);
}
#undef HOW_CELL_IJK

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
    const CTFields f = ct_fields(c.ct);
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
