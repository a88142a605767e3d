// ct_kernels.cu -- 4th-order constrained transport (src/fluxct.cpp:786-899).
//
// The reference builds O2 over [0,n+3], smooths over [1,n+4] and updates face
// B over [1,n+3], each followed by a full ghost fill that overwrites every
// index outside [3, n+2] (src/fluxct.cpp:826, 846, 880).  Only active-index
// results survive those fills, so these kernels compute active cells only.
// O2, O and face B are then ghost-filled as there; the flux arrays are not,
// and their reader goes through bc_map, which returns what the fill would
// have left at a ghost index.  Face B: bxb(i) is the x-face at i+1/2.
#include "cell_ops.cuh"

namespace how {

namespace {

#define HOW_CELL_IJK                                                   \
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;           \
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;                  \
    if (i > g.nx + 2) return

// The flux arrays are never ghost-filled here: k_emf2 reads them through
// bc_map (BCMap::on = 1), except in cells whose neighbours two out along
// every stencilled axis are active, where the map is the identity and the
// plain offsets serve.
__device__ __forceinline__ bool ct_inner(const Grid& g, int i, int j, int k) {
    return (g.nx == 1 || (i >= 5 && i <= g.nx)) && (g.ny == 1 || (j >= 5 && j <= g.ny)) &&
           (g.nz == 1 || (k >= 5 && k <= g.nz));
}

__global__ void k_emf2(Grid g, CTFields f, BCMap m, int use_Ox, int use_Oy, int use_Oz) {
    HOW_CELL_IJK;
    if (ct_inner(g, i, j, k)) op_emf2_cell(g, f, BCMap{0, 0, 0, 0}, use_Ox, use_Oy, use_Oz, i, j, k);
    else op_emf2_cell(g, f, m, use_Ox, use_Oy, use_Oz, i, j, k);
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
                              double pgmin, int prot_too) {
    HOW_CELL_IJK;
    op_interp_prot_cell(g, b, q, use_x, use_y, use_z, gam, rhomin, pgmin, i, j, k, prot_too != 0);
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

// fluxct (src/fluxct.cpp:786-899) for stage iw, followed by prot when
// prot_too (as ssprk runs it).  Requires the sweeps of the stage to have
// filled the CT flux arrays at active faces.  The face-B base is the stage's
// copied (or, for stage 5, combined) base formed from b0/b2/b3 in place;
// base_from_stage reads it from face B(iw) itself instead, as the standalone
// fluxct does after the caller's copy_bfield_stage.
static void run_ct(Ctx& c, int iw, double k1, double k3, double c4, double c5, int stage5, bool prot_too,
                   bool base_from_stage) {
    const Grid& g = c.g;
    const int use_x = g.nx > 1, use_y = g.ny > 1, use_z = g.nz > 1;
    const int use_Ox = use_x && use_y, use_Oy = use_y && use_z, use_Oz = use_x && use_z;
    const CTFields f = ct_fields(c.ct);
    // bound_ct_fluxes (src/fluxct.cpp:765-772) is read through bc_map
    // instead of run
    const BCMap m{c.p.bc[0] == HOW_BC_PERIODIC, c.p.bc[1] == HOW_BC_PERIODIC, c.p.bc[2] == HOW_BC_PERIODIC, 1};
    const dim3 grid((g.nx + 127) / 128, g.ny, g.nz);
    k_emf2<<<grid, 128, 0, c.stream>>>(g, f, m, use_Ox, use_Oy, use_Oz);
    ++c.launches;
    {
        // the O2 ghost fill (src/fluxct.cpp:826)
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
        // O is ghost-filled for the face-B update: its four-point differences
        // reach two cells out, and a plain ghost fill costs less than mapping
        // each of its nine neighbour offsets
        double* fl[3];
        int n = 0;
        if (use_Ox) fl[n++] = c.ct[9];
        if (use_Oy) fl[n++] = c.ct[10];
        if (use_Oz) fl[n++] = c.ct[11];
        launch_bound(c, fl, n);
    }
    BArgs a = make_bargs(c, iw, k1, k3, c4, c5, stage5);
    if (base_from_stage) { a.b0 = c.b[iw]; a.stage5 = 0; }
    k_update_b<<<grid, 128, 0, c.stream>>>(g, f, a, use_Ox, use_Oy, use_Oz);
    ++c.launches;
    double* bf[3] = {c.b[iw], c.b[iw] + g.fs, c.b[iw] + 2 * g.fs};
    launch_bound(c, bf, 3);
    k_interp_prot<<<grid, 128, 0, c.stream>>>(g, c.b[iw], c.q[iw], use_x, use_y, use_z, c.p.gam,
                                              c.p.rhomin, c.p.pgmin, prot_too ? 1 : 0);
    ++c.launches;
}

void launch_ct(Ctx& c, int iw, double k1, double k3, double c4, double c5, int stage5) {
    run_ct(c, iw, k1, k3, c4, c5, stage5, true, false);
}

// The same chain for a part of a z-decomposed domain, cut where the
// reference exchanges halos (src/fluxct.cpp:287-479, 554-751; the q halos of
// src/bound.cpp:132-271): each segment ends with the local ghost fills of the
// arrays whose z halos the caller then copies from the neighbours
// (part_halo_fields names them).  The CT flux arrays are ghost-filled here
// and read at plain offsets, as the reference does.
//   seg 0  fill the six CT flux arrays
//   seg 1  corner EMFs (fluxct_build_O2), fill O2
//   seg 2  smoothing (fluxct_smooth_O), fill O
//   seg 3  face-B update, fill face B(iw)
//   seg 4  face-to-centre B + prot, fill q(iw)
void launch_ct_part(Ctx& c, int seg, int iw, double k1, double k3, double c4, double c5, int stage5) {
    const Grid& g = c.g;
    const int use_x = g.nx > 1, use_y = g.ny > 1, use_z = g.nz > 1;
    const int use_Ox = use_x && use_y, use_Oy = use_y && use_z, use_Oz = use_x && use_z;
    const CTFields f = ct_fields(c.ct);
    const dim3 grid((g.nx + 127) / 128, g.ny, g.nz);
    double* fl[12];
    const int n = part_halo_fields(c, seg, iw, fl);
    if (seg == 1) {
        k_emf2<<<grid, 128, 0, c.stream>>>(g, f, BCMap{0, 0, 0, 0}, use_Ox, use_Oy, use_Oz);
        ++c.launches;
    } else if (seg == 2) {
        k_emf<<<grid, 128, 0, c.stream>>>(g, f, use_Ox, use_Oy, use_Oz);
        ++c.launches;
    } else if (seg == 3) {
        BArgs a = make_bargs(c, iw, k1, k3, c4, c5, stage5);
        k_update_b<<<grid, 128, 0, c.stream>>>(g, f, a, use_Ox, use_Oy, use_Oz);
        ++c.launches;
    } else if (seg == 4) {
        k_interp_prot<<<grid, 128, 0, c.stream>>>(g, c.b[iw], c.q[iw], use_x, use_y, use_z, c.p.gam,
                                                  c.p.rhomin, c.p.pgmin, 1);
        ++c.launches;
    }
    launch_bound(c, fl, n);
}

// Arrays whose z halos are exchanged after segment `seg` of stage iw.
int part_halo_fields(Ctx& c, int seg, int iw, double** out) {
    const Grid& g = c.g;
    const int use_Ox = g.nx > 1 && g.ny > 1, use_Oy = g.ny > 1 && g.nz > 1, use_Oz = g.nx > 1 && g.nz > 1;
    int n = 0;
    if (seg == 0) {
        for (int a = 0; a < 6; ++a) out[n++] = c.ct[a];
    } else if (seg == 1 || seg == 2) {
        const int base = seg == 1 ? 6 : 9;
        if (use_Ox) out[n++] = c.ct[base];
        if (use_Oy) out[n++] = c.ct[base + 1];
        if (use_Oz) out[n++] = c.ct[base + 2];
    } else if (seg == 3) {
        for (int k = 0; k < 3; ++k) out[n++] = c.b[iw] + k * g.fs;
    } else {
        for (int v = 0; v < 8; ++v) out[n++] = c.q[iw] + v * g.fs;
    }
    return n;
}

void launch_fluxct(Ctx& c, int iw, double k1, double k3) {
    run_ct(c, iw, k1, k3, 0.0, 0.0, 0, false, true);
}

}  // namespace how
