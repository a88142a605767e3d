// state_kernels.cu -- layout conversion, ghost fill, face-B initialisation,
// the CFL reduction and the positivity floor.  All memory-bound; one thread
// per cell or per ghost column, coalesced along the x-fastest rows.
#include "cell_ops.cuh"

#include <cmath>

namespace how {

namespace {

constexpr int TILE = 32;

// reference layout (v, i, j, k) k-fastest  ->  device (v field, k, j, i) i-fastest.
// 32x32 (i, k) tiles through shared memory for each (v, j).
__global__ void k_ref_to_dev(Grid g, const double* __restrict__ ref, double* __restrict__ dst) {
    __shared__ double tile[TILE][TILE + 1];
    const int k0 = blockIdx.x * TILE, i0 = blockIdx.y * TILE;
    const int j = blockIdx.z % g.P1, v = blockIdx.z / g.P1;
    const long long vbase = (long long)v * g.P0 * g.P1 * g.P2;
    for (int r = threadIdx.y; r < TILE; r += blockDim.y) {
        const int i = i0 + r, k = k0 + threadIdx.x;
        if (i < g.P0 && k < g.P2)
            tile[r][threadIdx.x] = ref[vbase + ((long long)i * g.P1 + j) * g.P2 + k];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < TILE; r += blockDim.y) {
        const int k = k0 + r, i = i0 + threadIdx.x;
        if (i < g.P0 && k < g.P2) dst[(long long)v * g.fs + g.idx(i, j, k)] = tile[threadIdx.x][r];
    }
}

__global__ void k_dev_to_ref(Grid g, const double* __restrict__ src, double* __restrict__ ref) {
    __shared__ double tile[TILE][TILE + 1];
    const int k0 = blockIdx.x * TILE, i0 = blockIdx.y * TILE;
    const int j = blockIdx.z % g.P1, v = blockIdx.z / g.P1;
    const long long vbase = (long long)v * g.P0 * g.P1 * g.P2;
    for (int r = threadIdx.y; r < TILE; r += blockDim.y) {
        const int k = k0 + r, i = i0 + threadIdx.x;
        if (i < g.P0 && k < g.P2) tile[threadIdx.x][r] = src[(long long)v * g.fs + g.idx(i, j, k)];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < TILE; r += blockDim.y) {
        const int i = i0 + r, k = k0 + threadIdx.x;
        if (i < g.P0 && k < g.P2)
            ref[vbase + ((long long)i * g.P1 + j) * g.P2 + k] = tile[r][threadIdx.x];
    }
}

struct FieldList { double* f[12]; int n; };

// Ghost fill along one axis for every listed field, one thread per column.
template <int AX>
__global__ void k_bound_axis(Grid g, FieldList fl, int periodic, int sides) {
    op_bound_column<AX>(g, fl.f[blockIdx.z], blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y, periodic, sides);
}

// initialize_bfield_from_q (src/fluxct.cpp:76-102): i,j,k in [1, n+3]
__global__ void k_init_faceb(Grid g, const double* __restrict__ q0, double* __restrict__ b0) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.nx + 3) return;
    const double* Bx = q0 + 4 * g.fs;
    const double* By = q0 + 5 * g.fs;
    const double* Bz = q0 + 6 * g.fs;
    const long long c = g.idx(i, j, k);
    const long long sj = g.pitch, sk = (long long)g.pitch * g.P1;
    b0[c] = (-Bx[c - 1] + 9.0 * Bx[c] + 9.0 * Bx[c + 1] - Bx[c + 2]) / 16.0;
    b0[g.fs + c] = (-By[c - sj] + 9.0 * By[c] + 9.0 * By[c + sj] - By[c + 2 * sj]) / 16.0;
    b0[2 * g.fs + c] = (-Bz[c - sk] + 9.0 * Bz[c] + 9.0 * Bz[c + sk] - Bz[c + 2 * sk]) / 16.0;
}

// tstep (src/tstep.cpp:28-83): max over active cells of |v_d| + c_f,d.  A
// non-finite conserved value anywhere sets HOW_STATUS_NONFINITE_STATE (the
// reference's reduction skips such cells through fmax and notices only a
// non-finite time, src/main.cpp:207-212; here the caller learns of the bad
// state before stepping on it).
__global__ void k_tstep(Grid g, const double* __restrict__ q, double gam, double rhomin,
                        double pgmin, DevScalars* sc) {
    double mx = 0.0, my = 0.0, mz = 0.0;
    bool ok = true;
    const long long ncell = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x)
        ok &= op_tstep_cell(g, q, gam, rhomin, pgmin, t, mx, my, mz);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(&sc->status, HOW_STATUS_NONFINITE_STATE);
    block_max3_to(mx, my, mz, sc->vmax_bits);
}

__global__ void k_tstep_finalize(DevScalars* sc, int gnx, int gny, int gnz, double dx, double dy,
                                 double dz, double cour, double time, double target, int clamp) {
    op_tstep_finalize(sc, gnx, gny, gnz, dx, dy, dz, cour, time, target, clamp);
}

__global__ void k_set_dt(DevScalars* sc, double dx, double dy, double dz) {
    fill_dtdl(sc, sc->dt, dx, dy, dz);
}

// prot (src/prot.cpp:10-51) on active cells
__global__ void k_prot(Grid g, double* __restrict__ q, double gam, double rhomin, double pgmin) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i > g.nx + 2) return;
    op_prot_cell(g, q, gam, rhomin, pgmin, i, 3 + blockIdx.y, 3 + blockIdx.z);
}

// prepare_stage5 (src/ssprk.cpp:121-140) on active cells
__global__ void k_stage5_base(Grid g, const double* __restrict__ q0, const double* __restrict__ q2,
                              const double* __restrict__ q3, double* __restrict__ q5, double c4, double c5) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i > g.nx + 2) return;
    op_stage5_cell(g, q0, q2, q3, q5, c4, c5, i, 3 + blockIdx.y, 3 + blockIdx.z);
}

__global__ void k_copy(double* __restrict__ dst, const double* __restrict__ src, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        dst[t] = src[t];
}

}  // namespace

void launch_ref_to_dev(Ctx& c, const double* ref_dev, double* dst, int nvar) {
    const Grid& g = c.g;
    dim3 grid((g.P2 + TILE - 1) / TILE, (g.P0 + TILE - 1) / TILE, g.P1 * nvar);
    k_ref_to_dev<<<grid, dim3(TILE, 8), 0, c.stream>>>(g, ref_dev, dst);
    ++c.launches;
}

void launch_dev_to_ref(Ctx& c, const double* src, double* ref_dev, int nvar) {
    const Grid& g = c.g;
    dim3 grid((g.P2 + TILE - 1) / TILE, (g.P0 + TILE - 1) / TILE, g.P1 * nvar);
    k_dev_to_ref<<<grid, dim3(TILE, 8), 0, c.stream>>>(g, src, ref_dev);
    ++c.launches;
}

void launch_bound(Ctx& c, double* const* fields, int nfields) {
    const Grid& g = c.g;
    for (int f0 = 0; f0 < nfields; f0 += 12) {
        FieldList fl;
        fl.n = nfields - f0 < 12 ? nfields - f0 : 12;
        for (int f = 0; f < fl.n; ++f) fl.f[f] = fields[f0 + f];
        k_bound_axis<0><<<dim3((g.P1 + 127) / 128, g.P2, fl.n), 128, 0, c.stream>>>(g, fl, c.p.bc[0] == HOW_BC_PERIODIC, 3);
        k_bound_axis<1><<<dim3((g.P0 + 127) / 128, g.P2, fl.n), 128, 0, c.stream>>>(g, fl, c.p.bc[1] == HOW_BC_PERIODIC, 3);
        c.launches += 2;
        // z: both sides, or for a part of a decomposed domain its physical
        // sides only (the others arrive from the neighbours)
        if (c.z_sides) {
            k_bound_axis<2><<<dim3((g.P0 + 127) / 128, g.P1, fl.n), 128, 0, c.stream>>>(
                g, fl, c.p.bc[2] == HOW_BC_PERIODIC, c.z_sides);
            ++c.launches;
        }
    }
}

void launch_init_faceb(Ctx& c) {
    const Grid& g = c.g;
    k_init_faceb<<<dim3((g.nx + 3 + 127) / 128, g.ny + 3, g.nz + 3), 128, 0, c.stream>>>(g, c.q[0], c.b[0]);
    ++c.launches;
    double* f[3] = {c.b[0], c.b[0] + g.fs, c.b[0] + 2 * g.fs};
    launch_bound(c, f, 3);
}

void launch_tstep_reduce(Ctx& c) {
    const Grid& g = c.g;
    long long ncell = (long long)g.nx * g.ny * g.nz;
    int blocks = (int)((ncell + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    k_tstep<<<blocks, 256, 0, c.stream>>>(g, c.q[0], c.p.gam, c.p.rhomin, c.p.pgmin, c.dsc);
    ++c.launches;
}

// dt from the maxima: the grid sizes of the axes count as the global ones
// (a part of a decomposed domain passes the global nz through gnz)
void launch_tstep_finish(Ctx& c, double time, double target, int clamp) {
    k_tstep_finalize<<<1, 1, 0, c.stream>>>(c.dsc, c.p.nx, c.p.ny, c.part >= 0 ? c.gnz : c.p.nz, c.p.dx, c.p.dy,
                                            c.p.dz, c.p.cour, time, target, clamp);
    ++c.launches;
}

void launch_tstep(Ctx& c, double time, double target, int clamp) {
    launch_tstep_reduce(c);
    launch_tstep_finish(c, time, target, clamp);
}

void launch_set_dt(Ctx& c) {
    k_set_dt<<<1, 1, 0, c.stream>>>(c.dsc, c.p.dx, c.p.dy, c.p.dz);
    ++c.launches;
}

void launch_prot(Ctx& c, int stage) {
    const Grid& g = c.g;
    k_prot<<<dim3((g.nx + 127) / 128, g.ny, g.nz), 128, 0, c.stream>>>(g, c.q[stage], c.p.gam,
                                                                      c.p.rhomin, c.p.pgmin);
    ++c.launches;
}

void launch_stage5_base(Ctx& c, double c4, double c5) {
    const Grid& g = c.g;
    k_stage5_base<<<dim3((g.nx + 127) / 128, g.ny, g.nz), 128, 0, c.stream>>>(g, c.q[0], c.q[2], c.q[3], c.q[5],
                                                                            c4, c5);
    ++c.launches;
}

void launch_copy_fields(Ctx& c, double* dst, const double* src, int nfields) {
    long long n = (long long)nfields * c.g.fs;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_copy<<<blocks, 256, 0, c.stream>>>(dst, src, n);
    ++c.launches;
}

}  // namespace how
