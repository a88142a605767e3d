// state_kernels.cu -- layout conversion, ghost fill, face-B initialisation,
// the CFL reduction and the positivity floor.  All memory-bound; one thread
// per cell or per ghost column, coalesced along the x-fastest rows.
#include "how_internal.cuh"

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

// Ghost fill along one axis for every listed field, one thread per column,
// in the reference's statement order (src/bound.cpp:19-107): periodic
// A(0)=A(n) A(1)=A(n+1) A(2)=A(n+2) A(n+3)=A(3) A(n+4)=A(4) A(n+5)=A(5);
// open A(0..2)=A(3), A(n+3..5)=A(n+2).  The same rule fills face B
// (src/fluxct.cpp:141-205) and the CT arrays (src/fluxct.cpp:510-552).
template <int AX>
__global__ void k_bound_axis(Grid g, FieldList fl, int periodic) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;   // fastest transverse
    const int b = blockIdx.y;                                // slower transverse
    const int f = blockIdx.z;
    int n, ta, tb;
    long long stride, base;
    if (AX == 0) { n = g.nx; ta = g.P1; tb = g.P2; if (a >= ta) return; base = g.idx(0, a, b); stride = 1; }
    else if (AX == 1) { n = g.ny; ta = g.P0; tb = g.P2; if (a >= ta) return; base = g.idx(a, 0, b); stride = g.pitch; }
    else { n = g.nz; ta = g.P0; tb = g.P1; if (a >= ta) return; base = g.idx(a, b, 0); stride = (long long)g.pitch * g.P1; }
    (void)tb;
    double* A = fl.f[f] + base;
    auto at = [&](int s) -> double& { return A[s * stride]; };
    if (periodic) {
        at(0) = at(n); at(1) = at(n + 1); at(2) = at(n + 2);
        at(n + 3) = at(3); at(n + 4) = at(4); at(n + 5) = at(5);
    } else {
        const double lo = at(3);
        at(0) = lo; at(1) = lo; at(2) = lo;
        const double hi = at(n + 2);
        at(n + 3) = hi; at(n + 4) = hi; at(n + 5) = hi;
    }
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

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// tstep (src/tstep.cpp:28-83): max over active cells of |v_d| + c_f,d.
// Block reduction by warp shuffles, then one atomicMax per block on the bit
// pattern (non-negative doubles order like their bit patterns).
__global__ void k_tstep(Grid g, const double* __restrict__ q, double gam, double rhomin,
                        double pgmin, DevScalars* sc) {
    double mx = 0.0, my = 0.0, mz = 0.0;
    const long long ncell = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = 3 + (int)(t % g.nx);
        const long long r = t / g.nx;
        const int j = 3 + (int)(r % g.ny);
        const int k = 3 + (int)(r / g.ny);
        const long long c = g.idx(i, j, k);
        const double DD = q[c], Mx = q[g.fs + c], My = q[2 * g.fs + c], Mz = q[3 * g.fs + c];
        const double Bx = q[4 * g.fs + c], By = q[5 * g.fs + c], Bz = q[6 * g.fs + c];
        const double EE = q[7 * g.fs + c];
        const double rho = fmax(DD, rhomin);
        const double vx = Mx / rho, vy = My / rho, vz = Mz / rho;
        const double vv2 = vx * vx + vy * vy + vz * vz;
        const double BB2 = Bx * Bx + By * By + Bz * Bz;
        const double pg = fmax(pgmin, (gam - 1.0) * (EE - 0.5 * (rho * vv2 + BB2)));
        const double bbn2 = BB2 / rho;
        const double cs2 = fmax(0.0, gam * pg / rho);
        const double bnx2 = Bx * Bx / rho, bny2 = By * By / rho, bnz2 = Bz * Bz / rho;
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
    }
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
            atomicMax(&sc->vmax_bits[0], (unsigned long long)__double_as_longlong(mx));
            atomicMax(&sc->vmax_bits[1], (unsigned long long)__double_as_longlong(my));
            atomicMax(&sc->vmax_bits[2], (unsigned long long)__double_as_longlong(mz));
        }
    }
}

__device__ void fill_dtdl(DevScalars* sc, double dt, double dx, double dy, double dz) {
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
// clamp to the output time (src/main.cpp:170-172).
__global__ void k_tstep_finalize(DevScalars* sc, int gnx, int gny, int gnz, double dx, double dy,
                                 double dz, double cour, double time, double target, int clamp) {
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
}

__global__ void k_set_dt(DevScalars* sc, double dx, double dy, double dz) {
    fill_dtdl(sc, sc->dt, dx, dy, dz);
}

// prot (src/prot.cpp:10-51) on active cells
__global__ void k_prot(Grid g, double* __restrict__ q, double gam, double rhomin, double pgmin) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;
    if (i > g.nx + 2) return;
    const long long c = g.idx(i, j, k);
    double rho = q[c];
    const double Mx = q[g.fs + c], My = q[2 * g.fs + c], Mz = q[3 * g.fs + c];
    const double Bx = q[4 * g.fs + c], By = q[5 * g.fs + c], Bz = q[6 * g.fs + c];
    double E = q[7 * g.fs + c];
    rho = fmax(rho, rhomin);
    const double vx = Mx / rho, vy = My / rho, vz = Mz / rho;
    const double vv2 = vx * vx + vy * vy + vz * vz;
    const double BB2 = Bx * Bx + By * By + Bz * Bz;
    double pg = (gam - 1.0) * (E - 0.5 * (rho * vv2 + BB2));
    pg = fmax(pg, pgmin);
    E = pg / (gam - 1.0) + 0.5 * (rho * vv2 + BB2);
    q[c] = rho;
    q[7 * g.fs + c] = E;
}

// prepare_stage5 (src/ssprk.cpp:121-140) on active cells:
// q5 = q0 + (k4/k1) q2 + (k5/k1) q3, all 8 variables.
__global__ void k_stage5_base(Grid g, const double* __restrict__ q0, const double* __restrict__ q2,
                              const double* __restrict__ q3, double* __restrict__ q5, double c4, double c5) {
    const int i = 3 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y, k = 3 + blockIdx.z;
    if (i > g.nx + 2) return;
    const long long c = g.idx(i, j, k);
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const long long o = v * g.fs + c;
        q5[o] = q0[o] + c4 * q2[o] + c5 * q3[o];
    }
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
        k_bound_axis<0><<<dim3((g.P1 + 127) / 128, g.P2, fl.n), 128, 0, c.stream>>>(g, fl, c.p.bc[0] == HOW_BC_PERIODIC);
        k_bound_axis<1><<<dim3((g.P0 + 127) / 128, g.P2, fl.n), 128, 0, c.stream>>>(g, fl, c.p.bc[1] == HOW_BC_PERIODIC);
        k_bound_axis<2><<<dim3((g.P0 + 127) / 128, g.P1, fl.n), 128, 0, c.stream>>>(g, fl, c.p.bc[2] == HOW_BC_PERIODIC);
        c.launches += 3;
    }
}

void launch_init_faceb(Ctx& c) {
    const Grid& g = c.g;
    k_init_faceb<<<dim3((g.nx + 3 + 127) / 128, g.ny + 3, g.nz + 3), 128, 0, c.stream>>>(g, c.q[0], c.b[0]);
    ++c.launches;
    double* f[3] = {c.b[0], c.b[0] + g.fs, c.b[0] + 2 * g.fs};
    launch_bound(c, f, 3);
}

void launch_tstep(Ctx& c, double time, double target, int clamp) {
    const Grid& g = c.g;
    long long ncell = (long long)g.nx * g.ny * g.nz;
    int blocks = (int)((ncell + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    k_tstep<<<blocks, 256, 0, c.stream>>>(g, c.q[0], c.p.gam, c.p.rhomin, c.p.pgmin, c.dsc);
    k_tstep_finalize<<<1, 1, 0, c.stream>>>(c.dsc, c.p.nx, c.p.ny, c.p.nz, c.p.dx, c.p.dy, c.p.dz,
                                            c.p.cour, time, target, clamp);
    c.launches += 2;
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
