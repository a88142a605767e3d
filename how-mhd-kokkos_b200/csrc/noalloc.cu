// noalloc.cu -- an allocation-free CFL time step for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs this solver's time-step selection inside a
// host application that owns every byte of GPU memory -- a Kokkos or AMReX
// application whose memory pool has already reserved the device, a plugin
// loaded into such a process, or a caller running under an allocator that
// forbids cudaMalloc/cudaFree once its set-up is over.  Those callers can
// hand us their state and a place for the result, but we may not allocate.
//
// How: the reduction keeps its per-line partial maxima in a file-scope
// __device__ array of fixed size (HOW_NOALLOC_MAX_LINES lines x 3 doubles,
// 6 MiB per GPU).  In host code the array's name is only a host-side
// stand-in, so every call looks up its device address on the current device
// with cudaGetSymbolAddress and passes that to the kernels (a cached address
// would go stale after a device reset).  Under CUDA's default lazy module
// loading, this file's module -- and with it the array -- is placed on a
// device by the first such lookup there: the first call on each device takes
// the 6 MiB, and the array stays until the process exits.  Callers make that
// first call during set-up, before a memory pool reserves the device, or set
// CUDA_MODULE_LOADING=EAGER so the array is placed when the library loads.
#include "how_internal.cuh"

namespace how {
namespace {

constexpr int kNoAllocMaxLines = HOW_NOALLOC_MAX_LINES;

static __device__ __align__(256) double g_cfl_line_max[3 * kNoAllocMaxLines];


// Pass 1: one warp per (i, j) line along k (contiguous in the reference
// layout), lanes striding k; writes the line's three maxima of |v_d| + c_f,d
// (the per-cell formula of src/tstep.cpp:35-78).
__global__ void k_cfl_lines(const double* __restrict__ q, int nx, int ny, int nz, double gam,
                            double rhomin, double pgmin, double* __restrict__ line_max) {
    const int warps_per_block = blockDim.x >> 5;
    const long long line = (long long)blockIdx.x * warps_per_block + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const long long nlines = (long long)nx * ny;
    if (line >= nlines) return;
    const int i = 3 + (int)(line / ny), j = 3 + (int)(line % ny);
    const long long P0 = nx + 6, P1 = ny + 6, P2 = nz + 6;
    const long long vs = P0 * P1 * P2;
    double mx = 0.0, my = 0.0, mz = 0.0;
    for (int k = 3 + lane; k < nz + 3; k += 32) {
        const long long c = ((long long)i * P1 + j) * P2 + k;
        const double DD = q[c], Mx = q[vs + c], My = q[2 * vs + c], Mz = q[3 * vs + c];
        const double Bx = q[4 * vs + c], By = q[5 * vs + c], Bz = q[6 * vs + c], EE = q[7 * vs + c];
        const double rho = fmax(DD, rhomin);
        const double vx = Mx / rho, vy = My / rho, vz = Mz / rho;
        const double vv2 = vx * vx + vy * vy + vz * vz;
        const double BB2 = Bx * Bx + By * By + Bz * Bz;
        const double pg = fmax(pgmin, (gam - 1.0) * (EE - 0.5 * (rho * vv2 + BB2)));
        const double bbn2 = BB2 / rho;
        const double cs2 = fmax(0.0, gam * pg / rho);
        const double s = (bbn2 + cs2) * (bbn2 + cs2);
        const double lfx = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 + sqrt(fmax(0.0, s - 4.0 * (Bx * Bx / rho) * cs2)))));
        const double lfy = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 + sqrt(fmax(0.0, s - 4.0 * (By * By / rho) * cs2)))));
        const double lfz = sqrt(fmax(0.0, 0.5 * (bbn2 + cs2 + sqrt(fmax(0.0, s - 4.0 * (Bz * Bz / rho) * cs2)))));
        mx = fmax(mx, fabs(vx) + lfx);
        my = fmax(my, fabs(vy) + lfy);
        mz = fmax(mz, fabs(vz) + lfz);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        my = fmax(my, __shfl_xor_sync(0xffffffffu, my, o));
        mz = fmax(mz, __shfl_xor_sync(0xffffffffu, mz, o));
    }
    if (lane == 0) {
        line_max[3 * line] = mx;
        line_max[3 * line + 1] = my;
        line_max[3 * line + 2] = mz;
    }
}

// Pass 2: one block reduces every line written by pass 1 (all of them are
// rewritten on each call, so nothing needs clearing) and forms
// dt = cour / sum_d(vmax_d / d_d) over the axes with more than one cell
// (src/tstep.cpp:123-135).
__global__ void k_cfl_finish(const double* __restrict__ line_max, long long nlines, int nx, int ny, int nz,
                             double dx, double dy, double dz, double cour, double* __restrict__ dt_out) {
    double mx = 0.0, my = 0.0, mz = 0.0;
    for (long long l = threadIdx.x; l < nlines; l += blockDim.x) {
        mx = fmax(mx, line_max[3 * l]);
        my = fmax(my, line_max[3 * l + 1]);
        mz = fmax(mz, line_max[3 * l + 2]);
    }
    __shared__ double red[3][32];
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        my = fmax(my, __shfl_xor_sync(0xffffffffu, my, o));
        mz = fmax(mz, __shfl_xor_sync(0xffffffffu, mz, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red[0][w] = mx; red[1][w] = my; red[2][w] = mz; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            mx = fmax(mx, red[0][k]); my = fmax(my, red[1][k]); mz = fmax(mz, red[2][k]);
        }
        const double tiny = 1.0e-300;
        double invdt = 0.0;
        if (nx > 1) invdt += fmax(mx, tiny) / dx;
        if (ny > 1) invdt += fmax(my, tiny) / dy;
        if (nz > 1) invdt += fmax(mz, tiny) / dz;
        if (invdt <= 0.0) invdt = fmax(mx, tiny) / dx;
        *dt_out = cour / invdt;
    }
}

// Device address of the scratch array on the current device (the device
// the kernels below launch on).  The first lookup on a device places the
// module there; later ones only read its address.
int scratch_for_current_device(double** out) {
    double* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_cfl_line_max);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_cfl_line_max)");
    *out = p;
    return HOW_OK;
}

}  // namespace
}  // namespace how

extern "C" int how_tstep_noalloc(const double* q_dev, const how_params* p, double* dt_dev, void* stream) {
    using namespace how;
    if (!q_dev || !p || !dt_dev) { set_error("how_tstep_noalloc: null argument"); return HOW_ERR_ARG; }
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0) { set_error("how_tstep_noalloc: non-positive grid"); return HOW_ERR_ARG; }
    const long long nlines = (long long)p->nx * p->ny;
    if (nlines > kNoAllocMaxLines) {
        set_error("how_tstep_noalloc: nx*ny = %lld lines exceeds the fixed scratch of %d lines "
                  "(HOW_NOALLOC_MAX_LINES); use how_tstep on a context instead", nlines, kNoAllocMaxLines);
        return HOW_ERR_ARG;
    }
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int threads = 256, warps = threads / 32;
    const long long blocks = (nlines + warps - 1) / warps;
    k_cfl_lines<<<(unsigned)blocks, threads, 0, s>>>(q_dev, p->nx, p->ny, p->nz, p->gam, p->rhomin, p->pgmin, scratch);
    const double dx = p->xsize / (double)p->nx, dy = p->ysize / (double)p->ny, dz = p->zsize / (double)p->nz;
    k_cfl_finish<<<1, 1024, 0, s>>>(scratch, nlines, p->nx, p->ny, p->nz, dx, dy, dz, p->cour, dt_dev);
    HOW_CUDA_CHECK(cudaGetLastError());
    return HOW_OK;
}
