// how_internal.cuh -- device-side geometry, context and kernel entry points
// shared by the translation units of libhowmhd.so.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "how_mhd.h"

namespace how {

// Device layout: one padded 3-D array ("field") per (stage, variable), x
// fastest.  Index (i, j, k) -> (k * P1 + j) * pitch + i with i,j,k in the
// reference's padded ranges [0, n+6).  pitch >= P0 and a multiple of 8 so
// every row starts on a 64-byte boundary; fields are 256-byte aligned.
struct Grid {
    int nx, ny, nz;
    int P0, P1, P2;
    int pitch;
    long long fs;   // doubles between consecutive fields
    __host__ __device__ inline long long idx(int i, int j, int k) const {
        return ((long long)k * P1 + j) * pitch + i;
    }
};

inline Grid make_grid(int nx, int ny, int nz) {
    Grid g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.P0 = nx + 6; g.P1 = ny + 6; g.P2 = nz + 6;
    g.pitch = (g.P0 + 7) / 8 * 8;
    long long f = (long long)g.pitch * g.P1 * g.P2;
    g.fs = (f + 31) / 32 * 32;
    return g;
}

// x / d, correctly rounded, for d > 0 given y = RN(1/d) (a compile-time
// constant, or one IEEE division shared by several quotients): one multiply
// and two FMAs in place of the division subroutine.  This is the correction
// step of Markstein's division (IBM RS/6000, 1990): q0 = RN(x y) is within an
// ulp of x/d, the remainder x - q0 d is exact in one FMA, and RN(q0 + rem y)
// = RN(x/d).  A zero is returned as it is (x/d keeps its sign); when x or q0
// is outside [2^-900, 2^900], where the remainder could leave the normal
// range, or not finite, the plain division runs.
__device__ __forceinline__ double div_const(double x, double d, double y) {
    const double q0 = __dmul_rn(x, y);
    const double q = __fma_rn(__fma_rn(-q0, d, x), y, q0);
    const double ax = fabs(x), aq = fabs(q0);
    if (ax >= 0x1p-900 && ax <= 0x1p+900 && aq >= 0x1p-900 && aq <= 0x1p+900) return q;
    if (x == 0.0) return x;
    return x / d;
}

// Per-face byte arrays of the learned router (decisions, priors), one per
// sweep direction, laid out line-major so that a line's faces along the sweep
// are contiguous in every direction: the face at padded index s of the line
// through transverse padded indices (t1, t2) (x sweep: j, k; y sweep: i, k;
// z sweep: i, j) is byte route_line(g, dir, t1, t2) + s.  A direction's
// array holds at most P0 P1 P2 <= fs bytes.
__host__ __device__ inline long long route_line(const Grid& g, int dir, int t1, int t2) {
    if (dir == 0) return ((long long)t2 * g.P1 + t1) * g.P0;
    if (dir == 1) return ((long long)t2 * g.P0 + t1) * g.P1;
    return ((long long)t2 * g.P0 + t1) * g.P2;
}

// SSPRK(5,4) coefficients (src/ssprk.cpp:66-94)
struct RKCoeff { double k1, k2, k3, k4, k5; };
inline RKCoeff rk_coeff(int iw) {
    switch (iw) {
        case 1: return {1.0, 0.39175222700392, 0.0, 0.0, 0.0};
        case 2: return {0.44437049406734, 0.36841059262959, 0.55562950593266, 0.0, 0.0};
        case 3: return {0.62010185138540, 0.25189177424738, 0.37989814861460, 0.0, 0.0};
        case 4: return {0.17807995410773, 0.54497475021237, 0.82192004589227, 0.0, 0.0};
        default: return {-2.081261929715610e-02, 0.22600748319395, 5.03580947213895e-1,
                         0.51723167208978, -6.518979800418380e-12};
    }
}

// Device scalars of a context (one cache line each group).
struct DevScalars {
    unsigned long long vmax_bits[3];   // tstep reduction (max of non-negative doubles)
    unsigned int status;               // HOW_STATUS_* bits set by kernels
    unsigned int pad0;
    double dt;                         // current step's dt
    double dtdl[6][3];                 // k2(iw) * dt / d(x,y,z), iw = 1..5
    double dt_raw;                     // dt before the output-time clamp
};

enum : unsigned int { HOW_STATUS_NONFINITE_DT = 1u, HOW_STATUS_TMA_TIMEOUT = 2u, HOW_STATUS_TMA_ALIGN = 4u,
                      HOW_STATUS_NONFINITE_STATE = 8u };

// Arguments of one directional sweep launch.
struct SweepArgs {
    CUtensorMap tm_in;     // stage iw-1: the pencil tile (with halo) of all 8 variables
    CUtensorMap tm_out;    // the update's read operand: q(iw) (accumulate) or the RK base
    Grid g;
    const double* qprev;   // stage iw-1, field 0 (vars at + v * fs)
    double* qout;          // stage iw
    const double* q0;      // stage 0 (RK base)
    const double* q2;      // stage 2 (stage-5 base only)
    const double* q3;      // stage 3 (stage-5 base only)
    double* cta;           // CT flux array fed by the B_t1 row
    double* ctb;           // CT flux array fed by the B_t2 row
    const double* dtdl;    // device: k2 * dt / d_dir for this stage
    double k1, k3, c4, c5; // c4 = k4 / k1, c5 = k5 / k1
    int mode;              // 0 accumulate, 1 first sweep with RK combine, 2 first sweep base+delta
    int stage5;            // base = q0 + c4 q2 + c5 q3
    int ct4;               // 4-point face average of B_n v_t in the CT terms (else 2-point)
    double gam, rhomin, pgmin;
    unsigned long long* prof;   // optional per-phase cycle counters (instrumentation)
    unsigned int* status;       // device status word (HOW_STATUS_* bits)
    // learned routing (MODE 1/2) and label collection (MODE 3)
    const float* router;        // packed MLP weights (RouterLayout), FP32
    const unsigned char* route_prev;  // per face: 1 if sent to full WENO by this direction's previous sweep
    unsigned char* route_next;        // this sweep's decisions (the two arrays swap every sweep)
    unsigned long long* route_count;   // [0] full, [1] cheap interfaces (active faces)
    float* collect;             // records of 8 floats: 6 features, label, weight deviation
    unsigned int* collect_n;    // records written
    unsigned int collect_cap;   // buffer capacity (records)
    unsigned int collect_every; // sample 1 tile in N
    float route_thr;            // logit threshold for full WENO
    float guard_jump;           // hard guard: relative jump of rho or p above this -> full WENO
    float guard_floor;          // hard guard: rho or p below this multiple of the floors -> full WENO
    // batched ensembles (ENS kernels): member m's arguments for this launch
    // are ens_tab[m * ens_stride + ens_off + ens_par[m]]
    const SweepArgs* ens_tab;
    const long long* ens_tile_start;   // [ens_n + 1]: prefix of the members' tile counts
    const int* ens_par;                // per member: stage-0 / stage-5 buffer parity
    const int* ens_active;             // per member: 1 while it is stepping
    int ens_n, ens_stride, ens_off;
    // failure-detection tests: nonzero makes the compute threads' tile waits
    // give up at once (the issuer's drain of copies in flight keeps its
    // full limit), so the launch ends early with HOW_STATUS_TMA_TIMEOUT
    int wait_expire;
};

// Packed router weights (FP32): W1[32][6], b1[32], W2[32][32], b2[32], w3[32], b3.
struct RouterLayout {
    static constexpr int H = 32, NF = 6;
    static constexpr int oW1 = 0, ob1 = oW1 + H * NF, oW2 = ob1 + H, ob2 = oW2 + H * H, ow3 = ob2 + H,
                         ob3 = ow3 + H, total = ob3 + 1;
};

struct Ctx {
    how_params p;
    Grid g;
    int dev = 0;
    cudaStream_t stream = nullptr;
    double* mem = nullptr;          // one allocation for every field
    size_t mem_bytes = 0;
    double* q[6] = {};              // stage s, field 0; var v at + v * fs
    double* qbuf[6] = {};           // the six physical stage buffers (q[] is a permutation)
    CUtensorMap tm_in[6][3];        // per physical buffer and sweep direction: input tile
    CUtensorMap tm_out[6][3];       // per physical buffer and sweep direction: update tile
    double* b[6] = {};              // face B stage s: comps at + c * fs
    double* ct[12] = {};            // fsy fsz gsx gsz hsx hsy Ox2 Oy2 Oz2 Ox Oy Oz
    double* stage_buf = nullptr;    // device staging for layout conversion (8 fields)
    DevScalars* dsc = nullptr;      // device scalars
    DevScalars* hsc = nullptr;      // pinned host mirror
    long launches = 0;
    int precision = HOW_PREC_FP64;
    bool have_state = false;
    unsigned long long* prof = nullptr;   // device phase counters while profiling
    // learned routing
    int route_mode = 0;                   // 0 off, 1 learned, 2 guard only, 3 collect labels
    float* router_w = nullptr;            // device RouterLayout weights
    unsigned char* route_prev = nullptr;  // 3 directions x 2 (read / write) x fs bytes
    int route_par[3] = {0, 0, 0};         // which of a direction's two arrays is read next
    unsigned long long* route_count = nullptr;
    float* collect = nullptr;
    unsigned int* collect_n = nullptr;
    unsigned int collect_cap = 0, collect_every = 1;
    float route_thr = 0.0f, guard_jump = 0.25f, guard_floor = 100.0f;
    int route_refresh = 5;                // learned routing: fresh decisions every this many stages (1..5, 10)
    int cur_stage = 1;                    // SSPRK stage being launched (1..5)
    // learned routing: whether the decision arrays hold the network's
    // decisions for the current run (cleared by any change of the state or
    // of the router), stages since they were formed, and whether the stage
    // being launched forms fresh ones
    bool route_valid = false;
    long long route_age = 0;
    bool route_due = true;
    int wait_expire = 0;                  // failure-detection test hook (SweepArgs::wait_expire)
    // part of a domain decomposed into z slabs (how_group_*): the global z
    // index of local plane 3 minus 3, and which z ghost layers this context
    // fills itself (bit 0 low, bit 1 high: 3 for a whole domain; a side shared
    // with a neighbour is filled by the neighbour's planes instead)
    int part = -1, kstart = 0, gnz = 0;
    int z_sides = 3;
    struct DumpJob* dump = nullptr;       // asynchronous dump file in flight (output.cu)
};

// ---- kernels / launchers (defined in the .cu files) ------------------------
void launch_ref_to_dev(Ctx& c, const double* ref_dev, double* dst, int nvar);
void launch_dev_to_ref(Ctx& c, const double* src, double* ref_dev, int nvar);
void launch_bound(Ctx& c, double* const* fields, int nfields);
void launch_init_faceb(Ctx& c);
void launch_tstep(Ctx& c, double time, double target, int clamp);
void launch_set_dt(Ctx& c);     // dt already in dsc->dt: fill dtdl
void launch_sweep(Ctx& c, int dir, const SweepArgs& a);
// learned-router decisions of every interface of sweep `dir` (route_prepass.cu)
void launch_route(Ctx& c, int dir, const double* q, const unsigned char* prev, unsigned char* next);
void launch_ct(Ctx& c, int iw, double k1, double k3, double c4, double c5, int stage5);
// standalone fluxct(q, iw, k1, k3): face B(iw) = k1 B(iw) + k3 B(iw-1) + CT update, no prot
void launch_fluxct(Ctx& c, int iw, double k1, double k3);
// a part of a z-decomposed domain: CT + prot of stage iw in segments 0..4,
// each ending with the local fills of the arrays part_halo_fields names
void launch_ct_part(Ctx& c, int seg, int iw, double k1, double k3, double c4, double c5, int stage5);
int part_halo_fields(Ctx& c, int seg, int iw, double** out);
// the .pvts master file of a z-decomposed domain's .vts pieces (output.cu)
int write_pvts(const how_params& gp, int nparts, const int* kstart, const int* nzl, int step, const char* dir);
// the sweeps of stage iw (with the stage-5 base), before its CT (capi.cu)
void stage_sweeps(Ctx& c, int iw);
// CFL reduction of stage 0 into the device maxima, and dt from them
void launch_tstep_reduce(Ctx& c);
void launch_tstep_finish(Ctx& c, double time, double target, int clamp);
void launch_faceb_base(Ctx& c, int iw, double c4, double c5, int stage5);
void launch_prot(Ctx& c, int stage);
void launch_stage5_base(Ctx& c, double c4, double c5);
int make_sweep_tensor_maps(Ctx& c);
void launch_copy_fields(Ctx& c, double* dst, const double* src, int nfields);

// asynchronous dump files (output.cu): join the writer, free its buffers
void dump_release(Ctx& c);

void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);

// event timing of kernel launches (instrument.cu)
void timer_begin(Ctx& c, cudaEvent_t* pair_out);
void timer_end(Ctx& c, cudaEvent_t* pair);

}  // namespace how

// The opaque handle of the C ABI is the context itself.
struct how_ctx : how::Ctx {};

#define HOW_CUDA_CHECK(expr)                                   \
    do {                                                       \
        cudaError_t e_ = (expr);                               \
        if (e_ != cudaSuccess) return how::cuda_fail(e_, #expr); \
    } while (0)
