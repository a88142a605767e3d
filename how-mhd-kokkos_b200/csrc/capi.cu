// capi.cu -- the C ABI (include/how_mhd.h): device state, upload/download with
// layout conversion, and the SSPRK(5,4) stage sequence of src/ssprk.cpp:1277-1329
// expressed as kernel launches on the context's stream.
#include "how_internal.cuh"
#include "tma.cuh"

#include <nvtx3/nvToolsExt.h>   // header-only NVTX: named ranges for profilers, no cost without one

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace how {
int router_enable_default(how_ctx* c);

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

int cuda_fail(cudaError_t e, const char* what) {
    set_error("CUDA error %s (%s) in %s", cudaGetErrorName(e), cudaGetErrorString(e), what);
    return HOW_ERR_CUDA;
}

static size_t ref_count(const Grid& g) { return (size_t)g.P0 * g.P1 * g.P2; }

// cuTensorMapEncodeTiled through the runtime's driver entry point.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_tensor_map_4d(CUtensorMap* map, const void* base, const uint64_t dims[4],
                         const uint64_t strides_bytes[3], const uint32_t box[4]) {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) {
            set_error("cuTensorMapEncodeTiled entry point unavailable");
            return HOW_ERR_CUDA;
        }
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    cuuint64_t gd[4] = {dims[0], dims[1], dims[2], dims[3]};
    cuuint64_t gs[3] = {strides_bytes[0], strides_bytes[1], strides_bytes[2]};
    cuuint32_t bx[4] = {box[0], box[1], box[2], box[3]};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(base), gd, gs, bx, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d): box %u x %u x %u x %u", (int)r, box[0], box[1], box[2], box[3]);
        return HOW_ERR_CUDA;
    }
    return HOW_OK;
}

// ---------------------------------------------------------------- one stage
// Stage iw of ssprk (src/ssprk.cpp:1281-1325).  The reference's per-stage
// zero_ct_fluxes, copy_stage / prepare_stage5 and the leading bound(q, iw-1)
// are folded away: the first sweep reads the RK base directly, every CT
// flux the EMFs read is rewritten by the sweeps before its ghost fill, and
// q(iw-1) already had its ghosts filled at the end of the previous stage.
void stage_sweeps(Ctx& c, int iw) {
    const Grid& g = c.g;
    c.cur_stage = iw;
    const RKCoeff k = rk_coeff(iw);
    const double c4 = iw == 5 ? k.k4 / k.k1 : 0.0;
    const double c5 = iw == 5 ? k.k5 / k.k1 : 0.0;
    const int stage5 = iw == 5;
    // learned routing: fresh decisions at a step's first stage and then every
    // route_refresh stages within the step (1..5), or at the first stage of
    // every second step (10); always when the arrays do not hold this run's
    if (!c.route_valid) c.route_age = 0;
    c.route_due = !c.route_valid ||
                  (c.route_refresh <= 5 ? (iw - 1) % c.route_refresh == 0 : c.route_age % c.route_refresh == 0);
    SweepArgs a;
    a.g = g;
    a.qprev = c.q[iw - 1];
    a.qout = c.q[iw];
    a.q0 = c.q[0];
    a.q2 = c.q[2];
    a.q3 = c.q[3];
    a.k1 = k.k1; a.k3 = k.k3; a.c4 = c4; a.c5 = c5;
    a.stage5 = stage5;
    a.gam = c.p.gam; a.rhomin = c.p.rhomin; a.pgmin = c.p.pgmin;
    if (stage5) {
        // prepare_stage5 (src/ssprk.cpp:121-140) on active cells: the first
        // sweep then reads its RK base from q(5) like every other stage's q(0)
        launch_stage5_base(c, c4, c5);
    }
    bool first = true;
    // x_sweep stores k1 q(iw) + k3 q(iw-1) + dq (src/ssprk.cpp:424-427); y/z add.
    // With nx == 1 there is no x sweep and q(iw) keeps the copied base.
    const int ct_a[3] = {0, 3, 4};   // fsy, gsz, hsx
    const int ct_b[3] = {1, 2, 5};   // fsz, gsx, hsy
    const int nd[3] = {g.nx, g.ny, g.nz};
    for (int d = 0; d < 3; ++d) {
        if (nd[d] <= 1) continue;
        a.mode = first ? (d == 0 ? 1 : 2) : 0;
        a.cta = c.ct[ct_a[d]];
        a.ctb = c.ct[ct_b[d]];
        a.dtdl = &c.dsc->dtdl[iw][d];
        launch_sweep(c, d, a);
        first = false;
    }
    if (first) {
        // no sweep at all (1x1x1): q(iw) = base
        launch_copy_fields(c, c.q[iw], c.q[0], 8);
    }
    if (c.route_mode == 1 && !first) {
        if (c.route_due) c.route_age = 0;
        c.route_valid = true;
        ++c.route_age;
    }
}

static void run_stage(Ctx& c, int iw) {
    static const char* const kStageName[6] = {"", "stage 1", "stage 2", "stage 3", "stage 4", "stage 5"};
    nvtxRangePushA(kStageName[iw]);
    const Grid& g = c.g;
    stage_sweeps(c, iw);
    const RKCoeff k = rk_coeff(iw);
    const double c4 = iw == 5 ? k.k4 / k.k1 : 0.0;
    const double c5 = iw == 5 ? k.k5 / k.k1 : 0.0;
    const int stage5 = iw == 5;
    const bool any_ct = (g.nx > 1 && g.ny > 1) || (g.ny > 1 && g.nz > 1) || (g.nx > 1 && g.nz > 1);
    if (any_ct) {
        launch_ct(c, iw, k.k1, k.k3, c4, c5, stage5);
    } else {
        launch_faceb_base(c, iw, c4, c5, stage5);
        launch_prot(c, iw);
    }
    double* qf[8];
    for (int v = 0; v < 8; ++v) qf[v] = c.q[iw] + v * g.fs;
    launch_bound(c, qf, 8);
    nvtxRangePop();
}

static void run_ssprk(Ctx& c) {
    nvtxRangePushA("ssprk");
    for (int iw = 1; iw <= 5; ++iw) run_stage(c, iw);
    nvtxRangePop();
    // copy_stage(q, 0, 5); copy_bfield_to_stage0 (src/ssprk.cpp:1327-1328): swap
    std::swap(c.q[0], c.q[5]);
    std::swap(c.b[0], c.b[5]);
}

static int check_ctx(Ctx* c) {
    if (!c) { set_error("null context"); return HOW_ERR_ARG; }
    HOW_CUDA_CHECK(cudaSetDevice(c->dev));
    return HOW_OK;
}

static int check_stage(int s) {
    if (s < 0 || s > 5) { set_error("stage %d out of range 0..5", s); return HOW_ERR_ARG; }
    return HOW_OK;
}

static int sync_and_status(Ctx& c) {
    HOW_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    HOW_CUDA_CHECK(cudaGetLastError());
    unsigned int st = 0;
    HOW_CUDA_CHECK(cudaMemcpy(&st, &c.dsc->status, sizeof(st), cudaMemcpyDeviceToHost));
    if (st & (HOW_STATUS_TMA_TIMEOUT | HOW_STATUS_TMA_ALIGN | HOW_STATUS_NONFINITE_STATE)) {
        HOW_CUDA_CHECK(cudaMemset(&c.dsc->status, 0, sizeof(st)));
        if (st & (HOW_STATUS_TMA_TIMEOUT | HOW_STATUS_TMA_ALIGN)) {
            set_error("device status 0x%x: %s", st,
                      (st & HOW_STATUS_TMA_ALIGN) ? "misaligned tensor copy refused" : "bounded TMA wait expired");
            return HOW_ERR_CUDA;
        }
        set_error("non-finite value in the conserved state (stage 0, active cells)");
        return HOW_ERR_NONFINITE;
    }
    return HOW_OK;
}

int sync_status(Ctx& c) { return sync_and_status(c); }

}  // namespace how

using namespace how;

extern "C" {

const char* how_last_error(void) { return g_err.c_str(); }

int how_create(const how_params* p, how_ctx** out) {
    if (!p || !out) { set_error("null argument"); return HOW_ERR_ARG; }
    *out = nullptr;
    how_params pp = *p;
    int rc = how_finalize_params(&pp);
    if (rc) return rc;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_error("no CUDA device available (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
        return HOW_ERR_NODEVICE;
    }
    how_ctx* c = new (std::nothrow) how_ctx();
    if (!c) { set_error("out of host memory"); return HOW_ERR_ARG; }
    c->p = pp;
    c->precision = pp.precision;
    c->g = make_grid(pp.nx, pp.ny, pp.nz);
    cudaGetDevice(&c->dev);
    const Grid& g = c->g;
    const int nfields = 6 * 8 + 6 * 3 + 12 + 8;
    c->mem_bytes = (size_t)nfields * g.fs * sizeof(double);
    e = cudaMalloc(&c->mem, c->mem_bytes);
    if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaMalloc(state)"); }
    double* m = c->mem;
    for (int s = 0; s < 6; ++s) { c->q[s] = c->qbuf[s] = m; m += 8 * g.fs; }
    for (int s = 0; s < 6; ++s) { c->b[s] = m; m += 3 * g.fs; }
    for (int a = 0; a < 12; ++a) { c->ct[a] = m; m += g.fs; }
    c->stage_buf = m;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->dsc, sizeof(DevScalars));
    if (e == cudaSuccess) e = cudaMallocHost(&c->hsc, sizeof(DevScalars));
    if (e == cudaSuccess) e = cudaMemsetAsync(c->mem, 0, c->mem_bytes, c->stream);   // Views start zeroed
    if (e == cudaSuccess) e = cudaMemsetAsync(c->dsc, 0, sizeof(DevScalars), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { how_destroy(c); return cuda_fail(e, "context set-up"); }
    std::memset(c->hsc, 0, sizeof(DevScalars));
    if ((rc = make_sweep_tensor_maps(*c))) { how_destroy(c); return rc; }
    if (pp.router && (rc = router_enable_default(c))) { how_destroy(c); return rc; }
    *out = c;
    return HOW_OK;
}

int how_destroy(how_ctx* c) {
    if (!c) return HOW_OK;
    cudaSetDevice(c->dev);
    dump_release(*c);   // an asynchronous dump still being written finishes first
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->mem) cudaFree(c->mem);
    if (c->router_w) cudaFree(c->router_w);
    if (c->route_prev) cudaFree(c->route_prev);
    if (c->route_count) cudaFree(c->route_count);
    if (c->collect) cudaFree(c->collect);
    if (c->collect_n) cudaFree(c->collect_n);
    if (c->dsc) cudaFree(c->dsc);
    if (c->hsc) cudaFreeHost(c->hsc);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return HOW_OK;
}

int how_get_params(const how_ctx* c, how_params* out) {
    if (!c || !out) { set_error("null argument"); return HOW_ERR_ARG; }
    *out = c->p;
    return HOW_OK;
}

size_t how_device_bytes(const how_ctx* c) { return c ? c->mem_bytes + sizeof(DevScalars) : 0; }
long how_kernel_launches(const how_ctx* c) { return c ? c->launches : 0; }
void* how_stream(how_ctx* c) { return c ? (void*)c->stream : nullptr; }

int how_sync(how_ctx* c) {
    int rc = check_ctx(c);
    if (rc) return rc;
    return sync_and_status(*c);
}

int how_set_state(how_ctx* c, int stage, const double* q) {
    int rc = check_ctx(c);
    if (rc || (rc = check_stage(stage))) return rc;
    if (!q) { set_error("null state pointer"); return HOW_ERR_ARG; }
    const size_t n = 8 * ref_count(c->g);
    HOW_CUDA_CHECK(cudaMemcpyAsync(c->stage_buf, q, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch_ref_to_dev(*c, c->stage_buf, c->q[stage], 8);
    if (stage == 0) c->have_state = true;
    c->route_valid = false;   // routing decisions are of the previous state
    return sync_and_status(*c);
}

int how_get_state(how_ctx* c, int stage, double* q) {
    int rc = check_ctx(c);
    if (rc || (rc = check_stage(stage))) return rc;
    if (!q) { set_error("null state pointer"); return HOW_ERR_ARG; }
    const size_t n = 8 * ref_count(c->g);
    launch_dev_to_ref(*c, c->q[stage], c->stage_buf, 8);
    HOW_CUDA_CHECK(cudaMemcpyAsync(q, c->stage_buf, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return sync_and_status(*c);
}

int how_set_face_b(how_ctx* c, int stage, const double* bx, const double* by, const double* bz) {
    int rc = check_ctx(c);
    if (rc || (rc = check_stage(stage))) return rc;
    if (!bx || !by || !bz) { set_error("null face-B pointer"); return HOW_ERR_ARG; }
    const size_t n = ref_count(c->g);
    const double* src[3] = {bx, by, bz};
    for (int k = 0; k < 3; ++k) {
        HOW_CUDA_CHECK(cudaMemcpyAsync(c->stage_buf + k * c->g.fs, src[k], n * sizeof(double),
                                       cudaMemcpyHostToDevice, c->stream));
        launch_ref_to_dev(*c, c->stage_buf + k * c->g.fs, c->b[stage] + k * c->g.fs, 1);
    }
    return sync_and_status(*c);
}

int how_get_face_b(how_ctx* c, int stage, double* bx, double* by, double* bz) {
    int rc = check_ctx(c);
    if (rc || (rc = check_stage(stage))) return rc;
    if (!bx || !by || !bz) { set_error("null face-B pointer"); return HOW_ERR_ARG; }
    const size_t n = ref_count(c->g);
    double* dst[3] = {bx, by, bz};
    for (int k = 0; k < 3; ++k) {
        launch_dev_to_ref(*c, c->b[stage] + k * c->g.fs, c->stage_buf + k * c->g.fs, 1);
        HOW_CUDA_CHECK(cudaMemcpyAsync(dst[k], c->stage_buf + k * c->g.fs, n * sizeof(double),
                                       cudaMemcpyDeviceToHost, c->stream));
    }
    return sync_and_status(*c);
}

int how_get_ct_array(how_ctx* c, int which, double* host) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (which < 0 || which > 11 || !host) { set_error("bad CT array index or null pointer"); return HOW_ERR_ARG; }
    launch_dev_to_ref(*c, c->ct[which], c->stage_buf, 1);
    HOW_CUDA_CHECK(cudaMemcpyAsync(host, c->stage_buf, ref_count(c->g) * sizeof(double),
                                   cudaMemcpyDeviceToHost, c->stream));
    return sync_and_status(*c);
}

int how_bound(how_ctx* c, int stage) {
    int rc = check_ctx(c);
    if (rc || (rc = check_stage(stage))) return rc;
    double* f[8];
    for (int v = 0; v < 8; ++v) f[v] = c->q[stage] + v * c->g.fs;
    launch_bound(*c, f, 8);
    return sync_and_status(*c);
}

int how_bound_bfield(how_ctx* c, int stage) {
    int rc = check_ctx(c);
    if (rc || (rc = check_stage(stage))) return rc;
    double* f[3] = {c->b[stage], c->b[stage] + c->g.fs, c->b[stage] + 2 * c->g.fs};
    launch_bound(*c, f, 3);
    return sync_and_status(*c);
}

int how_init_bfield_from_q(how_ctx* c) {
    int rc = check_ctx(c);
    if (rc) return rc;
    launch_init_faceb(*c);
    return sync_and_status(*c);
}

int how_init_problem(how_ctx* c) {
    int rc = check_ctx(c);
    if (rc) return rc;
    const size_t n = 8 * ref_count(c->g);
    double* h = nullptr;
    HOW_CUDA_CHECK(cudaMallocHost(&h, n * sizeof(double)));
    rc = how_problem_init_host(&c->p, h);
    if (rc == HOW_OK) rc = how_set_state(c, 0, h);
    cudaFreeHost(h);
    if (rc) return rc;
    // bound(q, 0); initialize_bfield_from_q (src/main.cpp:127-130)
    double* f[8];
    for (int v = 0; v < 8; ++v) f[v] = c->q[0] + v * c->g.fs;
    launch_bound(*c, f, 8);
    launch_init_faceb(*c);
    c->have_state = true;
    c->route_valid = false;
    return sync_and_status(*c);
}

int how_tstep(how_ctx* c, double* dt) {
    int rc = check_ctx(c);
    if (rc) return rc;
    launch_tstep(*c, 0.0, 0.0, 0);
    HOW_CUDA_CHECK(cudaMemcpyAsync(c->hsc, c->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
    rc = sync_and_status(*c);
    if (rc) return rc;
    if (dt) *dt = c->hsc->dt;
    if (!std::isfinite(c->hsc->dt)) { set_error("tstep: non-finite dt"); return HOW_ERR_NONFINITE; }
    return HOW_OK;
}

static int upload_dt(how_ctx* c, double dt) {
    c->hsc->dt = dt;
    HOW_CUDA_CHECK(cudaMemcpyAsync(&c->dsc->dt, &c->hsc->dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch_set_dt(*c);
    return HOW_OK;
}

int how_ssprk(how_ctx* c, double dt) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!(dt > 0.0) || !std::isfinite(dt)) { set_error("ssprk: dt must be positive and finite"); return HOW_ERR_DT; }
    if ((rc = upload_dt(c, dt))) return rc;
    run_ssprk(*c);
    return sync_and_status(*c);
}

int how_prot(how_ctx* c, int stage) {
    int rc = check_ctx(c);
    if (rc || (rc = check_stage(stage))) return rc;
    launch_prot(*c, stage);
    return sync_and_status(*c);
}

int how_sweep(how_ctx* c, int dir, double dt) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (dir < 0 || dir > 2) { set_error("sweep direction %d out of range", dir); return HOW_ERR_ARG; }
    const int n = dir == 0 ? c->g.nx : dir == 1 ? c->g.ny : c->g.nz;
    if (n <= 1) { set_error("no sweep along an axis with one cell"); return HOW_ERR_ARG; }
    if ((rc = upload_dt(c, dt))) return rc;
    c->cur_stage = 1;
    c->route_valid = false;   // a lone sweep routes from its own state
    c->route_due = true;
    // stage 1: copy_stage(q, 1, 0), copy_bfield_stage(1, 0), then the sweep
    // (src/ssprk.cpp:1288-1289, 1306-1317)
    launch_copy_fields(*c, c->q[1], c->q[0], 8);
    launch_copy_fields(*c, c->b[1], c->b[0], 3);
    const RKCoeff k = rk_coeff(1);
    SweepArgs a;
    a.g = c->g;
    a.qprev = c->q[0]; a.qout = c->q[1]; a.q0 = c->q[0]; a.q2 = c->q[2]; a.q3 = c->q[3];
    a.k1 = k.k1; a.k3 = k.k3; a.c4 = 0.0; a.c5 = 0.0; a.stage5 = 0;
    a.gam = c->p.gam; a.rhomin = c->p.rhomin; a.pgmin = c->p.pgmin;
    a.mode = dir == 0 ? 1 : 0;
    const int ct_a[3] = {0, 3, 4}, ct_b[3] = {1, 2, 5};
    a.cta = c->ct[ct_a[dir]];
    a.ctb = c->ct[ct_b[dir]];
    a.dtdl = &c->dsc->dtdl[1][dir];
    launch_sweep(*c, dir, a);
    return sync_and_status(*c);
}

int how_fluxct(how_ctx* c, int iw, double k1, double k3) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (iw < 1 || iw > 5) { set_error("fluxct stage %d out of range 1..5", iw); return HOW_ERR_ARG; }
    const Grid& g = c->g;
    const bool any_ct = (g.nx > 1 && g.ny > 1) || (g.ny > 1 && g.nz > 1) || (g.nx > 1 && g.nz > 1);
    if (!any_ct) return HOW_OK;   // 1-D: fluxct returns at once (src/fluxct.cpp:793)
    // bound_bfield(iw - 1) precedes fluxct in ssprk (src/ssprk.cpp:1319)
    double* f[3] = {c->b[iw - 1], c->b[iw - 1] + g.fs, c->b[iw - 1] + 2 * g.fs};
    launch_bound(*c, f, 3);
    launch_fluxct(*c, iw, k1, k3);
    return sync_and_status(*c);
}

int how_set_wait_limit(how_ctx* c, int expire_at_once) {
    if (!c) { set_error("null context"); return HOW_ERR_ARG; }
    c->wait_expire = expire_at_once ? 1 : 0;
    return HOW_OK;
}

int how_set_precision(how_ctx* c, int mode) {
    if (!c) { set_error("null context"); return HOW_ERR_ARG; }
    if (mode != HOW_PREC_FP64 && mode != HOW_PREC_MIXED) { set_error("unknown precision %d", mode); return HOW_ERR_ARG; }
    c->precision = mode;
    c->p.precision = mode;
    return HOW_OK;
}

int how_run(how_ctx* c, double* time, long max_steps, long* steps, double* dts, long dts_cap) {
    int rc = check_ctx(c);
    if (rc) return rc;
    if (!time || !steps) { set_error("null time/steps"); return HOW_ERR_ARG; }
    const double dtout = c->p.tend / (double)c->p.nt;
    long taken = 0;
    // src/main.cpp:158-223: nt output intervals, CFL steps clamped to each end
    for (int out_step = 1; out_step <= c->p.nt; ++out_step) {
        const double target = dtout * (double)out_step;
        while (*time < target) {
            if (max_steps >= 0 && taken >= max_steps) { *steps += taken; return HOW_OK; }
            nvtxRangePushA("tstep");
            launch_tstep(*c, *time, target, 1);
            const cudaError_t ce =
                cudaMemcpyAsync(c->hsc, c->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream);
            nvtxRangePop();
            HOW_CUDA_CHECK(ce);
            rc = sync_and_status(*c);
            if (rc) { *steps += taken; return rc; }
            const double dt = c->hsc->dt;
            // src/main.cpp:175-183: a non-positive dt stops the run (a NaN dt
            // passes this test there too, and the time check below stops it)
            if (dt <= 0.0) {
                *steps += taken;
                set_error("non-positive dt detected: time=%.17g target=%.17g dt=%.17g", *time, target, dt);
                return HOW_ERR_DT;
            }
            run_ssprk(*c);
            *time += dt;
            if (dts && taken < dts_cap) dts[taken] = dt;
            ++taken;
            if (!std::isfinite(*time)) { *steps += taken; set_error("time became non-finite"); return HOW_ERR_NONFINITE; }
        }
    }
    *steps += taken;
    return HOW_OK;
}

}  // extern "C"
