// ensemble.cu -- batched ensembles of independent runs (members) of uneven
// sizes.  Each kernel of an SSPRK(5,4) step is launched once for all members:
// the sweeps as one persistent launch per direction over every member's
// tiles (ensemble_sweep.cu), the memory-bound kernels with blocks assigned to
// members by prefix sums.  The step -- CFL reduction, dt with each member's
// own output-time clamp, five stages, time advance -- runs entirely on the
// device, so one CUDA graph of one step is replayed until every member has
// reached its end time.  Members that are done skip their work.
//
// Every member computes exactly what how_run computes for it alone: the
// per-cell bodies are the single-domain kernels' own (cell_ops.cuh,
// sweep_core.cuh), and dt follows src/main.cpp:158-223 (nt output intervals,
// each step clamped to the interval's end) on the device.
#include "cell_ops.cuh"
#include "ensemble.cuh"

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

namespace how {

namespace {

enum EnsCellOp { OP_STAGE5, OP_EMF2, OP_EMF, OP_UPDATE_B, OP_FACEB_BASE, OP_INTERP_PROT, OP_PROT };
enum EnsBoundKind { BK_Q, BK_B, BK_CTFLUX, BK_O2, BK_O, BK_COUNT };
enum EnsClass { CL_ALL, CL_CT, CL_NOCT, CL_COUNT };

struct EnsDev {
    const EnsMember* mem;
    EnsState* st;
    int* par;
    int* step;      // 1 while the member takes the current step
    int nm;
};

__device__ __forceinline__ int find_member(const long long* start, int nm, long long b) {
    int lo = 0, hi = nm - 1;   // last member whose first block is <= b
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__host__ __device__ __forceinline__ int phys_stage(int par, int s) {
    return (par && (s == 0 || s == 5)) ? 5 - s : s;
}

__device__ __forceinline__ double* ens_field(const EnsMember& M, int par, int kind, int iw, int f) {
    const long long fs = M.g.fs;
    if (kind == BK_Q) return M.qbuf[phys_stage(par, iw)] + f * fs;
    if (kind == BK_B) return M.bbuf[phys_stage(par, iw)] + f * fs;
    // CT arrays in launch_ct's order
    int list[6], n = 0;
    if (kind == BK_CTFLUX) {
        if (M.use_Ox) { list[n++] = 2; list[n++] = 0; }   // gsx, fsy
        if (M.use_Oy) { list[n++] = 5; list[n++] = 3; }   // hsy, gsz
        if (M.use_Oz) { list[n++] = 1; list[n++] = 4; }   // fsz, hsx
    } else {
        const int base = kind == BK_O2 ? 6 : 9;
        if (M.use_Ox) list[n++] = base;
        if (M.use_Oy) list[n++] = base + 1;
        if (M.use_Oz) list[n++] = base + 2;
    }
    return M.ct[list[f < n ? f : 0]];
}

__global__ void k_ens_tstep(EnsDev d, const long long* __restrict__ start) {
    const long long b = blockIdx.x;
    const int m = find_member(start, d.nm, b);
    if (d.st[m].done) return;   // uniform over the block
    const EnsMember& M = d.mem[m];
    const Grid& g = M.g;
    const long long lb = b - start[m], nb = start[m + 1] - start[m];
    const double* q = M.qbuf[phys_stage(d.par[m], 0)];
    const long long ncell = (long long)g.nx * g.ny * g.nz;
    double mx = 0.0, my = 0.0, mz = 0.0;
    for (long long t = lb * blockDim.x + threadIdx.x; t < ncell; t += nb * blockDim.x)
        op_tstep_cell(g, q, M.gam, M.rhomin, M.pgmin, t, mx, my, mz);
    block_max3_to(mx, my, mz, M.dsc->vmax_bits);
}

// dt of each member for this step (src/main.cpp:158-223 on the device)
__global__ void k_ens_finalize(EnsDev d) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= d.nm) return;
    EnsState& S = d.st[m];
    const EnsMember& M = d.mem[m];
    d.step[m] = 0;
    if (S.done) return;
    while (S.out_step <= M.nt && !(S.time < M.dtout * (double)S.out_step)) ++S.out_step;
    if (S.out_step > M.nt) {
        S.done = 1;
        M.dsc->vmax_bits[0] = M.dsc->vmax_bits[1] = M.dsc->vmax_bits[2] = 0ull;
        return;
    }
    const double target = M.dtout * (double)S.out_step;
    const double dt = op_tstep_finalize(M.dsc, M.g.nx, M.g.ny, M.g.nz, M.dx, M.dy, M.dz, M.cour, S.time, target, 1);
    if (!(dt > 0.0)) {   // how_run stops with HOW_ERR_DT
        S.err = 1;
        S.done = 1;
        return;
    }
    d.step[m] = 1;
}

__global__ void k_ens_finish(EnsDev d, unsigned int* count) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= d.nm || !d.step[m]) return;
    EnsState& S = d.st[m];
    S.time += d.mem[m].dsc->dt;
    S.steps += 1;
    d.par[m] ^= 1;   // copy_stage(q, 0, 5): stage 5 becomes stage 0
    atomicAdd(count, 1u);
}

template <int OP>
__global__ void k_ens_cell(EnsDev d, const long long* __restrict__ start, int iw, double k1, double k3, double c4,
                           double c5, int stage5) {
    const long long b = blockIdx.x;
    const int m = find_member(start, d.nm, b);
    if (!d.step[m]) return;
    const EnsMember& M = d.mem[m];
    const Grid& g = M.g;
    const long long lb = b - start[m];
    const int gx = (g.nx + 127) / 128;
    const long long r = lb / gx;
    const int i = 3 + (int)(lb % gx) * 128 + threadIdx.x;
    const int j = 3 + (int)(r % g.ny), k = 3 + (int)(r / g.ny);
    if (i > g.nx + 2) return;
    const int par = d.par[m];
    if constexpr (OP == OP_STAGE5) {
        op_stage5_cell(g, M.qbuf[phys_stage(par, 0)], M.qbuf[2], M.qbuf[3], M.qbuf[phys_stage(par, 5)], c4, c5, i, j,
                       k);
    } else if constexpr (OP == OP_PROT) {
        op_prot_cell(g, M.qbuf[phys_stage(par, iw)], M.gam, M.rhomin, M.pgmin, i, j, k);
    } else if constexpr (OP == OP_INTERP_PROT) {
        op_interp_prot_cell(g, M.bbuf[phys_stage(par, iw)], M.qbuf[phys_stage(par, iw)], M.use_x, M.use_y, M.use_z,
                            M.gam, M.rhomin, M.pgmin, i, j, k);
    } else if constexpr (OP == OP_EMF2 || OP == OP_EMF) {
        const CTFields f = ct_fields(const_cast<double* const*>(M.ct));
        if constexpr (OP == OP_EMF2) op_emf2_cell(g, f, BCMap{0, 0, 0, 0}, M.use_Ox, M.use_Oy, M.use_Oz, i, j, k);
        else op_emf_cell(g, f, M.use_Ox, M.use_Oy, M.use_Oz, i, j, k);
    } else {
        BArgs a;
        a.bout = M.bbuf[phys_stage(par, iw)];
        a.bprev = M.bbuf[phys_stage(par, iw - 1)];
        a.b0 = M.bbuf[phys_stage(par, 0)];
        a.b2 = M.bbuf[2];
        a.b3 = M.bbuf[3];
        a.k1 = k1; a.k3 = k3; a.c4 = c4; a.c5 = c5; a.stage5 = stage5;
        a.dtdl = &M.dsc->dtdl[iw][0];
        if constexpr (OP == OP_UPDATE_B) {
            const CTFields f = ct_fields(const_cast<double* const*>(M.ct));
            op_update_b_cell(g, f, a, M.use_Ox, M.use_Oy, M.use_Oz, i, j, k);
        } else {
            op_faceb_base_cell(g, a, i, j, k);
        }
    }
}

template <int AX>
__global__ void k_ens_bound(EnsDev d, const long long* __restrict__ start, int kind, int iw) {
    const long long b = blockIdx.x;
    const int m = find_member(start, d.nm, b);
    if (!d.step[m]) return;
    const EnsMember& M = d.mem[m];
    const Grid& g = M.g;
    int ta, tb;
    bound_plane<AX>(g, ta, tb);
    const long long lb = b - start[m];
    const int gx = (ta + 127) / 128;
    const long long per = (long long)gx * tb;
    const int f = (int)(lb / per);
    const long long r = lb % per;
    op_bound_column<AX>(g, ens_field(M, d.par[m], kind, iw, f), (int)(r % gx) * 128 + threadIdx.x, (int)(r / gx),
                        M.periodic[AX]);
}

int bound_fields(const EnsMember& M, int kind) {
    const int no = M.use_Ox + M.use_Oy + M.use_Oz;
    switch (kind) {
        case BK_Q: return 8;
        case BK_B: return 3;
        case BK_CTFLUX: return M.any_ct ? 2 * no : 0;
        default: return M.any_ct ? no : 0;
    }
}

}  // namespace
}  // namespace how

using namespace how;

struct how_ensemble {
    int dev = 0;
    cudaStream_t stream = nullptr;
    std::vector<how_ctx*> members;
    std::vector<EnsMember> hmem;
    std::vector<EnsState> hst;
    std::vector<int> hpar;
    // device
    EnsMember* d_mem = nullptr;
    EnsState* d_st = nullptr;
    int* d_par = nullptr;
    int* d_step = nullptr;
    unsigned int* d_count = nullptr;   // members that stepped in the last step
    unsigned int* d_status = nullptr;  // sweep status bits (HOW_STATUS_*)
    long long* d_prefix = nullptr;     // all prefix arrays below, (nm + 1) each
    long long* p_cell[CL_COUNT] = {};
    long long* p_bound[3][BK_COUNT] = {};
    long long* p_tstep = nullptr;
    long long* p_tiles[3] = {};
    long long n_cell[CL_COUNT] = {}, n_bound[3][BK_COUNT] = {}, n_tstep = 0, n_tiles[3] = {};
    SweepArgs* d_tab = nullptr;
    int shape[3] = {-1, -1, -1};
    cudaGraphExec_t exec = nullptr;
    double sweep_ms[3][kEnsShapes] = {};
    long graph_launches = 0;
};

namespace {

constexpr int kTabStride = 6 * 3 * 2;   // [stage 0..5][dir][par]

long long* prefix_slot(how_ensemble* e, int k) { return e->d_prefix + (size_t)k * (e->members.size() + 1); }

int upload_prefix(how_ensemble* e, long long* dst, const std::vector<long long>& counts, long long* total) {
    std::vector<long long> pre(counts.size() + 1, 0);
    for (size_t m = 0; m < counts.size(); ++m) pre[m + 1] = pre[m] + counts[m];
    *total = pre.back();
    HOW_CUDA_CHECK(cudaMemcpy(dst, pre.data(), pre.size() * sizeof(long long), cudaMemcpyHostToDevice));
    return HOW_OK;
}

// Sweep argument table and tile prefixes for shape set e->shape.
int build_sweep_tables(how_ensemble* e) {
    const int nm = (int)e->members.size();
    std::vector<SweepArgs> tab((size_t)nm * kTabStride);
    std::memset((void*)tab.data(), 0, tab.size() * sizeof(SweepArgs));
    const int ct_a[3] = {0, 3, 4}, ct_b[3] = {1, 2, 5};
    for (int m = 0; m < nm; ++m) {
        const Ctx& c = *e->members[m];
        const EnsMember& M = e->hmem[m];
        const int nd[3] = {c.g.nx, c.g.ny, c.g.nz};
        for (int d = 0; d < 3; ++d) {
            if (nd[d] <= 1) continue;
            CUtensorMap tin[6], tout[6];
            int rc = ens_encode_maps(c, d, e->shape[d], tin, tout);
            if (rc) return rc;
            for (int iw = 1; iw <= 5; ++iw) {
                const RKCoeff k = rk_coeff(iw);
                for (int par = 0; par < 2; ++par) {
                    SweepArgs& a = tab[(size_t)m * kTabStride + (iw * 3 + d) * 2 + par];
                    auto Q = [&](int s) { return M.qbuf[phys_stage(par, s)]; };
                    a.g = c.g;
                    a.qprev = Q(iw - 1);
                    a.qout = Q(iw);
                    a.q0 = Q(0);
                    a.q2 = Q(2);
                    a.q3 = Q(3);
                    a.k1 = k.k1; a.k3 = k.k3;
                    a.c4 = iw == 5 ? k.k4 / k.k1 : 0.0;
                    a.c5 = iw == 5 ? k.k5 / k.k1 : 0.0;
                    a.stage5 = iw == 5;
                    // the first sweep of a stage combines (run_stage); members have nx > 1
                    a.mode = d == 0 ? 1 : 0;
                    a.cta = c.ct[ct_a[d]];
                    a.ctb = c.ct[ct_b[d]];
                    a.dtdl = &c.dsc->dtdl[iw][d];
                    a.gam = c.p.gam; a.rhomin = c.p.rhomin; a.pgmin = c.p.pgmin;
                    a.ct4 = c.p.ct_avg == 4;
                    a.status = e->d_status;
                    const int bin = phys_stage(par, iw - 1);
                    const int bout = phys_stage(par, (a.mode == 0 || a.stage5) ? iw : 0);
                    a.tm_in = tin[bin];
                    a.tm_out = tout[bout];
                    a.collect_every = 1;
                }
            }
        }
    }
    if (!e->d_tab) HOW_CUDA_CHECK(cudaMalloc(&e->d_tab, tab.size() * sizeof(SweepArgs)));
    HOW_CUDA_CHECK(cudaMemcpy(e->d_tab, tab.data(), tab.size() * sizeof(SweepArgs), cudaMemcpyHostToDevice));
    for (int d = 0; d < 3; ++d) {
        std::vector<long long> cnt(nm);
        for (int m = 0; m < nm; ++m) cnt[m] = ens_tiles(e->members[m]->g, d, e->shape[d]);
        int rc = upload_prefix(e, e->p_tiles[d], cnt, &e->n_tiles[d]);
        if (rc) return rc;
    }
    if (e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
    return HOW_OK;
}

template <int OP>
void cell_launch(how_ensemble* e, const EnsDev& D, int cls, int iw, double k1, double k3, double c4, double c5,
                 int stage5) {
    if (e->n_cell[cls] == 0) return;
    k_ens_cell<OP><<<(unsigned)e->n_cell[cls], 128, 0, e->stream>>>(D, e->p_cell[cls], iw, k1, k3, c4, c5, stage5);
}

void bound_launch(how_ensemble* e, const EnsDev& D, int kind, int iw) {
    if (e->n_bound[0][kind])
        k_ens_bound<0><<<(unsigned)e->n_bound[0][kind], 128, 0, e->stream>>>(D, e->p_bound[0][kind], kind, iw);
    if (e->n_bound[1][kind])
        k_ens_bound<1><<<(unsigned)e->n_bound[1][kind], 128, 0, e->stream>>>(D, e->p_bound[1][kind], kind, iw);
    if (e->n_bound[2][kind])
        k_ens_bound<2><<<(unsigned)e->n_bound[2][kind], 128, 0, e->stream>>>(D, e->p_bound[2][kind], kind, iw);
}

// One SSPRK(5,4) step of every member still running, enqueued on e->stream.
// With `ev` (3 x 5 x 2 events) each sweep launch is bracketed for timing.
void enqueue_step(how_ensemble* e, cudaEvent_t* ev) {
    const EnsDev D{e->d_mem, e->d_st, e->d_par, e->d_step, (int)e->members.size()};
    const int nm = (int)e->members.size();
    cudaMemsetAsync(e->d_count, 0, sizeof(unsigned int), e->stream);
    k_ens_tstep<<<(unsigned)e->n_tstep, 256, 0, e->stream>>>(D, e->p_tstep);
    k_ens_finalize<<<(nm + 63) / 64, 64, 0, e->stream>>>(D);
    for (int iw = 1; iw <= 5; ++iw) {
        const RKCoeff k = rk_coeff(iw);
        const double c4 = iw == 5 ? k.k4 / k.k1 : 0.0, c5 = iw == 5 ? k.k5 / k.k1 : 0.0;
        const int stage5 = iw == 5;
        if (stage5) cell_launch<OP_STAGE5>(e, D, CL_ALL, iw, 0, 0, c4, c5, stage5);
        for (int d = 0; d < 3; ++d) {
            if (e->n_tiles[d] == 0) continue;
            SweepArgs a0;
            std::memset((void*)&a0, 0, sizeof(a0));
            a0.ens_tab = e->d_tab;
            a0.ens_tile_start = e->p_tiles[d];
            a0.ens_par = e->d_par;
            a0.ens_active = e->d_step;
            a0.ens_n = nm;
            a0.ens_stride = kTabStride;
            a0.ens_off = (iw * 3 + d) * 2;
            a0.status = e->d_status;
            if (ev) cudaEventRecord(ev[(d * 5 + iw - 1) * 2], e->stream);
            ens_launch_sweep(d, e->shape[d], a0, e->stream, e->dev);
            if (ev) cudaEventRecord(ev[(d * 5 + iw - 1) * 2 + 1], e->stream);
        }
        // fluxct (CT members) or face-B base (1-D members), then prot and the ghost fill
        bound_launch(e, D, BK_CTFLUX, iw);
        cell_launch<OP_EMF2>(e, D, CL_CT, iw, 0, 0, 0, 0, 0);
        bound_launch(e, D, BK_O2, iw);
        cell_launch<OP_EMF>(e, D, CL_CT, iw, 0, 0, 0, 0, 0);
        bound_launch(e, D, BK_O, iw);
        cell_launch<OP_UPDATE_B>(e, D, CL_CT, iw, k.k1, k.k3, c4, c5, stage5);
        cell_launch<OP_FACEB_BASE>(e, D, CL_NOCT, iw, 1.0, 0.0, c4, c5, stage5);
        bound_launch(e, D, BK_B, iw);
        cell_launch<OP_INTERP_PROT>(e, D, CL_CT, iw, 0, 0, 0, 0, 0);
        cell_launch<OP_PROT>(e, D, CL_NOCT, iw, 0, 0, 0, 0, 0);
        bound_launch(e, D, BK_Q, iw);
    }
    k_ens_finish<<<(nm + 63) / 64, 64, 0, e->stream>>>(D, e->d_count);
}

// Pull the members' stage parity from their contexts (a member may have been
// stepped on its own in between) and push times / parity to the device.
int upload_state(how_ensemble* e) {
    const int nm = (int)e->members.size();
    for (int m = 0; m < nm; ++m) {
        how_ctx* c = e->members[m];
        HOW_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        e->hpar[m] = c->q[0] == c->qbuf[0] ? 0 : 1;
    }
    HOW_CUDA_CHECK(cudaMemcpy(e->d_par, e->hpar.data(), nm * sizeof(int), cudaMemcpyHostToDevice));
    HOW_CUDA_CHECK(cudaMemcpy(e->d_st, e->hst.data(), nm * sizeof(EnsState), cudaMemcpyHostToDevice));
    return HOW_OK;
}

// Read times / parity back and make each member context's stage pointers match.
int download_state(how_ensemble* e) {
    const int nm = (int)e->members.size();
    HOW_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    HOW_CUDA_CHECK(cudaMemcpy(e->hpar.data(), e->d_par, nm * sizeof(int), cudaMemcpyDeviceToHost));
    HOW_CUDA_CHECK(cudaMemcpy(e->hst.data(), e->d_st, nm * sizeof(EnsState), cudaMemcpyDeviceToHost));
    for (int m = 0; m < nm; ++m) {
        how_ctx* c = e->members[m];
        const EnsMember& M = e->hmem[m];
        for (int s = 0; s < 6; ++s) {
            c->q[s] = M.qbuf[phys_stage(e->hpar[m], s)];
            c->b[s] = M.bbuf[phys_stage(e->hpar[m], s)];
        }
    }
    return HOW_OK;
}

int check_status(how_ensemble* e) {
    unsigned int st = 0;
    HOW_CUDA_CHECK(cudaMemcpy(&st, e->d_status, sizeof(st), cudaMemcpyDeviceToHost));
    if (st & (HOW_STATUS_TMA_TIMEOUT | HOW_STATUS_TMA_ALIGN)) {
        cudaMemset(e->d_status, 0, sizeof(st));
        set_error("ensemble device status 0x%x: %s", st,
                  (st & HOW_STATUS_TMA_ALIGN) ? "misaligned tensor copy refused" : "bounded TMA wait expired");
        return HOW_ERR_CUDA;
    }
    return HOW_OK;
}

// Autotune: one real step per candidate shape set (shape s in every
// direction), the sweeps timed per direction; then each direction takes its
// fastest shape.  A direction's time is its sweeps of stages 2-5, scaled by
// 5/4: the stage-1 launch of a shape is that kernel's first, and can carry
// its one-time module load.  The steps advance the members like any other
// step (the tile shape does not change the arithmetic).
int autotune(how_ensemble* e, long* steps_done) {
    cudaEvent_t ev[30];
    for (auto& x : ev) HOW_CUDA_CHECK(cudaEventCreate(&x));
    for (int s = 0; s < kEnsShapes; ++s) {
        e->shape[0] = e->shape[1] = e->shape[2] = s;
        int rc = build_sweep_tables(e);
        if (rc) return rc;
        enqueue_step(e, ev);
        HOW_CUDA_CHECK(cudaStreamSynchronize(e->stream));
        HOW_CUDA_CHECK(cudaGetLastError());
        if ((rc = check_status(e))) return rc;
        for (int d = 0; d < 3; ++d) {
            double ms = 0.0;
            if (e->n_tiles[d] > 0)
                for (int iw = 1; iw < 5; ++iw) {
                    float t = 0.f;
                    cudaEventElapsedTime(&t, ev[(d * 5 + iw) * 2], ev[(d * 5 + iw) * 2 + 1]);
                    ms += t;
                }
            e->sweep_ms[d][s] = 1.25 * ms;
        }
        ++*steps_done;
    }
    for (auto& x : ev) cudaEventDestroy(x);
    for (int d = 0; d < 3; ++d) {
        int best = 0;
        for (int s = 1; s < kEnsShapes; ++s)
            if (e->sweep_ms[d][s] < e->sweep_ms[d][best]) best = s;
        e->shape[d] = best;
    }
    return build_sweep_tables(e);
}

int capture(how_ensemble* e) {
    cudaGraph_t g = nullptr;
    HOW_CUDA_CHECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed));
    enqueue_step(e, nullptr);
    HOW_CUDA_CHECK(cudaStreamEndCapture(e->stream, &g));
    cudaError_t err = cudaGraphInstantiate(&e->exec, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) { e->exec = nullptr; return cuda_fail(err, "cudaGraphInstantiate"); }
    return HOW_OK;
}

}  // namespace

extern "C" {

int how_ensemble_create(const how_params* params, int n, how_ensemble** out) {
    if (!params || n <= 0 || !out) { set_error("ensemble: need at least one member"); return HOW_ERR_ARG; }
    *out = nullptr;
    how_ensemble* e = new (std::nothrow) how_ensemble();
    if (!e) { set_error("out of host memory"); return HOW_ERR_ARG; }
    for (int m = 0; m < n; ++m) {
        if (params[m].nx <= 1) {
            how_ensemble_destroy(e);
            set_error("ensemble member %d: nx must be > 1", m);
            return HOW_ERR_ARG;
        }
        if (params[m].precision != HOW_PREC_FP64 || params[m].router) {
            how_ensemble_destroy(e);
            set_error("ensemble member %d: members run the plain FP64 method", m);
            return HOW_ERR_ARG;
        }
        how_ctx* c = nullptr;
        int rc = how_create(&params[m], &c);
        if (rc) { how_destroy(c); how_ensemble_destroy(e); return rc; }
        e->members.push_back(c);
    }
    e->dev = e->members[0]->dev;
    const int nm = n;
    e->hmem.resize(nm);
    e->hst.assign(nm, EnsState{0.0, 0, 1, 0, 0, 0});
    e->hpar.assign(nm, 0);
    std::vector<long long> cnt_cell[CL_COUNT], cnt_bound[3][BK_COUNT], cnt_tstep;
    for (int m = 0; m < nm; ++m) {
        how_ctx* c = e->members[m];
        EnsMember& M = e->hmem[m];
        std::memset((void*)&M, 0, sizeof(M));
        M.g = c->g;
        const int par0 = c->q[0] == c->qbuf[0] ? 0 : 1;
        for (int s = 0; s < 6; ++s) {
            M.qbuf[s] = c->qbuf[s];
            M.bbuf[s] = c->b[phys_stage(par0, s)];
        }
        for (int a = 0; a < 12; ++a) M.ct[a] = c->ct[a];
        M.dsc = c->dsc;
        M.gam = c->p.gam; M.rhomin = c->p.rhomin; M.pgmin = c->p.pgmin; M.cour = c->p.cour;
        M.dx = c->p.dx; M.dy = c->p.dy; M.dz = c->p.dz;
        M.nt = c->p.nt;
        M.dtout = c->p.tend / (double)c->p.nt;
        for (int a = 0; a < 3; ++a) M.periodic[a] = c->p.bc[a] == HOW_BC_PERIODIC;
        M.use_x = c->g.nx > 1; M.use_y = c->g.ny > 1; M.use_z = c->g.nz > 1;
        M.use_Ox = M.use_x && M.use_y; M.use_Oy = M.use_y && M.use_z; M.use_Oz = M.use_x && M.use_z;
        M.any_ct = M.use_Ox || M.use_Oy || M.use_Oz;
        const Grid& g = c->g;
        const long long cells = (long long)((g.nx + 127) / 128) * g.ny * g.nz;
        cnt_cell[CL_ALL].push_back(cells);
        cnt_cell[CL_CT].push_back(M.any_ct ? cells : 0);
        cnt_cell[CL_NOCT].push_back(M.any_ct ? 0 : cells);
        for (int ax = 0; ax < 3; ++ax) {
            int ta = ax == 0 ? g.P1 : g.P0, tb = ax == 2 ? g.P1 : g.P2;
            for (int k = 0; k < BK_COUNT; ++k)
                cnt_bound[ax][k].push_back((long long)((ta + 127) / 128) * tb * bound_fields(M, k));
        }
        const long long ncell = (long long)g.nx * g.ny * g.nz;
        long long blocks = (ncell + 255) / 256;
        if (blocks > 148 * 8) blocks = 148 * 8;
        cnt_tstep.push_back(blocks < 1 ? 1 : blocks);
    }
    cudaError_t err = cudaSetDevice(e->dev);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaMalloc(&e->d_mem, nm * sizeof(EnsMember));
    if (err == cudaSuccess) err = cudaMalloc(&e->d_st, nm * sizeof(EnsState));
    if (err == cudaSuccess) err = cudaMalloc(&e->d_par, nm * sizeof(int));
    if (err == cudaSuccess) err = cudaMalloc(&e->d_step, nm * sizeof(int));
    if (err == cudaSuccess) err = cudaMalloc(&e->d_count, sizeof(unsigned int));
    if (err == cudaSuccess) err = cudaMalloc(&e->d_status, sizeof(unsigned int));
    const int nslots = CL_COUNT + 3 * BK_COUNT + 1 + 3;
    if (err == cudaSuccess) err = cudaMalloc(&e->d_prefix, (size_t)nslots * (nm + 1) * sizeof(long long));
    if (err == cudaSuccess) err = cudaMemset(e->d_status, 0, sizeof(unsigned int));
    if (err == cudaSuccess) err = cudaMemset(e->d_step, 0, nm * sizeof(int));
    if (err == cudaSuccess)
        err = cudaMemcpy(e->d_mem, e->hmem.data(), nm * sizeof(EnsMember), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) { how_ensemble_destroy(e); return cuda_fail(err, "ensemble set-up"); }
    int slot = 0, rc = 0;
    for (int k = 0; k < CL_COUNT && !rc; ++k) {
        e->p_cell[k] = prefix_slot(e, slot++);
        rc = upload_prefix(e, e->p_cell[k], cnt_cell[k], &e->n_cell[k]);
    }
    for (int ax = 0; ax < 3 && !rc; ++ax)
        for (int k = 0; k < BK_COUNT && !rc; ++k) {
            e->p_bound[ax][k] = prefix_slot(e, slot++);
            rc = upload_prefix(e, e->p_bound[ax][k], cnt_bound[ax][k], &e->n_bound[ax][k]);
        }
    if (!rc) {
        e->p_tstep = prefix_slot(e, slot++);
        rc = upload_prefix(e, e->p_tstep, cnt_tstep, &e->n_tstep);
    }
    for (int d = 0; d < 3; ++d) e->p_tiles[d] = prefix_slot(e, slot++);
    if (rc) { how_ensemble_destroy(e); return rc; }
    *out = e;
    return HOW_OK;
}

int how_ensemble_destroy(how_ensemble* e) {
    if (!e) return HOW_OK;
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    for (how_ctx* c : e->members) how_destroy(c);
    cudaFree(e->d_mem); cudaFree(e->d_st); cudaFree(e->d_par); cudaFree(e->d_step);
    cudaFree(e->d_count); cudaFree(e->d_status); cudaFree(e->d_prefix); cudaFree(e->d_tab);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return HOW_OK;
}

int how_ensemble_size(const how_ensemble* e) { return e ? (int)e->members.size() : 0; }

how_ctx* how_ensemble_member(how_ensemble* e, int m) {
    if (!e || m < 0 || m >= (int)e->members.size()) { set_error("ensemble member %d out of range", m); return nullptr; }
    return e->members[m];
}

int how_ensemble_init(how_ensemble* e) {
    if (!e) return HOW_ERR_ARG;
    for (how_ctx* c : e->members) {
        int rc = how_init_problem(c);
        if (rc) return rc;
    }
    for (auto& s : e->hst) s = EnsState{0.0, 0, 1, 0, 0, 0};
    return HOW_OK;
}

int how_ensemble_set_shapes(how_ensemble* e, int sx, int sy, int sz) {
    if (!e) return HOW_ERR_ARG;
    const int s[3] = {sx, sy, sz};
    for (int d = 0; d < 3; ++d)
        if (s[d] < 0 || s[d] >= kEnsShapes) { set_error("tile shape %d out of range 0..%d", s[d], kEnsShapes - 1); return HOW_ERR_ARG; }
    HOW_CUDA_CHECK(cudaSetDevice(e->dev));
    for (int d = 0; d < 3; ++d) e->shape[d] = s[d];
    return build_sweep_tables(e);
}

int how_ensemble_get_shapes(const how_ensemble* e, int* shapes, double* sweep_ms) {
    if (!e) return HOW_ERR_ARG;
    for (int d = 0; d < 3; ++d) {
        if (shapes) shapes[d] = e->shape[d];
        if (sweep_ms)
            for (int s = 0; s < kEnsShapes; ++s) sweep_ms[d * kEnsShapes + s] = e->sweep_ms[d][s];
    }
    return HOW_OK;
}

int how_ensemble_shape_info(int dir, int shape, int* lines, int* cells) {
    if (dir < 0 || dir > 2 || shape < 0 || shape >= kEnsShapes || !lines || !cells) return HOW_ERR_ARG;
    ens_shape(dir, shape, lines, cells);
    return HOW_OK;
}

int how_ensemble_run(how_ensemble* e, long max_steps, long* steps_out) {
    if (!e) { set_error("null ensemble"); return HOW_ERR_ARG; }
    HOW_CUDA_CHECK(cudaSetDevice(e->dev));
    long steps = 0;
    int rc = upload_state(e);
    if (rc) return rc;
    if (e->shape[0] < 0) {
        if (max_steps < 0 || max_steps >= kEnsShapes) rc = autotune(e, &steps);
        else { e->shape[0] = e->shape[1] = e->shape[2] = 0; rc = build_sweep_tables(e); }
        if (rc) { download_state(e); return rc; }
    }
    if (!e->exec && (rc = capture(e))) { download_state(e); return rc; }
    // replay the one-step graph, checking after every batch whether any member still runs
    bool running = true;
    while (running && (max_steps < 0 || steps < max_steps)) {
        long batch = 16;
        if (max_steps >= 0 && max_steps - steps < batch) batch = max_steps - steps;
        for (long s = 0; s < batch; ++s) {
            HOW_CUDA_CHECK(cudaGraphLaunch(e->exec, e->stream));
            ++e->graph_launches;
        }
        steps += batch;
        unsigned int cnt = 0;
        HOW_CUDA_CHECK(cudaMemcpyAsync(&cnt, e->d_count, sizeof(cnt), cudaMemcpyDeviceToHost, e->stream));
        HOW_CUDA_CHECK(cudaStreamSynchronize(e->stream));
        if ((rc = check_status(e))) { download_state(e); return rc; }
        running = cnt > 0;
    }
    if ((rc = download_state(e))) return rc;
    long most = 0;
    for (const EnsState& s : e->hst) most = std::max(most, (long)s.steps);
    if (steps_out) *steps_out = most;
    for (size_t m = 0; m < e->hst.size(); ++m)
        if (e->hst[m].err) {
            set_error("ensemble member %zu: non-positive dt at time %.17g", m, e->hst[m].time);
            return HOW_ERR_DT;
        }
    return HOW_OK;
}

int how_ensemble_member_status(const how_ensemble* e, int m, double* time, long* steps, int* done) {
    if (!e || m < 0 || m >= (int)e->members.size()) { set_error("ensemble member %d out of range", m); return HOW_ERR_ARG; }
    const EnsState& s = e->hst[m];
    if (time) *time = s.time;
    if (steps) *steps = (long)s.steps;
    if (done) *done = s.done;
    return HOW_OK;
}

long how_ensemble_graph_launches(const how_ensemble* e) { return e ? e->graph_launches : 0; }
void* how_ensemble_stream(how_ensemble* e) { return e ? (void*)e->stream : nullptr; }

}  // extern "C"
