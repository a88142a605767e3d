// group.cu -- one domain decomposed into z slabs ("parts"), one context per
// part, possibly on different GPUs, stepped together by one host thread.
//
// This is the reference's MPI build re-designed for GPUs in one node: its
// Cartesian split (setup_mpi_domain, src/mpi_domain.cpp:93-155) becomes a
// split along z; its host-staged halo exchanges (q: src/bound.cpp:132-271;
// face B and the CT arrays: src/fluxct.cpp:287-479, 554-751) become copies of
// whole z planes from a part's own buffers straight into its neighbour's
// ghost planes (the device layout is x fastest, so a z plane of a field is
// one contiguous run: nothing is packed), peer-to-peer over NVLink between
// GPUs; its dt allreduce (src/tstep.cpp:87-121) becomes a max over the parts'
// CFL maxima.  The parts run the same kernels as a whole domain, so a
// decomposed run equals the undecomposed one bit for bit.
//
// The reference's apply_physical_boundaries_q fills open boundaries on both
// sides of a rank that has only one physical side (src/bound.cpp:273-291);
// here each part fills only its physical sides and takes the others from its
// neighbours.
//
// Ordering: each part works on its own stream.  Before a copy out of part A
// the receiving stream waits for A's fills (event `ready`); after the copies
// A's stream waits for its neighbours' copies to finish (event `done`)
// before it may overwrite the planes they read.
#include "how_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace how {
int sync_status(Ctx& c);
}

using namespace how;

struct how_group {
    how_params global{};
    int n = 0;
    bool periodic_z = true;
    std::vector<how_ctx*> parts;
    std::vector<int> kstart, nzl, dev;
    std::vector<cudaEvent_t> ready, done;
};

namespace {

int set_dev(const how_group* g, int p) {
    HOW_CUDA_CHECK(cudaSetDevice(g->dev[p]));
    return HOW_OK;
}

// Copies the z halos of one list of arrays (the same arrays in every part,
// `fields[p][f]`) between neighbouring parts: the lower part's top three
// active planes into the upper part's planes 0..2, the upper part's planes
// 3..5 into the lower part's planes nz+3..nz+5.
int halo_exchange(how_group* g, const std::vector<std::vector<double*>>& fields) {
    const int n = g->n;
    if (n < 2) return HOW_OK;
    const Grid& gr = g->parts[0]->g;
    const size_t plane = (size_t)gr.P1 * gr.pitch;
    const size_t bytes = 3 * plane * sizeof(double);
    for (int p = 0; p < n; ++p) {
        HOW_CUDA_CHECK(cudaSetDevice(g->dev[p]));
        HOW_CUDA_CHECK(cudaEventRecord(g->ready[p], g->parts[p]->stream));
    }
    const int nb = g->periodic_z ? n : n - 1;   // boundaries: lower part b, upper part (b + 1) % n
    for (int b = 0; b < nb; ++b) {
        const int lo = b, up = (b + 1) % n;
        Ctx& L = *g->parts[lo];
        Ctx& U = *g->parts[up];
        HOW_CUDA_CHECK(cudaSetDevice(g->dev[up]));
        HOW_CUDA_CHECK(cudaStreamWaitEvent(U.stream, g->ready[lo], 0));
        how_part_info pl, pu;
        how_part_plan(g->global.nz, n, g->periodic_z, lo, &pl);
        how_part_plan(g->global.nz, n, g->periodic_z, up, &pu);
        for (size_t f = 0; f < fields[up].size(); ++f)
            HOW_CUDA_CHECK(cudaMemcpyPeerAsync(fields[up][f] + (size_t)pu.recv_lo_first * plane, g->dev[up],
                                               fields[lo][f] + (size_t)pl.send_up_first * plane, g->dev[lo],
                                               bytes, U.stream));
        HOW_CUDA_CHECK(cudaSetDevice(g->dev[lo]));
        HOW_CUDA_CHECK(cudaStreamWaitEvent(L.stream, g->ready[up], 0));
        for (size_t f = 0; f < fields[lo].size(); ++f)
            HOW_CUDA_CHECK(cudaMemcpyPeerAsync(fields[lo][f] + (size_t)pl.recv_hi_first * plane, g->dev[lo],
                                               fields[up][f] + (size_t)pu.send_down_first * plane, g->dev[up],
                                               bytes, L.stream));
    }
    for (int p = 0; p < n; ++p) {
        HOW_CUDA_CHECK(cudaSetDevice(g->dev[p]));
        HOW_CUDA_CHECK(cudaEventRecord(g->done[p], g->parts[p]->stream));
    }
    for (int b = 0; b < nb; ++b) {
        const int lo = b, up = (b + 1) % n;
        HOW_CUDA_CHECK(cudaSetDevice(g->dev[lo]));
        HOW_CUDA_CHECK(cudaStreamWaitEvent(g->parts[lo]->stream, g->done[up], 0));
        HOW_CUDA_CHECK(cudaSetDevice(g->dev[up]));
        HOW_CUDA_CHECK(cudaStreamWaitEvent(g->parts[up]->stream, g->done[lo], 0));
    }
    return HOW_OK;
}

// the arrays `seg` names in every part (part_halo_fields), exchanged
int exchange_seg(how_group* g, int seg, int iw) {
    std::vector<std::vector<double*>> f(g->n);
    for (int p = 0; p < g->n; ++p) {
        double* arr[12];
        const int k = part_halo_fields(*g->parts[p], seg, iw, arr);
        f[p].assign(arr, arr + k);
    }
    return halo_exchange(g, f);
}

int exchange_stage_q(how_group* g, int stage) {
    std::vector<std::vector<double*>> f(g->n);
    for (int p = 0; p < g->n; ++p)
        for (int v = 0; v < 8; ++v) f[p].push_back(g->parts[p]->q[stage] + v * g->parts[p]->g.fs);
    return halo_exchange(g, f);
}

int exchange_stage_b(how_group* g, int stage) {
    std::vector<std::vector<double*>> f(g->n);
    for (int p = 0; p < g->n; ++p)
        for (int k = 0; k < 3; ++k) f[p].push_back(g->parts[p]->b[stage] + k * g->parts[p]->g.fs);
    return halo_exchange(g, f);
}

int sync_all(how_group* g) {
    int first = HOW_OK;
    for (int p = 0; p < g->n; ++p) {
        int rc = set_dev(g, p);
        if (!rc) rc = sync_status(*g->parts[p]);
        if (rc && first == HOW_OK) first = rc;
    }
    return first;
}

// ghost fill of stage `stage` of q (local fills, then the halos)
int bound_q(how_group* g, int stage) {
    for (int p = 0; p < g->n; ++p) {
        int rc = set_dev(g, p);
        if (rc) return rc;
        Ctx& c = *g->parts[p];
        double* f[8];
        for (int v = 0; v < 8; ++v) f[v] = c.q[stage] + v * c.g.fs;
        launch_bound(c, f, 8);
    }
    return exchange_stage_q(g, stage);
}

// one SSPRK(5,4) step of every part (src/ssprk.cpp:1277-1329)
int step(how_group* g) {
    for (int iw = 1; iw <= 5; ++iw) {
        const RKCoeff k = rk_coeff(iw);
        const double c4 = iw == 5 ? k.k4 / k.k1 : 0.0;
        const double c5 = iw == 5 ? k.k5 / k.k1 : 0.0;
        for (int seg = 0; seg <= 4; ++seg) {
            for (int p = 0; p < g->n; ++p) {
                int rc = set_dev(g, p);
                if (rc) return rc;
                if (seg == 0) stage_sweeps(*g->parts[p], iw);
                launch_ct_part(*g->parts[p], seg, iw, k.k1, k.k3, c4, c5, iw == 5);
            }
            int rc = exchange_seg(g, seg, iw);
            if (rc) return rc;
        }
    }
    for (int p = 0; p < g->n; ++p) {
        std::swap(g->parts[p]->q[0], g->parts[p]->q[5]);
        std::swap(g->parts[p]->b[0], g->parts[p]->b[5]);
    }
    return HOW_OK;
}

// tstep over every part (the allreduce of src/tstep.cpp:87-121 as a max of
// the parts' maxima; non-negative doubles order like their bit patterns),
// then dt with the clamp to the output time
int tstep_all(how_group* g, double time, double target, int clamp, double* dt) {
    for (int p = 0; p < g->n; ++p) {
        int rc = set_dev(g, p);
        if (rc) return rc;
        launch_tstep_reduce(*g->parts[p]);
    }
    unsigned long long mx[3] = {0, 0, 0};
    for (int p = 0; p < g->n; ++p) {
        int rc = set_dev(g, p);
        if (rc) return rc;
        Ctx& c = *g->parts[p];
        rc = sync_status(c);
        if (rc) return rc;
        unsigned long long v[3];
        HOW_CUDA_CHECK(cudaMemcpy(v, c.dsc->vmax_bits, sizeof(v), cudaMemcpyDeviceToHost));
        for (int d = 0; d < 3; ++d) mx[d] = std::max(mx[d], v[d]);
    }
    for (int p = 0; p < g->n; ++p) {
        int rc = set_dev(g, p);
        if (rc) return rc;
        Ctx& c = *g->parts[p];
        HOW_CUDA_CHECK(cudaMemcpyAsync(c.dsc->vmax_bits, mx, sizeof(mx), cudaMemcpyHostToDevice, c.stream));
        launch_tstep_finish(c, time, target, clamp);
        HOW_CUDA_CHECK(cudaMemcpyAsync(c.hsc, c.dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c.stream));
    }
    int rc = sync_all(g);
    if (rc) return rc;
    *dt = g->parts[0]->hsc->dt;
    return HOW_OK;
}

// reference layout (v, i, j, k), k fastest
inline size_t ref_at(size_t P0, size_t P1, size_t P2, int v, int i, int j, int k) {
    return (((size_t)v * P0 + i) * P1 + j) * P2 + k;
}

}  // namespace

extern "C" {

int how_part_plan(int nz, int nparts, int periodic_z, int part, how_part_info* out) {
    if (!out || nparts < 1 || part < 0 || part >= nparts || nz < 3 * nparts) {
        set_error("no plan for part %d of %d over %d z planes (at least 3 planes per part)", part, nparts, nz);
        return HOW_ERR_ARG;
    }
    how_part_info r;
    r.kstart = 0;
    for (int p = 0; p < part; ++p) r.kstart += nz / nparts + (p < nz % nparts ? 1 : 0);
    r.nz = nz / nparts + (part < nz % nparts ? 1 : 0);
    if (nparts == 1) {
        r.z_sides = 3;
        r.lo_part = r.hi_part = -1;
    } else {
        r.z_sides = periodic_z ? 0 : ((part == 0 ? 1 : 0) | (part == nparts - 1 ? 2 : 0));
        r.lo_part = part > 0 ? part - 1 : (periodic_z ? nparts - 1 : -1);
        r.hi_part = part < nparts - 1 ? part + 1 : (periodic_z ? 0 : -1);
    }
    // the ghost fill's planes: the top three active planes n .. n+2 become
    // the upper neighbour's low ghosts 0..2, the bottom three 3..5 the lower
    // neighbour's high ghosts n+3 .. n+5 (src/bound.cpp:19-107 across parts)
    r.nplanes = 3;
    r.send_up_first = r.nz;
    r.recv_lo_first = 0;
    r.send_down_first = 3;
    r.recv_hi_first = r.nz + 3;
    *out = r;
    return HOW_OK;
}

int how_group_create(const how_params* global, int nparts, const int* devices, how_group** out) {
    if (!global || !out) { set_error("null argument"); return HOW_ERR_ARG; }
    *out = nullptr;
    how_params gp = *global;
    int rc = how_finalize_params(&gp);
    if (rc) return rc;
    if (nparts < 1) { set_error("group of %d parts", nparts); return HOW_ERR_ARG; }
    if (gp.nx < 2 || gp.ny < 2 || gp.nz < 3 * nparts) {
        set_error("a group needs a 3-D grid with at least 3 z planes per part (nx %d ny %d nz %d, %d parts)",
                  gp.nx, gp.ny, gp.nz, nparts);
        return HOW_ERR_ARG;
    }
    how_group* g = new (std::nothrow) how_group();
    if (!g) { set_error("out of host memory"); return HOW_ERR_ARG; }
    g->global = gp;
    g->n = nparts;
    g->periodic_z = gp.bc[2] == HOW_BC_PERIODIC;
    int cur = 0;
    cudaGetDevice(&cur);
    std::vector<how_part_info> plan(nparts);
    for (int p = 0; p < nparts; ++p) {
        how_part_plan(gp.nz, nparts, g->periodic_z, p, &plan[p]);
        g->kstart.push_back(plan[p].kstart);
        g->nzl.push_back(plan[p].nz);
        g->dev.push_back(devices ? devices[p] : cur);
    }
    for (int p = 0; p < nparts; ++p) {
        if ((rc = set_dev(g, p))) { how_group_destroy(g); return rc; }
        for (int q = 0; q < nparts; ++q) {
            if (g->dev[q] == g->dev[p]) continue;
            int ok = 0;
            cudaDeviceCanAccessPeer(&ok, g->dev[p], g->dev[q]);
            if (ok) {
                const cudaError_t e = cudaDeviceEnablePeerAccess(g->dev[q], 0);
                if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
            }
        }
        how_params pp = gp;
        pp.nz = g->nzl[p];
        how_ctx* c = nullptr;
        if ((rc = how_create(&pp, &c))) { how_group_destroy(g); return rc; }
        g->parts.push_back(c);
        // the part's cells have the global spacing (its own zsize / nz may
        // round differently)
        c->p.dz = gp.dz;
        c->part = p;
        c->kstart = g->kstart[p];
        c->gnz = gp.nz;
        c->z_sides = plan[p].z_sides;
        cudaEvent_t a = nullptr, b = nullptr;
        if (cudaEventCreateWithFlags(&a, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&b, cudaEventDisableTiming) != cudaSuccess) {
            how_group_destroy(g);
            return cuda_fail(cudaGetLastError(), "cudaEventCreate");
        }
        g->ready.push_back(a);
        g->done.push_back(b);
    }
    cudaSetDevice(cur);
    *out = g;
    return HOW_OK;
}

int how_group_destroy(how_group* g) {
    if (!g) return HOW_OK;
    for (size_t p = 0; p < g->parts.size(); ++p) {
        cudaSetDevice(g->dev[p]);
        how_destroy(g->parts[p]);
    }
    for (size_t p = 0; p < g->ready.size(); ++p) {
        cudaSetDevice(g->dev[p]);
        cudaEventDestroy(g->ready[p]);
        cudaEventDestroy(g->done[p]);
    }
    delete g;
    return HOW_OK;
}

int how_group_size(const how_group* g) { return g ? g->n : 0; }

how_ctx* how_group_part(how_group* g, int part) {
    return (g && part >= 0 && part < g->n) ? g->parts[part] : nullptr;
}

int how_group_part_range(const how_group* g, int part, int* kstart, int* nz) {
    if (!g || part < 0 || part >= g->n) { set_error("bad group or part"); return HOW_ERR_ARG; }
    if (kstart) *kstart = g->kstart[part];
    if (nz) *nz = g->nzl[part];
    return HOW_OK;
}

int how_group_set_state(how_group* g, const double* q) {
    if (!g || !q) { set_error("null argument"); return HOW_ERR_ARG; }
    const how_params& gp = g->global;
    const size_t P0 = gp.nx + 6, P1 = gp.ny + 6, P2 = gp.nz + 6;
    for (int p = 0; p < g->n; ++p) {
        const size_t L2 = (size_t)g->nzl[p] + 6;
        std::vector<double> loc(8 * P0 * P1 * L2);
        // global planes kstart .. kstart + nz + 5 are the part's 0 .. nz + 5
        for (int v = 0; v < 8; ++v)
            for (size_t i = 0; i < P0; ++i)
                for (size_t j = 0; j < P1; ++j)
                    std::memcpy(&loc[ref_at(P0, P1, L2, v, (int)i, (int)j, 0)],
                                &q[ref_at(P0, P1, P2, v, (int)i, (int)j, g->kstart[p])], L2 * sizeof(double));
        int rc = set_dev(g, p);
        if (!rc) rc = how_set_state(g->parts[p], 0, loc.data());
        if (rc) return rc;
    }
    // bound(q, 0) and initialize_bfield_from_q (src/main.cpp:127-130)
    int rc = bound_q(g, 0);
    if (rc) return rc;
    for (int p = 0; p < g->n; ++p) {
        if ((rc = set_dev(g, p))) return rc;
        launch_init_faceb(*g->parts[p]);
        g->parts[p]->have_state = true;
    }
    if ((rc = exchange_stage_b(g, 0))) return rc;
    return sync_all(g);
}

int how_group_init(how_group* g) {
    if (!g) { set_error("null group"); return HOW_ERR_ARG; }
    const how_params& gp = g->global;
    std::vector<double> q((size_t)8 * (gp.nx + 6) * (gp.ny + 6) * (gp.nz + 6), 0.0);
    int rc = how_problem_init_host(&gp, q.data());
    if (rc) return rc;
    return how_group_set_state(g, q.data());
}

int how_group_run(how_group* g, double* time, long max_steps, long* steps, double* dts, long dts_cap) {
    if (!g || !time || !steps) { set_error("null argument"); return HOW_ERR_ARG; }
    const how_params& gp = g->global;
    const double dtout = gp.tend / (double)gp.nt;
    long taken = 0;
    int rc = HOW_OK;
    // src/main.cpp:158-223
    for (int out_step = 1; out_step <= gp.nt && rc == HOW_OK; ++out_step) {
        const double target = dtout * (double)out_step;
        while (*time < target) {
            if (max_steps >= 0 && taken >= max_steps) { *steps += taken; return HOW_OK; }
            double dt = 0.0;
            if ((rc = tstep_all(g, *time, target, 1, &dt))) break;
            if (dt <= 0.0) {
                set_error("non-positive dt detected: time=%.17g target=%.17g dt=%.17g", *time, target, dt);
                rc = HOW_ERR_DT;
                break;
            }
            if ((rc = step(g))) break;
            *time += dt;
            if (dts && taken < dts_cap) dts[taken] = dt;
            ++taken;
            if (!std::isfinite(*time)) { set_error("time became non-finite"); rc = HOW_ERR_NONFINITE; break; }
        }
    }
    *steps += taken;
    if (rc) return rc;
    return sync_all(g);
}

int how_group_get_state(how_group* g, double* q) {
    if (!g || !q) { set_error("null argument"); return HOW_ERR_ARG; }
    const how_params& gp = g->global;
    const size_t P0 = gp.nx + 6, P1 = gp.ny + 6, P2 = gp.nz + 6;
    for (int p = 0; p < g->n; ++p) {
        const size_t L2 = (size_t)g->nzl[p] + 6;
        std::vector<double> loc(8 * P0 * P1 * L2);
        int rc = set_dev(g, p);
        if (!rc) rc = how_get_state(g->parts[p], 0, loc.data());
        if (rc) return rc;
        // active planes 3 .. nz + 2 of the part into the global array
        for (int v = 0; v < 8; ++v)
            for (size_t i = 0; i < P0; ++i)
                for (size_t j = 0; j < P1; ++j)
                    std::memcpy(&q[ref_at(P0, P1, P2, v, (int)i, (int)j, g->kstart[p] + 3)],
                                &loc[ref_at(P0, P1, L2, v, (int)i, (int)j, 3)], g->nzl[p] * sizeof(double));
    }
    return HOW_OK;
}

int how_group_output(how_group* g, int step, double time, const char* dir) {
    if (!g) { set_error("null group"); return HOW_ERR_ARG; }
    // every part writes its piece, named and headed as the reference's MPI
    // rank of the same slab writes it (src/output.cpp:21-38, 85-91, 383-402)
    for (int p = 0; p < g->n; ++p) {
        int rc = set_dev(g, p);
        if (!rc) rc = how_output(g->parts[p], step, time, dir);
        if (rc) return rc;
    }
    const std::string fmt = g->global.output_format;
    if (fmt != "vts" && fmt != "vtk") return HOW_OK;
    return write_pvts(g->global, g->n, g->kstart.data(), g->nzl.data(), step, dir);
}

int how_group_get_face_b(how_group* g, double* bx, double* by, double* bz) {
    if (!g || !bx || !by || !bz) { set_error("null argument"); return HOW_ERR_ARG; }
    const how_params& gp = g->global;
    const size_t P0 = gp.nx + 6, P1 = gp.ny + 6, P2 = gp.nz + 6;
    double* out[3] = {bx, by, bz};
    for (int p = 0; p < g->n; ++p) {
        const size_t L2 = (size_t)g->nzl[p] + 6;
        std::vector<double> b[3];
        for (auto& x : b) x.resize(P0 * P1 * L2);
        int rc = set_dev(g, p);
        if (!rc) rc = how_get_face_b(g->parts[p], 0, b[0].data(), b[1].data(), b[2].data());
        if (rc) return rc;
        for (int c = 0; c < 3; ++c)
            for (size_t i = 0; i < P0; ++i)
                for (size_t j = 0; j < P1; ++j)
                    std::memcpy(&out[c][ref_at(P0, P1, P2, 0, (int)i, (int)j, g->kstart[p] + 3)],
                                &b[c][ref_at(P0, P1, L2, 0, (int)i, (int)j, 3)], g->nzl[p] * sizeof(double));
    }
    return HOW_OK;
}

}  // extern "C"
