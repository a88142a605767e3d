// sweep_kernels.cu -- single-domain launches of the fused directional sweep
// (sweep_core.cuh): tile shapes, TMA tensor maps and the instantiations for
// {FP64, mixed} x {plain, learned routing, guard-only routing, label
// collection}.
#include "sweep_core.cuh"

namespace how {

namespace {

template <int DIR, int NL, int T, int NT, typename R, int MINB, int MODE>
void launch_one(Ctx& c, const SweepArgs& a) {
    using TL = Tile<DIR, NL, T, R>;
    constexpr size_t bytes = (MODE == 0 ? TL::bytes_plain : MODE == 1 ? TL::bytes_learned : TL::bytes_route) + 128;
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(k_sweep<DIR, NL, T, NT, R, MINB, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bytes);
        attr_done = true;
    }
    const Grid& g = c.g;
    const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
    const int nt1 = DIR == 0 ? g.ny : g.nx;
    const int nt2 = DIR == 2 ? g.ny : g.nz;
    const long long ntx = (n + T - 1) / T;
    const long long nty = DIR == 0 ? (nt1 + NL - 1) / NL : (nt1 + 1 + NL - 1) / NL;
    const long long ntiles = ntx * nty * nt2;
    int nsm = 148, occ = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.dev);
    // persistent grid: exactly the blocks that are resident at once
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sweep<DIR, NL, T, NT, R, MINB, MODE>, NT, bytes);
    if (occ < 1) occ = 1;
    const long long resident = (long long)nsm * occ;
    const int grid = (int)(ntiles < resident ? ntiles : resident);
    cudaEvent_t ev[2];
    timer_begin(c, ev);
    k_sweep<DIR, NL, T, NT, R, MINB, MODE><<<grid, NT, bytes, c.stream>>>(a);
    timer_end(c, ev);
    ++c.launches;
}

}  // namespace

// Sweep tile shapes: x sweeps 1 line x 32 cells, y/z sweeps 2 lines x 16 cells.
template <int DIR> struct SweepShape;
template <> struct SweepShape<0> { static constexpr int NL = 1, T = 32; };
template <> struct SweepShape<1> { static constexpr int NL = 2, T = 16; };
template <> struct SweepShape<2> { static constexpr int NL = 2, T = 16; };

template <int DIR>
static int make_maps_dir(Ctx& c) {
    using S = SweepShape<DIR>;
    using TL = Tile<DIR, S::NL, S::T, double>;   // the TMA boxes do not depend on R
    const Grid& g = c.g;
    const uint64_t dims[4] = {(uint64_t)g.P0, (uint64_t)g.P1, (uint64_t)g.P2, 8};
    const uint64_t strides[3] = {(uint64_t)g.pitch * 8, (uint64_t)g.pitch * g.P1 * 8, (uint64_t)g.fs * 8};
    uint32_t bin[4], bout[4];
    if (DIR == 0) { bin[0] = TL::C; bin[1] = S::NL; bin[2] = 1; bout[0] = TL::TO; bout[1] = S::NL; bout[2] = 1; }
    else if (DIR == 1) { bin[0] = S::NL; bin[1] = TL::C; bin[2] = 1; bout[0] = S::NL; bout[1] = TL::TO; bout[2] = 1; }
    else { bin[0] = S::NL; bin[1] = 1; bin[2] = TL::C; bout[0] = S::NL; bout[1] = 1; bout[2] = TL::TO; }
    bin[3] = 8; bout[3] = 8;
    for (int b = 0; b < 6; ++b) {
        int rc = encode_tensor_map_4d(&c.tm_in[b][DIR], c.qbuf[b], dims, strides, bin);
        if (!rc) rc = encode_tensor_map_4d(&c.tm_out[b][DIR], c.qbuf[b], dims, strides, bout);
        if (rc) return rc;
    }
    return 0;
}

int make_sweep_tensor_maps(Ctx& c) {
    int rc = make_maps_dir<0>(c);
    if (!rc) rc = make_maps_dir<1>(c);
    if (!rc) rc = make_maps_dir<2>(c);
    return rc;
}

static int buffer_of(const Ctx& c, const double* p) {
    for (int b = 0; b < 6; ++b) if (c.qbuf[b] == p) return b;
    return -1;
}

// a.qprev / a.qout / a.q0 choose the tensor maps: the tile comes from qprev;
// the update operand is q(iw) when accumulating (mode 0) or when the base was
// prepared in q(iw) (stage 5), else q(0).
void launch_sweep(Ctx& c, int dir, const SweepArgs& a_in) {
    SweepArgs a = a_in;
    a.prof = c.prof;
    a.status = &c.dsc->status;
    const int bin = buffer_of(c, a.qprev);
    const int bout = buffer_of(c, (a.mode == 0 || a.stage5) ? a.qout : a.q0);
    a.tm_in = c.tm_in[bin][dir];
    a.tm_out = c.tm_out[bout][dir];
    a.router = c.router_w;
    a.route_prev = c.route_prev ? c.route_prev + (size_t)(2 * dir + c.route_par[dir]) * c.g.fs : nullptr;
    a.route_next = c.route_prev ? c.route_prev + (size_t)(2 * dir + 1 - c.route_par[dir]) * c.g.fs : nullptr;
    a.route_count = c.route_count;
    a.collect = c.collect;
    a.collect_n = c.collect_n;
    a.collect_cap = c.collect_cap;
    a.collect_every = c.collect_every > 0 ? c.collect_every : 1;
    a.route_thr = c.route_thr;
    a.guard_jump = c.guard_jump;
    a.guard_floor = c.guard_floor;
    a.ct4 = c.p.ct_avg == 4;
    a.wait_expire = c.wait_expire;
    const bool mixed = c.precision == HOW_PREC_MIXED;
    const int mode = c.route_mode;
    if (mode == 1) {
        // learned routing: the routing pass forms fresh decisions (on the
        // stages stage_sweeps marks due) into the other half of this
        // direction's pair, which then becomes the current one; the sweep
        // reads the current decisions
        if (c.route_due) {
            launch_route(c, dir, a.qprev, a.route_prev, a.route_next);
            c.route_par[dir] ^= 1;
        }
        a.route_next = c.route_prev + (size_t)(2 * dir + c.route_par[dir]) * c.g.fs;
        a.route_prev = nullptr;
    }
    // instantiations: {fp64, mixed} x {plain, learned, guard-only}; label
    // collection runs the FP64 method
    // Blocks per SM (the launch bound that caps registers): six for the plain
    // FP64 sweep (80 registers, one interface per thread in P3), seven for
    // the learned one (72 registers), six for the plain mixed one (80
    // registers, no spills); measured at 256^3 against 4/5 and 6/8 (FP64),
    // 6 (learned) and 7 (plain mixed).
#define HOW_SWEEP_CASES(D)                                                                              \
    do {                                                                                                \
        using S = SweepShape<D>;                                                                        \
        if (mode == 3) { launch_one<D, S::NL, S::T, 128, double, 3, 3>(c, a); break; }                  \
        if (mixed) {                                                                                    \
            if (mode == 1) launch_one<D, S::NL, S::T, 128, float, 7, 1>(c, a);                          \
            else if (mode == 2) launch_one<D, S::NL, S::T, 128, float, 5, 2>(c, a);                     \
            else launch_one<D, S::NL, S::T, 128, float, 6, 0>(c, a);                                    \
        } else {                                                                                        \
            if (mode == 1) launch_one<D, S::NL, S::T, 128, double, 3, 1>(c, a);                         \
            else if (mode == 2) launch_one<D, S::NL, S::T, 128, double, 3, 2>(c, a);                    \
            else launch_one<D, S::NL, S::T, 128, double, 6, 0>(c, a);                                   \
        }                                                                                               \
    } while (0)
    if (dir == 0) HOW_SWEEP_CASES(0);
    else if (dir == 1) HOW_SWEEP_CASES(1);
    else HOW_SWEEP_CASES(2);
    if (mode == 2 || mode == 3) {
        // guard-only routing and label collection write the decision arrays
        c.route_par[dir] ^= 1;
        c.route_valid = false;
    }
#undef HOW_SWEEP_CASES
}

}  // namespace how
