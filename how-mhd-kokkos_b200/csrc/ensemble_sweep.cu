// ensemble_sweep.cu -- the fused sweep over every member of a batched
// ensemble in one persistent launch, for each tile shape the autotuner may
// pick.  Member m's tiles occupy [tile_start[m], tile_start[m+1]) of the
// launch's tile space; each tile reads its member's arguments (geometry,
// stage pointers, TMA tensor maps, dt) from a device table.
#include "sweep_core.cuh"
#include "ensemble.cuh"

namespace how {

namespace {

// Candidate tile shapes (lines x active cells) per direction.  y/z lines are
// consecutive i from an even start, so NL is even there (16-byte TMA rule).
struct ShapeDef { int nl, t, minb; };
constexpr ShapeDef kShapes[3][kEnsShapes] = {
    {{1, 32, 4}, {1, 64, 2}, {2, 16, 4}},
    {{2, 16, 4}, {2, 32, 2}, {4, 8, 4}},
    {{2, 16, 4}, {2, 16, 4}, {2, 16, 4}},
};

template <int DIR, int NL, int T, int MINB>
void launch_ens(const SweepArgs& a0, cudaStream_t st, int dev) {
    using TL = Tile<DIR, NL, T, double>;
    constexpr size_t bytes = TL::bytes_plain + 128;
    auto kern = k_sweep<DIR, NL, T, 128, double, MINB, 0, true>;
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        attr_done = true;
    }
    int nsm = 148, occ = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 128, bytes);
    if (occ < 1) occ = 1;
    kern<<<nsm * occ, 128, bytes, st>>>(a0);
}

}  // namespace

void ens_shape(int dir, int s, int* nl, int* t) {
    *nl = kShapes[dir][s].nl;
    *t = kShapes[dir][s].t;
}

long long ens_tiles(const Grid& g, int dir, int s) {
    const int NL = kShapes[dir][s].nl, T = kShapes[dir][s].t;
    const int n = dir == 0 ? g.nx : dir == 1 ? g.ny : g.nz;
    if (n <= 1) return 0;
    const int nt1 = dir == 0 ? g.ny : g.nx;
    const int nt2 = dir == 2 ? g.ny : g.nz;
    const long long ntx = (n + T - 1) / T;
    const long long nty = dir == 0 ? (nt1 + NL - 1) / NL : (nt1 + 1 + NL - 1) / NL;
    return ntx * nty * nt2;
}

// Tensor maps of the 6 stage buffers of a context for shape s of direction dir.
int ens_encode_maps(const Ctx& c, int dir, int s, CUtensorMap* tm_in, CUtensorMap* tm_out) {
    const int NL = kShapes[dir][s].nl, T = kShapes[dir][s].t;
    const int C = T + 6, TO = dir == 0 ? T + 2 : T;
    const Grid& g = c.g;
    const uint64_t dims[4] = {(uint64_t)g.P0, (uint64_t)g.P1, (uint64_t)g.P2, 8};
    const uint64_t strides[3] = {(uint64_t)g.pitch * 8, (uint64_t)g.pitch * g.P1 * 8, (uint64_t)g.fs * 8};
    uint32_t bin[4], bout[4];
    if (dir == 0) { bin[0] = C; bin[1] = NL; bin[2] = 1; bout[0] = TO; bout[1] = NL; bout[2] = 1; }
    else if (dir == 1) { bin[0] = NL; bin[1] = C; bin[2] = 1; bout[0] = NL; bout[1] = TO; bout[2] = 1; }
    else { bin[0] = NL; bin[1] = 1; bin[2] = C; bout[0] = NL; bout[1] = 1; bout[2] = TO; }
    bin[3] = 8; bout[3] = 8;
    for (int b = 0; b < 6; ++b) {
        int rc = encode_tensor_map_4d(&tm_in[b], c.qbuf[b], dims, strides, bin);
        if (!rc) rc = encode_tensor_map_4d(&tm_out[b], c.qbuf[b], dims, strides, bout);
        if (rc) return rc;
    }
    return 0;
}

void ens_launch_sweep(int dir, int s, const SweepArgs& a0, cudaStream_t st, int dev) {
#define HOW_ENS_CASE(D, S)                                                                             \
    if (dir == D && s == S) {                                                                          \
        launch_ens<D, kShapes[D][S].nl, kShapes[D][S].t, kShapes[D][S].minb>(a0, st, dev);             \
        return;                                                                                        \
    }
    HOW_ENS_CASE(0, 0) HOW_ENS_CASE(0, 1) HOW_ENS_CASE(0, 2)
    HOW_ENS_CASE(1, 0) HOW_ENS_CASE(1, 1) HOW_ENS_CASE(1, 2)
    if (dir == 2) launch_ens<2, kShapes[2][0].nl, kShapes[2][0].t, kShapes[2][0].minb>(a0, st, dev);
#undef HOW_ENS_CASE
}

}  // namespace how
