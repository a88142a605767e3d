// route_prepass.cu -- the learned router's decisions for every interface of a
// sweep, computed before the sweep in one batched pass.
//
// The routing values of each interface's 6 stencil cells come from the stage
// input (the sweep's primitive floors; fast speed along the sweep normal),
// then the 6 features and the guard (router.cuh); a warp's 32 interfaces are
// two 16-row groups of the BF16 tensor-core network.  Groups whose stencils
// are all uniform take the precomputed logit of a flat stencil.
// The decision (1: full characteristic WENO) lands in the per-face byte array
// the sweep reads and the next stage's prior comes from.
#include "how_internal.cuh"
#include "router.cuh"

namespace how {

namespace {

__device__ __forceinline__ int route_perm(int dir, int v) {
    // line variable v -> conserved index (x: identity; y: rho,My,Mz,Mx,By,Bz,Bx,E;
    // z: rho,Mz,Mx,My,Bz,Bx,By,E), the sweeps' order
    return dir == 0 ? v
         : dir == 1 ? (v == 1 ? 2 : v == 2 ? 3 : v == 3 ? 1 : v == 4 ? 5 : v == 5 ? 6 : v == 6 ? 4 : v)
                    : (v == 1 ? 3 : v == 2 ? 1 : v == 3 ? 2 : v == 4 ? 6 : v == 5 ? 4 : v == 6 ? 5 : v);
}

struct RouteArgs {
    Grid g;
    const double* q;            // stage input, field 0 (var v at + v * fs)
    const unsigned char* prev;  // previous decisions of this direction (the prior)
    unsigned char* next;        // this sweep's decisions
    const float* w;             // network (RouterLayout)
    float thr, guard_jump, guard_floor;
    double gam, rhomin, pgmin;
    unsigned long long* groups; // [0] tensor-core groups, [1] flat groups (may be null)
};

constexpr int kRouteThreads = 256;

// Routing values of one cell: floored density and pressure (the sweep's
// primit floors, src/ssprk.cpp:479-512), |B|, |v| and the fast speed along
// the sweep normal.  Density, velocity and pressure in FP64 (one division);
// the square roots of the fast speed in FP32, which is all the features keep.
__device__ __forceinline__ StencilCell route_cell(const double* q, long long fs, long long c, int dir, double gam,
                                                  double rhomin, double pgmin) {
    const double DD = q[c];
    const double Mx = q[route_perm(dir, 1) * fs + c], My = q[route_perm(dir, 2) * fs + c];
    const double Mz = q[route_perm(dir, 3) * fs + c];
    const double Bx = q[route_perm(dir, 4) * fs + c], By = q[route_perm(dir, 5) * fs + c];
    const double Bz = q[route_perm(dir, 6) * fs + c];
    const double EE = q[7 * fs + c];
    const double irho0 = 1.0 / DD;
    const double vx = Mx * irho0, vy = My * irho0, vz = Mz * irho0;
    const double vv2 = vx * vx + vy * vy + vz * vz;
    const double BB2 = Bx * Bx + By * By + Bz * Bz;
    const double pg = fmax(pgmin, (gam - 1.0) * (EE - 0.5 * (DD * vv2 + BB2)));
    const double rho = fmax(rhomin, DD);
    const float irho = 1.0f / (float)rho;
    const float bbn2 = (float)BB2 * irho, bnx2 = (float)(Bx * Bx) * irho;
    const float cs2 = fmaxf(0.0f, (float)gam * fabsf((float)pg * irho));
    const float root = sqrtf(fmaxf(0.0f, (bbn2 + cs2) * (bbn2 + cs2) - 4.0f * bnx2 * cs2));
    const float lf = sqrtf(fmaxf(0.0f, 0.5f * (bbn2 + cs2 + root)));
    return StencilCell{(float)rho, (float)pg, sqrtf((float)BB2), sqrtf((float)vv2), lf};
}

// A warp's 32 interfaces as two 16-row groups of the network: features to the
// BF16 operand rows, the tensor-core logits (or the flat logit of a group of
// uniform stencils), the decision.  Every lane of the warp calls this.
struct RouteShared {
    RouterSmem rs;
    __align__(16) __nv_bfloat16 X[kRouteThreads / 32][32][16];
    float lg[kRouteThreads / 32][32];
    float flat_logit[2];
    unsigned int cnt[2];
};

__device__ __forceinline__ void route_decide(RouteShared& S, const RouteArgs& a, int warp, int lane,
                                             const float* ft, bool flat, bool guard, bool live, long long face) {
    uint4 v0;
    v0.x = pack_bf16(ft[0], ft[1]); v0.y = pack_bf16(ft[2], ft[3]);
    v0.z = pack_bf16(ft[4], ft[5]); v0.w = 0u;
    reinterpret_cast<uint4*>(&S.X[warp][lane][0])[0] = v0;
    reinterpret_cast<uint4*>(&S.X[warp][lane][0])[1] = make_uint4(0u, 0u, 0u, 0u);
    // 0: needs the network; 1 + prior: uniform stencil (flat logit);
    // 3: guarded or no face (decided without a logit)
    const int code = (guard || !live) ? 3 : flat ? 1 + (ft[5] > 0.5f ? 1 : 0) : 0;
    __syncwarp();
    float logit = 0.0f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const unsigned int needs = __ballot_sync(0xffffffffu, code == 0);
        const unsigned int half = h == 0 ? 0x0000ffffu : 0xffff0000u;
        if ((needs & half) == 0u) {
            if ((lane >> 4) == h && code < 3) logit = S.flat_logit[code - 1];
            if (lane == 0) atomicAdd(&S.cnt[1], 1u);
        } else {
            router_mma_16rows(&S.rs, S.X[warp] + 16 * h, S.lg[warp] + 16 * h);
            __syncwarp();
            if ((lane >> 4) == h) logit = S.lg[warp][lane];
            if (lane == 0) atomicAdd(&S.cnt[0], 1u);
        }
    }
    if (live) a.next[face] = (guard || logit > a.thr) ? 1 : 0;
    __syncwarp();
}

// The network in shared memory and the logits of a uniform stencil with prior
// 0 and 1, through the same code as every face (runtime cell values).
__device__ __forceinline__ void route_setup(RouteShared& S, const RouteArgs& a) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    router_load_smem(&S.rs, a.w, tid, blockDim.x);
    if (tid < 2) S.cnt[tid] = 0u;
    __syncthreads();
    if (warp == 0) {
        StencilCell sc[6];
        const float u = (float)a.gam;
        for (int k = 0; k < 6; ++k) sc[k] = StencilCell{u, u, u, u, u};
        float ff[kRouterNF];
        bool flat;
        router_features(sc, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, ff, &flat);
        for (int e = lane; e < 256; e += 32) {
            const int r = e / 16, k = e % 16;
            S.X[0][r][k] = __float2bfloat16_rn(k < 5 ? ff[k] : k == 5 ? (float)(r & 1) : 0.0f);
        }
        __syncwarp();
        router_mma_16rows(&S.rs, S.X[0], S.lg[0]);
        __syncwarp();
        if (lane < 2) S.flat_logit[lane] = S.lg[0][lane];
    }
    __syncthreads();
}

__device__ __forceinline__ void route_finish(RouteShared& S, const RouteArgs& a) {
    __syncthreads();
    if (threadIdx.x == 0 && a.groups) {
        atomicAdd(&a.groups[0], (unsigned long long)S.cnt[0]);
        atomicAdd(&a.groups[1], (unsigned long long)S.cnt[1]);
    }
}

// x sweeps: a warp takes 32 consecutive faces of one line; its lanes form
// the values of 37 consecutive cells (coalesced along x) into shared memory
// and each lane reads its face's 6.
// (four blocks per SM: 63 registers without spills; the y/z kernels would spill)
__global__ void __launch_bounds__(kRouteThreads, 4) k_route_x(const __grid_constant__ RouteArgs a) {
    __shared__ RouteShared S;
    __shared__ float cv[kRouteThreads / 32][37][5];
    route_setup(S, a);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Grid& g = a.g;
    const int n = g.nx;
    const int nseg = (n + 1 + 31) / 32;
    const long long nwork = (long long)g.ny * g.nz * nseg;   // (segment, line)
    const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long wi = (long long)blockIdx.x * (blockDim.x >> 5) + warp; wi < nwork; wi += wstride) {
        const int seg = (int)(wi % nseg);
        const long long ln = wi / nseg;
        const int lj = 3 + (int)(ln % g.ny), lk = 3 + (int)(ln / g.ny);
        const long long line = g.idx(0, lj, lk);
        const long long rl = route_line(g, 0, lj, lk);   // the line in the per-face arrays
        const int f0 = seg * 32;
        for (int k = lane; k < 37; k += 32) {
            const int s = f0 + k;   // padded cell index
            StencilCell v = StencilCell{0.f, 0.f, 0.f, 0.f, 0.f};
            if (s <= n + 5) v = route_cell(a.q, g.fs, line + s, 0, a.gam, a.rhomin, a.pgmin);
            cv[warp][k][0] = v.rho; cv[warp][k][1] = v.p; cv[warp][k][2] = v.bmag;
            cv[warp][k][3] = v.vmag; cv[warp][k][4] = v.cf;
        }
        __syncwarp();
        const int iface = f0 + lane;
        const bool live = iface <= n;
        float ft[kRouterNF] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        bool flat = true, guard = false;
        const long long face = rl + iface + 2;
        if (live) {
            StencilCell sc[6];
#pragma unroll
            for (int k = 0; k < 6; ++k)
                sc[k] = StencilCell{cv[warp][lane + k][0], cv[warp][lane + k][1], cv[warp][lane + k][2],
                                    cv[warp][lane + k][3], cv[warp][lane + k][4]};
            guard = router_features(sc, 0.0f /* prior-stage feature held at 0 */, (float)a.rhomin, (float)a.pgmin, a.guard_jump,
                                    a.guard_floor, ft, &flat);
        }
        route_decide(S, a, warp, lane, ft, flat, guard, live, face);
    }
    route_finish(S, a);
}

// y/z sweeps: each thread walks one segment of kSeg interfaces of one line
// along the sweep direction with a sliding window of its 6 stencil cells, so
// every cell's routing values are formed once per segment (kSeg + 5 cells for
// kSeg faces); lanes of a warp hold x-adjacent lines (coalesced loads), and at
// every step the warp's 32 interfaces are two 16-row groups of the network.
constexpr int kSeg = 32;

// y and z sweeps (see above): sliding windows along the sweep direction.
template <int DIR>
__global__ void __launch_bounds__(kRouteThreads) k_route(const __grid_constant__ RouteArgs a) {
    __shared__ RouteShared S;
    route_setup(S, a);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Grid& g = a.g;
    const int n = DIR == 1 ? g.ny : g.nz;
    const long long stride = DIR == 1 ? (long long)g.pitch : (long long)g.pitch * g.P1;
    // lines: DIR 1 (i, k); DIR 2 (i, j) -- i fastest
    const int la = g.nx;
    const int lb = DIR == 2 ? g.ny : g.nz;
    const long long nlines = (long long)la * lb;
    const int nseg = (n + 1 + kSeg - 1) / kSeg;
    const long long nwork = nlines * nseg;   // (segment, line), line fastest
    for (long long base = (long long)blockIdx.x * blockDim.x; base < nwork; base += (long long)gridDim.x * blockDim.x) {
        const long long widx = base + tid;
        const bool valid = widx < nwork;
        long long line = 0, rl = 0;
        int f0 = 0;
        if (valid) {
            const long long ln = widx % nlines;
            f0 = (int)(widx / nlines) * kSeg;
            const int ia = (int)(ln % la), ib = (int)(ln / la);
            line = DIR == 1 ? g.idx(3 + ia, 0, 3 + ib) : g.idx(3 + ia, 3 + ib, 0);
            rl = route_line(g, DIR, 3 + ia, 3 + ib);   // the line in the per-face arrays
        }
        // window: stencil cells f .. f+5 of face f (padded cells)
        StencilCell win[6];
        if (valid) {
#pragma unroll
            for (int k = 0; k < 5; ++k)
                win[k] = route_cell(a.q, g.fs, line + (long long)(f0 + k) * stride, DIR, a.gam, a.rhomin, a.pgmin);
        }
        for (int s = 0; s < kSeg; ++s) {
            const int iface = f0 + s;
            const bool live = valid && iface <= n;
            float ft[kRouterNF] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            bool flat = true, guard = false;
            const long long face = rl + iface + 2;
            if (live) {
                win[5] = route_cell(a.q, g.fs, line + (long long)(iface + 5) * stride, DIR, a.gam, a.rhomin, a.pgmin);
                guard = router_features(win, 0.0f /* prior-stage feature held at 0 */, (float)a.rhomin, (float)a.pgmin, a.guard_jump,
                                        a.guard_floor, ft, &flat);
#pragma unroll
                for (int k = 0; k < 5; ++k) win[k] = win[k + 1];
            }
            // every lane of the warp reaches here kSeg times (uniform trip count)
            route_decide(S, a, warp, lane, ft, flat, guard, live, face);
        }
    }
    route_finish(S, a);
}

}  // namespace

// Decisions of sweep `dir` over stage input q into c.route_prev's write half.
void launch_route(Ctx& c, int dir, const double* q, const unsigned char* prev, unsigned char* next) {
    RouteArgs a;
    a.g = c.g;
    a.q = q;
    a.prev = prev;
    a.next = next;
    a.w = c.router_w;
    a.thr = c.route_thr;
    a.guard_jump = c.guard_jump;
    a.guard_floor = c.guard_floor;
    a.gam = c.p.gam;
    a.rhomin = c.p.rhomin;
    a.pgmin = c.p.pgmin;
    a.groups = c.route_count ? c.route_count + 2 : nullptr;
    const Grid& g = c.g;
    const int n = dir == 0 ? g.nx : dir == 1 ? g.ny : g.nz;
    const long long nlines = dir == 0 ? (long long)g.ny * g.nz : dir == 1 ? (long long)g.nx * g.nz
                                                                        : (long long)g.nx * g.ny;
    // x: one warp per (32-face segment, line); y/z: one thread per (kSeg-face segment, line)
    const long long nwork = dir == 0 ? nlines * ((n + 1 + 31) / 32) * 32 : nlines * ((n + 1 + kSeg - 1) / kSeg);
    long long blocks = (nwork + kRouteThreads - 1) / kRouteThreads;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.dev);
    if (blocks > (long long)nsm * 8) blocks = (long long)nsm * 8;
    if (blocks < 1) blocks = 1;
    if (dir == 0) k_route_x<<<(unsigned)blocks, kRouteThreads, 0, c.stream>>>(a);
    else if (dir == 1) k_route<1><<<(unsigned)blocks, kRouteThreads, 0, c.stream>>>(a);
    else k_route<2><<<(unsigned)blocks, kRouteThreads, 0, c.stream>>>(a);
    ++c.launches;
}

}  // namespace how
