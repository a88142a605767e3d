// instrument.cu -- measurement hooks: CUDA-event timing of the sweep kernels
// inside a running step, and an FP64 FMA-pipe throughput probe that gives the
// roofline denominator for this FP64-bound path.
#include "how_internal.cuh"

#include <vector>

namespace how {

struct TimerPool {
    std::vector<cudaEvent_t> ev;   // pairs
    size_t used = 0;
    bool on = false;
};

static TimerPool& pool(Ctx& c) {
    static thread_local std::vector<std::pair<Ctx*, TimerPool>> pools;
    for (auto& p : pools) if (p.first == &c) return p.second;
    pools.push_back({&c, TimerPool{}});
    return pools.back().second;
}

void timer_begin(Ctx& c, cudaEvent_t* pair_out) {
    TimerPool& tp = pool(c);
    pair_out[0] = pair_out[1] = nullptr;
    if (!tp.on) return;
    if (tp.used + 2 > tp.ev.size()) {
        for (int k = 0; k < 64; ++k) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return;
            tp.ev.push_back(e);
        }
    }
    pair_out[0] = tp.ev[tp.used];
    pair_out[1] = tp.ev[tp.used + 1];
    tp.used += 2;
    cudaEventRecord(pair_out[0], c.stream);
}

void timer_end(Ctx& c, cudaEvent_t* pair) {
    if (pair[1]) cudaEventRecord(pair[1], c.stream);
}

namespace {

// Eight independent FMA chains per thread keep the FP64 pipe saturated.
__global__ void k_fp64_fma(double* out, int iters, double a, double b) {
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
    double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1.2345678) out[blockIdx.x] = s;   // keeps the chains live
}

}  // namespace
}  // namespace how

using namespace how;

extern "C" {

// Enable/disable event timing of sweep launches; enabling clears the record.
int how_set_kernel_timing(how_ctx* cp, int on) {
    Ctx* c = cp;
    if (!c) return HOW_ERR_ARG;
    TimerPool& tp = pool(*c);
    tp.on = on != 0;
    tp.used = 0;
    return HOW_OK;
}

// Sum of the device durations (ms) and count of the sweep launches timed
// since timing was enabled.  Synchronises the context's stream.
int how_get_kernel_timing(how_ctx* cp, double* total_ms, long* launches) {
    Ctx* c = cp;
    if (!c || !total_ms || !launches) return HOW_ERR_ARG;
    HOW_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    TimerPool& tp = pool(*c);
    double tot = 0.0;
    for (size_t k = 0; k + 1 < tp.used; k += 2) {
        float ms = 0.f;
        HOW_CUDA_CHECK(cudaEventElapsedTime(&ms, tp.ev[k], tp.ev[k + 1]));
        tot += ms;
    }
    *total_ms = tot;
    *launches = (long)(tp.used / 2);
    return HOW_OK;
}

// Per-phase cycle accounting of one directional sweep of stage 1 (the
// how_sweep semantics): out[k] = mean cycles per block spent in phase k
// (0 load, 1 primitives/centre, 2 differences + interface scalars,
// 3 eigenvector rows, 4 projection + WENO, 5 back-projection + CT,
// 6 update), measured by thread 0 of each block with clock64.
int how_sweep_phase_profile(how_ctx* cp, int dir, double dt, double* out, int nout) {
    Ctx* c = cp;
    if (!c || !out) return HOW_ERR_ARG;
    unsigned long long* d = nullptr;
    HOW_CUDA_CHECK(cudaMalloc(&d, 12 * sizeof(unsigned long long)));
    HOW_CUDA_CHECK(cudaMemset(d, 0, 12 * sizeof(unsigned long long)));
    c->prof = d;
    const int rc = how_sweep(cp, dir, dt);
    c->prof = nullptr;
    unsigned long long h[12] = {0};
    cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (rc) return rc;
    for (int k = 0; k < nout && k < 12; ++k)
        out[k] = k < 11 ? (h[11] ? (double)h[k] / (double)h[11] : 0.0) : (double)h[11];
    return HOW_OK;
}

// Measured FP64 FMA throughput of the current device in TFLOP/s (2 flops per
// FMA), best of `reps` launches of 8 independent FMA chains per thread.
int how_measure_fp64_peak(double* tflops, int reps) {
    if (!tflops) return HOW_ERR_ARG;
    int dev = 0, nsm = 0;
    HOW_CUDA_CHECK(cudaGetDevice(&dev));
    HOW_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    double* out = nullptr;
    HOW_CUDA_CHECK(cudaMalloc(&out, sizeof(double) * nsm * 8));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = nsm * 8, threads = 256, iters = 2048;
    k_fp64_fma<<<blocks, threads>>>(out, 64, 1.0000001, 1e-7);   // warm-up
    double best = 0.0;
    for (int r = 0; r < (reps > 0 ? reps : 5); ++r) {
        cudaEventRecord(e0);
        k_fp64_fma<<<blocks, threads>>>(out, iters, 1.0000001, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        const double tf = flops / (ms * 1e-3) / 1e12;
        if (tf > best) best = tf;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    HOW_CUDA_CHECK(cudaGetLastError());
    *tflops = best;
    return HOW_OK;
}

}  // extern "C"
