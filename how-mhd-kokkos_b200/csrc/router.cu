// router.cu -- training and batched inference of the learned WENO router
// (router.cuh holds the network, the features and the BF16 tensor-core
// inference used inside the sweep kernel).
//
// Training is FP32 and hand-written: per sample, the forward pass and the
// backward pass down to the layer activations (k_fwd_bwd); per weight, the
// gradient as a deterministic reduction over the batch (k_grad_reduce);
// Adam (k_adam).  Loss: binary cross-entropy on the logit, with positives
// (interfaces whose nonlinear WENO weights depart from the linear ones)
// weighted by pos_weight.
#include "how_internal.cuh"
#include "router.cuh"
#include "router_default.inc"

#include <cmath>
#include <cstring>
#include <vector>

namespace how {
namespace {

constexpr int H = kRouterH, NF = kRouterNF;
constexpr int NW = RouterLayout::total;   // 1313 parameters
constexpr int ACT = NF + 4 * H + 2;       // per-sample record: x, z1, h1, dz2, h2, dlogit, loss

// per sample: forward, loss, backward to activations.  act[s] = {x[6], dz1[32],
// h1[32], dz2[32], h2[32], dlogit, loss}
__global__ void k_fwd_bwd(const float* __restrict__ w, const float* __restrict__ feats,
                          const float* __restrict__ labels, const int* __restrict__ idx, int nb,
                          float pos_weight, float inv_norm, float* __restrict__ act) {
    __shared__ float sw[NW];
    for (int t = threadIdx.x; t < NW; t += blockDim.x) sw[t] = w[t];
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nb) return;
    const int src = idx ? idx[s] : s;
    const float* W1 = sw + RouterLayout::oW1;
    const float* b1 = sw + RouterLayout::ob1;
    const float* W2 = sw + RouterLayout::oW2;
    const float* b2 = sw + RouterLayout::ob2;
    const float* w3 = sw + RouterLayout::ow3;
    float x[NF];
#pragma unroll
    for (int i = 0; i < NF; ++i) x[i] = feats[(size_t)src * NF + i];
    const float y = labels[src];
    float z1[H], h1[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        float a = b1[j];
#pragma unroll
        for (int i = 0; i < NF; ++i) a += W1[j * NF + i] * x[i];
        z1[j] = a;
        h1[j] = gelu_tanh(a);
    }
    float z2[H], logit = sw[RouterLayout::ob3];
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
        float a = b2[j];
#pragma unroll
        for (int i = 0; i < H; ++i) a += W2[j * H + i] * h1[i];
        z2[j] = a;
        logit += w3[j] * gelu_tanh(a);
    }
    // weighted BCE with logits: pw y log(1+e^-z) + (1-y) log(1+e^z)
    const float sp_pos = logit > 0.f ? log1pf(expf(-logit)) : -logit + log1pf(expf(logit));
    const float sp_neg = sp_pos + logit;
    const float loss = pos_weight * y * sp_pos + (1.0f - y) * sp_neg;
    const float sig = 1.0f / (1.0f + expf(-logit));
    const float dlogit = (pos_weight * y * (sig - 1.0f) + (1.0f - y) * sig) * inv_norm;
    float* A = act + (size_t)s * ACT;
#pragma unroll
    for (int i = 0; i < NF; ++i) A[i] = x[i];
    float dh1[H];
#pragma unroll
    for (int i = 0; i < H; ++i) dh1[i] = 0.f;
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
        const float dz2 = dlogit * w3[j] * gelu_tanh_grad(z2[j]);
        A[NF + 2 * H + j] = dz2;
        A[NF + 3 * H + j] = gelu_tanh(z2[j]);
#pragma unroll
        for (int i = 0; i < H; ++i) dh1[i] += W2[j * H + i] * dz2;
    }
#pragma unroll
    for (int j = 0; j < H; ++j) {
        A[NF + j] = dh1[j] * gelu_tanh_grad(z1[j]);   // dz1
        A[NF + H + j] = h1[j];
    }
    A[NF + 4 * H] = dlogit;
    A[NF + 4 * H + 1] = loss * inv_norm;
}

// one block per parameter: gradient = sum over the batch, fixed order
__global__ void k_grad_reduce(const float* __restrict__ act, int nb, float* __restrict__ grad, float* loss_out) {
    const int p = blockIdx.x;   // parameter index in RouterLayout, or NW for the loss
    float acc = 0.f;
    for (int s = threadIdx.x; s < nb; s += blockDim.x) {
        const float* A = act + (size_t)s * ACT;
        float v;
        if (p < RouterLayout::ob1) { const int j = p / NF, i = p % NF; v = A[NF + j] * A[i]; }
        else if (p < RouterLayout::oW2) v = A[NF + (p - RouterLayout::ob1)];
        else if (p < RouterLayout::ob2) { const int q = p - RouterLayout::oW2, j = q / H, i = q % H; v = A[NF + 2 * H + j] * A[NF + H + i]; }
        else if (p < RouterLayout::ow3) v = A[NF + 2 * H + (p - RouterLayout::ob2)];
        else if (p < RouterLayout::ob3) v = A[NF + 4 * H] * A[NF + 3 * H + (p - RouterLayout::ow3)];
        else if (p == RouterLayout::ob3) v = A[NF + 4 * H];
        else v = A[NF + 4 * H + 1];
        acc += v;
    }
    __shared__ float red[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        if (p < NW) grad[p] = t; else *loss_out = t;
    }
}

__global__ void k_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                       float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

__global__ void k_infer_fp32(const float* __restrict__ w, const float* __restrict__ feats, long n,
                             float* __restrict__ out) {
    const long s = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[NF];
    for (int i = 0; i < NF; ++i) x[i] = feats[s * NF + i];
    out[s] = router_logit_fp32(w, x);
}

// the sweep kernel's tensor-core path on a batch: 16 rows per warp pass
__global__ void k_infer_mma(const float* __restrict__ w, const float* __restrict__ feats, long n,
                            float* __restrict__ out) {
    __shared__ RouterSmem rs;
    __shared__ __nv_bfloat16 X[4][16][16];
    __shared__ float lg[4][16];
    router_load_smem(&rs, w, threadIdx.x, blockDim.x);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long row0 = (blockIdx.x * 4 + warp) * 16l;
    for (int e = lane; e < 256; e += 32) {
        const int r = e / 16, k = e % 16;
        const long s = row0 + r;
        X[warp][r][k] = __float2bfloat16_rn((k < NF && s < n) ? feats[s * NF + k] : 0.0f);
    }
    __syncwarp();
    router_mma_16rows(&rs, X[warp], lg[warp]);
    __syncwarp();
    if (lane < 16 && row0 + lane < n) out[row0 + lane] = lg[warp][lane];
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace
}  // namespace how

using namespace how;

extern "C" {

// Gradient of the mean weighted BCE over n samples (FP32, one pass): the
// check target of the CPU restatement.  All pointers host.
int how_router_grad(const float* w, const float* feats, const float* labels, long n, float pos_weight,
                    float* grad_out, float* loss_out) {
    if (!w || !feats || !labels || n <= 0 || !grad_out) { set_error("router_grad: bad argument"); return HOW_ERR_ARG; }
    DevBuf dw, df, dl, da, dg, dloss;
    HOW_CUDA_CHECK(cudaMalloc(&dw.p, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&df.p, n * NF * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&dl.p, n * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&da.p, n * ACT * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&dg.p, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&dloss.p, sizeof(float)));
    HOW_CUDA_CHECK(cudaMemcpy(dw.p, w, NW * sizeof(float), cudaMemcpyHostToDevice));
    HOW_CUDA_CHECK(cudaMemcpy(df.p, feats, n * NF * sizeof(float), cudaMemcpyHostToDevice));
    HOW_CUDA_CHECK(cudaMemcpy(dl.p, labels, n * sizeof(float), cudaMemcpyHostToDevice));
    k_fwd_bwd<<<(unsigned)((n + 127) / 128), 128>>>((float*)dw.p, (float*)df.p, (float*)dl.p, nullptr, (int)n,
                                                   pos_weight, 1.0f / (float)n, (float*)da.p);
    k_grad_reduce<<<NW + 1, 256>>>((float*)da.p, (int)n, (float*)dg.p, (float*)dloss.p);
    HOW_CUDA_CHECK(cudaGetLastError());
    HOW_CUDA_CHECK(cudaMemcpy(grad_out, dg.p, NW * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss_out) HOW_CUDA_CHECK(cudaMemcpy(loss_out, dloss.p, sizeof(float), cudaMemcpyDeviceToHost));
    return HOW_OK;
}

// Train in place: w (host, RouterLayout) is the starting point and receives
// the result.  Mini-batches of `batch` samples drawn by a seeded host
// generator; Adam with learning rate lr.  loss_hist (may be NULL) receives
// the mean loss of each iteration.
int how_router_train(float* w, const float* feats, const float* labels, long n, float pos_weight, int iters,
                     int batch, float lr, unsigned long long seed, float* loss_hist) {
    if (!w || !feats || !labels || n <= 0 || iters <= 0 || batch <= 0) { set_error("router_train: bad argument"); return HOW_ERR_ARG; }
    if (batch > n) batch = (int)n;
    DevBuf dw, df, dl, da, dg, dm, dv, didx, dloss;
    HOW_CUDA_CHECK(cudaMalloc(&dw.p, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&df.p, n * NF * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&dl.p, n * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&da.p, (size_t)batch * ACT * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&dg.p, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&dm.p, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&dv.p, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&didx.p, (size_t)batch * sizeof(int)));
    HOW_CUDA_CHECK(cudaMalloc(&dloss.p, sizeof(float)));
    HOW_CUDA_CHECK(cudaMemcpy(dw.p, w, NW * sizeof(float), cudaMemcpyHostToDevice));
    HOW_CUDA_CHECK(cudaMemcpy(df.p, feats, n * NF * sizeof(float), cudaMemcpyHostToDevice));
    HOW_CUDA_CHECK(cudaMemcpy(dl.p, labels, n * sizeof(float), cudaMemcpyHostToDevice));
    HOW_CUDA_CHECK(cudaMemset(dm.p, 0, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMemset(dv.p, 0, NW * sizeof(float)));
    std::vector<int> idx(batch);
    unsigned long long st = seed ? seed : 1ull;
    auto next = [&]() { st ^= st << 13; st ^= st >> 7; st ^= st << 17; return st; };   // xorshift64
    const float b1 = 0.9f, b2 = 0.999f;
    for (int it = 0; it < iters; ++it) {
        for (int k = 0; k < batch; ++k) idx[k] = (int)(next() % (unsigned long long)n);
        HOW_CUDA_CHECK(cudaMemcpy(didx.p, idx.data(), batch * sizeof(int), cudaMemcpyHostToDevice));
        k_fwd_bwd<<<(batch + 127) / 128, 128>>>((float*)dw.p, (float*)df.p, (float*)dl.p, (int*)didx.p, batch,
                                               pos_weight, 1.0f / (float)batch, (float*)da.p);
        k_grad_reduce<<<NW + 1, 256>>>((float*)da.p, batch, (float*)dg.p, (float*)dloss.p);
        const float bc1 = 1.f - powf(b1, (float)(it + 1)), bc2 = 1.f - powf(b2, (float)(it + 1));
        k_adam<<<(NW + 255) / 256, 256>>>((float*)dw.p, (float*)dg.p, (float*)dm.p, (float*)dv.p, NW, lr, b1, b2,
                                          1e-8f, bc1, bc2);
        if (loss_hist) HOW_CUDA_CHECK(cudaMemcpy(&loss_hist[it], dloss.p, sizeof(float), cudaMemcpyDeviceToHost));
    }
    HOW_CUDA_CHECK(cudaGetLastError());
    HOW_CUDA_CHECK(cudaMemcpy(w, dw.p, NW * sizeof(float), cudaMemcpyDeviceToHost));
    return HOW_OK;
}

// Logits of n feature rows: out_fp32 by the FP32 network, out_bf16 by the
// sweep kernel's BF16 tensor-core path (either may be NULL).
int how_router_infer(const float* w, const float* feats, long n, float* out_fp32, float* out_bf16) {
    if (!w || !feats || n <= 0) { set_error("router_infer: bad argument"); return HOW_ERR_ARG; }
    DevBuf dw, df, d1, d2;
    HOW_CUDA_CHECK(cudaMalloc(&dw.p, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&df.p, n * NF * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&d1.p, n * sizeof(float)));
    HOW_CUDA_CHECK(cudaMalloc(&d2.p, n * sizeof(float)));
    HOW_CUDA_CHECK(cudaMemcpy(dw.p, w, NW * sizeof(float), cudaMemcpyHostToDevice));
    HOW_CUDA_CHECK(cudaMemcpy(df.p, feats, n * NF * sizeof(float), cudaMemcpyHostToDevice));
    k_infer_fp32<<<(unsigned)((n + 127) / 128), 128>>>((float*)dw.p, (float*)df.p, n, (float*)d1.p);
    k_infer_mma<<<(unsigned)((n + 63) / 64), 128>>>((float*)dw.p, (float*)df.p, n, (float*)d2.p);
    HOW_CUDA_CHECK(cudaGetLastError());
    if (out_fp32) HOW_CUDA_CHECK(cudaMemcpy(out_fp32, d1.p, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (out_bf16) HOW_CUDA_CHECK(cudaMemcpy(out_bf16, d2.p, n * sizeof(float), cudaMemcpyDeviceToHost));
    return HOW_OK;
}

int how_router_param_count(void) { return NW; }

// The built-in trained weights and their logit threshold.
int how_router_default(float* w, int n, float* threshold) {
    if (n != NW) { set_error("router_default: need %d floats", NW); return HOW_ERR_ARG; }
    if (w) std::memcpy(w, kRouterDefaultWeights, sizeof(kRouterDefaultWeights));
    if (threshold) *threshold = kRouterDefaultThreshold;
    return HOW_OK;
}

// ---- per-context routing controls ---------------------------------------
int how_router_set_weights(how_ctx* c, const float* w, int n);
int how_router_configure(how_ctx* c, int mode, float threshold, float guard_jump, float guard_floor);
int how_router_set_weights(how_ctx* c, const float* w, int n) {
    if (!c || !w || n != NW) { set_error("router_set_weights: need %d floats", NW); return HOW_ERR_ARG; }
    HOW_CUDA_CHECK(cudaSetDevice(c->dev));
    if (!c->router_w) HOW_CUDA_CHECK(cudaMalloc(&c->router_w, NW * sizeof(float)));
    HOW_CUDA_CHECK(cudaMemcpy(c->router_w, w, NW * sizeof(float), cudaMemcpyHostToDevice));
    c->route_valid = false;
    return HOW_OK;
}

// mode: 0 off (plain), 1 learned network + guard, 2 guard only.
int how_router_configure(how_ctx* c, int mode, float threshold, float guard_jump, float guard_floor) {
    if (!c || mode < 0 || mode > 2) { set_error("router_configure: mode 0..2"); return HOW_ERR_ARG; }
    if (mode == 1 && !c->router_w) { set_error("router_configure: no weights set"); return HOW_ERR_STATE; }
    HOW_CUDA_CHECK(cudaSetDevice(c->dev));
    if (mode != 0 && !c->route_prev) {
        HOW_CUDA_CHECK(cudaMalloc(&c->route_prev, 6 * (size_t)c->g.fs));
        HOW_CUDA_CHECK(cudaMemset(c->route_prev, 1, 6 * (size_t)c->g.fs));
    }
    if (!c->route_count) {
        HOW_CUDA_CHECK(cudaMalloc(&c->route_count, 4 * sizeof(unsigned long long)));
        HOW_CUDA_CHECK(cudaMemset(c->route_count, 0, 4 * sizeof(unsigned long long)));
    }
    c->route_mode = mode;
    c->route_valid = false;
    c->route_thr = threshold;
    c->guard_jump = guard_jump;
    c->guard_floor = guard_floor;
    return HOW_OK;
}

// Learned routing forms the network's decisions every `stages` stages of a
// step, from its first (5: once per step, the default; 1: every stage), or
// with 10 at the first stage of every second step; in between the sweeps
// reuse them, and re-evaluate the hard guard on each stage's own state.
// Reuse over two steps stays inside the decisions' one-face dilation: at a
// Courant number <= 0.4 no signal crosses more than 0.8 cells in two steps.
int how_router_set_refresh(how_ctx* c, int stages) {
    if (!c || stages < 1 || (stages > 5 && stages != 10)) {
        set_error("router refresh: 1..5 or 10 stages");
        return HOW_ERR_ARG;
    }
    c->route_refresh = stages;
    c->route_valid = false;
    return HOW_OK;
}

// Interfaces (active faces) sent to full WENO and to the linear flux since
// the last reset.
int how_router_stats4(how_ctx* c, unsigned long long* full, unsigned long long* cheap,
                      unsigned long long* mma_groups, unsigned long long* flat_groups, int reset);
int how_router_stats(how_ctx* c, unsigned long long* full, unsigned long long* cheap, int reset) {
    return how_router_stats4(c, full, cheap, nullptr, nullptr, reset);
}

// ... and the 16-interface groups whose logits came from the tensor cores or,
// all their stencils being uniform, from the precomputed flat logits.
int how_router_stats4(how_ctx* c, unsigned long long* full, unsigned long long* cheap,
                      unsigned long long* mma_groups, unsigned long long* flat_groups, int reset) {
    if (!c) return HOW_ERR_ARG;
    unsigned long long h[4] = {0, 0, 0, 0};
    if (c->route_count) {
        HOW_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        HOW_CUDA_CHECK(cudaMemcpy(h, c->route_count, sizeof(h), cudaMemcpyDeviceToHost));
        if (reset) HOW_CUDA_CHECK(cudaMemset(c->route_count, 0, sizeof(h)));
    }
    if (full) *full = h[0];
    if (cheap) *cheap = h[1];
    if (mma_groups) *mma_groups = h[2];
    if (flat_groups) *flat_groups = h[3];
    return HOW_OK;
}

// Label collection: while active, every sweep runs the plain FP64 method and
// records (6 features, label, weight deviation) of one tile in `every`
// (labels: 1 if any field's nonlinear weights depart from the linear ones by
// more than 0.1).
int how_collect_begin(how_ctx* c, unsigned int capacity, unsigned int every) {
    if (!c || capacity == 0) return HOW_ERR_ARG;
    HOW_CUDA_CHECK(cudaSetDevice(c->dev));
    if (c->collect) { cudaFree(c->collect); c->collect = nullptr; }
    if (!c->collect_n) HOW_CUDA_CHECK(cudaMalloc(&c->collect_n, sizeof(unsigned int)));
    HOW_CUDA_CHECK(cudaMalloc(&c->collect, (size_t)capacity * 8 * sizeof(float)));
    HOW_CUDA_CHECK(cudaMemset(c->collect_n, 0, sizeof(unsigned int)));
    if (!c->route_prev) {
        HOW_CUDA_CHECK(cudaMalloc(&c->route_prev, 6 * (size_t)c->g.fs));
        HOW_CUDA_CHECK(cudaMemset(c->route_prev, 1, 6 * (size_t)c->g.fs));
    }
    c->collect_cap = capacity;
    c->collect_every = every ? every : 1;
    c->route_mode = 3;
    return HOW_OK;
}

// Copies up to `cap` records (8 floats each) to `out`; returns the count in
// *n and ends collection (routing off).
int how_collect_end(how_ctx* c, float* out, unsigned int cap, unsigned int* n) {
    if (!c || !n) return HOW_ERR_ARG;
    HOW_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    unsigned int cnt = 0;
    if (c->collect_n) HOW_CUDA_CHECK(cudaMemcpy(&cnt, c->collect_n, sizeof(cnt), cudaMemcpyDeviceToHost));
    if (cnt > c->collect_cap) cnt = c->collect_cap;
    if (cnt > cap) cnt = cap;
    if (out && cnt) HOW_CUDA_CHECK(cudaMemcpy(out, c->collect, (size_t)cnt * 8 * sizeof(float), cudaMemcpyDeviceToHost));
    *n = cnt;
    if (c->collect) { cudaFree(c->collect); c->collect = nullptr; }
    c->collect_cap = 0;
    c->route_mode = 0;
    return HOW_OK;
}

}  // extern "C"

namespace how {
// `router on` in the parameters: the built-in network and threshold.
int router_enable_default(how_ctx* c) {
    int rc = how_router_set_weights(c, kRouterDefaultWeights, NW);
    if (!rc) rc = how_router_configure(c, 1, kRouterDefaultThreshold, 0.25f, 100.0f);
    return rc;
}
}  // namespace how
