// router.cuh -- the learned WENO router's device pieces, shared by the sweep
// kernel (inference inside a tile) and router.cu (training, batched
// inference, gradient checks).
//
// Network: 6 features -> 32 -> 32 (GELU, tanh form) -> 1 logit.  Inference
// runs on the tensor cores with mma.sync m16n8k16 BF16 x BF16 -> FP32 and the
// hardware tanh (the per-tile batch is at most a few dozen interfaces, far
// below a tcgen05 128-row tile); training is FP32 (router.cu).
//
// Features of the interface between cells c+2 and c+3 over its 6-cell
// stencil c..c+5 (all dimensionless, log10 with a 1e-6 floor):
//   0  max |d rho| / min rho
//   1  max |d p|   / min p
//   2  max |d |B|| / (max |B| + sqrt(min p))
//   3  max |d |v|| / max c_f
//   4  max |d c_f| / min c_f
//   5  1 if this face was sent to full WENO in the previous stage, else 0
// The hard guard (jump of rho or p above guard_jump, or rho / p within
// guard_floor times the floors) overrides the network toward full WENO.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace how {

constexpr int kRouterH = 32;
constexpr int kRouterNF = 6;

__device__ __forceinline__ float gelu_tanh(float x) {
    // 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.0f + tanhf(u));
}

__device__ __forceinline__ float gelu_tanh_grad(float x) {
    const float x2 = x * x;
    const float u = 0.7978845608028654f * (x + 0.044715f * x2 * x);
    const float th = tanhf(u);
    const float du = 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * x2);
    return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * du;
}

// GELU with the hardware tanh approximation (MUFU, |error| ~ 2^-10.7): the
// tensor-core inference path, whose operands are BF16 anyway.
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float gelu_fast(float x) {
    // sqrt(2/pi) (x + 0.044715 x^3) = x (0.79788456 + 0.03567741 x^2)
    const float u = x * fmaf(0.0356774081363001f, x * x, 0.7978845608028654f);
    const float hx = 0.5f * x;
    return fmaf(hx, tanh_fast(u), hx);
}

// Features from the stencil's cell values; returns the guard decision.
struct StencilCell { float rho, p, bmag, vmag, cf; };

// *flat: every jump is exactly zero (a uniform stencil), so feat[0..4] are all
// log10f(1e-6f).
__device__ __forceinline__ bool router_features(const StencilCell* s, float prior, float rhomin, float pgmin,
                                                float guard_jump, float guard_floor, float* feat, bool* flat) {
    float minrho = s[0].rho, minp = s[0].p, maxb = s[0].bmag, maxcf = s[0].cf, mincf = s[0].cf;
    float drho = 0.f, dp = 0.f, db = 0.f, dv = 0.f, dcf = 0.f;
#pragma unroll
    for (int k = 1; k < 6; ++k) {
        minrho = fminf(minrho, s[k].rho); minp = fminf(minp, s[k].p);
        maxb = fmaxf(maxb, s[k].bmag); maxcf = fmaxf(maxcf, s[k].cf); mincf = fminf(mincf, s[k].cf);
        drho = fmaxf(drho, fabsf(s[k].rho - s[k - 1].rho));
        dp = fmaxf(dp, fabsf(s[k].p - s[k - 1].p));
        db = fmaxf(db, fabsf(s[k].bmag - s[k - 1].bmag));
        dv = fmaxf(dv, fabsf(s[k].vmag - s[k - 1].vmag));
        dcf = fmaxf(dcf, fabsf(s[k].cf - s[k - 1].cf));
    }
    const float tiny = 1e-30f;
    const float jr = drho / fmaxf(minrho, tiny), jp = dp / fmaxf(minp, tiny);
    feat[0] = log10f(1e-6f + jr);
    feat[1] = log10f(1e-6f + jp);
    feat[2] = log10f(1e-6f + db / fmaxf(maxb + sqrtf(fmaxf(minp, 0.f)), tiny));
    feat[3] = log10f(1e-6f + dv / fmaxf(maxcf, tiny));
    feat[4] = log10f(1e-6f + dcf / fmaxf(mincf, tiny));
    feat[5] = prior;
    *flat = drho == 0.0f && dp == 0.0f && db == 0.0f && dv == 0.0f && dcf == 0.0f;
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 6; ++k) sum += s[k].rho + s[k].p;
    const bool bad = !(sum == sum) || !(jr == jr) || !(jp == jp);   // NaN anywhere: full method
    return bad || jr > guard_jump || jp > guard_jump || minrho < guard_floor * rhomin ||
           minp < guard_floor * pgmin;
}

// The guard from 6 consecutive densities and pressures, without divisions
// (jump > guard_jump * min is the same test; a NaN fails every comparison).
__device__ __forceinline__ bool router_guard_rp(const float* rho, const float* p, float rhomin, float pgmin,
                                                float guard_jump, float guard_floor) {
    float minrho = rho[0], minp = p[0], drho = 0.f, dp = 0.f, sum = rho[0] + p[0];
#pragma unroll
    for (int k = 1; k < 6; ++k) {
        minrho = fminf(minrho, rho[k]);
        minp = fminf(minp, p[k]);
        drho = fmaxf(drho, fabsf(rho[k] - rho[k - 1]));
        dp = fmaxf(dp, fabsf(p[k] - p[k - 1]));
        sum += rho[k] + p[k];   // NaN anywhere makes the sum NaN (fminf/fmaxf drop it)
    }
    const float tiny = 1e-30f;
    const bool ok = sum == sum && drho <= guard_jump * fmaxf(minrho, tiny) && dp <= guard_jump * fmaxf(minp, tiny) &&
                    minrho >= guard_floor * rhomin && minp >= guard_floor * pgmin;
    return !ok;
}

// FP32 reference of the network (training, checks): w packed as RouterLayout.
__device__ __forceinline__ float router_logit_fp32(const float* w, const float* x) {
    constexpr int H = kRouterH, NF = kRouterNF;
    float h1[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        float s = w[H * NF + j];
#pragma unroll
        for (int i = 0; i < NF; ++i) s += w[j * NF + i] * x[i];
        h1[j] = gelu_tanh(s);
    }
    const float* W2 = w + H * NF + H;
    const float* b2 = W2 + H * H;
    const float* w3 = b2 + H;
    float out = w3[H];
    for (int j = 0; j < H; ++j) {
        float s = b2[j];
#pragma unroll 8
        for (int i = 0; i < H; ++i) s += W2[j * H + i] * h1[i];
        out += w3[j] * gelu_tanh(s);
    }
    return out;
}

// ---------------------------------------------------------------- BF16 MMA
// Shared-memory copy of the network for the tensor-core path.
struct RouterSmem {
    __nv_bfloat16 W1[kRouterH][16];        // [n][k], k = 6 features padded to 16
    __nv_bfloat16 W2[kRouterH][kRouterH];  // [n][k]
    float b1[kRouterH], b2[kRouterH], w3[kRouterH], b3;
};

__device__ __forceinline__ void router_load_smem(RouterSmem* rs, const float* w, int tid, int nt) {
    constexpr int H = kRouterH, NF = kRouterNF;
    for (int t = tid; t < H * 16; t += nt) {
        const int n = t / 16, k = t % 16;
        rs->W1[n][k] = __float2bfloat16_rn(k < NF ? w[n * NF + k] : 0.0f);
    }
    for (int t = tid; t < H * H; t += nt) rs->W2[t / H][t % H] = __float2bfloat16_rn(w[H * NF + H + t]);
    for (int t = tid; t < H; t += nt) {
        rs->b1[t] = w[H * NF + t];
        rs->b2[t] = w[H * NF + H + H * H + t];
        rs->w3[t] = w[H * NF + H + H * H + H + t];
    }
    if (tid == 0) rs->b3 = w[H * NF + H + H * H + 2 * H];
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x = lo (low 16 bits)
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One warp: logits of 16 rows.  X is the rows' features as BF16 [16][16]
// (row-major, 6 used); out[r] receives the logit of row r (lanes 4g write
// rows g and g + 8).  Fragment layout of m16n8k16 (PTX ISA): with g = lane/4,
// t = lane%4, A regs {(g,2t..2t+1), (g+8,2t..), (g,2t+8..), (g+8,2t+8..)},
// B regs {(k=2t..2t+1, n=g), (k=2t+8.., n=g)}, C {(g,2t..2t+1), (g+8,2t..)}.
// A layer's C fragments of n-tiles 2j, 2j+1 are exactly the next layer's A
// fragment of k-tile j, so the hidden layer never leaves registers.
__device__ __forceinline__ void router_mma_16rows(const RouterSmem* rs, const __nv_bfloat16 (*X)[16], float* out) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint32_t a[4];
    a[0] = *reinterpret_cast<const uint32_t*>(&X[g][2 * t]);
    a[1] = *reinterpret_cast<const uint32_t*>(&X[g + 8][2 * t]);
    a[2] = *reinterpret_cast<const uint32_t*>(&X[g][2 * t + 8]);
    a[3] = *reinterpret_cast<const uint32_t*>(&X[g + 8][2 * t + 8]);
    // layer 1: [16 x 16] x [16 x 32]
    float h[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        uint32_t b[2];
        b[0] = *reinterpret_cast<const uint32_t*>(&rs->W1[8 * j + g][2 * t]);
        b[1] = *reinterpret_cast<const uint32_t*>(&rs->W1[8 * j + g][2 * t + 8]);
        h[j][0] = h[j][1] = h[j][2] = h[j][3] = 0.0f;
        mma_bf16_16816(h[j], a, b);
        const float bb0 = rs->b1[8 * j + 2 * t], bb1 = rs->b1[8 * j + 2 * t + 1];
        h[j][0] = gelu_fast(h[j][0] + bb0); h[j][1] = gelu_fast(h[j][1] + bb1);
        h[j][2] = gelu_fast(h[j][2] + bb0); h[j][3] = gelu_fast(h[j][3] + bb1);
    }
    // layer 2: [16 x 32] x [32 x 32], A from the layer-1 accumulators
    uint32_t a2[2][4];
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
        a2[kt][0] = pack_bf16(h[2 * kt][0], h[2 * kt][1]);
        a2[kt][1] = pack_bf16(h[2 * kt][2], h[2 * kt][3]);
        a2[kt][2] = pack_bf16(h[2 * kt + 1][0], h[2 * kt + 1][1]);
        a2[kt][3] = pack_bf16(h[2 * kt + 1][2], h[2 * kt + 1][3]);
    }
    float part0 = 0.0f, part1 = 0.0f;   // rows g, g + 8
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) {
            uint32_t b[2];
            b[0] = *reinterpret_cast<const uint32_t*>(&rs->W2[8 * j + g][16 * kt + 2 * t]);
            b[1] = *reinterpret_cast<const uint32_t*>(&rs->W2[8 * j + g][16 * kt + 2 * t + 8]);
            mma_bf16_16816(d, a2[kt], b);
        }
        const int n0 = 8 * j + 2 * t;
        const float c0 = rs->b2[n0], c1 = rs->b2[n0 + 1];
        const float w0 = rs->w3[n0], w1 = rs->w3[n0 + 1];
        part0 += w0 * gelu_fast(d[0] + c0) + w1 * gelu_fast(d[1] + c1);
        part1 += w0 * gelu_fast(d[2] + c0) + w1 * gelu_fast(d[3] + c1);
    }
    part0 += __shfl_xor_sync(0xffffffffu, part0, 1);
    part0 += __shfl_xor_sync(0xffffffffu, part0, 2);
    part1 += __shfl_xor_sync(0xffffffffu, part1, 1);
    part1 += __shfl_xor_sync(0xffffffffu, part1, 2);
    if (t == 0) {
        out[g] = part0 + rs->b3;
        out[g + 8] = part1 + rs->b3;
    }
}

}  // namespace how
