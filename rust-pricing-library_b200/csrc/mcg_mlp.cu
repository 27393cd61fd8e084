// mcg_mlp.cu -- the learned continuation value of the early-exercise engine.
//
// No counterpart in the reference (whose continuation value is the CPQR
// polynomial of crates/pricing/src/engine/mc/lsm.rs:2067-2247): a
// 2 -> 64 -> 64 -> 1 network with SiLU activations,
//   f(x) = W3 . silu(W2 silu(W1 x + b1) + b2) + b3,
// of the scaled spot 4 (S - K) / K and the scaled time 2 t / T - 1, predicting
// the scaled continuation value 10 C / K.  Master parameters are FP32; the
// 64 x 64 layer runs on the tensor cores with BF16 operands and FP32
// accumulation (mma.sync m16n8k16), forward and backward; the thin input and
// output layers run on the FP32 pipe.
//
// Training step (one launch + one Adam launch): each CTA takes tiles of 128
// rows, four warps of 32.  A warp runs layer 1 for its rows into shared
// memory, the 64 x 64 layer and the output, the output error, and back
// through both hidden layers; the CTA then forms its share of dLoss/dW2 =
// dH2^T H1 with each warp owning 16 output rows of W2 in registers.  Every
// gradient sum is taken in a fixed order (lanes, warps, CTAs), so a step is
// reproducible bit for bit.
#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "mcg_kernels.cuh"
#include "mcg_mlp.cuh"

namespace mcg {
namespace {

constexpr int kH = kMlpHidden;
constexpr int kStride = kH + 8;  // padded BF16 row: conflict-free fragment loads
constexpr int kMlpWarps = 4;
constexpr int kMlpThreads = 32 * kMlpWarps;
constexpr int kTileRows = kMlpThreads;  // rows per CTA iteration
constexpr int kSmall = 2 * kH + kH + kH + kH + 1;  // W1, b1, b2, W3, b3 gradients

struct NetShared {
    float w1[kH][2];
    float b1[kH];
    float b2[kH];
    float w3[kH];
    float b3;
    __align__(16) __nv_bfloat16 w2[kH][kStride];   // [out][in]
    __align__(16) __nv_bfloat16 w2t[kH][kStride];  // [in][out]
};

__device__ void load_net(NetShared& s, const float* __restrict__ p) {
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
        const int o = i / kH, in = i % kH;
        const __nv_bfloat16 w = __float2bfloat16_rn(p[kMlpW2 + i]);
        s.w2[o][in] = w;
        s.w2t[in][o] = w;
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        s.w1[i][0] = p[kMlpW1 + 2 * i];
        s.w1[i][1] = p[kMlpW1 + 2 * i + 1];
        s.b1[i] = p[kMlpB1 + i];
        s.b2[i] = p[kMlpB2 + i];
        s.w3[i] = p[kMlpW3 + i];
    }
    if (threadIdx.x == 0) s.b3 = p[kMlpB3];
    __syncthreads();
}

// Logistic function on the special-function unit (exp2 and reciprocal
// approximations, ~2 ulp): the network is an approximation itself, and the
// gradient checks bound the whole forward/backward pass.
__device__ __forceinline__ float sigmoid(float x) { return __fdividef(1.0f, 1.0f + __expf(-x)); }
__device__ __forceinline__ float silu(float x) { return x * sigmoid(x); }
__device__ __forceinline__ float silu_grad(float x) {
    const float s = sigmoid(x);
    return s * (1.0f + x * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return static_cast<uint32_t>(__bfloat16_as_ushort(lo)) |
           (static_cast<uint32_t>(__bfloat16_as_ushort(hi)) << 16);
}

__device__ __forceinline__ uint32_t ld2(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D = A B + D for one 16 x 8 x 16 tile: A row-major BF16, B column-major BF16,
// D FP32 (PTX mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32).
__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Layer 1 for the lane's own row: silu(W1 x + b1) as BF16 into `row`.
__device__ __forceinline__ void layer1(const NetShared& net, __nv_bfloat16* row, float x0, float x1) {
#pragma unroll 8
    for (int i = 0; i < kH; i += 2) {
        const float a = net.w1[i][0] * x0 + net.w1[i][1] * x1 + net.b1[i];
        const float b = net.w1[i + 1][0] * x0 + net.w1[i + 1][1] * x1 + net.b1[i + 1];
        *reinterpret_cast<uint32_t*>(row + i) = pack2(__float2bfloat16_rn(silu(a)), __float2bfloat16_rn(silu(b)));
    }
}

// acc = X W^T + bias for the warp's 32 rows of X (row-major [32][kStride]) and
// a [64][kStride] weight matrix W (row n holds output n).  Fragment layout of
// acc[mt][nt]: rows mt*16 + g (+8), columns nt*8 + 2t (+1), g = lane / 4, t = lane % 4.
__device__ __forceinline__ void gemm_rows(const __nv_bfloat16* X, const __nv_bfloat16 (*W)[kStride],
                                          const float* bias, float (&acc)[2][8][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float b0 = bias ? bias[nt * 8 + 2 * t] : 0.0f;
        const float b1 = bias ? bias[nt * 8 + 2 * t + 1] : 0.0f;
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            acc[mt][nt][0] = b0;
            acc[mt][nt][1] = b1;
            acc[mt][nt][2] = b0;
            acc[mt][nt][3] = b1;
        }
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        uint32_t a[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const __nv_bfloat16* r0 = X + (mt * 16 + g) * kStride + kt * 16 + 2 * t;
            const __nv_bfloat16* r1 = r0 + 8 * kStride;
            a[mt][0] = ld2(r0);
            a[mt][1] = ld2(r1);
            a[mt][2] = ld2(r0 + 8);
            a[mt][3] = ld2(r1 + 8);
        }
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const __nv_bfloat16* wr = &W[nt * 8 + g][kt * 16 + 2 * t];
            const uint32_t b0 = ld2(wr), b1 = ld2(wr + 8);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) mma16816(acc[mt][nt], a[mt][0], a[mt][1], a[mt][2], a[mt][3], b0, b1);
        }
    }
}

// Network output for the warp's rows given the layer-2 pre-activations; every
// lane returns the output of its own row (row = lane).
__device__ __forceinline__ float output_rows(const NetShared& net, const float (&acc)[2][8][4]) {
    const int lane = threadIdx.x & 31, t = lane & 3;
    float part[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};  // [mt][half]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) part[mt][e >> 1] += silu(acc[mt][nt][e]) * net.w3[nt * 8 + 2 * t + (e & 1)];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            part[mt][h] += __shfl_xor_sync(0xffffffffu, part[mt][h], 1);
            part[mt][h] += __shfl_xor_sync(0xffffffffu, part[mt][h], 2);
        }
    // row r = mt*16 + h*8 + g lives in quad g = r % 8
    const int src = (lane & 7) * 4;
    const float o00 = __shfl_sync(0xffffffffu, part[0][0], src);
    const float o01 = __shfl_sync(0xffffffffu, part[0][1], src);
    const float o10 = __shfl_sync(0xffffffffu, part[1][0], src);
    const float o11 = __shfl_sync(0xffffffffu, part[1][1], src);
    const int mt = lane >> 4, h = (lane >> 3) & 1;
    const float own = mt ? (h ? o11 : o10) : (h ? o01 : o00);
    return own + net.b3;
}

// Forward pass for the warp: every lane passes its row's inputs and gets its
// output.  `h1` is the warp's [32][kStride] scratch.  All 32 lanes take part.
__device__ __forceinline__ float forward_warp(const NetShared& net, __nv_bfloat16* h1, float x0, float x1) {
    const int lane = threadIdx.x & 31;
    layer1(net, h1 + lane * kStride, x0, x1);
    __syncwarp();
    float acc[2][8][4];
    gemm_rows(h1, net.w2, net.b2, acc);
    const float out = output_rows(net, acc);
    __syncwarp();
    return out;
}

// Sum over the 8 lane groups that share t (lanes t, t+4, ..., t+28).
__device__ __forceinline__ float sum_groups(float v) {
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

struct GradShared {
    NetShared net;
    __align__(16) __nv_bfloat16 h1[kTileRows][kStride];  // silu(layer 1), BF16
    __align__(16) __nv_bfloat16 d2[kTileRows][kStride];  // dLoss / d(layer-2 pre-activation), BF16
    float small[kMlpWarps][kSmall];        // per-warp W1, b1, b2, W3, b3 gradient sums
    float loss[kMlpWarps], rows[kMlpWarps];
};

// Loads row r of a step: inputs, scaled target and mask.
__device__ __forceinline__ void load_row(const MlpRows& R, uint64_t r, float& x0, float& x1, float& y, float& m) {
    x0 = 0.0f;
    x1 = 0.0f;
    y = 0.0f;
    m = 0.0f;
    if (r >= R.count) return;
    if (R.x) {
        x0 = R.x[2 * r];
        x1 = R.x[2 * r + 1];
        y = R.y[r];
        m = R.mask[r] ? 1.0f : 0.0f;
        return;
    }
    const uint64_t p = R.first + r;
    const double s = R.spots[p];
    const double in = R.side == MCG_CALL ? s - R.strike : R.strike - s;
    const double imm = (in >= 0.0 ? in : 0.0) * R.notional;
    if (!(imm > R.itm_tol)) return;
    x0 = static_cast<float>(4.0 * (s - R.strike) / R.strike);
    x1 = static_cast<float>(R.time_input);
    y = static_cast<float>(10.0 * (R.cf[p] / R.df) / R.strike);
    m = 1.0f;
}

// One gradient pass of the CTA over its tiles of the step's rows (tiles
// blockIdx.x, + gridDim.x, ...), written as the CTA's partial record.
__device__ __forceinline__ void gradient_pass(GradShared& S, const float* __restrict__ params, const MlpRows& R,
                                              float* __restrict__ partials) {
    load_net(S.net, params);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int i = lane; i < kSmall; i += 32) S.small[warp][i] = 0.0f;
    float loss = 0.0f, rows = 0.0f;
    float gw2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) gw2[nt][e] = 0.0f;
    const uint64_t tiles = (R.count + kTileRows - 1) / kTileRows;
    __nv_bfloat16* h1w = &S.h1[warp * 32][0];
    __nv_bfloat16* d2w = &S.d2[warp * 32][0];
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        float x0, x1, y, m;
        load_row(R, tile * kTileRows + warp * 32 + lane, x0, x1, y, m);
        // forward
        layer1(S.net, h1w + lane * kStride, x0, x1);
        __syncwarp();
        float acc[2][8][4];
        gemm_rows(h1w, S.net.w2, S.net.b2, acc);
        const float out = output_rows(S.net, acc);
        const float err = out - y;
        loss += m * err * err;
        rows += m;
        const float delta = 2.0f * m * err;  // dLoss/dout of the own row
        float dlt[2][2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) dlt[mt][h] = __shfl_sync(0xffffffffu, delta, mt * 16 + h * 8 + g);
        // output layer and layer 2 backward: dW3, db2, dH2
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float gw3v[2] = {0.0f, 0.0f}, gb2v[2] = {0.0f, 0.0f};
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    float dh[2];
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const float v = acc[mt][nt][2 * h + j];
                        const int col = nt * 8 + 2 * t + j;
                        const float sg = sigmoid(v);  // one logistic for silu and its derivative
                        gw3v[j] += dlt[mt][h] * (v * sg);
                        dh[j] = dlt[mt][h] * S.net.w3[col] * (sg * (1.0f + v * (1.0f - sg)));
                        gb2v[j] += dh[j];
                    }
                    *reinterpret_cast<uint32_t*>(d2w + (mt * 16 + h * 8 + g) * kStride + nt * 8 + 2 * t) =
                        pack2(__float2bfloat16_rn(dh[0]), __float2bfloat16_rn(dh[1]));
                }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const float a = sum_groups(gw3v[j]);
                const float b = sum_groups(gb2v[j]);
                if (g == 0) {
                    S.small[warp][4 * kH + nt * 8 + 2 * t + j] += a;   // W3
                    S.small[warp][3 * kH + nt * 8 + 2 * t + j] += b;   // b2
                }
            }
        }
        {
            float db3 = delta;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) db3 += __shfl_xor_sync(0xffffffffu, db3, off);
            if (lane == 0) S.small[warp][5 * kH] += db3;
        }
        __syncwarp();
        // layer 1 backward: dH1 = (dH2 W2) * silu'(layer-1 pre-activation)
        gemm_rows(d2w, S.net.w2t, nullptr, acc);
        float xr[2][2][2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                xr[mt][h][0] = __shfl_sync(0xffffffffu, x0, mt * 16 + h * 8 + g);
                xr[mt][h][1] = __shfl_sync(0xffffffffu, x1, mt * 16 + h * 8 + g);
            }
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float gw1v[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}}, gb1v[2] = {0.0f, 0.0f};
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const int col = nt * 8 + 2 * t + j;
                        const float pre = S.net.w1[col][0] * xr[mt][h][0] + S.net.w1[col][1] * xr[mt][h][1] +
                                          S.net.b1[col];
                        const float dh1 = acc[mt][nt][2 * h + j] * silu_grad(pre);
                        gw1v[j][0] += dh1 * xr[mt][h][0];
                        gw1v[j][1] += dh1 * xr[mt][h][1];
                        gb1v[j] += dh1;
                    }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const float a0 = sum_groups(gw1v[j][0]);
                const float a1 = sum_groups(gw1v[j][1]);
                const float b = sum_groups(gb1v[j]);
                if (g == 0) {
                    const int col = nt * 8 + 2 * t + j;
                    S.small[warp][2 * col] += a0;       // W1[col][0]
                    S.small[warp][2 * col + 1] += a1;   // W1[col][1]
                    S.small[warp][2 * kH + col] += b;   // b1
                }
            }
        }
        __syncthreads();
        // dW2 = dH2^T H1 over the CTA's 128 rows; warp w owns outputs 16w .. 16w+15.
        const int o0 = warp * 16;
#pragma unroll
        for (int kt = 0; kt < kTileRows / 16; ++kt) {
            const int s0 = kt * 16 + 2 * t;
            const uint32_t a0 = pack2(S.d2[s0][o0 + g], S.d2[s0 + 1][o0 + g]);
            const uint32_t a1 = pack2(S.d2[s0][o0 + g + 8], S.d2[s0 + 1][o0 + g + 8]);
            const uint32_t a2 = pack2(S.d2[s0 + 8][o0 + g], S.d2[s0 + 9][o0 + g]);
            const uint32_t a3 = pack2(S.d2[s0 + 8][o0 + g + 8], S.d2[s0 + 9][o0 + g + 8]);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const uint32_t b0 = pack2(S.h1[s0][nt * 8 + g], S.h1[s0 + 1][nt * 8 + g]);
                const uint32_t b1 = pack2(S.h1[s0 + 8][nt * 8 + g], S.h1[s0 + 9][nt * 8 + g]);
                mma16816(gw2[nt], a0, a1, a2, a3, b0, b1);
            }
        }
        __syncthreads();
    }
    // per-CTA partial record
    float* out = partials + static_cast<size_t>(blockIdx.x) * kMlpPartial;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int o = warp * 16 + g + (e >> 1) * 8;
            const int i = nt * 8 + 2 * t + (e & 1);
            out[kMlpW2 + o * kH + i] = gw2[nt][e];
        }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        loss += __shfl_xor_sync(0xffffffffu, loss, off);
        rows += __shfl_xor_sync(0xffffffffu, rows, off);
    }
    if (lane == 0) {
        S.loss[warp] = loss;
        S.rows[warp] = rows;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSmall; i += blockDim.x) {
        float v = S.small[0][i];
        for (int w = 1; w < kMlpWarps; ++w) v += S.small[w][i];
        int dst;
        if (i < 2 * kH) dst = kMlpW1 + i;
        else if (i < 3 * kH) dst = kMlpB1 + (i - 2 * kH);
        else if (i < 4 * kH) dst = kMlpB2 + (i - 3 * kH);
        else if (i < 5 * kH) dst = kMlpW3 + (i - 4 * kH);
        else dst = kMlpB3;
        out[dst] = v;
    }
    if (threadIdx.x == 0) {
        float l = 0.0f, r = 0.0f;
        for (int w = 0; w < kMlpWarps; ++w) {
            l += S.loss[w];
            r += S.rows[w];
        }
        out[kMlpParams] = l;
        out[kMlpParams + 1] = r;
    }
}

__global__ void __launch_bounds__(kMlpThreads) mlp_gradient_kernel(const float* __restrict__ params, const MlpRows R,
                                                                   float* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradShared& S = *reinterpret_cast<GradShared*>(smem_raw);
    gradient_pass(S, params, R, partials);
}

// Sums the per-CTA records in CTA order and takes one Adam step on the mean
// gradient (beta1 0.9, beta2 0.999, eps 1e-8) for parameter i.  moments = [m | v].
__device__ __forceinline__ void adam_param(int i, const float* __restrict__ partials, unsigned ctas,
                                           float* __restrict__ params, float* __restrict__ moments, uint32_t step,
                                           float lr, float* loss_out) {
    float rows = 0.0f, gsum = 0.0f;
#pragma unroll 8
    for (unsigned c = 0; c < ctas; ++c) {  // in CTA order; the loads run ahead of the adds
        gsum += partials[static_cast<size_t>(c) * kMlpPartial + i];
        rows += partials[static_cast<size_t>(c) * kMlpPartial + kMlpParams + 1];
    }
    if (rows <= 0.0f) return;
    const float grad = gsum / rows;
    const float b1 = 0.9f, b2 = 0.999f;
    const float m = b1 * moments[i] + (1.0f - b1) * grad;
    const float v = b2 * moments[kMlpParams + i] + (1.0f - b2) * grad * grad;
    moments[i] = m;
    moments[kMlpParams + i] = v;
    const float mhat = m / (1.0f - powf(b1, static_cast<float>(step)));
    const float vhat = v / (1.0f - powf(b2, static_cast<float>(step)));
    params[i] -= lr * mhat / (sqrtf(vhat) + 1e-8f);
    if (i == 0 && loss_out) {
        float l = 0.0f;
        for (unsigned c = 0; c < ctas; ++c) l += partials[static_cast<size_t>(c) * kMlpPartial + kMlpParams];
        *loss_out = l / rows;
    }
}

__global__ void mlp_adam_kernel(const float* __restrict__ partials, unsigned ctas, float* __restrict__ params,
                                float* __restrict__ moments, uint32_t step, float lr, float* loss_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    adam_param(i, partials, ctas, params, moments, step, lr, loss_out);
}

// A date's whole training in one cooperative launch: per step, every CTA's
// gradient pass over its tiles of batch (k mod nbatch), a grid barrier, the
// Adam update spread over the grid's threads, a grid barrier.  The same
// arithmetic in the same order as alternating mlp_gradient_kernel and
// mlp_adam_kernel launches (a CTA whose tiles run out writes a zero record,
// which adds nothing), without two launches per step.
__global__ void __launch_bounds__(kMlpThreads) mlp_train_kernel(float* __restrict__ params,
                                                                float* __restrict__ moments,
                                                                float* __restrict__ partials, MlpRows R0,
                                                                uint64_t total, uint64_t batch, uint32_t steps,
                                                                uint32_t step0, float lr, float* loss_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradShared& S = *reinterpret_cast<GradShared*>(smem_raw);
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const uint64_t nbatch = (total + batch - 1) / batch;
    for (uint32_t k = 0; k < steps; ++k) {
        MlpRows R = R0;
        R.first = (k % nbatch) * batch;
        R.count = min(batch, total - R.first);
        gradient_pass(S, params, R, partials);
        grid.sync();
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x)
            adam_param(i, partials, gridDim.x, params, moments, step0 + k + 1, lr, k + 1 == steps ? loss_out : nullptr);
        grid.sync();
    }
}

// Plain sums of the per-CTA records (gradient of the summed loss, the loss).
__global__ void mlp_sum_kernel(const float* __restrict__ partials, unsigned ctas, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpPartial) return;
    float s = 0.0f;
    for (unsigned c = 0; c < ctas; ++c) s += partials[static_cast<size_t>(c) * kMlpPartial + i];
    out[i] = s;
}

struct ForwardShared {
    NetShared net;
    __align__(16) __nv_bfloat16 h1[kTileRows][kStride];
};

__global__ void __launch_bounds__(kMlpThreads) mlp_forward_kernel(const float* __restrict__ params,
                                                                  const float* __restrict__ x, uint32_t count,
                                                                  float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ForwardShared& S = *reinterpret_cast<ForwardShared*>(smem_raw);
    load_net(S.net, params);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t tiles = (count + 31) / 32;
    for (uint64_t tile = static_cast<uint64_t>(blockIdx.x) * kMlpWarps + warp; tile < tiles;
         tile += static_cast<uint64_t>(gridDim.x) * kMlpWarps) {
        const uint64_t r = tile * 32 + lane;
        const float x0 = r < count ? x[2 * r] : 0.0f, x1 = r < count ? x[2 * r + 1] : 0.0f;
        const float f = forward_warp(S.net, &S.h1[warp * 32][0], x0, x1);
        if (r < count) out[r] = f;
    }
}

// The network's exercise decision at one training date for every path:
// exercise an ITM path when immediate > continuation.
__global__ void __launch_bounds__(kMlpThreads) mlp_decide_kernel(const float* __restrict__ params,
                                                                 const MlpDecision D) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ForwardShared& S = *reinterpret_cast<ForwardShared*>(smem_raw);
    load_net(S.net, params);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t tiles = (D.paths + 31) / 32;
    for (uint64_t tile = static_cast<uint64_t>(blockIdx.x) * kMlpWarps + warp; tile < tiles;
         tile += static_cast<uint64_t>(gridDim.x) * kMlpWarps) {
        const uint64_t p = tile * 32 + lane;
        const double s = p < D.paths ? D.spots[p] : D.strike;
        const double in = D.side == MCG_CALL ? s - D.strike : D.strike - s;
        const double imm = (in >= 0.0 ? in : 0.0) * D.notional;
        const float x0 = static_cast<float>(4.0 * (s - D.strike) / D.strike);
        const float f = forward_warp(S.net, &S.h1[warp * 32][0], x0, static_cast<float>(D.time_input));
        const double cont = static_cast<double>(f) * D.strike / 10.0;
        if (p < D.paths && imm > D.itm_tol && imm > cont) {
            D.cf[p] = imm * D.df;
            D.stop[p] = D.date;
        }
    }
}

// Valuation paths under the network's policy (cf. lsm_bs_value_kernel): the
// warp evaluates the network for its 32 units (and their mates) at each date,
// with the weights the training held when it decided that date
// (`params` + date * MCG_MLP_PARAMS), so the valued policy is the trained one.
__global__ void __launch_bounds__(kMlpThreads) lsm_bs_value_mlp_kernel(const DevicePlan P, LsmValueArgs V,
                                                                       const float* __restrict__ params,
                                                                       double inv_horizon) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ForwardShared& S = *reinterpret_cast<ForwardShared*>(smem_raw);
    unsigned int* s_counts = reinterpret_cast<unsigned int*>(smem_raw + sizeof(ForwardShared));
    for (uint32_t i = threadIdx.x; i < V.dates; i += blockDim.x) s_counts[i] = 0;
    const int warp = threadIdx.x >> 5;
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool valid = point < P.units;
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = valid ? point : 0;
    ns.gray = static_cast<uint32_t>(ns.unit ^ (ns.unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    ns.domain = 0;
    const uint64_t unit = static_cast<uint64_t>(scramble) * P.units + point;
    const int pairs = P.antithetic ? 2 : 1;
    const uint32_t n = P.observation_count;
    double w[2] = {0.0, 0.0};
    double realized[2] = {0.0, 0.0};
    uint32_t stop[2] = {n - 1, n - 1};
    bool open[2] = {valid, valid && pairs == 2};
    const double* row = V.spots && valid ? V.spots + unit * pairs : nullptr;
    for (uint32_t i = 0; i < n; ++i) {
        // CTA-uniform: every warp finished the previous date before the weights change
        if (!__syncthreads_or(open[0] || open[1])) break;
        if (i + 1 < n) load_net(S.net, params + static_cast<size_t>(i) * kMlpParams);
        const double z = (P.zero_variance || !valid || V.spots) ? 0.0 : ns.normal(i);
        const double t = P.obs_time[i];
        const double tv = P.vol * P.vol * t;
        const float tin = static_cast<float>(2.0 * t * inv_horizon - 1.0);
        for (int e = 0; e < pairs; ++e) {
            const double ze = e == 0 ? z : -z;
            double f;
            if (V.spots) {
                f = row ? row[static_cast<size_t>(i) * V.paths + e] : V.strike;
            } else if (n == 1) {
                f = P.obs_fwd[0] * 1.0 * exp(-0.5 * tv + sqrt(tv) * ze);
            } else {
                w[e] += P.obs_sqrt_step[i] * ze;
                f = P.obs_fwd[i] * 1.0 * exp(-0.5 * tv + P.vol * w[e]);
            }
            const double in = V.side == MCG_CALL ? f - V.strike : V.strike - f;
            const double imm = (in >= 0.0 ? in : 0.0) * V.notional;
            if (i + 1 == n) {
                if (open[e]) {
                    realized[e] = imm;
                    open[e] = false;
                }
                continue;
            }
            const float x0 = static_cast<float>(4.0 * (f - V.strike) / V.strike);
            const float out = forward_warp(S.net, &S.h1[warp * 32][0], x0, tin);
            const double cont = static_cast<double>(out) * V.strike / 10.0;
            if (open[e] && imm > 0.0 && imm > cont) {
                realized[e] = imm;
                stop[e] = i;
                open[e] = false;
            }
        }
    }
    if (valid) {
        const double d0 = realized[0] * V.df[stop[0]];
        double value = d0;
        if (pairs == 2) value = (d0 + realized[1] * V.df[stop[1]]) * 0.5;
        V.unit_values[unit] = value;
        for (int e = 0; e < pairs; ++e) {
            atomicAdd(&s_counts[stop[e]], 1u);
            if (V.stops) V.stops[unit * pairs + e] = stop[e];
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < V.dates; i += blockDim.x)
        if (s_counts[i]) atomicAdd(&V.counts[i], static_cast<unsigned long long>(s_counts[i]));
}

int device_sms() {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    return sms;
}

}  // namespace

unsigned mlp_gradient_ctas(uint64_t rows) {
    const uint64_t tiles = (rows + kTileRows - 1) / kTileRows;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(tiles, static_cast<uint64_t>(device_sms()))));
}

cudaError_t launch_mlp_gradient(const float* params, const MlpRows& rows, float* partials, unsigned ctas,
                                cudaStream_t stream) {
    const size_t smem = sizeof(GradShared);
    cudaError_t e = cudaFuncSetAttribute(mlp_gradient_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    mlp_gradient_kernel<<<ctas, kMlpThreads, smem, stream>>>(params, rows, partials);
    return cudaGetLastError();
}

cudaError_t launch_mlp_train(float* params, float* moments, float* partials, const MlpRows& rows, uint64_t total,
                             uint64_t batch, uint32_t steps, uint32_t step0, float learning_rate, float* loss_out,
                             cudaStream_t stream) {
    const size_t smem = sizeof(GradShared);
    cudaError_t e = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mlp_train_kernel, kMlpThreads, smem);
    if (e != cudaSuccess) return e;
    // as many CTAs as a full batch has tiles, all co-resident
    const unsigned ctas = std::min<unsigned>(mlp_gradient_ctas(std::min(batch, total)),
                                             static_cast<unsigned>(std::max(per_sm, 1) * device_sms()));
    MlpRows r = rows;
    void* args[] = {&params, &moments, &partials, &r, &total, &batch, &steps, &step0, &learning_rate, &loss_out};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(mlp_train_kernel), dim3(ctas), dim3(kMlpThreads),
                                       args, smem, stream);
}

cudaError_t launch_mlp_adam(const float* partials, unsigned ctas, float* params, float* moments, uint32_t step,
                            float learning_rate, float* loss_out, cudaStream_t stream) {
    mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, stream>>>(partials, ctas, params, moments, step,
                                                                   learning_rate, loss_out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_sum(const float* partials, unsigned ctas, float* out, cudaStream_t stream) {
    mlp_sum_kernel<<<(kMlpPartial + 255) / 256, 256, 0, stream>>>(partials, ctas, out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const float* params, const float* x, uint32_t count, float* out,
                               cudaStream_t stream) {
    const size_t smem = sizeof(ForwardShared);
    cudaError_t e = cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const unsigned tiles = (count + 31) / 32;
    const unsigned ctas = std::max(1u, std::min<unsigned>((tiles + kMlpWarps - 1) / kMlpWarps, 4u * device_sms()));
    mlp_forward_kernel<<<ctas, kMlpThreads, smem, stream>>>(params, x, count, out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_decide(const float* params, const MlpDecision& D, cudaStream_t stream) {
    const size_t smem = sizeof(ForwardShared);
    cudaError_t e = cudaFuncSetAttribute(mlp_decide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const uint64_t tiles = (D.paths + 31) / 32;
    const unsigned ctas = static_cast<unsigned>(
        std::max<uint64_t>(1, std::min<uint64_t>((tiles + kMlpWarps - 1) / kMlpWarps, 8ull * device_sms())));
    mlp_decide_kernel<<<ctas, kMlpThreads, smem, stream>>>(params, D);
    return cudaGetLastError();
}

cudaError_t launch_lsm_bs_value_mlp(const DevicePlan& P, const LsmValueArgs& V, const float* params,
                                    double inv_horizon, cudaStream_t stream) {
    const size_t smem = sizeof(ForwardShared) + V.dates * sizeof(unsigned int);
    cudaError_t e = cudaFuncSetAttribute(lsm_bs_value_mlp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const dim3 grid(static_cast<unsigned>((P.units + kMlpThreads - 1) / kMlpThreads), P.scramble_count);
    lsm_bs_value_mlp_kernel<<<grid, kMlpThreads, smem, stream>>>(P, V, params, inv_horizon);
    return cudaGetLastError();
}

}  // namespace mcg
