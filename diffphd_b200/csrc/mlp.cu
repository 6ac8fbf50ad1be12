// Learned warm start of the PD fixed point: a per-node MLP 15 -> 128 -> 128 -> 3 (GELU), BF16 weights and
// activations on the tensor cores (mma.sync m16n8k16, FP32 accumulation), FP32 master weights and AdamW.
//
// Layout.  Rows are nodes (one sample = one node at one time step).  Every warp owns 16 rows; a CTA of 8
// warps owns 128 rows.  The three layers are chained in registers: the FP32 accumulator fragment of one layer
// is the BF16 A-operand fragment of the next (columns 16kk..16kk+15 of the next layer's K are the n-tiles
// 2kk, 2kk+1 of the previous layer's output).  Weight matrices live in shared memory in the "col" layout the
// B operand wants (W^T, i.e. [out][in] with `in` contiguous).
//
// Training step (k_mlp_train): forward with the activations kept in registers, backward through the same
// fragments, then the CTA's rows are staged in shared memory and its weight-gradient partials
// (x^T dz1, a1^T dz2, a2^T dz3) are formed by tensor-core MMAs over the 128 rows; k_mlp_adamw sums the CTA
// partials in a fixed order (deterministic), applies AdamW to the FP32 master weights and re-packs the BF16
// copies.  Features are built on the device by k_mlp_features.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace dphd {

constexpr int kIn = 16, kHid = 128, kOut = 8, kOutUsed = 4;
constexpr int kRowsPerCta = 128;
// per-CTA gradient partial: W1 [16][128], W2 [128][128], W3 [128][8], b1, b2 [128], b3 [8], loss
constexpr int kPartW1 = 0, kPartW2 = kPartW1 + kIn * kHid, kPartW3 = kPartW2 + kHid * kHid;
constexpr int kPartB1 = kPartW3 + kHid * kOut, kPartB2 = kPartB1 + kHid, kPartB3 = kPartB2 + kHid;
constexpr int kPartLoss = kPartB3 + kOut, kPartSize = kPartLoss + 8;

struct MlpParams {
    // FP32 masters (row-major [in][out]) and biases
    float* W1;  // 16 x 128
    float* W2;  // 128 x 128
    float* W3;  // 128 x 8
    float* b1;
    float* b2;
    float* b3;
    // BF16 operand copies
    __nv_bfloat16* W1T;  // [128][16]  forward layer 1 (B, col)
    __nv_bfloat16* W2T;  // [128][128] forward layer 2
    __nv_bfloat16* W3T;  // [8][128]   forward layer 3
    __nv_bfloat16* W2b;  // [128][128] backward through layer 2 ([in][out])
    __nv_bfloat16* W3b;  // [128][16]  backward through layer 3 ([hidden][out], out padded to 16)
};

namespace {

__device__ __forceinline__ void mma16816(float* c, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ uint32_t pair16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.3989422804014327f * expf(-0.5f * x * x);
}

struct Smem {
    __nv_bfloat16 W1T[kHid * kIn];
    __nv_bfloat16 W2T[kHid * kHid];
    __nv_bfloat16 W3T[kOut * kHid];
    float b1[kHid], b2[kHid], b3[kOut];
};
struct SmemTrain {
    Smem f;
    __nv_bfloat16 W2b[kHid * kHid];
    __nv_bfloat16 W3b[kHid * 16];
    // staged CTA rows for the weight gradients
    __nv_bfloat16 x[kRowsPerCta * kIn];
    __nv_bfloat16 a1[kRowsPerCta * kHid];
    __nv_bfloat16 a2[kRowsPerCta * kHid];
    __nv_bfloat16 dz1[kRowsPerCta * kHid];
    __nv_bfloat16 dz2[kRowsPerCta * kHid];
    __nv_bfloat16 dz3[kRowsPerCta * 16];
    float red[8][kHid * 2 + kOut + 1];
};

__device__ void load_weights(Smem& s, const MlpParams& p) {
    for (int i = threadIdx.x; i < kHid * kIn; i += blockDim.x) s.W1T[i] = p.W1T[i];
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) s.W2T[i] = p.W2T[i];
    for (int i = threadIdx.x; i < kOut * kHid; i += blockDim.x) s.W3T[i] = p.W3T[i];
    for (int i = threadIdx.x; i < kHid; i += blockDim.x) {
        s.b1[i] = p.b1[i];
        s.b2[i] = p.b2[i];
    }
    if (threadIdx.x < kOut) s.b3[threadIdx.x] = p.b3[threadIdx.x];
}

// A fragment of the 16-row input tile (rows r0.., 16 features, row stride kIn), zero rows beyond n.
__device__ __forceinline__ void load_x(const __nv_bfloat16* X, int r0, int n, uint32_t* a) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int ra = r0 + g, rb = r0 + g + 8;
    a[0] = ra < n ? ld32(X + (size_t)ra * kIn + 2 * t) : 0u;
    a[1] = rb < n ? ld32(X + (size_t)rb * kIn + 2 * t) : 0u;
    a[2] = ra < n ? ld32(X + (size_t)ra * kIn + 2 * t + 8) : 0u;
    a[3] = rb < n ? ld32(X + (size_t)rb * kIn + 2 * t + 8) : 0u;
}

// Layer 1 pre-activations (16 x 128) for one warp.
__device__ __forceinline__ void layer1(const Smem& s, const uint32_t* ax, float (*z)[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const uint32_t b[2] = {ld32(&s.W1T[(8 * j + g) * kIn + 2 * t]), ld32(&s.W1T[(8 * j + g) * kIn + 2 * t + 8])};
        z[j][0] = s.b1[8 * j + 2 * t];
        z[j][1] = s.b1[8 * j + 2 * t + 1];
        z[j][2] = z[j][0];
        z[j][3] = z[j][1];
        mma16816(z[j], ax, b);
    }
}

// 16x128 activation (FP32 fragments) -> 8 BF16 A fragments.
__device__ __forceinline__ void to_afrag(float (*c)[4], uint32_t (*a)[4]) {
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        a[kk][0] = pack_bf16(c[2 * kk][0], c[2 * kk][1]);
        a[kk][1] = pack_bf16(c[2 * kk][2], c[2 * kk][3]);
        a[kk][2] = pack_bf16(c[2 * kk + 1][0], c[2 * kk + 1][1]);
        a[kk][3] = pack_bf16(c[2 * kk + 1][2], c[2 * kk + 1][3]);
    }
}

// C (16 x 128) = A (16 x 128, 8 k-steps) * B, B from [n][k] storage with row stride 128, plus bias.
__device__ __forceinline__ void layer_hh(const __nv_bfloat16* BT, const float* bias, uint32_t (*a)[4],
                                         float (*c)[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        c[j][0] = bias ? bias[8 * j + 2 * t] : 0.f;
        c[j][1] = bias ? bias[8 * j + 2 * t + 1] : 0.f;
        c[j][2] = c[j][0];
        c[j][3] = c[j][1];
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const uint32_t b[2] = {ld32(&BT[(8 * j + g) * kHid + 16 * kk + 2 * t]),
                                   ld32(&BT[(8 * j + g) * kHid + 16 * kk + 2 * t + 8])};
            mma16816(c[j], a[kk], b);
        }
    }
}

__device__ __forceinline__ void layer3(const Smem& s, uint32_t (*a)[4], float* c) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    c[0] = s.b3[2 * t];
    c[1] = s.b3[2 * t + 1];
    c[2] = c[0];
    c[3] = c[1];
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        const uint32_t b[2] = {ld32(&s.W3T[g * kHid + 16 * kk + 2 * t]), ld32(&s.W3T[g * kHid + 16 * kk + 2 * t + 8])};
        mma16816(c, a[kk], b);
    }
}

__global__ void __launch_bounds__(256) k_mlp_forward(MlpParams p, const __nv_bfloat16* __restrict__ X, int n,
                                                     float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& s = *reinterpret_cast<Smem*>(smem_raw);
    load_weights(s, p);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int r0 = blockIdx.x * kRowsPerCta + warp * 16;
    if (r0 >= n) return;
    uint32_t ax[4];
    load_x(X, r0, n, ax);
    float z[16][4];
    layer1(s, ax, z);
#pragma unroll
    for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) z[j][e] = gelu(z[j][e]);
    uint32_t a[8][4];
    to_afrag(z, a);
    layer_hh(s.W2T, s.b2, a, z);
#pragma unroll
    for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) z[j][e] = gelu(z[j][e]);
    to_afrag(z, a);
    float o[4];
    layer3(s, a, o);
    const int ra = r0 + g, rb = r0 + g + 8;
    if (ra < n) { out[(size_t)ra * kOut + 2 * t] = o[0]; out[(size_t)ra * kOut + 2 * t + 1] = o[1]; }
    if (rb < n) { out[(size_t)rb * kOut + 2 * t] = o[2]; out[(size_t)rb * kOut + 2 * t + 1] = o[3]; }
}

// Column sums over the warp's 16 rows of a 16x8 FP32 fragment (valid in lanes 0..3: cols 2t, 2t+1).
__device__ __forceinline__ void colsum(const float* c, float& s0, float& s1) {
    s0 = c[0] + c[2];
    s1 = c[1] + c[3];
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
}

// One training step over rows [128*blockIdx, +128): MSE(out[:, :3], Y) / n_total, per-CTA gradient partials.
__global__ void __launch_bounds__(256) k_mlp_train(MlpParams p, const __nv_bfloat16* __restrict__ X,
                                                   const float* __restrict__ Y, int n, float inv_n,
                                                   float* __restrict__ part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemTrain& s = *reinterpret_cast<SmemTrain*>(smem_raw);
    load_weights(s.f, p);
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) s.W2b[i] = p.W2b[i];
    for (int i = threadIdx.x; i < kHid * 16; i += blockDim.x) s.W3b[i] = p.W3b[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int rl = warp * 16;  // local row base
    const int r0 = blockIdx.x * kRowsPerCta + rl;
    // Rows of the warp's tiles are staged in shared memory as soon as they are final (A-fragment order back
    // to row-major), so that only the packed GELU derivatives stay live across the backward pass.
    auto stage = [&](__nv_bfloat16* dst, int ld, const uint32_t (*fr)[4], int ksteps) {
        for (int kk = 0; kk < ksteps; ++kk) {
            *reinterpret_cast<uint32_t*>(&dst[(rl + g) * ld + 16 * kk + 2 * t]) = fr[kk][0];
            *reinterpret_cast<uint32_t*>(&dst[(rl + g + 8) * ld + 16 * kk + 2 * t]) = fr[kk][1];
            *reinterpret_cast<uint32_t*>(&dst[(rl + g) * ld + 16 * kk + 2 * t + 8]) = fr[kk][2];
            *reinterpret_cast<uint32_t*>(&dst[(rl + g + 8) * ld + 16 * kk + 2 * t + 8]) = fr[kk][3];
        }
    };
    // ---- forward ----
    uint32_t ax[1][4];
    load_x(X, r0, n, ax[0]);
    stage(s.x, kIn, ax, 1);
    float c[16][4];
    layer1(s.f, ax[0], c);  // z1
    // gelu'(z1) and gelu'(z2) are parked (BF16, accumulator order) in the dz1 / dz2 tiles, which each thread
    // later overwrites at the same positions with its own dz values
    auto park = [&](__nv_bfloat16* dst, int j, uint32_t lo, uint32_t hi) {
        *reinterpret_cast<uint32_t*>(&dst[(rl + g) * kHid + 8 * j + 2 * t]) = lo;
        *reinterpret_cast<uint32_t*>(&dst[(rl + g + 8) * kHid + 8 * j + 2 * t]) = hi;
    };
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        park(s.dz1, j, pack_bf16(gelu_d(c[j][0]), gelu_d(c[j][1])), pack_bf16(gelu_d(c[j][2]), gelu_d(c[j][3])));
#pragma unroll
        for (int e = 0; e < 4; ++e) c[j][e] = gelu(c[j][e]);
    }
    uint32_t af[8][4];
    to_afrag(c, af);  // a1
    stage(s.a1, kHid, af, 8);
    layer_hh(s.f.W2T, s.f.b2, af, c);  // z2
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        park(s.dz2, j, pack_bf16(gelu_d(c[j][0]), gelu_d(c[j][1])), pack_bf16(gelu_d(c[j][2]), gelu_d(c[j][3])));
#pragma unroll
        for (int e = 0; e < 4; ++e) c[j][e] = gelu(c[j][e]);
    }
    to_afrag(c, af);  // a2
    stage(s.a2, kHid, af, 8);
    float o[4];
    layer3(s.f, af, o);
    // ---- loss gradient dz3 = 2 (pred - y) / n (3 used outputs), and the loss ----
    const int ra = r0 + g, rb = r0 + g + 8;
    float dz3[4] = {0.f, 0.f, 0.f, 0.f}, lsum = 0.f;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int row = e < 2 ? ra : rb, col = 2 * t + (e & 1);
        if (row < n && col < kOutUsed) {
            const float d = o[e] - Y[(size_t)row * kOutUsed + col];
            dz3[e] = 2.f * d * inv_n;
            lsum += d * d;
        }
    }
    // ---- backward ----
    const uint32_t adz3[1][4] = {{pack_bf16(dz3[0], dz3[1]), pack_bf16(dz3[2], dz3[3]), 0u, 0u}};
    stage(s.dz3, 16, adz3, 1);
    float bs[2];
    colsum(dz3, bs[0], bs[1]);
    if (lane < 4) {
        s.red[warp][2 * kHid + 2 * lane] = bs[0];
        s.red[warp][2 * kHid + 2 * lane + 1] = bs[1];
    }
    float ls = lsum;
#pragma unroll
    for (int of = 16; of > 0; of >>= 1) ls += __shfl_xor_sync(0xffffffffu, ls, of);
    if (lane == 0) s.red[warp][2 * kHid + kOut] = ls;
    auto unpack_mul = [&](float* cj, const __nv_bfloat16* src, int j) {
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&src[(rl + g) * kHid + 8 * j + 2 * t]));
        const float2 hi =
            __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&src[(rl + g + 8) * kHid + 8 * j + 2 * t]));
        cj[0] *= lo.x;
        cj[1] *= lo.y;
        cj[2] *= hi.x;
        cj[3] *= hi.y;
    };
    // da2 = dz3 W3^T  (K = outputs padded to 16); dz2 = da2 * gelu'(z2)
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
        const uint32_t b[2] = {ld32(&s.W3b[(8 * j + g) * 16 + 2 * t]), ld32(&s.W3b[(8 * j + g) * 16 + 2 * t + 8])};
        mma16816(c[j], adz3[0], b);
        unpack_mul(c[j], s.dz2, j);
        colsum(c[j], bs[0], bs[1]);
        if (lane < 4) {
            s.red[warp][kHid + 8 * j + 2 * lane] = bs[0];
            s.red[warp][kHid + 8 * j + 2 * lane + 1] = bs[1];
        }
    }
    to_afrag(c, af);  // dz2
    stage(s.dz2, kHid, af, 8);
    // da1 = dz2 W2^T, B from W2b ([in][out]); dz1 = da1 * gelu'(z1)
    layer_hh(s.W2b, nullptr, af, c);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        unpack_mul(c[j], s.dz1, j);
        colsum(c[j], bs[0], bs[1]);
        if (lane < 4) {
            s.red[warp][8 * j + 2 * lane] = bs[0];
            s.red[warp][8 * j + 2 * lane + 1] = bs[1];
        }
    }
    to_afrag(c, af);  // dz1
    stage(s.dz1, kHid, af, 8);
    __syncthreads();
    float* P = part + (size_t)blockIdx.x * kPartSize;
    // biases and loss (fixed warp order)
    for (int i = threadIdx.x; i < 2 * kHid + kOut + 1; i += blockDim.x) {
        float v = 0.f;
        for (int w = 0; w < 8; ++w) v += s.red[w][i];
        if (i < kHid) P[kPartB1 + i] = v;
        else if (i < 2 * kHid) P[kPartB2 + i - kHid] = v;
        else if (i < 2 * kHid + kOut) P[kPartB3 + i - 2 * kHid] = v;
        else P[kPartLoss] = v;
    }
    // ---- weight gradients over the CTA's 128 rows: D[m][n] = sum_r L[r][m] R[r][n] ----
    // A[m][k] = L[k][m] (transposed tile), B[k][n] = R[k][n].
    auto wgrad = [&](const __nv_bfloat16* L, int ldl, int m0, const __nv_bfloat16* R, int ldr, int n0, float* acc) {
        acc[0] = acc[1] = acc[2] = acc[3] = 0.f;
        for (int kk = 0; kk < kRowsPerCta / 16; ++kk) {
            const int k0 = 16 * kk;
            uint32_t a[4], b[2];
            a[0] = pair16(L[(k0 + 2 * t) * ldl + m0 + g], L[(k0 + 2 * t + 1) * ldl + m0 + g]);
            a[1] = pair16(L[(k0 + 2 * t) * ldl + m0 + g + 8], L[(k0 + 2 * t + 1) * ldl + m0 + g + 8]);
            a[2] = pair16(L[(k0 + 2 * t + 8) * ldl + m0 + g], L[(k0 + 2 * t + 9) * ldl + m0 + g]);
            a[3] = pair16(L[(k0 + 2 * t + 8) * ldl + m0 + g + 8], L[(k0 + 2 * t + 9) * ldl + m0 + g + 8]);
            b[0] = pair16(R[(k0 + 2 * t) * ldr + n0 + g], R[(k0 + 2 * t + 1) * ldr + n0 + g]);
            b[1] = pair16(R[(k0 + 2 * t + 8) * ldr + n0 + g], R[(k0 + 2 * t + 9) * ldr + n0 + g]);
            mma16816(acc, a, b);
        }
    };
    auto store = [&](float* dst, int ld, int m0, int n0, const float* acc) {
        dst[(m0 + g) * ld + n0 + 2 * t] = acc[0];
        dst[(m0 + g) * ld + n0 + 2 * t + 1] = acc[1];
        dst[(m0 + g + 8) * ld + n0 + 2 * t] = acc[2];
        dst[(m0 + g + 8) * ld + n0 + 2 * t + 1] = acc[3];
    };
    // dW2 [in][out] = a1^T dz2: warp owns input rows [16w, 16w+16)
    for (int j = 0; j < 16; ++j) {
        float acc[4];
        wgrad(s.a1, kHid, 16 * warp, s.dz2, kHid, 8 * j, acc);
        store(P + kPartW2, kHid, 16 * warp, 8 * j, acc);
    }
    // dW1 [in=16][out] = x^T dz1: warp owns output n-tiles 2w, 2w+1
    for (int jj = 0; jj < 2; ++jj) {
        float acc[4];
        wgrad(s.x, kIn, 0, s.dz1, kHid, 8 * (2 * warp + jj), acc);
        store(P + kPartW1, kHid, 0, 8 * (2 * warp + jj), acc);
    }
    // dW3 [hidden][out=8] = a2^T dz3: warp owns hidden rows [16w, 16w+16)
    {
        float acc[4];
        wgrad(s.a2, kHid, 16 * warp, s.dz3, 16, 0, acc);
        store(P + kPartW3, kOut, 16 * warp, 0, acc);
    }
}

// Sum of the CTA partials (fixed order), AdamW on the FP32 masters, BF16 re-pack; one thread per parameter.
__global__ void k_mlp_adamw(MlpParams p, const float* __restrict__ part, int nblocks, float lr, float beta1,
                            float beta2, float eps, float wd, int step, float* __restrict__ m, float* __restrict__ v,
                            float* __restrict__ grad_out, float* __restrict__ loss_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && loss_out) {
        float l = 0.f;
        for (int b = 0; b < nblocks; ++b) l += part[(size_t)b * kPartSize + kPartLoss];
        *loss_out = l;
    }
    if (i >= kPartLoss) return;
    float gsum = 0.f;
    for (int b = 0; b < nblocks; ++b) gsum += part[(size_t)b * kPartSize + i];
    // masked entries: the unused input column 15, unused outputs 3..7
    bool used = true;
    float* w = nullptr;
    bool decay = true;
    if (i < kPartW2) {
        const int in = i / kHid;
        used = in < 15;
        w = p.W1 + i;
    } else if (i < kPartW3) {
        w = p.W2 + (i - kPartW2);
    } else if (i < kPartB1) {
        const int o = (i - kPartW3) % kOut;
        used = o < kOutUsed;
        w = p.W3 + (i - kPartW3);
    } else if (i < kPartB2) {
        w = p.b1 + (i - kPartB1);
        decay = false;
    } else if (i < kPartB3) {
        w = p.b2 + (i - kPartB2);
        decay = false;
    } else {
        const int o = i - kPartB3;
        used = o < kOutUsed;
        w = p.b3 + o;
        decay = false;
    }
    if (grad_out) grad_out[i] = used ? gsum : 0.f;
    if (!used || lr == 0.f) return;
    const float b1c = 1.f - powf(beta1, (float)step), b2c = 1.f - powf(beta2, (float)step);
    m[i] = beta1 * m[i] + (1.f - beta1) * gsum;
    v[i] = beta2 * v[i] + (1.f - beta2) * gsum * gsum;
    const float mh = m[i] / b1c, vh = v[i] / b2c;
    float wv = *w;
    if (decay) wv -= lr * wd * wv;
    wv -= lr * mh / (sqrtf(vh) + eps);
    *w = wv;
}

__global__ void k_mlp_pack(MlpParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kIn * kHid) {  // W1 [in][out] -> W1T [out][in]
        const int in = i / kHid, o = i % kHid;
        p.W1T[o * kIn + in] = __float2bfloat16_rn(in < 15 ? p.W1[i] : 0.f);
    }
    if (i < kHid * kHid) {  // W2 [in][out] -> W2T [out][in] and W2b = W2
        const int in = i / kHid, o = i % kHid;
        const __nv_bfloat16 w = __float2bfloat16_rn(p.W2[i]);
        p.W2T[o * kHid + in] = w;
        p.W2b[i] = w;
    }
    if (i < kHid * kOut) {  // W3 [hidden][out] -> W3T [out][hidden], W3b [hidden][16]
        const int h = i / kOut, o = i % kOut;
        const __nv_bfloat16 w = __float2bfloat16_rn(o < kOutUsed ? p.W3[i] : 0.f);
        p.W3T[o * kHid + h] = w;
        p.W3b[h * 16 + o] = w;
        p.W3b[h * 16 + o + 8] = __float2bfloat16_rn(0.f);
    }
}

}  // namespace

size_t mlp_forward_smem() { return sizeof(Smem); }
size_t mlp_train_smem() { return sizeof(SmemTrain); }

void launch_mlp_forward(const MlpParams& p, const void* X, int n, float* out, cudaStream_t st) {
    // per device and cheap: set on every call
    cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
    const int blocks = (n + kRowsPerCta - 1) / kRowsPerCta;
    if (blocks > 0)
        k_mlp_forward<<<blocks, 256, sizeof(Smem), st>>>(p, reinterpret_cast<const __nv_bfloat16*>(X), n, out);
}

int launch_mlp_train(const MlpParams& p, const void* X, const float* Y, int n, float* part, cudaStream_t st) {
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SmemTrain));
    const int blocks = (n + kRowsPerCta - 1) / kRowsPerCta;
    if (blocks > 0)
        k_mlp_train<<<blocks, 256, sizeof(SmemTrain), st>>>(p, reinterpret_cast<const __nv_bfloat16*>(X), Y, n,
                                                             1.f / (float)n, part);
    return blocks;
}

void launch_mlp_adamw(const MlpParams& p, const float* part, int nblocks, float lr, float b1, float b2, float eps,
                      float wd, int step, float* m, float* v, float* grad_out, float* loss_out, cudaStream_t st) {
    k_mlp_adamw<<<(kPartLoss + 255) / 256, 256, 0, st>>>(p, part, nblocks, lr, b1, b2, eps, wd, step, m, v, grad_out,
                                                         loss_out);
    k_mlp_pack<<<(kHid * kHid + 255) / 256, 256, 0, st>>>(p);
}

void launch_mlp_pack(const MlpParams& p, cudaStream_t st) { k_mlp_pack<<<(kHid * kHid + 255) / 256, 256, 0, st>>>(p); }

int mlp_part_size() { return kPartSize; }
int mlp_param_count() { return kPartLoss; }
int mlp_rows_per_block() { return kRowsPerCta; }
int mlp_packed_count() { return kHid * kIn + kHid * kHid + kOut * kHid + kHid * kHid + kHid * 16; }

static MlpParams flat_params(float* master, void* packed) {
    MlpParams p;
    p.W1 = master + kPartW1;
    p.W2 = master + kPartW2;
    p.W3 = master + kPartW3;
    p.b1 = master + kPartB1;
    p.b2 = master + kPartB2;
    p.b3 = master + kPartB3;
    __nv_bfloat16* b = reinterpret_cast<__nv_bfloat16*>(packed);
    p.W1T = b;
    p.W2T = p.W1T + kHid * kIn;
    p.W3T = p.W2T + kHid * kHid;
    p.W2b = p.W3T + kOut * kHid;
    p.W3b = p.W2b + kHid * kHid;
    return p;
}

void mlp_pack_flat(float* master, void* packed, cudaStream_t st) { launch_mlp_pack(flat_params(master, packed), st); }
void mlp_forward_flat(float* master, void* packed, const void* X, int n, float* out, cudaStream_t st) {
    launch_mlp_forward(flat_params(master, packed), X, n, out, st);
}
void launch_mlp_forward_tc(const void* W1T, const void* W2T, const void* W3T, const float* b1, const float* b2,
                           const float* b3, const void* X, int n, float* out, int* err, int max_ctas, cudaStream_t st);
void mlp_forward_tc_flat(float* master, void* packed, const void* X, int n, float* out, int* err, cudaStream_t st) {
    const MlpParams p = flat_params(master, packed);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    launch_mlp_forward_tc(p.W1T, p.W2T, p.W3T, p.b1, p.b2, p.b3, X, n, out, err, 2 * (sms > 0 ? sms : 148), st);
}
int mlp_train_flat(float* master, void* packed, const void* X, const float* Y, int n, float* part, cudaStream_t st) {
    return launch_mlp_train(flat_params(master, packed), X, Y, n, part, st);
}
void mlp_adamw_flat(float* master, void* packed, const float* part, int nblocks, float lr, float b1, float b2,
                    float eps, float wd, int step, float* m, float* v, float* grad_out, float* loss_out,
                    cudaStream_t st) {
    launch_mlp_adamw(flat_params(master, packed), part, nblocks, lr, b1, b2, eps, wd, step, m, v, grad_out, loss_out,
                     st);
}

}  // namespace dphd

namespace dphd {

namespace {

// Per-node features (16): displacement (q - X)/dx, last step (q - q_prev)/dx, the last step's correction
// (q - q_tilde_prev)/dx (0 without a previous prediction), h^2/m f_ext/dx, height above the contact plane /dx,
// log10 of the node's mean PD stiffness / 7, Dirichlet flag, and the node's current contact multiplier (the
// previous frame's lambda) in the output's scale h^2/(m dx), clipped at 4 (0 off the contact set); also the inertial
// prediction q_tilde = q + h v + h^2/m (f_ext + m g) (the warm start is q_tilde + dx * MLP).
__global__ void k_mlp_features(FeatureArgs a, const double* __restrict__ q, const double* __restrict__ qp,
                               const double* __restrict__ v, const double* __restrict__ f,
                               const double* __restrict__ prev_base, const float* __restrict__ lam_node,
                               __nv_bfloat16* __restrict__ X, double* __restrict__ base) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    float feat[16];
    double qt[3];
    for (int d = 0; d < 3; ++d) {
        const int k = 3 * i + d;
        qt[d] = q[k] + a.h * v[k] + a.h2m * f[k] + a.h2m * a.gforce[d];
        base[k] = qt[d];
        feat[d] = (float)((q[k] - a.X[k]) * a.inv_dx);
        feat[3 + d] = (float)((q[k] - qp[k]) * a.inv_dx);
        feat[6 + d] = prev_base ? (float)((q[k] - prev_base[k]) * a.inv_dx) : 0.f;
        feat[9 + d] = (float)(a.h2m * f[k] * a.inv_dx);
    }
    // height above the contact plane in cells, clamped to [-2, 2]: only the layer next to the plane is told apart
    // (unclamped, the feature would grow with the body's size and leave the training range on larger meshes)
    feat[12] = a.plane ? fminf(2.f, fmaxf(-2.f, (float)((a.pn[0] * q[3 * i] + a.pn[1] * q[3 * i + 1] +
                                                         a.pn[2] * q[3 * i + 2] + a.poff) * a.inv_dx)))
                       : 0.f;
    feat[13] = a.wlog[i];
    feat[14] = a.fixed[i] ? 1.f : 0.f;
    feat[15] = lam_node ? lam_node[i] : 0.f;
    for (int c = 0; c < 16; ++c) X[(size_t)i * 16 + c] = __float2bfloat16_rn(feat[c]);
}

__global__ void k_mlp_apply(int n3, const double* __restrict__ base, const float* __restrict__ out, double dx,
                            const unsigned char* __restrict__ fixed_dof, const double* __restrict__ fval,
                            double* __restrict__ q_init) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n3) return;
    q_init[k] = fixed_dof[k] ? fval[k] : base[k] + dx * (double)out[(size_t)(k / 3) * 8 + k % 3];
}

// The scaled multipliers are clipped at kLamClip in the feature and the target: impact frames reach tens of the
// resting values, and a few such rows would dominate the squared loss of a warm start.
constexpr double kLamClip = 4.0;

// Training targets, 4 per node: (q_next - q_tilde)/dx and the frame's contact multiplier in the scale h^2/(m dx)
// (column 3: 0 here, the candidates' values are written by k_mlp_target_lambda after this kernel).
__global__ void k_mlp_target(int n3, const double* __restrict__ q_next, const double* __restrict__ base,
                             double inv_dx, float* __restrict__ Y) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n3) return;
    Y[(size_t)(k / 3) * 4 + k % 3] = (float)((q_next[k] - base[k]) * inv_dx);
    if (k % 3 == 0) Y[(size_t)(k / 3) * 4 + 3] = 0.f;
}

// Column 3: the change of the multiplier over the frame, (lambda_final - lambda_prev) * scale, clipped to
// [-kLamClip, kLamClip] (the network predicts a correction of the previous frame's multiplier).
__global__ void k_mlp_target_lambda(int K, const int* __restrict__ cand, const double* __restrict__ lam,
                                    const double* __restrict__ lam_prev, double scale, float* __restrict__ Y) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const double d = (lam[k] - (lam_prev ? lam_prev[k] : 0.0)) * scale;
    Y[(size_t)cand[k] * 4 + 3] = (float)fmax(-kLamClip, fmin(d, kLamClip));
}

// Node-indexed contact multipliers in the network's scale (the lambda feature): 0 off the candidate set.
__global__ void k_mlp_lambda_zero(int n, float* __restrict__ lam_node) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lam_node[i] = 0.f;
}
__global__ void k_mlp_lambda_scatter(int K, const int* __restrict__ cand, const double* __restrict__ lam, double scale,
                                     float* __restrict__ lam_node) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) lam_node[cand[k]] = (float)fmin(lam[k] * scale, kLamClip);
}

// The predicted initial contact multipliers: lambda_k <- max(0, lambda_k + out[node_k][3] / scale), the previous
// frame's multiplier corrected by the network.
__global__ void k_mlp_lambda_apply(int K, const int* __restrict__ cand, const float* __restrict__ out, double inv_scale,
                                   double* __restrict__ lam) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const double v = lam[k] + (double)out[(size_t)cand[k] * 8 + 3] * inv_scale;
    lam[k] = v > 0.0 ? v : 0.0;
}

}  // namespace

void launch_mlp_features(const FeatureArgs& a, const double* q, const double* qp, const double* v, const double* f,
                         const double* prev_base, const float* lam_node, void* X, double* base, cudaStream_t st) {
    k_mlp_features<<<(a.n + 255) / 256, 256, 0, st>>>(a, q, qp, v, f, prev_base, lam_node,
                                                      reinterpret_cast<__nv_bfloat16*>(X), base);
}
void launch_mlp_lambda_nodes(int n, int K, const int* cand, const double* lam, double scale, float* lam_node,
                             cudaStream_t st) {
    k_mlp_lambda_zero<<<(n + 255) / 256, 256, 0, st>>>(n, lam_node);
    if (K > 0) k_mlp_lambda_scatter<<<(K + 255) / 256, 256, 0, st>>>(K, cand, lam, scale, lam_node);
}
void launch_mlp_target_lambda(int K, const int* cand, const double* lam, const double* lam_prev, double scale,
                              float* Y, cudaStream_t st) {
    if (K > 0) k_mlp_target_lambda<<<(K + 255) / 256, 256, 0, st>>>(K, cand, lam, lam_prev, scale, Y);
}
void launch_mlp_lambda_apply(int K, const int* cand, const float* out, double inv_scale, double* lam, cudaStream_t st) {
    if (K > 0) k_mlp_lambda_apply<<<(K + 255) / 256, 256, 0, st>>>(K, cand, out, inv_scale, lam);
}
void launch_mlp_apply(int n3, const double* base, const float* out, double dx, const unsigned char* fixed_dof,
                      const double* fval, double* q_init, cudaStream_t st) {
    k_mlp_apply<<<(n3 + 255) / 256, 256, 0, st>>>(n3, base, out, dx, fixed_dof, fval, q_init);
}
// The learned start at the contact candidates.  Mode 1: a candidate in contact in the previous frame (lambda > 0)
// keeps its previous gap (a resting contact stays at rest), the others are moved out of the half space if the
// prediction penetrates it; the tangential components stay as predicted.  Mode 2: a candidate in contact keeps
// its previous position altogether (the plain solver's start there), the others keep the prediction.
__global__ void k_ws_contact_start(int K, int mode, const int* __restrict__ cand, const double* __restrict__ lam,
                                   double n0, double n1, double n2, double off,
                                   const unsigned char* __restrict__ fixed_dof, const double* __restrict__ q_prev,
                                   double* __restrict__ q_init) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const int i = cand[k];
    if (fixed_dof[3 * i] || fixed_dof[3 * i + 1] || fixed_dof[3 * i + 2]) return;
    double* x = q_init + 3 * (size_t)i;
    const double* xp = q_prev + 3 * (size_t)i;
    if (mode == 2) {
        if (lam[k] > 0.0) {
            x[0] = xp[0];
            x[1] = xp[1];
            x[2] = xp[2];
        }
        return;
    }
    const double d = n0 * x[0] + n1 * x[1] + n2 * x[2] + off;
    const double dp = n0 * xp[0] + n1 * xp[1] + n2 * xp[2] + off;
    const double target = lam[k] > 0.0 ? dp : (d < 0.0 ? 0.0 : d);
    const double s = target - d;
    x[0] += s * n0;
    x[1] += s * n1;
    x[2] += s * n2;
}

void launch_ws_contact_start(int K, int mode, const int* cand, const double* lam, const double* n, double off,
                             const unsigned char* fixed_dof, const double* q_prev, double* q_init, cudaStream_t st) {
    if (K > 0)
        k_ws_contact_start<<<(K + 255) / 256, 256, 0, st>>>(K, mode, cand, lam, n[0], n[1], n[2], off, fixed_dof,
                                                             q_prev, q_init);
}

void launch_mlp_target(int n3, const double* q_next, const double* base, double inv_dx, float* Y, cudaStream_t st) {
    k_mlp_target<<<(n3 + 255) / 256, 256, 0, st>>>(n3, q_next, base, inv_dx, Y);
}

}  // namespace dphd
