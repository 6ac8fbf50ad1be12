// Warm-start MLP inference (16 -> 128 -> 128 -> 8, GELU; the first 4 outputs are used) on the 5th-generation
// tensor cores: tcgen05.mma with
// BF16 operands in shared memory, FP32 accumulators in tensor memory (TMEM), read back with tcgen05.ld.
//
// One CTA of 128 threads works on tiles of 128 rows (nodes); thread t owns row t, which is TMEM lane t of every
// accumulator (M = 128, cta_group::1).  Per tile:
//   layer 1: D1[128 x 128] = X[128 x 16] W1^T        1 MMA  (K = 16 per instruction)
//   layer 2: D2[128 x 128] = gelu(D1 + b1) W2^T       8 MMAs
//   layer 3: D3[128 x 16]  = gelu(D2 + b2) W3^T       8 MMAs (N = 16: outputs 0..7 used, 8..15 zero rows)
// Between layers each thread reads its row of the accumulator (tcgen05.ld 32x32b), adds the bias, applies
// GELU, rounds to BF16 and writes the row into the next layer's A tile; thread 0 issues the
// MMAs and commits them to an mbarrier that every thread waits on (bounded).  The weights are staged into
// shared memory once per CTA; CTAs loop over tiles.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout of the UMMA descriptors: "core matrices"
// of 8 rows x 16 bytes (8 BF16 along K) stored contiguously (128 B), ordered [k / 8][row / 8].  For the MMA of
// K-slice ki the descriptor starts at core column 2 ki; the two 8-wide K halves of the slice are LBO =
// (rows / 8) * 128 bytes apart and consecutive 8-row groups SBO = 128 bytes apart.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace dphd {

namespace {

constexpr int kTcRows = 128;                     // M: rows per tile, one per thread
constexpr int kIn = 16, kHid = 128, kOut8 = 8, kN3 = 16;
constexpr uint32_t kTmemCols = 128;              // one FP32 accumulator of N <= 128 columns
constexpr long long kWaitPolls = 1ll << 22;      // bound of every mbarrier wait

struct __align__(128) SmemTc {
    __nv_bfloat16 A1[kTcRows * kIn];   // X tile
    __nv_bfloat16 A2[kTcRows * kHid];  // layer-2 input, then layer-3 input
    __nv_bfloat16 B1[kHid * kIn];      // W1^T  [N = 128][K = 16]
    __nv_bfloat16 B2[kHid * kHid];     // W2^T  [N = 128][K = 128]
    __nv_bfloat16 B3[kN3 * kHid];      // W3^T  [N = 16][K = 128], rows 8..15 zero
    float b1[kHid], b2[kHid], b3[kN3];
    unsigned long long mbar;
    uint32_t tmem_base;
};

// Element offset of (row, k) in a K-major no-swizzle canonical tile of `rows` rows.
__device__ __forceinline__ int cm_off(int row, int k, int rows) {
    return ((k >> 3) * (rows >> 3) + (row >> 3)) * 64 + (row & 7) * 8 + (k & 7);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor (no swizzle, K-major): start address, leading (K) and stride (row-group) byte
// offsets, all in 16-byte units; version 1 (sm_100); base offset 0; layout type 0.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, N and M encoded.
__host__ __device__ constexpr uint32_t make_idesc(int M, int N) {
    return (1u << 4)                       // D format: F32
           | (1u << 7)                     // A format: BF16
           | (1u << 10)                    // B format: BF16
           | ((uint32_t)(N >> 3) << 17)    // N / 8
           | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase, long long polls) {
    for (long long i = 0; i < polls; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (taddr: the warp's lane block and the first column); the
// wait is in the same asm statement, so no use of the outputs can be scheduled before it.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// bias + GELU on 32 columns [c0, c0 + 32) of this thread's row; written as BF16 into the K-major A tile.
__device__ __forceinline__ void gelu_to_tile(const float* v, const float* bias, int c0, int row,
                                             __nv_bfloat16* A) {
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        uint4 w;
        w.x = pack2(gelu(v[8 * g + 0] + bias[c0 + 8 * g + 0]), gelu(v[8 * g + 1] + bias[c0 + 8 * g + 1]));
        w.y = pack2(gelu(v[8 * g + 2] + bias[c0 + 8 * g + 2]), gelu(v[8 * g + 3] + bias[c0 + 8 * g + 3]));
        w.z = pack2(gelu(v[8 * g + 4] + bias[c0 + 8 * g + 4]), gelu(v[8 * g + 5] + bias[c0 + 8 * g + 5]));
        w.w = pack2(gelu(v[8 * g + 6] + bias[c0 + 8 * g + 6]), gelu(v[8 * g + 7] + bias[c0 + 8 * g + 7]));
        *reinterpret_cast<uint4*>(A + cm_off(row, c0 + 8 * g, kTcRows)) = w;
    }
}

__global__ void __launch_bounds__(128) k_mlp_forward_tc(const __nv_bfloat16* __restrict__ W1T,
                                                        const __nv_bfloat16* __restrict__ W2T,
                                                        const __nv_bfloat16* __restrict__ W3T,
                                                        const float* __restrict__ b1, const float* __restrict__ b2,
                                                        const float* __restrict__ b3,
                                                        const __nv_bfloat16* __restrict__ X, int n,
                                                        float* __restrict__ out, int* __restrict__ err,
                                                        long long wait_polls) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    SmemTc& s = *reinterpret_cast<SmemTc*>(smem_raw);
    const int t = threadIdx.x, warp = t >> 5;
    // weights and biases, once per CTA, into the canonical layouts: 8 consecutive K values of one row are one
    // 16-byte core-matrix row, so every copy is a 16-byte load and store
    for (int c = t; c < kHid * kIn / 8; c += blockDim.x)
        *reinterpret_cast<uint4*>(s.B1 + cm_off(c >> 1, (c & 1) * 8, kHid)) =
            *reinterpret_cast<const uint4*>(W1T + c * 8);
    for (int c = t; c < kHid * kHid / 8; c += blockDim.x)
        *reinterpret_cast<uint4*>(s.B2 + cm_off(c >> 4, (c & 15) * 8, kHid)) =
            *reinterpret_cast<const uint4*>(W2T + c * 8);
    for (int c = t; c < kN3 * kHid / 8; c += blockDim.x) {
        const int r = c >> 4;
        *reinterpret_cast<uint4*>(s.B3 + cm_off(r, (c & 15) * 8, kN3)) =
            r < kOut8 ? *reinterpret_cast<const uint4*>(W3T + c * 8) : make_uint4(0, 0, 0, 0);
    }
    for (int i = t; i < kHid; i += blockDim.x) {
        s.b1[i] = b1[i];
        s.b2[i] = b2[i];
    }
    if (t < kN3) s.b3[t] = t < kOut8 ? b3[t] : 0.f;
    const uint32_t mbar = smem_addr(&s.mbar);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = s.tmem_base;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 TMEM lanes
    const uint32_t id128 = make_idesc(kTcRows, kHid), id16 = make_idesc(kTcRows, kN3);
    const uint32_t a1 = smem_addr(s.A1), a2 = smem_addr(s.A2), bb1 = smem_addr(s.B1), bb2 = smem_addr(s.B2),
                   bb3 = smem_addr(s.B3);
    // descriptor byte offsets: LBO = (rows / 8) * 128 between the two K halves, SBO = 128 between row groups
    const uint32_t lbo_rows128 = (kTcRows / 8) * 128, lbo_rows16 = (kN3 / 8) * 128;
    uint32_t phase = 0;
    bool ok = true;
    // Waits for the MMAs committed to the barrier; the result is made CTA-uniform before any .sync.aligned
    // tcgen05.ld depends on it.
    auto wait_mma = [&]() -> bool {
        const bool r = __syncthreads_and(mbar_wait(mbar, phase, wait_polls));
        phase ^= 1u;
        fence_after_sync();
        return r;
    };
    // Generic-proxy shared-memory writes become visible to the tensor cores, and this thread's TMEM reads are
    // ordered before the next MMA.
    auto publish = [&]() {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
    };
    const int ntiles = (n + kTcRows - 1) / kTcRows;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int row = tile * kTcRows + t;
        // X tile: this thread's row (16 BF16 = two 16-byte core rows), zero beyond n
        uint4 x0 = make_uint4(0, 0, 0, 0), x1 = make_uint4(0, 0, 0, 0);
        if (row < n) {
            x0 = *reinterpret_cast<const uint4*>(X + (size_t)row * kIn);
            x1 = *reinterpret_cast<const uint4*>(X + (size_t)row * kIn + 8);
        }
        *reinterpret_cast<uint4*>(s.A1 + cm_off(t, 0, kTcRows)) = x0;
        *reinterpret_cast<uint4*>(s.A1 + cm_off(t, 8, kTcRows)) = x1;
        publish();
        // layer 1: one K = 16 slice
        if (t == 0) {
            mma_bf16(tmem, make_desc(a1, lbo_rows128, 128), make_desc(bb1, lbo_rows128, 128), id128, 0u);
            mma_commit(mbar);
        }
        if (!(ok = wait_mma())) break;
        float v[32];
#pragma unroll
        for (int c0 = 0; c0 < kHid; c0 += 32) {
            tmem_ld32(lane_addr + c0, v);
            gelu_to_tile(v, s.b1, c0, t, s.A2);
        }
        publish();
        // layer 2: eight K-slices of 16
        if (t == 0) {
#pragma unroll
            for (int ki = 0; ki < kHid / 16; ++ki)
                mma_bf16(tmem, make_desc(a2 + ki * 2 * lbo_rows128, lbo_rows128, 128),
                         make_desc(bb2 + ki * 2 * lbo_rows128, lbo_rows128, 128), id128, ki > 0 ? 1u : 0u);
            mma_commit(mbar);
        }
        if (!(ok = wait_mma())) break;
        // layer 2 has finished reading A2: the layer-3 input overwrites it
#pragma unroll
        for (int c0 = 0; c0 < kHid; c0 += 32) {
            tmem_ld32(lane_addr + c0, v);
            gelu_to_tile(v, s.b2, c0, t, s.A2);
        }
        publish();
        // layer 3: N = 16 (rows 8..15 of W3^T are zero)
        if (t == 0) {
#pragma unroll
            for (int ki = 0; ki < kHid / 16; ++ki)
                mma_bf16(tmem, make_desc(a2 + ki * 2 * lbo_rows128, lbo_rows128, 128),
                         make_desc(bb3 + ki * 2 * lbo_rows16, lbo_rows16, 128), id16, ki > 0 ? 1u : 0u);
            mma_commit(mbar);
        }
        if (!(ok = wait_mma())) break;
        tmem_ld16(lane_addr, v);
        if (row < n) {
            float4* o = reinterpret_cast<float4*>(out + (size_t)row * kOut8);
            o[0] = make_float4(v[0] + s.b3[0], v[1] + s.b3[1], v[2] + s.b3[2], v[3] + s.b3[3]);
            o[1] = make_float4(v[4] + s.b3[4], v[5] + s.b3[5], v[6] + s.b3[6], v[7] + s.b3[7]);
        }
        // the next tile's X write and barrier (publish) order these TMEM reads before its layer-1 MMA
    }
    if (!ok) {
        if (t == 0) atomicExch(err, 1);
        // the MMAs of the wait that gave up may still be in flight: drain them (the full bound) before TMEM goes
        __syncthreads_and(mbar_wait(mbar, phase ^ 1u, kWaitPolls));
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
}

static_assert(sizeof(SmemTc) < 200 * 1024, "shared memory of the tcgen05 MLP kernel");
static_assert(make_idesc(128, 128) == ((1u << 4) | (1u << 7) | (1u << 10) | (16u << 17) | (8u << 24)),
              "instruction descriptor");

}  // namespace

size_t mlp_tc_smem() { return sizeof(SmemTc) + 1024; }

long long g_mma_wait_polls = kWaitPolls;  // bound of the completion waits (lowered only by a failure-path test)
void set_mma_wait_polls(long long polls) { g_mma_wait_polls = polls >= 0 ? polls : kWaitPolls; }

void launch_mlp_forward_tc(const void* W1T, const void* W2T, const void* W3T, const float* b1, const float* b2,
                           const float* b3, const void* X, int n, float* out, int* err, int max_ctas,
                           cudaStream_t st) {
    const int ntiles = (n + kTcRows - 1) / kTcRows;
    if (ntiles == 0) return;
    const int smem = (int)mlp_tc_smem();
    cudaFuncSetAttribute(k_mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const int grid = ntiles < max_ctas ? ntiles : max_ctas;
    k_mlp_forward_tc<<<grid, 128, smem, st>>>(
        reinterpret_cast<const __nv_bfloat16*>(W1T), reinterpret_cast<const __nv_bfloat16*>(W2T),
        reinterpret_cast<const __nv_bfloat16*>(W3T), b1, b2, b3, reinterpret_cast<const __nv_bfloat16*>(X), n, out,
        err, g_mma_wait_polls);
}

}  // namespace dphd
