// Allocation-free A^-1 apply (x = S^T S b) for callers that must not allocate GPU memory at call time.
//
// Some callers cannot call cudaMalloc during a step: code that runs inside a memory-budgeted real-time
// loop, code embedded in another framework that owns the device allocator, or code that must never trigger
// an implicit device synchronisation (cudaMalloc/cudaFree can synchronise the device).  They set the
// deformable up once (which allocates S in HBM), then call dphd_ainv_noalloc every step: it launches kernels
// only, and keeps its temporaries in the fixed static device array below instead of allocating them.
//
// The array is kNoAllocScratchBytes (32 MiB) per GPU and stays resident for as long as the library is
// loaded on that device.  Every call shares it and it keeps the previous call's contents: each call first
// zeroes what must start at zero (its control block) and overwrites the rest before reading it.  Calls that
// overlap on the GPU (two streams, or two host threads) race on the array and must be serialised by the
// caller.  The first call on a device looks the array's device address up (cudaGetSymbolAddress, with that
// device current) and caches it; make that first call before any stream capture.  The cached address belongs
// to the device's primary context as it was then: after a cudaDeviceReset in the same process the module is
// loaded again and the cached address is stale, so this entry point is not for use across a device reset.
// The handle's device must be current (the engine checks it before the lookup).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "dphd_internal.h"
#include "kernels.cuh"

namespace dphd {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
void* g_addr[kMaxDevices] = {nullptr};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Device address of the scratch array on the current device, looked up once per device.
void* scratch_address() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    DPHD_CHECK(e == cudaSuccess, std::string("cudaGetDevice failed: ") + cudaGetErrorString(e));
    DPHD_CHECK(dev >= 0 && dev < kMaxDevices, "device index out of range for the scratch table");
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        DPHD_CHECK(e == cudaSuccess && p, std::string("cudaGetSymbolAddress(scratch) failed: ") + cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    return g_addr[dev];
}

// Zeroes the control block, then writes b (node-major, 3n) as the permuted SoA right-hand side with
// Dirichlet nodes set to zero (the same input the forward step hands to the S^T S pair) and clears the
// padding columns, all inside the scratch array.
template <typename T>
__global__ void k_noalloc_prepare(int n, int npad, const double* __restrict__ b, const unsigned char* __restrict__ fixed,
                                  const int* __restrict__ perm, size_t ctrl_off, size_t v_off) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (int)(sizeof(Ctrl) / sizeof(int))) reinterpret_cast<int*>(g_noalloc_scratch + ctrl_off)[t] = 0;
    if (t >= npad) return;
    T* v = reinterpret_cast<T*>(g_noalloc_scratch + v_off);
    if (t >= n) {
        v[t] = T(0);
        v[npad + t] = T(0);
        v[2 * (size_t)npad + t] = T(0);
        return;
    }
    const int node = perm[t];
    const bool fx = fixed[node] != 0;
    v[t] = fx ? T(0) : (T)b[3 * node];
    v[npad + t] = fx ? T(0) : (T)b[3 * node + 1];
    v[2 * (size_t)npad + t] = fx ? T(0) : (T)b[3 * node + 2];
}

template <typename T>
void run(const SpmvPlan<T>& plan, const unsigned char* fixed_node, const double* d_b, double* d_x, cudaStream_t st) {
    const int n = plan.n, npad = plan.npad;
    const size_t ctrl_off = 0;
    const size_t v_off = align256(sizeof(Ctrl));
    const size_t y_off = v_off + align256((size_t)3 * npad * sizeof(T));
    const size_t yp_off = y_off + align256((size_t)3 * npad * sizeof(T));
    const size_t xp_off = yp_off + align256((size_t)std::max(1, plan.n_items) * 3 * sizeof(T));
    const size_t need = xp_off + align256((size_t)plan.n_chunks * 3 * kTileCols * sizeof(T));
    DPHD_CHECK(need <= kNoAllocScratchBytes,
               "dphd_ainv_noalloc: this mesh needs " + std::to_string(need) + " bytes of scratch, more than the " +
                   std::to_string(kNoAllocScratchBytes) + "-byte static array; use dphd_debug_ainv or the step "
                   "entry points, which allocate their buffers");
    unsigned char* base = static_cast<unsigned char*>(scratch_address());
    SpmvPlan<T> p = plan;
    p.ypart = reinterpret_cast<T*>(base + yp_off);
    p.xpart = reinterpret_cast<T*>(base + xp_off);
    p.x_base = nullptr;
    p.yrow = nullptr;  // the S^T pass sums each row's item partials itself: no buffer outside the static array
    p.row_cnt = nullptr;
    const Ctrl* ctrl = reinterpret_cast<const Ctrl*>(base + ctrl_off);
    const int threads = 256, blocks = (std::max(npad, 64) + threads - 1) / threads;
    k_noalloc_prepare<T><<<blocks, threads, 0, st>>>(n, npad, d_b, fixed_node, plan.perm, ctrl_off, v_off);
    launch_sts<T>(p, reinterpret_cast<const T*>(base + v_off), reinterpret_cast<T*>(base + y_off), d_x, ctrl, st);
    const cudaError_t e = cudaGetLastError();
    DPHD_CHECK(e == cudaSuccess, std::string("dphd_ainv_noalloc launch failed: ") + cudaGetErrorString(e));
}

}  // namespace

void ainv_noalloc(const SpmvPlan<double>& p64, const SpmvPlan<float>& p32, const unsigned char* fixed_node,
                  const double* d_b, double* d_x, bool fp32, cudaStream_t st) {
    if (fp32) run<float>(p32, fixed_node, d_b, d_x, st);
    else run<double>(p64, fixed_node, d_b, d_x, st);
}

}  // namespace dphd
