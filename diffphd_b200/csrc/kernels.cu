// sm_100a kernels of the projective-dynamics step and its adjoint.
//
// All reductions are deterministic: fixed grids, per-block partials, and a last-arriving block that sums
// the partials in block order.  No floating-point atomics are used.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <utility>

#include "kernels.cuh"

namespace dphd {

namespace {

constexpr int kThreads = 256;

// Programmatic dependent launch.  The kernels of an iteration body are launched with programmatic stream
// serialization (launch_k below), so each grid is launched while its predecessor drains; every such kernel
// begins with pdl_enter: it lets its own successor launch, then waits (griddepcontrol.wait) until the
// predecessor grid has completed and its memory is visible, before reading anything.  Launched without the
// attribute, the wait returns at once.  Every such kernel then reads ctrl->done with an ordinary load (ordered
// after the wait's memory clobber) and branches on it before it touches data a predecessor wrote: loads through
// the read-only path (ld.global.nc, which the compiler may treat as invariant and move across the wait) stay
// behind that branch, so none is issued before the wait.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values per thread; result valid in thread 0.  `sh` holds NV * 32 doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double* v, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double s = warp_sum(v[i]);
        if (lane == 0) sh[i * 32 + wid] = s;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = lane < nw ? sh[i * 32 + lane] : 0.0;
            s = warp_sum(s);
            v[i] = s;
        }
    }
    __syncthreads();
}

// Last-block election after each block stored its partials.
__device__ __forceinline__ bool arrive_last(unsigned int* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return last;
}

// Sum NV partial values over `nb` blocks (layout part[b * NV + i]) with all threads of the calling block in a
// fixed order (thread t takes blocks t, t + blockDim, ...; then a fixed tree); result valid in thread 0.
template <int NV>
__device__ __forceinline__ void sum_partials(const double* part, int nb, double* out, double* sh) {
    double v[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] += __ldcg(part + (size_t)b * NV + i);
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int i = 0; i < NV; ++i) out[i] = v[i];
}

template <typename T>
__device__ __forceinline__ T ld_weight(const ElemEnergyDev& en, int e);
template <>
__device__ __forceinline__ double ld_weight<double>(const ElemEnergyDev& en, int e) {
    return en.per_element ? __ldg(en.w + e) : en.w_mean;
}
template <>
__device__ __forceinline__ float ld_weight<float>(const ElemEnergyDev& en, int e) {
    return en.per_element ? __ldg(en.w32 + e) : (float)en.w_mean;
}

// Deformation gradient F(i,j) = sum_a x_a[i] grad_a[j] over the element's nodes (FP64 accumulation).
template <int K>
__device__ __forceinline__ void def_grad(const int* __restrict__ E, int e, const double* __restrict__ x,
                                         const double* __restrict__ g, double* F) {
#pragma unroll
    for (int i = 0; i < 9; ++i) F[i] = 0.0;
#pragma unroll
    for (int a = 0; a < K; ++a) {
        const int node = __ldg(E + (size_t)e * K + a);
        const double x0 = x[3 * node], x1 = x[3 * node + 1], x2 = x[3 * node + 2];
        const double g0 = __ldg(g + a * 3), g1 = __ldg(g + a * 3 + 1), g2 = __ldg(g + a * 3 + 2);
        F[0] += x0 * g0; F[1] += x1 * g0; F[2] += x2 * g0;
        F[3] += x0 * g1; F[4] += x1 * g1; F[5] += x2 * g1;
        F[6] += x0 * g2; F[7] += x1 * g2; F[8] += x2 * g2;
    }
}

// ------------------------------------------------------------------------------------------------
// Forward local step (deformable_projective_dynamics_forward.cpp:186-292), one thread per (element, sample);
// for hexes the 8 samples of an element are 8 consecutive lanes and are summed by a shuffle butterfly.
// ------------------------------------------------------------------------------------------------
// FP64: P = sum_en w (Bp - F_bound), the reference's expression.  FP32 (mixed precision): the SVD and the
// projections run in FP32 on F, but only their small correction Bp - F = U diag(s* - sig) V^T is rounded to
// FP32; P = sum_en w ((F - F_bound) in FP64 + (Bp - F) in FP32).  Node contributions are accumulated in FP64.
template <typename T, int K, int S>
__global__ void __launch_bounds__(kThreads) k_elem_fwd(int m, const int* __restrict__ E, const double* __restrict__ q,
                                                       const double* __restrict__ qb,
                                                       const unsigned char* __restrict__ elem_dir,
                                                       const double* __restrict__ grad, double vol_over_s,
                                                       EnergyPack ep, double* __restrict__ out, Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = t / S, smp = t % S;
    const bool valid = e < m;
    double acc[K][3];
#pragma unroll
    for (int a = 0; a < K; ++a) acc[a][0] = acc[a][1] = acc[a][2] = 0.0;
    if (valid) {
        const double* g = (S == 8) ? grad + smp * 24 : grad + (size_t)e * 12;
        double Fd[9], Fbd[9];
        def_grad<K>(E, e, q, g, Fd);
        if (elem_dir[e]) def_grad<K>(E, e, qb, g, Fbd);
        else {
#pragma unroll
            for (int i = 0; i < 9; ++i) Fbd[i] = 0.0;
        }
        T F[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) F[i] = (T)Fd[i];
        T U[9], V[9], sig[3];
        svd3<T>(F, U, sig, V);
        double P[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) P[i] = 0.0;
        bool ok = true;
        for (int k = 0; k < ep.count; ++k) {
            const ElemEnergyDev& en = ep.en[k];
            if (en.mask && !en.mask[e]) continue;
            const double w = ld_weight<double>(en, e) * vol_over_s;
            T Bp[9];
            if (sizeof(T) == 8) {
                ok = project<T>(en.type, (T)en.mu, (T)en.la, (T)en.w_mean, U, sig, V, Bp) && ok;
#pragma unroll
                for (int i = 0; i < 9; ++i) P[i] += w * ((double)Bp[i] - Fbd[i]);
            } else {
                ok = project_delta<T>(en.type, (T)en.mu, (T)en.la, (T)en.w_mean, U, sig, V, Bp) && ok;
#pragma unroll
                for (int i = 0; i < 9; ++i) P[i] += w * ((Fd[i] - Fbd[i]) + (double)Bp[i]);
            }
        }
        if (!ok) atomicOr(&ctrl->status, (int)kStatusSingularF);
#pragma unroll
        for (int a = 0; a < K; ++a) {
            const double g0 = __ldg(g + a * 3), g1 = __ldg(g + a * 3 + 1), g2 = __ldg(g + a * 3 + 2);
#pragma unroll
            for (int i = 0; i < 3; ++i) acc[a][i] = P[i] * g0 + P[i + 3] * g1 + P[i + 6] * g2;
        }
    }
    if (S == 8) {
#pragma unroll
        for (int o = 4; o > 0; o >>= 1)
#pragma unroll
            for (int a = 0; a < K; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) acc[a][i] += __shfl_xor_sync(0xffffffffu, acc[a][i], o);
        if (valid) {
#pragma unroll
            for (int a = 0; a < K; ++a)
                if (a == smp) {
                    double* o = out + ((size_t)e * K + a) * 3;
                    o[0] = acc[a][0]; o[1] = acc[a][1]; o[2] = acc[a][2];
                }
        }
    } else if (valid) {
#pragma unroll
        for (int a = 0; a < K; ++a) {
            double* o = out + ((size_t)e * K + a) * 3;
            o[0] = acc[a][0]; o[1] = acc[a][1]; o[2] = acc[a][2];
        }
    }
}

// Node gathers run kGatherLanes lanes per node (strided over the node's incident element outputs and its CSR
// row of A) and combine them with xor shuffles in a fixed order: deterministic, and eight times the memory
// parallelism of one thread per node on meshes of a few thousand nodes.

template <typename T>
__device__ __forceinline__ void group_sum(T& a) {
#pragma unroll
    for (int o = kGatherLanes / 2; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
}


// Sum of a node's incident element contributions eo[node_inc[idx]] (3 doubles each) over idx in [b, e), this
// lane taking idx = b + lane, b + lane + kGatherLanes, ...; four indices are loaded before their values so
// that a lane has several independent loads in flight instead of a chain of dependent ones.
__device__ __forceinline__ void sum_incident(const int* __restrict__ node_inc, const double* __restrict__ eo, int b,
                                             int e, int lane, double* p) {
    for (int idx = b + lane; idx < e; idx += 4 * kGatherLanes) {
        int k[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) k[u] = idx + u * kGatherLanes < e ? __ldg(node_inc + idx + u * kGatherLanes) : -1;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k[u] >= 0) {
                const double* c = eo + (size_t)k[u] * 3;
                p[0] += c[0]; p[1] += c[1]; p[2] += c[2];
            }
    }
}

// sum_k A.v[k] x[3 A.ci[k] + d] over this lane's share of the row [r0, r1), batched like sum_incident
__device__ __forceinline__ void csr_row_product(const NodeCsr& A, const double* __restrict__ x, int r0, int r1, int lane,
                                                double* acc) {
    for (int k0 = r0 + lane; k0 < r1; k0 += 4 * kGatherLanes) {
        int c[4];
        double a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u * kGatherLanes;
            c[u] = k < r1 ? __ldg(A.ci + k) : -1;
            a[u] = k < r1 ? __ldg(A.v + k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (c[u] >= 0) {
                acc[0] += a[u] * x[3 * c[u]];
                acc[1] += a[u] * x[3 * c[u] + 1];
                acc[2] += a[u] * x[3 * c[u] + 2];
            }
    }
}

template <typename T>
__global__ void __launch_bounds__(kGatherMaxThreads) k_gather_fwd(int n, const int* __restrict__ node_ptr,
                                                         const int* __restrict__ node_inc, const double* __restrict__ eo,
                                                         const double* __restrict__ qt, double inv_h2m,
                                                         const unsigned char* __restrict__ fixed,
                                                         const int* __restrict__ iperm, T* __restrict__ v, int npad,
                                                         double* __restrict__ prev, double* __restrict__ part,
                                                         NodeCsr A, const double* __restrict__ q, int zero_dirichlet,
                                                         double* __restrict__ r_out, Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    __shared__ double sh[2 * 32];
    double acc[2] = {0.0, 0.0};
    const int lane = threadIdx.x & (kGatherLanes - 1);
    const int per_block = (int)blockDim.x / kGatherLanes;
    for (int base = blockIdx.x * per_block; base < n; base += gridDim.x * per_block) {
        const int i = base + (int)threadIdx.x / kGatherLanes;
        const bool valid = i < n;
        const bool fx = valid ? fixed[i] != 0 : true;
        double p[3] = {0.0, 0.0, 0.0}, aq[3] = {0.0, 0.0, 0.0};
        if (valid) {
            sum_incident(node_inc, eo, node_ptr[i], node_ptr[i + 1], lane, p);
            if (A.rp && !fx) csr_row_product(A, q, A.rp[i], A.rp[i + 1], lane, aq);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            group_sum(p[d]);
            group_sum(aq[d]);
        }
        if (valid && lane == 0) {
            const int j = iperm[i];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double pr = prev[3 * i + d];
                acc[0] += (p[d] - pr) * (p[d] - pr);
                acc[1] += pr * pr;
                prev[3 * i + d] = p[d];
                const double val = (fx && zero_dirichlet) ? 0.0 : inv_h2m * qt[3 * i + d] + p[d] - aq[d];
                v[(size_t)d * npad + j] = (T)val;
                if (r_out) r_out[3 * i + d] = val;
            }
        }
    }
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2] = acc[0];
        part[blockIdx.x * 2 + 1] = acc[1];
    }
}

// ------------------------------------------------------------------------------------------------
// Sparse-inverse SpMV pair.  S row i is a dense segment of row_len[i] values starting at column row_a[i]
// (both multiples of 4, zero-padded), so loads are 16-byte vectors with implicit column indices.
// ------------------------------------------------------------------------------------------------
template <typename T> struct Vec4;
template <> struct Vec4<float> {
    float v[4];
    __device__ __forceinline__ void load(const float* p) {
        const float4 x = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    }
    __device__ __forceinline__ void load_stream(const float* p) {
        const float4 x = __ldcs(reinterpret_cast<const float4*>(p));
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    }
    // S values: kept in L2 across iterations when the factor fits there, streamed (evict-first) otherwise
    __device__ __forceinline__ void load_s(const float* p, int keep) {
        if (keep) load(p);
        else load_stream(p);
    }
};
template <> struct Vec4<double> {
    double v[4];
    __device__ __forceinline__ void load(const double* p) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    __device__ __forceinline__ void load_stream(const double* p) {
        const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
        const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    __device__ __forceinline__ void load_s(const double* p, int keep) {
        if (keep) load(p);
        else load_stream(p);
    }
};

// One thread per finished item of a row cut into several items: after its partial is stored, it counts itself
// in; the last one sums the row's partials in slot order (the order the S^T pass would use) into yrow.
template <typename T>
__device__ __forceinline__ void row_arrive(const SpmvPlan<T>& p, int z, int w) {
    __threadfence();
    const unsigned int prev = atomicAdd(p.row_cnt + z, 1u);
    if (prev != (unsigned int)(w - z - 1)) return;
    p.row_cnt[z] = 0u;  // ready for the next apply
    __threadfence();
    T s0 = T(0), s1 = T(0), s2 = T(0);
    for (int k = z; k < w; ++k) {
        s0 += __ldcg(p.ypart + 3 * (size_t)k);
        s1 += __ldcg(p.ypart + 3 * (size_t)k + 1);
        s2 += __ldcg(p.ypart + 3 * (size_t)k + 2);
    }
    T* o = p.yrow + 3 * (size_t)z;
    o[0] = s0;
    o[1] = s1;
    o[2] = s2;
}

// y = S v, stage 1: one warp per work item (a row segment of <= kSegCols columns), four 16-byte loads of S
// in flight per lane, v through L1 (the CTA's warps share the segment's columns).
template <typename T>
__device__ __forceinline__ void s_items_body(const SpmvPlan<T>& p, const T* __restrict__ v, int vb, const Ctrl* ctrl) {
    const int done = ctrl->done;  // in flight together with the descriptor loads, tested after them
    const int it = (vb * (int)blockDim.x + (int)threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (it >= p.n_items) return;
    const int4 dsc = __ldg(p.item_desc + it);
    const int slot = __ldg(p.item_slot + it);
    const int2 rs = p.yrow ? __ldg(p.item_rslots + it) : make_int2(0, 1);
    if (done) return;
    const T* __restrict__ sv = p.vals + ((int64_t)(uint32_t)dsc.x | ((int64_t)dsc.y << 32));
    const int a = dsc.z, nc = dsc.w;
    const T* __restrict__ v0 = v + a;
    const T* __restrict__ v1 = v + p.npad + a;
    const T* __restrict__ v2 = v + 2 * (size_t)p.npad + a;
    T s0 = T(0), s1 = T(0), s2 = T(0);
    int c = lane * 4;
    for (; c + 384 < nc; c += 512) {
        Vec4<T> s[4], x0[4], x1[4], x2[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) s[u].load_s(sv + c + 128 * u, p.keep_in_l2);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            x0[u].load(v0 + c + 128 * u);
            x1[u].load(v1 + c + 128 * u);
            x2[u].load(v2 + c + 128 * u);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                s0 += s[u].v[q] * x0[u].v[q];
                s1 += s[u].v[q] * x1[u].v[q];
                s2 += s[u].v[q] * x2[u].v[q];
            }
    }
    for (; c < nc; c += 128) {
        Vec4<T> s, x0, x1, x2;
        s.load_s(sv + c, p.keep_in_l2);
        x0.load(v0 + c);
        x1.load(v1 + c);
        x2.load(v2 + c);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            s0 += s.v[q] * x0.v[q];
            s1 += s.v[q] * x1.v[q];
            s2 += s.v[q] * x2.v[q];
        }
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    if (lane == 0) {
        T* o = p.ypart + (size_t)slot * 3;
        o[0] = s0; o[1] = s1; o[2] = s2;
        if (rs.y - rs.x > 1) row_arrive(p, rs.x, rs.y);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_spmv_S_items(SpmvPlan<T> p, const T* __restrict__ v, const Ctrl* ctrl) {
    pdl_enter();
    s_items_body(p, v, blockIdx.x, ctrl);
}

// y = S v, stage 1 by row groups (FP32): one warp per unit (up to kUnitRows rows of one nested-dissection
// group over one column segment).  Each lane loads the three float4 of v at its columns once and the float4
// of S of every row of the unit, so v is read once per unit instead of once per row, and every lane keeps up to
// kUnitRows + 3 independent 16-byte loads in flight.  Rows shorter than the unit's widest row are masked per
// float4 (row lengths and segment starts are multiples of 4).  Partial sums go to the rows' item slots.
__global__ void __launch_bounds__(256) k_spmv_S_units(SpmvPlan<float> p, const float* __restrict__ v,
                                                      const Ctrl* ctrl) {
    pdl_enter();
    const int done = ctrl->done;  // in flight together with the unit descriptor, tested after it
    const int u = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (u >= p.n_units) return;
    const int4 ud = __ldg(p.unit_desc + u);
    if (done) return;
    const int first = ud.x, nr = ud.y, a = ud.z, ncmax = ud.w;
    const float* sp[kUnitRows];
    int nc[kUnitRows];
#pragma unroll
    for (int r = 0; r < kUnitRows; ++r) {
        sp[r] = p.vals;
        nc[r] = 0;
        if (r < nr) {
            const int4 d = __ldg(p.unit_item_desc + first + r);
            sp[r] = p.vals + ((int64_t)(uint32_t)d.x | ((int64_t)d.y << 32));
            nc[r] = d.w;
        }
    }
    const size_t npad = (size_t)p.npad;
    const float* v0 = v + a;
    const float* v1 = v + npad + a;
    const float* v2 = v + 2 * npad + a;
    float acc[kUnitRows][3];
#pragma unroll
    for (int r = 0; r < kUnitRows; ++r) acc[r][0] = acc[r][1] = acc[r][2] = 0.f;
    for (int c = lane * 4; c < ncmax; c += 128) {
        Vec4<float> x0, x1, x2, sv[kUnitRows];
        x0.load(v0 + c);
        x1.load(v1 + c);
        x2.load(v2 + c);
#pragma unroll
        for (int r = 0; r < kUnitRows; ++r) {
            if (c < nc[r]) sv[r].load_s(sp[r] + c, p.keep_in_l2);
            else sv[r].v[0] = sv[r].v[1] = sv[r].v[2] = sv[r].v[3] = 0.f;
        }
#pragma unroll
        for (int r = 0; r < kUnitRows; ++r)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                acc[r][0] += sv[r].v[q] * x0.v[q];
                acc[r][1] += sv[r].v[q] * x1.v[q];
                acc[r][2] += sv[r].v[q] * x2.v[q];
            }
    }
#pragma unroll
    for (int r = 0; r < kUnitRows; ++r)
        if (r < nr) {
            acc[r][0] = warp_sum(acc[r][0]);
            acc[r][1] = warp_sum(acc[r][1]);
            acc[r][2] = warp_sum(acc[r][2]);
        }
    if (lane < nr) {  // lane r stores row r's partial (the values are warp-uniform after the sums)
        float o0 = 0.f, o1 = 0.f, o2 = 0.f;
#pragma unroll
        for (int r = 0; r < kUnitRows; ++r)
            if (r == lane) {
                o0 = acc[r][0];
                o1 = acc[r][1];
                o2 = acc[r][2];
            }
        float* o = p.ypart + (size_t)__ldg(p.unit_item_slot + first + lane) * 3;
        o[0] = o0;
        o[1] = o1;
        o[2] = o2;
        if (p.yrow) {
            const int2 rs = __ldg(p.unit_item_rslots + first + lane);
            if (rs.y - rs.x > 1) row_arrive(p, rs.x, rs.y);
        }
    }
}

// y = S v, stage 2: per row, the item partials in item order.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_spmv_S_fin(SpmvPlan<T> p, T* __restrict__ y, const Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    T s0 = T(0), s1 = T(0), s2 = T(0);
    for (int k = __ldg(p.row_yptr + i); k < __ldg(p.row_yptr + i + 1); ++k) {
        const T* o = p.ypart + (size_t)k * 3;
        s0 += o[0]; s1 += o[1]; s2 += o[2];
    }
    if (p.y_accumulate) {
        y[i] += s0;
        y[p.npad + i] += s1;
        y[2 * (size_t)p.npad + i] += s2;
    } else {
        y[i] = s0;
        y[p.npad + i] = s1;
        y[2 * (size_t)p.npad + i] = s2;
    }
}

// x = S^T y, stage 1: one CTA per (column tile, chunk of the tile's row list); partial tile sums are written
// to xpart[chunk] and summed in chunk order by stage 2.  The CTA first stages the chunk's row descriptors (first
// column, length, S offset) and y values in shared memory -- one coalesced pass, so that the S loads below do
// not wait on a descriptor load each -- then each warp takes every 8th row and keeps kStRows rows in flight.
// FROM_ITEMS: y_r is summed here from the S pass's row-contiguous item partials (in slot order, as the S fix-up
// kernel would), so the pair needs no separate fix-up launch.
template <typename T, bool FROM_ITEMS, int kStRows>
__device__ __forceinline__ void st_part_body(const SpmvPlan<T>& p, const T* __restrict__ y, int ch, const Ctrl* ctrl) {
    __shared__ T red[8][3][kTileCols];
    __shared__ int2 s_cl[kStChunkMax];        // per row of the chunk: first column, length of its padded segment
    __shared__ long long s_off[kStChunkMax];  // S offset of the row's first value
    __shared__ T s_y[3][kStChunkMax];
    const int done = ctrl->done;  // in flight together with the chunk's bounds; the same in every thread
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = __ldg(p.chunk_tile + ch);
    const int c = tile * kTileCols + lane * 4;
    const int npad = p.npad;
    T acc[3][4];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[d][q] = T(0);
    const int pe = __ldg(p.chunk_p1 + ch), p0 = __ldg(p.chunk_p0 + ch);
    if (done) return;
    const int cnt = pe - p0;  // <= kStChunkMax (the schedule's chunk rows)
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        const int q = p0 + t;
        const int4 dd = __ldg(p.trow_desc + q);
        s_cl[t] = make_int2(dd.x, dd.y);
        s_off[t] = __ldg(p.trow_off + q);
        T y0 = T(0), y1 = T(0), y2 = T(0);
        if (FROM_ITEMS) {
            if (p.yrow) {  // one load per row: the item partial, or the row total of a multi-item row
                if (dd.z < dd.w) {
                    const T* src = (dd.w - dd.z > 1 ? p.yrow : p.ypart) + 3 * (size_t)dd.z;
                    y0 = __ldg(src);
                    y1 = __ldg(src + 1);
                    y2 = __ldg(src + 2);
                }
            } else {
                for (int k = dd.z; k < dd.w; ++k) {
                    y0 += __ldg(p.ypart + 3 * (size_t)k);
                    y1 += __ldg(p.ypart + 3 * (size_t)k + 1);
                    y2 += __ldg(p.ypart + 3 * (size_t)k + 2);
                }
            }
        } else {
            const int i = __ldg(p.tile_rows + q);
            y0 = __ldg(y + i);
            y1 = __ldg(y + npad + i);
            y2 = __ldg(y + 2 * (size_t)npad + i);
        }
        s_y[0][t] = y0;
        s_y[1][t] = y1;
        s_y[2][t] = y2;
    }
    __syncthreads();
    for (int b = wid; b < cnt; b += 8 * kStRows) {
        Vec4<T> sv[kStRows];
        bool in[kStRows];
#pragma unroll
        for (int u = 0; u < kStRows; ++u) {
            const int t = b + 8 * u;
            in[u] = false;
            if (t < cnt) {
                const int2 cl = s_cl[t];
                in[u] = cl.y > 0 && c >= cl.x && c + 4 <= cl.x + cl.y;
                if (in[u]) sv[u].load_s(p.vals + s_off[t] + (c - cl.x), p.keep_in_l2);
            }
        }
#pragma unroll
        for (int u = 0; u < kStRows; ++u)
            if (in[u]) {
                const int t = b + 8 * u;
                const T y0 = s_y[0][t], y1 = s_y[1][t], y2 = s_y[2][t];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    acc[0][q] += sv[u].v[q] * y0;
                    acc[1][q] += sv[u].v[q] * y1;
                    acc[2][q] += sv[u].v[q] * y2;
                }
            }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int q = 0; q < 4; ++q) red[wid][d][lane * 4 + q] = acc[d][q];
    __syncthreads();
    for (int t = threadIdx.x; t < 3 * kTileCols; t += 256) {
        const int d = t / kTileCols, col = t % kTileCols;
        T s = T(0);
#pragma unroll
        for (int w = 0; w < 8; ++w) s += red[w][d][col];
        p.xpart[(size_t)ch * 3 * kTileCols + t] = s;
    }
    __syncthreads();  // `red` is reused by the next chunk of a persistent CTA
}

template <typename T, bool FROM_ITEMS, int kStRows>
__global__ void __launch_bounds__(256) k_spmv_ST_part(SpmvPlan<T> p, const T* __restrict__ y, const Ctrl* ctrl) {
    pdl_enter();
    st_part_body<T, FROM_ITEMS, kStRows>(p, y, blockIdx.x, ctrl);
}

// x = S^T y, stage 2: per tile column, sum the chunk partials in order and scatter to node-major x.
template <typename T>
__device__ __forceinline__ void st_fin_body(const SpmvPlan<T>& p, double* __restrict__ x_out, int vb,
                                            const Ctrl* ctrl) {
    const int done = ctrl->done;  // in flight together with the tile's chunk range, tested after it
    const int t = vb * (int)blockDim.x + (int)threadIdx.x;
    if (t >= p.ntiles * 3 * kTileCols) return;
    const int tile = t / (3 * kTileCols), r = t % (3 * kTileCols);
    const int d = r / kTileCols, col = r % kTileCols;
    const int j = tile * kTileCols + col;
    if (j >= p.n) return;
    double s = 0.0;
    const int c0 = __ldg(p.tile_chunk_ptr + tile), c1 = __ldg(p.tile_chunk_ptr + tile + 1);
    if (done) return;
    for (int ch = c0; ch < c1; ch += 8) {  // eight independent loads in flight, summed in chunk order
        T t8[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) t8[u] = ch + u < c1 ? p.xpart[(size_t)(ch + u) * 3 * kTileCols + r] : T(0);
#pragma unroll
        for (int u = 0; u < 8; ++u) s += (double)t8[u];
    }
    const size_t o = 3 * (size_t)__ldg(p.perm + j) + d;
    x_out[o] = p.x_base ? p.x_base[o] + s : s;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_spmv_ST_fin(SpmvPlan<T> p, double* __restrict__ x_out,
                                                          const Ctrl* ctrl) {
    pdl_enter();
    st_fin_body(p, x_out, blockIdx.x, ctrl);
}


// ------------------------------------------------------------------------------------------------
// Type-II Anderson acceleration (forward_gpu.cpp:1340-1379; backward_gpu.cpp:825-859) and the gate.
// History: `count` entries (x_prev, g); differences dG, dX live in a ring of `window` slots starting at
// `head`.  k_aa_reduce pushes the new entry, forms the Gram system and solves it in the last block;
// k_aa_update applies the extrapolation, re-imposes Dirichlet values and evaluates the stop rule.
// ------------------------------------------------------------------------------------------------
constexpr int kAaVals = 2 * kMaxWindow + 2;  // new Gram column, right-hand side, |g|^2, |x_raw|^2

__global__ void __launch_bounds__(kThreads) k_aa_reduce(int n3, const double* __restrict__ x,
                                                        const double* __restrict__ xr,
                                                        const unsigned char* __restrict__ fixed,
                                                        const double* __restrict__ fval, double* __restrict__ dG,
                                                        double* __restrict__ dX, double* __restrict__ lg,
                                                        double* __restrict__ lx, int ld, double* __restrict__ part,
                                                        Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    __shared__ double sh[kAaVals * 32];
    const int W = ctrl->window, count = ctrl->count, head = ctrl->head, mode = ctrl->mode;
    const int m = W > 0 ? count : 0;  // differences after this push (the newest is j = m - 1)
    double acc[kAaVals];
#pragma unroll
    for (int i = 0; i < kAaVals; ++i) acc[i] = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n3; r += gridDim.x * blockDim.x) {
        const double xp = x[r];
        double xv = xr[r];
        if (fixed[r]) xv = mode == 0 ? fval[r] : 0.0;
        const double g = xv - xp;
        if (W > 0) {
            double gnew = 0.0;
            if (count >= 1) {
                const int s = (head + count - 1) % W;
                gnew = g - lg[r];
                dG[(size_t)s * ld + r] = gnew;
                dX[(size_t)s * ld + r] = xp - lx[r];
            }
            lg[r] = g;
            lx[r] = xp;
#pragma unroll
            for (int j = 0; j < kMaxWindow; ++j)
                if (j < m) {
                    const double dgj = (j == m - 1) ? gnew : dG[(size_t)((head + j) % W) * ld + r];
                    acc[j] += gnew * dgj;
                    acc[kMaxWindow + j] += dgj * g;
                }
        }
        acc[kAaVals - 2] += g * g;
        acc[kAaVals - 1] += xv * xv;
    }
    block_sum<kAaVals>(acc, sh);
    if (threadIdx.x == 0)
        for (int i = 0; i < kAaVals; ++i) part[blockIdx.x * kAaVals + i] = acc[i];
    if (!arrive_last(&ctrl->arrive[0])) return;
    double tot[kAaVals];
    sum_partials<kAaVals>(part, gridDim.x, tot, sh);
    if (threadIdx.x != 0) return;
    ctrl->arrive[0] = 0;
    ctrl->err = sqrt(tot[kAaVals - 2]);
    ctrl->xn = sqrt(tot[kAaVals - 1]);
    ctrl->m = m;
    ctrl->accept = 0;
    ctrl->restart = 0;
    if (mode == 1 && (!(ctrl->xn == ctrl->xn) || ctrl->xn > 1e300 ||
                      (ctrl->clip > 0 && ctrl->xn > ctrl->clip))) {
        ctrl->status |= (ctrl->xn == ctrl->xn && ctrl->xn <= 1e300) ? (int)kStatusDiverged
                                                                    : (int)(kStatusDiverged | kStatusNonFinite);
        return;
    }
    if (m < 1) return;
    // Extend the stored Gram matrix by the new difference's column, then solve
    // (dG^T dG + reg I) gamma = dG^T g, reg = max(1e-6 |dG|_F^2 / m, 1e-12), by Cholesky.  All loops run to
    // kMaxWindow with guards so that the small arrays stay in registers; the stored entries are loaded
    // independently (one round trip) rather than inside the factorisation.
    const int snew = (head + m - 1) % W;
    double A[kMaxWindow][kMaxWindow], b[kMaxWindow];
#pragma unroll
    for (int i = 0; i < kMaxWindow; ++i)
#pragma unroll
        for (int j = 0; j < kMaxWindow; ++j)
            if (i < m && j < m)
                A[i][j] = (i == m - 1) ? tot[j] : (j == m - 1) ? tot[i] : ctrl->gram[(head + i) % W][(head + j) % W];
#pragma unroll
    for (int j = 0; j < kMaxWindow; ++j)
        if (j < m) {
            const int sj = (head + j) % W;
            ctrl->gram[snew][sj] = tot[j];
            ctrl->gram[sj][snew] = tot[j];
        }
    double fro = 0;
#pragma unroll
    for (int j = 0; j < kMaxWindow; ++j)
        if (j < m) fro += A[j][j];
    const double reg = fmax(1e-6 * fro / m, 1e-12);
#pragma unroll
    for (int i = 0; i < kMaxWindow; ++i)
        if (i < m) {
            A[i][i] += reg;
            b[i] = tot[kMaxWindow + i];
        }
    // one reciprocal per column (a single thread runs this: FP64 divisions dominate its latency)
    double inv_diag[kMaxWindow];
#pragma unroll
    for (int j = 0; j < kMaxWindow; ++j) {
        inv_diag[j] = 0.0;
        if (j < m) {
            double d = A[j][j];
#pragma unroll
            for (int k = 0; k < kMaxWindow; ++k)
                if (k < j) d -= A[j][k] * A[j][k];
            d = sqrt(fmax(d, 1e-300));
            A[j][j] = d;
            const double inv = 1.0 / d;
            inv_diag[j] = inv;
#pragma unroll
            for (int i = 0; i < kMaxWindow; ++i)
                if (i > j && i < m) {
                    double t = A[i][j];
#pragma unroll
                    for (int k = 0; k < kMaxWindow; ++k)
                        if (k < j) t -= A[i][k] * A[j][k];
                    A[i][j] = t * inv;
                }
        }
    }
#pragma unroll
    for (int i = 0; i < kMaxWindow; ++i)
        if (i < m) {
            double t = b[i];
#pragma unroll
            for (int k = 0; k < kMaxWindow; ++k)
                if (k < i) t -= A[i][k] * b[k];
            b[i] = t * inv_diag[i];
        }
#pragma unroll
    for (int i = kMaxWindow - 1; i >= 0; --i)
        if (i < m) {
            double t = b[i];
#pragma unroll
            for (int k = 0; k < kMaxWindow; ++k)
                if (k > i && k < m) t -= A[k][i] * b[k];
            b[i] = t * inv_diag[i];
        }
    double gn = 0;
#pragma unroll
    for (int i = 0; i < kMaxWindow; ++i)
        if (i < m) gn += b[i] * b[i];
    gn = sqrt(gn);
    if (!(gn < 10.0)) {
        ctrl->restart = 1;
    } else {
        ctrl->accept = 1;
#pragma unroll
        for (int i = 0; i < kMaxWindow; ++i)
            if (i < m) ctrl->gamma[i] = b[i];
    }
}

__global__ void __launch_bounds__(kThreads) k_aa_update(int n3, double* __restrict__ x, const double* __restrict__ xr,
                                                        const unsigned char* __restrict__ fixed,
                                                        const double* __restrict__ fval,
                                                        const double* __restrict__ dG, const double* __restrict__ dX,
                                                        int ld, double* __restrict__ part,
                                                        const double* __restrict__ gate_part, int gate_blocks,
                                                        Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    __shared__ double sh[3 * 32];
    const int W = ctrl->window, head = ctrl->head, mode = ctrl->mode;
    const int accept = ctrl->accept, m = ctrl->m;
    double gam[kMaxWindow];
#pragma unroll
    for (int j = 0; j < kMaxWindow; ++j) gam[j] = (accept && j < m) ? ctrl->gamma[j] : 0.0;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n3; r += gridDim.x * blockDim.x) {
        const double xp = x[r];
        double xv = xr[r];
        const bool fx = fixed[r] != 0;
        if (fx) xv = mode == 0 ? fval[r] : 0.0;
        double xn = xv;
        if (accept) {
            xn = xv;  // = xp + g
#pragma unroll
            for (int j = 0; j < kMaxWindow; ++j)
                if (j < m) {
                    const size_t s = (size_t)((head + j) % W) * ld + r;
                    xn -= (dX[s] + dG[s]) * gam[j];
                }
            if (fx) xn = mode == 0 ? fval[r] : 0.0;
        }
        x[r] = xn;
        acc[0] += (xn - xp) * (xn - xp);
        acc[1] += xp * xp;
        acc[2] += xn * xn;
    }
    block_sum<3>(acc, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x * 3] = acc[0];
        part[blockIdx.x * 3 + 1] = acc[1];
        part[blockIdx.x * 3 + 2] = acc[2];
    }
    if (!arrive_last(&ctrl->arrive[1])) return;
    double tt[3], gp[2] = {0.0, 0.0};
    sum_partials<3>(part, gridDim.x, tt, sh);
    if (mode == 0) sum_partials<2>(gate_part, gate_blocks, gp, sh);
    if (threadIdx.x != 0) return;
    const double t0 = tt[0], t1 = tt[1], t2 = tt[2];
    ctrl->arrive[1] = 0;
    const double dq = sqrt(t0), rn = sqrt(t1), xnorm = sqrt(t2);
    bool conv = false;
    const int it = ctrl->iter;
    if (mode == 0) {
        const double pdc = sqrt(gp[0]), pdr = sqrt(gp[1]);
        ctrl->dq = dq; ctrl->rn = rn; ctrl->pdc = pdc; ctrl->pdr = pdr;
        conv = it > 0 && dq <= ctrl->rel_tol * rn + ctrl->abs_tol && pdc <= ctrl->rel_tol * pdr + ctrl->abs_tol;
        if (!(dq == dq) || !(pdc == pdc)) ctrl->status |= kStatusNonFinite;
        if (!conv && it > 0 && ctrl->stall_window > 0) {
            const double ratio = fmax(dq / (ctrl->rel_tol * rn + ctrl->abs_tol), pdc / (ctrl->rel_tol * pdr + ctrl->abs_tol));
            if (ratio < 0.5 * ctrl->best_ratio) {
                ctrl->best_ratio = ratio;
                ctrl->best_it = it;
            } else if (it - ctrl->best_it >= ctrl->stall_window) {
                ctrl->stalled = 1;
                ctrl->done = 1;
            }
        }
    } else {
        ctrl->dq = dq; ctrl->rn = xnorm;
        conv = it > 0 && ctrl->err < ctrl->rel_tol * xnorm + ctrl->abs_tol;
        if (!(xnorm == xnorm)) ctrl->status |= kStatusNonFinite | kStatusDiverged;
        else if (ctrl->clip > 0 && xnorm > ctrl->clip) ctrl->status |= kStatusDiverged;
    }
    if (W > 0) {
        if (ctrl->restart) {
            ctrl->count = 0;
            ctrl->head = 0;
        } else {
            int c = ctrl->count + 1;
            if (c > W) {
                c = W;
                ctrl->head = (ctrl->head + 1) % W;
            }
            ctrl->count = c;
        }
    }
    ctrl->iter = it + 1;
    if (conv) ctrl->converged = 1;
    if (conv || ctrl->iter >= ctrl->max_iter || (ctrl->status & (kStatusNonFinite | kStatusDiverged))) ctrl->done = 1;
}

__global__ void k_qtilde(int n3, const double* q, const double* v, const double* f, double h, double h2m,
                         const double* gf, double* qt) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n3) return;
    qt[r] = q[r] + h * v[r] + h2m * f[r] + h2m * gf[r % 3];
}

__global__ void k_velocity(int n3, const double* qn, const double* q, double inv_h, double* vn) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n3) return;
    vn[r] = (qn[r] - q[r]) * inv_h;
}

// ------------------------------------------------------------------------------------------------
// Adjoint kernels
// ------------------------------------------------------------------------------------------------
// Cyclic Jacobi eigen-decomposition of a symmetric 9x9 matrix (row-major), eigenvectors in Q (columns).
__device__ void jacobi_eig9(double* A, double* Q) {
    for (int i = 0; i < 81; ++i) Q[i] = (i % 10 == 0) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 30; ++sweep) {
        double off = 0, diag = 0;
        for (int i = 0; i < 9; ++i)
            for (int j = 0; j < 9; ++j) (i == j ? diag : off) += A[i * 9 + j] * A[i * 9 + j];
        if (off <= 1e-30 * diag) break;
        for (int p = 0; p < 8; ++p)
            for (int q = p + 1; q < 9; ++q) {
                const double apq = A[p * 9 + q];
                if (fabs(apq) < 1e-300) continue;
                const double tau = (A[q * 9 + q] - A[p * 9 + p]) / (2 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1 + tau * tau));
                const double c = 1 / sqrt(1 + t * t), s = t * c;
                for (int k = 0; k < 9; ++k) {  // columns p,q
                    const double akp = A[k * 9 + p], akq = A[k * 9 + q];
                    A[k * 9 + p] = c * akp - s * akq;
                    A[k * 9 + q] = s * akp + c * akq;
                }
                for (int k = 0; k < 9; ++k) {  // rows p,q
                    const double apk = A[p * 9 + k], aqk = A[q * 9 + k];
                    A[p * 9 + k] = c * apk - s * aqk;
                    A[q * 9 + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 9; ++k) {
                    const double qkp = Q[k * 9 + p], qkq = Q[k * 9 + q];
                    Q[k * 9 + p] = c * qkp - s * qkq;
                    Q[k * 9 + q] = s * qkp + c * qkq;
                }
            }
    }
}

// FP32 copy of a symmetric 9x9 Jacobian (the projections' differentials are Hessians of scalar functions):
// upper triangle, row by row, (J_ic + J_ci) / 2, padded to 48 floats for 16-byte loads.
constexpr int kJ32Stride = 48;
__device__ __forceinline__ void pack_sym32(const double* Jt, float* o) {
    int k = 0;
    for (int i = 0; i < 9; ++i)
        for (int c = i; c < 9; ++c) o[k++] = (float)(0.5 * (Jt[c * 9 + i] + Jt[i * 9 + c]));
    for (; k < kJ32Stride; ++k) o[k] = 0.f;
}

template <int K, int S>
__global__ void __launch_bounds__(128) k_jac_build(int m, const int* __restrict__ E, const double* __restrict__ q,
                                                   const double* __restrict__ grad, double vol_over_s, EnergyPack ep,
                                                   int mean_w, int filter, double* __restrict__ J,
                                                   float* __restrict__ J32, Ctrl* ctrl) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = t / S, smp = t % S;
    if (e >= m) return;
    const double* g = (S == 8) ? grad + smp * 24 : grad + (size_t)e * 12;
    double F[9], U[9], V[9], sig[3];
    def_grad<K>(E, e, q, g, F);
    svd3<double>(F, U, sig, V);
    double* Jt = J + (size_t)t * 81;
    double wsum = 0;
    for (int col = 0; col < 9; ++col) {
        double dF[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) dF[i] = (i == col) ? 1.0 : 0.0;
        double out[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) out[i] = 0.0;
        for (int k = 0; k < ep.count; ++k) {
            const ElemEnergyDev& en = ep.en[k];
            if (en.mask && !en.mask[e]) continue;
            const double w = (mean_w ? en.w_mean : ld_weight<double>(en, e)) * vol_over_s;
            if (col == 0) wsum += w;
            double d[9];
            project_diff<double>(en.type, en.mu, en.la, en.w_mean, U, sig, V, dF, d);
#pragma unroll
            for (int i = 0; i < 9; ++i) out[i] += w * d[i];
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) Jt[col * 9 + i] = out[i];  // column col (column-major 9x9)
    }
    if (filter == 0) {
        if (J32) pack_sym32(Jt, J32 + (size_t)t * kJ32Stride);
        return;
    }
    // State-adaptive filter of the local Hessian H = wsum I - J (the PD energy's per-sample Hessian), with the
    // rule of ProjectedNewtonMatrix (cpp/core/src/fem/deformable_newton_forward.cpp:394-434): kept as is when
    // diagonally dominant (|H_kk| >= sum_j |H_kj| + 1e-5 in every row); otherwise eigen-decomposed and its
    // eigenvalues clamped at 0 (filter 1) or replaced by |lambda| (filter 2).
    double H[81];
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) H[i * 9 + j] = (i == j ? wsum : 0.0) - 0.5 * (Jt[j * 9 + i] + Jt[i * 9 + j]);
    bool dd = true;
    for (int i = 0; i < 9 && dd; ++i) {
        double off = 0;
        for (int j = 0; j < 9; ++j)
            if (j != i) off += fabs(H[i * 9 + j]);
        dd = !(fabs(H[i * 9 + i]) < off + 1e-5);
    }
    if (dd) {
        if (J32) pack_sym32(Jt, J32 + (size_t)t * kJ32Stride);
        return;
    }
    double Q[81];
    jacobi_eig9(H, Q);
    double lam[9];
    for (int i = 0; i < 9; ++i) {
        const double l = H[i * 9 + i];
        lam[i] = filter == 1 ? fmax(l, 0.0) : fabs(l);
    }
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) {
            double h = 0;
            for (int k = 0; k < 9; ++k) h += Q[i * 9 + k] * lam[k] * Q[j * 9 + k];
            Jt[j * 9 + i] = (i == j ? wsum : 0.0) - h;
        }
    atomicAdd(&ctrl->arrive[3], 1u);  // number of filtered samples (diagnostic)
    if (J32) pack_sym32(Jt, J32 + (size_t)t * kJ32Stride);
}

template <int K, int S>
__global__ void __launch_bounds__(kThreads) k_kpd_elem(int m, const int* __restrict__ E, const double* __restrict__ u,
                                                       const double* __restrict__ grad, const double* __restrict__ J,
                                                       double* __restrict__ out, const Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = t / S, smp = t % S;
    const bool valid = e < m;
    double acc[K][3];
#pragma unroll
    for (int a = 0; a < K; ++a) acc[a][0] = acc[a][1] = acc[a][2] = 0.0;
    if (valid) {
        const double* g = (S == 8) ? grad + smp * 24 : grad + (size_t)e * 12;
        double dF[9];
        def_grad<K>(E, e, u, g, dF);
        const double* Jt = J + (size_t)t * 81;
        double P[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) P[i] = 0.0;
#pragma unroll
        for (int col = 0; col < 9; ++col) {
            const double f = dF[col];
#pragma unroll
            for (int i = 0; i < 9; ++i) P[i] += __ldg(Jt + col * 9 + i) * f;
        }
#pragma unroll
        for (int a = 0; a < K; ++a) {
            const double g0 = __ldg(g + a * 3), g1 = __ldg(g + a * 3 + 1), g2 = __ldg(g + a * 3 + 2);
#pragma unroll
            for (int i = 0; i < 3; ++i) acc[a][i] = P[i] * g0 + P[i + 3] * g1 + P[i + 6] * g2;
        }
    }
    if (S == 8) {
#pragma unroll
        for (int o = 4; o > 0; o >>= 1)
#pragma unroll
            for (int a = 0; a < K; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) acc[a][i] += __shfl_xor_sync(0xffffffffu, acc[a][i], o);
        if (valid) {
#pragma unroll
            for (int a = 0; a < K; ++a)
                if (a == smp) {
                    double* o = out + ((size_t)e * K + a) * 3;
                    o[0] = acc[a][0]; o[1] = acc[a][1]; o[2] = acc[a][2];
                }
        }
    } else if (valid) {
#pragma unroll
        for (int a = 0; a < K; ++a) {
            double* o = out + ((size_t)e * K + a) * 3;
            o[0] = acc[a][0]; o[1] = acc[a][1]; o[2] = acc[a][2];
        }
    }
}

// K_pd u from the FP32 packed symmetric Jacobians (mixed precision): P = J dF in FP32, element sums in FP64.
template <int K, int S>
__global__ void __launch_bounds__(kThreads) k_kpd_elem32(int m, const int* __restrict__ E,
                                                         const double* __restrict__ u, const double* __restrict__ grad,
                                                         const float* __restrict__ J32, double* __restrict__ out,
                                                         const Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = t / S, smp = t % S;
    const bool valid = e < m;
    double acc[K][3];
#pragma unroll
    for (int a = 0; a < K; ++a) acc[a][0] = acc[a][1] = acc[a][2] = 0.0;
    if (valid) {
        const double* g = (S == 8) ? grad + smp * 24 : grad + (size_t)e * 12;
        float Mv[kJ32Stride];
        const float4* src = reinterpret_cast<const float4*>(J32 + (size_t)t * kJ32Stride);
#pragma unroll
        for (int k = 0; k < kJ32Stride / 4; ++k) {
            const float4 x = __ldg(src + k);
            Mv[4 * k] = x.x; Mv[4 * k + 1] = x.y; Mv[4 * k + 2] = x.z; Mv[4 * k + 3] = x.w;
        }
        double dFd[9];
        def_grad<K>(E, e, u, g, dFd);
        float dF[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) dF[i] = (float)dFd[i];
        float P[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) P[i] = 0.f;
        int k = 0;
#pragma unroll
        for (int i = 0; i < 9; ++i)
#pragma unroll
            for (int c = i; c < 9; ++c, ++k) {
                P[i] += Mv[k] * dF[c];
                if (c != i) P[c] += Mv[k] * dF[i];
            }
#pragma unroll
        for (int a = 0; a < K; ++a) {
            const double g0 = __ldg(g + a * 3), g1 = __ldg(g + a * 3 + 1), g2 = __ldg(g + a * 3 + 2);
#pragma unroll
            for (int i = 0; i < 3; ++i)
                acc[a][i] = (double)P[i] * g0 + (double)P[i + 3] * g1 + (double)P[i + 6] * g2;
        }
    }
    if (S == 8) {
#pragma unroll
        for (int o = 4; o > 0; o >>= 1)
#pragma unroll
            for (int a = 0; a < K; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) acc[a][i] += __shfl_xor_sync(0xffffffffu, acc[a][i], o);
        if (valid) {
#pragma unroll
            for (int a = 0; a < K; ++a)
                if (a == smp) {
                    double* o = out + ((size_t)e * K + a) * 3;
                    o[0] = acc[a][0]; o[1] = acc[a][1]; o[2] = acc[a][2];
                }
        }
    } else if (valid) {
#pragma unroll
        for (int a = 0; a < K; ++a) {
            double* o = out + ((size_t)e * K + a) * 3;
            o[0] = acc[a][0]; o[1] = acc[a][1]; o[2] = acc[a][2];
        }
    }
}

__global__ void __launch_bounds__(kGatherMaxThreads) k_gather_bwd(int n, const int* __restrict__ node_ptr,
                                                         const int* __restrict__ node_inc,
                                                         const double* __restrict__ eo, const double* __restrict__ gbar,
                                                         const unsigned char* __restrict__ fixed,
                                                         const int* __restrict__ iperm, double* __restrict__ v,
                                                         int npad, const Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    const int lane = threadIdx.x & (kGatherLanes - 1);
    const int per_block = (int)blockDim.x / kGatherLanes;
    for (int base = blockIdx.x * per_block; base < n; base += gridDim.x * per_block) {
        const int i = base + (int)threadIdx.x / kGatherLanes;
        const bool valid = i < n;
        double pp[3] = {0.0, 0.0, 0.0};
        if (valid) sum_incident(node_inc, eo, node_ptr[i], node_ptr[i + 1], lane, pp);
        double p0 = pp[0], p1 = pp[1], p2 = pp[2];
        group_sum(p0);
        group_sum(p1);
        group_sum(p2);
        if (valid && lane == 0) {
            const int j = iperm[i];
            const bool fx = fixed[i] != 0;
            v[j] = fx ? 0.0 : gbar[3 * i] + p0;
            v[npad + j] = fx ? 0.0 : gbar[3 * i + 1] + p1;
            v[2 * (size_t)npad + j] = fx ? 0.0 : gbar[3 * i + 2] + p2;
        }
    }
}

// d(prox)/d(mu_bar), d(prox)/d(la_bar) of the Neo-Hookean proximal map with k = 2 mu_bar.
__device__ void nh_param_diff(double mu, double la, const double* U, const double* sig, const double* V, double* dPm,
                              double* dPl) {
    const double k = 2 * mu;
    double ss[3];
    nh_prox<double>(mu, la, k, sig, ss);
    double H[9];
    nh_hessian<double>(mu, la, k, ss, H);
    H[0] += 1e-9; H[4] += 1e-9; H[8] += 1e-9;
    const double L = log(fmax(ss[0] * ss[1] * ss[2], 1e-12));
    double gm[3], gl[3], H2[9];
    for (int i = 0; i < 3; ++i) {
        gm[i] = -(ss[i] - 1 / ss[i] + 2 * (ss[i] - sig[i]));
        gl[i] = -(L / ss[i]);
    }
    for (int i = 0; i < 9; ++i) H2[i] = H[i];
    small_solve<double, 3>(H, gm);
    small_solve<double, 3>(H2, gl);
    for (int i = 0; i < 3; ++i)
        if (ss[i] <= 1e-4) { gm[i] = 0; gl[i] = 0; }
    usvt(U, gm, V, dPm);
    usvt(U, gl, V, dPl);
}

template <int K, int S>
__global__ void __launch_bounds__(128) k_param_grad(int m, const int* __restrict__ E, const double* __restrict__ q,
                                                    const double* __restrict__ mu, const double* __restrict__ grad,
                                                    double vol_over_s, EnergyPack ep, double* __restrict__ gw,
                                                    double* __restrict__ gmat, double* __restrict__ gnh) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = t / S, smp = t % S;
    const bool valid = e < m;
    double r[kMaxEnergies][4];
#pragma unroll
    for (int k = 0; k < kMaxEnergies; ++k) r[k][0] = r[k][1] = r[k][2] = r[k][3] = 0.0;
    if (valid) {
        const double* g = (S == 8) ? grad + smp * 24 : grad + (size_t)e * 12;
        double F[9], U[9], V[9], sig[3];
        def_grad<K>(E, e, q, g, F);
        svd3<double>(F, U, sig, V);
        // G(i,j) = sum_a mu_a[i] grad_a[j]: then mu_e^T A_s^T M = <G, M>
        double G[9];
        def_grad<K>(E, e, mu, g, G);
        for (int k = 0; k < ep.count && k < kMaxEnergies; ++k) {
            const ElemEnergyDev& en = ep.en[k];
            if (en.mask && !en.mask[e]) continue;
            double Bp[9];
            project<double>(en.type, en.mu, en.la, en.w_mean, U, sig, V, Bp);
            double dot = 0;
#pragma unroll
            for (int i = 0; i < 9; ++i) dot += G[i] * (F[i] - Bp[i]);
            r[k][0] = -vol_over_s * dot;
            if (en.type == 2) {
                // reference dl_dmat_w term: NH first Piola stress over the mean stiffness
                const double Jd = F[0] * (F[4] * F[8] - F[7] * F[5]) - F[3] * (F[1] * F[8] - F[7] * F[2]) +
                                  F[6] * (F[1] * F[5] - F[4] * F[2]);
                const double lj = log(fmax(Jd, 1e-12));
                double FiT[9];  // F^-T = cofactor(F) / det
                FiT[0] = (F[4] * F[8] - F[5] * F[7]) / Jd;
                FiT[1] = (F[5] * F[6] - F[3] * F[8]) / Jd;
                FiT[2] = (F[3] * F[7] - F[4] * F[6]) / Jd;
                FiT[3] = (F[2] * F[7] - F[1] * F[8]) / Jd;
                FiT[4] = (F[0] * F[8] - F[2] * F[6]) / Jd;
                FiT[5] = (F[1] * F[6] - F[0] * F[7]) / Jd;
                FiT[6] = (F[1] * F[5] - F[2] * F[4]) / Jd;
                FiT[7] = (F[2] * F[3] - F[0] * F[5]) / Jd;
                FiT[8] = (F[0] * F[4] - F[1] * F[3]) / Jd;
                double dp = 0;
#pragma unroll
                for (int i = 0; i < 9; ++i) dp += G[i] * (en.mu * (F[i] - FiT[i]) + en.la * lj * FiT[i]) / en.w_mean;
                r[k][1] = -vol_over_s * dp;
                double dPm[9], dPl[9];
                nh_param_diff(en.mu, en.la, U, sig, V, dPm, dPl);
                const double w = ld_weight<double>(en, e) * vol_over_s;
                double a1 = 0, a2 = 0;
#pragma unroll
                for (int i = 0; i < 9; ++i) { a1 += G[i] * dPm[i]; a2 += G[i] * dPl[i]; }
                r[k][2] = w * a1;
                r[k][3] = w * a2;
            } else {
                r[k][1] = r[k][0];
            }
        }
    }
    if (S == 8) {
#pragma unroll
        for (int o = 4; o > 0; o >>= 1)
#pragma unroll
            for (int k = 0; k < kMaxEnergies; ++k)
#pragma unroll
                for (int i = 0; i < 4; ++i) r[k][i] += __shfl_xor_sync(0xffffffffu, r[k][i], o);
    }
    if (valid && smp == 0) {
        for (int k = 0; k < ep.count && k < kMaxEnergies; ++k) {
            gw[(size_t)k * m + e] = r[k][0];
            gmat[(size_t)k * m + e] = r[k][1];
            gnh[((size_t)k * m + e) * 2] = r[k][2];
            gnh[((size_t)k * m + e) * 2 + 1] = r[k][3];
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Conjugate-gradient adjoint
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kGatherMaxThreads) k_pcg_gather(int n, NodeCsr A, const double* __restrict__ p,
                                                         const int* __restrict__ node_ptr,
                                                         const int* __restrict__ node_inc,
                                                         const double* __restrict__ eo,
                                                         const unsigned char* __restrict__ fixed,
                                                         double* __restrict__ w, double* __restrict__ part,
                                                         Ctrl* ctrl, int init) {
    pdl_enter();
    if (ctrl->done) return;
    __shared__ double sh[32];
    double acc[1] = {0.0};
    const int lane = threadIdx.x & (kGatherLanes - 1);
    const int per_block = (int)blockDim.x / kGatherLanes;
    for (int base = blockIdx.x * per_block; base < n; base += gridDim.x * per_block) {
        const int i = base + (int)threadIdx.x / kGatherLanes;
        const bool valid = i < n;
        const bool fx = valid ? fixed[i] != 0 : true;
        double a0 = 0, a1 = 0, a2 = 0;
        if (valid && !fx) {
            double ap[3] = {0.0, 0.0, 0.0}, kp[3] = {0.0, 0.0, 0.0};
            csr_row_product(A, p, A.rp[i], A.rp[i + 1], lane, ap);
            sum_incident(node_inc, eo, node_ptr[i], node_ptr[i + 1], lane, kp);
            a0 = ap[0] - kp[0];
            a1 = ap[1] - kp[1];
            a2 = ap[2] - kp[2];
        }
        group_sum(a0);
        group_sum(a1);
        group_sum(a2);
        if (valid && lane == 0) {
            w[3 * i] = a0; w[3 * i + 1] = a1; w[3 * i + 2] = a2;  // zero on Dirichlet nodes
            acc[0] += a0 * p[3 * i] + a1 * p[3 * i + 1] + a2 * p[3 * i + 2];
        }
    }
    if (init) return;  // w = (A - K_pd) x0 for a start vector: no step length, no curvature test
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
    if (!arrive_last(&ctrl->arrive[2])) return;
    double t[1];
    sum_partials<1>(part, gridDim.x, t, sh);
    if (threadIdx.x != 0) return;
    ctrl->arrive[2] = 0;
    const double pw = t[0];
    if (!(pw > 0.0) || !(pw < 1e300)) {
        ctrl->status |= kStatusIndefinite;
        ctrl->done = 1;
        ctrl->alpha = 0.0;
        return;
    }
    ctrl->alpha = ctrl->rz / pw;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_pcg_update1(int n, double* __restrict__ mu, double* __restrict__ r,
                                                          const double* __restrict__ p, const double* __restrict__ w,
                                                          const unsigned char* __restrict__ fixed,
                                                          const int* __restrict__ iperm, T* __restrict__ v, int npad,
                                                          double* __restrict__ part, Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    __shared__ double sh[32];
    const double alpha = ctrl->alpha;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int j = iperm[i];
        const bool fx = fixed[i] != 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int k = 3 * i + d;
            const double m = mu[k] + alpha * p[k];
            const double rr = r[k] - alpha * w[k];
            mu[k] = m;
            r[k] = rr;
            acc[0] += m * m;
            v[(size_t)d * npad + j] = fx ? T(0) : (T)rr;
        }
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

__device__ __forceinline__ void pcg_update2_tail(const double* __restrict__ part, const double* __restrict__ mu_part,
                                                 int mu_blocks, Ctrl* ctrl, double* sh);

__global__ void __launch_bounds__(kThreads) k_pcg_update2(int n3, const double* __restrict__ r,
                                                          const double* __restrict__ z, double* __restrict__ part,
                                                          const double* __restrict__ mu_part, int mu_blocks,
                                                          Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    __shared__ double sh[2 * 32];
    double acc[2] = {0.0, 0.0};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += gridDim.x * blockDim.x) {
        acc[0] += r[k] * z[k];
        acc[1] += z[k] * z[k];
    }
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2] = acc[0];
        part[blockIdx.x * 2 + 1] = acc[1];
    }
    pcg_update2_tail(part, mu_part, mu_blocks, ctrl, sh);
}

// Last-block part of the z-side update: r.z and |z| summed over the blocks' partials, beta, the stop rule.
__device__ __forceinline__ void pcg_update2_tail(const double* __restrict__ part, const double* __restrict__ mu_part,
                                                 int mu_blocks, Ctrl* ctrl, double* sh) {
    if (!arrive_last(&ctrl->arrive[1])) return;
    double t[2], mu2[1] = {0.0};
    sum_partials<2>(part, gridDim.x, t, sh);
    if (!ctrl->pcg_init) sum_partials<1>(mu_part, mu_blocks, mu2, sh);
    if (threadIdx.x != 0) return;
    ctrl->arrive[1] = 0;
    const double rz = t[0], zn = sqrt(t[1]), mun = sqrt(mu2[0]);
    if (ctrl->pcg_init) {
        ctrl->pcg_init = 0;
        ctrl->beta = 0.0;
        ctrl->rz = rz;
        return;
    }
    ctrl->beta = ctrl->rz > 0 ? rz / ctrl->rz : 0.0;
    ctrl->rz = rz;
    ctrl->err = zn;
    ctrl->rn = mun;
    const int it = ctrl->iter;
    const bool conv = it > 0 && zn < ctrl->rel_tol * mun + ctrl->abs_tol;
    if (!(zn == zn) || !(mun == mun)) ctrl->status |= kStatusNonFinite | kStatusDiverged;
    else if (ctrl->clip > 0 && mun > ctrl->clip) ctrl->status |= kStatusDiverged;
    ctrl->iter = it + 1;
    if (conv) ctrl->converged = 1;
    if (conv || ctrl->iter >= ctrl->max_iter || (ctrl->status & (kStatusNonFinite | kStatusDiverged)))
        ctrl->done = 1;
}

// x = S^T y stage 2 fused with the z-side update of the conjugate-gradient adjoint: each thread finishes one
// column of z = S^T S r (the chunk partials summed in order, scattered to node order) and adds its r.z and
// z.z terms to the block's partials; the last block sums them (pcg_update2_tail).  Replaces the ST fin +
// k_pcg_update2 pair when z is not projected afterwards.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_spmv_ST_fin_cg(SpmvPlan<T> p, double* __restrict__ z_out,
                                                             const double* __restrict__ r, double* __restrict__ part,
                                                             const double* __restrict__ mu_part, int mu_blocks,
                                                             Ctrl* ctrl) {
    pdl_enter();
    __shared__ double sh[2 * 32];
    const int done = ctrl->done;
    const int t = blockIdx.x * (int)blockDim.x + (int)threadIdx.x;
    double acc[2] = {0.0, 0.0};
    int rr = 0, d = 0, j = -1, c0 = 0, c1 = 0;
    if (t < p.ntiles * 3 * kTileCols) {
        const int tile = t / (3 * kTileCols);
        rr = t % (3 * kTileCols);
        d = rr / kTileCols;
        j = tile * kTileCols + rr % kTileCols;
        c0 = __ldg(p.tile_chunk_ptr + tile);
        c1 = __ldg(p.tile_chunk_ptr + tile + 1);
    }
    if (done) return;  // the same in every block: no block arrives, no tail runs
    if (j >= 0 && j < p.n) {
        double sum = 0.0;
        for (int ch = c0; ch < c1; ch += 8) {  // eight independent loads in flight, summed in chunk order
            T t8[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) t8[u] = ch + u < c1 ? p.xpart[(size_t)(ch + u) * 3 * kTileCols + rr] : T(0);
#pragma unroll
            for (int u = 0; u < 8; ++u) sum += (double)t8[u];
        }
        const size_t o = 3 * (size_t)__ldg(p.perm + j) + d;
        const double zv = p.x_base ? p.x_base[o] + sum : sum;
        z_out[o] = zv;
        acc[0] = r[o] * zv;
        acc[1] = zv * zv;
    }
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2] = acc[0];
        part[blockIdx.x * 2 + 1] = acc[1];
    }
    pcg_update2_tail(part, mu_part, mu_blocks, ctrl, sh);
}

__global__ void k_pcg_p(int n3, double* __restrict__ p, const double* __restrict__ z, const Ctrl* ctrl) {
    pdl_enter();
    if (ctrl->done) return;
    const double beta = ctrl->beta;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += gridDim.x * blockDim.x) p[k] = z[k] + beta * p[k];
}

// r = g_bar - w (w = (A - K_pd) mu_0 for a warm start, null for mu_0 = 0); v = r in the S ordering.
template <typename T>
__global__ void k_pcg_init(int n, const double* __restrict__ gbar, const double* __restrict__ w,
                           const unsigned char* __restrict__ fixed, const int* __restrict__ iperm,
                           double* __restrict__ r, T* __restrict__ v, int npad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool fx = fixed[i] != 0;
    const int j = iperm[i];
    for (int d = 0; d < 3; ++d) {
        const double g = fx ? 0.0 : gbar[3 * i + d] - (w ? w[3 * i + d] : 0.0);
        r[3 * i + d] = g;
        v[(size_t)d * npad + j] = (T)g;
    }
}

__global__ void __launch_bounds__(kThreads) k_adj_prepare(int n3, const double* __restrict__ gq,
                                                          const double* __restrict__ gv, double inv_h,
                                                          double* __restrict__ gbar, double* __restrict__ dq,
                                                          double* __restrict__ part, double* norm_out,
                                                          unsigned int* arrive) {
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n3; r += gridDim.x * blockDim.x) {
        const double g = gq[r] + gv[r] * inv_h;
        gbar[r] = g;
        dq[r] = -gv[r] * inv_h;
        acc[0] += g * g;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
    if (!arrive_last(arrive)) return;
    double t[1];
    sum_partials<1>(part, gridDim.x, t, sh);
    if (threadIdx.x == 0) {
        norm_out[0] = sqrt(t[0]);
        *arrive = 0;
    }
}

__global__ void __launch_bounds__(kThreads) k_adj_route(int n3, const double* __restrict__ mu, double mu_norm,
                                                        const double* __restrict__ gbar_norm, double inv_h2m, double h,
                                                        double h2m, double mass, int cap, int gravity,
                                                        double* __restrict__ dq, double* __restrict__ dv,
                                                        double* __restrict__ df, double* __restrict__ dstate,
                                                        double* __restrict__ part, unsigned int* arrive) {
    __shared__ double sh[3 * 32];
    double s = 1.0;
    if (cap) {
        const double c = gbar_norm[0] + 1.0, in = inv_h2m * mu_norm;
        if (in > c) s = c / in;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n3; r += gridDim.x * blockDim.x) {
        const double inj = s * inv_h2m * mu[r];
        dq[r] += inj;
        dv[r] = h * inj;
        df[r] = h2m * inj;
        acc[r % 3] += h2m * inj * mass;
    }
    block_sum<3>(acc, sh);
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) part[blockIdx.x * 3 + d] = acc[d];
    if (!arrive_last(arrive)) return;
    double t[3];
    sum_partials<3>(part, gridDim.x, t, sh);
    if (threadIdx.x == 0) {
        if (gravity)
            for (int d = 0; d < 3; ++d) dstate[d] = t[d];
        *arrive = 0;
    }
}

// One block per energy: fixed-order sums (deterministic).
__global__ void k_param_reduce(int m, const int* __restrict__ np_k, const int* __restrict__ type_k,
                               const int* __restrict__ off_k, const double* __restrict__ gw,
                               const double* __restrict__ gmat, const double* __restrict__ gnh,
                               double* __restrict__ dmat, double* __restrict__ dpar) {
    __shared__ double sh[4 * 32];
    const int k = blockIdx.x;
    const int npk = np_k[k], type = type_k[k], off = off_k[k];
    const double* w = gw + (size_t)k * m;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int e = threadIdx.x; e < m; e += blockDim.x) {
        acc[0] += gmat[(size_t)k * m + e];
        acc[1] += w[e];
        acc[2] += gnh[((size_t)k * m + e) * 2];
        acc[3] += gnh[((size_t)k * m + e) * 2 + 1];
    }
    block_sum<4>(acc, sh);
    __shared__ double tot[4];
    if (threadIdx.x == 0)
        for (int i = 0; i < 4; ++i) tot[i] = acc[i];
    __syncthreads();
    if (threadIdx.x == 0) dmat[k] = tot[0];
    if (type != 2) {
        if (npk == 1) {
            if (threadIdx.x == 0) dpar[off] = tot[1];
        } else {
            for (int e = threadIdx.x; e < m; e += blockDim.x) dpar[off + e] = w[e];
        }
    } else {
        if (npk == 2) {
            if (threadIdx.x == 0) {
                dpar[off] = 2 * tot[1] + tot[2];
                dpar[off + 1] = tot[3];
            }
        } else {
            for (int e = threadIdx.x; e < m; e += blockDim.x) {
                dpar[off + 2 * e] = 2 * w[e] + tot[2] / m;
                dpar[off + 2 * e + 1] = tot[3] / m;
            }
        }
    }
}

inline int blocks_for(long long work, int threads) { return (int)((work + threads - 1) / threads); }
bool g_pdl = true;  // programmatic dependent launch of the iteration-body kernels (process-wide)

// Launches `kern` with programmatic stream serialization when g_pdl is set: the grid may start while its
// predecessor in the stream drains (the kernel's pdl_enter waits for the predecessor's completion before it
// reads anything).  Inside stream capture this becomes a programmatic edge of the graph.
template <typename... KArgs, typename... Args>
void launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g_pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}


}  // namespace

void set_pdl(bool on) { g_pdl = on; }

int device_sms() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = sms > 0 ? sms : 148;
    }
    return cached[dev];
}

void even_grid(long long threads, int max_bs, int max_grid, int* grid, int* bs) {
    const long long sms = device_sms();
    if (threads <= 0) {
        *grid = 1;
        *bs = 32;
        return;
    }
    const long long k = std::max(1LL, (threads + (long long)max_bs * sms - 1) / ((long long)max_bs * sms));
    long long per = (threads + k * sms - 1) / (k * sms);
    per = std::min<long long>(max_bs, (per + 31) / 32 * 32);
    const long long g = (threads + per - 1) / per;
    *bs = (int)per;
    *grid = (int)std::max(1LL, std::min<long long>(g, max_grid));
}

int gather_grid(int n) {
    int g, b;
    even_grid((long long)n * kGatherLanes, kGatherMaxThreads, kMaxRedBlocks, &g, &b);
    return g;
}
int gather_bs(int n) {
    int g, b;
    even_grid((long long)n * kGatherLanes, kGatherMaxThreads, kMaxRedBlocks, &g, &b);
    return b;
}

namespace {

}  // namespace

// ------------------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------------------
template <typename T>
void launch_elem_fwd(int m, int k, int s, const int* E, const double* q, const double* qb, const unsigned char* elem_dir,
                     const double* grad, int hex, double vol_over_s, const EnergyPack& ep, double* elem_out, Ctrl* ctrl,
                     cudaStream_t st) {
    int grid, bs;
    even_grid((long long)m * s, kThreads, 1 << 30, &grid, &bs);
    if (hex) launch_k(k_elem_fwd<T, 8, 8>, grid, bs, 0, st, m, E, q, qb, elem_dir, grad, vol_over_s, ep, elem_out, ctrl);
    else launch_k(k_elem_fwd<T, 4, 1>, grid, bs, 0, st, m, E, q, qb, elem_dir, grad, vol_over_s, ep, elem_out, ctrl);
}

template <typename T>
void launch_gather_fwd(int n, const int* node_ptr, const int* node_inc, const double* elem_out, const double* qt,
                       double inv_h2m, const unsigned char* fixed_node, const int* iperm, T* v_perm, int npad,
                       double* prev_pd, double* part, int blocks, NodeCsr A, const double* q, int zero_dirichlet,
                       Ctrl* ctrl, cudaStream_t st, double* r_out) {
    launch_k(k_gather_fwd<T>, blocks, gather_bs(n), 0, st, n, node_ptr, node_inc, elem_out, qt, inv_h2m, fixed_node, iperm,
                                                     v_perm, npad, prev_pd, part, A, q, zero_dirichlet, r_out, ctrl);
}

// stage 1 of x = S^T y with the plan's rows in flight per warp
template <typename T, bool FROM_ITEMS>
static void launch_st_part(const SpmvPlan<T>& p, const T* y, const Ctrl* ctrl, cudaStream_t st) {
    if (p.st_rows == 8) launch_k(k_spmv_ST_part<T, FROM_ITEMS, 8>, p.n_chunks, 256, 0, st, p, y, ctrl);
    else launch_k(k_spmv_ST_part<T, FROM_ITEMS, 4>, p.n_chunks, 256, 0, st, p, y, ctrl);
}

// stage 1 of y = S v: the row-group kernel for FP32 factors with a unit schedule, else one warp per item
template <typename T>
static void launch_s_items(const SpmvPlan<T>& p, const T* v, const Ctrl* ctrl, cudaStream_t st) {
    if constexpr (std::is_same<T, float>::value) {
        if (p.use_units && p.n_units > 0) {
            launch_k(k_spmv_S_units, blocks_for((long long)p.n_units * 32, 256), 256, 0, st, p, v, ctrl);
            return;
        }
    }
    launch_k(k_spmv_S_items<T>, blocks_for((long long)p.n_items * 32, 256), 256, 0, st, p, v, ctrl);
}

template <typename T>
void launch_sts(const SpmvPlan<T>& p, const T* v, T* y, double* x_out, const Ctrl* ctrl, cudaStream_t st) {
    launch_s_items(p, v, ctrl, st);
    if (p.y_accumulate) {
        launch_k(k_spmv_S_fin<T>, blocks_for(p.n, kThreads), kThreads, 0, st, p, y, ctrl);
        launch_st_part<T, false>(p, y, ctrl, st);
    } else {
        launch_st_part<T, true>(p, nullptr, ctrl, st);
    }
    launch_k(k_spmv_ST_fin<T>, blocks_for((long long)p.ntiles * 3 * kTileCols, kThreads), kThreads, 0, st, p, x_out, ctrl);
}

void launch_aa_reduce(int n3, const double* x, const double* x_raw, const unsigned char* fixed_dof,
                      const double* fixed_val, double* dG, double* dX, double* last_g, double* last_x, int ld,
                      double* part, int blocks, Ctrl* ctrl, cudaStream_t st) {
    launch_k(k_aa_reduce, blocks, kThreads, 0, st, n3, x, x_raw, fixed_dof, fixed_val, dG, dX, last_g, last_x, ld, part,
                                                ctrl);
}

void launch_aa_update(int n3, double* x, const double* x_raw, const unsigned char* fixed_dof, const double* fixed_val,
                      const double* dG, const double* dX, int ld, double* part, const double* gate_part,
                      int gate_blocks, int blocks, Ctrl* ctrl, cudaStream_t st) {
    launch_k(k_aa_update, blocks, kThreads, 0, st, n3, x, x_raw, fixed_dof, fixed_val, dG, dX, ld, part, gate_part,
                                                gate_blocks, ctrl);
}

void launch_qtilde(int n3, const double* q, const double* v, const double* f_ext, double h, double h2m,
                   const double* grav_force, double* qt, cudaStream_t st) {
    k_qtilde<<<blocks_for(n3, kThreads), kThreads, 0, st>>>(n3, q, v, f_ext, h, h2m, grav_force, qt);
}

void launch_velocity(int n3, const double* q_next, const double* q, double inv_h, double* v_next, cudaStream_t st) {
    k_velocity<<<blocks_for(n3, kThreads), kThreads, 0, st>>>(n3, q_next, q, inv_h, v_next);
}

void launch_jac_build(int m, int k, int s, const int* E, const double* q, const double* grad, int hex,
                      double vol_over_s, const EnergyPack& ep, int mean_w, int filter, double* J, float* J32,
                      Ctrl* ctrl, cudaStream_t st) {
    (void)k;
    const int grid = blocks_for((long long)m * s, 128);
    if (hex) k_jac_build<8, 8><<<grid, 128, 0, st>>>(m, E, q, grad, vol_over_s, ep, mean_w, filter, J, J32, ctrl);
    else k_jac_build<4, 1><<<grid, 128, 0, st>>>(m, E, q, grad, vol_over_s, ep, mean_w, filter, J, J32, ctrl);
}

void launch_kpd_elem32(int m, int k, int s, const int* E, const double* u, const double* grad, int hex,
                       const float* J32, double* elem_out, const Ctrl* ctrl, cudaStream_t st) {
    (void)k;
    int grid, bs;
    even_grid((long long)m * s, kThreads, 1 << 30, &grid, &bs);
    if (hex) launch_k(k_kpd_elem32<8, 8>, grid, bs, 0, st, m, E, u, grad, J32, elem_out, ctrl);
    else launch_k(k_kpd_elem32<4, 1>, grid, bs, 0, st, m, E, u, grad, J32, elem_out, ctrl);
}

void launch_kpd_elem(int m, int k, int s, const int* E, const double* u, const double* grad, int hex, const double* J,
                     double* elem_out, const Ctrl* ctrl, cudaStream_t st) {
    (void)k;
    int grid, bs;
    even_grid((long long)m * s, kThreads, 1 << 30, &grid, &bs);
    if (hex) launch_k(k_kpd_elem<8, 8>, grid, bs, 0, st, m, E, u, grad, J, elem_out, ctrl);
    else launch_k(k_kpd_elem<4, 1>, grid, bs, 0, st, m, E, u, grad, J, elem_out, ctrl);
}

void launch_gather_bwd(int n, const int* node_ptr, const int* node_inc, const double* elem_out, const double* gbar,
                       const unsigned char* fixed_node, const int* iperm, double* v_perm, int npad, const Ctrl* ctrl,
                       cudaStream_t st) {
    const int blocks = std::max(1, std::min(kMaxRedBlocks, (n * kGatherLanes + kThreads - 1) / kThreads));
    launch_k(k_gather_bwd, blocks, gather_bs(n), 0, st, n, node_ptr, node_inc, elem_out, gbar, fixed_node, iperm, v_perm, npad,
                                              ctrl);
}

void launch_param_grad(int m, int k, int s, const int* E, const double* q, const double* mu, const double* grad,
                       int hex, double vol_over_s, const EnergyPack& ep, double* gw, double* gmat, double* gnh,
                       cudaStream_t st) {
    (void)k;
    const int grid = blocks_for((long long)m * s, 128);
    if (hex) k_param_grad<8, 8><<<grid, 128, 0, st>>>(m, E, q, mu, grad, vol_over_s, ep, gw, gmat, gnh);
    else k_param_grad<4, 1><<<grid, 128, 0, st>>>(m, E, q, mu, grad, vol_over_s, ep, gw, gmat, gnh);
}

template void launch_elem_fwd<double>(int, int, int, const int*, const double*, const double*, const unsigned char*,
                                      const double*, int, double, const EnergyPack&, double*, Ctrl*, cudaStream_t);
template void launch_elem_fwd<float>(int, int, int, const int*, const double*, const double*, const unsigned char*,
                                     const double*, int, double, const EnergyPack&, double*, Ctrl*, cudaStream_t);
template void launch_gather_fwd<double>(int, const int*, const int*, const double*, const double*, double,
                                        const unsigned char*, const int*, double*, int, double*, double*, int, NodeCsr,
                                        const double*, int, Ctrl*, cudaStream_t, double*);
template void launch_gather_fwd<float>(int, const int*, const int*, const double*, const double*, double,
                                       const unsigned char*, const int*, float*, int, double*, double*, int, NodeCsr,
                                       const double*, int, Ctrl*, cudaStream_t, double*);

void launch_pcg_gather(int n, NodeCsr A, const double* p, const int* node_ptr, const int* node_inc,
                       const double* elem_out, const unsigned char* fixed_node, double* w, double* part, int blocks,
                       Ctrl* ctrl, cudaStream_t st, int init) {
    launch_k(k_pcg_gather, blocks, gather_bs(n), 0, st, n, A, p, node_ptr, node_inc, elem_out, fixed_node, w, part, ctrl,
                                              init);
}

// ---- contact-aware material adjoint ------------------------------------------------------------------
// u_c <- (I - sum_k d_k d_k^T) u_c at the constrained nodes (orthonormal directions d_k, at most 3 per node);
// with vperm, the projected values are also written to the S-ordered copy.
template <typename T>
__global__ void k_wb_project(const int* __restrict__ count, const int* __restrict__ nodes,
                             const double* __restrict__ dirs, const int* __restrict__ ndir, double* __restrict__ u,
                             T* __restrict__ vperm, const int* __restrict__ iperm, int npad, const Ctrl* ctrl) {
    if (ctrl && ctrl->done) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *count) return;
    const int node = nodes[k];
    double x[3] = {u[3 * node], u[3 * node + 1], u[3 * node + 2]};
    for (int j = 0; j < ndir[k]; ++j) {
        const double* d = dirs + 9 * (size_t)k + 3 * j;
        const double t = d[0] * x[0] + d[1] * x[1] + d[2] * x[2];
        x[0] -= t * d[0];
        x[1] -= t * d[1];
        x[2] -= t * d[2];
    }
    u[3 * node] = x[0];
    u[3 * node + 1] = x[1];
    u[3 * node + 2] = x[2];
    if (vperm) {
        const int j = iperm[node];
        vperm[j] = (T)x[0];
        vperm[npad + j] = (T)x[1];
        vperm[2 * (size_t)npad + j] = (T)x[2];
    }
}

template <typename T>
void launch_wb_project(int capacity, const int* count, const int* nodes, const double* dirs, const int* ndir,
                       double* u, T* vperm, const int* iperm, int npad, const Ctrl* ctrl, cudaStream_t st) {
    k_wb_project<T><<<blocks_for(std::max(capacity, 1), kThreads), kThreads, 0, st>>>(count, nodes, dirs, ndir, u,
                                                                                     vperm, iperm, npad, ctrl);
}
template void launch_wb_project<double>(int, const int*, const int*, const double*, const int*, double*, double*,
                                        const int*, int, const Ctrl*, cudaStream_t);
template void launch_wb_project<float>(int, const int*, const int*, const double*, const int*, double*, float*,
                                       const int*, int, const Ctrl*, cudaStream_t);

// out[k] = u at node cand[k] (3 values per candidate)
__global__ void k_gather_nodes(int K, const int* __restrict__ cand, const double* __restrict__ u,
                               double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const int node = cand[k];
    out[3 * k] = u[3 * node];
    out[3 * k + 1] = u[3 * node + 1];
    out[3 * k + 2] = u[3 * node + 2];
}
void launch_gather_nodes(int K, const int* cand, const double* u, double* out, cudaStream_t st) {
    if (K > 0) k_gather_nodes<<<blocks_for(K, kThreads), kThreads, 0, st>>>(K, cand, u, out);
}

// res = {|a - b|^2, |a|^2, |b|^2} (one CTA: a tape comparison per backward call, off the iteration path)
__global__ void __launch_bounds__(1024) k_diff_norms(int n, const double* __restrict__ a,
                                                     const double* __restrict__ b, double* __restrict__ res) {
    __shared__ double sh[3 * 32];
    double acc[3] = {0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = a[i], y = b[i];
        acc[0] += (x - y) * (x - y);
        acc[1] += x * x;
        acc[2] += y * y;
    }
    block_sum<3>(acc, sh);
    if (threadIdx.x == 0) {
        res[0] = acc[0];
        res[1] = acc[1];
        res[2] = acc[2];
    }
}
void launch_diff_norms(int n, const double* a, const double* b, double* res, cudaStream_t st) {
    k_diff_norms<<<1, 1024, 0, st>>>(n, a, b, res);
}
template <typename T>
void launch_pcg_update1(int n, double* mu, double* r, const double* p, const double* w,
                        const unsigned char* fixed_node, const int* iperm, T* v_perm, int npad, double* part,
                        int blocks, Ctrl* ctrl, cudaStream_t st) {
    launch_k(k_pcg_update1<T>, blocks, kThreads, 0, st, n, mu, r, p, w, fixed_node, iperm, v_perm, npad, part, ctrl);
}
void launch_pcg_update2(int n3, const double* r, const double* z, double* part, const double* mu_part, int mu_blocks,
                        int blocks, Ctrl* ctrl, cudaStream_t st) {
    launch_k(k_pcg_update2, blocks, kThreads, 0, st, n3, r, z, part, mu_part, mu_blocks, ctrl);
}
template <typename T>
void launch_sts_cg(const SpmvPlan<T>& p, const T* v, double* z, const double* r, double* part, const double* mu_part,
                   int mu_blocks, Ctrl* ctrl, cudaStream_t st) {
    launch_s_items(p, v, ctrl, st);
    launch_st_part<T, true>(p, nullptr, ctrl, st);
    launch_k(k_spmv_ST_fin_cg<T>, blocks_for((long long)p.ntiles * 3 * kTileCols, kThreads), kThreads, 0, st, 
        p, z, r, part, mu_part, mu_blocks, ctrl);
}
template void launch_sts_cg<float>(const SpmvPlan<float>&, const float*, double*, const double*, double*,
                                   const double*, int, Ctrl*, cudaStream_t);
template void launch_sts_cg<double>(const SpmvPlan<double>&, const double*, double*, const double*, double*,
                                    const double*, int, Ctrl*, cudaStream_t);

__global__ void k_extrapolate(int n3, const double* __restrict__ a, const double* __restrict__ b,
                              double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n3) out[k] = 2.0 * a[k] - b[k];
}
void launch_extrapolate(int n3, const double* a, const double* b, double* out, cudaStream_t st) {
    k_extrapolate<<<blocks_for(n3, kThreads), kThreads, 0, st>>>(n3, a, b, out);
}
__global__ void k_extrapolate3(int n3, const double* __restrict__ a, const double* __restrict__ b,
                               const double* __restrict__ c, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n3) out[k] = 3.0 * (a[k] - b[k]) + c[k];
}
void launch_extrapolate3(int n3, const double* a, const double* b, const double* c, double* out, cudaStream_t st) {
    k_extrapolate3<<<blocks_for(n3, kThreads), kThreads, 0, st>>>(n3, a, b, c, out);
}
__global__ void k_extrapolate4(int n3, const double* __restrict__ a, const double* __restrict__ b,
                               const double* __restrict__ c, const double* __restrict__ d, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n3) out[k] = 4.0 * (a[k] + c[k]) - 6.0 * b[k] - d[k];
}
void launch_extrapolate4(int n3, const double* a, const double* b, const double* c, const double* d, double* out,
                         cudaStream_t st) {
    k_extrapolate4<<<blocks_for(n3, kThreads), kThreads, 0, st>>>(n3, a, b, c, d, out);
}

void launch_pcg_p(int n3, double* p, const double* z, const Ctrl* ctrl, cudaStream_t st) {
    launch_k(k_pcg_p, std::max(1, std::min(kMaxRedBlocks, (n3 + 255) / 256)), kThreads, 0, st, n3, p, z, ctrl);
}
template <typename T>
void launch_pcg_init(int n, const double* gbar, const double* w, const unsigned char* fixed_node, const int* iperm,
                     double* r, T* v_perm, int npad, cudaStream_t st) {
    k_pcg_init<T><<<blocks_for(n, kThreads), kThreads, 0, st>>>(n, gbar, w, fixed_node, iperm, r, v_perm, npad);
}
template void launch_pcg_update1<double>(int, double*, double*, const double*, const double*, const unsigned char*,
                                         const int*, double*, int, double*, int, Ctrl*, cudaStream_t);
template void launch_pcg_update1<float>(int, double*, double*, const double*, const double*, const unsigned char*,
                                        const int*, float*, int, double*, int, Ctrl*, cudaStream_t);
template void launch_pcg_init<double>(int, const double*, const double*, const unsigned char*, const int*, double*,
                                      double*, int, cudaStream_t);
template void launch_pcg_init<float>(int, const double*, const double*, const unsigned char*, const int*, double*,
                                     float*, int, cudaStream_t);
void launch_adj_prepare(int n3, const double* gq, const double* gv, double inv_h, double* gbar, double* dq,
                        double* part, double* norm_out, cudaStream_t st) {
    // norm_out[1] doubles as the arrival counter of this kernel (zeroed by the caller)
    k_adj_prepare<<<std::max(1, std::min(kRedBlocks, (n3 + 2047) / 2048)), kThreads, 0, st>>>(
        n3, gq, gv, inv_h, gbar, dq, part, norm_out, reinterpret_cast<unsigned int*>(norm_out + 1));
}

void launch_adj_route(int n3, const double* mu, double mu_norm, const double* gbar_norm, double inv_h2m, double h,
                      double h2m, double mass, int cap, int gravity, double* dl_dq, double* dl_dv, double* dl_df,
                      double* dl_dstate_p, double* part, unsigned int* arrive, cudaStream_t st) {
    k_adj_route<<<std::max(1, std::min(kRedBlocks, (n3 + 2047) / 2048)), kThreads, 0, st>>>(
        n3, mu, mu_norm, gbar_norm, inv_h2m, h, h2m, mass, cap, gravity, dl_dq, dl_dv, dl_df, dl_dstate_p, part,
        arrive);
}

void launch_param_reduce(int m, int ne, const int* np_k, const int* type_k, const int* off_k, const double* gw,
                         const double* gmat, const double* gnh, double* dl_dmat_w, double* dl_dparams,
                         cudaStream_t st) {
    if (ne > 0) k_param_reduce<<<ne, kThreads, 0, st>>>(m, np_k, type_k, off_k, gw, gmat, gnh, dl_dmat_w, dl_dparams);
}

template <typename T>
void launch_s_only(const SpmvPlan<T>& p, const T* v, T* y, const Ctrl* ctrl, cudaStream_t st) {
    launch_s_items(p, v, ctrl, st);
    launch_k(k_spmv_S_fin<T>, blocks_for(p.n, kThreads), kThreads, 0, st, p, y, ctrl);
}
template <typename T>
void launch_st_only(const SpmvPlan<T>& p, const T* y, double* x_out, const Ctrl* ctrl, cudaStream_t st) {
    launch_st_part<T, false>(p, y, ctrl, st);
    launch_k(k_spmv_ST_fin<T>, blocks_for((long long)p.ntiles * 3 * kTileCols, kThreads), kThreads, 0, st, p, x_out, ctrl);
}
template void launch_s_only<double>(const SpmvPlan<double>&, const double*, double*, const Ctrl*, cudaStream_t);
template void launch_s_only<float>(const SpmvPlan<float>&, const float*, float*, const Ctrl*, cudaStream_t);
template void launch_st_only<double>(const SpmvPlan<double>&, const double*, double*, const Ctrl*, cudaStream_t);
template void launch_st_only<float>(const SpmvPlan<float>&, const float*, double*, const Ctrl*, cudaStream_t);

__global__ void k_loop_cond(cudaGraphConditionalHandle h, Ctrl* ctrl, int cap) {
    const int loops = ctrl->loops + 1;
    ctrl->loops = loops;
    cudaGraphSetConditional(h, (!ctrl->done && loops < cap) ? 1u : 0u);
}

__global__ void k_axpy(int n, double a, const double* __restrict__ x, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}
__global__ void k_sub(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] - b[i];
}
void launch_axpy(int n, double a, const double* x, double* y, cudaStream_t st) {
    if (n > 0) k_axpy<<<(n + 255) / 256, 256, 0, st>>>(n, a, x, y);
}
void launch_sub(int n, const double* a, const double* b, double* out, cudaStream_t st) {
    if (n > 0) k_sub<<<(n + 255) / 256, 256, 0, st>>>(n, a, b, out);
}

void launch_loop_cond(cudaGraphConditionalHandle h, Ctrl* ctrl, int cap, cudaStream_t st) {
    k_loop_cond<<<1, 1, 0, st>>>(h, ctrl, cap);
}


template void launch_sts<double>(const SpmvPlan<double>&, const double*, double*, double*, const Ctrl*,
                                 cudaStream_t);
template void launch_sts<float>(const SpmvPlan<float>&, const float*, float*, double*, const Ctrl*, cudaStream_t);

}  // namespace dphd
