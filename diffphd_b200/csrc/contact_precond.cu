// Preconditioner of the contact-aware material adjoint (the reference's Woodbury correction,
// cpp/core/src/fem/deformable_projective_dynamics_backward_gpu.cpp:937-1208, solved here as one projected CG):
// the exact inverse of A on the constrained subspace.
//
// For r with J r = 0 (J: the selected unit directions d_b, b in {n, t1, t2}, at the constrained nodes), the
// minimiser of z^T A z / 2 - r^T z subject to J z = 0 is  z = A^-1 (r - J^T lam),  lam = (J A^-1 J^T)^-1 J A^-1 r.
// The directions form one orthonormal basis shared by every node and A is the same for x, y and z, so J A^-1 J^T
// is block diagonal over the three directions, each block the node block G of A^-1 restricted to that
// direction's nodes; their inverse factors X_b = L_b^-1 (G_b = L_b L_b^T) are formed once per adjoint step.
// Per CG iteration:  y = S r;  u_b = d_b . (A^-1 r) at the constrained nodes (dots of their S column paths with y);
// lam_b = X_b^T X_b u_b;  y -= S J^T lam (by the constrained candidates' S column paths);  z = S^T y.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace dphd {

namespace {

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__global__ void __launch_bounds__(256) k_wbp_jdot(const int* __restrict__ count, const int* __restrict__ wcand,
                                                  const int* __restrict__ wpos, ContactDev c, const T* __restrict__ y,
                                                  int npad, WbpDirs dirs, int cap, double* __restrict__ u,
                                                  const Ctrl* ctrl) {
    if (ctrl->done) return;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= *count) return;
    const int k = wcand[i];
    const int64_t o = c.off[k];
    const int L = (int)(c.off[k + 1] - o);
    double s0 = 0, s1 = 0, s2 = 0;
    for (int d = lane; d < L; d += 32) {
        const int r = c.prow[o + d];
        const double v = c.pval[o + d];
        s0 += v * (double)y[r];
        s1 += v * (double)y[npad + r];
        s2 += v * (double)y[2 * (size_t)npad + r];
    }
    s0 = wsum(s0);
    s1 = wsum(s1);
    s2 = wsum(s2);
    if (lane == 0)
        for (int b = 0; b < 3; ++b) {
            const int pos = wpos[3 * i + b];
            if (pos >= 0) u[b * cap + pos] = dirs.d[b][0] * s0 + dirs.d[b][1] * s1 + dirs.d[b][2] * s2;
        }
}

// w_b = X_b u_b (X_b lower triangular at X + b * ld * ld, leading dimension ld); one warp per row.
__global__ void __launch_bounds__(256) k_wbp_trmv(const int* __restrict__ nb, const double* __restrict__ X, int ld,
                                                  const double* __restrict__ u, double* __restrict__ w, int cap,
                                                  const Ctrl* ctrl) {
    if (ctrl->done) return;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int b = (int)(gw / cap), i = (int)(gw % cap);
    if (b >= 3 || i >= nb[b]) return;
    const double* Xi = X + (size_t)b * ld * ld + (size_t)i * ld;
    const double* ub = u + (size_t)b * cap;
    double s = 0.0;
    for (int j = lane; j <= i; j += 32) s += Xi[j] * ub[j];
    s = wsum(s);
    if (lane == 0) w[(size_t)b * cap + i] = s;
}

// lam_b = X_b^T w_b from the stored transpose Xt_b (row j holds column j of X_b from its diagonal on); one warp
// per row.
__global__ void __launch_bounds__(256) k_wbp_trmvt(const int* __restrict__ nb, const double* __restrict__ Xt, int ld,
                                                   const double* __restrict__ w, double* __restrict__ lam, int cap,
                                                   const Ctrl* ctrl) {
    if (ctrl->done) return;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int b = (int)(gw / cap), j = (int)(gw % cap);
    if (b >= 3) return;
    const int n = nb[b];
    if (j >= n) return;
    const double* Xj = Xt + (size_t)b * ld * ld + (size_t)j * ld;
    const double* wb = w + (size_t)b * cap;
    double s = 0.0;
    for (int i = j + lane; i < n; i += 32) s += Xj[i] * wb[i];
    s = wsum(s);
    if (lane == 0) lam[(size_t)b * cap + j] = s;
}

// Xt = the transpose of the lower triangle of X (n x n, leading dimension ld), 32 x 32 tiles through shared memory.
__global__ void k_wbp_transpose(int n, const double* __restrict__ X, double* __restrict__ Xt, int ld) {
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // source rows by.., columns bx..
    if (bx > by + 31) return;                              // entirely above the diagonal: nothing to copy
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = by + r, j = bx + threadIdx.x;
        tile[r][threadIdx.x] = (i < n && j < n && j <= i) ? X[(size_t)i * ld + j] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = bx + r, j = by + threadIdx.x;  // destination row i (= source column), column j (= source row)
        if (i < n && j < n && j >= i) Xt[(size_t)i * ld + j] = tile[threadIdx.x][r];
    }
}

// The S-pass input -J^T lam at the constrained candidates (zero at the others), per candidate: S (-J^T lam) is
// then applied by the candidates' S column paths.
__global__ void k_wbp_scatter(const int* __restrict__ count, const int* __restrict__ wcand, const int* __restrict__ wpos,
                              WbpDirs dirs, int cap, const double* __restrict__ lam, double* __restrict__ vk,
                              const Ctrl* ctrl) {
    if (ctrl->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count) return;
    double v[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < 3; ++b) {
        const int pos = wpos[3 * i + b];
        if (pos < 0) continue;
        const double l = lam[(size_t)b * cap + pos];
        for (int d = 0; d < 3; ++d) v[d] -= l * dirs.d[b][d];
    }
    double* o = vk + 3 * (size_t)wcand[i];
    o[0] = v[0];
    o[1] = v[1];
    o[2] = v[2];
}

// G_b (the direction's constrained candidates, identity-padded to n_pad) and X_b = I before the factorisation.
__global__ void k_wbp_gather_g(int n, int n_pad, const int* __restrict__ idx, const double* __restrict__ G, int K,
                               double* __restrict__ M, double* __restrict__ X, int ldx) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n_pad * n_pad) return;
    const int i = (int)(t / n_pad), j = (int)(t % n_pad);
    M[t] = (i < n && j < n) ? G[(size_t)idx[i] * K + idx[j]] : (i == j ? 1.0 : 0.0);
    X[(size_t)i * ldx + j] = i == j ? 1.0 : 0.0;
}

}  // namespace

template <typename T>
void launch_wbp_precond_parts(int stage, int cap, const int* count, const int* wcand, const int* wpos, const int* nb,
                              const ContactDev& c, const WbpDirs& dirs, const T* y, int npad, const double* X, int ld,
                              double* u, double* w, double* lam, double* vk, const Ctrl* ctrl, cudaStream_t st) {
    if (cap <= 0) return;
    if (stage == 0) {  // u = J A^-1 r, lam = (J A^-1 J^T)^-1 u (X: three blocks, then their three transposes)
        const double* Xt = X + (size_t)3 * ld * ld;
        k_wbp_jdot<T><<<(cap * 32 + 255) / 256, 256, 0, st>>>(count, wcand, wpos, c, y, npad, dirs, cap, u, ctrl);
        k_wbp_trmv<<<(unsigned)(((long long)3 * cap * 32 + 255) / 256), 256, 0, st>>>(nb, X, ld, u, w, cap, ctrl);
        k_wbp_trmvt<<<(unsigned)(((long long)3 * cap * 32 + 255) / 256), 256, 0, st>>>(nb, Xt, ld, w, lam, cap, ctrl);
    } else {  // the S-pass input -J^T lam, per candidate
        k_wbp_scatter<<<(cap + 255) / 256, 256, 0, st>>>(count, wcand, wpos, dirs, cap, lam, vk, ctrl);
    }
}
template void launch_wbp_precond_parts<double>(int, int, const int*, const int*, const int*, const int*,
                                               const ContactDev&, const WbpDirs&, const double*, int, const double*,
                                               int, double*, double*, double*, double*, const Ctrl*, cudaStream_t);
template void launch_wbp_precond_parts<float>(int, int, const int*, const int*, const int*, const int*,
                                              const ContactDev&, const WbpDirs&, const float*, int, const double*,
                                              int, double*, double*, double*, double*, const Ctrl*, cudaStream_t);

void launch_wbp_transpose(int n, const double* X, double* Xt, int ld, cudaStream_t st) {
    if (n <= 0) return;
    const int nt = (n + 31) / 32;
    k_wbp_transpose<<<dim3(nt, nt), dim3(32, 8), 0, st>>>(n, X, Xt, ld);
}

void launch_wbp_gather_g(int n, int n_pad, const int* idx, const double* G, int K, double* M, double* X, int ldx,
                         cudaStream_t st) {
    const long long t = (long long)n_pad * n_pad;
    if (t > 0) k_wbp_gather_g<<<(unsigned)((t + 255) / 256), 256, 0, st>>>(n, n_pad, idx, G, K, M, X, ldx);
}

}  // namespace dphd
