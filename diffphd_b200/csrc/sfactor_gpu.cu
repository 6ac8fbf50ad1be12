// Device construction of the sparse-inverse factor S (the plan and its formulas are in sfactor_plan.cpp).
//
// Per device-built supernode s = rows [a, a + w) (postorder, so every descendant row is final):
//   k_sfb_w        X = [W | I] with W[r][p] = sum_{d in A-row a+r, lo_k <= d <= k} A[a+r][d] S[k][d], k = B_s[p]
//   k_sfb_init_c   C = A[s, s] (padding rows / columns: identity)
//   k_sfb_syrk     C -= W W^T (lower 64 x 64 tiles)
//   k_sfb_chol     C = L L^T and X <- L^-1 X  (one cooperative grid, blocked right-looking, bounded barriers)
//   k_sfb_gemm     S[a + r][c] = -sum_p V[r][p] S[B_p][c] for c in [lo_s, a)   (V = X's first nB columns)
//   k_sfb_tri      S[a + r][a + c] = T[r][c], c <= r                                (T = X's last w columns)
// All FP64; the FP32 copy is rounded from it afterwards.  S values live in the padded row layout of the SpMV
// pair: row i at vals[row_off[i]], columns row_a[i] .. row_a[i] + row_len[i] (zero outside [lo_i, i]).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "engine.h"

namespace dphd {

namespace {

constexpr int kT = kSbTile;       // 64
constexpr int kLd = kT + 1;       // padded smem row
constexpr int kThr = 256;
constexpr long long kSpinLimit = 1ll << 24;

enum : int { kSfbBarrierTimeout = 1, kSfbNotPositive = 2 };

__device__ __forceinline__ double s_at(const double* __restrict__ vals, const int64_t* __restrict__ ro,
                                       const int* __restrict__ ra, const int* __restrict__ rl, int k, int c) {
    const int a = __ldg(ra + k);
    const int l = __ldg(rl + k);
    return (c >= a && c < a + l) ? vals[__ldg(ro + k) + (c - a)] : 0.0;
}

__global__ void k_sfb_w(int a, int w, int wpad, int nB, const int* __restrict__ B, const int64_t* __restrict__ arp,
                        const int* __restrict__ aci, const double* __restrict__ av, const int* __restrict__ lo,
                        const double* __restrict__ vals, const int64_t* __restrict__ ro, const int* __restrict__ ra,
                        const int* __restrict__ rl, double* __restrict__ X, int ldx) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)wpad * ldx;
    if (t >= total) return;
    const int r = (int)(t / ldx), p = (int)(t % ldx);
    double v = 0.0;
    if (r < w) {
        if (p < nB) {
            const int k = __ldg(B + p);
            const int lk = __ldg(lo + k);
            const int j = a + r;
            for (int64_t q = __ldg(arp + j); q < __ldg(arp + j + 1); ++q) {
                const int d = __ldg(aci + q);
                if (d >= lk && d <= k) v += __ldg(av + q) * s_at(vals, ro, ra, rl, k, d);
            }
        } else {
            v = (p - nB == r) ? 1.0 : 0.0;
        }
    }
    X[t] = v;
}

// C = A[s, s] (dense, ld = wpad), padding rows: identity.  One CTA per row.
__global__ void k_sfb_init_c(int a, int w, int wpad, const int64_t* __restrict__ arp, const int* __restrict__ aci,
                             const double* __restrict__ av, double* __restrict__ C) {
    const int r = blockIdx.x;
    double* row = C + (size_t)r * wpad;
    for (int c = threadIdx.x; c < wpad; c += blockDim.x) row[c] = (r >= w && c == r) ? 1.0 : 0.0;
    __syncthreads();
    if (r >= w || threadIdx.x != 0) return;
    const int j = a + r;
    for (int64_t q = arp[j]; q < arp[j + 1]; ++q) {
        const int d = aci[q];
        if (d >= a && d < a + w) row[d - a] += av[q];
    }
}

// 64 x 64 tile product acc += A B^T with A, B given k-major in shared memory (sA[k][r], sB[k][c]).
__device__ __forceinline__ void tile_fma(const double* sA, const double* sB, int kk, double (&acc)[4][4]) {
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll 4
    for (int k = 0; k < kk; ++k) {
        double av[4], bv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) av[u] = sA[k * kLd + ty * 4 + u];
#pragma unroll
        for (int v = 0; v < 4; ++v) bv[v] = sB[k * kLd + tx * 4 + v];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] += av[u] * bv[v];
    }
}

// C[i][j] -= sum_p W[i][p] W[j][p] over the lower tiles (j <= i); W = X's first nB columns (rows >= w are 0).
__global__ void __launch_bounds__(kThr) k_sfb_syrk(int wpad, int nB, const double* __restrict__ X, int ldx,
                                                   double* __restrict__ C) {
    constexpr int kK = 32;  // reduction chunk (two 32 x 65 operand tiles stay within static shared memory)
    __shared__ double sA[kK * kLd], sB[kK * kLd];
    const int w = blockIdx.x;
    int ti = (int)((sqrt(8.0 * (double)w + 1.0) - 1.0) * 0.5);
    while ((ti + 1) * (ti + 2) / 2 <= w) ++ti;
    while (ti * (ti + 1) / 2 > w) --ti;
    const int tj = w - ti * (ti + 1) / 2;
    double acc[4][4] = {};
    for (int p0 = 0; p0 < nB; p0 += kK) {
        __syncthreads();
        for (int t = threadIdx.x; t < kK * kT; t += blockDim.x) {
            const int r = t / kK, k = t % kK;
            const bool in = p0 + k < nB;
            sA[k * kLd + r] = in ? X[(size_t)(ti * kT + r) * ldx + p0 + k] : 0.0;
            sB[k * kLd + r] = in ? X[(size_t)(tj * kT + r) * ldx + p0 + k] : 0.0;
        }
        __syncthreads();
        tile_fma(sA, sB, kK, acc);
    }
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) C[(size_t)(ti * kT + ty * 4 + u) * wpad + tj * kT + tx * 4 + v] -= acc[u][v];
}

__device__ __forceinline__ bool sfb_grid_sync(unsigned int* bar, int* status) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vbar = bar;
        int ok = vbar[2] == 0u;
        if (ok) {
            const unsigned int gen = vbar[1];
            __threadfence();
            const unsigned int arrived = atomicAdd(bar, 1u);
            if (arrived == gridDim.x - 1) {
                vbar[0] = 0u;
                __threadfence();
                atomicAdd(bar + 1, 1u);
            } else {
                long long spins = 0;
                while (vbar[1] == gen) {
                    if (vbar[2] != 0u || ++spins > kSpinLimit) {
                        ok = 0;
                        break;
                    }
                    __nanosleep(64);
                }
                if (!ok && vbar[2] == 0u) {
                    atomicExch(bar + 2, 1u);
                    atomicOr(status, kSfbBarrierTimeout);
                }
            }
            __threadfence();
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// C = L L^T (lower, ld = n = nb * 64) and X <- L^-1 X (n rows, ncols columns, ld ldx), blocked right-looking.
__global__ void __launch_bounds__(kThr, 1) k_sfb_chol(double* __restrict__ M, int n, double* __restrict__ X, int ldx,
                                                     int ncols, unsigned int* bar, int* status) {
    extern __shared__ double sm[];
    double* sD = sm;               // diagonal block, row-major
    double* sA = sm + kT * kLd;    // panel / k-major operand
    double* sB = sm + 2 * kT * kLd;
    __shared__ double piv;
    const int tid = threadIdx.x, nt = blockDim.x, G = gridDim.x, bid = blockIdx.x;
    const int nb = n / kT, nxc = (ncols + kT - 1) / kT;
    for (int kb = 0; kb < nb; ++kb) {
        const int below = nb - kb - 1;
        // every CTA factors the diagonal block (it needs L_kk for its panels and right-hand-side chunks)
        const double* Dg = M + (size_t)kb * kT * n + kb * kT;
        for (int t = tid; t < kT * kT; t += nt) {
            const int r = t / kT, l = t % kT;
            if (l <= r) sD[r * kLd + l] = Dg[(size_t)r * n + l];
        }
        __syncthreads();
        for (int j = 0; j < kT; ++j) {
            if (tid == 0) {
                const double d = sD[j * kLd + j];
                if (!(d > 0.0) && bid == 0) atomicOr(status, kSfbNotPositive);
                piv = sqrt(d > 1e-300 ? d : 1e-300);
                sD[j * kLd + j] = piv;
            }
            __syncthreads();
            const double inv = 1.0 / piv;
            for (int r = j + 1 + tid; r < kT; r += nt) sD[r * kLd + j] *= inv;
            __syncthreads();
            const int rem = kT - j - 1;
            for (int t = tid; t < rem * rem; t += nt) {
                const int r = j + 1 + t / rem, l = j + 1 + t % rem;
                if (l <= r) sD[r * kLd + l] -= sD[r * kLd + j] * sD[l * kLd + j];
            }
            __syncthreads();
        }
        // panel tiles L[i, kb] = M[i, kb] L_kk^-T and right-hand-side chunks Y_kb = L_kk^-1 X_kb
        for (int item = bid; item < below + nxc; item += G) {
            __syncthreads();
            if (item < below) {
                double* Pg = M + (size_t)(kb + 1 + item) * kT * n + kb * kT;
                for (int t = tid; t < kT * kT; t += nt) sA[(t / kT) * kLd + t % kT] = Pg[(size_t)(t / kT) * n + t % kT];
                __syncthreads();
                if (tid < kT) {  // row tid: x L_kk^T = m, four independent partial sums per dot
                    double* row = sA + tid * kLd;
                    for (int j = 0; j < kT; ++j) {
                        const double* Lj = sD + j * kLd;
                        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                        int l = 0;
                        for (; l + 4 <= j; l += 4) {
                            s0 += row[l] * Lj[l];
                            s1 += row[l + 1] * Lj[l + 1];
                            s2 += row[l + 2] * Lj[l + 2];
                            s3 += row[l + 3] * Lj[l + 3];
                        }
                        for (; l < j; ++l) s0 += row[l] * Lj[l];
                        row[j] = (row[j] - ((s0 + s1) + (s2 + s3))) / Lj[j];
                    }
                }
                __syncthreads();
                for (int t = tid; t < kT * kT; t += nt) Pg[(size_t)(t / kT) * n + t % kT] = sA[(t / kT) * kLd + t % kT];
            } else {
                const int c0 = (item - below) * kT;
                double* Xg = X + (size_t)kb * kT * ldx + c0;
                for (int t = tid; t < kT * kT; t += nt) {
                    const int r = t / kT, c = t % kT;
                    sA[r * kLd + c] = (c0 + c < ncols) ? Xg[(size_t)r * ldx + c] : 0.0;
                }
                __syncthreads();
                if (tid < kT) {  // column tid: forward substitution with L_kk (four partial sums per dot)
                    for (int r = 0; r < kT; ++r) {
                        const double* Lr = sD + r * kLd;
                        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                        int l = 0;
                        for (; l + 4 <= r; l += 4) {
                            s0 += Lr[l] * sA[l * kLd + tid];
                            s1 += Lr[l + 1] * sA[(l + 1) * kLd + tid];
                            s2 += Lr[l + 2] * sA[(l + 2) * kLd + tid];
                            s3 += Lr[l + 3] * sA[(l + 3) * kLd + tid];
                        }
                        for (; l < r; ++l) s0 += Lr[l] * sA[l * kLd + tid];
                        sA[r * kLd + tid] = (sA[r * kLd + tid] - ((s0 + s1) + (s2 + s3))) / Lr[r];
                    }
                }
                __syncthreads();
                for (int t = tid; t < kT * kT; t += nt) {
                    const int r = t / kT, c = t % kT;
                    if (c0 + c < ncols) Xg[(size_t)r * ldx + c] = sA[r * kLd + c];
                }
            }
        }
        if (!sfb_grid_sync(bar, status)) return;
        if (bid == 0) {  // every CTA has read M[kb][kb]: store L_kk
            double* Dw = M + (size_t)kb * kT * n + kb * kT;
            for (int t = tid; t < kT * kT; t += nt) {
                const int r = t / kT, l = t % kT;
                if (l <= r) Dw[(size_t)r * n + l] = sD[r * kLd + l];
            }
        }
        // trailing updates: M[i][j] -= L[i,kb] L[j,kb]^T (kb < j <= i) and X_i -= L[i,kb] Y_kb
        const int ntri = below * (below + 1) / 2;
        const int ty = tid >> 4, tx = tid & 15;
        for (int item = bid; item < ntri + below * nxc; item += G) {
            __syncthreads();
            int i, j = -1, c0 = 0;
            if (item < ntri) {
                int ii = (int)((sqrt(8.0 * (double)item + 1.0) - 1.0) * 0.5);
                while ((ii + 1) * (ii + 2) / 2 <= item) ++ii;
                while (ii * (ii + 1) / 2 > item) --ii;
                i = kb + 1 + ii;
                j = kb + 1 + (item - ii * (ii + 1) / 2);
            } else {
                const int q = item - ntri;
                i = kb + 1 + q / nxc;
                c0 = (q % nxc) * kT;
            }
            const double* Pi = M + (size_t)i * kT * n + kb * kT;
            for (int t = tid; t < kT * kT; t += nt) {
                const int r = t / kT, k = t % kT;
                sA[k * kLd + r] = Pi[(size_t)r * n + k];
            }
            if (j >= 0) {
                const double* Pj = M + (size_t)j * kT * n + kb * kT;
                for (int t = tid; t < kT * kT; t += nt) {
                    const int r = t / kT, k = t % kT;
                    sB[k * kLd + r] = Pj[(size_t)r * n + k];
                }
            } else {
                const double* Yg = X + (size_t)kb * kT * ldx + c0;
                for (int t = tid; t < kT * kT; t += nt) {
                    const int k = t / kT, c = t % kT;
                    sB[k * kLd + c] = (c0 + c < ncols) ? Yg[(size_t)k * ldx + c] : 0.0;
                }
            }
            __syncthreads();
            double acc[4][4] = {};
            tile_fma(sA, sB, kT, acc);
            if (j >= 0) {
                double* Cg = M + (size_t)i * kT * n + j * kT;
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 4; ++v) Cg[(size_t)(ty * 4 + u) * n + tx * 4 + v] -= acc[u][v];
            } else {
                double* Xi = X + (size_t)i * kT * ldx + c0;
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 4; ++v)
                        if (c0 + tx * 4 + v < ncols) Xi[(size_t)(ty * 4 + u) * ldx + tx * 4 + v] -= acc[u][v];
            }
        }
        if (!sfb_grid_sync(bar, status)) return;
    }
}

// S[a + r][c] = -sum_{p in list(ct)} V[r][p] S[B_p][c], output tile (64 rows of s) x (64 columns from ra + 64 ct),
// written for c in [lo, a).
__global__ void __launch_bounds__(kThr) k_sfb_gemm(int a, int w, int lo, int ra, int nB, const int* __restrict__ B,
                                                   const int64_t* __restrict__ ct_ptr, const int* __restrict__ ct_p,
                                                   const double* __restrict__ X, int ldx, double* __restrict__ vals,
                                                   const int64_t* __restrict__ ro, const int* __restrict__ rra,
                                                   const int* __restrict__ rl) {
    constexpr int kK = 16;
    __shared__ double sA[kK * kLd], sB[kK * kLd];
    __shared__ int sk[kK], sp[kK];
    const int rt = blockIdx.y, ct = blockIdx.x;
    const int64_t q0 = ct_ptr[ct], q1 = ct_ptr[ct + 1];
    const int c0 = ra + ct * kT;
    double acc[4][4] = {};
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
    for (int64_t qb = q0; qb < q1; qb += kK) {
        __syncthreads();
        if (threadIdx.x < kK) {
            const int64_t q = qb + threadIdx.x;
            const int p = q < q1 ? ct_p[q] : -1;
            sp[threadIdx.x] = p;
            sk[threadIdx.x] = p >= 0 ? B[p] : -1;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < kK * kT; t += blockDim.x) {
            const int kk = t / kT, x = t % kT;
            const int p = sp[kk], k = sk[kk];
            // V[r][p]: row rt*64 + x of X (rows >= w of X are zero)
            sA[kk * kLd + x] = p >= 0 ? X[(size_t)(rt * kT + x) * ldx + p] : 0.0;
            sB[kk * kLd + x] = k >= 0 ? s_at(vals, ro, rra, rl, k, c0 + x) : 0.0;
        }
        __syncthreads();
        tile_fma(sA, sB, kK, acc);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int r = rt * kT + ty * 4 + u;
        if (r >= w) continue;
        double* row = vals + ro[a + r] - ra;  // row a + r starts at column ra (all rows of s share lo)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int c = c0 + tx * 4 + v;
            if (c >= lo && c < a) row[c] = -acc[u][v];
        }
    }
}

__global__ void k_sfb_tri(int a, int w, int ra, int nB, const double* __restrict__ X, int ldx,
                          double* __restrict__ vals, const int64_t* __restrict__ ro) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)w * w) return;
    const int r = (int)(t / w), c = (int)(t % w);
    if (c > r) return;
    vals[ro[a + r] + (a + c - ra)] = X[(size_t)r * ldx + nB + c];
}

__global__ void k_to_f32(const double* __restrict__ in, float* __restrict__ out, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

__global__ void k_path_vals(int K, const int64_t* __restrict__ off, const int* __restrict__ prow,
                            const int* __restrict__ cand, const int* __restrict__ iperm, const double* __restrict__ vals,
                            const int64_t* __restrict__ ro, const int* __restrict__ ra, double* __restrict__ pval) {
    const int c = blockIdx.x;
    if (c >= K) return;
    const int col = iperm[cand[c]];
    for (int64_t q = off[c] + threadIdx.x; q < off[c + 1]; q += blockDim.x) {
        const int r = prow[q];
        pval[q] = vals[ro[r] + (col - ra[r])];
    }
}

template <typename T>
void upload_vec(DeviceBuffer& b, const std::vector<T>& v) {
    b.alloc(std::max<size_t>(1, v.size()) * sizeof(T));
    if (!v.empty()) CUDA_OK(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}

}  // namespace

void device_build_factor(const SBuildPlan& P, const std::vector<int>& lo, const int64_t* d_ro, const int* d_ra,
                         const int* d_rl, double* d_vals, cudaStream_t st) {
    DeviceBuffer d_lo, d_arp, d_aci, d_av, d_B, d_ctptr, d_ctp, d_X, d_C, d_bar, d_status;
    upload_vec(d_lo, lo);
    upload_vec(d_arp, P.a_rp);
    upload_vec(d_aci, P.a_ci);
    upload_vec(d_av, P.a_v);
    upload_vec(d_B, P.B);
    upload_vec(d_ctptr, P.ct_ptr);
    upload_vec(d_ctp, P.ct_p);
    d_X.alloc(std::max<int64_t>(1, P.max_x) * sizeof(double));
    const size_t wpad_max = (size_t)(P.max_w + kT - 1) / kT * kT;
    d_C.alloc(std::max<size_t>(1, wpad_max * wpad_max) * sizeof(double));
    d_bar.alloc(4 * sizeof(unsigned int));
    d_status.alloc(sizeof(int));
    CUDA_OK(cudaMemsetAsync(d_bar.p, 0, d_bar.bytes, st));
    CUDA_OK(cudaMemsetAsync(d_status.p, 0, sizeof(int), st));
    const size_t chol_smem = (size_t)3 * kT * kLd * sizeof(double);
    CUDA_OK(cudaFuncSetAttribute(k_sfb_chol, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chol_smem));
    const int sms = device_sms();
    for (const SBigSuper& s : P.sup) {
        const int w = s.b - s.a, wpad = (w + kT - 1) / kT * kT, nB = s.nB, ldx = nB + w;
        const int* B = d_B.as<int>() + s.B_off;
        double* X = d_X.as<double>();
        double* C = d_C.as<double>();
        const long long nx = (long long)wpad * ldx;
        k_sfb_w<<<(unsigned)((nx + 255) / 256), 256, 0, st>>>(s.a, w, wpad, nB, B, d_arp.as<int64_t>(), d_aci.as<int>(),
                                                              d_av.as<double>(), d_lo.as<int>(), d_vals, d_ro, d_ra,
                                                              d_rl, X, ldx);
        k_sfb_init_c<<<wpad, 256, 0, st>>>(s.a, w, wpad, d_arp.as<int64_t>(), d_aci.as<int>(), d_av.as<double>(), C);
        const int nbw = wpad / kT;
        if (nB > 0) k_sfb_syrk<<<nbw * (nbw + 1) / 2, kThr, 0, st>>>(wpad, nB, X, ldx, C);
        {
            const int nxc = (ldx + kT - 1) / kT;
            const int grid = std::max(1, std::min(sms, nbw * nxc));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(grid);
            cfg.blockDim = dim3(kThr);
            cfg.dynamicSmemBytes = chol_smem;
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            CUDA_OK(cudaLaunchKernelEx(&cfg, k_sfb_chol, C, wpad, X, ldx, ldx, d_bar.as<unsigned int>(),
                                       d_status.as<int>()));
        }
        if (nB > 0 && s.nct > 0)
            k_sfb_gemm<<<dim3(s.nct, nbw), kThr, 0, st>>>(s.a, w, s.lo, s.ra, nB, B, d_ctptr.as<int64_t>() + s.ct_off,
                                                          d_ctp.as<int>(), X, ldx, d_vals, d_ro, d_ra, d_rl);
        k_sfb_tri<<<(unsigned)(((long long)w * w + 255) / 256), 256, 0, st>>>(s.a, w, s.ra, nB, X, ldx, d_vals, d_ro);
        CUDA_OK(cudaGetLastError());
    }
    int status = 0;
    CUDA_OK(cudaMemcpyAsync(&status, d_status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    DPHD_CHECK(!(status & kSfbBarrierTimeout), "device factor build: a grid barrier timed out");
    DPHD_CHECK(!(status & kSfbNotPositive), "PD matrix is not positive definite (device factor build)");
}

void dense_chol_solve(double* M, int n, double* X, int ldx, int ncols, cudaStream_t st) {
    DPHD_CHECK(n % kT == 0, "dense_chol_solve: n must be a multiple of 64");
    if (n == 0) return;
    DeviceBuffer d_bar, d_status;
    d_bar.alloc(4 * sizeof(unsigned int));
    d_status.alloc(sizeof(int));
    CUDA_OK(cudaMemsetAsync(d_bar.p, 0, d_bar.bytes, st));
    CUDA_OK(cudaMemsetAsync(d_status.p, 0, sizeof(int), st));
    const size_t chol_smem = (size_t)3 * kT * kLd * sizeof(double);
    CUDA_OK(cudaFuncSetAttribute(k_sfb_chol, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chol_smem));
    const int nbw = n / kT, nxc = (ncols + kT - 1) / kT;
    const int grid = std::max(1, std::min(device_sms(), nbw * std::max(nxc, 1)));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kThr);
    cfg.dynamicSmemBytes = chol_smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_OK(cudaLaunchKernelEx(&cfg, k_sfb_chol, M, n, X, ldx, ncols, d_bar.as<unsigned int>(), d_status.as<int>()));
    int status = 0;
    CUDA_OK(cudaMemcpyAsync(&status, d_status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    DPHD_CHECK(!(status & kSfbBarrierTimeout), "dense Cholesky: a grid barrier timed out");
    DPHD_CHECK(!(status & kSfbNotPositive), "dense Cholesky: matrix is not positive definite");
}

void device_round_f32(const double* d_in, float* d_out, long long n, cudaStream_t st) {
    if (n <= 0) return;
    k_to_f32<<<4 * device_sms(), 256, 0, st>>>(d_in, d_out, n);
    CUDA_OK(cudaGetLastError());
}

void device_path_vals(int K, const int64_t* d_off, const int* d_prow, const int* d_cand, const int* d_iperm,
                      const double* d_vals, const int64_t* d_ro, const int* d_ra, double* d_pval, cudaStream_t st) {
    if (K <= 0) return;
    k_path_vals<<<K, 256, 0, st>>>(K, d_off, d_prow, d_cand, d_iperm, d_vals, d_ro, d_ra, d_pval);
    CUDA_OK(cudaGetLastError());
}

}  // namespace dphd
