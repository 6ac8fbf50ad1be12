// Signorini–Coulomb contact for a planar frictional boundary, inside the PD iteration
// (ForwardProjectiveDynamicsAlgPhd, cpp/core/src/fem/deformable_projective_dynamics_forward_gpu.cpp:461-528,
// 849-1061, 1116-1321, 1483-1545).
//
// Delassus operator.  With one node-level A for all axes, (A^-1 (n_j e_j))_i = G_ij n_j with G the node block
// of A^-1 = S^T S at the candidates, so W_ij = (n_i . n_j) G_ij and the tangential 2x2 blocks are G_ii I.  A does
// not change between frames, so G is formed once per factor build: G_ij is the dot product of two S columns,
// whose nonzeros are the etree paths of the two columns, i.e. a dot product over the shared root-first prefix.
//
// Each PD iteration: (1) delta_j = n . q_j + offset for every candidate; candidates with lambda_j = 0 and
// delta_j > 0 have omega_j = 0, E_j = r_j, phi_j = 0, so their rows and columns of M = Omega W Omega + E
// decouple with Delta lambda_j = 0 exactly — only the others (the active set) enter the dense solve;
// (2) A^-1 b at active nodes from y = S b through the S column paths; (3) M Delta lambda = h - J A^-1 g by a
// dense Cholesky factorisation, clamp lambda to [0, 1e8], Coulomb cone per contact; (4) the contact impulse
// J^T f is written as a sparse right-hand side so that y += S J^T f before the single S^T pass.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace dphd {

namespace {

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// G_ij for i <= j, one warp per pair (prefix of matching rows from the root).
__global__ void __launch_bounds__(256) k_delassus(int K, const int64_t* __restrict__ off, const int* __restrict__ prow,
                                                  const double* __restrict__ pval, double* __restrict__ G) {
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long npairs = (long long)K * (K + 1) / 2;
    if (w >= npairs) return;
    // w -> (i, j) with i <= j, row-major over the upper triangle
    long long i = (long long)((sqrt(8.0 * (double)w + 1.0) - 1.0) / 2.0);  // j index in tri ordering
    while ((i + 1) * (i + 2) / 2 <= w) ++i;
    while (i * (i + 1) / 2 > w) --i;
    const int j = (int)i;
    const int ii = (int)(w - i * (i + 1) / 2);  // ii <= j
    const int64_t oa = off[ii], ob = off[j];
    const int la = (int)(off[ii + 1] - oa), lb = (int)(off[j + 1] - ob);
    const int L = min(la, lb);
    double s = 0.0;
    bool matching = true;
    for (int base = 0; base < L && matching; base += 32) {
        const int d = base + lane;
        const bool in = d < L;
        const bool eq = in && prow[oa + d] == prow[ob + d];
        const unsigned mism = __ballot_sync(0xffffffffu, in && !eq);
        const int first_bad = mism ? __ffs(mism) - 1 : 32;
        if (lane < first_bad && in) s += pval[oa + d] * pval[ob + d];
        if (mism) matching = false;
    }
    s = warp_sum_d(s);
    if (lane == 0) {
        G[(size_t)ii * K + j] = s;
        G[(size_t)j * K + ii] = s;
    }
}

// Block-wide exclusive scan of 0/1 flags over K candidates (one CTA), producing the ordered active list.
__global__ void __launch_bounds__(1024) k_ncp_prepare(ContactDev c, const double* __restrict__ x, Ctrl* ctrl) {
    if (ctrl->done) return;
    __shared__ int warp_tot[32];
    __shared__ int base_s;
    if (threadIdx.x == 0) base_s = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int b0 = 0; b0 < c.K; b0 += blockDim.x) {
        const int k = b0 + threadIdx.x;
        int act = 0;
        if (k < c.K) {
            const int node = c.cand[k];
            const double dj = c.n[0] * x[3 * node] + c.n[1] * x[3 * node + 1] + c.n[2] * x[3 * node + 2] + c.offset;
            const double lj = c.lam[k], rj = c.rprec[k];
            double den = sqrt(dj * dj + rj * rj * lj * lj);
            if (den < 1e-14) den = 1e-14;
            const double om = 1.0 - dj / den;
            const double E = (1.0 - rj * lj / den) * rj;
            const double phi = dj + rj * lj - den;
            const double Hq = dj - c.offset;
            c.omega[k] = om;
            c.Ediag[k] = E;
            c.hvec[k] = -phi + om * Hq;
            act = (lj > 0.0 || dj <= 0.0) ? 1 : 0;
        }
        // scan
        const unsigned bal = __ballot_sync(0xffffffffu, act);
        const int pre = __popc(bal & ((1u << lane) - 1u));
        if (lane == 0) warp_tot[wid] = __popc(bal);
        __syncthreads();
        int woff = 0;
        for (int w = 0; w < wid; ++w) woff += warp_tot[w];
        if (act) c.act[base_s + woff + pre] = k;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += warp_tot[w];
            base_s += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) c.kact[0] = base_s;
}

// A^-1 b at active candidate nodes: dot of the node's S column path with y = S b (3 right-hand sides).
template <typename T>
__global__ void __launch_bounds__(256) k_ncp_ainvb(ContactDev c, const T* __restrict__ y, int npad,
                                                   const double* __restrict__ x_base, const Ctrl* ctrl) {
    if (ctrl->done) return;
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= c.kact[0]) return;
    const int k = c.act[a];
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
    s0 = warp_sum_d(s0);
    s1 = warp_sum_d(s1);
    s2 = warp_sum_d(s2);
    if (lane == 0) {
        const int node = c.cand[k];
        c.ainvb[3 * a] = s0 + (x_base ? x_base[3 * node] : 0.0);
        c.ainvb[3 * a + 1] = s1 + (x_base ? x_base[3 * node + 1] : 0.0);
        c.ainvb[3 * a + 2] = s2 + (x_base ? x_base[3 * node + 2] : 0.0);
    }
}

// ---- Dense solve of the active NCP system (multi-CTA, one cooperative launch per PD iteration) -------------
//
// M = Omega G Omega + E over the ka active candidates (ka <= K, known only on the device) is factored by a
// blocked right-looking Cholesky in 64 x 64 tiles, and M dlambda = h - J A^-1 g solved, by every CTA of one
// cooperative grid (all CTAs co-resident) with grid-wide barriers between the dependent phases:
//   A  assemble M (lower triangle, padded to a multiple of 64 with identity rows) and the right-hand side;
//   B  per block column kb: factor the 64 x 64 diagonal block (redundantly in every CTA that needs it) and
//      solve its panel tiles; barrier; update the trailing lower tiles and the right-hand side; barrier;
//   C  backward substitution by block rows, one barrier per block;
//   D  clamp lambda to [0, 1e8]; barrier; Coulomb cone per active contact and the contact right-hand side.
// The barrier is a counter + generation word with a bounded spin: a CTA that waits too long sets
// kStatusBarrierTimeout and `done` in the control block and every later barrier returns at once, so the
// kernel always ends (the host turns the status into an error).
constexpr int kNcpTile = 64;
constexpr int kNcpThreads = 256;
constexpr int kNcpLd = kNcpTile + 1;  // padded smem row (doubles) for the row-major 64 x 64 tiles
constexpr long long kBarrierSpins = 1ll << 24;

// Returns false when the grid is aborting (a barrier timed out somewhere): the caller returns.
__device__ __forceinline__ bool ncp_grid_sync(unsigned int* bar, Ctrl* ctrl) {
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
                    if (vbar[2] != 0u || ++spins > kBarrierSpins) {
                        ok = 0;
                        break;
                    }
                    __nanosleep(64);
                }
                if (!ok && vbar[2] == 0u) {
                    atomicExch(bar + 2, 1u);
                    atomicOr(&ctrl->status, (int)kStatusBarrierTimeout);
                    ctrl->done = 1;
                }
            }
            __threadfence();
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Cholesky of the 64 x 64 lower block sD (row-major, ld kNcpLd) in place, the reference's pivot guard
// (sqrt(max(d, 1e-300))); all threads of the CTA take part.
__device__ void ncp_tile_cholesky(double* sD) {
    __shared__ double piv;
    for (int j = 0; j < kNcpTile; ++j) {
        if (threadIdx.x == 0) {
            const double d = sD[j * kNcpLd + j];
            piv = sqrt(d > 1e-300 ? d : 1e-300);
            sD[j * kNcpLd + j] = piv;
        }
        __syncthreads();
        const double inv = 1.0 / piv;
        for (int r = j + 1 + (int)threadIdx.x; r < kNcpTile; r += blockDim.x) sD[r * kNcpLd + j] *= inv;
        __syncthreads();
        const int rem = kNcpTile - j - 1;
        for (int t = threadIdx.x; t < rem * rem; t += blockDim.x) {
            const int r = j + 1 + t / rem, l = j + 1 + t % rem;
            if (l <= r) sD[r * kNcpLd + l] -= sD[r * kNcpLd + j] * sD[l * kNcpLd + j];
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(kNcpThreads, 1)
k_ncp_block_solve(ContactDev c, const double* __restrict__ q0, const int* __restrict__ iperm, T* __restrict__ vcon,
                  int npad, const double* __restrict__ r64, Ctrl* ctrl) {
    extern __shared__ double smem[];
    double* sA = smem;                           // 64 x kNcpLd: diagonal block / k-major panel i
    double* sB = smem + kNcpTile * kNcpLd;       // 64 x kNcpLd: panel tile / k-major panel j
    double* sy = smem + 2 * kNcpTile * kNcpLd;   // 64: the block's right-hand side / solution
    if (ctrl->done) return;  // every CTA reads the same value: no CTA reaches a barrier the others skip
    const int K = c.K, ka = c.kact[0];
    const int tid = threadIdx.x, nt = blockDim.x, G = gridDim.x, bid = blockIdx.x;
    const int gt = bid * nt + tid, nthr = G * nt;
    const int lane = tid & 31, gw = gt >> 5, nwarps = nthr >> 5;
    const double n0 = c.n[0], n1 = c.n[1], n2 = c.n[2];
    // clear the previous contact right-hand side at every candidate node
    for (int k = gt; k < K; k += nthr) {
        const int node = c.cand[k], j = iperm[node];
        vcon[j] = r64 ? (T)r64[3 * node] : T(0);
        vcon[npad + j] = r64 ? (T)r64[3 * node + 1] : T(0);
        vcon[2 * (size_t)npad + j] = r64 ? (T)r64[3 * node + 2] : T(0);
        for (int d = 0; d < 3; ++d) c.vc[3 * (size_t)k + d] = r64 ? r64[3 * node + d] : 0.0;
    }
    if (ka == 0) {
        for (int k = gt; k < K; k += nthr) c.lt1[k] = c.lt2[k] = 0.0;
        return;
    }
    const int nb = (ka + kNcpTile - 1) / kNcpTile, ld = nb * kNcpTile;
    double* M = c.Mwork;  // ld x ld, row-major, lower triangle used
    double* rhs = c.rhs;  // ld
    // ---- A: M and the right-hand side h - J A^-1 g (one warp per row) ----
    for (int a = gw; a < ld; a += nwarps) {
        double* Ma = M + (size_t)a * ld;
        if (a >= ka) {  // identity padding row
            for (int b = lane; b <= a; b += 32) Ma[b] = (a == b) ? 1.0 : 0.0;
            if (lane == 0) rhs[a] = 0.0;
            continue;
        }
        const int k = c.act[a];
        const double om = c.omega[k];
        const double* Gk = c.G + (size_t)k * K;
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
        for (int b = lane; b < ka; b += 32) {
            const int kb = c.act[b];
            const double Gab = Gk[kb];
            const double fn = c.omega[kb] * c.lam[kb];
            const double f1 = c.lt1[kb], f2 = c.lt2[kb];
            g0 += Gab * (fn * n0 + f1 * c.t1[0] + f2 * c.t2[0]);
            g1 += Gab * (fn * n1 + f1 * c.t1[1] + f2 * c.t2[1]);
            g2 += Gab * (fn * n2 + f1 * c.t1[2] + f2 * c.t2[2]);
            if (b <= a) Ma[b] = om * Gab * c.omega[kb] + (a == b ? c.Ediag[k] : 0.0);
        }
        g0 = warp_sum_d(g0);
        g1 = warp_sum_d(g1);
        g2 = warp_sum_d(g2);
        if (lane == 0) {
            g0 += c.ainvb[3 * a];
            g1 += c.ainvb[3 * a + 1];
            g2 += c.ainvb[3 * a + 2];
            rhs[a] = c.hvec[k] - om * (n0 * g0 + n1 * g1 + n2 * g2);
        }
    }
    if (!ncp_grid_sync(c.bar, ctrl)) return;
    // ---- B: blocked factorisation with the forward substitution folded in ----
    for (int kb = 0; kb < nb; ++kb) {
        const int below = nb - kb - 1;
        if (bid == 0 || bid < below) {
            const double* Dg = M + (size_t)kb * kNcpTile * ld + kb * kNcpTile;
            for (int t = tid; t < kNcpTile * kNcpTile; t += nt) {
                const int r = t / kNcpTile, l = t % kNcpTile;
                if (l <= r) sA[r * kNcpLd + l] = Dg[(size_t)r * ld + l];
            }
            if (bid == 0 && tid < kNcpTile) sy[tid] = rhs[kb * kNcpTile + tid];
            __syncthreads();
            ncp_tile_cholesky(sA);
            if (bid == 0) {  // y_kb = L_kk^-1 rhs_kb (one warp, column-oriented); L_kk goes back after the barrier
                if (tid < 32) {
                    for (int j = 0; j < kNcpTile; ++j) {
                        double yj = 0.0;
                        if (lane == 0) sy[j] /= sA[j * kNcpLd + j];
                        __syncwarp();
                        yj = sy[j];
                        for (int r = j + 1 + lane; r < kNcpTile; r += 32) sy[r] -= sA[r * kNcpLd + j] * yj;
                        __syncwarp();
                    }
                }
                __syncthreads();
                if (tid < kNcpTile) rhs[kb * kNcpTile + tid] = sy[tid];  // no other CTA reads rhs_kb in this phase
            }
            // panel tiles L[i, kb] = M[i, kb] L_kk^-T
            for (int i = kb + 1 + bid; i < nb; i += G) {
                double* Pg = M + (size_t)i * kNcpTile * ld + kb * kNcpTile;
                __syncthreads();
                for (int t = tid; t < kNcpTile * kNcpTile; t += nt) {
                    const int r = t / kNcpTile, l = t % kNcpTile;
                    sB[r * kNcpLd + l] = Pg[(size_t)r * ld + l];
                }
                __syncthreads();
                if (tid < kNcpTile) {  // row tid: x L_kk^T = m, four independent partial sums per dot
                    double* row = sB + tid * kNcpLd;
                    for (int j = 0; j < kNcpTile; ++j) {
                        const double* Lj = sA + j * kNcpLd;
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
                for (int t = tid; t < kNcpTile * kNcpTile; t += nt) {
                    const int r = t / kNcpTile, l = t % kNcpTile;
                    Pg[(size_t)r * ld + l] = sB[r * kNcpLd + l];
                }
            }
        }
        if (!ncp_grid_sync(c.bar, ctrl)) return;
        // every CTA has now read M[kb][kb]: CTA 0 stores L_kk (still in its sA) in its place
        if (bid == 0) {
            double* Dw = M + (size_t)kb * kNcpTile * ld + kb * kNcpTile;
            for (int t = tid; t < kNcpTile * kNcpTile; t += nt) {
                const int r = t / kNcpTile, l = t % kNcpTile;
                if (l <= r) Dw[(size_t)r * ld + l] = sA[r * kNcpLd + l];
            }
        }
        // trailing update M[i][j] -= L[i,kb] L[j,kb]^T for kb < j <= i, and rhs_i -= L[i,kb] y_kb
        const int ntri = below * (below + 1) / 2;
        const int ty = tid >> 4, tx = tid & 15;
        for (int w = bid; w < ntri + below; w += G) {
            __syncthreads();
            if (w < ntri) {
                int ii = (int)((sqrt(8.0 * (double)w + 1.0) - 1.0) * 0.5);
                while ((ii + 1) * (ii + 2) / 2 <= w) ++ii;
                while (ii * (ii + 1) / 2 > w) --ii;
                const int jj = w - ii * (ii + 1) / 2;
                const int i = kb + 1 + ii, j = kb + 1 + jj;
                const double* Pi = M + (size_t)i * kNcpTile * ld + kb * kNcpTile;
                const double* Pj = M + (size_t)j * kNcpTile * ld + kb * kNcpTile;
                // k-major copies: sA[k][r] = L[i*64 + r, kb*64 + k]
                for (int t = tid; t < kNcpTile * kNcpTile; t += nt) {
                    const int r = t / kNcpTile, k = t % kNcpTile;
                    sA[k * kNcpLd + r] = Pi[(size_t)r * ld + k];
                    sB[k * kNcpLd + r] = Pj[(size_t)r * ld + k];
                }
                __syncthreads();
                double acc[4][4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
#pragma unroll 4
                for (int k = 0; k < kNcpTile; ++k) {
                    double av[4], bv[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) av[u] = sA[k * kNcpLd + ty * 4 + u];
#pragma unroll
                    for (int v = 0; v < 4; ++v) bv[v] = sB[k * kNcpLd + tx * 4 + v];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) acc[u][v] += av[u] * bv[v];
                }
                double* Cg = M + (size_t)i * kNcpTile * ld + j * kNcpTile;
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 4; ++v) Cg[(size_t)(ty * 4 + u) * ld + tx * 4 + v] -= acc[u][v];
            } else {
                const int i = kb + 1 + (w - ntri);
                if (tid < kNcpTile) {
                    const double* Li = M + (size_t)(i * kNcpTile + tid) * ld + kb * kNcpTile;
                    const double* y = rhs + kb * kNcpTile;
                    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                    for (int k = 0; k < kNcpTile; k += 4) {
                        s0 += Li[k] * y[k];
                        s1 += Li[k + 1] * y[k + 1];
                        s2 += Li[k + 2] * y[k + 2];
                        s3 += Li[k + 3] * y[k + 3];
                    }
                    rhs[i * kNcpTile + tid] -= (s0 + s1) + (s2 + s3);
                }
            }
        }
        if (!ncp_grid_sync(c.bar, ctrl)) return;
    }
    // ---- C: backward substitution L^T x = y by block rows ----
    for (int kb = nb - 1; kb >= 0; --kb) {
        if (bid == 0 || bid < kb) {
            const double* Dg = M + (size_t)kb * kNcpTile * ld + kb * kNcpTile;
            __syncthreads();
            for (int t = tid; t < kNcpTile * kNcpTile; t += nt) {
                const int r = t / kNcpTile, l = t % kNcpTile;
                if (l <= r) sA[r * kNcpLd + l] = Dg[(size_t)r * ld + l];
            }
            if (tid < kNcpTile) sy[tid] = rhs[kb * kNcpTile + tid];
            __syncthreads();
            if (tid < 32) {
                for (int j = kNcpTile - 1; j >= 0; --j) {
                    if (lane == 0) sy[j] /= sA[j * kNcpLd + j];
                    __syncwarp();
                    const double xj = sy[j];
                    for (int l = lane; l < j; l += 32) sy[l] -= sA[j * kNcpLd + l] * xj;
                    __syncwarp();
                }
            }
            __syncthreads();
            if (bid == 0 && tid < kNcpTile) c.xsol[kb * kNcpTile + tid] = sy[tid];
            // rhs_p -= L[kb, p]^T x_kb for the block rows p < kb (rhs_kb itself is only read in this phase)
            for (int p = bid; p < kb; p += G) {
                if (tid < kNcpTile) {
                    const double* Lkp = M + (size_t)kb * kNcpTile * ld + p * kNcpTile + tid;
                    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                    for (int i = 0; i < kNcpTile; i += 4) {
                        s0 += Lkp[(size_t)i * ld] * sy[i];
                        s1 += Lkp[(size_t)(i + 1) * ld] * sy[i + 1];
                        s2 += Lkp[(size_t)(i + 2) * ld] * sy[i + 2];
                        s3 += Lkp[(size_t)(i + 3) * ld] * sy[i + 3];
                    }
                    rhs[p * kNcpTile + tid] -= (s0 + s1) + (s2 + s3);
                }
            }
        }
        if (!ncp_grid_sync(c.bar, ctrl)) return;
    }
    // ---- D: multipliers, Coulomb cone (forward_gpu.cpp:1255-1302), contact right-hand side ----
    for (int a = gt; a < ka; a += nthr) {
        const int k = c.act[a];
        double l = c.lam[k] + c.xsol[a];
        l = l < 0.0 ? 0.0 : (l > 1e8 ? 1e8 : l);
        c.lam[k] = l;
    }
    for (int k = gt; k < K; k += nthr) c.lt1[k] = c.lt2[k] = 0.0;  // non-active candidates carry no friction
    if (!ncp_grid_sync(c.bar, ctrl)) return;
    for (int a = gw; a < ka; a += nwarps) {
        const int k = c.act[a];
        double t1v = 0.0, t2v = 0.0;
        if (c.mu > 0.0 && c.lam[k] > 0.0) {
            const double* Gk = c.G + (size_t)k * K;
            double f = 0.0;
            for (int b = lane; b < ka; b += 32) {
                const int kb = c.act[b];
                f += c.omega[kb] * c.lam[kb] * Gk[kb];
            }
            f = warp_sum_d(f);
            const int node = c.cand[k];
            const double qn0 = c.ainvb[3 * a] + f * n0, qn1 = c.ainvb[3 * a + 1] + f * n1,
                         qn2 = c.ainvb[3 * a + 2] + f * n2;
            const double s0 = qn0 - q0[3 * node], s1 = qn1 - q0[3 * node + 1], s2 = qn2 - q0[3 * node + 2];
            const double sn = s0 * n0 + s1 * n1 + s2 * n2;
            const double u0 = s0 - sn * n0, u1 = s1 - sn * n1, u2 = s2 - sn * n2;
            const double ut1 = u0 * c.t1[0] + u1 * c.t1[1] + u2 * c.t1[2];
            const double ut2 = u0 * c.t2[0] + u1 * c.t2[1] + u2 * c.t2[2];
            const double Gkk = Gk[k];
            double st1 = 0.0, st2 = 0.0;
            if (fabs(Gkk * Gkk) > 1e-20) {
                st1 = -ut1 / Gkk;
                st2 = -ut2 / Gkk;
            }
            const double cone = c.mu * c.lam[k];
            if (sqrt(st1 * st1 + st2 * st2) <= cone + 1e-14) {
                t1v = st1;
                t2v = st2;
            } else {
                const double um = sqrt(ut1 * ut1 + ut2 * ut2);
                if (um > 1e-14) {
                    t1v = -cone * ut1 / um;
                    t2v = -cone * ut2 / um;
                }
            }
        }
        if (lane == 0) {
            c.lt1[k] = t1v;
            c.lt2[k] = t2v;
            // contact right-hand side J^T f at the node (omega from this iteration times the new lambda)
            const double fn = c.omega[k] * c.lam[k];
            const int node = c.cand[k], j = iperm[node];
            const double r0 = r64 ? r64[3 * node] : 0.0, r1 = r64 ? r64[3 * node + 1] : 0.0,
                         r2 = r64 ? r64[3 * node + 2] : 0.0;
            const double w0 = r0 + fn * n0 + t1v * c.t1[0] + t2v * c.t2[0];
            const double w1 = r1 + fn * n1 + t1v * c.t1[1] + t2v * c.t2[1];
            const double w2 = r2 + fn * n2 + t1v * c.t1[2] + t2v * c.t2[2];
            vcon[j] = (T)w0;
            vcon[npad + j] = (T)w1;
            vcon[2 * (size_t)npad + j] = (T)w2;
            c.vc[3 * (size_t)k] = w0;
            c.vc[3 * (size_t)k + 1] = w1;
            c.vc[3 * (size_t)k + 2] = w2;
        }
    }
}

// Restitution (forward_gpu.cpp:1483-1531), planar boundary.
__global__ void k_restitution(ContactDev c, double* __restrict__ q, const double* __restrict__ q0,
                              const double* __restrict__ v0, double h, double e, double slop) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.K || !(c.lam[k] > 0.0)) return;
    const int node = c.cand[k];
    const double* n = c.n;
    const double sd = n[0] * q[3 * node] + n[1] * q[3 * node + 1] + n[2] * q[3 * node + 2] + c.offset;
    if (sd > slop) return;
    const double vin = v0[3 * node] * n[0] + v0[3 * node + 1] * n[1] + v0[3 * node + 2] * n[2];
    if (!(vin < 0)) return;
    double vo = 0;
    for (int d = 0; d < 3; ++d) vo += (q[3 * node + d] - q0[3 * node + d]) / h * n[d];
    const double dv = -e * vin - vo;
    if (dv > 0)
        for (int d = 0; d < 3; ++d) q[3 * node + d] += h * dv * n[d];
}

}  // namespace

int ncp_grid() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 148;
}

size_t ncp_matrix_capacity(int K) {
    const size_t kp = ((size_t)K + kNcpTile - 1) / kNcpTile * kNcpTile;
    return kp;
}

void launch_delassus(int K, const int64_t* off, const int* prow, const double* pval, double* G, cudaStream_t st) {
    const long long npairs = (long long)K * (K + 1) / 2;
    const long long blocks = (npairs * 32 + 255) / 256;
    if (npairs > 0) k_delassus<<<(unsigned)blocks, 256, 0, st>>>(K, off, prow, pval, G);
}

template <typename T>
void launch_ncp_iteration(const ContactDev& c, const double* x, const T* y, int npad, const double* x_base,
                          const double* q0, const int* iperm, T* vcon, const double* r64, Ctrl* ctrl,
                          cudaStream_t st) {
    k_ncp_prepare<<<1, 1024, 0, st>>>(c, x, ctrl);
    k_ncp_ainvb<T><<<(c.K * 32 + 255) / 256, 256, 0, st>>>(c, y, npad, x_base, ctrl);
    if (c.cached) {
        launch_ncp_cached_solve<T>(c, q0, iperm, vcon, npad, r64, ctrl, st);
        return;
    }
    // one cooperative grid of one CTA per SM (the barrier needs every CTA resident)
    const size_t smem = (size_t)(2 * kNcpTile * kNcpLd + kNcpTile) * sizeof(double);
    static bool attr_set[2] = {false, false};
    void (*kern)(ContactDev, const double*, const int*, T*, int, const double*, Ctrl*) = k_ncp_block_solve<T>;
    if (!attr_set[sizeof(T) == 8]) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set[sizeof(T) == 8] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ncp_grid());
    cfg.blockDim = dim3(kNcpThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, c, q0, iperm, vcon, npad, r64, ctrl);
}
template void launch_ncp_iteration<double>(const ContactDev&, const double*, const double*, int, const double*,
                                           const double*, const int*, double*, const double*, Ctrl*, cudaStream_t);
template void launch_ncp_iteration<float>(const ContactDev&, const double*, const float*, int, const double*,
                                          const double*, const int*, float*, const double*, Ctrl*, cudaStream_t);

namespace {
template <typename TI, typename TO>
__global__ void __launch_bounds__(256) k_path_apply(ContactDev c, const double* __restrict__ vsrc, int from_nodes,
                                                    const TI* yin, TO* yout, int npad, const Ctrl* ctrl) {
    if (ctrl->done) return;
    const int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (u >= c.nU) return;
    const int row = c.tp_row[u];
    const int64_t e0 = c.tp_ptr[u], e1 = c.tp_ptr[u + 1];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int64_t e = e0 + lane; e < e1; e += 32) {
        const int k = c.tp_k[e];
        const double v = c.tp_val[e];
        const double* src = vsrc + 3 * (size_t)(from_nodes ? c.cand[k] : k);
        s0 += v * src[0];
        s1 += v * src[1];
        s2 += v * src[2];
    }
    s0 = warp_sum_d(s0);
    s1 = warp_sum_d(s1);
    s2 = warp_sum_d(s2);
    if (lane == 0) {
        const double a0 = (double)yin[row], a1 = (double)yin[npad + row], a2 = (double)yin[2 * (size_t)npad + row];
        yout[row] = (TO)(a0 + s0);
        yout[npad + row] = (TO)(a1 + s1);
        yout[2 * (size_t)npad + row] = (TO)(a2 + s2);
    }
}

__global__ void k_cand_zero(ContactDev c, const int* __restrict__ iperm, float* __restrict__ v, int npad,
                            const Ctrl* ctrl) {
    if (ctrl->done) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.K) return;
    const int j = iperm[c.cand[k]];
    v[j] = 0.0f;
    v[npad + j] = 0.0f;
    v[2 * (size_t)npad + j] = 0.0f;
}

__global__ void k_path_gather_vals(long long E, const int64_t* __restrict__ src_e, const double* __restrict__ pval,
                                   double* __restrict__ tp_val) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < E) tp_val[i] = pval[src_e[i]];
}
}  // namespace

template <typename TI, typename TO>
void launch_path_apply(const ContactDev& c, const double* v_src, int from_nodes, const TI* y_in, TO* y_out, int npad,
                       const Ctrl* ctrl, cudaStream_t st) {
    if (c.nU <= 0) return;
    k_path_apply<TI, TO><<<(unsigned)(((long long)c.nU * 32 + 255) / 256), 256, 0, st>>>(c, v_src, from_nodes, y_in,
                                                                                        y_out, npad, ctrl);
}
template void launch_path_apply<double, double>(const ContactDev&, const double*, int, const double*, double*, int,
                                                const Ctrl*, cudaStream_t);
template void launch_path_apply<float, double>(const ContactDev&, const double*, int, const float*, double*, int,
                                               const Ctrl*, cudaStream_t);
template void launch_path_apply<float, float>(const ContactDev&, const double*, int, const float*, float*, int,
                                              const Ctrl*, cudaStream_t);

void launch_cand_zero(const ContactDev& c, const int* iperm, float* v, int npad, const Ctrl* ctrl, cudaStream_t st) {
    if (c.K > 0) k_cand_zero<<<(c.K + 255) / 256, 256, 0, st>>>(c, iperm, v, npad, ctrl);
}

void launch_path_gather_vals(long long E, const int64_t* src_e, const double* pval, double* tp_val, cudaStream_t st) {
    if (E > 0) k_path_gather_vals<<<(unsigned)((E + 255) / 256), 256, 0, st>>>(E, src_e, pval, tp_val);
}

void launch_restitution(const ContactDev& c, double* q, const double* q0, const double* v0, double h, double e,
                        double slop, cudaStream_t st) {
    if (c.K > 0) k_restitution<<<(c.K + 255) / 256, 256, 0, st>>>(c, q, q0, v0, h, e, slop);
}

}  // namespace dphd
