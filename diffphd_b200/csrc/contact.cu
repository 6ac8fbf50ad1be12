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

// Dense solve of the active NCP system, multiplier updates and the contact right-hand side (one CTA).
// vcon: without r64, J^T f (zero elsewhere); with r64 (the FP64 residual of the refinement form), the S-pass
// input itself, overwritten at the candidates with r + J^T f formed in FP64 (no FP32 cancellation of the two).
template <typename T>
__global__ void __launch_bounds__(1024) k_ncp_solve(ContactDev c, const double* __restrict__ q0,
                                                    const int* __restrict__ iperm, T* __restrict__ vcon, int npad,
                                                    const double* __restrict__ r64, Ctrl* ctrl) {
    if (ctrl->done) return;
    const int K = c.K, ka = c.kact[0];
    const int tid = threadIdx.x, nt = blockDim.x;
    const double n0 = c.n[0], n1 = c.n[1], n2 = c.n[2];
    // clear the previous contact right-hand side at every candidate node
    for (int k = tid; k < K; k += nt) {
        const int node = c.cand[k], j = iperm[node];
        vcon[j] = r64 ? (T)r64[3 * node] : T(0);
        vcon[npad + j] = r64 ? (T)r64[3 * node + 1] : T(0);
        vcon[2 * (size_t)npad + j] = r64 ? (T)r64[3 * node + 2] : T(0);
    }
    if (ka == 0) {
        for (int k = tid; k < K; k += nt) c.lt1[k] = c.lt2[k] = 0.0;
        return;
    }
    double* M = c.Mwork;      // ka x ka, row-major
    double* rhs = c.rhs;      // ka
    // A^-1 g at active nodes and the right-hand side h - J A^-1 g
    for (int a = tid; a < ka; a += nt) {
        const int k = c.act[a];
        double g0 = c.ainvb[3 * a], g1 = c.ainvb[3 * a + 1], g2 = c.ainvb[3 * a + 2];
        for (int b = 0; b < ka; ++b) {
            const int kb = c.act[b];
            const double Gab = c.G[(size_t)k * K + kb];
            const double fn = c.omega[kb] * c.lam[kb];
            const double f1 = c.lt1[kb], f2 = c.lt2[kb];
            g0 += Gab * (fn * n0 + f1 * c.t1[0] + f2 * c.t2[0]);
            g1 += Gab * (fn * n1 + f1 * c.t1[1] + f2 * c.t2[1]);
            g2 += Gab * (fn * n2 + f1 * c.t1[2] + f2 * c.t2[2]);
        }
        rhs[a] = c.hvec[k] - c.omega[k] * (n0 * g0 + n1 * g1 + n2 * g2);
        for (int b = 0; b < ka; ++b) {
            const int kb = c.act[b];
            M[(size_t)a * ka + b] = c.omega[k] * c.G[(size_t)k * K + kb] * c.omega[kb] + (a == b ? c.Ediag[k] : 0.0);
        }
    }
    __syncthreads();
    // Cholesky M = L L^T in place (lower triangle), right-looking
    for (int j = 0; j < ka; ++j) {
        __shared__ double piv;
        if (tid == 0) {
            double d = M[(size_t)j * ka + j];
            piv = sqrt(d > 1e-300 ? d : 1e-300);
            M[(size_t)j * ka + j] = piv;
        }
        __syncthreads();
        for (int i = j + 1 + tid; i < ka; i += nt) M[(size_t)i * ka + j] /= piv;
        __syncthreads();
        const int rem = ka - j - 1;
        for (long long t = tid; t < (long long)rem * rem; t += nt) {
            const int i = j + 1 + (int)(t / rem), l = j + 1 + (int)(t % rem);
            if (l <= i) M[(size_t)i * ka + l] -= M[(size_t)i * ka + j] * M[(size_t)l * ka + j];
        }
        __syncthreads();
    }
    // forward / backward substitution, column-oriented so that each step is parallel over the rows
    for (int k = 0; k < ka; ++k) {
        if (tid == 0) rhs[k] /= M[(size_t)k * ka + k];
        __syncthreads();
        const double rk = rhs[k];
        for (int i = k + 1 + tid; i < ka; i += nt) rhs[i] -= M[(size_t)i * ka + k] * rk;
        __syncthreads();
    }
    for (int i = ka - 1; i >= 0; --i) {
        if (tid == 0) rhs[i] /= M[(size_t)i * ka + i];
        __syncthreads();
        const double ri = rhs[i];
        for (int k = tid; k < i; k += nt) rhs[k] -= M[(size_t)i * ka + k] * ri;
        __syncthreads();
    }
    for (int a = tid; a < ka; a += nt) {
        const int k = c.act[a];
        double l = c.lam[k] + rhs[a];
        l = l < 0.0 ? 0.0 : (l > 1e8 ? 1e8 : l);
        c.lam[k] = l;
    }
    __syncthreads();
    // Coulomb cone (forward_gpu.cpp:1255-1302); non-active candidates have lambda = 0 and no friction
    for (int k = tid; k < K; k += nt) c.ltmp[k] = 0.0;
    __syncthreads();
    for (int a = tid; a < ka; a += nt) {
        const int k = c.act[a];
        double t1v = 0.0, t2v = 0.0;
        if (c.mu > 0.0 && c.lam[k] > 0.0) {
            const int node = c.cand[k];
            double qn0 = c.ainvb[3 * a], qn1 = c.ainvb[3 * a + 1], qn2 = c.ainvb[3 * a + 2];
            for (int b = 0; b < ka; ++b) {
                const int kb = c.act[b];
                const double f = c.omega[kb] * c.lam[kb] * c.G[(size_t)k * K + kb];
                qn0 += f * n0;
                qn1 += f * n1;
                qn2 += f * n2;
            }
            const double s0 = qn0 - q0[3 * node], s1 = qn1 - q0[3 * node + 1], s2 = qn2 - q0[3 * node + 2];
            const double sn = s0 * n0 + s1 * n1 + s2 * n2;
            const double u0 = s0 - sn * n0, u1 = s1 - sn * n1, u2 = s2 - sn * n2;
            const double ut1 = u0 * c.t1[0] + u1 * c.t1[1] + u2 * c.t1[2];
            const double ut2 = u0 * c.t2[0] + u1 * c.t2[1] + u2 * c.t2[2];
            const double Gkk = c.G[(size_t)k * K + k];
            const double det = Gkk * Gkk;
            double st1 = 0.0, st2 = 0.0;
            if (fabs(det) > 1e-20) {
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
        c.ltmp[k] = t1v;
        c.ltmp[K + k] = t2v;
    }
    __syncthreads();
    for (int k = tid; k < K; k += nt) {
        c.lt1[k] = c.ltmp[k];
        c.lt2[k] = c.ltmp[K + k];
    }
    __syncthreads();
    // contact right-hand side J^T f at the active nodes (omega from this iteration times the new lambda)
    for (int a = tid; a < ka; a += nt) {
        const int k = c.act[a];
        const double fn = c.omega[k] * c.lam[k];
        const int node = c.cand[k], j = iperm[node];
        const double r0 = r64 ? r64[3 * node] : 0.0, r1 = r64 ? r64[3 * node + 1] : 0.0,
                     r2 = r64 ? r64[3 * node + 2] : 0.0;
        vcon[j] = (T)(r0 + fn * n0 + c.lt1[k] * c.t1[0] + c.lt2[k] * c.t2[0]);
        vcon[npad + j] = (T)(r1 + fn * n1 + c.lt1[k] * c.t1[1] + c.lt2[k] * c.t2[1]);
        vcon[2 * (size_t)npad + j] = (T)(r2 + fn * n2 + c.lt1[k] * c.t1[2] + c.lt2[k] * c.t2[2]);
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
    k_ncp_solve<T><<<1, 1024, 0, st>>>(c, q0, iperm, vcon, npad, r64, ctrl);
}
template void launch_ncp_iteration<double>(const ContactDev&, const double*, const double*, int, const double*,
                                           const double*, const int*, double*, const double*, Ctrl*, cudaStream_t);
template void launch_ncp_iteration<float>(const ContactDev&, const double*, const float*, int, const double*,
                                          const double*, const int*, float*, const double*, Ctrl*, cudaStream_t);

void launch_restitution(const ContactDev& c, double* q, const double* q0, const double* v0, double h, double e,
                        double slop, cudaStream_t st) {
    if (c.K > 0) k_restitution<<<(c.K + 255) / 256, 256, 0, st>>>(c, q, q0, v0, h, e, slop);
}

}  // namespace dphd
