// The NCP's dense solve M dlambda = rhs (M = Omega G Omega + E over the ka active candidates) with a cached
// factor: the reference factors M at every PD iteration (forward_gpu.cpp:1238-1240).  Here one cooperative
// launch per PD iteration
//   A  assembles M (full rows, identity-padded to a multiple of 64) and the right-hand side, and counts the active
//      candidates that are not in the list act_ref the cached factor was built for;
//   B  when a cached factor X = L_ref^-1 of an earlier M_ref of this frame exists and the two lists differ in at
//      most kNcpMaxListChange candidates: conjugate gradients on M to |r| <= tol |rhs| (option ncp_cg_tol, 1e-13
//      by default: looser steps leave multipliers just above 0 and change the active list more often),
//      preconditioned by D^-1 X^T X D^-1 on the candidates in both lists (D = Omega Omega_ref^-1, see phase B)
//      and diag(M)^-1 on the others.  X^T X restricted to a subset of its list is the inverse of a Schur
//      complement of M_ref, so P M differs from I by the change of E between the PD iterations plus a term of
//      rank <= (dropped + 2 x new candidates); near the fixed point a few iterations suffice.  X is applied from
//      FP32 copies (the preconditioner only has to be symmetric positive definite; the residual and the iterate
//      are FP64);
//   C  otherwise (no factor, a large change of the list, or CG not converged): the blocked Cholesky of M with the
//      triangular solve of the identity folded in (X = L^-1, only the lower blocks, kept as the new cached factor),
//      then dlambda = X^T (X rhs);
//   D  clamp, Coulomb cone and the contact right-hand side, as k_ncp_block_solve.
// Both paths solve the same system (to the CG tolerance), so the iterates match the refactor-every-iteration
// solve (option ncp_solver = 0) to that level.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace dphd {

namespace {

constexpr int kT = 64;
constexpr int kLd = kT + 1;
constexpr int kThr = 256;
constexpr int kNcpPcgIters = 40;       // CG iteration cap for an unchanged list; + 2 per changed candidate
constexpr int kNcpMaxListChange = 32;  // larger changes of the active list refactor at once
constexpr double kOmegaMin = 1e-6;     // |omega| below this: the candidate's row is decoupled (E only)
constexpr double kEDrift = 0.1;        // |E - (omega / omega_ref)^2 E_ref| above this fraction of M_kk: diagonal
constexpr long long kSpins = 1ll << 24;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ bool gsync(unsigned int* bar, Ctrl* ctrl) {
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
                    if (vbar[2] != 0u || ++spins > kSpins) {
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

// Sum of one value per CTA (part[0 .. G)), the same in every CTA: each CTA sums the partials in block order.
__device__ double grid_total(const double* part) {
    __shared__ double sh[32];
    __shared__ double tot;
    double v = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += __ldcg(part + b);
    v = wsum(v);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
        tot = s;
    }
    __syncthreads();
    return tot;
}

// CTA partial of a value that each warp accumulated in `v` (lane 0 holds the warp's share): written to part[bid].
__device__ void cta_partial(double v, double* part) {
    __shared__ double sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
        part[blockIdx.x] = s;
    }
    __syncthreads();
}

// 64x64 Cholesky of sD (row-major, ld kLd) in place; the reference's pivot guard.
__device__ void tile_chol(double* sD) {
    __shared__ double piv;
    for (int j = 0; j < kT; ++j) {
        if (threadIdx.x == 0) {
            const double d = sD[j * kLd + j];
            piv = sqrt(d > 1e-300 ? d : 1e-300);
            sD[j * kLd + j] = piv;
        }
        __syncthreads();
        const double inv = 1.0 / piv;
        for (int r = j + 1 + (int)threadIdx.x; r < kT; r += blockDim.x) sD[r * kLd + j] *= inv;
        __syncthreads();
        const int rem = kT - j - 1;
        for (int t = threadIdx.x; t < rem * rem; t += blockDim.x) {
            const int r = j + 1 + t / rem, l = j + 1 + t % rem;
            if (l <= r) sD[r * kLd + l] -= sD[r * kLd + j] * sD[l * kLd + j];
        }
        __syncthreads();
    }
}

// acc -= A B^T for 64x64 tiles given k-major in shared memory.
__device__ __forceinline__ void tile_fma(const double* sA, const double* sB, double (&acc)[4][4]) {
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll 4
    for (int k = 0; k < kT; ++k) {
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

template <typename T>
__global__ void __launch_bounds__(kThr, 1)
k_ncp_cached_solve(ContactDev c, const double* __restrict__ q0, const int* __restrict__ iperm, T* __restrict__ vcon,
                   int npad, const double* __restrict__ r64, Ctrl* ctrl) {
    extern __shared__ double smem[];
    double* sD = smem;
    double* sA = smem + kT * kLd;
    double* sB = smem + 2 * kT * kLd;
    if (ctrl->done) return;
    const int K = c.K, ka = c.kact[0];
    const int tid = threadIdx.x, nt = blockDim.x, G = gridDim.x, bid = blockIdx.x;
    const int gt = bid * nt + tid, nthr = G * nt;
    const int lane = tid & 31, gw = gt >> 5, nwarps = nthr >> 5;
    const double n0 = c.n[0], n1 = c.n[1], n2 = c.n[2];
    const int ldx = (int)c.kcap;
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
    const int nb = (ka + kT - 1) / kT, ld = nb * kT;
    double* M = c.Mwork;
    double* rhs = c.rhs;
    double* x = c.xsol;
    double* dg = c.pcg + 5 * (size_t)ldx;    // diag(M)
    double* part = c.pcg + 9 * (size_t)ldx;  // per-CTA partial sums (omega_ref and E_ref, kept with the factor,
                                             // at 7 ldx and 8 ldx)
    // [0] cached factor valid, [1] its ka, [2] candidates not in its list (this launch), [3] the last CG fell back
    int* flags = c.ncp_flags;
    const bool have = flags[0] != 0;
    const int ka_ref = have ? flags[1] : 0;
    const int ld_ref = (ka_ref + kT - 1) / kT * kT;
    // ---- A: M (full rows), diag(M), rhs, and the active candidates that are new to the cached factor's list ----
    for (int a = gt; a < ka_ref; a += nthr) c.ref_inv[a] = -1;
    int n_new_w = 0;
    for (int a = gw; a < ld; a += nwarps) {
        double* Ma = M + (size_t)a * ld;
        if (a >= ka) {
            for (int b = lane; b < ld; b += 32) Ma[b] = (a == b) ? 1.0 : 0.0;
            if (lane == 0) {
                rhs[a] = 0.0;
                dg[a] = 1.0;
            }
            continue;
        }
        const int k = c.act[a];
        if (have && lane == 0 && c.ref_pos[k] < 0) ++n_new_w;
        const double om = c.omega[k];
        const double* Gk = c.G + (size_t)k * K;
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
        for (int b = lane; b < ld; b += 32) {
            if (b >= ka) {
                Ma[b] = 0.0;
                continue;
            }
            const int kb = c.act[b];
            const double Gab = Gk[kb];
            const double fn = c.omega[kb] * c.lam[kb];
            const double f1 = c.lt1[kb], f2 = c.lt2[kb];
            g0 += Gab * (fn * n0 + f1 * c.t1[0] + f2 * c.t2[0]);
            g1 += Gab * (fn * n1 + f1 * c.t1[1] + f2 * c.t2[1]);
            g2 += Gab * (fn * n2 + f1 * c.t1[2] + f2 * c.t2[2]);
            const double m = om * Gab * c.omega[kb] + (a == b ? c.Ediag[k] : 0.0);
            Ma[b] = m;
            if (a == b) dg[a] = m;
        }
        g0 = wsum(g0);
        g1 = wsum(g1);
        g2 = wsum(g2);
        if (lane == 0) {
            g0 += c.ainvb[3 * a];
            g1 += c.ainvb[3 * a + 1];
            g2 += c.ainvb[3 * a + 2];
            rhs[a] = c.hvec[k] - om * (n0 * g0 + n1 * g1 + n2 * g2);
        }
    }
    if (n_new_w) atomicAdd(flags + 2, n_new_w);
    if (!gsync(c.bar, ctrl)) return;
    // candidates whose positions changed: new to the list, or dropped from it
    const int n_new = have ? __ldcg(flags + 2) : 0;
    const int n_chg = n_new + (ka_ref - (ka - n_new));
    bool solved = false;
    if (have && n_chg <= kNcpMaxListChange) {
        // ---- B: CG on M, preconditioned by the cached factor on the common candidates, diag(M) on the others ----
        // M = Omega G Omega + E and M_ref = Omega_r G Omega_r + E_r, so with D = Omega Omega_r^-1 (diagonal)
        // M = D M_ref D + (E - D^2 E_r): the preconditioner D^-1 X^T X D^-1 follows the change of Omega between PD
        // iterations exactly and leaves only the diagonal change of E (small for resting contacts) to CG.
        // Candidates with omega or omega_ref near 0 (decoupled rows E only), or whose E moved away from D^2 E_r by
        // more than kEDrift of their diagonal (a contact opening or closing), take the diagonal preconditioner.
        double* r = c.pcg;
        double* p = c.pcg + ldx;
        double* w = c.pcg + 2 * (size_t)ldx;
        double* t = c.pcg + 3 * (size_t)ldx;
        double* zr = c.pcg + 4 * (size_t)ldx;  // X^T X (D^-1 r) over the cached list
        double* sc = c.pcg + 6 * (size_t)ldx;  // omega_ref / omega at a scaled common candidate, else 0
        const double* om_ref = c.pcg + 7 * (size_t)ldx;
        const double* e_ref = c.pcg + 8 * (size_t)ldx;
        for (int a = gt; a < ld; a += nthr) {
            double f = 0.0;
            if (a < ka) {
                const int k = c.act[a];
                const int pr = c.ref_pos[k];
                const double om = c.omega[k];
                if (pr >= 0 && fabs(om) >= kOmegaMin && fabs(om_ref[pr]) >= kOmegaMin) {
                    const double g = om / om_ref[pr];
                    if (fabs(c.Ediag[k] - g * g * e_ref[pr]) <= kEDrift * dg[a]) {
                        f = 1.0 / g;
                        c.ref_inv[pr] = a;
                    }
                }
            }
            sc[a] = f;
        }
        if (!gsync(c.bar, ctrl)) return;
        // r = rhs, x = 0, |rhs|^2
        double acc = 0.0;
        for (int a = gt; a < ld; a += nthr) {
            const double v = a < ka ? rhs[a] : 0.0;
            r[a] = v;
            x[a] = 0.0;
            acc += v * v;
        }
        cta_partial(wsum(acc), part);
        if (!gsync(c.bar, ctrl)) return;
        const double rhs2 = grid_total(part);
        if (!gsync(c.bar, ctrl)) return;
        double rz = 0.0;
        int it = 0;
        bool conv = rhs2 == 0.0;
        // after an attempt that fell back, the next one gets a quarter of the cap (a system far from the cached one)
        const int cap = (__ldcg(flags + 3) != 0 ? kNcpPcgIters / 4 : kNcpPcgIters) + 2 * n_chg;
        while (!conv && it < cap) {
            // t = X (D^-1 r)_ref over the cached list (one warp per row; 0 at dropped or unscaled candidates)
            for (int a = gw; a < ld_ref; a += nwarps) {
                const float* Xa = c.X32 + (size_t)a * ldx;
                double s = 0.0;
                for (int b = lane; b <= a && b < ka_ref; b += 32) {
                    const int nb_ = __ldcg(c.ref_inv + b);
                    if (nb_ >= 0) s += (double)Xa[b] * (__ldcg(r + nb_) * __ldcg(sc + nb_));
                }
                s = wsum(s);
                if (lane == 0) t[a] = s;
            }
            if (!gsync(c.bar, ctrl)) return;
            // zr = X^T t (one warp per row of the stored transpose)
            for (int b = gw; b < ld_ref; b += nwarps) {
                const float* Xb = c.Xt32 + (size_t)b * ldx;
                double s = 0.0;
                for (int a = b + lane; a < ld_ref; a += 32) s += (double)Xb[a] * __ldcg(t + a);
                s = wsum(s);
                if (lane == 0) zr[b] = s;
            }
            if (!gsync(c.bar, ctrl)) return;
            // z on the current list (kept in w): D^-1 zr at the scaled candidates, r / M_aa elsewhere; rz = r . z
            acc = 0.0;
            for (int a = gt; a < ld; a += nthr) {
                const double ra = __ldcg(r + a);
                double z = ra;
                if (a < ka) {
                    const double f = __ldcg(sc + a);
                    z = f != 0.0 ? __ldcg(zr + c.ref_pos[c.act[a]]) * f : (dg[a] > 0.0 ? ra / dg[a] : ra);
                }
                w[a] = z;
                acc += ra * z;
            }
            cta_partial(wsum(acc), part);
            if (!gsync(c.bar, ctrl)) return;
            const double rz_new = grid_total(part);
            const double beta = it == 0 ? 0.0 : rz_new / rz;
            rz = rz_new;
            for (int a = gt; a < ld; a += nthr) p[a] = __ldcg(w + a) + beta * (it == 0 ? 0.0 : __ldcg(p + a));
            if (!gsync(c.bar, ctrl)) return;
            // w = M p (one warp per row), p . w
            acc = 0.0;
            for (int a = gw; a < ld; a += nwarps) {
                const double* Ma = M + (size_t)a * ld;
                double s = 0.0;
                for (int b = lane; b < ld; b += 32) s += Ma[b] * __ldcg(p + b);
                s = wsum(s);
                if (lane == 0) {
                    w[a] = s;
                    acc += s * __ldcg(p + a);
                }
            }
            cta_partial(wsum(acc), part);
            if (!gsync(c.bar, ctrl)) return;
            const double pw = grid_total(part);
            const double alpha = pw > 0.0 ? rz / pw : 0.0;
            acc = 0.0;
            for (int a = gt; a < ld; a += nthr) {
                x[a] += alpha * __ldcg(p + a);
                const double rv = __ldcg(r + a) - alpha * __ldcg(w + a);
                r[a] = rv;
                acc += rv * rv;
            }
            cta_partial(wsum(acc), part);
            if (!gsync(c.bar, ctrl)) return;
            const double rr = grid_total(part);
            ++it;
            conv = pw > 0.0 && rr <= c.cg_tol * c.cg_tol * rhs2;
            if (!gsync(c.bar, ctrl)) return;
        }
        solved = conv;
        if (gt == 0) {
            c.ncp_stats[2] += it;         // CG iterations
            if (!conv) c.ncp_stats[3] += 1;  // CG attempts that fall back to a factorisation
            flags[3] = conv ? 0 : 1;
        }
    }
    if (!solved) {
        // ---- C: blocked Cholesky of M with X = L^-1 (identity solved in place), then x = X^T X rhs ----
        double* X = c.Xinv;
        for (int k = gt; k < K; k += nthr) c.ref_pos[k] = -1;  // read no more in this launch (after its CG)
        for (size_t e = (size_t)gt; e < (size_t)ld * ld; e += (size_t)nthr) {
            const int a = (int)(e / ld), b = (int)(e % ld);
            X[(size_t)a * ldx + b] = a == b ? 1.0 : 0.0;
        }
        if (!gsync(c.bar, ctrl)) return;
        for (int kb = 0; kb < nb; ++kb) {
            const int below = nb - kb - 1;
            // every CTA with a panel tile or an X chunk of this block row factors the diagonal block
            const int n_items = below + (kb + 1);  // panels, then X_kb chunks of block columns 0..kb
            if (bid < n_items) {
                const double* Dg = M + (size_t)kb * kT * ld + kb * kT;
                for (int e = tid; e < kT * kT; e += nt) {
                    const int rr = e / kT, ll = e % kT;
                    if (ll <= rr) sD[rr * kLd + ll] = Dg[(size_t)rr * ld + ll];
                }
                __syncthreads();
                tile_chol(sD);
            }
            for (int item = bid; item < n_items; item += G) {
                __syncthreads();
                if (item < below) {  // panel L[i, kb] = M[i, kb] L_kk^-T
                    double* Pg = M + (size_t)(kb + 1 + item) * kT * ld + kb * kT;
                    for (int e = tid; e < kT * kT; e += nt) sA[(e / kT) * kLd + e % kT] = Pg[(size_t)(e / kT) * ld + e % kT];
                    __syncthreads();
                    if (tid < kT) {
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
                    for (int e = tid; e < kT * kT; e += nt) Pg[(size_t)(e / kT) * ld + e % kT] = sA[(e / kT) * kLd + e % kT];
                } else {  // X_kb[:, block column cc] <- L_kk^-1 X_kb[:, cc] (cc <= kb; blocks right of kb stay 0)
                    const int cc = item - below;
                    double* Xg = X + (size_t)kb * kT * ldx + cc * kT;
                    for (int e = tid; e < kT * kT; e += nt) sA[(e / kT) * kLd + e % kT] = Xg[(size_t)(e / kT) * ldx + e % kT];
                    __syncthreads();
                    if (tid < kT) {
                        for (int rr = 0; rr < kT; ++rr) {
                            const double* Lr = sD + rr * kLd;
                            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                            int l = 0;
                            for (; l + 4 <= rr; l += 4) {
                                s0 += Lr[l] * sA[l * kLd + tid];
                                s1 += Lr[l + 1] * sA[(l + 1) * kLd + tid];
                                s2 += Lr[l + 2] * sA[(l + 2) * kLd + tid];
                                s3 += Lr[l + 3] * sA[(l + 3) * kLd + tid];
                            }
                            for (; l < rr; ++l) s0 += Lr[l] * sA[l * kLd + tid];
                            sA[rr * kLd + tid] = (sA[rr * kLd + tid] - ((s0 + s1) + (s2 + s3))) / Lr[rr];
                        }
                    }
                    __syncthreads();
                    for (int e = tid; e < kT * kT; e += nt) Xg[(size_t)(e / kT) * ldx + e % kT] = sA[(e / kT) * kLd + e % kT];
                }
            }
            if (!gsync(c.bar, ctrl)) return;
            if (bid == 0) {  // every CTA has read M[kb][kb]: store L_kk (the trailing updates read only panels)
                double* Dw = M + (size_t)kb * kT * ld + kb * kT;
                for (int e = tid; e < kT * kT; e += nt) {
                    const int rr = e / kT, ll = e % kT;
                    if (ll <= rr) Dw[(size_t)rr * ld + ll] = sD[rr * kLd + ll];
                }
            }
            // trailing updates: M[i][j] -= L[i,kb] L[j,kb]^T (kb < j <= i); X[i][cc] -= L[i,kb] X[kb][cc] (cc <= kb)
            const int ntri = below * (below + 1) / 2, nx = below * (kb + 1);
            const int ty = tid >> 4, tx = tid & 15;
            for (int item = bid; item < ntri + nx; item += G) {
                __syncthreads();
                int i, j = -1, cc = 0;
                if (item < ntri) {
                    int ii = (int)((sqrt(8.0 * (double)item + 1.0) - 1.0) * 0.5);
                    while ((ii + 1) * (ii + 2) / 2 <= item) ++ii;
                    while (ii * (ii + 1) / 2 > item) --ii;
                    i = kb + 1 + ii;
                    j = kb + 1 + (item - ii * (ii + 1) / 2);
                } else {
                    const int q = item - ntri;
                    i = kb + 1 + q / (kb + 1);
                    cc = q % (kb + 1);
                }
                const double* Pi = M + (size_t)i * kT * ld + kb * kT;
                for (int e = tid; e < kT * kT; e += nt) {
                    const int rr = e / kT, k = e % kT;
                    sA[k * kLd + rr] = Pi[(size_t)rr * ld + k];
                }
                if (j >= 0) {
                    const double* Pj = M + (size_t)j * kT * ld + kb * kT;
                    for (int e = tid; e < kT * kT; e += nt) {
                        const int rr = e / kT, k = e % kT;
                        sB[k * kLd + rr] = Pj[(size_t)rr * ld + k];
                    }
                } else {
                    const double* Yg = X + (size_t)kb * kT * ldx + cc * kT;
                    for (int e = tid; e < kT * kT; e += nt) {
                        const int k = e / kT, cl = e % kT;
                        sB[k * kLd + cl] = Yg[(size_t)k * ldx + cl];
                    }
                }
                __syncthreads();
                double acc4[4][4] = {};
                tile_fma(sA, sB, acc4);
                if (j >= 0) {
                    double* Cg = M + (size_t)i * kT * ld + j * kT;
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) Cg[(size_t)(ty * 4 + u) * ld + tx * 4 + v] -= acc4[u][v];
                } else {
                    double* Xi = X + (size_t)i * kT * ldx + cc * kT;
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) Xi[(size_t)(ty * 4 + u) * ldx + tx * 4 + v] -= acc4[u][v];
                }
            }
            if (!gsync(c.bar, ctrl)) return;
        }
        // the transpose of X (its lower triangle), for row-wise X^T products; then x = X^T (X rhs)
        for (size_t e = (size_t)gt; e < (size_t)ld * ld; e += (size_t)nthr) {
            const int a = (int)(e / ld), b = (int)(e % ld);
            if (b <= a) {
                const double v = X[(size_t)a * ldx + b];
                c.Xt[(size_t)b * ldx + a] = v;
                c.X32[(size_t)a * ldx + b] = (float)v;
                c.Xt32[(size_t)b * ldx + a] = (float)v;
            }
        }
        double* t = c.pcg + 3 * (size_t)ldx;
        for (int a = gw; a < ld; a += nwarps) {
            const double* Xa = X + (size_t)a * ldx;
            double s = 0.0;
            for (int b = lane; b <= a; b += 32) s += Xa[b] * rhs[b];
            s = wsum(s);
            if (lane == 0) t[a] = s;
        }
        if (!gsync(c.bar, ctrl)) return;
        for (int b = gw; b < ld; b += nwarps) {
            const double* Xb = c.Xt + (size_t)b * ldx;
            double s = 0.0;
            for (int a = b + lane; a < ld; a += 32) s += Xb[a] * __ldcg(t + a);
            s = wsum(s);
            if (lane == 0) x[b] = s;
        }
        // the new cached factor: its active list, the candidates' positions in it and their omega
        for (int a = gt; a < ka; a += nthr) {
            c.act_ref[a] = c.act[a];
            c.ref_pos[c.act[a]] = a;
            c.pcg[7 * (size_t)ldx + a] = c.omega[c.act[a]];
            c.pcg[8 * (size_t)ldx + a] = c.Ediag[c.act[a]];
        }
        if (gt == 0) {
            flags[0] = 1;
            flags[1] = ka;
            c.ncp_stats[1] += 1;  // refactorisations
        }
    } else if (gt == 0) {
        c.ncp_stats[0] += 1;  // solves by the cached factor
    }
    if (!gsync(c.bar, ctrl)) return;
    if (gt == 0) flags[2] = 0;  // re-armed for the next launch
    // ---- D: multipliers, Coulomb cone, contact right-hand side ----
    for (int a = gt; a < ka; a += nthr) {
        const int k = c.act[a];
        double l = c.lam[k] + x[a];
        l = l < 0.0 ? 0.0 : (l > 1e8 ? 1e8 : l);
        c.lam[k] = l;
    }
    for (int k = gt; k < K; k += nthr) c.lt1[k] = c.lt2[k] = 0.0;
    if (!gsync(c.bar, ctrl)) return;
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
            f = wsum(f);
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

}  // namespace

template <typename T>
void launch_ncp_cached_solve(const ContactDev& c, const double* q0, const int* iperm, T* vcon, int npad,
                             const double* r64, Ctrl* ctrl, cudaStream_t st) {
    const size_t smem = (size_t)(3 * kT * kLd) * sizeof(double);
    static bool attr_set[2] = {false, false};
    void (*kern)(ContactDev, const double*, const int*, T*, int, const double*, Ctrl*) = k_ncp_cached_solve<T>;
    if (!attr_set[sizeof(T) == 8]) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set[sizeof(T) == 8] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ncp_grid());
    cfg.blockDim = dim3(kThr);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, c, q0, iperm, vcon, npad, r64, ctrl);
}
template void launch_ncp_cached_solve<double>(const ContactDev&, const double*, const int*, double*, int,
                                              const double*, Ctrl*, cudaStream_t);
template void launch_ncp_cached_solve<float>(const ContactDev&, const double*, const int*, float*, int,
                                             const double*, Ctrl*, cudaStream_t);

}  // namespace dphd
