// Host side of the device construction of the sparse-inverse factor S = L~^-1 P (A = P^T L~ L~^T P, L~ the
// Cholesky factor; the reference builds S = D^-1/2 L^-1 P from an LDL^T, which is the same matrix:
// RealSim/src/Scomponent/tools/math/SparseLDLT.cpp:226-347, deformable_projective_dynamics_forward_gpu.cpp:593-764).
//
// The etree postorder makes row i of S dense on [lo_i, i].  The rows split into two kinds:
//  * small subtrees (at most `small_max` nodes under a root whose parent's subtree is larger) are built on the
//    host by the up-looking LDL^T and the row recurrence of build_sfactor, restricted to the subtree (each
//    subtree is independent, so they run in parallel; the values are bit-identical to build_sfactor's);
//  * every other row belongs to a "big" supernode: a chain s = [a, b) of the etree (each node the only child of
//    the next), whose rows all start at lo_s = lo_a and whose descendants are D = [lo_s, a).  Its rows follow from
//    the descendants' rows (Schur complement of A on s given D, with A_DD^-1 = S_DD^T S_DD):
//        W   = A[s, D] S_DD^T                     (|s| x |B_s|: only the columns B_s of rows k in D that are
//                                                   ancestors-or-self of a D-neighbour of s are non-zero)
//        C   = A[s, s] - W W^T = L~_ss L~_ss^T
//        [V | T] = L~_ss^-1 [W | I]
//        S[s, D] = -V S[B_s, D],   S[s, s] = T.
//    The device does these per supernode in postorder (descendants first).  This file builds the index plan.
#include <algorithm>
#include <cmath>
#include <functional>
#include <numeric>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "dphd_internal.h"

namespace dphd {

SBuildPlan plan_sfactor_build(const SFactor& S, const PermUpper& U, int small_max) {
    const int n = S.n;
    SBuildPlan P;
    P.small_max = small_max;
    std::vector<int> nchild(n, 0);
    for (int j = 0; j < n; ++j)
        if (S.parent[j] >= 0) nchild[S.parent[j]]++;
    auto size_of = [&](int j) { return j - S.lo[j] + 1; };
    // small subtree roots, ascending (subtrees are disjoint index ranges [lo_r, r])
    std::vector<uint8_t> small(n, 0);
    for (int j = 0; j < n; ++j) {
        if (size_of(j) > small_max) continue;
        const int p = S.parent[j];
        if (p < 0 || size_of(p) > small_max) P.small_roots.push_back(j);
    }
    for (int r : P.small_roots)
        for (int j = S.lo[r]; j <= r; ++j) small[j] = 1;
    // big supernodes: maximal chains of big nodes
    for (int j = 0; j < n;) {
        if (small[j]) {
            ++j;
            continue;
        }
        int e = j + 1;
        while (e < n && !small[e] && S.parent[e - 1] == e && nchild[e] == 1) ++e;
        SBigSuper s;
        s.a = j;
        s.b = e;
        s.lo = S.lo[j];
        s.ra = s.lo & ~3;
        P.sup.push_back(s);
        j = e;
    }
    // full symmetric permuted A by rows (the entries of the rows of big supernodes are what the device reads)
    {
        std::vector<int64_t> cnt(n + 1, 0);
        for (int c = 0; c < n; ++c)
            for (int q = U.Cp[c]; q < U.Cp[c + 1]; ++q) {
                const int r = U.Ci[q];
                cnt[r + 1]++;
                if (r != c) cnt[c + 1]++;
            }
        for (int i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
        P.a_rp.assign(cnt.begin(), cnt.end());
        P.a_ci.assign(cnt[n], 0);
        P.a_v.assign(cnt[n], 0.0);
        std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
        for (int c = 0; c < n; ++c)
            for (int q = U.Cp[c]; q < U.Cp[c + 1]; ++q) {
                const int r = U.Ci[q];
                P.a_ci[pos[r]] = c;
                P.a_v[pos[r]++] = U.Cx[q];
                if (r != c) {
                    P.a_ci[pos[c]] = r;
                    P.a_v[pos[c]++] = U.Cx[q];
                }
            }
    }
    // B_s and the per-column-tile lists of the S[s, D] product
    std::vector<int> mark(n, -1);
    std::vector<int> tcount;
    P.ct_ptr.push_back(0);
    for (size_t si = 0; si < P.sup.size(); ++si) {
        SBigSuper& s = P.sup[si];
        std::vector<int> B;
        for (int j = s.a; j < s.b; ++j)
            for (int64_t q = P.a_rp[j]; q < P.a_rp[j + 1]; ++q) {
                int k = P.a_ci[q];
                if (k >= s.a) continue;  // in s or above: not a descendant
                while (k < s.a && mark[k] != (int)si) {
                    mark[k] = (int)si;
                    B.push_back(k);
                    k = S.parent[k];
                }
            }
        std::sort(B.begin(), B.end());
        s.B_off = (int64_t)P.B.size();
        s.nB = (int)B.size();
        P.B.insert(P.B.end(), B.begin(), B.end());
        s.nct = (s.a - s.ra + kSbTile - 1) / kSbTile;
        s.ct_off = (int64_t)P.ct_ptr.size() - 1;
        tcount.assign(s.nct + 1, 0);
        for (int k : B) {
            const int t0 = (S.lo[k] - s.ra) / kSbTile, t1 = (k - s.ra) / kSbTile;
            for (int t = t0; t <= t1; ++t) tcount[t + 1]++;
        }
        for (int t = 0; t < s.nct; ++t) tcount[t + 1] += tcount[t];
        const int64_t base = (int64_t)P.ct_p.size();
        P.ct_p.resize(base + tcount[s.nct]);
        std::vector<int> tpos(tcount.begin(), tcount.end() - 1);
        for (int p = 0; p < s.nB; ++p) {
            const int k = B[p];
            const int t0 = (S.lo[k] - s.ra) / kSbTile, t1 = (k - s.ra) / kSbTile;
            for (int t = t0; t <= t1; ++t) P.ct_p[base + tpos[t]++] = p;
        }
        for (int t = 0; t < s.nct; ++t) P.ct_ptr.push_back(base + tcount[t + 1]);
        P.max_w = std::max(P.max_w, s.b - s.a);
        P.max_nB = std::max(P.max_nB, s.nB);
        P.max_x = std::max<int64_t>(P.max_x, (int64_t)((s.b - s.a + kSbTile - 1) / kSbTile * kSbTile) *
                                                  (int64_t)(s.nB + (s.b - s.a)));
    }
    return P;
}

// Rows of the small subtrees, computed as build_sfactor does (up-looking LDL^T of the subtree, then the row
// recurrence row_i(L^-1) = e_i - sum_k l_ik row_k(L^-1), scaled by D^-1/2), written through row_ptr(i), which
// returns where column lo_i of row i goes.  Subtrees run in parallel; each one serially, so the values do not
// depend on the thread count.
void sfactor_small_rows(const SFactor& S, const PermUpper& U, const std::vector<int>& roots, int threads,
                        const std::function<double*(int)>& row_ptr) {
    const int nr = (int)roots.size();
    const int nthr = threads > 0 ? threads : 0;
    int bad_root = -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthr > 0 ? nthr : omp_get_max_threads())
    for (int ri = 0; ri < nr; ++ri) {
        const int root = roots[ri], lo = S.lo[root], m = root - lo + 1;
        // local indices: node lo + t
        std::vector<int> lnz(m, 0), flag(m, -1), pattern(m);
        for (int k = 0; k < m; ++k) {
            flag[k] = k;
            const int kg = lo + k;
            for (int q = U.Cp[kg]; q < U.Cp[kg + 1]; ++q)
                for (int i = U.Ci[q] - lo; i < k && flag[i] != k; i = S.parent[lo + i] - lo) {
                    lnz[i]++;
                    flag[i] = k;
                }
        }
        std::vector<int64_t> Lp(m + 1, 0);
        for (int k = 0; k < m; ++k) Lp[k + 1] = Lp[k] + lnz[k];
        std::vector<int> Li(Lp[m]);
        std::vector<double> Lx(Lp[m]), D(m), Y(m, 0.0);
        std::vector<int64_t> Rp(m + 1, 0);
        std::vector<int> Rj;
        std::vector<double> Rx;
        Rj.reserve(Lp[m]);
        Rx.reserve(Lp[m]);
        std::fill(lnz.begin(), lnz.end(), 0);
        std::fill(flag.begin(), flag.end(), -1);
        bool ok = true;
        for (int k = 0; k < m; ++k) {
            int top = m;
            flag[k] = k;
            const int kg = lo + k;
            for (int q = U.Cp[kg]; q < U.Cp[kg + 1]; ++q) {
                int i = U.Ci[q] - lo;
                Y[i] += U.Cx[q];
                int len = 0;
                for (; flag[i] != k; i = S.parent[lo + i] - lo) {
                    pattern[len++] = i;
                    flag[i] = k;
                }
                while (len > 0) pattern[--top] = pattern[--len];
            }
            double dk = Y[k];
            Y[k] = 0;
            for (; top < m; ++top) {
                const int i = pattern[top];
                const double yi = Y[i];
                Y[i] = 0;
                const int64_t p2 = Lp[i] + lnz[i];
                for (int64_t p = Lp[i]; p < p2; ++p) Y[Li[p]] -= Lx[p] * yi;
                const double lki = yi / D[i];
                dk -= lki * yi;
                Li[p2] = k;
                Lx[p2] = lki;
                lnz[i]++;
                Rj.push_back(i);
                Rx.push_back(lki);
            }
            Rp[k + 1] = (int64_t)Rj.size();
            if (!(dk > 0 && std::isfinite(dk))) ok = false;
            D[k] = dk > 0 ? dk : 1.0;
        }
        if (!ok) {  // reported after the loop (no throw inside the parallel region)
#pragma omp critical(dphd_small_rows)
            bad_root = std::max(bad_root, root);
            continue;
        }
        for (int i = 0; i < m; ++i) {
            const int ig = lo + i, li = S.lo[ig] - lo;
            double* out = row_ptr(ig) - li;  // out[c] for local columns c in [li, i]
            for (int c = li; c <= i; ++c) out[c] = (c == i) ? 1.0 : 0.0;
            for (int64_t p = Rp[i]; p < Rp[i + 1]; ++p) {
                const int k = Rj[p];
                const double l = Rx[p];
                const int lk = S.lo[lo + k] - lo;
                const double* rk = row_ptr(lo + k) - lk;
                for (int c = lk; c <= k; ++c) out[c] -= l * rk[c];
            }
        }
        for (int i = 0; i < m; ++i) {
            const int ig = lo + i;
            double* r = row_ptr(ig);
            const double sc = 1.0 / std::sqrt(D[i]);
            for (int c = 0; c < ig - S.lo[ig] + 1; ++c) r[c] *= sc;
        }
    }
    DPHD_CHECK(bad_root < 0, "PD matrix is not positive definite (LDL^T pivot in the subtree of row " +
                                 std::to_string(bad_root) + ")");
}

}  // namespace dphd
