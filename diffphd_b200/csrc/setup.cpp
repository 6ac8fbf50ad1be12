// Host-side set-up of the B200 projective-dynamics step: finite-element samples, the node-level PD matrix
// A, a nested-dissection ordering, and the sparse-inverse factor S = D^-1/2 L^-1 P with A^-1 = S^T S.
//
// Reference behaviour followed:
//   * FE samples: hex  cpp/core/src/fem/hex_deformable.cpp:3-51 (8 Gauss points, trilinear gradients),
//                 tet  cpp/core/src/fem/tet_deformable.cpp:3-42 (one constant-gradient sample).
//   * A = diag(m/h^2, 1 on Dirichlet) + sum_e w_e (vol/s) sum_s A_s^T A_s, Dirichlet rows/cols skipped
//     (cpp/core/src/fem/deformable_projective_dynamics_forward.cpp:9-96).  Because A_s^T A_s couples only
//     equal axes, one node-level matrix serves x, y and z whenever Dirichlet constraints fix whole nodes.
//   * S factor: the reference builds S = sqrt(D^-1) L^-1 from a METIS ordering and an up-looking LDL^T
//     (RealSim/src/Scomponent/tools/math/SparseLDLT.cpp:111-347; forward_gpu.cpp:593-635).  Here the
//     ordering is nested dissection by recursive coordinate bisection followed by an etree postorder, so
//     every row of L^-1 is one dense contiguous segment [lo_i, i] and needs no column indices.
#include <algorithm>
#include <cmath>
#include <numeric>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "dphd_internal.h"

namespace dphd {

void init_samples(HostModel& M) {
    if (M.hex) {
        const double r = 1.0 / std::sqrt(3.0);
        const double dx = std::pow(M.vol, 1.0 / 3.0);
        const double inv_dx = 1.0 / dx;
        M.grad.assign(8 * 8 * 3, 0.0);
        for (int smp = 0; smp < 8; ++smp) {
            double p[3];
            const int bits[3] = {(smp >> 2) & 1, (smp >> 1) & 1, smp & 1};
            for (int d = 0; d < 3; ++d) p[d] = ((bits[d] - 0.5) * r + 0.5) * dx * inv_dx;
            const double lin[3][2] = {{1 - p[0], p[0]}, {1 - p[1], p[1]}, {1 - p[2], p[2]}};
            const double slope[2] = {-inv_dx, inv_dx};
            for (int node = 0; node < 8; ++node) {
                const int a = (node >> 2) & 1, b = (node >> 1) & 1, c = node & 1;
                double* g = &M.grad[(smp * 8 + node) * 3];
                g[0] = slope[a] * lin[1][b] * lin[2][c];
                g[1] = lin[0][a] * slope[b] * lin[2][c];
                g[2] = lin[0][a] * lin[1][b] * slope[c];
            }
        }
        return;
    }
    M.grad.assign((size_t)M.m * 12, 0.0);
    for (int e = 0; e < M.m; ++e) {
        const int* v = &M.E[(size_t)e * 4];
        double B[3][3];  // columns X1-X0, X2-X0, X3-X0
        for (int c = 0; c < 3; ++c)
            for (int d = 0; d < 3; ++d) B[d][c] = M.X[3 * v[c + 1] + d] - M.X[3 * v[0] + d];
        const double det = B[0][0] * (B[1][1] * B[2][2] - B[1][2] * B[2][1]) -
                           B[0][1] * (B[1][0] * B[2][2] - B[1][2] * B[2][0]) +
                           B[0][2] * (B[1][0] * B[2][1] - B[1][1] * B[2][0]);
        DPHD_CHECK(det != 0.0, "Degenerate tetrahedron " + std::to_string(e));
        double Bi[3][3];  // inverse: Bi[i][j] = cofactor(j,i)/det
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const int r0 = (j + 1) % 3, r1 = (j + 2) % 3, c0 = (i + 1) % 3, c1 = (i + 2) % 3;
                Bi[i][j] = (B[r0][c0] * B[r1][c1] - B[r0][c1] * B[r1][c0]) / det;
            }
        double* g = &M.grad[(size_t)e * 12];
        for (int d = 0; d < 3; ++d) {
            g[d] = -Bi[0][d] - Bi[1][d] - Bi[2][d];
            g[3 + d] = Bi[0][d];
            g[6 + d] = Bi[1][d];
            g[9 + d] = Bi[2][d];
        }
    }
}

double element_volume(const HostModel& M, int e) {
    const int* v = &M.E[(size_t)e * M.k];
    auto d = [&](int a, int b, int c) { return M.X[3 * v[a] + c] - M.X[3 * v[b] + c]; };
    double A[3][3];
    if (M.hex) {  // |det[v001-v000, v010-v000, v100-v000]|  (mesh.cpp Mesh<3,8>::ComputeElementVolume)
        for (int c = 0; c < 3; ++c) {
            A[c][0] = d(1, 0, c);
            A[c][1] = d(2, 0, c);
            A[c][2] = d(4, 0, c);
        }
    } else {
        for (int c = 0; c < 3; ++c) {
            A[c][0] = d(1, 0, c);
            A[c][1] = d(2, 0, c);
            A[c][2] = d(3, 0, c);
        }
    }
    const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                       A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                       A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    return M.hex ? std::fabs(det) : std::fabs(det / 6.0);
}

NodeMatrix assemble_A(const HostModel& M, double dt) {
    const int n = M.n;
    const double inv_h2m = M.mass() / (dt * dt);
    std::vector<uint8_t> fixed(n, 0);
    for (const auto& kv : M.dirichlet) fixed[kv.first / 3] = 1;
    struct Trip {
        int r, c;
        double v;
    };
    std::vector<Trip> t;
    t.reserve((size_t)M.m * M.k * M.k + n);
    for (int i = 0; i < n; ++i) t.push_back({i, i, fixed[i] ? 1.0 : inv_h2m});
    std::vector<double> blk((size_t)M.k * M.k);
    for (int e = 0; e < M.m; ++e) {
        double w = 0;
        for (const auto& en : M.energies)
            if (en.all_elements || en.in_set[e]) w += en.elem_w(e);
        std::fill(blk.begin(), blk.end(), 0.0);
        for (int smp = 0; smp < M.s; ++smp) {
            const double* g = M.g(e, smp);
            const double scale = w * M.vol / M.s;
            for (int a = 0; a < M.k; ++a)
                for (int b = 0; b < M.k; ++b)
                    blk[a * M.k + b] += (g[a * 3] * g[b * 3] + g[a * 3 + 1] * g[b * 3 + 1] + g[a * 3 + 2] * g[b * 3 + 2]) * scale;
        }
        const int* v = &M.E[(size_t)e * M.k];
        for (int a = 0; a < M.k; ++a)
            for (int b = 0; b < M.k; ++b) {
                if (fixed[v[a]] || fixed[v[b]]) continue;
                t.push_back({v[a], v[b], blk[a * M.k + b]});
            }
    }
    std::sort(t.begin(), t.end(), [](const Trip& x, const Trip& y) { return x.r != y.r ? x.r < y.r : x.c < y.c; });
    NodeMatrix A;
    A.n = n;
    A.rp.assign(n + 1, 0);
    for (size_t p = 0; p < t.size();) {
        size_t q = p;
        double s = 0;
        while (q < t.size() && t[q].r == t[p].r && t[q].c == t[p].c) s += t[q++].v;
        A.ci.push_back(t[p].c);
        A.v.push_back(s);
        A.rp[t[p].r + 1]++;
        p = q;
    }
    for (int i = 0; i < n; ++i) A.rp[i + 1] += A.rp[i];
    return A;
}

// Nested dissection by recursive coordinate bisection on the rest configuration: split at the median
// coordinate of the longest extent; the separator is the set of lower-side nodes adjacent to the upper
// side; order = [lower part, upper part, separator], recursively.
std::vector<int> nested_dissection(const HostModel& M, const NodeMatrix& A) {
    const int n = M.n;
    std::vector<int> order;
    order.reserve(n);
    std::vector<int8_t> side(n, 0);
    struct Job {
        std::vector<int> nodes;
        int stage;  // 0: split, 1: emit separator
        std::vector<int> sep;
    };
    std::vector<Job> stack;
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    stack.push_back({all, 0, {}});
    while (!stack.empty()) {
        Job job = std::move(stack.back());
        stack.pop_back();
        if (job.stage == 1) {
            order.insert(order.end(), job.sep.begin(), job.sep.end());
            continue;
        }
        std::vector<int>& nodes = job.nodes;
        if (nodes.size() <= 32) {
            order.insert(order.end(), nodes.begin(), nodes.end());
            continue;
        }
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int v : nodes)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::min(lo[d], M.X[3 * v + d]);
                hi[d] = std::max(hi[d], M.X[3 * v + d]);
            }
        int ax = 0;
        for (int d = 1; d < 3; ++d)
            if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
        std::vector<double> c;
        c.reserve(nodes.size());
        for (int v : nodes) c.push_back(M.X[3 * v + ax]);
        std::nth_element(c.begin(), c.begin() + c.size() / 2, c.end());
        const double cut = c[c.size() / 2];
        for (int v : nodes) side[v] = M.X[3 * v + ax] < cut ? 1 : 2;
        std::vector<int> L, R, S;
        for (int v : nodes) {
            if (side[v] != 1) continue;
            for (int p = A.rp[v]; p < A.rp[v + 1]; ++p)
                if (side[A.ci[p]] == 2) {
                    S.push_back(v);
                    break;
                }
        }
        for (int v : S) side[v] = 3;
        for (int v : nodes) {
            if (side[v] == 1) L.push_back(v);
            else if (side[v] == 2) R.push_back(v);
        }
        for (int v : nodes) side[v] = 0;
        if (L.empty() || R.empty()) {
            order.insert(order.end(), nodes.begin(), nodes.end());
            continue;
        }
        // processed in stack order: L first, then R, then the separator
        stack.push_back({{}, 1, std::move(S)});
        stack.push_back({std::move(R), 0, {}});
        stack.push_back({std::move(L), 0, {}});
    }
    DPHD_CHECK((int)order.size() == n, "nested dissection lost nodes");
    return order;
}

namespace {

// Upper triangle (row <= col) of P A P^T by columns, for order[k] = original node at position k.
void permuted_upper(const NodeMatrix& A, const std::vector<int>& order, std::vector<int>& Cp, std::vector<int>& Ci,
                    std::vector<double>& Cx) {
    const int n = A.n;
    std::vector<int> ip(n);
    for (int k = 0; k < n; ++k) ip[order[k]] = k;
    Cp.assign(n + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int p = A.rp[r]; p < A.rp[r + 1]; ++p)
            if (ip[r] <= ip[A.ci[p]]) Cp[ip[A.ci[p]] + 1]++;
    for (int k = 0; k < n; ++k) Cp[k + 1] += Cp[k];
    Ci.assign(Cp[n], 0);
    Cx.assign(Cp[n], 0);
    std::vector<int> pos(Cp.begin(), Cp.end() - 1);
    for (int r = 0; r < n; ++r)
        for (int p = A.rp[r]; p < A.rp[r + 1]; ++p) {
            const int pr = ip[r], pc = ip[A.ci[p]];
            if (pr <= pc) {
                Ci[pos[pc]] = pr;
                Cx[pos[pc]++] = A.v[p];
            }
        }
}

// Elimination tree (Liu's algorithm with path compression).
std::vector<int> etree(int n, const std::vector<int>& Cp, const std::vector<int>& Ci) {
    std::vector<int> parent(n, -1), anc(n, -1);
    for (int k = 0; k < n; ++k)
        for (int p = Cp[k]; p < Cp[k + 1]; ++p) {
            int i = Ci[p];
            while (i != -1 && i < k) {
                const int nx = anc[i];
                anc[i] = k;
                if (nx == -1) parent[i] = k;
                i = nx;
            }
        }
    return parent;
}

}  // namespace

void sfactor_symbolic(const NodeMatrix& A, const std::vector<int>& order0, SFactor& S, PermUpper& U) {
    const int n = A.n;
    std::vector<int>& Cp = U.Cp;
    std::vector<int>& Ci = U.Ci;
    std::vector<double>& Cx = U.Cx;
    permuted_upper(A, order0, Cp, Ci, Cx);
    std::vector<int> par = etree(n, Cp, Ci);
    // postorder (children visited in increasing index order)
    std::vector<int> head(n, -1), next(n, -1);
    for (int j = n - 1; j >= 0; --j)
        if (par[j] != -1) {
            next[j] = head[par[j]];
            head[par[j]] = j;
        }
    std::vector<int> post;
    post.reserve(n);
    std::vector<int> stk;
    for (int r = 0; r < n; ++r) {
        if (par[r] != -1) continue;
        stk.push_back(r);
        while (!stk.empty()) {
            const int top = stk.back();
            const int c = head[top];
            if (c == -1) {
                post.push_back(top);
                stk.pop_back();
            } else {
                head[top] = next[c];
                stk.push_back(c);
            }
        }
    }
    DPHD_CHECK((int)post.size() == n, "etree postorder incomplete");
    S.n = n;
    S.perm.resize(n);
    for (int k = 0; k < n; ++k) S.perm[k] = order0[post[k]];
    S.iperm.assign(n, 0);
    for (int k = 0; k < n; ++k) S.iperm[S.perm[k]] = k;
    permuted_upper(A, S.perm, Cp, Ci, Cx);
    S.parent = etree(n, Cp, Ci);
    // subtree sizes -> lo; depth
    std::vector<int> size(n, 1);
    for (int j = 0; j < n; ++j)
        if (S.parent[j] != -1) size[S.parent[j]] += size[j];
    S.lo.resize(n);
    for (int j = 0; j < n; ++j) {
        S.lo[j] = j - size[j] + 1;
        DPHD_CHECK(S.lo[j] >= 0, "postorder violated");
    }
    {
        std::vector<int> depth(n, 0);
        for (int j = n - 1; j >= 0; --j) depth[j] = S.parent[j] == -1 ? 0 : depth[S.parent[j]] + 1;
        S.max_depth = n ? *std::max_element(depth.begin(), depth.end()) : 0;
    }
    S.row_ptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) S.row_ptr[i + 1] = S.row_ptr[i] + (i - S.lo[i] + 1);
}

void build_sfactor(const NodeMatrix& A, const std::vector<int>& order0, SFactor& S, int threads) {
    PermUpper U;
    sfactor_symbolic(A, order0, S, U);
    sfactor_numeric_host(U, S, threads);
}

void sfactor_numeric_host(const PermUpper& U, SFactor& S, int threads) {
    const int n = S.n;
    const std::vector<int>& Cp = U.Cp;
    const std::vector<int>& Ci = U.Ci;
    const std::vector<double>& Cx = U.Cx;
    // Up-looking LDL^T (Davis, ACM TOMS Algorithm 849): row k of L is computed from a sparse triangular
    // solve whose pattern is the row subtree of k.  Rows of L are kept for the L^-1 recurrence below.
    std::vector<int> lnz(n, 0), flag(n, -1);
    for (int k = 0; k < n; ++k) {
        flag[k] = k;
        for (int p = Cp[k]; p < Cp[k + 1]; ++p)
            for (int i = Ci[p]; i < k && flag[i] != k; i = S.parent[i]) {
                lnz[i]++;
                flag[i] = k;
            }
    }
    std::vector<int64_t> Lp(n + 1, 0);
    for (int k = 0; k < n; ++k) Lp[k + 1] = Lp[k] + lnz[k];
    S.nnz_L = Lp[n];
    std::vector<int> Li(Lp[n]);
    std::vector<double> Lx(Lp[n]), D(n), Y(n, 0.0);
    std::vector<int> pattern(n);
    std::vector<int64_t> Rp(n + 1, 0);  // rows of L: row k has (Lp-style) entries appended at step k
    std::vector<int> Rj;
    std::vector<double> Rx;
    Rj.reserve(Lp[n]);
    Rx.reserve(Lp[n]);
    std::fill(lnz.begin(), lnz.end(), 0);
    std::fill(flag.begin(), flag.end(), -1);
    for (int k = 0; k < n; ++k) {
        int top = n;
        flag[k] = k;
        for (int p = Cp[k]; p < Cp[k + 1]; ++p) {
            int i = Ci[p];
            Y[i] += Cx[p];
            int len = 0;
            for (; flag[i] != k; i = S.parent[i]) {
                pattern[len++] = i;
                flag[i] = k;
            }
            while (len > 0) pattern[--top] = pattern[--len];
        }
        double dk = Y[k];
        Y[k] = 0;
        for (; top < n; ++top) {
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
        DPHD_CHECK(dk > 0 && std::isfinite(dk), "PD matrix is not positive definite (LDL^T pivot " +
                                                    std::to_string(dk) + " at row " + std::to_string(k) + ")");
        D[k] = dk;
    }
    // S rows: row_i(L^-1) = e_i - sum_{k in row_i(L)} l_ik row_k(L^-1), each row dense on [lo_i, i].
    S.vals.assign(S.row_ptr[n], 0.0);
    S.Dinv_sqrt.resize(n);
    for (int i = 0; i < n; ++i) S.Dinv_sqrt[i] = 1.0 / std::sqrt(D[i]);
    // Column c of L^-1 depends only on column c of the rows above it, so the recurrence runs over independent
    // column blocks in parallel; inside a block the rows go in increasing order (every row k < i that row i
    // needs is done by then).  Each entry is summed in the same order as a row-at-a-time sweep would.
    // the thread count goes to these two loops only (num_threads clauses), not to the process-wide default
    const int nthr = threads > 0 ? threads : 0;
    auto row_span = [&](int i, int c0, int c1) {
        // accumulate columns [c0, c1) of row i
        double* out = &S.vals[S.row_ptr[i]] - S.lo[i];
        for (int c = c0; c < c1; ++c) out[c] = (c == i) ? 1.0 : 0.0;
        for (int64_t p = Rp[i]; p < Rp[i + 1]; ++p) {
            const int k = Rj[p];
            const double l = Rx[p];
            const int a = std::max(c0, S.lo[k]), b = std::min(c1, k + 1);
            if (a >= b) continue;
            const double* rk = &S.vals[S.row_ptr[k]] - S.lo[k];
            for (int c = a; c < b; ++c) out[c] -= l * rk[c];
        }
    };
    constexpr int kColBlock = 64;
    const int nblk = (n + kColBlock - 1) / kColBlock;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthr > 0 ? nthr : omp_get_max_threads())
    for (int blk = 0; blk < nblk; ++blk) {
        const int c0 = blk * kColBlock, c1 = std::min(n, c0 + kColBlock);
        for (int i = c0; i < n; ++i)
            if (S.lo[i] < c1) row_span(i, std::max(c0, S.lo[i]), std::min(c1, i + 1));
    }
    // scale rows by D^-1/2
#pragma omp parallel for schedule(static) num_threads(nthr > 0 ? nthr : omp_get_max_threads())
    for (int i = 0; i < n; ++i) {
        double* r = &S.vals[S.row_ptr[i]];
        const int64_t len = S.row_ptr[i + 1] - S.row_ptr[i];
        for (int64_t c = 0; c < len; ++c) r[c] *= S.Dinv_sqrt[i];
    }
}

// Without a host copy of the S values (a device-built factor) only the path rows are filled; the values are
// then gathered on the device.
ContactPaths build_contact_paths(const SFactor& S, const std::vector<int>& cand_nodes) {
    ContactPaths P;
    const int K = (int)cand_nodes.size();
    P.off.assign(K + 1, 0);
    std::vector<std::vector<int>> paths(K);
    for (int c = 0; c < K; ++c) {
        const int col = S.iperm[cand_nodes[c]];
        for (int r = col; r != -1; r = S.parent[r]) paths[c].push_back(r);
        std::reverse(paths[c].begin(), paths[c].end());
        P.off[c + 1] = P.off[c] + (int64_t)paths[c].size();
        P.max_depth = std::max(P.max_depth, (int)paths[c].size());
    }
    P.row.resize(P.off[K]);
    if (!S.vals.empty()) P.val.resize(P.off[K]);
    for (int c = 0; c < K; ++c) {
        const int col = S.iperm[cand_nodes[c]];
        for (size_t k = 0; k < paths[c].size(); ++k) {
            const int r = paths[c][k];
            P.row[P.off[c] + k] = r;
            if (!S.vals.empty()) P.val[P.off[c] + k] = S.vals[S.row_ptr[r] + (col - S.lo[r])];
        }
    }
    return P;
}

}  // namespace dphd
