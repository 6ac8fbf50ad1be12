// ORACLE — test infrastructure only. Never linked into, or called by, the product path.
//
// CPU FP64 restatement of the reference's projective-dynamics "AlgPhd" time step and its adjoint
// (DiffPhD, method "pd_eigen_alg_phd"), as the reference runs it without CUDA: every A^-1 apply is a
// sparse LDL^T solve (cpp/core/src/fem/deformable_projective_dynamics_forward_gpu.cpp:837 falls back to
// pd_eigen_solver_[d].solve; the backward always uses it, deformable_projective_dynamics_backward_gpu.cpp:763-775).
//
// Parity status: the reference cannot be compiled in this environment (its Eigen submodule is empty and
// there is no network), and it ships no golden vectors, so this restatement is "parity unpinned" against
// the reference binary. Its building blocks are pinned instead against independent implementations in the
// CPU test-suite: the 3x3 SVD and polar factor against LAPACK (numpy), A^-1 against SciPy's sparse solver,
// projections against their defining optimality conditions, and the adjoint against central finite
// differences of this forward.
//
// Eigen calls the reference makes are restated here from the published algorithms:
//   * Eigen::JacobiSVD (3x3)        -> two-sided cyclic Jacobi SVD (Forsythe & Henrici 1960; the 2x2
//                                      symmetrise-then-diagonalise step of Brent & Luk 1985), singular
//                                      values >= 0 sorted descending, U and V orthogonal (det may be -1).
//   * Eigen::SimplicialLDLT         -> up-looking sparse LDL^T (Davis, ACM TOMS Algorithm 849) on a
//                                      nested-dissection ordering by recursive coordinate bisection.
//   * small dense LDLT / inverse    -> Gaussian elimination with partial pivoting.
// Build: oracle/Makefile  ->  oracle/_build/libpd_oracle.so  (ctypes, C ABI below).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef double real;
thread_local std::string g_err;

struct OracleError {
    std::string msg;
};
#define ORC_CHECK(cond, msg)                  \
    do {                                      \
        if (!(cond)) throw OracleError{(msg)}; \
    } while (0)

// ------------------------------------------------------------------------------------------------
// Small dense 3x3 helpers. Matrices are column-major 9-vectors, F(i,j) = F[i + 3j]
// (Flatten/Unflatten, cpp/core/src/common/geometry.cpp:192-200).
// ------------------------------------------------------------------------------------------------
struct M3 {
    real a[9];
    real& operator()(int i, int j) { return a[i + 3 * j]; }
    real operator()(int i, int j) const { return a[i + 3 * j]; }
};
static M3 zero3() { M3 m; for (int i = 0; i < 9; ++i) m.a[i] = 0; return m; }
static M3 eye3() { M3 m = zero3(); m(0, 0) = m(1, 1) = m(2, 2) = 1; return m; }
static M3 mul(const M3& A, const M3& B) {
    M3 C = zero3();
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            real s = 0;
            for (int k = 0; k < 3; ++k) s += A(i, k) * B(k, j);
            C(i, j) = s;
        }
    return C;
}
static M3 transpose(const M3& A) {
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C(i, j) = A(j, i);
    return C;
}
static real det3(const M3& A) {
    return A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) - A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
           A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
}
// U diag(s) V^T
static M3 usvt(const M3& U, const real* s, const M3& V) {
    M3 C = zero3();
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            real acc = 0;
            for (int k = 0; k < 3; ++k) acc += U(i, k) * s[k] * V(j, k);
            C(i, j) = acc;
        }
    return C;
}
// Solve a small dense system (n <= 8) by Gaussian elimination with partial pivoting.
static void dense_solve(int n, std::vector<real> A, std::vector<real>& b) {
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        if (piv != c) {
            for (int k = 0; k < n; ++k) std::swap(A[c * n + k], A[piv * n + k]);
            std::swap(b[c], b[piv]);
        }
        const real d = A[c * n + c];
        for (int r = c + 1; r < n; ++r) {
            const real f = A[r * n + c] / d;
            if (f == 0) continue;
            for (int k = c; k < n; ++k) A[r * n + k] -= f * A[c * n + k];
            b[r] -= f * b[c];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        real s = b[c];
        for (int k = c + 1; k < n; ++k) s -= A[c * n + k] * b[k];
        b[c] = s / A[c * n + c];
    }
}

// ------------------------------------------------------------------------------------------------
// 3x3 SVD, restating Eigen::JacobiSVD's contract (deformation_gradient_auxiliary_data.cpp:6,
// geometry.cpp:24-31): F = U diag(sig) V^T, sig >= 0 descending.
// Two-sided Jacobi: for each pair (p,q) a rotation on the left symmetrises the 2x2 block, then a
// symmetric Jacobi rotation diagonalises it; sweeps run until the off-diagonal is below eps*max|diag|.
// ------------------------------------------------------------------------------------------------
static void svd3(const M3& F, M3& U, real* sig, M3& V) {
    M3 A = F;
    U = eye3();
    V = eye3();
    const real eps = std::numeric_limits<real>::epsilon();
    const real tiny = std::numeric_limits<real>::min();
    for (int sweep = 0; sweep < 64; ++sweep) {
        bool changed = false;
        real maxdiag = 0;
        for (int i = 0; i < 3; ++i) maxdiag = std::max(maxdiag, std::fabs(A(i, i)));
        const real thr = std::max(tiny, 2 * eps * maxdiag);
        for (int p = 1; p < 3; ++p)
            for (int q = 0; q < p; ++q) {
                if (!(std::fabs(A(p, q)) > thr || std::fabs(A(q, p)) > thr)) continue;
                changed = true;
                // 2x2 block [[a b],[c d]] on rows/cols (q,p).
                const real a = A(q, q), b = A(q, p), c = A(p, q), d = A(p, p);
                // Left rotation G1 = [[c1, s1],[-s1, c1]] making G1*block symmetric:
                // (G1 B)(0,1) == (G1 B)(1,0)  ->  c1*b + s1*d == -s1*a + c1*c
                real c1 = 1, s1 = 0;
                const real t = a + d, dd = c - b;
                if (std::fabs(dd) > tiny) {
                    const real u = t / dd;
                    const real tmp = std::sqrt(1 + u * u);
                    s1 = 1 / tmp;
                    c1 = u / tmp;
                    // orientation: require c1*b + s1*d == -s1*a + c1*c
                }
                // symmetric block after left rotation
                real m00 = c1 * a + s1 * c, m01 = c1 * b + s1 * d;
                real m10 = -s1 * a + c1 * c, m11 = -s1 * b + c1 * d;
                (void)m10;
                // Jacobi rotation J = [[cj, sj],[-sj, cj]] with J^T M J diagonal.
                real cj = 1, sj = 0;
                if (std::fabs(m01) > tiny) {
                    const real tau = (m11 - m00) / (2 * m01);
                    const real tt = (tau >= 0 ? 1 : -1) / (std::fabs(tau) + std::sqrt(1 + tau * tau));
                    cj = 1 / std::sqrt(1 + tt * tt);
                    sj = tt * cj;
                }
                // Left total: L = J^T G1 ; right: R = J.  Block -> L B R diagonal.
                const real l00 = cj * c1 + sj * s1, l01 = cj * s1 - sj * c1;
                const real l10 = sj * c1 - cj * s1, l11 = sj * s1 + cj * c1;
                // rows q,p of A <- L * rows
                for (int k = 0; k < 3; ++k) {
                    const real x = A(q, k), y = A(p, k);
                    A(q, k) = l00 * x + l01 * y;
                    A(p, k) = l10 * x + l11 * y;
                }
                // cols q,p of A <- cols * J
                for (int k = 0; k < 3; ++k) {
                    const real x = A(k, q), y = A(k, p);
                    A(k, q) = cj * x - sj * y;
                    A(k, p) = sj * x + cj * y;
                }
                // U <- U * L^T ; V <- V * J
                for (int k = 0; k < 3; ++k) {
                    const real x = U(k, q), y = U(k, p);
                    U(k, q) = l00 * x + l01 * y;
                    U(k, p) = l10 * x + l11 * y;
                }
                for (int k = 0; k < 3; ++k) {
                    const real x = V(k, q), y = V(k, p);
                    V(k, q) = cj * x - sj * y;
                    V(k, p) = sj * x + cj * y;
                }
            }
        if (!changed) break;
    }
    // Make singular values non-negative (flip U's column) and sort descending.
    real s[3];
    for (int i = 0; i < 3; ++i) {
        s[i] = A(i, i);
        if (s[i] < 0) {
            s[i] = -s[i];
            for (int k = 0; k < 3; ++k) U(k, i) = -U(k, i);
        }
    }
    int idx[3] = {0, 1, 2};
    std::sort(idx, idx + 3, [&](int x, int y) { return s[x] > s[y]; });
    M3 U2, V2;
    for (int j = 0; j < 3; ++j) {
        sig[j] = s[idx[j]];
        for (int k = 0; k < 3; ++k) {
            U2(k, j) = U(k, idx[j]);
            V2(k, j) = V(k, idx[j]);
        }
    }
    U = U2;
    V = V2;
}

// dSVD (Townsend, "Differentiating the singular value decomposition"), restating
// cpp/core/src/common/geometry.cpp:159-186 including its 10*eps skip of near-equal singular values.
static void dsvd3(const M3& U, const real* sig, const M3& V, const M3& dF, M3& dU, real* dsig, M3& dV) {
    const M3 dP = mul(mul(transpose(U), dF), V);
    for (int i = 0; i < 3; ++i) dsig[i] = dP(i, i);
    const real eps = 10 * std::numeric_limits<real>::epsilon();
    M3 Sij = zero3();
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j)
            if (sig[i] - sig[j] > eps) {
                Sij(i, j) = 1 / (sig[j] * sig[j] - sig[i] * sig[i]);
                Sij(j, i) = -Sij(i, j);
            }
    M3 wU = zero3(), wV = zero3();
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            // (dP S + S dP^T)_ij and (S dP + dP^T S)_ij
            const real a = dP(i, j) * sig[j] + sig[i] * dP(j, i);
            const real b = sig[i] * dP(i, j) + dP(j, i) * sig[j];
            wU(i, j) = Sij(i, j) * a;
            wV(i, j) = Sij(i, j) * b;
        }
    dU = mul(U, wU);
    dV = mul(V, wV);
}

// ------------------------------------------------------------------------------------------------
// Projections ("ProjectToManifold") and their differentials.
// ------------------------------------------------------------------------------------------------
enum EnergyType { kCorotated = 0, kVolume = 1, kNeoHookean = 2 };

struct SvdData {
    M3 F, U, V, R, S;
    real sig[3];
};
static SvdData make_svd(const M3& F) {
    SvdData d;
    d.F = F;
    svd3(F, d.U, d.sig, d.V);
    d.R = mul(d.U, transpose(d.V));
    d.S = usvt(d.V, d.sig, d.V);
    return d;
}

// Volume projection: Newton iterations on D with prod(sig + D) = 1
// (volume_pd_element_energy.cpp:22-59).
static void volume_D(const real* sig, real* D) {
    const real eps = std::numeric_limits<real>::epsilon();
    ORC_CHECK(std::min(sig[0], std::min(sig[1], sig[2])) >= eps, "Singular F.");
    const real prod = sig[0] * sig[1] * sig[2];
    const real cr = std::pow(prod, real(1) / 3);
    for (int i = 0; i < 3; ++i) D[i] = sig[i] / cr - sig[i];
    for (int it = 0; it < 50; ++it) {
        const real C = (sig[0] + D[0]) * (sig[1] + D[1]) * (sig[2] + D[2]) - 1;
        real g[3];
        for (int j = 0; j < 3; ++j) {
            g[j] = 1;
            for (int k = 0; k < 3; ++k)
                if (k != j) g[j] *= (sig[k] + D[k]);
        }
        const real gd = g[0] * D[0] + g[1] * D[1] + g[2] * D[2];
        const real gg = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
        real Dn[3], diff = 0;
        for (int j = 0; j < 3; ++j) {
            Dn[j] = (gd - C) / gg * g[j];
            diff = std::max(diff, std::fabs(Dn[j] - D[j]));
        }
        if (diff <= eps) break;
        for (int j = 0; j < 3; ++j) D[j] = Dn[j];
    }
}

// Neo-Hookean proximal map on singular values (neohookean_pd_element_energy.cpp:38-104).
struct NhParams {
    real mu, la, k;
};
static void nh_hessian(const NhParams& p, const real* s, real* H) {
    const real prod = s[0] * s[1] * s[2];
    const real L = std::log(std::max(prod, real(1e-12)));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            H[i * 3 + j] = (i == j) ? p.mu + (p.mu + p.la - p.la * L) / (s[i] * s[i]) + p.k : p.la / (s[i] * s[j]);
}
static void nh_solve_prox(const NhParams& p, const real* sigF, real* sig) {
    const real sig_min = 1e-4, tol = 1e-10;
    for (int i = 0; i < 3; ++i) sig[i] = std::max(sigF[i], sig_min);
    for (int it = 0; it < 32; ++it) {
        const real prod = sig[0] * sig[1] * sig[2];
        const real L = std::log(std::max(prod, real(1e-12)));
        real g[3];
        for (int i = 0; i < 3; ++i)
            g[i] = p.mu * sig[i] - p.mu / sig[i] + p.la * L / sig[i] + p.k * (sig[i] - sigF[i]);
        if (std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) < tol) break;
        real H[9];
        nh_hessian(p, sig, H);
        for (int i = 0; i < 3; ++i) H[i * 3 + i] += 1e-9;
        std::vector<real> Hv(H, H + 9), dv(g, g + 3);
        dense_solve(3, Hv, dv);
        real alpha = 1, sn[3];
        for (int i = 0; i < 3; ++i) sn[i] = sig[i] - alpha * dv[i];
        for (int ls = 0; ls < 20; ++ls) {
            const real mn = std::min(sn[0], std::min(sn[1], sn[2]));
            if (mn > sig_min * 0.5) break;
            alpha *= 0.5;
            for (int i = 0; i < 3; ++i) sn[i] = sig[i] - alpha * dv[i];
        }
        real step = 0;
        for (int i = 0; i < 3; ++i) step = std::max(step, std::fabs(sn[i] - sig[i]));
        for (int i = 0; i < 3; ++i) sig[i] = std::max(sn[i], sig_min);
        if (step < tol) break;
    }
}

// dR from dF (geometry.cpp:60-113).
static M3 dR_from_dF(const M3& R, const M3& S, const M3& dF) {
    const M3 lhs = [&] {
        M3 a = mul(transpose(R), dF), b = mul(transpose(dF), R), c;
        for (int i = 0; i < 9; ++i) c.a[i] = a.a[i] - b.a[i];
        return c;
    }();
    std::vector<real> A(9);
    A[0] = S(0, 0) + S(1, 1);
    A[4] = S(0, 0) + S(2, 2);
    A[8] = S(1, 1) + S(2, 2);
    A[1] = A[3] = S(1, 2);
    A[2] = A[6] = -S(0, 2);
    A[5] = A[7] = S(0, 1);
    std::vector<real> b = {lhs(0, 1), lhs(0, 2), lhs(1, 2)};
    dense_solve(3, A, b);
    M3 W = zero3();
    W(0, 1) = b[0];
    W(0, 2) = b[1];
    W(1, 0) = -b[0];
    W(1, 2) = b[2];
    W(2, 0) = -b[1];
    W(2, 1) = -b[2];
    return mul(R, W);
}

struct Energy {
    int type;
    std::vector<real> params;       // as passed to AddPdEnergy
    std::vector<real> w_elem;       // element_stiffness(e), empty when homogeneous
    real w_mean;                    // stiffness()
    real mu, la;                    // NH means (projection uses means)
    std::vector<char> in_set;       // element membership
    real elem_w(int e) const { return w_elem.empty() ? w_mean : w_elem[e]; }
    NhParams nh() const { return NhParams{mu, la, w_mean}; }
};

static M3 project(const Energy& en, const SvdData& d) {
    if (en.type == kCorotated) return d.R;
    if (en.type == kVolume) {
        real D[3];
        volume_D(d.sig, D);
        real s[3] = {d.sig[0] + D[0], d.sig[1] + D[1], d.sig[2] + D[2]};
        return usvt(d.U, s, d.V);
    }
    real s[3];
    nh_solve_prox(en.nh(), d.sig, s);
    return usvt(d.U, s, d.V);
}

// d(project)/dF along dF (corotated: geometry.cpp dRFromdF; volume: volume_pd_element_energy.cpp:61-155;
// NH: neohookean_pd_element_energy.cpp:133-165).
static M3 project_diff(const Energy& en, const SvdData& d, const M3& dF) {
    if (en.type == kCorotated) return dR_from_dF(d.R, d.S, dF);
    const real* sig = d.sig;
    M3 dU, dV;
    real dsig[3];
    dsvd3(d.U, sig, d.V, dF, dU, dsig, dV);
    if (en.type == kVolume) {
        real D[3];
        volume_D(sig, D);
        real g[3];
        for (int j = 0; j < 3; ++j) {
            g[j] = 1;
            for (int k = 0; k < 3; ++k)
                if (k != j) g[j] *= (sig[k] + D[k]);
        }
        real H[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                if (i == j) { H[i * 3 + j] = 0; continue; }
                real h = 1;
                for (int k = 0; k < 3; ++k)
                    if (k != i && k != j) h *= (sig[k] + D[k]);
                H[i * 3 + j] = h;
            }
        const real Dn = std::sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
        const real gn = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        const real la_abs = Dn / gn;
        real la = la_abs, e1 = 0, e2 = 0;
        for (int i = 0; i < 3; ++i) {
            e1 += (D[i] - la_abs * g[i]) * (D[i] - la_abs * g[i]);
            e2 += (D[i] + la_abs * g[i]) * (D[i] + la_abs * g[i]);
        }
        if (e1 < e2) la = -la_abs;
        std::vector<real> A(16, 0), b(4, 0);
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) A[i * 4 + j] = (i == j ? 1 : 0) + la * H[i * 3 + j];
            A[i * 4 + 3] = g[i];
            A[3 * 4 + i] = g[i];
            real hd = 0;
            for (int j = 0; j < 3; ++j) hd += H[i * 3 + j] * dsig[j];
            b[i] = -la * hd;
        }
        b[3] = -(g[0] * dsig[0] + g[1] * dsig[1] + g[2] * dsig[2]);
        dense_solve(4, A, b);
        const real dD[3] = {b[0], b[1], b[2]};
        const M3 t1 = usvt(dU, D, d.V), t2 = usvt(d.U, dD, d.V), t3 = usvt(d.U, D, dV);
        M3 out;
        for (int i = 0; i < 9; ++i) out.a[i] = dF.a[i] + t1.a[i] + t2.a[i] + t3.a[i];
        return out;
    }
    // Neo-Hookean
    const NhParams p = en.nh();
    real ss[3];
    nh_solve_prox(p, sig, ss);
    real H[9];
    nh_hessian(p, ss, H);
    for (int i = 0; i < 3; ++i) H[i * 3 + i] += 1e-9;
    std::vector<real> Hv(H, H + 9), rhs = {p.k * dsig[0], p.k * dsig[1], p.k * dsig[2]};
    dense_solve(3, Hv, rhs);
    const real ds[3] = {rhs[0], rhs[1], rhs[2]};
    const M3 t1 = usvt(dU, ss, d.V), t2 = usvt(d.U, ds, d.V), t3 = usvt(d.U, ss, dV);
    M3 out;
    for (int i = 0; i < 9; ++i) out.a[i] = t1.a[i] + t2.a[i] + t3.a[i];
    return out;
}

// d(project)/d(mu_bar) and d(project)/d(la_bar) for the NH proximal map with k = 2*mu_bar
// (implicit function theorem on the prox optimality g(sig*) = 0; components clamped at sig_min get 0).
static void nh_param_diff(const Energy& en, const SvdData& d, M3& dP_dmu, M3& dP_dla) {
    const NhParams p = en.nh();
    real ss[3];
    nh_solve_prox(p, d.sig, ss);
    real H[9];
    nh_hessian(p, ss, H);
    for (int i = 0; i < 3; ++i) H[i * 3 + i] += 1e-9;
    const real prod = ss[0] * ss[1] * ss[2];
    const real L = std::log(std::max(prod, real(1e-12)));
    std::vector<real> gm(3), gl(3);
    for (int i = 0; i < 3; ++i) {
        gm[i] = -(ss[i] - 1 / ss[i] + 2 * (ss[i] - d.sig[i]));
        gl[i] = -(L / ss[i]);
    }
    std::vector<real> Hv(H, H + 9);
    dense_solve(3, Hv, gm);
    Hv.assign(H, H + 9);
    dense_solve(3, Hv, gl);
    real a[3], b[3];
    for (int i = 0; i < 3; ++i) {
        const bool clamped = ss[i] <= 1e-4;
        a[i] = clamped ? 0 : gm[i];
        b[i] = clamped ? 0 : gl[i];
    }
    dP_dmu = usvt(d.U, a, d.V);
    dP_dla = usvt(d.U, b, d.V);
}

// ------------------------------------------------------------------------------------------------
// Sparse LDL^T (Davis, Algorithm 849) on a nested-dissection ordering.
// ------------------------------------------------------------------------------------------------
struct Ldl {
    int n = 0;
    std::vector<int> perm, iperm;    // perm[k] = original index placed at position k
    std::vector<int> Lp, Li, parent;
    std::vector<real> Lx, D;
    // A given as symmetric adjacency (both triangles) CSR in original indexing.
    void factor(int n_, const std::vector<int>& Ap, const std::vector<int>& Ai, const std::vector<real>& Ax,
                const std::vector<int>& order) {
        n = n_;
        perm = order;
        iperm.assign(n, 0);
        for (int k = 0; k < n; ++k) iperm[perm[k]] = k;
        // Upper triangle of C = P A P^T, column-wise: column k holds rows i <= k.
        std::vector<int> Cp(n + 1, 0), cnt(n, 0);
        for (int r = 0; r < n; ++r)
            for (int p = Ap[r]; p < Ap[r + 1]; ++p) {
                const int c = Ai[p];
                const int pr = iperm[r], pc = iperm[c];
                if (pr <= pc) cnt[pc]++;
            }
        for (int k = 0; k < n; ++k) Cp[k + 1] = Cp[k] + cnt[k];
        std::vector<int> Ci(Cp[n]), pos(Cp.begin(), Cp.end() - 1);
        std::vector<real> Cx(Cp[n]);
        for (int r = 0; r < n; ++r)
            for (int p = Ap[r]; p < Ap[r + 1]; ++p) {
                const int c = Ai[p];
                const int pr = iperm[r], pc = iperm[c];
                if (pr <= pc) {
                    Ci[pos[pc]] = pr;
                    Cx[pos[pc]++] = Ax[p];
                }
            }
        // symbolic
        parent.assign(n, -1);
        std::vector<int> flag(n), lnz(n, 0);
        for (int k = 0; k < n; ++k) {
            flag[k] = k;
            for (int p = Cp[k]; p < Cp[k + 1]; ++p) {
                int i = Ci[p];
                if (i < k) {
                    for (; flag[i] != k; i = parent[i]) {
                        if (parent[i] == -1) parent[i] = k;
                        lnz[i]++;
                        flag[i] = k;
                    }
                }
            }
        }
        Lp.assign(n + 1, 0);
        for (int k = 0; k < n; ++k) Lp[k + 1] = Lp[k] + lnz[k];
        Li.assign(Lp[n], 0);
        Lx.assign(Lp[n], 0);
        D.assign(n, 0);
        // numeric (up-looking)
        std::vector<real> Y(n, 0);
        std::vector<int> pattern(n);
        std::fill(lnz.begin(), lnz.end(), 0);
        for (int k = 0; k < n; ++k) {
            Y[k] = 0;
            int top = n;
            flag[k] = k;
            for (int p = Cp[k]; p < Cp[k + 1]; ++p) {
                int i = Ci[p];
                Y[i] += Cx[p];
                int len = 0;
                for (; flag[i] != k; i = parent[i]) {
                    pattern[len++] = i;
                    flag[i] = k;
                }
                while (len > 0) pattern[--top] = pattern[--len];
            }
            D[k] = Y[k];
            Y[k] = 0;
            for (; top < n; ++top) {
                const int i = pattern[top];
                const real yi = Y[i];
                Y[i] = 0;
                const int p2 = Lp[i] + lnz[i];
                for (int p = Lp[i]; p < p2; ++p) Y[Li[p]] -= Lx[p] * yi;
                const real lki = yi / D[i];
                D[k] -= lki * yi;
                Li[p2] = k;
                Lx[p2] = lki;
                lnz[i]++;
            }
            ORC_CHECK(D[k] != 0, "LDLT factorization failed: zero pivot.");
        }
    }
    void solve(const real* b, real* x) const {
        std::vector<real> y(n);
        for (int k = 0; k < n; ++k) y[k] = b[perm[k]];
        for (int j = 0; j < n; ++j)
            for (int p = Lp[j]; p < Lp[j + 1]; ++p) y[Li[p]] -= Lx[p] * y[j];
        for (int j = 0; j < n; ++j) y[j] /= D[j];
        for (int j = n - 1; j >= 0; --j)
            for (int p = Lp[j]; p < Lp[j + 1]; ++p) y[j] -= Lx[p] * y[Li[p]];
        for (int k = 0; k < n; ++k) x[perm[k]] = y[k];
    }
};

// Nested dissection by recursive coordinate bisection; the separator is the set of left-side vertices
// adjacent to the right side (a vertex separator of the node graph).
static void nd_order(const std::vector<int>& adjp, const std::vector<int>& adji, const std::vector<real>& X,
                     std::vector<int> nodes, std::vector<int>& out, std::vector<int>& side) {
    if (nodes.size() <= 48) {
        out.insert(out.end(), nodes.begin(), nodes.end());
        return;
    }
    real lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int v : nodes)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], X[3 * v + d]);
            hi[d] = std::max(hi[d], X[3 * v + d]);
        }
    int ax = 0;
    for (int d = 1; d < 3; ++d)
        if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
    std::vector<real> cs;
    cs.reserve(nodes.size());
    for (int v : nodes) cs.push_back(X[3 * v + ax]);
    std::nth_element(cs.begin(), cs.begin() + cs.size() / 2, cs.end());
    const real cut = cs[cs.size() / 2];
    // side: 1 = left, 2 = right, 3 = separator (tags only valid for current node set)
    for (int v : nodes) side[v] = X[3 * v + ax] < cut ? 1 : 2;
    std::vector<int> L, R, S;
    for (int v : nodes) {
        if (side[v] != 1) continue;
        bool touches = false;
        for (int p = adjp[v]; p < adjp[v + 1] && !touches; ++p)
            if (side[adji[p]] == 2) touches = true;
        if (touches) S.push_back(v);
    }
    for (int v : S) side[v] = 3;
    for (int v : nodes) {
        if (side[v] == 1) L.push_back(v);
        else if (side[v] == 2) R.push_back(v);
    }
    for (int v : nodes) side[v] = 0;
    if (L.empty() || R.empty()) {  // degenerate split: stop recursing
        out.insert(out.end(), nodes.begin(), nodes.end());
        return;
    }
    nd_order(adjp, adji, X, L, out, side);
    nd_order(adjp, adji, X, R, out, side);
    out.insert(out.end(), S.begin(), S.end());
}

// ------------------------------------------------------------------------------------------------
// The model (Deformable<3,8> / Deformable<3,4> state relevant to the AlgPhd path).
// ------------------------------------------------------------------------------------------------
struct Model {
    int n = 0, m = 0, k = 0, s = 0;
    std::vector<real> X;     // 3n rest positions
    std::vector<int> E;      // m*k connectivity
    real density = 0, vol = 0;
    std::vector<real> grad;  // per (element, sample): k x 3 gradient rows, row-major [node][dim]
    bool hex = true;
    std::map<int, real> dirichlet;
    std::vector<Energy> energies;
    std::vector<real> gravity;  // empty or 3
    // planar frictional boundary
    bool has_plane = false;
    real pn[3] = {0, 0, 1}, poff = 0;
    std::vector<int> contact_nodes;  // sorted unique
    // solver cache
    bool ready = false;
    real ready_dt = 0;
    Ldl ldl[3];
    std::vector<int> adjp, adji;
    // lambda warm start (forward_gpu.cpp:1074-1084, 1544-1545)
    std::vector<int> prev_cand;
    std::vector<real> prev_lambda;
    // forward tape of contact frames (AlgPhdReplayCache, deformable.h:336-355; pushed forward_gpu.cpp:1547-1593,
    // popped backward_gpu.cpp:716-742): active candidates (lambda > 0), their last-iteration omega and lambda
    struct TapeFrame {
        std::vector<real> q_sol;
        std::vector<int> active;
        std::vector<real> omega, lambda;
    };
    std::vector<TapeFrame> tape;
    // statistics of the last forward call
    int last_iters = 0, last_converged = 0;
    int last_filtered = 0;  // samples whose Hessian the last backward filtered

    const real* g(int e, int smp) const { return &grad[((size_t)(hex ? 0 : e) * s + smp) * k * 3]; }
    real mass() const { return density * vol; }
};

static void init_samples(Model& M) {
    if (M.hex) {
        // hex_deformable.cpp:3-51 — 8 Gauss points at dx*(1/2 +- 1/(2 sqrt 3)), trilinear shape gradients.
        const real r = real(1 / std::sqrt(3.0));
        const real dx = std::pow(M.vol, real(1) / 3);
        const real inv_dx = real(1) / dx;
        M.grad.assign(8 * 8 * 3, 0);
        for (int smp = 0; smp < 8; ++smp) {
            const int sb[3] = {(smp >> 2) & 1, (smp >> 1) & 1, smp & 1};
            real xs[3];
            for (int d = 0; d < 3; ++d) xs[d] = ((sb[d] - real(0.5)) * r + real(0.5)) * dx;
            const real nx = xs[0] * inv_dx, ny = xs[1] * inv_dx, nz = xs[2] * inv_dx;
            const real cnx = 1 - nx, cny = 1 - ny, cnz = 1 - nz;
            const real fx[2] = {cnx, nx}, fy[2] = {cny, ny}, fz[2] = {cnz, nz};
            const real gx[2] = {-inv_dx, inv_dx};
            for (int node = 0; node < 8; ++node) {
                const int a = (node >> 2) & 1, b = (node >> 1) & 1, c = node & 1;
                real* gr = &M.grad[(smp * 8 + node) * 3];
                gr[0] = gx[a] * fy[b] * fz[c];
                gr[1] = fx[a] * gx[b] * fz[c];
                gr[2] = fx[a] * fy[b] * gx[c];
            }
        }
    } else {
        // tet_deformable.cpp:3-42 — one constant-gradient sample, B = [X1-X0, X2-X0, X3-X0]^-1.
        M.grad.assign((size_t)M.m * 4 * 3, 0);
        for (int e = 0; e < M.m; ++e) {
            const int* v = &M.E[e * 4];
            M3 Bi;
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d) Bi(d, c) = M.X[3 * v[c + 1] + d] - M.X[3 * v[0] + d];
            // inverse via adjugate
            const real det = det3(Bi);
            ORC_CHECK(det != 0, "Degenerate tetrahedron.");
            M3 B;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const int i1 = (j + 1) % 3, i2 = (j + 2) % 3, j1 = (i + 1) % 3, j2 = (i + 2) % 3;
                    B(i, j) = (Bi(i1, j1) * Bi(i2, j2) - Bi(i1, j2) * Bi(i2, j1)) / det;
                }
            real* gr = &M.grad[(size_t)e * 12];
            for (int d = 0; d < 3; ++d) {
                gr[0 * 3 + d] = -B(0, d) - B(1, d) - B(2, d);
                gr[1 * 3 + d] = B(0, d);
                gr[2 * 3 + d] = B(1, d);
                gr[3 * 3 + d] = B(2, d);
            }
        }
    }
}

static real element_volume(const Model& M, int e) {
    const int* v = &M.E[e * M.k];
    auto P = [&](int i, int d) { return M.X[3 * v[i] + d]; };
    if (M.hex) {  // mesh.cpp: |det[v001-v000, v010-v000, v100-v000]|
        M3 A;
        for (int d = 0; d < 3; ++d) {
            A(d, 0) = P(1, d) - P(0, d);
            A(d, 1) = P(2, d) - P(0, d);
            A(d, 2) = P(4, d) - P(0, d);
        }
        return std::fabs(det3(A));
    }
    real a[3], b[3], c[3];
    for (int d = 0; d < 3; ++d) {
        a[d] = P(1, d) - P(0, d);
        b[d] = P(2, d) - P(0, d);
        c[d] = P(3, d) - P(0, d);
    }
    const real bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
    return std::fabs((a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2]) / 6);
}

// F(i,j) = sum_k x_k[i] * grad(k,j)
static M3 def_grad(const Model& M, int e, int smp, const real* q) {
    const real* gr = M.g(e, smp);
    const int* v = &M.E[(size_t)e * M.k];
    M3 F = zero3();
    for (int a = 0; a < M.k; ++a)
        for (int i = 0; i < 3; ++i) {
            const real x = q[3 * v[a] + i];
            for (int j = 0; j < 3; ++j) F(i, j) += x * gr[a * 3 + j];
        }
    return F;
}
// Add w * A_s^T P into per-element node forces (node a gets P grad_a^T).
static void add_At(const Model& M, int e, int smp, const M3& P, real w, real* out_e /* k*3 */) {
    const real* gr = M.g(e, smp);
    for (int a = 0; a < M.k; ++a)
        for (int i = 0; i < 3; ++i) {
            real acc = 0;
            for (int j = 0; j < 3; ++j) acc += P(i, j) * gr[a * 3 + j];
            out_e[a * 3 + i] += w * acc;
        }
}

// SetupProjectiveDynamicsSolver (deformable_projective_dynamics_forward.cpp:9-156), per-axis A_d and its LDL^T.
static void setup_solver(Model& M, real dt) {
    if (M.ready && M.ready_dt == dt) return;
    const int n = M.n;
    const real inv_h2m = M.mass() / (dt * dt);
    std::vector<std::map<int, real>> rows[3];
    for (int d = 0; d < 3; ++d) rows[d].assign(n, {});
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < n; ++i) rows[d][i][i] += M.dirichlet.count(3 * i + d) ? 1 : inv_h2m;
    for (int e = 0; e < M.m; ++e) {
        real w_e = 0;
        for (const auto& en : M.energies)
            if (en.in_set[e]) w_e += en.elem_w(e);
        const int* v = &M.E[(size_t)e * M.k];
        for (int smp = 0; smp < M.s; ++smp) {
            const real* gr = M.g(e, smp);
            for (int a = 0; a < M.k; ++a)
                for (int b = 0; b < M.k; ++b) {
                    real gg = 0;
                    for (int j = 0; j < 3; ++j) gg += gr[a * 3 + j] * gr[b * 3 + j];
                    const real val = gg * w_e * M.vol / M.s;
                    for (int d = 0; d < 3; ++d) {
                        if (M.dirichlet.count(3 * v[a] + d) || M.dirichlet.count(3 * v[b] + d)) continue;
                        rows[d][v[a]][v[b]] += val;
                    }
                }
        }
    }
    // node adjacency (pattern of axis 0 plus element coupling) for the ordering
    std::vector<std::set<int>> adj(n);
    for (int e = 0; e < M.m; ++e)
        for (int a = 0; a < M.k; ++a)
            for (int b = 0; b < M.k; ++b)
                if (a != b) adj[M.E[(size_t)e * M.k + a]].insert(M.E[(size_t)e * M.k + b]);
    M.adjp.assign(n + 1, 0);
    M.adji.clear();
    for (int i = 0; i < n; ++i) {
        M.adji.insert(M.adji.end(), adj[i].begin(), adj[i].end());
        M.adjp[i + 1] = (int)M.adji.size();
    }
    std::vector<int> order, side(n, 0), all(n);
    std::iota(all.begin(), all.end(), 0);
    nd_order(M.adjp, M.adji, M.X, all, order, side);
    ORC_CHECK((int)order.size() == n, "ordering lost vertices");
    for (int d = 0; d < 3; ++d) {
        std::vector<int> Ap(n + 1, 0), Ai;
        std::vector<real> Ax;
        for (int i = 0; i < n; ++i) {
            for (const auto& kv : rows[d][i]) {
                Ai.push_back(kv.first);
                Ax.push_back(kv.second);
            }
            Ap[i + 1] = (int)Ai.size();
        }
        M.ldl[d].factor(n, Ap, Ai, Ax, order);
    }
    M.ready = true;
    M.ready_dt = dt;
}

// A_d^-1 applied to a node-major interleaved 3n vector, axis by axis.
static void apply_ainv(const Model& M, const real* b, real* x) {
    const int n = M.n;
#pragma omp parallel for
    for (int d = 0; d < 3; ++d) {
        std::vector<real> bd(n), xd(n);
        for (int i = 0; i < n; ++i) bd[i] = b[3 * i + d];
        M.ldl[d].solve(bd.data(), xd.data());
        for (int i = 0; i < n; ++i) x[3 * i + d] = xd[i];
    }
}

// ProjectiveDynamicsLocalStep (deformable_projective_dynamics_forward.cpp:186-292):
// rhs = sum_e w_e (vol/s) sum_s A_s^T (Bp(F_s) - F_bound_s).
static void local_step(const Model& M, const real* q, real* rhs) {
    const int n3 = 3 * M.n;
    std::vector<real> qb(n3, 0);
    for (const auto& kv : M.dirichlet) qb[kv.first] = kv.second;
    std::vector<real> per((size_t)M.m * M.k * 3, 0);
    for (const auto& en : M.energies) {
#pragma omp parallel for schedule(static)
        for (int e = 0; e < M.m; ++e) {
            if (!en.in_set[e]) continue;
            const real w = en.elem_w(e) * M.vol / M.s;
            for (int smp = 0; smp < M.s; ++smp) {
                const M3 F = def_grad(M, e, smp, q);
                const M3 Fb = def_grad(M, e, smp, qb.data());
                const SvdData d = make_svd(F);
                const M3 Bp = project(en, d);
                M3 diff;
                for (int i = 0; i < 9; ++i) diff.a[i] = Bp.a[i] - Fb.a[i];
                add_At(M, e, smp, diff, w, &per[(size_t)e * M.k * 3]);
            }
        }
    }
    std::fill(rhs, rhs + n3, 0.0);
    for (int e = 0; e < M.m; ++e)
        for (int a = 0; a < M.k; ++a)
            for (int i = 0; i < 3; ++i) rhs[3 * M.E[(size_t)e * M.k + a] + i] += per[((size_t)e * M.k + a) * 3 + i];
}

static real norm(const std::vector<real>& v) {
    real s = 0;
    for (real x : v) s += x * x;
    return std::sqrt(s);
}

struct Options {
    int max_pd_iter = 0;
    real abs_tol = 0, rel_tol = 0;
    int aa_window = 5;
    real friction_mu = 0, restitution = 0, contact_slop = 1e-8;
    real clip = 1e6;
    int mean_stiffness_bwd = 0;  // reference backward semantics: mean stiffness in K_pd
    int cascade_cap = 1;
    int verbose = 0;
    // contact-aware material adjoint (backward_gpu.cpp:937-1208)
    int skip_woodbury = 0, skip_material_grad = 0;
    real tangent_lambda_min = 1e-8, rhs_prune_rel = 1e-3, rhs_prune_abs = 1e-12;
    int basis_topk = 0, wt_max_iter = 120;
    int eigen_filter = 0;  // 0 off, 1 clamp at 0, 2 absolute value (deformable_newton_forward.cpp:394-434)
};

// Type-II Anderson acceleration with the reference's regularisation and restart rule
// (forward_gpu.cpp:1346-1379; backward_gpu.cpp:825-859).
struct Anderson {
    int window;
    std::vector<std::vector<real>> xh, gh;
    // returns true when the candidate was accepted and written to x_out
    bool step(const std::vector<real>& x_prev, const std::vector<real>& gk, std::vector<real>& x_out) {
        bool accepted = false;
        if (window <= 0) return false;
        xh.push_back(x_prev);
        gh.push_back(gk);
        const int m = (int)gh.size() - 1;
        if (m >= 1) {
            const size_t N = gk.size();
            std::vector<real> GtG(m * m, 0), rhs(m, 0);
            real fro = 0;
            std::vector<std::vector<real>> dG(m, std::vector<real>(N)), dQ(m, std::vector<real>(N));
            for (int i = 0; i < m; ++i)
                for (size_t r = 0; r < N; ++r) {
                    dG[i][r] = gh[i + 1][r] - gh[i][r];
                    dQ[i][r] = xh[i + 1][r] - xh[i][r];
                }
            for (int i = 0; i < m; ++i) {
                for (int j = 0; j < m; ++j) {
                    real s = 0;
                    for (size_t r = 0; r < N; ++r) s += dG[i][r] * dG[j][r];
                    GtG[i * m + j] = s;
                }
                real s = 0;
                for (size_t r = 0; r < N; ++r) s += dG[i][r] * gk[r];
                rhs[i] = s;
                fro += GtG[i * m + i];
            }
            const real reg = std::max(1e-6 * fro / std::max(m, 1), 1e-12);
            for (int i = 0; i < m; ++i) GtG[i * m + i] += reg;
            dense_solve(m, GtG, rhs);
            real gn = 0;
            for (int i = 0; i < m; ++i) gn += rhs[i] * rhs[i];
            gn = std::sqrt(gn);
            if (gn >= 10.0) {
                xh.clear();
                gh.clear();
            } else {
                x_out.resize(N);
                for (size_t r = 0; r < N; ++r) {
                    real c = x_prev[r] + gk[r];
                    for (int i = 0; i < m; ++i) c -= (dQ[i][r] + dG[i][r]) * rhs[i];
                    x_out[r] = c;
                }
                accepted = true;
            }
        }
        while ((int)xh.size() > window) {
            xh.erase(xh.begin());
            gh.erase(gh.begin());
        }
        return accepted;
    }
};

static std::vector<real> q_tilde(const Model& M, const real* q, const real* v, const real* f_ext, real h) {
    const int n3 = 3 * M.n;
    const real h2m = h * h / M.mass();
    std::vector<real> qt(n3);
    for (int i = 0; i < n3; ++i) {
        const real fs = M.gravity.empty() ? 0 : M.mass() * M.gravity[i % 3];
        qt[i] = q[i] + h * v[i] + h2m * f_ext[i] + h2m * fs;
    }
    return qt;
}

// ForwardProjectiveDynamicsAlgPhd (forward_gpu.cpp:387-1594), planar frictional boundary only.
static void forward(Model& M, const real* q, const real* v, const real* f_ext, real h, const Options& opt,
                    real* q_next, real* v_next, std::vector<int>& active) {
    setup_solver(M, h);
    const int n = M.n, n3 = 3 * n;
    const real inv_h2m = M.mass() / (h * h);
    const std::vector<real> qt = q_tilde(M, q, v, f_ext, h);
    // contact candidates: every listed boundary node (planar: no prefilter), frames from GetLocalFrame
    const std::vector<int>& cand = M.has_plane ? M.contact_nodes : std::vector<int>();
    const int K = (int)cand.size();
    real t1[3] = {0, 0, 0}, t2[3] = {0, 0, 0};
    const real* nrm = M.pn;
    if (K > 0) {  // planar_frictional_boundary.cpp:25-40
        real best = -1;
        for (int i = 0; i < 3; ++i) {
            real e[3] = {0, 0, 0};
            e[i] = 1;
            const real x[3] = {nrm[1] * e[2] - nrm[2] * e[1], nrm[2] * e[0] - nrm[0] * e[2], nrm[0] * e[1] - nrm[1] * e[0]};
            const real sq = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (sq > best) {
                best = sq;
                t1[0] = x[0]; t1[1] = x[1]; t1[2] = x[2];
            }
        }
        const real l1 = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
        for (int d = 0; d < 3; ++d) t1[d] /= l1;
        t2[0] = nrm[1] * t1[2] - nrm[2] * t1[1];
        t2[1] = nrm[2] * t1[0] - nrm[0] * t1[2];
        t2[2] = nrm[0] * t1[1] - nrm[1] * t1[0];
        const real l2 = std::sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
        for (int d = 0; d < 3; ++d) t2[d] /= l2;
    }
    // Delassus columns Ainv_cols[d][ci] = A_d^-1 (n_d e_ci) and W
    std::vector<std::vector<real>> Acol[3], At1[3], At2[3];
    std::vector<real> W((size_t)K * K, 0);
    const bool fric = K > 0 && opt.friction_mu > 0;
    for (int d = 0; d < 3; ++d) {
        Acol[d].assign(K, {});
        if (fric) { At1[d].assign(K, {}); At2[d].assign(K, {}); }
    }
#pragma omp parallel for schedule(dynamic)
    for (int job = 0; job < 3 * K; ++job) {
        const int d = job / K, ci = job % K;
        std::vector<real> rhs(n, 0), x(n);
        rhs[cand[ci]] = nrm[d];
        M.ldl[d].solve(rhs.data(), x.data());
        Acol[d][ci] = x;
        if (fric) {
            rhs[cand[ci]] = t1[d];
            M.ldl[d].solve(rhs.data(), x.data());
            At1[d][ci] = x;
            rhs[cand[ci]] = t2[d];
            M.ldl[d].solve(rhs.data(), x.data());
            At2[d][ci] = x;
        }
    }
    for (int ci = 0; ci < K; ++ci)
        for (int cj = ci; cj < K; ++cj) {
            real w = 0;
            for (int d = 0; d < 3; ++d) w += nrm[d] * Acol[d][ci][cand[cj]];
            W[(size_t)ci * K + cj] = W[(size_t)cj * K + ci] = w;
        }
    std::vector<real> Wtt(4 * (size_t)K, 0);
    if (fric)
        for (int ci = 0; ci < K; ++ci) {
            real w11 = 0, w12 = 0, w22 = 0;
            for (int d = 0; d < 3; ++d) {
                w11 += t1[d] * At1[d][ci][cand[ci]];
                w12 += t1[d] * At2[d][ci][cand[ci]];
                w22 += t2[d] * At2[d][ci][cand[ci]];
            }
            Wtt[4 * ci + 0] = w11; Wtt[4 * ci + 1] = w12; Wtt[4 * ci + 2] = w12; Wtt[4 * ci + 3] = w22;
        }
    std::vector<real> rp(K);
    for (int ci = 0; ci < K; ++ci) rp[ci] = std::max(h * h * W[(size_t)ci * K + ci], 1e-10);
    std::vector<real> lam(K, 0), lt1(K, 0), lt2(K, 0);
    if (!M.prev_cand.empty() && M.prev_lambda.size() == M.prev_cand.size()) {
        std::unordered_map<int, int> pi;
        for (size_t i = 0; i < M.prev_cand.size(); ++i) pi[M.prev_cand[i]] = (int)i;
        for (int ci = 0; ci < K; ++ci) {
            auto it = pi.find(cand[ci]);
            if (it != pi.end()) lam[ci] = M.prev_lambda[it->second];
        }
    }
    std::vector<real> qs(q, q + n3), qp(q, q + n3), prev_rhs(n3, 0), pd(n3), b(n3), x(n3);
    Anderson aa{opt.aa_window, {}, {}};
    bool converged = false;
    int iters = 0;
    std::vector<real> om_last(K, 0);
    for (int it = 0; it < opt.max_pd_iter; ++it) {
        local_step(M, qs.data(), pd.data());
        for (int i = 0; i < n3; ++i) b[i] = inv_h2m * qt[i] + pd[i];
        qp = qs;
        if (K > 0) {
            std::vector<real> dn(K), om(K), Ed(K);
            for (int ci = 0; ci < K; ++ci) {
                const int node = cand[ci];
                dn[ci] = nrm[0] * qs[3 * node] + nrm[1] * qs[3 * node + 1] + nrm[2] * qs[3 * node + 2] + M.poff;
                real den = std::sqrt(dn[ci] * dn[ci] + rp[ci] * rp[ci] * lam[ci] * lam[ci]);
                if (den < 1e-14) den = 1e-14;
                om[ci] = 1.0 - dn[ci] / den;
                Ed[ci] = (1.0 - rp[ci] * lam[ci] / den) * rp[ci];
            }
            om_last = om;
            std::vector<real> Ms((size_t)K * K);
            for (int i = 0; i < K; ++i)
                for (int j = 0; j < K; ++j) Ms[(size_t)i * K + j] = om[i] * W[(size_t)i * K + j] * om[j];
            for (int i = 0; i < K; ++i) Ms[(size_t)i * K + i] += Ed[i];
            std::vector<real> hv(K);
            for (int ci = 0; ci < K; ++ci) {
                const real dj = dn[ci], lj = lam[ci], rj = rp[ci];
                real den = std::sqrt(dj * dj + rj * rj * lj * lj);
                if (den < 1e-14) den = 1e-14;
                const real phi = dj + rj * lj - den;
                const int node = cand[ci];
                const real Hq = nrm[0] * qs[3 * node] + nrm[1] * qs[3 * node + 1] + nrm[2] * qs[3 * node + 2];
                hv[ci] = -phi + om[ci] * Hq;
            }
            apply_ainv(M, b.data(), x.data());  // Ainv_b (node-major)
            std::vector<real> Ag(x);
            for (int ci = 0; ci < K; ++ci)
                for (int d = 0; d < 3; ++d) {
                    const real c0 = om[ci] * lam[ci];
                    const real c1 = fric ? lt1[ci] : 0, c2 = fric ? lt2[ci] : 0;
                    const std::vector<real>& col = Acol[d][ci];
                    for (int nd = 0; nd < n; ++nd) {
                        real add = c0 * col[nd];
                        if (fric) add += c1 * At1[d][ci][nd] + c2 * At2[d][ci][nd];
                        Ag[3 * nd + d] += add;
                    }
                }
            std::vector<real> rc(K);
            for (int ci = 0; ci < K; ++ci) {
                const int node = cand[ci];
                real val = 0;
                for (int d = 0; d < 3; ++d) val += nrm[d] * Ag[3 * node + d];
                rc[ci] = hv[ci] - om[ci] * val;
            }
            dense_solve(K, Ms, rc);
            for (int ci = 0; ci < K; ++ci) lam[ci] = std::min(std::max(lam[ci] + rc[ci], 0.0), 1e8);
            std::vector<real> oln(K);
            for (int ci = 0; ci < K; ++ci) oln[ci] = om[ci] * lam[ci];
            if (fric) {  // Coulomb cone (forward_gpu.cpp:1255-1302)
                for (int ci = 0; ci < K; ++ci) {
                    if (lam[ci] <= 0.0) { lt1[ci] = lt2[ci] = 0; continue; }
                    const int node = cand[ci];
                    real qn[3];
                    for (int d = 0; d < 3; ++d) {
                        qn[d] = x[3 * node + d];
                        for (int cj = 0; cj < K; ++cj) qn[d] += oln[cj] * Acol[d][cj][node];
                    }
                    real st[3];
                    for (int d = 0; d < 3; ++d) st[d] = qn[d] - q[3 * node + d];
                    const real sn = st[0] * nrm[0] + st[1] * nrm[1] + st[2] * nrm[2];
                    real ut[3];
                    for (int d = 0; d < 3; ++d) ut[d] = st[d] - sn * nrm[d];
                    const real u1 = ut[0] * t1[0] + ut[1] * t1[1] + ut[2] * t1[2];
                    const real u2 = ut[0] * t2[0] + ut[1] * t2[1] + ut[2] * t2[2];
                    const real* Wt = &Wtt[4 * ci];
                    const real det = Wt[0] * Wt[3] - Wt[1] * Wt[2];
                    real s1 = 0, s2 = 0;
                    if (std::fabs(det) > 1e-20) {
                        s1 = (Wt[3] * -u1 - Wt[1] * -u2) / det;
                        s2 = (-Wt[2] * -u1 + Wt[0] * -u2) / det;
                    }
                    const real cone = opt.friction_mu * lam[ci];
                    if (std::sqrt(s1 * s1 + s2 * s2) <= cone + 1e-14) {
                        lt1[ci] = s1; lt2[ci] = s2;
                    } else {
                        const real um = std::sqrt(u1 * u1 + u2 * u2);
                        if (um > 1e-14) { lt1[ci] = -cone * u1 / um; lt2[ci] = -cone * u2 / um; }
                        else lt1[ci] = lt2[ci] = 0;
                    }
                }
            }
            for (int nd = 0; nd < n; ++nd)
                for (int d = 0; d < 3; ++d) qs[3 * nd + d] = x[3 * nd + d];
            for (int ci = 0; ci < K; ++ci)
                for (int d = 0; d < 3; ++d) {
                    const std::vector<real>& col = Acol[d][ci];
                    for (int nd = 0; nd < n; ++nd) {
                        real add = oln[ci] * col[nd];
                        if (fric) add += lt1[ci] * At1[d][ci][nd] + lt2[ci] * At2[d][ci][nd];
                        qs[3 * nd + d] += add;
                    }
                }
        } else {
            std::vector<real> bb(b);
            for (const auto& kv : M.dirichlet) bb[kv.first] = 0;
            apply_ainv(M, bb.data(), qs.data());
        }
        ++iters;
        for (const auto& kv : M.dirichlet) qs[kv.first] = kv.second;
        {
            std::vector<real> gk(n3), cand_q;
            for (int i = 0; i < n3; ++i) gk[i] = qs[i] - qp[i];
            if (aa.step(qp, gk, cand_q)) {
                qs = cand_q;
                for (const auto& kv : M.dirichlet) qs[kv.first] = kv.second;
            }
        }
        std::vector<real> dq(n3), drhs(n3);
        for (int i = 0; i < n3; ++i) { dq[i] = qs[i] - qp[i]; drhs[i] = pd[i] - prev_rhs[i]; }
        const real abs_err = norm(dq), rn = norm(qp), pc = norm(drhs), pr = norm(prev_rhs);
        prev_rhs = pd;
        if (opt.verbose > 1) std::printf("oracle PD iter %d dq=%.3e (tol %.3e) drhs=%.3e (tol %.3e)\n", it, abs_err, opt.rel_tol * rn + opt.abs_tol, pc, opt.rel_tol * pr + opt.abs_tol);
        if (it > 0 && abs_err <= opt.rel_tol * rn + opt.abs_tol && pc <= opt.rel_tol * pr + opt.abs_tol) {
            converged = true;
            break;
        }
    }
    M.last_iters = iters;
    M.last_converged = converged ? 1 : 0;
    // restitution (forward_gpu.cpp:1483-1531), planar boundary
    if (opt.restitution > 0) {
        for (int ci = 0; ci < K; ++ci) {
            if (lam[ci] <= 0) continue;
            const int node = cand[ci];
            const real sd = nrm[0] * qs[3 * node] + nrm[1] * qs[3 * node + 1] + nrm[2] * qs[3 * node + 2] + M.poff;
            if (sd > opt.contact_slop) continue;
            const real vin = v[3 * node] * nrm[0] + v[3 * node + 1] * nrm[1] + v[3 * node + 2] * nrm[2];
            if (vin < 0) {
                real vo = 0;
                for (int d = 0; d < 3; ++d) vo += (qs[3 * node + d] - q[3 * node + d]) / h * nrm[d];
                const real dv = -opt.restitution * vin - vo;
                if (dv > 0)
                    for (int d = 0; d < 3; ++d) qs[3 * node + d] += h * dv * nrm[d];
            }
        }
    }
    for (int i = 0; i < n3; ++i) {
        q_next[i] = qs[i];
        v_next[i] = (qs[i] - q[i]) / h;
    }
    active.clear();
    for (int ci = 0; ci < K; ++ci)
        if (lam[ci] > 0) active.push_back(cand[ci]);
    M.prev_cand = cand;
    M.prev_lambda = lam;
    if (K > 0) {
        Model::TapeFrame fr;
        fr.q_sol.assign(q_next, q_next + n3);
        for (int ci = 0; ci < K; ++ci)
            if (lam[ci] > 0) {
                fr.active.push_back(cand[ci]);
                fr.omega.push_back(om_last[ci]);
                fr.lambda.push_back(lam[ci]);
            }
        M.tape.push_back(std::move(fr));
        if (M.tape.size() > 8192) M.tape.erase(M.tape.begin());
    }
}

// K_pd u: sum_e (vol/s) sum_s A_s^T [w dBp/dF](A_s u)  (deformable_projective_dynamics_backward.cpp:10-139)
static void apply_kpd(const Model& M, const std::vector<std::vector<SvdData>>& svd, const real* u, real* out,
                      bool mean_w) {
    const int n3 = 3 * M.n;
    std::vector<real> per((size_t)M.m * M.k * 3, 0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < M.m; ++e) {
        for (int smp = 0; smp < M.s; ++smp) {
            const M3 dF = def_grad(M, e, smp, u);
            M3 acc = zero3();
            for (const auto& en : M.energies) {
                if (!en.in_set[e]) continue;
                const real w = (mean_w ? en.w_mean : en.elem_w(e)) * M.vol / M.s;
                const M3 dB = project_diff(en, svd[e][smp], dF);
                for (int i = 0; i < 9; ++i) acc.a[i] += w * dB.a[i];
            }
            add_At(M, e, smp, acc, 1.0, &per[(size_t)e * M.k * 3]);
        }
    }
    std::fill(out, out + n3, 0.0);
    for (int e = 0; e < M.m; ++e)
        for (int a = 0; a < M.k; ++a)
            for (int i = 0; i < 3; ++i) out[3 * M.E[(size_t)e * M.k + a] + i] += per[((size_t)e * M.k + a) * 3 + i];
}

// Symmetric eigen-decomposition A = Q diag(A') Q^T by cyclic Jacobi rotations (n x n, row-major, in place).
static void sym_eig(int n, std::vector<real>& A, std::vector<real>& Q) {
    Q.assign((size_t)n * n, 0);
    for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1;
    for (int sweep = 0; sweep < 100; ++sweep) {
        real off = 0, tot = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const real a = A[(size_t)i * n + j];
                tot += a * a;
                if (i != j) off += a * a;
            }
        if (off <= 1e-32 * tot) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const real apq = A[(size_t)p * n + q];
                if (apq == 0) continue;
                const real theta = 0.5 * std::atan2(2 * apq, A[(size_t)q * n + q] - A[(size_t)p * n + p]);
                const real c = std::cos(theta), s = std::sin(theta);
                for (int k = 0; k < n; ++k) {
                    const real akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - s * akq;
                    A[(size_t)k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const real apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - s * aqk;
                    A[(size_t)q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const real qkp = Q[(size_t)k * n + p], qkq = Q[(size_t)k * n + q];
                    Q[(size_t)k * n + p] = c * qkp - s * qkq;
                    Q[(size_t)k * n + q] = s * qkp + c * qkq;
                }
            }
    }
}

// Per-sample 9x9 Jacobian of the weighted projections, J[col * 9 + i] = d(sum_en w Bp)_i / dF_col, with the
// state-adaptive eigen filter of H = (sum w) I - sym(J) applied when `filter` is set (the diagonal-dominance
// test and eigenvalue clamp / absolute value of ProjectedNewtonMatrix, deformable_newton_forward.cpp:394-434).
static int build_filtered_jacobians(const Model& M, const std::vector<std::vector<SvdData>>& svd, bool mean_w,
                                    int filter, std::vector<real>& Jall) {
    Jall.assign((size_t)M.m * M.s * 81, 0);
    int nfilt = 0;
#pragma omp parallel for schedule(static) reduction(+ : nfilt)
    for (int e = 0; e < M.m; ++e)
        for (int smp = 0; smp < M.s; ++smp) {
            real* J = &Jall[((size_t)e * M.s + smp) * 81];
            real wsum = 0;
            for (const auto& en : M.energies)
                if (en.in_set[e]) wsum += (mean_w ? en.w_mean : en.elem_w(e)) * M.vol / M.s;
            for (int col = 0; col < 9; ++col) {
                M3 dF = zero3();
                dF.a[col] = 1;
                for (const auto& en : M.energies) {
                    if (!en.in_set[e]) continue;
                    const real w = (mean_w ? en.w_mean : en.elem_w(e)) * M.vol / M.s;
                    const M3 dB = project_diff(en, svd[e][smp], dF);
                    for (int i = 0; i < 9; ++i) J[col * 9 + i] += w * dB.a[i];
                }
            }
            if (!filter) continue;
            std::vector<real> H(81), Q;
            for (int i = 0; i < 9; ++i)
                for (int j = 0; j < 9; ++j) H[i * 9 + j] = (i == j ? wsum : 0.0) - 0.5 * (J[j * 9 + i] + J[i * 9 + j]);
            bool dd = true;
            for (int i = 0; i < 9 && dd; ++i) {
                real off = 0;
                for (int j = 0; j < 9; ++j)
                    if (j != i) off += std::fabs(H[i * 9 + j]);
                if (std::fabs(H[i * 9 + i]) < off + 1e-5) dd = false;
            }
            if (dd) continue;
            sym_eig(9, H, Q);
            real lam[9];
            for (int k = 0; k < 9; ++k) lam[k] = filter == 1 ? std::max(H[k * 9 + k], real(0)) : std::fabs(H[k * 9 + k]);
            for (int i = 0; i < 9; ++i)
                for (int j = 0; j < 9; ++j) {
                    real h = 0;
                    for (int k = 0; k < 9; ++k) h += Q[i * 9 + k] * lam[k] * Q[j * 9 + k];
                    J[j * 9 + i] = (i == j ? wsum : 0.0) - h;
                }
            ++nfilt;
        }
    return nfilt;
}

// K_pd u from the per-sample Jacobians of build_filtered_jacobians.
static void apply_kpd_J(const Model& M, const std::vector<real>& Jall, const real* u, real* out) {
    const int n3 = 3 * M.n;
    std::vector<real> per((size_t)M.m * M.k * 3, 0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < M.m; ++e)
        for (int smp = 0; smp < M.s; ++smp) {
            const M3 dF = def_grad(M, e, smp, u);
            const real* J = &Jall[((size_t)e * M.s + smp) * 81];
            M3 P = zero3();
            for (int col = 0; col < 9; ++col)
                for (int i = 0; i < 9; ++i) P.a[i] += J[col * 9 + i] * dF.a[col];
            add_At(M, e, smp, P, 1.0, &per[(size_t)e * M.k * 3]);
        }
    std::fill(out, out + n3, 0.0);
    for (int e = 0; e < M.m; ++e)
        for (int a = 0; a < M.k; ++a)
            for (int i = 0; i < 3; ++i) out[3 * M.E[(size_t)e * M.k + a] + i] += per[((size_t)e * M.k + a) * 3 + i];
}

static int count_params(const Model& M) {
    int t = 0;
    for (const auto& en : M.energies) t += (int)en.params.size();
    return t;
}

// BackwardProjectiveDynamicsAlgPhd (backward_gpu.cpp:648-1250): backbone adjoint (A - K_pd) mu = g_bar by the
// AA fixed point mu <- clip(A^-1 (g_bar + K_pd mu)), downstream routing, and parameter gradients.
// Parameter gradients are returned for the exact parameter vector of each AddPdEnergy call
// (1 scalar, m per-element values, or 2m interleaved [mu_e, la_e] for pd_neohookean), with z_q = mu.
static void backward(Model& M, const real* q, const real* v, const real* f_ext, real h, const real* q_next,
                     const real* dl_dq_next, const real* dl_dv_next, const Options& opt, real* dl_dq, real* dl_dv,
                     real* dl_df, real* dl_dmat_w, real* dl_dparams, real* dl_dstate_p, int* iters_out) {
    setup_solver(M, h);
    const int n3 = 3 * M.n;
    const real inv_h2m = M.mass() / (h * h), h2m = h * h / M.mass();
    std::vector<real> gbar(n3);
    for (int i = 0; i < n3; ++i) {
        dl_dq[i] = -dl_dv_next[i] / h;
        dl_dv[i] = 0;
        dl_df[i] = 0;
        gbar[i] = dl_dq_next[i] + dl_dv_next[i] / h;
    }
    std::vector<std::vector<SvdData>> svd(M.m, std::vector<SvdData>(M.s));
#pragma omp parallel for
    for (int e = 0; e < M.m; ++e)
        for (int smp = 0; smp < M.s; ++smp) svd[e][smp] = make_svd(def_grad(M, e, smp, q_next));
    std::vector<real> Jf;
    int nfilt = 0;
    if (opt.eigen_filter) nfilt = build_filtered_jacobians(M, svd, opt.mean_stiffness_bwd != 0, opt.eigen_filter, Jf);
    M.last_filtered = nfilt;
    auto kpd_apply = [&](const real* u, real* out) {
        if (opt.eigen_filter) apply_kpd_J(M, Jf, u, out);
        else apply_kpd(M, svd, u, out, opt.mean_stiffness_bwd != 0);
    };
    std::vector<real> mu(n3, 0), kpd(n3), rhs(n3), nx(n3);
    auto clip = [&](std::vector<real>& x) {
        for (auto& val : x)
            if (!std::isfinite(val)) val = 0;
        const real nn = norm(x);
        if (opt.clip > 0 && std::isfinite(nn) && nn > opt.clip)
            for (auto& val : x) val *= opt.clip / nn;
    };
    Anderson aa{opt.aa_window, {}, {}};
    int iters = 0;
    for (int it = 0; it < opt.max_pd_iter; ++it) {
        kpd_apply(mu.data(), kpd.data());
        for (int i = 0; i < n3; ++i) rhs[i] = gbar[i] + kpd[i];
        apply_ainv(M, rhs.data(), nx.data());
        for (const auto& kv : M.dirichlet) nx[kv.first] = 0;
        clip(nx);
        std::vector<real> dd(n3);
        for (int i = 0; i < n3; ++i) dd[i] = nx[i] - mu[i];
        const real err = norm(dd);
        std::vector<real> cand_x;
        if (aa.step(mu, dd, cand_x)) {
            nx = cand_x;
            clip(nx);
        }
        mu = nx;
        iters = it + 1;
        if (it > 0 && err < opt.rel_tol * norm(mu) + opt.abs_tol) break;
    }
    if (iters_out) *iters_out = iters;
    const bool diverged = opt.clip > 0 && norm(mu) >= opt.clip * 0.999;
    const int np = count_params(M);
    for (size_t k = 0; k < M.energies.size(); ++k) dl_dmat_w[k] = 0;
    for (int i = 0; i < np; ++i) dl_dparams[i] = 0;
    for (int d = 0; d < 3; ++d) dl_dstate_p[d] = 0;
    if (diverged) return;
    std::vector<real> inj(n3);
    for (int i = 0; i < n3; ++i) inj[i] = inv_h2m * mu[i];
    if (opt.cascade_cap) {
        const real cap = norm(gbar) + 1.0, in = norm(inj);
        if (in > cap)
            for (auto& val : inj) val *= cap / in;
    }
    for (int i = 0; i < n3; ++i) {
        dl_dq[i] += inj[i];
        dl_df[i] += h2m * inj[i];
        dl_dv[i] += h * inj[i];
    }
    if (!M.gravity.empty())
        for (int i = 0; i < n3; ++i) dl_dstate_p[i % 3] += h2m * inj[i] * M.mass();
    if (opt.skip_material_grad) return;
    // Contact-aware adjoint for the material gradients (backward_gpu.cpp:937-1208):
    // z_q = mu - W_T G_T^-1 (J_basis mu), W_T[k] = (A - K_pd)^-1 j_k by the Anderson fixed point.
    std::vector<real> zq = mu;
    Model::TapeFrame fr;
    bool have = false;
    if (M.has_plane) {
        if (!M.tape.empty()) {  // tape pop (backward_gpu.cpp:716-742)
            const Model::TapeFrame& tail = M.tape.back();
            std::vector<real> dd(n3);
            for (int i = 0; i < n3; ++i) dd[i] = tail.q_sol[i] - q_next[i];
            const real denom = std::max<real>(1, std::max(norm(tail.q_sol), norm(std::vector<real>(q_next, q_next + n3))));
            const real rel = norm(dd) / denom;
            if (rel <= 1e-8) {
                fr = tail;
                M.tape.pop_back();
                have = true;
            } else if (rel > 1e-6) {
                M.tape.clear();
            }
        }
        if (!have) {  // replay: the forward step again from (q, v, f_ext), lambda warm start preserved
            const std::vector<int> pc = M.prev_cand;
            const std::vector<real> pl = M.prev_lambda;
            std::vector<real> tq(n3), tv(n3);
            std::vector<int> act;
            forward(M, q, v, f_ext, h, opt, tq.data(), tv.data(), act);
            fr = M.tape.back();
            M.tape.pop_back();
            M.prev_cand = pc;
            M.prev_lambda = pl;
            have = true;
        }
    }
    if (have && !opt.skip_woodbury && !fr.active.empty()) {
        const real* nrm = M.pn;
        // tangent basis of the backward (backward_gpu.cpp:958-981): axis of the smallest |n_d|
        int axis = 0;
        for (int d = 1; d < 3; ++d)
            if (std::fabs(nrm[d]) < std::fabs(nrm[axis])) axis = d;
        real e[3] = {0, 0, 0};
        e[axis] = 1;
        const real ne = nrm[0] * e[0] + nrm[1] * e[1] + nrm[2] * e[2];
        real t1[3] = {e[0] - ne * nrm[0], e[1] - ne * nrm[1], e[2] - ne * nrm[2]};
        real l1 = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
        if (l1 > 1e-12) for (auto& x : t1) x /= l1;
        else { t1[0] = 1; t1[1] = 0; t1[2] = 0; }
        real t2[3] = {nrm[1] * t1[2] - nrm[2] * t1[1], nrm[2] * t1[0] - nrm[0] * t1[2], nrm[0] * t1[1] - nrm[1] * t1[0]};
        const real l2 = std::sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
        if (l2 > 1e-12) for (auto& x : t2) x /= l2;
        else { t2[0] = 0; t2[1] = 1; t2[2] = 0; }
        const bool tang = opt.friction_mu > 0;
        struct Basis { int ai, b; };
        std::vector<Basis> full;
        for (int ai = 0; ai < (int)fr.active.size(); ++ai) {
            if (fr.omega[ai] < 0.5) continue;
            full.push_back({ai, 0});
            if (tang && fr.lambda[ai] > opt.tangent_lambda_min) {
                full.push_back({ai, 1});
                full.push_back({ai, 2});
            }
        }
        auto basis_dir = [&](const Basis& bc, real* dir, real& scale) {
            const real* src = bc.b == 0 ? nrm : (bc.b == 1 ? t1 : t2);
            for (int d = 0; d < 3; ++d) dir[d] = src[d];
            scale = bc.b == 0 ? fr.omega[bc.ai] : 1.0;
        };
        auto project = [&](const Basis& bc, const std::vector<real>& x) {
            real dir[3], sc;
            basis_dir(bc, dir, sc);
            const int node = fr.active[bc.ai];
            return sc * (dir[0] * x[3 * node] + dir[1] * x[3 * node + 1] + dir[2] * x[3 * node + 2]);
        };
        const int nbf = (int)full.size();
        std::vector<real> rfull(nbf);
        real rmax = 0;
        for (int i = 0; i < nbf; ++i) {
            rfull[i] = project(full[i], zq);
            rmax = std::max(rmax, std::fabs(rfull[i]));
        }
        const real gate = std::max(opt.rhs_prune_abs, opt.rhs_prune_rel * rmax);
        std::vector<int> sel;
        for (int i = 0; i < nbf; ++i)
            if (std::fabs(rfull[i]) >= gate) sel.push_back(i);
        if (opt.basis_topk > 0 && (int)sel.size() > opt.basis_topk) {
            std::nth_element(sel.begin(), sel.begin() + opt.basis_topk, sel.end(),
                             [&](int a, int b) { return std::fabs(rfull[a]) > std::fabs(rfull[b]); });
            sel.resize(opt.basis_topk);
        }
        const int nb = (int)sel.size();
        if (nb > 0) {
            const int wmax = std::min(opt.max_pd_iter, std::max(1, opt.wt_max_iter));
            std::vector<std::vector<real>> WT(nb);
            for (int k = 0; k < nb; ++k) {
                const Basis bc = full[sel[k]];
                real dir[3], sc;
                basis_dir(bc, dir, sc);
                std::vector<real> j(n3, 0), sv(n3, 0), kp(n3), rh(n3), sn(n3);
                const int node = fr.active[bc.ai];
                for (int d = 0; d < 3; ++d) j[3 * node + d] = sc * dir[d];
                Anderson wa{opt.aa_window, {}, {}};
                for (int it = 0; it < wmax; ++it) {
                    kpd_apply(sv.data(), kp.data());
                    for (int i = 0; i < n3; ++i) rh[i] = j[i] + kp[i];
                    apply_ainv(M, rh.data(), sn.data());
                    for (const auto& kv : M.dirichlet) sn[kv.first] = 0;
                    clip(sn);
                    std::vector<real> dd(n3);
                    for (int i = 0; i < n3; ++i) dd[i] = sn[i] - sv[i];
                    const real err = norm(dd);
                    std::vector<real> cx;
                    if (wa.step(sv, dd, cx)) {
                        sn = cx;
                        clip(sn);
                    }
                    sv = sn;
                    if (it > 0 && err < opt.rel_tol * norm(sv) + opt.abs_tol) break;
                }
                WT[k] = sv;
            }
            std::vector<real> GT((size_t)nb * nb), al(nb);
            for (int k = 0; k < nb; ++k)
                for (int l = 0; l < nb; ++l) GT[(size_t)l * nb + k] = project(full[sel[l]], WT[k]);
            for (int i = 0; i < nb; ++i) al[i] = rfull[sel[i]];
            dense_solve(nb, GT, al);
            for (int k = 0; k < nb; ++k)
                for (int i = 0; i < n3; ++i) zq[i] -= al[k] * WT[k][i];
            clip(zq);
        }
    }
    mu = zq;  // the material gradients below use the contact-aware adjoint
    // parameter gradients: dl/dw_e = -(vol/s) sum_s mu_e^T A_s^T (F_s - Bp_s); reference-style dl_dmat_w
    // uses the stress over the energy's mean stiffness (deformable_pd_energy.cpp:368-403).
    int off = 0;
    for (size_t ei = 0; ei < M.energies.size(); ++ei) {
        const Energy& en = M.energies[ei];
        std::vector<real> gw(M.m, 0), gmu_bar_e(M.m, 0), gla_bar_e(M.m, 0), gmat(M.m, 0);
#pragma omp parallel for schedule(static)
        for (int e = 0; e < M.m; ++e) {
            if (!en.in_set[e]) continue;
            const int* vv = &M.E[(size_t)e * M.k];
            for (int smp = 0; smp < M.s; ++smp) {
                const SvdData& d = svd[e][smp];
                const M3 Bp = project(en, d);
                M3 FmB;
                for (int i = 0; i < 9; ++i) FmB.a[i] = d.F.a[i] - Bp.a[i];
                std::vector<real> f(M.k * 3, 0);
                add_At(M, e, smp, FmB, -M.vol / M.s, f.data());
                real dot = 0;
                for (int a = 0; a < M.k; ++a)
                    for (int i = 0; i < 3; ++i) dot += mu[3 * vv[a] + i] * f[a * 3 + i];
                gw[e] += dot;
                // reference dl_dmat_w: stress / mean stiffness
                if (en.type == kNeoHookean) {
                    const M3& F = d.F;
                    const real J = det3(F);
                    const real lj = std::log(std::max(J, real(1e-12)));
                    M3 Finv;
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            const int i1 = (j + 1) % 3, i2 = (j + 2) % 3, j1 = (i + 1) % 3, j2 = (i + 2) % 3;
                            Finv(i, j) = (F(i1, j1) * F(i2, j2) - F(i1, j2) * F(i2, j1)) / J;
                        }
                    const M3 FiT = transpose(Finv);
                    M3 P;
                    for (int i = 0; i < 9; ++i) P.a[i] = (en.mu * (F.a[i] - FiT.a[i]) + en.la * lj * FiT.a[i]) / en.w_mean;
                    std::vector<real> fp(M.k * 3, 0);
                    add_At(M, e, smp, P, -M.vol / M.s, fp.data());
                    real dp = 0;
                    for (int a = 0; a < M.k; ++a)
                        for (int i = 0; i < 3; ++i) dp += mu[3 * vv[a] + i] * fp[a * 3 + i];
                    gmat[e] += dp;
                    // mean-parameter dependence of the proximal map
                    M3 dPm, dPl;
                    nh_param_diff(en, d, dPm, dPl);
                    std::vector<real> fm(M.k * 3, 0), fl(M.k * 3, 0);
                    const real w = en.elem_w(e) * M.vol / M.s;
                    add_At(M, e, smp, dPm, w, fm.data());
                    add_At(M, e, smp, dPl, w, fl.data());
                    real a1 = 0, a2 = 0;
                    for (int a = 0; a < M.k; ++a)
                        for (int i = 0; i < 3; ++i) {
                            a1 += mu[3 * vv[a] + i] * fm[a * 3 + i];
                            a2 += mu[3 * vv[a] + i] * fl[a * 3 + i];
                        }
                    gmu_bar_e[e] += a1;
                    gla_bar_e[e] += a2;
                } else {
                    gmat[e] += dot;
                }
            }
        }
        real tot = 0;
        for (int e = 0; e < M.m; ++e) tot += gmat[e];
        dl_dmat_w[ei] = tot;
        const int np_e = (int)en.params.size();
        if (en.type != kNeoHookean) {
            if (np_e == 1) {
                real s = 0;
                for (int e = 0; e < M.m; ++e) s += gw[e];
                dl_dparams[off] = s;
            } else {
                for (int e = 0; e < M.m; ++e) dl_dparams[off + e] = gw[e];
            }
        } else {
            real gmb = 0, glb = 0;
            for (int e = 0; e < M.m; ++e) { gmb += gmu_bar_e[e]; glb += gla_bar_e[e]; }
            if (np_e == 2) {
                real s = 0;
                for (int e = 0; e < M.m; ++e) s += gw[e];
                dl_dparams[off] = 2 * s + gmb;
                dl_dparams[off + 1] = glb;
            } else {
                const real inv_m = 1.0 / M.m;
                for (int e = 0; e < M.m; ++e) {
                    dl_dparams[off + 2 * e] = 2 * gw[e] + gmb * inv_m;
                    dl_dparams[off + 2 * e + 1] = glb * inv_m;
                }
            }
        }
        off += np_e;
    }
}

struct Handle {
    Model M;
};

Options parse_opts(const char** keys, const double* vals, int n) {
    Options o;
    std::map<std::string, double> m;
    for (int i = 0; i < n; ++i) m[keys[i]] = vals[i];
    for (const char* req : {"max_pd_iter", "abs_tol", "rel_tol", "verbose", "thread_ct"})
        ORC_CHECK(m.count(req), std::string("Missing option ") + req + ".");
    o.max_pd_iter = (int)m["max_pd_iter"];
    o.abs_tol = m["abs_tol"];
    o.rel_tol = m["rel_tol"];
    o.verbose = (int)m["verbose"];
    if (m.count("aa_window")) o.aa_window = (int)m["aa_window"];
    if (m.count("friction_mu")) o.friction_mu = m["friction_mu"];
    if (m.count("restitution")) o.restitution = m["restitution"];
    if (m.count("friction_contact_slop")) o.contact_slop = m["friction_contact_slop"];
    if (m.count("alg_phd_bwd_clip_norm")) o.clip = m["alg_phd_bwd_clip_norm"];
    if (m.count("bwd_mean_stiffness")) o.mean_stiffness_bwd = (int)m["bwd_mean_stiffness"];
    if (m.count("bwd_cascade_cap")) o.cascade_cap = (int)m["bwd_cascade_cap"];
    if (m.count("skip_contact_woodbury")) o.skip_woodbury = m["skip_contact_woodbury"] > 0.5;
    if (m.count("skip_material_grad")) o.skip_material_grad = m["skip_material_grad"] > 0.5;
    if (m.count("alg_phd_bwd_tangent_lambda_min")) o.tangent_lambda_min = m["alg_phd_bwd_tangent_lambda_min"];
    if (m.count("alg_phd_bwd_rhs_prune_rel")) o.rhs_prune_rel = m["alg_phd_bwd_rhs_prune_rel"];
    if (m.count("alg_phd_bwd_rhs_prune_abs")) o.rhs_prune_abs = m["alg_phd_bwd_rhs_prune_abs"];
    if (m.count("alg_phd_bwd_basis_topk")) o.basis_topk = (int)m["alg_phd_bwd_basis_topk"];
    if (m.count("alg_phd_bwd_wt_max_iter")) o.wt_max_iter = (int)m["alg_phd_bwd_wt_max_iter"];
    if (m.count("bwd_eigen_filter")) o.eigen_filter = (int)m["bwd_eigen_filter"];
#ifdef _OPENMP
    if ((int)m["thread_ct"] > 0) omp_set_num_threads((int)m["thread_ct"]);
#endif
    return o;
}

}  // namespace

#define ORC_API extern "C" __attribute__((visibility("default")))
#define ORC_GUARD(...)                  \
    try {                               \
        __VA_ARGS__;                    \
        return 0;                       \
    } catch (const OracleError& e) {    \
        g_err = e.msg;                  \
        return 1;                       \
    } catch (const std::exception& e) { \
        g_err = e.what();               \
        return 2;                       \
    }

ORC_API const char* orc_last_error() { return g_err.c_str(); }

ORC_API void* orc_create(const double* verts, int n, const int* elems, int m, int k, double density) {
    try {
        Handle* H = new Handle();
        Model& M = H->M;
        ORC_CHECK(k == 8 || k == 4, "element_dim must be 8 (hex) or 4 (tet)");
        M.n = n; M.m = m; M.k = k; M.hex = (k == 8); M.s = (k == 8) ? 8 : 1;
        M.X.assign(verts, verts + 3 * (size_t)n);
        M.E.assign(elems, elems + (size_t)k * m);
        M.density = density;
        real sum = 0;
        for (int e = 0; e < m; ++e) sum += element_volume(M, e);
        M.vol = sum / m;
        init_samples(M);
        return H;
    } catch (const OracleError& e) {
        g_err = e.msg;
        return nullptr;
    }
}
ORC_API void orc_destroy(void* h) { delete (Handle*)h; }

ORC_API int orc_set_dirichlet(void* h, int dof, double val) {
    ORC_GUARD({
        Model& M = ((Handle*)h)->M;
        if (!M.dirichlet.count(dof)) M.ready = false;
        M.dirichlet[dof] = val;
    })
}

ORC_API int orc_add_pd_energy(void* h, const char* type, const double* params, int np, const int* idx, int nidx) {
    ORC_GUARD({
        Model& M = ((Handle*)h)->M;
        Energy en;
        const std::string t(type);
        if (t == "corotated") en.type = kCorotated;
        else if (t == "volume") en.type = kVolume;
        else if (t == "pd_neohookean") en.type = kNeoHookean;
        else ORC_CHECK(false, "Unsupported PD energy: " + t);
        en.params.assign(params, params + np);
        if (en.type != kNeoHookean) {
            ORC_CHECK(np == 1 || np == M.m, "Inconsistent param size.");
            if (np == 1) en.w_mean = params[0];
            else {
                en.w_elem.assign(params, params + np);
                en.w_mean = std::accumulate(en.w_elem.begin(), en.w_elem.end(), 0.0) / np;
            }
            en.mu = en.la = 0;
        } else {
            ORC_CHECK(np == 2 || np == 2 * M.m, "pd_neohookean expects [mu, lambda] or 2*element_num params");
            if (np == 2) {
                en.mu = params[0]; en.la = params[1]; en.w_mean = 2 * params[0];
            } else {
                real sm = 0, sl = 0;
                en.w_elem.resize(M.m);
                for (int e = 0; e < M.m; ++e) {
                    sm += params[2 * e]; sl += params[2 * e + 1];
                    en.w_elem[e] = 2 * params[2 * e];
                }
                en.mu = sm / M.m; en.la = sl / M.m;
                en.w_mean = std::accumulate(en.w_elem.begin(), en.w_elem.end(), 0.0) / M.m;
            }
        }
        en.in_set.assign(M.m, nidx == 0 ? 1 : 0);
        for (int i = 0; i < nidx; ++i) {
            ORC_CHECK(idx[i] >= 0 && idx[i] < M.m, "Element index out of bound.");
            en.in_set[idx[i]] = 1;
        }
        M.energies.push_back(en);
        M.ready = false;
    })
}

ORC_API int orc_add_gravity(void* h, const double* g) {
    ORC_GUARD({
        Model& M = ((Handle*)h)->M;
        M.gravity.assign(g, g + 3);
    })
}

ORC_API int orc_set_planar_boundary(void* h, const double* p4, const int* idx, int nidx) {
    ORC_GUARD({
        Model& M = ((Handle*)h)->M;
        const real nn = std::sqrt(p4[0] * p4[0] + p4[1] * p4[1] + p4[2] * p4[2]);
        ORC_CHECK(nn > std::numeric_limits<real>::epsilon(), "Singular normal.");
        for (int d = 0; d < 3; ++d) M.pn[d] = p4[d] / nn;
        M.poff = p4[3] / nn;
        std::set<int> u(idx, idx + nidx);
        ORC_CHECK((int)u.size() == nidx, "Duplicated vertex elements.");
        M.contact_nodes.assign(u.begin(), u.end());
        M.has_plane = true;
        M.ready = false;
    })
}

ORC_API int orc_num_params(void* h) { return count_params(((Handle*)h)->M); }
ORC_API double orc_mass(void* h) { return ((Handle*)h)->M.mass(); }
ORC_API int orc_last_iters(void* h) { return ((Handle*)h)->M.last_iters; }
ORC_API int orc_last_filtered(void* h) { return ((Handle*)h)->M.last_filtered; }
ORC_API int orc_last_converged(void* h) { return ((Handle*)h)->M.last_converged; }
ORC_API void orc_reset_warm_start(void* h) {
    ((Handle*)h)->M.prev_cand.clear();
    ((Handle*)h)->M.prev_lambda.clear();
}

ORC_API int orc_forward(void* h, const double* q, const double* v, const double* f_ext, double dt, const char** keys,
                        const double* vals, int nopt, double* q_next, double* v_next, int* active, int* n_active) {
    ORC_GUARD({
        Model& M = ((Handle*)h)->M;
        const Options o = parse_opts(keys, vals, nopt);
        std::vector<int> act;
        forward(M, q, v, f_ext, dt, o, q_next, v_next, act);
        for (size_t i = 0; i < act.size(); ++i) active[i] = act[i];
        *n_active = (int)act.size();
    })
}

ORC_API int orc_backward(void* h, const double* q, const double* v, const double* f_ext, double dt,
                         const double* q_next, const double* dl_dq_next, const double* dl_dv_next, const char** keys,
                         const double* vals, int nopt, double* dl_dq, double* dl_dv, double* dl_df,
                         double* dl_dmat_w, double* dl_dparams, double* dl_dstate_p, int* iters) {
    ORC_GUARD({
        Model& M = ((Handle*)h)->M;
        const Options o = parse_opts(keys, vals, nopt);
        backward(M, q, v, f_ext, dt, q_next, dl_dq_next, dl_dv_next, o, dl_dq, dl_dv, dl_df, dl_dmat_w, dl_dparams,
                 dl_dstate_p, iters);
    })
}

// Building blocks exposed for unit tests.
ORC_API int orc_ainv(void* h, double dt, const double* b, double* x) {
    ORC_GUARD({
        Model& M = ((Handle*)h)->M;
        setup_solver(M, dt);
        apply_ainv(M, b, x);
    })
}
ORC_API int orc_local_step(void* h, const double* q, double* rhs) {
    ORC_GUARD({ local_step(((Handle*)h)->M, q, rhs); })
}
ORC_API void orc_svd3(const double* F9, double* U9, double* sig3, double* V9) {
    M3 F, U, V;
    for (int i = 0; i < 9; ++i) F.a[i] = F9[i];
    svd3(F, U, sig3, V);
    for (int i = 0; i < 9; ++i) { U9[i] = U.a[i]; V9[i] = V.a[i]; }
}
// type: 0 corotated, 1 volume, 2 NH (mu, la, k given)
ORC_API int orc_project(int type, const double* F9, double mu, double la, double k, double* P9) {
    ORC_GUARD({
        Energy en;
        en.type = type; en.mu = mu; en.la = la; en.w_mean = k;
        M3 F;
        for (int i = 0; i < 9; ++i) F.a[i] = F9[i];
        const M3 P = project(en, make_svd(F));
        for (int i = 0; i < 9; ++i) P9[i] = P.a[i];
    })
}
ORC_API int orc_project_diff(int type, const double* F9, double mu, double la, double k, const double* dF9,
                             double* dP9) {
    ORC_GUARD({
        Energy en;
        en.type = type; en.mu = mu; en.la = la; en.w_mean = k;
        M3 F, dF;
        for (int i = 0; i < 9; ++i) { F.a[i] = F9[i]; dF.a[i] = dF9[i]; }
        const M3 P = project_diff(en, make_svd(F), dF);
        for (int i = 0; i < 9; ++i) dP9[i] = P.a[i];
    })
}
// Assembled A (axis d) as dense row-major n*n, for small-case tests.
ORC_API int orc_dense_A(void* h, double dt, int axis, double* out) {
    ORC_GUARD({
        Model& M = ((Handle*)h)->M;
        setup_solver(M, dt);
        const int n = M.n;
        std::vector<real> e(n, 0), col(n);
        // reconstruct A from the factors: A = P^T L D L^T P, column by column
        const Ldl& F = M.ldl[axis];
        for (int c = 0; c < n; ++c) {
            std::vector<real> y(n, 0);
            y[F.iperm[c]] = 1;                        // P e_c
            for (int j = 0; j < n; ++j)                // L^T y (ascending: rows below j still hold inputs)
                for (int p = F.Lp[j]; p < F.Lp[j + 1]; ++p) y[j] += F.Lx[p] * y[F.Li[p]];
            for (int j = 0; j < n; ++j) y[j] *= F.D[j];
            for (int j = n - 1; j >= 0; --j) {         // L y (column-oriented, descending keeps inputs intact)
                for (int p = F.Lp[j]; p < F.Lp[j + 1]; ++p) y[F.Li[p]] += F.Lx[p] * y[j];
            }
            for (int r = 0; r < n; ++r) out[(size_t)F.perm[r] * n + c] = y[r];
        }
    })
}
