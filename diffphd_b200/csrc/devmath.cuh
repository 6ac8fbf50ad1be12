// Register-resident 3x3 numerics for the element kernels (FP32 and FP64).
//
// Matrices are column-major 9-vectors, A(i,j) = a[i + 3j], the reference's Flatten order
// (cpp/core/src/common/geometry.cpp:192-200).
//
// SVD: one-sided Jacobi (Hestenes 1958; convergence analysis Demmel & Veselic 1992) — plane rotations
// applied on the right orthogonalise the columns of B = F V; singular values are the column norms, U the
// normalised columns.  The result follows Eigen::JacobiSVD's contract that the reference relies on
// (deformation_gradient_auxiliary_data.cpp:4-12): sig >= 0 sorted descending, U and V orthogonal with
// det(U) det(V) = sign(det F), so R = U V^T is a reflection for inverted elements exactly as in the
// reference (geometry.cpp:24-31).
#pragma once
#include <cfloat>
#include <cmath>

namespace dphd {

template <typename T> struct Eps;
template <> struct Eps<double> { static constexpr double v = DBL_EPSILON; static constexpr int sweeps = 12; };
template <> struct Eps<float> { static constexpr float v = FLT_EPSILON; static constexpr int sweeps = 8; };

template <typename T> __device__ __forceinline__ T dsqrt(T x) { return sqrt(x); }
template <typename T> __device__ __forceinline__ T dabs(T x) { return fabs(x); }

#define M3(a, i, j) a[(i) + 3 * (j)]

template <typename T>
__device__ __forceinline__ void mat3_mul(const T* A, const T* B, T* C) {
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) M3(C, i, j) = M3(A, i, 0) * M3(B, 0, j) + M3(A, i, 1) * M3(B, 1, j) + M3(A, i, 2) * M3(B, 2, j);
}
// C = U diag(s) V^T
template <typename T>
__device__ __forceinline__ void usvt(const T* U, const T* s, const T* V, T* C) {
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i)
            M3(C, i, j) = M3(U, i, 0) * s[0] * M3(V, j, 0) + M3(U, i, 1) * s[1] * M3(V, j, 1) + M3(U, i, 2) * s[2] * M3(V, j, 2);
}

template <typename T>
__device__ __forceinline__ void jacobi_rotate_cols(T* B, T* V, int p, int q) {
    const T alpha = M3(B, 0, p) * M3(B, 0, p) + M3(B, 1, p) * M3(B, 1, p) + M3(B, 2, p) * M3(B, 2, p);
    const T beta = M3(B, 0, q) * M3(B, 0, q) + M3(B, 1, q) * M3(B, 1, q) + M3(B, 2, q) * M3(B, 2, q);
    const T gamma = M3(B, 0, p) * M3(B, 0, q) + M3(B, 1, p) * M3(B, 1, q) + M3(B, 2, p) * M3(B, 2, q);
    if (gamma == T(0) || dabs(gamma) <= T(4) * Eps<T>::v * dsqrt(alpha * beta)) return;
    const T zeta = (beta - alpha) / (T(2) * gamma);
    const T t = (zeta >= T(0) ? T(1) : T(-1)) / (dabs(zeta) + dsqrt(T(1) + zeta * zeta));
    const T c = T(1) / dsqrt(T(1) + t * t);
    const T s = c * t;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const T bp = M3(B, r, p), bq = M3(B, r, q);
        M3(B, r, p) = c * bp - s * bq;
        M3(B, r, q) = s * bp + c * bq;
        const T vp = M3(V, r, p), vq = M3(V, r, q);
        M3(V, r, p) = c * vp - s * vq;
        M3(V, r, q) = s * vp + c * vq;
    }
}

template <typename T>
__device__ __forceinline__ bool cols_orthogonal(const T* B) {
    bool ok = true;
#pragma unroll
    for (int pq = 0; pq < 3; ++pq) {
        const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
        const T a = M3(B, 0, p) * M3(B, 0, p) + M3(B, 1, p) * M3(B, 1, p) + M3(B, 2, p) * M3(B, 2, p);
        const T b = M3(B, 0, q) * M3(B, 0, q) + M3(B, 1, q) * M3(B, 1, q) + M3(B, 2, q) * M3(B, 2, q);
        const T g = M3(B, 0, p) * M3(B, 0, q) + M3(B, 1, p) * M3(B, 1, q) + M3(B, 2, p) * M3(B, 2, q);
        ok = ok && (g == T(0) || dabs(g) <= T(4) * Eps<T>::v * dsqrt(a * b));
    }
    return ok;
}

template <typename T>
__device__ __forceinline__ void swap_cols(T* A, int p, int q) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const T t = M3(A, r, p);
        M3(A, r, p) = M3(A, r, q);
        M3(A, r, q) = t;
    }
}

template <typename T>
__device__ void svd3(const T* F, T* U, T* sig, T* V) {
    T B[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) { B[i] = F[i]; V[i] = T(0); }
    V[0] = V[4] = V[8] = T(1);
    for (int sweep = 0; sweep < Eps<T>::sweeps; ++sweep) {
        jacobi_rotate_cols(B, V, 0, 1);
        jacobi_rotate_cols(B, V, 0, 2);
        jacobi_rotate_cols(B, V, 1, 2);
        if (cols_orthogonal(B)) break;
    }
    T s[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) s[i] = dsqrt(M3(B, 0, i) * M3(B, 0, i) + M3(B, 1, i) * M3(B, 1, i) + M3(B, 2, i) * M3(B, 2, i));
    // sort descending (3-element network), permuting columns of B and V alongside
    if (s[0] < s[1]) { T t = s[0]; s[0] = s[1]; s[1] = t; swap_cols(B, 0, 1); swap_cols(V, 0, 1); }
    if (s[1] < s[2]) { T t = s[1]; s[1] = s[2]; s[2] = t; swap_cols(B, 1, 2); swap_cols(V, 1, 2); }
    if (s[0] < s[1]) { T t = s[0]; s[0] = s[1]; s[1] = t; swap_cols(B, 0, 1); swap_cols(V, 0, 1); }
    const T tiny = T(64) * Eps<T>::v * (s[0] > T(0) ? s[0] : T(1));
    // U columns: normalised B columns; rank-deficient columns completed to an orthonormal basis
    if (s[0] > T(0)) {
#pragma unroll
        for (int r = 0; r < 3; ++r) M3(U, r, 0) = M3(B, r, 0) / s[0];
    } else {
        M3(U, 0, 0) = T(1); M3(U, 1, 0) = T(0); M3(U, 2, 0) = T(0);
    }
    if (s[1] > tiny) {
#pragma unroll
        for (int r = 0; r < 3; ++r) M3(U, r, 1) = M3(B, r, 1) / s[1];
    } else {
        // any unit vector orthogonal to U0: cross with the least-aligned axis
        const T ax = dabs(M3(U, 0, 0)), ay = dabs(M3(U, 1, 0)), az = dabs(M3(U, 2, 0));
        T e[3] = {T(0), T(0), T(0)};
        if (ax <= ay && ax <= az) e[0] = T(1); else if (ay <= az) e[1] = T(1); else e[2] = T(1);
        T c[3] = {M3(U, 1, 0) * e[2] - M3(U, 2, 0) * e[1], M3(U, 2, 0) * e[0] - M3(U, 0, 0) * e[2],
                  M3(U, 0, 0) * e[1] - M3(U, 1, 0) * e[0]};
        const T cn = dsqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
#pragma unroll
        for (int r = 0; r < 3; ++r) M3(U, r, 1) = c[r] / cn;
    }
    if (s[2] > tiny) {
#pragma unroll
        for (int r = 0; r < 3; ++r) M3(U, r, 2) = M3(B, r, 2) / s[2];
    } else {
        M3(U, 0, 2) = M3(U, 1, 0) * M3(U, 2, 1) - M3(U, 2, 0) * M3(U, 1, 1);
        M3(U, 1, 2) = M3(U, 2, 0) * M3(U, 0, 1) - M3(U, 0, 0) * M3(U, 2, 1);
        M3(U, 2, 2) = M3(U, 0, 0) * M3(U, 1, 1) - M3(U, 1, 0) * M3(U, 0, 1);
    }
    sig[0] = s[0]; sig[1] = s[1]; sig[2] = s[2];
}

// Small dense solve (n <= 4) by Gaussian elimination with partial pivoting; A row-major, overwritten.
template <typename T, int N>
__device__ __forceinline__ void small_solve(T* A, T* b) {
#pragma unroll
    for (int c = 0; c < N; ++c) {
        int piv = c;
#pragma unroll
        for (int r = c + 1; r < N; ++r)
            if (dabs(A[r * N + c]) > dabs(A[piv * N + c])) piv = r;
        if (piv != c) {
#pragma unroll
            for (int k = 0; k < N; ++k) { T t = A[c * N + k]; A[c * N + k] = A[piv * N + k]; A[piv * N + k] = t; }
            T t = b[c]; b[c] = b[piv]; b[piv] = t;
        }
        const T d = A[c * N + c];
#pragma unroll
        for (int r = c + 1; r < N; ++r) {
            const T f = A[r * N + c] / d;
#pragma unroll
            for (int k = c; k < N; ++k) A[r * N + k] -= f * A[c * N + k];
            b[r] -= f * b[c];
        }
    }
#pragma unroll
    for (int c = N - 1; c >= 0; --c) {
        T s = b[c];
#pragma unroll
        for (int k = c + 1; k < N; ++k) s -= A[c * N + k] * b[k];
        b[c] = s / A[c * N + c];
    }
}

// Volume projection onto prod(sig*) = 1: Newton iterations on D = sig* - sig exactly as
// cpp/core/src/pd_energy/volume_pd_element_energy.cpp:22-59 (initial guess sig/cbrt(prod) - sig,
// <= 50 iterations, stop when max|dD| <= eps).  Returns false on a singular F (sig_min < eps).
template <typename T>
__device__ __forceinline__ bool volume_D(const T* sig, T* D) {
    const T eps = Eps<T>::v;
    if (sig[2] < eps) return false;
    const T cr = pow(sig[0] * sig[1] * sig[2], T(1) / T(3));
#pragma unroll
    for (int i = 0; i < 3; ++i) D[i] = sig[i] / cr - sig[i];
    for (int it = 0; it < 50; ++it) {
        const T a0 = sig[0] + D[0], a1 = sig[1] + D[1], a2 = sig[2] + D[2];
        const T C = a0 * a1 * a2 - T(1);
        const T g0 = a1 * a2, g1 = a0 * a2, g2 = a0 * a1;
        const T f = (g0 * D[0] + g1 * D[1] + g2 * D[2] - C) / (g0 * g0 + g1 * g1 + g2 * g2);
        const T n0 = f * g0, n1 = f * g1, n2 = f * g2;
        const T diff = fmax(fmax(dabs(n0 - D[0]), dabs(n1 - D[1])), dabs(n2 - D[2]));
        if (diff <= eps) break;
        D[0] = n0; D[1] = n1; D[2] = n2;
    }
    return true;
}

// Neo-Hookean proximal map on singular values
// (cpp/core/src/pd_energy/neohookean_pd_element_energy.cpp:38-104): minimise psi(sig) + k/2 |sig - sig_F|^2
// by <= 32 damped Newton steps with a positivity-guarded backtracking line search.
template <typename T>
__device__ __forceinline__ void nh_hessian(T mu, T la, T k, const T* s, T* H) {
    const T prod = s[0] * s[1] * s[2];
    const T L = log(fmax(prod, T(1e-12)));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            H[i * 3 + j] = (i == j) ? mu + (mu + la - la * L) / (s[i] * s[i]) + k : la / (s[i] * s[j]);
}
template <typename T>
__device__ void nh_prox(T mu, T la, T k, const T* sF, T* s) {
    // FP64: the reference's tolerances.  FP32: the step test at 1e-6 (1e-10 is below FP32 resolution).
    const T sig_min = T(1e-4), tol = sizeof(T) == 4 ? T(1e-6) : T(1e-10);
#pragma unroll
    for (int i = 0; i < 3; ++i) s[i] = sF[i] < sig_min ? sig_min : sF[i];
    for (int it = 0; it < 32; ++it) {
        const T L = log(fmax(s[0] * s[1] * s[2], T(1e-12)));
        T g[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) g[i] = mu * s[i] - mu / s[i] + la * L / s[i] + k * (s[i] - sF[i]);
        if (dsqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) < tol) break;
        T H[9];
        nh_hessian(mu, la, k, s, H);
        H[0] += T(1e-9); H[4] += T(1e-9); H[8] += T(1e-9);
        small_solve<T, 3>(H, g);
        T alpha = T(1), sn[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) sn[i] = s[i] - alpha * g[i];
        for (int ls = 0; ls < 20; ++ls) {
            if (fmin(fmin(sn[0], sn[1]), sn[2]) > sig_min * T(0.5)) break;
            alpha *= T(0.5);
#pragma unroll
            for (int i = 0; i < 3; ++i) sn[i] = s[i] - alpha * g[i];
        }
        const T step = fmax(fmax(dabs(sn[0] - s[0]), dabs(sn[1] - s[1])), dabs(sn[2] - s[2]));
#pragma unroll
        for (int i = 0; i < 3; ++i) s[i] = sn[i] < sig_min ? sig_min : sn[i];
        if (step < tol) break;
    }
}

// dSVD (Townsend's closed form, with the reference's 10*eps skip of near-equal singular values,
// cpp/core/src/common/geometry.cpp:159-186).
template <typename T>
__device__ void dsvd3(const T* U, const T* sig, const T* V, const T* dF, T* dU, T* dsig, T* dV) {
    T tmp[9], dP[9], Ut[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) M3(Ut, i, j) = M3(U, j, i);
    mat3_mul(Ut, dF, tmp);
    mat3_mul(tmp, V, dP);
#pragma unroll
    for (int i = 0; i < 3; ++i) dsig[i] = M3(dP, i, i);
    const T eps = T(10) * Eps<T>::v;
    T wU[9], wV[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T sij = T(0);
            if (i < j && sig[i] - sig[j] > eps) sij = T(1) / (sig[j] * sig[j] - sig[i] * sig[i]);
            if (i > j && sig[j] - sig[i] > eps) sij = -T(1) / (sig[i] * sig[i] - sig[j] * sig[j]);
            M3(wU, i, j) = sij * (M3(dP, i, j) * sig[j] + sig[i] * M3(dP, j, i));
            M3(wV, i, j) = sij * (sig[i] * M3(dP, i, j) + M3(dP, j, i) * sig[j]);
        }
    mat3_mul(U, wU, dU);
    mat3_mul(V, wV, dV);
}

struct ElemEnergyDev {
    int type;          // 0 corotated, 1 volume, 2 Neo-Hookean
    int per_element;   // w read from w[e] when set, else w_mean
    double w_mean;
    double mu, la;     // Neo-Hookean means (proximal penalty k = w_mean)
    const double* w;   // per-element stiffness (FP64)
    const float* w32;  // per-element stiffness (FP32 copy)
    const unsigned char* mask;  // element membership, null = all elements
};

// Projection Bp(F) for one energy, given the SVD of F.  Returns false on a singular F for the volume energy.
template <typename T>
__device__ __forceinline__ bool project(int type, T mu, T la, T k, const T* U, const T* sig, const T* V, T* P) {
    if (type == 0) {
        const T one[3] = {T(1), T(1), T(1)};
        usvt(U, one, V, P);
        return true;
    }
    if (type == 1) {
        T D[3];
        if (!volume_D(sig, D)) {
#pragma unroll
            for (int i = 0; i < 9; ++i) P[i] = T(0);
            return false;
        }
        const T s[3] = {sig[0] + D[0], sig[1] + D[1], sig[2] + D[2]};
        usvt(U, s, V, P);
        return true;
    }
    T s[3];
    nh_prox(mu, la, k, sig, s);
    usvt(U, s, V, P);
    return true;
}

// Bp(F) - F = U diag(s* - sig) V^T, evaluated without cancellation against F (used by the FP32 path, which
// keeps the linear part F - F_bound in FP64).
template <typename T>
__device__ __forceinline__ bool project_delta(int type, T mu, T la, T k, const T* U, const T* sig, const T* V, T* D) {
    T d[3];
    bool ok = true;
    if (type == 0) {
        d[0] = T(1) - sig[0]; d[1] = T(1) - sig[1]; d[2] = T(1) - sig[2];
    } else if (type == 1) {
        ok = volume_D(sig, d);
        if (!ok) d[0] = d[1] = d[2] = T(0);
    } else {
        T s[3];
        nh_prox(mu, la, k, sig, s);
        d[0] = s[0] - sig[0]; d[1] = s[1] - sig[1]; d[2] = s[2] - sig[2];
    }
    usvt(U, d, V, D);
    return ok;
}

// Directional derivative of Bp along dF (corotated: dR from the 3x3 system of geometry.cpp:60-80;
// volume: KKT system of volume_pd_element_energy.cpp:61-155; Neo-Hookean: implicit function theorem on the
// proximal optimality, neohookean_pd_element_energy.cpp:133-165).
template <typename T>
__device__ void project_diff(int type, T mu, T la, T k, const T* U, const T* sig, const T* V, const T* dF, T* out) {
    if (type == 0) {
        T R[9], S[9], one[3] = {T(1), T(1), T(1)};
        usvt(U, one, V, R);
        usvt(V, sig, V, S);
        // lhs = R^T dF - dF^T R (only the strictly-upper entries are used)
        T lhs01 = T(0), lhs02 = T(0), lhs12 = T(0);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            lhs01 += M3(R, r, 0) * M3(dF, r, 1) - M3(dF, r, 0) * M3(R, r, 1);
            lhs02 += M3(R, r, 0) * M3(dF, r, 2) - M3(dF, r, 0) * M3(R, r, 2);
            lhs12 += M3(R, r, 1) * M3(dF, r, 2) - M3(dF, r, 1) * M3(R, r, 2);
        }
        T A[9] = {M3(S, 0, 0) + M3(S, 1, 1), M3(S, 1, 2), -M3(S, 0, 2),
                  M3(S, 1, 2), M3(S, 0, 0) + M3(S, 2, 2), M3(S, 0, 1),
                  -M3(S, 0, 2), M3(S, 0, 1), M3(S, 1, 1) + M3(S, 2, 2)};
        T b[3] = {lhs01, lhs02, lhs12};
        small_solve<T, 3>(A, b);
        T W[9] = {T(0), -b[0], -b[1], b[0], T(0), -b[2], b[1], b[2], T(0)};  // column-major skew
        mat3_mul(R, W, out);
        return;
    }
    T dU[9], dV[9], ds[3];
    dsvd3(U, sig, V, dF, dU, ds, dV);
    if (type == 1) {
        T D[3];
        volume_D(sig, D);
        const T a0 = sig[0] + D[0], a1 = sig[1] + D[1], a2 = sig[2] + D[2];
        const T g[3] = {a1 * a2, a0 * a2, a0 * a1};
        // H(i,j) = prod over the remaining index (i != j), 0 on the diagonal
        const T H[9] = {T(0), a2, a1, a2, T(0), a0, a1, a0, T(0)};
        const T Dn = dsqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
        const T gn = dsqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
        const T la_abs = Dn / gn;
        T e1 = T(0), e2 = T(0);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            e1 += (D[i] - la_abs * g[i]) * (D[i] - la_abs * g[i]);
            e2 += (D[i] + la_abs * g[i]) * (D[i] + la_abs * g[i]);
        }
        const T lam = e1 < e2 ? -la_abs : la_abs;
        T A[16], b[4];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
#pragma unroll
            for (int j = 0; j < 3; ++j) A[i * 4 + j] = (i == j ? T(1) : T(0)) + lam * H[i * 3 + j];
            A[i * 4 + 3] = g[i];
            A[12 + i] = g[i];
            b[i] = -lam * (H[i * 3] * ds[0] + H[i * 3 + 1] * ds[1] + H[i * 3 + 2] * ds[2]);
        }
        A[15] = T(0);
        b[3] = -(g[0] * ds[0] + g[1] * ds[1] + g[2] * ds[2]);
        small_solve<T, 4>(A, b);
        T t1[9], t2[9], t3[9];
        usvt(dU, D, V, t1);
        usvt(U, b, V, t2);
        usvt(U, D, dV, t3);
#pragma unroll
        for (int i = 0; i < 9; ++i) out[i] = dF[i] + t1[i] + t2[i] + t3[i];
        return;
    }
    T ss[3];
    nh_prox(mu, la, k, sig, ss);
    T H[9];
    nh_hessian(mu, la, k, ss, H);
    H[0] += T(1e-9); H[4] += T(1e-9); H[8] += T(1e-9);
    T r[3] = {k * ds[0], k * ds[1], k * ds[2]};
    small_solve<T, 3>(H, r);
    T t1[9], t2[9], t3[9];
    usvt(dU, ss, V, t1);
    usvt(U, r, V, t2);
    usvt(U, ss, dV, t3);
#pragma unroll
    for (int i = 0; i < 9; ++i) out[i] = t1[i] + t2[i] + t3[i];
}

}  // namespace dphd
