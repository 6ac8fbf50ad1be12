// Kernel launch interface of the B200 projective-dynamics step.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "devmath.cuh"

namespace dphd {

constexpr int kMaxEnergies = 4;
constexpr int kMaxWindow = 8;
constexpr int kTileCols = 128;       // S^T column tile width (32 lanes x 4 columns)
constexpr int kRedBlocks = 296;      // fixed grid of the reduction kernels (2 x 148 SMs)
constexpr int kAaSlots = 24;         // per-block partial slots of the AA reduction

// Status bits written by kernels (never a trap).
enum StatusBits : int {
    kStatusSingularF = 1,        // volume projection met sig_min < eps
    kStatusNonFinite = 2,        // NaN/Inf in an iterate
    kStatusDiverged = 4,         // adjoint iterate exceeded the clip norm
};

// Device-resident control block of one fixed-point solve (forward PD loop or backbone adjoint).
struct Ctrl {
    int iter, done, converged, status;
    int count, head, m, accept, restart;
    int max_iter, window, mode;          // mode 0: forward, 1: adjoint
    double rel_tol, abs_tol, clip;
    double gamma[kMaxWindow];
    double dq, rn, pdc, pdr, err, xn;    // last gate quantities
    unsigned int arrive[4];
};

struct EnergyPack {
    int count;
    ElemEnergyDev en[kMaxEnergies];
};

// Element kernels --------------------------------------------------------------------------------
// Forward local step: per-element node contributions of sum_energies w_e (vol/s) A_s^T (Bp(F_s) - F_bound,s).
template <typename T>
void launch_elem_fwd(int m, int k, int s, const int* E, const double* q, const double* qb, const unsigned char* elem_dir,
                     const double* grad, int hex, double vol_over_s, const EnergyPack& ep, T* elem_out, Ctrl* ctrl,
                     cudaStream_t st);
// Per-node gather of element contributions: b = inv_h2m q_tilde + pd (Dirichlet rows zero), written to the
// permuted SoA right-hand side; pd kept node-major with the gate partial norms.
template <typename T>
void launch_gather_fwd(int n, const int* node_ptr, const int* node_inc, const T* elem_out, const double* qt,
                       double inv_h2m, const unsigned char* fixed_node, const int* iperm, T* v_perm, int npad,
                       double* pd, double* prev_pd, double* part, Ctrl* ctrl, cudaStream_t st);
// y = S v and x = S^T y (x scattered to node-major FP64 through perm).
template <typename T>
void launch_spmv_S(int n, const int64_t* row_off, const int* row_a, const int* row_len, const T* vals, const T* v,
                   int npad, T* y, const Ctrl* ctrl, cudaStream_t st);
template <typename T>
void launch_spmv_ST(int n, int ntiles, const int* tile_ptr, const int* tile_rows, const int64_t* row_off,
                    const int* row_a, const int* row_len, const T* vals, const T* y, int npad, const int* perm,
                    double* x_out, const Ctrl* ctrl, cudaStream_t st);

// Anderson acceleration + gate ------------------------------------------------------------------
void launch_aa_reduce(int n3, const double* x, const double* x_raw, const unsigned char* fixed_dof,
                      const double* fixed_val, double* dG, double* dX, double* last_g, double* last_x, int ld,
                      double* part, Ctrl* ctrl, cudaStream_t st);
void launch_aa_update(int n3, double* x, const double* x_raw, const unsigned char* fixed_dof, const double* fixed_val,
                      const double* dG, const double* dX, int ld, double* part, const double* gate_part,
                      int gate_blocks, Ctrl* ctrl, cudaStream_t st);

// Misc vector kernels
void launch_qtilde(int n3, const double* q, const double* v, const double* f_ext, double h, double h2m,
                   const double* grav_force, double* qt, cudaStream_t st);
void launch_velocity(int n3, const double* q_next, const double* q, double inv_h, double* v_next, cudaStream_t st);

// Adjoint ------------------------------------------------------------------------------------------
// Per-sample 9x9 local Jacobians J_s = sum_energies w (vol/s) dBp/dF at q_next (optionally eigen-filtered).
void launch_jac_build(int m, int k, int s, const int* E, const double* q, const double* grad, int hex,
                      double vol_over_s, const EnergyPack& ep, int mean_w, int filter, double* J, Ctrl* ctrl,
                      cudaStream_t st);
// K_pd u element contributions from the cached Jacobians.
void launch_kpd_elem(int m, int k, int s, const int* E, const double* u, const double* grad, int hex, const double* J,
                     double* elem_out, const Ctrl* ctrl, cudaStream_t st);
// rhs = gbar + K_pd u, Dirichlet rows zero, permuted SoA.
void launch_gather_bwd(int n, const int* node_ptr, const int* node_inc, const double* elem_out, const double* gbar,
                       const unsigned char* fixed_node, const int* iperm, double* v_perm, int npad, const Ctrl* ctrl,
                       cudaStream_t st);
// Parameter gradients at q_next for adjoint mu: per element and energy dl/dw_e = -(vol/s) sum_s mu_e^T A_s^T (F - Bp),
// the reference-style stress term, and the Neo-Hookean mean-parameter terms.
void launch_param_grad(int m, int k, int s, const int* E, const double* q, const double* mu, const double* grad,
                       int hex, double vol_over_s, const EnergyPack& ep, double* gw /* [energies][m] */,
                       double* gmat /* [energies][m] */, double* gnh /* [energies][m][2] */, cudaStream_t st);

}  // namespace dphd
