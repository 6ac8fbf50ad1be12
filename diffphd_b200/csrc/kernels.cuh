// Kernel launch interface of the B200 projective-dynamics step.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "devmath.cuh"

namespace dphd {

constexpr int kMaxEnergies = 4;
constexpr int kMaxWindow = 8;
constexpr int kTileCols = 128;       // S^T column tile width (32 lanes x 4 columns)
constexpr int kRedBlocks = 296;      // grid of the small adjoint reductions (2 x 148 SMs)
constexpr int kMaxRedBlocks = 1184;  // upper bound of the per-iteration reduction grids (8 x 148 SMs)

// Status bits written by kernels (never a trap).
enum StatusBits : int {
    kStatusSingularF = 1,        // volume projection met sig_min < eps
    kStatusNonFinite = 2,        // NaN/Inf in an iterate
    kStatusDiverged = 4,         // adjoint iterate exceeded the clip norm
    kStatusIndefinite = 8,       // conjugate-gradient curvature p^T (A - K) p <= 0
    kStatusBarrierTimeout = 16,  // a grid-wide barrier of a cooperative kernel gave up waiting
};

// Device-resident control block of one fixed-point solve (forward PD loop or backbone adjoint).
struct Ctrl {
    int iter, done, converged, status;
    int count, head, m, accept, restart;
    int max_iter, window, mode;          // mode 0: forward, 1: adjoint
    double rel_tol, abs_tol, clip;
    double gamma[kMaxWindow];
    double gram[kMaxWindow][kMaxWindow];  // dG_i . dG_j by ring slot (incrementally extended)
    double dq, rn, pdc, pdr, err, xn;    // last gate quantities
    double rz, alpha, beta;              // conjugate-gradient scalars of the adjoint solve
    int pcg_init;
    unsigned int arrive[4];
    int loops;  // iterations run by the device-side while loop (k_loop_cond)
    // stall detection of the forward loop (mixed precision): the solve stops with `stalled` set when the gate
    // ratio max(|dq| / (rtol |q| + atol), |d pd| / (rtol |pd| + atol)) has not halved for stall_window iterations
    int stall_window, stalled, best_it;
    double best_ratio;
};

struct EnergyPack {
    int count;
    ElemEnergyDev en[kMaxEnergies];
};

// Element kernels --------------------------------------------------------------------------------
// Forward local step: per-element node contributions of sum_energies w_e (vol/s) A_s^T (Bp(F_s) - F_bound,s).
template <typename T>
void launch_elem_fwd(int m, int k, int s, const int* E, const double* q, const double* qb, const unsigned char* elem_dir,
                     const double* grad, int hex, double vol_over_s, const EnergyPack& ep, double* elem_out, Ctrl* ctrl,
                     cudaStream_t st);
// Per-node gather of element contributions: b = inv_h2m q_tilde + pd (Dirichlet rows zero), written to the
// permuted SoA right-hand side; pd kept node-major with the gate partial norms.
// When A_rp is non-null the residual form is written instead: v = b - A q (refinement of an inexact A^-1).
struct NodeCsr {
    const int* rp = nullptr;
    const int* ci = nullptr;
    const double* v = nullptr;
};
template <typename T>
void launch_gather_fwd(int n, const int* node_ptr, const int* node_inc, const double* elem_out, const double* qt,
                       double inv_h2m, const unsigned char* fixed_node, const int* iperm, T* v_perm, int npad,
                       double* prev_pd, double* part, int blocks, NodeCsr A, const double* q, int zero_dirichlet,
                       Ctrl* ctrl, cudaStream_t st,
                       double* r_out = nullptr);
// Sparse-inverse SpMV pair x = S^T (S v) (3 right-hand sides, permuted SoA v and y, x node-major FP64).
// S row i: row_len[i] values from column row_a[i] (both multiples of 4) at vals[row_off[i]].
template <typename T>
struct SpmvPlan {
    int n = 0, npad = 0;
    const int64_t* row_off = nullptr;
    const int* row_a = nullptr;
    const int* row_len = nullptr;
    const T* vals = nullptr;
    int keep_in_l2 = 0;  // S fits comfortably in L2: ordinary cached loads instead of evict-first streaming
    // y = S v: work items (row, first column, column count) of at most kSegCols columns, one warp each;
    // items of the same nested-dissection separator and column segment are adjacent so that the warps of
    // one CTA read the same slice of v (L1 reuse).  Partial sums ypart[item][3] are summed per row in item
    // order by the fix-up kernel (rows own items [row_item_ptr[r], row_item_ptr[r+1]) via row_items).
    int n_items = 0;
    const int4* item_desc = nullptr;    // per item: S offset of its first value (lo, hi words), first column, count
    const int* item_slot = nullptr;     // per item: its slot in ypart; row r owns slots [row_yptr[r], row_yptr[r+1])
    const int* row_yptr = nullptr;
    const int4* trow_desc = nullptr;    // per S^T tile-row position: first column, length, slot range of the row
    const int64_t* trow_off = nullptr;  // per S^T tile-row position: S offset of the row's first value
    const int* item_row = nullptr;
    const int* item_c0 = nullptr;
    const int* item_nc = nullptr;
    const int* row_item_ptr = nullptr;
    const int* row_items = nullptr;
    T* ypart = nullptr;
    // x = S^T y: column tiles of kTileCols, each tile's row list split into chunks (one CTA each); st_rows: rows
    // in flight per warp (4 or 8)
    int n_chunks = 0, ntiles = 0, st_rows = 4;
    const int* chunk_tile = nullptr;
    const int* chunk_p0 = nullptr;
    const int* chunk_p1 = nullptr;
    const int* tile_rows = nullptr;
    const int* tile_chunk_ptr = nullptr;
    T* xpart = nullptr;
    const int* perm = nullptr;
    const double* x_base = nullptr;  // when set, x_out = x_base + S^T S v (refinement form)
    int y_accumulate = 0;            // when set, y += S v instead of y = S v
    // y = S v by row groups (FP32 factors): unit u = the items of one group of at most kUnitRows rows that
    // share a column segment (unit_desc: first item, rows, first column, widest row's columns); one warp
    // reads the segment of v once for all rows.  use_units = 0 selects the one-warp-per-item kernel.
    // Rows cut into several items: the warp whose item of such a row finishes last sums the row's slot
    // partials in slot order into yrow[3 z] (z = the row's first slot), so that the S^T pass reads one value
    // per row.  item_rslots / unit_item_rslots: (first slot, end slot) of each item's row, in the launch order
    // of the item kernel and in emission order; row_cnt: per-row arrival counters indexed by z (zero between
    // applies: the last arrival resets its counter).  Null yrow keeps the S^T pass summing the slots itself.
    T* yrow = nullptr;
    unsigned int* row_cnt = nullptr;
    const int2* item_rslots = nullptr;
    const int2* unit_item_rslots = nullptr;
    int n_units = 0, use_units = 0;
    const int4* unit_desc = nullptr;
    const int4* unit_item_desc = nullptr;  // the items in emission order (a unit's rows are consecutive here)
    const int* unit_item_slot = nullptr;
};
constexpr int kSegCols = 2048;       // columns per S v work item
constexpr int kUnitRows = 8;         // rows per S v unit (the row-group cap of the item schedule)
constexpr int kChunkRows = 512;      // rows per S^T chunk CTA for large factors (64^3 contact block: 64 -> 512
                                     // rows took the FP32 pair from 4.05 to 3.60 ms)
constexpr int kChunkRowsSmall = 64;  // for factors of at most kChunkLargeValues values (more CTAs to fill the GPU)
constexpr long long kChunkLargeValues = 1ll << 28;
constexpr int kStChunkMax = 512;     // largest S^T chunk (its row descriptors are staged in shared memory)
constexpr int kGatherLanes = 8;      // lanes per node in the node gathers
constexpr int kGatherMaxThreads = 512;  // block-size bound of the node gathers

// Launch shapes spread evenly over the SMs: `threads` independent threads in at most `max_grid` blocks of at
// most `max_bs` threads (a multiple of 32), with the fewest blocks per SM that fit and equal-sized blocks, so
// that no SM holds a block more than the others (a partly filled last wave doubles a short kernel's time).
int device_sms();
// Programmatic dependent launch of the iteration-body kernels (default on; process-wide).  Graphs captured
// afterwards use the setting; already captured graphs keep theirs.
void set_pdl(bool on);
void even_grid(long long threads, int max_bs, int max_grid, int* grid, int* bs);
int gather_grid(int n);  // grid of the node gathers for n nodes (also the count of their per-block partials)
int gather_bs(int n);    // block size of the node gathers for n nodes

template <typename T>
void launch_sts(const SpmvPlan<T>& p, const T* v, T* y, double* x_out, const Ctrl* ctrl, cudaStream_t st);
// z = S^T S v (y = S v without its fix-up stage) whose last stage also performs the conjugate-gradient z-side
// update: r.z, |z|, beta and the stop rule, as launch_pcg_update2 over (r, z) would (p.y_accumulate must be 0).
template <typename T>
void launch_sts_cg(const SpmvPlan<T>& p, const T* v, double* z, const double* r, double* part, const double* mu_part,
                   int mu_blocks, Ctrl* ctrl, cudaStream_t st);


// Anderson acceleration + gate ------------------------------------------------------------------
void launch_aa_reduce(int n3, const double* x, const double* x_raw, const unsigned char* fixed_dof,
                      const double* fixed_val, double* dG, double* dX, double* last_g, double* last_x, int ld,
                      double* part, int blocks, Ctrl* ctrl, cudaStream_t st);
void launch_aa_update(int n3, double* x, const double* x_raw, const unsigned char* fixed_dof, const double* fixed_val,
                      const double* dG, const double* dX, int ld, double* part, const double* gate_part,
                      int gate_blocks, int blocks, Ctrl* ctrl, cudaStream_t st);

// Misc vector kernels
void launch_qtilde(int n3, const double* q, const double* v, const double* f_ext, double h, double h2m,
                   const double* grav_force, double* qt, cudaStream_t st);
void launch_velocity(int n3, const double* q_next, const double* q, double inv_h, double* v_next, cudaStream_t st);

// Adjoint ------------------------------------------------------------------------------------------
// Per-sample 9x9 local Jacobians J_s = sum_energies w (vol/s) dBp/dF at q_next (optionally eigen-filtered).
// With J32 set, also an FP32 packed symmetric copy (48 floats per sample) for the mixed-precision adjoint.
void launch_jac_build(int m, int k, int s, const int* E, const double* q, const double* grad, int hex,
                      double vol_over_s, const EnergyPack& ep, int mean_w, int filter, double* J, float* J32,
                      Ctrl* ctrl, cudaStream_t st);
// K_pd u element contributions from the cached Jacobians.
void launch_kpd_elem(int m, int k, int s, const int* E, const double* u, const double* grad, int hex, const double* J,
                     double* elem_out, const Ctrl* ctrl, cudaStream_t st);
void launch_kpd_elem32(int m, int k, int s, const int* E, const double* u, const double* grad, int hex,
                       const float* J32, double* elem_out, const Ctrl* ctrl, cudaStream_t st);
// rhs = gbar + K_pd u, Dirichlet rows zero, permuted SoA.
void launch_gather_bwd(int n, const int* node_ptr, const int* node_inc, const double* elem_out, const double* gbar,
                       const unsigned char* fixed_node, const int* iperm, double* v_perm, int npad, const Ctrl* ctrl,
                       cudaStream_t st);
// Parameter gradients at q_next for adjoint mu: per element and energy dl/dw_e = -(vol/s) sum_s mu_e^T A_s^T (F - Bp),
// the reference-style stress term, and the Neo-Hookean mean-parameter terms.
void launch_param_grad(int m, int k, int s, const int* E, const double* q, const double* mu, const double* grad,
                       int hex, double vol_over_s, const EnergyPack& ep, double* gw /* [energies][m] */,
                       double* gmat /* [energies][m] */, double* gnh /* [energies][m][2] */, cudaStream_t st);

// Preconditioned conjugate gradients for the adjoint (A - K_pd) mu = g_bar on the free DoFs, preconditioner
// A^-1 = S^T S.  Kernels of one iteration, in order: K p (launch_kpd_elem), w = (A - K) p and alpha,
// mu += alpha p / r -= alpha w (also the permuted right-hand side of the preconditioner), S^T S, r.z and the
// stop rule |z| < rtol |mu| + atol, p = z + beta p.
void launch_pcg_gather(int n, NodeCsr A, const double* p, const int* node_ptr, const int* node_inc,
                       const double* elem_out, const unsigned char* fixed_node, double* w, double* part, int blocks,
                       Ctrl* ctrl, cudaStream_t st, int init = 0);
template <typename T>
void launch_pcg_update1(int n, double* mu, double* r, const double* p, const double* w,
                        const unsigned char* fixed_node, const int* iperm, T* v_perm, int npad, double* part,
                        int blocks, Ctrl* ctrl, cudaStream_t st);
void launch_pcg_update2(int n3, const double* r, const double* z, double* part, const double* mu_part, int mu_blocks,
                        int blocks, Ctrl* ctrl, cudaStream_t st);
void launch_pcg_p(int n3, double* p, const double* z, const Ctrl* ctrl, cudaStream_t st);
// y += a x;  out = a - b
void launch_axpy(int n, double a, const double* x, double* y, cudaStream_t st);
void launch_sub(int n, const double* a, const double* b, double* out, cudaStream_t st);
// out = 2 a - b (linear extrapolation of the last two adjoints for the next solve's start)
void launch_extrapolate(int n3, const double* a, const double* b, double* out, cudaStream_t st);
// out = 3 (a - b) + c (quadratic extrapolation of the last three adjoints)
void launch_extrapolate3(int n3, const double* a, const double* b, const double* c, double* out, cudaStream_t st);
// out = 4 (a + c) - 6 b - d (cubic extrapolation of the last four adjoints)
void launch_extrapolate4(int n3, const double* a, const double* b, const double* c, const double* d, double* out,
                         cudaStream_t st);
// r = g_bar - w on free DoFs (0 on Dirichlet; w = (A - K_pd) mu_0 or null for mu_0 = 0), permuted right-hand
// side for the first preconditioner apply.
template <typename T>
void launch_pcg_init(int n, const double* gbar, const double* w, const unsigned char* fixed_node, const int* iperm,
                     double* r, T* v_perm, int npad, cudaStream_t st);

// Planar contact state on the device (see contact.cu).
struct ContactDev {
    int K = 0;                       // candidates (every listed boundary node, ascending)
    const int* cand = nullptr;       // node of each candidate
    double n[3] = {0, 0, 1}, t1[3] = {1, 0, 0}, t2[3] = {0, 1, 0};
    double offset = 0, mu = 0;
    const int64_t* off = nullptr;    // root-first S column paths of the candidates
    const int* prow = nullptr;
    const double* pval = nullptr;
    const double* G = nullptr;       // K x K node block of A^-1
    const double* rprec = nullptr;   // r_j = max(h^2 G_jj, 1e-10)
    double* lam = nullptr;           // normal multipliers (warm-started across frames)
    double* lt1 = nullptr;           // tangential multipliers (reset every frame)
    double* lt2 = nullptr;
    double* omega = nullptr;
    double* Ediag = nullptr;
    double* hvec = nullptr;
    int* act = nullptr;              // ordered active candidate list
    int* kact = nullptr;             // its length
    double* ainvb = nullptr;         // 3 per active candidate
    double* rhs = nullptr;           // kcap: right-hand side, then the forward-substituted y
    double* xsol = nullptr;          // kcap: the solution dlambda of the active system
    double* Mwork = nullptr;         // active system, kcap x kcap capacity (kcap = K rounded up to 64)
    unsigned int* bar = nullptr;     // grid barrier of the NCP solve: count, generation, abort
    // cached-factor solve (ncp_cached.cu): kcap = padded capacity; X = L_ref^-1 (lower) and its transpose for the
    // active list act_ref, with FP32 copies for the CG preconditioner; ref_pos[k] = the position of candidate k
    // in act_ref (-1: not in it), ref_inv[a] = the position of act_ref[a] in the current list (-1: dropped); CG
    // work vectors and per-CTA partials; flags (factor valid, its ka, candidates new to the list this launch);
    // stats (solves by the cached factor, refactorisations, CG iterations, CG attempts that fell back)
    size_t kcap = 0;
    double* Xinv = nullptr;
    double* Xt = nullptr;
    float* X32 = nullptr;
    float* Xt32 = nullptr;
    double* pcg = nullptr;
    int* act_ref = nullptr;
    int* ref_pos = nullptr;
    int* ref_inv = nullptr;
    int* ncp_flags = nullptr;
    unsigned long long* ncp_stats = nullptr;
    int cached = 1;                  // 1: the cached-factor solve, 0: a fresh factorisation every PD iteration
    double cg_tol = 1e-13;           // relative residual of the cached-factor CG
    // S v for v supported on the candidates, row by row: the rows of U (the union of the candidates' column
    // paths), each with its (candidate, S value) entries in candidate order
    int nU = 0;
    const int* tp_row = nullptr;     // nU: row of S
    const int64_t* tp_ptr = nullptr; // nU + 1
    const int* tp_k = nullptr;       // entries: candidate
    const double* tp_val = nullptr;  // entries: S[row, column of the candidate]
    double* vc = nullptr;            // 3 K: the S-pass input at the candidates after the NCP step (FP64)
};
template <typename T>
void launch_ncp_cached_solve(const ContactDev& c, const double* q0, const int* iperm, T* vcon, int npad,
                             const double* r64, Ctrl* ctrl, cudaStream_t st);
// The preconditioner of the contact-aware adjoint (contact_precond.cu): the three unit directions of the
// constraint basis, the parts of one application (stage 0: u = J A^-1 r from y = S r, lam = X^T X u per direction
// block; stage 1: the S-pass input -J^T lam), and the set-up gather of G_b with an identity X_b.
struct WbpDirs {
    double d[3][3];
};
template <typename T>
void launch_wbp_precond_parts(int stage, int cap, const int* count, const int* wcand, const int* wpos, const int* nb,
                              const ContactDev& c, const WbpDirs& dirs, const T* y, int npad, const double* X, int ld,
                              double* u, double* w, double* lam, double* vk, const Ctrl* ctrl, cudaStream_t st);
void launch_wbp_gather_g(int n, int n_pad, const int* idx, const double* G, int K, double* M, double* X, int ldx,
                         cudaStream_t st);
// Xt = transpose of the lower triangle of X (n x n, leading dimension ld)
void launch_wbp_transpose(int n, const double* X, double* Xt, int ld, cudaStream_t st);
// Dense Cholesky M = L L^T (n rows, a multiple of 64, identity-padded, ld n) with X <- L^-1 X (ldx, ncols), one
// cooperative grid (sfactor_gpu.cu); throws on a barrier timeout or a non-positive pivot.
void dense_chol_solve(double* M, int n, double* X, int ldx, int ncols, cudaStream_t st);
// Side of the padded active-system capacity for K candidates (K rounded up to the 64 x 64 tile).
size_t ncp_matrix_capacity(int K);
int ncp_grid();
void launch_delassus(int K, const int64_t* off, const int* prow, const double* pval, double* G, cudaStream_t st);
// One NCP iteration: y (T) holds S r for the iteration's right-hand side (S b in FP64; S (b - A x) in the
// FP32 refinement form, where x_base = x adds the current iterate back).  vcon (T) receives J^T f; with r64
// (FP64 r, refinement form) vcon is the S-pass input and receives r + J^T f at the candidates instead.
template <typename T>
void launch_ncp_iteration(const ContactDev& c, const double* x, const T* y, int npad, const double* x_base,
                          const double* q0, const int* iperm, T* vcon, const double* r64, Ctrl* ctrl,
                          cudaStream_t st);
// y_out = y_in + S v at the rows of U, v supported on the candidates (one warp per row, FP64 sums):
// v_k = v_src[3 cand[k] + d] (node order, from_nodes) or v_src[3 k + d].  y_in may alias y_out.
template <typename TI, typename TO>
void launch_path_apply(const ContactDev& c, const double* v_src, int from_nodes, const TI* y_in, TO* y_out, int npad,
                       const Ctrl* ctrl, cudaStream_t st);
// zero the candidates' entries of a permuted S-pass input
void launch_cand_zero(const ContactDev& c, const int* iperm, float* v, int npad, const Ctrl* ctrl, cudaStream_t st);
// the values of the row-wise path entries from the column paths (set-up)
void launch_path_gather_vals(long long E, const int64_t* src_e, const double* pval, double* tp_val, cudaStream_t st);
void launch_restitution(const ContactDev& c, double* q, const double* q0, const double* v0, double h, double e,
                        double slop, cudaStream_t st);
// y (+)= S v only (first half of the pair), and x = S^T y only (second half).
template <typename T>
void launch_s_only(const SpmvPlan<T>& p, const T* v, T* y, const Ctrl* ctrl, cudaStream_t st);
template <typename T>
void launch_st_only(const SpmvPlan<T>& p, const T* y, double* x_out, const Ctrl* ctrl, cudaStream_t st);

// Contact-aware material adjoint: projection of node vectors onto the complement of the constrained contact
// directions, candidate-node gather, and the |a - b|, |a|, |b| norms of a tape comparison.
template <typename T>
void launch_wb_project(int capacity, const int* count, const int* nodes, const double* dirs, const int* ndir,
                       double* u, T* vperm, const int* iperm, int npad, const Ctrl* ctrl, cudaStream_t st);
void launch_gather_nodes(int K, const int* cand, const double* u, double* out, cudaStream_t st);
void launch_diff_norms(int n, const double* a, const double* b, double* res, cudaStream_t st);

// Device construction of the sparse-inverse factor (sfactor_gpu.cu): fills the device-built supernodes' rows of
// d_vals (FP64, padded row layout; the small-subtree rows must already be there), then the FP32 copy.
struct SBuildPlan;
void device_build_factor(const SBuildPlan& P, const std::vector<int>& lo, const int64_t* d_ro, const int* d_ra,
                         const int* d_rl, double* d_vals, cudaStream_t st);
void device_round_f32(const double* d_in, float* d_out, long long n, cudaStream_t st);
void device_path_vals(int K, const int64_t* d_off, const int* d_prow, const int* d_cand, const int* d_iperm,
                      const double* d_vals, const int64_t* d_ro, const int* d_ra, double* d_pval, cudaStream_t st);

// Device-side loop control of a graph WHILE node: counts the iteration and keeps looping while the gate has
// not set `done` and fewer than `cap` iterations ran (cap > max_iter: a bound even if a gate kernel is skipped).
void launch_loop_cond(cudaGraphConditionalHandle h, Ctrl* ctrl, int cap, cudaStream_t st);

// Learned warm start (mlp.cu) -----------------------------------------------------------------------
struct FeatureArgs {
    int n = 0;
    const double* X = nullptr;             // rest positions
    const unsigned char* fixed = nullptr;  // per node
    const float* wlog = nullptr;           // log10 of the node's mean PD stiffness
    double inv_dx = 1, h = 0, h2m = 0;
    double gforce[3] = {0, 0, 0};          // m g
    int plane = 0;
    double pn[3] = {0, 0, 1}, poff = 0;
};
// Per-node MLP 15 -> 128 -> 128 -> 3 (mlp.cu).  `master` holds the FP32 weights in one flat array
// (W1 [16][128], W2 [128][128], W3 [128][8], b1 [128], b2 [128], b3 [8]); `packed` the BF16 operand copies.
int mlp_param_count();    // floats in `master` (= gradient length)
int mlp_packed_count();   // bf16 values in `packed`
int mlp_part_size();      // floats of one CTA's gradient partial
int mlp_rows_per_block(); // rows (nodes) per CTA
void mlp_pack_flat(float* master, void* packed, cudaStream_t st);
void mlp_forward_flat(float* master, void* packed, const void* X, int n, float* out, cudaStream_t st);
// Same network on tcgen05 MMAs (mlp_tc.cu): BF16 operands in shared memory, FP32 accumulators in TMEM; *err is
// set to 1 when a completion wait gave up (the outputs of that CTA's remaining rows are then not written).
void mlp_forward_tc_flat(float* master, void* packed, const void* X, int n, float* out, int* err, cudaStream_t st);
// Bound (polls) of the tcgen05 kernel's completion waits (0: every wait gives up at once); < 0 restores the
// default (4M).  Process-wide.
void set_mma_wait_polls(long long polls);
int mlp_train_flat(float* master, void* packed, const void* X, const float* Y, int n, float* part, cudaStream_t st);
void mlp_adamw_flat(float* master, void* packed, const float* part, int nblocks, float lr, float b1, float b2,
                    float eps, float wd, int step, float* m, float* v, float* grad_out, float* loss_out,
                    cudaStream_t st);
void launch_mlp_features(const FeatureArgs& a, const double* q, const double* qp, const double* v, const double* f,
                         const double* prev_base, const float* lam_node, void* X, double* base, cudaStream_t st);
// contact multipliers <-> the network: node-indexed feature column, training target column 3 of Y [n][4], and the
// predicted initial multipliers (scale = h^2 / (m dx))
void launch_mlp_lambda_nodes(int n, int K, const int* cand, const double* lam, double scale, float* lam_node,
                             cudaStream_t st);
void launch_mlp_target_lambda(int K, const int* cand, const double* lam, const double* lam_prev, double scale,
                              float* Y, cudaStream_t st);
void launch_mlp_lambda_apply(int K, const int* cand, const float* out, double inv_scale, double* lam, cudaStream_t st);
void launch_mlp_apply(int n3, const double* base, const float* out, double dx, const unsigned char* fixed_dof,
                      const double* fval, double* q_init, cudaStream_t st);
void launch_mlp_target(int n3, const double* q_next, const double* base, double inv_dx, float* Y, cudaStream_t st);
void launch_ws_contact_start(int K, int mode, const int* cand, const double* lam, const double* n, double off,
                             const unsigned char* fixed_dof, const double* q_prev, double* q_init, cudaStream_t st);

// Device-side adjoint routing (backward_gpu.cpp:881-917) and parameter-gradient reductions.
// g_bar = dl_dq_next + dl_dv_next / h;  dl_dq = -dl_dv_next / h;  |g_bar| into norm_out[0].
void launch_adj_prepare(int n3, const double* dl_dq_next, const double* dl_dv_next, double inv_h, double* gbar,
                        double* dl_dq, double* part, double* norm_out, cudaStream_t st);
// inj = s * inv_h2m * mu with s = min(1, (|g_bar| + 1) / |inj|) when cap is set; dl_dq += inj, dl_dv = h inj,
// dl_df = h2m inj, gravity parameter gradient (3 values) = sum over axis of h2m * inj * mass.
void launch_adj_route(int n3, const double* mu, double mu_norm, const double* gbar_norm, double inv_h2m, double h,
                      double h2m, double mass, int cap, int gravity, double* dl_dq, double* dl_dv, double* dl_df,
                      double* dl_dstate_p, double* part, unsigned int* arrive, cudaStream_t st);
// per energy: dl_dmat_w[k] = sum_e gmat[k][e]; dl_dparams from gw / gnh in the parameter layout of the energy.
void launch_param_reduce(int m, int ne, const int* np_k, const int* type_k, const int* off_k, const double* gw,
                         const double* gmat, const double* gnh, double* dl_dmat_w, double* dl_dparams,
                         cudaStream_t st);

}  // namespace dphd
