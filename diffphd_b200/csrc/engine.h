// Engine: one Deformable<3,k> on one GPU — builder state, the sparse-inverse factor in HBM, and the
// forward / adjoint drivers of the projective-dynamics step.
#pragma once
#include <cuda_runtime.h>

#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "dphd_internal.h"
#include "kernels.cuh"

#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e__ = (x);                                                                        \
        if (e__ != cudaSuccess)                                                                       \
            throw ::dphd::Error(std::string("CUDA error: ") + cudaGetErrorString(e__) + " at " +      \
                                __FILE__ + ":" + std::to_string(__LINE__));                           \
    } while (0)

namespace dphd {

struct Options {
    int max_pd_iter = 0;
    double abs_tol = 0, rel_tol = 0;
    int verbose = 0, thread_ct = 0;
    int aa_window = 5;
    double friction_mu = 0, restitution = 0, contact_slop = 1e-8;
    double bwd_clip = 1e6;
    int bwd_mean_stiffness = 0;  // reference backward semantics: mean stiffness inside K_pd
    int bwd_cascade_cap = 1;     // reference cap of the injected adjoint at |g_bar| + 1
    int bwd_eigen_filter = 0;    // 0 off (exact adjoint), 1 clamp, 2 abs
    int debug_force_bwd_fallback = 0;  // take the CG -> fixed-point fallback path (failure-path tests)
    int bwd_contact_precond = 1; // contact-aware adjoint preconditioner: 1 exact inverse of A on the constrained
                                 // subspace (Woodbury with the Delassus block), 0 P A^-1 P
    int fp32_bulk = 0;           // projection and S/S^T SpMVs in FP32
    int bwd_solver = 0;          // 0: Anderson-accelerated fixed point (reference), 1: preconditioned CG
    int bwd_warm_start = 0;      // CG adjoint starts from the previous backward call's solution (reverse sweeps)
    // contact-aware material adjoint (backward_gpu.cpp:937-1208)
    int skip_woodbury = 0, skip_material_grad = 0, basis_topk = 0;
    double tangent_lambda_min = 1e-8, rhs_prune_rel = 1e-3, rhs_prune_abs = 1e-12;
    int poll_chunk = 8;
    int graph_while = 1;         // device-side WHILE graph per solve (0: host polling every poll_chunk iterations)
    int ws_tcgen05 = 1;          // warm-start inference on tcgen05 MMAs with TMEM accumulators (0: mma.sync)
    int ncp_solver = 1;          // NCP dense solve: 1 CG preconditioned by a cached factor (refactored when the
                                 // active list changes or CG stalls), 0 a fresh Cholesky every PD iteration
    double ncp_cg_tol = 1e-13;   // relative residual of the cached-factor CG (1e-10 measured slower on the 64^3
                                 // contact rollout: inexact steps leave multipliers just above 0, and the active
                                 // list, hence the cached factor, changes more often)
    int ws_contact_start = 0;    // with a warm-start network and contact: 1 keeps the previous gap of the
                                 // candidates in contact and lifts predicted penetrations to the plane; 2 keeps
                                 // the candidates in contact at their previous positions
    int ws_lambda = 0;           // with a warm-start network and contact: 1 starts each frame's NCP from the
                                 // network's predicted multipliers instead of the previous frame's (measured
                                 // slower on the 64^3 contact rollout, so off by default)
    int fp32_projection = -1;    // mixed precision: 1 FP32 local projections, 0 FP64 projections with FP32 S
                                 // passes, -1 automatic (FP32 without a contact set, FP64 with one)
    int fp32_stall_window = 40;  // mixed precision: iterations without the gate ratio halving before the rest of
                                 // the frame continues in FP64 (0: never)
    static Options parse(const std::map<std::string, double>& m);
};

struct DeviceBuffer {
    void* p = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { release(); }
    void release();
    void alloc(size_t b);
    template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
    template <typename T> void upload(const std::vector<T>& v) {
        alloc(v.size() * sizeof(T));
        if (!v.empty()) copy_in(v.data(), v.size() * sizeof(T));
    }
    void copy_in(const void* src, size_t b);
};

struct StepStats {
    std::vector<int> frame_iters, frame_converged;
    int fp64_escalations = 0;  // mixed-precision frames finished in FP64 after the FP32 iteration stalled
    int last_bwd_iters = 0, last_filtered = 0, bwd_fallbacks = 0;
    // last backward's contact-aware material adjoint: frame source (0 no contact / skipped by option,
    // 1 forward tape, 2 replayed forward step, 3 tape miss without replay inputs), constraints, CG iterations
    int contact_source = 0, contact_constraints = 0, contact_iters = 0;
};

// One forward contact frame kept for the adjoint (the reference's AlgPhdReplayCache): the step's output and,
// per candidate, the final normal multiplier and the last NCP iteration's omega.
struct TapeFrame {
    DeviceBuffer q_sol, lam, omega;
};

class Engine {
public:
    Engine(int vertex_dim, int element_dim);
    ~Engine();

    // builder (mirrors Deformable's Python-facing API)
    void init_from_arrays(const double* verts, int n, const int* elems, int m, double density,
                          const std::string& material, double E, double nu);
    void set_dirichlet(int dof, double val);
    void add_pd_energy(const std::string& type, const double* params, int np, const int* idx, int nidx);
    void add_state_force(const std::string& type, const double* params, int np);
    void set_frictional_boundary(const std::string& type, const double* params, int np, const int* idx, int nidx);

    int dofs() const { return 3 * M.n; }
    int num_pd_energies() const { return (int)M.energies.size(); }
    int num_pd_params() const;
    int num_state_params() const { return M.has_gravity ? 3 : 0; }
    long long s_memory_bytes() const;
    long long s_nnz() const { return S.nnz(); }
    long long s_padded_values() const { return (long long)(d_vals64.bytes / sizeof(double)); }
    int num_nodes() const { return M.n; }
    int s_depth() const { return S.max_depth; }

    // host-pointer step (drop-in for PyForward / PyBackward)
    void forward(const double* q, const double* v, const double* f_ext, double dt, const Options& o, double* q_next,
                 double* v_next, std::vector<int>& active);
    void backward(const double* q, const double* v, const double* f_ext, double dt, const double* q_next,
                  const double* v_next, const double* dl_dq_next, const double* dl_dv_next, const Options& o,
                  double* dl_dq, double* dl_dv, double* dl_df, double* dl_dmat_w, double* dl_dparams,
                  double* dl_dstate_p);
    // device-pointer step (inputs and outputs already in HBM, launched on `stream`)
    void forward_device(const double* d_q, const double* d_v, const double* d_f, double dt, const Options& o,
                        double* d_q_next, double* d_v_next, cudaStream_t stream);

    // forward step whose PD iteration starts from d_q_init instead of q (the learned warm start)
    void forward_device_init(const double* d_q, const double* d_v, const double* d_f, double dt, const Options& o,
                             const double* d_q_init, double* d_q_next, double* d_v_next, cudaStream_t stream);
    // warm-start features / application / training targets (see mlp.cu)
    void ws_features(double dt, const double* d_q, const double* d_qp, const double* d_v, const double* d_f,
                     const double* d_prev_base, void* X, double* d_base, cudaStream_t st);
    void ws_apply(double dt, const double* d_base, const float* out, double* d_q_init, cudaStream_t st);
    void ws_target(double dt, const double* d_q_next, const double* d_base, float* Y, cudaStream_t st);
    double ws_dx() const;
    double ws_lambda_scale(double dt) const;  // h^2 / (m dx): contact multipliers in the network's scale
    // Attach a trained warm-start network (device pointers; copied into engine memory) or detach (null): while
    // attached, every forward step whose caller gives no initial guess starts its PD loop from the network's
    // prediction.  The previous step's q and q_tilde are engine state (reset by reset_warm_start).
    void set_ws_net(const float* d_master, const void* d_packed);
    // contact candidates and their normal multipliers (the lambda warm start carried across frames)
    int contact_candidates() const;
    void contact_lambda_device(double* d_buf, bool set, cudaStream_t st);
    // NCP solves by the cached factor and refactorisations since the contact set-up
    void ncp_stats(long long* cached, long long* refactors, long long* cg_iters, long long* cg_fallbacks);
    bool ws_net_attached() const { return ws_net_; }
    // the learned start's frame-to-frame state (whether a previous step exists, its q and its q_tilde): copied to
    // (set = false) or from (set = true) a device array of 2 * 3n doubles, so that a checkpointed rollout can
    // recompute a segment exactly as the forward pass ran it
    void ws_state(double* d_buf, int* valid, bool set, cudaStream_t st);
    // selects the row-group or the one-warp-per-item kernel of the FP32 y = S v pass (overriding the choice
    // timed at factor build); drops the captured iteration graphs
    void set_s_units(bool on);
    void drop_captured_graphs() { drop_graphs(); }

    void backward_device(const double* d_q_next, const double* d_gq, const double* d_gv, double dt, const Options& o,
                         double* d_dq, double* d_dv, double* d_df, double* d_dmat_w, double* d_dparams,
                         double* d_dstate_p, cudaStream_t stream);
    // time `reps` applications of the S^T S pair on the device; returns ms per application
    double time_ainv(double dt, int reps, bool fp32, bool flush_l2);
    long long kernel_launches() const { return launches_; }
    // how the sparse-inverse factor is built: 0 automatic (on the device above kDeviceBuildNnz values, on the
    // host below), 1 host, 2 device; a change takes effect at the next factor build
    void set_factor_build(int mode, int small_subtree_max);
    // the S^T pass's schedule: rows per chunk CTA and rows in flight per warp (4 or 8); takes effect at the next
    // factor build
    void set_st_schedule(int chunk_rows, int rows_in_flight);
    // the candidates' S column paths: total entries, rows of their union, longest path (0 without contact)
    void contact_path_stats(long long* entries, int* rows, int* max_depth) const {
        *entries = has_contact_ ? path_entries_ : 0;
        *rows = has_contact_ ? contact_.nU : 0;
        *max_depth = has_contact_ ? path_max_depth_ : 0;
    }
    int factor_built_on_device() const { return factor_on_device_ ? 1 : 0; }
    static constexpr long long kDeviceBuildNnz = 32ll << 20;
    // CUDA device that holds this handle's GPU state (-1 until the first call that builds it); every later
    // call must be made with that device current
    int device() const { return device_; }

    // contact state: normal multipliers of the planar candidates (the frame-to-frame warm start)
    void reset_warm_start();
    std::vector<double> contact_lambda();
    int num_contact_candidates() const { return (int)M.contact_nodes.size(); }

    // x = A^-1 b on device pointers without allocating (temporaries in a static device array); the factor
    // for this dt must already be built by an earlier (allocating) call on this handle.
    void ainv_noalloc(double dt, const double* d_b, double* d_x, bool fp32, cudaStream_t stream);

    // diagnostics used by the tests
    void apply_ainv(double dt, const double* b, double* x, bool fp32);
    void host_sts_apply(double dt, const double* b, double* x);
    void local_step(double dt, const double* q, double* rhs);

    StepStats stats;
    HostModel M;

private:
    void ensure_built(double dt, int threads);
    void build_device(int threads);
    EnergyPack energy_pack() const;
    void run_forward_loop(const double* d_q, double h, const Options& o, cudaStream_t st,
                          const double* d_init = nullptr);
    void launch_ainv(bool fp32, cudaStream_t st, const double* x_base = nullptr);  // d_vperm -> d_xraw
    void enqueue_pcg_iteration(bool fp32, cudaStream_t st, bool projected = false, bool woodbury = false);
    // x_raw = the contact-aware adjoint's preconditioner applied to the permuted S-pass input (P A^-1 P without
    // the constrained-inverse correction, or the exact inverse of A on the constrained subspace with it)
    void enqueue_contact_precond(bool fp32, bool woodbury, cudaStream_t st);
    void backward_core(const double* d_q_next, const double* d_gq, const double* d_gv, double dt, const Options& o,
                       double* d_dq, double* d_dv, double* d_df, double* d_dmat_w, double* d_dparams,
                       double* d_dstate_p, cudaStream_t st, const double* d_q, const double* d_v, const double* d_f);
    // forward contact tape
    std::deque<std::unique_ptr<TapeFrame>> tape_;
    std::vector<std::unique_ptr<TapeFrame>> tape_free_;
    void tape_push(const double* d_q_next, cudaStream_t st);
    bool tape_take(const double* d_q_next, std::unique_ptr<TapeFrame>& out, cudaStream_t st);
    void replay_step(const double* d_q, const double* d_v, const double* d_f, double dt, const Options& o,
                     cudaStream_t st);
    void contact_adjoint(const Options& o, const TapeFrame& fr, cudaStream_t st);
    DeviceBuffer d_wb_nodes, d_wb_dirs, d_wb_ndir, d_wb_count, d_wb_gath, d_wb_mu, d_cmp, d_rq, d_rv;
    DeviceBuffer d_z1;  // constraint correction z - mu of the last contact-aware adjoint of a reverse sweep
    // constrained-inverse preconditioner: per constrained node its candidate and its position in each direction's
    // block, the block sizes, the blocks' inverse Cholesky factors, work vectors and the sparse S-pass input
    DeviceBuffer d_wbp_cand, d_wbp_pos, d_wbp_nb, d_wbp_idx, d_wbp_X, d_wbp_M, d_wbp_u, d_wbp_w, d_wbp_lam, d_wbp_vk;
    WbpDirs wbp_dirs_ = {};
    int z_hist_ = 0;
    double* h_cmp_ = nullptr;
    void enqueue_contact_iteration(cudaStream_t st, bool f32);
    void enqueue_contact_iteration64(cudaStream_t st);
    void build_contact(double dt);
    void enqueue_fwd_iteration(bool fp32, cudaStream_t st);
    void enqueue_bwd_iteration(cudaStream_t st);
    // mode 0 fwd64, 1 fwd mixed, 2 adjoint fixed point, 3 adjoint PCG (FP64 preconditioner), 4 PCG (FP32 precond.)
    void run_iterations(int mode, const Options& o, cudaStream_t st);
    void drop_graphs();
    void check_status(const char* where);
    void check_device() const;
    int device_ = -1;
    int factor_mode_ = 0, small_subtree_max_ = 512;
    int st_chunk_rows_ = 0, st_rows_ = 4;  // chunk rows 0: by the factor's size
    bool proj32_ = true;  // precision of the projections captured in the mixed-precision iteration graphs
    // the contact-adjoint preconditioner's direction factors X_b: the G they were built from (generation of the
    // contact set-up) and their constrained candidates, reused while both are unchanged
    long long contact_gen_ = 0, wbp_gen_[3] = {-1, -1, -1};
    long long path_entries_ = 0;  // entries of the candidates' S column paths; their longest path
    int path_max_depth_ = 0;
    std::vector<int> wbp_idx_prev_[3];
    bool factor_on_device_ = false;
    std::unique_ptr<SBuildPlan> sb_plan_;   // device build: plan and the permuted upper triangle of A, kept from
    std::unique_ptr<PermUpper> sb_upper_;   // the symbolic step until build_device runs the numeric one

    bool built_ = false;
    double built_dt_ = -1;
    SFactor S;
    NodeMatrix A;
    int npad_ = 0, ntiles_ = 0, red_blocks_ = 1, gather_blocks_ = 1;
    double graph_dt_ = -1, graph_mu_ = 0;
    // 0 fwd64, 1 fwd mixed, 2 adjoint fixed point, 3/4 CG adjoint f64/f32, 5 contact f64, 6/7 projected CG
    // f64/f32, 8 contact mixed
    // 9/10 projected CG f64/f32 with the constrained-inverse preconditioner
    static constexpr int kModes = 11;
    cudaGraphExec_t graphs_[kModes] = {};
    size_t graph_nodes_[kModes] = {};
    bool graph_is_while_[kModes] = {};
    int graph_cap_[kModes] = {};
    bool while_ok_ = true;
    void enqueue_iteration(int mode, cudaStream_t cap);
    bool build_while_graph(int mode, int cap_iters);
    ContactDev contact_;
    bool has_contact_ = false;
    NodeCsr Acsr_;
    long long launches_ = 0;
    SpmvPlan<double> plan64_;
    SpmvPlan<float> plan32_;
    bool device_ready_ = false;
    cudaStream_t stream_ = nullptr;

    DeviceBuffer dE, dX, dgrad, d_elem_dir, d_fixed_node, d_fixed_dof, d_fixed_val, d_qb;
    DeviceBuffer d_node_ptr, d_node_inc, d_perm, d_iperm;
    DeviceBuffer d_row_off, d_row_a, d_row_len, d_vals64, d_vals32, d_tile_ptr, d_tile_rows;
    DeviceBuffer d_short_rows, d_grp_row0, d_grp_g, d_chunk_tile, d_chunk_p0, d_chunk_p1, d_tile_chunk_ptr;
    DeviceBuffer d_xpart64, d_xpart32, d_ypart64, d_ypart32, d_row_item_ptr, d_row_items;
    DeviceBuffer d_w[kMaxEnergies], d_w32[kMaxEnergies], d_mask[kMaxEnergies];
    DeviceBuffer d_q, d_v, d_f, d_qt, d_x, d_xraw, d_prev_pd, d_dG, d_dX, d_lg, d_lx;
    DeviceBuffer d_part_gate, d_part_aa, d_part_upd, d_gravf;
    DeviceBuffer d_elem_out64, d_elem_out32, d_vperm64, d_vperm32, d_y64, d_y32;
    DeviceBuffer d_qn, d_vn, d_gbar, d_J, d_gw, d_gmat, d_gnh;
    DeviceBuffer d_ctrl, d_adjnorm, d_part_adj, d_np_k, d_type_k, d_off_k, d_dmat_dev, d_dpar_dev, d_dstate_dev;
    DeviceBuffer d_item_desc, d_item_slot, d_trow_desc, d_trow_off, d_J32;
    DeviceBuffer d_unit_desc, d_unit_item_desc, d_unit_item_slot;  // row-group units of the FP32 y = S v pass
    DeviceBuffer d_item_rslots, d_unit_item_rslots, d_row_cnt, d_yrow32, d_yrow64;  // multi-item row totals
    bool s_units_ = false;       // chosen by timing both kernels when the factor is built
    DeviceBuffer d_gq, d_gv, d_dq, d_dv, d_df, d_A_rp, d_A_ci, d_A_v, d_r, d_pp, d_wv, d_wlog, d_mu_prev;
    bool mu_prev_valid_ = false, mu_prev2_valid_ = false, mu_prev3_valid_ = false, mu_prev4_valid_ = false;
    DeviceBuffer d_mu_prev2, d_mu_prev3, d_mu_prev4;  // the adjoints before d_mu_prev (bwd_warm_start 2-4)
    const double* ws_predict(const double* d_q, const double* d_v, const double* d_f, double dt, bool tcgen05,
                             cudaStream_t st);
    bool ws_net_ = false, ws_prev_valid_ = false;
    int ws_which_ = 0;
    DeviceBuffer d_ws_master, d_ws_packed, d_ws_X, d_ws_out, d_ws_base0, d_ws_base1, d_ws_qprev, d_ws_qinit;
    DeviceBuffer d_ws_err;       // set by the tcgen05 inference kernel when a tensor-core wait gave up
    DeviceBuffer d_ws_lamnode;   // node-indexed contact multipliers (the lambda feature)
    DeviceBuffer d_ws_lamprev;   // the multipliers at the last features call (the training target's baseline)
    bool ws_lambda_ = true;
    int ws_contact_start_ = 0;
    int* h_ws_err_ = nullptr;    // pinned copy, read after the forward loop's synchronisation
    DeviceBuffer dc_cand, dc_off, dc_prow, dc_pval, dc_G, dc_rprec, dc_lam, dc_lt1, dc_lt2, dc_omega, dc_E, dc_h,
        dc_act, dc_kact, dc_ainvb, dc_rhs, dc_xsol, dc_bar, dc_M, d_vcon, d_r64, d_q0, dc_Xinv, dc_Xt, dc_pcg,
        dc_actref, dc_flags, dc_stats, dc_X32, dc_Xt32, dc_refpos, dc_refinv, dc_tprow, dc_tpptr, dc_tpk, dc_tpval,
        dc_vc;
    Ctrl* h_ctrl_ = nullptr;  // pinned mirror
};

}  // namespace dphd
