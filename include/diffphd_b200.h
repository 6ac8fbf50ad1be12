/*
 * diffphd_b200 — C ABI of the B200 (sm_100a) projective-dynamics time step and its adjoint.
 *
 * Drop-in boundary for DiffPhD's `Deformable<3,8>` / `Deformable<3,4>` on the "pd_eigen_alg_phd" path.
 * Every entry point returns 0 on success and a non-zero status otherwise; the message of the last error
 * on the calling thread is returned by dphd_last_error().  No C++ exception crosses this boundary.
 * Vectors are node-major interleaved xyz, FP64 (the layout of the reference's q, v, f_ext).
 * Option dictionaries are passed as parallel arrays of keys and values (the reference's
 * std::map<std::string, real>, converted from a Python dict by common.py:195-200 `to_std_map`).
 */
#ifndef DIFFPHD_B200_H
#define DIFFPHD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dphd_deformable dphd_deformable;

/* Message of the last failed call on this thread (empty string when none). */
const char* dphd_last_error(void);

/* Replaces the HexDeformable()/TetDeformable() constructors (cpp/core/src/py_diff_pd_core.i:60-68;
 * Deformable<vertex_dim, element_dim>, cpp/core/include/fem/deformable.h:17-21).
 * vertex_dim must be 3; element_dim 8 (hex) or 4 (tet). */
int dphd_create(int vertex_dim, int element_dim, dphd_deformable** out);
int dphd_destroy(dphd_deformable* h);

/* Deformable::Initialize(bin_file, density, material_type, E, nu) (deformable.h:24-28).
 * Only material_type "none" is accepted on this path (elasticity comes from AddPdEnergy). */
int dphd_init_from_bin(dphd_deformable* h, const char* bin_file, double density, const char* material_type,
                       double youngs_modulus, double poissons_ratio);
/* Deformable::Initialize(vertices, elements, ...) (deformable.h:26-28); verts: n*3 FP64 node-major,
 * elems: m*element_dim int32. */
int dphd_init_from_arrays(dphd_deformable* h, const double* verts, int n, const int* elems, int m, double density,
                          const char* material_type, double youngs_modulus, double poissons_ratio);

/* Deformable::SetDirichletBoundaryCondition(dof, val) (deformable.h:70-73). */
int dphd_set_dirichlet(dphd_deformable* h, int dof, double val);
/* Deformable::AddPdEnergy(type, params, indices) (cpp/core/src/fem/deformable_pd_energy.cpp:43-153);
 * type "corotated" | "volume" (params: 1 or element_num values) | "pd_neohookean" (params: [mu, la] or
 * 2*element_num interleaved); nidx == 0 means every element. */
int dphd_add_pd_energy(dphd_deformable* h, const char* type, const double* params, int nparams, const int* indices,
                       int nidx);
/* Deformable::AddStateForce("gravity", [gx, gy, gz]) (cpp/core/src/fem/deformable_state_force.cpp:10-20). */
int dphd_add_state_force(dphd_deformable* h, const char* type, const double* params, int nparams);
/* Deformable::SetFrictionalBoundary("planar", [nx, ny, nz, offset], node_indices)
 * (cpp/core/src/fem/deformable_friction.cpp:7-31). */
int dphd_set_frictional_boundary(dphd_deformable* h, const char* type, const double* params, int nparams,
                                 const int* indices, int nidx);

/* Accessors (deformable.h:45-64): dofs(), act_dofs(), NumOfPdElementEnergies(), NumOfStateForceParameters();
 * dphd_num_pd_params is the total length of all AddPdEnergy parameter arrays (size of dl_dparams). */
int dphd_dofs(const dphd_deformable* h);
int dphd_act_dofs(const dphd_deformable* h);
int dphd_num_pd_element_energies(const dphd_deformable* h);
int dphd_num_state_force_parameters(const dphd_deformable* h);
int dphd_num_pd_params(const dphd_deformable* h);

/* Deformable::PyForward(method, q, v, a, f_ext, dt, options, q_next&, v_next&, active_contact_idx&)
 * (deformable.h:132-134; AlgPhd implementation forward_gpu.cpp:387-1594).  method: "pd_eigen_alg_phd" or
 * its alias "pd_eigen_pcg_proj_gpu".  active_idx: capacity *n_active on input, count on output. */
int dphd_forward(dphd_deformable* h, const char* method, const double* q, const double* v, const double* a,
                 const double* f_ext, double dt, const char** opt_keys, const double* opt_vals, int nopts,
                 double* q_next, double* v_next, int* active_idx, int* n_active);

/* Deformable::PyBackward(method, q, v, a, f_ext, dt, q_next, v_next, active_contact_idx, dl_dq_next,
 * dl_dv_next, options, dl_dq&, dl_dv&, dl_da&, dl_df_ext&, dl_dmat_w&, dl_dact_w&, dl_dstate_p&)
 * (deformable.h:135-141; AlgPhd implementation backward_gpu.cpp:648-1250). */
int dphd_backward(dphd_deformable* h, const char* method, const double* q, const double* v, const double* a,
                  const double* f_ext, double dt, const double* q_next, const double* v_next, const int* active_idx,
                  int n_active, const double* dl_dq_next, const double* dl_dv_next, const char** opt_keys,
                  const double* opt_vals, int nopts, double* dl_dq, double* dl_dv, double* dl_da, double* dl_df_ext,
                  double* dl_dmat_w, double* dl_dact_w, double* dl_dstate_p);
/* Extension of dphd_backward: also returns dl_dparams, the gradient w.r.t. every AddPdEnergy parameter
 * array concatenated in call order (per-element stiffnesses, or interleaved [mu_e, la_e]); the reference
 * only returns one scalar per energy (dl_dmat_w). */
int dphd_backward_ex(dphd_deformable* h, const char* method, const double* q, const double* v, const double* a,
                     const double* f_ext, double dt, const double* q_next, const double* v_next,
                     const int* active_idx, int n_active, const double* dl_dq_next, const double* dl_dv_next,
                     const char** opt_keys, const double* opt_vals, int nopts, double* dl_dq, double* dl_dv,
                     double* dl_da, double* dl_df_ext, double* dl_dmat_w, double* dl_dact_w, double* dl_dstate_p,
                     double* dl_dparams);

/* Device-pointer forward step: q, v, f_ext, q_next, v_next are device pointers (3n FP64) and the step is
 * enqueued on `stream` (a cudaStream_t, NULL = legacy default).  Same semantics as dphd_forward. */
int dphd_forward_device(dphd_deformable* h, const char* method, const double* d_q, const double* d_v,
                        const double* d_f_ext, double dt, const char** opt_keys, const double* opt_vals, int nopts,
                        double* d_q_next, double* d_v_next, void* stream);

/* Device-pointer adjoint step (BackwardProjectiveDynamicsAlgPhd, backward_gpu.cpp:648-1250, contact-free): reads
 * q_next, dl_dq_next, dl_dv_next (device, 3n FP64) and writes dl_dq, dl_dv, dl_df_ext (device, 3n) and, when
 * non-null, dl_dmat_w (device, #energies), dl_dparams (device, dphd_num_pd_params) and dl_dstate_p (device, 3). */
int dphd_backward_device(dphd_deformable* h, const char* method, const double* d_q_next, const double* d_dl_dq_next,
                         const double* d_dl_dv_next, double dt, const char** opt_keys, const double* opt_vals,
                         int nopts, double* d_dl_dq, double* d_dl_dv, double* d_dl_df_ext, double* d_dl_dmat_w,
                         double* d_dl_dparams, double* d_dl_dstate_p, void* stream);

/* Clears the frame-to-frame warm start of the contact multipliers (the reference keeps them in
 * alg_phd_prev_lambda_, forward_gpu.cpp:1074-1084, 1544-1545, across every later call). */
int dphd_reset_warm_start(dphd_deformable* h);

/* Number of kernels this library launched on the GPU since the handle was created (graph nodes included). */
long long dphd_kernel_launches(const dphd_deformable* h);
/* Bound, in polls, of the completion waits of the tcgen05 warm-start inference kernel (default 4M; 0 makes every
 * wait give up at once; < 0 restores the default; process-wide).  A wait that runs out sets the kernel's error flag, drains the MMAs in flight, frees its
 * TMEM and returns; the forward step then fails with an error.  For failure-path tests.  No counterpart in the
 * reference. */
int dphd_debug_set_mma_wait_polls(long long polls);
/* Where the sparse-inverse factor S is built (the reference builds it on the host from an LDL^T and uploads it,
 * forward_gpu.cpp:593-764): 0 automatic (on the device when S has more than 32 Mi values, else on the host),
 * 1 host, 2 device (rows of etree subtrees of at most small_subtree_max nodes, 512 when <= 0, on the host; every
 * larger separator chain on the GPU from the Schur complement of its descendants).  Takes effect at the next
 * factor build.  No counterpart in the reference. */
int dphd_debug_set_factor_build(dphd_deformable* h, int mode, int small_subtree_max);
/* Schedule of the x = S^T y pass: rows of a column tile's row list per CTA (chunk_rows, 8..512; by default 512 for factors above 2^28 values, else 64) and
 * rows each warp keeps in flight (4 or 8, default 4).  Changes the order of the partial sums, so results differ
 * at the rounding level between schedules.  Takes effect at the next factor build.  No counterpart in the
 * reference. */
int dphd_debug_set_st_schedule(dphd_deformable* h, int chunk_rows, int rows_in_flight);
/* The contact candidates' S column paths (after the factor build): total entries, rows of their union (the
 * rows a path product S v writes for v supported on the candidates), longest path.  Zeros without a contact
 * plane.  No counterpart in the reference. */
int dphd_contact_path_stats(dphd_deformable* h, long long* entries, int* rows, int* max_depth);
/* 1 when the current factor was built on the device, 0 on the host, -1 for a null handle. */
int dphd_factor_built_on_device(const dphd_deformable* h);
/* CUDA device that holds this handle's GPU state: -1 until the first call that builds the factor (it records
 * the device current then), -2 for a null handle.  Later calls made while another device is current fail with
 * an error instead of mixing pointers of two devices.  No counterpart in the reference (fixed to device 0,
 * forward_gpu.cpp:579). */
int dphd_device(const dphd_deformable* h);

/* Per-frame statistics (AlgPhdFrameIters / AlgPhdFrameConverged / AlgPhdResetFrameStats,
 * cpp/core/include/fem/alg_phd_gpu_memory.h:25-27; forward_gpu.cpp:324-332). */
int dphd_num_frames(const dphd_deformable* h);
int dphd_frame_stats(const dphd_deformable* h, int* frame_iters, int* frame_converged);
int dphd_reset_frame_stats(dphd_deformable* h);
int dphd_last_backward_iters(const dphd_deformable* h);
/* The learned start's frame-to-frame state: *valid (a previous step exists) and, when valid, the previous step's
 * q and q_tilde in d_buf (device, 2 * 3n FP64), copied out (set = 0) or restored (set = 1) on `stream`.  A
 * checkpointed rollout saves it with each checkpoint (with the contact multipliers) so that recomputing a segment
 * repeats the forward pass exactly.  No counterpart in the reference. */
int dphd_warm_start_state(dphd_deformable* h, double* d_buf, int* valid, int set, void* stream);
/* The NCP's dense solves since the contact set-up (option ncp_solver 1, the default; ncp_solver 0 factors at
 * every PD iteration as the reference does, forward_gpu.cpp:1238-1240): solves by conjugate gradients
 * preconditioned with the cached factor of an earlier PD iteration's system of the same frame (its active list
 * may differ by a few candidates), fresh factorisations, the CG iterations of all cached solves, and the CG
 * attempts that did not converge and fell back to a factorisation.  Any pointer may be NULL.  No counterpart in
 * the reference. */
int dphd_ncp_solve_stats(dphd_deformable* h, long long* cached, long long* refactors, long long* cg_iters,
                         long long* cg_fallbacks);
/* Mixed-precision forward frames (option fp32_bulk) whose FP32 iteration stalled and that finished in FP64 from
 * the FP32 iterate, since the handle was created (option fp32_stall_window: iterations without the gate ratio
 * halving, default 40; 0 never switches).  No counterpart in the reference. */
int dphd_fp64_escalations(const dphd_deformable* h);
/* Adjoint solves that left the conjugate-gradient solver for the reference fixed point (negative curvature of
 * A - K_pd) or, in the contact-aware solve, for the unconstrained adjoint, since the handle was created.  No
 * counterpart in the reference. */
int dphd_backward_fallbacks(const dphd_deformable* h);
/* Samples whose 9x9 local Hessian the last backward call eigen-filtered (option bwd_eigen_filter 1 clamp /
 * 2 absolute value; the diagonal-dominance test of ProjectedNewtonMatrix, deformable_newton_forward.cpp:394-434). */
int dphd_last_filtered_samples(const dphd_deformable* h);
/* The last backward call's contact-aware material adjoint (backward_gpu.cpp:937-1208): where its contact frame
 * came from (0 none / skipped by option, 1 the forward tape, 2 a replayed forward step, 3 a tape miss on the
 * device-pointer entry, which has no q, v to replay from: material gradients then use the plain adjoint),
 * the number of contact basis constraints kept, and the conjugate-gradient iterations of the constrained solve. */
int dphd_contact_adjoint_stats(const dphd_deformable* h, int* source, int* constraints, int* iters);
/* AlgPhdSMemoryBytes / AlgPhdSNnz (forward_gpu.cpp:302-315): bytes of the S factor in HBM and its nnz. */
long long dphd_s_memory_bytes(const dphd_deformable* h);
long long dphd_s_nnz(const dphd_deformable* h);
/* Stored S values including the 16-byte alignment padding of each row segment. */
long long dphd_s_padded_values(const dphd_deformable* h);

/* Selects the kernel of the FP32 y = S v pass: 1 one warp per row group of up to 8 rows that share a column
 * segment (v read once per group); 0 one warp per row segment.  Both give bit-identical sums; by default the
 * faster one on the factor is chosen by timing both when the factor is built.  Captured iteration graphs are
 * dropped.  No counterpart in the reference (profiling and A/B timing). */
int dphd_debug_set_s_kernel(dphd_deformable* h, int row_groups);
/* Programmatic dependent launch of the kernels inside the iteration graphs (1, the default: each kernel may
 * launch while its predecessor drains and waits for it on the device; 0: plain stream order).  The setting is
 * process-wide; this handle's captured graphs are dropped so that they are captured again with it.  No
 * counterpart in the reference (A/B timing). */
int dphd_debug_set_pdl(dphd_deformable* h, int on);
/* x = A^-1 b through the S^T S pair on device pointers (b, x: 3n FP64 node-major; Dirichlet rows of b are
 * taken as zero, as in the forward step), allocating no GPU memory: its temporaries live in a static 32 MiB
 * device array instead.  No counterpart in the reference.  For callers that cannot call cudaMalloc during a
 * step (a fixed memory budget, a host framework that owns the allocator, or no implicit device syncs).
 * Requires the factor for this dt to be on the device already (one earlier allocating call on the handle);
 * fails with a clear error when the mesh needs more scratch than the array holds.  All calls share the
 * array: calls that overlap on the GPU race and must be serialised by the caller.  The first call on a
 * device looks up the array's address; make it before any stream capture.  That cached address is not valid
 * across a cudaDeviceReset in the same process.  The handle's device (dphd_device) must be current. */
int dphd_ainv_noalloc(dphd_deformable* h, double dt, const double* d_b, double* d_x, int fp32, void* stream);

/* Contact candidates of the frictional boundary (0 without one; -1 before the first forward call builds them)
 * and their normal multipliers lambda, the warm start the reference carries across frames
 * (forward_gpu.cpp:1074-1084): copied to (set = 0) or from (set = 1) a device array of that length.  A
 * checkpointed rollout saves them with each checkpoint so that recomputing a segment repeats the forward. */
int dphd_num_contact_candidates(const dphd_deformable* h);
int dphd_contact_lambda_device(dphd_deformable* h, double* d_lambda, int set, void* stream);

/* ---- Learned warm start (no counterpart in the reference: the reference starts every PD loop from q). ----
 * A forward step whose PD loop starts from d_q_init (3n FP64) instead of q.  The loop still runs to the same
 * dual gate, so the start only changes the iteration count, never the accepted fixed point's tolerance. */
int dphd_forward_device_init(dphd_deformable* h, const char* method, const double* d_q, const double* d_v,
                             const double* d_f, double dt, const char** keys, const double* vals, int nopts,
                             const double* d_q_init, double* d_q_next, double* d_v_next, void* stream);
/* Attach a trained warm-start network to the deformable (device pointers in the dphd_mlp_* layout below;
 * copied, so the caller may free them), or detach it (d_master = null).  While attached, dphd_forward and
 * dphd_forward_device start every PD loop from q_tilde + dx * MLP(features) (features from this and the
 * previous forward call's state, kept by the handle and cleared by dphd_reset_warm_start) instead of q, and
 * still run it to the same dual gate: drop-in for the reference's PyForward, with only the iteration count
 * changed. */
int dphd_set_warm_start_network(dphd_deformable* h, const float* d_master, const void* d_packed);
/* Per-node MLP 15 -> 128 -> 128 -> 3 (GELU), BF16 tensor-core kernels with FP32 accumulation.
 * d_master: FP32 weights in one flat array (W1 [16][128], W2 [128][128], W3 [128][8], b1 [128], b2 [128],
 * b3 [8]; row 15 of W1 and columns 3..7 of W3/b3 are unused and kept at zero by training);
 * d_packed: the BF16 operand copies (dphd_mlp_pack writes them).  Inputs X are BF16 [n][16]; outputs FP32
 * [n][8] (columns 0..2 used). */
int dphd_mlp_sizes(int* n_master, int* n_packed, int* part_floats_per_block, int* rows_per_block);
int dphd_mlp_pack(float* d_master, void* d_packed, void* stream);
int dphd_mlp_forward(float* d_master, void* d_packed, const void* d_X, int n, float* d_out, void* stream);
/* The same inference on the 5th-generation tensor cores (tcgen05.mma, BF16 operands in shared memory, FP32
 * accumulators in tensor memory); the engine's warm start uses it unless the option ws_tcgen05 = 0.  d_err: one
 * device int the caller zeroes; the kernel sets it to 1 if a tensor-core completion wait gave up (bounded
 * wait; the rows that CTA had not finished are then left unwritten).  d_packed, d_X and d_out 16-byte aligned. */
int dphd_mlp_forward_tc(float* d_master, void* d_packed, const void* d_X, int n, float* d_out, int* d_err,
                        void* stream);
/* One training step on rows [0, n): loss = sum over rows and the 3 outputs of (pred - Y)^2 / n (Y: FP32
 * [n][3]); d_part holds ceil(n / rows_per_block) * part_floats_per_block floats of per-block gradient
 * partials, summed in a fixed order (deterministic); AdamW (bias-corrected, decoupled decay on weights only)
 * updates d_master and re-packs d_packed.  lr = 0 computes the gradient only.  d_grad (n_master floats) and
 * d_loss (1 float) may be null. */
int dphd_mlp_train_step(float* d_master, void* d_packed, const void* d_X, const float* d_Y, int n, float* d_part,
                        float lr, float beta1, float beta2, float eps, float weight_decay, int step, float* d_m,
                        float* d_v, float* d_grad, float* d_loss, void* stream);
/* Features of every node for one step (BF16 [n][16]: (q - X)/dx, (q - q_prev)/dx, the previous step's
 * correction (q - q_tilde_prev)/dx (zero when d_prev_base is null), h^2 f_ext/(m dx), signed height above the
 * contact plane / dx, log10(mean stiffness)/7, Dirichlet flag, 0) and the inertial prediction
 * q_tilde = q + h v + h^2/m (f_ext + m g) (3n FP64, d_base).  dx = cube root of the mean element volume.  Builds
 * the handle's factor for this dt first if no forward call has. */
int dphd_warmstart_features(dphd_deformable* h, double dt, const double* d_q, const double* d_q_prev,
                            const double* d_v, const double* d_f, const double* d_prev_base, void* d_X,
                            double* d_base, void* stream);
/* q_init = q_tilde + dx * out[:, :3] (Dirichlet dofs take their fixed values). */
int dphd_warmstart_apply(dphd_deformable* h, double dt, const double* d_base, const float* d_out, double* d_q_init,
                         void* stream);
/* Training target Y = (q_next - q_tilde) / dx (FP32 [n][3]). */
int dphd_warmstart_target(dphd_deformable* h, double dt, const double* d_q_next, const double* d_base, float* d_Y,
                          void* stream);

/* Diagnostics used by the tests: x = A^-1 b through the GPU S^T S pair (fp32 = 0 or 1), the same product
 * with the host copy of S (the set-up self-check of forward_gpu.cpp:653-670), and the GPU local step
 * (ProjectiveDynamicsLocalStep, deformable_projective_dynamics_forward.cpp:186-292). */
int dphd_debug_ainv(dphd_deformable* h, double dt, const double* b, double* x, int fp32);
/* Host-only structure of the sparse inverse factor (no GPU needed): per S row its first column lo_i (row i is
 * dense on [lo_i, i]) and the node at each permuted position. */
int dphd_debug_s_rows(dphd_deformable* h, double dt, int* row_lo, int* perm);
int dphd_debug_host_sts(dphd_deformable* h, double dt, const double* b, double* x);
int dphd_debug_local_step(dphd_deformable* h, double dt, const double* q, double* rhs);
/* Average device time (ms, CUDA events on the library's stream) of one S^T S pair over `reps` applications,
 * optionally writing 256 MB between applications so that S is not served from L2. */
int dphd_debug_time_ainv(dphd_deformable* h, double dt, int reps, int fp32, int flush_l2, double* ms_per_apply);

#ifdef __cplusplus
}
#endif
#endif /* DIFFPHD_B200_H */
