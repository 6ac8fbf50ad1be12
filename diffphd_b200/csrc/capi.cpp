// extern "C" boundary: status codes + thread-local last-error message, no exceptions across the ABI
// (the reference maps CheckError's ExceptionWithCallStack to a Python RuntimeError through SWIG,
// cpp/core/src/py_diff_pd_core.i:17-27; here the Python layer raises RuntimeError from the message).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "../../include/diffphd_b200.h"
#include "engine.h"

using dphd::Engine;
using dphd::Error;

struct dphd_deformable {
    Engine* eng;
};

namespace {
thread_local std::string g_last_error;

template <typename F>
int guard(F&& f) {
    try {
        g_last_error.clear();
        f();
        return 0;
    } catch (const Error& e) {
        g_last_error = e.what();
        return 1;
    } catch (const std::bad_alloc&) {
        g_last_error = "out of host memory";
        return 3;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 2;
    }
}

std::map<std::string, double> to_map(const char** keys, const double* vals, int n) {
    std::map<std::string, double> m;
    for (int i = 0; i < n; ++i) {
        DPHD_CHECK(keys && keys[i], "null option key");
        m[keys[i]] = vals[i];
    }
    return m;
}

void check_method(const char* method) {
    DPHD_CHECK(method != nullptr, "null method");
    const std::string s(method);
    DPHD_CHECK(s == "pd_eigen_alg_phd" || s == "pd_eigen_pcg_proj_gpu",
               "Unsupported method on this path: " + s + " (expected pd_eigen_alg_phd)");
}

Engine& E(dphd_deformable* h) {
    DPHD_CHECK(h && h->eng, "null deformable handle");
    return *h->eng;
}
const Engine& E(const dphd_deformable* h) {
    DPHD_CHECK(h && h->eng, "null deformable handle");
    return *h->eng;
}

// .bin reader (cpp/core/src/mesh/mesh.cpp:4-31, file_helper.cpp:169-184)
void read_bin(const char* path, int k_expect, std::vector<double>& verts, std::vector<int>& elems, int& n, int& m) {
    std::ifstream f(path, std::ios::binary);
    DPHD_CHECK(f.good(), std::string("Cannot open mesh file: ") + path);
    int vdim = 0, edim = 0, r = 0, c = 0;
    f.read((char*)&vdim, 4);
    f.read((char*)&edim, 4);
    DPHD_CHECK(f.good() && vdim == 3 && edim == k_expect, std::string("Corrupted mesh file: ") + path);
    f.read((char*)&r, 4);
    f.read((char*)&c, 4);
    DPHD_CHECK(f.good() && r == 3 && c > 0, "Inconsistent mesh matrix size.");
    std::vector<double> vt((size_t)r * c);
    f.read((char*)vt.data(), vt.size() * 8);
    n = c;
    verts.resize((size_t)3 * n);
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) verts[3 * i + d] = vt[(size_t)d * n + i];
    int r2 = 0, c2 = 0;
    f.read((char*)&r2, 4);
    f.read((char*)&c2, 4);
    DPHD_CHECK(f.good() && r2 == k_expect && c2 > 0, "Inconsistent mesh matrix size.");
    std::vector<int> et((size_t)r2 * c2);
    f.read((char*)et.data(), et.size() * 4);
    DPHD_CHECK(f.good(), std::string("Truncated mesh file: ") + path);
    m = c2;
    elems.resize((size_t)k_expect * m);
    for (int e = 0; e < m; ++e)
        for (int a = 0; a < k_expect; ++a) elems[(size_t)e * k_expect + a] = et[(size_t)a * m + e];
}
}  // namespace

extern "C" {

const char* dphd_last_error(void) { return g_last_error.c_str(); }

int dphd_create(int vertex_dim, int element_dim, dphd_deformable** out) {
    return guard([&] {
        DPHD_CHECK(out, "null output handle");
        *out = nullptr;
        auto* h = new dphd_deformable{nullptr};
        try {
            h->eng = new Engine(vertex_dim, element_dim);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int dphd_destroy(dphd_deformable* h) {
    return guard([&] {
        if (!h) return;
        delete h->eng;
        delete h;
    });
}

int dphd_init_from_bin(dphd_deformable* h, const char* bin_file, double density, const char* material_type,
                       double E_, double nu) {
    return guard([&] {
        Engine& e = E(h);
        std::vector<double> v;
        std::vector<int> el;
        int n = 0, m = 0;
        read_bin(bin_file, e.M.k, v, el, n, m);
        e.init_from_arrays(v.data(), n, el.data(), m, density, material_type ? material_type : "", E_, nu);
    });
}

int dphd_init_from_arrays(dphd_deformable* h, const double* verts, int n, const int* elems, int m, double density,
                          const char* material_type, double E_, double nu) {
    return guard([&] {
        DPHD_CHECK(verts && elems, "null mesh arrays");
        E(h).init_from_arrays(verts, n, elems, m, density, material_type ? material_type : "", E_, nu);
    });
}

int dphd_set_dirichlet(dphd_deformable* h, int dof, double val) {
    return guard([&] { E(h).set_dirichlet(dof, val); });
}

int dphd_add_pd_energy(dphd_deformable* h, const char* type, const double* params, int np, const int* idx,
                       int nidx) {
    return guard([&] {
        DPHD_CHECK(type && (params || np == 0) && (idx || nidx == 0), "null argument");
        E(h).add_pd_energy(type, params, np, idx, nidx);
    });
}

int dphd_add_state_force(dphd_deformable* h, const char* type, const double* params, int np) {
    return guard([&] {
        DPHD_CHECK(type && (params || np == 0), "null argument");
        E(h).add_state_force(type, params, np);
    });
}

int dphd_set_frictional_boundary(dphd_deformable* h, const char* type, const double* params, int np,
                                 const int* idx, int nidx) {
    return guard([&] {
        DPHD_CHECK(type && (params || np == 0) && (idx || nidx == 0), "null argument");
        E(h).set_frictional_boundary(type, params, np, idx, nidx);
    });
}

int dphd_dofs(const dphd_deformable* h) { return h && h->eng ? h->eng->dofs() : -1; }
int dphd_act_dofs(const dphd_deformable* h) { return h && h->eng ? 0 : -1; }
int dphd_num_pd_element_energies(const dphd_deformable* h) { return h && h->eng ? h->eng->num_pd_energies() : -1; }
int dphd_num_state_force_parameters(const dphd_deformable* h) {
    return h && h->eng ? h->eng->num_state_params() : -1;
}
int dphd_num_pd_params(const dphd_deformable* h) { return h && h->eng ? h->eng->num_pd_params() : -1; }

int dphd_forward(dphd_deformable* h, const char* method, const double* q, const double* v, const double* a,
                 const double* f_ext, double dt, const char** keys, const double* vals, int nopts, double* q_next,
                 double* v_next, int* active_idx, int* n_active) {
    (void)a;
    return guard([&] {
        check_method(method);
        DPHD_CHECK(q && v && f_ext && q_next && v_next, "null vector argument");
        DPHD_CHECK(dt > 0, "dt must be positive");
        const dphd::Options o = dphd::Options::parse(to_map(keys, vals, nopts));
        std::vector<int> act;
        E(h).forward(q, v, f_ext, dt, o, q_next, v_next, act);
        if (n_active) {
            DPHD_CHECK((int)act.size() <= *n_active || !active_idx, "active_idx capacity too small");
            for (size_t i = 0; i < act.size() && active_idx; ++i) active_idx[i] = act[i];
            *n_active = (int)act.size();
        }
    });
}

static int backward_impl(dphd_deformable* h, const char* method, const double* q, const double* v, const double* f,
                         double dt, const double* qn, const double* vn, const double* gq, const double* gv,
                         const char** keys, const double* vals, int nopts, double* dq, double* dv, double* df,
                         double* dmat, double* dstate, double* dparams) {
    return guard([&] {
        check_method(method);
        DPHD_CHECK(q && v && f && qn && vn && gq && gv && dq && dv && df, "null vector argument");
        DPHD_CHECK(dt > 0, "dt must be positive");
        Engine& e = E(h);
        const dphd::Options o = dphd::Options::parse(to_map(keys, vals, nopts));
        std::vector<double> mat(std::max(1, e.num_pd_energies())), st(3), par(std::max(1, e.num_pd_params()));
        e.backward(q, v, f, dt, qn, vn, gq, gv, o, dq, dv, df, mat.data(), par.data(), st.data());
        if (dmat)
            for (int i = 0; i < e.num_pd_energies(); ++i) dmat[i] = mat[i];
        if (dstate)
            for (int i = 0; i < e.num_state_params(); ++i) dstate[i] = st[i];
        if (dparams)
            for (int i = 0; i < e.num_pd_params(); ++i) dparams[i] = par[i];
    });
}

int dphd_backward(dphd_deformable* h, const char* method, const double* q, const double* v, const double* a,
                  const double* f_ext, double dt, const double* q_next, const double* v_next, const int* active_idx,
                  int n_active, const double* dl_dq_next, const double* dl_dv_next, const char** keys,
                  const double* vals, int nopts, double* dl_dq, double* dl_dv, double* dl_da, double* dl_df_ext,
                  double* dl_dmat_w, double* dl_dact_w, double* dl_dstate_p) {
    (void)a; (void)active_idx; (void)n_active; (void)dl_da; (void)dl_dact_w;
    return backward_impl(h, method, q, v, f_ext, dt, q_next, v_next, dl_dq_next, dl_dv_next, keys, vals, nopts,
                         dl_dq, dl_dv, dl_df_ext, dl_dmat_w, dl_dstate_p, nullptr);
}

int dphd_backward_ex(dphd_deformable* h, const char* method, const double* q, const double* v, const double* a,
                     const double* f_ext, double dt, const double* q_next, const double* v_next,
                     const int* active_idx, int n_active, const double* dl_dq_next, const double* dl_dv_next,
                     const char** keys, const double* vals, int nopts, double* dl_dq, double* dl_dv, double* dl_da,
                     double* dl_df_ext, double* dl_dmat_w, double* dl_dact_w, double* dl_dstate_p,
                     double* dl_dparams) {
    (void)a; (void)active_idx; (void)n_active; (void)dl_da; (void)dl_dact_w;
    return backward_impl(h, method, q, v, f_ext, dt, q_next, v_next, dl_dq_next, dl_dv_next, keys, vals, nopts,
                         dl_dq, dl_dv, dl_df_ext, dl_dmat_w, dl_dstate_p, dl_dparams);
}

int dphd_forward_device(dphd_deformable* h, const char* method, const double* d_q, const double* d_v,
                        const double* d_f, double dt, const char** keys, const double* vals, int nopts,
                        double* d_qn, double* d_vn, void* stream) {
    return guard([&] {
        check_method(method);
        DPHD_CHECK(d_q && d_v && d_f && d_qn && d_vn, "null device pointer");
        DPHD_CHECK(dt > 0, "dt must be positive");
        const dphd::Options o = dphd::Options::parse(to_map(keys, vals, nopts));
        E(h).forward_device(d_q, d_v, d_f, dt, o, d_qn, d_vn, (cudaStream_t)stream);
    });
}

int dphd_forward_device_init(dphd_deformable* h, const char* method, const double* d_q, const double* d_v,
                             const double* d_f, double dt, const char** keys, const double* vals, int nopts,
                             const double* d_q_init, double* d_qn, double* d_vn, void* stream) {
    return guard([&] {
        check_method(method);
        DPHD_CHECK(d_q && d_v && d_f && d_q_init && d_qn && d_vn, "null device pointer");
        DPHD_CHECK(dt > 0, "dt must be positive");
        const dphd::Options o = dphd::Options::parse(to_map(keys, vals, nopts));
        E(h).forward_device_init(d_q, d_v, d_f, dt, o, d_q_init, d_qn, d_vn, (cudaStream_t)stream);
    });
}

int dphd_set_warm_start_network(dphd_deformable* h, const float* d_master, const void* d_packed) {
    return guard([&] { E(h).set_ws_net(d_master, d_packed); });
}

int dphd_num_contact_candidates(const dphd_deformable* h) {
    return h && h->eng ? h->eng->contact_candidates() : -1;
}

int dphd_contact_lambda_device(dphd_deformable* h, double* d_lambda, int set, void* stream) {
    return guard([&] {
        DPHD_CHECK(d_lambda || E(h).contact_candidates() == 0, "null device pointer");
        E(h).contact_lambda_device(d_lambda, set != 0, (cudaStream_t)stream);
    });
}

int dphd_mlp_sizes(int* n_master, int* n_packed, int* part_floats_per_block, int* rows_per_block) {
    return guard([&] {
        if (n_master) *n_master = dphd::mlp_param_count();
        if (n_packed) *n_packed = dphd::mlp_packed_count();
        if (part_floats_per_block) *part_floats_per_block = dphd::mlp_part_size();
        if (rows_per_block) *rows_per_block = dphd::mlp_rows_per_block();
    });
}

int dphd_mlp_pack(float* d_master, void* d_packed, void* stream) {
    return guard([&] {
        DPHD_CHECK(d_master && d_packed, "null device pointer");
        dphd::mlp_pack_flat(d_master, d_packed, (cudaStream_t)stream);
        CUDA_OK(cudaGetLastError());
    });
}

int dphd_mlp_forward(float* d_master, void* d_packed, const void* d_X, int n, float* d_out, void* stream) {
    return guard([&] {
        DPHD_CHECK(d_master && d_packed && d_X && d_out, "null device pointer");
        DPHD_CHECK(n >= 0, "negative row count");
        dphd::mlp_forward_flat(d_master, d_packed, d_X, n, d_out, (cudaStream_t)stream);
        CUDA_OK(cudaGetLastError());
    });
}

int dphd_mlp_forward_tc(float* d_master, void* d_packed, const void* d_X, int n, float* d_out, int* d_err,
                        void* stream) {
    return guard([&] {
        DPHD_CHECK(d_master && d_packed && d_X && d_out && d_err, "null device pointer");
        DPHD_CHECK(n >= 0, "negative row count");
        DPHD_CHECK(((uintptr_t)d_X & 15) == 0 && ((uintptr_t)d_out & 15) == 0 && ((uintptr_t)d_packed & 15) == 0,
                   "packed weights, X and out must be 16-byte aligned");
        dphd::mlp_forward_tc_flat(d_master, d_packed, d_X, n, d_out, d_err, (cudaStream_t)stream);
        CUDA_OK(cudaGetLastError());
    });
}

int dphd_mlp_train_step(float* d_master, void* d_packed, const void* d_X, const float* d_Y, int n, float* d_part,
                        float lr, float beta1, float beta2, float eps, float weight_decay, int step, float* d_m,
                        float* d_v, float* d_grad, float* d_loss, void* stream) {
    return guard([&] {
        DPHD_CHECK(d_master && d_packed && d_X && d_Y && d_part && d_m && d_v, "null device pointer");
        DPHD_CHECK(n > 0, "empty training batch");
        DPHD_CHECK(step >= 1, "AdamW step counter starts at 1");
        const cudaStream_t st = (cudaStream_t)stream;
        const int blocks = dphd::mlp_train_flat(d_master, d_packed, d_X, d_Y, n, d_part, st);
        dphd::mlp_adamw_flat(d_master, d_packed, d_part, blocks, lr, beta1, beta2, eps, weight_decay, step, d_m, d_v,
                             d_grad, d_loss, st);
        CUDA_OK(cudaGetLastError());
    });
}

int dphd_warmstart_features(dphd_deformable* h, double dt, const double* d_q, const double* d_q_prev,
                            const double* d_v, const double* d_f, const double* d_prev_base, void* d_X,
                            double* d_base, void* stream) {
    return guard([&] {
        DPHD_CHECK(d_q && d_q_prev && d_v && d_f && d_X && d_base, "null device pointer");
        E(h).ws_features(dt, d_q, d_q_prev, d_v, d_f, d_prev_base, d_X, d_base, (cudaStream_t)stream);
        CUDA_OK(cudaGetLastError());
    });
}

int dphd_warmstart_apply(dphd_deformable* h, double dt, const double* d_base, const float* d_out, double* d_q_init,
                         void* stream) {
    return guard([&] {
        DPHD_CHECK(d_base && d_out && d_q_init, "null device pointer");
        E(h).ws_apply(dt, d_base, d_out, d_q_init, (cudaStream_t)stream);
        CUDA_OK(cudaGetLastError());
    });
}

int dphd_warmstart_target(dphd_deformable* h, double dt, const double* d_q_next, const double* d_base, float* d_Y,
                          void* stream) {
    return guard([&] {
        DPHD_CHECK(d_q_next && d_base && d_Y, "null device pointer");
        E(h).ws_target(dt, d_q_next, d_base, d_Y, (cudaStream_t)stream);
        CUDA_OK(cudaGetLastError());
    });
}

int dphd_backward_device(dphd_deformable* h, const char* method, const double* d_q_next, const double* d_dl_dq_next,
                         const double* d_dl_dv_next, double dt, const char** keys, const double* vals, int nopts,
                         double* d_dl_dq, double* d_dl_dv, double* d_dl_df_ext, double* d_dl_dmat_w,
                         double* d_dl_dparams, double* d_dl_dstate_p, void* stream) {
    return guard([&] {
        check_method(method);
        DPHD_CHECK(d_q_next && d_dl_dq_next && d_dl_dv_next && d_dl_dq && d_dl_dv && d_dl_df_ext,
                   "null device pointer");
        DPHD_CHECK(dt > 0, "dt must be positive");
        const dphd::Options o = dphd::Options::parse(to_map(keys, vals, nopts));
        E(h).backward_device(d_q_next, d_dl_dq_next, d_dl_dv_next, dt, o, d_dl_dq, d_dl_dv, d_dl_df_ext,
                             d_dl_dmat_w, d_dl_dparams, d_dl_dstate_p, (cudaStream_t)stream);
    });
}

int dphd_reset_warm_start(dphd_deformable* h) {
    return guard([&] { E(h).reset_warm_start(); });
}

int dphd_debug_set_mma_wait_polls(long long polls) {
    return guard([&] { dphd::set_mma_wait_polls(polls); });
}
int dphd_debug_set_factor_build(dphd_deformable* h, int mode, int small_subtree_max) {
    return guard([&] { E(h).set_factor_build(mode, small_subtree_max); });
}
int dphd_debug_set_st_schedule(dphd_deformable* h, int chunk_rows, int rows_in_flight) {
    return guard([&] { E(h).set_st_schedule(chunk_rows, rows_in_flight); });
}
int dphd_contact_path_stats(dphd_deformable* h, long long* entries, int* rows, int* max_depth) {
    return guard([&] {
        DPHD_CHECK(entries && rows && max_depth, "contact path stats: null pointer");
        E(h).contact_path_stats(entries, rows, max_depth);
    });
}
int dphd_factor_built_on_device(const dphd_deformable* h) {
    return h && h->eng ? h->eng->factor_built_on_device() : -1;
}
int dphd_device(const dphd_deformable* h) { return h && h->eng ? h->eng->device() : -2; }

long long dphd_kernel_launches(const dphd_deformable* h) { return h && h->eng ? h->eng->kernel_launches() : -1; }

int dphd_debug_time_ainv(dphd_deformable* h, double dt, int reps, int fp32, int flush_l2, double* ms_per_apply) {
    return guard([&] {
        DPHD_CHECK(ms_per_apply && reps > 0, "bad arguments");
        *ms_per_apply = E(h).time_ainv(dt, reps, fp32 != 0, flush_l2 != 0);
    });
}

int dphd_debug_set_s_kernel(dphd_deformable* h, int row_groups) {
    return guard([&] { E(h).set_s_units(row_groups != 0); });
}

int dphd_debug_set_pdl(dphd_deformable* h, int on) {
    return guard([&] {
        dphd::set_pdl(on != 0);
        E(h).drop_captured_graphs();
    });
}

int dphd_ainv_noalloc(dphd_deformable* h, double dt, const double* d_b, double* d_x, int fp32, void* stream) {
    return guard([&] { E(h).ainv_noalloc(dt, d_b, d_x, fp32 != 0, (cudaStream_t)stream); });
}

long long dphd_s_padded_values(const dphd_deformable* h) { return h && h->eng ? h->eng->s_padded_values() : -1; }

int dphd_num_frames(const dphd_deformable* h) {
    return h && h->eng ? (int)h->eng->stats.frame_iters.size() : -1;
}
int dphd_frame_stats(const dphd_deformable* h, int* it, int* cv) {
    return guard([&] {
        const Engine& e = E(h);
        for (size_t i = 0; i < e.stats.frame_iters.size(); ++i) {
            if (it) it[i] = e.stats.frame_iters[i];
            if (cv) cv[i] = e.stats.frame_converged[i];
        }
    });
}
int dphd_reset_frame_stats(dphd_deformable* h) {
    return guard([&] {
        E(h).stats.frame_iters.clear();
        E(h).stats.frame_converged.clear();
    });
}
int dphd_backward_fallbacks(const dphd_deformable* h) { return h && h->eng ? h->eng->stats.bwd_fallbacks : -1; }
int dphd_warm_start_state(dphd_deformable* h, double* d_buf, int* valid, int set, void* stream) {
    return guard([&] { E(h).ws_state(d_buf, valid, set != 0, static_cast<cudaStream_t>(stream)); });
}
int dphd_ncp_solve_stats(dphd_deformable* h, long long* cached, long long* refactors, long long* cg_iters,
                         long long* cg_fallbacks) {
    return guard([&] { E(h).ncp_stats(cached, refactors, cg_iters, cg_fallbacks); });
}
int dphd_fp64_escalations(const dphd_deformable* h) { return h && h->eng ? h->eng->stats.fp64_escalations : -1; }
int dphd_last_backward_iters(const dphd_deformable* h) { return h && h->eng ? h->eng->stats.last_bwd_iters : -1; }
int dphd_last_filtered_samples(const dphd_deformable* h) {
    return h && h->eng ? h->eng->stats.last_filtered : -1;
}
int dphd_contact_adjoint_stats(const dphd_deformable* h, int* source, int* constraints, int* iters) {
    return guard([&] {
        DPHD_CHECK(h && h->eng, "null handle");
        const auto& st = h->eng->stats;
        if (source) *source = st.contact_source;
        if (constraints) *constraints = st.contact_constraints;
        if (iters) *iters = st.contact_iters;
    });
}
long long dphd_s_memory_bytes(const dphd_deformable* h) { return h && h->eng ? h->eng->s_memory_bytes() : -1; }
long long dphd_s_nnz(const dphd_deformable* h) { return h && h->eng ? h->eng->s_nnz() : -1; }

int dphd_debug_s_rows(dphd_deformable* h, double dt, int* row_lo, int* perm) {
    return guard([&] {
        dphd::Engine& e = E(h);
        DPHD_CHECK(e.M.n > 0, "Deformable is not initialized.");
        dphd::init_samples(e.M);
        const dphd::NodeMatrix A = dphd::assemble_A(e.M, dt);
        const std::vector<int> order = dphd::nested_dissection(e.M, A);
        dphd::SFactor S;
        dphd::build_sfactor(A, order, S, 0);
        for (int i = 0; i < S.n; ++i) {
            if (row_lo) row_lo[i] = S.lo[i];
            if (perm) perm[i] = S.perm[i];
        }
    });
}

int dphd_debug_ainv(dphd_deformable* h, double dt, const double* b, double* x, int fp32) {
    return guard([&] { E(h).apply_ainv(dt, b, x, fp32 != 0); });
}
int dphd_debug_host_sts(dphd_deformable* h, double dt, const double* b, double* x) {
    return guard([&] { E(h).host_sts_apply(dt, b, x); });
}
int dphd_debug_local_step(dphd_deformable* h, double dt, const double* q, double* rhs) {
    return guard([&] { E(h).local_step(dt, q, rhs); });
}

}  // extern "C"
