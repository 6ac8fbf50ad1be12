// Forward and adjoint drivers of the B200 projective-dynamics step.
//
// Forward (ForwardProjectiveDynamicsAlgPhd, cpp/core/src/fem/deformable_projective_dynamics_forward_gpu.cpp:387-1594,
// contact-free branch): q_tilde, then PD iterations  pd = local_step(q); q_raw = A^-1 (m/h^2 q_tilde + pd)
// with Dirichlet rows zeroed; Dirichlet reset; Type-II Anderson acceleration; dual gate
// |dq| <= rtol |q_prev| + atol and |d pd| <= rtol |pd_prev| + atol for iter > 0.  Every iteration is six
// kernels on one stream; the stop decision is taken on the device and polled every `poll_chunk` iterations.
//
// Adjoint (BackwardProjectiveDynamicsAlgPhd, deformable_projective_dynamics_backward_gpu.cpp:648-917): the
// backbone fixed point mu <- A^-1 (g_bar + K_pd mu) with the same acceleration, then the downstream routing
// to dl/dq, dl/dv, dl/df_ext and the gravity parameters, and per-element parameter gradients.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <set>
#include <type_traits>

#include "engine.h"

namespace dphd {

void DeviceBuffer::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}
void DeviceBuffer::alloc(size_t b) {
    if (b == bytes && p) return;
    release();
    if (b == 0) return;
    CUDA_OK(cudaMalloc(&p, b));
    bytes = b;
}
void DeviceBuffer::copy_in(const void* src, size_t b) { CUDA_OK(cudaMemcpy(p, src, b, cudaMemcpyHostToDevice)); }

Options Options::parse(const std::map<std::string, double>& m) {
    Options o;
    for (const char* req : {"max_pd_iter", "abs_tol", "rel_tol", "verbose", "thread_ct"})
        DPHD_CHECK(m.count(req), std::string("Missing option ") + req + ".");
    o.max_pd_iter = (int)m.at("max_pd_iter");
    o.abs_tol = m.at("abs_tol");
    o.rel_tol = m.at("rel_tol");
    o.verbose = (int)m.at("verbose");
    o.thread_ct = (int)m.at("thread_ct");
    auto get = [&](const char* k, double def) { return m.count(k) ? m.at(k) : def; };
    o.aa_window = (int)get("aa_window", 5);
    o.friction_mu = get("friction_mu", 0);
    o.restitution = get("restitution", 0);
    o.contact_slop = get("friction_contact_slop", 1e-8);
    o.bwd_clip = get("alg_phd_bwd_clip_norm", 1e6);
    o.bwd_mean_stiffness = (int)get("bwd_mean_stiffness", 0);
    o.bwd_cascade_cap = (int)get("bwd_cascade_cap", 1);
    o.bwd_eigen_filter = (int)get("bwd_eigen_filter", 0);
    o.bwd_contact_precond = (int)get("bwd_contact_precond", 1);
    o.debug_force_bwd_fallback = (int)get("debug_force_bwd_fallback", 0);
    o.fp32_bulk = (int)get("fp32_bulk", 0);
    o.bwd_solver = (int)get("alg_phd_bwd_solver", 0);
    o.bwd_warm_start = (int)get("alg_phd_bwd_warm_start", 0);
    o.skip_woodbury = get("skip_contact_woodbury", 0) > 0.5;
    o.skip_material_grad = get("skip_material_grad", 0) > 0.5;
    o.tangent_lambda_min = get("alg_phd_bwd_tangent_lambda_min", 1e-8);
    o.rhs_prune_rel = get("alg_phd_bwd_rhs_prune_rel", 1e-3);
    o.rhs_prune_abs = get("alg_phd_bwd_rhs_prune_abs", 1e-12);
    o.basis_topk = (int)get("alg_phd_bwd_basis_topk", 0);
    o.poll_chunk = std::max(1, (int)get("poll_chunk", 8));
    o.graph_while = (int)get("graph_while", 1);
    o.ws_tcgen05 = (int)get("ws_tcgen05", 1);
    o.fp32_stall_window = std::max(0, (int)get("fp32_stall_window", 40));
    o.fp32_projection = (int)get("fp32_projection", -1);
    o.ws_lambda = (int)get("ws_lambda", 0);
    o.ws_contact_start = (int)get("ws_contact_start", 0);
    o.ncp_solver = (int)get("ncp_solver", 1);
    o.ncp_cg_tol = get("ncp_cg_tol", 1e-13);
    DPHD_CHECK(o.ncp_cg_tol > 0.0 && o.ncp_cg_tol < 1.0, "ncp_cg_tol must lie in (0, 1)");
    DPHD_CHECK(o.aa_window >= 0 && o.aa_window <= kMaxWindow,
               "aa_window must be in [0, " + std::to_string(kMaxWindow) + "]");
    DPHD_CHECK(o.max_pd_iter > 0, "max_pd_iter must be positive.");
    return o;
}

Engine::Engine(int vertex_dim, int element_dim) {
    DPHD_CHECK(vertex_dim == 3, "Only 3D deformables (vertex_dim = 3) are supported on this path.");
    DPHD_CHECK(element_dim == 8 || element_dim == 4, "element_dim must be 8 (hex) or 4 (tet).");
    M.k = element_dim;
    M.hex = element_dim == 8;
    M.s = M.hex ? 8 : 1;
}

void Engine::drop_graphs() {
    for (auto& g : graphs_)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

Engine::~Engine() {
    drop_graphs();
    if (h_ctrl_) cudaFreeHost(h_ctrl_);
    if (h_cmp_) cudaFreeHost(h_cmp_);
    if (h_ws_err_) cudaFreeHost(h_ws_err_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Engine::init_from_arrays(const double* verts, int n, const int* elems, int m, double density,
                              const std::string& material, double E, double nu) {
    (void)E;
    (void)nu;
    DPHD_CHECK(material == "none",
               "Only material 'none' (elasticity from AddPdEnergy) is supported on the AlgPhd path; got '" +
                   material + "'.");
    DPHD_CHECK(n > 0 && m > 0, "Empty mesh.");
    M.n = n;
    M.m = m;
    M.X.assign(verts, verts + 3 * (size_t)n);
    M.E.assign(elems, elems + (size_t)m * M.k);
    for (int v : M.E) DPHD_CHECK(v >= 0 && v < n, "Element references a vertex out of range.");
    M.density = density;
    double sum = 0;
    for (int e = 0; e < m; ++e) sum += element_volume(M, e);
    M.vol = sum / m;
    init_samples(M);
    built_ = false;
}

void Engine::set_dirichlet(int dof, double val) {
    DPHD_CHECK(dof >= 0 && dof < dofs(), "Dirichlet dof out of range.");
    if (!M.dirichlet.count(dof)) built_ = false;
    M.dirichlet[dof] = val;
    device_ready_ = false;
}

void Engine::add_pd_energy(const std::string& type, const double* params, int np, const int* idx, int nidx) {
    DPHD_CHECK(M.n > 0, "Initialize the mesh before adding energies.");
    DPHD_CHECK((int)M.energies.size() < kMaxEnergies, "At most 4 PD element energies are supported.");
    PdEnergy en;
    if (type == "corotated") en.type = kCorotated;
    else if (type == "volume") en.type = kVolume;
    else if (type == "pd_neohookean") en.type = kNeoHookean;
    else throw Error("Unsupported PD energy: " + type);
    en.params.assign(params, params + np);
    if (en.type != kNeoHookean) {
        DPHD_CHECK(np == 1 || np == M.m, "Inconsistent param size: expected 1 (homogeneous) or element_num=" +
                                             std::to_string(M.m) + " (per-element), got " + std::to_string(np));
        if (np == 1) {
            en.w_mean = params[0];
        } else {
            en.w_elem.assign(params, params + np);
            en.w_mean = std::accumulate(en.w_elem.begin(), en.w_elem.end(), 0.0) / np;
        }
    } else {
        DPHD_CHECK(np == 2 || np == 2 * M.m, "pd_neohookean expects params = [mu, lambda] or per-element "
                                             "[mu_1, la_1, ..., mu_n, la_n] of length 2*element_num=" +
                                                 std::to_string(2 * M.m) + ", got " + std::to_string(np));
        if (np == 2) {
            en.mu = params[0];
            en.la = params[1];
            en.w_mean = 2 * params[0];
        } else {
            double sm = 0, sl = 0;
            en.w_elem.resize(M.m);
            for (int e = 0; e < M.m; ++e) {
                sm += params[2 * e];
                sl += params[2 * e + 1];
                en.w_elem[e] = 2 * params[2 * e];
            }
            en.mu = sm / M.m;
            en.la = sl / M.m;
            en.w_mean = std::accumulate(en.w_elem.begin(), en.w_elem.end(), 0.0) / M.m;
        }
    }
    en.all_elements = (nidx == 0);
    en.in_set.assign(M.m, en.all_elements ? 1 : 0);
    for (int i = 0; i < nidx; ++i) {
        DPHD_CHECK(idx[i] >= 0 && idx[i] < M.m, "Element index out of bound.");
        en.in_set[idx[i]] = 1;
    }
    M.energies.push_back(en);
    built_ = false;
}

void Engine::add_state_force(const std::string& type, const double* params, int np) {
    DPHD_CHECK(type == "gravity", "Unsupported state force on this path: " + type);
    DPHD_CHECK(np == 3, "Inconsistent params for GravitionalStateForce.");
    DPHD_CHECK(!M.has_gravity, "Gravity was already added.");
    M.has_gravity = true;
    for (int d = 0; d < 3; ++d) M.gravity[d] = params[d];
}

void Engine::set_frictional_boundary(const std::string& type, const double* params, int np, const int* idx,
                                     int nidx) {
    DPHD_CHECK(type == "planar", "Unsupported frictional boundary on this path: " + type);
    DPHD_CHECK(np == 4, "Incompatible parameter number.");
    const double nn = std::sqrt(params[0] * params[0] + params[1] * params[1] + params[2] * params[2]);
    DPHD_CHECK(nn > 2.220446049250313e-16, "Singular normal.");
    for (int d = 0; d < 3; ++d) M.plane_n[d] = params[d] / nn;
    M.plane_off = params[3] / nn;
    std::set<int> u(idx, idx + nidx);
    DPHD_CHECK((int)u.size() == nidx, "Duplicated vertex elements.");
    for (int v : u) DPHD_CHECK(v >= 0 && v < M.n, "Frictional boundary vertex out of range.");
    M.contact_nodes.assign(u.begin(), u.end());
    M.has_plane = true;
    device_ready_ = false;
}

int Engine::num_pd_params() const {
    int t = 0;
    for (const auto& e : M.energies) t += (int)e.params.size();
    return t;
}

long long Engine::s_memory_bytes() const {
    return (long long)d_vals64.bytes + (long long)d_vals32.bytes + (long long)d_row_off.bytes + d_row_a.bytes +
           d_row_len.bytes + d_tile_ptr.bytes + d_tile_rows.bytes;
}

void Engine::set_factor_build(int mode, int small_subtree_max) {
    DPHD_CHECK(mode >= 0 && mode <= 2, "factor build mode must be 0 (automatic), 1 (host) or 2 (device)");
    const int sm = small_subtree_max > 0 ? small_subtree_max : 512;
    if (mode != factor_mode_ || sm != small_subtree_max_) built_ = false;
    factor_mode_ = mode;
    small_subtree_max_ = sm;
}

void Engine::set_st_schedule(int chunk_rows, int rows_in_flight) {
    DPHD_CHECK(chunk_rows >= 8 && chunk_rows <= kStChunkMax,
               "S^T chunk rows must lie in [8, " + std::to_string(kStChunkMax) + "]");
    DPHD_CHECK(rows_in_flight == 4 || rows_in_flight == 8, "S^T rows in flight must be 4 or 8");
    if (chunk_rows != st_chunk_rows_ || rows_in_flight != st_rows_) built_ = false;
    st_chunk_rows_ = chunk_rows;
    st_rows_ = rows_in_flight;
}

void Engine::check_device() const {
    if (device_ < 0) return;
    int cur = -1;
    CUDA_OK(cudaGetDevice(&cur));
    DPHD_CHECK(cur == device_, "this deformable's GPU state lives on device " + std::to_string(device_) +
                                   " but device " + std::to_string(cur) +
                                   " is current; make its device current (cudaSetDevice) before the call");
}

void Engine::ensure_built(double dt, int threads) {
    DPHD_CHECK(M.n > 0, "Deformable is not initialized.");
    DPHD_CHECK(!M.energies.empty(), "No PD energy was added.");
    check_device();
    if (built_ && built_dt_ == dt) {
        if (!device_ready_) build_device(threads);
        return;
    }
    // One node-level factor serves all three axes only when Dirichlet constraints fix whole nodes.
    std::map<int, int> per_node;
    for (const auto& kv : M.dirichlet) per_node[kv.first / 3]++;
    for (const auto& kv : per_node)
        DPHD_CHECK(kv.second == 3, "Dirichlet constraints must fix all three DoFs of a node on this path (node " +
                                       std::to_string(kv.first) + ").");
    A = assemble_A(M, dt);
    const std::vector<int> order = nested_dissection(M, A);
    S = SFactor();
    sb_upper_.reset(new PermUpper());
    sfactor_symbolic(A, order, S, *sb_upper_);
    factor_on_device_ = factor_mode_ == 2 || (factor_mode_ == 0 && S.nnz() > kDeviceBuildNnz);
    if (factor_on_device_) {
        sb_plan_.reset(new SBuildPlan(plan_sfactor_build(S, *sb_upper_, small_subtree_max_)));
    } else {
        sfactor_numeric_host(*sb_upper_, S, threads);
        sb_upper_.reset();
        sb_plan_.reset();
    }
    built_ = true;
    built_dt_ = dt;
    device_ready_ = false;
    build_device(threads);
}

void Engine::build_device(int threads) {
    (void)threads;
    if (device_ < 0) CUDA_OK(cudaGetDevice(&device_));
    if (!stream_) CUDA_OK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    if (!h_ctrl_) CUDA_OK(cudaMallocHost(&h_ctrl_, sizeof(Ctrl)));
    const int n = M.n, m = M.m, k = M.k;
    const int n3 = 3 * n;
    npad_ = ((n + kTileCols - 1) / kTileCols) * kTileCols;
    ntiles_ = npad_ / kTileCols;
    // S rows, padded to 16-byte (4-value) aligned segments
    std::vector<int> ra(n), rl(n);
    std::vector<int64_t> ro(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        ra[i] = S.lo[i] & ~3;
        rl[i] = ((i + 1 - ra[i]) + 3) & ~3;
        ro[i + 1] = ro[i] + rl[i];
    }
    if (!factor_on_device_) {
        std::vector<double> v64(ro[n], 0.0);
        for (int i = 0; i < n; ++i) {
            const double* src = &S.vals[S.row_ptr[i]];
            std::copy(src, src + (i - S.lo[i] + 1), &v64[ro[i] + (S.lo[i] - ra[i])]);
        }
        std::vector<float> v32(v64.begin(), v64.end());
        d_vals64.upload(v64);
        d_vals32.upload(v32);
    }
    d_row_a.upload(ra);
    d_row_len.upload(rl);
    d_row_off.upload(ro);
    if (factor_on_device_) {
        DPHD_CHECK(sb_plan_ && sb_upper_, "device factor build: the symbolic plan is missing");
        d_vals64.alloc((size_t)ro[n] * sizeof(double));
        CUDA_OK(cudaMemsetAsync(d_vals64.p, 0, d_vals64.bytes, stream_));
        // rows of the small subtrees: on the host into one zeroed staging array in the padded layout
        const std::vector<int>& roots = sb_plan_->small_roots;
        std::vector<int64_t> soff(roots.size() + 1, 0);
        for (size_t q = 0; q < roots.size(); ++q) soff[q + 1] = soff[q] + (ro[roots[q] + 1] - ro[S.lo[roots[q]]]);
        std::vector<double> staging(soff.back(), 0.0);
        std::vector<int64_t> rowbase(n, 0);
        for (size_t q = 0; q < roots.size(); ++q)
            for (int i = S.lo[roots[q]]; i <= roots[q]; ++i) rowbase[i] = soff[q] - ro[S.lo[roots[q]]];
        sfactor_small_rows(S, *sb_upper_, roots, threads,
                           [&](int i) { return staging.data() + rowbase[i] + ro[i] + (S.lo[i] - ra[i]); });
        for (size_t q = 0; q < roots.size(); ++q)
            CUDA_OK(cudaMemcpyAsync(d_vals64.as<double>() + ro[S.lo[roots[q]]], staging.data() + soff[q],
                                    (soff[q + 1] - soff[q]) * sizeof(double), cudaMemcpyHostToDevice, stream_));
        device_build_factor(*sb_plan_, S.lo, d_row_off.as<int64_t>(), d_row_a.as<int>(), d_row_len.as<int>(),
                            d_vals64.as<double>(), stream_);
        d_vals32.alloc((size_t)ro[n] * sizeof(float));
        device_round_f32(d_vals64.as<double>(), d_vals32.as<float>(), (long long)ro[n], stream_);
        CUDA_OK(cudaStreamSynchronize(stream_));
        sb_plan_.reset();
        sb_upper_.reset();
    }
    // column tiles of S^T: rows whose padded segment meets the tile, ascending
    std::vector<int> tcnt(ntiles_ + 1, 0);
    for (int i = 0; i < n; ++i)
        for (int t = ra[i] / kTileCols; t <= (ra[i] + rl[i] - 1) / kTileCols; ++t) tcnt[t + 1]++;
    for (int t = 0; t < ntiles_; ++t) tcnt[t + 1] += tcnt[t];
    std::vector<int> trows(tcnt[ntiles_]), tpos(tcnt.begin(), tcnt.end() - 1);
    for (int i = 0; i < n; ++i)
        for (int t = ra[i] / kTileCols; t <= (ra[i] + rl[i] - 1) / kTileCols; ++t) trows[tpos[t]++] = i;
    // y = S v schedule: rows cut into segments of <= kSegCols columns.  Segments of consecutive rows that
    // share their first column (one separator) are emitted row-fastest so one CTA reads one slice of v.
    // The items of one group and segment form one unit of the row-group kernel (first item, rows, first column,
    // widest row's columns).
    std::vector<int> it_row, it_c0, it_nc;
    std::vector<int4> units;
    for (int i = 0; i < n;) {
        int j = i + 1;
        while (j < n && ra[j] == ra[i] && j - i < kUnitRows) ++j;
        int glen = 0;
        for (int r = i; r < j; ++r) glen = std::max(glen, rl[r]);
        for (int c0 = 0; c0 < glen; c0 += kSegCols) {
            const int first = (int)it_row.size();
            int ncmax = 0;
            for (int r = i; r < j; ++r)
                if (c0 < rl[r]) {
                    it_row.push_back(r);
                    it_c0.push_back(c0);
                    it_nc.push_back(std::min(kSegCols, rl[r] - c0));
                    ncmax = std::max(ncmax, it_nc.back());
                }
            units.push_back(make_int4(first, (int)it_row.size() - first, ra[i] + c0, ncmax));
        }
        i = j;
    }
    std::vector<int> r_ptr(n + 1, 0), r_items(it_row.size());
    for (int r : it_row) r_ptr[r + 1]++;
    for (int i = 0; i < n; ++i) r_ptr[i + 1] += r_ptr[i];
    {
        std::vector<int> pos(r_ptr.begin(), r_ptr.end() - 1);
        for (size_t t = 0; t < it_row.size(); ++t) r_items[pos[it_row[t]]++] = (int)t;
    }
    // x = S^T y schedule: each tile's row list in chunks of `chunk` rows (long chunks for large factors, where
    // they keep more bytes in flight per CTA; short ones for small factors, where they make enough CTAs)
    const int chunk = st_chunk_rows_ > 0 ? st_chunk_rows_ : ((long long)ro[n] > kChunkLargeValues ? kChunkRows
                                                                                                  : kChunkRowsSmall);
    std::vector<int> c_tile, c_p0, c_p1, t_cptr(ntiles_ + 1, 0);
    for (int t = 0; t < ntiles_; ++t) {
        for (int p0 = tcnt[t]; p0 < tcnt[t + 1]; p0 += chunk) {
            c_tile.push_back(t);
            c_p0.push_back(p0);
            c_p1.push_back(std::min(p0 + chunk, tcnt[t + 1]));
        }
        if (tcnt[t] == tcnt[t + 1]) {  // keep every tile covered so stage 2 writes zeros
            c_tile.push_back(t);
            c_p0.push_back(tcnt[t]);
            c_p1.push_back(tcnt[t]);
        }
        t_cptr[t + 1] = (int)c_tile.size();
    }
    // Packed descriptors (one 16-byte load per work item / S^T row instead of a chain of dependent loads).
    // Item partial sums go to row-contiguous slots so that the S^T pass can sum a row's items itself.
    std::vector<int> slot(it_row.size());
    {
        std::vector<int> pos(r_ptr.begin(), r_ptr.end() - 1);
        for (size_t t = 0; t < it_row.size(); ++t) slot[t] = pos[it_row[t]]++;
    }
    std::vector<int4> idesc(it_row.size());
    for (size_t t = 0; t < it_row.size(); ++t) {
        const int r = it_row[t];
        const int64_t off = ro[r] + it_c0[t];
        idesc[t] = make_int4((int)(uint32_t)(off & 0xffffffffll), (int)(off >> 32), ra[r] + it_c0[t], it_nc[t]);
    }
    std::vector<int4> tdesc(trows.size());
    std::vector<int64_t> toff(trows.size());
    for (size_t q = 0; q < trows.size(); ++q) {
        const int r = trows[q];
        tdesc[q] = make_int4(ra[r], rl[r], r_ptr[r], r_ptr[r + 1]);
        toff[q] = ro[r];
    }
    // Launch orders, longest work first so that the last wave is made of short work items: the
    // one-warp-per-item kernel takes (descriptor, slot) pairs sorted by decreasing length; the row-group kernel
    // reads its rows from the pairs in emission order and takes its units sorted by decreasing size.
    {
        std::vector<int> ord(idesc.size());
        for (size_t t = 0; t < ord.size(); ++t) ord[t] = (int)t;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return idesc[x].w > idesc[y].w; });
        std::vector<int4> od(ord.size());
        std::vector<int> os(ord.size());
        for (size_t t = 0; t < ord.size(); ++t) {
            od[t] = idesc[ord[t]];
            os[t] = slot[ord[t]];
        }
        d_item_desc.upload(od);
        d_item_slot.upload(os);
        std::vector<int2> ors(ord.size());
        for (size_t t = 0; t < ord.size(); ++t) {
            const int r = it_row[ord[t]];
            ors[t] = make_int2(r_ptr[r], r_ptr[r + 1]);
        }
        d_item_rslots.upload(ors);
        std::stable_sort(units.begin(), units.end(),
                         [](const int4& x, const int4& y) { return (long long)x.y * x.w > (long long)y.y * y.w; });
    }
    d_unit_item_desc.upload(idesc);
    d_unit_item_slot.upload(slot);
    {
        std::vector<int2> rs(it_row.size());
        for (size_t t = 0; t < it_row.size(); ++t) rs[t] = make_int2(r_ptr[it_row[t]], r_ptr[it_row[t] + 1]);
        d_unit_item_rslots.upload(rs);
        d_row_cnt.alloc(std::max<size_t>(1, it_row.size()) * sizeof(unsigned int));
        CUDA_OK(cudaMemset(d_row_cnt.p, 0, d_row_cnt.bytes));
        d_yrow32.alloc(std::max<size_t>(1, it_row.size()) * 3 * sizeof(float));
        d_yrow64.alloc(std::max<size_t>(1, it_row.size()) * 3 * sizeof(double));
    }
    d_unit_desc.upload(units);
    d_trow_desc.upload(tdesc);
    d_trow_off.upload(toff);
    d_short_rows.upload(it_row);
    d_grp_row0.upload(it_c0);
    d_grp_g.upload(it_nc);
    d_row_item_ptr.upload(r_ptr);
    d_row_items.upload(r_items);
    d_ypart64.alloc(std::max<size_t>(1, it_row.size()) * 3 * sizeof(double));
    d_ypart32.alloc(std::max<size_t>(1, it_row.size()) * 3 * sizeof(float));
    d_chunk_tile.upload(c_tile);
    d_chunk_p0.upload(c_p0);
    d_chunk_p1.upload(c_p1);
    d_tile_chunk_ptr.upload(t_cptr);
    d_xpart64.alloc(c_tile.size() * 3 * kTileCols * sizeof(double));
    d_xpart32.alloc(c_tile.size() * 3 * kTileCols * sizeof(float));
    d_tile_ptr.upload(tcnt);
    d_tile_rows.upload(trows);
    d_perm.upload(S.perm);
    d_iperm.upload(S.iperm);
    auto fill_plan = [&](auto& P, const void* vals) {
        using PT = std::remove_reference_t<decltype(P)>;
        P = PT();
        P.n = n;
        P.npad = npad_;
        P.row_off = d_row_off.as<int64_t>();
        P.row_a = d_row_a.as<int>();
        P.row_len = d_row_len.as<int>();
        P.n_items = (int)it_row.size();
        P.item_desc = d_item_desc.as<int4>();
        P.item_slot = d_item_slot.as<int>();
        P.row_yptr = d_row_item_ptr.as<int>();
        P.trow_desc = d_trow_desc.as<int4>();
        P.trow_off = d_trow_off.as<int64_t>();
        P.item_row = d_short_rows.as<int>();
        P.item_c0 = d_grp_row0.as<int>();
        P.item_nc = d_grp_g.as<int>();
        P.row_item_ptr = d_row_item_ptr.as<int>();
        P.row_items = d_row_items.as<int>();
        P.n_chunks = (int)c_tile.size();
        P.st_rows = st_rows_;
        P.ntiles = ntiles_;
        P.chunk_tile = d_chunk_tile.as<int>();
        P.chunk_p0 = d_chunk_p0.as<int>();
        P.chunk_p1 = d_chunk_p1.as<int>();
        P.tile_rows = d_tile_rows.as<int>();
        P.tile_chunk_ptr = d_tile_chunk_ptr.as<int>();
        P.perm = d_perm.as<int>();
        (void)vals;
    };
    fill_plan(plan64_, nullptr);
    fill_plan(plan32_, nullptr);
    plan64_.vals = d_vals64.as<double>();
    plan64_.xpart = d_xpart64.as<double>();
    plan64_.ypart = d_ypart64.as<double>();
    plan32_.ypart = d_ypart32.as<float>();
    plan32_.vals = d_vals32.as<float>();
    plan32_.xpart = d_xpart32.as<float>();
    // the factor stays in L2 across PD iterations when it takes at most about half of it (126 MB on B200)
    plan64_.keep_in_l2 = d_vals64.bytes <= (64ull << 20) ? 1 : 0;
    plan32_.keep_in_l2 = d_vals32.bytes <= (64ull << 20) ? 1 : 0;
    plan32_.n_units = (int)units.size();
    plan32_.unit_desc = d_unit_desc.as<int4>();
    plan32_.unit_item_desc = d_unit_item_desc.as<int4>();
    plan32_.unit_item_rslots = d_unit_item_rslots.as<int2>();
    for (auto* P : {&plan32_}) {
        P->yrow = d_yrow32.as<float>();
        P->row_cnt = d_row_cnt.as<unsigned int>();
        P->item_rslots = d_item_rslots.as<int2>();
    }
    plan64_.yrow = d_yrow64.as<double>();
    plan64_.row_cnt = d_row_cnt.as<unsigned int>();
    plan64_.item_rslots = d_item_rslots.as<int2>();
    plan32_.unit_item_slot = d_unit_item_slot.as<int>();
    plan32_.use_units = s_units_ ? 1 : 0;
    // mesh, samples, constraints
    dE.upload(M.E);
    dX.upload(M.X);
    dgrad.upload(M.grad);
    std::vector<unsigned char> fn(n, 0), fd(n3, 0), ed(m, 0);
    std::vector<double> fv(n3, 0.0), qb(n3, 0.0);
    for (const auto& kv : M.dirichlet) {
        fn[kv.first / 3] = 1;
        fd[kv.first] = 1;
        fv[kv.first] = kv.second;
        qb[kv.first] = kv.second;
    }
    for (int e = 0; e < m; ++e)
        for (int a = 0; a < k; ++a)
            if (fn[M.E[(size_t)e * k + a]]) ed[e] = 1;
    d_fixed_node.upload(fn);
    d_fixed_dof.upload(fd);
    d_fixed_val.upload(fv);
    d_qb.upload(qb);
    d_elem_dir.upload(ed);
    // node <- (element, corner) incidence, ascending element order (deterministic gather)
    std::vector<int> np(n + 1, 0);
    for (int v : M.E) np[v + 1]++;
    for (int i = 0; i < n; ++i) np[i + 1] += np[i];
    std::vector<int> inc(np[n]), ip(np.begin(), np.end() - 1);
    for (int e = 0; e < m; ++e)
        for (int a = 0; a < k; ++a) inc[ip[M.E[(size_t)e * k + a]]++] = e * k + a;
    d_node_ptr.upload(np);
    d_node_inc.upload(inc);
    // energies
    for (int i = 0; i < kMaxEnergies; ++i) {
        d_w[i].release();
        d_w32[i].release();
        d_mask[i].release();
    }
    for (size_t i = 0; i < M.energies.size(); ++i) {
        const PdEnergy& en = M.energies[i];
        if (!en.w_elem.empty()) {
            d_w[i].upload(en.w_elem);
            std::vector<float> w32(en.w_elem.begin(), en.w_elem.end());
            d_w32[i].upload(w32);
        }
        if (!en.all_elements) d_mask[i].upload(en.in_set);
    }
    // work buffers
    const size_t ld = (size_t)n3;
    for (DeviceBuffer* b : {&d_q, &d_v, &d_f, &d_qt, &d_x, &d_xraw, &d_prev_pd, &d_lg, &d_lx, &d_qn, &d_vn, &d_gbar})
        b->alloc(ld * sizeof(double));
    d_dG.alloc(ld * kMaxWindow * sizeof(double));
    d_dX.alloc(ld * kMaxWindow * sizeof(double));
    red_blocks_ = std::max(1, std::min(kMaxRedBlocks, (n3 + 255) / 256));
    gather_blocks_ = gather_grid(n);
    d_part_gate.alloc(kMaxRedBlocks * 2 * sizeof(double));
    d_part_aa.alloc(kMaxRedBlocks * 64 * sizeof(double));
    d_part_upd.alloc(kMaxRedBlocks * 3 * sizeof(double));
    d_gravf.alloc(3 * sizeof(double));
    d_elem_out64.alloc((size_t)m * k * 3 * sizeof(double));
    d_elem_out32.alloc((size_t)m * k * 3 * sizeof(float));
    d_vperm64.alloc((size_t)npad_ * 3 * sizeof(double));
    d_vperm32.alloc((size_t)npad_ * 3 * sizeof(float));
    d_y64.alloc((size_t)npad_ * 3 * sizeof(double));
    d_y32.alloc((size_t)npad_ * 3 * sizeof(float));
    CUDA_OK(cudaMemset(d_vperm64.p, 0, d_vperm64.bytes));
    CUDA_OK(cudaMemset(d_vperm32.p, 0, d_vperm32.bytes));
    CUDA_OK(cudaMemset(d_y64.p, 0, d_y64.bytes));
    CUDA_OK(cudaMemset(d_y32.p, 0, d_y32.bytes));
    d_ctrl.alloc(sizeof(Ctrl));
    CUDA_OK(cudaMemset(d_ctrl.p, 0, sizeof(Ctrl)));
    // The two FP32 y = S v kernels (one warp per row segment, one warp per row group) give bit-identical sums
    // (the same per-lane order); which is faster depends on the factor's shape, so both are timed once here on
    // this factor (a warm-up and 5 launches each) and the faster one is kept.
    {
        cudaEvent_t e0, e1;
        CUDA_OK(cudaEventCreate(&e0));
        CUDA_OK(cudaEventCreate(&e1));
        float ms[2] = {0.f, 0.f};
        const Ctrl* c = d_ctrl.as<Ctrl>();
        for (int which = 0; which < 2; ++which) {
            SpmvPlan<float> p = plan32_;
            p.use_units = which;
            launch_s_only<float>(p, d_vperm32.as<float>(), d_y32.as<float>(), c, stream_);
            CUDA_OK(cudaEventRecord(e0, stream_));
            for (int r = 0; r < 5; ++r) launch_s_only<float>(p, d_vperm32.as<float>(), d_y32.as<float>(), c, stream_);
            CUDA_OK(cudaEventRecord(e1, stream_));
            CUDA_OK(cudaEventSynchronize(e1));
            CUDA_OK(cudaEventElapsedTime(&ms[which], e0, e1));
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        s_units_ = ms[1] < ms[0];
        plan32_.use_units = s_units_ ? 1 : 0;
        launches_ += 24;
    }
    double gf[3] = {0, 0, 0};
    if (M.has_gravity)
        for (int d = 0; d < 3; ++d) gf[d] = M.mass() * M.gravity[d];
    d_gravf.copy_in(gf, sizeof(gf));
    {
        std::vector<int> npk, tk, ok;
        int off = 0;
        for (const auto& en : M.energies) {
            npk.push_back((int)en.params.size());
            tk.push_back(en.type);
            ok.push_back(off);
            off += (int)en.params.size();
        }
        d_np_k.upload(npk);
        d_type_k.upload(tk);
        d_off_k.upload(ok);
        d_dmat_dev.alloc(std::max<size_t>(1, npk.size()) * sizeof(double));
        d_dpar_dev.alloc(std::max(1, off) * sizeof(double));
        d_dstate_dev.alloc(3 * sizeof(double));
        d_adjnorm.alloc(2 * sizeof(double));
        CUDA_OK(cudaMemset(d_adjnorm.p, 0, 2 * sizeof(double)));
        d_part_adj.alloc(kMaxRedBlocks * 3 * sizeof(double));
        for (DeviceBuffer* b : {&d_gq, &d_gv, &d_dq, &d_dv, &d_df, &d_r, &d_pp, &d_wv}) b->alloc(ld * sizeof(double));
        d_A_rp.upload(A.rp);
        d_A_ci.upload(A.ci);
        d_A_v.upload(A.v);
        Acsr_.rp = d_A_rp.as<int>();
        Acsr_.ci = d_A_ci.as<int>();
        Acsr_.v = d_A_v.as<double>();
    }
    d_q0.alloc(ld * sizeof(double));
    d_vcon.alloc((size_t)npad_ * 3 * sizeof(double));
    CUDA_OK(cudaMemset(d_vcon.p, 0, d_vcon.bytes));
    d_r64.alloc((size_t)n3 * sizeof(double));
    build_contact(built_dt_);
    drop_graphs();
    device_ready_ = true;
}

// Planar contact candidates (every listed boundary node, ascending, as frictional_boundary_vertex_indices_
// orders them), the local frame of PlanarFrictionalBoundary::GetLocalFrame
// (cpp/core/src/friction/planar_frictional_boundary.cpp:25-40), the candidates' S column paths and the
// Delassus node block G.
void Engine::build_contact(double dt) {
    has_contact_ = M.has_plane && !M.contact_nodes.empty();
    contact_ = ContactDev();
    ++contact_gen_;  // G is rebuilt: factors cached from the old one are stale
    if (!has_contact_) return;
    const int K = (int)M.contact_nodes.size();
    DPHD_CHECK((double)K * K * 8 * 2 < 64e9, "too many contact candidates for the dense Delassus block");
    ContactDev& c = contact_;
    c.K = K;
    for (int d = 0; d < 3; ++d) c.n[d] = M.plane_n[d];
    c.offset = M.plane_off;
    double best = -1, t1[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        double e[3] = {0, 0, 0};
        e[i] = 1;
        const double x[3] = {c.n[1] * e[2] - c.n[2] * e[1], c.n[2] * e[0] - c.n[0] * e[2], c.n[0] * e[1] - c.n[1] * e[0]};
        const double sq = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (sq > best) {
            best = sq;
            t1[0] = x[0]; t1[1] = x[1]; t1[2] = x[2];
        }
    }
    const double l1 = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    for (int d = 0; d < 3; ++d) c.t1[d] = t1[d] / l1;
    double t2[3] = {c.n[1] * c.t1[2] - c.n[2] * c.t1[1], c.n[2] * c.t1[0] - c.n[0] * c.t1[2],
                    c.n[0] * c.t1[1] - c.n[1] * c.t1[0]};
    const double l2 = std::sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
    for (int d = 0; d < 3; ++d) c.t2[d] = t2[d] / l2;
    const ContactPaths P = build_contact_paths(S, M.contact_nodes);
    dc_cand.upload(M.contact_nodes);
    dc_off.upload(P.off);
    dc_prow.upload(P.row);
    if (!P.val.empty()) {
        dc_pval.upload(P.val);
    } else {  // device-built factor: gather the path values from the device copy of S
        dc_pval.alloc(std::max<size_t>(1, P.row.size()) * sizeof(double));
        device_path_vals(K, dc_off.as<int64_t>(), dc_prow.as<int>(), dc_cand.as<int>(), d_iperm.as<int>(),
                         d_vals64.as<double>(), d_row_off.as<int64_t>(), d_row_a.as<int>(), dc_pval.as<double>(), 0);
        CUDA_OK(cudaDeviceSynchronize());
    }
    // The same entries by row: S v for v supported on the candidates is sum_k v_k S[:, j_k], and column j_k of
    // S = L~^-1 P is nonzero only on the etree path of j_k, so the rows of U (the union of the paths) take it in
    // O(path entries) instead of a full S pass.  Entries of a row in candidate order (a fixed summation order).
    {
        const int64_t E = P.off[K];
        std::vector<int> cnt(M.n, 0);
        for (int64_t e = 0; e < E; ++e) cnt[P.row[e]]++;
        std::vector<int> urow;
        std::vector<int64_t> uptr(1, 0), rpos(M.n, -1);
        for (int r = 0; r < M.n; ++r)
            if (cnt[r]) {
                rpos[r] = uptr.back();
                urow.push_back(r);
                uptr.push_back(uptr.back() + cnt[r]);
            }
        std::vector<int> tk(E);
        std::vector<int64_t> te(E);
        for (int k = 0; k < K; ++k)
            for (int64_t e = P.off[k]; e < P.off[k + 1]; ++e) {
                const int64_t q = rpos[P.row[e]]++;
                tk[q] = k;
                te[q] = e;
            }
        dc_tprow.upload(urow);
        dc_tpptr.upload(uptr);
        dc_tpk.upload(tk);
        DeviceBuffer src;
        src.upload(te);
        dc_tpval.alloc(std::max<size_t>(1, (size_t)E) * sizeof(double));
        launch_path_gather_vals((long long)E, src.as<int64_t>(), dc_pval.as<double>(), dc_tpval.as<double>(), 0);
        CUDA_OK(cudaDeviceSynchronize());
        c.nU = (int)urow.size();
        path_entries_ = (long long)E;
        path_max_depth_ = P.max_depth;
        c.tp_row = dc_tprow.as<int>();
        c.tp_ptr = dc_tpptr.as<int64_t>();
        c.tp_k = dc_tpk.as<int>();
        c.tp_val = dc_tpval.as<double>();
        dc_vc.alloc((size_t)3 * K * sizeof(double));
        CUDA_OK(cudaMemset(dc_vc.p, 0, dc_vc.bytes));
        c.vc = dc_vc.as<double>();
    }
    dc_G.alloc((size_t)K * K * sizeof(double));
    launch_delassus(K, dc_off.as<int64_t>(), dc_prow.as<int>(), dc_pval.as<double>(), dc_G.as<double>(), 0);
    CUDA_OK(cudaDeviceSynchronize());
    std::vector<double> gdiag(K), rp(K);
    CUDA_OK(cudaMemcpy2D(gdiag.data(), sizeof(double), dc_G.p, (K + 1) * sizeof(double), sizeof(double), K,
                         cudaMemcpyDeviceToHost));
    for (int k = 0; k < K; ++k) rp[k] = std::max(dt * dt * gdiag[k], 1e-10);
    dc_rprec.upload(rp);
    for (DeviceBuffer* b : {&dc_lam, &dc_lt1, &dc_lt2, &dc_omega, &dc_E, &dc_h}) {
        b->alloc((size_t)K * sizeof(double));
        CUDA_OK(cudaMemset(b->p, 0, b->bytes));
    }
    const size_t kcap = ncp_matrix_capacity(K);
    for (DeviceBuffer* b : {&dc_rhs, &dc_xsol}) {
        b->alloc(kcap * sizeof(double));
        CUDA_OK(cudaMemset(b->p, 0, b->bytes));
    }
    dc_bar.alloc(4 * sizeof(unsigned int));
    CUDA_OK(cudaMemset(dc_bar.p, 0, dc_bar.bytes));
    dc_Xinv.alloc(kcap * kcap * sizeof(double));
    dc_Xt.alloc(kcap * kcap * sizeof(double));
    dc_X32.alloc(kcap * kcap * sizeof(float));
    dc_Xt32.alloc(kcap * kcap * sizeof(float));
    dc_pcg.alloc((9 * kcap + 1024) * sizeof(double));
    dc_actref.alloc((size_t)K * sizeof(int));
    dc_refpos.alloc((size_t)K * sizeof(int));
    CUDA_OK(cudaMemset(dc_refpos.p, 0xff, dc_refpos.bytes));  // -1: no candidate is in a cached list yet
    dc_refinv.alloc(kcap * sizeof(int));
    dc_flags.alloc(4 * sizeof(int));
    CUDA_OK(cudaMemset(dc_flags.p, 0, dc_flags.bytes));
    dc_stats.alloc(4 * sizeof(unsigned long long));
    CUDA_OK(cudaMemset(dc_stats.p, 0, dc_stats.bytes));
    dc_act.alloc((size_t)K * sizeof(int));
    dc_kact.alloc(sizeof(int));
    CUDA_OK(cudaMemset(dc_kact.p, 0, sizeof(int)));
    dc_ainvb.alloc((size_t)3 * K * sizeof(double));
    dc_M.alloc(kcap * kcap * sizeof(double));
    c.cand = dc_cand.as<int>();
    c.off = dc_off.as<int64_t>();
    c.prow = dc_prow.as<int>();
    c.pval = dc_pval.as<double>();
    c.G = dc_G.as<double>();
    c.rprec = dc_rprec.as<double>();
    c.lam = dc_lam.as<double>();
    c.lt1 = dc_lt1.as<double>();
    c.lt2 = dc_lt2.as<double>();
    c.omega = dc_omega.as<double>();
    c.Ediag = dc_E.as<double>();
    c.hvec = dc_h.as<double>();
    c.act = dc_act.as<int>();
    c.kact = dc_kact.as<int>();
    c.ainvb = dc_ainvb.as<double>();
    c.rhs = dc_rhs.as<double>();
    c.Mwork = dc_M.as<double>();
    c.xsol = dc_xsol.as<double>();
    c.bar = dc_bar.as<unsigned int>();
    c.kcap = kcap;
    c.Xinv = dc_Xinv.as<double>();
    c.Xt = dc_Xt.as<double>();
    c.X32 = dc_X32.as<float>();
    c.Xt32 = dc_Xt32.as<float>();
    c.pcg = dc_pcg.as<double>();
    c.act_ref = dc_actref.as<int>();
    c.ref_pos = dc_refpos.as<int>();
    c.ref_inv = dc_refinv.as<int>();
    c.ncp_flags = dc_flags.as<int>();
    c.ncp_stats = dc_stats.as<unsigned long long>();
}

void Engine::ncp_stats(long long* cached, long long* refactors, long long* cg_iters, long long* cg_fallbacks) {
    unsigned long long h[4] = {0, 0, 0, 0};
    if (has_contact_ && dc_stats.p) CUDA_OK(cudaMemcpy(h, dc_stats.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (cached) *cached = (long long)h[0];
    if (refactors) *refactors = (long long)h[1];
    if (cg_iters) *cg_iters = (long long)h[2];
    if (cg_fallbacks) *cg_fallbacks = (long long)h[3];
}

void Engine::reset_warm_start() {
    if (has_contact_ && dc_lam.p) CUDA_OK(cudaMemset(dc_lam.p, 0, dc_lam.bytes));
    z_hist_ = 0;
    mu_prev_valid_ = false;
    mu_prev2_valid_ = false;
    mu_prev3_valid_ = false;
    mu_prev4_valid_ = false;
    ws_prev_valid_ = false;
}

int Engine::contact_candidates() const { return M.has_plane ? (int)M.contact_nodes.size() : 0; }

void Engine::contact_lambda_device(double* d_out, bool set, cudaStream_t st) {
    const int K = contact_candidates();
    if (K == 0) return;
    const size_t b = (size_t)K * sizeof(double);
    if (!has_contact_ || !dc_lam.p) {  // before the first forward call: the multipliers are zero
        DPHD_CHECK(!set, "contact multipliers: make one forward call before setting them");
        CUDA_OK(cudaMemsetAsync(d_out, 0, b, st));
        return;
    }
    if (set) CUDA_OK(cudaMemcpyAsync(dc_lam.p, d_out, b, cudaMemcpyDeviceToDevice, st));
    else CUDA_OK(cudaMemcpyAsync(d_out, dc_lam.p, b, cudaMemcpyDeviceToDevice, st));
}

std::vector<double> Engine::contact_lambda() {
    std::vector<double> l(has_contact_ ? contact_.K : 0);
    if (!l.empty()) CUDA_OK(cudaMemcpy(l.data(), dc_lam.p, l.size() * sizeof(double), cudaMemcpyDeviceToHost));
    return l;
}

// One PD iteration with contact (FP64): b (Dirichlet rows kept, as the reference's contact branch),
// y = S b, NCP on the active set, y += S J^T f, x_raw = S^T y, Anderson + gate.
void Engine::enqueue_contact_iteration(cudaStream_t st, bool f32) {
    const int n = M.n, n3 = 3 * n;
    const double inv_h2m = M.mass() / (graph_dt_ * graph_dt_);
    const EnergyPack ep = energy_pack();
    Ctrl* c = d_ctrl.as<Ctrl>();
    if (f32) {
        // Mixed precision: FP32 projections and SpMVs in refinement form.  r = b - A x (FP64 against the node
        // CSR of A, also kept in FP64), y = S r in FP32; the NCP sees A^-1 b = x + S^T-path(y) at the
        // candidates and solves in FP64; the S input becomes r + J^T f (summed in FP64 at the candidates:
        // near the fixed point the two nearly cancel there), y = S (r + J^T f), x_raw = x + S^T y.
        if (proj32_)
            launch_elem_fwd<float>(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), d_qb.as<double>(),
                                   d_elem_dir.as<unsigned char>(), dgrad.as<double>(), M.hex, M.vol / M.s, ep,
                                   d_elem_out64.as<double>(), c, st);
        else
            launch_elem_fwd<double>(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), d_qb.as<double>(),
                                    d_elem_dir.as<unsigned char>(), dgrad.as<double>(), M.hex, M.vol / M.s, ep,
                                    d_elem_out64.as<double>(), c, st);
        launch_gather_fwd<float>(n, d_node_ptr.as<int>(), d_node_inc.as<int>(), d_elem_out64.as<double>(),
                                 d_qt.as<double>(), inv_h2m, d_fixed_node.as<unsigned char>(), d_iperm.as<int>(),
                                 d_vperm32.as<float>(), npad_, d_prev_pd.as<double>(), d_part_gate.as<double>(),
                                 gather_blocks_, Acsr_, d_x.as<double>(), 1, c, st, d_r64.as<double>());
        // One S pass on the residual away from the candidates (small near the fixed point), the candidates' part
        // by their S column paths in FP64: r carries -J^T f there, so its FP32 image would put rounding noise
        // into the contact gaps, and after the NCP step the S input there becomes r + J^T f (small again).
        launch_cand_zero(contact_, d_iperm.as<int>(), d_vperm32.as<float>(), npad_, c, st);
        launch_s_only<float>(plan32_, d_vperm32.as<float>(), d_y32.as<float>(), c, st);  // y = S r_nc
        // S r at the rows of U, for A^-1 b = x + S^T-path(S r) at the candidates
        launch_path_apply<float, double>(contact_, d_r64.as<double>(), 1, d_y32.as<float>(), d_y64.as<double>(), npad_,
                                         c, st);
        launch_ncp_iteration<double>(contact_, d_x.as<double>(), d_y64.as<double>(), npad_, d_x.as<double>(),
                                     d_q0.as<double>(), d_iperm.as<int>(), d_vcon.as<double>(), d_r64.as<double>(),
                                     c, st);
        // y = S (r + J^T f): the candidates' inputs r + J^T f (FP64, from the NCP step) by their paths
        launch_path_apply<float, float>(contact_, contact_.vc, 0, d_y32.as<float>(), d_y32.as<float>(), npad_, c,
                                        st);
        SpmvPlan<float> ref = plan32_;
        ref.x_base = d_x.as<double>();
        launch_st_only<float>(ref, d_y32.as<float>(), d_xraw.as<double>(), c, st);
    } else {
        enqueue_contact_iteration64(st);
    }
    launch_aa_reduce(n3, d_x.as<double>(), d_xraw.as<double>(), d_fixed_dof.as<unsigned char>(),
                     d_fixed_val.as<double>(), d_dG.as<double>(), d_dX.as<double>(), d_lg.as<double>(),
                     d_lx.as<double>(), n3, d_part_aa.as<double>(), red_blocks_, c, st);
    launch_aa_update(n3, d_x.as<double>(), d_xraw.as<double>(), d_fixed_dof.as<unsigned char>(),
                     d_fixed_val.as<double>(), d_dG.as<double>(), d_dX.as<double>(), n3, d_part_upd.as<double>(),
                     d_part_gate.as<double>(), gather_blocks_, red_blocks_, c, st);
}

void Engine::enqueue_contact_iteration64(cudaStream_t st) {
    const int n = M.n;
    const double inv_h2m = M.mass() / (graph_dt_ * graph_dt_);
    const EnergyPack ep = energy_pack();
    Ctrl* c = d_ctrl.as<Ctrl>();
    launch_elem_fwd<double>(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), d_qb.as<double>(),
                            d_elem_dir.as<unsigned char>(), dgrad.as<double>(), M.hex, M.vol / M.s, ep,
                            d_elem_out64.as<double>(), c, st);
    launch_gather_fwd<double>(n, d_node_ptr.as<int>(), d_node_inc.as<int>(), d_elem_out64.as<double>(),
                              d_qt.as<double>(), inv_h2m, d_fixed_node.as<unsigned char>(), d_iperm.as<int>(),
                              d_vperm64.as<double>(), npad_, d_prev_pd.as<double>(), d_part_gate.as<double>(),
                              gather_blocks_, NodeCsr(), nullptr, 0, c, st);
    launch_s_only<double>(plan64_, d_vperm64.as<double>(), d_y64.as<double>(), c, st);
    launch_ncp_iteration<double>(contact_, d_x.as<double>(), d_y64.as<double>(), npad_, nullptr,
                                 d_q0.as<double>(), d_iperm.as<int>(), d_vcon.as<double>(), nullptr, c, st);
    // y += S J^T f by the candidates' S column paths (J^T f lives on the candidates only)
    launch_path_apply<double, double>(contact_, contact_.vc, 0, d_y64.as<double>(), d_y64.as<double>(), npad_, c, st);
    launch_st_only<double>(plan64_, d_y64.as<double>(), d_xraw.as<double>(), c, st);
}

EnergyPack Engine::energy_pack() const {
    EnergyPack ep{};
    ep.count = (int)M.energies.size();
    for (int i = 0; i < ep.count; ++i) {
        const PdEnergy& en = M.energies[i];
        ElemEnergyDev& d = ep.en[i];
        d.type = en.type;
        d.per_element = en.w_elem.empty() ? 0 : 1;
        d.w_mean = en.w_mean;
        d.mu = en.mu;
        d.la = en.la;
        d.w = d_w[i].as<double>();
        d.w32 = d_w32[i].as<float>();
        d.mask = d_mask[i].as<unsigned char>();
    }
    return ep;
}

void Engine::launch_ainv(bool fp32, cudaStream_t st, const double* x_base) {
    Ctrl* c = d_ctrl.as<Ctrl>();
    if (fp32) {
        SpmvPlan<float> p = plan32_;
        p.x_base = x_base;
        launch_sts<float>(p, d_vperm32.as<float>(), d_y32.as<float>(), d_xraw.as<double>(), c, st);
    } else {
        SpmvPlan<double> p = plan64_;
        p.x_base = x_base;
        launch_sts<double>(p, d_vperm64.as<double>(), d_y64.as<double>(), d_xraw.as<double>(), c, st);
    }
}

// One PD iteration: local step, gather to the permuted right-hand side, A^-1 pair, Anderson + gate.
void Engine::enqueue_fwd_iteration(bool f32, cudaStream_t st) {
    const int n = M.n, n3 = 3 * n;
    const double inv_h2m = M.mass() / (graph_dt_ * graph_dt_);
    const double vol_over_s = M.vol / M.s;
    const EnergyPack ep = energy_pack();
    Ctrl* c = d_ctrl.as<Ctrl>();
    if (f32) {
        if (proj32_)
            launch_elem_fwd<float>(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), d_qb.as<double>(),
                                   d_elem_dir.as<unsigned char>(), dgrad.as<double>(), M.hex, vol_over_s, ep,
                                   d_elem_out64.as<double>(), c, st);
        else
            launch_elem_fwd<double>(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), d_qb.as<double>(),
                                    d_elem_dir.as<unsigned char>(), dgrad.as<double>(), M.hex, vol_over_s, ep,
                                    d_elem_out64.as<double>(), c, st);
        launch_gather_fwd<float>(n, d_node_ptr.as<int>(), d_node_inc.as<int>(), d_elem_out64.as<double>(),
                                 d_qt.as<double>(), inv_h2m, d_fixed_node.as<unsigned char>(), d_iperm.as<int>(),
                                 d_vperm32.as<float>(), npad_, d_prev_pd.as<double>(), d_part_gate.as<double>(),
                                 gather_blocks_, Acsr_, d_x.as<double>(), 1, c, st);
    } else {
        launch_elem_fwd<double>(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), d_qb.as<double>(),
                                d_elem_dir.as<unsigned char>(), dgrad.as<double>(), M.hex, vol_over_s, ep,
                                d_elem_out64.as<double>(), c, st);
        launch_gather_fwd<double>(n, d_node_ptr.as<int>(), d_node_inc.as<int>(), d_elem_out64.as<double>(),
                                  d_qt.as<double>(), inv_h2m, d_fixed_node.as<unsigned char>(), d_iperm.as<int>(),
                                  d_vperm64.as<double>(), npad_, d_prev_pd.as<double>(), d_part_gate.as<double>(),
                                  gather_blocks_, NodeCsr(), nullptr, 1, c, st);
    }
    // FP32 S^T S in refinement form: x_raw = x + A~^-1 (b - A x) with the residual in FP64
    launch_ainv(f32, st, f32 ? d_x.as<double>() : nullptr);
    launch_aa_reduce(n3, d_x.as<double>(), d_xraw.as<double>(), d_fixed_dof.as<unsigned char>(),
                     d_fixed_val.as<double>(), d_dG.as<double>(), d_dX.as<double>(), d_lg.as<double>(),
                     d_lx.as<double>(), n3, d_part_aa.as<double>(), red_blocks_, c, st);
    launch_aa_update(n3, d_x.as<double>(), d_xraw.as<double>(), d_fixed_dof.as<unsigned char>(),
                     d_fixed_val.as<double>(), d_dG.as<double>(), d_dX.as<double>(), n3, d_part_upd.as<double>(),
                     d_part_gate.as<double>(), gather_blocks_, red_blocks_, c, st);
}

// One adjoint iteration: K_pd mu, gather of g_bar + K_pd mu, A^-1 pair, Anderson + gate.
void Engine::enqueue_bwd_iteration(cudaStream_t st) {
    const int n = M.n, n3 = 3 * n;
    Ctrl* c = d_ctrl.as<Ctrl>();
    launch_kpd_elem(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), dgrad.as<double>(), M.hex, d_J.as<double>(),
                    d_elem_out64.as<double>(), c, st);
    launch_gather_bwd(n, d_node_ptr.as<int>(), d_node_inc.as<int>(), d_elem_out64.as<double>(), d_gbar.as<double>(),
                      d_fixed_node.as<unsigned char>(), d_iperm.as<int>(), d_vperm64.as<double>(), npad_, c, st);
    launch_ainv(false, st);
    launch_aa_reduce(n3, d_x.as<double>(), d_xraw.as<double>(), d_fixed_dof.as<unsigned char>(),
                     d_fixed_val.as<double>(), d_dG.as<double>(), d_dX.as<double>(), d_lg.as<double>(),
                     d_lx.as<double>(), n3, d_part_aa.as<double>(), red_blocks_, c, st);
    launch_aa_update(n3, d_x.as<double>(), d_xraw.as<double>(), d_fixed_dof.as<unsigned char>(),
                     d_fixed_val.as<double>(), d_dG.as<double>(), d_dX.as<double>(), n3, d_part_upd.as<double>(),
                     d_part_gate.as<double>(), 0, red_blocks_, c, st);
}

// One conjugate-gradient iteration of the adjoint (A - K_pd) mu = g_bar, preconditioned by S^T S.
void Engine::enqueue_contact_precond(bool f32, bool woodbury, cudaStream_t st) {
    if (!woodbury) {
        launch_ainv(f32, st);
        return;
    }
    Ctrl* c = d_ctrl.as<Ctrl>();
    const int K = contact_.K, ld = (int)ncp_matrix_capacity(K);
    if (f32) {
        launch_s_only<float>(plan32_, d_vperm32.as<float>(), d_y32.as<float>(), c, st);
        for (int stage = 0; stage < 2; ++stage)
            launch_wbp_precond_parts<float>(stage, K, d_wb_count.as<int>(), d_wbp_cand.as<int>(), d_wbp_pos.as<int>(),
                                            d_wbp_nb.as<int>(), contact_, wbp_dirs_, d_y32.as<float>(), npad_,
                                            d_wbp_X.as<double>(), ld, d_wbp_u.as<double>(), d_wbp_w.as<double>(),
                                            d_wbp_lam.as<double>(), d_wbp_vk.as<double>(), c, st);
        // y -= S J^T lam by the constrained candidates' S column paths (FP64 sums)
        launch_path_apply<float, float>(contact_, d_wbp_vk.as<double>(), 0, d_y32.as<float>(), d_y32.as<float>(),
                                        npad_, c, st);
        launch_st_only<float>(plan32_, d_y32.as<float>(), d_xraw.as<double>(), c, st);
    } else {
        launch_s_only<double>(plan64_, d_vperm64.as<double>(), d_y64.as<double>(), c, st);
        for (int stage = 0; stage < 2; ++stage)
            launch_wbp_precond_parts<double>(stage, K, d_wb_count.as<int>(), d_wbp_cand.as<int>(),
                                             d_wbp_pos.as<int>(), d_wbp_nb.as<int>(), contact_, wbp_dirs_,
                                             d_y64.as<double>(), npad_, d_wbp_X.as<double>(), ld,
                                             d_wbp_u.as<double>(), d_wbp_w.as<double>(), d_wbp_lam.as<double>(),
                                             d_wbp_vk.as<double>(), c, st);
        launch_path_apply<double, double>(contact_, d_wbp_vk.as<double>(), 0, d_y64.as<double>(),
                                          d_y64.as<double>(), npad_, c, st);
        launch_st_only<double>(plan64_, d_y64.as<double>(), d_xraw.as<double>(), c, st);
    }
}

void Engine::enqueue_pcg_iteration(bool f32, cudaStream_t st, bool projected, bool woodbury) {
    const int n = M.n, n3 = 3 * n;
    Ctrl* c = d_ctrl.as<Ctrl>();
    const int capK = has_contact_ ? contact_.K : 0;
    if (f32)  // mixed precision: FP32 packed symmetric Jacobians (a quarter of the bytes), FP64 sums
        launch_kpd_elem32(M.m, M.k, M.s, dE.as<int>(), d_pp.as<double>(), dgrad.as<double>(), M.hex,
                          d_J32.as<float>(), d_elem_out64.as<double>(), c, st);
    else
        launch_kpd_elem(M.m, M.k, M.s, dE.as<int>(), d_pp.as<double>(), dgrad.as<double>(), M.hex, d_J.as<double>(),
                        d_elem_out64.as<double>(), c, st);
    launch_pcg_gather(n, Acsr_, d_pp.as<double>(), d_node_ptr.as<int>(), d_node_inc.as<int>(),
                      d_elem_out64.as<double>(), d_fixed_node.as<unsigned char>(), d_wv.as<double>(),
                      d_part_gate.as<double>(), gather_blocks_, c, st);
    if (projected)  // w = P (A - K_pd) p  (p lies in range(P), so p.w above is unchanged)
        launch_wb_project<double>(capK, d_wb_count.as<int>(), d_wb_nodes.as<int>(), d_wb_dirs.as<double>(),
                                  d_wb_ndir.as<int>(), d_wv.as<double>(), nullptr, nullptr, npad_, c, st);
    if (f32)
        launch_pcg_update1<float>(n, d_x.as<double>(), d_r.as<double>(), d_pp.as<double>(), d_wv.as<double>(),
                                  d_fixed_node.as<unsigned char>(), d_iperm.as<int>(), d_vperm32.as<float>(), npad_,
                                  d_part_upd.as<double>(), gather_blocks_, c, st);
    else
        launch_pcg_update1<double>(n, d_x.as<double>(), d_r.as<double>(), d_pp.as<double>(), d_wv.as<double>(),
                                   d_fixed_node.as<unsigned char>(), d_iperm.as<int>(), d_vperm64.as<double>(), npad_,
                                   d_part_upd.as<double>(), gather_blocks_, c, st);
    if (projected) {  // z = P M^-1 P r (M^-1 the preconditioner), then the z-side update
        enqueue_contact_precond(f32, woodbury, st);
        launch_wb_project<double>(capK, d_wb_count.as<int>(), d_wb_nodes.as<int>(), d_wb_dirs.as<double>(),
                                  d_wb_ndir.as<int>(), d_xraw.as<double>(), nullptr, nullptr, npad_, c, st);
        launch_pcg_update2(n3, d_r.as<double>(), d_xraw.as<double>(), d_part_aa.as<double>(),
                           d_part_upd.as<double>(), gather_blocks_, red_blocks_, c, st);
    } else if (f32) {  // z = A^-1 r with the z-side update in the S^T pass's last stage
        launch_sts_cg<float>(plan32_, d_vperm32.as<float>(), d_xraw.as<double>(), d_r.as<double>(),
                             d_part_aa.as<double>(), d_part_upd.as<double>(), gather_blocks_, c, st);
    } else {
        launch_sts_cg<double>(plan64_, d_vperm64.as<double>(), d_xraw.as<double>(), d_r.as<double>(),
                              d_part_aa.as<double>(), d_part_upd.as<double>(), gather_blocks_, c, st);
    }
    launch_pcg_p(n3, d_pp.as<double>(), d_xraw.as<double>(), c, st);
}

// Runs iterations until the device-side gate sets `done`: one iteration is captured once as a CUDA graph and
// replayed; the control block is read back every few iterations (doubling up to poll_chunk).
// Runs iterations until the device-side gate sets `done`.  Default: one launch of a graph whose WHILE node
// replays the captured iteration until k_loop_cond clears its condition (no host round trip inside a solve).
// Fallback (graph_while = 0, or a driver without conditional nodes): the iteration graph is replayed from the
// host and the control block polled every few iterations (doubling up to poll_chunk).
void Engine::enqueue_iteration(int mode, cudaStream_t cap) {
    if (mode == 2) enqueue_bwd_iteration(cap);
    else if (mode == 5 || mode == 8) enqueue_contact_iteration(cap, mode == 8);
    else if (mode == 6 || mode == 7) enqueue_pcg_iteration(mode == 7, cap, true);
    else if (mode == 9 || mode == 10) enqueue_pcg_iteration(mode == 10, cap, true, true);
    else if (mode == 3 || mode == 4) enqueue_pcg_iteration(mode == 4, cap);
    else enqueue_fwd_iteration(mode == 1, cap);
}

bool Engine::build_while_graph(int mode, int cap_iters) {
    Ctrl* c = d_ctrl.as<Ctrl>();
    cudaGraph_t graph = nullptr;
    if (cudaGraphCreate(&graph, 0) != cudaSuccess) return false;
    cudaGraphConditionalHandle handle;
    bool ok = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNode_t node;
    cudaGraphNodeParams cp = {};
    if (ok) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        ok = cudaGraphAddNode(&node, graph, nullptr, 0, &cp) == cudaSuccess;
    }
    if (ok) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaStream_t cs;
        CUDA_OK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        ok = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
             cudaSuccess;
        if (ok) {
            enqueue_iteration(mode, cs);
            launch_loop_cond(handle, c, cap_iters, cs);
            cudaGraph_t out = body;
            ok = cudaStreamEndCapture(cs, &out) == cudaSuccess;
            size_t nn = 0;
            if (ok) ok = cudaGraphGetNodes(body, nullptr, &nn) == cudaSuccess;
            graph_nodes_[mode] = nn;
        }
        CUDA_OK(cudaStreamDestroy(cs));
    }
    if (ok) ok = cudaGraphInstantiate(&graphs_[mode], graph, 0) == cudaSuccess;
    cudaGraphDestroy(graph);
    if (!ok) {
        graphs_[mode] = nullptr;
        (void)cudaGetLastError();
    }
    return ok;
}

void Engine::run_iterations(int mode, const Options& o, cudaStream_t st) {
    Ctrl* c = d_ctrl.as<Ctrl>();
    cudaGraphExec_t& g = graphs_[mode];
    const bool use_while = o.graph_while && while_ok_;
    if (g && graph_is_while_[mode] != use_while) {
        cudaGraphExecDestroy(g);
        g = nullptr;
    }
    const int cap_iters = o.max_pd_iter + 8;
    if (g && graph_is_while_[mode] && graph_cap_[mode] != cap_iters) {
        cudaGraphExecDestroy(g);
        g = nullptr;
    }
    if (!g && use_while) {
        if (build_while_graph(mode, cap_iters)) {
            graph_is_while_[mode] = true;
            graph_cap_[mode] = cap_iters;
        } else {
            while_ok_ = false;
        }
    }
    if (g && graph_is_while_[mode]) {
        CUDA_OK(cudaGraphLaunch(g, st));
        CUDA_OK(cudaMemcpyAsync(h_ctrl_, c, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        launches_ += (long long)h_ctrl_->loops * (long long)graph_nodes_[mode];
        return;
    }
    if (!g) {
        cudaStream_t cap;
        CUDA_OK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t graph;
        CUDA_OK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        enqueue_iteration(mode, cap);
        CUDA_OK(cudaStreamEndCapture(cap, &graph));
        CUDA_OK(cudaGraphGetNodes(graph, nullptr, &graph_nodes_[mode]));
        CUDA_OK(cudaGraphInstantiate(&g, graph, 0));
        CUDA_OK(cudaGraphDestroy(graph));
        CUDA_OK(cudaStreamDestroy(cap));
        graph_is_while_[mode] = false;
    }
    int launched = 0, chunk = std::min(o.poll_chunk, 4);
    while (launched < o.max_pd_iter) {
        const int todo = std::min(chunk, o.max_pd_iter - launched);
        for (int it = 0; it < todo; ++it) CUDA_OK(cudaGraphLaunch(g, st));
        launched += todo;
        launches_ += (long long)todo * (long long)graph_nodes_[mode];
        CUDA_OK(cudaMemcpyAsync(h_ctrl_, c, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        if (h_ctrl_->done) break;
        chunk = std::min(chunk * 2, std::max(o.poll_chunk, 4));
    }
}

static void init_ctrl(Ctrl* h, int mode, const Options& o, int max_iter, double clip) {
    std::memset(h, 0, sizeof(Ctrl));
    h->max_iter = max_iter;
    h->window = o.aa_window;
    h->mode = mode;
    h->rel_tol = o.rel_tol;
    h->abs_tol = o.abs_tol;
    h->clip = clip;
    h->best_ratio = 1e300;
}

void Engine::check_status(const char* where) {
    if (h_ctrl_->status & kStatusNonFinite)  // first: a NaN input can also trip the singular-F test
        throw Error(std::string(where) + ": non-finite PD iterate (NaN or Inf in q, v, f_ext or the solve)");
    if (h_ctrl_->status & kStatusSingularF) throw Error("Singular F.");
    if (h_ctrl_->status & kStatusBarrierTimeout)
        throw Error(std::string(where) + ": the contact solve's grid barrier timed out (CTAs not co-resident)");
}

void Engine::run_forward_loop(const double* dq_in, double h, const Options& o, cudaStream_t st,
                              const double* d_init) {
    const int n3 = 3 * M.n;
    Ctrl* c = d_ctrl.as<Ctrl>();
    CUDA_OK(cudaMemcpyAsync(d_x.p, d_init ? d_init : dq_in, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_OK(cudaMemsetAsync(d_prev_pd.p, 0, n3 * sizeof(double), st));
    init_ctrl(h_ctrl_, 0, o, o.max_pd_iter, 0.0);
    CUDA_OK(cudaMemcpyAsync(c, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    if (graph_dt_ != h) {
        drop_graphs();
        graph_dt_ = h;
    }
    // FP32 projections by default only without contact: with a contact set their rounding slows the coupled
    // PD / NCP iteration (measured on the 64^3 contact block), so FP64 projections feed the FP32 S passes there
    const bool want32 = o.fp32_projection < 0 ? !has_contact_ : o.fp32_projection != 0;
    if (want32 != proj32_) {  // the projection precision is captured in the mixed graphs
        proj32_ = want32;
        for (int md : {1, 8})
            if (graphs_[md]) {
                cudaGraphExecDestroy(graphs_[md]);
                graphs_[md] = nullptr;
            }
    }
    if (has_contact_) {
        contact_.mu = o.friction_mu;
        if ((o.ncp_solver != 0) != (contact_.cached != 0)) {  // the NCP solver is captured in the contact graphs
            contact_.cached = o.ncp_solver != 0 ? 1 : 0;
            for (int md : {5, 8})
                if (graphs_[md]) {
                    cudaGraphExecDestroy(graphs_[md]);
                    graphs_[md] = nullptr;
                }
        }
        CUDA_OK(cudaMemsetAsync(dc_lt1.p, 0, dc_lt1.bytes, st));
        CUDA_OK(cudaMemsetAsync(dc_lt2.p, 0, dc_lt2.bytes, st));
        // the friction coefficient and the NCP's CG tolerance are captured in the contact iteration graphs
        if (graph_mu_ != o.friction_mu || contact_.cg_tol != o.ncp_cg_tol)
            for (int md : {5, 8})
                if (graphs_[md]) {
                    cudaGraphExecDestroy(graphs_[md]);
                    graphs_[md] = nullptr;
                }
        graph_mu_ = o.friction_mu;
        contact_.cg_tol = o.ncp_cg_tol;
        CUDA_OK(cudaMemsetAsync(dc_bar.p, 0, dc_bar.bytes, st));  // clears an abort left by an earlier solve
        // every frame starts without a cached NCP factor, so that a frame's result depends on its inputs (and the
        // multipliers' warm start) alone: a recomputed frame repeats the original bit for bit
        CUDA_OK(cudaMemsetAsync(dc_flags.p, 0, dc_flags.bytes, st));
    }
    const int mode64 = has_contact_ ? 5 : 0, mode32 = has_contact_ ? 8 : 1;
    if (o.fp32_bulk && o.fp32_stall_window > 0) {
        h_ctrl_->stall_window = o.fp32_stall_window;
        CUDA_OK(cudaMemcpyAsync(c, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    }
    run_iterations(o.fp32_bulk ? mode32 : mode64, o, st);
    check_status("forward");
    int iters = h_ctrl_->iter;
    if (o.fp32_bulk && h_ctrl_->stalled && !h_ctrl_->converged && iters < o.max_pd_iter) {
        // the FP32 iteration stopped improving: the rest of the frame runs in FP64 from the current iterate, with a
        // fresh Anderson history and the same gate (the iterations of both parts count against max_pd_iter)
        Options o64 = o;
        o64.max_pd_iter = o.max_pd_iter - iters;
        CUDA_OK(cudaMemsetAsync(d_prev_pd.p, 0, n3 * sizeof(double), st));
        init_ctrl(h_ctrl_, 0, o64, o64.max_pd_iter, 0.0);
        CUDA_OK(cudaMemcpyAsync(c, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
        run_iterations(mode64, o, st);  // o: the captured loop's iteration cap; the device gate stops at o64's
        check_status("forward");
        iters += h_ctrl_->iter;
        stats.fp64_escalations++;
    }
    stats.frame_iters.push_back(iters);
    stats.frame_converged.push_back(h_ctrl_->converged);
    if (!h_ctrl_->converged && o.verbose >= 0)
        std::fprintf(stderr, "frame: %zu alg_phd: PD loop did not converge.\n", stats.frame_iters.size());
}

void Engine::forward_device(const double* dq, const double* dv, const double* df, double dt, const Options& o,
                            double* dqn, double* dvn, cudaStream_t st) {
    forward_device_init(dq, dv, df, dt, o, nullptr, dqn, dvn, st);
}

void Engine::forward_device_init(const double* dq, const double* dv, const double* df, double dt, const Options& o,
                                 const double* d_init, double* dqn, double* dvn, cudaStream_t st) {
    ensure_built(dt, o.thread_ct);
    const int n3 = dofs();
    const double h2m = dt * dt / M.mass();
    const bool learned = !d_init && ws_net_;
    ws_lambda_ = o.ws_lambda != 0;
    ws_contact_start_ = o.ws_contact_start;
    if (learned) d_init = ws_predict(dq, dv, df, dt, o.ws_tcgen05 != 0, st);
    // new-rollout detection of the contact tape (forward_gpu.cpp:437-449): the input must continue the last
    // frame; the comparison is read after the solve's own synchronisation
    const bool check_tape = has_contact_ && !tape_.empty();
    if (check_tape) {
        d_cmp.alloc(4 * sizeof(double));
        if (!h_cmp_) CUDA_OK(cudaMallocHost(&h_cmp_, 4 * sizeof(double)));
        launch_diff_norms(n3, tape_.back()->q_sol.as<double>(), dq, d_cmp.as<double>(), st);
        CUDA_OK(cudaMemcpyAsync(h_cmp_, d_cmp.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    launch_qtilde(n3, dq, dv, df, dt, h2m, d_gravf.as<double>(), d_qt.as<double>(), st);
    CUDA_OK(cudaMemcpyAsync(d_q0.p, dq, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    run_forward_loop(dq, dt, o, st, d_init);
    if (learned && *h_ws_err_) {  // the loop's synchronisation has landed the flag
        *h_ws_err_ = 0;
        CUDA_OK(cudaMemsetAsync(d_ws_err.p, 0, sizeof(int), st));
        throw Error("warm-start MLP: a tensor-core completion wait timed out.");
    }
    if (learned) {
        CUDA_OK(cudaMemcpyAsync(d_ws_qprev.p, dq, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        ws_which_ ^= 1;
        ws_prev_valid_ = true;
    }
    if (has_contact_ && o.restitution > 0) {
        launch_restitution(contact_, d_x.as<double>(), dq, dv, dt, o.restitution, o.contact_slop, st);
        launches_ += 1;
    }
    if (check_tape) {
        const double denom = std::max(1.0, std::max(std::sqrt(h_cmp_[1]), std::sqrt(h_cmp_[2])));
        if (!(std::sqrt(h_cmp_[0]) <= 1e-8 * denom))
            while (!tape_.empty()) {
                tape_free_.push_back(std::move(tape_.back()));
                tape_.pop_back();
            }
    }
    if (has_contact_) tape_push(d_x.as<double>(), st);
    CUDA_OK(cudaMemcpyAsync(dqn, d_x.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    launch_velocity(n3, d_x.as<double>(), dq, 1.0 / dt, dvn, st);
    launches_ += 2;
    CUDA_OK(cudaGetLastError());
}

void Engine::set_s_units(bool on) {
    drop_graphs();
    s_units_ = on;
    plan32_.use_units = on ? 1 : 0;
}

double Engine::ws_dx() const { return std::pow(M.vol, 1.0 / 3.0); }

void Engine::ws_state(double* d_buf, int* valid, bool set, cudaStream_t st) {
    const size_t n3 = (size_t)3 * M.n;
    DPHD_CHECK(d_buf && valid, "warm-start state: null pointer");
    if (!set) {
        *valid = ws_prev_valid_ ? 1 : 0;
        if (ws_prev_valid_) {
            CUDA_OK(cudaMemcpyAsync(d_buf, d_ws_qprev.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
            const DeviceBuffer& pb = ws_which_ ? d_ws_base0 : d_ws_base1;  // the next step's prev_base
            CUDA_OK(cudaMemcpyAsync(d_buf + n3, pb.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        }
        return;
    }
    ws_prev_valid_ = *valid != 0;
    if (!ws_prev_valid_) return;
    for (DeviceBuffer* b : {&d_ws_qprev, &d_ws_base0, &d_ws_base1}) b->alloc(n3 * sizeof(double));
    CUDA_OK(cudaMemcpyAsync(d_ws_qprev.p, d_buf, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    DeviceBuffer& pb = ws_which_ ? d_ws_base0 : d_ws_base1;
    CUDA_OK(cudaMemcpyAsync(pb.p, d_buf + n3, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
}

void Engine::set_ws_net(const float* d_master, const void* d_packed) {
    if (!d_master) {
        ws_net_ = false;
        ws_prev_valid_ = false;
        return;
    }
    DPHD_CHECK(d_packed, "warm-start network: null packed weights");
    d_ws_master.alloc((size_t)mlp_param_count() * sizeof(float));
    d_ws_packed.alloc((size_t)mlp_packed_count() * 2);
    CUDA_OK(cudaMemcpy(d_ws_master.p, d_master, d_ws_master.bytes, cudaMemcpyDeviceToDevice));
    CUDA_OK(cudaMemcpy(d_ws_packed.p, d_packed, d_ws_packed.bytes, cudaMemcpyDeviceToDevice));
    ws_net_ = true;
    ws_prev_valid_ = false;
}

const double* Engine::ws_predict(const double* dq, const double* dv, const double* df, double dt, bool tcgen05,
                                 cudaStream_t st) {
    const int n = M.n, n3 = 3 * n;
    if (!d_ws_err.p) {
        d_ws_err.alloc(sizeof(int));
        CUDA_OK(cudaMemsetAsync(d_ws_err.p, 0, sizeof(int), st));
    }
    if (!h_ws_err_) {
        CUDA_OK(cudaMallocHost(&h_ws_err_, sizeof(int)));
        *h_ws_err_ = 0;
    }
    d_ws_X.alloc((size_t)n * 16 * 2);
    d_ws_out.alloc((size_t)n * 8 * sizeof(float));
    d_ws_base0.alloc(n3 * sizeof(double));
    d_ws_base1.alloc(n3 * sizeof(double));
    d_ws_qprev.alloc(n3 * sizeof(double));
    d_ws_qinit.alloc(n3 * sizeof(double));
    double* base = (ws_which_ ? d_ws_base1 : d_ws_base0).as<double>();
    const double* prev_base = ws_prev_valid_ ? (ws_which_ ? d_ws_base0 : d_ws_base1).as<double>() : nullptr;
    const double* qp = ws_prev_valid_ ? d_ws_qprev.as<double>() : dq;
    ws_features(dt, dq, qp, dv, df, prev_base, d_ws_X.p, base, st);
    if (tcgen05) {
        mlp_forward_tc_flat(d_ws_master.as<float>(), d_ws_packed.p, d_ws_X.p, n, d_ws_out.as<float>(),
                            d_ws_err.as<int>(), st);
        CUDA_OK(cudaMemcpyAsync(h_ws_err_, d_ws_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    } else {
        mlp_forward_flat(d_ws_master.as<float>(), d_ws_packed.p, d_ws_X.p, n, d_ws_out.as<float>(), st);
    }
    ws_apply(dt, base, d_ws_out.as<float>(), d_ws_qinit.as<double>(), st);
    launches_ += 1;
    if (has_contact_ && ws_contact_start_ > 0) {
        launch_ws_contact_start(contact_.K, ws_contact_start_, dc_cand.as<int>(), dc_lam.as<double>(), contact_.n,
                                contact_.offset, d_fixed_dof.as<unsigned char>(), dq, d_ws_qinit.as<double>(), st);
        launches_ += 1;
    }
    if (has_contact_ && ws_lambda_) {  // the predicted initial contact multipliers replace the previous frame's
        launch_mlp_lambda_apply(contact_.K, dc_cand.as<int>(), d_ws_out.as<float>(), 1.0 / ws_lambda_scale(dt),
                                dc_lam.as<double>(), st);
        launches_ += 1;
    }
    return d_ws_qinit.as<double>();
}

void Engine::ws_features(double dt, const double* dq, const double* dqp, const double* dv, const double* df,
                         const double* d_prev_base, void* X, double* d_base, cudaStream_t st) {
    ensure_built(dt, 0);
    if (!d_wlog.p) {
        // log10 of each node's mean PD stiffness over its incident elements
        std::vector<double> acc(M.n, 0.0);
        std::vector<int> cnt(M.n, 0);
        for (int e = 0; e < M.m; ++e) {
            double w = 0;
            for (const auto& en : M.energies)
                if (en.all_elements || en.in_set[e]) w += en.elem_w(e);
            for (int a = 0; a < M.k; ++a) {
                acc[M.E[(size_t)e * M.k + a]] += w;
                cnt[M.E[(size_t)e * M.k + a]]++;
            }
        }
        std::vector<float> wl(M.n);
        for (int i = 0; i < M.n; ++i) wl[i] = (float)std::log10(std::max(acc[i] / std::max(cnt[i], 1), 1.0)) / 7.0f;
        d_wlog.upload(wl);
    }
    FeatureArgs a;
    a.n = M.n;
    a.X = dX.as<double>();
    a.fixed = d_fixed_node.as<unsigned char>();
    a.wlog = d_wlog.as<float>();
    a.inv_dx = 1.0 / ws_dx();
    a.h = dt;
    a.h2m = dt * dt / M.mass();
    for (int d = 0; d < 3; ++d) a.gforce[d] = M.has_gravity ? M.mass() * M.gravity[d] : 0.0;
    a.plane = M.has_plane ? 1 : 0;
    for (int d = 0; d < 3; ++d) a.pn[d] = M.plane_n[d];
    a.poff = M.plane_off;
    const float* lam_node = nullptr;
    if (has_contact_ && dc_lam.p) {  // the current multipliers (the previous frame's) as the 16th feature
        d_ws_lamprev.alloc((size_t)contact_.K * sizeof(double));  // kept for the training target's change
        CUDA_OK(cudaMemcpyAsync(d_ws_lamprev.p, dc_lam.p, d_ws_lamprev.bytes, cudaMemcpyDeviceToDevice, st));
        d_ws_lamnode.alloc((size_t)M.n * sizeof(float));
        launch_mlp_lambda_nodes(M.n, contact_.K, dc_cand.as<int>(), dc_lam.as<double>(), ws_lambda_scale(dt),
                                d_ws_lamnode.as<float>(), st);
        lam_node = d_ws_lamnode.as<float>();
        launches_ += 2;
    }
    launch_mlp_features(a, dq, dqp, dv, df, d_prev_base, lam_node, X, d_base, st);
    launches_ += 1;
}

double Engine::ws_lambda_scale(double dt) const { return dt * dt / (M.mass() * ws_dx()); }

void Engine::ws_apply(double dt, const double* d_base, const float* out, double* d_q_init, cudaStream_t st) {
    ensure_built(dt, 0);
    launch_mlp_apply(dofs(), d_base, out, ws_dx(), d_fixed_dof.as<unsigned char>(), d_fixed_val.as<double>(), d_q_init,
                     st);
    launches_ += 1;
}

void Engine::ws_target(double dt, const double* d_q_next, const double* d_base, float* Y, cudaStream_t st) {
    ensure_built(dt, 0);
    launch_mlp_target(dofs(), d_q_next, d_base, 1.0 / ws_dx(), Y, st);
    launches_ += 1;
    if (has_contact_ && dc_lam.p) {  // column 3: the multipliers' change over the frame (final - at the features)
        const double* prev = d_ws_lamprev.bytes == (size_t)contact_.K * sizeof(double) ? d_ws_lamprev.as<double>()
                                                                                        : nullptr;
        launch_mlp_target_lambda(contact_.K, dc_cand.as<int>(), dc_lam.as<double>(), prev, ws_lambda_scale(dt), Y,
                                 st);
        launches_ += 1;
    }
}

void Engine::forward(const double* q, const double* v, const double* f_ext, double dt, const Options& o,
                     double* q_next, double* v_next, std::vector<int>& active) {
    ensure_built(dt, o.thread_ct);
    const int n3 = dofs();
    cudaStream_t st = stream_;
    CUDA_OK(cudaMemcpyAsync(d_q.p, q, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d_v.p, v, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d_f.p, f_ext, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    forward_device(d_q.as<double>(), d_v.as<double>(), d_f.as<double>(), dt, o, d_qn.as<double>(),
                   d_vn.as<double>(), st);
    CUDA_OK(cudaMemcpyAsync(q_next, d_qn.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(v_next, d_vn.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    active.clear();
    if (has_contact_) {  // active_contact_idx = candidates with lambda > 0 (forward_gpu.cpp:1537-1541)
        const std::vector<double> l = contact_lambda();
        for (int k = 0; k < (int)l.size(); ++k)
            if (l[k] > 0) active.push_back(M.contact_nodes[k]);
    }
}

// ---- forward contact tape (forward_gpu.cpp:1547-1593; backward_gpu.cpp:716-742) -----------------------------
void Engine::tape_push(const double* d_qn, cudaStream_t st) {
    const int n3 = 3 * M.n, K = contact_.K;
    std::unique_ptr<TapeFrame> fr;
    if (!tape_free_.empty()) {
        fr = std::move(tape_free_.back());
        tape_free_.pop_back();
    } else {
        fr.reset(new TapeFrame());
    }
    fr->q_sol.alloc(n3 * sizeof(double));
    fr->lam.alloc((size_t)K * sizeof(double));
    fr->omega.alloc((size_t)K * sizeof(double));
    CUDA_OK(cudaMemcpyAsync(fr->q_sol.p, d_qn, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_OK(cudaMemcpyAsync(fr->lam.p, dc_lam.p, K * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_OK(cudaMemcpyAsync(fr->omega.p, dc_omega.p, K * sizeof(double), cudaMemcpyDeviceToDevice, st));
    tape_.push_back(std::move(fr));
    if (tape_.size() > 8192) {
        tape_free_.push_back(std::move(tape_.front()));
        tape_.pop_front();
    }
}

// Pops the newest frame when its q_sol matches q_next (relative 1e-8); clears the tape on a clear mismatch
// (relative > 1e-6), as the reference does.
bool Engine::tape_take(const double* d_qn, std::unique_ptr<TapeFrame>& out, cudaStream_t st) {
    if (tape_.empty()) return false;
    const int n3 = 3 * M.n;
    d_cmp.alloc(4 * sizeof(double));
    if (!h_cmp_) CUDA_OK(cudaMallocHost(&h_cmp_, 4 * sizeof(double)));
    launch_diff_norms(n3, tape_.back()->q_sol.as<double>(), d_qn, d_cmp.as<double>(), st);
    CUDA_OK(cudaMemcpyAsync(h_cmp_, d_cmp.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    const double denom = std::max(1.0, std::max(std::sqrt(h_cmp_[1]), std::sqrt(h_cmp_[2])));
    const double rel = std::sqrt(h_cmp_[0]) / denom;
    if (rel <= 1e-8) {
        out = std::move(tape_.back());
        tape_.pop_back();
        return true;
    }
    if (rel > 1e-6) {
        while (!tape_.empty()) {
            tape_free_.push_back(std::move(tape_.back()));
            tape_.pop_back();
        }
    }
    return false;
}

// Replays the forward step from (q, v, f_ext) to regenerate the contact frame of a tape miss.  The lambda warm
// start, the frame statistics and the learned-start state are left as they were.
void Engine::replay_step(const double* dq, const double* dv, const double* df, double dt, const Options& o,
                         cudaStream_t st) {
    const int n3 = 3 * M.n, K = contact_.K;
    std::vector<double> lam(K);
    CUDA_OK(cudaMemcpyAsync(lam.data(), dc_lam.p, K * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    const size_t nf = stats.frame_iters.size();
    const bool net = ws_net_;
    ws_net_ = false;
    d_rq.alloc(n3 * sizeof(double));
    d_rv.alloc(n3 * sizeof(double));
    forward_device_init(dq, dv, df, dt, o, nullptr, d_rq.as<double>(), d_rv.as<double>(), st);
    ws_net_ = net;
    stats.frame_iters.resize(nf);
    stats.frame_converged.resize(nf);
    CUDA_OK(cudaMemcpyAsync(dc_lam.p, lam.data(), K * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaStreamSynchronize(st));
}

// Contact-aware adjoint for the material gradients (backward_gpu.cpp:937-1208).  The reference forms
// z_q = mu - W_T G_T^-1 J mu with W_T[k] = (A - K_pd)^-1 j_k from one fixed-point solve per basis vector.  That is
// the (A - K_pd)-orthogonal projection of mu onto {z : J z = 0}, i.e. the adjoint system solved with the selected
// contact directions held at zero:  P (A - K_pd) P z = P g_bar,  z in range(P),  P = I - sum_k d_k d_k^T per node.
// It is solved here by one conjugate-gradient run (preconditioner P S^T S P, started from P mu) instead of one
// solve per constraint.  Selection (omega >= 0.5, tangents when friction_mu > 0 and lambda above the threshold,
// right-hand-side pruning, top-k) follows the reference.  d_x holds mu on entry and z_q on exit.
void Engine::contact_adjoint(const Options& o, const TapeFrame& fr, cudaStream_t st) {
    const int K = contact_.K, n = M.n, n3 = 3 * n;
    stats.contact_constraints = 0;
    stats.contact_iters = 0;
    d_wb_gath.alloc((size_t)3 * K * sizeof(double));
    launch_gather_nodes(K, dc_cand.as<int>(), d_x.as<double>(), d_wb_gath.as<double>(), st);
    std::vector<double> muc(3 * (size_t)K), lam(K), om(K);
    CUDA_OK(cudaMemcpyAsync(muc.data(), d_wb_gath.p, muc.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(lam.data(), fr.lam.p, K * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(om.data(), fr.omega.p, K * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    const double* nrm = M.plane_n;
    // tangent basis of the backward (backward_gpu.cpp:958-981)
    int axis = 0;
    for (int d = 1; d < 3; ++d)
        if (std::fabs(nrm[d]) < std::fabs(nrm[axis])) axis = d;
    double e[3] = {0, 0, 0};
    e[axis] = 1;
    const double ne = nrm[0] * e[0] + nrm[1] * e[1] + nrm[2] * e[2];
    double t1[3] = {e[0] - ne * nrm[0], e[1] - ne * nrm[1], e[2] - ne * nrm[2]};
    const double l1 = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    if (l1 > 1e-12) for (double& x : t1) x /= l1;
    else { t1[0] = 1; t1[1] = 0; t1[2] = 0; }
    double t2[3] = {nrm[1] * t1[2] - nrm[2] * t1[1], nrm[2] * t1[0] - nrm[0] * t1[2], nrm[0] * t1[1] - nrm[1] * t1[0]};
    const double l2 = std::sqrt(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
    if (l2 > 1e-12) for (double& x : t2) x /= l2;
    else { t2[0] = 0; t2[1] = 1; t2[2] = 0; }
    const double* dirs3[3] = {nrm, t1, t2};
    const bool tang = o.friction_mu > 0;
    struct Basis { int k, b; };
    std::vector<Basis> full;
    for (int k = 0; k < K; ++k) {  // the frame's active set: lambda > 0
        if (!(lam[k] > 0) || om[k] < 0.5) continue;
        full.push_back({k, 0});
        if (tang && lam[k] > o.tangent_lambda_min) {
            full.push_back({k, 1});
            full.push_back({k, 2});
        }
    }
    const int nbf = (int)full.size();
    std::vector<double> rfull(nbf);
    double rmax = 0;
    for (int i = 0; i < nbf; ++i) {
        const double* d = dirs3[full[i].b];
        const double sc = full[i].b == 0 ? om[full[i].k] : 1.0;
        const double* u = &muc[3 * (size_t)full[i].k];
        rfull[i] = sc * (d[0] * u[0] + d[1] * u[1] + d[2] * u[2]);
        rmax = std::max(rmax, std::fabs(rfull[i]));
    }
    const double gate = std::max(o.rhs_prune_abs, o.rhs_prune_rel * rmax);
    std::vector<int> sel;
    for (int i = 0; i < nbf; ++i)
        if (std::fabs(rfull[i]) >= gate) sel.push_back(i);
    if (o.basis_topk > 0 && (int)sel.size() > o.basis_topk) {
        std::nth_element(sel.begin(), sel.begin() + o.basis_topk, sel.end(),
                         [&](int a, int b) { return std::fabs(rfull[a]) > std::fabs(rfull[b]); });
        sel.resize(o.basis_topk);
    }
    if (sel.empty()) return;
    // per constrained node: its selected directions (orthonormal: n, t1, t2)
    std::map<int, std::vector<int>> per;
    for (int i : sel) per[full[i].k].push_back(full[i].b);
    std::vector<int> nodes, ndir;
    std::vector<double> dirs;
    for (const auto& kv : per) {
        if (M.dirichlet.count(3 * M.contact_nodes[kv.first])) continue;  // a fixed node has no free direction
        nodes.push_back(M.contact_nodes[kv.first]);
        ndir.push_back((int)kv.second.size());
        for (int j = 0; j < 3; ++j)
            for (int d = 0; d < 3; ++d)
                dirs.push_back(j < (int)kv.second.size() ? dirs3[kv.second[j]][d] : 0.0);
    }
    const int count = (int)nodes.size();
    stats.contact_constraints = (int)sel.size();
    if (count == 0) return;
    // per direction b of the basis: its constrained candidates (the blocks of J A^-1 J^T), and each constrained
    // node's position in them
    std::vector<int> wcand, wpos, idx[3];
    for (const auto& kv : per) {
        if (M.dirichlet.count(3 * M.contact_nodes[kv.first])) continue;
        int pos[3] = {-1, -1, -1};
        for (int b : kv.second) {
            pos[b] = (int)idx[b].size();
            idx[b].push_back(kv.first);
        }
        wcand.push_back(kv.first);
        for (int b = 0; b < 3; ++b) wpos.push_back(pos[b]);
    }
    d_wb_nodes.alloc((size_t)K * sizeof(int));
    d_wb_ndir.alloc((size_t)K * sizeof(int));
    d_wb_dirs.alloc((size_t)9 * K * sizeof(double));
    d_wb_count.alloc(sizeof(int));
    CUDA_OK(cudaMemcpyAsync(d_wb_nodes.p, nodes.data(), count * sizeof(int), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d_wb_ndir.p, ndir.data(), count * sizeof(int), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d_wb_dirs.p, dirs.data(), dirs.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d_wb_count.p, &count, sizeof(int), cudaMemcpyHostToDevice, st));
    // keep mu: the fallback when the projected system shows negative curvature
    d_wb_mu.alloc(n3 * sizeof(double));
    CUDA_OK(cudaMemcpyAsync(d_wb_mu.p, d_x.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    const bool f32 = o.fp32_bulk != 0;
    const bool woodbury = o.bwd_contact_precond != 0;
    if (woodbury) {
        const size_t ld = ncp_matrix_capacity(K);
        d_wbp_cand.alloc((size_t)K * sizeof(int));
        d_wbp_pos.alloc((size_t)3 * K * sizeof(int));
        d_wbp_nb.alloc(3 * sizeof(int));
        d_wbp_idx.alloc((size_t)3 * K * sizeof(int));
        d_wbp_X.alloc(6 * ld * ld * sizeof(double));  // the three X_b, then their transposes
        d_wbp_M.alloc(ld * ld * sizeof(double));
        for (DeviceBuffer* b : {&d_wbp_u, &d_wbp_w, &d_wbp_lam}) b->alloc((size_t)3 * K * sizeof(double));
        d_wbp_vk.alloc((size_t)3 * K * sizeof(double));  // zero at the candidates without a constraint
        CUDA_OK(cudaMemsetAsync(d_wbp_vk.p, 0, d_wbp_vk.bytes, st));
        CUDA_OK(cudaMemcpyAsync(d_wbp_cand.p, wcand.data(), wcand.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(d_wbp_pos.p, wpos.data(), wpos.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        int nb[3] = {(int)idx[0].size(), (int)idx[1].size(), (int)idx[2].size()};
        CUDA_OK(cudaMemcpyAsync(d_wbp_nb.p, nb, sizeof(nb), cudaMemcpyHostToDevice, st));
        for (int b = 0; b < 3; ++b) {
            for (int d = 0; d < 3; ++d) wbp_dirs_.d[b][d] = dirs3[b][d];
            if (nb[b] == 0) continue;
            // G_b depends only on A and the direction's constrained candidates: a reverse sweep whose consecutive
            // steps constrain the same candidates keeps the factor of the previous step
            if (wbp_gen_[b] == contact_gen_ && wbp_idx_prev_[b] == idx[b]) continue;
            wbp_gen_[b] = contact_gen_;
            wbp_idx_prev_[b] = idx[b];
            int* db_idx = d_wbp_idx.as<int>() + (size_t)b * K;
            CUDA_OK(cudaMemcpyAsync(db_idx, idx[b].data(), nb[b] * sizeof(int), cudaMemcpyHostToDevice, st));
            const int npd = (nb[b] + 63) / 64 * 64;
            double* Xb = d_wbp_X.as<double>() + (size_t)b * ld * ld;
            launch_wbp_gather_g(nb[b], npd, db_idx, dc_G.as<double>(), K, d_wbp_M.as<double>(), Xb, (int)ld, st);
            dense_chol_solve(d_wbp_M.as<double>(), npd, Xb, (int)ld, npd, st);  // X_b = L_b^-1
            launch_wbp_transpose(nb[b], Xb, d_wbp_X.as<double>() + (size_t)(3 + b) * ld * ld, (int)ld, st);
            launches_ += 3;  // gather, cooperative Cholesky, transpose
        }
    }
    Ctrl* c = d_ctrl.as<Ctrl>();
    init_ctrl(h_ctrl_, 1, o, o.max_pd_iter, o.bwd_clip);
    h_ctrl_->pcg_init = 1;
    CUDA_OK(cudaMemcpyAsync(c, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemsetAsync(d_pp.p, 0, n3 * sizeof(double), st));
    auto proj = [&](double* u, void* vperm) {
        if (f32)
            launch_wb_project<float>(K, d_wb_count.as<int>(), d_wb_nodes.as<int>(), d_wb_dirs.as<double>(),
                                     d_wb_ndir.as<int>(), u, reinterpret_cast<float*>(vperm), d_iperm.as<int>(),
                                     npad_, c, st);
        else
            launch_wb_project<double>(K, d_wb_count.as<int>(), d_wb_nodes.as<int>(), d_wb_dirs.as<double>(),
                                      d_wb_ndir.as<int>(), u, reinterpret_cast<double*>(vperm), d_iperm.as<int>(),
                                      npad_, c, st);
    };
    // start: P mu, or (reverse sweeps, bwd_warm_start) P (mu + (z - mu) of the later step): the constraint
    // correction carried over from the previous call (the projection makes any start admissible)
    if (o.bwd_warm_start && z_hist_ > 0) launch_axpy(n3, 1.0, d_z1.as<double>(), d_x.as<double>(), st);
    proj(d_x.as<double>(), nullptr);  // z_0 = P mu (or P (mu + correction))
    launch_kpd_elem(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), dgrad.as<double>(), M.hex, d_J.as<double>(),
                    d_elem_out64.as<double>(), c, st);
    launch_pcg_gather(n, Acsr_, d_x.as<double>(), d_node_ptr.as<int>(), d_node_inc.as<int>(),
                      d_elem_out64.as<double>(), d_fixed_node.as<unsigned char>(), d_wv.as<double>(),
                      d_part_gate.as<double>(), gather_blocks_, c, st, 1);
    proj(d_wv.as<double>(), nullptr);
    void* vp = f32 ? d_vperm32.p : d_vperm64.p;
    if (f32)
        launch_pcg_init<float>(n, d_gbar.as<double>(), d_wv.as<double>(), d_fixed_node.as<unsigned char>(),
                               d_iperm.as<int>(), d_r.as<double>(), d_vperm32.as<float>(), npad_, st);
    else
        launch_pcg_init<double>(n, d_gbar.as<double>(), d_wv.as<double>(), d_fixed_node.as<unsigned char>(),
                                d_iperm.as<int>(), d_r.as<double>(), d_vperm64.as<double>(), npad_, st);
    proj(d_r.as<double>(), vp);  // r_0 = P (g_bar - (A - K_pd) z_0)
    enqueue_contact_precond(f32, woodbury, st);
    proj(d_xraw.as<double>(), nullptr);
    launch_pcg_update2(n3, d_r.as<double>(), d_xraw.as<double>(), d_part_aa.as<double>(), d_part_upd.as<double>(),
                       gather_blocks_, red_blocks_, c, st);
    launch_pcg_p(n3, d_pp.as<double>(), d_xraw.as<double>(), c, st);
    launches_ += 12;
    run_iterations(woodbury ? (f32 ? 10 : 9) : (f32 ? 7 : 6), o, st);
    stats.contact_iters = h_ctrl_->iter;
    if (h_ctrl_->status & (kStatusIndefinite | kStatusNonFinite | kStatusDiverged)) {
        CUDA_OK(cudaMemcpyAsync(d_x.p, d_wb_mu.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        stats.bwd_fallbacks++;
        z_hist_ = 0;
    } else if (o.bwd_warm_start) {  // the constraint correction z - mu, for the next (earlier) step's start
        d_z1.alloc(n3 * sizeof(double));
        launch_sub(n3, d_x.as<double>(), d_wb_mu.as<double>(), d_z1.as<double>(), st);
        z_hist_ = 1;
    }
}

void Engine::backward_device(const double* d_q_next, const double* d_gq, const double* d_gv, double dt,
                             const Options& o, double* d_dq, double* d_dv, double* d_df, double* d_dmat_w,
                             double* d_dparams, double* d_dstate_p, cudaStream_t st) {
    backward_core(d_q_next, d_gq, d_gv, dt, o, d_dq, d_dv, d_df, d_dmat_w, d_dparams, d_dstate_p, st, nullptr,
                  nullptr, nullptr);
}

void Engine::backward_core(const double* d_q_next, const double* d_gq, const double* d_gv, double dt,
                           const Options& o, double* d_dq, double* d_dv, double* d_df, double* d_dmat_w,
                           double* d_dparams, double* d_dstate_p, cudaStream_t st, const double* d_q,
                           const double* d_v, const double* d_f) {
    ensure_built(dt, o.thread_ct);
    const int n3 = 3 * M.n, m = M.m;
    // the contact frame of this step (tape, or a replayed forward step), before anything below uses d_x
    std::unique_ptr<TapeFrame> frame;
    stats.contact_source = 0;
    stats.contact_constraints = stats.contact_iters = 0;
    if (has_contact_ && !o.skip_material_grad && !o.skip_woodbury) {
        if (tape_take(d_q_next, frame, st)) {
            stats.contact_source = 1;
        } else if (d_q && d_v && d_f) {
            replay_step(d_q, d_v, d_f, dt, o, st);
            frame = std::move(tape_.back());
            tape_.pop_back();
            stats.contact_source = 2;
        } else {
            stats.contact_source = 3;
        }
    }
    const double h = dt, mass = M.mass(), inv_h2m = mass / (h * h), h2m = h * h / mass;
    const EnergyPack ep = energy_pack();
    const double vol_over_s = M.vol / M.s;
    launch_adj_prepare(n3, d_gq, d_gv, 1.0 / h, d_gbar.as<double>(), d_dq, d_part_adj.as<double>(),
                       d_adjnorm.as<double>(), st);
    d_J.alloc((size_t)m * M.s * 81 * sizeof(double));
    Ctrl* c = d_ctrl.as<Ctrl>();
    init_ctrl(h_ctrl_, 1, o, o.max_pd_iter, o.bwd_clip);
    CUDA_OK(cudaMemcpyAsync(c, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    const bool j32 = o.fp32_bulk && o.bwd_solver == 1;
    if (j32) d_J32.alloc((size_t)m * M.s * 48 * sizeof(float));
    launch_jac_build(m, M.k, M.s, dE.as<int>(), d_q_next, dgrad.as<double>(), M.hex, vol_over_s, ep,
                     o.bwd_mean_stiffness, o.bwd_eigen_filter, d_J.as<double>(), j32 ? d_J32.as<float>() : nullptr, c,
                     st);
    CUDA_OK(cudaMemsetAsync(d_x.p, 0, n3 * sizeof(double), st));
    launches_ += 2;
    if (graph_dt_ != h) {
        drop_graphs();
        graph_dt_ = h;
    }
    if (o.bwd_solver == 1) {
        // r = g_bar, z = A^-1 r, p = z (the first update2 call only records r.z)
        const bool f32 = o.fp32_bulk != 0;
        h_ctrl_->pcg_init = 1;
        CUDA_OK(cudaMemcpyAsync(c, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemsetAsync(d_pp.p, 0, n3 * sizeof(double), st));
        // warm start from the previous call's adjoint (the next time step of a reverse sweep): mu_0 = mu_prev,
        // r_0 = g_bar - (A - K_pd) mu_0; the gate is unchanged, so only the iteration count moves
        const bool warm = o.bwd_warm_start && mu_prev_valid_ && d_mu_prev.bytes == n3 * sizeof(double);
        const double* w0 = nullptr;
        if (warm) {
            if (o.bwd_warm_start == 4 && mu_prev4_valid_)  // cubic extrapolation of the last four
                launch_extrapolate4(n3, d_mu_prev.as<double>(), d_mu_prev2.as<double>(), d_mu_prev3.as<double>(),
                                    d_mu_prev4.as<double>(), d_x.as<double>(), st);
            else if (o.bwd_warm_start >= 3 && mu_prev3_valid_)  // quadratic extrapolation of the last three
                launch_extrapolate3(n3, d_mu_prev.as<double>(), d_mu_prev2.as<double>(), d_mu_prev3.as<double>(),
                                    d_x.as<double>(), st);
            else if (o.bwd_warm_start >= 2 && mu_prev2_valid_)  // linear extrapolation of the last two adjoints
                launch_extrapolate(n3, d_mu_prev.as<double>(), d_mu_prev2.as<double>(), d_x.as<double>(), st);
            else
                CUDA_OK(cudaMemcpyAsync(d_x.p, d_mu_prev.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
            // the start's residual uses the iteration's own K_pd (FP32 Jacobians in mixed mode), so that the
            // solve converges to the same adjoint whatever the start
            if (f32)
                launch_kpd_elem32(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), dgrad.as<double>(), M.hex,
                                  d_J32.as<float>(), d_elem_out64.as<double>(), c, st);
            else
                launch_kpd_elem(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), dgrad.as<double>(), M.hex,
                                d_J.as<double>(), d_elem_out64.as<double>(), c, st);
            launch_pcg_gather(M.n, Acsr_, d_x.as<double>(), d_node_ptr.as<int>(), d_node_inc.as<int>(),
                              d_elem_out64.as<double>(), d_fixed_node.as<unsigned char>(), d_wv.as<double>(),
                              d_part_gate.as<double>(), gather_blocks_, c, st, 1);
            w0 = d_wv.as<double>();
            launches_ += 2;
        }
        if (f32)
            launch_pcg_init<float>(M.n, d_gbar.as<double>(), w0, d_fixed_node.as<unsigned char>(), d_iperm.as<int>(),
                                   d_r.as<double>(), d_vperm32.as<float>(), npad_, st);
        else
            launch_pcg_init<double>(M.n, d_gbar.as<double>(), w0, d_fixed_node.as<unsigned char>(),
                                    d_iperm.as<int>(), d_r.as<double>(), d_vperm64.as<double>(), npad_, st);
        launch_ainv(f32, st);
        launch_pcg_update2(n3, d_r.as<double>(), d_xraw.as<double>(), d_part_aa.as<double>(), d_part_upd.as<double>(),
                           gather_blocks_, red_blocks_, c, st);
        launch_pcg_p(n3, d_pp.as<double>(), d_xraw.as<double>(), c, st);
        launches_ += 8;
        run_iterations(f32 ? 4 : 3, o, st);
        if ((h_ctrl_->status & kStatusIndefinite) || o.debug_force_bwd_fallback) {
            // negative curvature of (A - K_pd): fall back to the reference fixed point for this step (the debug
            // option takes this path without the curvature test failing, for the failure-path tests)
            init_ctrl(h_ctrl_, 1, o, o.max_pd_iter, o.bwd_clip);
            CUDA_OK(cudaMemcpyAsync(c, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
            CUDA_OK(cudaMemsetAsync(d_x.p, 0, n3 * sizeof(double), st));
            run_iterations(2, o, st);
            stats.bwd_fallbacks++;
        }
    } else {
        if (o.bwd_warm_start && mu_prev_valid_ && d_mu_prev.bytes == n3 * sizeof(double))
            CUDA_OK(cudaMemcpyAsync(d_x.p, d_mu_prev.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        run_iterations(2, o, st);
    }
    stats.last_bwd_iters = h_ctrl_->iter;
    stats.last_filtered = (int)h_ctrl_->arrive[3];
    const int ne = (int)M.energies.size(), np = num_pd_params();
    const bool diverged = (h_ctrl_->status & (kStatusDiverged | kStatusNonFinite)) != 0;
    if (diverged) {  // reference: a diverged backbone contributes nothing downstream (backward_gpu.cpp:873-880)
        if (frame) tape_free_.push_back(std::move(frame));
        CUDA_OK(cudaMemsetAsync(d_dv, 0, n3 * sizeof(double), st));
        CUDA_OK(cudaMemsetAsync(d_df, 0, n3 * sizeof(double), st));
        if (d_dmat_w && ne) CUDA_OK(cudaMemsetAsync(d_dmat_w, 0, ne * sizeof(double), st));
        if (d_dparams && np) CUDA_OK(cudaMemsetAsync(d_dparams, 0, np * sizeof(double), st));
        if (d_dstate_p && M.has_gravity) CUDA_OK(cudaMemsetAsync(d_dstate_p, 0, 3 * sizeof(double), st));
        return;
    }
    if (o.bwd_warm_start) {
        if (o.bwd_warm_start == 4 && mu_prev3_valid_) {
            d_mu_prev4.alloc(n3 * sizeof(double));
            CUDA_OK(cudaMemcpyAsync(d_mu_prev4.p, d_mu_prev3.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
            mu_prev4_valid_ = true;
        }
        if (o.bwd_warm_start >= 3 && mu_prev2_valid_) {
            d_mu_prev3.alloc(n3 * sizeof(double));
            CUDA_OK(cudaMemcpyAsync(d_mu_prev3.p, d_mu_prev2.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
            mu_prev3_valid_ = true;
        }
        if (o.bwd_warm_start >= 2 && mu_prev_valid_) {
            d_mu_prev2.alloc(n3 * sizeof(double));
            CUDA_OK(cudaMemcpyAsync(d_mu_prev2.p, d_mu_prev.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
            mu_prev2_valid_ = true;
        }
        d_mu_prev.alloc(n3 * sizeof(double));
        CUDA_OK(cudaMemcpyAsync(d_mu_prev.p, d_x.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        mu_prev_valid_ = true;
    }
    launch_adj_route(n3, d_x.as<double>(), h_ctrl_->rn, d_adjnorm.as<double>(), inv_h2m, h, h2m, mass,
                     o.bwd_cascade_cap, M.has_gravity ? 1 : 0, d_dq, d_dv, d_df,
                     d_dstate_p ? d_dstate_p : d_dstate_dev.as<double>(), d_part_adj.as<double>(),
                     reinterpret_cast<unsigned int*>(d_adjnorm.as<double>() + 1), st);
    if (o.skip_material_grad) {
        if (frame) tape_free_.push_back(std::move(frame));
        if (d_dmat_w && ne) CUDA_OK(cudaMemsetAsync(d_dmat_w, 0, ne * sizeof(double), st));
        if (d_dparams && np) CUDA_OK(cudaMemsetAsync(d_dparams, 0, np * sizeof(double), st));
        CUDA_OK(cudaGetLastError());
        return;
    }
    if (frame) {  // d_x: mu -> z_q (the routing above already read mu, in stream order)
        contact_adjoint(o, *frame, st);
        tape_free_.push_back(std::move(frame));
    }
    d_gw.alloc((size_t)kMaxEnergies * m * sizeof(double));
    d_gmat.alloc((size_t)kMaxEnergies * m * sizeof(double));
    d_gnh.alloc((size_t)kMaxEnergies * m * 2 * sizeof(double));
    launch_param_grad(m, M.k, M.s, dE.as<int>(), d_q_next, d_x.as<double>(), dgrad.as<double>(), M.hex, vol_over_s,
                      ep, d_gw.as<double>(), d_gmat.as<double>(), d_gnh.as<double>(), st);
    launch_param_reduce(m, ne, d_np_k.as<int>(), d_type_k.as<int>(), d_off_k.as<int>(), d_gw.as<double>(),
                        d_gmat.as<double>(), d_gnh.as<double>(), d_dmat_w ? d_dmat_w : d_dmat_dev.as<double>(),
                        d_dparams ? d_dparams : d_dpar_dev.as<double>(), st);
    launches_ += 3;
    CUDA_OK(cudaGetLastError());
}

void Engine::backward(const double* q, const double* v, const double* f_ext, double dt, const double* q_next,
                      const double* v_next, const double* dl_dq_next, const double* dl_dv_next, const Options& o,
                      double* dl_dq, double* dl_dv, double* dl_df, double* dl_dmat_w, double* dl_dparams,
                      double* dl_dstate_p) {
    (void)v_next;
    ensure_built(dt, o.thread_ct);
    const int n3 = dofs();
    cudaStream_t st = stream_;
    CUDA_OK(cudaMemcpyAsync(d_qn.p, q_next, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d_gq.p, dl_dq_next, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(d_gv.p, dl_dv_next, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    const bool replayable = has_contact_ && q && v && f_ext;
    if (replayable) {  // inputs of a possible replay of the forward step (a tape miss)
        CUDA_OK(cudaMemcpyAsync(d_q.p, q, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(d_v.p, v, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(d_f.p, f_ext, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    backward_core(d_qn.as<double>(), d_gq.as<double>(), d_gv.as<double>(), dt, o, d_dq.as<double>(),
                  d_dv.as<double>(), d_df.as<double>(), d_dmat_dev.as<double>(), d_dpar_dev.as<double>(),
                  d_dstate_dev.as<double>(), st, replayable ? d_q.as<double>() : nullptr,
                  replayable ? d_v.as<double>() : nullptr, replayable ? d_f.as<double>() : nullptr);
    const int ne = (int)M.energies.size(), np = num_pd_params();
    CUDA_OK(cudaMemcpyAsync(dl_dq, d_dq.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(dl_dv, d_dv.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(dl_df, d_df.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (ne) CUDA_OK(cudaMemcpyAsync(dl_dmat_w, d_dmat_dev.p, ne * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (np) CUDA_OK(cudaMemcpyAsync(dl_dparams, d_dpar_dev.p, np * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (M.has_gravity)
        CUDA_OK(cudaMemcpyAsync(dl_dstate_p, d_dstate_dev.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
}

void ainv_noalloc(const SpmvPlan<double>& p64, const SpmvPlan<float>& p32, const unsigned char* fixed_node,
                  const double* d_b, double* d_x, bool fp32, cudaStream_t st);

void Engine::ainv_noalloc(double dt, const double* d_b, double* d_x, bool fp32, cudaStream_t st) {
    DPHD_CHECK(built_ && built_dt_ == dt && device_ready_,
               "dphd_ainv_noalloc: the factor for this dt is not on the device yet; make one allocating call "
               "first (dphd_forward, dphd_forward_device or dphd_debug_ainv with the same dt)");
    DPHD_CHECK(d_b && d_x, "null device pointer");
    check_device();  // the factor and the scratch address used below must belong to the same device
    dphd::ainv_noalloc(plan64_, plan32_, d_fixed_node.as<unsigned char>(), d_b, d_x, fp32, st);
    launches_ += 5;
}

double Engine::time_ainv(double dt, int reps, bool fp32, bool flush_l2) {
    ensure_built(dt, 0);
    cudaStream_t st = stream_;
    init_ctrl(h_ctrl_, 0, Options(), 1, 0);
    CUDA_OK(cudaMemcpyAsync(d_ctrl.p, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    DeviceBuffer flush;
    if (flush_l2) flush.alloc((size_t)256 << 20);  // larger than the 126 MB L2
    launch_ainv(fp32, st);  // warm
    cudaEvent_t e0, e1;
    CUDA_OK(cudaEventCreate(&e0));
    CUDA_OK(cudaEventCreate(&e1));
    double total = 0;
    for (int r = 0; r < reps; ++r) {
        if (flush_l2) CUDA_OK(cudaMemsetAsync(flush.p, r & 0xff, flush.bytes, st));
        CUDA_OK(cudaEventRecord(e0, st));
        launch_ainv(fp32, st);
        CUDA_OK(cudaEventRecord(e1, st));
        CUDA_OK(cudaEventSynchronize(e1));
        float ms = 0;
        CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
        total += ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CUDA_OK(cudaGetLastError());
    launches_ += 4LL * (reps + 1);
    return total / reps;
}

void Engine::apply_ainv(double dt, const double* b, double* x, bool fp32) {
    ensure_built(dt, 0);
    const int n = M.n, n3 = 3 * n;
    cudaStream_t st = stream_;
    // permuted SoA input, Dirichlet rows zero (as the forward's b_bc)
    std::vector<double> v((size_t)npad_ * 3, 0.0);
    std::vector<unsigned char> fixed(n, 0);
    for (const auto& kv : M.dirichlet) fixed[kv.first / 3] = 1;
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) v[(size_t)d * npad_ + S.iperm[i]] = fixed[i] ? 0.0 : b[3 * i + d];
    init_ctrl(h_ctrl_, 0, Options(), 1, 0);
    CUDA_OK(cudaMemcpyAsync(d_ctrl.p, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    if (fp32) {
        std::vector<float> v32(v.begin(), v.end());
        CUDA_OK(cudaMemcpyAsync(d_vperm32.p, v32.data(), v32.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        launch_ainv(true, st);
        CUDA_OK(cudaStreamSynchronize(st));
    } else {
        CUDA_OK(cudaMemcpyAsync(d_vperm64.p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        launch_ainv(false, st);
    }
    CUDA_OK(cudaMemcpyAsync(x, d_xraw.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
}

// Host self-check of the factor (the reference runs the same S^T S v vs LDL^T solve check on the host,
// forward_gpu.cpp:653-670): x = S^T (S v) with the host copy of S, Dirichlet rows zero.
void Engine::host_sts_apply(double dt, const double* b, double* x) {
    DPHD_CHECK(M.n > 0 && !M.energies.empty(), "Deformable is not initialized.");
    if (!(built_ && built_dt_ == dt)) {
        std::map<int, int> per_node;
        for (const auto& kv : M.dirichlet) per_node[kv.first / 3]++;
        for (const auto& kv : per_node) DPHD_CHECK(kv.second == 3, "Dirichlet constraints must fix whole nodes.");
        A = assemble_A(M, dt);
        S = SFactor();
        build_sfactor(A, nested_dissection(M, A), S, 0);
        built_ = true;
        built_dt_ = dt;
        device_ready_ = false;
    }
    DPHD_CHECK(!S.vals.empty(), "the factor was built on the device: no host copy of S to apply");
    const int n = M.n;
    std::vector<unsigned char> fixed(n, 0);
    for (const auto& kv : M.dirichlet) fixed[kv.first / 3] = 1;
    for (int d = 0; d < 3; ++d) {
        std::vector<double> v(n), y(n, 0.0), z(n, 0.0);
        for (int i = 0; i < n; ++i) v[S.iperm[i]] = fixed[i] ? 0.0 : b[3 * i + d];
        for (int i = 0; i < n; ++i) {
            const double* r = &S.vals[S.row_ptr[i]] - S.lo[i];
            double s = 0;
            for (int c = S.lo[i]; c <= i; ++c) s += r[c] * v[c];
            y[i] = s;
        }
        for (int i = 0; i < n; ++i) {
            const double* r = &S.vals[S.row_ptr[i]] - S.lo[i];
            for (int c = S.lo[i]; c <= i; ++c) z[c] += r[c] * y[i];
        }
        for (int i = 0; i < n; ++i) x[3 * i + d] = z[S.iperm[i]];
    }
}

void Engine::local_step(double dt, const double* q, double* rhs) {
    ensure_built(dt, 0);
    const int n = M.n, n3 = 3 * n;
    cudaStream_t st = stream_;
    CUDA_OK(cudaMemcpyAsync(d_x.p, q, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemsetAsync(d_prev_pd.p, 0, n3 * sizeof(double), st));
    CUDA_OK(cudaMemsetAsync(d_qt.p, 0, n3 * sizeof(double), st));
    init_ctrl(h_ctrl_, 0, Options(), 1, 0);
    CUDA_OK(cudaMemcpyAsync(d_ctrl.p, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    const EnergyPack ep = energy_pack();
    launch_elem_fwd<double>(M.m, M.k, M.s, dE.as<int>(), d_x.as<double>(), d_qb.as<double>(),
                            d_elem_dir.as<unsigned char>(), dgrad.as<double>(), M.hex, M.vol / M.s, ep,
                            d_elem_out64.as<double>(), d_ctrl.as<Ctrl>(), st);
    launch_gather_fwd<double>(n, d_node_ptr.as<int>(), d_node_inc.as<int>(), d_elem_out64.as<double>(),
                              d_qt.as<double>(), 0.0, d_fixed_node.as<unsigned char>(), d_iperm.as<int>(),
                              d_vperm64.as<double>(), npad_, d_prev_pd.as<double>(), d_part_gate.as<double>(),
                              gather_blocks_, NodeCsr(), nullptr, 1, d_ctrl.as<Ctrl>(), st);
    // the gather leaves pd (node-major) in prev_pd
    CUDA_OK(cudaMemcpyAsync(rhs, d_prev_pd.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(h_ctrl_, d_ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
    check_status("local_step");
}

}  // namespace dphd
