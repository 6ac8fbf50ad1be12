// Internal data structures of the B200 projective-dynamics step (not part of the C ABI).
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace dphd {

struct Error : std::runtime_error {
    explicit Error(const std::string& s) : std::runtime_error(s) {}
};
#define DPHD_CHECK(cond, msg)                  \
    do {                                       \
        if (!(cond)) throw ::dphd::Error(msg); \
    } while (0)

enum EnergyType { kCorotated = 0, kVolume = 1, kNeoHookean = 2 };

// One AddPdEnergy call (cpp/core/src/fem/deformable_pd_energy.cpp:43-153).
struct PdEnergy {
    int type = kCorotated;
    std::vector<double> params;      // exactly as passed
    std::vector<double> w_elem;      // per-element stiffness; empty when homogeneous
    double w_mean = 0;               // stiffness(): mean of w_elem, or the scalar
    double mu = 0, la = 0;           // Neo-Hookean means used by the proximal map
    std::vector<uint8_t> in_set;     // element membership
    bool all_elements = true;
    double elem_w(int e) const { return w_elem.empty() ? w_mean : w_elem[e]; }
};

// Host model: the Deformable<3,k> state the AlgPhd path reads.
struct HostModel {
    int n = 0, m = 0, k = 0, s = 0;  // nodes, elements, nodes per element, samples per element
    bool hex = true;
    std::vector<double> X;           // 3n rest positions (node-major xyz)
    std::vector<int> E;              // m*k connectivity
    double density = 0, vol = 0;     // density, average element volume
    std::vector<double> grad;        // hex: 8 samples x 8 nodes x 3; tet: m x 4 x 3
    std::map<int, double> dirichlet;
    std::vector<PdEnergy> energies;
    bool has_gravity = false;
    double gravity[3] = {0, 0, 0};
    bool has_plane = false;
    double plane_n[3] = {0, 0, 1}, plane_off = 0;
    std::vector<int> contact_nodes;  // sorted unique
    double mass() const { return density * vol; }
    const double* g(int e, int smp) const { return &grad[((size_t)(hex ? 0 : e) * s + smp) * k * 3]; }
};

// Sparse-inverse factor S = D^-1/2 L^-1 P of the node-level PD matrix (A = P^T L D L^T P, shared by the
// three axes because Dirichlet constraints fix whole nodes).  P is a nested-dissection ordering followed
// by an elimination-tree postorder, so row i of L^-1 is dense on [lo_i, i] (its etree descendants form a
// contiguous range): S is stored as one contiguous segment per row, column indices implicit.
struct SFactor {
    int n = 0;
    std::vector<int> perm;           // perm[j] = node at permuted position j
    std::vector<int> iperm;          // iperm[node] = position
    std::vector<int> lo;             // first column of row i (= i - subtree_size + 1)
    std::vector<int> parent;         // etree parent (permuted indices), -1 at roots
    std::vector<double> Dinv_sqrt;
    // values: row i occupies vals[row_ptr[i] .. row_ptr[i+1]) for columns lo[i]..i
    std::vector<int64_t> row_ptr;
    std::vector<double> vals;
    int64_t nnz() const { return row_ptr.empty() ? 0 : row_ptr.back(); }
    int64_t nnz_L = 0;
    int max_depth = 0;
};

// Node-level PD matrix in CSR (original node order): A = diag(m/h^2 or 1) + sum_e w_e vol/s sum_s G_s G_s^T.
struct NodeMatrix {
    int n = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
};

// Root-first etree paths of the S columns of contact candidates: for candidate c (permuted column col_c),
// entries k = 0 .. depth_c-1 walk from the etree root down to col_c; path_row[off_c + k] is the S row and
// path_val[off_c + k] = S(row, col_c).  Two candidates' paths share exactly the prefix from the root to
// their lowest common ancestor, so (A^-1)_{ij} = sum over the shared prefix of path_val_i * path_val_j.
struct ContactPaths {
    std::vector<int64_t> off;   // K + 1
    std::vector<int> row;
    std::vector<double> val;
    int max_depth = 0;
};
ContactPaths build_contact_paths(const SFactor& S, const std::vector<int>& cand_nodes);

// Upper triangle (row <= col) of P A P^T by columns, in the factor's permuted order.
struct PermUpper {
    std::vector<int> Cp, Ci;
    std::vector<double> Cx;
};

// Plan of the device construction of S (sfactor_plan.cpp, sfactor_gpu.cu).
constexpr int kSbTile = 64;  // column tile of the S[s, D] product
struct SBigSuper {
    int a = 0, b = 0;   // rows [a, b) of an etree chain (permuted indices)
    int lo = 0, ra = 0; // first column of the rows' segments, and its 4-aligned start in storage
    int64_t B_off = 0;  // its B_s rows: plan.B[B_off .. B_off + nB)
    int nB = 0;
    int64_t ct_off = 0; // column tile t's contributing B positions: ct_p[ct_ptr[ct_off + t] .. ct_ptr[ct_off + t + 1])
    int nct = 0;        // column tiles of kSbTile columns from ra up to a
};
struct SBuildPlan {
    int small_max = 0;
    std::vector<int> small_roots;   // roots of the host-built subtrees, ascending
    std::vector<SBigSuper> sup;     // device-built supernodes in postorder
    std::vector<int> B;
    std::vector<int64_t> ct_ptr;
    std::vector<int> ct_p;
    std::vector<int64_t> a_rp;      // P A P^T, both triangles, by rows (permuted indices)
    std::vector<int> a_ci;
    std::vector<double> a_v;
    int max_w = 0, max_nB = 0;
    int64_t max_x = 0;              // largest [W | I] work array (rows padded to kSbTile) in doubles
};
SBuildPlan plan_sfactor_build(const struct SFactor& S, const struct PermUpper& U, int small_max);
void sfactor_small_rows(const struct SFactor& S, const struct PermUpper& U, const std::vector<int>& roots, int threads,
                        const std::function<double*(int)>& row_ptr);

void init_samples(HostModel& M);
double element_volume(const HostModel& M, int e);
NodeMatrix assemble_A(const HostModel& M, double dt);
std::vector<int> nested_dissection(const HostModel& M, const NodeMatrix& A);
void build_sfactor(const NodeMatrix& A, const std::vector<int>& order, SFactor& S, int threads);
// The symbolic half of build_sfactor: postorder permutation, etree, row ranges lo and row_ptr (no values) ...
void sfactor_symbolic(const NodeMatrix& A, const std::vector<int>& order, SFactor& S, PermUpper& U);
// ... and its numeric half on the host (up-looking LDL^T and the row recurrence into S.vals).
void sfactor_numeric_host(const PermUpper& U, SFactor& S, int threads);

}  // namespace dphd
