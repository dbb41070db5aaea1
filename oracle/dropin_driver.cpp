// TEST INFRASTRUCTURE ONLY: a driver in the shape of the reference's
// src/main_hodlr.cpp and src/main_hss.cpp that runs the reference's serial HODLRMatrix
// and HSSMatrix and the drop-in HODLRMatrixCUDA / HSSMatrixCUDA
// (include/hodlr_routines_cuda.h) on the same dense operators and prints one JSON line
// with their differences.  Built by oracle/Makefile into
// oracle/_ref/dropin_hodlr against the reference headers and libhmat_b200.so; the
// reference's RNG is seeded as in oracle/ref_harness.cpp.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <thread>

static unsigned g_seed = 7;
namespace std {
struct hmref_seeded_device {
    using result_type = unsigned int;
    result_type operator()() const { return g_seed; }
};
}  // namespace std
#define random_device hmref_seeded_device
#include "hodlr_routines.h"
#include "hss_routines.h"
#undef random_device
#include "hodlr_routines_cuda.h"

static double rel(const Matrix& a, const Matrix& b) {
    double num = 0, den = 0;
    for (int i = 0; i < a.rows() * a.cols(); ++i) {
        double d = a.data()[i] - b.data()[i];
        num += d * d;
        den += a.data()[i] * a.data()[i];
    }
    return den == 0 ? 0 : std::sqrt(num / den);
}

int main() {
    const int N = 2048, leaf = 64;
    const double tol = 1e-8;
    Matrix A(N, N);  // configuration-1 operator: 1/(x_i - y_j), x_i = i/N, y_j = (j+0.5)/N
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) A(i, j) = 1.0 / ((double)i / N - (j + 0.5) / N);
    Matrix x(N, 1), b(N, 1);
    std::mt19937 g(1);
    std::normal_distribution<double> nd;
    for (int i = 0; i < N; ++i) { x(i, 0) = nd(g); b(i, 0) = nd(g); }

    HODLRMatrix ref(tol);
    ref.rsvd_rank = 16;
    std::thread t([&] { ref.build_from_dense(A, leaf); });  // fresh thread: seeded generator
    t.join();
    Matrix y_ref = ref.multiply(x);
    Matrix s_ref = ref.solve(b);

    HODLRMatrixCUDA gpu(tol);
    gpu.rsvd_rank = 16;
    gpu.opts.seed = g_seed;
    gpu.build_from_dense(A, leaf);
    Matrix y = gpu.multiply(x);
    Matrix s = gpu.solve(b);
    gpu.download_factors();

    // tree layout and ranks against the reference's pre-order walk
    int mismatched = 0, count = 0;
    std::vector<HODLRNode*> stack{ref.root};
    std::vector<HODLRNode*> pre;
    while (!stack.empty()) {
        HODLRNode* n = stack.back();
        stack.pop_back();
        pre.push_back(n);
        if (!n->is_leaf) { stack.push_back(n->right); stack.push_back(n->left); }
    }
    for (size_t i = 0; i < pre.size() && i < gpu.nodes.size(); ++i, ++count) {
        HODLRNode* a = pre[i];
        HODLRNode* c = gpu.nodes[i];
        bool ok = a->idx_start == c->idx_start && a->idx_end == c->idx_end && a->is_leaf == c->is_leaf;
        if (!a->is_leaf) ok = ok && a->B_12.rows() == c->B_12.rows() && a->B_21.rows() == c->B_21.rows();
        mismatched += !ok;
    }

    // HSS: Gaussian h = 0.05 + 1e-2 I on sorted uniform points, N = 512, leaf 64 (leaf
    // strips narrower than 256 take the full SVD: no sketch draws)
    const int Nh = 512, leafh = 64;
    std::vector<double> px(Nh);
    std::uniform_real_distribution<double> ud(0.0, 1.0);
    std::mt19937 gp(2);
    for (auto& v : px) v = ud(gp);
    std::sort(px.begin(), px.end());
    Matrix H(Nh, Nh);
    for (int j = 0; j < Nh; ++j)
        for (int i = 0; i < Nh; ++i) {
            const double d = px[i] - px[j];
            H(i, j) = std::exp(-d * d / (2 * 0.05 * 0.05)) + (i == j ? 1e-2 : 0.0);
        }
    Matrix xh(Nh, 1), bh(Nh, 1);
    for (int i = 0; i < Nh; ++i) { xh(i, 0) = nd(g); bh(i, 0) = nd(g); }
    HSSMatrix href(1e-10);
    std::thread th([&] { href.build_from_dense(H, leafh); });
    th.join();
    Matrix yh_ref = href.multiply(xh);
    Matrix sh_ref = href.solve(bh);
    HSSMatrixCUDA hgpu(1e-10);
    hgpu.opts.seed = g_seed;
    hgpu.build_from_dense(H, leafh);
    Matrix yh = hgpu.multiply(xh);
    Matrix sh = hgpu.solve(bh);
    hgpu.download_factors();
    int hmis = 0;
    for (size_t i = 0; i < href.nodes.size() && i < hgpu.nodes.size(); ++i) {
        HSSNode* a = href.nodes[i];
        HSSNode* c = hgpu.nodes[i];
        bool ok = a->id == c->id && a->idx_start == c->idx_start && a->idx_end == c->idx_end &&
                  a->is_leaf == c->is_leaf && a->rank_U == c->rank_U && a->rank_V == c->rank_V &&
                  (a->parent ? a->parent->id : -1) == (c->parent ? c->parent->id : -1);
        if (!a->is_leaf) ok = ok && a->B.rows() == c->B.rows() && a->B.cols() == c->B.cols();
        else ok = ok && a->U.cols() == c->U.cols() && a->V.cols() == c->V.cols();
        hmis += !ok;
    }
    std::printf("{\"nodes_ref\": %zu, \"nodes_gpu\": %zu, \"tree_mismatches\": %d, "
                "\"multiply_rel\": %.3e, \"solve_rel\": %.3e, \"root_children_linked\": %d, "
                "\"hss_nodes_ref\": %zu, \"hss_nodes_gpu\": %zu, \"hss_tree_mismatches\": %d, "
                "\"hss_multiply_rel\": %.3e, \"hss_solve_rel\": %.3e}\n",
                pre.size(), gpu.nodes.size(), mismatched, rel(y_ref, y), rel(s_ref, s),
                (int)(gpu.root && gpu.root->left && gpu.root->right), href.nodes.size(), hgpu.nodes.size(), hmis,
                rel(yh_ref, yh), rel(sh_ref, sh));
    return 0;
}
