// hodlr_routines_cuda.h — drop-in C++ classes for the reference's HODLRMatrix and
// HSSMatrix (chenxinye/hmat-omp include/hodlr_routines.h:8-176, hss_routines.h:10-307)
// running on the B200 library through its C ABI (hmat_b200.h).
//
// Same public members (root, nodes, N, tolerance, rsvd_rank) and methods
// (build_from_dense, multiply, solve) as the reference, on the reference's Matrix and
// HODLRNode/HSSNode types (include it after the reference's utils.h is reachable on
// the include path).  After a build, `root`/`nodes` hold the tree with the reference's
// index ranges; the factors stay on the device unless download_factors() copies them
// into the nodes' D/U/V/B fields.  Errors throw std::runtime_error with the library's
// message (the reference itself asserts or ignores LAPACK info).
#ifndef HODLR_ROUTINES_CUDA_H
#define HODLR_ROUTINES_CUDA_H

#include <stdexcept>
#include <string>
#include <vector>

#include "hmat_b200.h"
#include "utils.h"

namespace hmat_b200_detail {

inline void check(int rc, hm_handle* h) {
    if (rc != HM_OK) throw std::runtime_error(std::string("hmat_b200: ") + hm_last_error(h));
}

// Download factor `which` of node `node` into M (left untouched when absent).
inline void get_factor(hm_handle* h, size_t node, int which, Matrix& M, bool present) {
    if (!present) return;
    int r = 0, c = 0;
    check(hm_get_factor(h, (int)node, which, nullptr, &r, &c), h);
    M = Matrix(r, c);
    if (r * c) check(hm_get_factor(h, (int)node, which, M.data(), &r, &c), h);
}

// A fresh handle with the caller's options (tolerance and RSVD rank from the members).
inline hm_handle* new_handle(hm_opts& opts, double tol, int rsvd_rank, hm_handle* old) {
    opts.tol = tol;
    opts.rsvd_rank = rsvd_rank;
    if (old) hm_destroy(old);
    hm_handle* h = nullptr;
    if (hm_create(&opts, &h) != HM_OK) throw std::runtime_error("hmat_b200: hm_create failed (no GPU?)");
    return h;
}

}  // namespace hmat_b200_detail

class HODLRMatrixCUDA {
public:
    HODLRNode* root;
    std::vector<HODLRNode*> nodes;   // all nodes, pre-order (the reference keeps only the root)
    int N;
    double tolerance;
    int rsvd_rank;
    hm_opts opts;                    // extension options (precision, sketch, rank cap, ...)

    explicit HODLRMatrixCUDA(double tol = 1e-6) : root(nullptr), N(0), tolerance(tol), rsvd_rank(64), h_(nullptr) {
        hm_opts_default(&opts);
    }
    ~HODLRMatrixCUDA() {
        clear_tree();
        if (h_) hm_destroy(h_);
    }
    HODLRMatrixCUDA(const HODLRMatrixCUDA&) = delete;
    HODLRMatrixCUDA& operator=(const HODLRMatrixCUDA&) = delete;

    // hodlr_routines.h:20
    void build_from_dense(const Matrix& A, int leaf_size) {
        ensure_handle();
        N = A.rows();
        hmat_b200_detail::check(hm_hodlr_build_from_dense(h_, A.data(), N, N, leaf_size), h_);
        fill_tree();
    }

    // hodlr_routines.h:66 (all columns of x; the reference uses column 0 only)
    Matrix multiply(const Matrix& x) {
        Matrix y(N, x.cols());
        hmat_b200_detail::check(hm_multiply(h_, x.data(), x.cols(), N, y.data(), N), h_);
        return y;
    }

    // hodlr_routines.h:108 (factors once, then solves; the reference re-factors per call)
    Matrix solve(const Matrix& b) {
        Matrix x(N, b.cols());
        hmat_b200_detail::check(hm_solve(h_, b.data(), b.cols(), N, x.data(), N, nullptr), h_);
        return x;
    }

    // Copy D (leaves), U, V (non-root) and B_12/B_21 (internal) into the nodes.
    void download_factors() {
        for (size_t i = 0; i < nodes.size(); ++i) {
            HODLRNode* n = nodes[i];
            get(i, 0, n->D, n->is_leaf);
            get(i, 1, n->U, i > 0);
            get(i, 2, n->V, i > 0);
            get(i, 3, n->B_12, !n->is_leaf);
            get(i, 4, n->B_21, !n->is_leaf);
        }
    }

    hm_handle* handle() { return h_; }

private:
    hm_handle* h_;

    void ensure_handle() { h_ = hmat_b200_detail::new_handle(opts, tolerance, rsvd_rank, h_); }

    void get(size_t node, int which, Matrix& M, bool present) { hmat_b200_detail::get_factor(h_, node, which, M, present); }

    void clear_tree() {
        for (auto* n : nodes) delete n;
        nodes.clear();
        root = nullptr;
    }

    void fill_tree() {
        clear_tree();
        const int n = hm_num_nodes(h_);
        std::vector<int> s(n), e(n), leaf(n), depth(n), r12(n), r21(n);
        hmat_b200_detail::check(
            hm_export_tree(h_, s.data(), e.data(), leaf.data(), depth.data(), r12.data(), r21.data()), h_);
        nodes.resize(n);
        for (int i = 0; i < n; ++i) {
            nodes[i] = new HODLRNode();
            nodes[i]->idx_start = s[i];
            nodes[i]->idx_end = e[i];
            nodes[i]->is_leaf = leaf[i] != 0;
        }
        // pre-order: the left child follows its parent, the right child follows the left subtree
        if (n) link(0);
        root = n ? nodes[0] : nullptr;
    }

    int link(int i) {  // returns the index after node i's subtree
        if (nodes[i]->is_leaf) return i + 1;
        nodes[i]->left = nodes[i + 1];
        const int r = link(i + 1);
        nodes[i]->right = nodes[r];
        return link(r);
    }
};

class HSSMatrixCUDA {
public:
    HSSNode* root;
    std::vector<HSSNode*> nodes;   // build_topo id order (hss_routines.h:293-306)
    int N;
    double tolerance;
    int rsvd_rank;
    hm_opts opts;                  // extension options (sketch, seed, refinement, ...)

    explicit HSSMatrixCUDA(double tol = 1e-9) : root(nullptr), N(0), tolerance(tol), rsvd_rank(64), h_(nullptr) {
        hm_opts_default(&opts);
    }
    ~HSSMatrixCUDA() {
        clear_tree();
        if (h_) hm_destroy(h_);
    }
    HSSMatrixCUDA(const HSSMatrixCUDA&) = delete;
    HSSMatrixCUDA& operator=(const HSSMatrixCUDA&) = delete;

    // hss_routines.h:50
    void build_from_dense(const Matrix& A, int leaf_size) {
        h_ = hmat_b200_detail::new_handle(opts, tolerance, rsvd_rank, h_);
        N = A.rows();
        hmat_b200_detail::check(hm_hss_build_from_dense(h_, A.data(), N, N, leaf_size), h_);
        fill_tree();
    }

    // hss_routines.h:118 (all columns of x)
    Matrix multiply(const Matrix& x) {
        Matrix y(N, x.cols());
        hmat_b200_detail::check(hm_multiply(h_, x.data(), x.cols(), N, y.data(), N), h_);
        return y;
    }

    // hss_routines.h:197 (factors once, then solves every column together)
    Matrix solve(const Matrix& b) {
        Matrix x(N, b.cols());
        hmat_b200_detail::check(hm_solve(h_, b.data(), b.cols(), N, x.data(), N, nullptr), h_);
        return x;
    }

    // Copy D, U, V (leaves), R, W, B (internal) into the nodes, as HSSMatrix holds them.
    void download_factors() {
        for (size_t i = 0; i < nodes.size(); ++i) {
            HSSNode* n = nodes[i];
            hmat_b200_detail::get_factor(h_, i, 0, n->D, n->is_leaf);
            hmat_b200_detail::get_factor(h_, i, 1, n->U, n->is_leaf);
            hmat_b200_detail::get_factor(h_, i, 2, n->V, n->is_leaf);
            hmat_b200_detail::get_factor(h_, i, 3, n->R, !n->is_leaf);
            hmat_b200_detail::get_factor(h_, i, 4, n->W, !n->is_leaf);
            hmat_b200_detail::get_factor(h_, i, 5, n->B, !n->is_leaf);
        }
    }

    hm_handle* handle() { return h_; }

private:
    hm_handle* h_;

    void clear_tree() {
        for (auto* n : nodes) delete n;
        nodes.clear();
        root = nullptr;
    }

    void fill_tree() {
        clear_tree();
        const int n = hm_num_nodes(h_);
        std::vector<int> s(n), e(n), leaf(n), depth(n), ru(n), rv(n);
        hmat_b200_detail::check(
            hm_export_tree(h_, s.data(), e.data(), leaf.data(), depth.data(), ru.data(), rv.data()), h_);
        nodes.resize(n);
        for (int i = 0; i < n; ++i) {
            nodes[i] = new HSSNode();
            nodes[i]->id = i;
            nodes[i]->idx_start = s[i];
            nodes[i]->idx_end = e[i];
            nodes[i]->is_leaf = leaf[i] != 0;
            nodes[i]->rank_U = ru[i];
            nodes[i]->rank_V = rv[i];
        }
        // build_topo numbers both children of a node before descending into the left one
        int next = 1;
        if (n) link(0, next);
        root = n ? nodes[0] : nullptr;
    }

    void link(int i, int& next) {
        if (nodes[i]->is_leaf) return;
        HSSNode* l = nodes[next];
        HSSNode* r = nodes[next + 1];
        next += 2;
        nodes[i]->left = l;
        nodes[i]->right = r;
        l->parent = r->parent = nodes[i];
        link(l->id, next);
        link(r->id, next);
    }
};

#endif  // HODLR_ROUTINES_CUDA_H
