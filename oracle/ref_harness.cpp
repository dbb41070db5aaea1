// TEST INFRASTRUCTURE ONLY — the oracle.  Compiled by oracle/Makefile against the
// unmodified reference headers (chenxinye/hmat-omp include/*.h) into
// oracle/_ref/libhmatref.so.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load it, as the checker or the timed CPU reference; the product
// library never links or calls it.
//
// What this file adds around the reference (without editing it):
//  * Seed injection.  Matrix::Random (include/matrix.h:50-57) seeds a thread_local
//    std::mt19937 from std::random_device{}().  `random_device` is redirected to a
//    functor returning a process-global seed, and every reference call that draws
//    random numbers runs on a fresh std::thread so its thread_local generator is
//    constructed anew from that seed.  The serial routines therefore draw their
//    sketches deterministically, in the serial post-order of the build.
//  * A Gaussian variant (HMREF_GAUSSIAN): uniform_real_distribution is redirected
//    to normal_distribution, giving the N(0,1) sketch that the configs name.
//  * Flat C entry points: build, tree export in the reference's node order,
//    factor download, multiply, solve, and the RNG stream itself.
#include <random>
#include <thread>
#include <vector>
#include <cstring>
#include <cstdint>

static unsigned g_hmref_seed = 0;
namespace std {
struct hmref_seeded_device {
    using result_type = unsigned int;
    result_type operator()() const { return g_hmref_seed; }
};
}  // namespace std
#define random_device hmref_seeded_device
#ifdef HMREF_GAUSSIAN
#define uniform_real_distribution normal_distribution
#endif

#include "hodlr_routines.h"
#include "hodlr_routines_omp.h"
#include "hss_routines.h"
#include "hss_routines_omp.h"

#undef random_device

namespace {

template <class F>
void on_fresh_thread(F&& f) {
    std::thread t(std::forward<F>(f));
    t.join();
}

Matrix from_ptr(const double* p, int rows, int cols, int ld) {
    Matrix M(rows, cols);
    for (int j = 0; j < cols; ++j)
        for (int i = 0; i < rows; ++i) M(i, j) = p[(size_t)j * ld + i];
    return M;
}

void to_ptr(const Matrix& M, double* p) {
    if (M.rows() * M.cols() > 0) std::memcpy(p, M.data(), sizeof(double) * M.rows() * M.cols());
}

struct HodlrBox {
    int omp = 0;
    HODLRMatrix* ser = nullptr;
    HODLRMatrixOMP* par = nullptr;
    std::vector<HODLRNode*> pre;   // pre-order (root, left subtree, right subtree)
    std::vector<int> depth;
    HODLRNode* root() const { return omp ? par->root : ser->root; }
};

void preorder(HodlrBox* b, HODLRNode* n, int d) {
    b->pre.push_back(n);
    b->depth.push_back(d);
    if (!n->is_leaf) {
        preorder(b, n->left, d + 1);
        preorder(b, n->right, d + 1);
    }
}

void free_subtree(HODLRNode* n, HODLRNode* keep) {
    // The reference deletes only `nodes` (= the root); children are never freed
    // (include/hodlr_routines.h:17,39-40).  Free them here so tests do not leak.
    if (!n) return;
    free_subtree(n->left, keep);
    free_subtree(n->right, keep);
    if (n != keep) delete n;
}

struct HssBox {
    int omp = 0;
    HSSMatrix* ser = nullptr;
    HSSMatrixOMP* par = nullptr;
    std::vector<HSSNode*>& nodes() { return omp ? par->nodes : ser->nodes; }
};

}  // namespace

extern "C" {

// ---- RNG stream as the reference draws it (Matrix::Random, column-major fill) ----
void hmref_random(unsigned seed, int rows, int cols, double* out) {
    g_hmref_seed = seed;
    on_fresh_thread([&] { to_ptr(Matrix::Random(rows, cols), out); });
}

// ---- compression.h entry points ----
int hmref_compress_svd(const double* A, int m, int n, int lda, double tol,
                       double* U, double* V, double* S) {
    Compression::LowRank lr;
    lr = Compression::compress_svd(from_ptr(A, m, n, lda), tol);
    to_ptr(lr.U, U);
    to_ptr(lr.V, V);
    for (int i = 0; i < lr.rank; ++i) S[i] = lr.B(i, i);
    return lr.rank;
}

int hmref_compress_rsvd(const double* A, int m, int n, int lda, double tol, int rank_guess,
                        unsigned seed, double* U, double* V, double* S) {
    Compression::LowRank lr;
    g_hmref_seed = seed;
    Matrix Am = from_ptr(A, m, n, lda);
    on_fresh_thread([&] { lr = Compression::compress_rsvd(Am, tol, rank_guess); });
    to_ptr(lr.U, U);
    to_ptr(lr.V, V);
    for (int i = 0; i < lr.rank; ++i) S[i] = lr.B(i, i);
    return lr.rank;
}

// ---- HODLR (include/hodlr_routines.h, include/hodlr_routines_omp.h) ----
void* hmref_hodlr_build(const double* A, int N, int lda, int leaf, double tol, int rsvd_rank,
                        unsigned seed, int omp) {
    auto* b = new HodlrBox();
    b->omp = omp;
    Matrix Am = from_ptr(A, N, N, lda);
    g_hmref_seed = seed;
    if (omp) {
        b->par = new HODLRMatrixOMP(tol);
        b->par->rsvd_rank = rsvd_rank;
        b->par->build_from_dense(Am, leaf);
    } else {
        b->ser = new HODLRMatrix(tol);
        b->ser->rsvd_rank = rsvd_rank;
        on_fresh_thread([&] { b->ser->build_from_dense(Am, leaf); });
    }
    preorder(b, b->root(), 0);
    return b;
}

void hmref_hodlr_free(void* h) {
    auto* b = static_cast<HodlrBox*>(h);
    free_subtree(b->root(), b->root());
    delete b->ser;
    delete b->par;
    delete b;
}

int hmref_hodlr_num_nodes(void* h) { return (int)static_cast<HodlrBox*>(h)->pre.size(); }

// Per node in pre-order: idx_start, idx_end, is_leaf, depth, rank12 (= B_12 rows),
// rank21 (= B_21 rows); ranks are 0 for leaves.
void hmref_hodlr_tree(void* h, int* start, int* end, int* is_leaf, int* depth, int* rank12,
                      int* rank21) {
    auto* b = static_cast<HodlrBox*>(h);
    for (size_t i = 0; i < b->pre.size(); ++i) {
        HODLRNode* n = b->pre[i];
        start[i] = n->idx_start;
        end[i] = n->idx_end;
        is_leaf[i] = n->is_leaf ? 1 : 0;
        depth[i] = b->depth[i];
        rank12[i] = n->is_leaf ? 0 : n->B_12.rows();
        rank21[i] = n->is_leaf ? 0 : n->B_21.rows();
    }
}

// which: 0 = D, 1 = U, 2 = V, 3 = B_12, 4 = B_21.  Returns rows*cols written
// (shape via hmref_hodlr_factor_shape).
void hmref_hodlr_factor_shape(void* h, int node, int which, int* rows, int* cols) {
    HODLRNode* n = static_cast<HodlrBox*>(h)->pre[node];
    const Matrix* M = which == 0 ? &n->D : which == 1 ? &n->U : which == 2 ? &n->V
                      : which == 3 ? &n->B_12 : &n->B_21;
    *rows = M->rows();
    *cols = M->cols();
}

void hmref_hodlr_factor(void* h, int node, int which, double* out) {
    HODLRNode* n = static_cast<HodlrBox*>(h)->pre[node];
    const Matrix* M = which == 0 ? &n->D : which == 1 ? &n->U : which == 2 ? &n->V
                      : which == 3 ? &n->B_12 : &n->B_21;
    to_ptr(*M, out);
}

// multiply() uses column 0 only (include/hodlr_routines.h:75,85).
void hmref_hodlr_multiply(void* h, const double* x, double* y) {
    auto* b = static_cast<HodlrBox*>(h);
    int N = b->omp ? b->par->N : b->ser->N;
    Matrix xm = from_ptr(x, N, 1, N);
    Matrix ym = b->omp ? b->par->multiply(xm) : b->ser->multiply(xm);
    to_ptr(ym, y);
}

void hmref_hodlr_solve(void* h, const double* rhs, int nrhs, double* x) {
    auto* b = static_cast<HodlrBox*>(h);
    int N = b->omp ? b->par->N : b->ser->N;
    Matrix bm = from_ptr(rhs, N, nrhs, N);
    Matrix xm = b->omp ? b->par->solve(bm) : b->ser->solve(bm);
    to_ptr(xm, x);
}

// HODLRMatrixOMP::solve (hodlr_routines_omp.h:137-240) on the tree of a serial build:
// the OpenMP class is pointed at the serial build's nodes (same HODLRNode type), so
// the timed solve is the reference's OpenMP path without its OpenMP build, whose tasks
// copy the whole dense A each (include/hodlr_routines_omp.h:48-56).
void hmref_hodlr_solve_omp(void* h, const double* rhs, int nrhs, double* x) {
    auto* b = static_cast<HodlrBox*>(h);
    HODLRMatrixOMP view(b->ser ? b->ser->tolerance : b->par->tolerance);
    view.root = b->root();
    view.N = b->ser ? b->ser->N : b->par->N;
    Matrix bm = from_ptr(rhs, view.N, nrhs, view.N);
    Matrix xm = view.solve(bm);
    to_ptr(xm, x);
    view.root = nullptr;  // nodes stay owned by the box (view.nodes is empty)
}

int hmref_omp_max_threads() { return omp_get_max_threads(); }

// ---- HSS (include/hss_routines.h, include/hss_routines_omp.h) ----
void* hmref_hss_build(const double* A, int N, int lda, int leaf, double tol, int rsvd_rank,
                      unsigned seed, int omp) {
    auto* b = new HssBox();
    b->omp = omp;
    Matrix Am = from_ptr(A, N, N, lda);
    g_hmref_seed = seed;
    if (omp) {
        b->par = new HSSMatrixOMP(tol);
        b->par->rsvd_rank = rsvd_rank;
        b->par->build_from_dense(Am, leaf);
    } else {
        b->ser = new HSSMatrix(tol);
        b->ser->rsvd_rank = rsvd_rank;
        on_fresh_thread([&] { b->ser->build_from_dense(Am, leaf); });
    }
    return b;
}

void hmref_hss_free(void* h) {
    auto* b = static_cast<HssBox*>(h);
    delete b->ser;
    delete b->par;
    delete b;
}

int hmref_hss_num_nodes(void* h) { return (int)static_cast<HssBox*>(h)->nodes().size(); }

// Per node in `nodes` (id) order: id, idx_start, idx_end, is_leaf, left id, right id,
// parent id, rank_U, rank_V (-1 for a missing link).
void hmref_hss_tree(void* h, int* id, int* start, int* end, int* is_leaf, int* left, int* right,
                    int* parent, int* rank_u, int* rank_v) {
    auto& nodes = static_cast<HssBox*>(h)->nodes();
    for (size_t i = 0; i < nodes.size(); ++i) {
        HSSNode* n = nodes[i];
        id[i] = n->id;
        start[i] = n->idx_start;
        end[i] = n->idx_end;
        is_leaf[i] = n->is_leaf ? 1 : 0;
        left[i] = n->left ? n->left->id : -1;
        right[i] = n->right ? n->right->id : -1;
        parent[i] = n->parent ? n->parent->id : -1;
        rank_u[i] = n->rank_U;
        rank_v[i] = n->rank_V;
    }
}

// which: 0 = D, 1 = U, 2 = V, 3 = R, 4 = W, 5 = B
static const Matrix& hss_mat(HSSNode* n, int which) {
    switch (which) {
        case 0: return n->D;
        case 1: return n->U;
        case 2: return n->V;
        case 3: return n->R;
        case 4: return n->W;
        default: return n->B;
    }
}

void hmref_hss_factor_shape(void* h, int node, int which, int* rows, int* cols) {
    const Matrix& M = hss_mat(static_cast<HssBox*>(h)->nodes()[node], which);
    *rows = M.rows();
    *cols = M.cols();
}

void hmref_hss_factor(void* h, int node, int which, double* out) {
    to_ptr(hss_mat(static_cast<HssBox*>(h)->nodes()[node], which), out);
}

void hmref_hss_multiply(void* h, const double* x, double* y) {
    auto* b = static_cast<HssBox*>(h);
    int N = b->omp ? b->par->N : b->ser->N;
    Matrix xm = from_ptr(x, N, 1, N);
    Matrix ym = b->omp ? b->par->multiply(xm) : b->ser->multiply(xm);
    to_ptr(ym, y);
}

// The serial solve handles several columns (solve_multi_rhs, hss_routines.h:281-290);
// the OMP solve reads column 0 only (hss_routines_omp.h:235-245).
void hmref_hss_solve(void* h, const double* rhs, int nrhs, double* x) {
    auto* b = static_cast<HssBox*>(h);
    int N = b->omp ? b->par->N : b->ser->N;
    if (b->omp) {
        for (int j = 0; j < nrhs; ++j) {
            Matrix bm = from_ptr(rhs + (size_t)j * N, N, 1, N);
            to_ptr(b->par->solve(bm), x + (size_t)j * N);
        }
    } else {
        Matrix bm = from_ptr(rhs, N, nrhs, N);
        to_ptr(b->ser->solve(bm), x);
    }
}

}  // extern "C"
