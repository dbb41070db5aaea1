// extern "C" entry points of libhmat_b200.so (declared in include/hmat_b200.h).
// Every call converts C++ exceptions to an HM_* status and keeps the message in the
// handle for hm_last_error().
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>

#include "hm_engine.h"

struct hm_handle {
    hm_opts opts;
    std::string err;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::unique_ptr<hm::Engine> eng;
    std::vector<int> fix12, fix21;   // rank profile for the next HODLR builds
    bool hss_nested = false;          // next HSS builds: nested bases (hm_hss_set_nested)
};

namespace {

template <class F>
int guard(hm_handle* h, F&& f) {
    if (!h) return HM_ERR_ARG;
    try {
        f();
        h->err.clear();
        return HM_OK;
    } catch (const hm::Error& e) {
        h->err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return HM_ERR_CUDA;
    } catch (const std::exception& e) {
        h->err = e.what();
        return HM_ERR_CUDA;
    }
}

hm::Engine& engine(hm_handle* h, hm::Engine::Kind kind) {
    if (!h->eng || h->eng->kind() != kind) {
        h->eng = std::make_unique<hm::Engine>(h->opts, kind);
        h->eng->set_stream(h->stream);
        h->eng->set_rank_profile(h->fix12, h->fix21);
        h->eng->set_hss_nested(h->hss_nested);
    }
    return *h->eng;
}

hm::Engine& built(hm_handle* h) {
    if (!h->eng) throw hm::Error(HM_ERR_STATE, "no operator built on this handle");
    return *h->eng;
}

void validate(const hm_opts& o) {
    HM_CHECK(o.tol == o.tol, HM_ERR_ARG, "tol is NaN");
    HM_CHECK(o.rsvd_rank >= 0 && o.oversample >= 0 && o.rsvd_min_dim >= 1, HM_ERR_ARG, "bad rsvd options");
    HM_CHECK(o.rsvd_rank + o.oversample <= hm::SKETCH_MAX, HM_ERR_UNSUPPORTED,
             "rsvd_rank + oversample above the supported sketch width (160)");
    HM_CHECK(o.power_iters >= 0 && o.max_rank >= 0, HM_ERR_ARG, "bad power_iters/max_rank");
    HM_CHECK(o.sketch >= HM_SKETCH_REFERENCE_UNIFORM && o.sketch <= HM_SKETCH_DEVICE_NORMAL, HM_ERR_ARG,
             "bad sketch");
    HM_CHECK(o.precision == HM_FP64 || o.precision == HM_MIXED, HM_ERR_ARG, "bad precision");
}

template <typename T>
void gemm_batched(hm_handle* h, int count, const int* m, const int* n, const int* k, T alpha, const T* const* A,
                  const int* lda, int opA, const T* const* B, const int* ldb, int opB, T beta, T* const* C,
                  const int* ldc, int ksplit, int flags) {
    HM_CHECK(count >= 0 && (count == 0 || (m && n && k && A && lda && B && ldb && C && ldc)), HM_ERR_ARG,
             "gemm_batched: null array");
    HM_CHECK((opA == hm::OP_N || opA == hm::OP_T) && (opB == hm::OP_N || opB == hm::OP_T), HM_ERR_ARG,
             "gemm_batched: op must be 0 or 1");
    const int mode = flags & 3;
    const bool stall = (flags & HM_GEMM_TEST_STALL) != 0;
    HM_CHECK(mode <= 2 && (flags & ~(3 | HM_GEMM_TEST_STALL)) == 0, HM_ERR_ARG, "gemm_batched: bad flags");
    HM_CHECK(!stall || (mode == HM_GEMM_TENSOR_CORES && sizeof(T) == 4), HM_ERR_ARG,
             "gemm_batched: HM_GEMM_TEST_STALL needs HM_GEMM_TENSOR_CORES on FP32");
    HM_CHECK(ksplit >= 0, HM_ERR_ARG, "gemm_batched: ksplit must be >= 0");
    if (count == 0) return;
    cudaStream_t s = h->stream;
    hm::GemmBatch<T> batch;
    batch.set_tag("gemm_batched");
    batch.set_kernel(mode);
    batch.set_test_stall(stall);
    for (int i = 0; i < count; ++i) {
        HM_CHECK(m[i] >= 0 && n[i] >= 0 && k[i] >= 0, HM_ERR_ARG, "gemm_batched: negative size");
        const int ar = opA == hm::OP_N ? m[i] : k[i], br = opB == hm::OP_N ? k[i] : n[i];
        HM_CHECK(lda[i] >= std::max(1, ar) && ldb[i] >= std::max(1, br) && ldc[i] >= std::max(1, m[i]), HM_ERR_ARG,
                 "gemm_batched: leading dimension below the row count");
        if (m[i] == 0 || n[i] == 0) continue;
        HM_CHECK(C[i] && (k[i] == 0 || (A[i] && B[i])), HM_ERR_ARG, "gemm_batched: null matrix");
        int ks = ksplit;
        if (ks == 0 && beta != T(0) && beta != T(1)) ks = 1;
        batch.add(m[i], n[i], k[i], alpha, A[i], lda[i], opA, B[i], ldb[i], opB, beta, C[i], ldc[i], nullptr, ks);
    }
    if (batch.empty()) return;
    batch.finalize(s);
    hm::DBuf<int> status(1);
    status.zero(s);
    batch.launch(s, hm::GenParams(), status.p);
    hm::count_launch(batch.nlaunch());
    int st = 0;
    HM_CUDA(cudaMemcpyAsync(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    HM_CUDA(cudaStreamSynchronize(s));
    if (st & hm::ST_TIMEOUT) throw hm::Error(HM_ERR_TIMEOUT, "gemm_batched: tensor-core pipeline wait timed out");
}

}  // namespace

extern "C" {

void hm_opts_default(hm_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-6;           // HODLRMatrix(double tol = 1e-6)  hodlr_routines.h:16
    o->rsvd_rank = 64;       // rsvd_rank(64)                   hodlr_routines.h:16
    o->oversample = 10;      // k = rank_guess + 10              compression.h:74
    o->rsvd_min_dim = 256;   // m < 256 || n < 256 -> full SVD   compression.h:72
    o->power_iters = 0;
    o->max_rank = 0;
    o->sketch = HM_SKETCH_REFERENCE_UNIFORM;
    o->seed = 0;
    o->precision = HM_FP64;
    o->ir_tol = 1e-10;
    o->ir_max_iter = 30;
    o->refine_steps = 0;
}

int hm_create(const hm_opts* o, hm_handle** out) {
    if (!out) return HM_ERR_ARG;
    *out = nullptr;
    auto h = std::make_unique<hm_handle>();
    if (o) h->opts = *o;
    else hm_opts_default(&h->opts);
    int rc = guard(h.get(), [&] {
        validate(h->opts);
        int ndev = 0;
        HM_CUDA(cudaGetDeviceCount(&ndev));
        HM_CHECK(ndev > 0, HM_ERR_CUDA, "no CUDA device");
        HM_CUDA(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
        h->stream = h->own;
    });
    if (rc != HM_OK) return rc;
    *out = h.release();
    return HM_OK;
}

int hm_destroy(hm_handle* h) {
    if (!h) return HM_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->eng.reset();
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
    return HM_OK;
}

const char* hm_last_error(const hm_handle* h) { return h ? h->err.c_str() : "null handle"; }

int hm_set_stream(hm_handle* h, void* stream) {
    return guard(h, [&] {
        h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own;
        if (h->eng) h->eng->set_stream(h->stream);
    });
}

int hm_set_precision(hm_handle* h, int precision) {
    return guard(h, [&] {
        HM_CHECK(precision == HM_FP64 || precision == HM_MIXED, HM_ERR_ARG, "bad precision");
        h->opts.precision = precision;
        if (h->eng) h->eng->set_precision(precision);
    });
}

int hm_hodlr_build_from_dense_device(hm_handle* h, const double* dA, int N, int lda, int leaf) {
    return guard(h, [&] {
        engine(h, hm::Engine::HODLR).build_dense_device(dA, N, lda, leaf);
    });
}

int hm_hodlr_build_from_dense(hm_handle* h, const double* A, int N, int lda, int leaf) {
    return guard(h, [&] {
        HM_CHECK(A && N > 0 && lda >= N, HM_ERR_ARG, "build_from_dense: bad arguments");
        hm::DBuf<double> d((size_t)N * N);
        HM_CUDA(cudaMemcpy2DAsync(d.p, (size_t)N * sizeof(double), A, (size_t)lda * sizeof(double),
                                  (size_t)N * sizeof(double), N, cudaMemcpyHostToDevice, h->stream));
        engine(h, hm::Engine::HODLR).build_dense_device(d.p, N, N, leaf);
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

static void build_from_kernel(hm_handle* h, hm::Engine::Kind kind, int kernel, const double* points, int dim,
                              int N, const double* params, int nparams, int leaf) {
    HM_CHECK(points && N > 0 && dim >= 1, HM_ERR_ARG, "build_from_kernel: bad arguments");
    HM_CHECK(nparams >= 2 && params, HM_ERR_ARG, "build_from_kernel: two parameters expected");
    int gen = kernel == HM_KERNEL_CAUCHY ? hm::GEN_CAUCHY
              : kernel == HM_KERNEL_GAUSSIAN ? hm::GEN_GAUSSIAN
              : kernel == HM_KERNEL_COULOMB ? hm::GEN_COULOMB : -1;
    HM_CHECK(gen > 0, HM_ERR_ARG, "build_from_kernel: unknown kernel");
    HM_CHECK(kernel != HM_KERNEL_CAUCHY || dim == 1, HM_ERR_ARG, "Cauchy points are 1-D");
    size_t npts = kernel == HM_KERNEL_CAUCHY ? 2 * (size_t)N : (size_t)N * dim;
    engine(h, kind).build_kernel(gen, points, npts, dim, N, params[0], params[1], leaf);
    HM_CUDA(cudaStreamSynchronize(h->stream));
}

int hm_hodlr_build_from_kernel(hm_handle* h, int kernel, const double* points, int dim, int N,
                               const double* params, int nparams, int leaf) {
    return guard(h, [&] { build_from_kernel(h, hm::Engine::HODLR, kernel, points, dim, N, params, nparams, leaf); });
}

int hm_hss_build_from_kernel(hm_handle* h, int kernel, const double* points, int dim, int N,
                             const double* params, int nparams, int leaf) {
    return guard(h, [&] { build_from_kernel(h, hm::Engine::HSS, kernel, points, dim, N, params, nparams, leaf); });
}

int hm_hss_build_from_dense(hm_handle* h, const double* A, int N, int lda, int leaf) {
    return guard(h, [&] {
        HM_CHECK(A && N > 0 && lda >= N, HM_ERR_ARG, "build_from_dense: bad arguments");
        hm::DBuf<double> d((size_t)N * N);
        HM_CUDA(cudaMemcpy2DAsync(d.p, (size_t)N * sizeof(double), A, (size_t)lda * sizeof(double),
                                  (size_t)N * sizeof(double), N, cudaMemcpyHostToDevice, h->stream));
        engine(h, hm::Engine::HSS).build_dense_device(d.p, N, N, leaf);
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int hm_hss_set_nested(hm_handle* h, int nested) {
    return guard(h, [&] {
        h->hss_nested = nested != 0;
        if (h->eng) h->eng->set_hss_nested(h->hss_nested);
    });
}

int hm_hss_is_nested(const hm_handle* h) {
    return h && h->eng && h->eng->kind() == hm::Engine::HSS && h->eng->hss_nested() ? 1 : 0;
}

int hm_set_rank_profile(hm_handle* h, int nnodes, const int* rank12, const int* rank21) {
    return guard(h, [&] {
        if (!rank12 || !rank21 || nnodes <= 0) {
            h->fix12.clear();
            h->fix21.clear();
        } else {
            for (int i = 0; i < nnodes; ++i)
                HM_CHECK(rank12[i] >= 0 && rank21[i] >= 0, HM_ERR_ARG, "rank profile: negative rank");
            h->fix12.assign(rank12, rank12 + nnodes);
            h->fix21.assign(rank21, rank21 + nnodes);
        }
        if (h->eng) h->eng->set_rank_profile(h->fix12, h->fix21);
    });
}

int hm_hodlr_import(hm_handle* h, int N, int leaf, const int* r12, const int* r21, const double* const* D,
                    const double* const* U, const double* const* V, const double* const* B12,
                    const double* const* B21) {
    return guard(h, [&] { engine(h, hm::Engine::HODLR).import_hodlr(N, leaf, r12, r21, D, U, V, B12, B21); });
}

int hm_save(hm_handle* h, const char* path) {
    return guard(h, [&] { built(h).save(path); });
}

int hm_load(hm_handle* h, const char* path) {
    return guard(h, [&] {
        const auto kind = static_cast<hm::Engine::Kind>(hm::Engine::file_kind(path));
        engine(h, kind).load(path);
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int hm_num_nodes(const hm_handle* h) {
    if (!h || !h->eng) return 0;
    return (int)h->eng->nodes().size();
}

int hm_export_tree(const hm_handle* h, int* start, int* end, int* is_leaf, int* depth, int* r12, int* r21) {
    return guard(const_cast<hm_handle*>(h), [&] {
        built(const_cast<hm_handle*>(h)).export_tree(start, end, is_leaf, depth, r12, r21);
    });
}

int hm_get_factor(const hm_handle* h, int node, int which, double* out, int* rows, int* cols) {
    return guard(const_cast<hm_handle*>(h), [&] {
        built(const_cast<hm_handle*>(h)).get_factor(node, which, out, rows, cols);
    });
}

int hm_multiply_device(hm_handle* h, const double* dx, int nrhs, int ldx, double* dy, int ldy) {
    return guard(h, [&] { built(h).multiply_device(dx, nrhs, ldx, dy, ldy); });
}

int hm_multiply(hm_handle* h, const double* x, int nrhs, int ldx, double* y, int ldy) {
    return guard(h, [&] {
        built(h).multiply_device(x, nrhs, ldx, y, ldy);   // host pointers: unified addressing
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int hm_factor(hm_handle* h) {
    return guard(h, [&] { built(h).factor(); });
}

int hm_solve_device(hm_handle* h, const double* db, int nrhs, int ldb, double* dx, int ldx,
                    hm_solve_stats* st) {
    return guard(h, [&] { built(h).solve_device(db, nrhs, ldb, dx, ldx, st); });
}

int hm_solve(hm_handle* h, const double* b, int nrhs, int ldb, double* x, int ldx, hm_solve_stats* st) {
    return guard(h, [&] {
        built(h).solve_device(b, nrhs, ldb, x, ldx, st);    // host pointers: unified addressing
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int hm_factor_solve(hm_handle* h, const double* b, int nrhs, int ldb, double* x, int ldx, hm_solve_stats* st) {
    return guard(h, [&] {
        built(h).factor_solve(b, nrhs, ldb, x, ldx, st);
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int hm_solve_exact_device(hm_handle* h, const double* db, int nrhs, int ldb, double* dx, int ldx, double tol,
                          int max_iter, hm_solve_stats* st) {
    return guard(h, [&] { built(h).solve_exact_device(db, nrhs, ldb, dx, ldx, tol, max_iter, st); });
}

int hm_solve_gmres(hm_handle* h, const double* b, int nrhs, int ldb, double* x, int ldx, double tol, int restart,
                   int max_iter, hm_solve_stats* st) {
    return guard(h, [&] { built(h).solve_gmres_device(b, nrhs, ldb, x, ldx, tol, restart, max_iter, st); });
}

int hm_residual_exact(hm_handle* h, const double* b, int nrhs, int ldb, const double* x, int ldx, double* rel) {
    return guard(h, [&] { built(h).residual_exact(b, ldb, x, ldx, nrhs, rel); });
}

int hm_solve_exact(hm_handle* h, const double* b, int nrhs, int ldb, double* x, int ldx, double tol, int max_iter,
                   hm_solve_stats* st) {
    return guard(h, [&] {
        built(h).solve_exact_device(b, nrhs, ldb, x, ldx, tol, max_iter, st);   // host pointers: unified addressing
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int hm_batch_build_from_kernel(hm_handle* h, int kernel, const double* points, int dim, int nsys, const int* N,
                               const double* params, int leaf) {
    return guard(h, [&] {
        HM_CHECK(params && nsys >= 1, HM_ERR_ARG, "batch build: bad arguments");
        const int gen = kernel == HM_KERNEL_GAUSSIAN ? hm::GEN_GAUSSIAN : kernel == HM_KERNEL_COULOMB ? hm::GEN_COULOMB : -1;
        HM_CHECK(gen > 0, HM_ERR_ARG, "batch build: Gaussian or Coulomb kernel");
        std::vector<double> p0(nsys), p1(nsys);
        for (int k = 0; k < nsys; ++k) { p0[k] = params[2 * k]; p1[k] = params[2 * k + 1]; }
        engine(h, hm::Engine::HODLR).build_batch_kernel(gen, points, dim, nsys, N, p0.data(), p1.data(), leaf);
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int hm_num_systems(const hm_handle* h) { return (h && h->eng) ? h->eng->num_systems() : 0; }

int hm_batch_solve(hm_handle* h, const double* b, const int* nrhs, double* x) {
    return guard(h, [&] { built(h).batch_solve(b, nrhs, x); });
}

int hm_batch_multiply(hm_handle* h, const double* x, const int* nrhs, double* y) {
    return guard(h, [&] { built(h).batch_multiply(x, nrhs, y); });
}

int hm_solve_transpose_device(hm_handle* h, const double* dg, int nrhs, int ldg, double* dl, int ldl) {
    return guard(h, [&] { built(h).solve_transpose_device(dg, nrhs, ldg, dl, ldl); });
}

int hm_solve_transpose(hm_handle* h, const double* g, int nrhs, int ldg, double* lam, int ldl) {
    return guard(h, [&] {
        built(h).solve_transpose_device(g, nrhs, ldg, lam, ldl);   // host pointers: unified addressing
        HM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int hm_gradients(hm_handle* h, const double* x, int ldx, const double* lam, int ldl, int nrhs, double* dparams) {
    return guard(h, [&] { built(h).gradients(x, ldx, lam, ldl, nrhs, dparams); });
}

int hm_get_gradient(const hm_handle* h, int node, int which, double* out, int* rows, int* cols) {
    return guard(const_cast<hm_handle*>(h), [&] {
        built(const_cast<hm_handle*>(h)).get_gradient(node, which, out, rows, cols);
    });
}

int hm_multiply_device_noalloc(hm_handle* h, const double* dx, int nrhs, int ldx, double* dy, int ldy) {
    return guard(h, [&] {
        hm::Engine& e = built(h);
        hm::multiply_noalloc(e.view(), dx, nrhs, ldx, dy, ldy, e.stream());
    });
}

void hm_profile_enable(int on) {
    hm::Profiler& p = hm::Profiler::get();
    p.enabled = on != 0;
    p.reset();
}

long long hm_launch_count(void) { return hm::Profiler::get().launches; }

static size_t copy_out_text(const std::string& r, char* buf, size_t len) {
    if (buf && len) {
        size_t n = std::min(len - 1, r.size());
        std::memcpy(buf, r.data(), n);
        buf[n] = 0;
    }
    return r.size() + 1;
}

size_t hm_profile_report(char* buf, size_t len) {
    std::string r;
    try {
        r = hm::Profiler::get().report();
    } catch (const std::exception& e) {
        r = std::string("{\"error\": \"") + e.what() + "\"}";
    }
    return copy_out_text(r, buf, len);
}

size_t hm_profile_sequence(char* buf, size_t len) {
    std::string r;
    try {
        r = hm::Profiler::get().sequence();
    } catch (const std::exception& e) {
        r = std::string("[[\"error: ") + e.what() + "\", 0, 0, 0, 0]]";
    }
    return copy_out_text(r, buf, len);
}

int hm_tile_table_load(const char* path) { return hm::tile_table_load(path) ? HM_OK : HM_ERR_ARG; }

int hm_tile_table_size(void) { return hm::tile_table_size(); }

}  // extern "C"

extern "C" {

int hm_gemm_batched_f32_device(hm_handle* h, int count, const int* m, const int* n, const int* k, float alpha,
                               const float* const* A, const int* lda, int opA, const float* const* B, const int* ldb,
                               int opB, float beta, float* const* C, const int* ldc, int ksplit, int flags) {
    return guard(h, [&] { gemm_batched<float>(h, count, m, n, k, alpha, A, lda, opA, B, ldb, opB, beta, C, ldc, ksplit,
                                              flags); });
}

int hm_gemm_batched_f64_device(hm_handle* h, int count, const int* m, const int* n, const int* k, double alpha,
                               const double* const* A, const int* lda, int opA, const double* const* B,
                               const int* ldb, int opB, double beta, double* const* C, const int* ldc, int ksplit,
                               int flags) {
    return guard(h, [&] { gemm_batched<double>(h, count, m, n, k, alpha, A, lda, opA, B, ldb, opB, beta, C, ldc,
                                               ksplit, flags); });
}

int hm_inverse_batched_device(hm_handle* h, int count, const int* n, const double* const* A, const int* lda,
                              double* const* X, const int* ldx) {
    return guard(h, [&] {
        HM_CHECK(count >= 0 && (count == 0 || (n && A && lda && X && ldx)), HM_ERR_ARG, "inverse_batched: null array");
        std::vector<hm::InvProblem> probs;
        for (int i = 0; i < count; ++i) {
            HM_CHECK(n[i] >= 0 && lda[i] >= std::max(1, n[i]) && ldx[i] >= std::max(1, n[i]), HM_ERR_ARG,
                     "inverse_batched: bad order or leading dimension");
            if (n[i] == 0) continue;
            HM_CHECK(A[i] && X[i], HM_ERR_ARG, "inverse_batched: null matrix");
            probs.push_back({A[i], lda[i], X[i], ldx[i], n[i]});
        }
        if (probs.empty()) return;
        cudaStream_t s = h->stream;
        hm::Plan plan;
        hm::plan_inverse(plan, probs, s);
        hm::DBuf<int> status(1);
        status.zero(s);
        plan.run(s, status.p);
        int st = 0;
        HM_CUDA(cudaMemcpyAsync(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        HM_CUDA(cudaStreamSynchronize(s));
        if (st & hm::ST_SINGULAR) throw hm::Error(HM_ERR_SINGULAR, "inverse_batched: zero or non-finite pivot");
    });
}

int hm_kernel_block_product_device(hm_handle* h, int kernel, const double* points, int dim, int N,
                                   const double* params, int nparams, int r0, int r1, int c0, int c1, int trans,
                                   const double* dX, int ldx, int nrhs, double* dY, int ldy) {
    return guard(h, [&] {
        HM_CHECK(points && N > 0 && dim >= 1 && dim <= 3 && params && nparams >= 2, HM_ERR_ARG,
                 "kernel_block_product: bad arguments");
        const int gen = kernel == HM_KERNEL_CAUCHY ? hm::GEN_CAUCHY
                        : kernel == HM_KERNEL_GAUSSIAN ? hm::GEN_GAUSSIAN
                        : kernel == HM_KERNEL_COULOMB ? hm::GEN_COULOMB : -1;
        HM_CHECK(gen > 0, HM_ERR_ARG, "kernel_block_product: unknown kernel");
        HM_CHECK(kernel != HM_KERNEL_CAUCHY || dim == 1, HM_ERR_ARG, "Cauchy points are 1-D");
        HM_CHECK(0 <= r0 && r0 <= r1 && r1 <= N && 0 <= c0 && c0 <= c1 && c1 <= N, HM_ERR_ARG,
                 "kernel_block_product: row or column range outside [0, N)");
        const int m = trans ? c1 - c0 : r1 - r0, k = trans ? r1 - r0 : c1 - c0;
        HM_CHECK(nrhs >= 0 && ldx >= std::max(1, k) && ldy >= std::max(1, m), HM_ERR_ARG,
                 "kernel_block_product: bad column count or leading dimension");
        if (m == 0 || nrhs == 0) return;
        HM_CHECK(dY && (k == 0 || dX), HM_ERR_ARG, "kernel_block_product: null matrix");
        const size_t npts = kernel == HM_KERNEL_CAUCHY ? 2 * (size_t)N : (size_t)N * dim;
        for (size_t i = 0; i < npts; ++i)
            HM_CHECK(std::isfinite(points[i]), HM_ERR_NONFINITE, "kernel_block_product: non-finite point");
        cudaStream_t s = h->stream;
        hm::DBuf<double> dp(npts);
        HM_CUDA(cudaMemcpyAsync(dp.p, points, npts * sizeof(double), cudaMemcpyHostToDevice, s));
        hm::GenParams gp;
        gp.pts = dp.p;
        gp.N = N;
        gp.dim = dim;
        gp.p0 = params[0];
        gp.p1 = params[1];
        // the generated operand is op(A) with A(i, j) = entry(r0 + i, c0 + j)
        hm::GemmBatch<double> batch(nrhs <= 16 ? hm::CFG_N_SKINNY : hm::CFG_64x64, gen);
        batch.set_tag("kernel_block_product");
        batch.add(m, nrhs, k, 1.0, nullptr, 0, trans ? hm::OP_T : hm::OP_N, dX, ldx, hm::OP_N, 0.0, dY, ldy, nullptr, 0,
                  r0, c0);
        batch.finalize(s);
        hm::DBuf<int> status(1);
        status.zero(s);
        batch.launch(s, gp, status.p);
        hm::count_launch(batch.nlaunch());
        HM_CUDA(cudaStreamSynchronize(s));   // the points buffer outlives the launch
    });
}

}  // extern "C"
