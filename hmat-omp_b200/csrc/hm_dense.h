// Small batched dense kernels (one CTA per problem) and the host plans that chain
// them with the batched GEMM: inverses, Gram/Jacobi SVDs, copies.
#pragma once

#include <cstdlib>

#include <algorithm>
#include <memory>
#include <string>

#include "hm_gemm.h"

namespace hm {

// Largest matrix inverted directly (in registers) by Gauss-Jordan; larger inverses run
// the block Gauss-Jordan sweep with panel pivoting (plan_inverse).
constexpr int GJ_MAX = 128;
// Widest sketch (rsvd_rank + oversample) and full-SVD block the Jacobi kernels take.
constexpr int SKETCH_MAX = 160;
// Largest Gram matrix held in shared memory by the Jacobi eigen-solver, and the largest
// whose eigenvector matrix is accumulated there too (both: 2 k^2 doubles <= ~190 KB).
constexpr int JAC_SMEM_MAX = 128;
constexpr int JAC_W_SMEM_MAX = 108;

struct GJDesc {
    const double* A;
    int lda;
    double* X;
    int ldx;
    int n;
};

struct EigDesc {
    double* G;     // k x k symmetric (overwritten)
    int ldg;
    double* W;     // k x k eigenvectors (output)
    int ldw;
    double* lam;   // k eigenvalues (output, unsorted)
    int k;
};

// Column norms of a tall block.
struct NormDesc {
    const double* X;
    int ld;
    int rows, k;
    double* out;         // k
};

// Sort singular values (descending) and derive the truncation rank.
struct PrepDesc {
    const double* sig_in;  // k, unsorted
    double* sigma;         // k, sorted (nullptr allowed)
    int* perm;             // k: sorted position -> source column
    int* rank;             // truncation rank (nullptr allowed)
    int k;
};

// dst[:, c] = src[:, perm[c]] / sig[c]  (sig == nullptr: no scaling; sig[c] == 0: zero column)
struct PermDesc {
    const double* src;
    int lds;
    double* dst;
    int ldd;
    int rows, k;
    const int* perm;
    const double* sig;
};

struct CopyDesc {
    const void* src;     // double, or float when src_f32
    int lds;
    void* dst;           // double, or float when dst_f32
    int ldd;
    int rows, cols;      // of the destination
    int trans;           // dst(i,j) = src(j,i)
    int src_f32 = 0;
    int dst_f32 = 0;
};

struct IdentDesc {
    double* X;
    int ldx;
    int rows, cols;
    double diag;
};

template <typename T>
struct DevTable {
    std::vector<T> h;
    DBuf<T> d;
    void upload(cudaStream_t s) {
        if (h.empty()) return;
        d.alloc(h.size());
        HM_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    int size() const { return (int)h.size(); }
};

void launch_gj(const DevTable<GJDesc>& t, int nb, int* status, cudaStream_t s);
void launch_jacobi(const DevTable<EigDesc>& t, int* status, cudaStream_t s, int max_sweeps = 60);
void launch_prep(const DevTable<PrepDesc>& t, double tol, int max_rank, cudaStream_t s);
void launch_norms(const DevTable<NormDesc>& t, cudaStream_t s);
void launch_permute(const DevTable<PermDesc>& t, cudaStream_t s);
void launch_copy(const DevTable<CopyDesc>& t, cudaStream_t s);
void launch_ident(const DevTable<IdentDesc>& t, cudaStream_t s);

// Process-wide launch counter and optional per-step CUDA-event timing.
struct Profiler {
    struct Rec {
        std::string name;
        cudaEvent_t a, b;
        double flops, bytes;
        int launches;
        std::string sig;   // tuning signature and tile choice of a GEMM step ("" otherwise)
    };
    bool enabled = false;
    long long launches = 0;
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    static Profiler& get();
    cudaEvent_t event();
    void reset();
    // {"name": [launches, ms, flops, bytes], ...} (synchronises)
    std::string report();
    // [["name", launches, ms, flops, bytes, "signature#bn,small,tc"], ...] in record
    // order (synchronises)
    std::string sequence();
};
inline void count_launch(int n = 1) { Profiler::get().launches += n; }

// A recorded sequence of batched launches (the unit that is replayed or captured).
class Plan {
  public:
    struct Step {
        virtual ~Step() = default;
        virtual void run(cudaStream_t s, int* status) const = 0;
        virtual const char* name() const = 0;
        virtual int nlaunch() const { return 1; }
        virtual double flops() const { return 0; }
        virtual double bytes() const { return 0; }
        virtual std::string sig() const { return ""; }
    };
    void add(std::unique_ptr<Step> st) { steps_.push_back(std::move(st)); }
    // Runs the steps in order on s.  The first run launches them one by one; the second
    // captures them into a CUDA graph (one per plan, i.e. per tree shape and column
    // count) and every run from then on replays that graph.  Runs launch one by one
    // instead while the profiler is on, on the legacy default stream, on a stream the
    // caller is already capturing (the launches then join the caller's graph), or with
    // HM_CUDA_GRAPHS=0.  A plan captured with one status word is re-captured if run
    // with another.
    void run(cudaStream_t s, int* status) const;
    bool empty() const { return steps_.empty(); }
    // device scratch owned by the plan (bump-allocated from large chunks)
    double* scratch(size_t count) { return static_cast<double*>(bump(count * sizeof(double))); }
    float* scratch_f(size_t count) { return static_cast<float*>(bump(count * sizeof(float))); }
    int* scratch_i(size_t count) { return static_cast<int*>(bump(count * sizeof(int))); }
    void clear() {
        graph_.reset();
        runs_ = 0;
        steps_.clear();
        chunks_.clear();
        used_ = cap_ = 0;
        ext_ = nullptr;
        ext_cap_ = ext_used_ = 0;
    }
    size_t scratch_bytes() const {
        size_t b = 0;
        for (auto& c : chunks_) b += c.n;
        return b;
    }
    // Serve scratch from caller-owned device memory first (the plan neither frees it nor
    // may outlive it); requests that no longer fit fall back to owned chunks.  Loops that
    // build one plan per chunk of work reuse one workspace this way instead of allocating
    // and freeing (a device synchronisation) their scratch chunk by chunk.
    void use_arena(void* base, size_t bytes) {
        ext_ = static_cast<unsigned char*>(base);
        ext_cap_ = bytes;
        ext_used_ = 0;
    }

  private:
    void* bump(size_t bytes) {
        bytes = align_up(std::max<size_t>(bytes, 1), 256);
        if (ext_ && ext_used_ + bytes <= ext_cap_) {
            void* p = ext_ + ext_used_;
            ext_used_ += bytes;
            return p;
        }
        if (chunks_.empty() || used_ + bytes > cap_) {
            size_t c = std::max<size_t>(bytes, size_t(64) << 20);
            chunks_.emplace_back(c);
            used_ = 0;
            cap_ = c;
        }
        void* p = chunks_.back().p + used_;
        used_ += bytes;
        return p;
    }
    void capture(cudaStream_t s, int* status) const;
    std::vector<std::unique_ptr<Step>> steps_;
    std::vector<DBuf<unsigned char>> chunks_;
    size_t used_ = 0, cap_ = 0;
    unsigned char* ext_ = nullptr;
    size_t ext_cap_ = 0, ext_used_ = 0;
    mutable std::shared_ptr<CUgraphExec_st> graph_;
    mutable int* graph_status_ = nullptr;
    mutable int runs_ = 0;
};
bool graphs_enabled();

// Which labelled FP32 steps may run on the tensor cores.  By default the bulk updates of
// the factorization (leaf_apply, update_project, update_small, update_correct) and the
// solve's correction (solve.correct: k = a node's rank, short).  The rest of the
// mixed-precision path feeds the refinement more directly: on the tensor cores the
// projection K = V^T Q (amplified by the capacitance matrices) or the solve's long-k
// steps weaken the refinement contraction (measured at N = 2^18, 64 right-hand sides:
// residual after two sweeps 2.6e-10 with K added, 1.1e-10 with the solve's leaf step
// added, against 5.5e-11 with the default set).  HM_FP32_TENSOR_CORES overrides: "0"
// none, "1" every eligible step, otherwise a comma-separated label list.
inline bool tensor_cores_allowed(const char* label) {
    const char* e = std::getenv("HM_FP32_TENSOR_CORES");
    const std::string l(label);
    if (!e || !*e)
        return l == "factor.leaf_apply" || l == "factor.update_project" || l == "factor.update_small" ||
               l == "factor.update_correct" || l == "solve.correct";
    if (e[0] == '1' && e[1] == 0) return true;
    if (e[0] == '0' && e[1] == 0) return false;
    const std::string list = std::string(",") + e + ",";
    return list.find("," + l + ",") != std::string::npos;
}

// Whether the tensor-core kernel takes this label's batches even when their inner
// dimension is short (fewer than 4 k-blocks per tile): the default short-k steps, or the
// labels HM_FP32_TENSOR_CORES names explicitly.
inline bool tensor_cores_named(const char* label) {
    const char* e = std::getenv("HM_FP32_TENSOR_CORES");
    if (!e || !*e) {   // the default short-k steps (3 k-blocks of 32 per tile)
        const std::string l(label);
        return l == "factor.update_correct" || l == "solve.correct";
    }
    if ((e[0] == '1' && e[1] == 0) || (e[0] == '0' && e[1] == 0)) return false;
    const std::string list = std::string(",") + e + ",";
    return list.find("," + std::string(label) + ",") != std::string::npos;
}

template <typename T>
struct GemmStep : Plan::Step {
    GemmBatch<T> batch;
    GenParams gp;
    std::string label;      // optional profile label (which step of which phase)
    std::string label_tc;   // the same when the batch runs on the tensor cores
    explicit GemmStep(int cfg = CFG_64x64, int gen = GEN_DENSE) : batch(cfg, gen) {}
    GemmStep(const char* lbl) : batch(CFG_64x64, GEN_DENSE) {
        batch.set_tag(lbl);
        label = std::string(sizeof(T) == 8 ? "gemm_f64:" : "gemm_f32:") + lbl;
        label_tc = std::string("tc_tf32x4:") + lbl;
        batch.allow_tensor_cores(tensor_cores_allowed(lbl), tensor_cores_named(lbl));
    }
    void run(cudaStream_t s, int* st) const override { batch.launch(s, gp, st); }
    const char* name() const override {
        if (batch.on_tensor_cores()) return label.empty() ? "tc_tf32x4" : label_tc.c_str();
        if (!label.empty()) return label.c_str();
        if (batch.gen() != GEN_DENSE) return "gemm_kernel_gen_f64";
        return sizeof(T) == 8 ? "gemm_f64" : "gemm_f32";
    }
    int nlaunch() const override { return batch.nlaunch(); }
    double flops() const override { return batch.flops(); }
    double bytes() const override { return batch.bytes(); }
    std::string sig() const override { return batch.signature() + "#" + batch.choice(); }
};

struct GJStep : Plan::Step {
    DevTable<GJDesc> t[4];   // n <= 32, <= 64, <= 96, <= 128
    void run(cudaStream_t s, int* st) const override {
        launch_gj(t[0], 32, st, s);
        launch_gj(t[1], 64, st, s);
        launch_gj(t[2], 96, st, s);
        launch_gj(t[3], 128, st, s);
    }
    const char* name() const override { return "gauss_jordan_inverse"; }
    int nlaunch() const override {
        return !t[0].h.empty() + !t[1].h.empty() + !t[2].h.empty() + !t[3].h.empty();
    }
    double flops() const override {
        double f = 0;
        for (auto& tb : t)
            for (auto& d : tb.h) f += 2.0 * d.n * d.n * (double)d.n;
        return f;
    }
    double bytes() const override {
        double b = 0;
        for (auto& tb : t)
            for (auto& d : tb.h) b += 16.0 * d.n * d.n;
        return b;
    }
};
struct EigStep : Plan::Step {
    DevTable<EigDesc> t;
    void run(cudaStream_t s, int* st) const override { launch_jacobi(t, st, s); }
    const char* name() const override { return "jacobi_eigen"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};
struct PrepStep : Plan::Step {
    DevTable<PrepDesc> t;
    double tol = 0;
    int max_rank = 0;
    void run(cudaStream_t s, int*) const override { launch_prep(t, tol, max_rank, s); }
    const char* name() const override { return "sort_rank"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};
struct NormStep : Plan::Step {
    DevTable<NormDesc> t;
    void run(cudaStream_t s, int*) const override { launch_norms(t, s); }
    const char* name() const override { return "column_norms"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};
struct PermStep : Plan::Step {
    DevTable<PermDesc> t;
    void run(cudaStream_t s, int*) const override { launch_permute(t, s); }
    const char* name() const override { return "permute_scale"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};
struct GenFillStep : Plan::Step {
    DevTable<GenFillDesc> t;
    int gen = GEN_DENSE;
    GenParams gp;
    void run(cudaStream_t s, int*) const override {
        int mx = 0;
        for (auto& d : t.h) mx = std::max(mx, d.rows * d.cols);
        launch_gen_fill(t.d.p, t.size(), mx, gen, gp, s);
    }
    const char* name() const override { return "kernel_fill"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};
struct CopyStep : Plan::Step {
    DevTable<CopyDesc> t;
    void run(cudaStream_t s, int*) const override { launch_copy(t, s); }
    const char* name() const override { return "copy"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};
struct IdentStep : Plan::Step {
    DevTable<IdentDesc> t;
    void run(cudaStream_t s, int*) const override { launch_ident(t, s); }
    const char* name() const override { return "identity_fill"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};

// X_i = inv(A_i) for a batch of square FP64 matrices (n <= 16384), with partial
// pivoting at every size: Gauss-Jordan up to the threshold (64 unless HM_GJ_MAX says
// otherwise), block Gauss-Jordan with panel pivoting above it.  X may alias A.
// Appends the launches to `plan`.
struct InvProblem {
    const double* A;
    int lda;
    double* X;
    int ldx;
    int n;
};
void plan_inverse(Plan& plan, const std::vector<InvProblem>& probs, cudaStream_t s);
// The same for matrices known to be symmetric positive definite: unpivoted 2 x 2 block
// elimination above order 64 (backward stable for SPD).  X may not alias A.
void plan_inverse_spd(Plan& plan, const std::vector<InvProblem>& probs, cudaStream_t s);

// Orthonormal basis Q_i (rows x k) of range(X_i) by shifted CholeskyQR3 (Gram matrices,
// batched Cholesky, X R^{-1}); directions X_i does not contain give zero columns.  Q may
// not alias X.
struct QrProblem {
    const double* X;
    int ldx;
    int rows, k;
    double* Q;
    int ldq;
};
void plan_cholqr3(Plan& plan, const std::vector<QrProblem>& probs, cudaStream_t s);

// Gram/Jacobi SVD of tall X_i (rows x k): X = L diag(sigma) R^T with L (rows x k)
// orthonormal columns and R (k x k) orthogonal, sigma sorted descending; optionally
// the truncation rank.  Each round rotates X by the eigenvectors of its Gram matrix
// (X <- X W, W from Jacobi on X^T X); a Gram matrix resolves about half of the double
// precision range of singular values relative to its own columns, so three rounds
// separate the full range (sigma down to ~1e-16 sigma_0).  sigma is taken from the
// column norms of the final rotated X, not from the Gram diagonal.
struct SvdProblem {
    const double* X;
    int ldx;
    int rows, k;
    double* L;      // rows x k (may alias X; nullptr: not needed)
    int ldl;
    double* R;      // k x k (nullptr: not needed, e.g. orthonormalisation only)
    int ldr;
    double* sigma;  // k (nullptr allowed)
    int* rank;      // nullptr allowed
    bool sort;
};
void plan_gram_svd(Plan& plan, const std::vector<SvdProblem>& probs, double tol, int max_rank,
                   cudaStream_t s, int rounds = 3);

}  // namespace hm
