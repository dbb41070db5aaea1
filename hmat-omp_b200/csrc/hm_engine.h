// Host-side engine: tree planning, device storage of the factors, and the recorded
// level-synchronous launch sequences (build, factor, solve, multiply).
#pragma once

#include <map>
#include <memory>

#include "hm_dense.h"

namespace hm {

// One tree node.  HODLR nodes are kept in pre-order (root, left subtree, right
// subtree: the recursion order of hodlr_routines.h:27-45); HSS nodes in build_topo id
// order (hss_routines.h:293-306).
struct Node {
    int start = 0, end = 0, depth = 0;
    int is_leaf = 0;
    int left = -1, right = -1, parent = -1;
    int sys = 0;   // independent system this node belongs to (batches); rows are global
    int len() const { return end - start; }
    int mid() const { return (start + end) / 2; }
    // Basis blocks owned by a non-root node (rows of this node):
    //   U: len x rankU (HODLR: from the parent's block with this node as row side)
    //   V: len x rankV
    size_t offU = 0, offV = 0;
    int capU = 0, capV = 0;
    int rankU = 0, rankV = 0;
    // Leaf: D (len x len).  Internal: dense B12 (p1 x q2), B21 (p2 x q1).
    size_t offD = 0;
    size_t offB12 = 0, offB21 = 0;
    // factor storage (internal): Minv ((q1+q2)^2, FP64) and P ((p1+p2) x (q1+q2))
    size_t offM = 0, offP = 0;
    // FP32 factor store: P with a zero gap after its first block (rows p1 .. p1 rounded up
    // to 4), so delta's second block starts 16-byte aligned for the tensor-core kernel
    size_t offP32 = 0;
};

class Engine;
std::vector<Node> hodlr_tree(int N, int leaf);
std::vector<Node> hss_tree(int N, int leaf);

// Where the operator's entries come from during a build: a dense device matrix, or a
// kernel generator evaluated from point coordinates (matrix-free).
struct Source {
    const double* dA = nullptr;
    int lda = 0;
    int gen = GEN_DENSE;
    GenParams gp;
    bool dense() const { return gen == GEN_DENSE; }
    const double* blk(int r0, int c0) const { return dense() ? dA + r0 + (size_t)c0 * lda : nullptr; }
};

// Per-precision factorization storage.
template <typename T>
struct FactorStore {
    DBuf<T> Q;      // like U: A_child^{-1} U_child
    DBuf<T> V;      // V in precision T (FP64: unused, the FP64 V is used)
    DBuf<T> P;      // B^ Minv per internal node
    DBuf<T> Dinv;   // leaf inverses in precision T (FP64: unused)
    bool ready = false;
    bool planned = false;
    DBuf<T> Utmp;                              // U in precision T (FP32 only)
    std::vector<std::unique_ptr<Plan>> plans;  // leaf step, then one per level
    std::unique_ptr<Plan> setup;               // once per build: bases converted to T
    bool setup_done = false;
};

class Engine {
  public:
    enum Kind { HODLR = 0, HSS = 1 };
    Engine(const hm_opts& o, Kind kind) : opts_(o), kind_(kind) {}
    virtual ~Engine() = default;

    Kind kind() const { return kind_; }
    int N() const { return N_; }
    const std::vector<Node>& nodes() const { return nodes_; }

    void set_stream(cudaStream_t s) { stream_ = s; }
    // Fixed kept ranks for the next HODLR builds (B_12 / B_21 size per node, pre-order),
    // instead of the truncation rule; empty vectors restore the rule.
    void set_rank_profile(const std::vector<int>& r12, const std::vector<int>& r21) {
        fix12_ = r12;
        fix21_ = r21;
    }
    // Next HSS builds: nested bases with compressed transfers R / W (true) or the
    // reference's identity transfers (false, the default).
    void set_hss_nested(bool on) { hss_nested_ = on; }
    bool hss_nested() const { return hss_.nested; }
    void set_precision(int p) {
        if (p != opts_.precision) factored_ = false;
        opts_.precision = p;
    }
    cudaStream_t stream() const { return stream_; }

    // builds
    void build_dense_device(const double* dA, int N, int lda, int leaf);
    // Matrix-free build: points (host) in the layout GenParams documents.
    void build_kernel(int gen, const double* pts_host, size_t npts, int dim, int N, double p0, double p1,
                      int leaf);
    // Many independent HODLR systems built from one kernel with per-system parameters
    // (points concatenated system after system); all share every launch.
    void build_batch_kernel(int gen, const double* pts_host, int dim, int nsys, const int* Ns,
                            const double* p0s, const double* p1s, int leaf);
    // Packed right-hand sides: system k's N_k x s_k block at offset sum_{j<k} N_j s_j.
    void batch_solve(const double* b, const int* nrhs, double* x);
    void batch_multiply(const double* x, const int* nrhs, double* y);
    int num_systems() const { return (int)sys_N_.size(); }
    void import_hodlr(int N, int leaf, const int* r12, const int* r21, const double* const* D,
                      const double* const* U, const double* const* V, const double* const* B12,
                      const double* const* B21);
    // operations on device buffers
    void multiply_device(const double* dx, int s, int ldx, double* dy, int ldy);
    void factor();
    void solve_device(const double* db, int s, int ldb, double* dx, int ldx, hm_solve_stats* st);
    // factor, then solve (host or device b/x); a host b is copied while the factor runs
    void factor_solve(const double* b, int s, int ldb, double* x, int ldx, hm_solve_stats* st);
    // refinement against the exact kernel operator (matrix-free builds)
    void solve_exact_device(const double* db, int s, int ldb, double* dx, int ldx, double tol, int max_iter,
                            hm_solve_stats* st);
    // flexible GMRES(restart) against the exact kernel operator, right-preconditioned by
    // the compressed factorization (hm_krylov.cu)
    void solve_gmres_device(const double* db, int s, int ldb, double* dx, int ldx, double tol, int restart,
                            int max_iter, hm_solve_stats* st);
    // dx = A~^{-1} db with the handle's factorization, once (mixed: one FP32 sweep); ld N
    void precondition_device(const double* db, int s, double* dx);
    // per-column ||b - A x|| / ||b|| against the exact kernel operator (matrix-free builds)
    void residual_exact(const double* db, int ldb, const double* dx, int ldx, int s, double* rel);
    // adjoint solve and gradient accumulation
    void solve_transpose_device(const double* dg, int s, int ldg, double* dl, int ldl);
    void gradients(const double* dx, int ldx, const double* dl, int ldl, int s, double* dparams);
    void get_gradient(int node, int which, double* out, int* rows, int* cols) const;

    // serialized operators (hm_io.cu): the built operator to / from one file
    void save(const char* path) const;
    void load(const char* path);
    static int file_kind(const char* path);   // HODLR or HSS, after checking the header

    // introspection
    void export_tree(int* start, int* end, int* is_leaf, int* depth, int* r12, int* r21) const;
    void get_factor(int node, int which, double* out, int* rows, int* cols) const;

    // Read-only view of the FP64 operator storage (for entry points that build their
    // own launch tables).
    struct View {
        const std::vector<Node>* nodes;
        const std::vector<int>* leaves;
        const std::vector<std::vector<int>>* levels;
        const double *D, *U, *V, *B;
        int N;
        bool built;
        int device;   // the CUDA device the operator's storage lives on
    };
    View view() const { return {&nodes_, &leaves_, &levels_, dD.p, dU.p, dV.p, dB.p, N_, built_, device_}; }

  protected:
    void plan_levels();
    void alloc_bases();
    void alloc_D();
    void alloc_UV();
    // sketches for RSVD blocks, in draw order: host mt19937 stream or device normals
    void make_sketches(DBuf<double>& dOmega, const std::vector<std::pair<size_t, size_t>>& blocks);
    void begin_build(int N, int leaf);
    void build_hodlr(const Source& src);
    void build_hss(const Source& src);
    // nested-basis levels above the leaf strips (hm_hss_nested.cu)
    void build_hss_nested(const Source& src);
    // telescoping product of a nested-basis operator (hm_hss_nested.cu): X, Y ld N
    void add_matvec_nested(Plan& pl, const double* X, double* Y, int s);
    void reduce_hss_coupling(const std::vector<std::vector<int>>& under);
    // Append steps materialising blocks (dense copy or generator fill).
    void add_block_fill(Plan& plan, const Source& src,
                        const std::vector<std::tuple<int, int, int, int, int, double*, int>>& blocks);
    void check_status(const char* what);
    template <typename T> void factor_t(FactorStore<T>& fs);
    template <typename T> void plan_factor(FactorStore<T>& fs);
    template <typename T> Plan& solve_plan(FactorStore<T>& fs, const std::vector<int>& sc);
    Plan& matvec_plan(const std::vector<int>& sc);
    std::vector<int> uniform(int s) const { return std::vector<int>(sys_N_.size(), s); }
    Plan& solveT_plan(int s);
    Plan& exact_plan(int s);
    Plan grad_plan(int s);
    void ensure_io(int s);
    std::vector<int> path_of(int n) const;   // n and its ancestors below the root
    void solve_fp64(const double* db, int s, int ldb, double* dx, int ldx);
    const double* refined_fp64(const std::vector<int>& sc, int smax);
    void solve_mixed(const double* db, int s, int ldb, double* dx, int ldx, hm_solve_stats* st);

    hm_opts opts_;
    Kind kind_;
    cudaStream_t stream_ = nullptr;
    int N_ = 0, leaf_ = 0;
    int device_ = 0;   // current device when the operator was built (or loaded)
    std::vector<Node> nodes_;
    std::vector<std::vector<int>> levels_;   // internal nodes by depth
    std::vector<int> leaves_;
    // FP64 operator storage
    DBuf<double> dD, dU, dV, dB;
    DBuf<int> dstatus;
    DBuf<double> dPts;             // generator points (matrix-free builds)
    // HSS: compressed leaf bases (offset into dLeafB, rank) per leaf node
    DBuf<double> dLeafB;
    std::vector<std::pair<size_t, int>> leafU_, leafV_;
    // HSS: the reference's representation, kept for export: rank_U / rank_V of every
    // node (sums over its leaves) and the coupling blocks at those widths.  The operator
    // in nodes_/dU/dV/dB that factor, solve and multiply use is its recompressed
    // two-block form (reduce_hss_coupling).
    // Nested-basis builds keep here their compressed transfers instead: R of internal node
    // t is (rankU[left] + rankU[right]) x rankU[t] at RW + offR[t], W likewise, B12/B21
    // at the nested ranks, and the root's ranks are 0 (it has no off-diagonal strip).
    struct HssForm {
        std::vector<int> rankU, rankV;
        std::vector<size_t> offB12, offB21;
        DBuf<double> B;
        bool nested = false;
        std::vector<size_t> offR, offW;
        DBuf<double> RW;
    } hss_;
    bool hss_nested_ = false;   // mode of the next HSS build
    bool built_ = false;
    // factorizations
    FactorStore<double> f64_;
    FactorStore<float> f32_;
    DBuf<double> dDinv, dMinv;    // FP64 leaf and capacitance inverses
    size_t sizeM_ = 0, sizeP_ = 0;
    bool factored_ = false;
    // I/O staging buffers (ld = N)
    DBuf<double> ioX, ioY, ioR, ioNorm, ioAcc;
    DBuf<float> ioXf, ioYf;
    int io_cols_ = 0;
    std::map<std::vector<int>, Plan> mv_plans_, solve64_plans_, solve32_plans_;
    std::map<int, Plan> solveT_plans_;
    // factor_solve: device copy of a host b, and the stream/event that carry it
    DBuf<double> fsB_;
    std::shared_ptr<CUstream_st> copy_stream_;
    std::shared_ptr<CUevent_st> copy_done_, x_ready_;
    void ensure_copy_stream();
    // exact-operator refinement: b, x, r, correction (N x ex_cols_), norms, A x plans
    DBuf<double> exB_, exX_, exR_, exD_, exNorm_;
    int ex_cols_ = 0;
    std::map<int, Plan> exact_plans_;
    // independent systems sharing the launches: size and first global row of each
    std::vector<int> sys_N_{0}, sys_off_{0};
    DBuf<int> dRowSys;
    DBuf<double> dSysP0, dSysP1, ioPacked;
    // the build's operator source (kernel generator and its parameters) and gradients
    int gen_ = GEN_DENSE;
    GenParams gp_;
    // every diagonal (leaf) block is symmetric positive definite: Gaussian and Coulomb
    // kernels with positive scale and non-negative shift (positive definite radial
    // functions), set by the kernel builds; dense builds and imports stay false
    bool leaves_spd_ = false;
    std::vector<int> fix12_, fix21_;   // fixed rank profile (empty: the truncation rule)
    static bool kernel_spd(int gen, double p0, double p1) {
        return (gen == GEN_GAUSSIAN || gen == GEN_COULOMB) && p0 > 0 && p1 >= 0;
    }
    DBuf<double> gD_, gU_, gV_, gB_, gAcc_;
    std::map<int, Plan> grad_plans_;   // per column count, recorded once per operator
    bool grads_ready_ = false;
};

}  // namespace hm

namespace hm {
// The multiply of Engine::multiply_device without device allocation: intermediates and
// launch tables in a fixed file-scope device array (hm_noalloc.cu).
void multiply_noalloc(const Engine::View& v, const double* dx, int s, int ldx, double* dy, int ldy,
                      cudaStream_t st);
}  // namespace hm
