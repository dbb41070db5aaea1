// Level-synchronous HODLR engine: every phase is a short sequence of batched launches
// per tree level, each launch covering all nodes of that level.
//
// Operator (per internal node n with children c1 = [s, mid), c2 = [mid, e)):
//   A_n = [[A_c1, U1 B12 V2^T], [U2 B21 V1^T, A_c2]]
// HODLR (hodlr_routines.h:55-61): U1 = left.U, V2 = right.V, B12 = diag(S) of A12's
// compression; U2 = right.U, V1 = left.V, B21 = diag(S) of A21's.
//
// Factorization (bottom-up; replaces the per-call recursion of hodlr_routines.h:112-175):
//   leaves:  Dinv = D^{-1};  Q_c[rows of leaf] = Dinv U_c[rows of leaf] for every basis
//            block c on the leaf's path to the root.
//   level d (deepest first), node n:  K1 = V1^T Q1, K2 = V2^T Q2,
//            M = [[I, K1 B12], [K2 B21, I]]  (= I + K B^, the stable capacitance form of
//            hss_routines.h:253-254), P = B^ M^{-1},
//            then for every basis block W on n's path: t = [V1^T W1; V2^T W2],
//            delta = P t, W1 -= Q1 delta_1, W2 -= Q2 delta_2.
// Solve: z = Dinv b per leaf, then the same update per level on z.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <random>

#include "hm_engine.h"

namespace hm {

// Rows of P in the FP32 factor store: p1 rounded up to a multiple of 4, then p2.
static inline int padded_p(int p1, int p2) { return (p1 + 3) / 4 * 4 + p2; }

template <> Plan& Engine::solve_plan<double>(FactorStore<double>& fs, const std::vector<int>& sc);
template <> Plan& Engine::solve_plan<float>(FactorStore<float>& fs, const std::vector<int>& sc);

// ---------------------------------------------------------------------------------
// Trees
// ---------------------------------------------------------------------------------
std::vector<Node> hodlr_tree(int N, int leaf) {
    std::vector<Node> out;
    std::function<int(int, int, int, int)> rec = [&](int s, int e, int d, int parent) -> int {
        int id = (int)out.size();
        out.emplace_back();
        out[id].start = s;
        out[id].end = e;
        out[id].depth = d;
        out[id].parent = parent;
        if (e - s <= leaf) {
            out[id].is_leaf = 1;
        } else {
            int m = (s + e) / 2;
            int l = rec(s, m, d + 1, id);
            int r = rec(m, e, d + 1, id);
            out[id].left = l;
            out[id].right = r;
        }
        return id;
    };
    rec(0, N, 0, -1);
    return out;
}

std::vector<Node> hss_tree(int N, int leaf) {
    std::vector<Node> out(1);
    out[0].start = 0;
    out[0].end = N;
    std::function<void(int)> rec = [&](int id) {
        Node n = out[id];
        if (n.end - n.start <= leaf) {
            out[id].is_leaf = 1;
            return;
        }
        int m = (n.start + n.end) / 2;
        int l = (int)out.size();
        out.emplace_back();
        out[l].start = n.start; out[l].end = m; out[l].depth = n.depth + 1; out[l].parent = id;
        int r = (int)out.size();
        out.emplace_back();
        out[r].start = m; out[r].end = n.end; out[r].depth = n.depth + 1; out[r].parent = id;
        out[id].left = l;
        out[id].right = r;
        rec(l);
        rec(r);
    };
    rec(0);
    return out;
}

// ---------------------------------------------------------------------------------
// Small device kernels used by the engine
// ---------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), keyed by the seed; one N(0,1)
// value per element via Box-Muller on the first two output words.
__device__ __forceinline__ void philox_round(uint32_t (&c)[4], uint32_t (&k)[2]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    uint32_t n0 = hi1 ^ c[1] ^ k[0], n1 = lo1, n2 = hi0 ^ c[3] ^ k[1], n3 = lo0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k[0] += 0x9E3779B9u;
    k[1] += 0xBB67AE85u;
}

__global__ void normal_fill_kernel(double* out, size_t count, unsigned long long seed,
                                   unsigned long long base) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count;
         e += (size_t)gridDim.x * blockDim.x) {
        unsigned long long g = base + e;
        uint32_t c[4] = {(uint32_t)g, (uint32_t)(g >> 32), 0x5eedu, 0u};
        uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
#pragma unroll
        for (int r = 0; r < 10; ++r) philox_round(c, k);
        const double u1 = ((double)c[0] + 1.0) * 2.3283064365386963e-10;  // (0, 1]
        const double u2 = (double)c[1] * 2.3283064365386963e-10;          // [0, 1)
        out[e] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    }
}

// r = b - r (in place on r), rf = float(r), per-column sums of r^2 and b^2.
__global__ void residual_kernel(const double* __restrict__ b, double* __restrict__ r,
                                float* __restrict__ rf, int N, int s, double* __restrict__ nr2,
                                double* __restrict__ nb2) {
    const int j = blockIdx.y;
    double a2 = 0.0, c2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        size_t e = i + (size_t)j * N;
        double bv = b[e];
        double rv = bv - r[e];
        r[e] = rv;
        if (rf) rf[e] = (float)rv;
        a2 += rv * rv;
        c2 += bv * bv;
    }
    for (int off = 16; off > 0; off >>= 1) {
        a2 += __shfl_down_sync(0xffffffffu, a2, off);
        c2 += __shfl_down_sync(0xffffffffu, c2, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&nr2[j], a2);
        atomicAdd(&nb2[j], c2);
    }
}

// out = a*x + b*y (out may alias x or y)
__global__ void axpby_kernel(double* out, const double* x, double a, const double* y, double b, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        out[e] = a * x[e] + b * y[e];
}

// x += double(d)
__global__ void accumulate_kernel(double* __restrict__ x, const float* __restrict__ d, size_t n,
                                  int first) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x)
        x[e] = first ? (double)d[e] : x[e] + (double)d[e];
}

__global__ void to_float_kernel(const double* __restrict__ a, float* __restrict__ b, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x)
        b[e] = (float)a[e];
}

__global__ void nonfinite_kernel(const double* __restrict__ a, size_t n, int* status) {
    bool bad = false;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x)
        bad |= !isfinite(a[e]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, ST_NONFINITE);
}

static int grid_for(size_t n, int bs = 256, int cap = 148 * 16) {
    return (int)std::min<size_t>(std::max<size_t>(1, (n + bs - 1) / bs), (size_t)cap);
}

// ---------------------------------------------------------------------------------
// Planning helpers
// ---------------------------------------------------------------------------------
std::vector<int> Engine::path_of(int n) const {
    std::vector<int> p;
    for (int c = n; c >= 0 && nodes_[c].parent >= 0; c = nodes_[c].parent) p.push_back(c);
    return p;
}

void Engine::plan_levels() {
    levels_.clear();
    leaves_.clear();
    int maxd = 0;
    for (auto& n : nodes_) maxd = std::max(maxd, n.depth);
    levels_.resize(maxd + 1);
    for (int i = 0; i < (int)nodes_.size(); ++i) {
        if (nodes_[i].is_leaf) leaves_.push_back(i);
        else levels_[nodes_[i].depth].push_back(i);
    }
    while (!levels_.empty() && levels_.back().empty()) levels_.pop_back();
}

void Engine::check_status(const char* what) {
    int st = 0;
    HM_CUDA(cudaMemcpyAsync(&st, dstatus.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HM_CUDA(cudaStreamSynchronize(stream_));
    if (st & ST_SINGULAR) throw Error(HM_ERR_SINGULAR, std::string(what) + ": singular pivot");
    if (st & ST_NONFINITE) throw Error(HM_ERR_NONFINITE, std::string(what) + ": non-finite values");
    if (st & ST_TIMEOUT) throw Error(HM_ERR_TIMEOUT, std::string(what) + ": tensor-core pipeline wait timed out");
    if (st & ST_NO_CONVERGE)
        throw Error(HM_ERR_NO_CONVERGE, std::string(what) + ": Jacobi sweep limit reached");
}

// Column capacity of each basis block from the compression rules (compression.h:72-75).
void Engine::alloc_bases() {
    alloc_D();
    alloc_UV();
}

void Engine::alloc_D() {
    size_t offD = 0;
    for (auto& n : nodes_) {
        if (n.is_leaf) {
            n.offD = offD;
            offD += (size_t)n.len() * n.len();
        }
    }
    dD.alloc(std::max<size_t>(offD, 1));
}

void Engine::alloc_UV() {
    size_t offU = 0, offV = 0;
    for (auto& n : nodes_) {
        if (n.parent < 0) continue;
        n.offU = offU;
        offU += (size_t)n.len() * n.capU;
        n.offV = offV;
        offV += (size_t)n.len() * n.capV;
    }
    dU.alloc(std::max<size_t>(offU, 1));
    dV.alloc(std::max<size_t>(offV, 1));
    dU.zero(stream_);
    dV.zero(stream_);
}

// blocks: (offset, count) of each sketch in the reference's draw order.
void Engine::make_sketches(DBuf<double>& dOmega, const std::vector<std::pair<size_t, size_t>>& blocks) {
    size_t total = 0;
    for (auto& b : blocks) total = std::max(total, b.first + b.second);
    dOmega.alloc(std::max<size_t>(total, 1));
    if (!total) return;
    if (opts_.sketch == HM_SKETCH_DEVICE_NORMAL) {
        normal_fill_kernel<<<grid_for(total), 256, 0, stream_>>>(dOmega.p, total, opts_.seed, 0ull);
        HM_CUDA(cudaGetLastError());
        count_launch();
        return;
    }
    // Matrix::Random (matrix.h:50-57): one std::mt19937 seeded once, a fresh
    // distribution per call, column-major fill, calls in build order.
    std::vector<double> host(total);
    std::mt19937 gen((std::mt19937::result_type)opts_.seed);
    for (auto& b : blocks) {
        double* o = host.data() + b.first;
        if (opts_.sketch == HM_SKETCH_REFERENCE_NORMAL) {
            std::normal_distribution<double> dist(0.0, 1.0);
            for (size_t i = 0; i < b.second; ++i) o[i] = dist(gen);
        } else {
            std::uniform_real_distribution<double> dist(0.0, 1.0);
            for (size_t i = 0; i < b.second; ++i) o[i] = dist(gen);
        }
    }
    HM_CUDA(cudaMemcpyAsync(dOmega.p, host.data(), total * sizeof(double), cudaMemcpyHostToDevice, stream_));
    HM_CUDA(cudaStreamSynchronize(stream_));
}

// ---------------------------------------------------------------------------------
// Build from a dense device matrix (hodlr_routines.h:20-63 + compression.h)
// ---------------------------------------------------------------------------------
namespace {
struct Block {
    int node, which;   // which: 0 = A12 (rows c1, cols c2), 1 = A21 (rows c2, cols c1)
    int m, n, r0, c0, crow, ccol;
    bool rsvd;
    int k;
    size_t omega = 0;  // offset of Omega in the sketch buffer
    int slot = 0;      // rank / sigma slot
};
}  // namespace

void Engine::begin_build(int N, int leaf) {
    HM_CHECK(N > 0 && leaf > 0, HM_ERR_ARG, "build: N and leaf_size must be positive");
    HM_CUDA(cudaGetDevice(&device_));
    N_ = N;
    leaf_ = leaf;
    built_ = factored_ = false;
    f64_.ready = f32_.ready = false;
    f64_.planned = f32_.planned = false;
    f64_.plans.clear();
    f32_.plans.clear();
    dDinv.release();
    mv_plans_.clear();
    solve64_plans_.clear();
    solve32_plans_.clear();
    solveT_plans_.clear();
    exact_plans_.clear();
    grad_plans_.clear();
    io_cols_ = 0;        // staging buffers are sized N x columns: a new N needs new ones
    ex_cols_ = 0;
    grads_ready_ = false;
    gen_ = GEN_DENSE;
    gp_ = GenParams();
    leaves_spd_ = false;
    nodes_ = kind_ == HODLR ? hodlr_tree(N, leaf) : hss_tree(N, leaf);
    sys_N_ = {N};
    sys_off_ = {0};
    plan_levels();
    if (!dstatus.p) dstatus.alloc(1);
    dstatus.zero(stream_);
}

void Engine::build_dense_device(const double* dA, int N, int lda, int leaf) {
    HM_CHECK(N > 0 && leaf > 0 && lda >= N && dA, HM_ERR_ARG, "build_from_dense: bad arguments");
    begin_build(N, leaf);
    {   // reject non-finite input before any compression
        if (lda == N) {
            const size_t cnt = (size_t)N * N;
            nonfinite_kernel<<<grid_for(cnt), 256, 0, stream_>>>(dA, cnt, dstatus.p);
        } else {
            for (int c = 0; c < N; ++c)
                nonfinite_kernel<<<grid_for(N), 256, 0, stream_>>>(dA + (size_t)c * lda, N, dstatus.p);
        }
        HM_CUDA(cudaGetLastError());
        check_status("build_from_dense: input");
    }
    Source src;
    src.dA = dA;
    src.lda = lda;
    if (kind_ == HODLR) build_hodlr(src);
    else build_hss(src);
    built_ = true;
}

void Engine::build_batch_kernel(int gen, const double* pts, int dim, int nsys, const int* Ns, const double* p0s,
                                const double* p1s, int leaf) {
    HM_CHECK(kind_ == HODLR, HM_ERR_UNSUPPORTED, "batches are HODLR systems");
    HM_CHECK(gen == GEN_GAUSSIAN || gen == GEN_COULOMB, HM_ERR_ARG, "batch kernel: Gaussian or Coulomb");
    HM_CHECK(nsys >= 1 && Ns && p0s && p1s && pts && dim >= 1 && dim <= 3 && leaf > 0, HM_ERR_ARG,
             "batch build: bad arguments");
    std::vector<int> off(nsys + 1, 0);
    for (int k = 0; k < nsys; ++k) {
        HM_CHECK(Ns[k] > 0, HM_ERR_ARG, "batch build: system sizes must be positive");
        HM_CHECK((long long)off[k] + Ns[k] < (1LL << 31), HM_ERR_UNSUPPORTED, "batch too large");
        off[k + 1] = off[k] + Ns[k];
    }
    const int Ntot = off[nsys];
    for (size_t i = 0; i < (size_t)Ntot * dim; ++i)
        HM_CHECK(std::isfinite(pts[i]), HM_ERR_NONFINITE, "batch build: non-finite point");
    begin_build(Ntot, leaf);
    // forest: each system's pre-order tree on its own rows
    nodes_.clear();
    for (int k = 0; k < nsys; ++k) {
        std::vector<Node> t = hodlr_tree(Ns[k], leaf);
        const int base = (int)nodes_.size();
        for (auto& n : t) {
            n.start += off[k];
            n.end += off[k];
            n.sys = k;
            if (n.parent >= 0) n.parent += base;
            if (n.left >= 0) n.left += base;
            if (n.right >= 0) n.right += base;
            nodes_.push_back(n);
        }
    }
    sys_N_.assign(Ns, Ns + nsys);
    sys_off_.assign(off.begin(), off.end() - 1);
    plan_levels();
    std::vector<int> rs(Ntot);
    for (int k = 0; k < nsys; ++k)
        for (int i = off[k]; i < off[k + 1]; ++i) rs[i] = k;
    dPts.alloc((size_t)Ntot * dim);
    dRowSys.alloc(Ntot);
    dSysP0.alloc(nsys);
    dSysP1.alloc(nsys);
    HM_CUDA(cudaMemcpyAsync(dPts.p, pts, (size_t)Ntot * dim * sizeof(double), cudaMemcpyHostToDevice, stream_));
    HM_CUDA(cudaMemcpyAsync(dRowSys.p, rs.data(), rs.size() * sizeof(int), cudaMemcpyHostToDevice, stream_));
    HM_CUDA(cudaMemcpyAsync(dSysP0.p, p0s, nsys * sizeof(double), cudaMemcpyHostToDevice, stream_));
    HM_CUDA(cudaMemcpyAsync(dSysP1.p, p1s, nsys * sizeof(double), cudaMemcpyHostToDevice, stream_));
    HM_CUDA(cudaStreamSynchronize(stream_));
    Source src;
    src.gen = gen;
    src.gp.pts = dPts.p;
    src.gp.N = Ntot;
    src.gp.dim = dim;
    src.gp.row_sys = dRowSys.p;
    src.gp.p0v = dSysP0.p;
    src.gp.p1v = dSysP1.p;
    build_hodlr(src);
    leaves_spd_ = true;
    for (int k = 0; k < nsys; ++k) leaves_spd_ = leaves_spd_ && kernel_spd(gen, p0s[k], p1s[k]);
    built_ = true;  // no kernel-parameter gradient for batches (gen_ stays dense)
}

// packed (system k: N_k x s_k at offset sum_{j<k} N_j s_j) <-> staging (rows global, ld N)
static std::vector<CopyDesc> packed_copies(const std::vector<int>& Ns, const std::vector<int>& off,
                                           const std::vector<int>& sc, double* packed, double* staging, int N,
                                           bool to_staging, size_t* total) {
    std::vector<CopyDesc> out;
    size_t p = 0;
    for (size_t k = 0; k < Ns.size(); ++k) {
        if (sc[k] > 0) {
            CopyDesc c{};
            if (to_staging) {
                c.src = packed + p; c.lds = Ns[k]; c.dst = staging + off[k]; c.ldd = N;
            } else {
                c.src = staging + off[k]; c.lds = N; c.dst = packed + p; c.ldd = Ns[k];
            }
            c.rows = Ns[k];
            c.cols = sc[k];
            out.push_back(c);
        }
        p += (size_t)Ns[k] * sc[k];
    }
    *total = p;
    return out;
}

void Engine::batch_solve(const double* b, const int* nrhs, double* x) {
    HM_CHECK(built_, HM_ERR_STATE, "batch solve before build");
    HM_CHECK(b && nrhs && x, HM_ERR_ARG, "batch solve: bad arguments");
    HM_CHECK(opts_.precision == HM_FP64, HM_ERR_UNSUPPORTED, "batched solves run in FP64");
    std::vector<int> sc(nrhs, nrhs + sys_N_.size());
    int smax = 0;
    for (int s : sc) {
        HM_CHECK(s >= 0, HM_ERR_ARG, "batch solve: negative column count");
        smax = std::max(smax, s);
    }
    if (smax == 0) return;
    if (!factored_) factor();
    ensure_io(smax);
    size_t total = 0;
    auto in = packed_copies(sys_N_, sys_off_, sc, nullptr, ioX.p, N_, true, &total);
    if (ioPacked.n < total) ioPacked.alloc(total);
    const bool refine = opts_.refine_steps > 0;
    if (refine && ioAcc.n < (size_t)N_ * smax) ioAcc.alloc((size_t)N_ * smax);
    in = packed_copies(sys_N_, sys_off_, sc, ioPacked.p, refine ? ioR.p : ioX.p, N_, true, &total);
    auto outc = packed_copies(sys_N_, sys_off_, sc, ioPacked.p, refine ? ioAcc.p : ioY.p, N_, false, &total);
    HM_CUDA(cudaMemcpyAsync(ioPacked.p, b, total * sizeof(double), cudaMemcpyDefault, stream_));
    CopyStep cin, cout;
    cin.t.h = in;
    cout.t.h = outc;
    cin.t.upload(stream_);
    cout.t.upload(stream_);
    cin.run(stream_, dstatus.p);
    count_launch();
    if (refine) refined_fp64(sc, smax);
    else solve_plan<double>(f64_, sc).run(stream_, dstatus.p);
    cout.run(stream_, dstatus.p);
    count_launch();
    HM_CUDA(cudaMemcpyAsync(x, ioPacked.p, total * sizeof(double), cudaMemcpyDefault, stream_));
    HM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::batch_multiply(const double* xin, const int* nrhs, double* y) {
    HM_CHECK(built_, HM_ERR_STATE, "batch multiply before build");
    HM_CHECK(xin && nrhs && y, HM_ERR_ARG, "batch multiply: bad arguments");
    std::vector<int> sc(nrhs, nrhs + sys_N_.size());
    int smax = 0;
    for (int s : sc) smax = std::max(smax, s);
    if (smax == 0) return;
    ensure_io(smax);
    size_t total = 0;
    packed_copies(sys_N_, sys_off_, sc, nullptr, ioX.p, N_, true, &total);
    if (ioPacked.n < total) ioPacked.alloc(total);
    auto in = packed_copies(sys_N_, sys_off_, sc, ioPacked.p, ioX.p, N_, true, &total);
    auto outc = packed_copies(sys_N_, sys_off_, sc, ioPacked.p, ioY.p, N_, false, &total);
    HM_CUDA(cudaMemcpyAsync(ioPacked.p, xin, total * sizeof(double), cudaMemcpyDefault, stream_));
    CopyStep cin, cout;
    cin.t.h = in;
    cout.t.h = outc;
    cin.t.upload(stream_);
    cout.t.upload(stream_);
    cin.run(stream_, dstatus.p);
    matvec_plan(sc).run(stream_, dstatus.p);
    cout.run(stream_, dstatus.p);
    count_launch(2);
    HM_CUDA(cudaMemcpyAsync(y, ioPacked.p, total * sizeof(double), cudaMemcpyDefault, stream_));
    HM_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::build_kernel(int gen, const double* pts, size_t npts, int dim, int N, double p0, double p1,
                          int leaf) {
    HM_CHECK(gen == GEN_CAUCHY || gen == GEN_GAUSSIAN || gen == GEN_COULOMB, HM_ERR_ARG, "unknown kernel");
    HM_CHECK(pts && dim >= 1 && dim <= 3, HM_ERR_ARG, "build_from_kernel: bad points");
    for (size_t i = 0; i < npts; ++i)
        HM_CHECK(std::isfinite(pts[i]), HM_ERR_NONFINITE, "build_from_kernel: non-finite point");
    begin_build(N, leaf);
    dPts.alloc(npts);
    HM_CUDA(cudaMemcpyAsync(dPts.p, pts, npts * sizeof(double), cudaMemcpyHostToDevice, stream_));
    Source src;
    src.gen = gen;
    src.gp.pts = dPts.p;
    src.gp.N = N;
    src.gp.dim = dim;
    src.gp.p0 = p0;
    src.gp.p1 = p1;
    if (kind_ == HODLR) build_hodlr(src);
    else build_hss(src);
    gen_ = src.gen;
    gp_ = src.gp;
    leaves_spd_ = kernel_spd(gen, p0, p1);
    built_ = true;
}

void Engine::add_block_fill(Plan& plan, const Source& src,
                            const std::vector<std::tuple<int, int, int, int, int, double*, int>>& blocks) {
    // (r0, c0, rows, cols, trans, dst, ldd): dst = trans ? A[r0.., c0..]^T : A[r0.., c0..]
    if (blocks.empty()) return;
    if (src.dense()) {
        auto cp = std::make_unique<CopyStep>();
        for (auto& b : blocks) {
            auto [r0, c0, rows, cols, trans, dst, ldd] = b;
            cp->t.h.push_back({src.blk(r0, c0), src.lda, dst, ldd, rows, cols, trans, 0, 0});
        }
        cp->t.upload(stream_);
        plan.add(std::move(cp));
    } else {
        auto gf = std::make_unique<GenFillStep>();
        gf->gen = src.gen;
        gf->gp = src.gp;
        for (auto& b : blocks) {
            auto [r0, c0, rows, cols, trans, dst, ldd] = b;
            gf->t.h.push_back({r0, c0, rows, cols, trans, dst, ldd});
        }
        gf->t.upload(stream_);
        plan.add(std::move(gf));
    }
}

void Engine::build_hodlr(const Source& src) {
    const int kguess = opts_.rsvd_rank + opts_.oversample;
    HM_CHECK(opts_.rsvd_rank >= 0 && opts_.oversample >= 0, HM_ERR_ARG, "bad rsvd_rank/oversample");
    // blocks in the reference's serial post-order (hodlr_routines.h:43-53)
    std::vector<Block> blocks;
    std::function<void(int)> post = [&](int id) {
        const Node& n = nodes_[id];
        if (n.is_leaf) return;
        post(n.left);
        post(n.right);
        const Node& L = nodes_[n.left];
        const Node& R = nodes_[n.right];
        for (int w = 0; w < 2; ++w) {
            Block b{};
            b.node = id;
            b.which = w;
            if (w == 0) { b.m = L.len(); b.n = R.len(); b.r0 = L.start; b.c0 = R.start; b.crow = n.left; b.ccol = n.right; }
            else { b.m = R.len(); b.n = L.len(); b.r0 = R.start; b.c0 = L.start; b.crow = n.right; b.ccol = n.left; }
            b.rsvd = b.m >= opts_.rsvd_min_dim && b.n >= opts_.rsvd_min_dim;  // compression.h:72
            b.k = b.rsvd ? std::min(kguess, std::min(b.m, b.n)) : std::min(b.m, b.n);
            b.slot = (int)blocks.size();
            blocks.push_back(b);
        }
    };
    for (size_t r = 0; r < nodes_.size(); ++r)  // every system's root, system after system
        if (nodes_[r].parent < 0) post((int)r);
    HM_CHECK((int)blocks.size() <= 1 << 26, HM_ERR_UNSUPPORTED, "tree too large");
    // capacities
    for (auto& b : blocks) {
        nodes_[b.crow].capU = b.k;
        nodes_[b.ccol].capV = b.k;
    }
    alloc_bases();
    // leaf blocks D (hodlr_routines.h:32-34)
    {
        Plan lp;
        std::vector<std::tuple<int, int, int, int, int, double*, int>> fill;
        for (int l : leaves_) {
            const Node& n = nodes_[l];
            fill.emplace_back(n.start, n.start, n.len(), n.len(), 0, dD.p + n.offD, n.len());
            if (fill.size() == 60000) { add_block_fill(lp, src, fill); fill.clear(); }
        }
        add_block_fill(lp, src, fill);
        lp.run(stream_, dstatus.p);
        HM_CUDA(cudaStreamSynchronize(stream_));
    }
    // sketches
    size_t omega_total = 0;
    for (auto& b : blocks)
        if (b.rsvd) { b.omega = omega_total; omega_total += (size_t)b.n * b.k; }
    DBuf<double> dOmega;
    {
        std::vector<std::pair<size_t, size_t>> om;
        for (auto& b : blocks)
            if (b.rsvd) om.emplace_back(b.omega, (size_t)b.n * b.k);
        make_sketches(dOmega, om);
    }
    // Mixed-precision matrix-free builds: the sketch, power-iteration and projection
    // products run in FP32 on the tensor cores with A's entries generated in the kernel;
    // Omega in FP32, each block 16-byte aligned for the TMA
    const bool tc_sketch = opts_.precision == HM_MIXED && !src.dense();
    DBuf<float> dOmega32;
    std::vector<size_t> om32(blocks.size(), 0);
    if (tc_sketch && omega_total) {
        size_t tot32 = 0;
        for (auto& b : blocks)
            if (b.rsvd) { om32[b.slot] = tot32; tot32 = align_up(tot32 + (size_t)b.n * b.k, 4); }
        dOmega32.alloc(std::max<size_t>(tot32, 1));
        Plan cv;
        auto st = std::make_unique<CopyStep>();
        for (auto& b : blocks)
            if (b.rsvd) st->t.h.push_back({dOmega.p + b.omega, b.n, dOmega32.p + om32[b.slot], b.n, b.n, b.k, 0, 0, 1});
        st->t.upload(stream_);
        cv.add(std::move(st));
        cv.run(stream_, dstatus.p);
        HM_CUDA(cudaStreamSynchronize(stream_));
    }
    // per-block sigma and rank
    std::vector<size_t> sig_off(blocks.size());
    size_t sig_total = 0;
    for (auto& b : blocks) { sig_off[b.slot] = sig_total; sig_total += b.k; }
    DBuf<double> dSig(std::max<size_t>(sig_total, 1));
    DBuf<int> dRank(std::max<size_t>(blocks.size(), 1));
    dSig.zero(stream_);
    dRank.zero(stream_);

    // one batched pipeline per tree level
    std::map<int, std::vector<Block*>> by_depth;
    for (auto& b : blocks) by_depth[nodes_[b.node].depth].push_back(&b);
    for (auto& kv : by_depth) {
        Plan plan;
        auto& lvl = kv.second;
        std::vector<Block*> rs, fs;
        for (auto* b : lvl) (b->rsvd ? rs : fs).push_back(b);
        // ---- full SVDs (compression.h:18-64) on the tall orientation ----
        if (!fs.empty()) {
            std::vector<std::tuple<int, int, int, int, int, double*, int>> fill;
            std::vector<SvdProblem> sv;
            for (auto* b : fs) {
                const bool tall = b->m >= b->n;
                const int rows = tall ? b->m : b->n, p = tall ? b->n : b->m;
                double* X = plan.scratch((size_t)rows * p);
                fill.emplace_back(b->r0, b->c0, rows, p, tall ? 0 : 1, X, rows);
                Node& cr = nodes_[b->crow];
                Node& cc = nodes_[b->ccol];
                double* Uo = dU.p + cr.offU;
                double* Vo = dV.p + cc.offV;
                SvdProblem q{};
                q.X = X; q.ldx = rows; q.rows = rows; q.k = p;
                q.sigma = dSig.p + sig_off[b->slot];
                q.rank = dRank.p + b->slot;
                q.sort = true;
                if (tall) { q.L = Uo; q.ldl = cr.len(); q.R = Vo; q.ldr = cc.len(); }
                else { q.L = Vo; q.ldl = cc.len(); q.R = Uo; q.ldr = cr.len(); }
                sv.push_back(q);
            }
            add_block_fill(plan, src, fill);
            plan_gram_svd(plan, sv, opts_.tol, opts_.max_rank, stream_);
        }
        // ---- randomized SVDs (compression.h:67-99) ----
        if (!rs.empty() && tc_sketch) {
            // FP32 products of generated A on the tensor cores (FP32 accumulation of TF32
            // hi/lo splits), basis by shifted CholeskyQR3 in FP64, small SVD in FP64
            struct W { double *Y, *Q, *X, *Ub; float *Y32, *Q32, *X32; };
            std::vector<W> ws(rs.size());
            auto mk32 = [&](const char* tag) {
                auto g = std::make_unique<GemmStep<float>>(CFG_64x64, src.gen);
                g->gp = src.gp;
                g->batch.set_tag(tag);
                g->label = std::string("gemm_gen_f32:") + tag;
                g->label_tc = std::string("tc_tf32x4_gen:") + tag;
                return g;
            };
            for (size_t i = 0; i < rs.size(); ++i) {
                Block* b = rs[i];
                ws[i].Y = plan.scratch((size_t)b->m * b->k);
                ws[i].Q = plan.scratch((size_t)b->m * b->k);
                ws[i].X = plan.scratch((size_t)b->n * b->k);
                ws[i].Ub = plan.scratch((size_t)b->k * b->k);
                ws[i].Y32 = plan.scratch_f((size_t)b->m * b->k);
                ws[i].Q32 = plan.scratch_f(std::max((size_t)b->m, (size_t)b->n) * b->k);
                ws[i].X32 = plan.scratch_f((size_t)b->n * b->k);
            }
            auto to64 = [&](const std::vector<std::tuple<float*, double*, int, int>>& l) {
                auto st = std::make_unique<CopyStep>();
                for (auto& t : l) st->t.h.push_back({std::get<0>(t), std::get<2>(t), std::get<1>(t), std::get<2>(t),
                                                     std::get<2>(t), std::get<3>(t), 0, 1, 0});
                st->t.upload(stream_);
                plan.add(std::move(st));
            };
            auto to32 = [&](const std::vector<std::tuple<double*, float*, int, int>>& l) {
                auto st = std::make_unique<CopyStep>();
                for (auto& t : l) st->t.h.push_back({std::get<0>(t), std::get<2>(t), std::get<1>(t), std::get<2>(t),
                                                     std::get<2>(t), std::get<3>(t), 0, 0, 1});
                st->t.upload(stream_);
                plan.add(std::move(st));
            };
            // Y = A_blk Omega  (compression.h:79), then Q = orthonormal basis of range(Y)
            auto sketchY = [&](bool from_omega) {
                auto g = mk32("build.sketch");
                std::vector<std::tuple<float*, double*, int, int>> cv;
                for (size_t i = 0; i < rs.size(); ++i) {
                    Block* b = rs[i];
                    const float* Bm = from_omega ? dOmega32.p + om32[b->slot] : ws[i].Q32;
                    g->batch.add(b->m, b->k, b->n, 1.0f, nullptr, 0, OP_N, Bm, b->n, OP_N, 0.0f, ws[i].Y32, b->m,
                                 nullptr, 0, b->r0, b->c0);
                    cv.emplace_back(ws[i].Y32, ws[i].Y, b->m, b->k);
                }
                g->batch.finalize(stream_);
                plan.add(std::move(g));
                to64(cv);
                std::vector<QrProblem> qr;
                for (size_t i = 0; i < rs.size(); ++i)
                    qr.push_back({ws[i].Y, rs[i]->m, rs[i]->m, rs[i]->k, ws[i].Q, rs[i]->m});
                plan_cholqr3(plan, qr, stream_);
            };
            // X = A_blk^T Q (the projection, compression.h:87, and the power iteration's Z)
            auto project = [&]() {
                std::vector<std::tuple<double*, float*, int, int>> c32;
                for (size_t i = 0; i < rs.size(); ++i) c32.emplace_back(ws[i].Q, ws[i].Q32, rs[i]->m, rs[i]->k);
                to32(c32);
                auto g = mk32("build.project");
                std::vector<std::tuple<float*, double*, int, int>> cv;
                for (size_t i = 0; i < rs.size(); ++i) {
                    Block* b = rs[i];
                    g->batch.add(b->n, b->k, b->m, 1.0f, nullptr, 0, OP_T, ws[i].Q32, b->m, OP_N, 0.0f, ws[i].X32, b->n,
                                 nullptr, 0, b->r0, b->c0);
                    cv.emplace_back(ws[i].X32, ws[i].X, b->n, b->k);
                }
                g->batch.finalize(stream_);
                plan.add(std::move(g));
                to64(cv);
            };
            sketchY(true);
            for (int it = 0; it < opts_.power_iters; ++it) {  // extension
                project();
                std::vector<QrProblem> qr;
                for (size_t i = 0; i < rs.size(); ++i) {
                    double* Z = plan.scratch((size_t)rs[i]->n * rs[i]->k);
                    qr.push_back({ws[i].X, rs[i]->n, rs[i]->n, rs[i]->k, Z, rs[i]->n});
                }
                plan_cholqr3(plan, qr, stream_);
                std::vector<std::tuple<double*, float*, int, int>> c32;
                for (size_t i = 0; i < rs.size(); ++i) c32.emplace_back(qr[i].Q, ws[i].Q32, rs[i]->n, rs[i]->k);
                to32(c32);
                sketchY(false);
            }
            project();
            // SVD of Q^T A (compression.h:90): X = V_b S U_b^T, then U = Q U_b (compression.h:94)
            std::vector<SvdProblem> sv;
            for (size_t i = 0; i < rs.size(); ++i) {
                Block* b = rs[i];
                Node& cc = nodes_[b->ccol];
                SvdProblem q{};
                q.X = ws[i].X; q.ldx = b->n; q.rows = b->n; q.k = b->k;
                q.L = dV.p + cc.offV; q.ldl = cc.len();
                q.R = ws[i].Ub; q.ldr = b->k;
                q.sigma = dSig.p + sig_off[b->slot];
                q.rank = dRank.p + b->slot;
                q.sort = true;
                sv.push_back(q);
            }
            plan_gram_svd(plan, sv, opts_.tol, opts_.max_rank, stream_);
            auto gU = std::make_unique<GemmStep<double>>();
            for (size_t i = 0; i < rs.size(); ++i) {
                Block* b = rs[i];
                Node& cr = nodes_[b->crow];
                gU->batch.add(b->m, b->k, b->k, 1.0, ws[i].Q, b->m, OP_N, ws[i].Ub, b->k, OP_N, 0.0,
                              dU.p + cr.offU, cr.len());
            }
            gU->batch.finalize(stream_);
            plan.add(std::move(gU));
        } else if (!rs.empty()) {
            struct W { double *Y, *Q, *X, *Ub; };
            std::vector<W> ws(rs.size());
            auto mkA = [&]() {
                auto g = std::make_unique<GemmStep<double>>(CFG_64x64, src.gen);
                g->gp = src.gp;
                return g;
            };
            auto gY = mkA();
            for (size_t i = 0; i < rs.size(); ++i) {
                Block* b = rs[i];
                ws[i].Y = plan.scratch((size_t)b->m * b->k);
                ws[i].Q = plan.scratch((size_t)b->m * b->k);
                ws[i].X = plan.scratch((size_t)b->n * b->k);
                ws[i].Ub = plan.scratch((size_t)b->k * b->k);
                // Y = A_blk Omega  (compression.h:79)
                gY->batch.add(b->m, b->k, b->n, 1.0, src.blk(b->r0, b->c0), src.lda, OP_N,
                              dOmega.p + b->omega, b->n, OP_N, 0.0, ws[i].Y, b->m, nullptr, 0, b->r0, b->c0);
            }
            gY->batch.finalize(stream_);
            plan.add(std::move(gY));
            auto orthY = [&]() {
                std::vector<SvdProblem> sv;
                for (size_t i = 0; i < rs.size(); ++i) {
                    Block* b = rs[i];
                    SvdProblem q{};
                    q.X = ws[i].Y; q.ldx = b->m; q.rows = b->m; q.k = b->k;
                    q.L = ws[i].Q; q.ldl = b->m;
                    q.sort = false;
                    sv.push_back(q);
                }
                plan_gram_svd(plan, sv, opts_.tol, 0, stream_);
            };
            orthY();  // Q = orthonormal basis of range(Y)  (compression.h:83-84)
            for (int it = 0; it < opts_.power_iters; ++it) {  // extension
                auto gZ = mkA();
                for (size_t i = 0; i < rs.size(); ++i) {
                    Block* b = rs[i];
                    gZ->batch.add(b->n, b->k, b->m, 1.0, src.blk(b->r0, b->c0), src.lda, OP_T,
                                  ws[i].Q, b->m, OP_N, 0.0, ws[i].X, b->n, nullptr, 0, b->r0, b->c0);
                }
                gZ->batch.finalize(stream_);
                plan.add(std::move(gZ));
                std::vector<SvdProblem> sv;
                for (size_t i = 0; i < rs.size(); ++i) {
                    Block* b = rs[i];
                    SvdProblem q{};
                    q.X = ws[i].X; q.ldx = b->n; q.rows = b->n; q.k = b->k;
                    q.L = ws[i].X; q.ldl = b->n;
                    sv.push_back(q);
                }
                plan_gram_svd(plan, sv, opts_.tol, 0, stream_);
                auto gY2 = mkA();
                for (size_t i = 0; i < rs.size(); ++i) {
                    Block* b = rs[i];
                    gY2->batch.add(b->m, b->k, b->n, 1.0, src.blk(b->r0, b->c0), src.lda, OP_N,
                                   ws[i].X, b->n, OP_N, 0.0, ws[i].Y, b->m, nullptr, 0, b->r0, b->c0);
                }
                gY2->batch.finalize(stream_);
                plan.add(std::move(gY2));
                orthY();
            }
            // X = A_blk^T Q = (Q^T A_blk)^T  (compression.h:87)
            auto gX = mkA();
            for (size_t i = 0; i < rs.size(); ++i) {
                Block* b = rs[i];
                gX->batch.add(b->n, b->k, b->m, 1.0, src.blk(b->r0, b->c0), src.lda, OP_T,
                              ws[i].Q, b->m, OP_N, 0.0, ws[i].X, b->n, nullptr, 0, b->r0, b->c0);
            }
            gX->batch.finalize(stream_);
            plan.add(std::move(gX));
            // SVD of Q^T A (compression.h:90): X = V_b S U_b^T
            std::vector<SvdProblem> sv;
            for (size_t i = 0; i < rs.size(); ++i) {
                Block* b = rs[i];
                Node& cc = nodes_[b->ccol];
                SvdProblem q{};
                q.X = ws[i].X; q.ldx = b->n; q.rows = b->n; q.k = b->k;
                q.L = dV.p + cc.offV; q.ldl = cc.len();
                q.R = ws[i].Ub; q.ldr = b->k;
                q.sigma = dSig.p + sig_off[b->slot];
                q.rank = dRank.p + b->slot;
                q.sort = true;
                sv.push_back(q);
            }
            plan_gram_svd(plan, sv, opts_.tol, opts_.max_rank, stream_);
            // U = Q U_b  (compression.h:94)
            auto gU = std::make_unique<GemmStep<double>>();
            for (size_t i = 0; i < rs.size(); ++i) {
                Block* b = rs[i];
                Node& cr = nodes_[b->crow];
                gU->batch.add(b->m, b->k, b->k, 1.0, ws[i].Q, b->m, OP_N, ws[i].Ub, b->k, OP_N, 0.0,
                              dU.p + cr.offU, cr.len());
            }
            gU->batch.finalize(stream_);
            plan.add(std::move(gU));
        }
        plan.run(stream_, dstatus.p);
        HM_CUDA(cudaStreamSynchronize(stream_));
    }
    check_status("build");
    // ranks and singular values to the host; B = diag(S[:rank]) (compression.h:57-63)
    std::vector<int> ranks(blocks.size());
    std::vector<double> sig(sig_total);
    HM_CUDA(cudaMemcpyAsync(ranks.data(), dRank.p, ranks.size() * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    if (sig_total)
        HM_CUDA(cudaMemcpyAsync(sig.data(), dSig.p, sig_total * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    HM_CUDA(cudaStreamSynchronize(stream_));
    // kept rank of every block: the truncation rule's, or a fixed profile (set_rank_profile)
    if (!fix12_.empty())
        HM_CHECK(fix12_.size() == nodes_.size() && fix21_.size() == nodes_.size() && kind_ == HODLR &&
                     sys_N_.size() == 1,
                 HM_ERR_ARG, "rank profile: its node count does not match this HODLR tree");
    for (auto& b : blocks) {
        int r = std::min(ranks[b.slot], b.k);
        if (!fix12_.empty()) r = std::max(1, std::min(b.k, (b.which == 0 ? fix12_ : fix21_)[b.node]));
        ranks[b.slot] = r;
    }
    std::vector<int> r12(nodes_.size(), 0), r21(nodes_.size(), 0);
    std::vector<double> s12, s21;
    size_t tot = 0;
    for (auto& b : blocks) {
        int r = std::min(ranks[b.slot], b.k);
        Node& n = nodes_[b.node];
        (b.which == 0 ? r12 : r21)[b.node] = r;
        tot += (size_t)r * r;
        (void)n;
    }
    std::vector<double> hB(std::max<size_t>(tot, 1), 0.0);
    size_t off = 0;
    for (auto& b : blocks) {
        int r = std::min(ranks[b.slot], b.k);
        Node& n = nodes_[b.node];
        size_t o = off;
        for (int i = 0; i < r; ++i) hB[o + i + (size_t)i * r] = sig[sig_off[b.slot] + i];
        if (b.which == 0) {
            n.offB12 = o;
            nodes_[b.crow].rankU = r;   // left.U
            nodes_[b.ccol].rankV = r;   // right.V
        } else {
            n.offB21 = o;
            nodes_[b.crow].rankU = r;   // right.U
            nodes_[b.ccol].rankV = r;   // left.V
        }
        off += (size_t)r * r;
    }
    dB.alloc(hB.size());
    HM_CUDA(cudaMemcpyAsync(dB.p, hB.data(), hB.size() * sizeof(double), cudaMemcpyHostToDevice, stream_));
    HM_CUDA(cudaStreamSynchronize(stream_));
}

// HSS build (hss_routines.h:50-113).  Leaves, in reverse id order, compress their row
// strip A[leaf, :] and their transposed column strip A[:, leaf]^T, each with the diagonal
// block zeroed, keeping only the left singular vectors (the leaf's U and V).  Transfers
// are identities (hss_routines.h:86-90), so a node's basis is the block diagonal of its
// leaves' bases and B12 = UL^T A12 VR is the set of leaf-pair blocks U_l^T A_lm V_m.
// Those come from the panels Pt_l = A[l, :]^T U_l (N x rank_U(l)): block (l, m) of B is
// Pt_l[m rows]^T V_m.  reduce_hss_coupling then derives the operator that the factor,
// solve and multiply run on.
void Engine::build_hss(const Source& src) {
    const int N = N_;
    const int kguess = opts_.rsvd_rank + opts_.oversample;
    struct Strip {
        int leaf, which;  // which 0: row strip (U), 1: column strip (V)
        bool rsvd;
        int m, k;
        size_t omega = 0, out = 0;
    };
    std::vector<Strip> strips;
    for (int i = (int)nodes_.size() - 1; i >= 0; --i) {  // reverse id order (hss_routines.h:57)
        if (!nodes_[i].is_leaf) continue;
        for (int w = 0; w < 2; ++w) {
            Strip s;
            s.leaf = i;
            s.which = w;
            s.m = nodes_[i].len();
            s.rsvd = s.m >= opts_.rsvd_min_dim && N >= opts_.rsvd_min_dim;  // compression.h:72
            s.k = s.rsvd ? std::min(kguess, std::min(s.m, N)) : std::min(s.m, N);
            strips.push_back(s);
        }
    }
    size_t omega_total = 0, out_total = 0;
    for (auto& s : strips) {
        if (s.rsvd) { s.omega = omega_total; omega_total += (size_t)N * s.k; }
        s.out = out_total;
        out_total += (size_t)s.m * s.k;
    }
    DBuf<double> dOmega;
    {
        std::vector<std::pair<size_t, size_t>> om;
        for (auto& s : strips)
            if (s.rsvd) om.emplace_back(s.omega, (size_t)N * s.k);
        make_sketches(dOmega, om);
    }
    alloc_D();
    {
        Plan lp;
        std::vector<std::tuple<int, int, int, int, int, double*, int>> fill;
        for (int l : leaves_) {
            const Node& n = nodes_[l];
            fill.emplace_back(n.start, n.start, n.len(), n.len(), 0, dD.p + n.offD, n.len());
        }
        add_block_fill(lp, src, fill);
        lp.run(stream_, dstatus.p);
    }
    dLeafB.alloc(std::max<size_t>(out_total, 1));
    DBuf<int> dRank(std::max<size_t>(strips.size(), 1));
    // chunks of strips bounded by a workspace budget; one workspace serves every chunk
    const size_t budget = size_t(16) << 30;
    std::vector<std::pair<size_t, size_t>> chunks;
    size_t ws_bytes = 0;
    for (size_t i0 = 0; i0 < strips.size();) {
        size_t i1 = i0, bytes = 0;
        while (i1 < strips.size()) {
            const Strip& s = strips[i1];
            const size_t b = 8 * ((size_t)s.m * N + 5 * (size_t)N * s.k + 6 * (size_t)s.m * s.k + 8 * (size_t)s.k * s.k) +
                             (size_t(1) << 20);   // alignment and small tables
            if (i1 > i0 && bytes + b > budget) break;
            bytes += b;
            ++i1;
        }
        chunks.emplace_back(i0, i1);
        ws_bytes = std::max(ws_bytes, bytes);
        i0 = i1;
    }
    DBuf<unsigned char> ws(std::max<size_t>(ws_bytes, 1));
    for (const auto& ch : chunks) {
        const size_t i0 = ch.first, i1 = ch.second;
        Plan plan;
        plan.use_arena(ws.p, ws.n);
        std::vector<std::tuple<int, int, int, int, int, double*, int>> fill;
        auto zero = std::make_unique<IdentStep>();
        std::vector<SvdProblem> full;
        struct R { const Strip* s; double *S, *Y, *Q, *X, *Ub; };
        std::vector<R> rs;
        for (size_t i = i0; i < i1; ++i) {
            const Strip& s = strips[i];
            const Node& n = nodes_[s.leaf];
            const int slot = (int)i;
            if (!s.rsvd) {
                // tall X = strip^T (N x m); strip = R S L^T, U_strip = R
                double* X = plan.scratch((size_t)N * s.m);
                if (s.which == 0) fill.emplace_back(n.start, 0, N, s.m, 1, X, N);
                else fill.emplace_back(0, n.start, N, s.m, 0, X, N);
                zero->t.h.push_back({X + n.start, N, s.m, s.m, 0.0});
                SvdProblem q{};
                q.X = X; q.ldx = N; q.rows = N; q.k = s.m;
                q.L = nullptr;
                q.R = dLeafB.p + s.out; q.ldr = s.m;
                q.rank = dRank.p + slot;
                q.sort = true;
                full.push_back(q);
            } else {
                R r{&s, nullptr, nullptr, nullptr, nullptr, nullptr};
                r.S = plan.scratch((size_t)s.m * N);  // the strip, m x N
                if (s.which == 0) fill.emplace_back(n.start, 0, s.m, N, 0, r.S, s.m);
                else fill.emplace_back(0, n.start, s.m, N, 1, r.S, s.m);
                zero->t.h.push_back({r.S + (size_t)n.start * s.m, s.m, s.m, s.m, 0.0});
                r.Y = plan.scratch((size_t)s.m * s.k);
                r.Q = plan.scratch((size_t)s.m * s.k);
                r.X = plan.scratch((size_t)N * s.k);
                r.Ub = plan.scratch((size_t)s.k * s.k);
                rs.push_back(r);
            }
        }
        add_block_fill(plan, src, fill);
        zero->t.upload(stream_);
        plan.add(std::move(zero));
        plan_gram_svd(plan, full, opts_.tol, opts_.max_rank, stream_);
        if (!rs.empty()) {
            auto gY = std::make_unique<GemmStep<double>>();
            for (auto& r : rs)  // Y = S Omega  (compression.h:79)
                gY->batch.add(r.s->m, r.s->k, N, 1.0, r.S, r.s->m, OP_N, dOmega.p + r.s->omega, N, OP_N, 0.0,
                              r.Y, r.s->m);
            gY->batch.finalize(stream_);
            plan.add(std::move(gY));
            std::vector<SvdProblem> sq;
            for (auto& r : rs) {  // Q = orthonormal basis of range(Y)
                SvdProblem q{};
                q.X = r.Y; q.ldx = r.s->m; q.rows = r.s->m; q.k = r.s->k;
                q.L = r.Q; q.ldl = r.s->m;
                sq.push_back(q);
            }
            plan_gram_svd(plan, sq, opts_.tol, 0, stream_);
            auto gX = std::make_unique<GemmStep<double>>();
            for (auto& r : rs)  // X = S^T Q
                gX->batch.add(N, r.s->k, r.s->m, 1.0, r.S, r.s->m, OP_T, r.Q, r.s->m, OP_N, 0.0, r.X, N);
            gX->batch.finalize(stream_);
            plan.add(std::move(gX));
            std::vector<SvdProblem> sv;
            for (auto& r : rs) {  // SVD of Q^T S: X = V_b diag(S) U_b^T
                SvdProblem q{};
                q.X = r.X; q.ldx = N; q.rows = N; q.k = r.s->k;
                q.L = nullptr;
                q.R = r.Ub; q.ldr = r.s->k;
                q.rank = dRank.p + (r.s - strips.data());
                q.sort = true;
                sv.push_back(q);
            }
            plan_gram_svd(plan, sv, opts_.tol, opts_.max_rank, stream_);
            auto gU = std::make_unique<GemmStep<double>>();
            for (auto& r : rs)  // U = Q U_b  (compression.h:94)
                gU->batch.add(r.s->m, r.s->k, r.s->k, 1.0, r.Q, r.s->m, OP_N, r.Ub, r.s->k, OP_N, 0.0,
                              dLeafB.p + r.s->out, r.s->m);
            gU->batch.finalize(stream_);
            plan.add(std::move(gU));
        }
        plan.run(stream_, dstatus.p);
        HM_CUDA(cudaStreamSynchronize(stream_));
        check_status("hss build: leaf strips");
    }
    ws.release();
    // ranks: leaves from their strips, internal nodes the sums (hss_routines.h:82-83)
    std::vector<int> rk(strips.size());
    if (!strips.empty())
        HM_CUDA(cudaMemcpy(rk.data(), dRank.p, rk.size() * sizeof(int), cudaMemcpyDeviceToHost));
    leafU_.assign(nodes_.size(), {0, 0});
    leafV_.assign(nodes_.size(), {0, 0});
    for (size_t i = 0; i < strips.size(); ++i) {
        const Strip& s = strips[i];
        Node& n = nodes_[s.leaf];
        const int r = std::min(rk[i], s.k);
        if (s.which == 0) { n.rankU = r; leafU_[s.leaf] = {s.out, r}; }
        else { n.rankV = r; leafV_[s.leaf] = {s.out, r}; }
    }
    hss_.nested = false;
    hss_.offR.clear();
    hss_.offW.clear();
    hss_.RW.release();
    if (hss_nested_) {
        build_hss_nested(src);
        return;
    }
    for (int i = (int)nodes_.size() - 1; i >= 0; --i) {
        Node& n = nodes_[i];
        if (n.is_leaf) continue;
        n.rankU = nodes_[n.left].rankU + nodes_[n.right].rankU;
        n.rankV = nodes_[n.left].rankV + nodes_[n.right].rankV;
    }
    std::vector<std::vector<int>> under(nodes_.size());  // leaves under each node, left to right
    for (int i = (int)nodes_.size() - 1; i >= 0; --i) {
        if (nodes_[i].is_leaf) under[i] = {i};
        else {
            under[i] = under[nodes_[i].left];
            under[i].insert(under[i].end(), under[nodes_[i].right].begin(), under[nodes_[i].right].end());
        }
    }
    // coupling blocks
    size_t totB = 0;
    for (auto& n : nodes_) {
        if (n.is_leaf) continue;
        const Node& L = nodes_[n.left];
        const Node& R = nodes_[n.right];
        n.offB12 = totB;
        totB += (size_t)L.rankU * R.rankV;
        n.offB21 = totB;
        totB += (size_t)R.rankU * L.rankV;
    }
    dB.alloc(std::max<size_t>(totB, 1));
    dB.zero(stream_);
    if (!levels_.empty()) {
        size_t totP = 0;
        std::vector<size_t> offP(nodes_.size(), 0);
        for (int l : leaves_) { offP[l] = totP; totP += (size_t)N * nodes_[l].rankU; }
        DBuf<double> Pt(std::max<size_t>(totP, 1));
        Plan pp;
        {   // Pt_l = A[l rows, :]^T U_l
            auto g = std::make_unique<GemmStep<double>>(CFG_64x64, src.gen);
            g->gp = src.gp;
            for (int l : leaves_) {
                const Node& L = nodes_[l];
                g->batch.add(N, L.rankU, L.len(), 1.0, src.blk(L.start, 0), src.lda, OP_T,
                             dLeafB.p + leafU_[l].first, L.len(), OP_N, 0.0, Pt.p + offP[l], N, nullptr, 0,
                             L.start, 0);
            }
            g->batch.finalize(stream_);
            pp.add(std::move(g));
        }
        auto gB = std::make_unique<GemmStep<double>>();
        auto flush = [&]() {
            if (gB->batch.empty()) return;
            gB->batch.finalize(stream_);
            pp.add(std::move(gB));
            gB = std::make_unique<GemmStep<double>>();
        };
        for (auto& lvl : levels_)
            for (int id : lvl) {
                const Node& n = nodes_[id];
                const int lc = n.left, rc = n.right;
                const int p1 = nodes_[lc].rankU, p2 = nodes_[rc].rankU;
                // B12[(l in lc), (m in rc)] = Pt_l[m rows]^T V_m ; B21 likewise with roles swapped
                for (int side = 0; side < 2; ++side) {
                    const int rowc = side == 0 ? lc : rc, colc = side == 0 ? rc : lc;
                    double* Bn = dB.p + (side == 0 ? n.offB12 : n.offB21);
                    const int ldb = side == 0 ? p1 : p2;
                    int ro = 0;
                    for (int l : under[rowc]) {
                        const Node& L = nodes_[l];
                        int co = 0;
                        for (int m : under[colc]) {
                            const Node& Mn = nodes_[m];
                            gB->batch.add(L.rankU, Mn.rankV, Mn.len(), 1.0, Pt.p + offP[l] + Mn.start, N, OP_T,
                                          dLeafB.p + leafV_[m].first, Mn.len(), OP_N, 0.0,
                                          Bn + ro + (size_t)co * ldb, ldb);
                            co += Mn.rankV;
                        }
                        ro += L.rankU;
                    }
                    if (gB->batch.size() > 200000) flush();
                }
            }
        flush();
        pp.run(stream_, dstatus.p);
        HM_CUDA(cudaStreamSynchronize(stream_));
    }
    check_status("hss build");
    reduce_hss_coupling(under);
}

// The reference's transfers are identities (hss_routines.h:86-90): a node's basis is the
// block diagonal of its leaves' bases, so its coupling blocks B12 (p1 x q2) and B21 are
// as wide as the sums of its leaves' ranks (2.5K at the top for N = 65536, leaf 128)
// while their numerical rank is that of the kernel block between the two children
// (tens).  A Woodbury factorization over that wide form carries capacitance systems of
// the same width, and its error grows with them (relative residual 2.6e-3 at
// N = 65536 against 1e-8 for the HODLR of the same kernel).  So each coupling block is
// recompressed once, B = F H^T with F orthonormal (p x r) and the singular values
// above 1e-15 s_0 kept in H (q x r), and the operator that factor, solve and multiply
// use is the two-block form U' = U F, V' = V H, B' = I -- equal to the HSS operator to
// rounding.  F and H come from a randomized range finder with an adaptive width:
// Y = B Omega (q x k Gaussian), Q = orth(Y), Z = B^T Q = W S R^T (Gram/Jacobi SVD),
// F = Q R, H = Z R; a block whose rank comes within 8 of k (k < min(p, q)) is redone
// with 2k.  The reference's leaf bases and B stay in hss_ and dLeafB for export.
void Engine::reduce_hss_coupling(const std::vector<std::vector<int>>& under) {
    const int nn = (int)nodes_.size();
    hss_.rankU.assign(nn, 0);
    hss_.rankV.assign(nn, 0);
    hss_.offB12.assign(nn, 0);
    hss_.offB21.assign(nn, 0);
    for (int i = 0; i < nn; ++i) {
        hss_.rankU[i] = nodes_[i].rankU;
        hss_.rankV[i] = nodes_[i].rankV;
        hss_.offB12[i] = nodes_[i].offB12;
        hss_.offB21[i] = nodes_[i].offB21;
    }
    hss_.B = std::move(dB);
    struct Cpl {
        int node, side, rowc, colc, p, q;
        int k = 0, r = 0;
        const double* B = nullptr;
        const double *F = nullptr, *H = nullptr;  // p x k, q x k (ld p, q)
    };
    std::vector<Cpl> cp;
    for (const auto& lvl : levels_)
        for (int id : lvl) {
            const Node& n = nodes_[id];
            for (int side = 0; side < 2; ++side) {
                Cpl c;
                c.node = id;
                c.side = side;
                c.rowc = side == 0 ? n.left : n.right;
                c.colc = side == 0 ? n.right : n.left;
                c.p = hss_.rankU[c.rowc];
                c.q = hss_.rankV[c.colc];
                c.B = hss_.B.p + (side == 0 ? hss_.offB12[id] : hss_.offB21[id]);
                if (c.p > 0 && c.q > 0) cp.push_back(c);
            }
        }
    std::vector<std::unique_ptr<Plan>> keep;   // owns the F/H scratch of every attempt
    std::vector<int> want(cp.size(), 96);
    std::vector<size_t> pending(cp.size());
    for (size_t i = 0; i < cp.size(); ++i) pending[i] = i;
    while (!pending.empty()) {
        keep.push_back(std::make_unique<Plan>());
        Plan& plan = *keep.back();
        size_t omega_total = 0;
        std::vector<size_t> om(pending.size());
        for (size_t j = 0; j < pending.size(); ++j) {
            Cpl& c = cp[pending[j]];
            c.k = std::min(std::min(c.p, c.q), want[pending[j]]);
            om[j] = omega_total;
            omega_total += (size_t)c.q * c.k;
        }
        double* Om = plan.scratch(omega_total);
        normal_fill_kernel<<<grid_for(omega_total), 256, 0, stream_>>>(Om, omega_total, opts_.seed,
                                                                        0x4853530000000000ull + omega_total);
        HM_CUDA(cudaGetLastError());
        count_launch();
        DBuf<int> dRank(pending.size());
        auto gY = std::make_unique<GemmStep<double>>();
        auto gZ = std::make_unique<GemmStep<double>>();
        auto gF = std::make_unique<GemmStep<double>>();
        std::vector<SvdProblem> s1, s2;
        struct W { double *Y, *Q, *Z, *R, *F, *H; };
        std::vector<W> w(pending.size());
        for (size_t j = 0; j < pending.size(); ++j) {
            Cpl& c = cp[pending[j]];
            W& x = w[j];
            x.Y = plan.scratch((size_t)c.p * c.k);
            x.Q = plan.scratch((size_t)c.p * c.k);
            x.Z = plan.scratch((size_t)c.q * c.k);
            x.R = plan.scratch((size_t)c.k * c.k);
            x.F = plan.scratch((size_t)c.p * c.k);
            x.H = plan.scratch((size_t)c.q * c.k);
            gY->batch.add(c.p, c.k, c.q, 1.0, c.B, c.p, OP_N, Om + om[j], c.q, OP_N, 0.0, x.Y, c.p);
            SvdProblem a{};
            a.X = x.Y; a.ldx = c.p; a.rows = c.p; a.k = c.k;
            a.L = x.Q; a.ldl = c.p;
            s1.push_back(a);
            gZ->batch.add(c.q, c.k, c.p, 1.0, c.B, c.p, OP_T, x.Q, c.p, OP_N, 0.0, x.Z, c.q);
            SvdProblem b{};
            b.X = x.Z; b.ldx = c.q; b.rows = c.q; b.k = c.k;
            b.R = x.R; b.ldr = c.k;
            b.rank = dRank.p + j;
            b.sort = true;
            s2.push_back(b);
            gF->batch.add(c.p, c.k, c.k, 1.0, x.Q, c.p, OP_N, x.R, c.k, OP_N, 0.0, x.F, c.p);
            gF->batch.add(c.q, c.k, c.k, 1.0, x.Z, c.q, OP_N, x.R, c.k, OP_N, 0.0, x.H, c.q);
        }
        gY->batch.finalize(stream_);
        plan.add(std::move(gY));
        plan_gram_svd(plan, s1, 0.0, 0, stream_);
        gZ->batch.finalize(stream_);
        plan.add(std::move(gZ));
        plan_gram_svd(plan, s2, 1e-15, 0, stream_);
        gF->batch.finalize(stream_);
        plan.add(std::move(gF));
        plan.run(stream_, dstatus.p);
        std::vector<int> rk(pending.size());
        HM_CUDA(cudaMemcpyAsync(rk.data(), dRank.p, rk.size() * sizeof(int), cudaMemcpyDeviceToHost, stream_));
        HM_CUDA(cudaStreamSynchronize(stream_));
        check_status("hss coupling recompression");
        std::vector<size_t> next;
        for (size_t j = 0; j < pending.size(); ++j) {
            Cpl& c = cp[pending[j]];
            if (rk[j] > c.k - 8 && c.k < std::min(c.p, c.q)) {
                want[pending[j]] = 2 * c.k;
                next.push_back(pending[j]);
            } else {
                c.r = std::min(rk[j], c.k);
                c.F = w[j].F;
                c.H = w[j].H;
            }
        }
        pending.swap(next);
    }
    // the two-block operator: ranks, bases U F / V H leaf by leaf, B' = I
    for (auto& n : nodes_) n.rankU = n.rankV = 0;
    for (const Cpl& c : cp) {
        nodes_[c.rowc].rankU = c.r;
        nodes_[c.colc].rankV = c.r;
    }
    for (auto& n : nodes_) {
        n.capU = n.rankU;
        n.capV = n.rankV;
    }
    alloc_UV();
    size_t totB = 0;
    for (auto& n : nodes_) {
        if (n.is_leaf) continue;
        n.offB12 = totB;
        totB += (size_t)nodes_[n.left].rankU * nodes_[n.right].rankV;
        n.offB21 = totB;
        totB += (size_t)nodes_[n.right].rankU * nodes_[n.left].rankV;
    }
    dB.alloc(std::max<size_t>(totB, 1));
    dB.zero(stream_);
    Plan bp;
    auto gb = std::make_unique<GemmStep<double>>();
    auto id = std::make_unique<IdentStep>();
    for (const Cpl& c : cp) {
        if (c.r == 0) continue;
        const Node& Rw = nodes_[c.rowc];
        const Node& Cl = nodes_[c.colc];
        int ro = 0;
        for (int l : under[c.rowc]) {
            const Node& L = nodes_[l];
            const int rl = leafU_[l].second;
            if (rl)
                gb->batch.add(L.len(), c.r, rl, 1.0, dLeafB.p + leafU_[l].first, L.len(), OP_N, c.F + ro, c.p, OP_N,
                              0.0, dU.p + Rw.offU + (L.start - Rw.start), Rw.len());
            ro += rl;
        }
        int co = 0;
        for (int m : under[c.colc]) {
            const Node& M = nodes_[m];
            const int rm = leafV_[m].second;
            if (rm)
                gb->batch.add(M.len(), c.r, rm, 1.0, dLeafB.p + leafV_[m].first, M.len(), OP_N, c.H + co, c.q, OP_N,
                              0.0, dV.p + Cl.offV + (M.start - Cl.start), Cl.len());
            co += rm;
        }
        const Node& n = nodes_[c.node];
        id->t.h.push_back({dB.p + (c.side == 0 ? n.offB12 : n.offB21), c.r, c.r, c.r, 1.0});
    }
    gb->batch.finalize(stream_);
    bp.add(std::move(gb));
    id->t.upload(stream_);
    bp.add(std::move(id));
    bp.run(stream_, dstatus.p);
    HM_CUDA(cudaStreamSynchronize(stream_));
    check_status("hss two-block form");
}

// ---------------------------------------------------------------------------------
// Import reference factors
// ---------------------------------------------------------------------------------
void Engine::import_hodlr(int N, int leaf, const int* r12, const int* r21, const double* const* D,
                          const double* const* U, const double* const* V, const double* const* B12,
                          const double* const* B21) {
    HM_CHECK(kind_ == HODLR, HM_ERR_STATE, "import is for HODLR handles");
    HM_CHECK(N > 0 && leaf > 0 && r12 && r21 && D && U && V && B12 && B21, HM_ERR_ARG, "import: bad arguments");
    begin_build(N, leaf);
    for (size_t i = 0; i < nodes_.size(); ++i) {
        Node& n = nodes_[i];
        if (n.is_leaf) continue;
        HM_CHECK(r12[i] >= 0 && r21[i] >= 0, HM_ERR_ARG, "import: negative rank");
        nodes_[n.left].capU = nodes_[n.left].rankU = r12[i];
        nodes_[n.right].capV = nodes_[n.right].rankV = r12[i];
        nodes_[n.right].capU = nodes_[n.right].rankU = r21[i];
        nodes_[n.left].capV = nodes_[n.left].rankV = r21[i];
    }
    alloc_bases();
    size_t tot = 0;
    for (size_t i = 0; i < nodes_.size(); ++i) {
        Node& n = nodes_[i];
        if (n.is_leaf) continue;
        n.offB12 = tot;
        tot += (size_t)r12[i] * r12[i];
        n.offB21 = tot;
        tot += (size_t)r21[i] * r21[i];
    }
    dB.alloc(std::max<size_t>(tot, 1));
    auto up = [&](double* dst, const double* src, size_t cnt) {
        if (!cnt) return;
        HM_CHECK(src, HM_ERR_ARG, "import: missing factor");
        HM_CUDA(cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyHostToDevice, stream_));
    };
    for (size_t i = 0; i < nodes_.size(); ++i) {
        Node& n = nodes_[i];
        if (n.is_leaf) up(dD.p + n.offD, D[i], (size_t)n.len() * n.len());
        else {
            up(dB.p + n.offB12, B12[i], (size_t)r12[i] * r12[i]);
            up(dB.p + n.offB21, B21[i], (size_t)r21[i] * r21[i]);
        }
        if (n.parent >= 0) {
            up(dU.p + n.offU, U[i], (size_t)n.len() * n.rankU);
            up(dV.p + n.offV, V[i], (size_t)n.len() * n.rankV);
        }
    }
    HM_CUDA(cudaStreamSynchronize(stream_));
    built_ = true;
}

// ---------------------------------------------------------------------------------
// Factorization
// ---------------------------------------------------------------------------------
static CopyDesc flat_copy(const void* src, bool sf, void* dst, bool df, size_t n) {
    CopyDesc c{};
    c.src = src; c.lds = (int)n; c.dst = dst; c.ldd = (int)n;
    c.rows = (int)n; c.cols = 1; c.trans = 0;
    c.src_f32 = sf; c.dst_f32 = df;
    return c;
}

template <typename T>
void Engine::plan_factor(FactorStore<T>& fs) {
    constexpr bool F32 = std::is_same<T, float>::value;
    cudaStream_t s = stream_;
    fs.plans.clear();
    fs.setup.reset();
    fs.setup_done = false;
    size_t offM = 0, offP = 0;
    for (auto& n : nodes_) {
        if (n.is_leaf) continue;
        const Node& L = nodes_[n.left];
        const Node& R = nodes_[n.right];
        const int p = L.rankU + R.rankU, q = L.rankV + R.rankV;
        n.offM = offM;
        offM += (size_t)q * q;
        if constexpr (F32) {
            n.offP32 = offP;
            offP += (size_t)padded_p(L.rankU, R.rankU) * q;
        } else {
            n.offP = offP;
            offP += (size_t)p * q;
        }
    }
    size_t totU = 1, totV = 1, totD = 1;
    for (auto& n : nodes_) {
        if (n.parent >= 0) {
            totU = std::max(totU, n.offU + (size_t)n.len() * n.capU);
            totV = std::max(totV, n.offV + (size_t)n.len() * n.capV);
        }
        if (n.is_leaf) totD = std::max(totD, n.offD + (size_t)n.len() * n.len());
    }
    fs.plans.push_back(std::make_unique<Plan>());
    Plan& plan = *fs.plans.back();
    {   // FP64 leaf inverses
        if (dDinv.n < totD) dDinv.alloc(totD);
        std::vector<InvProblem> inv;
        for (int l : leaves_) {
            const Node& n = nodes_[l];
            inv.push_back({dD.p + n.offD, n.len(), dDinv.p + n.offD, n.len(), n.len()});
        }
        if (leaves_spd_) plan_inverse_spd(plan, inv, s);   // SPD leaves: no pivoting needed
        else plan_inverse(plan, inv, s);
    }
    if (dMinv.n < std::max<size_t>(offM, 1)) dMinv.alloc(std::max<size_t>(offM, 1));
    sizeM_ = offM;
    if (fs.Q.n < totU) fs.Q.alloc(totU);
    if (fs.P.n < std::max<size_t>(offP, 1)) fs.P.alloc(std::max<size_t>(offP, 1));
    sizeP_ = offP;
    const T* Dinv;
    const T* Vt;
    const T* Ut;
    DBuf<T>& Utmp = fs.Utmp;
    if constexpr (F32) {
        if (fs.Dinv.n < totD) fs.Dinv.alloc(totD);
        if (fs.V.n < totV) fs.V.alloc(totV);
        Utmp.alloc(totU);
        // the bases depend on the built operator only: converted once per build
        auto cb = std::make_unique<CopyStep>();
        cb->t.h.push_back(flat_copy(dV.p, false, fs.V.p, true, totV));
        cb->t.h.push_back(flat_copy(dU.p, false, Utmp.p, true, totU));
        cb->t.upload(s);
        fs.setup = std::make_unique<Plan>();
        fs.setup->add(std::move(cb));
        auto cp = std::make_unique<CopyStep>();
        cp->t.h.push_back(flat_copy(dDinv.p, false, fs.Dinv.p, true, totD));
        cp->t.upload(s);
        plan.add(std::move(cp));
        Dinv = fs.Dinv.p;
        Vt = fs.V.p;
        Ut = Utmp.p;
    } else {
        Dinv = reinterpret_cast<const T*>(dDinv.p);
        Vt = reinterpret_cast<const T*>(dV.p);
        Ut = reinterpret_cast<const T*>(dU.p);
    }
    {   // Q_c[rows of leaf] = Dinv U_c[rows of leaf] for every basis block on the path
        auto g = std::make_unique<GemmStep<T>>("factor.leaf_apply");
        for (int l : leaves_) {
            const Node& n = nodes_[l];
            for (int c : path_of(l)) {
                const Node& C = nodes_[c];
                if (C.rankU == 0) continue;
                const size_t o = C.offU + (size_t)(n.start - C.start);
                g->batch.add(n.len(), C.rankU, n.len(), T(1), Dinv + n.offD, n.len(), OP_N, Ut + o,
                             C.len(), OP_N, T(0), fs.Q.p + o, C.len());
            }
        }
        g->batch.finalize(s);
        plan.add(std::move(g));
    }
    for (int d = (int)levels_.size() - 1; d >= 0; --d) {
        fs.plans.push_back(std::make_unique<Plan>());
        Plan& lp = *fs.plans.back();
        const auto& lvl = levels_[d];
        auto gK = std::make_unique<GemmStep<T>>("factor.K");
        auto cvK = std::make_unique<CopyStep>();
        auto ident = std::make_unique<IdentStep>();
        auto gM = std::make_unique<GemmStep<double>>("factor.M");
        auto gS = std::make_unique<GemmStep<double>>("factor.M");
        auto gZ = std::make_unique<GemmStep<double>>("factor.M");
        auto gTop = std::make_unique<GemmStep<double>>("factor.M");
        std::vector<InvProblem> inv;
        auto gP = std::make_unique<GemmStep<double>>("factor.P");
        auto cvP = std::make_unique<CopyStep>();
        auto gT = std::make_unique<GemmStep<T>>("factor.update_project");
        auto gD = std::make_unique<GemmStep<T>>("factor.update_small");
        auto gC = std::make_unique<GemmStep<T>>("factor.update_correct");
        for (int id : lvl) {
            const Node& n = nodes_[id];
            const Node& L = nodes_[n.left];
            const Node& R = nodes_[n.right];
            const int p1 = L.rankU, p2 = R.rankU, q1 = L.rankV, q2 = R.rankV;
            const int q = q1 + q2, p = p1 + p2;
            const size_t kn = (size_t)q1 * p1 + (size_t)q2 * p2;
            T* Kt;
            double* K64;
            if constexpr (F32) {
                Kt = lp.scratch_f(std::max<size_t>(kn, 1));
                K64 = lp.scratch(std::max<size_t>(kn, 1));
                if (kn) cvK->t.h.push_back(flat_copy(Kt, true, K64, false, kn));
            } else {
                K64 = lp.scratch(std::max<size_t>(kn, 1));
                Kt = K64;
            }
            // K1 = V1^T Q1, K2 = V2^T Q2
            gK->batch.add(q1, p1, L.len(), T(1), Vt + L.offV, L.len(), OP_T, fs.Q.p + L.offU, L.len(),
                          OP_N, T(0), Kt, q1);
            gK->batch.add(q2, p2, R.len(), T(1), Vt + R.offV, R.len(), OP_T, fs.Q.p + R.offU, R.len(),
                          OP_N, T(0), Kt + (size_t)q1 * p1, q2);
            // M = [[I, X], [Y, I]] with X = K1 B12, Y = K2 B21.  Its inverse through the
            // Schur complement of the identity block, S = I - Y X:
            //   Minv[q1:, :] = [-S^-1 Y, S^-1],   Minv[:q1, :] = [I, 0] - X Minv[q1:, :]
            // (one inversion of order q2 instead of one of order q1 + q2).
            double* M = lp.scratch(std::max<size_t>((size_t)q * q, 1));
            double* Minv = dMinv.p + n.offM;
            const double* B12 = dB.p + n.offB12;
            const double* B21 = dB.p + n.offB21;
            double* X = M + (size_t)q1 * q;
            double* Y = M + q1;
            gM->batch.add(q1, q2, p1, 1.0, K64, q1, OP_N, B12, p1, OP_N, 0.0, X, q);
            gM->batch.add(q2, q1, p2, 1.0, K64 + (size_t)q1 * p1, q2, OP_N, B21, p2, OP_N, 0.0, Y, q);
            double* Sinv = Minv + q1 + (size_t)q1 * q;
            if (q2) {
                double* S = lp.scratch((size_t)q2 * q2);
                ident->t.h.push_back({S, q2, q2, q2, 1.0});
                gS->batch.add(q2, q2, q1, -1.0, Y, q, OP_N, X, q, OP_N, 1.0, S, q2);
                inv.push_back({S, q2, Sinv, q, q2});
                gZ->batch.add(q2, q1, q2, -1.0, Sinv, q, OP_N, Y, q, OP_N, 0.0, Minv + q1, q);
            }
            if (q1) {
                ident->t.h.push_back({Minv, q, q1, q, 1.0});
                if (q2) gTop->batch.add(q1, q, q2, -1.0, X, q, OP_N, Minv + q1, q, OP_N, 1.0, Minv, q);
            }
            // P = B^ Minv: P[0:p1,:] = B12 Minv[q1:,:], P[o2:o2+p2,:] = B21 Minv[0:q1,:]
            // (o2 = p1 in FP64; in FP32 p1 rounded up to 4, the gap rows zero)
            const int pp = F32 ? padded_p(p1, p2) : p, o2 = F32 ? pp - p2 : p1;
            double* P64;
            if constexpr (F32) {
                P64 = lp.scratch(std::max<size_t>((size_t)pp * q, 1));
                if (o2 > p1 && q) ident->t.h.push_back({P64 + p1, pp, o2 - p1, q, 0.0});
                if ((size_t)pp * q) cvP->t.h.push_back(flat_copy(P64, false, fs.P.p + n.offP32, true, (size_t)pp * q));
            } else {
                P64 = fs.P.p + n.offP;
            }
            gP->batch.add(p1, q, q2, 1.0, B12, p1, OP_N, Minv + q1, q, OP_N, 0.0, P64, pp);
            gP->batch.add(p2, q, q1, 1.0, B21, p2, OP_N, Minv, q, OP_N, 0.0, P64 + o2, pp);
            // every basis block on n's path: W <- A_n^{-1} W (given blockdiag-solved W)
            const T* Pn = fs.P.p + (F32 ? n.offP32 : n.offP);
            const int ldD = F32 ? (pp + 3) / 4 * 4 : p;
            for (int c : path_of(id)) {
                const Node& C = nodes_[c];
                const int w = C.rankU;
                if (w == 0) continue;
                T* W = fs.Q.p + C.offU + (size_t)(n.start - C.start);
                const int ldw = C.len();
                T* Tt = F32 ? reinterpret_cast<T*>(lp.scratch_f(std::max<size_t>((size_t)q * w, 1)))
                            : reinterpret_cast<T*>(lp.scratch(std::max<size_t>((size_t)q * w, 1)));
                T* Dt = F32 ? reinterpret_cast<T*>(lp.scratch_f(std::max<size_t>((size_t)ldD * w, 1)))
                            : reinterpret_cast<T*>(lp.scratch(std::max<size_t>((size_t)ldD * w, 1)));
                gT->batch.add(q1, w, L.len(), T(1), Vt + L.offV, L.len(), OP_T, W, ldw, OP_N, T(0), Tt, q);
                gT->batch.add(q2, w, R.len(), T(1), Vt + R.offV, R.len(), OP_T, W + L.len(), ldw, OP_N,
                              T(0), Tt + q1, q);
                gD->batch.add(pp, w, q, T(1), Pn, pp, OP_N, Tt, q, OP_N, T(0), Dt, ldD);
                gC->batch.add(L.len(), w, p1, T(-1), fs.Q.p + L.offU, L.len(), OP_N, Dt, ldD, OP_N, T(1), W, ldw);
                gC->batch.add(R.len(), w, p2, T(-1), fs.Q.p + R.offU, R.len(), OP_N, Dt + o2, ldD, OP_N,
                              T(1), W + L.len(), ldw);
            }
        }
        gK->batch.finalize(s);
        lp.add(std::move(gK));
        if (!cvK->t.h.empty()) { cvK->t.upload(s); lp.add(std::move(cvK)); }
        ident->t.upload(s);
        lp.add(std::move(ident));
        gM->batch.finalize(s);
        lp.add(std::move(gM));
        gS->batch.finalize(s);
        lp.add(std::move(gS));
        plan_inverse(lp, inv, s);
        gZ->batch.finalize(s);
        lp.add(std::move(gZ));
        gTop->batch.finalize(s);
        lp.add(std::move(gTop));
        gP->batch.finalize(s);
        lp.add(std::move(gP));
        if (!cvP->t.h.empty()) { cvP->t.upload(s); lp.add(std::move(cvP)); }
        gT->batch.finalize(s);
        lp.add(std::move(gT));
        gD->batch.finalize(s);
        lp.add(std::move(gD));
        gC->batch.finalize(s);
        lp.add(std::move(gC));
    }
    fs.planned = true;
}

// Run the recorded factorization (planned once per operator), then check the status
// word once: singular pivots anywhere are reported after the last level.
template <typename T>
void Engine::factor_t(FactorStore<T>& fs) {
    if (!fs.planned) plan_factor(fs);
    dstatus.zero(stream_);
    if (fs.setup && !fs.setup_done) {
        fs.setup->run(stream_, dstatus.p);
        fs.setup_done = true;
    }
    for (auto& p : fs.plans) p->run(stream_, dstatus.p);
    check_status("factor");
    fs.ready = true;
}

// Recomputes every time it is called (a rebuild or a new operator needs no flag).
void Engine::factor() {
    HM_CHECK(built_, HM_ERR_STATE, "factor before build");
    factored_ = false;
    if (opts_.precision == HM_MIXED) factor_t<float>(f32_);
    else factor_t<double>(f64_);
    factored_ = true;
}

// ---------------------------------------------------------------------------------
// Solve and multiply plans on the staging buffers (ld = N)
// ---------------------------------------------------------------------------------
void Engine::ensure_io(int s) {
    if (s <= io_cols_) return;
    const size_t n = (size_t)N_ * s;
    ioX.alloc(n);
    ioY.alloc(n);
    ioR.alloc(n);
    ioXf.alloc(n);
    ioYf.alloc(n);
    ioNorm.alloc(2 * (size_t)s);
    io_cols_ = s;
    grad_plans_.clear();
    mv_plans_.clear();
    solve64_plans_.clear();
    solve32_plans_.clear();
    solveT_plans_.clear();
}

// y = A x for s columns: in = x (ld N), out = y (ld N)
// sc[k]: right-hand-side columns of system k (rows of all systems share ld N)
static void add_matvec(Plan& pl, const std::vector<Node>& nodes, const std::vector<int>& leaves,
                       const std::vector<std::vector<int>>& levels, const double* dD, const double* dU,
                       const double* dV, const double* dB, const double* X, double* Y, int N,
                       const std::vector<int>& sc, cudaStream_t st) {
    // Projections and couplings of every level first (independent of y):
    //   t = [V1^T x1; V2^T x2],  delta = [B12 t2; B21 t1]  per internal node;
    // then one launch per leaf row block accumulates y = D x + sum over the leaf's path of
    // U_c delta_c in registers (a chain of GEMM problems) and writes y once.
    auto gT = std::make_unique<GemmStep<double>>("matvec.project");
    auto gD = std::make_unique<GemmStep<double>>("matvec.couple");
    std::vector<const double*> delta(nodes.size(), nullptr);   // delta_c of child c
    std::vector<int> ldd(nodes.size(), 0);
    for (size_t d = 0; d < levels.size(); ++d) {
        for (int id : levels[d]) {
            const Node& n = nodes[id];
            const Node& L = nodes[n.left];
            const Node& R = nodes[n.right];
            const int p1 = L.rankU, p2 = R.rankU, q1 = L.rankV, q2 = R.rankV;
            const int s = sc[n.sys];
            if (s == 0) continue;
            double* T = pl.scratch(std::max<size_t>((size_t)(q1 + q2) * s, 1));
            double* Dl = pl.scratch(std::max<size_t>((size_t)(p1 + p2) * s, 1));
            // T1 = V1^T x1, T2 = V2^T x2
            gT->batch.add(q1, s, L.len(), 1.0, dV + L.offV, L.len(), OP_T, X + L.start, N, OP_N, 0.0, T, q1 + q2);
            gT->batch.add(q2, s, R.len(), 1.0, dV + R.offV, R.len(), OP_T, X + R.start, N, OP_N, 0.0,
                          T + q1, q1 + q2);
            // delta1 = B12 T2, delta2 = B21 T1
            gD->batch.add(p1, s, q2, 1.0, dB + n.offB12, p1, OP_N, T + q1, q1 + q2, OP_N, 0.0, Dl, p1 + p2);
            gD->batch.add(p2, s, q1, 1.0, dB + n.offB21, p2, OP_N, T, q1 + q2, OP_N, 0.0, Dl + p1, p1 + p2);
            delta[n.left] = Dl;
            delta[n.right] = Dl + p1;
            ldd[n.left] = ldd[n.right] = p1 + p2;
        }
    }
    auto gY = std::make_unique<GemmStep<double>>("matvec.leaf_expand");
    for (int l : leaves) {
        const Node& n = nodes[l];
        const int s = sc[n.sys];
        if (s == 0) continue;
        gY->batch.add(n.len(), s, n.len(), 1.0, dD + n.offD, n.len(), OP_N, X + n.start, N, OP_N, 0.0, Y + n.start,
                      N, nullptr, 1);
        for (int c = l; nodes[c].parent >= 0; c = nodes[c].parent) {
            const Node& C = nodes[c];
            if (C.rankU == 0 || !delta[c]) continue;
            gY->batch.add_chained(n.len(), s, C.rankU, 1.0, dU + C.offU + (n.start - C.start), C.len(), OP_N,
                                  delta[c], ldd[c], OP_N);
        }
    }
    gT->batch.finalize(st);
    pl.add(std::move(gT));
    gD->batch.finalize(st);
    pl.add(std::move(gD));
    gY->batch.finalize(st);
    pl.add(std::move(gY));
}

Plan& Engine::matvec_plan(const std::vector<int>& sc) {
    auto it = mv_plans_.find(sc);
    if (it != mv_plans_.end()) return it->second;
    Plan& pl = mv_plans_[sc];
    if (kind_ == HSS && hss_.nested) add_matvec_nested(pl, ioX.p, ioY.p, sc[0]);
    else add_matvec(pl, nodes_, leaves_, levels_, dD.p, dU.p, dV.p, dB.p, ioX.p, ioY.p, N_, sc, stream_);
    return pl;
}

// z = A^{-1} x in precision T: in = X (ld N), out = Z (ld N)
template <typename T>
static void add_solve(Plan& pl, const std::vector<Node>& nodes, const std::vector<int>& leaves,
                      const std::vector<std::vector<int>>& levels, const T* Dinv, const T* Vt,
                      const T* Q, const T* P, const T* X, T* Z, int N, const std::vector<int>& sc,
                      cudaStream_t st) {
    constexpr bool F32 = std::is_same<T, float>::value;
    auto gLeaf = std::make_unique<GemmStep<T>>("solve.leaf");
    for (int l : leaves) {
        const Node& n = nodes[l];
        const int s = sc[n.sys];
        gLeaf->batch.add(n.len(), s, n.len(), T(1), Dinv + n.offD, n.len(), OP_N, X + n.start, N, OP_N,
                         T(0), Z + n.start, N);
    }
    gLeaf->batch.finalize(st);
    pl.add(std::move(gLeaf));
    for (int d = (int)levels.size() - 1; d >= 0; --d) {
        auto gT = std::make_unique<GemmStep<T>>("solve.project");
        auto gD = std::make_unique<GemmStep<T>>("solve.small");
        auto gC = std::make_unique<GemmStep<T>>("solve.correct");

        for (int id : levels[d]) {
            const Node& n = nodes[id];
            const Node& L = nodes[n.left];
            const Node& R = nodes[n.right];
            const int p1 = L.rankU, p2 = R.rankU, q1 = L.rankV, q2 = R.rankV;
            const int p = p1 + p2, q = q1 + q2;
            const int s = sc[n.sys];
            if (s == 0) continue;
            T* Tt = F32 ? reinterpret_cast<T*>(pl.scratch_f(std::max<size_t>((size_t)q * s, 1)))
                        : reinterpret_cast<T*>(pl.scratch(std::max<size_t>((size_t)q * s, 1)));
            // FP32: P in its padded layout (second block at o2 = p1 rounded up to 4)
            const int pp = F32 ? padded_p(p1, p2) : p, o2 = F32 ? pp - p2 : p1;
            const int ldD = F32 ? (pp + 3) / 4 * 4 : p;
            T* Dt = F32 ? reinterpret_cast<T*>(pl.scratch_f(std::max<size_t>((size_t)ldD * s, 1)))
                        : reinterpret_cast<T*>(pl.scratch(std::max<size_t>((size_t)ldD * s, 1)));
            gT->batch.add(q1, s, L.len(), T(1), Vt + L.offV, L.len(), OP_T, Z + L.start, N, OP_N, T(0), Tt, q);
            gT->batch.add(q2, s, R.len(), T(1), Vt + R.offV, R.len(), OP_T, Z + R.start, N, OP_N, T(0),
                          Tt + q1, q);
            gD->batch.add(pp, s, q, T(1), P + (F32 ? n.offP32 : n.offP), pp, OP_N, Tt, q, OP_N, T(0), Dt, ldD);
            gC->batch.add(L.len(), s, p1, T(-1), Q + L.offU, L.len(), OP_N, Dt, ldD, OP_N, T(1), Z + L.start, N);
            gC->batch.add(R.len(), s, p2, T(-1), Q + R.offU, R.len(), OP_N, Dt + o2, ldD, OP_N, T(1),
                          Z + R.start, N);
        }
        gT->batch.finalize(st);
        pl.add(std::move(gT));
        gD->batch.finalize(st);
        pl.add(std::move(gD));
        gC->batch.finalize(st);
        pl.add(std::move(gC));
    }
}

template <>
Plan& Engine::solve_plan<double>(FactorStore<double>& fs, const std::vector<int>& sc) {
    auto it = solve64_plans_.find(sc);
    if (it != solve64_plans_.end()) return it->second;
    Plan& pl = solve64_plans_[sc];
    add_solve<double>(pl, nodes_, leaves_, levels_, dDinv.p, dV.p, fs.Q.p, fs.P.p, ioX.p, ioY.p, N_, sc,
                      stream_);
    return pl;
}

template <>
Plan& Engine::solve_plan<float>(FactorStore<float>& fs, const std::vector<int>& sc) {
    auto it = solve32_plans_.find(sc);
    if (it != solve32_plans_.end()) return it->second;
    Plan& pl = solve32_plans_[sc];
    add_solve<float>(pl, nodes_, leaves_, levels_, fs.Dinv.p, fs.V.p, fs.Q.p, fs.P.p, ioXf.p, ioYf.p,
                     N_, sc, stream_);
    return pl;
}

// Host or device source/destination (unified addressing decides the direction).
static void copy_in(double* dst, const double* src, int N, int s, int ld, cudaStream_t st) {
    HM_CUDA(cudaMemcpy2DAsync(dst, (size_t)N * sizeof(double), src, (size_t)ld * sizeof(double),
                              (size_t)N * sizeof(double), s, cudaMemcpyDefault, st));
}
static void copy_out(double* dst, int ld, const double* src, int N, int s, cudaStream_t st) {
    HM_CUDA(cudaMemcpy2DAsync(dst, (size_t)ld * sizeof(double), src, (size_t)N * sizeof(double),
                              (size_t)N * sizeof(double), s, cudaMemcpyDefault, st));
}

void Engine::multiply_device(const double* dx, int s, int ldx, double* dy, int ldy) {
    HM_CHECK(built_, HM_ERR_STATE, "multiply before build");
    HM_CHECK(s >= 1 && ldx >= N_ && ldy >= N_ && dx && dy, HM_ERR_ARG, "multiply: bad arguments");
    ensure_io(s);
    copy_in(ioX.p, dx, N_, s, ldx, stream_);
    matvec_plan(uniform(s)).run(stream_, dstatus.p);
    copy_out(dy, ldy, ioY.p, N_, s, stream_);
}

void Engine::solve_fp64(const double* db, int s, int ldb, double* dx, int ldx) {
    ensure_io(s);
    if (opts_.refine_steps <= 0) {
        copy_in(ioX.p, db, N_, s, ldb, stream_);
        solve_plan<double>(f64_, uniform(s)).run(stream_, dstatus.p);
        copy_out(dx, ldx, ioY.p, N_, s, stream_);
        return;
    }
    copy_in(ioR.p, db, N_, s, ldb, stream_);
    copy_out(dx, ldx, refined_fp64(uniform(s), s), N_, s, stream_);
}

// b in ioR (staging, ld N); returns the staging buffer holding x after the direct solve
// and opts_.refine_steps steps of x += A^{-1}(b - A x), all in FP64 with one factorization.
const double* Engine::refined_fp64(const std::vector<int>& sc, int smax) {
    const size_t n = (size_t)N_ * smax;
    if (ioAcc.n < n) ioAcc.alloc(n);
    Plan& sp = solve_plan<double>(f64_, sc);
    HM_CUDA(cudaMemcpyAsync(ioX.p, ioR.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    sp.run(stream_, dstatus.p);
    HM_CUDA(cudaMemcpyAsync(ioAcc.p, ioY.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    Plan& mp = matvec_plan(sc);
    for (int it = 0; it < opts_.refine_steps; ++it) {
        HM_CUDA(cudaMemcpyAsync(ioX.p, ioAcc.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        mp.run(stream_, dstatus.p);                                   // ioY = A x
        axpby_kernel<<<grid_for(n), 256, 0, stream_>>>(ioX.p, ioR.p, 1.0, ioY.p, -1.0, n);  // r = b - A x
        sp.run(stream_, dstatus.p);                                   // ioY = A^{-1} r
        axpby_kernel<<<grid_for(n), 256, 0, stream_>>>(ioAcc.p, ioAcc.p, 1.0, ioY.p, 1.0, n);
        count_launch(2);
    }
    return ioAcc.p;
}

// Mixed precision: FP32 factor sweeps, refined against the FP64 operator
// (x += A32^{-1} r, r = b - A64 x) until max_j ||r_j|| / ||b_j|| <= ir_tol.
void Engine::solve_mixed(const double* db, int s, int ldb, double* dx, int ldx, hm_solve_stats* st) {
    ensure_io(s);
    cudaStream_t q = stream_;
    // ioR = b, ioX = x (also the matvec input), ioY = A x then r, ioXf = float(r),
    // ioYf = the FP32 correction.
    double* bcopy = ioR.p;
    copy_in(bcopy, db, N_, s, ldb, q);
    to_float_kernel<<<grid_for((size_t)N_ * s), 256, 0, q>>>(bcopy, ioXf.p, (size_t)N_ * s);
    count_launch();
    Plan& sp = solve_plan<float>(f32_, uniform(s));
    Plan& mp = matvec_plan(uniform(s));
    // x into page-locked host memory: each sweep's x is copied out on the copy stream while
    // the residual of that x is computed; the copy of the sweep that converges is the answer
    cudaPointerAttributes pa{};
    HM_CUDA(cudaPointerGetAttributes(&pa, dx));
    const bool spec_out = pa.type == cudaMemoryTypeHost;
    if (spec_out) ensure_copy_stream();
    std::vector<double> hn(2 * (size_t)s);
    double worst = 0.0;
    int it = 0;
    for (; it < std::max(1, opts_.ir_max_iter); ++it) {
        sp.run(q, dstatus.p);                                   // ioYf = A32^{-1} r
        if (spec_out && it > 0) HM_CUDA(cudaStreamWaitEvent(q, copy_done_.get(), 0));   // previous copy read x
        accumulate_kernel<<<grid_for((size_t)N_ * s), 256, 0, q>>>(ioX.p, ioYf.p, (size_t)N_ * s, it == 0);
        count_launch();
        if (spec_out) {
            HM_CUDA(cudaEventRecord(x_ready_.get(), q));
            HM_CUDA(cudaStreamWaitEvent(copy_stream_.get(), x_ready_.get(), 0));
            copy_out(dx, ldx, ioX.p, N_, s, copy_stream_.get());
            HM_CUDA(cudaEventRecord(copy_done_.get(), copy_stream_.get()));
        }
        mp.run(q, dstatus.p);                                   // ioY = A64 x
        HM_CUDA(cudaMemsetAsync(ioNorm.p, 0, 2 * (size_t)s * sizeof(double), q));
        residual_kernel<<<dim3(std::min(64, ceil_div(N_, 256)), s), 256, 0, q>>>(
            bcopy, ioY.p, ioXf.p, N_, s, ioNorm.p, ioNorm.p + s);  // ioY = b - A x, ioXf = float(r)
        count_launch();
        HM_CUDA(cudaMemcpyAsync(hn.data(), ioNorm.p, 2 * s * sizeof(double), cudaMemcpyDeviceToHost, q));
        HM_CUDA(cudaStreamSynchronize(q));
        worst = 0.0;
        for (int j = 0; j < s; ++j) {
            double den = std::sqrt(hn[s + j]);
            double rel = den > 0 ? std::sqrt(hn[j]) / den : std::sqrt(hn[j]);
            worst = max_nan(worst, rel);
        }
        if (!(worst == worst)) break;  // NaN
        if (worst <= opts_.ir_tol) { ++it; break; }
    }
    if (spec_out) HM_CUDA(cudaStreamSynchronize(copy_stream_.get()));
    else copy_out(dx, ldx, ioX.p, N_, s, q);
    HM_CUDA(cudaStreamSynchronize(q));
    if (st) {
        st->ir_iters = it;
        st->rel_residual = worst;
    }
    if (!(worst <= opts_.ir_tol)) {
        char msg[128];
        snprintf(msg, sizeof msg, "iterative refinement stopped at relative residual %.3e after %d sweeps", worst, it);
        throw Error(HM_ERR_IR, msg);
    }
}

// Refinement against the exact kernel operator of a matrix-free build:
//   x = A~^{-1} b;  repeat r = b - A x (A generated on the device, 2 N^2 s flops),
//   stop when max_j ||r_j|| / ||b_j|| <= tol, else x += A~^{-1} r,
// with A~^{-1} the compressed factorization in the handle's precision.  Each sweep
// contracts the error by about ||A - A~|| ||A~^{-1}||.
Plan& Engine::exact_plan(int s) {
    auto it = exact_plans_.find(s);
    if (it != exact_plans_.end()) return it->second;
    Plan& pl = exact_plans_[s];
    auto g = std::make_unique<GemmStep<double>>(s <= 16 ? CFG_N_SKINNY : CFG_64x64, gen_);
    g->gp = gp_;
    g->batch.add(N_, s, N_, 1.0, nullptr, 0, OP_N, exX_.p, N_, OP_N, 0.0, exR_.p, N_, nullptr, 0, 0, 0);
    g->batch.finalize(stream_);
    pl.add(std::move(g));
    return pl;
}

void Engine::solve_exact_device(const double* db, int s, int ldb, double* dx, int ldx, double tol, int max_iter,
                                hm_solve_stats* st) {
    HM_CHECK(built_, HM_ERR_STATE, "solve_exact before build");
    HM_CHECK(gen_ != GEN_DENSE && sys_N_.size() == 1, HM_ERR_STATE,
             "solve_exact needs a single operator built from a kernel (hm_*_build_from_kernel)");
    HM_CHECK(s >= 1 && ldb >= N_ && ldx >= N_ && db && dx && tol > 0 && max_iter >= 0, HM_ERR_ARG,
             "solve_exact: bad arguments");
    const size_t n = (size_t)N_ * s;
    if (s > ex_cols_) {
        exB_.alloc(n);
        exX_.alloc(n);
        exR_.alloc(n);
        exD_.alloc(n);
        exNorm_.alloc(2 * (size_t)s);
        ex_cols_ = s;
        exact_plans_.clear();
    }
    cudaStream_t q = stream_;
    HM_CUDA(cudaMemcpy2DAsync(exB_.p, (size_t)N_ * sizeof(double), db, (size_t)ldb * sizeof(double),
                              (size_t)N_ * sizeof(double), s, cudaMemcpyDefault, q));
    solve_device(exB_.p, s, N_, exX_.p, N_, nullptr);
    Plan& ap = exact_plan(s);
    std::vector<double> hn(2 * (size_t)s);
    double worst = 0.0;
    int it = 0;
    for (;; ++it) {
        ap.run(q, dstatus.p);   // exR = A x
        HM_CUDA(cudaMemsetAsync(exNorm_.p, 0, 2 * (size_t)s * sizeof(double), q));
        residual_kernel<<<dim3(std::min(64, ceil_div(N_, 256)), s), 256, 0, q>>>(
            exB_.p, exR_.p, nullptr, N_, s, exNorm_.p, exNorm_.p + s);   // exR = b - A x
        count_launch();
        HM_CUDA(cudaMemcpyAsync(hn.data(), exNorm_.p, 2 * s * sizeof(double), cudaMemcpyDeviceToHost, q));
        HM_CUDA(cudaStreamSynchronize(q));
        check_status("solve_exact");
        worst = 0.0;
        for (int j = 0; j < s; ++j) {
            const double den = std::sqrt(hn[s + j]);
            worst = max_nan(worst, den > 0 ? std::sqrt(hn[j]) / den : std::sqrt(hn[j]));
        }
        if (!(worst == worst) || worst <= tol || it >= max_iter) break;
        solve_device(exR_.p, s, N_, exD_.p, N_, nullptr);
        axpby_kernel<<<grid_for(n), 256, 0, q>>>(exX_.p, exX_.p, 1.0, exD_.p, 1.0, n);
        count_launch();
    }
    HM_CUDA(cudaMemcpy2DAsync(dx, (size_t)ldx * sizeof(double), exX_.p, (size_t)N_ * sizeof(double),
                              (size_t)N_ * sizeof(double), s, cudaMemcpyDefault, q));
    HM_CUDA(cudaStreamSynchronize(q));
    if (st) {
        st->ir_iters = it;
        st->rel_residual = worst;
    }
    if (!(worst <= tol)) {
        char msg[160];
        snprintf(msg, sizeof msg, "exact-operator refinement stopped at relative residual %.3e after %d sweeps",
                 worst, it);
        throw Error(HM_ERR_IR, msg);
    }
}

// dx = A~^{-1} db once with the handle's factorization (ld N both): the FP64 solve, or in
// mixed precision one FP32 sweep without refinement (a preconditioner application).
void Engine::precondition_device(const double* db, int s, double* dx) {
    HM_CHECK(built_, HM_ERR_STATE, "precondition before build");
    if (!factored_) factor();
    if (opts_.precision != HM_MIXED) {
        solve_fp64(db, s, N_, dx, N_);
        return;
    }
    ensure_io(s);
    const size_t n = (size_t)N_ * s;
    to_float_kernel<<<grid_for(n), 256, 0, stream_>>>(db, ioXf.p, n);
    count_launch();
    solve_plan<float>(f32_, uniform(s)).run(stream_, dstatus.p);   // ioYf = A32^{-1} float(b)
    accumulate_kernel<<<grid_for(n), 256, 0, stream_>>>(dx, ioYf.p, n, 1);
    count_launch();
    HM_CUDA(cudaGetLastError());
}

// rel[j] = ||b_j - A x_j|| / ||b_j|| with A the exact kernel operator, its entries
// generated inside the batched FP64 product (2 N^2 s flops; A never stored).
void Engine::residual_exact(const double* db, int ldb, const double* dx, int ldx, int s, double* rel) {
    HM_CHECK(built_, HM_ERR_STATE, "residual_exact before build");
    HM_CHECK(gen_ != GEN_DENSE && sys_N_.size() == 1, HM_ERR_STATE,
             "residual_exact needs a single operator built from a kernel (hm_*_build_from_kernel)");
    HM_CHECK(s >= 1 && ldb >= N_ && ldx >= N_ && db && dx && rel, HM_ERR_ARG, "residual_exact: bad arguments");
    const size_t n = (size_t)N_ * s;
    if (s > ex_cols_) {
        exB_.alloc(n);
        exX_.alloc(n);
        exR_.alloc(n);
        exD_.alloc(n);
        exNorm_.alloc(2 * (size_t)s);
        ex_cols_ = s;
        exact_plans_.clear();
    }
    cudaStream_t q = stream_;
    HM_CUDA(cudaMemcpy2DAsync(exB_.p, (size_t)N_ * sizeof(double), db, (size_t)ldb * sizeof(double),
                              (size_t)N_ * sizeof(double), s, cudaMemcpyDefault, q));
    HM_CUDA(cudaMemcpy2DAsync(exX_.p, (size_t)N_ * sizeof(double), dx, (size_t)ldx * sizeof(double),
                              (size_t)N_ * sizeof(double), s, cudaMemcpyDefault, q));
    exact_plan(s).run(q, dstatus.p);   // exR = A x
    HM_CUDA(cudaMemsetAsync(exNorm_.p, 0, 2 * (size_t)s * sizeof(double), q));
    residual_kernel<<<dim3(std::min(64, ceil_div(N_, 256)), s), 256, 0, q>>>(exB_.p, exR_.p, nullptr, N_, s,
                                                                           exNorm_.p, exNorm_.p + s);
    HM_CUDA(cudaGetLastError());
    count_launch();
    std::vector<double> hn(2 * (size_t)s);
    HM_CUDA(cudaMemcpyAsync(hn.data(), exNorm_.p, 2 * s * sizeof(double), cudaMemcpyDeviceToHost, q));
    HM_CUDA(cudaStreamSynchronize(q));
    check_status("residual_exact");
    for (int j = 0; j < s; ++j) {
        const double den = std::sqrt(hn[s + j]);
        rel[j] = den > 0 ? std::sqrt(hn[j]) / den : std::sqrt(hn[j]);
    }
}

void Engine::ensure_copy_stream() {
    if (copy_stream_) return;
    cudaStream_t cs = nullptr;
    HM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    copy_stream_.reset(cs, [](cudaStream_t q) { cudaStreamDestroy(q); });
    cudaEvent_t e = nullptr, r = nullptr;
    HM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    copy_done_.reset(e, [](cudaEvent_t v) { cudaEventDestroy(v); });
    HM_CUDA(cudaEventCreateWithFlags(&r, cudaEventDisableTiming));
    x_ready_.reset(r, [](cudaEvent_t v) { cudaEventDestroy(v); });
}

// The reference's solve(b) (factor and solve in one call): a host b is staged to the
// device on a copy stream while the factorization runs on the handle's stream.
void Engine::factor_solve(const double* b, int s, int ldb, double* x, int ldx, hm_solve_stats* st) {
    HM_CHECK(built_, HM_ERR_STATE, "solve before build");
    HM_CHECK(s >= 1 && ldb >= N_ && ldx >= N_ && b && x, HM_ERR_ARG, "solve: bad arguments");
    cudaPointerAttributes pa{};
    HM_CUDA(cudaPointerGetAttributes(&pa, b));
    const bool host = pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged;
    if (!host) {
        factor();
        solve_device(b, s, ldb, x, ldx, st);
        return;
    }
    const size_t n = (size_t)N_ * s;
    if (fsB_.n < n) fsB_.alloc(n);
    ensure_copy_stream();
    HM_CUDA(cudaMemcpy2DAsync(fsB_.p, (size_t)N_ * sizeof(double), b, (size_t)ldb * sizeof(double),
                              (size_t)N_ * sizeof(double), s, cudaMemcpyHostToDevice, copy_stream_.get()));
    HM_CUDA(cudaEventRecord(copy_done_.get(), copy_stream_.get()));
    try {
        factor();
    } catch (...) {
        cudaEventSynchronize(copy_done_.get());   // fsB_ stays in use until the copy lands
        throw;
    }
    HM_CUDA(cudaStreamWaitEvent(stream_, copy_done_.get(), 0));
    solve_device(fsB_.p, s, N_, x, ldx, st);
}

void Engine::solve_device(const double* db, int s, int ldb, double* dx, int ldx, hm_solve_stats* st) {
    HM_CHECK(built_, HM_ERR_STATE, "solve before build");
    HM_CHECK(s >= 1 && ldb >= N_ && ldx >= N_ && db && dx, HM_ERR_ARG, "solve: bad arguments");
    if (!factored_) factor();
    if (st) { st->ir_iters = 0; st->rel_residual = -1.0; }
    if (opts_.precision == HM_MIXED) solve_mixed(db, s, ldb, dx, ldx, st);
    else solve_fp64(db, s, ldb, dx, ldx);
}

// ---------------------------------------------------------------------------------
// Adjoint: A^T lam = g with the FP64 factors.  A^{-1} = F_0 ... F_{L-1} Dinv with
// F_d = I - Q P V~^T per node of level d, so A^{-T} = Dinv^T F_{L-1}^T ... F_0^T:
// root level first, t = [Q1^T l1; Q2^T l2], gamma = P^T t, l1 -= V1 gamma_1,
// l2 -= V2 gamma_2; then lam_leaf = Dinv^T l_leaf.
// ---------------------------------------------------------------------------------
Plan& Engine::solveT_plan(int s) {
    auto it = solveT_plans_.find(s);
    if (it != solveT_plans_.end()) return it->second;
    Plan& pl = solveT_plans_[s];
    const int N = N_;
    double* Z = ioX.p;
    for (size_t d = 0; d < levels_.size(); ++d) {
        auto gT = std::make_unique<GemmStep<double>>();
        auto gG = std::make_unique<GemmStep<double>>();
        auto gC = std::make_unique<GemmStep<double>>();
        for (int id : levels_[d]) {
            const Node& n = nodes_[id];
            const Node& L = nodes_[n.left];
            const Node& R = nodes_[n.right];
            const int p1 = L.rankU, p2 = R.rankU, q1 = L.rankV, q2 = R.rankV;
            const int p = p1 + p2, q = q1 + q2;
            double* T = pl.scratch(std::max<size_t>((size_t)p * s, 1));
            double* G = pl.scratch(std::max<size_t>((size_t)q * s, 1));
            gT->batch.add(p1, s, L.len(), 1.0, f64_.Q.p + L.offU, L.len(), OP_T, Z + L.start, N, OP_N, 0.0, T, p);
            gT->batch.add(p2, s, R.len(), 1.0, f64_.Q.p + R.offU, R.len(), OP_T, Z + R.start, N, OP_N, 0.0, T + p1, p);
            gG->batch.add(q, s, p, 1.0, f64_.P.p + n.offP, p, OP_T, T, p, OP_N, 0.0, G, q);
            gC->batch.add(L.len(), s, q1, -1.0, dV.p + L.offV, L.len(), OP_N, G, q, OP_N, 1.0, Z + L.start, N);
            gC->batch.add(R.len(), s, q2, -1.0, dV.p + R.offV, R.len(), OP_N, G + q1, q, OP_N, 1.0, Z + R.start, N);
        }
        gT->batch.finalize(stream_);
        pl.add(std::move(gT));
        gG->batch.finalize(stream_);
        pl.add(std::move(gG));
        gC->batch.finalize(stream_);
        pl.add(std::move(gC));
    }
    auto gL = std::make_unique<GemmStep<double>>();
    for (int l : leaves_) {
        const Node& n = nodes_[l];
        gL->batch.add(n.len(), s, n.len(), 1.0, dDinv.p + n.offD, n.len(), OP_T, Z + n.start, N, OP_N, 0.0,
                      ioY.p + n.start, N);
    }
    gL->batch.finalize(stream_);
    pl.add(std::move(gL));
    return pl;
}

void Engine::solve_transpose_device(const double* dg, int s, int ldg, double* dl, int ldl) {
    HM_CHECK(built_, HM_ERR_STATE, "solve_transpose before build");
    HM_CHECK(s >= 1 && ldg >= N_ && ldl >= N_ && dg && dl, HM_ERR_ARG, "solve_transpose: bad arguments");
    if (!f64_.ready) factor_t<double>(f64_);
    ensure_io(s);
    copy_in(ioX.p, dg, N_, s, ldg, stream_);
    solveT_plan(s).run(stream_, dstatus.p);
    copy_out(dl, ldl, ioY.p, N_, s, stream_);
}

// Gradients of a loss L through x = A^{-1} b, given x and lam = A^{-T} dL/dx, so that
// dL/dA = -lam x^T: per leaf dD = -lam x^T; per node, with A12 = U1 B12 V2^T and
// A21 = U2 B21 V1^T, dU1 = -lam1 (B12 V2^T x2)^T, dV2 = -x2 (B12^T U1^T lam1)^T,
// dB12 = -(U1^T lam1)(V2^T x2)^T, and likewise for A21.  For a kernel-generated
// operator also dL/dp0 and dL/dp1 of the exact kernel (matrix-free, O(N^2 s)).
void Engine::gradients(const double* dx, int ldx, const double* dl, int ldl, int s, double* dparams) {
    HM_CHECK(built_, HM_ERR_STATE, "gradients before build");
    HM_CHECK(s >= 1 && ldx >= N_ && ldl >= N_ && dx && dl, HM_ERR_ARG, "gradients: bad arguments");
    const int N = N_;
    ensure_io(s);
    // stage x in ioX and lam in ioY (ld N)
    copy_in(ioX.p, dx, N, s, ldx, stream_);
    copy_in(ioY.p, dl, N, s, ldl, stream_);
    // gradient storage like the factors' (kept across calls); the launch plan per column
    // count is recorded once per operator
    bool fresh = false;
    for (auto pr : {std::make_pair(&gD_, dD.n), std::make_pair(&gU_, dU.n), std::make_pair(&gV_, dV.n),
                    std::make_pair(&gB_, dB.n)}) {
        if (pr.first->n != std::max<size_t>(pr.second, 1)) {
            pr.first->alloc(std::max<size_t>(pr.second, 1));
            fresh = true;
        }
    }
    if (fresh) grad_plans_.clear();
    if (!gAcc_.p) gAcc_.alloc(2);
    gU_.zero(stream_);
    gV_.zero(stream_);
    auto found = grad_plans_.find(s);
    if (found == grad_plans_.end()) found = grad_plans_.emplace(s, grad_plan(s)).first;
    found->second.run(stream_, dstatus.p);
    if (dparams) {
        dparams[0] = dparams[1] = std::nan("");
        if (gen_ != GEN_DENSE) {
            gAcc_.zero(stream_);
            launch_param_grad(gen_, gp_, ioX.p, ioY.p, N, s, gAcc_.p, stream_);
            count_launch();
            double h[2];
            HM_CUDA(cudaMemcpyAsync(h, gAcc_.p, sizeof h, cudaMemcpyDeviceToHost, stream_));
            HM_CUDA(cudaStreamSynchronize(stream_));
            dparams[0] = h[0];
            dparams[1] = h[1];
        }
    }
    HM_CUDA(cudaStreamSynchronize(stream_));
    grads_ready_ = true;
}

// dL/d(factors) for s columns staged in ioX (x) and ioY (lam), into gD_/gU_/gV_/gB_.
Plan Engine::grad_plan(int s) {
    const int N = N_;
    Plan pl;
    const double *X = ioX.p, *Lm = ioY.p;
    auto gLeaf = std::make_unique<GemmStep<double>>();
    for (int l : leaves_) {
        const Node& n = nodes_[l];
        gLeaf->batch.add(n.len(), n.len(), s, -1.0, Lm + n.start, N, OP_N, X + n.start, N, OP_T, 0.0,
                         gD_.p + n.offD, n.len());
    }
    auto gProj = std::make_unique<GemmStep<double>>();
    auto gMid = std::make_unique<GemmStep<double>>();
    auto gOut = std::make_unique<GemmStep<double>>();
    for (auto& lvl : levels_)
        for (int id : lvl) {
            const Node& n = nodes_[id];
            const Node& L = nodes_[n.left];
            const Node& R = nodes_[n.right];
            const int p1 = L.rankU, p2 = R.rankU, q1 = L.rankV, q2 = R.rankV;
            double* t1 = pl.scratch(std::max<size_t>((size_t)q1 * s, 1));   // V1^T x1
            double* t2 = pl.scratch(std::max<size_t>((size_t)q2 * s, 1));   // V2^T x2
            double* w1 = pl.scratch(std::max<size_t>((size_t)p1 * s, 1));   // U1^T lam1
            double* w2 = pl.scratch(std::max<size_t>((size_t)p2 * s, 1));   // U2^T lam2
            double* u1 = pl.scratch(std::max<size_t>((size_t)p1 * s, 1));   // B12 t2
            double* u2 = pl.scratch(std::max<size_t>((size_t)p2 * s, 1));   // B21 t1
            double* v2 = pl.scratch(std::max<size_t>((size_t)q2 * s, 1));   // B12^T w1
            double* v1 = pl.scratch(std::max<size_t>((size_t)q1 * s, 1));   // B21^T w2
            const double* B12 = dB.p + n.offB12;
            const double* B21 = dB.p + n.offB21;
            gProj->batch.add(q1, s, L.len(), 1.0, dV.p + L.offV, L.len(), OP_T, X + L.start, N, OP_N, 0.0, t1, q1);
            gProj->batch.add(q2, s, R.len(), 1.0, dV.p + R.offV, R.len(), OP_T, X + R.start, N, OP_N, 0.0, t2, q2);
            gProj->batch.add(p1, s, L.len(), 1.0, dU.p + L.offU, L.len(), OP_T, Lm + L.start, N, OP_N, 0.0, w1, p1);
            gProj->batch.add(p2, s, R.len(), 1.0, dU.p + R.offU, R.len(), OP_T, Lm + R.start, N, OP_N, 0.0, w2, p2);
            gMid->batch.add(p1, s, q2, 1.0, B12, p1, OP_N, t2, q2, OP_N, 0.0, u1, p1);
            gMid->batch.add(p2, s, q1, 1.0, B21, p2, OP_N, t1, q1, OP_N, 0.0, u2, p2);
            gMid->batch.add(q2, s, p1, 1.0, B12, p1, OP_T, w1, p1, OP_N, 0.0, v2, q2);
            gMid->batch.add(q1, s, p2, 1.0, B21, p2, OP_T, w2, p2, OP_N, 0.0, v1, q1);
            // dU1 = -lam1 u1^T, dU2 = -lam2 u2^T, dV2 = -x2 v2^T, dV1 = -x1 v1^T
            gOut->batch.add(L.len(), p1, s, -1.0, Lm + L.start, N, OP_N, u1, p1, OP_T, 0.0, gU_.p + L.offU, L.len());
            gOut->batch.add(R.len(), p2, s, -1.0, Lm + R.start, N, OP_N, u2, p2, OP_T, 0.0, gU_.p + R.offU, R.len());
            gOut->batch.add(R.len(), q2, s, -1.0, X + R.start, N, OP_N, v2, q2, OP_T, 0.0, gV_.p + R.offV, R.len());
            gOut->batch.add(L.len(), q1, s, -1.0, X + L.start, N, OP_N, v1, q1, OP_T, 0.0, gV_.p + L.offV, L.len());
            // dB12 = -w1 t2^T, dB21 = -w2 t1^T
            gOut->batch.add(p1, q2, s, -1.0, w1, p1, OP_N, t2, q2, OP_T, 0.0, gB_.p + n.offB12, p1);
            gOut->batch.add(p2, q1, s, -1.0, w2, p2, OP_N, t1, q1, OP_T, 0.0, gB_.p + n.offB21, p2);
        }
    for (auto* g : {gLeaf.get(), gProj.get(), gMid.get(), gOut.get()}) g->batch.finalize(stream_);
    pl.add(std::move(gLeaf));
    pl.add(std::move(gProj));
    pl.add(std::move(gMid));
    pl.add(std::move(gOut));
    return pl;
}

void Engine::get_gradient(int node, int which, double* out, int* rows, int* cols) const {
    HM_CHECK(grads_ready_, HM_ERR_STATE, "get_gradient before gradients");
    HM_CHECK(kind_ == HODLR, HM_ERR_UNSUPPORTED, "factor gradients are for HODLR operators");
    HM_CHECK(node >= 0 && node < (int)nodes_.size(), HM_ERR_ARG, "get_gradient: bad node");
    const Node& n = nodes_[node];
    const double* src = nullptr;
    int r = 0, c = 0, ld = 0;
    switch (which) {
        case 0: if (n.is_leaf) { src = gD_.p + n.offD; r = c = ld = n.len(); } break;
        case 1: if (n.parent >= 0) { src = gU_.p + n.offU; r = ld = n.len(); c = n.rankU; } break;
        case 2: if (n.parent >= 0) { src = gV_.p + n.offV; r = ld = n.len(); c = n.rankV; } break;
        case 3: if (!n.is_leaf) { src = gB_.p + n.offB12; r = ld = nodes_[n.left].rankU; c = nodes_[n.right].rankV; } break;
        case 4: if (!n.is_leaf) { src = gB_.p + n.offB21; r = ld = nodes_[n.right].rankU; c = nodes_[n.left].rankV; } break;
        default: throw Error(HM_ERR_ARG, "get_gradient: bad selector");
    }
    if (rows) *rows = r;
    if (cols) *cols = c;
    if (out && r * c > 0)
        HM_CUDA(cudaMemcpy2D(out, (size_t)r * sizeof(double), src, (size_t)ld * sizeof(double),
                             (size_t)r * sizeof(double), c, cudaMemcpyDeviceToHost));
}

// ---------------------------------------------------------------------------------
// Introspection
// ---------------------------------------------------------------------------------
void Engine::export_tree(int* start, int* end, int* is_leaf, int* depth, int* r12, int* r21) const {
    for (size_t i = 0; i < nodes_.size(); ++i) {
        const Node& n = nodes_[i];
        if (start) start[i] = n.start;
        if (end) end[i] = n.end;
        if (is_leaf) is_leaf[i] = n.is_leaf;
        if (depth) depth[i] = n.depth;
        int a = 0, b = 0;
        if (kind_ == HSS) {  // rank_U, rank_V (utils.h:41-42)
            a = hss_.rankU[i];
            b = hss_.rankV[i];
        } else if (!n.is_leaf) {  // B_12, B_21 sizes (hodlr_routines.h:140-141)
            a = nodes_[n.left].rankU;
            b = nodes_[n.right].rankU;
        }
        if (r12) r12[i] = a;
        if (r21) r21[i] = b;
    }
}

void Engine::get_factor(int node, int which, double* out, int* rows, int* cols) const {
    HM_CHECK(built_, HM_ERR_STATE, "get_factor before build");
    HM_CHECK(node >= 0 && node < (int)nodes_.size(), HM_ERR_ARG, "get_factor: bad node");
    const Node& n = nodes_[node];
    const double* src = nullptr;
    int r = 0, c = 0, ld = 0;
    if (kind_ == HSS) {  // HSSNode fields (utils.h:32-55)
        std::vector<double> host;
        switch (which) {
            case 0: if (n.is_leaf) { src = dD.p + n.offD; r = c = ld = n.len(); } break;
            case 1: if (n.is_leaf) { src = dLeafB.p + leafU_[node].first; r = ld = n.len(); c = leafU_[node].second; } break;
            case 2: if (n.is_leaf) { src = dLeafB.p + leafV_[node].first; r = ld = n.len(); c = leafV_[node].second; } break;
            case 3:  // R = I (hss_routines.h:86-87); nested builds: the compressed transfer
            case 4: {  // W = I (hss_routines.h:89-90)
                if (hss_.nested) {
                    const auto& rk = which == 3 ? hss_.rankU : hss_.rankV;
                    if (n.is_leaf || n.parent < 0 || rk[node] == 0) break;
                    src = hss_.RW.p + (which == 3 ? hss_.offR[node] : hss_.offW[node]);
                    r = ld = rk[n.left] + rk[n.right];
                    c = rk[node];
                    break;
                }
                const int k = which == 3 ? hss_.rankU[node] : hss_.rankV[node];
                if (n.is_leaf || k == 0) break;
                r = c = k;
                if (out)
                    for (int j = 0; j < k; ++j)
                        for (int i = 0; i < k; ++i) out[i + (size_t)j * k] = i == j;
                if (rows) *rows = r;
                if (cols) *cols = c;
                return;
            }
            case 5: {  // B = [[0, B12], [B21, 0]] at (0, lc.rank_V) and (lc.rank_U, 0) (hss_routines.h:105-107)
                const auto& hu = hss_.rankU;
                const auto& hv = hss_.rankV;
                if (n.is_leaf) break;
                const int lc = n.left, rc = n.right;
                r = hu[lc] + hu[rc];   // = rank_U of the node in the reference form
                c = hv[lc] + hv[rc];
                if (r == 0 || c == 0) { r = c = 0; break; }
                if (out) {
                    std::fill(out, out + (size_t)r * c, 0.0);
                    std::vector<double> b12((size_t)hu[lc] * hv[rc]), b21((size_t)hu[rc] * hv[lc]);
                    if (!b12.empty())
                        HM_CUDA(cudaMemcpy(b12.data(), hss_.B.p + hss_.offB12[node], b12.size() * 8,
                                           cudaMemcpyDeviceToHost));
                    if (!b21.empty())
                        HM_CUDA(cudaMemcpy(b21.data(), hss_.B.p + hss_.offB21[node], b21.size() * 8,
                                           cudaMemcpyDeviceToHost));
                    for (int j = 0; j < hv[rc]; ++j)
                        for (int i = 0; i < hu[lc]; ++i)
                            out[i + (size_t)(hv[lc] + j) * r] = b12[i + (size_t)j * hu[lc]];
                    for (int j = 0; j < hv[lc]; ++j)
                        for (int i = 0; i < hu[rc]; ++i)
                            out[(hu[lc] + i) + (size_t)j * r] = b21[i + (size_t)j * hu[rc]];
                }
                if (rows) *rows = r;
                if (cols) *cols = c;
                return;
            }
            default: throw Error(HM_ERR_ARG, "get_factor: bad selector");
        }
        if (rows) *rows = r;
        if (cols) *cols = c;
        if (out && r * c > 0)
            HM_CUDA(cudaMemcpy2D(out, (size_t)r * sizeof(double), src, (size_t)ld * sizeof(double),
                                 (size_t)r * sizeof(double), c, cudaMemcpyDeviceToHost));
        return;
    }
    switch (which) {
        case 0: if (n.is_leaf) { src = dD.p + n.offD; r = c = ld = n.len(); } break;
        case 1: if (n.parent >= 0) { src = dU.p + n.offU; r = ld = n.len(); c = n.rankU; } break;
        case 2: if (n.parent >= 0) { src = dV.p + n.offV; r = ld = n.len(); c = n.rankV; } break;
        case 3: if (!n.is_leaf) { src = dB.p + n.offB12; r = ld = nodes_[n.left].rankU; c = nodes_[n.right].rankV; } break;
        case 4: if (!n.is_leaf) { src = dB.p + n.offB21; r = ld = nodes_[n.right].rankU; c = nodes_[n.left].rankV; } break;
        default: throw Error(HM_ERR_ARG, "get_factor: bad selector");
    }
    if (rows) *rows = r;
    if (cols) *cols = c;
    if (out && r * c > 0) {
        HM_CUDA(cudaMemcpy2D(out, (size_t)r * sizeof(double), src, (size_t)ld * sizeof(double),
                             (size_t)r * sizeof(double), c, cudaMemcpyDeviceToHost));
    }
}

template void Engine::factor_t<double>(FactorStore<double>&);
template void Engine::factor_t<float>(FactorStore<float>&);

}  // namespace hm
