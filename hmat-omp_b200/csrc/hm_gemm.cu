// Batched variable-size GEMM for sm_100a (FP64 DFMA / FP32 FFMA register tiles).
//
// One CTA computes one BM x BN output tile of one problem over one k-slice.  The
// problem is found by binary search of the tile prefix sums in the descriptor table.
// Operand tiles are staged through double-buffered shared memory with a register
// prefetch of the next k-tile; each thread owns a TM x TN block of the tile strided by
// the thread grid so that shared-memory reads and global stores are conflict-free and
// coalesced along the column-major row index.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "hm_gemm.h"

#include <dlfcn.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <mutex>
#include <sstream>
#include <unordered_map>

namespace hm {

// ---------------------------------------------------------------------------------
// Matrix-free operator entries (FP64 math; the FP32 engine rounds the result).
// ---------------------------------------------------------------------------------
template <int GEN>
__device__ __forceinline__ double gen_entry(const GenParams& g, int r, int c) {
    const double p0 = g.p0v ? g.p0v[g.row_sys[r]] : g.p0;
    const double p1 = g.p1v ? g.p1v[g.row_sys[r]] : g.p1;
    if constexpr (GEN == GEN_CAUCHY) {
        double x = g.pts[r], y = g.pts[g.N + c];
        double v = 1.0 / (x - y);
        return r == c ? v + p0 : v;
    } else if constexpr (GEN == GEN_GAUSSIAN) {
        double d2 = 0.0;
        for (int t = 0; t < g.dim; ++t) {
            double d = g.pts[(size_t)r * g.dim + t] - g.pts[(size_t)c * g.dim + t];
            d2 += d * d;
        }
        double v = exp(-d2 / (2.0 * p0 * p0));
        return r == c ? v + p1 : v;
    } else if constexpr (GEN == GEN_COULOMB) {
        double d2 = 0.0;
        for (int t = 0; t < g.dim; ++t) {
            double d = g.pts[(size_t)r * g.dim + t] - g.pts[(size_t)c * g.dim + t];
            d2 += d * d;
        }
        double v = 1.0 / (sqrt(d2) + p0);
        return r == c ? v + p1 : v;
    } else {
        return 0.0;
    }
}

template <typename T, int BM, int BN, int BK, int TM, int TN, int GEN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
gemm_batched_kernel(const GemmDesc<T>* __restrict__ descs, int ndesc, GenParams gp) {
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int TX = BM / TM;
    constexpr int TY = BN / TN;
    constexpr int LA = BM * BK / NT;
    constexpr int LB = BN * BK / NT;
    static_assert(BM * BK % NT == 0 && BN * BK % NT == 0, "tile/threads mismatch");
    __shared__ __align__(16) T As[2][BK][BM + 1];
    __shared__ __align__(16) T Bs[2][BK][BN + 1];

    const int tile = blockIdx.x;
    int lo = 0, hi = ndesc - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (descs[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    const GemmDesc<T>& D = descs[lo];
    const int m = D.m, n = D.n, k = D.k;
    const int lda = D.lda, ldb = D.ldb;
    const int opA = D.opA, opB = D.opB;
    const T* __restrict__ A = D.A;
    const T* __restrict__ B = D.B;
    const T* __restrict__ ks = D.kscale;
    int t = tile - D.tile0;
    const int tm = t % D.tiles_m;
    t /= D.tiles_m;
    const int tn = t % D.tiles_n;
    const int kslice = t / D.tiles_n;
    const int m0 = tm * BM, n0 = tn * BN;
    int kper = (k + D.ksplit - 1) / D.ksplit;
    kper = (kper + BK - 1) / BK * BK;
    const int kb = kslice * kper;
    const int ke = min(k, kb + kper);

    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;

    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

    T ra[LA], rb[LB];

    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < LA; ++q) {
            int e = tid + NT * q;
            int i, kk;
            if (opA == OP_N) { i = e % BM; kk = e / BM; } else { i = e / BK; kk = e % BK; }
            int gi = m0 + i, gk = k0 + kk;
            T v = T(0);
            if (gi < m && gk < ke) {
                if constexpr (GEN == GEN_DENSE) {
                    v = opA == OP_N ? A[gi + (size_t)gk * lda] : A[gk + (size_t)gi * lda];
                } else {
                    v = opA == OP_N ? (T)gen_entry<GEN>(gp, D.ga_r0 + gi, D.ga_c0 + gk)
                                    : (T)gen_entry<GEN>(gp, D.ga_r0 + gk, D.ga_c0 + gi);
                }
            }
            ra[q] = v;
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            int e = tid + NT * q;
            int j, kk;
            if (opB == OP_N) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
            int gj = n0 + j, gk = k0 + kk;
            T v = T(0);
            if (gj < n && gk < ke) {
                v = opB == OP_N ? B[gk + (size_t)gj * ldb] : B[gj + (size_t)gk * ldb];
                if (ks) v *= ks[gk];
            }
            rb[q] = v;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < LA; ++q) {
            int e = tid + NT * q;
            int i, kk;
            if (opA == OP_N) { i = e % BM; kk = e / BM; } else { i = e / BK; kk = e % BK; }
            As[buf][kk][i] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            int e = tid + NT * q;
            int j, kk;
            if (opB == OP_N) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
            Bs[buf][kk][j] = rb[q];
        }
    };

    const int nk = (ke - kb + BK - 1) / BK;
    if (nk > 0) {
        load(kb);
        store(0);
        __syncthreads();
        for (int it = 0; it < nk; ++it) {
            const int buf = it & 1;
            if (it + 1 < nk) load(kb + (it + 1) * BK);
#pragma unroll
            for (int kk = 0; kk < BK; ++kk) {
                T a[TM], b[TN];
#pragma unroll
                for (int i = 0; i < TM; ++i) a[i] = As[buf][kk][tx + TX * i];
#pragma unroll
                for (int j = 0; j < TN; ++j) b[j] = Bs[buf][kk][ty + TY * j];
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
            }
            if (it + 1 < nk) store(buf ^ 1);
            __syncthreads();
        }
    }

    T* __restrict__ C = D.C;
    const int ldc = D.ldc;
    const T alpha = D.alpha, beta = D.beta;
    const bool split = D.ksplit > 1;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        int gi = m0 + tx + TX * i;
        if (gi >= m) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            int gj = n0 + ty + TY * j;
            if (gj >= n) continue;
            T v = alpha * acc[i][j];
            T* c = C + gi + (size_t)gj * ldc;
            if (split) atomicAdd(c, v);
            else *c = (beta == T(0)) ? v : fma(beta, *c, v);
        }
    }
}

#include "hm_gemm_tile.cuh"
#include "hm_gemm_dmma.cuh"
#include "hm_gemm_tc.cuh"

template <typename T>
__global__ void zero_regions_kernel(const ZeroRegion<T>* __restrict__ z, int count) {
    // one block per region, block-stride inside
    int r = blockIdx.x;
    if (r >= count) return;
    ZeroRegion<T> q = z[r];
    size_t total = (size_t)q.m * q.n;
    for (size_t e = threadIdx.x; e < total; e += blockDim.x) {
        int i = (int)(e % q.m), j = (int)(e / q.m);
        q.C[i + (size_t)j * q.ldc] = T(0);
    }
}

template <int GEN>
__global__ void gen_fill_kernel(const GenFillDesc* __restrict__ descs, GenParams gp) {
    const GenFillDesc d = descs[blockIdx.x];
    const size_t total = (size_t)d.rows * d.cols;
    for (size_t e = blockIdx.y * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.y * blockDim.x) {
        const int i = (int)(e % d.rows), j = (int)(e / d.rows);
        d.dst[i + (size_t)j * d.ldd] =
            d.trans ? gen_entry<GEN>(gp, d.r0 + j, d.c0 + i) : gen_entry<GEN>(gp, d.r0 + i, d.c0 + j);
    }
}

void launch_gen_fill(const GenFillDesc* d_descs, int count, int max_elems, int gen, const GenParams& gp,
                     cudaStream_t s) {
    if (count <= 0) return;
    dim3 grid((unsigned)count, (unsigned)std::min(std::max(1, (max_elems + 255) / 256), 2048));
    switch (gen) {
        case GEN_CAUCHY: gen_fill_kernel<GEN_CAUCHY><<<grid, 256, 0, s>>>(d_descs, gp); break;
        case GEN_GAUSSIAN: gen_fill_kernel<GEN_GAUSSIAN><<<grid, 256, 0, s>>>(d_descs, gp); break;
        case GEN_COULOMB: gen_fill_kernel<GEN_COULOMB><<<grid, 256, 0, s>>>(d_descs, gp); break;
        default: throw Error(HM_ERR_ARG, "unknown kernel generator");
    }
    HM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------
// dL/dp of the exact kernel operator: dL/dA = -lam x^T, so
//   dL/dp0 = -sum_ij dA_ij/dp0 * sum_k lam_ik x_jk,  dL/dp1 = -sum_i sum_k lam_ik x_ik
// (p1 is the diagonal shift of the Gaussian and Coulomb kernels; for Cauchy the shift is
// p0 and has no off-diagonal part).  One CTA: 128 rows x PG_COLS columns, both operand
// panels staged in shared memory as [k][index].
// ---------------------------------------------------------------------------------
constexpr int PG_ROWS = 128, PG_COLS = 1024, PG_TILE = 128;

// dA_ij/dp0 with the parameter-only factors precomputed (c1, c2: Gaussian 1/(2h^2), 1/h^3;
// Coulomb: the softening p0, unused): no division per pair for the Gaussian.
template <int GEN>
__device__ __forceinline__ double gen_dparam(const GenParams& g, int r, int c, double c1, double c2) {
    if constexpr (GEN == GEN_GAUSSIAN) {
        double d2 = 0.0;
        for (int t = 0; t < g.dim; ++t) {
            const double d = g.pts[(size_t)r * g.dim + t] - g.pts[(size_t)c * g.dim + t];
            d2 += d * d;
        }
        return exp(-d2 * c1) * d2 * c2;
    } else if constexpr (GEN == GEN_COULOMB) {
        double d2 = 0.0;
        for (int t = 0; t < g.dim; ++t) {
            const double d = g.pts[(size_t)r * g.dim + t] - g.pts[(size_t)c * g.dim + t];
            d2 += d * d;
        }
        const double den = sqrt(d2) + c1;
        return -1.0 / (den * den);
    } else {
        return r == c ? 1.0 : 0.0;  // Cauchy: p0 is the diagonal shift
    }
}

// SYM (kernels symmetric in i, j: Gaussian, Coulomb): only pairs j >= i are visited and an
// off-diagonal pair adds g_ij (Lam_ij + Lam_ji), Lam = lam x^T summed over the columns;
// CTAs whose whole column range lies below their rows return at once.
template <int GEN, bool SYM>
__global__ void __launch_bounds__(PG_ROWS) param_grad_kernel(GenParams gp, const double* __restrict__ X,
                                                             const double* __restrict__ L, int N, int s,
                                                             double* acc) {
    extern __shared__ double sm[];
    double* Lr = sm;                                     // [s][PG_ROWS]  lam of this CTA's rows
    double* Xr = Lr + (size_t)s * PG_ROWS;               // [s][PG_ROWS]  x of the rows (SYM)
    double* Xc = Xr + (SYM ? (size_t)s * PG_ROWS : 0);   // [s][PG_TILE]  x of the column tile
    double* Lc = Xc + (size_t)s * PG_TILE;               // [s][PG_TILE]  lam of the column tile (SYM)
    const int i0 = blockIdx.x * PG_ROWS, j0 = blockIdx.y * PG_COLS;
    if (SYM && j0 + PG_COLS <= i0) return;
    const int t = threadIdx.x, i = i0 + t;
    for (int k = 0; k < s; ++k) {
        Lr[k * PG_ROWS + t] = i < N ? L[i + (size_t)k * N] : 0.0;
        if (SYM) Xr[k * PG_ROWS + t] = i < N ? X[i + (size_t)k * N] : 0.0;
    }
    double c1 = gp.p0, c2 = 0.0;
    if (GEN == GEN_GAUSSIAN) {
        const double h = gp.p0;
        c1 = 1.0 / (2.0 * h * h);
        c2 = 1.0 / (h * h * h);
    }
    double a0 = 0.0, a1 = 0.0;
    for (int jt = j0; jt < min(N, j0 + PG_COLS); jt += PG_TILE) {
        __syncthreads();
        for (int k = 0; k < s; ++k) {
            const int j = jt + t;
            Xc[k * PG_TILE + t] = j < N ? X[j + (size_t)k * N] : 0.0;
            if (SYM) Lc[k * PG_TILE + t] = j < N ? L[j + (size_t)k * N] : 0.0;
        }
        __syncthreads();
        if (i >= N) continue;
        if (SYM && jt + PG_TILE <= i) continue;   // this tile lies below row i
        const int jn = min(PG_TILE, N - jt);
        for (int jj = 0; jj < jn; ++jj) {
            const int j = jt + jj;
            if (SYM && j < i) continue;
            double dot = 0.0;
            for (int k = 0; k < s; ++k) dot = fma(Lr[k * PG_ROWS + t], Xc[k * PG_TILE + jj], dot);
            if (i == j) a1 += dot;
            if (SYM && j > i)
                for (int k = 0; k < s; ++k) dot = fma(Lc[k * PG_TILE + jj], Xr[k * PG_ROWS + t], dot);
            a0 = fma(gen_dparam<GEN>(gp, i, j, c1, c2), dot, a0);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        a0 += __shfl_down_sync(0xffffffffu, a0, off);
        a1 += __shfl_down_sync(0xffffffffu, a1, off);
    }
    if ((t & 31) == 0) {
        atomicAdd(&acc[0], -a0);
        atomicAdd(&acc[1], GEN == GEN_CAUCHY ? 0.0 : -a1);
    }
}

template <int GEN, bool SYM>
static void launch_pg(dim3 grid, size_t smem, const GenParams& gp, const double* X, const double* L, int N, int s,
                      double* acc, cudaStream_t st) {
    static size_t cur = 0;
    ensure_dyn_smem(param_grad_kernel<GEN, SYM>, smem, cur);
    param_grad_kernel<GEN, SYM><<<grid, PG_ROWS, smem, st>>>(gp, X, L, N, s, acc);
}

void launch_param_grad(int gen, const GenParams& gp, const double* X, const double* L, int N, int s,
                       double* acc, cudaStream_t st) {
    HM_CHECK(s >= 1 && s <= 96, HM_ERR_UNSUPPORTED, "kernel-parameter gradient supports 1..96 columns");
    // the symmetric pass stages twice the operands: up to 48 columns within shared memory
    const bool sym = (gen == GEN_GAUSSIAN || gen == GEN_COULOMB) && s <= 48;
    const size_t smem = (size_t)s * (PG_ROWS + PG_TILE) * sizeof(double) * (sym ? 2 : 1);
    dim3 grid((unsigned)ceil_div(N, PG_ROWS), (unsigned)ceil_div(N, PG_COLS));
    switch (gen) {
        case GEN_GAUSSIAN:
            if (sym) launch_pg<GEN_GAUSSIAN, true>(grid, smem, gp, X, L, N, s, acc, st);
            else launch_pg<GEN_GAUSSIAN, false>(grid, smem, gp, X, L, N, s, acc, st);
            break;
        case GEN_COULOMB:
            if (sym) launch_pg<GEN_COULOMB, true>(grid, smem, gp, X, L, N, s, acc, st);
            else launch_pg<GEN_COULOMB, false>(grid, smem, gp, X, L, N, s, acc, st);
            break;
        case GEN_CAUCHY: launch_pg<GEN_CAUCHY, false>(grid, smem, gp, X, L, N, s, acc, st); break;
        default: throw Error(HM_ERR_ARG, "parameter gradient needs a kernel-generated operator");
    }
    HM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------
struct CfgShape { int BM, BN, BK; };
static CfgShape cfg_shape(int cfg) {
    switch (cfg) {
        case CFG_N_SKINNY: return {128, 16, 16};
        default: return {64, 64, 16};
    }
}

// Target k per slice when a long-k problem with few output tiles is split (atomically
// reduced slices).  Each slice accumulates in T, so the FP32 slice length bounds the
// rounding of the FP32 projections that the mixed refinement's contraction depends on
// (at 1024 the headline's refinement needs a third sweep).  HM_KSPLIT_K (FP32) and
// HM_KSPLIT_K_F64 override the default of 256.
template <typename T>
static int ksplit_k() {
    static const int v = [] {
        const char* e = std::getenv(sizeof(T) == 8 ? "HM_KSPLIT_K_F64" : "HM_KSPLIT_K");
        const int x = e ? std::atoi(e) : 256;
        return x >= 32 ? x : 256;
    }();
    return v;
}

template <typename T>
void GemmBatch<T>::add(int m, int n, int k, T alpha, const T* A, int lda, int opA, const T* B,
                       int ldb, int opB, T beta, T* C, int ldc, const T* kscale, int ksplit,
                       int ga_r0, int ga_c0) {
    if (m <= 0 || n <= 0) return;
    HM_CHECK(!finalized_, HM_ERR_STATE, "GemmBatch::add after finalize");
    CfgShape cs = cfg_shape(cfg_);
    GemmDesc<T> d{};
    d.A = A; d.B = B; d.C = C; d.kscale = kscale;
    d.alpha = alpha; d.beta = beta;
    d.m = m; d.n = n; d.k = std::max(k, 0);
    d.lda = lda; d.ldb = ldb; d.ldc = ldc;
    d.opA = opA; d.opB = opB;
    d.tiles_m = ceil_div(m, cs.BM);
    d.tiles_n = ceil_div(n, cs.BN);
    d.ga_r0 = ga_r0; d.ga_c0 = ga_c0;
    d.next = -1;
    d.is_link = 0;
    if (ksplit <= 0) {
        int tiles = d.tiles_m * d.tiles_n;
        ksplit = 1;
        const int kk = ksplit_k<T>();
        if (tiles < 32 && k >= 2 * kk) ksplit = std::min(std::max(1, k / kk), std::max(1, 128 / tiles));
    }
    ksplit = std::max(1, std::min(ksplit, std::max(1, ceil_div(std::max(k, 1), cs.BK))));
    if (ksplit > 1 && beta != T(0)) {
        HM_CHECK(beta == T(1), HM_ERR_ARG, "split-K GEMM needs beta 0 or 1");
    }
    d.ksplit = ksplit;
    if (ksplit > 1 && beta == T(0)) hz_.push_back({C, m, n, ldc});
    if (k <= 0 && beta == T(0)) {
        // empty product: C = 0
        d.ksplit = 1;
    }
    h_.push_back(d);
    chain_head_ = chain_tail_ = (int)h_.size() - 1;
}

template <typename T>
void GemmBatch<T>::add_chained(int m, int n, int k, T alpha, const T* A, int lda, int opA, const T* B, int ldb,
                               int opB) {
    HM_CHECK(!finalized_, HM_ERR_STATE, "GemmBatch::add_chained after finalize");
    HM_CHECK(chain_head_ >= 0 && gen_ == GEN_DENSE, HM_ERR_STATE, "add_chained: no dense head problem");
    const GemmDesc<T>& hd = h_[chain_head_];
    HM_CHECK(hd.m == m && hd.n == n && hd.alpha == alpha && hd.ksplit == 1 && hd.kscale == nullptr, HM_ERR_ARG,
             "add_chained: the link must match its head (m, n, alpha; head ksplit 1, no kscale)");
    if (k <= 0) return;
    GemmDesc<T> d = hd;
    d.A = A; d.B = B; d.lda = lda; d.ldb = ldb; d.opA = opA; d.opB = opB; d.k = k;
    d.tiles_m = d.tiles_n = 0;
    d.next = -1;
    d.is_link = 1;
    h_.push_back(d);
    h_[chain_tail_].next = (int)h_.size() - 1;
    chain_tail_ = (int)h_.size() - 1;
    has_chains_ = true;
}

// ---------------------------------------------------------------------------------
// Tile-choice table (autotune.py writes it; finalize consults it)
// ---------------------------------------------------------------------------------
namespace {
struct TileTable {
    std::mutex mu;
    bool loaded = false;
    std::unordered_map<std::string, TileChoice> map;
};
TileTable& tile_table() {
    static TileTable t;
    return t;
}

bool valid_choice(const TileChoice& c) {
    return (c.bn == 32 || c.bn == 64 || c.bn == 96 || c.bn == 128) && (c.small >= 0 && c.small <= 3) &&
           (c.tc == 0 || c.tc == 1);
}

// {"signature": [bn, small, tc], ...}; nothing else is accepted
bool parse_tile_table(const std::string& txt, std::unordered_map<std::string, TileChoice>& out) {
    size_t i = 0;
    auto peek = [&]() -> char { return i < txt.size() ? txt[i] : '\0'; };
    auto skip = [&] { while (i < txt.size() && std::isspace((unsigned char)txt[i])) ++i; };
    skip();
    if (peek() != '{') return false;
    ++i;
    skip();
    if (peek() == '}') return true;
    for (;;) {
        skip();
        if (peek() != '"') return false;
        const size_t j = txt.find('"', i + 1);
        if (j == std::string::npos) return false;
        const std::string key = txt.substr(i + 1, j - i - 1);
        i = j + 1;
        skip();
        if (peek() != ':') return false;
        ++i;
        skip();
        if (peek() != '[') return false;
        ++i;
        long v[3];
        for (int q = 0; q < 3; ++q) {
            skip();
            const char* b = txt.c_str() + i;
            char* e = nullptr;
            v[q] = std::strtol(b, &e, 10);
            if (e == b) return false;
            i += (size_t)(e - b);
            skip();
            if (q < 2) {
                if (peek() != ',') return false;
                ++i;
            }
        }
        if (peek() != ']') return false;
        ++i;
        TileChoice c;
        c.bn = (int)v[0];
        c.small = (int)v[1];
        c.tc = (int)v[2];
        if (!valid_choice(c)) return false;
        out[key] = c;
        skip();
        if (peek() == ',') { ++i; continue; }
        if (peek() == '}') return true;
        return false;
    }
}

bool read_tile_table(const std::string& path, std::unordered_map<std::string, TileChoice>& out) {
    std::ifstream f(path);
    if (!f) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    std::unordered_map<std::string, TileChoice> m;
    if (!parse_tile_table(ss.str(), m)) return false;
    out.swap(m);
    return true;
}

std::string library_dir() {
    Dl_info info{};
    if (!dladdr(reinterpret_cast<void*>(&tile_table_size), &info) || !info.dli_fname) return "";
    std::string p(info.dli_fname);
    const size_t slash = p.rfind('/');
    return slash == std::string::npos ? std::string(".") : p.substr(0, slash);
}

const TileChoice* forced_choice() {
    static TileChoice c;
    static const bool on = [] {
        const char* e = std::getenv("HM_TILE_FORCE");
        if (!e || !*e) return false;
        int bn = 0, sm = 0, tc = 0;
        HM_CHECK(std::sscanf(e, "%d,%d,%d", &bn, &sm, &tc) == 3, HM_ERR_ARG, "HM_TILE_FORCE: expected bn,small,tc");
        c.bn = bn;
        c.small = sm;
        c.tc = tc;
        HM_CHECK(valid_choice(c), HM_ERR_ARG, "HM_TILE_FORCE: bn in {32,64,96,128}, shape 0-3, tc 0 or 1");
        return true;
    }();
    return on ? &c : nullptr;
}
}  // namespace

bool tile_choice(const std::string& sig, TileChoice& out) {
    if (const TileChoice* f = forced_choice()) {
        out = *f;
        return true;
    }
    TileTable& t = tile_table();
    std::lock_guard<std::mutex> g(t.mu);
    if (!t.loaded) {
        t.loaded = true;
        const char* e = std::getenv("HM_TILE_TABLE");
        if (e && *e) {
            HM_CHECK(read_tile_table(e, t.map), HM_ERR_ARG, std::string("HM_TILE_TABLE: cannot read ") + e);
        } else {
            const std::string dir = library_dir();
            if (!dir.empty()) read_tile_table(dir + "/tile_table.json", t.map);  // optional
        }
    }
    auto it = t.map.find(sig);
    if (it == t.map.end()) return false;
    out = it->second;
    return true;
}

bool tile_table_load(const char* path) {
    TileTable& t = tile_table();
    std::lock_guard<std::mutex> g(t.mu);
    t.loaded = true;
    if (!path || !*path) {
        t.map.clear();
        return true;
    }
    return read_tile_table(path, t.map);
}

int tile_table_size() {
    TileTable& t = tile_table();
    std::lock_guard<std::mutex> g(t.mu);
    return (int)t.map.size();
}

static int pow2_ceil(long long v) {
    int p = 1;
    while (p < v && p < (1 << 30)) p <<= 1;
    return p;
}

template <typename T>
std::string GemmBatch<T>::choice() const {
    return std::to_string(gen_tc_ ? gen_bn_ : pipe_bn_) + "," + std::to_string(pipe_shape_) + "," +
           (use_tc_ || use_dmma_ ? "1" : "0");
}

// HM_FP64_BIG=1 gives FP64 batches without a table entry that would take the default
// warp-tiled shape the 8 x 8-per-lane shape instead (a measurement switch).
static bool fp64_big_forced() {
    static const bool on = [] {
        const char* e = std::getenv("HM_FP64_BIG");
        return e && e[0] == '1' && e[1] == 0;
    }();
    return on;
}

// 96-row tiles for batches of tile width <= 64 whose every problem has a multiple of 96
// rows (projections onto rank-96 bases of 64 right-hand sides) that the chosen shape would
// pad, on top of the tile table's choice (not of HM_TILE_FORCE's); HM_TILE96=0 turns this
// off.  At width 96 (V^T Q, V^T W of the factorization) the 96 x 96 tile measured slower
// than the table's choice: 1 CTA of 6 warps per SM in FP64.
static bool tile96_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("HM_TILE96");
        return !(e && e[0] == '0' && e[1] == 0);
    }();
    return on;
}

// HM_FP64_DMMA=1 puts every FP64 batch the warp-tiled kernel would run on the FP64 MMA
// kernel (tile-table entries choose it per batch through their tc flag otherwise).
static bool fp64_dmma_forced() {
    static const bool on = [] {
        const char* e = std::getenv("HM_FP64_DMMA");
        return e && e[0] == '1' && e[1] == 0;
    }();
    return on;
}

template <typename T>
void GemmBatch<T>::finalize(cudaStream_t s) {
    int t = 0;
    flops_ = bytes_ = 0;
    for (auto& d : h_) {
        d.tile0 = t;
        t += d.tiles_m * d.tiles_n * d.ksplit;
        flops_ += 2.0 * d.m * (double)d.n * d.k;
        const double a = (gen_ == GEN_DENSE) ? (double)d.m * d.k : 0.0;
        bytes_ += sizeof(T) * (a + (double)d.k * d.n + (double)d.m * d.n * (d.beta != T(0) ? 2 : 1));
    }
    total_tiles_ = t;
    {   // tuning signature
        int mmax = 0, nmax = 0;
        std::vector<int> ks;
        ks.reserve(h_.size());
        for (auto& d : h_) {
            mmax = std::max(mmax, d.m);
            nmax = std::max(nmax, d.n);
            ks.push_back(d.k);
        }
        int kmed = 0;
        if (!ks.empty()) {
            std::nth_element(ks.begin(), ks.begin() + ks.size() / 2, ks.end());
            kmed = ks[ks.size() / 2];
        }
        sig_ = tag_ + (sizeof(T) == 4 ? "|f32" : "|f64") + "|p" + std::to_string(pow2_ceil((long long)h_.size())) +
               "|m" + std::to_string(pow2_ceil(mmax)) + "|n" + std::to_string(ceil_div(nmax, 32) * 32) + "|k" +
               std::to_string(pow2_ceil(kmed));
    }
    // dense batches run the warp-tiled kernel: tile counts for its shape in a device-side
    // copy of the table (BN fitted to the widest problem: ranks are usually <= 96)
    pipe_bn_ = 0;
    if (gen_ == GEN_DENSE && cfg_ == CFG_64x64 && !h_.empty()) {
        bool any_scale = false;
        int nmax = 0;
        for (auto& d : h_) {
            any_scale |= d.kscale != nullptr;
            nmax = std::max(nmax, d.n);
        }
        if (!any_scale) pipe_bn_ = nmax <= 32 ? 32 : nmax <= 64 ? 64 : nmax <= 96 ? 96 : 128;
    }
    // generated-operand batches (matrix-free sketches: n = sketch width, ~100): 128-wide
    // tiles so each generated entry of A feeds the whole width once
    gen_wide_ = false;
    if (gen_ != GEN_DENSE && cfg_ == CFG_64x64 && !h_.empty()) {
        int nmax = 0;
        for (auto& d : h_) nmax = std::max(nmax, d.n);
        if (nmax > 64) {
            gen_wide_ = true;
            int tt = 0;
            for (auto& d : h_) {
                d.tiles_m = ceil_div(d.m, 64);
                d.tiles_n = ceil_div(d.n, 128);
                d.tile0 = tt;
                tt += d.tiles_m * d.tiles_n * d.ksplit;
            }
            total_tiles_ = tt;
        }
    }
    TileChoice tuned;
    const bool have_tuned = pipe_bn_ && tile_choice(sig_, tuned);
    if (have_tuned) pipe_bn_ = tuned.bn;
    // FP64 batches: the FP64 MMA kernel when the table's tc flag or HM_FP64_DMMA asks
    use_dmma_ = std::is_same<T, double>::value && pipe_bn_ && (fp64_dmma_forced() || (have_tuned && tuned.tc));
    if (kernel_mode_ == 1) use_dmma_ = std::is_same<T, double>::value && pipe_bn_;
    if (kernel_mode_ == 2) use_dmma_ = false;
    if (pipe_bn_) {
        // 64-row tiles when the batch's problems are short enough that 128-row (or
        // 256-row) tiles would pad more than a quarter of the rows
        const int big = tile::bm_for(sizeof(T), pipe_bn_);
        double rows = 0, pad_big = 0, pad_small = 0;
        for (auto& d : h_) {
            rows += d.m;
            pad_big += (double)ceil_div(d.m, big) * big - d.m;
            pad_small += (double)ceil_div(d.m, 64) * 64 - d.m;
        }
        pipe_shape_ = have_tuned ? tuned.small : (big > 64 && pad_big > 0.25 * rows && pad_small < pad_big ? 1 : 0);
        if (!have_tuned && pipe_shape_ == 0 && fp64_big_forced()) pipe_shape_ = 2;
        pipe_shape_ = tile::shape_for(sizeof(T), pipe_shape_);
        if (use_dmma_ || (has_chains_ && pipe_shape_ == 3)) pipe_shape_ = 0;   // no 96-row chain kernel
        if (!use_dmma_ && !has_chains_ && pipe_shape_ != 3 && pipe_bn_ <= 64 && tile96_enabled() &&
            !forced_choice()) {
            const int bmc = tile::bm_for(sizeof(T), pipe_bn_, pipe_shape_);
            bool all96 = true, pads = false;
            for (auto& d : h_) {
                all96 &= d.m % 96 == 0;
                pads |= d.m % bmc != 0;
            }
            if (all96 && pads) pipe_shape_ = 3;
        }
        const int BM = use_dmma_ ? dmma::bm_for(pipe_bn_) : tile::bm_for(sizeof(T), pipe_bn_, pipe_shape_);
        std::vector<GemmDesc<T>> dv(h_);
        int tt = 0;
        for (auto& d : dv) {
            d.tiles_m = d.is_link ? 0 : ceil_div(d.m, BM);
            d.tiles_n = d.is_link ? 0 : ceil_div(d.n, pipe_bn_);
            d.tile0 = tt;
            tt += d.tiles_m * d.tiles_n * d.ksplit;
        }
        pipe_tiles_ = tt;
        std::vector<int> tp((size_t)tt);
        for (size_t i = 0; i < dv.size(); ++i) {
            const auto& d = dv[i];
            std::fill(tp.begin() + d.tile0, tp.begin() + d.tile0 + d.tiles_m * d.tiles_n * d.ksplit, (int)i);
        }
        d_.alloc(dv.size());
        tmap_.alloc(std::max<size_t>(tp.size(), 1));
        HM_CUDA(cudaMemcpyAsync(d_.p, dv.data(), dv.size() * sizeof(GemmDesc<T>), cudaMemcpyHostToDevice, s));
        if (!tp.empty())
            HM_CUDA(cudaMemcpyAsync(tmap_.p, tp.data(), tp.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        HM_CUDA(cudaStreamSynchronize(s));  // dv and tp are local vectors
    } else if (!h_.empty()) {
        HM_CHECK(!has_chains_, HM_ERR_STATE, "chained GEMM problems need the warp-tiled kernel");
        d_.alloc(h_.size());
        HM_CUDA(cudaMemcpyAsync(d_.p, h_.data(), h_.size() * sizeof(GemmDesc<T>),
                                cudaMemcpyHostToDevice, s));
    }
    use_tc_ = false;
    if constexpr (std::is_same<T, float>::value) {
        if (kernel_mode_ == 1) {
            HM_CHECK(pipe_bn_ && !has_chains_, HM_ERR_UNSUPPORTED, "tensor-core GEMM: batch not eligible");
            finalize_tc(s, true);
            HM_CHECK(use_tc_, HM_ERR_UNSUPPORTED,
                     "tensor-core GEMM: operands not TMA-addressable (16-byte aligned, ld a multiple of 4)");
        } else if (kernel_mode_ == 0 && pipe_bn_ && tc_allowed_ && !has_chains_ && (!have_tuned || tuned.tc)) {
            finalize_tc(s, tc_any_k_);
        }
        gen_tc_ = false;
        if (gen_ != GEN_DENSE && cfg_ == CFG_64x64 && tc_allowed_ && kernel_mode_ != 2 && !h_.empty())
            finalize_tc_gen(s);
    }
    if (!hz_.empty()) {
        dz_.alloc(hz_.size());
        HM_CUDA(cudaMemcpyAsync(dz_.p, hz_.data(), hz_.size() * sizeof(ZeroRegion<T>),
                                cudaMemcpyHostToDevice, s));
    }
    // the host vectors must outlive the async copies: keep them
    finalized_ = true;
}

// FP32 batches whose tiles average at least 4 k-blocks of 32 (k >= 128) and whose
// operands the TMA can address run on the tensor cores (3xTF32); short-k batches keep
// the FMA kernel, which is as fast there.
template <typename T>
void GemmBatch<T>::finalize_tc(cudaStream_t s, bool force) {
    if constexpr (std::is_same<T, float>::value) {
        std::vector<GemmDesc<float>> dv(h_);
        long long kblocks = 0;
        int tt = 0;
        static const bool dbg = std::getenv("HM_TC_DEBUG") != nullptr;
        for (auto& d : dv) {
            if (!tc::tma_ok(d)) {
                if (dbg)
                    fprintf(stderr, "[tc] %s: operand not TMA-addressable (A%%16=%d B%%16=%d lda=%d ldb=%d)\n",
                            tag_.c_str(), (int)(reinterpret_cast<uintptr_t>(d.A) & 15),
                            (int)(reinterpret_cast<uintptr_t>(d.B) & 15), d.lda, d.ldb);
                return;
            }
            d.tiles_m = ceil_div(d.m, tc::BM);
            d.tiles_n = ceil_div(d.n, pipe_bn_);
            d.tile0 = tt;
            const int tiles = d.tiles_m * d.tiles_n * d.ksplit;
            tt += tiles;
            kblocks += (long long)d.tiles_m * d.tiles_n * ceil_div(std::max(d.k, 1), tc::BK);
        }
        if (tt == 0 || (!force && kblocks < 4LL * tt)) return;
        std::vector<CUtensorMap> maps;
        if (!tc::encode_maps(dv, pipe_bn_, maps)) {
            if (dbg) fprintf(stderr, "[tc] %s: tensor-map encoding refused\n", tag_.c_str());
            return;
        }
        std::vector<int> tp((size_t)tt);
        for (size_t i = 0; i < dv.size(); ++i)
            std::fill(tp.begin() + dv[i].tile0, tp.begin() + dv[i].tile0 + dv[i].tiles_m * dv[i].tiles_n * dv[i].ksplit,
                      (int)i);
        tcd_.alloc(dv.size());
        tct_.alloc(tp.size());
        tcmaps_.alloc(maps.size() * sizeof(CUtensorMap));
        tcstatus_.alloc(1);
        tcstatus_.zero(s);
        HM_CUDA(cudaMemcpyAsync(tcd_.p, dv.data(), dv.size() * sizeof(GemmDesc<float>), cudaMemcpyHostToDevice, s));
        HM_CUDA(cudaMemcpyAsync(tct_.p, tp.data(), tp.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        HM_CUDA(cudaMemcpyAsync(tcmaps_.p, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s));
        HM_CUDA(cudaStreamSynchronize(s));   // the host vectors are locals
        tc_tiles_ = tt;
        // at most 4 k-blocks per tile on average: the epilogue bounds the tile rate, so
        // it gets twice the warps
        tc_epw_ = kblocks <= 4LL * tt ? 8 : 4;
        use_tc_ = true;
    }
}

template <typename T>
void GemmBatch<T>::finalize_tc_gen(cudaStream_t s) {
    if constexpr (std::is_same<T, float>::value) {
        static const bool dbg = std::getenv("HM_TC_DEBUG") != nullptr;
        int nmax = 0;
        for (auto& d : h_) nmax = std::max(nmax, d.n);
        if (nmax > 128) return;
        const int bn = nmax <= 32 ? 32 : nmax <= 64 ? 64 : nmax <= 96 ? 96 : 128;
        std::vector<GemmDesc<float>> dv(h_);
        int tt = 0;
        for (auto& d : dv) {
            if (!tc::tma_ok(d, true)) {
                if (dbg) fprintf(stderr, "[tc] %s: sketch operand not TMA-addressable (ldb=%d)\n", tag_.c_str(), d.ldb);
                return;
            }
            d.tiles_m = ceil_div(d.m, tc::BM);
            d.tiles_n = ceil_div(d.n, bn);
            d.tile0 = tt;
            tt += d.tiles_m * d.tiles_n * d.ksplit;
        }
        if (tt == 0) return;
        std::vector<CUtensorMap> maps;
        if (!tc::encode_maps(dv, bn, maps, true)) {
            if (dbg) fprintf(stderr, "[tc] %s: tensor-map encoding refused\n", tag_.c_str());
            return;
        }
        std::vector<int> tp((size_t)tt);
        for (size_t i = 0; i < dv.size(); ++i)
            std::fill(tp.begin() + dv[i].tile0, tp.begin() + dv[i].tile0 + dv[i].tiles_m * dv[i].tiles_n * dv[i].ksplit,
                      (int)i);
        tcd_.alloc(dv.size());
        tct_.alloc(tp.size());
        tcmaps_.alloc(maps.size() * sizeof(CUtensorMap));
        tcstatus_.alloc(1);
        tcstatus_.zero(s);
        HM_CUDA(cudaMemcpyAsync(tcd_.p, dv.data(), dv.size() * sizeof(GemmDesc<float>), cudaMemcpyHostToDevice, s));
        HM_CUDA(cudaMemcpyAsync(tct_.p, tp.data(), tp.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        HM_CUDA(cudaMemcpyAsync(tcmaps_.p, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s));
        HM_CUDA(cudaStreamSynchronize(s));   // the host vectors are locals
        tc_tiles_ = tt;
        gen_bn_ = bn;
        gen_tc_ = true;
        use_tc_ = true;
    }
}

template <int GEN>
static void launch_tc_gen(int bn, int tiles, int sms, cudaStream_t s, const GemmDesc<float>* d, const int* tp,
                          const CUtensorMap* maps, int* st, int stall, const GenParams& gp) {
    // the entry generation in the converter warps bounds these: 12 of them
    if (bn == 32) tc::launch<32, GEN, 4, 12>(tiles, sms, s, d, tp, maps, st, stall, gp);
    else if (bn == 64) tc::launch<64, GEN, 4, 12>(tiles, sms, s, d, tp, maps, st, stall, gp);
    else if (bn == 96) tc::launch<96, GEN, 4, 12>(tiles, sms, s, d, tp, maps, st, stall, gp);
    else tc::launch<128, GEN, 4, 12>(tiles, sms, s, d, tp, maps, st, stall, gp);
}

static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        HM_CUDA(cudaGetDevice(&dev));
        HM_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    }
    return n;
}

template <typename T>
void GemmBatch<T>::clear() {
    h_.clear();
    hz_.clear();
    d_.release();
    dz_.release();
    tmap_.release();
    tcd_.release();
    tct_.release();
    tcmaps_.release();
    use_tc_ = false;
    gen_tc_ = false;
    total_tiles_ = 0;
    finalized_ = false;
}

template <typename T, int BM, int BN, int BK, int TM, int TN>
static void launch_gen(int gen, int grid, cudaStream_t s, const GemmDesc<T>* d, int nd,
                       const GenParams& gp) {
    constexpr int NT = (BM / TM) * (BN / TN);
    switch (gen) {
        case GEN_CAUCHY:
            gemm_batched_kernel<T, BM, BN, BK, TM, TN, GEN_CAUCHY><<<grid, NT, 0, s>>>(d, nd, gp);
            break;
        case GEN_GAUSSIAN:
            gemm_batched_kernel<T, BM, BN, BK, TM, TN, GEN_GAUSSIAN><<<grid, NT, 0, s>>>(d, nd, gp);
            break;
        case GEN_COULOMB:
            gemm_batched_kernel<T, BM, BN, BK, TM, TN, GEN_COULOMB><<<grid, NT, 0, s>>>(d, nd, gp);
            break;
        default:
            gemm_batched_kernel<T, BM, BN, BK, TM, TN, GEN_DENSE><<<grid, NT, 0, s>>>(d, nd, gp);
    }
}

// warp-tiled kernel for tile width bn and shape SHAPE (SHAPE 2 exists for FP64 only)
template <typename T, int SHAPE, bool CHAIN>
static void launch_tile(int bn, int tiles, cudaStream_t s, const GemmDesc<T>* d, const int* tp) {
    if constexpr (SHAPE == 2 && !std::is_same<T, double>::value) {
        throw Error(HM_ERR_STATE, "FP64-only tile shape on an FP32 batch");
    } else {
        if (bn == 32) tile::launch<T, 32, SHAPE, CHAIN>(tiles, s, d, tp);
        else if (bn == 64) tile::launch<T, 64, SHAPE, CHAIN>(tiles, s, d, tp);
        else if (bn == 96) tile::launch<T, 96, SHAPE, CHAIN>(tiles, s, d, tp);
        else tile::launch<T, 128, SHAPE, CHAIN>(tiles, s, d, tp);
    }
}

template <typename T>
void GemmBatch<T>::launch(cudaStream_t s, const GenParams& gp, int* status) const {
    if (h_.empty()) return;
    HM_CHECK(finalized_, HM_ERR_STATE, "GemmBatch::launch before finalize");
    if (!hz_.empty())
        zero_regions_kernel<T><<<(int)hz_.size(), 256, 0, s>>>(dz_.p, (int)hz_.size());
    if constexpr (std::is_same<T, float>::value) {
        if (use_tc_) {
            const auto* maps = reinterpret_cast<const CUtensorMap*>(tcmaps_.p);
            int* st = status ? status : tcstatus_.p;
            const int sms = sm_count();
            if (gen_tc_) {
                const int stall = tc_stall_ ? 1 : 0;
                if (gen_ == GEN_CAUCHY) launch_tc_gen<GEN_CAUCHY>(gen_bn_, tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall, gp);
                else if (gen_ == GEN_GAUSSIAN) launch_tc_gen<GEN_GAUSSIAN>(gen_bn_, tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall, gp);
                else launch_tc_gen<GEN_COULOMB>(gen_bn_, tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall, gp);
                HM_CUDA(cudaGetLastError());
                return;
            }
            const int stall = tc_stall_ ? 1 : 0;
            if (tc_epw_ == 8) {
                if (pipe_bn_ == 32) tc::launch<32, GEN_DENSE, 8>(tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall);
                else if (pipe_bn_ == 64) tc::launch<64, GEN_DENSE, 8>(tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall);
                else if (pipe_bn_ == 96) tc::launch<96, GEN_DENSE, 8>(tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall);
                else tc::launch<128, GEN_DENSE, 8>(tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall);
            } else {
                if (pipe_bn_ == 32) tc::launch<32>(tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall);
                else if (pipe_bn_ == 64) tc::launch<64>(tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall);
                else if (pipe_bn_ == 96) tc::launch<96>(tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall);
                else tc::launch<128>(tc_tiles_, sms, s, tcd_.p, tct_.p, maps, st, stall);
            }
            HM_CUDA(cudaGetLastError());
            return;
        }
    }
    if constexpr (std::is_same<T, double>::value) {
        if (use_dmma_) {
            if (has_chains_) {
                if (pipe_bn_ == 32) dmma::launch<32, true>(pipe_tiles_, s, d_.p, tmap_.p);
                else if (pipe_bn_ == 64) dmma::launch<64, true>(pipe_tiles_, s, d_.p, tmap_.p);
                else if (pipe_bn_ == 96) dmma::launch<96, true>(pipe_tiles_, s, d_.p, tmap_.p);
                else dmma::launch<128, true>(pipe_tiles_, s, d_.p, tmap_.p);
            } else {
                if (pipe_bn_ == 32) dmma::launch<32, false>(pipe_tiles_, s, d_.p, tmap_.p);
                else if (pipe_bn_ == 64) dmma::launch<64, false>(pipe_tiles_, s, d_.p, tmap_.p);
                else if (pipe_bn_ == 96) dmma::launch<96, false>(pipe_tiles_, s, d_.p, tmap_.p);
                else dmma::launch<128, false>(pipe_tiles_, s, d_.p, tmap_.p);
            }
            HM_CUDA(cudaGetLastError());
            return;
        }
    }
    if (has_chains_) {   // chained batches (the FP64 matvec's leaf + expansion)
        if constexpr (std::is_same<T, double>::value) {
            if (pipe_shape_ == 2) launch_tile<T, 2, true>(pipe_bn_, pipe_tiles_, s, d_.p, tmap_.p);
            else if (pipe_shape_ == 1) launch_tile<T, 1, true>(pipe_bn_, pipe_tiles_, s, d_.p, tmap_.p);
            else launch_tile<T, 0, true>(pipe_bn_, pipe_tiles_, s, d_.p, tmap_.p);
            HM_CUDA(cudaGetLastError());
            return;
        }
        throw Error(HM_ERR_UNSUPPORTED, "chained GEMM problems are FP64 only");
    }
    if (pipe_bn_) {
        if (pipe_shape_ == 3) launch_tile<T, 3, false>(pipe_bn_, pipe_tiles_, s, d_.p, tmap_.p);
        else if (pipe_shape_ == 2) launch_tile<T, 2, false>(pipe_bn_, pipe_tiles_, s, d_.p, tmap_.p);
        else if (pipe_shape_ == 1) launch_tile<T, 1, false>(pipe_bn_, pipe_tiles_, s, d_.p, tmap_.p);
        else launch_tile<T, 0, false>(pipe_bn_, pipe_tiles_, s, d_.p, tmap_.p);
    }
    else if (gen_wide_)
        launch_gen<T, 64, 128, 8, 4, 8>(gen_, total_tiles_, s, d_.p, (int)h_.size(), gp);
    else if (cfg_ == CFG_N_SKINNY)
        launch_gen<T, 128, 16, 16, 4, 2>(gen_, total_tiles_, s, d_.p, (int)h_.size(), gp);
    else
        launch_gen<T, 64, 64, 16, 4, 4>(gen_, total_tiles_, s, d_.p, (int)h_.size(), gp);
    HM_CUDA(cudaGetLastError());
}

// Launch a batch whose descriptor and zeroing tables are already in device memory
// that the caller owns (tile offsets assigned as GemmBatch::packed() does).
void gemm_launch_tables(const GemmDesc<double>* dtab, int ndesc, int total_tiles,
                        const ZeroRegion<double>* dzero, int nzero, cudaStream_t s) {
    if (ndesc <= 0 || total_tiles <= 0) return;
    if (nzero > 0) zero_regions_kernel<double><<<nzero, 256, 0, s>>>(dzero, nzero);
    launch_gen<double, 64, 64, 16, 4, 4>(GEN_DENSE, total_tiles, s, dtab, ndesc, GenParams());
    HM_CUDA(cudaGetLastError());
}

template class GemmBatch<double>;
template class GemmBatch<float>;

}  // namespace hm
