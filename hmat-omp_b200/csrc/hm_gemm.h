// Variable-size batched GEMM: every node of a tree level (and every system of a
// batch) is one problem in a descriptor table; one launch covers the whole table.
//
//   C = alpha * op(A) * diag(kscale) * op(B) + beta * C
//
// op(X) is X or X^T of a column-major block with an explicit leading dimension.
// A may instead be generated on the fly from point coordinates (matrix-free kernel
// blocks).  Problems whose k is long and whose output is small are split along k
// ("split-K"); their partial products are added with atomics, so C must already
// hold beta*C (the batch zeroes C first when beta == 0).
#pragma once

#include <string>

#include "hm_common.h"

namespace hm {

enum : int { OP_N = 0, OP_T = 1 };

// Matrix-free A source.  Element (r, c) of the global N x N operator.
enum : int { GEN_DENSE = 0, GEN_CAUCHY = 1, GEN_GAUSSIAN = 2, GEN_COULOMB = 3 };

struct GenParams {
    const double* pts = nullptr;  // GEN_CAUCHY: x = pts[0:N], y = pts[N:2N]; else N x dim, point-major
    int N = 0;
    int dim = 1;
    double p0 = 0, p1 = 0;        // kernel parameters (see hmat_b200.h HM_KERNEL_*)
    // Batches of independent systems: row -> system, and per-system p0/p1 (override
    // p0/p1 when set).  Blocks never couple two systems.
    const int* row_sys = nullptr;
    const double* p0v = nullptr;
    const double* p1v = nullptr;
};

template <typename T>
struct ZeroRegion {
    T* C;
    int m, n, ldc;
};

template <typename T>
struct GemmDesc {
    const T* A;
    const T* B;
    T* C;
    const T* kscale;   // optional, length k
    T alpha, beta;
    int m, n, k;
    int lda, ldb, ldc;
    int opA, opB;
    int ksplit;
    int tiles_m, tiles_n;
    int tile0;         // first global tile index of this problem
    int ga_r0, ga_c0;  // generated A: origin of the block in the global operator
    // Chains (warp-tiled dense kernel only): a problem with next >= 0 is followed, in the
    // same CTA and register accumulators, by problem `next` (same m and n; its product is
    // added before the head's epilogue writes C).  Linked problems own no tiles.
    int next;
    int is_link;
};

// Materialise a block of a generated operator: dst(i,j) = trans ? G(r0+j, c0+i) : G(r0+i, c0+j)
struct GenFillDesc {
    int r0, c0, rows, cols, trans;
    double* dst;
    int ldd;
};
void launch_gen_fill(const GenFillDesc* d_descs, int count, int max_elems, int gen, const GenParams& gp,
                     cudaStream_t s);

// acc[0] += dL/dp0, acc[1] += dL/dp1 of the exact kernel operator, given x and
// lam = A^{-T} dL/dx (both N x s, ld N); dL/dA = -lam x^T.
void launch_param_grad(int gen, const GenParams& gp, const double* X, const double* L, int N, int s,
                       double* acc, cudaStream_t st);

template <typename T> struct GemmDesc;
template <typename T> struct ZeroRegion;
void gemm_launch_tables(const GemmDesc<double>* dtab, int ndesc, int total_tiles,
                        const ZeroRegion<double>* dzero, int nzero, cudaStream_t s);

// Tile configurations.
enum : int { CFG_64x64 = 0, CFG_N_SKINNY = 1 };

// Autotuned tile choices for the dense batched GEMM.  A batch is identified by its
// signature (step tag, element type and bucketed problem count / m / n / k, see
// GemmBatch::signature); the choice is the warp-tiled kernel's tile width BN, its shape
// (0 default, 1 64-row tiles, 2 8 x 8 outputs per lane, FP64 only), and tc: an eligible
// FP32 batch on the tcgen05 kernel, an FP64 batch on the FP64 MMA kernel.
// Sources, first match wins: HM_TILE_FORCE="bn,small,tc" (every batch; the offline
// sweep's switch), then the table in the JSON file HM_TILE_TABLE names, else
// tile_table.json beside the loaded library ({"signature": [bn, small, tc], ...},
// written by autotune.py).  Batches without an entry keep the built-in heuristics.
struct TileChoice {
    int bn = 0, small = 0, tc = 1;   // small: the shape (0 default, 1 64-row, 2 FP64 8 x 8, 3 96-row)
};
bool tile_choice(const std::string& sig, TileChoice& out);
// Replace the table with the one in `path` (an empty path clears it); false if the file
// cannot be read or parsed.
bool tile_table_load(const char* path);
int tile_table_size();

template <typename T>
class GemmBatch {
  public:
    explicit GemmBatch(int cfg = CFG_64x64, int gen = GEN_DENSE) : cfg_(cfg), gen_(gen) {}
    // Add C = alpha op(A) diag(kscale) op(B) + beta C.  ksplit <= 0 picks a split.
    void add(int m, int n, int k, T alpha, const T* A, int lda, int opA, const T* B, int ldb,
             int opB, T beta, T* C, int ldc, const T* kscale = nullptr, int ksplit = 0,
             int ga_r0 = 0, int ga_c0 = 0);
    // Add op(A) op(B) (m x n, same alpha) to the C tile of the last problem added with
    // add() (ksplit 1): the whole chain is accumulated in registers and C is written once.
    void add_chained(int m, int n, int k, T alpha, const T* A, int lda, int opA, const T* B, int ldb, int opB);
    bool empty() const { return h_.empty(); }
    size_t size() const { return h_.size(); }
    // step name used in the tuning signature
    void set_tag(const std::string& t) { tag_ = t; }
    // "<tag>|<f32|f64>|p<count>|m<max m>|n<max n>|k<median k>" (counts and m/k rounded up
    // to powers of two, n to multiples of 32); set by finalize
    const std::string& signature() const { return sig_; }
    // "bn,small,tc" as finalize chose it (bn 0: not the warp-tiled kernel)
    std::string choice() const;
    // Upload the table (once); later launches reuse it (and may be graph-captured).
    void finalize(cudaStream_t s);
    void finalize_tc(cudaStream_t s, bool force = false);
    // FP32 batches whose A is generated from a kernel: the tcgen05 kernel evaluates A's
    // entries into its stages (the TMA brings B only)
    void finalize_tc_gen(cudaStream_t s);
    bool on_tensor_cores() const { return use_tc_; }
    bool on_fp64_mma() const { return use_dmma_; }
    // Kernel selection for finalize: 0 the built-in rules and tile table; 1 the tensor-core
    // kernel (tcgen05 for FP32 -- finalize throws HM_ERR_UNSUPPORTED if the operands are
    // not TMA-addressable; the FP64 MMA kernel for FP64); 2 the warp-tiled FMA kernel.
    void set_kernel(int mode) { kernel_mode_ = mode; }
    // Test of the tensor-core kernel's timeout path: its producer issues no copies and its
    // role waits give up after ~0.5 ms, so the launch sets ST_TIMEOUT with nothing in flight.
    void set_test_stall(bool on) { tc_stall_ = on; }
    // whether finalize may put this (FP32) batch on the tensor cores
    // any_k: also when the inner dimension is short (fewer than 4 k-blocks per tile)
    void allow_tensor_cores(bool on, bool any_k = false) {
        tc_allowed_ = on;
        tc_any_k_ = any_k;
    }
    // status: device status word for the tensor-core kernel's bounded waits (may be null
    // for batches that never take that kernel)
    void launch(cudaStream_t s, const GenParams& gp = GenParams(), int* status = nullptr) const;
    void clear();
    int cfg() const { return cfg_; }
    int gen() const { return gen_; }
    // Descriptors with tile offsets assigned (total tile count in *tiles), and the
    // split-K zeroing regions: for launching from tables the caller places itself.
    std::vector<GemmDesc<T>> packed(int* tiles) const {
        std::vector<GemmDesc<T>> out(h_);
        int t = 0;
        for (auto& d : out) {
            d.tile0 = t;
            t += d.tiles_m * d.tiles_n * d.ksplit;
        }
        *tiles = t;
        return out;
    }
    const std::vector<ZeroRegion<T>>& zero_regions() const { return hz_; }
    int nlaunch() const { return h_.empty() ? 0 : (hz_.empty() ? 1 : 2); }
    // algorithmic work of one launch: 2mnk flops; operand and result bytes
    double flops() const { return flops_; }
    double bytes() const { return bytes_; }

  private:
    int cfg_, gen_;
    std::string tag_, sig_;
    std::vector<GemmDesc<T>> h_;
    int chain_head_ = -1, chain_tail_ = -1;
    bool has_chains_ = false;
    DBuf<GemmDesc<T>> d_;
    // regions to zero before a split-K launch
    std::vector<ZeroRegion<T>> hz_;
    DBuf<ZeroRegion<T>> dz_;
    int total_tiles_ = 0;
    bool finalized_ = false;
    double flops_ = 0, bytes_ = 0;
    int pipe_bn_ = 0, pipe_tiles_ = 0;   // warp-tiled dense kernel: tile width and tile count
    int pipe_shape_ = 0;                 // its shape: 0 default, 1 64-row tiles, 2 8 x 8 per lane (FP64)
    bool gen_wide_ = false;              // generated-A batch on 64 x 128 tiles
    bool use_dmma_ = false;              // FP64 batch on the FP64 MMA kernel (same tables)
    DBuf<int> tmap_;                     // its tile -> problem table
    // FP32 batches with long k on the tensor cores: tile count, tables, tensor maps
    bool use_tc_ = false, tc_allowed_ = true, tc_stall_ = false, tc_any_k_ = false;
    int kernel_mode_ = 0;
    bool gen_tc_ = false;   // generated-A batch on the tensor cores
    int gen_bn_ = 0;        // its tile width
    int tc_tiles_ = 0;
    int tc_epw_ = 4;   // epilogue warps of the tensor-core kernel (8 for short-k batches)
    DBuf<GemmDesc<T>> tcd_;
    DBuf<int> tct_;
    DBuf<unsigned char> tcmaps_;
    DBuf<int> tcstatus_;
};

}  // namespace hm
