/* hmat_b200.h — C ABI of the B200 hierarchical-matrix library (libhmat_b200.so).
 *
 * The reference (chenxinye/hmat-omp) is a header-only C++ library whose callers use
 * four classes — HODLRMatrix[OMP] and HSSMatrix[OMP] — with the same three methods:
 *   ctor(double tol)                          include/hodlr_routines.h:16, hss_routines.h:18
 *   void build_from_dense(const Matrix&, int) include/hodlr_routines.h:20, hss_routines.h:50
 *   Matrix multiply(const Matrix& x)          include/hodlr_routines.h:66, hss_routines.h:118
 *   Matrix solve(const Matrix& b)             include/hodlr_routines.h:108, hss_routines.h:197
 * and the public fields root/nodes/N/tolerance/rsvd_rank (hodlr_routines.h:10-14).
 * Each entry point below names the reference interface it replaces.  Matrices are
 * column-major FP64 with an explicit leading dimension, as Matrix stores them
 * (include/matrix.h:36).  Every function returns an HM_* status; 0 is success and
 * hm_last_error() holds the message of the last failure on a handle.
 *
 * Device work runs on the handle's CUDA stream (hm_set_stream).  Host-buffer entry
 * points copy in and out and return when the result is on the host.  Calls on one
 * handle must not overlap; different handles may be used from different threads.
 */
#ifndef HMAT_B200_H
#define HMAT_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define HM_API __attribute__((visibility("default")))
#else
#define HM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
enum {
    HM_OK = 0,
    HM_ERR_ARG = 1,          /* invalid argument (shape, pointer, option) */
    HM_ERR_CUDA = 2,         /* CUDA runtime error */
    HM_ERR_SINGULAR = 3,     /* zero or non-finite pivot in a leaf or capacitance inverse */
    HM_ERR_NO_CONVERGE = 4,  /* a Jacobi eigen/SVD iteration hit its sweep limit */
    HM_ERR_NONFINITE = 5,    /* non-finite input or result */
    HM_ERR_STATE = 6,        /* call out of order (e.g. solve before build) */
    HM_ERR_UNSUPPORTED = 7,  /* size or option outside what this build supports */
    HM_ERR_IR = 8,           /* iterative refinement did not reach ir_tol */
    HM_ERR_TIMEOUT = 9       /* a device-side wait of a kernel's own pipeline gave up (bounded waits) */
};

/* ---- sketch sources for the randomized SVD (compression.h:78) ---- */
enum {
    HM_SKETCH_REFERENCE_UNIFORM = 0, /* std::mt19937(seed) + uniform_real_distribution<double>(0,1),
                                        drawn on the host in the reference's serial build order
                                        (Matrix::Random, matrix.h:50-57): bit-identical sketches */
    HM_SKETCH_REFERENCE_NORMAL = 1,  /* same stream through normal_distribution<double>(0,1) */
    HM_SKETCH_DEVICE_NORMAL = 2      /* N(0,1) from a counter-based generator on the device */
};

enum { HM_FP64 = 0, HM_MIXED = 1 };

/* Matrix-free kernel generators (hm_hodlr_build_from_kernel). */
enum {
    HM_KERNEL_CAUCHY = 1,   /* A_ij = 1/(x_i - y_j) + p0*delta_ij; rows x = pts[0:N], cols y = pts[N:2N] */
    HM_KERNEL_GAUSSIAN = 2, /* A_ij = exp(-|p_i - p_j|^2 / (2 p0^2)) + p1*delta_ij */
    HM_KERNEL_COULOMB = 3   /* A_ij = 1/(|p_i - p_j| + p0) + p1*delta_ij */
};

typedef struct hm_opts {
    double tol;          /* truncation tolerance: HODLRMatrix(tol) (hodlr_routines.h:16) */
    int rsvd_rank;       /* rank guess, public field rsvd_rank = 64 (hodlr_routines.h:16) */
    int oversample;      /* k = rsvd_rank + oversample (compression.h:74: 10) */
    int rsvd_min_dim;    /* blocks with m or n below this use a full SVD (compression.h:72: 256) */
    int power_iters;     /* extension (0 = reference behaviour) */
    int max_rank;        /* extension: cap on every block rank (0 = no cap, the reference) */
    int sketch;          /* HM_SKETCH_* */
    unsigned long long seed;
    int precision;       /* HM_FP64, or HM_MIXED (FP32 bulk + FP64 LUs + FP64-residual refinement) */
    double ir_tol;       /* HM_MIXED: target max_j ||b_j - A x_j|| / ||b_j|| */
    int ir_max_iter;     /* HM_MIXED: refinement iteration limit */
    int refine_steps;    /* HM_FP64: steps of x += A^{-1}(b - A x) with the same factors after the
                            direct solve (0 = the reference's single solve); restores the backward
                            error of ill-conditioned operators */
} hm_opts;

typedef struct hm_handle hm_handle;

typedef struct hm_solve_stats {
    int ir_iters;          /* refinement iterations taken (0 in FP64 mode) */
    double rel_residual;   /* max_j ||b_j - A~ x_j|| / ||b_j|| against the FP64 compressed operator
                              (computed in HM_MIXED mode; -1 when not computed) */
} hm_solve_stats;

/* Defaults mirror the reference: tol 1e-6, rsvd_rank 64, oversample 10, min dim 256,
 * no power iteration, no rank cap, reference uniform sketch with seed 0, FP64. */
HM_API void hm_opts_default(hm_opts* o);

/* Replaces the constructors HODLRMatrix(tol) / HSSMatrix(tol) (hodlr_routines.h:16,
 * hss_routines.h:18): options, stream and device memory live in the handle. */
HM_API int hm_create(const hm_opts* o, hm_handle** out);
/* Replaces ~HODLRMatrix / ~HSSMatrix (hodlr_routines.h:17, hss_routines.h:19). */
HM_API int hm_destroy(hm_handle* h);
HM_API const char* hm_last_error(const hm_handle* h);
/* Work is enqueued on `stream` (a cudaStream_t); NULL = the handle's own stream. */
HM_API int hm_set_stream(hm_handle* h, void* stream);

/* Switch the factor/solve precision of an existing operator (HM_FP64 or HM_MIXED); the
 * next solve refactors.  No counterpart in the reference (FP64 only). */
HM_API int hm_set_precision(hm_handle* h, int precision);

/* HODLRMatrix::build_from_dense(A, leaf_size) (hodlr_routines.h:20-63): tree split
 * mid=(s+e)/2, leaf iff len <= leaf; A12 -> (left.U, right.V, B_12), A21 -> (right.U,
 * left.V, B_21) by compress_rsvd (compression.h:67-99).  A: host, N x N, column-major. */
HM_API int hm_hodlr_build_from_dense(hm_handle* h, const double* A, int N, int lda, int leaf_size);
/* Same, with A already in device memory. */
HM_API int hm_hodlr_build_from_dense_device(hm_handle* h, const double* dA, int N, int lda, int leaf_size);

/* Matrix-free counterpart of build_from_dense for operators given by a kernel on
 * points (the reference fills a dense A from include/kernel.h:30-89 and compresses its
 * blocks; here the blocks' entries are evaluated on the device where the sketch GEMMs
 * consume them, so A is never stored).  points (host): Cauchy: x[0:N] then y[0:N]
 * (dim 1); Gaussian/Coulomb: N x dim, point-major.  params[0..1] = p0, p1 of the
 * HM_KERNEL_* formula.  Same tree, compression rules and sketch stream as
 * hm_hodlr_build_from_dense. */
HM_API int hm_hodlr_build_from_kernel(hm_handle* h, int kernel, const double* points, int dim, int N,
                                      const double* params, int nparams, int leaf_size);

/* HSSMatrix::build_from_dense(A, leaf_size) (hss_routines.h:50-113): build_topo ids,
 * leaf row/column bases of the off-diagonal strips, identity transfers, dense B — the
 * factors hm_export_tree / hm_get_factor return.  Multiply, factor and solve run on the
 * same operator with each coupling block recompressed to its numerical rank (singular
 * values above 1e-15 of the largest), which keeps the Woodbury capacitance systems small
 * and the solve accurate. */
HM_API int hm_hss_build_from_dense(hm_handle* h, const double* A, int N, int lda, int leaf_size);
/* Matrix-free counterpart of HSSMatrix::build_from_dense (hss_routines.h:50-113): the
 * leaf strips and coupling blocks are evaluated from the kernel on the device (same
 * points/params layout as hm_hodlr_build_from_kernel), so A is never stored.  Same
 * tree, ranks and sketch stream as hm_hss_build_from_dense on the matrix the kernel
 * defines. */
HM_API int hm_hss_build_from_kernel(hm_handle* h, int kernel, const double* points, int dim, int N,
                                    const double* params, int nparams, int leaf_size);

/* Nested-basis HSS (no counterpart: the reference's transfers are identities,
 * hss_routines.h:86-90).  nested != 0 makes the next hm_hss_build_from_dense /
 * hm_hss_build_from_kernel on this handle keep the leaf bases of the reference form and
 * compress every internal node's off-diagonal strip onto its children's bases:
 * U_t = diag(U_left, U_right) R_t, V_t = diag(V_left, V_right) W_t, with R_t / W_t the
 * leading singular vectors of the projected strips, truncated by the rule every other
 * block uses (#{s > tol s_0}, at least 1, capped by max_rank).  Ranks then stay at the
 * numerical rank of each strip instead of growing with the number of leaves below.
 * hm_export_tree returns the nested ranks (0 at the root); hm_get_factor returns the
 * leaf U / V, R (rank_U(left) + rank_U(right)) x rank_U, W likewise, and B at the nested
 * ranks.  Multiply, factor and solve run on the same operator; hm_save / hm_load keep
 * the form.  nested = 0 restores the reference form.  hm_hss_is_nested: 1 when the
 * handle's current operator is a nested-basis HSS, else 0. */
HM_API int hm_hss_set_nested(hm_handle* h, int nested);
HM_API int hm_hss_is_nested(const hm_handle* h);

/* ---- serialized operators (no counterpart in the reference, which has no format) ----
 * hm_save writes the built operator (tree, leaf blocks, bases, coupling blocks; for HSS
 * also the reference-form leaf bases and B that hm_get_factor exports; for kernel builds
 * the kernel, its parameters and points) to one binary file; hm_load replaces the
 * handle's operator with the file's (HODLR or HSS as saved), ready to multiply, factor and
 * solve without recompressing.  Factorizations are not stored (the first solve factors).
 * The handle's options (precision, refinement) apply to the loaded operator.  Errors:
 * HM_ERR_STATE (save before build), HM_ERR_UNSUPPORTED (batches), HM_ERR_ARG (unreadable,
 * truncated or inconsistent file; a load that fails after the header leaves the handle
 * with no operator). */
HM_API int hm_save(hm_handle* h, const char* path);
HM_API int hm_load(hm_handle* h, const char* path);

/* Fix the kept rank of every compressed block for the next HODLR builds on this handle
 * (no counterpart in the reference, whose compress_rsvd truncates by tolerance,
 * compression.h:42-46): node i's B_12 / B_21 keep rank12[i] / rank21[i] singular triplets
 * (pre-order, as hm_export_tree lists them; capped by the sketch width, at least 1)
 * instead of #{S > tol S_0}.  A profile exported from one build and set before rebuilding
 * with perturbed kernel parameters gives an operator that is a smooth function of those
 * parameters (finite differences without re-truncation).  nnodes must equal the next
 * tree's node count (HM_ERR_ARG at build otherwise); NULL arrays or nnodes <= 0 clear it. */
HM_API int hm_set_rank_profile(hm_handle* h, int nnodes, const int* rank12, const int* rank21);

/* Upload a HODLR tree built elsewhere (e.g. by HODLRMatrix::build_from_dense) so the
 * device path can multiply/solve with exactly those factors.  Nodes in pre-order
 * (root, left subtree, right subtree); per node pointers to host column-major
 * blocks: D (leaf, len x len), U and V (non-root, len x rank from the parent's
 * compression), B12/B21 (internal, rank x rank).  NULL where the reference field is
 * empty.  ranks12/ranks21: B_12/B_21 sizes (0 for leaves). */
HM_API int hm_hodlr_import(hm_handle* h, int N, int leaf_size, const int* ranks12, const int* ranks21,
                    const double* const* D, const double* const* U, const double* const* V,
                    const double* const* B12, const double* const* B21);

/* Tree introspection, pre-order for HODLR (the reference's recursion order) and id
 * order for HSS (hss_routines.h:293-306).  rank12/rank21 are B_12/B_21 sizes for
 * HODLR and rank_U/rank_V for HSS. */
HM_API int hm_num_nodes(const hm_handle* h);
HM_API int hm_export_tree(const hm_handle* h, int* idx_start, int* idx_end, int* is_leaf, int* depth,
                   int* rank12, int* rank21);
/* Download one node's factor in the reference layout.  HODLR which: 0 D, 1 U, 2 V,
 * 3 B_12, 4 B_21 (utils.h:6-29).  HSS which: 0 D, 1 U, 2 V, 3 R, 4 W, 5 B (utils.h:32-55).
 * rows/cols receive the shape; out may be NULL to query the shape only. */
HM_API int hm_get_factor(const hm_handle* h, int node, int which, double* out, int* rows, int* cols);

/* multiply(x) (hodlr_routines.h:66-105, hss_routines.h:118-192) for nrhs columns. */
HM_API int hm_multiply(hm_handle* h, const double* x, int nrhs, int ldx, double* y, int ldy);
HM_API int hm_multiply_device(hm_handle* h, const double* dx, int nrhs, int ldx, double* dy, int ldy);

/* Factor once: leaf inverses and one Woodbury capacitance inverse per node, bottom-up
 * (the quantities the reference's solve recomputes on every call,
 * hodlr_routines.h:112-175, hss_routines.h:205-279).  solve() factors on demand. */
HM_API int hm_factor(hm_handle* h);

/* solve(b) (hodlr_routines.h:108-175, hss_routines.h:197-290) for nrhs columns. */
HM_API int hm_solve(hm_handle* h, const double* b, int nrhs, int ldb, double* x, int ldx,
             hm_solve_stats* stats);
HM_API int hm_solve_device(hm_handle* h, const double* db, int nrhs, int ldb, double* dx, int ldx,
                    hm_solve_stats* stats);

/* ---- many independent systems in shared launches (no counterpart in the reference,
 *      whose classes hold one operator each) ----
 * nsys HODLR operators, system k of size N[k] with kernel parameters
 * params[2k], params[2k+1] (p0, p1 of HM_KERNEL_GAUSSIAN / HM_KERNEL_COULOMB) on
 * points[sum_{j<k} N[j] .. +N[k]) (N x dim, point-major, concatenated).  Each system
 * gets the reference's tree and compression rules; every level of every system shares
 * one launch per step in the build, the factorization and the solve. */
HM_API int hm_batch_build_from_kernel(hm_handle* h, int kernel, const double* points, int dim, int nsys,
                                      const int* N, const double* params, int leaf_size);
HM_API int hm_num_systems(const hm_handle* h);
/* Packed right-hand sides (host or device): system k's N[k] x nrhs[k] column-major
 * block at offset sum_{j<k} N[j] nrhs[j]; nrhs[k] may be 0.  FP64; synchronises. */
HM_API int hm_batch_solve(hm_handle* h, const double* b, const int* nrhs, double* x);
HM_API int hm_batch_multiply(hm_handle* h, const double* x, const int* nrhs, double* y);

/* HODLRMatrix::solve(b) / HSSMatrix::solve(b) as the reference runs them: factor the
 * current operator, then solve (hodlr_routines.h:108-110 recomputes everything per call).
 * Here the factorization is recomputed and kept for later hm_solve calls; when b is in
 * host memory its copy to the device overlaps the factorization (page-locked b makes the
 * copy fully asynchronous).  Host or device b/x; synchronises before returning. */
HM_API int hm_factor_solve(hm_handle* h, const double* b, int nrhs, int ldb, double* x, int ldx,
                           hm_solve_stats* stats);

/* ---- exact-operator refinement (no counterpart in the reference) ----
 * For operators built by hm_*_build_from_kernel: solve A x = b with A the exact kernel
 * matrix, the compressed factorization serving as the preconditioner of an iterative
 * refinement x += A~^{-1}(b - A x) whose residual is computed with A's entries generated
 * on the device (2 N^2 nrhs flops per sweep; A is never stored).  Stops when
 * max_j ||b_j - A x_j|| / ||b_j|| <= tol (stats: sweeps, that residual) or returns
 * HM_ERR_IR after max_iter sweeps (x then holds the last iterate).  Each sweep contracts
 * the error by about ||A - A~|| ||A~^{-1}||: a few sweeps when the compression tolerance
 * times cond(A) is well below one.  HM_ERR_STATE for dense builds and batches.  Host or
 * device b/x; the _device form takes device pointers (it synchronises once per sweep to
 * read the residual norms). */
HM_API int hm_solve_exact(hm_handle* h, const double* b, int nrhs, int ldb, double* x, int ldx, double tol,
                          int max_iter, hm_solve_stats* stats);
HM_API int hm_solve_exact_device(hm_handle* h, const double* db, int nrhs, int ldb, double* dx, int ldx,
                                 double tol, int max_iter, hm_solve_stats* stats);

/* Krylov solve against the exact operator (no counterpart in the reference): flexible
 * GMRES(restart) for A x = b, A the exact kernel matrix of an operator built by
 * hm_*_build_from_kernel (entries generated on the device, A never stored), right-
 * preconditioned by the compressed factorization in the handle's precision; every column
 * runs its own Arnoldi process, all in shared launches.  Converges where hm_solve_exact's
 * stationary refinement diverges (compression error times ||A~^{-1}|| above one).  Stops
 * when max_j ||b_j - A x_j|| / ||b_j|| <= tol (stats: iterations, that residual) or returns
 * HM_ERR_IR after max_iter iterations (x holds the last iterate).  Host or device b/x;
 * synchronises. */
HM_API int hm_solve_gmres(hm_handle* h, const double* b, int nrhs, int ldb, double* x, int ldx, double tol,
                          int restart, int max_iter, hm_solve_stats* stats);

/* rel[j] = ||b_j - A x_j|| / ||b_j|| (j < nrhs, rel: host) with A the exact kernel matrix of an
 * operator built by hm_*_build_from_kernel, its entries generated on the device (2 N^2 nrhs
 * flops; A is never stored): the error of any solution against the exact operator rather
 * than the compressed one.  The reference's drivers print this quantity against their dense
 * A (main_hodlr.cpp:26-35).  Host or device b/x; synchronises. */
HM_API int hm_residual_exact(hm_handle* h, const double* b, int nrhs, int ldb, const double* x, int ldx,
                             double* rel);

/* ---- adjoint (no counterpart in the reference) ----
 * A^T lam = g with the FP64 factorization run transposed in reverse level order
 * (the transpose of the Woodbury recursion of hodlr_routines.h:112-175); factors in FP64
 * on demand.  Host or device g/lam; the _device form does not synchronise. */
HM_API int hm_solve_transpose(hm_handle* h, const double* g, int nrhs, int ldg, double* lam, int ldl);
HM_API int hm_solve_transpose_device(hm_handle* h, const double* dg, int nrhs, int ldg, double* dlam, int ldl);
/* Gradients of a loss L through x = A^{-1} b given x and lam = A^{-T} dL/dx (so dL/db = lam
 * and dL/dA = -lam x^T), accumulated into the factors of the HODLR representation
 * (leaf D, U, V, B_12, B_21; read with hm_get_gradient, same selectors as
 * hm_get_factor) and, for operators built by hm_hodlr_build_from_kernel, dparams[0..1] =
 * dL/dp0, dL/dp1 of the exact kernel (Gaussian: p0 = length-scale h; NaN for dense
 * builds).  dparams may be NULL. */
HM_API int hm_gradients(hm_handle* h, const double* x, int ldx, const double* lam, int ldl, int nrhs,
                        double* dparams);
HM_API int hm_get_gradient(const hm_handle* h, int node, int which, double* out, int* rows, int* cols);

/* multiply(x) like hm_multiply_device, but allocating no device memory: for callers
 * that may not call cudaMalloc when they multiply (a real-time or callback thread that
 * must not block in the device allocator, an application that owns all device memory
 * through its own pool).  No counterpart in the reference.  Intermediates and launch
 * tables live in one fixed 32 MiB device array that every GPU loading the library
 * keeps until exit; operators needing more fail with HM_ERR_UNSUPPORTED.  The operator's
 * device must be current (HM_ERR_ARG otherwise); the first call on a device looks up
 * that array's device address.  All calls share the array: calls whose work overlaps on
 * the GPU race.  Each call copies its launch tables from host memory, which waits for
 * the work already queued on the stream.  dx/dy: device, N x nrhs, column-major, on the
 * handle's stream. */
HM_API int hm_multiply_device_noalloc(hm_handle* h, const double* dx, int nrhs, int ldx, double* dy,
                                      int ldy);

/* ---- dense building blocks on the device ----
 * Kernel choice for the batched GEMMs. */
enum {
    HM_GEMM_AUTO = 0,          /* the library's own rules (tile table, tensor-core eligibility) */
    HM_GEMM_TENSOR_CORES = 1,  /* FP32: the tcgen05 kernel (TF32 hi/lo split, FP32 accumulation);
                                  FP64: the FP64 MMA kernel.  HM_ERR_UNSUPPORTED when the operands
                                  are not 16-byte aligned with leading dimensions a multiple of 4 */
    HM_GEMM_FMA = 2,           /* the warp-tiled FMA kernel */
    HM_GEMM_TEST_STALL = 16    /* or-ed with HM_GEMM_TENSOR_CORES (FP32): exercises the timeout path.
                                  The kernel's producer issues no copy, so its pipeline waits run out
                                  (after ~0.5 ms) with nothing in flight and the call returns
                                  HM_ERR_TIMEOUT; C is left unspecified.  For tests. */
};
/* Matrix::operator* (matrix.h:93-104: C = A * B through dgemm_) for `count` independent
 * products in one launch: C_i = alpha op(A_i) op(B_i) + beta C_i, C_i m_i x n_i, inner
 * dimension k_i, op = transpose when opA / opB is 1.  Size and pointer arrays are host
 * memory; the matrices are device memory, column-major.  ksplit: 0 lets the library split
 * long inner dimensions across CTAs (partial products added atomically; only when beta is
 * 0 or 1), 1 keeps one CTA per output tile.  Runs on the handle's stream; synchronises. */
HM_API int hm_gemm_batched_f32_device(hm_handle* h, int count, const int* m, const int* n, const int* k,
                                      float alpha, const float* const* A, const int* lda, int opA,
                                      const float* const* B, const int* ldb, int opB, float beta,
                                      float* const* C, const int* ldc, int ksplit, int flags);
HM_API int hm_gemm_batched_f64_device(hm_handle* h, int count, const int* m, const int* n, const int* k,
                                      double alpha, const double* const* A, const int* lda, int opA,
                                      const double* const* B, const int* ldb, int opB, double beta,
                                      double* const* C, const int* ldc, int ksplit, int flags);
/* Matrix::inverse (matrix.h:133-149: getrf + getri) for `count` square FP64 device matrices:
 * X_i = inv(A_i), n_i <= 16384, with partial pivoting at every size (Gauss-Jordan up to 64,
 * block Gauss-Jordan with panel pivoting above).  X may alias A.  HM_ERR_SINGULAR when a
 * pivot is zero or non-finite.  Runs on the handle's stream; synchronises. */
HM_API int hm_inverse_batched_device(hm_handle* h, int count, const int* n, const double* const* A,
                                     const int* lda, double* const* X, const int* ldx);
/* Y = A[r0:r1, c0:c1] X (trans 0) or Y = A[r0:r1, c0:c1]^T X (trans 1) for a kernel matrix
 * A generated on the device from `points` (the layout and kernels of
 * hm_hodlr_build_from_kernel; params p0, p1), entries never stored: FP64, 2 m k nrhs
 * flops.  The product a rank needs to compress its rows of a coupling block without
 * forming it (the sharded build of hmat_shard.build_top_sharded; the reference forms its
 * blocks densely, compression.h:77-87).  X (k x nrhs, ld ldx) and Y (m x nrhs, ld ldy) are
 * device memory, column-major, with m = r1 - r0 and k = c1 - c0 (swapped for trans).
 * Runs on the handle's stream; synchronises. */
HM_API int hm_kernel_block_product_device(hm_handle* h, int kernel, const double* points, int dim, int N,
                                          const double* params, int nparams, int r0, int r1, int c0, int c1,
                                          int trans, const double* dX, int ldx, int nrhs, double* dY, int ldy);

/* ---- instrumentation (no counterpart in the reference, which only wall-clocks its
 *      drivers: main_hodlr.cpp:14-24) ---- */
/* Count of kernels this library has launched in the process (always on). */
HM_API long long hm_launch_count(void);
/* Turn per-step CUDA-event timing on/off (clears recorded steps). */
HM_API void hm_profile_enable(int on);
/* JSON {"step": [launches, ms, algorithmic flops, algorithmic bytes], ...} of the steps
 * recorded since hm_profile_enable(1); synchronises.  Returns the length needed
 * (including the terminating NUL); writes at most len bytes. */
HM_API size_t hm_profile_report(char* buf, size_t len);
/* The same records in launch order, one per recorded step execution:
 * JSON [["step", launches, ms, algorithmic flops, algorithmic bytes, "tuning"], ...]
 * (lines up with a profiler's kernel list, step by step); "tuning" is
 * "<signature>#<bn>,<small>,<tc>" for batched-GEMM steps (see hm_tile_table_load), ""
 * otherwise; same buffer convention. */
HM_API size_t hm_profile_sequence(char* buf, size_t len);

/* ---- tile autotuning (no counterpart in the reference) ----
 * Batched-GEMM steps pick their kernel and tile shape (width BN of the warp-tiled kernel;
 * shape 0 default, 1 64-row tiles, 2 8 x 8 outputs per lane for FP64, 3 96-row tiles;
 * batches of tile width <= 64 whose rows all come in multiples of 96 take 96-row tiles
 * unless the table's shape already fits them or HM_TILE96=0; tc: the tcgen05
 * kernel for eligible FP32 batches, the FP64 MMA kernel for FP64 batches) from a table
 * keyed by the batch's signature (step, element type, bucketed problem count and m/n/k),
 * written by hmat-omp_b200/autotune.py from timed sweeps:
 * JSON {"signature": [bn, shape, tc], ...}.
 * The table is read from HM_TILE_TABLE if set, else from tile_table.json beside the
 * library, at the first batch finalised; entries apply to operators planned afterwards.
 * Batches without an entry keep the built-in heuristics.  hm_tile_table_load replaces
 * the table (NULL or "" clears it); returns HM_OK or HM_ERR_ARG if the file cannot be
 * read or parsed.  hm_tile_table_size: entries in the table. */
HM_API int hm_tile_table_load(const char* path);
HM_API int hm_tile_table_size(void);

#ifdef __cplusplus
}
#endif
#endif /* HMAT_B200_H */
