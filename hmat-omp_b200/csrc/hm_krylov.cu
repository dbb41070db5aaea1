// Flexible GMRES against the exact kernel operator, right-preconditioned by the
// compressed factorization (hm_solve_gmres).
//
// Every right-hand side j runs its own Arnoldi process; all of them advance together,
// so each step is one preconditioner application over all columns (the handle's
// factorization: the FP64 solve, or in mixed precision one FP32 sweep, which the flexible
// form tolerates), one product with the exact operator A (entries generated inside the
// batched FP64 GEMM, A never stored) and column-wise classical Gram-Schmidt with one
// reorthogonalisation (CGS2).  The Krylov basis is stored column-interleaved,
// V[(i s + j) N + r] = row r of basis vector i of right-hand side j, so the dot products
// and updates of all columns are single launches.  Rotations, least-squares updates and
// back substitutions run on the host (at most restart x restart per column).  With the
// preconditioner in the search space (flexible form: the preconditioned vectors Z_i are
// kept) the method converges where the stationary refinement x += A~^{-1}(b - A x) does
// not, i.e. when the compression error times ||A~^{-1}|| exceeds one.
#include <cmath>

#include "hm_engine.h"

namespace hm {

namespace {

constexpr int DOT_BLOCKS = 64;   // fixed partition of the rows: deterministic sums

// part[((i s + j) DOT_BLOCKS) + bx] = sum over this block's rows of V_i[:, j] . w[:, j]
__global__ void krylov_dot_partial(const double* __restrict__ V, int nv, const double* __restrict__ w, int N,
                                   int s, double* __restrict__ part) {
    const int j = blockIdx.y, i = blockIdx.z;
    if (i >= nv) return;
    const double* v = V + ((size_t)i * s + j) * N;
    const double* x = w + (size_t)j * N;
    const int chunk = (N + gridDim.x - 1) / gridDim.x;
    const int r0 = blockIdx.x * chunk, r1 = min(N, r0 + chunk);
    double acc = 0.0;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) acc = fma(v[r], x[r], acc);
    __shared__ double red[8];
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        part[((size_t)i * s + j) * gridDim.x + blockIdx.x] = t;
    }
}

// out[i s + j] = sum of the partials, in a fixed order
__global__ void krylov_dot_final(const double* __restrict__ part, int count, int nb, double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += part[(size_t)e * nb + b];
    out[e] = t;
}

// w[:, j] += sign * sum_{i < nv} h[i s + j] V_i[:, j]
__global__ void krylov_update(double* __restrict__ w, const double* __restrict__ V, int nv,
                              const double* __restrict__ h, int N, int s, double sign) {
    const int j = blockIdx.y;
    double* x = w + (size_t)j * N;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int i = 0; i < nv; ++i) acc = fma(h[(size_t)i * s + j], V[((size_t)i * s + j) * N + r], acc);
        x[r] = fma(sign, acc, x[r]);
    }
}

// dst[:, j] = f[j] * src[:, j]
__global__ void krylov_scale(double* __restrict__ dst, const double* __restrict__ src, const double* __restrict__ f,
                             int N, int s) {
    const int j = blockIdx.y;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x)
        dst[(size_t)j * N + r] = f[j] * src[(size_t)j * N + r];
}

// dst = a - b (N x s, ld N)
__global__ void krylov_sub(double* __restrict__ dst, const double* __restrict__ a, const double* __restrict__ b,
                           size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        dst[e] = a[e] - b[e];
}

int row_blocks(int N) { return std::max(1, std::min(256, (N + 255) / 256)); }

}  // namespace

void Engine::solve_gmres_device(const double* db, int s, int ldb, double* dx, int ldx, double tol, int restart,
                                int max_iter, hm_solve_stats* st) {
    HM_CHECK(built_, HM_ERR_STATE, "solve_gmres before build");
    HM_CHECK(gen_ != GEN_DENSE && sys_N_.size() == 1, HM_ERR_STATE,
             "solve_gmres needs a single operator built from a kernel (hm_*_build_from_kernel)");
    HM_CHECK(s >= 1 && ldb >= N_ && ldx >= N_ && db && dx && tol > 0 && restart >= 1 && restart <= 200 &&
                 max_iter >= 1,
             HM_ERR_ARG, "solve_gmres: bad arguments");
    const int N = N_, m = restart;
    const size_t ns = (size_t)N * s;
    if (s > ex_cols_) {
        exB_.alloc(ns);
        exX_.alloc(ns);
        exR_.alloc(ns);
        exD_.alloc(ns);
        exNorm_.alloc(2 * (size_t)s);
        ex_cols_ = s;
        exact_plans_.clear();
    }
    cudaStream_t q = stream_;
    DBuf<double> V((size_t)(m + 1) * ns), Z((size_t)m * ns), X(ns);
    DBuf<double> part((size_t)(m + 1) * s * DOT_BLOCKS), dots((size_t)(m + 1) * s), coef((size_t)(m + 1) * s);
    std::vector<double> hdots((size_t)(m + 1) * s), hcoef((size_t)(m + 1) * s);
    const dim3 rows_grid(row_blocks(N), s);
    // column dot products of V_0..V_{nv-1} with w -> host hdots[i s + j]
    auto col_dots = [&](const double* Vb, int nv, const double* w) {
        krylov_dot_partial<<<dim3(DOT_BLOCKS, s, nv), 256, 0, q>>>(Vb, nv, w, N, s, part.p);
        const int cnt = nv * s;
        krylov_dot_final<<<ceil_div(cnt, 128), 128, 0, q>>>(part.p, cnt, DOT_BLOCKS, dots.p);
        HM_CUDA(cudaGetLastError());
        count_launch(2);
        HM_CUDA(cudaMemcpyAsync(hdots.data(), dots.p, (size_t)cnt * sizeof(double), cudaMemcpyDeviceToHost, q));
        HM_CUDA(cudaStreamSynchronize(q));
    };
    auto upload_coef = [&](int nv) {
        HM_CUDA(cudaMemcpyAsync(coef.p, hcoef.data(), (size_t)nv * s * sizeof(double), cudaMemcpyHostToDevice, q));
    };
    Plan& ap = exact_plan(s);   // exR = A exX
    // b, its column norms, and the first iterate x = A~^{-1} b
    HM_CUDA(cudaMemcpy2DAsync(exB_.p, (size_t)N * sizeof(double), db, (size_t)ldb * sizeof(double),
                              (size_t)N * sizeof(double), s, cudaMemcpyDefault, q));
    col_dots(exB_.p, 1, exB_.p);
    std::vector<double> bnorm(s);
    for (int j = 0; j < s; ++j) bnorm[j] = std::sqrt(hdots[j]) > 0 ? std::sqrt(hdots[j]) : 1.0;
    precondition_device(exB_.p, s, X.p);
    std::vector<double> H((size_t)s * (m + 1) * m), cs((size_t)s * m), sn((size_t)s * m), g((size_t)s * (m + 1));
    std::vector<int> steps(s);
    std::vector<char> active(s);
    int total = 0;
    double worst = 0.0;
    for (;;) {
        // r = b - A x into V_0, then beta = ||r|| per column
        HM_CUDA(cudaMemcpyAsync(exX_.p, X.p, ns * sizeof(double), cudaMemcpyDeviceToDevice, q));
        ap.run(q, dstatus.p);
        krylov_sub<<<std::min<size_t>(4096, (ns + 255) / 256), 256, 0, q>>>(V.p, exB_.p, exR_.p, ns);
        count_launch();
        col_dots(V.p, 1, V.p);
        check_status("solve_gmres");
        worst = 0.0;
        for (int j = 0; j < s; ++j) {
            const double beta = std::sqrt(hdots[j]);
            worst = max_nan(worst, beta / bnorm[j]);
            g[(size_t)j * (m + 1)] = beta;
            for (int i = 1; i <= m; ++i) g[(size_t)j * (m + 1) + i] = 0.0;
            hcoef[j] = beta > 0 ? 1.0 / beta : 0.0;
            steps[j] = 0;
            active[j] = beta / bnorm[j] > tol;
        }
        if (!(worst == worst) || worst <= tol || total >= max_iter) break;
        upload_coef(1);
        krylov_scale<<<rows_grid, 256, 0, q>>>(V.p, V.p, coef.p, N, s);
        count_launch();
        int k = 0;
        for (; k < m && total < max_iter; ++k, ++total) {
            double* Vk = V.p + (size_t)k * ns;
            double* Zk = Z.p + (size_t)k * ns;
            precondition_device(Vk, s, Zk);                              // Z_k = A~^{-1} V_k
            HM_CUDA(cudaMemcpyAsync(exX_.p, Zk, ns * sizeof(double), cudaMemcpyDeviceToDevice, q));
            ap.run(q, dstatus.p);                                        // w = A Z_k (in exR)
            std::vector<double> h((size_t)(k + 1) * s, 0.0);
            for (int pass = 0; pass < 2; ++pass) {                       // CGS2
                col_dots(V.p, k + 1, exR_.p);
                for (size_t e = 0; e < h.size(); ++e) h[e] += hdots[e];
                std::copy(hdots.begin(), hdots.begin() + (k + 1) * s, hcoef.begin());
                upload_coef(k + 1);
                krylov_update<<<rows_grid, 256, 0, q>>>(exR_.p, V.p, k + 1, coef.p, N, s, -1.0);
                count_launch();
            }
            col_dots(exR_.p, 1, exR_.p);
            check_status("solve_gmres");
            bool any = false;
            for (int j = 0; j < s; ++j) {
                const double hn = std::sqrt(hdots[j]);
                hcoef[j] = 0.0;
                if (!active[j]) continue;
                double* Hj = H.data() + (size_t)j * (m + 1) * m;   // column-major (m + 1) x m
                double* col = Hj + (size_t)k * (m + 1);
                for (int i = 0; i <= k; ++i) col[i] = h[(size_t)i * s + j];
                col[k + 1] = hn;
                for (int i = 0; i < k; ++i) {   // previous rotations
                    const double c = cs[(size_t)j * m + i], sv = sn[(size_t)j * m + i];
                    const double a = col[i], b = col[i + 1];
                    col[i] = c * a + sv * b;
                    col[i + 1] = -sv * a + c * b;
                }
                const double a = col[k], b = col[k + 1];
                const double rr = std::hypot(a, b);
                const double c = rr > 0 ? a / rr : 1.0, sv = rr > 0 ? b / rr : 0.0;
                cs[(size_t)j * m + k] = c;
                sn[(size_t)j * m + k] = sv;
                col[k] = rr;
                col[k + 1] = 0.0;
                double* gj = g.data() + (size_t)j * (m + 1);
                gj[k + 1] = -sv * gj[k];
                gj[k] = c * gj[k];
                steps[j] = k + 1;
                if (rr == 0.0) {                 // exact breakdown: nothing more to gain
                    active[j] = 0;
                    steps[j] = k;
                    continue;
                }
                if (std::fabs(gj[k + 1]) / bnorm[j] <= 0.5 * tol || hn <= 1e-300) active[j] = 0;
                else hcoef[j] = 1.0 / hn;
                any = any || active[j];
            }
            upload_coef(1);
            krylov_scale<<<rows_grid, 256, 0, q>>>(V.p + (size_t)(k + 1) * ns, exR_.p, coef.p, N, s);
            count_launch();
            if (!any) { ++k; ++total; break; }
        }
        // x += Z y with H y = g (upper triangular, per column)
        const int kk = k;
        std::fill(hcoef.begin(), hcoef.end(), 0.0);
        for (int j = 0; j < s; ++j) {
            const int nj = std::min(steps[j], kk);
            const double* Hj = H.data() + (size_t)j * (m + 1) * m;
            const double* gj = g.data() + (size_t)j * (m + 1);
            std::vector<double> y(nj);
            for (int i = nj - 1; i >= 0; --i) {
                double t = gj[i];
                for (int c = i + 1; c < nj; ++c) t -= Hj[(size_t)c * (m + 1) + i] * y[c];
                const double d = Hj[(size_t)i * (m + 1) + i];
                y[i] = d != 0.0 ? t / d : 0.0;
            }
            for (int i = 0; i < nj; ++i) hcoef[(size_t)i * s + j] = y[i];
        }
        if (kk > 0) {
            upload_coef(kk);
            krylov_update<<<rows_grid, 256, 0, q>>>(X.p, Z.p, kk, coef.p, N, s, 1.0);
            count_launch();
        }
    }
    HM_CUDA(cudaMemcpy2DAsync(dx, (size_t)ldx * sizeof(double), X.p, (size_t)N * sizeof(double),
                              (size_t)N * sizeof(double), s, cudaMemcpyDefault, q));
    HM_CUDA(cudaStreamSynchronize(q));
    if (st) {
        st->ir_iters = total;
        st->rel_residual = worst;
    }
    if (!(worst <= tol)) {
        char msg[160];
        snprintf(msg, sizeof msg, "GMRES stopped at relative residual %.3e after %d iterations", worst, total);
        throw Error(HM_ERR_IR, msg);
    }
}

}  // namespace hm
