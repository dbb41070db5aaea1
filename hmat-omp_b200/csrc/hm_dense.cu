// Small batched dense kernels for sm_100a: one CTA per problem.
//
//  * gj_inverse_kernel  — Gauss-Jordan inversion with partial pivoting, the matrix held
//                          in registers (n <= GJ_MAX; used up to the threshold of
//                          plan_inverse).  Larger inverses are built by block
//                          Gauss-Jordan with panel pivoting over these plus batched
//                          GEMMs (panel_pivot_kernel, unscramble_kernel).
//  * jacobi_kernel      — cyclic two-sided Jacobi for symmetric positive semi-definite
//                          Gram matrices, parallel (round-robin) pair ordering, rotation
//                          test relative to the diagonal so graded matrices keep small
//                          eigenvalues to high relative accuracy (Demmel & Veselic, 1992).
//  * prep_kernel        — sort eigenpairs, form the scaled/permuted rotation and the
//                          truncation rank of compression.h:42-46.
//  * copy / identity utilities.
#include "hm_dense.h"

#include <algorithm>
#include <map>
#include <cstdlib>
#include <cmath>

namespace hm {

// ---------------------------------------------------------------------------------
// Profiler and plan execution
// ---------------------------------------------------------------------------------
Profiler& Profiler::get() {
    static Profiler p;
    return p;
}

cudaEvent_t Profiler::event() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    HM_CUDA(cudaEventCreate(&e));
    return e;
}

void Profiler::reset() {
    for (auto& r : recs) {
        pool.push_back(r.a);
        pool.push_back(r.b);
    }
    recs.clear();
}

std::string Profiler::report() {
    struct Agg { long long n = 0; double ms = 0, flops = 0, bytes = 0; };
    std::vector<std::pair<std::string, Agg>> agg;
    for (auto& r : recs) {
        HM_CUDA(cudaEventSynchronize(r.b));
        float ms = 0;
        HM_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        auto it = std::find_if(agg.begin(), agg.end(), [&](auto& x) { return x.first == r.name; });
        if (it == agg.end()) { agg.push_back({r.name, Agg{}}); it = agg.end() - 1; }
        it->second.n += r.launches;
        it->second.ms += ms;
        it->second.flops += r.flops;
        it->second.bytes += r.bytes;
    }
    std::string out = "{";
    char buf[256];
    for (size_t i = 0; i < agg.size(); ++i) {
        snprintf(buf, sizeof buf, "%s\"%s\": [%lld, %.6f, %.6e, %.6e]", i ? ", " : "", agg[i].first.c_str(),
                 agg[i].second.n, agg[i].second.ms, agg[i].second.flops, agg[i].second.bytes);
        out += buf;
    }
    return out + "}";
}

std::string Profiler::sequence() {
    std::string out = "[";
    char buf[512];
    for (size_t i = 0; i < recs.size(); ++i) {
        const Rec& r = recs[i];
        HM_CUDA(cudaEventSynchronize(r.b));
        float ms = 0;
        HM_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        snprintf(buf, sizeof buf, "%s[\"%s\", %d, %.6f, %.6e, %.6e, \"%s\"]", i ? ", " : "", r.name.c_str(),
                 r.launches, ms, r.flops, r.bytes, r.sig.c_str());
        out += buf;
    }
    return out + "]";
}

bool graphs_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("HM_CUDA_GRAPHS");
        return !(e && e[0] == '0' && e[1] == 0);
    }();
    return on;
}

void Plan::capture(cudaStream_t s, int* status) const {
    graph_.reset();
    cudaGraph_t g = nullptr;
    HM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
        for (auto& st : steps_) st->run(s, status);
    } catch (...) {
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    HM_CUDA(cudaStreamEndCapture(s, &g));
    cudaGraphExec_t e = nullptr;
    const cudaError_t rc = cudaGraphInstantiate(&e, g, 0);
    cudaGraphDestroy(g);
    HM_CUDA(rc);
    graph_.reset(e, [](cudaGraphExec_t x) { cudaGraphExecDestroy(x); });
    graph_status_ = status;
}

void Plan::run(cudaStream_t s, int* status) const {
    Profiler& P = Profiler::get();
    if (runs_ >= 1 && !steps_.empty() && !P.enabled && s != nullptr && s != cudaStreamLegacy && graphs_enabled()) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        HM_CUDA(cudaStreamIsCapturing(s, &cs));
        if (cs == cudaStreamCaptureStatusNone) {
            if (!graph_ || graph_status_ != status) capture(s, status);
            HM_CUDA(cudaGraphLaunch(graph_.get(), s));
            for (auto& st : steps_) P.launches += st->nlaunch();
            ++runs_;
            return;
        }
    }
    ++runs_;
    for (auto& st : steps_) {
        const int nl = st->nlaunch();
        if (P.enabled && nl > 0) {
            Profiler::Rec r{st->name(), P.event(), P.event(), st->flops(), st->bytes(), nl, st->sig()};
            HM_CUDA(cudaEventRecord(r.a, s));
            st->run(s, status);
            HM_CUDA(cudaEventRecord(r.b, s));
            P.recs.push_back(r);
        } else {
            st->run(s, status);
        }
        P.launches += nl;
    }
}

// ---------------------------------------------------------------------------------
// Gauss-Jordan inverse, register resident, implicit pivoting
//
// Thread (lane, warp) holds rows lane + 32*rr and columns warp + W*cc of an NB x NB
// tile (the matrix padded with identity).  Step j picks the pivot row p_j among rows not
// yet used (partial pivoting) and applies the in-place Gauss-Jordan update
//     a[p][c] <- a[p][c] / a[p][j]   (c != j),   a[p][j] <- 1 / a[p][j],
//     a[i][c] <- a[i][c] - a[i][j] a[p][c]      (i != p, c != j),
//     a[i][j] <- -a[i][j] / a[p][j]  (i != p),
// without swapping rows: at the end X[q[r], p[c]] = B[r, c] (q = inverse of the pivot
// sequence).  Each step is one fused multiply-add per element: column j is zeroed by its
// owner first (so the same FMA yields -a[i][j]/a[p][j]) and the pivot row's multiplier
// is zero (its scaled values are written afterwards by the owning lane).
//
// The owner of column j+1 searches its pivot right after its own update of step j, while
// the other warps still update, and publishes it (one CTA barrier per step).  The search
// key is the high word of |a[i][j]| with its low 8 bits replaced by 255 - i: one warp
// max-reduction picks a pivot within a relative 2^-12 of the largest candidate (ties to
// the lowest row), which keeps partial pivoting's stability bound.
// ---------------------------------------------------------------------------------
template <int NB, int W>
__global__ void __launch_bounds__(32 * W, 1) gj_inverse_kernel(const GJDesc* __restrict__ descs, int* status) {
    constexpr int RT = NB / 32, CT = NB / W;
    static_assert(NB % 32 == 0 && NB % W == 0 && NB <= 256, "Gauss-Jordan tile");
    __shared__ double colv[2][NB];
    __shared__ double s_inv[2];
    __shared__ int s_p[2];
    __shared__ int piv[NB];
    __shared__ int qinv[NB];
    const GJDesc d = descs[blockIdx.x];
    const int n = d.n;
    if (n <= 0) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double a[RT][CT];
#pragma unroll
    for (int rr = 0; rr < RT; ++rr)
#pragma unroll
        for (int cc = 0; cc < CT; ++cc) {
            const int i = lane + 32 * rr, c = warp + W * cc;
            a[rr][cc] = (i < n && c < n) ? d.A[i + (size_t)c * d.lda] : (i == c ? 1.0 : 0.0);
        }
    unsigned used = 0;   // bit rr: row lane + 32 rr is already a pivot row

    // pivot search of column j by its owning warp: colv[buf], s_p[buf], s_inv[buf]
    // (s_p = -1 marks a zero or non-finite pivot)
    auto search = [&](int j, int buf) {
        const int ccj = j / W;
        unsigned best = 0;
#pragma unroll
        for (int cc = 0; cc < CT; ++cc) {
            if (cc != ccj) continue;
#pragma unroll
            for (int rr = 0; rr < RT; ++rr) {
                const int i = lane + 32 * rr;
                const double v = a[rr][cc];
                colv[buf][i] = v;
                if (i < n && !((used >> rr) & 1u)) {
                    const unsigned hi = (unsigned)((unsigned long long)__double_as_longlong(fabs(v)) >> 32);
                    best = max(best, (hi & 0xFFFFFF00u) | (unsigned)(255 - i));
                }
            }
        }
        best = __reduce_max_sync(0xffffffffu, best);
        __syncwarp();
        if (lane == 0) {
            const int p = 255 - (int)(best & 0xFFu);
            const double pv = best ? colv[buf][p] : 0.0;
            const bool ok = best != 0 && pv != 0.0 && isfinite(pv);
            s_p[buf] = ok ? p : -1;
            s_inv[buf] = ok ? 1.0 / pv : 0.0;
        }
    };

    if (warp == 0) search(0, 0);
    __syncthreads();
    bool bad = false;
    for (int j = 0; j < n; ++j) {
        const int buf = j & 1;
        const int p = s_p[buf];
        if (p < 0) { bad = true; break; }   // uniform: every thread read the same word
        const double inv = s_inv[buf];
        if (threadIdx.x == 0) piv[j] = p;
        const int prr = p >> 5, plane = p & 31;
        if (lane == plane) used |= 1u << prr;
        // scaled pivot row, broadcast from its owning lane
        double r[CT];
#pragma unroll
        for (int cc = 0; cc < CT; ++cc) {
            double v = 0.0;
#pragma unroll
            for (int rr = 0; rr < RT; ++rr)
                if (rr == prr) v = a[rr][cc];
            r[cc] = __shfl_sync(0xffffffffu, v, plane) * inv;
        }
        // column j: zeroed by its owner, its pivot-row entry becomes 1 / a[p][j]
        if (warp == j % W) {
            const int ccj = j / W;
#pragma unroll
            for (int cc = 0; cc < CT; ++cc) {
                if (cc != ccj) continue;
                r[cc] = inv;
#pragma unroll
                for (int rr = 0; rr < RT; ++rr) a[rr][cc] = 0.0;
            }
        }
        double cv[RT];
#pragma unroll
        for (int rr = 0; rr < RT; ++rr) cv[rr] = (rr == prr && lane == plane) ? 0.0 : colv[buf][lane + 32 * rr];
#pragma unroll
        for (int rr = 0; rr < RT; ++rr)
#pragma unroll
            for (int cc = 0; cc < CT; ++cc) a[rr][cc] = fma(-cv[rr], r[cc], a[rr][cc]);
#pragma unroll
        for (int rr = 0; rr < RT; ++rr) {
            if (rr != prr) continue;
#pragma unroll
            for (int cc = 0; cc < CT; ++cc) a[rr][cc] = (lane == plane) ? r[cc] : a[rr][cc];
        }
        if (j + 1 < n && warp == (j + 1) % W) search(j + 1, buf ^ 1);
        __syncthreads();
    }
    if (bad) {
        if (threadIdx.x == 0) atomicOr(status, ST_SINGULAR);
        for (int e = threadIdx.x; e < n * n; e += 32 * W) d.X[(e % n) + (size_t)(e / n) * d.ldx] = nan("");
        return;
    }
    for (int j = threadIdx.x; j < n; j += 32 * W) qinv[piv[j]] = j;
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < RT; ++rr) {
        const int i = lane + 32 * rr;
        if (i >= n) continue;
        const int row = qinv[i];
#pragma unroll
        for (int cc = 0; cc < CT; ++cc) {
            const int c = warp + W * cc;
            if (c < n) d.X[row + (size_t)piv[c] * d.ldx] = a[rr][cc];
        }
    }
}

void launch_gj(const DevTable<GJDesc>& t, int nb, int* status, cudaStream_t s) {
    if (t.h.empty()) return;
    switch (nb) {
        case 32: gj_inverse_kernel<32, 4><<<t.size(), 128, 0, s>>>(t.d.p, status); break;
        case 64: gj_inverse_kernel<64, 8><<<t.size(), 256, 0, s>>>(t.d.p, status); break;
        case 96: gj_inverse_kernel<96, 12><<<t.size(), 384, 0, s>>>(t.d.p, status); break;
        case 128: gj_inverse_kernel<128, 16><<<t.size(), 512, 0, s>>>(t.d.p, status); break;
        default: throw Error(HM_ERR_UNSUPPORTED, "Gauss-Jordan block size");
    }
    HM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------
// Cyclic Jacobi for symmetric PSD matrices (parallel round-robin ordering)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void jac_pair(int r, int i, int kk, int& p, int& q) {
    // circle method on kk (even) players: player kk-1 fixed
    const int m = kk - 1;
    if (i == 0) { p = m; q = r; }
    else { p = (r + i) % m; q = (r - i + m) % m; }
    if (p > q) { int t = p; p = q; q = t; }
}

__global__ void __launch_bounds__(256) jacobi_kernel(const EigDesc* __restrict__ descs, int* status,
                                                     int max_sweeps, int use_smem, int w_smem) {
    extern __shared__ double sm[];
    const EigDesc d = descs[blockIdx.x];
    const int k = d.k;
    if (k <= 0) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    const bool in_smem = use_smem != 0;
    const int ld = in_smem ? k : d.ldg;
    double* g = in_smem ? sm : d.G;
    double* cs = in_smem ? sm + k * k : sm;   // rotation cosines  (k/2+1)
    const int kk = (k + 1) & ~1;              // even number of players (k = dummy if odd)
    const int half = kk / 2;
    double* sn = cs + half;
    // the eigenvector matrix accumulates in shared memory when it fits (every rotation
    // round reads and writes two of its columns), and is written out once at the end
    const bool w_in_smem = in_smem && w_smem != 0;
    double* W = w_in_smem ? sn + half : d.W;
    const int ldw = w_in_smem ? k : d.ldw;
    __shared__ int s_rot;
    if (in_smem)
        for (int e = tid; e < k * k; e += nt) {
            int i = e % k, j = e / k;
            g[e] = d.G[i + (size_t)j * d.ldg];
        }
    for (int e = tid; e < k * k; e += nt) {
        int i = e % k, j = e / k;
        W[i + (size_t)j * ldw] = (i == j) ? 1.0 : 0.0;
    }
    // Rotation test: |a_pq| > eps sqrt(a_pp a_qq), relative, so graded matrices keep their
    // small eigenvalues to high relative accuracy.  Columns whose diagonal is at most 1e-30
    // of the largest (singular values below 1e-15 sigma_0: rounding, not signal) are dead:
    // they are not rotated, and the caller turns them into zero columns.  Orthogonalising
    // noise among itself to relative precision would take tens of sweeps (and never ends
    // once entries reach the denormal range) without changing any result above 1e-15.
    __shared__ double s_dmax;
    if (tid == 0) {
        double dm = 0.0;
        for (int i = 0; i < k; ++i) dm = fmax(dm, fabs(g[i + i * ld]));
        s_dmax = dm;
    }
    __syncthreads();
    const double dead = 1e-30 * s_dmax;
    const double floor_abs = 1e-290;
    const double eps = 4.0 * 2.220446049250313e-16;
    int sweep = 0;
    bool converged = (k == 1) || s_dmax == 0.0;
    for (; sweep < max_sweeps && !converged; ++sweep) {
        if (tid == 0) s_rot = 0;
        __syncthreads();
        for (int r = 0; r < kk - 1; ++r) {
            for (int t = tid; t < half; t += nt) {
                int p, q;
                jac_pair(r, t, kk, p, q);
                double c = 1.0, s = 0.0;
                if (q < k) {
                    const double app = g[p + p * ld], aqq = g[q + q * ld], apq = g[p + q * ld];
                    const double thr = eps * sqrt(fabs(app)) * sqrt(fabs(aqq));
                    if (app > dead && aqq > dead && fabs(apq) > thr && fabs(apq) > floor_abs) {
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + hypot(1.0, tau));
                        c = 1.0 / sqrt(1.0 + tt * tt);
                        s = tt * c;
                        s_rot = 1;
                    }
                }
                cs[t] = c;
                sn[t] = s;
            }
            __syncthreads();
            // G <- G J (columns p, q), W <- W J
            for (int e = tid; e < half * k; e += nt) {
                const int t = e / k, i = e % k;
                const double s = sn[t];
                if (s == 0.0) continue;
                int p, q;
                jac_pair(r, t, kk, p, q);
                const double c = cs[t];
                const double gp = g[i + p * ld], gq = g[i + q * ld];
                g[i + p * ld] = c * gp - s * gq;
                g[i + q * ld] = s * gp + c * gq;
                const double wp = W[i + (size_t)p * ldw], wq = W[i + (size_t)q * ldw];
                W[i + (size_t)p * ldw] = c * wp - s * wq;
                W[i + (size_t)q * ldw] = s * wp + c * wq;
            }
            __syncthreads();
            // G <- J^T G (rows p, q); the annihilated pair (p, q), (q, p) set to exact zeros
            // (only this pair's own updates touch those two entries)
            for (int e = tid; e < half * k; e += nt) {
                const int t = e / k, j = e % k;
                const double s = sn[t];
                if (s == 0.0) continue;
                int p, q;
                jac_pair(r, t, kk, p, q);
                const double c = cs[t];
                const double gp = g[p + j * ld], gq = g[q + j * ld];
                g[p + j * ld] = j == q ? 0.0 : c * gp - s * gq;
                g[q + j * ld] = j == p ? 0.0 : s * gp + c * gq;
            }
            __syncthreads();
        }
        converged = (s_rot == 0);
        __syncthreads();
    }
    if (!converged && tid == 0) atomicOr(status, ST_NO_CONVERGE);
    for (int i = tid; i < k; i += nt) d.lam[i] = g[i + i * ld];
    if (w_in_smem) {
        __syncthreads();
        for (int e = tid; e < k * k; e += nt) {
            const int i = e % k, j = e / k;
            d.W[i + (size_t)j * d.ldw] = W[e];
        }
    }
}

void launch_jacobi(const DevTable<EigDesc>& t, int* status, cudaStream_t s, int max_sweeps) {
    if (t.h.empty()) return;
    int kmax = 0;
    for (auto& d : t.h) kmax = std::max(kmax, d.k);
    const bool g_smem = kmax <= JAC_SMEM_MAX;
    const bool w_smem = g_smem && kmax <= JAC_W_SMEM_MAX;
    size_t smem = (g_smem ? (size_t)kmax * kmax * 8 : 0) + ((size_t)kmax + 2) * 8 +
                  (w_smem ? (size_t)kmax * kmax * 8 : 0);
    static size_t cur = 0;
    ensure_dyn_smem(jacobi_kernel, smem, cur);
    jacobi_kernel<<<t.size(), 256, smem, s>>>(t.d.p, status, max_sweeps, g_smem, w_smem);
    HM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------
// Column norms, sort + truncation rank, permute/scale
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) norms_kernel(const NormDesc* __restrict__ descs) {
    const NormDesc d = descs[blockIdx.x];
    const int c = blockIdx.y;
    if (c >= d.k) return;
    const double* x = d.X + (size_t)c * d.ld;
    // scaled sum of squares (no overflow/underflow for tiny or huge columns)
    double mx = 0.0;
    for (int i = threadIdx.x; i < d.rows; i += blockDim.x) mx = fmax(mx, fabs(x[i]));
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        mx = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
        if (threadIdx.x == 0) red[0] = mx;
    }
    __syncthreads();
    mx = red[0];
    __syncthreads();
    if (mx == 0.0) {
        if (threadIdx.x == 0) d.out[c] = 0.0;
        return;
    }
    const double inv = 1.0 / mx;
    double s = 0.0;
    for (int i = threadIdx.x; i < d.rows; i += blockDim.x) {
        const double v = x[i] * inv;
        s = fma(v, v, s);
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (threadIdx.x == 0) d.out[c] = mx * sqrt(s);
    }
}

void launch_norms(const DevTable<NormDesc>& t, cudaStream_t s) {
    if (t.h.empty()) return;
    int kmax = 0;
    for (auto& d : t.h) kmax = std::max(kmax, d.k);
    HM_CHECK(kmax <= 65535, HM_ERR_UNSUPPORTED, "too many columns");
    norms_kernel<<<dim3(t.size(), kmax), 256, 0, s>>>(t.d.p);
    HM_CUDA(cudaGetLastError());
}

__global__ void __launch_bounds__(256) prep_kernel(const PrepDesc* __restrict__ descs, double tol,
                                                   int max_rank) {
    extern __shared__ double sm[];
    const PrepDesc d = descs[blockIdx.x];
    const int k = d.k;
    if (k <= 0) return;
    double* sg = sm;
    int* perm = reinterpret_cast<int*>(sg + k);
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < k; i += nt) sg[i] = d.sig_in[i];
    __syncthreads();
    // position of each entry in descending order (ties by index)
    for (int i = tid; i < k; i += nt) {
        const double v = sg[i];
        int pos = 0;
        for (int j = 0; j < k; ++j) {
            const double w = sg[j];
            pos += (w > v) || (w == v && j < i);
        }
        perm[pos] = i;
    }
    __syncthreads();
    // singular values at or below 1e-15 of the largest are rounding (dead Jacobi columns):
    // zero, so the permute step writes zero columns for them
    const double smax = sg[perm[0]];
    for (int c = tid; c < k; c += nt) {
        d.perm[c] = perm[c];
        const double v = sg[perm[c]];
        if (d.sigma) d.sigma[c] = v > 1e-15 * smax ? v : 0.0;
    }
    if (d.rank && tid == 0) {
        // compression.h:42-46: #{S_i > tol*S_0} when S_0 > 1e-15, at least 1
        const double s0 = sg[perm[0]];
        int r = 0;
        if (s0 > 1e-15)
            for (int c = 0; c < k; ++c) r += sg[perm[c]] > tol * s0;
        if (r == 0) r = 1;
        if (max_rank > 0 && r > max_rank) r = max_rank;
        *d.rank = r;
    }
}

void launch_prep(const DevTable<PrepDesc>& t, double tol, int max_rank, cudaStream_t s) {
    if (t.h.empty()) return;
    int kmax = 0;
    for (auto& d : t.h) kmax = std::max(kmax, d.k);
    size_t smem = (size_t)kmax * 12 + 16;
    prep_kernel<<<t.size(), 256, smem, s>>>(t.d.p, tol, max_rank);
    HM_CUDA(cudaGetLastError());
}

// Table kernels: blockIdx.x = problem (no 65535 limit), blockIdx.y = slice of its elements.
__global__ void permute_kernel(const PermDesc* __restrict__ descs) {
    const PermDesc d = descs[blockIdx.x];
    const size_t total = (size_t)d.rows * d.k;
    for (size_t e = blockIdx.y * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.y * blockDim.x) {
        const int i = (int)(e % d.rows), c = (int)(e / d.rows);
        const int src = d.perm[c];
        double v = d.src[i + (size_t)src * d.lds];
        if (d.sig) {
            const double sg = d.sig[c];
            v = sg > 0.0 ? v / sg : 0.0;
        }
        d.dst[i + (size_t)c * d.ldd] = v;
    }
}

void launch_permute(const DevTable<PermDesc>& t, cudaStream_t s) {
    if (t.h.empty()) return;
    size_t mx = 0;
    for (auto& d : t.h) mx = std::max(mx, (size_t)d.rows * d.k);
    int gx = (int)std::min<size_t>(std::max<size_t>(1, (mx + 255) / 256), 1024);
    permute_kernel<<<dim3(t.size(), gx), 256, 0, s>>>(t.d.p);
    HM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------
// Copies (optionally transposed, optionally to FP32) and identity fills
// ---------------------------------------------------------------------------------
__global__ void copy_kernel(const CopyDesc* __restrict__ descs) {
    const CopyDesc d = descs[blockIdx.x];
    const size_t total = (size_t)d.rows * d.cols;
    for (size_t e = blockIdx.y * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.y * blockDim.x) {
        const int i = (int)(e % d.rows), j = (int)(e / d.rows);
        const size_t si = d.trans ? j + (size_t)i * d.lds : i + (size_t)j * d.lds;
        const double v = d.src_f32 ? (double)static_cast<const float*>(d.src)[si]
                                   : static_cast<const double*>(d.src)[si];
        const size_t di = i + (size_t)j * d.ldd;
        if (d.dst_f32) static_cast<float*>(d.dst)[di] = (float)v;
        else static_cast<double*>(d.dst)[di] = v;
    }
}

void launch_copy(const DevTable<CopyDesc>& t, cudaStream_t s) {
    if (t.h.empty()) return;
    size_t mx = 0;
    for (auto& d : t.h) mx = std::max(mx, (size_t)d.rows * d.cols);
    int gx = (int)std::min<size_t>(std::max<size_t>(1, (mx + 255) / 256), 2048);
    copy_kernel<<<dim3(t.size(), gx), 256, 0, s>>>(t.d.p);
    HM_CUDA(cudaGetLastError());
}

__global__ void ident_kernel(const IdentDesc* __restrict__ descs) {
    const IdentDesc d = descs[blockIdx.x];
    const size_t total = (size_t)d.rows * d.cols;
    for (size_t e = blockIdx.y * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.y * blockDim.x) {
        const int i = (int)(e % d.rows), j = (int)(e / d.rows);
        d.X[i + (size_t)j * d.ldx] = (i == j) ? d.diag : 0.0;
    }
}

void launch_ident(const DevTable<IdentDesc>& t, cudaStream_t s) {
    if (t.h.empty()) return;
    size_t mx = 0;
    for (auto& d : t.h) mx = std::max(mx, (size_t)d.rows * d.cols);
    int gx = (int)std::min<size_t>(std::max<size_t>(1, (mx + 255) / 256), 1024);
    ident_kernel<<<dim3(t.size(), gx), 256, 0, s>>>(t.d.p);
    HM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------
// Plans
// ---------------------------------------------------------------------------------
// Largest order inverted by one Gauss-Jordan kernel (pivoting over all rows); larger
// ones go through the block Gauss-Jordan sweep below, whose bulk runs as batched GEMMs.
// 128 by default (every capacitance matrix of rank <= 64 per side is one launch per
// level); HM_GJ_MAX (32, 64, 96 or 128) overrides it.
static int gj_max() {
    static const int v = [] {
        const char* e = std::getenv("HM_GJ_MAX");
        const int x = e ? std::atoi(e) : 128;
        return (x == 32 || x == 64 || x == 96 || x == 128) ? x : 128;
    }();
    return v;
}

// ---------------------------------------------------------------------------------
// Block Gauss-Jordan with partial pivoting by panels (inverses above the Gauss-Jordan
// threshold), in place on a column-major work copy W of A.  It is the sweep of the
// transposed problem: pivots are chosen among columns, so every exchange moves whole
// (contiguous) columns.  For each block of w rows K = [k0, k0 + kw), with O the other
// indices:
//   1. panel_pivot_kernel: Gaussian elimination with partial pivoting on the transposed
//      panel W[K, k0:]^T (in shared memory) chooses kw pivot columns, which are swapped
//      into columns K; the exchanges are recorded in ipiv.
//   2. PD = inv(W[K, K]) (Gauss-Jordan kernel);
//   3. T = W[O, K] PD,  Z = -PD W[K, O];
//   4. W[O, O] += W[O, K] Z;
//   5. W[K, K] = PD, W[O, K] = T, W[K, O] = Z.
// At the end row c of W is row where[c] of inv(A), where[] being the exchanges applied in
// order to the identity permutation (unscramble_kernel).  The pivots are those of LU with
// partial pivoting of A^T panel by panel, so every inverted block W[K, K] is as well
// conditioned as LU's diagonal blocks: a leaf whose leading block is singular while the
// leaf is not (which getrf handles, matrix.h:120-131) inverts like any other.
// ---------------------------------------------------------------------------------
struct PanelDesc {
    double* W;
    int ld, n, k0, kw;
    int* ipiv;    // n entries: column position i was exchanged with column ipiv[i]
};

struct ScatterDesc {
    const double* W;
    int ldw;
    double* X;
    int ldx, n;
    const int* ipiv;
};

// Panel width for order n: the padded (n + 1) x w panel fits in 136 KB of shared memory
// (w = 64 up to n = 271).
static int bgj_width(int n) {
    int w = 64;
    while (w > 1 && (size_t)(n + 1) * w * sizeof(double) > (size_t)136 * 1024) w /= 2;
    return w;
}
static size_t panel_smem(int m, int kw) {
    return (size_t)(m + 1) * kw * sizeof(double) + 2 * (size_t)m * sizeof(int);
}

__global__ void __launch_bounds__(256) panel_pivot_kernel(const PanelDesc* __restrict__ descs, int* status) {
    extern __shared__ double sm[];   // panel: (m + 1) x kw column-major (then the move buffer); 2m ints
    __shared__ unsigned red_k[2][8];
    __shared__ int prow[64];
    __shared__ int mv_pos[128], mv_src[128];
    __shared__ int s_bad, s_nmv;
    const PanelDesc d = descs[blockIdx.x];
    const int m = d.n - d.k0, kw = d.kw, LDP = m + 1, tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    double* pan = sm;
    int* at = reinterpret_cast<int*>(sm + (size_t)LDP * kw);
    int* pos = at + m;
    if (tid == 0) s_bad = 0;
    // logical panel element (i, j) = W[k0 + j, k0 + i]: rows K of the columns k0.. (contiguous in j)
    for (int e = tid; e < m * kw; e += nt) {
        const int j = e % kw, i = e / kw;
        pan[i + (size_t)j * LDP] = d.W[(d.k0 + j) + (size_t)(d.k0 + i) * d.ld];
    }
    // Right-looking elimination without row exchanges: a row chosen as pivot is flagged
    // (bit k of `used` for row tid + k nt) and left in place.  Each thread updates its own
    // rows and, in the same pass, offers its best candidate for the next column, so one
    // barrier per column separates the steps.  Candidates are compared by a 32-bit key:
    // the high word of |value| with its low ib bits replaced by (mask - row), so one warp
    // max-reduction picks a pivot within a relative 2^(ib - 20) of the largest (ties to
    // the lowest row), which keeps partial pivoting's stability bound.
    const int ib = 32 - __clz(max(m - 1, 1));
    const unsigned mask = (1u << ib) - 1u;
    auto key = [&](double v, int i) -> unsigned {
        if (!(v == v)) return 0u;   // NaN never wins
        const unsigned hi = (unsigned)((unsigned long long)__double_as_longlong(fabs(v)) >> 32);
        return (hi & ~mask) | (mask - (unsigned)i);
    };
    auto offer = [&](unsigned k, int buf) {
        k = __reduce_max_sync(0xffffffffu, k);
        if (lane == 0) red_k[buf][warp] = k;
    };
    auto choose = [&](int buf) {
        unsigned k = red_k[buf][0];
        for (int w = 1; w < nw; ++w) k = max(k, red_k[buf][w]);
        return k;
    };
    unsigned long long used = 0;
    __syncthreads();
    {
        unsigned best = 0;
        for (int i = tid; i < m; i += nt) best = max(best, key(pan[i], i));
        offer(best, 0);
    }
    __syncthreads();
    for (int j = 0; j < kw; ++j) {
        const unsigned kb = choose(j & 1);
        const int p = (int)(mask - (kb & mask));
        const bool pin = kb != 0u && p >= 0 && p < m;   // false when no candidate is a number
        const double pv = pin ? pan[p + (size_t)j * LDP] : 0.0;
        const bool ok = pin && fabs(pv) > 0.0 && isfinite(pv);
        if (tid == 0) {
            prow[j] = pin ? p : -1;
            if (!ok) s_bad = 1;
        }
        if (pin && p % nt == tid) used |= 1ull << (p / nt);
        const double rinv = ok ? 1.0 / pv : 0.0;
        unsigned best = 0;
        for (int k = 0, i = tid; i < m; ++k, i += nt) {
            if ((used >> k) & 1ull) continue;
            if (ok) {
                // 8 columns at a time, every load of a chunk before its stores (the row is
                // never the pivot row, but the compiler cannot know that)
                const double l = pan[i + (size_t)j * LDP] * rinv;
                double* ri = pan + i;
                const double* rp = pan + p;
                for (int c0 = j + 1; c0 < kw; c0 += 8) {
                    double a[8], b[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int c = c0 + u;
                        a[u] = c < kw ? ri[(size_t)c * LDP] : 0.0;
                        b[u] = c < kw ? rp[(size_t)c * LDP] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (c0 + u < kw) ri[(size_t)(c0 + u) * LDP] = fma(-l, b[u], a[u]);
                }
            }
            if (j + 1 < kw) best = max(best, key(pan[i + (size_t)(j + 1) * LDP], i));
        }
        if (j + 1 < kw) offer(best, (j + 1) & 1);
        __syncthreads();
    }
    // The pivot rows as the exchange sequence of LU with partial pivoting (position j
    // exchanged with position ipiv[j]), and as one permutation of the columns k0..n-1:
    // column k0 + i receives column k0 + at[i]; only the moved ones (at most 2 kw) are listed.
    for (int i = tid; i < m; i += nt) at[i] = pos[i] = i;
    if (tid == 0) s_nmv = 0;
    __syncthreads();
    if (tid == 0) {
        if (s_bad) atomicOr(status, ST_SINGULAR);
        for (int j = 0; j < kw; ++j) {
            const int r = (prow[j] >= 0 && prow[j] < m) ? prow[j] : j;
            const int q = pos[r] >= j ? pos[r] : j;   // a repeated row (only after a bad pivot) stays put
            d.ipiv[d.k0 + j] = d.k0 + q;
            const int x = at[j], y = at[q];
            at[j] = y; at[q] = x;
            pos[y] = j; pos[x] = q;
        }
    }
    __syncthreads();
    for (int i = tid; i < m; i += nt)   // the moved positions, in any order (at most 2 kw)
        if (at[i] != i) {
            const int sl = atomicAdd(&s_nmv, 1);
            if (sl < 128) { mv_pos[sl] = i; mv_src[sl] = at[i]; }
        }
    __syncthreads();
    const int nmv = min(s_nmv, 128);
    if (nmv == 0) return;
    // move the columns through shared memory (the panel's space), rc rows at a time: all
    // reads of a chunk, then all writes (coalesced along the rows)
    const int rc = min(d.n, (int)(((size_t)LDP * kw) / (size_t)nmv));
    for (int r0 = 0; r0 < d.n; r0 += rc) {
        const int rows = min(rc, d.n - r0);
        for (int e = tid; e < nmv * rows; e += nt) {
            const int l = e / rows, r = e % rows;
            pan[(size_t)l * rows + r] = d.W[(r0 + r) + (size_t)(d.k0 + mv_src[l]) * d.ld];
        }
        __syncthreads();
        for (int e = tid; e < nmv * rows; e += nt) {
            const int l = e / rows, r = e % rows;
            d.W[(r0 + r) + (size_t)(d.k0 + mv_pos[l]) * d.ld] = pan[(size_t)l * rows + r];
        }
        __syncthreads();
    }
}

// X[where[c], :] = W[c, :], where[] = the exchanges of ipiv applied in order to the
// identity; done as the gather X[r, :] = W[src[r], :] with src the inverse of where
// (coalesced writes, reads within the same column).
__global__ void __launch_bounds__(256) unscramble_kernel(const ScatterDesc* __restrict__ descs) {
    extern __shared__ int where[];   // where[n], then src[n]
    const ScatterDesc d = descs[blockIdx.x];
    int* src = where + d.n;
    if (threadIdx.x == 0) {
        for (int i = 0; i < d.n; ++i) where[i] = i;
        for (int i = 0; i < d.n; ++i) {
            const int p = d.ipiv[i];
            const int t = where[i]; where[i] = where[p]; where[p] = t;
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < d.n; c += blockDim.x) src[where[c]] = c;
    __syncthreads();
    const size_t total = (size_t)d.n * d.n;
    for (size_t e = blockIdx.y * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.y * blockDim.x) {
        const int r = (int)(e % d.n), j = (int)(e / d.n);
        d.X[r + (size_t)j * d.ldx] = d.W[src[r] + (size_t)j * d.ldw];
    }
}

namespace {
struct PanelStep : Plan::Step {
    DevTable<PanelDesc> t;
    void run(cudaStream_t s, int* st) const override {
        if (t.h.empty()) return;
        size_t mx = 0;
        for (auto& d : t.h) mx = std::max(mx, panel_smem(d.n - d.k0, d.kw));
        static size_t cur = 0;
        ensure_dyn_smem(panel_pivot_kernel, mx, cur);
        panel_pivot_kernel<<<t.size(), 256, mx, s>>>(t.d.p, st);
        HM_CUDA(cudaGetLastError());
    }
    const char* name() const override { return "panel_pivot"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};
struct ScatterStep : Plan::Step {
    DevTable<ScatterDesc> t;
    void run(cudaStream_t s, int*) const override {
        if (t.h.empty()) return;
        int mx = 0;
        for (auto& d : t.h) mx = std::max(mx, d.n);
        static size_t cur = 0;
        ensure_dyn_smem(unscramble_kernel, 2 * (size_t)mx * sizeof(int), cur);
        const int gy = std::max(1, std::min(8, mx * mx / 16384));
        unscramble_kernel<<<dim3(t.size(), gy), 256, 2 * (size_t)mx * sizeof(int), s>>>(t.d.p);
        HM_CUDA(cudaGetLastError());
    }
    const char* name() const override { return "unscramble"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
    double bytes() const override {
        double b = 0;
        for (auto& d : t.h) b += 16.0 * d.n * d.n;
        return b;
    }
};
}  // namespace

void plan_inverse(Plan& plan, const std::vector<InvProblem>& probs, cudaStream_t s) {
    std::vector<InvProblem> small, large;
    const int gmax = gj_max();
    for (auto& p : probs) {
        if (p.n <= 0) continue;
        (p.n <= gmax ? small : large).push_back(p);
    }
    if (!small.empty()) {
        auto st = std::make_unique<GJStep>();
        for (auto& p : small)
            st->t[p.n <= 32 ? 0 : p.n <= 64 ? 1 : p.n <= 96 ? 2 : 3].h.push_back({p.A, p.lda, p.X, p.ldx, p.n});
        for (auto& tb : st->t) tb.upload(s);
        plan.add(std::move(st));
    }
    if (large.empty()) return;
    struct Work { const InvProblem* p; double *W, *PD, *T, *Z; int* ipiv; int w; };
    std::vector<Work> ws;
    int steps = 0;
    auto cp = std::make_unique<CopyStep>();
    for (auto& p : large) {
        HM_CHECK(p.n <= 16384, HM_ERR_UNSUPPORTED, "inverse: order above 16384");
        Work x{&p, nullptr, nullptr, nullptr, nullptr, nullptr, bgj_width(p.n)};
        x.W = plan.scratch((size_t)p.n * p.n);
        x.PD = plan.scratch((size_t)x.w * x.w);
        x.T = plan.scratch((size_t)p.n * x.w);   // n x kw, ld n (rows O used)
        x.Z = plan.scratch((size_t)x.w * p.n);   // kw x n, ld kw (columns O used)
        x.ipiv = plan.scratch_i(p.n);
        cp->t.h.push_back({p.A, p.lda, x.W, p.n, p.n, p.n, 0, 0, 0});
        ws.push_back(x);
        steps = std::max(steps, ceil_div(p.n, x.w));
    }
    cp->t.upload(s);
    plan.add(std::move(cp));
    for (int b = 0; b < steps; ++b) {
        auto pan = std::make_unique<PanelStep>();
        auto gj = std::make_unique<GJStep>();
        auto gTZ = std::make_unique<GemmStep<double>>("inverse.panel");
        auto gUp = std::make_unique<GemmStep<double>>("inverse.update");
        auto put = std::make_unique<CopyStep>();
        for (auto& x : ws) {
            const int n = x.p->n, k0 = b * x.w;
            if (k0 >= n) continue;
            const int kw = std::min(x.w, n - k0), e0 = k0 + kw, ld = n;
            double* W = x.W;
            pan->t.h.push_back({W, ld, n, k0, kw, x.ipiv});
            gj->t[kw <= 32 ? 0 : 1].h.push_back({W + k0 + (size_t)k0 * ld, ld, x.PD, kw, kw});
            // index ranges outside K: [0, k0) and [e0, n)
            const int r0[2] = {0, e0}, rl[2] = {k0, n - e0};
            for (int q = 0; q < 2; ++q) {
                if (rl[q] <= 0) continue;
                // T[Oq, :] = W[Oq, K] PD
                gTZ->batch.add(rl[q], kw, kw, 1.0, W + r0[q] + (size_t)k0 * ld, ld, OP_N, x.PD, kw, OP_N, 0.0,
                               x.T + r0[q], n);
                // Z[:, Oq] = -PD W[K, Oq]
                gTZ->batch.add(kw, rl[q], kw, -1.0, x.PD, kw, OP_N, W + k0 + (size_t)r0[q] * ld, ld, OP_N, 0.0,
                               x.Z + (size_t)r0[q] * kw, kw);
            }
            for (int qi = 0; qi < 2; ++qi)
                for (int qj = 0; qj < 2; ++qj) {
                    if (rl[qi] <= 0 || rl[qj] <= 0) continue;
                    // W[Oqi, Oqj] += W[Oqi, K] Z[:, Oqj]
                    gUp->batch.add(rl[qi], rl[qj], kw, 1.0, W + r0[qi] + (size_t)k0 * ld, ld, OP_N,
                                   x.Z + (size_t)r0[qj] * kw, kw, OP_N, 1.0, W + r0[qi] + (size_t)r0[qj] * ld, ld);
                }
            put->t.h.push_back({x.PD, kw, W + k0 + (size_t)k0 * ld, ld, kw, kw, 0, 0, 0});
            for (int q = 0; q < 2; ++q) {
                if (rl[q] <= 0) continue;
                put->t.h.push_back({x.T + r0[q], n, W + r0[q] + (size_t)k0 * ld, ld, rl[q], kw, 0, 0, 0});
                put->t.h.push_back({x.Z + (size_t)r0[q] * kw, kw, W + k0 + (size_t)r0[q] * ld, ld, kw, rl[q], 0, 0, 0});
            }
        }
        pan->t.upload(s);
        for (auto& tb : gj->t) tb.upload(s);
        gTZ->batch.finalize(s);
        gUp->batch.finalize(s);
        put->t.upload(s);
        plan.add(std::move(pan));
        plan.add(std::move(gj));
        if (!gTZ->batch.empty()) plan.add(std::move(gTZ));
        if (!gUp->batch.empty()) plan.add(std::move(gUp));
        plan.add(std::move(put));
    }
    auto sc = std::make_unique<ScatterStep>();
    for (auto& x : ws) sc->t.h.push_back({x.W, x.p->n, x.p->X, x.p->ldx, x.p->n, x.ipiv});
    sc->t.upload(s);
    plan.add(std::move(sc));
}

// ---------------------------------------------------------------------------------
// Shifted CholeskyQR3 (Fukaya, Kannan, Nakatsukasa, Yamamoto, Yanagisawa; SIAM J. Sci.
// Comput. 2020): X = Q R by Gram matrices.  Pass 1 factors G + s I with the shift
// s = 11 (m k + k (k + 1)) u tr(G), which brings cond(X R^{-1}) to about u^{-1/2}; passes
// 2 and 3 are plain CholeskyQR (CholeskyQR2), each X <- X R^{-1}.  chol_rinv_kernel
// factors one Gram matrix in shared memory and returns R^{-1} (upper triangular).  A pivot
// at or below 1e-24 of the largest diagonal entry marks a direction the sketch does not
// contain (a rank-deficient X): its column of R^{-1} is zero, so Q gets a zero column
// there rather than amplified rounding noise, and the later passes keep it zero.
// ---------------------------------------------------------------------------------
struct CholDesc {
    const double* G;
    int ldg;
    double* Rinv;   // k x k, upper triangular (zeros below)
    int ldr;
    int k, rows;
    int shift;      // 1: shifted pass
};

__global__ void __launch_bounds__(256) chol_rinv_kernel(const CholDesc* __restrict__ descs) {
    extern __shared__ double L[];   // k x k, column-major, ld k (lower triangle used); then k flags
    const CholDesc d = descs[blockIdx.x];
    const int k = d.k, tid = threadIdx.x, nt = blockDim.x;
    int* dead = reinterpret_cast<int*>(L + (size_t)k * k);
    __shared__ double s_diag_max, s_shift;
    for (int e = tid; e < k * k; e += nt) {
        const int i = e % k, j = e / k;
        L[e] = i >= j ? d.G[i + (size_t)j * d.ldg] : 0.0;
    }
    for (int j = tid; j < k; j += nt) dead[j] = 0;
    __syncthreads();
    if (tid == 0) {
        double tr = 0.0, mx = 0.0;
        for (int j = 0; j < k; ++j) {
            tr += L[j + (size_t)j * k];
            mx = fmax(mx, L[j + (size_t)j * k]);
        }
        const double u = 1.1102230246251565e-16;
        s_shift = d.shift ? 11.0 * ((double)d.rows * k + (double)k * (k + 1)) * u * tr : 0.0;
        s_diag_max = mx + s_shift;
    }
    __syncthreads();
    if (d.shift)
        for (int j = tid; j < k; j += nt) L[j + (size_t)j * k] += s_shift;
    __syncthreads();
    const double floor_piv = 1e-24 * s_diag_max;
    for (int j = 0; j < k; ++j) {
        // column j: pivot, scale, then the trailing lower triangle
        const double piv = L[j + (size_t)j * k];
        const bool ok = piv > floor_piv && isfinite(piv);
        const double r = ok ? sqrt(piv) : 1.0;
        __syncthreads();
        if (tid == 0) {
            L[j + (size_t)j * k] = r;
            if (!ok) dead[j] = 1;
        }
        for (int i = j + 1 + tid; i < k; i += nt) L[i + (size_t)j * k] = ok ? L[i + (size_t)j * k] / r : 0.0;
        __syncthreads();
        const int m = k - j - 1;
        for (int e = tid; e < m * m; e += nt) {
            const int i = j + 1 + e % m, c = j + 1 + e / m;
            if (i >= c) L[i + (size_t)c * k] -= L[i + (size_t)j * k] * L[c + (size_t)j * k];
        }
        __syncthreads();
    }
    // R^{-1} = (L^{-1})^T: column c of L^{-1} by forward substitution (one thread per
    // column), written as row c of R^{-1}; dead directions give zero columns of R^{-1}
    for (int c = tid; c < k; c += nt) {
        double* out = d.Rinv;
        for (int i = 0; i < k; ++i) {
            double v = 0.0;
            if (i >= c) {
                double acc = i == c ? 1.0 : 0.0;
                for (int t = c; t < i; ++t) acc -= L[i + (size_t)t * k] * out[c + (size_t)t * d.ldr];
                v = acc / L[i + (size_t)i * k];
            }
            out[c + (size_t)i * d.ldr] = v;   // R^{-1}(c, i) = L^{-1}(i, c)
        }
    }
    __syncthreads();
    for (int e = tid; e < k * k; e += nt) {
        const int i = e % k, j = e / k;
        if (dead[j] || dead[i]) d.Rinv[i + (size_t)j * d.ldr] = 0.0;
    }
}

namespace {
struct CholStep : Plan::Step {
    DevTable<CholDesc> t;
    void run(cudaStream_t s, int*) const override {
        if (t.h.empty()) return;
        int kmax = 1;
        for (auto& d : t.h) kmax = std::max(kmax, d.k);
        const size_t smem = (size_t)kmax * kmax * sizeof(double) + (size_t)kmax * sizeof(int);
        static size_t cur = 0;
        ensure_dyn_smem(chol_rinv_kernel, smem, cur);
        chol_rinv_kernel<<<t.size(), 256, smem, s>>>(t.d.p);
        HM_CUDA(cudaGetLastError());
    }
    const char* name() const override { return "cholesky_rinv"; }
    int nlaunch() const override { return t.h.empty() ? 0 : 1; }
};
}  // namespace

void plan_cholqr3(Plan& plan, const std::vector<QrProblem>& probs, cudaStream_t s) {
    if (probs.empty()) return;
    struct W { const QrProblem* p; const double* X; int ldx; };
    std::vector<W> ws;
    for (auto& p : probs)
        if (p.rows > 0 && p.k > 0) ws.push_back({&p, p.X, p.ldx});
    for (int pass = 0; pass < 3; ++pass) {
        auto gram = std::make_unique<GemmStep<double>>("build.cholqr_gram");
        auto chol = std::make_unique<CholStep>();
        auto rot = std::make_unique<GemmStep<double>>("build.cholqr_apply");
        for (auto& w : ws) {
            const int k = w.p->k, m = w.p->rows;
            double* G = plan.scratch((size_t)k * k);
            double* Ri = plan.scratch((size_t)k * k);
            double* Xn = pass == 2 ? w.p->Q : plan.scratch((size_t)m * k);
            const int ldn = pass == 2 ? w.p->ldq : m;
            gram->batch.add(k, k, m, 1.0, w.X, w.ldx, OP_T, w.X, w.ldx, OP_N, 0.0, G, k);
            chol->t.h.push_back({G, k, Ri, k, k, m, pass == 0 ? 1 : 0});
            rot->batch.add(m, k, k, 1.0, w.X, w.ldx, OP_N, Ri, k, OP_N, 0.0, Xn, ldn);
            w.X = Xn;
            w.ldx = ldn;
        }
        gram->batch.finalize(s);
        chol->t.upload(s);
        rot->batch.finalize(s);
        plan.add(std::move(gram));
        plan.add(std::move(chol));
        plan.add(std::move(rot));
    }
}

// Inverses of symmetric positive definite matrices: elimination without pivoting is
// backward stable for them, so the large ones are split 2 x 2 recursively down to
// Gauss-Jordan blocks of order <= 64 (X11 = inv(A11), T = X11 A12, W = A21 X11,
// S = A22 - A21 T, X22 = inv(S), X12 = -T X22, X21 = -X22 W, X11 -= X12 W): fewer,
// larger batched GEMMs than the pivoted sweep.  A zero or non-finite pivot (a matrix that
// was not SPD after all) still raises ST_SINGULAR in the Gauss-Jordan blocks.
void plan_inverse_spd(Plan& plan, const std::vector<InvProblem>& probs, cudaStream_t s) {
    std::vector<InvProblem> small, large;
    for (auto& p : probs) {
        if (p.n <= 0) continue;
        (p.n <= 64 ? small : large).push_back(p);
    }
    if (!small.empty()) plan_inverse(plan, small, s);
    if (large.empty()) return;
    std::vector<InvProblem> sub11, sub22;
    auto copyS = std::make_unique<CopyStep>();
    auto g1 = std::make_unique<GemmStep<double>>("inverse.spd");
    auto g2 = std::make_unique<GemmStep<double>>("inverse.spd");
    auto g3 = std::make_unique<GemmStep<double>>("inverse.spd");
    auto g4 = std::make_unique<GemmStep<double>>("inverse.spd");
    for (auto& p : large) {
        HM_CHECK(p.A != p.X, HM_ERR_ARG, "SPD block inverse cannot run in place");
        const int a = p.n / 2, b = p.n - a;
        const double* A11 = p.A;
        const double* A12 = p.A + (size_t)a * p.lda;
        const double* A21 = p.A + a;
        const double* A22 = p.A + a + (size_t)a * p.lda;
        double* X11 = p.X;
        double* X12 = p.X + (size_t)a * p.ldx;
        double* X21 = p.X + a;
        double* X22 = p.X + a + (size_t)a * p.ldx;
        double* T = plan.scratch((size_t)a * b);
        double* W = plan.scratch((size_t)b * a);
        double* S = plan.scratch((size_t)b * b);
        sub11.push_back({A11, p.lda, X11, p.ldx, a});
        copyS->t.h.push_back({A22, p.lda, S, b, b, b, 0, 0, 0});
        g1->batch.add(a, b, a, 1.0, X11, p.ldx, OP_N, A12, p.lda, OP_N, 0.0, T, a);
        g1->batch.add(b, a, a, 1.0, A21, p.lda, OP_N, X11, p.ldx, OP_N, 0.0, W, b);
        g2->batch.add(b, b, a, -1.0, A21, p.lda, OP_N, T, a, OP_N, 1.0, S, b);
        sub22.push_back({S, b, X22, p.ldx, b});
        g3->batch.add(a, b, b, -1.0, T, a, OP_N, X22, p.ldx, OP_N, 0.0, X12, p.ldx);
        g3->batch.add(b, a, b, -1.0, X22, p.ldx, OP_N, W, b, OP_N, 0.0, X21, p.ldx);
        g4->batch.add(a, a, b, -1.0, X12, p.ldx, OP_N, W, b, OP_N, 1.0, X11, p.ldx);
    }
    copyS->t.upload(s);
    plan.add(std::move(copyS));
    plan_inverse_spd(plan, sub11, s);
    g1->batch.finalize(s);
    plan.add(std::move(g1));
    g2->batch.finalize(s);
    plan.add(std::move(g2));
    plan_inverse_spd(plan, sub22, s);
    g3->batch.finalize(s);
    plan.add(std::move(g3));
    g4->batch.finalize(s);
    plan.add(std::move(g4));
}

void plan_gram_svd(Plan& plan, const std::vector<SvdProblem>& probs, double tol, int max_rank,
                   cudaStream_t s, int rounds) {
    if (probs.empty()) return;
    rounds = std::max(1, rounds);
    struct Work { const SvdProblem* p; const double* X; int ldx; double* Wt; };
    std::vector<Work> w;
    for (auto& p : probs)
        if (p.k > 0 && p.rows > 0) w.push_back({&p, p.X, p.ldx, nullptr});
    if (w.empty()) return;
    for (int r = 0; r < rounds; ++r) {
        auto gram = std::make_unique<GemmStep<double>>();
        auto eig = std::make_unique<EigStep>();
        auto rot = std::make_unique<GemmStep<double>>();
        auto acc = std::make_unique<GemmStep<double>>();
        for (auto& x : w) {
            const int k = x.p->k, m = x.p->rows;
            double* G = plan.scratch((size_t)k * k);
            double* W = plan.scratch((size_t)k * k);
            double* lam = plan.scratch(k);
            double* Xn = plan.scratch((size_t)m * k);
            gram->batch.add(k, k, m, 1.0, x.X, x.ldx, OP_T, x.X, x.ldx, OP_N, 0.0, G, k);
            eig->t.h.push_back({G, k, W, k, lam, k});
            rot->batch.add(m, k, k, 1.0, x.X, x.ldx, OP_N, W, k, OP_N, 0.0, Xn, m);
            if (x.p->R) {
                if (!x.Wt) {
                    x.Wt = W;
                } else {
                    double* Wn = plan.scratch((size_t)k * k);
                    acc->batch.add(k, k, k, 1.0, x.Wt, k, OP_N, W, k, OP_N, 0.0, Wn, k);
                    x.Wt = Wn;
                }
            }
            x.X = Xn;
            x.ldx = m;
        }
        gram->batch.finalize(s);
        eig->t.upload(s);
        rot->batch.finalize(s);
        acc->batch.finalize(s);
        plan.add(std::move(gram));
        plan.add(std::move(eig));
        plan.add(std::move(rot));
        if (!acc->batch.empty()) plan.add(std::move(acc));
    }
    auto nrm = std::make_unique<NormStep>();
    auto prep = std::make_unique<PrepStep>();
    auto perm = std::make_unique<PermStep>();
    prep->tol = tol;
    prep->max_rank = max_rank;
    for (auto& x : w) {
        const SvdProblem& p = *x.p;
        const int k = p.k, m = p.rows;
        double* raw = plan.scratch(k);
        double* sig = p.sigma ? p.sigma : plan.scratch(k);
        int* pm = plan.scratch_i(k);
        nrm->t.h.push_back({x.X, x.ldx, m, k, raw});
        prep->t.h.push_back({raw, sig, pm, p.rank, k});
        if (p.L) perm->t.h.push_back({x.X, x.ldx, p.L, p.ldl, m, k, pm, sig});
        if (p.R) perm->t.h.push_back({x.Wt, k, p.R, p.ldr, k, k, pm, nullptr});
    }
    nrm->t.upload(s);
    prep->t.upload(s);
    perm->t.upload(s);
    plan.add(std::move(nrm));
    plan.add(std::move(prep));
    plan.add(std::move(perm));
}

}  // namespace hm
