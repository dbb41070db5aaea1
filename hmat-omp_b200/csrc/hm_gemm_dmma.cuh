// FP64 batched GEMM on the FP64 tensor path (mma.sync m8n8k4 f64), included by
// hm_gemm.cu inside namespace hm after hm_gemm_tile.cuh.  Same problem tables as the
// warp-tiled kernel (per-tile problem index, split-K by atomics, chained problems).
//
// B200 issues FP64 MMA at the same peak as DFMA (~37 TF/s), but one m8n8k4 MMA does 256
// multiply-adds per warp instruction from one A and one B element per lane: with a warp
// computing 32 x 32 outputs (4 x 4 MMA tiles) it reads 8 doubles per lane from shared
// memory per 16 MMAs (4096 multiply-adds), a quarter of what the FMA kernel's register
// tiles read, so neither shared-memory bandwidth nor instruction issue sets the pace.
//
// Operands go global -> shared with cp.async (16-byte copies along a contiguous column of
// an MN-major operand, 8-byte copies transposed into place for a k-contiguous one, zero
// fill past the edges) through an ST-stage ring of [k][row] buffers whose row pitch is
// 8 (mod 16) doubles.  A fragment read (lane -> row lane/4, k lane%4) then touches each
// bank pair at most twice, the minimum for 32 x 8 bytes.
#pragma once

namespace dmma {

constexpr int BK = 16;

template <int WGM_, int WGN_, int ST_>
struct Cfg {
    static constexpr int WGM = WGM_, WGN = WGN_, ST = ST_;
    static constexpr int NT = 32 * WGM * WGN;
    static constexpr int BM = 32 * WGM, BN = 32 * WGN;
    static constexpr int PA = BM + 8, PB = BN + 8;
    static constexpr size_t smem = (size_t)ST * BK * (PA + PB) * sizeof(double);
};

template <int BN> struct For;
template <> struct For<32> { using C = Cfg<4, 1, 4>; };
template <> struct For<64> { using C = Cfg<2, 2, 4>; };
template <> struct For<96> { using C = Cfg<2, 3, 4>; };
template <> struct For<128> { using C = Cfg<2, 4, 4>; };

inline int bm_for(int bn) { return bn == 32 ? 128 : 64; }

__device__ __forceinline__ void mma884(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// cp.async of `bytes` (0, 8 or 16) valid bytes into a 16-byte slot, the rest zero-filled
__device__ __forceinline__ void cp16(double* s, const double* g, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"((unsigned)__cvta_generic_to_shared(s)),
                 "l"(g), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp8(double* s, const double* g, int bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"((unsigned)__cvta_generic_to_shared(s)),
                 "l"(g), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wait_groups() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// k-tile [k0, k0 + BK) of rows [r0, r0 + ROWS) of op(X) into s ([k][row], pitch P);
// rows >= rmax and k >= ke read as zero.  mn: X[r + k ld] (rows contiguous), else
// X[k + r ld].  vec: X 16-byte aligned and ld even (16-byte copies of row pairs).
template <int ROWS, int NT>
__device__ __forceinline__ void issue(double* s, int P, const double* __restrict__ X, int ld, bool mn, bool vec,
                                      int r0, int rmax, int k0, int ke, int tid) {
    if (mn && vec) {
        constexpr int NG = ROWS / 2 * BK;
#pragma unroll
        for (int q = 0; q < (NG + NT - 1) / NT; ++q) {
            const int e = tid + NT * q;
            if (NG % NT != 0 && e >= NG) break;
            const int kk = e / (ROWS / 2), r = 2 * (e % (ROWS / 2));
            const int gr = r0 + r, gk = k0 + kk;
            int bytes = 0;
            const double* src = X;
            if (gk < ke && gr < rmax) {
                bytes = gr + 1 < rmax ? 16 : 8;
                src = X + gr + (size_t)gk * ld;
            }
            cp16(s + kk * P + r, src, bytes);
        }
    } else {
        constexpr int NE = ROWS * BK;
#pragma unroll
        for (int q = 0; q < (NE + NT - 1) / NT; ++q) {
            const int e = tid + NT * q;
            if (NE % NT != 0 && e >= NE) break;
            int kk, r;
            if (mn) { kk = e / ROWS; r = e % ROWS; } else { r = e / BK; kk = e % BK; }
            const int gr = r0 + r, gk = k0 + kk;
            const bool v = gr < rmax && gk < ke;
            cp8(s + kk * P + r, v ? X + (mn ? gr + (size_t)gk * ld : gk + (size_t)gr * ld) : X, v ? 8 : 0);
        }
    }
}

template <class CF, bool CHAIN>
__global__ void __launch_bounds__(CF::NT)
gemm_dmma_kernel(const GemmDesc<double>* __restrict__ descs, const int* __restrict__ tile_problem) {
    constexpr int BM = CF::BM, BN = CF::BN, NT = CF::NT, PA = CF::PA, PB = CF::PB, ST = CF::ST;
    extern __shared__ __align__(16) unsigned char smraw[];
    double* As = reinterpret_cast<double*>(smraw);   // [ST][BK][PA]
    double* Bs = As + ST * BK * PA;                  // [ST][BK][PB]

    const int tile = blockIdx.x;
    const GemmDesc<double>& D = descs[tile_problem[tile]];
    const int m = D.m, n = D.n;
    int t = tile - D.tile0;
    const int tm = t % D.tiles_m;
    t /= D.tiles_m;
    const int tn = t % D.tiles_n;
    const int kslice = t / D.tiles_n;
    const int m0 = tm * BM, n0 = tn * BN;

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int wm0 = (w % CF::WGM) * 32, wn0 = (w / CF::WGM) * 32;
    const int fr = lane >> 2, fk = lane & 3;

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    // acc += op(A)[m0.., kb:ke) op(B)[kb:ke), n0..)
    auto mainloop = [&](const GemmDesc<double>& P, int kb, int ke) {
        const int nk = ke > kb ? (ke - kb + BK - 1) / BK : 0;
        if (nk <= 0) return;
        const double* __restrict__ A = P.A;
        const double* __restrict__ B = P.B;
        const int lda = P.lda, ldb = P.ldb;
        const bool a_mn = P.opA == OP_N, b_mn = P.opB == OP_T;
        const bool a_vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda % 2 == 0);
        const bool b_vec = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb % 2 == 0);
#pragma unroll
        for (int s = 0; s < ST - 1; ++s) {
            if (s < nk) {
                issue<BM, NT>(As + s * BK * PA, PA, A, lda, a_mn, a_vec, m0, m, kb + s * BK, ke, tid);
                issue<BN, NT>(Bs + s * BK * PB, PB, B, ldb, b_mn, b_vec, n0, n, kb + s * BK, ke, tid);
            }
            commit();
        }
        for (int it = 0; it < nk; ++it) {
            wait_groups<ST - 2>();   // this thread's copies of k-tile `it` have landed
            __syncthreads();         // everyone's have, and everyone is done with tile it - 1
            const int nx = it + ST - 1;
            if (nx < nk) {
                const int b = nx % ST;
                issue<BM, NT>(As + b * BK * PA, PA, A, lda, a_mn, a_vec, m0, m, kb + nx * BK, ke, tid);
                issue<BN, NT>(Bs + b * BK * PB, PB, B, ldb, b_mn, b_vec, n0, n, kb + nx * BK, ke, tid);
            }
            commit();
            const double* as = As + (it % ST) * BK * PA + wm0 + fr;
            const double* bs = Bs + (it % ST) * BK * PB + wn0 + fr;
#pragma unroll
            for (int k4 = 0; k4 < BK; k4 += 4) {
                double a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = as[(k4 + fk) * PA + 8 * i];
#pragma unroll
                for (int j = 0; j < 4; ++j) b[j] = bs[(k4 + fk) * PB + 8 * j];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) mma884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
            }
        }
        wait_groups<0>();
        __syncthreads();   // the ring is free for the next problem of a chain
    };

    {
        int kper = (D.k + D.ksplit - 1) / D.ksplit;
        kper = (kper + BK - 1) / BK * BK;
        const int kb = kslice * kper;
        mainloop(D, kb, min(D.k, kb + kper));
    }
    if constexpr (CHAIN) {
        for (int nx = D.next; nx >= 0; nx = descs[nx].next) mainloop(descs[nx], 0, descs[nx].k);
    }

    // lane holds rows wm0 + 8i + lane/4, columns wn0 + 8j + 2 (lane%4) + {0, 1}
    double* __restrict__ C = D.C;
    const int ldc = D.ldc;
    const double alpha = D.alpha, beta = D.beta;
    const bool split = D.ksplit > 1;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gi = m0 + wm0 + 8 * i + fr;
        if (gi >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = n0 + wn0 + 8 * j + 2 * fk + h;
                if (gj >= n) continue;
                double* c = C + gi + (size_t)gj * ldc;
                const double v = alpha * acc[i][j][h];
                if (split) atomicAdd(c, v);
                else *c = (beta == 0.0) ? v : fma(beta, *c, v);
            }
        }
    }
}

template <int BN, bool CHAIN>
void launch(int tiles, cudaStream_t s, const GemmDesc<double>* d, const int* tile_problem) {
    using CF = typename For<BN>::C;
    static size_t cur = 0;
    ensure_dyn_smem(gemm_dmma_kernel<CF, CHAIN>, CF::smem, cur);
    gemm_dmma_kernel<CF, CHAIN><<<tiles, CF::NT, CF::smem, s>>>(d, tile_problem);
}

}  // namespace dmma
