// FP64 batched GEMM on the FP64 tensor path (mma.sync m8n8k4 f64), included by
// hm_gemm.cu inside namespace hm after hm_gemm_tile.cuh (it reuses its register stage).
//
// B200 runs FP64 FMA and FP64 MMA at the same peak (measured ~37 TF/s each); one MMA does
// 256 multiply-adds per warp instruction against 32 for a DFMA, so the operand traffic
// per multiply-add through registers and shared memory is 8x lower and the FP64 pipe,
// not instruction issue, sets the pace.
//
// One CTA computes one BM x BN tile of one problem over one k-slice (per-tile problem
// table, split-K by atomics, as the FMA kernel).  WGM x WGN warps, each 32 x 32 outputs:
// 4 x 4 MMA tiles of 8 x 8, accumulators in registers (2 doubles per tile per lane).
// Operands are staged through registers into k-major shared tiles [k][row] whose row
// pitch is 8 (mod 16) doubles: a fragment load (lane -> row lane/4, k lane%4) then spans
// exactly two bank wavefronts.
#pragma once

namespace dmma {

template <int WGM_, int WGN_>
struct Cfg {
    static constexpr int WGM = WGM_, WGN = WGN_;
    static constexpr int NT = 32 * WGM * WGN;
    static constexpr int BM = 32 * WGM, BN = 32 * WGN, BK = 16;
    static constexpr int PA = BM + 8, PB = BN + 8;
    static constexpr size_t smem = 2 * (size_t)BK * (PA + PB) * sizeof(double);
};

template <int BN> struct For;
template <> struct For<128> { using C = Cfg<2, 4>; };
template <> struct For<96> { using C = Cfg<4, 3>; };
template <> struct For<64> { using C = Cfg<4, 2>; };
template <> struct For<32> { using C = Cfg<4, 1>; };

inline int bm_for(int bn) { return bn == 128 ? 64 : 128; }

__device__ __forceinline__ void mma884(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <class CF>
__global__ void __launch_bounds__(CF::NT)
gemm_dmma_kernel(const GemmDesc<double>* __restrict__ descs, const int* __restrict__ tile_problem) {
    constexpr int BM = CF::BM, BN = CF::BN, BK = CF::BK, NT = CF::NT, PA = CF::PA, PB = CF::PB;
    extern __shared__ __align__(16) unsigned char smraw[];
    double* As = reinterpret_cast<double*>(smraw);   // [2][BK][PA]
    double* Bs = As + 2 * BK * PA;                   // [2][BK][PB]

    const int tile = blockIdx.x;
    const GemmDesc<double>& D = descs[tile_problem[tile]];
    const int m = D.m, n = D.n, k = D.k, lda = D.lda, ldb = D.ldb;
    const double* __restrict__ A = D.A;
    const double* __restrict__ B = D.B;
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
    const int nk = ke > kb ? (ke - kb + BK - 1) / BK : 0;

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int wm0 = (w % CF::WGM) * 32, wn0 = (w / CF::WGM) * 32;
    const int fr = lane >> 2, fk = lane & 3;   // fragment row/column and k of this lane

    const bool a_mn = D.opA == OP_N, b_mn = D.opB == OP_T;
    const bool a_vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda % 2 == 0);
    const bool b_vec = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb % 2 == 0);

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    if (nk > 0) {
        tile::Stage<double, BM, BK, NT> sa;
        tile::Stage<double, BN, BK, NT> sb;
        sa.load(A, lda, a_mn, a_vec, m0, m, kb, ke, tid);
        sb.load(B, ldb, b_mn, b_vec, n0, n, kb, ke, tid);
        sa.store(As, PA, a_mn, tid);
        sb.store(Bs, PB, b_mn, tid);
        __syncthreads();
        for (int it = 0; it < nk; ++it) {
            const int buf = it & 1;
            const bool more = it + 1 < nk;
            if (more) {
                const int k1 = kb + (it + 1) * BK;
                sa.load(A, lda, a_mn, a_vec, m0, m, k1, ke, tid);
                sb.load(B, ldb, b_mn, b_vec, n0, n, k1, ke, tid);
            }
            const double* as = As + buf * BK * PA + wm0 + fr;
            const double* bs = Bs + buf * BK * PB + wn0 + fr;
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
            if (more) {
                sa.store(As + (buf ^ 1) * BK * PA, PA, a_mn, tid);
                sb.store(Bs + (buf ^ 1) * BK * PB, PB, b_mn, tid);
            }
            __syncthreads();
        }
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

template <int BN>
void launch(int tiles, cudaStream_t s, const GemmDesc<double>* d, const int* tile_problem) {
    using CF = typename For<BN>::C;
    static size_t cur = 0;
    ensure_dyn_smem(gemm_dmma_kernel<CF>, CF::smem, cur);
    gemm_dmma_kernel<CF><<<tiles, CF::NT, CF::smem, s>>>(d, tile_problem);
}

}  // namespace dmma
