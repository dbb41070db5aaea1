// Warp-tiled batched GEMM for dense operands (FP32 FFMA / FP64 DFMA), included by
// hm_gemm.cu inside namespace hm.
//
// One CTA computes one BM x BN output tile of one problem over one k-slice (a per-tile
// table names the problem).  The CTA
// has WGM x WGN warps; a warp covers (32 UM) x (16 UN) outputs with its lanes on an
// 8 (rows) x 4 (columns) grid, and a lane owns UM x UN blocks of 4 x 4 outputs, each
// made of 16-byte groups (4 floats or 2 doubles) placed so that 8 lanes read 128
// contiguous bytes of A and 4 lanes 64 contiguous bytes of B: every shared-memory read
// is a conflict-free 16-byte vector and the FMA pipe, not shared memory, sets the pace.
//
// Operands are staged through registers: 16-byte global loads along whichever
// dimension is contiguous in memory (the rows of op(A) = A, the k of op(A) = A^T, ...),
// stored into k-major shared tiles ([k][row], rows padded by 4 elements), double
// buffered, with the next k-tile's global loads in flight while the current tile is
// multiplied.  Operands whose base or leading dimension is not 16-byte aligned, and
// ragged edges, take element loads with zero fill.
#pragma once

namespace tile {

template <typename T, int WGM_, int WGN_, int UM_, int UN_, int MINB_ = 0>
struct Cfg {
    static constexpr int WGM = WGM_, WGN = WGN_, UM = UM_, UN = UN_;
    static constexpr int NT = 32 * WGM * WGN;
    // 8-deep k-tiles for the FP64 8 x 8-per-lane shape: its accumulators take half the
    // registers, so the next tile's staging registers must shrink
    static constexpr int BM = 32 * UM * WGM, BN = 16 * UN * WGN, BK = (sizeof(T) == 8 && UM * UN >= 4) ? 8 : 16;
    // padded k-rows: 16 bytes past a multiple of 128 (FP32 +4, FP64 +2 elements), which
    // spreads the transposed stores of k-contiguous operands over the banks and keeps
    // every row 16-byte aligned
    static constexpr int PAD = sizeof(T) == 4 ? 4 : 2;
    static constexpr int PA = BM + PAD, PB = BN + PAD;
    static constexpr size_t smem = 2 * (size_t)BK * (PA + PB) * sizeof(T);
    // resident CTAs per SM the register allocation must allow (default: two for the
    // 256-thread FP32 shapes, which caps registers at 128 without spills)
    static constexpr int MINB = MINB_ > 0 ? MINB_ : ((sizeof(T) == 4 && NT <= 256) ? 2 : 1);
};

// Tile shape per element type and tile width (the widest problem of the batch picks
// the width; ranks are usually <= 96).  Chosen by timing the factor's update shapes
// (m = node rows, n = rank, k = rank; m = n = rank, k = node rows) on B200.
// SHAPE 1: 64-row tiles, for batches of short problems (the many-system workload's leaves
// and nodes of <= 64 rows), where 128-row tiles would be half padding.
// SHAPE 2 (FP64): lanes own 8 x 8 outputs (UM = UN = 2), half the shared-memory reads per
// FMA of the 4 x 8 default at the cost of one CTA per SM.
template <typename T, int BN, int SHAPE = 0> struct For;
template <> struct For<float, 128> { using C = Cfg<float, 2, 4, 2, 2>; };
template <> struct For<float, 96> { using C = Cfg<float, 4, 2, 1, 3>; };
template <> struct For<float, 64> { using C = Cfg<float, 4, 2, 1, 2>; };
template <> struct For<float, 32> { using C = Cfg<float, 4, 2, 2, 1>; };
template <> struct For<double, 128> { using C = Cfg<double, 2, 4, 1, 2, 2>; };
template <> struct For<double, 96> { using C = Cfg<double, 4, 3, 1, 2>; };
template <> struct For<double, 64> { using C = Cfg<double, 4, 2, 1, 2, 2>; };
template <> struct For<double, 32> { using C = Cfg<double, 4, 2, 1, 1>; };
template <> struct For<float, 128, 1> { using C = Cfg<float, 2, 4, 1, 2>; };
template <> struct For<float, 96, 1> { using C = Cfg<float, 2, 3, 1, 2, 2>; };
template <> struct For<float, 64, 1> { using C = Cfg<float, 2, 2, 1, 2, 4>; };
template <> struct For<float, 32, 1> { using C = Cfg<float, 2, 2, 1, 1, 4>; };
template <> struct For<double, 128, 1> { using C = Cfg<double, 2, 4, 1, 2, 2>; };
template <> struct For<double, 96, 1> { using C = Cfg<double, 2, 3, 1, 2, 1>; };
template <> struct For<double, 64, 1> { using C = Cfg<double, 2, 2, 1, 2, 3>; };
template <> struct For<double, 32, 1> { using C = Cfg<double, 2, 2, 1, 1, 4>; };
template <> struct For<double, 128, 2> { using C = Cfg<double, 2, 4, 2, 2, 1>; };
template <> struct For<double, 96, 2> { using C = Cfg<double, 2, 3, 2, 2, 1>; };
template <> struct For<double, 64, 2> { using C = Cfg<double, 2, 2, 2, 2, 1>; };
template <> struct For<double, 32, 2> { using C = Cfg<double, 4, 1, 2, 2, 1>; };
// SHAPE 3: 96-row tiles (three warp rows), for batches whose rows come in multiples of 96
// (projections onto rank-96 bases: m = rank), where 64- or 128-row tiles pad a quarter
template <> struct For<float, 128, 3> { using C = Cfg<float, 3, 4, 1, 2>; };
template <> struct For<float, 96, 3> { using C = Cfg<float, 3, 2, 1, 3, 2>; };
template <> struct For<float, 64, 3> { using C = Cfg<float, 3, 2, 1, 2, 3>; };
template <> struct For<float, 32, 3> { using C = Cfg<float, 3, 2, 1, 1, 4>; };
template <> struct For<double, 128, 3> { using C = Cfg<double, 3, 4, 1, 2, 1>; };
template <> struct For<double, 96, 3> { using C = Cfg<double, 3, 2, 1, 3, 1>; };
template <> struct For<double, 64, 3> { using C = Cfg<double, 3, 2, 1, 2, 2>; };
template <> struct For<double, 32, 3> { using C = Cfg<double, 3, 2, 1, 1, 3>; };

// SHAPE 2 exists for FP64 only (FP32 batches fall back to SHAPE 0)
inline int shape_for(size_t elem, int shape) { return (shape == 2 && elem == 4) ? 0 : shape; }

inline int bm_for(size_t elem, int bn, int shape = 0) {
    shape = shape_for(elem, shape);
    if (shape == 1) return 64;
    if (shape == 3) return 96;
    if (shape == 2) return bn == 32 ? 256 : 128;
    if (elem == 4) return bn == 32 ? 256 : 128;
    return bn == 128 ? 64 : 128;
}

// one 16-byte vector (4 floats or 2 doubles)
template <typename T>
__device__ __forceinline__ void ld16(const T* p, T* o) {
    if constexpr (sizeof(T) == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
    } else {
        const double2 t = *reinterpret_cast<const double2*>(p);
        o[0] = t.x; o[1] = t.y;
    }
}
template <typename T>
__device__ __forceinline__ void st16(T* p, const T* v) {
    if constexpr (sizeof(T) == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}

// Register stage of one operand tile: BMN indices of op(X)'s row (A) or column (B)
// dimension by BK k-values.  mn_contig: element (r, k) is X[r + k*ld], else X[k + r*ld].
template <typename T, int BMN, int BK, int NT>
struct Stage {
    static constexpr int VW = 16 / (int)sizeof(T);
    static constexpr int NVEC = BMN * BK / VW;
    static constexpr int NV = (NVEC + NT - 1) / NT;
    static_assert(BMN % VW == 0 && BK % VW == 0, "vector width");
    T v[NV][VW];

    __device__ __forceinline__ void map(int e, bool mn_contig, int& r, int& kk) const {
        if (mn_contig) { r = (e % (BMN / VW)) * VW; kk = e / (BMN / VW); }
        else { kk = (e % (BK / VW)) * VW; r = e / (BK / VW); }
    }

    __device__ __forceinline__ void load(const T* __restrict__ X, int ld, bool mn_contig, bool vec_ok,
                                         int r0, int rmax, int k0, int ke, int tid) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const int e = tid + NT * q;
            if (NVEC % NT != 0 && e >= NVEC) continue;
            int r, kk;
            map(e, mn_contig, r, kk);
            const int gr = r0 + r, gk = k0 + kk;
            if (mn_contig) {
                const bool kin = gk < ke;
                if (vec_ok && kin && gr + VW <= rmax) {
                    ld16(X + gr + (size_t)gk * ld, v[q]);
                } else {
#pragma unroll
                    for (int u = 0; u < VW; ++u)
                        v[q][u] = (kin && gr + u < rmax) ? X[gr + u + (size_t)gk * ld] : T(0);
                }
            } else {
                const bool rin = gr < rmax;
                if (vec_ok && rin && gk + VW <= ke) {
                    ld16(X + gk + (size_t)gr * ld, v[q]);
                } else {
#pragma unroll
                    for (int u = 0; u < VW; ++u)
                        v[q][u] = (rin && gk + u < ke) ? X[gk + u + (size_t)gr * ld] : T(0);
                }
            }
        }
    }

    __device__ __forceinline__ void store(T* s, int P, bool mn_contig, int tid) const {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const int e = tid + NT * q;
            if (NVEC % NT != 0 && e >= NVEC) continue;
            int r, kk;
            map(e, mn_contig, r, kk);
            if (mn_contig) {
                st16(s + kk * P + r, v[q]);
            } else {
#pragma unroll
                for (int u = 0; u < VW; ++u) s[(kk + u) * P + r] = v[q][u];
            }
        }
    }
};

// The main loop of gemm_tile_kernel for one chained problem (whole k), accumulating
// into the caller's registers: only the chain instantiation uses it.
template <typename T, class CF>
__device__ __forceinline__ void chain_mainloop(const GemmDesc<T>& P, int m, int n, int m0, int n0, int am, int bn,
                                               T* As, T* Bs, T (&acc)[4 * CF::UM][4 * CF::UN]) {
    constexpr int BK = CF::BK, NT = CF::NT, PA = CF::PA, PB = CF::PB, UM = CF::UM, UN = CF::UN;
    constexpr int VW = 16 / (int)sizeof(T);
    constexpr int NG = 4 / VW;
    const int tid = threadIdx.x;
    const int k = P.k, lda = P.lda, ldb = P.ldb;
    const T* __restrict__ A = P.A;
    const T* __restrict__ B = P.B;
    const bool a_mn = P.opA == OP_N, b_mn = P.opB == OP_T;
    const bool a_vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda % VW == 0);
    const bool b_vec = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb % VW == 0);
    const int nk = (k + BK - 1) / BK;
    if (nk <= 0) return;
    Stage<T, CF::BM, BK, NT> sa;
    Stage<T, CF::BN, BK, NT> sb;
    sa.load(A, lda, a_mn, a_vec, m0, m, 0, k, tid);
    sb.load(B, ldb, b_mn, b_vec, n0, n, 0, k, tid);
    sa.store(As, PA, a_mn, tid);
    sb.store(Bs, PB, b_mn, tid);
    __syncthreads();
    for (int it = 0; it < nk; ++it) {
        const int buf = it & 1;
        const bool more = it + 1 < nk;
        if (more) {
            const int k1 = (it + 1) * BK;
            sa.load(A, lda, a_mn, a_vec, m0, m, k1, k, tid);
            sb.load(B, ldb, b_mn, b_vec, n0, n, k1, k, tid);
        }
        const T* as = As + buf * BK * PA + am;
        const T* bs = Bs + buf * BK * PB + bn;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T a[4 * UM], b[4 * UN];
#pragma unroll
            for (int u = 0; u < UM; ++u)
#pragma unroll
                for (int g = 0; g < NG; ++g) ld16(as + kk * PA + 32 * u + g * 8 * VW, a + 4 * u + g * VW);
#pragma unroll
            for (int v = 0; v < UN; ++v)
#pragma unroll
                for (int g = 0; g < NG; ++g) ld16(bs + kk * PB + 16 * v + g * 4 * VW, b + 4 * v + g * VW);
#pragma unroll
            for (int i = 0; i < 4 * UM; ++i)
#pragma unroll
                for (int j = 0; j < 4 * UN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (more) {
            sa.store(As + (buf ^ 1) * BK * PA, PA, a_mn, tid);
            sb.store(Bs + (buf ^ 1) * BK * PB, PB, b_mn, tid);
        }
        __syncthreads();
    }
}

// CHAIN: after the head problem, follow GemmDesc::next (problems accumulated into the
// head's tile; one CTA per SM of register budget, so the chain's extra state does not
// spill); the plain instantiation is the single-problem kernel.
template <typename T, class CF, bool CHAIN = false>
__global__ void __launch_bounds__(CF::NT, CHAIN ? 1 : CF::MINB)
gemm_tile_kernel(const GemmDesc<T>* __restrict__ descs, const int* __restrict__ tile_problem) {
    constexpr int BM = CF::BM, BN = CF::BN, BK = CF::BK, NT = CF::NT;
    constexpr int PA = CF::PA, PB = CF::PB, UM = CF::UM, UN = CF::UN;
    constexpr int VW = 16 / (int)sizeof(T);
    extern __shared__ __align__(16) unsigned char smraw[];
    T* As = reinterpret_cast<T*>(smraw);   // [2][BK][PA]
    T* Bs = As + 2 * BK * PA;              // [2][BK][PB]

    // tile -> problem from a per-tile table: two dependent loads instead of a search
    const int tile = blockIdx.x;
    const GemmDesc<T>& D = descs[tile_problem[tile]];
    const int m = D.m, n = D.n, k = D.k, lda = D.lda, ldb = D.ldb;
    const T* __restrict__ A = D.A;
    const T* __restrict__ B = D.B;
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

    // A lane's 4 rows of a 32-row block are NG groups of VW contiguous rows (16 bytes):
    // group g starts at g*8*VW + lx*VW, so 8 lanes read 128 contiguous bytes.  Columns
    // of a 16-column block likewise: group g at g*4*VW + ly*VW.
    constexpr int NG = 4 / VW;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int am = (w % CF::WGM) * 32 * UM + (lane & 7) * VW;
    const int bn = (w / CF::WGM) * 16 * UN + (lane >> 3) * VW;

    const bool a_mn = D.opA == OP_N, b_mn = D.opB == OP_T;
    const bool a_vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda % VW == 0);
    const bool b_vec = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb % VW == 0);

    // the epilogue reads C when beta != 0: start bringing this thread's C lines into L2
    if (D.beta != T(0) && D.ksplit == 1) {
        const T* Cp = D.C;
#pragma unroll
        for (int u = 0; u < UM; ++u)
#pragma unroll
            for (int gu = 0; gu < NG; ++gu) {
                const int gi = m0 + am + 32 * u + gu * 8 * VW;
                if (gi >= m) continue;
#pragma unroll
                for (int v = 0; v < UN; ++v)
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj) {
                        const int gj = n0 + bn + 16 * v + (jj / VW) * 4 * VW + (jj % VW);
                        if (gj < n)
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(Cp + gi + (size_t)gj * D.ldc));
                    }
            }
    }

    T acc[4 * UM][4 * UN];
#pragma unroll
    for (int i = 0; i < 4 * UM; ++i)
#pragma unroll
        for (int j = 0; j < 4 * UN; ++j) acc[i][j] = T(0);

    if (nk > 0) {
        Stage<T, BM, BK, NT> sa;
        Stage<T, BN, BK, NT> sb;
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
            const T* as = As + buf * BK * PA + am;
            const T* bs = Bs + buf * BK * PB + bn;
#pragma unroll
            for (int kk = 0; kk < BK; ++kk) {
                T a[4 * UM], b[4 * UN];
#pragma unroll
                for (int u = 0; u < UM; ++u)
#pragma unroll
                    for (int g = 0; g < NG; ++g) ld16(as + kk * PA + 32 * u + g * 8 * VW, a + 4 * u + g * VW);
#pragma unroll
                for (int v = 0; v < UN; ++v)
#pragma unroll
                    for (int g = 0; g < NG; ++g) ld16(bs + kk * PB + 16 * v + g * 4 * VW, b + 4 * v + g * VW);
#pragma unroll
                for (int i = 0; i < 4 * UM; ++i)
#pragma unroll
                    for (int j = 0; j < 4 * UN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
            }
            if (more) {
                sa.store(As + (buf ^ 1) * BK * PA, PA, a_mn, tid);
                sb.store(Bs + (buf ^ 1) * BK * PB, PB, b_mn, tid);
            }
            __syncthreads();
        }
    }

    if constexpr (CHAIN) {
        for (int nx = D.next; nx >= 0; nx = descs[nx].next)
            chain_mainloop<T, CF>(descs[nx], m, n, m0, n0, am, bn, As, Bs, acc);
    }

    T* __restrict__ C = D.C;
    const int ldc = D.ldc;
    const T alpha = D.alpha, beta = D.beta;
    const bool split = D.ksplit > 1;
    const bool c_vec = ((reinterpret_cast<uintptr_t>(C) & 15) == 0) && (ldc % VW == 0);
#pragma unroll
    for (int u = 0; u < UM; ++u) {
#pragma unroll
        for (int gu = 0; gu < NG; ++gu) {
            const int gi = m0 + am + 32 * u + gu * 8 * VW;
            if (gi >= m) continue;
#pragma unroll
            for (int v = 0; v < UN; ++v) {
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    const int gj = n0 + bn + 16 * v + (jj / VW) * 4 * VW + (jj % VW);
                    if (gj >= n) continue;
                    T* c = C + gi + (size_t)gj * ldc;
                    T val[VW];
#pragma unroll
                    for (int r = 0; r < VW; ++r) val[r] = alpha * acc[4 * u + gu * VW + r][4 * v + jj];
                    if (split) {
#pragma unroll
                        for (int r = 0; r < VW; ++r)
                            if (gi + r < m) atomicAdd(c + r, val[r]);
                    } else if (c_vec && gi + VW <= m) {
                        if (beta != T(0)) {
                            T old[VW];
                            ld16(c, old);
#pragma unroll
                            for (int r = 0; r < VW; ++r) val[r] = fma(beta, old[r], val[r]);
                        }
                        st16(c, val);
                    } else {
#pragma unroll
                        for (int r = 0; r < VW; ++r) {
                            if (gi + r >= m) continue;
                            c[r] = (beta == T(0)) ? val[r] : fma(beta, c[r], val[r]);
                        }
                    }
                }
            }
        }
    }
}

template <typename T, int BN, int SHAPE = 0, bool CHAIN = false>
void launch(int tiles, cudaStream_t s, const GemmDesc<T>* d, const int* tile_problem) {
    using CF = typename For<T, BN, SHAPE>::C;
    static size_t cur = 0;
    ensure_dyn_smem(gemm_tile_kernel<T, CF, CHAIN>, CF::smem, cur);
    gemm_tile_kernel<T, CF, CHAIN><<<tiles, CF::NT, CF::smem, s>>>(d, tile_problem);
}

}  // namespace tile
