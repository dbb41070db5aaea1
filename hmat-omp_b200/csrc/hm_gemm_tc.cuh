// FP32 batched GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32), included
// by hm_gemm.cu inside namespace hm.
//
// Precision: every operand element x is split in shared memory into two TF32 values,
// hi = tf32_rn(x) and lo = tf32_rn(x - hi) (together x to a relative 2^-23), and all four
// partial products are accumulated in FP32 in two tensor-memory accumulators,
//     main = sum A_hi B_hi,   correction = sum (A_lo B_lo + A_lo B_hi + A_hi B_lo),
// added in the epilogue.  The tensor core's FP32 accumulation error grows with the number
// of MMAs chained into one accumulator; keeping the three small products out of the main
// chain (and the lo x lo term in) brings the result to the accuracy of an FP32 FMA GEMM,
// which the mixed-precision factorization needs to keep its refinement contraction.  The
// MMAs are not this kernel's bottleneck, so the extra products cost little.
//
// Structure: a persistent kernel, one CTA per SM, tiles of BM = 128 rows by BN columns
// assigned round-robin (blockIdx.x + i * gridDim.x) from the same per-tile problem table
// as the FMA kernel.  Warp roles, decoupled by mbarriers:
//   warp 0     TMA producer (one lane): per k-block (32 deep) the tiles of op(A) and op(B)
//              by tensor maps (two per problem, encoded on the host when the batch is
//              finalized), into a stage laid out as the UMMA swizzled canonical layout
//              that matches the operand's contiguous dimension in global memory
//              (K-major, 128-byte swizzle, when k is contiguous; MN-major, 128-byte
//              swizzle with 32-byte granules, when rows/columns are); out-of-range rows
//              and k are zero-filled by the TMA.
//   warps 1..NCW converters (8, or 12 for generated-A batches): the hi/lo
//              split of a landed stage, hi in place and lo into a twin buffer; up to 4
//              stages in flight.
//   warp NCW+1 allocates the tensor memory (two accumulator buffers) and one lane issues the
//              MMAs: per k-block 4 k-steps x 4 products of 128 x BN x 8, then a commit
//              that frees the stage; after a tile's last k-block, a commit that hands the
//              accumulator to the epilogue.
//   the rest   epilogue: 4 warps, or for short-k batches 8 (two per TMEM lane quarter,
//              each taking half of the tile's columns): tcgen05.ld of the main and correction accumulators
//              (one wait per 16 columns) into the shared C tile (loaded first by TMA when
//              beta != 0: C = alpha acc + beta C), released accumulator, then one TMA store
//              of the tile (a TMA reduce-add for split-K), so a tile's epilogue overlaps
//              the next tile's MMAs.  (With four warps the epilogue bounded short-k tiles:
//              the MMA thread waited for a free accumulator 60% of the time.)
// Every wait on an mbarrier gives up after about a second of clock, sets ST_TIMEOUT in
// the status word and makes all roles leave; the tensor memory is always released.
// Teardown waits (copies and MMAs already issued) keep the one-second bound even when a
// role wait gave up early.  A stall switch (tests of this path only) makes the producer
// issue nothing and shortens the role waits, so they run out with nothing in flight.
#pragma once

namespace tc {

constexpr int BM = 128, BK = 32;
// Warps: 0 the TMA producer, 1..NCW the converters, NCW + 1 the MMA issuer, then EPW
// epilogue warps.  Threads of such a CTA:
template <int EPW, int NCW>
constexpr int nthreads() { return (NCW + 2 + EPW) * 32; }

template <int BN>
struct Shape {
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 128, "tile width");
    static constexpr int A_BYTES = BM * BK * 4;
    static constexpr int B_BYTES = BN * BK * 4;
    // stage: A (hi in place), A lo, B (hi in place), B lo
    static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int C_BYTES = BM * BN * 4;   // the epilogue's C tile (beta != 0)
    // as many stages (up to 4) as fit the 227 KB a CTA may hold, after the C tile,
    // alignment slack and the barrier area
    static constexpr int ST_FIT = (232448 - 1024 - 256 - C_BYTES) / STAGE;
    static constexpr int ST = ST_FIT < 4 ? ST_FIT : 4;
    static_assert(ST >= 2, "stages");
    // an accumulator buffer = main (hi x hi) + correction columns; two buffers
    static constexpr int HALF_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : 128;
    static constexpr int ACC_COLS = 2 * HALF_COLS;
    static constexpr int TMEM_COLS = 2 * ACC_COLS;
    static constexpr size_t SMEM = (size_t)ST * STAGE + C_BYTES + 1024 + 256;
};

// ---- shared layouts written by the TMA (and read by the MMA descriptors) ----
// K-major operand, box {32 k, R rows}, 128-byte swizzle: row r is a 128-byte line at
//   r * 128 whose 16-byte chunks are XOR-ed with r % 8 (8-row atoms of 1 KB).
// MN-major operand, R/32 boxes {32 rows, 32 k}, 128-byte swizzle with 32-byte granules:
//   box c at c * 4096; in it, k-line k is 128 bytes at k * 128 whose 32-byte granules are
//   XOR-ed with k % 4 (4-line atoms of 512 bytes).
// ---- PTX wrappers ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// TMA: 2-D tile of the tensor map at coordinates (x, y) into shared memory, completing
// transaction bytes on barrier b
__device__ __forceinline__ void tma2d(uint32_t dst, const void* tmap, int x, int y, uint32_t b) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
        "l"(tmap), "r"(x), "r"(y), "r"(b)
        : "memory");
}
// TMA: prefetch a tile of global memory into L2 (no shared memory, no completion)
__device__ __forceinline__ void tma2d_prefetch(const void* tmap, int x, int y) {
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];\n" ::"l"(tmap), "r"(x), "r"(y)
                 : "memory");
}
// TMA: shared tile -> global (store), or added into global (reduce-add), as a bulk group
__device__ __forceinline__ void tma2d_store(const void* tmap, int x, int y, uint32_t src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(tmap),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
}
__device__ __forceinline__ void tma2d_add(const void* tmap, int x, int y, uint32_t src) {
    asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(tmap),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect(uint32_t b, uint32_t bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(b), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t b, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(b), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t b) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(b) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(b), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Shared-memory matrix descriptor: start >> 4 | LBO >> 4 << 16 | SBO >> 4 << 32 |
// version 1 << 46 | layout << 61 (2: 128-byte swizzle, K-major here; 1: 128-byte swizzle
// with 32-byte granules, MN-major here).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}
__device__ __forceinline__ uint32_t idesc_tf32(bool a_mn, bool b_mn, int n) {
    // D f32 (bits 4-5 = 1), A/B tf32 (2 at bits 7-9, 10-12), majors (15, 16), N >> 3 (17-22), M >> 4 (24-28)
    return (1u << 4) | (2u << 7) | (2u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
// Two 16-column loads (the main and the correction accumulator) and one wait.
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, float* v, float* w) {
    uint32_t r[16], q[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(ta)
        : "memory");
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
          "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]), "=r"(q[15])
        : "r"(tb)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        v[i] = __uint_as_float(r[i]);
        w[i] = __uint_as_float(q[i]);
    }
}
__device__ __forceinline__ float lds_f32(uint32_t a) {
    float x;
    asm volatile("ld.shared.f32 %0, [%1];\n" : "=f"(x) : "r"(a));
    return x;
}
__device__ __forceinline__ void sts_f32(uint32_t a, float x) {
    asm volatile("st.shared.f32 [%0], %1;\n" ::"r"(a), "f"(x) : "memory");
}
__device__ __forceinline__ float tf32_rn(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Clock cycles a role wait (wait_bar) polls before it gives up: about a second.
constexpr long long ROLE_WAIT_CYCLES = 2000000000ll;
// With the stall switch (a test of the timeout path, set only through the batched-GEMM
// entry point's HM_GEMM_TEST_STALL flag) the producer issues no copy and the role waits
// give up after this many cycles instead (~0.5 ms).
constexpr long long STALL_WAIT_CYCLES = 1ll << 20;

// Wait for phase `parity` of barrier b, at most `limit` cycles; false on timeout (and
// the CTA-wide abort flag is raised).
__device__ __forceinline__ bool wait_bar(uint32_t b, uint32_t parity, volatile int* abort_flag, int* status,
                                         long long limit) {
    if (mbar_try(b, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (mbar_try(b, parity)) return true;
        if (*abort_flag) return false;
        if (clock64() - t0 > limit) {
            *abort_flag = 1;
            atomicOr(status, ST_TIMEOUT);
            return false;
        }
    }
}

// Teardown wait: ignores the abort flag (copies or MMAs this thread started must land
// before the CTA exits or frees tensor memory) but still gives up after about a second.
__device__ __forceinline__ void wait_bar_final(uint32_t b, uint32_t parity, int* status) {
    if (mbar_try(b, parity)) return;
    const long long t0 = clock64();
    while (!mbar_try(b, parity)) {
        if (clock64() - t0 > 2000000000ll) {
            atomicOr(status, ST_TIMEOUT);
            return;
        }
    }
}

// The same wait taken by a whole warp: lane 0 polls, the warp follows its verdict
// (keeps the warp converged for the .sync.aligned tensor-memory loads that follow).
__device__ __forceinline__ bool wait_bar_warp(uint32_t b, uint32_t parity, volatile int* abort_flag, int* status,
                                              long long limit) {
    int ok = 0;
    if ((threadIdx.x & 31) == 0) ok = wait_bar(b, parity, abort_flag, status, limit) ? 1 : 0;
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// Entry (r, c) of a generated operator for the tensor-core path: coordinate differences
// and squared distances in FP64 (no cancellation for close points), the exp / sqrt /
// reciprocal in FP32 (the hi/lo TF32 split carries FP32 accuracy, no more).
template <int GEN>
__device__ __forceinline__ float gen_entry_f32(const GenParams& g, int r, int c) {
    const double p0 = g.p0v ? g.p0v[g.row_sys[r]] : g.p0;
    const double p1 = g.p1v ? g.p1v[g.row_sys[r]] : g.p1;
    float v = 0.f;
    if constexpr (GEN == GEN_CAUCHY) {
        v = 1.0f / (float)(g.pts[r] - g.pts[g.N + c]);
        if (r == c) v += (float)p0;
    } else {
        double d2 = 0.0;
        for (int t = 0; t < g.dim; ++t) {
            const double d = g.pts[(size_t)r * g.dim + t] - g.pts[(size_t)c * g.dim + t];
            d2 = fma(d, d, d2);
        }
        if constexpr (GEN == GEN_GAUSSIAN) {
            v = __expf(-(float)(d2 / (2.0 * p0 * p0)));
        } else {
            v = 1.0f / (sqrtf((float)d2) + (float)p0);
        }
        if (r == c) v += (float)p1;
    }
    return v;
}

// The same entry from a squared distance d2 (symmetric kernels; r, c: global indices).
template <int GEN>
__device__ __forceinline__ float gen_from_d2(const GenParams& g, int r, int c, double d2) {
    const double p0 = g.p0v ? g.p0v[g.row_sys[r]] : g.p0;
    float v;
    if constexpr (GEN == GEN_GAUSSIAN) v = __expf(-(float)(d2 / (2.0 * p0 * p0)));
    else v = 1.0f / (sqrtf((float)d2) + (float)p0);
    if (r == c) v += (float)(g.p1v ? g.p1v[g.row_sys[r]] : g.p1);
    return v;
}

// C goes through the TMA (load for beta != 0, store / reduce-add) only when aligned;
// otherwise the epilogue reads and writes it row by row
__host__ __device__ inline bool c_tma_ok(const float* C, int ldc) {
    return (reinterpret_cast<uintptr_t>(C) & 15) == 0 && ldc % 4 == 0;
}

// Tile of this CTA -> problem, origin and k-range (same split rules as the FMA kernel).
struct TileInfo {
    int p, m0, n0, kb, ke, nk;
};
template <int BN>
__device__ __forceinline__ TileInfo decode(const GemmDesc<float>* __restrict__ descs,
                                           const int* __restrict__ tile_problem, int tile) {
    TileInfo t;
    t.p = tile_problem[tile];
    const GemmDesc<float>& D = descs[t.p];
    int r = tile - D.tile0;
    const int tm = r % D.tiles_m;
    r /= D.tiles_m;
    const int tn = r % D.tiles_n;
    const int ks = r / D.tiles_n;
    t.m0 = tm * BM;
    t.n0 = tn * BN;
    int kper = (D.k + D.ksplit - 1) / D.ksplit;
    kper = (kper + BK - 1) / BK * BK;
    t.kb = ks * kper;
    t.ke = min(D.k, t.kb + kper);
    t.nk = t.ke > t.kb ? (t.ke - t.kb + BK - 1) / BK : 0;
    return t;
}

// GEN != GEN_DENSE: A is not read from memory but evaluated by the converter warps from
// the kernel generator (entry (ga_r0 + i, ga_c0 + k) of op(A), or its transpose for
// opA = OP_T) straight into the K-major stage layout; the TMA brings only B.
template <int BN, int GEN, int EPW, int NCW>
__global__ void __launch_bounds__(nthreads<EPW, NCW>(), 1)
gemm_tc32_kernel(const GemmDesc<float>* __restrict__ descs, const int* __restrict__ tile_problem, int ntiles,
                 const CUtensorMap* __restrict__ tmaps, int* status, int stall, const GenParams gp) {
    constexpr int NCONV = NCW * 32;        // converter threads
    constexpr int MMA_WARP = NCW + 1;
    constexpr int EPI_WARP0 = NCW + 2;
    using S = Shape<BN>;
    constexpr int ST = S::ST;
    extern __shared__ unsigned char smraw[];
    // 1024-byte aligned stage area, then the barriers
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    float* cbuf = reinterpret_cast<float*>(sm + (size_t)ST * S::STAGE);   // [BN][BM], column-major
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + (size_t)ST * S::STAGE + S::C_BYTES);
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const uint32_t stage0 = smem_u32(sm);
    const uint32_t bar0 = smem_u32(bars);
    // raw[ST]: copies landed; full[ST]: split done; empty[ST]: MMAs done with the stage;
    // tfull[2] / tempty[2]: accumulator handed to / released by the epilogue; done
    auto raw = [&](int s) { return bar0 + 8u * s; };
    auto full = [&](int s) { return bar0 + 8u * (ST + s); };
    auto empty = [&](int s) { return bar0 + 8u * (2 * ST + s); };
    auto tfull = [&](int a) { return bar0 + 8u * (3 * ST + a); };
    auto tempty = [&](int a) { return bar0 + 8u * (3 * ST + 2 + a); };
    const uint32_t done = bar0 + 8u * (3 * ST + 4);
    const uint32_t cfull = bar0 + 8u * (3 * ST + 5);   // the C tile has landed
    const uint32_t cdone = bar0 + 8u * (3 * ST + 6);   // the epilogue has written its results into it
    const uint32_t cfree = bar0 + 8u * (3 * ST + 7);   // the last store has finished reading it

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == MMA_WARP) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                     "r"(S::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(raw(s), 1);
            mbar_init(full(s), NCONV);
            mbar_init(empty(s), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(tfull(a), 1);
            mbar_init(tempty(a), EPW * 32);
        }
        mbar_init(done, 1);
        mbar_init(cfull, 1);
        mbar_init(cdone, EPW * 32);
        mbar_init(cfree, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = s_tmem;
    volatile int* abort_flag = &s_abort;
    const long long lim = stall ? STALL_WAIT_CYCLES : ROLE_WAIT_CYCLES;

    if (warp == 0) {
        // ------------------------------ TMA producer ------------------------------
        if (lane == 0) {
            int slot = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok && !stall; tile += gridDim.x) {
                const TileInfo ti = decode<BN>(descs, tile_problem, tile);
                const GemmDesc<float>& D = descs[ti.p];
                const bool a_mn = GEN == GEN_DENSE && D.opA == OP_N, b_mn = D.opB == OP_T;
                const CUtensorMap* ma = tmaps + 3 * ti.p;
                const CUtensorMap* mb = ma + 1;
                // the next tile's first k-blocks (short-k tiles: all of it) into L2 while
                // this one's last ST k-blocks stream, so its stage loads do not wait on DRAM
                // latency (earlier, on long tiles, the lines would be evicted before use)
                auto prefetch_next = [&]() {
                    if (tile + (int)gridDim.x >= ntiles) return;
                    const TileInfo tn = decode<BN>(descs, tile_problem, tile + gridDim.x);
                    const GemmDesc<float>& Dn = descs[tn.p];
                    const bool na_mn = Dn.opA == OP_N, nb_mn = Dn.opB == OP_T;
                    const CUtensorMap* pa = tmaps + 3 * tn.p;
                    for (int kt = 0; kt < min(tn.nk, ST); ++kt) {
                        const int k0 = tn.kb + kt * BK;
                        if constexpr (GEN == GEN_DENSE) {
                            if (na_mn) {
#pragma unroll
                                for (int c = 0; c < BM / 32; ++c) tma2d_prefetch(pa, tn.m0 + 32 * c, k0);
                            } else {
                                tma2d_prefetch(pa, k0, tn.m0);
                            }
                        }
                        if (nb_mn) {
#pragma unroll
                            for (int c = 0; c < BN / 32; ++c) tma2d_prefetch(pa + 1, tn.n0 + 32 * c, k0);
                        } else {
                            tma2d_prefetch(pa + 1, k0, tn.n0);
                        }
                    }
                };
                if (ti.nk == 0) prefetch_next();
                for (int kt = 0; kt < ti.nk; ++kt, ++slot) {
                    const int st = slot % ST;
                    if (kt == max(0, ti.nk - ST)) prefetch_next();
                    if (!wait_bar(empty(st), ((slot / ST) & 1) ^ 1, abort_flag, status, lim)) { ok = false; break; }
                    const uint32_t base = stage0 + (uint32_t)st * S::STAGE;
                    const uint32_t bbase = base + 2 * S::A_BYTES;
                    const int k0 = ti.kb + kt * BK;
                    mbar_expect(raw(st), (uint32_t)((GEN == GEN_DENSE ? S::A_BYTES : 0) + S::B_BYTES));
                    if constexpr (GEN == GEN_DENSE) {
                        if (a_mn) {
#pragma unroll
                            for (int c = 0; c < BM / 32; ++c) tma2d(base + 4096u * c, ma, ti.m0 + 32 * c, k0, raw(st));
                        } else {
                            tma2d(base, ma, k0, ti.m0, raw(st));
                        }
                    }
                    if (b_mn) {
#pragma unroll
                        for (int c = 0; c < BN / 32; ++c) tma2d(bbase + 4096u * c, mb, ti.n0 + 32 * c, k0, raw(st));
                    } else {
                        tma2d(bbase, mb, k0, ti.n0, raw(st));
                    }
                }
            }
            // no copy may still be landing when the CTA exits (a no-op unless a wait
            // elsewhere gave up): the last ST stages issued have completed
            for (int sl = max(0, slot - ST); sl < slot; ++sl) wait_bar_final(raw(sl % ST), (sl / ST) & 1, status);
        }
        __syncwarp();
    } else if (warp < MMA_WARP) {
        // ------------------------- converters (hi/lo split) -------------------------
        const int t = tid - 32;
        int slot = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            const TileInfo ti = decode<BN>(descs, tile_problem, tile);
            const GemmDesc<float>& D = descs[ti.p];
            for (int kt = 0; kt < ti.nk; ++kt, ++slot) {
                const int st = slot % ST;
                if (!wait_bar_warp(raw(st), (slot / ST) & 1, abort_flag, status, lim)) { ok = false; break; }
                const uint32_t base = stage0 + (uint32_t)st * S::STAGE;
                constexpr int CA = S::A_BYTES / 16, CB = S::B_BYTES / 16;
                constexpr int NCH = (CA + CB + NCONV - 1) / NCONV;
                const int k0 = ti.kb + kt * BK;
                // all of this thread's 16-byte chunks are read (or, for a generated A,
                // evaluated) first, then split and written back
                float x[NCH][4];
                uint32_t off[NCH], lof[NCH];
#pragma unroll
                for (int i = 0; i < NCH; ++i) {
                    const int e = t + NCONV * i;
                    if (e >= CA + CB) continue;
                    off[i] = e < CA ? (uint32_t)e * 16 : (uint32_t)(2 * S::A_BYTES + (e - CA) * 16);
                    lof[i] = off[i] + (e < CA ? S::A_BYTES : S::B_BYTES);
                    if (GEN != GEN_DENSE && e < CA) {
                        // K-major line r (128 bytes), physical chunk e % 8 = logical k-group
                        // ((e % 8) ^ (r % 8)) of the 128-byte swizzle.  A thread's chunks all
                        // have the same k-group (r % 8 = (t / 8) % 8), so for the symmetric
                        // kernels in 1-D or 2-D the four column points are loaded once per
                        // stage and each row point once per chunk.
                        const int r = e >> 3, kg = (e & 7) ^ (r & 7);
                        const int row = ti.m0 + r;
                        if ((GEN == GEN_GAUSSIAN || GEN == GEN_COULOMB) && gp.dim <= 2) {
                            const bool nt = D.opA == OP_N;
                            const int rowg = (nt ? D.ga_r0 : D.ga_c0) + row;   // the tile row's point
                            const int colg0 = (nt ? D.ga_c0 : D.ga_r0) + k0 + 4 * kg;
                            const bool two = gp.dim == 2;
                            const double rx = row < D.m ? gp.pts[(size_t)rowg * gp.dim] : 0.0;
                            const double ry = (row < D.m && two) ? gp.pts[(size_t)rowg * 2 + 1] : 0.0;
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int kk = k0 + 4 * kg + u;
                                float v = 0.f;
                                if (row < D.m && kk < ti.ke) {
                                    const int cg = colg0 + u;
                                    const double dx = rx - gp.pts[(size_t)cg * gp.dim];
                                    const double dy = two ? ry - gp.pts[(size_t)cg * 2 + 1] : 0.0;
                                    v = gen_from_d2<GEN == GEN_GAUSSIAN ? GEN_GAUSSIAN : GEN_COULOMB>(
                                        gp, rowg, cg, fma(dx, dx, dy * dy));
                                }
                                x[i][u] = v;
                            }
                        } else {
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int kk = k0 + 4 * kg + u;
                                float v = 0.f;
                                if (row < D.m && kk < ti.ke)
                                    v = D.opA == OP_N ? gen_entry_f32<GEN>(gp, D.ga_r0 + row, D.ga_c0 + kk)
                                                      : gen_entry_f32<GEN>(gp, D.ga_r0 + kk, D.ga_c0 + row);
                                x[i][u] = v;
                            }
                        }
                    } else {
                        asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];\n"
                                     : "=f"(x[i][0]), "=f"(x[i][1]), "=f"(x[i][2]), "=f"(x[i][3])
                                     : "r"(base + off[i]));
                    }
                }
#pragma unroll
                for (int i = 0; i < NCH; ++i) {
                    const int e = t + NCONV * i;
                    if (e >= CA + CB) continue;
                    float h[4], l[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        h[u] = tf32_rn(x[i][u]);
                        l[u] = tf32_rn(x[i][u] - h[u]);
                    }
                    asm volatile("st.shared.v4.f32 [%0], {%1,%2,%3,%4};\n" ::"r"(base + off[i]), "f"(h[0]), "f"(h[1]),
                                 "f"(h[2]), "f"(h[3])
                                 : "memory");
                    asm volatile("st.shared.v4.f32 [%0], {%1,%2,%3,%4};\n" ::"r"(base + lof[i]), "f"(l[0]), "f"(l[1]),
                                 "f"(l[2]), "f"(l[3])
                                 : "memory");
                }
                fence_async_smem();
                mbar_arrive(full(st));
            }
        }
    } else if (warp == MMA_WARP) {
        // ------------------------------- MMA issue -------------------------------
        if (lane == 0) {
            int slot = 0, accn = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                const TileInfo ti = decode<BN>(descs, tile_problem, tile);
                const GemmDesc<float>& D = descs[ti.p];
                const bool a_mn = GEN == GEN_DENSE && D.opA == OP_N, b_mn = D.opB == OP_T;
                const int nt = min(BN, D.n - ti.n0);
                const int ninst = (nt + 15) / 16 * 16;
                const int acc = accn & 1;
                if (!wait_bar(tempty(acc), ((accn >> 1) & 1) ^ 1, abort_flag, status, lim)) break;
                tc_after();
                const uint32_t dt = tmem + (uint32_t)(acc * S::ACC_COLS);
                const uint32_t idesc = idesc_tf32(a_mn, b_mn, ninst);
                // descriptor strides: K-major (LBO 16, SBO 1024 between 8-row groups, k-step
                // +32 bytes inside the swizzled line); MN-major (LBO 4096 between 32-row
                // boxes, SBO 512 between 4-deep k-groups, k-step = 2 k-groups)
                const uint32_t a_lbo = a_mn ? 4096u : 16u, a_sbo = a_mn ? 512u : 1024u;
                const uint32_t b_lbo = b_mn ? 4096u : 16u, b_sbo = b_mn ? 512u : 1024u;
                const uint32_t a_step = a_mn ? 1024u : 32u, b_step = b_mn ? 1024u : 32u;
                const uint32_t a_lay = a_mn ? 1u : 2u, b_lay = b_mn ? 1u : 2u;
                for (int kt = 0; kt < ti.nk; ++kt, ++slot) {
                    const int st = slot % ST;
                    if (!wait_bar(full(st), (slot / ST) & 1, abort_flag, status, lim)) { ok = false; break; }
                    tc_after();
                    const uint32_t base = stage0 + (uint32_t)st * S::STAGE;
                    const uint32_t ahi = base, alo = base + S::A_BYTES;
                    const uint32_t bhi = base + 2 * S::A_BYTES, blo = bhi + S::B_BYTES;
#pragma unroll
                    for (int s = 0; s < BK / 8; ++s) {
                        const uint64_t dah = sdesc(ahi + s * a_step, a_lbo, a_sbo, a_lay);
                        const uint64_t dal = sdesc(alo + s * a_step, a_lbo, a_sbo, a_lay);
                        const uint64_t dbh = sdesc(bhi + s * b_step, b_lbo, b_sbo, b_lay);
                        const uint64_t dbl = sdesc(blo + s * b_step, b_lbo, b_sbo, b_lay);
                        const uint32_t first = (kt | s) != 0;
                        mma_tf32(dt + S::HALF_COLS, dal, dbl, idesc, first);
                        mma_tf32(dt + S::HALF_COLS, dal, dbh, idesc, 1);
                        mma_tf32(dt + S::HALF_COLS, dah, dbl, idesc, 1);
                        mma_tf32(dt, dah, dbh, idesc, first);
                    }
                    mma_commit(empty(st));
                }
                if (!ok) break;
                mma_commit(tfull(acc));
                ++accn;
            }
            // every MMA issued has completed before the tensor memory is released
            mma_commit(done);
            wait_bar_final(done, 0, status);
        }
        __syncwarp();
    } else {
        // -------------------------------- epilogue --------------------------------
        // The tile goes through the shared C buffer: C is loaded into it by TMA when
        // beta != 0, the results are written into it, and one TMA store (or, for
        // split-K, one TMA reduce-add) writes it back; the leader thread issues the
        // copies and orders the buffer's reuse.
        const int q = warp & 3;                          // TMEM lane quarter of this warp
        const int half = (warp - EPI_WARP0) >> 2;        // which half of the tile's columns
        const int row = 32 * q + lane;
        const bool leader = warp == EPI_WARP0 && lane == 0;
        int accn = 0, rdn = 0;    // tiles seen; tiles whose C tile was loaded
        bool c_pending = false;   // leader: a C-tile load not yet waited for
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const TileInfo ti = decode<BN>(descs, tile_problem, tile);
            const GemmDesc<float>& D = descs[ti.p];
            const float alpha = D.alpha, beta = D.beta;
            const bool split = D.ksplit > 1;
            const int nt = min(BN, D.n - ti.n0);
            const CUtensorMap* mc = tmaps + 3 * ti.p + 2;
            const bool rd = !split && beta != 0.f;
            // the TMA store writes whole 16-byte granules: a tile whose last valid row
            // ends inside one is written back row by row instead (it must not touch the
            // rows that follow C in memory)
            const int m = D.m;
            const bool c_tma = c_tma_ok(D.C, D.ldc);
            const bool via_tma = c_tma && ((m % 4 == 0) || (ti.m0 + BM <= m));
            const int gi = ti.m0 + row;
            float* crow = D.C + gi + (size_t)ti.n0 * D.ldc;
            if (leader) {
                // the previous tile's store has read the buffer: it may be reloaded / rewritten
                bulk_wait_read();
                if (rd && c_tma) {
                    mbar_expect(cfull, (uint32_t)S::C_BYTES);
                    tma2d(smem_u32(cbuf), mc, ti.m0, ti.n0, cfull);
                    c_pending = true;
                }
                mbar_arrive(cfree);
                // after a short-k tile, the next tile's C into L2: its load then waits on
                // L2, not DRAM (long tiles leave the load time to land anyway)
                if (ti.nk <= ST && tile + (int)gridDim.x < ntiles) {
                    const TileInfo tn = decode<BN>(descs, tile_problem, tile + gridDim.x);
                    const GemmDesc<float>& Dn = descs[tn.p];
                    if (Dn.ksplit <= 1 && Dn.beta != 0.f && c_tma_ok(Dn.C, Dn.ldc))
                        tma2d_prefetch(tmaps + 3 * tn.p + 2, tn.m0, tn.n0);
                }
            }
            const int acc = accn & 1;
            if (!wait_bar_warp(tfull(acc), (accn >> 1) & 1, abort_flag, status, lim)) break;
            if (!wait_bar_warp(cfree, accn & 1, abort_flag, status, lim)) break;
            if (rd && c_tma) {
                if (!wait_bar_warp(cfull, rdn & 1, abort_flag, status, lim)) break;
                if (leader) c_pending = false;
            }
            tc_after();
            const uint32_t tbase = tmem + (uint32_t)(acc * S::ACC_COLS) + ((uint32_t)(32 * q) << 16);
            const uint32_t cb0 = smem_u32(cbuf) + 4u * row;   // this row of column 0 of the C tile
            // 16 columns per round: the main and correction accumulators, then the round's
            // C reads all issued together, then the results (the 16-column body is unrolled;
            // the outer loop is not, to keep the kernel's code small: instruction fetch
            // stalls led this kernel's profile)
            constexpr int RH = BN / 16 / (EPW / 4);   // 16-column rounds per warp
#pragma unroll 1
            for (int c = half * RH; c < (half + 1) * RH; ++c) {
                if (16 * c >= nt) break;
                float v[16], w[16], cc[16];
                if (ti.nk > 0) {
                    tmem_ld16x2(tbase + (uint32_t)(16 * c), tbase + (uint32_t)(S::HALF_COLS + 16 * c), v, w);
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] = w[j] = 0.f;
                }
                if (rd && c_tma) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) cc[j] = lds_f32(cb0 + 4u * BM * (16 * c + j));
                } else if (rd) {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        cc[j] = (gi < m && 16 * c + j < nt) ? crow[(size_t)(16 * c + j) * D.ldc] : 0.f;
                }
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float a = alpha * (v[j] + w[j]);
                    const float val = rd ? fmaf(beta, cc[j], a) : a;
                    if (via_tma) {
                        sts_f32(cb0 + 4u * BM * (16 * c + j), val);
                    } else if (gi < m && 16 * c + j < nt) {
                        float* cw = crow + (size_t)(16 * c + j) * D.ldc;
                        if (split) atomicAdd(cw, val);
                        else *cw = val;
                    }
                }
            }
            tc_before();
            mbar_arrive(tempty(acc));
            fence_async_smem();
            mbar_arrive(cdone);
            if (leader) {
                if (!wait_bar(cdone, accn & 1, abort_flag, status, lim)) break;
                if (via_tma) {
                    if (split) tma2d_add(mc, ti.m0, ti.n0, smem_u32(cbuf));
                    else tma2d_store(mc, ti.m0, ti.n0, smem_u32(cbuf));
                    bulk_commit();
                }
            }
            if (rd && c_tma) ++rdn;
            ++accn;
        }
        if (leader) {
            if (c_pending) wait_bar_final(cfull, rdn & 1, status);
            bulk_wait_all();
        }
    }
    tc_before();
    __syncthreads();
    if (warp == MMA_WARP) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(S::TMEM_COLS)
                     : "memory");
    }
}

// EPW: epilogue warps, 8 for short-k batches (the epilogue bounds them), 4 otherwise.
// NCW: converter warps, 8, or 12 for generated-A batches, where the entry generation in
// the converters bounds the kernel (12 made the Coulomb sketch 17% faster; dense long-k
// batches, not converter-bound, were 2% slower with 12).
template <int BN, int GEN = GEN_DENSE, int EPW = 4, int NCW = 8>
void launch(int tiles, int sms, cudaStream_t s, const GemmDesc<float>* d, const int* tile_problem,
            const CUtensorMap* tmaps, int* status, int stall, const GenParams& gp = GenParams()) {
    static_assert(EPW == 4 || EPW == 8, "epilogue warps");
    static_assert(NCW == 8 || NCW == 12, "converter warps (a multiple of 2 keeps the chunk k-groups)");
    using S = Shape<BN>;
    static size_t cur = 0;
    ensure_dyn_smem(gemm_tc32_kernel<BN, GEN, EPW, NCW>, S::SMEM, cur);
    const int grid = std::max(1, std::min(tiles, sms));
    gemm_tc32_kernel<BN, GEN, EPW, NCW><<<grid, nthreads<EPW, NCW>(), S::SMEM, s>>>(d, tile_problem, tiles, tmaps,
                                                                                     status, stall, gp);
}

// Whether the tensor-core kernel can take a problem: the TMA wants 16-byte aligned bases
// and leading dimensions that are multiples of 4 floats.
inline bool tma_ok(const GemmDesc<float>& d, bool gen_a = false) {
    return (gen_a || ((reinterpret_cast<uintptr_t>(d.A) & 15) == 0 && d.lda % 4 == 0)) &&
           (reinterpret_cast<uintptr_t>(d.B) & 15) == 0 && d.ldb % 4 == 0 && d.kscale == nullptr;
}

// Tensor maps of every problem's operands (3 per problem: A, B, C), in the box shapes
// the kernel issues.  Returns false if the driver refuses one.
inline bool encode_maps(const std::vector<GemmDesc<float>>& probs, int bn, std::vector<CUtensorMap>& out,
                        bool gen_a = false) {
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    out.resize(3 * probs.size());
    for (size_t i = 0; i < probs.size(); ++i) {
        const GemmDesc<float>& d = probs[i];
        const cuuint64_t k = (cuuint64_t)std::max(d.k, 1);
        for (int w = gen_a ? 1 : 0; w < 2; ++w) {   // a generated A has no tensor map
            const bool mn = w == 0 ? d.opA == OP_N : d.opB == OP_T;
            const cuuint64_t rows = (cuuint64_t)(w == 0 ? d.m : d.n);
            const int ld = w == 0 ? d.lda : d.ldb;
            void* base = const_cast<float*>(w == 0 ? d.A : d.B);
            cuuint64_t dims[2], strides[1] = {(cuuint64_t)ld * 4};
            cuuint32_t box[2], es[2] = {1, 1};
            if (mn) { dims[0] = rows; dims[1] = k; box[0] = 32; box[1] = 32; }
            else { dims[0] = k; dims[1] = rows; box[0] = 32; box[1] = (cuuint32_t)(w == 0 ? BM : bn); }
            const CUresult r = enc(&out[3 * i + w], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE,
                                   mn ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return false;
        }
        if (c_tma_ok(d.C, d.ldc)) {   // C (m x n, column-major), box BM x bn, no swizzle
            cuuint64_t dims[2] = {(cuuint64_t)d.m, (cuuint64_t)d.n}, strides[1] = {(cuuint64_t)d.ldc * 4};
            cuuint32_t box[2] = {(cuuint32_t)BM, (cuuint32_t)bn}, es[2] = {1, 1};
            const CUresult r = enc(&out[3 * i + 2], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, d.C, dims, strides, box, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return false;
        }
    }
    return true;
}

}  // namespace tc
