// hm_multiply_device_noalloc: the HODLR multiply on caller-owned device buffers without
// any device allocation.
//
// Who needs it: code that may not call cudaMalloc at the moment it multiplies — a
// real-time or callback thread that must not block in the device allocator, or an
// application that hands out all device memory through its own pool and forbids other
// allocations.  Such callers build the operator once at set-up (that build allocates)
// and then multiply here.
//
// The per-node intermediates (t = V^T x, delta = B t) and the launch tables live in one
// file-scope __device__ array of NOALLOC_SCRATCH_BYTES (32 MiB).  Every GPU that loads
// the library holds that array until the process exits.  In host code the array's name
// is only a host-side stand-in, so its device address is fetched with
// cudaGetSymbolAddress once per device (the first call on a device, with that device
// current) and cached.  The operator's device must be the current device.  All calls
// share the array and it keeps the last call's contents: the split-K partial sums are
// zeroed by the launch itself before accumulation, and two calls whose work overlaps on
// the GPU (e.g. on two streams, or two handles) race on the array.  Each call copies its
// launch tables from host memory into the array with cudaMemcpyAsync; a copy from
// pageable host memory first waits for the work already queued on the stream, so the
// call returns once the stream has reached it.
#include <mutex>

#include "hm_engine.h"

namespace hm {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(32) << 20;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static unsigned char* noalloc_scratch_device() {
    static std::mutex mu;
    static void* addr[NOALLOC_MAX_DEVICES] = {};
    int dev = 0;
    HM_CUDA(cudaGetDevice(&dev));
    HM_CHECK(dev >= 0 && dev < NOALLOC_MAX_DEVICES, HM_ERR_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            throw Error(HM_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") +
                                         cudaGetErrorString(e));
        }
        addr[dev] = p;
    }
    return static_cast<unsigned char*>(addr[dev]);
}

void multiply_noalloc(const Engine::View& v, const double* dx, int s, int ldx, double* dy, int ldy,
                      cudaStream_t st) {
    HM_CHECK(v.built, HM_ERR_STATE, "multiply before build");
    HM_CHECK(dx && dy && s >= 1 && ldx >= v.N && ldy >= v.N, HM_ERR_ARG, "multiply_noalloc: bad arguments");
    {   // the scratch address is per device: the operator's device must be current
        int cur = 0;
        HM_CUDA(cudaGetDevice(&cur));
        HM_CHECK(cur == v.device, HM_ERR_ARG,
                 "multiply_noalloc: the current device (" + std::to_string(cur) + ") is not the operator's (" +
                     std::to_string(v.device) + ")");
    }
    const std::vector<Node>& nodes = *v.nodes;
    const std::vector<std::vector<int>>& levels = *v.levels;
    // 1) scratch offsets for t and delta of every internal node (first in the array)
    size_t off = 0;
    auto take = [&](size_t doubles) {
        size_t o = off;
        off += align_up(std::max<size_t>(doubles, 1) * sizeof(double), 256);
        return o;
    };
    struct Tmp { size_t T, D; };
    std::vector<Tmp> tmp(nodes.size(), Tmp{0, 0});
    for (size_t i = 0; i < nodes.size(); ++i) {
        const Node& n = nodes[i];
        if (n.is_leaf) continue;
        const Node& L = nodes[n.left];
        const Node& R = nodes[n.right];
        tmp[i].T = take((size_t)(L.rankV + R.rankV) * s);
        tmp[i].D = take((size_t)(L.rankU + R.rankU) * s);
    }
    const size_t scratch_bytes = off;
    HM_CHECK(scratch_bytes <= NOALLOC_SCRATCH_BYTES, HM_ERR_UNSUPPORTED,
             "multiply_noalloc: the intermediates need " + std::to_string(scratch_bytes) +
                 " bytes, above the fixed " + std::to_string(NOALLOC_SCRATCH_BYTES) + "-byte scratch");
    unsigned char* base = noalloc_scratch_device();
    auto P = [&](size_t o) { return reinterpret_cast<double*>(base + o); };
    // 2) the same launch sequence as the handle's multiply, on the caller's x and y
    std::vector<GemmBatch<double>> batches;
    batches.emplace_back();  // y_leaf = D x_leaf
    for (int l : *v.leaves) {
        const Node& n = nodes[l];
        batches.back().add(n.len(), s, n.len(), 1.0, v.D + n.offD, n.len(), OP_N, dx + n.start, ldx, OP_N,
                           0.0, dy + n.start, ldy);
    }
    batches.emplace_back();  // t = [V1^T x1; V2^T x2]
    GemmBatch<double>& gT = batches.back();
    for (size_t i = 0; i < nodes.size(); ++i) {
        const Node& n = nodes[i];
        if (n.is_leaf) continue;
        const Node& L = nodes[n.left];
        const Node& R = nodes[n.right];
        const int q1 = L.rankV, q2 = R.rankV;
        gT.add(q1, s, L.len(), 1.0, v.V + L.offV, L.len(), OP_T, dx + L.start, ldx, OP_N, 0.0, P(tmp[i].T), q1 + q2);
        gT.add(q2, s, R.len(), 1.0, v.V + R.offV, R.len(), OP_T, dx + R.start, ldx, OP_N, 0.0,
               P(tmp[i].T) + q1, q1 + q2);
    }
    batches.emplace_back();  // delta1 = B12 t2, delta2 = B21 t1
    GemmBatch<double>& gD = batches.back();
    for (size_t i = 0; i < nodes.size(); ++i) {
        const Node& n = nodes[i];
        if (n.is_leaf) continue;
        const Node& L = nodes[n.left];
        const Node& R = nodes[n.right];
        const int p1 = L.rankU, p2 = R.rankU, q1 = L.rankV, q2 = R.rankV;
        gD.add(p1, s, q2, 1.0, v.B + n.offB12, p1, OP_N, P(tmp[i].T) + q1, q1 + q2, OP_N, 0.0, P(tmp[i].D), p1 + p2);
        gD.add(p2, s, q1, 1.0, v.B + n.offB21, p2, OP_N, P(tmp[i].T), q1 + q2, OP_N, 0.0, P(tmp[i].D) + p1, p1 + p2);
    }
    for (size_t d = 0; d < levels.size(); ++d) {  // y += U delta, one level at a time
        batches.emplace_back();
        for (int id : levels[d]) {
            const Node& n = nodes[id];
            const Node& L = nodes[n.left];
            const Node& R = nodes[n.right];
            const int p1 = L.rankU, p2 = R.rankU;
            batches.back().add(L.len(), s, p1, 1.0, v.U + L.offU, L.len(), OP_N, P(tmp[id].D), p1 + p2, OP_N, 1.0,
                               dy + L.start, ldy);
            batches.back().add(R.len(), s, p2, 1.0, v.U + R.offU, R.len(), OP_N, P(tmp[id].D) + p1, p1 + p2, OP_N,
                               1.0, dy + R.start, ldy);
        }
    }
    // 3) launch tables after the intermediates, copied in (a copy, not an allocation)
    struct Placed { size_t desc, zero; int nd, nz, tiles; };
    std::vector<Placed> placed;
    std::vector<std::vector<GemmDesc<double>>> descs;
    for (auto& b : batches) {
        Placed p{};
        descs.push_back(b.packed(&p.tiles));
        p.nd = (int)descs.back().size();
        p.nz = (int)b.zero_regions().size();
        p.desc = take(sizeof(GemmDesc<double>) * p.nd / sizeof(double) + 1);
        p.zero = take(sizeof(ZeroRegion<double>) * p.nz / sizeof(double) + 1);
        placed.push_back(p);
    }
    HM_CHECK(off <= NOALLOC_SCRATCH_BYTES, HM_ERR_UNSUPPORTED,
             "multiply_noalloc: intermediates and launch tables need " + std::to_string(off) +
                 " bytes, above the fixed " + std::to_string(NOALLOC_SCRATCH_BYTES) + "-byte scratch");
    for (size_t i = 0; i < batches.size(); ++i) {
        const Placed& p = placed[i];
        if (p.nd)
            HM_CUDA(cudaMemcpyAsync(base + p.desc, descs[i].data(), sizeof(GemmDesc<double>) * p.nd,
                                    cudaMemcpyHostToDevice, st));
        if (p.nz)
            HM_CUDA(cudaMemcpyAsync(base + p.zero, batches[i].zero_regions().data(),
                                    sizeof(ZeroRegion<double>) * p.nz, cudaMemcpyHostToDevice, st));
    }
    for (size_t i = 0; i < batches.size(); ++i) {
        const Placed& p = placed[i];
        gemm_launch_tables(reinterpret_cast<const GemmDesc<double>*>(base + p.desc), p.nd, p.tiles,
                           reinterpret_cast<const ZeroRegion<double>*>(base + p.zero), p.nz, st);
        count_launch((p.nd ? 1 : 0) + (p.nz ? 1 : 0));
    }
    // the host-side tables above are pageable: each copy has staged them before
    // returning, so they may go out of scope now
}

}  // namespace hm
