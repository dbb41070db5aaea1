// Serialized operators: a built HODLR or HSS operator (tree, leaf blocks, bases,
// coupling blocks, and for HSS the reference-form export data; for matrix-free builds the
// kernel, its parameters and points) written to one file and read back into a handle, so
// a later process factors and solves without recompressing.  Factorizations are not
// stored: factoring is cheap next to the build and is redone on first use.
//
// Layout (native byte order, version 2; version 1 files, without the nested-basis
// section, still load):
//   "HMATB200" | u32 version | u32 kind | i64 N | i64 leaf | i64 nodes
//   nodes x Node (the planner's struct, offsets into the arrays below included)
//   array D | array U | array V | array B           (array = i64 count, count doubles)
//   i32 gen | i32 dim | f64 p0 | f64 p1 | array points
//   HSS only: array leafB | nodes x (i64 offU, i32 rankU, i64 offV, i32 rankV)
//             nodes x (i32 rankU, i32 rankV, i64 offB12, i64 offB21) | array B (reference form)
//             u32 nested | nested only: nodes x (i64 offR, i64 offW) | array RW
// The tree in the file must be the one the planner makes for (N, leaf); load checks it.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "hm_engine.h"

namespace hm {

namespace {
// [off, off + count) inside an array of n elements, without wrapping
inline bool fits(size_t off, size_t count, size_t n) { return off <= n && count <= n - off; }

constexpr char MAGIC[8] = {'H', 'M', 'A', 'T', 'B', '2', '0', '0'};
constexpr uint32_t VERSION = 2;
static_assert(std::is_trivially_copyable<Node>::value, "Node is written as raw bytes");

struct File {
    FILE* f = nullptr;
    std::string path;
    File(const char* p, const char* mode) : path(p ? p : "") {
        HM_CHECK(p && *p, HM_ERR_ARG, "operator file: empty path");
        f = std::fopen(p, mode);
        HM_CHECK(f, HM_ERR_ARG, "operator file: cannot open " + path);
    }
    ~File() {
        if (f) std::fclose(f);
    }
    void put(const void* p, size_t n) {
        HM_CHECK(n == 0 || std::fwrite(p, 1, n, f) == n, HM_ERR_ARG, "operator file: write failed: " + path);
    }
    void get(void* p, size_t n) {
        HM_CHECK(n == 0 || std::fread(p, 1, n, f) == n, HM_ERR_ARG, "operator file: truncated: " + path);
    }
    template <typename V> void put_v(const V& v) { put(&v, sizeof v); }
    template <typename V> V get_v() {
        V v;
        get(&v, sizeof v);
        return v;
    }
    void close_checked() {
        const int rc = std::fclose(f);
        f = nullptr;
        HM_CHECK(rc == 0, HM_ERR_ARG, "operator file: write failed: " + path);
    }
};

// device array -> file, staged through a bounded host buffer
void put_array(File& F, const double* d, size_t n, cudaStream_t s) {
    F.put_v<int64_t>((int64_t)n);
    const size_t chunk = size_t(1) << 24;
    std::vector<double> h(std::min(n, chunk));
    for (size_t o = 0; o < n; o += chunk) {
        const size_t c = std::min(chunk, n - o);
        HM_CUDA(cudaMemcpyAsync(h.data(), d + o, c * sizeof(double), cudaMemcpyDeviceToHost, s));
        HM_CUDA(cudaStreamSynchronize(s));
        F.put(h.data(), c * sizeof(double));
    }
}

void get_array(File& F, DBuf<double>& d, cudaStream_t s) {
    const int64_t n = F.get_v<int64_t>();
    HM_CHECK(n >= 0 && n < (int64_t(1) << 40), HM_ERR_ARG, "operator file: bad array size");
    d.alloc(std::max<size_t>((size_t)n, 1));
    const size_t chunk = size_t(1) << 24;
    std::vector<double> h(std::min((size_t)n, chunk));
    for (size_t o = 0; o < (size_t)n; o += chunk) {
        const size_t c = std::min(chunk, (size_t)n - o);
        F.get(h.data(), c * sizeof(double));
        HM_CUDA(cudaMemcpyAsync(d.p + o, h.data(), c * sizeof(double), cudaMemcpyHostToDevice, s));
        HM_CUDA(cudaStreamSynchronize(s));
    }
}
}  // namespace

int Engine::file_kind(const char* path) {
    File F(path, "rb");
    char m[8];
    F.get(m, 8);
    HM_CHECK(std::memcmp(m, MAGIC, 8) == 0, HM_ERR_ARG, "operator file: not an hmat_b200 operator: " + F.path);
    const uint32_t v = F.get_v<uint32_t>();
    HM_CHECK(v == 1 || v == VERSION, HM_ERR_ARG, "operator file: unsupported version " + std::to_string(v));
    const uint32_t k = F.get_v<uint32_t>();
    HM_CHECK(k == HODLR || k == HSS, HM_ERR_ARG, "operator file: bad kind");
    return (int)k;
}

void Engine::save(const char* path) const {
    HM_CHECK(built_, HM_ERR_STATE, "save before build");
    HM_CHECK(sys_N_.size() == 1, HM_ERR_UNSUPPORTED, "save: batches of systems are not serialized");
    File F(path, "wb");
    F.put(MAGIC, 8);
    F.put_v<uint32_t>(VERSION);
    F.put_v<uint32_t>((uint32_t)kind_);
    F.put_v<int64_t>(N_);
    F.put_v<int64_t>(leaf_);
    F.put_v<int64_t>((int64_t)nodes_.size());
    F.put(nodes_.data(), nodes_.size() * sizeof(Node));
    put_array(F, dD.p, dD.n, stream_);
    put_array(F, dU.p, dU.n, stream_);
    put_array(F, dV.p, dV.n, stream_);
    put_array(F, dB.p, dB.n, stream_);
    F.put_v<int32_t>(gen_);
    F.put_v<int32_t>(gp_.dim);
    F.put_v<double>(gp_.p0);
    F.put_v<double>(gp_.p1);
    put_array(F, dPts.p, gen_ == GEN_DENSE ? 0 : dPts.n, stream_);
    if (kind_ == HSS) {
        put_array(F, dLeafB.p, dLeafB.n, stream_);
        for (size_t i = 0; i < nodes_.size(); ++i) {
            F.put_v<int64_t>((int64_t)leafU_[i].first);
            F.put_v<int32_t>(leafU_[i].second);
            F.put_v<int64_t>((int64_t)leafV_[i].first);
            F.put_v<int32_t>(leafV_[i].second);
        }
        for (size_t i = 0; i < nodes_.size(); ++i) {
            F.put_v<int32_t>(hss_.rankU[i]);
            F.put_v<int32_t>(hss_.rankV[i]);
            F.put_v<int64_t>((int64_t)hss_.offB12[i]);
            F.put_v<int64_t>((int64_t)hss_.offB21[i]);
        }
        put_array(F, hss_.B.p, hss_.B.n, stream_);
        F.put_v<uint32_t>(hss_.nested ? 1u : 0u);
        if (hss_.nested) {
            for (size_t i = 0; i < nodes_.size(); ++i) {
                F.put_v<int64_t>((int64_t)hss_.offR[i]);
                F.put_v<int64_t>((int64_t)hss_.offW[i]);
            }
            put_array(F, hss_.RW.p, hss_.RW.n, stream_);
        }
    }
    F.close_checked();
}

void Engine::load(const char* path) {
    HM_CHECK(file_kind(path) == kind_, HM_ERR_ARG, "operator file: kind differs from the handle's engine");
    File F(path, "rb");
    char m[8];
    F.get(m, 8);
    const uint32_t version = F.get_v<uint32_t>();
    F.get_v<uint32_t>();
    const int64_t N = F.get_v<int64_t>(), leaf = F.get_v<int64_t>(), nn = F.get_v<int64_t>();
    HM_CHECK(N > 0 && N < (int64_t(1) << 31) && leaf > 0 && leaf <= N, HM_ERR_ARG, "operator file: bad N/leaf");
    begin_build((int)N, (int)leaf);
    HM_CHECK(nn == (int64_t)nodes_.size(), HM_ERR_ARG, "operator file: tree does not match (N, leaf)");
    std::vector<Node> nodes((size_t)nn);
    F.get(nodes.data(), nodes.size() * sizeof(Node));
    for (size_t i = 0; i < nodes.size(); ++i) {
        const Node &a = nodes[i], &b = nodes_[i];
        HM_CHECK(a.start == b.start && a.end == b.end && a.is_leaf == b.is_leaf && a.left == b.left &&
                     a.right == b.right && a.parent == b.parent && a.depth == b.depth && a.sys == 0,
                 HM_ERR_ARG, "operator file: tree does not match (N, leaf)");
    }
    DBuf<double> D, U, V, B;
    get_array(F, D, stream_);
    get_array(F, U, stream_);
    get_array(F, V, stream_);
    get_array(F, B, stream_);
    // every block the operator addresses must lie inside the arrays just read
    for (const Node& n : nodes) {
        HM_CHECK(n.rankU >= 0 && n.rankV >= 0 && n.rankU <= n.len() && n.rankV <= n.len(), HM_ERR_ARG,
                 "operator file: bad rank");
        const size_t len = (size_t)n.len();
        if (n.is_leaf) HM_CHECK(fits(n.offD, len * len, D.n), HM_ERR_ARG, "operator file: D range");
        if (n.parent >= 0) {
            HM_CHECK(fits(n.offU, len * n.rankU, U.n) && fits(n.offV, len * n.rankV, V.n), HM_ERR_ARG,
                     "operator file: U/V range");
        }
        if (!n.is_leaf) {
            const Node& L = nodes[n.left];
            const Node& R = nodes[n.right];
            HM_CHECK(fits(n.offB12, (size_t)L.rankU * R.rankV, B.n) && fits(n.offB21, (size_t)R.rankU * L.rankV, B.n),
                     HM_ERR_ARG, "operator file: B range");
        }
    }
    const int32_t gen = F.get_v<int32_t>();
    const int32_t dim = F.get_v<int32_t>();
    const double p0 = F.get_v<double>(), p1 = F.get_v<double>();
    DBuf<double> P;
    get_array(F, P, stream_);
    HM_CHECK(gen == GEN_DENSE || gen == GEN_CAUCHY || gen == GEN_GAUSSIAN || gen == GEN_COULOMB, HM_ERR_ARG,
             "operator file: bad kernel");
    if (gen != GEN_DENSE) {
        const size_t need = gen == GEN_CAUCHY ? 2 * (size_t)N : (size_t)N * dim;
        HM_CHECK(dim >= 1 && dim <= 3 && P.n >= need, HM_ERR_ARG, "operator file: bad points");
    }
    if (kind_ == HSS) {
        DBuf<double> LB, HB;
        get_array(F, LB, stream_);
        std::vector<std::pair<size_t, int>> lu(nodes.size()), lv(nodes.size());
        for (size_t i = 0; i < nodes.size(); ++i) {
            lu[i].first = (size_t)F.get_v<int64_t>();
            lu[i].second = F.get_v<int32_t>();
            lv[i].first = (size_t)F.get_v<int64_t>();
            lv[i].second = F.get_v<int32_t>();
            const size_t len = (size_t)nodes[i].len();
            HM_CHECK(lu[i].second >= 0 && lv[i].second >= 0 && fits(lu[i].first, len * lu[i].second, LB.n) &&
                         fits(lv[i].first, len * lv[i].second, LB.n),
                     HM_ERR_ARG, "operator file: leaf basis range");
        }
        HssForm h;
        h.rankU.resize(nodes.size());
        h.rankV.resize(nodes.size());
        h.offB12.resize(nodes.size());
        h.offB21.resize(nodes.size());
        for (size_t i = 0; i < nodes.size(); ++i) {
            h.rankU[i] = F.get_v<int32_t>();
            h.rankV[i] = F.get_v<int32_t>();
            h.offB12[i] = (size_t)F.get_v<int64_t>();
            h.offB21[i] = (size_t)F.get_v<int64_t>();
        }
        get_array(F, HB, stream_);
        h.nested = version >= 2 && F.get_v<uint32_t>() != 0;
        if (h.nested) {
            h.offR.resize(nodes.size());
            h.offW.resize(nodes.size());
            for (size_t i = 0; i < nodes.size(); ++i) {
                h.offR[i] = (size_t)F.get_v<int64_t>();
                h.offW[i] = (size_t)F.get_v<int64_t>();
            }
            get_array(F, h.RW, stream_);
        }
        for (size_t i = 0; i < nodes.size(); ++i) {
            const Node& n = nodes[i];
            if (n.is_leaf) {
                HM_CHECK(h.rankU[i] == lu[i].second && h.rankV[i] == lv[i].second, HM_ERR_ARG,
                         "operator file: HSS leaf ranks");
                continue;
            }
            const int su = h.rankU[n.left] + h.rankU[n.right], sv = h.rankV[n.left] + h.rankV[n.right];
            // reference form: a node's rank is the sum of its children's; nested form: at
            // most that sum, 0 at the root, with R / W inside RW
            const bool ranks_ok =
                h.nested ? (n.parent < 0 ? h.rankU[i] == 0 && h.rankV[i] == 0
                                         : h.rankU[i] >= 0 && h.rankV[i] >= 0 && h.rankU[i] <= su &&
                                               h.rankV[i] <= sv &&
                                               fits(h.offR[i], (size_t)su * h.rankU[i], h.RW.n) &&
                                               fits(h.offW[i], (size_t)sv * h.rankV[i], h.RW.n))
                         : h.rankU[i] == su && h.rankV[i] == sv;
            HM_CHECK(h.rankU[n.left] >= 0 && h.rankV[n.left] >= 0 && h.rankU[n.right] >= 0 &&
                         h.rankV[n.right] >= 0 && ranks_ok &&
                         fits(h.offB12[i], (size_t)h.rankU[n.left] * h.rankV[n.right], HB.n) &&
                         fits(h.offB21[i], (size_t)h.rankU[n.right] * h.rankV[n.left], HB.n),
                     HM_ERR_ARG, "operator file: HSS B range");
        }
        h.B = std::move(HB);
        dLeafB = std::move(LB);
        leafU_ = std::move(lu);
        leafV_ = std::move(lv);
        hss_ = std::move(h);
    }
    nodes_ = std::move(nodes);
    dD = std::move(D);
    dU = std::move(U);
    dV = std::move(V);
    dB = std::move(B);
    gen_ = gen;
    gp_ = GenParams();
    if (gen != GEN_DENSE) {
        dPts = std::move(P);
        gp_.pts = dPts.p;
        gp_.N = (int)N;
        gp_.dim = dim;
        gp_.p0 = p0;
        gp_.p1 = p1;
        leaves_spd_ = kernel_spd(gen, p0, p1);
    }
    built_ = true;
}

}  // namespace hm
