// Nested-basis HSS build: compressed transfers R / W in place of the reference's identity
// transfers (hss_routines.h:86-90), so that a node's basis has the numerical rank of its
// own off-diagonal strip instead of the sum of its leaves' ranks.  No counterpart in the
// reference; selected per handle (hm_hss_set_nested), the reference form stays the default.
//
// Node t with children a, b and rows I_t.  Leaves keep the bases of their strips exactly
// as the reference-form build computes them (Engine::build_hss).  Above them
//     U_t = diag(U_a, U_b) R_t,   V_t = diag(V_a, V_b) W_t,
//     A[I_a, I_b] ~ U_a B12_t V_b^T,   A[I_b, I_a] ~ U_b B21_t V_a^T.
// Bottom-up, one tree level per pass, reading A only through one product per leaf:
//   panels    PU_c = A[I_c, :]^T U_c (N x kU_c) and PV_c = A[:, I_c] V_c: a generated (or
//             dense) product for a leaf, XU_c R_c for an internal child (its rows inside
//             I_c are zero and never read again)
//   pair      XU_t = [PU_a | PU_b] with the rows I_t zeroed = the transpose of the
//             projected strip [U_a^T A[I_a, I_t^c]; U_b^T A[I_b, I_t^c]]
//   transfer  R_t = the leading right singular vectors of XU_t (the strip's left ones,
//             Gram/Jacobi SVD), rank by the rule every other block uses (#{s > tol s_0},
//             at least 1, capped by max_rank); W_t likewise from XV_t
//   coupling  B12_t = PU_a[I_b rows]^T V_b,  B21_t = PU_b[I_a rows]^T V_a (expanded V)
// PU_a[I_b rows] = A[I_a, I_b]^T U_a holds exactly at every level, so B is the
// projection of the true block onto the nested bases.  Only one level's pair buffers are
// alive at a time (N x the sum of the level's child ranks, for U and for V, plus those of
// the level below while its panels are formed); the SVD scratch (three N x k' rotations
// per pair) is bounded per chunk.  The expanded bases and B go into the engine's
// two-level storage (nodes_, dU, dV, dB), on which factor, solve and multiply run;
// R, W and B are kept in hss_ for export.
#include <algorithm>
#include <memory>
#include <vector>

#include "hm_engine.h"

namespace hm {

namespace {
// Device storage of one node while the nested levels are built.
struct NestedNode {
    double* XU = nullptr;   // internal: [PU_left | PU_right], N rows
    double* XV = nullptr;
    int kpU = 0, kpV = 0;   // their widths: the children's rank sums
    double* Rf = nullptr;   // kpU x kpU right singular vectors of XU, sorted; R = leading kU columns
    double* Wf = nullptr;
    double* EU = nullptr;   // expanded basis, len x kU (ld len)
    double* EV = nullptr;
    double* B12 = nullptr;  // internal: kU[left] x kV[right] (ld kU[left])
    double* B21 = nullptr;  // internal: kU[right] x kV[left]
};
}  // namespace

void Engine::build_hss_nested(const Source& src) {
    const int N = N_;
    const int nn = (int)nodes_.size();
    std::vector<int> kU(nn, 0), kV(nn, 0);
    std::vector<NestedNode> nb(nn);
    for (int l : leaves_) {
        kU[l] = leafU_[l].second;
        kV[l] = leafV_[l].second;
        nb[l].EU = dLeafB.p + leafU_[l].first;
        nb[l].EV = dLeafB.p + leafV_[l].first;
    }
    auto one = [](size_t n) { return std::max<size_t>(n, 1); };
    Plan keep;                          // arena: R/W, expanded bases and B of every node
    std::unique_ptr<Plan> below;        // pair buffers of the level below (in below_ws)
    DBuf<unsigned char> below_ws;
    auto al = [](size_t bytes) { return (std::max<size_t>(bytes, 1) + 255) / 256 * 256; };
    const size_t budget = size_t(8) << 30;   // SVD scratch per chunk
    DBuf<unsigned char> ws;                   // one workspace for the chunks' scratch
    for (int d = (int)levels_.size() - 1; d >= 0; --d) {
        const std::vector<int>& lvl = levels_[d];
        if (lvl.empty()) continue;
        size_t pair_bytes = 0;   // this level's pair buffers, in one allocation
        for (int t : lvl) {
            const Node& n = nodes_[t];
            pair_bytes += al(8 * (size_t)N * (kU[n.left] + kU[n.right])) + al(8 * (size_t)N * (kV[n.left] + kV[n.right]));
        }
        DBuf<unsigned char> pair_ws(pair_bytes);
        auto pairs = std::make_unique<Plan>();
        pairs->use_arena(pair_ws.p, pair_ws.n);
        for (int t : lvl) {
            const Node& n = nodes_[t];
            NestedNode& x = nb[t];
            x.kpU = kU[n.left] + kU[n.right];
            x.kpV = kV[n.left] + kV[n.right];
            x.XU = pairs->scratch(one((size_t)N * x.kpU));
            x.XV = pairs->scratch(one((size_t)N * x.kpV));
            x.B12 = keep.scratch(one((size_t)kU[n.left] * kV[n.right]));
            x.B21 = keep.scratch(one((size_t)kU[n.right] * kV[n.left]));
            if (d > 0) {
                x.Rf = keep.scratch(one((size_t)x.kpU * x.kpU));
                x.Wf = keep.scratch(one((size_t)x.kpV * x.kpV));
            }
            for (int c : {n.left, n.right})
                if (!nodes_[c].is_leaf) {
                    nb[c].EU = keep.scratch(one((size_t)nodes_[c].len() * kU[c]));
                    nb[c].EV = keep.scratch(one((size_t)nodes_[c].len() * kV[c]));
                }
        }
        DBuf<int> dRank(2 * lvl.size());
        dRank.zero(stream_);
        size_t i0 = 0;
        while (i0 < lvl.size()) {
            size_t i1 = i0, bytes = 0;
            while (i1 < lvl.size()) {
                const NestedNode& x = nb[lvl[i1]];
                const size_t b = 8 * (3 * (size_t)N * (x.kpU + x.kpV) + 8 * ((size_t)x.kpU * x.kpU + (size_t)x.kpV * x.kpV)) +
                                 (size_t(64) << 10);   // alignment and small tables
                if (i1 > i0 && bytes + b > budget) break;
                bytes += b;
                ++i1;
            }
            if (ws.n < bytes) ws.alloc(bytes);
            Plan plan;
            plan.use_arena(ws.p, ws.n);
            auto pre = std::make_unique<IdentStep>();      // expanded blocks under a rank-0 child
            auto gP = std::make_unique<GemmStep<double>>(CFG_64x64, src.gen);   // leaf panels
            gP->gp = src.gp;
            auto gM = std::make_unique<GemmStep<double>>();   // internal children: panels, bases
            auto gB = std::make_unique<GemmStep<double>>();   // couplings
            auto cut = std::make_unique<IdentStep>();      // rows I_t of the pairs
            std::vector<SvdProblem> sv;
            for (size_t i = i0; i < i1; ++i) {
                const int t = lvl[i];
                const Node& n = nodes_[t];
                NestedNode& x = nb[t];
                const int a = n.left, b = n.right;
                for (int side = 0; side < 2; ++side) {
                    const int c = side == 0 ? a : b;
                    const Node& C = nodes_[c];
                    double* pu = x.XU + (size_t)N * (side == 0 ? 0 : kU[a]);
                    double* pv = x.XV + (size_t)N * (side == 0 ? 0 : kV[a]);
                    if (C.is_leaf) {
                        if (kU[c])
                            gP->batch.add(N, kU[c], C.len(), 1.0, src.blk(C.start, 0), src.lda, OP_T, nb[c].EU,
                                          C.len(), OP_N, 0.0, pu, N, nullptr, 0, C.start, 0);
                        if (kV[c])
                            gP->batch.add(N, kV[c], C.len(), 1.0, src.blk(0, C.start), src.lda, OP_N, nb[c].EV,
                                          C.len(), OP_N, 0.0, pv, N, nullptr, 0, 0, C.start);
                        continue;
                    }
                    const NestedNode& y = nb[c];
                    const Node& C1 = nodes_[C.left];
                    const Node& C2 = nodes_[C.right];
                    const int k1u = kU[C.left], k2u = kU[C.right], k1v = kV[C.left], k2v = kV[C.right];
                    if (kU[c]) {
                        gM->batch.add(N, kU[c], y.kpU, 1.0, y.XU, N, OP_N, y.Rf, y.kpU, OP_N, 0.0, pu, N);
                        if (k1u)
                            gM->batch.add(C1.len(), kU[c], k1u, 1.0, nb[C.left].EU, C1.len(), OP_N, y.Rf, y.kpU,
                                          OP_N, 0.0, y.EU, C.len());
                        else
                            pre->t.h.push_back({y.EU, C.len(), C1.len(), kU[c], 0.0});
                        if (k2u)
                            gM->batch.add(C2.len(), kU[c], k2u, 1.0, nb[C.right].EU, C2.len(), OP_N, y.Rf + k1u,
                                          y.kpU, OP_N, 0.0, y.EU + C1.len(), C.len());
                        else
                            pre->t.h.push_back({y.EU + C1.len(), C.len(), C2.len(), kU[c], 0.0});
                    }
                    if (kV[c]) {
                        gM->batch.add(N, kV[c], y.kpV, 1.0, y.XV, N, OP_N, y.Wf, y.kpV, OP_N, 0.0, pv, N);
                        if (k1v)
                            gM->batch.add(C1.len(), kV[c], k1v, 1.0, nb[C.left].EV, C1.len(), OP_N, y.Wf, y.kpV,
                                          OP_N, 0.0, y.EV, C.len());
                        else
                            pre->t.h.push_back({y.EV, C.len(), C1.len(), kV[c], 0.0});
                        if (k2v)
                            gM->batch.add(C2.len(), kV[c], k2v, 1.0, nb[C.right].EV, C2.len(), OP_N, y.Wf + k1v,
                                          y.kpV, OP_N, 0.0, y.EV + C1.len(), C.len());
                        else
                            pre->t.h.push_back({y.EV + C1.len(), C.len(), C2.len(), kV[c], 0.0});
                    }
                }
                const Node& A_ = nodes_[a];
                const Node& B_ = nodes_[b];
                if (kU[a] && kV[b])   // B12 = PU_a[I_b rows]^T V_b
                    gB->batch.add(kU[a], kV[b], B_.len(), 1.0, x.XU + B_.start, N, OP_T, nb[b].EV, B_.len(), OP_N,
                                  0.0, x.B12, kU[a]);
                if (kU[b] && kV[a])   // B21 = PU_b[I_a rows]^T V_a
                    gB->batch.add(kU[b], kV[a], A_.len(), 1.0, x.XU + (size_t)N * kU[a] + A_.start, N, OP_T,
                                  nb[a].EV, A_.len(), OP_N, 0.0, x.B21, kU[b]);
                if (d == 0) continue;   // the root has no strip
                for (int w = 0; w < 2; ++w) {
                    const int kp = w == 0 ? x.kpU : x.kpV;
                    if (!kp) continue;
                    double* X = w == 0 ? x.XU : x.XV;
                    cut->t.h.push_back({X + n.start, N, n.len(), kp, 0.0});
                    SvdProblem q{};
                    q.X = X; q.ldx = N; q.rows = N; q.k = kp;
                    q.L = nullptr;
                    q.R = w == 0 ? x.Rf : x.Wf; q.ldr = kp;
                    q.rank = dRank.p + 2 * i + w;
                    q.sort = true;
                    sv.push_back(q);
                }
            }
            auto add_gemm = [&](std::unique_ptr<GemmStep<double>>& g) {
                if (g->batch.empty()) return;
                g->batch.finalize(stream_);
                plan.add(std::move(g));
            };
            if (!pre->t.h.empty()) {
                pre->t.upload(stream_);
                plan.add(std::move(pre));
            }
            add_gemm(gP);
            add_gemm(gM);
            add_gemm(gB);
            if (!cut->t.h.empty()) {
                cut->t.upload(stream_);
                plan.add(std::move(cut));
            }
            plan_gram_svd(plan, sv, opts_.tol, opts_.max_rank, stream_);
            plan.run(stream_, dstatus.p);
            HM_CUDA(cudaStreamSynchronize(stream_));
            check_status("hss nested build");
            i0 = i1;
        }
        if (d > 0) {
            std::vector<int> rk(2 * lvl.size());
            HM_CUDA(cudaMemcpy(rk.data(), dRank.p, rk.size() * sizeof(int), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < lvl.size(); ++i) {
                const NestedNode& x = nb[lvl[i]];
                kU[lvl[i]] = x.kpU ? std::min(std::max(rk[2 * i], 0), x.kpU) : 0;
                kV[lvl[i]] = x.kpV ? std::min(std::max(rk[2 * i + 1], 0), x.kpV) : 0;
            }
        }
        below = std::move(pairs);   // this level's pairs feed the next level's panels
        below_ws = std::move(pair_ws);
    }
    below.reset();
    below_ws.release();

    // The engine's two-level storage: expanded bases of every non-root node, B per node.
    for (int i = 0; i < nn; ++i) {
        Node& n = nodes_[i];
        n.rankU = n.parent >= 0 ? kU[i] : 0;
        n.rankV = n.parent >= 0 ? kV[i] : 0;
        n.capU = n.rankU;
        n.capV = n.rankV;
    }
    alloc_UV();
    size_t totB = 0, totRW = 0;
    hss_.offR.assign(nn, 0);
    hss_.offW.assign(nn, 0);
    for (int i = 0; i < nn; ++i) {
        Node& n = nodes_[i];
        if (n.is_leaf) continue;
        n.offB12 = totB;
        totB += (size_t)kU[n.left] * kV[n.right];
        n.offB21 = totB;
        totB += (size_t)kU[n.right] * kV[n.left];
        if (n.parent >= 0) {
            hss_.offR[i] = totRW;
            totRW += (size_t)nb[i].kpU * kU[i];
            hss_.offW[i] = totRW;
            totRW += (size_t)nb[i].kpV * kV[i];
        }
    }
    dB.alloc(one(totB));
    hss_.RW.alloc(one(totRW));
    CopyStep cp;
    for (int i = 0; i < nn; ++i) {
        const Node& n = nodes_[i];
        const int len = n.len();
        if (n.parent >= 0) {
            if (kU[i]) cp.t.h.push_back({nb[i].EU, len, dU.p + n.offU, len, len, kU[i], 0});
            if (kV[i]) cp.t.h.push_back({nb[i].EV, len, dV.p + n.offV, len, len, kV[i], 0});
        }
        if (n.is_leaf) continue;
        const int a = n.left, b = n.right;
        if (kU[a] && kV[b]) cp.t.h.push_back({nb[i].B12, kU[a], dB.p + n.offB12, kU[a], kU[a], kV[b], 0});
        if (kU[b] && kV[a]) cp.t.h.push_back({nb[i].B21, kU[b], dB.p + n.offB21, kU[b], kU[b], kV[a], 0});
        if (n.parent >= 0) {
            const NestedNode& x = nb[i];
            if (kU[i]) cp.t.h.push_back({x.Rf, x.kpU, hss_.RW.p + hss_.offR[i], x.kpU, x.kpU, kU[i], 0});
            if (kV[i]) cp.t.h.push_back({x.Wf, x.kpV, hss_.RW.p + hss_.offW[i], x.kpV, x.kpV, kV[i], 0});
        }
    }
    if (!cp.t.h.empty()) {
        cp.t.upload(stream_);
        cp.run(stream_, dstatus.p);
        count_launch();
    }
    hss_.rankU.assign(nn, 0);
    hss_.rankV.assign(nn, 0);
    hss_.offB12.assign(nn, 0);
    hss_.offB21.assign(nn, 0);
    for (int i = 0; i < nn; ++i) {
        hss_.rankU[i] = nodes_[i].is_leaf ? kU[i] : nodes_[i].rankU;   // a root leaf keeps its strip's rank
        hss_.rankV[i] = nodes_[i].is_leaf ? kV[i] : nodes_[i].rankV;
        hss_.offB12[i] = nodes_[i].offB12;
        hss_.offB21[i] = nodes_[i].offB21;
    }
    hss_.B.alloc(dB.n);
    HM_CUDA(cudaMemcpyAsync(hss_.B.p, dB.p, dB.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    hss_.nested = true;
    HM_CUDA(cudaStreamSynchronize(stream_));
    check_status("hss nested form");
}

// Telescoping product of a nested-basis HSS operator, y = A~ x, O(N k) work:
//   up     g_leaf = V_leaf^T x_leaf,  g_t = W_t^T [g_a; g_b]          (deepest level first)
//   down   [f_a; f_b] = [B12_t g_b; B21_t g_a] + R_t f_t              (root first, no R there)
//   leaves y_leaf = D_leaf x_leaf + U_leaf f_leaf
// Siblings' g (and f) are adjacent rows of one buffer per parent, so every transfer is one
// product; the coupling and transfer terms of a block are one register-accumulated chain.
// The reference-form operator keeps the two-level product (its bases are the
// expanded ones by construction).
void Engine::add_matvec_nested(Plan& pl, const double* X, double* Y, int s) {
    const int nn = (int)nodes_.size();
    if (s <= 0) return;
    std::vector<double*> gpair(nn, nullptr), fpair(nn, nullptr);
    std::vector<int> kpU(nn, 0), kpV(nn, 0);
    for (int i = 0; i < nn; ++i) {
        const Node& n = nodes_[i];
        if (n.is_leaf) continue;
        kpU[i] = nodes_[n.left].rankU + nodes_[n.right].rankU;
        kpV[i] = nodes_[n.left].rankV + nodes_[n.right].rankV;
        gpair[i] = pl.scratch(std::max<size_t>((size_t)kpV[i] * s, 1));
        fpair[i] = pl.scratch(std::max<size_t>((size_t)kpU[i] * s, 1));
    }
    // the rows of node c inside its parent's pair buffers
    auto gslot = [&](int c) {
        const Node& P = nodes_[nodes_[c].parent];
        return gpair[nodes_[c].parent] + (c == P.right ? nodes_[P.left].rankV : 0);
    };
    auto fslot = [&](int c) {
        const Node& P = nodes_[nodes_[c].parent];
        return fpair[nodes_[c].parent] + (c == P.right ? nodes_[P.left].rankU : 0);
    };
    auto push = [&](std::unique_ptr<GemmStep<double>>& g) {
        if (g->batch.empty()) return;
        g->batch.finalize(stream_);
        pl.add(std::move(g));
    };
    auto zero = std::make_unique<IdentStep>();
    auto up0 = std::make_unique<GemmStep<double>>("matvec.hss_up");
    for (int l : leaves_) {
        const Node& n = nodes_[l];
        if (n.parent >= 0 && n.rankV)
            up0->batch.add(n.rankV, s, n.len(), 1.0, dV.p + n.offV, n.len(), OP_T, X + n.start, N_, OP_N, 0.0,
                           gslot(l), kpV[n.parent]);
    }
    std::vector<std::unique_ptr<GemmStep<double>>> up, down;
    for (int d = (int)levels_.size() - 1; d >= 1; --d) {
        auto g = std::make_unique<GemmStep<double>>("matvec.hss_up");
        for (int t : levels_[d]) {
            const Node& n = nodes_[t];
            if (n.rankV && kpV[t])
                g->batch.add(n.rankV, s, kpV[t], 1.0, hss_.RW.p + hss_.offW[t], kpV[t], OP_T, gpair[t], kpV[t],
                             OP_N, 0.0, gslot(t), kpV[n.parent]);
        }
        up.push_back(std::move(g));
    }
    for (size_t d = 0; d < levels_.size(); ++d) {
        auto g = std::make_unique<GemmStep<double>>("matvec.hss_down");
        for (int t : levels_[d]) {
            const Node& n = nodes_[t];
            const int a = n.left, b = n.right;
            for (int side = 0; side < 2; ++side) {
                const int rows = side == 0 ? nodes_[a].rankU : nodes_[b].rankU;
                if (!rows) continue;
                double* F = fpair[t] + (side == 0 ? 0 : nodes_[a].rankU);
                const int kc = side == 0 ? nodes_[b].rankV : nodes_[a].rankV;   // coupling width
                const double* Bm = dB.p + (side == 0 ? n.offB12 : n.offB21);
                const double* gc = gpair[t] + (side == 0 ? nodes_[a].rankV : 0);
                const bool has_r = n.parent >= 0 && n.rankU > 0;
                const double* Rm = has_r ? hss_.RW.p + hss_.offR[t] + (side == 0 ? 0 : nodes_[a].rankU) : nullptr;
                if (kc) {
                    g->batch.add(rows, s, kc, 1.0, Bm, rows, OP_N, gc, kpV[t], OP_N, 0.0, F, kpU[t], nullptr, 1);
                    if (has_r) g->batch.add_chained(rows, s, n.rankU, 1.0, Rm, kpU[t], OP_N, fslot(t), kpU[n.parent], OP_N);
                } else if (has_r) {
                    g->batch.add(rows, s, n.rankU, 1.0, Rm, kpU[t], OP_N, fslot(t), kpU[n.parent], OP_N, 0.0, F,
                                 kpU[t]);
                } else {
                    zero->t.h.push_back({F, kpU[t], rows, s, 0.0});
                }
            }
        }
        down.push_back(std::move(g));
    }
    auto leaf = std::make_unique<GemmStep<double>>("matvec.leaf_expand");
    for (int l : leaves_) {
        const Node& n = nodes_[l];
        leaf->batch.add(n.len(), s, n.len(), 1.0, dD.p + n.offD, n.len(), OP_N, X + n.start, N_, OP_N, 0.0,
                        Y + n.start, N_, nullptr, 1);
        if (n.parent >= 0 && n.rankU)
            leaf->batch.add_chained(n.len(), s, n.rankU, 1.0, dU.p + n.offU, n.len(), OP_N, fslot(l),
                                    kpU[n.parent], OP_N);
    }
    if (!zero->t.h.empty()) {
        zero->t.upload(stream_);
        pl.add(std::move(zero));
    }
    push(up0);
    for (auto& g : up) push(g);
    for (auto& g : down) push(g);
    push(leaf);
}

}  // namespace hm
