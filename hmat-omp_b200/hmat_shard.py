"""Subtree sharding of one HODLR system across ranks (one process per GPU).

The reference parallelises one operator with OpenMP tasks over the subtrees of its
bisection tree (include/hodlr_routines_omp.h:48-56, 103-113, 164-174).  Here the same
tree is cut at depth p for P = 2^p ranks:

* rank g owns the depth-p subtree over rows [start_g, end_g) (the reference's split rule,
  mid = (s + e) / 2).  Its leaves, its subtree's couplings, their factorization and its
  part of every solve are local: a *local solver* applies A_g^{-1} (on a GPU the CUDA
  engine with the subtree's factors, hm_hodlr_import; on a CPU any object with a
  ``solve`` method).
* a top node n (depth < p) couples its children c1, c2 by A12 = U1 B12 V2^T and
  A21 = U2 B21 V1^T; the bases' rows are spread over the ranks under each child, B12 and
  B21 are replicated.  Its Woodbury factorization (the stable form I + K B^ of
  hss_routines.h:253-254, as the single-GPU engine uses) needs K = diag(V1^T Q1, V2^T Q2)
  and, for every basis block W on n's path, t = [V1^T W1; V2^T W2]: sums over rows, i.e.
  all-reduces of small matrices.  M^{-1} and P = B^ M^{-1} are computed redundantly.
* a solve is z = A_g^{-1} b_g locally, then per top level t = [V1^T z1; V2^T z2]
  (all-reduce of r x s), delta = P t, z -= Q delta on local rows.

Every rank issues the same collectives in the same order: one buffer per top depth packs
the contributions for all nodes of that depth (zeros where a rank has no rows), so shapes
agree across ranks.  Collectives are sums through the caller's ``allreduce`` (NCCL or
gloo through torch.distributed); no device kernel waits on another rank and no operand is
read from a peer's memory.
"""
from __future__ import annotations

from dataclasses import dataclass, field


# ------------------------------------------------------------------------------------
# Partition plan (pure host logic)
# ------------------------------------------------------------------------------------
@dataclass
class TopNode:
    depth: int
    start: int
    mid: int
    end: int
    slot: int            # position among the top nodes of its depth (left to right)
    ranks: tuple         # (first rank, one past the last rank) under this node


@dataclass
class ShardPlan:
    N: int
    leaf: int
    world: int
    p: int
    bounds: list                                   # rank -> (start, end)
    levels: list = field(default_factory=list)     # depth -> [TopNode, ...]

    def owner_range(self, rank: int):
        return self.bounds[rank]

    def path(self, rank: int):
        """Top nodes containing rank's rows, depth 0 first."""
        s, e = self.bounds[rank]
        return [next(n for n in lvl if n.start <= s and e <= n.end) for lvl in self.levels]

    def side(self, node: TopNode, rank: int) -> int:
        """0 if rank's rows are in the left child of node, 1 if in the right."""
        return 0 if self.bounds[rank][1] <= node.mid else 1


def partition(N: int, leaf: int, world: int) -> ShardPlan:
    """Cut the reference's tree (hodlr_routines.h:27-45: mid = (s+e)/2, leaf iff
    len <= leaf) at depth p = log2(world).  Every top node must be internal."""
    p = world.bit_length() - 1
    if world < 1 or (1 << p) != world:
        raise ValueError(f"subtree sharding needs a power-of-two number of ranks, got {world}")
    levels = []
    spans = [(0, N)]
    for d in range(p):
        lvl, nxt = [], []
        for i, (s, e) in enumerate(spans):
            if e - s <= leaf:
                raise ValueError(f"rows [{s}, {e}) form a leaf above depth {p}: too many ranks for N={N}, leaf={leaf}")
            m = (s + e) // 2
            per = world >> d
            lvl.append(TopNode(d, s, m, e, i, (i * per, (i + 1) * per)))
            nxt += [(s, m), (m, e)]
        levels.append(lvl)
        spans = nxt
    return ShardPlan(N, leaf, world, p, spans, levels)


# ------------------------------------------------------------------------------------
# Array back ends
# ------------------------------------------------------------------------------------
class NumpyOps:
    def __init__(self):
        import numpy as np
        self.np = np

    def zeros(self, r, c, like=None):
        return self.np.zeros((r, c))

    def eye(self, n, like=None):
        return self.np.eye(n)

    def inv(self, a):
        return self.np.linalg.inv(a)

    def hcat(self, xs):
        return self.np.concatenate(xs, axis=1)

    def copy(self, a):
        return a.copy()


class TorchOps:
    def __init__(self, device):
        import torch
        self.torch = torch
        self.device = device

    def zeros(self, r, c, like=None):
        return self.torch.zeros((r, c), dtype=self.torch.float64, device=self.device)

    def eye(self, n, like=None):
        return self.torch.eye(n, dtype=self.torch.float64, device=self.device)

    def inv(self, a):
        return self.torch.linalg.inv(a)

    def hcat(self, xs):
        return self.torch.cat(xs, dim=1)

    def copy(self, a):
        return a.clone()


def torch_allreduce(buf):
    """Sum over all ranks with torch.distributed (NCCL for device tensors, gloo on CPU)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(buf)
    return buf


def numpy_allreduce_gloo(buf):
    """Sum of a numpy array over all ranks through torch.distributed (gloo)."""
    import torch
    t = torch.from_numpy(buf.copy())
    torch_allreduce(t)
    return t.numpy()


# ------------------------------------------------------------------------------------
# Sharded factorization and solve
# ------------------------------------------------------------------------------------
@dataclass
class TopCoupling:
    """Node n's coupling, as rank g sees it: its rows of the bases of the child on its
    side, and the replicated coupling blocks and ranks."""
    B12: object          # p1 x q2
    B21: object          # p2 x q1
    U: object            # rows of this rank x p_side (the side child's U)
    V: object            # rows of this rank x q_side (the side child's V)


class ShardedHODLR:
    """Rank-local part of one HODLR operator sharded by subtrees.

    plan      ShardPlan from partition()
    rank      this rank
    local     object with solve(Y) -> A_g^{-1} Y for this rank's subtree (rows x cols)
    top       {depth: TopCoupling} for the top nodes on this rank's path
    ranks     {(depth, slot): (p1, p2, q1, q2)} for every top node (replicated metadata)
    ops       NumpyOps() or TorchOps(device)
    allreduce function summing an array over all ranks (in place or returning the sum)
    """

    def __init__(self, plan: ShardPlan, rank: int, local, top: dict, ranks: dict, ops, allreduce):
        self.plan, self.rank, self.local, self.top, self.ranks = plan, rank, local, top, ranks
        self.ops, self.allreduce = ops, allreduce
        self.path = plan.path(rank)
        self.factored = False
        self.collectives = 0

    # -- packing of per-depth collectives --------------------------------------------
    def _reduce_packed(self, d: int, shapes: list, mine):
        """All-reduce one buffer holding a block per top node of depth d (shapes[i] =
        (rows, cols) of node i's block); this rank fills its node's block with `mine`."""
        self.collectives += 1
        return _packed_allreduce(self.ops, self.allreduce, shapes, self.path[d].slot, mine)

    def _side_rows(self, d: int):
        n = self.path[d]
        p1, p2, q1, q2 = self.ranks[(d, n.slot)]
        side = self.plan.side(n, self.rank)
        return n, side, (p1, p2, q1, q2)

    # -- factorization ------------------------------------------------------------------
    def factor(self):
        """Bottom-up over the top levels, after the local subtree: Q = A_child^{-1} U on
        every basis block of this rank's path, K, M, P per top node."""
        ops, p = self.ops, self.plan.p
        # basis blocks on the path: W[d] = rows of this rank of U of the child at depth
        # d + 1 (the side child of the depth-d top node); first A_g^{-1} W locally
        blocks = [self.top[d].U for d in range(p)]
        widths = [b.shape[1] for b in blocks]
        Wall = self.local.solve(ops.hcat(blocks)) if sum(widths) else None
        W, c0 = [], 0
        for w in widths:
            W.append(Wall[:, c0:c0 + w] if w else blocks[0][:, :0])
            c0 += w
        self.Q, self.P = {}, {}
        for d in range(p - 1, -1, -1):
            n, side, (p1, p2, q1, q2) = self._side_rows(d)
            Qs, Vs = W[d], self.top[d].V
            # K = diag(V1^T Q1, V2^T Q2): this rank's rows contribute to its side's block
            shapes = [((lambda r: (r[2] + r[3], r[0] + r[1]))(self.ranks[(d, m.slot)])) for m in self.plan.levels[d]]
            mine = ops.zeros(q1 + q2, p1 + p2)
            if side == 0:
                mine[:q1, :p1] = Vs.T @ Qs
            else:
                mine[q1:, p1:] = Vs.T @ Qs
            K = self._reduce_packed(d, shapes, mine)
            Bh = ops.zeros(p1 + p2, q1 + q2)
            Bh[:p1, q1:] = self.top[d].B12
            Bh[p1:, :q1] = self.top[d].B21
            M = ops.eye(q1 + q2) + K @ Bh
            P = Bh @ ops.inv(M)
            self.Q[d], self.P[d] = ops.copy(Qs), P
            # every basis block on the path above this node: W <- A_n^{-1} W
            cols = [widths[e] for e in range(d)]
            if d > 0:
                shapes = [(self.ranks[(d, m.slot)][2] + self.ranks[(d, m.slot)][3],
                           sum(self._path_widths_for(d, m))) for m in self.plan.levels[d]]
                Wcat = ops.hcat([W[e] for e in range(d)])
                mine = ops.zeros(q1 + q2, Wcat.shape[1])
                if side == 0:
                    mine[:q1] = Vs.T @ Wcat
                else:
                    mine[q1:] = Vs.T @ Wcat
                t = self._reduce_packed(d, shapes, mine)
                delta = P @ t
                upd = Qs @ (delta[:p1] if side == 0 else delta[p1:])
                c0 = 0
                for e in range(d):
                    W[e] = W[e] - upd[:, c0:c0 + cols[e]]
                    c0 += cols[e]
        self.factored = True

    def _path_widths_for(self, d: int, node: TopNode):
        """Widths of the basis blocks on node's path above it (depths 0..d-1: the side
        child of each ancestor), from the replicated rank table."""
        out = []
        for e in range(d):
            anc = next(m for m in self.plan.levels[e] if m.start <= node.start and node.end <= m.end)
            p1, p2, _, _ = self.ranks[(e, anc.slot)]
            out.append(p1 if node.end <= anc.mid else p2)
        return out

    # -- solve ----------------------------------------------------------------------------
    def solve(self, b):
        """x = A^{-1} b on this rank's rows (b: rows x s)."""
        if not self.factored:
            self.factor()
        ops = self.ops
        z = self.local.solve(b)
        s = b.shape[1]
        for d in range(self.plan.p - 1, -1, -1):
            n, side, (p1, p2, q1, q2) = self._side_rows(d)
            shapes = [(self.ranks[(d, m.slot)][2] + self.ranks[(d, m.slot)][3], s) for m in self.plan.levels[d]]
            mine = ops.zeros(q1 + q2, s)
            if side == 0:
                mine[:q1] = self.top[d].V.T @ z
            else:
                mine[q1:] = self.top[d].V.T @ z
            t = self._reduce_packed(d, shapes, mine)
            delta = self.P[d] @ t
            z = z - self.Q[d] @ (delta[:p1] if side == 0 else delta[p1:])
        return z


# ------------------------------------------------------------------------------------
# Slicing a whole operator's factors into a rank's share
# ------------------------------------------------------------------------------------
def rank_share(plan: ShardPlan, rank: int, nodes):
    """From a whole-operator tree in the reference's pre-order (objects with start, end,
    is_leaf, depth, left, right and D/U/V/B12/B21), the rank's subtree nodes (re-indexed
    from its own root) and its TopCoupling per top depth, plus the replicated rank table.
    Used when every rank holds (or can export) the whole operator's factors."""
    s, e = plan.bounds[rank]
    by_range = {(n.start, n.end): n for n in nodes}
    top, table = {}, {}
    for d, lvl in enumerate(plan.levels):
        for m in lvl:
            n = by_range[(m.start, m.end)]
            table[(d, m.slot)] = (n.B12.shape[0], n.B21.shape[0], n.B21.shape[1], n.B12.shape[1])
    for d, m in enumerate(plan.path(rank)):
        n = by_range[(m.start, m.end)]
        child = n.left if e <= m.mid else n.right
        o0, o1 = s - child.start, e - child.start
        top[d] = TopCoupling(n.B12, n.B21, child.U[o0:o1], child.V[o0:o1])
    sub = [n for n in nodes if s <= n.start and n.end <= e]
    return sub, top, table


# ------------------------------------------------------------------------------------
# GPU side: the rank's subtree on the CUDA engine, shares exported from a built handle
# ------------------------------------------------------------------------------------
@dataclass
class TreeNode:
    start: int
    end: int
    depth: int
    is_leaf: bool
    left: "TreeNode | None" = None
    right: "TreeNode | None" = None
    index: int = 0
    D: object = None
    U: object = None
    V: object = None
    B12: object = None
    B21: object = None


def nodes_from_handle(h, rows):
    """The HODLR tree of a built handle (pre-order, hm_export_tree) as TreeNodes, with the
    factors (hm_get_factor) of the nodes inside rows = (start, end) and of the nodes above
    it (their coupling blocks and the bases of their children) downloaded."""
    t = h.tree()
    nodes = [TreeNode(int(t["start"][i]), int(t["end"][i]), int(t["depth"][i]), bool(t["is_leaf"][i]), index=i)
             for i in range(len(t["start"]))]
    stack = []
    for n in nodes:   # pre-order: a node's left child follows it, its right child starts at mid
        while stack and not (stack[-1].start <= n.start and n.end <= stack[-1].end):
            stack.pop()
        if stack:
            par = stack[-1]
            if par.left is None:
                par.left = n
            else:
                par.right = n
        if not n.is_leaf:
            stack.append(n)
    s, e = rows
    D, U, V, B12, B21 = 0, 1, 2, 3, 4
    for n in nodes:
        inside = s <= n.start and n.end <= e
        above = n.start <= s and e <= n.end and not inside
        if inside and n.is_leaf:
            n.D = h.get_factor(n.index, D)
        if inside or above:
            if not n.is_leaf:
                n.B12, n.B21 = h.get_factor(n.index, B12), h.get_factor(n.index, B21)
                for c in (n.left, n.right):
                    if c.U is None and c.index > 0:
                        c.U, c.V = h.get_factor(c.index, U), h.get_factor(c.index, V)
    return nodes


class EngineLocalSolver:
    """A_g^{-1} for a rank's subtree on the CUDA engine: the subtree's factors imported into
    a handle (hm_hodlr_import), FP64 factorization; solve() takes and returns torch
    tensors of rows x columns on the device.  The handle works on torch's current stream
    (or the given one), so its results are ordered with the torch operations around it."""

    def __init__(self, sub_nodes, start: int, leaf: int, stream_ptr: int | None = None):
        import torch

        import hmat_b200 as H
        if stream_ptr is None:
            # torch's default stream has handle 0, which hm_set_stream reads as "the
            # handle's own stream": name the legacy default stream (1) instead
            stream_ptr = torch.cuda.current_stream().cuda_stream or 1
        local = []
        for n in sub_nodes:
            c = TreeNode(n.start - start, n.end - start, n.depth, n.is_leaf, index=len(local), D=n.D, U=n.U, V=n.V,
                         B12=n.B12, B21=n.B21)
            local.append(c)
        self.N = local[0].end
        self.h = H.HODLRMatrix(1e-14)
        self.h.set_stream(stream_ptr)
        self.h.import_factors(self.N, leaf, local)

    @classmethod
    def from_handle(cls, h):
        """The whole operator of a built handle as the local solver (a single rank); the
        handle must work on torch's current stream (set_stream)."""
        self = cls.__new__(cls)
        self.h, self.N = h, h.N
        return self

    def factor(self):
        self.h.factor()

    def solve(self, Y):
        import torch
        Yc = Y.T.contiguous()                  # column-major rows x cols
        X = torch.empty_like(Yc)
        self.h.solve_device(Yc.data_ptr(), Yc.shape[0], self.N, X.data_ptr(), self.N)
        return X.T

    def close(self):
        self.h.close()


def to_torch_share(top: dict, device):
    """TopCouplings with numpy blocks -> the same with FP64 device tensors."""
    import torch
    cv = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device)
    return {d: TopCoupling(cv(c.B12), cv(c.B21), cv(c.U), cv(c.V)) for d, c in top.items()}


# ------------------------------------------------------------------------------------
# Sharded compression of the top-level couplings
# ------------------------------------------------------------------------------------
def _packed_allreduce(ops, allreduce, shapes: list, me: int, mine):
    """Sum over all ranks of one buffer holding block i (shapes[i] = (rows, cols)) side by
    side; this rank writes `mine` into block `me` and gets that block's sum back."""
    rows = max(max(r for r, _ in shapes), 1)
    offs, c0 = [], 0
    for _, c in shapes:
        offs.append(c0)
        c0 += c
    buf = ops.zeros(rows, max(c0, 1))
    r, c = shapes[me]
    if r and c and mine is not None:
        buf[:r, offs[me]:offs[me] + c] = mine
    out = allreduce(buf)
    out = buf if out is None else out
    return out[:r, offs[me]:offs[me] + c]


def build_top_sharded(plan: ShardPlan, rank: int, block_product, tol: float, max_rank: int, oversample: int = 10,
                      power_iters: int = 0, seed: int = 0, ops=None, allreduce=None):
    """Compress the couplings of every top node (depth < p) with their rows spread over
    the ranks, so that no rank builds more than its own rows of the operator.

    For top node n with children c1 = [start, mid) and c2 = [mid, end), the ranks under c1
    hold A12 = A[c1, c2] by rows and the ranks under c2 hold A21 = A[c2, c1].  Each block
    is compressed by a randomized range finder (the steps of compression.h:67-99) whose
    row dimension is distributed:
      Y_g = A[R_g, C] Omega          (local rows R_g; Omega |C| x k from (seed, depth,
                                      slot, side), the same on every rank of the block)
      [power iterations: Y_g = A[R_g, C] (sum_g A[R_g, C]^T Q_g)]
      Q_g = Y_g W L^{-1/2}            (Gram-eigen orthonormalisation, twice: G = sum_g
                                      Y_g^T Y_g is all-reduced, k x k; directions with
                                      eigenvalues below 1e-28 of the largest become zero)
      X   = sum_g A[R_g, C]^T Q_g     (all-reduced, |C| x k)
      X   = Z S W^T (SVD, redundantly on every rank of the block)
      A[R, C] ~= (Q W_r) diag(S_r) Z_r^T,  r = #{S_i > tol S_0} (<= max_rank, >= 1).
    U rows stay where they were computed; Z_r (the other child's basis) and S_r go to the
    ranks under the other child by one packed all-reduce per depth.

    block_product(r0, r1, c0, c1, X, trans) returns A[r0:r1, c0:c1] @ X (trans False) or
    A[r0:r1, c0:c1]^T @ X (trans True) in the ops back end.  Every rank issues the same
    collectives in the same order (packed per depth).  Returns (top, table, count):
    {depth: TopCoupling} for this rank's path, the replicated rank table
    {(depth, slot): (p1, p2, q1, q2)} that ShardedHODLR takes, and the number of
    collectives issued."""
    import numpy as np
    ops = ops or NumpyOps()
    allreduce = allreduce or numpy_allreduce_gloo
    k = max_rank + oversample
    s_g, e_g = plan.bounds[rank]
    top, table, count = {}, {}, 0

    def to_np(a):
        return a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)

    def from_np(a, like):
        if hasattr(like, "detach"):
            import torch
            return torch.as_tensor(a, dtype=torch.float64, device=like.device)
        return np.asarray(a, dtype=np.float64)

    for d, lvl in enumerate(plan.levels):
        me = plan.path(rank)[d]
        side = plan.side(me, rank)
        # block of node i, side j at position 2 i + j in every packed buffer
        pos = 2 * me.slot + side
        R0, R1 = (me.start, me.mid) if side == 0 else (me.mid, me.end)     # this block's rows
        C0, C1 = (me.mid, me.end) if side == 0 else (me.start, me.mid)     # its columns
        ncol = C1 - C0
        colsz = []
        for m in lvl:
            colsz += [m.end - m.mid, m.mid - m.start]

        def reduce_kk(mine):
            nonlocal count
            count += 1
            return _packed_allreduce(ops, allreduce, [(k, k)] * (2 * len(lvl)), pos, mine)

        def reduce_cols(mine):
            nonlocal count
            count += 1
            return _packed_allreduce(ops, allreduce, [(c, k) for c in colsz], pos, mine)

        def orth(Y):
            for _ in range(2):
                G = to_np(reduce_kk(Y.T @ Y))
                G = 0.5 * (G + G.T)
                lam, W = np.linalg.eigh(G)
                lmax = max(lam.max(), 0.0)
                keep = lam > 1e-28 * lmax if lmax > 0 else np.zeros_like(lam, dtype=bool)
                scale = np.where(keep, 1.0 / np.sqrt(np.where(keep, lam, 1.0)), 0.0)
                Y = Y @ from_np(W * scale[None, :], Y)
            return Y

        omega = np.random.default_rng([seed, d, me.slot, side]).standard_normal((ncol, k))
        like = ops.zeros(1, 1)
        Y = block_product(s_g, e_g, C0, C1, from_np(omega, like), False)
        for _ in range(power_iters):
            Q = orth(Y)
            Z = reduce_cols(block_product(s_g, e_g, C0, C1, Q, True))
            Y = block_product(s_g, e_g, C0, C1, Z, False)
        Q = orth(Y)
        X = to_np(reduce_cols(block_product(s_g, e_g, C0, C1, Q, True)))
        Zs, S, Wt = np.linalg.svd(X, full_matrices=False)
        r = 1
        if S.size and S[0] > 1e-15:
            r = max(1, min(int(np.sum(S > tol * S[0])), max_rank))
        U_rows = Q @ from_np(Wt.T[:, :r], Q)
        # ranks and singular values to everyone (only the first rank of each block
        # contributes, so the sums are the values)
        first = (s_g == R0)
        meta = np.zeros((1, 1 + max_rank))
        if first:
            meta[0, 0] = r
            meta[0, 1:1 + r] = S[:r]
        count += 1
        allmeta = to_np(allreduce(from_np(np.concatenate(
            [meta if i == pos else np.zeros_like(meta) for i in range(2 * len(lvl))], axis=1), like)))
        rk = [int(round(allmeta[0, i * (1 + max_rank)])) for i in range(2 * len(lvl))]
        sv = [allmeta[0, i * (1 + max_rank) + 1:i * (1 + max_rank) + 1 + rk[i]] for i in range(2 * len(lvl))]
        for i, m in enumerate(lvl):
            r12, r21 = rk[2 * i], rk[2 * i + 1]
            table[(d, m.slot)] = (r12, r21, r21, r12)
        # the other child's basis: block (2 i + j) carries Z_r of side j (|C_j| x r_j),
        # written by the block's first rank; each rank reads the opposite block
        shapes = [(colsz[i], rk[i]) for i in range(2 * len(lvl))]
        rows = max(max(c for c, _ in shapes), 1)
        offs, c0 = [], 0
        for _, c in shapes:
            offs.append(c0)
            c0 += c
        buf = ops.zeros(rows, max(c0, 1))
        if first:
            buf[:ncol, offs[pos]:offs[pos] + r] = from_np(Zs[:, :r], like)
        count += 1
        out = allreduce(buf)
        out = buf if out is None else out
        o = pos ^ 1
        Vother = out[:colsz[o], offs[o]:offs[o] + rk[o]]   # the basis of this rank's child, all rows
        B_mine = from_np(np.diag(sv[pos]), like)
        B_other = from_np(np.diag(sv[pos ^ 1]), like)
        V_rows = Vother[s_g - R0:e_g - R0]
        if side == 0:
            top[d] = TopCoupling(B_mine, B_other, U_rows, V_rows)
        else:
            top[d] = TopCoupling(B_other, B_mine, U_rows, V_rows)
    return top, table, count


def device_block_product(dense, kernel: int, points, params):
    """block_product for build_top_sharded on the device: A[r0:r1, c0:c1] @ X (or the
    transposed product) with A's entries generated by the engine
    (hm_kernel_block_product_device), never stored.  X and the result are FP64 torch
    tensors on the device; `dense` is an hmat_b200.Dense handle working on torch's current
    stream, `points` the host points of hm_hodlr_build_from_kernel's layout."""
    import torch

    def prod(r0, r1, c0, c1, X, trans):
        m = (c1 - c0) if trans else (r1 - r0)
        k, s = X.shape
        Xc = X.T.contiguous()                                   # column-major k x s
        Yc = torch.empty((s, m), dtype=torch.float64, device=X.device)
        dense.kernel_block_product(kernel, points, params, r0, r1, c0, c1, Xc.data_ptr(), max(k, 1), s,
                                   Yc.data_ptr(), max(m, 1), trans=trans)
        return Yc.T
    return prod
