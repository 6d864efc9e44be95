"""Node partition, split CSR and halo plan for running the SW2 linear algebra on
several ranks, and the distributed matrix-vector product and dot product over
torch.distributed (gloo on CPU here; the same plan serves NCCL ranks).

The layout restates the reference's distributed design:

* nodes split into contiguous ranges, ``npes`` ranges of ``nnodes // npes`` nodes
  with the remainder on the last rank (node_ind_ptr, src/structs/sgrid/sgrid_read.c:172-178);
* each rank owns the dofs of its nodes and holds a split CSR
  (src/structs/slin_sys/slin_sys.h:13-22): a diagonal block whose columns are local
  dof numbers, and an off-diagonal block whose columns are global dof numbers of
  ghost dofs, resolved through the rank's ``ghosts`` list (local number =
  nrows + position in ghosts, global_to_local);
* y = A x row by row, the diagonal block's entries first and then the off-diagonal
  block's, each in column order (split_CSR_mat_vec_mult, src/la/matrix_utilities.c:177-215).

The ghost values come from their owners before each product (the halo exchange the
reference leaves stubbed at src/la/bcgstab_solver.c:152-158).  Ghost dofs are kept in
increasing global order.  Host code: the arrays are numpy, the exchange is
torch.distributed point-to-point on CPU tensors.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List

import numpy as np


def node_ranges(nnodes: int, npes: int) -> np.ndarray:
    """node_ind_ptr: rank r owns nodes [ptr[r], ptr[r+1])."""
    per = nnodes // npes
    ptr = np.arange(npes + 1, dtype=np.int64) * per
    ptr[npes] = nnodes
    return ptr


@dataclass
class RankCSR:
    rank: int
    row0: int                      # first owned global dof
    nrows: int                     # owned dofs
    indptr_diag: np.ndarray
    cols_diag: np.ndarray          # local dof numbers
    vals_diag: np.ndarray
    indptr_off: np.ndarray
    cols_off: np.ndarray           # global dof numbers (ghosts)
    vals_off: np.ndarray
    ghosts: np.ndarray             # sorted global dof numbers of the ghost dofs
    send: Dict[int, np.ndarray] = field(default_factory=dict)   # peer -> owned global dofs the peer needs
    recv: Dict[int, np.ndarray] = field(default_factory=dict)   # peer -> positions in ghosts it fills


def split(indptr: np.ndarray, cols: np.ndarray, vals: np.ndarray, nnodes: int, npes: int) -> List[RankCSR]:
    """Every rank's split CSR of the global CSR (dof = 3 node + var) and the halo plan."""
    ptr = node_ranges(nnodes, npes)
    dof_ptr = 3 * ptr
    out = []
    for r in range(npes):
        r0, r1 = int(dof_ptr[r]), int(dof_ptr[r + 1])
        ip_d, c_d, v_d, ip_o, c_o, v_o = [0], [], [], [0], [], []
        for row in range(r0, r1):
            k0, k1 = int(indptr[row]), int(indptr[row + 1])
            c, v = cols[k0:k1], vals[k0:k1]
            own = (c >= r0) & (c < r1)
            c_d.append(c[own] - r0); v_d.append(v[own])
            c_o.append(c[~own]); v_o.append(v[~own])
            ip_d.append(ip_d[-1] + int(own.sum())); ip_o.append(ip_o[-1] + int((~own).sum()))
        cat = lambda a, dt: np.concatenate(a).astype(dt) if a else np.zeros(0, dt)   # noqa: E731
        cols_off = cat(c_o, np.int64)
        ghosts = np.unique(cols_off)
        out.append(RankCSR(r, r0, r1 - r0, np.array(ip_d, np.int64), cat(c_d, np.int64), cat(v_d, vals.dtype),
                           np.array(ip_o, np.int64), cols_off, cat(v_o, vals.dtype), ghosts))
    owner = lambda g: int(np.searchsorted(dof_ptr, g, side="right") - 1)   # noqa: E731
    for p in out:
        if p.ghosts.size == 0:
            continue
        owners = np.array([owner(g) for g in p.ghosts])
        for q in np.unique(owners):
            sel = np.nonzero(owners == q)[0]
            p.recv[int(q)] = sel
            out[int(q)].send[p.rank] = p.ghosts[sel]
    return out


def local_index(p: RankCSR, g: np.ndarray) -> np.ndarray:
    """global_to_local for ghost dofs: nrows + position in the ghost list."""
    return p.nrows + np.searchsorted(p.ghosts, g)


def matvec_local(p: RankCSR, x_ext: np.ndarray) -> np.ndarray:
    """split_CSR_mat_vec_mult on one rank: x_ext = owned values then ghost values."""
    y = np.zeros(p.nrows, dtype=x_ext.dtype)
    off_local = local_index(p, p.cols_off)
    for i in range(p.nrows):
        s = 0.0
        for j in range(p.indptr_diag[i], p.indptr_diag[i + 1]):
            s += p.vals_diag[j] * x_ext[p.cols_diag[j]]
        for k in range(p.indptr_off[i], p.indptr_off[i + 1]):
            s += p.vals_off[k] * x_ext[off_local[k]]
        y[i] = s
    return y


def halo_exchange(p: RankCSR, x_own: np.ndarray, dist) -> np.ndarray:
    """Owned values plus the ghost values received from their owners (point-to-point,
    every pair in the same order on both sides)."""
    import torch
    x_ext = np.concatenate([x_own, np.zeros(p.ghosts.size, x_own.dtype)])
    reqs, bufs = [], {}
    for q, dofs in sorted(p.send.items()):
        t = torch.from_numpy(np.ascontiguousarray(x_own[dofs - p.row0]))
        reqs.append(dist.isend(t, dst=q))
        bufs[("s", q)] = t
    for q, pos in sorted(p.recv.items()):
        t = torch.empty(len(pos), dtype=torch.float64 if x_own.dtype == np.float64 else torch.float32)
        reqs.append(dist.irecv(t, src=q))
        bufs[("r", q)] = t
    for rq in reqs:
        rq.wait()
    for q, pos in p.recv.items():
        x_ext[p.nrows + pos] = bufs[("r", q)].numpy()
    return x_ext


def matvec(p: RankCSR, x_own: np.ndarray, dist) -> np.ndarray:
    return matvec_local(p, halo_exchange(p, x_own, dist))


def dot(a_own: np.ndarray, b_own: np.ndarray, dist) -> float:
    """Global dot product: local sums, then one all-reduce (messg_dsum)."""
    import torch
    t = torch.tensor([float(np.dot(a_own, b_own))], dtype=torch.float64)
    dist.all_reduce(t)
    return float(t.item())


def _gmax(v: np.ndarray, dist) -> float:
    import torch
    t = torch.tensor([float(np.max(np.abs(v))) if v.size else 0.0], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def block_jacobi_inverse(p: RankCSR) -> np.ndarray:
    """Inverses of the owned nodes' 3x3 diagonal blocks (Gauss-Jordan with partial
    pivoting; a singular block is replaced by the identity).  The blocks lie in the
    diagonal part of the split CSR, so no exchange is needed."""
    nn = p.nrows // 3
    inv = np.zeros((nn, 3, 3))
    for b in range(nn):
        a = np.zeros((3, 6))
        a[:, 3:] = np.eye(3)
        for r in range(3):
            row = 3 * b + r
            for j in range(p.indptr_diag[row], p.indptr_diag[row + 1]):
                c = p.cols_diag[j] - 3 * b
                if 0 <= c < 3:
                    a[r, c] = p.vals_diag[j]
        ok = True
        for c in range(3):
            piv = c + int(np.argmax(np.abs(a[c:, c])))
            if a[piv, c] == 0.0:
                ok = False
                break
            if piv != c:
                a[[c, piv]] = a[[piv, c]]
            a[c] /= a[c, c]
            for r in range(3):
                if r != c:
                    a[r] -= a[r, c] * a[c]
        inv[b] = a[:, 3:] if ok else np.eye(3)
    return inv


def _bj_apply(inv: np.ndarray, v: np.ndarray) -> np.ndarray:
    w = v.reshape(-1, 3)
    return (inv[:, :, 0] * w[:, :1] + inv[:, :, 1] * w[:, 1:2] + inv[:, :, 2] * w[:, 2:3]).ravel()


def bicgstab_bj(p: RankCSR, x_own: np.ndarray, b_own: np.ndarray, scale_own: np.ndarray, dist,
                max_it: int = 100, tol: float = 1e-11):
    """The reference's left-preconditioned BiCGStab (solve_linear_sys_bcgstab,
    src/la/bcgstab_solver.c:65-230: x0 = M^-1 b, stop when max|r| <= tol + tol max|M^-1 b|)
    with the block-Jacobi preconditioner, on this rank's rows: every product goes
    through the halo exchange, every dot product and max-norm through an all-reduce.
    Returns (this rank's unscaled solution x + x_in, iterations; negative on breakdown)."""
    inv = block_jacobi_inverse(p)
    x0 = x_own.copy()
    b = _bj_apply(inv, b_own)
    x = b.copy()
    r = b - _bj_apply(inv, matvec(p, x, dist))
    q = r.copy()
    pv = np.zeros_like(r)
    Ap = np.zeros_like(r)
    rnorm, bnorm = _gmax(r, dist), _gmax(b, dist)
    rhop = alpha = omega = 1.0
    rho = dot(r, q, dist)
    it, status = 0, 0
    while rnorm > (tol + bnorm * tol) and it < max_it:
        it += 1
        beta = (rho * alpha) / (rhop * omega)
        pv = (pv - omega * Ap) * beta + r
        Ap = _bj_apply(inv, matvec(p, pv, dist))
        gamma = dot(q, Ap, dist)
        if gamma == 0.0 or not np.isfinite(gamma):
            status = -1
            break
        alpha = rho / gamma
        s = r - alpha * Ap
        As = _bj_apply(inv, matvec(p, s, dist))
        omega = dot(As, s, dist)
        gamma = dot(As, As, dist)
        if gamma == 0.0:
            x = x + alpha * pv
            r = s
            break
        omega = omega / gamma
        rhop = rho
        rho = -1.0 * omega * dot(As, q, dist)
        x = x + alpha * pv + omega * s
        r = s - omega * As
        rnorm = _gmax(r, dist)
        if not np.isfinite(rnorm):
            status = -1
            break
    x = (x + x0) * scale_own
    return x, (-it - 1 if status < 0 else it)


# ---------------------------------------------------------------------------- assembly
@dataclass
class AssemblyPart:
    """What one rank needs to assemble its own rows without exchanging element
    contributions: every triangle within two element rings of its nodes (the
    wet/dry flag of an element next to an owned node depends on the elements around
    that element's nodes), the boundary segments that touch its nodes, and the nodes
    all of them reference.  Elements keep their global order and nodes their global
    order, so each owned row sums the same element contributions in the same order
    as the single-process assembly."""
    rank: int
    lo: int
    hi: int
    tri_ids: np.ndarray     # global triangle ids, increasing
    seg_ids: np.ndarray     # global segment ids, increasing
    nodes: np.ndarray       # global node ids, increasing (local node k = nodes[k])

    def local(self, g: np.ndarray) -> np.ndarray:
        return np.searchsorted(self.nodes, g)

    @property
    def owned_local(self) -> np.ndarray:
        return self.local(np.arange(self.lo, self.hi))


def assembly_parts(tri: np.ndarray, seg: np.ndarray, nnodes: int, npes: int) -> List[AssemblyPart]:
    ptr = node_ranges(nnodes, npes)
    out = []
    for r in range(npes):
        lo, hi = int(ptr[r]), int(ptr[r + 1])
        owned = np.zeros(nnodes, bool)
        owned[lo:hi] = True
        ring1 = owned[tri].any(axis=1)
        n1 = np.zeros(nnodes, bool)
        n1[tri[ring1].ravel()] = True
        n1 |= owned
        ring2 = n1[tri].any(axis=1)
        sg = owned[seg].any(axis=1) if seg.size else np.zeros(0, bool)
        nodes = np.unique(np.concatenate([tri[ring2].ravel(), seg[sg].ravel(), np.arange(lo, hi)]))
        out.append(AssemblyPart(r, lo, hi, np.nonzero(ring2)[0], np.nonzero(sg)[0], nodes))
    return out


def part_case(case, part: AssemblyPart):
    """The rank's sub-mesh as a case in local numbering (same forcing and step)."""
    import dataclasses
    loc = part.local
    tri = loc(case.tri[part.tri_ids]).astype(np.int32)
    seg = loc(case.seg[part.seg_ids]).astype(np.int32).reshape(-1, 2)
    dofs = (3 * part.nodes[:, None] + np.arange(3)).ravel()
    return dataclasses.replace(case, xyz=case.xyz[part.nodes], tri=tri, seg=seg,
                               seg_kind=case.seg_kind[part.seg_ids], sol0=case.sol0[dofs]), dofs


def state_halo(parts: List[AssemblyPart], nnodes: int):
    """For each rank: {peer: global nodes it receives from that peer} and
    {peer: global nodes it sends}, node-wise (three dofs per node)."""
    ptr = node_ranges(nnodes, len(parts))
    recv = [dict() for _ in parts]
    send = [dict() for _ in parts]
    for p in parts:
        ghost = p.nodes[(p.nodes < p.lo) | (p.nodes >= p.hi)]
        owner = np.searchsorted(ptr, ghost, side="right") - 1
        for q in np.unique(owner):
            g = ghost[owner == q]
            recv[p.rank][int(q)] = g
            send[int(q)][p.rank] = g
    return send, recv


def exchange_state(part: AssemblyPart, send: Dict[int, np.ndarray], recv: Dict[int, np.ndarray],
                   state_own: np.ndarray, dist) -> np.ndarray:
    """This rank's state vector in the part's local node order: owned nodes from
    state_own (3 values per owned node), the others from their owners."""
    import torch
    out = np.zeros(3 * part.nodes.size, dtype=state_own.dtype)
    own = part.owned_local
    out.reshape(-1, 3)[own] = state_own.reshape(-1, 3)
    reqs, bufs = [], {}
    for q, g in sorted(send.items()):
        t = torch.from_numpy(np.ascontiguousarray(state_own.reshape(-1, 3)[g - part.lo].ravel()))
        reqs.append(dist.isend(t, dst=q))
        bufs[("s", q)] = t
    for q, g in sorted(recv.items()):
        t = torch.empty(3 * g.size, dtype=torch.float64)
        reqs.append(dist.irecv(t, src=q))
        bufs[("r", q)] = t
    for rq in reqs:
        rq.wait()
    for q, g in recv.items():
        out.reshape(-1, 3)[part.local(g)] = bufs[("r", q)].numpy().reshape(-1, 3)
    return out


# ---------------------------------------------------------------------------- Newton
def _gsum(v: float, dist) -> float:
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64)
    dist.all_reduce(t)
    return float(t.item())


class RankNewton:
    """fe_newton (src/newton/fe_newton.c:44-915) for one rank of a partitioned run:
    residual and Jacobian rows from the rank's halo sub-mesh (``make_model`` builds
    the element evaluator for it: an object with wd_flags / residual / jacobian on
    local states and the sub-mesh CSR row pointers, ``indptr`` or ``sparsity()`` --
    the CPU oracle, or the device model, which offers the same calls), check_diag, Dirichlet
    rows and columns, row and column scaling, block-Jacobi BiCGStab over the split
    CSR, the line search and the stop tests, with the norms and dot products reduced
    over the ranks.  Column operations read the ghost columns' Dirichlet marks and
    scale factors through the same halo as the products."""

    SMALL = float(np.finfo(np.float64).eps)

    def __init__(self, case, indptr, cols, npes, rank, make_model):
        self.case, self.npes, self.rank = case, npes, rank
        parts = assembly_parts(case.tri, case.seg, case.nnodes, npes)
        self.part = parts[rank]
        self.send, self.recv = state_halo(parts, case.nnodes)
        self.send, self.recv = self.send[rank], self.recv[rank]
        sub, _ = part_case(case, self.part)
        self.model = make_model(sub)
        self.sub_indptr = self.model.indptr if hasattr(self.model, "indptr") else self.model.sparsity()[0]
        self.plan = split(indptr, cols, np.zeros(len(cols)), case.nnodes, npes)[rank]
        self.r0, self.r1 = 3 * self.part.lo, 3 * self.part.hi
        rows = slice(int(indptr[self.r0]), int(indptr[self.r1]))
        self.row_cols = np.asarray(cols[rows], np.int64)
        self.row_ptr = np.asarray(indptr[self.r0:self.r1 + 1], np.int64) - int(indptr[self.r0])
        self.diag_mask = (self.row_cols >= self.r0) & (self.row_cols < self.r1)
        self.own_rows = (3 * self.part.owned_local[:, None] + np.arange(3)).ravel()
        row_of = np.repeat(np.arange(self.r1 - self.r0), np.diff(self.row_ptr))
        self.diag_slot = np.nonzero(self.row_cols == row_of + self.r0)[0]
        self.n_global = 3 * case.nnodes

    # -- helpers
    def _local(self, sol_own, dist):
        return exchange_state(self.part, self.send, self.recv, sol_own, dist)

    def _ghost_values(self, v_own, dist):
        return halo_exchange(self.plan, v_own, dist)[self.plan.nrows:]

    def _col_values(self, v_own, v_ghost):
        """v at every matrix entry's column (owned columns from v_own, ghosts from v_ghost)."""
        out = np.empty(self.row_cols.size)
        out[self.diag_mask] = v_own[self.row_cols[self.diag_mask] - self.r0]
        out[~self.diag_mask] = v_ghost[np.searchsorted(self.plan.ghosts, self.row_cols[~self.diag_mask])]
        return out

    def _residual(self, sol_own, old_loc, older_loc, dist):
        r = self.model.residual(self._local(sol_own, dist), old_loc, older_loc)
        return r[self.own_rows]

    def _jacobian(self, sol_own, old_loc, older_loc, dist):
        v = self.model.jacobian(self._local(sol_own, dist), old_loc, older_loc)
        ip = self.sub_indptr
        return np.concatenate([v[ip[r]:ip[r + 1]] for r in self.own_rows])

    def _norms(self, res, dsol, mask, dist):
        inc = mask != 1
        rmax = _gmax(res[inc], dist)
        l2 = _gsum(float(np.sum(res[inc] * res[inc])), dist)
        imax = _gmax(dsol[inc], dist)
        return rmax, np.sqrt(l2) / self.n_global, imax

    def solve(self, sol_old_own, sol_older_own, mask_own, dirichlet_own, dist, tol_nonlin=1e-8, inc_nonlin=1e-6,
              max_nonlin_it=10, max_cuts=5, krylov_max_it=100, krylov_tol=1e-11):
        old_loc = self._local(sol_old_own, dist)
        older_loc = self._local(sol_older_own, dist)
        n = self.r1 - self.r0
        # initialize_system (newton_tools.c:21-37) and fe_sw2_init's dry-node marks
        sol = sol_old_own.copy()
        self.model.wd_flags(self._local(sol, dist), old_loc)
        dry = np.nonzero(sol_old_own[0::3] <= 0.0)[0]
        mask_own[3 * dry + 1] = 1
        mask_own[3 * dry + 2] = 1
        sol[mask_own == 1] = dirichlet_own[mask_own == 1]
        res = self._residual(sol, old_loc, older_loc, dist)
        dsol = np.zeros(n)
        rmax, rl2, imax = self._norms(res, dsol, mask_own, dist)
        it, kry, ok, cuts_total = 0, 0, True, 0
        while True:
            vals = self._jacobian(sol, old_loc, older_loc, dist)
            mask_own[np.abs(vals[self.diag_slot]) < self.SMALL] = 1                 # check_diag
            mask_col = self._col_values(mask_own.astype(np.float64), self._ghost_values(mask_own.astype(np.float64), dist))
            vals[mask_col == 1.0] = 0.0                                                # Dirichlet columns
            for r in np.nonzero(mask_own == 1)[0]:                                     # Dirichlet rows
                k0, k1 = self.row_ptr[r], self.row_ptr[r + 1]
                vals[k0:k1] = (self.row_cols[k0:k1] == r + self.r0).astype(np.float64)
                res[r] = 0.0
            mx = np.array([np.max(np.abs(vals[self.row_ptr[r]:self.row_ptr[r + 1]])) for r in range(n)])
            s = np.where(mx < self.SMALL, 1.0 / np.sqrt(self.SMALL), 1.0 / np.sqrt(np.abs(mx)))
            b = res * s
            s_col = self._col_values(s, self._ghost_values(s, dist))
            row_of = np.repeat(np.arange(n), np.diff(self.row_ptr))
            vals = vals * (s[row_of] * s_col)
            p = self.plan
            p.vals_diag, p.vals_off = vals[self.diag_mask], vals[~self.diag_mask]
            dsol, kit = bicgstab_bj(p, np.zeros(n), b, s, dist, max_it=krylov_max_it, tol=krylov_tol)
            kry += kit if kit >= 0 else -kit - 1
            sol = sol + dsol
            dsol = -dsol
            old_l2 = rl2
            res = self._residual(sol, old_loc, older_loc, dist)
            rmax, rl2, imax = self._norms(res, dsol, mask_own, dist)
            if not np.isfinite(rl2):
                ok = False
            cuts = 0
            while rmax > tol_nonlin and rl2 > old_l2 and cuts < max_cuts:              # line search
                dsol = dsol * 0.5
                sol = sol + dsol
                res = self._residual(sol, old_loc, older_loc, dist)
                rmax, rl2, imax = self._norms(res, dsol, mask_own, dist)
                cuts += 1
            cuts_total += cuts
            it += 1
            if not (ok and it < max_nonlin_it and rmax < 1.0e20 and rmax > tol_nonlin and imax > inc_nonlin):
                break
        success = not (((rmax > tol_nonlin) and (imax > inc_nonlin)) or rmax >= 1.0e20 or not ok)
        if not success:                                                              # fe_newton.c:893-899
            sol = sol_old_own.copy()
            sol[mask_own == 1] = dirichlet_own[mask_own == 1]
        return sol, {"newton_its": it, "krylov_its": kry, "resid_max": rmax, "ok": success,
                     "linesearch_cuts": cuts_total}


class DeviceRankModel:
    """The device model (``capi.SW2Model``, the CUDA element and assembly kernels) as
    RankNewton's element evaluator for one rank's halo sub-mesh.  Like fe_sw2_init
    (src/models/sw2/fe_sw2_init.c), ``wd_flags`` fixes the wet/dry flags at the start of
    a Newton solve and every residual and Jacobian of that solve uses them
    (``sw2g_assemble_residual_wd`` / ``sw2g_assemble_jacobian_wd``)."""

    def __init__(self, sub_case):
        from .capi import SW2Model
        self.case = sub_case
        self.model = SW2Model(sub_case)
        self.indptr = self.model.sparsity()[0]
        self._wd = None
        self.set_bc_window(sub_case.t0, sub_case.t0 + sub_case.dt)

    def set_bc_window(self, t1: float, t2: float) -> None:
        """The step's dt and series averages over [t1, t2] (advance_time's series update)."""
        from .timeloop import series_step_average
        s = self.case.series
        vals = [series_step_average(*s[k], t1, t2) if k in s else 0.0 for k in (0, 1, 2)]
        self.model.set_step(t2 - t1, *vals)
        if 3 in s or 4 in s:
            qs = series_step_average(*s[3], t1, t2) if 3 in s else 0.0
            tw = series_step_average(*s[4], t1, t2) if 4 in s else 0.0
            self.model.set_bc_structures(qs, self.case.bc_conveyance, self.case.bc_rough_height, tw)
        if 5 in s:
            self.model.set_bc_flux(series_step_average(*s[5], t1, t2))

    def wd_flags(self, sol, sol_old):
        self._wd = self.model.wd_flags(sol, sol_old)
        return self._wd.copy()

    def residual(self, sol, sol_old, sol_older):
        return self.model.residual_wd(sol, sol_old, sol_older, self._wd)

    def jacobian(self, sol, sol_old, sol_older):
        return self.model.jacobian_wd(sol, sol_old, sol_older, self._wd)

    def close(self) -> None:
        self.model.close()
