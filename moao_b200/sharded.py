"""One reconstructor build spread over several GPUs (one rank per GPU).

For a system whose Cmm does not fit one device (the FP64 Cmm is 80 GB at
nmeas 100k), the matrix is held in column panels of width nb distributed
cyclically over the ranks (panel j on rank j mod P, all of its rows on or below
the diagonal), and the factorisation and both triangular solves run as
right-looking panel steps with one broadcast per step:

  factor + forward solve, k = 0 .. nt-1: the owner of panel k factors its
    diagonal block (L_kk and L_kk^-1), turns the rest of the panel into
    L_ik = A_ik L_kk^-T and its Ctm columns into X_k = B_k L_kk^-T, and
    broadcasts [status, L_(k+1:, k), X_k]; every rank then updates its own
    later panels, A_ij -= L_ik L_jk^T (i >= j), and their Ctm columns,
    B_j -= X_k L_jk^T;
  backward solve, c = nt-1 .. 0: the owner of panel c finishes
    R_c = B_c L_cc^-1 and broadcasts it; every rank updates its earlier
    columns, B_j -= R_c L_cj (L_cj is in the rank's own panel j).

Each rank generates its own panels of Cmm and columns of Ctm with the
covariance kernels (no communication), stores about 1/P of the lower part, and
ends with R's columns of its panels (gathered on request). The broadcasts move
n^2 / 2 + nmeasts n doubles in all. Every rank takes the same collective steps
in the same order, a factorisation failure included (its status travels with
the panel).

The reference's distributed path is ScaLAPACK (scalapack/moao_scalapack.c:
pdpotrf and two pdtrsm on a 2-D block-cyclic distribution); the result is
R = Ctm Cmm^-1 like lapack/compute/reconstructor.cpp:32-58.

Matrices are column-major: a local array of `ncols` columns and `nrows` rows is
a torch tensor of shape (ncols, nrows). Operands are (tensor, col, row) views
with the tensor's row stride as leading dimension.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

from ._lib import check, lib
from .api import Context, Tomo, default_context


@dataclass
class Layout:
    n: int      # nmeas
    m: int      # nmeasts
    nb: int     # panel width
    P: int      # ranks
    rank: int

    @property
    def nt(self) -> int:
        return (self.n + self.nb - 1) // self.nb

    def width(self, j: int) -> int:
        return min(self.nb, self.n - j * self.nb)

    def owner(self, j: int) -> int:
        return j % self.P

    @property
    def owned(self) -> list:
        return [j for j in range(self.nt) if j % self.P == self.rank]

    def local_col(self, j: int) -> int:
        """First local column of owned panel j."""
        c = 0
        for q in self.owned:
            if q == j:
                return c
            c += self.width(q)
        raise ValueError(f"panel {j} is not on rank {self.rank}")

    @property
    def local_cols(self) -> int:
        return sum(self.width(j) for j in self.owned)


class DeviceOps:
    """The operations of the sharded build on CUDA tensors, through the C ABI
    (moao_matcov_tile, moao_dense_potrf_inv, moao_dense_gemm), on the
    context's stream (which the caller sets to torch's current stream)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    @staticmethod
    def _ptr(v):
        t, col, row = v
        return C.c_void_p(t.data_ptr() + 8 * (col * t.stride(0) + row))

    def potrf_inv(self, v, n, Linv) -> int:
        info = C.c_int()
        st = lib().moao_dense_potrf_inv(self.ctx.handle, n, self._ptr(v), v[0].stride(0),
                                        self._ptr((Linv, 0, 0)), Linv.stride(0), C.byref(info))
        if st == 2:  # not SPD: reported through the broadcast status
            return info.value
        check(st, "moao_dense_potrf_inv")
        return 0

    def gemm(self, transB, lowerC, M, N, K, alpha, a, b, beta, c):
        check(lib().moao_dense_gemm(self.ctx.handle, int(transB), int(lowerC), M, N, K, alpha,
                                    self._ptr(a), a[0].stride(0), self._ptr(b), b[0].stride(0),
                                    beta, self._ptr(c), c[0].stride(0)), "moao_dense_gemm")

    def matcov(self, tomo: Tomo, v, nrows, ncols, xoff, yoff, type_mat):
        check(lib().moao_matcov_tile(self.ctx.handle, tomo.handle,
                                     C.cast(self._ptr(v), C.POINTER(C.c_double)), nrows, ncols,
                                     xoff, yoff, v[0].stride(0), type_mat), "moao_matcov_tile")


def generate(lay: Layout, A, B, ops, tomo) -> None:
    """This rank's panels of Cmm (rows from the panel's diagonal down) into A
    and its columns of Ctm into B, from the covariance model."""
    for j in lay.owned:
        j0, jb, lc = j * lay.nb, lay.width(j), lay.local_col(j)
        ops.matcov(tomo, (A, lc, j0), lay.n - j0, jb, j0, j0, 1)
        if lay.m:
            ops.matcov(tomo, (B, lc, 0), lay.m, jb, 0, j0, 3)


def factor_and_solve(lay: Layout, A, B, ops, dist=None, group=None) -> int:
    """Factors the distributed Cmm in A and turns the distributed Ctm columns in
    B into R's (in place). Returns 0, or the 1-based global column of the first
    non-positive pivot (then every rank stops after that step).

    With several ranks the factorisation looks one panel ahead: at step k the
    owner of panel k + 1 first applies panel k to that panel alone, factors it
    and starts its broadcast (asynchronously), and only then applies panel k
    to the rest of its panels, so that panel k + 1 travels while every rank
    updates. The collectives are the same broadcasts in the same order on every
    rank."""
    import torch
    n, m, nb, P, rank = lay.n, lay.m, lay.nb, lay.P, lay.rank
    dev, f64 = A.device, torch.float64
    owned = lay.owned
    linv = {}

    def bcast(buf, src):
        if P > 1:
            dist.broadcast(buf, src=src, group=group)

    def buffer(k):
        k0, kb = k * nb, lay.width(k)
        rest = n - k0 - kb
        return torch.empty(1 + (kb * rest + kb * m if P > 1 else 0), dtype=f64, device=dev)

    def factor_panel(k):
        """On the owner of panel k: L_kk and its inverse, the panel's rows
        below the diagonal block L_ik = A_ik L_kk^-T and X_k = B_k L_kk^-T;
        returns the broadcast buffer [status, L(k0+kb : n, k), X_k]."""
        k0, kb = k * nb, lay.width(k)
        rest = n - k0 - kb
        buf = buffer(k)
        lc = lay.local_col(k)
        Lk = torch.zeros((kb, kb), dtype=f64, device=dev)
        info = ops.potrf_inv((A, lc, k0), kb, Lk)
        linv[k] = Lk
        if info == 0:
            if rest:
                W = torch.empty((kb, rest), dtype=f64, device=dev)
                ops.gemm(True, False, rest, kb, kb, 1.0, (A, lc, k0 + kb), (Lk, 0, 0), 0.0,
                         (W, 0, 0))
                A[lc:lc + kb, k0 + kb:n] = W
            if m:
                W = torch.empty((kb, m), dtype=f64, device=dev)
                ops.gemm(True, False, m, kb, kb, 1.0, (B, lc, 0), (Lk, 0, 0), 0.0, (W, 0, 0))
                B[lc:lc + kb, :] = W
        buf[0] = float(info + k0 if info else 0)
        if P > 1:
            if rest:
                buf[1:1 + kb * rest].view(kb, rest).copy_(A[lc:lc + kb, k0 + kb:n])
            if m:
                buf[1 + kb * rest:].view(kb, m).copy_(B[lc:lc + kb, :])
        return buf

    def update(k, panels, buf):
        """Apply panel k (its broadcast buffer) to this rank's panels `panels`
        (consecutive in local storage, all after k)."""
        if not panels:
            return
        k0, kb = k * nb, lay.width(k)
        rest = n - k0 - kb
        Lp = buf[1:1 + kb * rest].view(kb, rest)   # L(k0+kb : n, panel k), ld rest
        Xk = buf[1 + kb * rest:].view(kb, m)       # X_k, ld m
        for j in panels:  # A(j0:n, panel j) -= L(j0:n, k) L(j0:j0+jb, k)^T, lower on its diagonal block
            j0, jb = j * nb, lay.width(j)
            r = j0 - (k0 + kb)
            ops.gemm(True, True, n - j0, jb, kb, -1.0, (Lp, 0, r), (Lp, 0, r), 1.0,
                     (A, lay.local_col(j), j0))
        if m:  # B(:, panels) -= X_k L(rows of the panels, k)^T in one product
            rows = torch.cat([torch.arange(j * nb - (k0 + kb), j * nb - (k0 + kb) + lay.width(j),
                                           device=dev) for j in panels])
            G = Lp[:, rows].contiguous()
            ops.gemm(True, False, m, int(rows.numel()), kb, -1.0, (Xk, 0, 0), (G, 0, 0), 1.0,
                     (B, lay.local_col(panels[0]), 0))

    if P == 1:
        for k in range(lay.nt):
            k0, kb = k * nb, lay.width(k)
            rest = n - k0 - kb
            info = int(factor_panel(k)[0].item())
            if info:
                return info
            later = [j for j in owned if j > k]
            if not later:
                continue
            # the later panels are the whole trailing matrix: one lower SYRK, L(k0+kb : n,
            # panel k) and X_k read in place
            lc = lay.local_col(k)
            Lv, Xv = (A, lc, k0 + kb), (B, lc, 0)
            ops.gemm(True, True, rest, rest, kb, -1.0, Lv, Lv, 1.0,
                     (A, lay.local_col(later[0]), k0 + kb))
            if m:
                ops.gemm(True, False, m, rest, kb, -1.0, Xv, Lv, 1.0,
                         (B, lay.local_col(later[0]), 0))
    else:
        def post(k, buf):
            return dist.broadcast(buf, src=lay.owner(k), group=group, async_op=True)

        buf = factor_panel(0) if rank == lay.owner(0) else buffer(0)
        work = post(0, buf)
        for k in range(lay.nt):
            work.wait()
            info = int(buf[0].item())
            if info:
                return info  # nothing posted beyond panel k: every rank stops here
            later = [j for j in owned if j > k]
            nxt = None
            if k + 1 < lay.nt:
                if rank == lay.owner(k + 1):
                    update(k, later[:1], buf)        # panel k + 1 is this rank's first later panel
                    later = later[1:]
                    nxt = factor_panel(k + 1)
                else:
                    nxt = buffer(k + 1)
                work = post(k + 1, nxt)
            update(k, later, buf)
            if nxt is not None:
                buf = nxt
    # backward solve, c = nt-1 .. 0: R_c = B_c L_cc^-1 on the owner of panel c, then
    # B(:, earlier panels) -= R_c L(c0 : c0+cb, earlier panels) on every rank
    if not m:
        return 0

    def finish(c, buf=None):
        """On the owner of panel c: R_c into B's columns (and into buf)."""
        cb, lc = lay.width(c), lay.local_col(c)
        W = torch.empty((cb, m), dtype=f64, device=dev)
        ops.gemm(False, False, m, cb, cb, 1.0, (B, lc, 0), (linv[c], 0, 0), 0.0, (W, 0, 0))
        B[lc:lc + cb, :] = W
        if buf is not None:
            buf.view(cb, m).copy_(W)
        return buf

    def back_update(c, Rc, col, ncols):
        """B(:, local columns col .. col+ncols) -= R_c L(c0 : c0+cb, those columns)."""
        if ncols:
            ops.gemm(False, False, m, ncols, lay.width(c), -1.0, (Rc, 0, 0), (A, col, c * nb),
                     1.0, (B, col, 0))

    def rbuf(c):
        return torch.empty(lay.width(c) * m, dtype=f64, device=dev)

    if P == 1:
        for c in reversed(range(lay.nt)):
            Rc = finish(c, rbuf(c)).view(lay.width(c), m)
            back_update(c, Rc, 0, lay.local_col(c))  # the earlier panels precede panel c
        return 0
    # several ranks: one panel ahead, as in the factorisation (the owner of panel
    # c - 1 updates that panel's columns with R_c, finishes R_(c-1) and posts it
    # before updating the rest of its earlier columns)
    def post(c, buf):
        return dist.broadcast(buf, src=lay.owner(c), group=group, async_op=True)

    c = lay.nt - 1
    buf = finish(c, rbuf(c)) if rank == lay.owner(c) else rbuf(c)
    work = post(c, buf)
    for c in reversed(range(lay.nt)):
        work.wait()
        Rc = buf.view(lay.width(c), m)
        earlier = [j for j in owned if j < c]
        nxt = None
        if c > 0:
            if rank == lay.owner(c - 1):
                lc1 = lay.local_col(c - 1)  # this rank's last earlier panel
                back_update(c, Rc, lc1, lay.width(c - 1))
                earlier = earlier[:-1]
                nxt = finish(c - 1, rbuf(c - 1))
            else:
                nxt = rbuf(c - 1)
            work = post(c - 1, nxt)
        back_update(c, Rc, 0, sum(lay.width(j) for j in earlier))
        if nxt is not None:
            buf = nxt
    return 0


def gather_R(lay: Layout, B, dist=None, group=None, root: int = 0):
    """R (nmeasts x nmeas, column-major: a tensor of shape (nmeas, nmeasts)) on
    rank `root`, None elsewhere; one broadcast per panel."""
    import torch
    R = torch.empty((lay.n, lay.m), dtype=torch.float64, device=B.device) if lay.rank == root else None
    for j in range(lay.nt):
        j0, jb, o = j * lay.nb, lay.width(j), lay.owner(j)
        if lay.P == 1:
            R[j0:j0 + jb] = B[lay.local_col(j):lay.local_col(j) + jb]
            continue
        buf = (B[lay.local_col(j):lay.local_col(j) + jb].contiguous() if lay.rank == o else
               torch.empty((jb, lay.m), dtype=torch.float64, device=B.device))
        dist.broadcast(buf, src=o, group=group)
        if lay.rank == root:
            R[j0:j0 + jb] = buf
    return R


def sharded_reconstructor(tomo: Tomo, nb: int = 1024, ctx: Optional[Context] = None,
                          dist=None, group=None, gather: bool = True):
    """Builds R for `tomo` with Cmm spread over the ranks of `group` (torch.distributed
    over NCCL, one rank per GPU; without `dist`, one rank). Returns (R on rank 0 or
    None, this rank's Layout, its local R columns)."""
    import torch
    ctx = ctx or default_context()
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    P = dist.get_world_size(group) if dist else 1
    rank = dist.get_rank(group) if dist else 0
    lay = Layout(tomo.getNMeas(), tomo.getNMeasTS(), nb, P, rank)
    A = torch.empty((lay.local_cols, lay.n), dtype=torch.float64, device="cuda")
    B = torch.empty((lay.local_cols, lay.m), dtype=torch.float64, device="cuda")
    ops = DeviceOps(ctx)
    generate(lay, A, B, ops, tomo)
    info = factor_and_solve(lay, A, B, ops, dist, group)
    if info:
        from ._lib import NotSPDError
        raise NotSPDError(2, "sharded_reconstructor", f"non-positive pivot at column {info}",
                          column=info)
    del A
    R = gather_R(lay, B, dist, group) if gather else None
    return R, lay, B
