"""The sharded build (moao_b200/sharded.py) on CPU ranks over gloo: the panel
distribution, the broadcast schedule and the per-rank updates, with the tile
operations done in numpy (the GPU runs the same schedule with the library's
kernels, tests/test_gpu_sharded.py). R gathered on rank 0 equals numpy's
Ctm Cmm^-1 for 1, 2 and 3 ranks, ragged panel widths included (with several
ranks the factorisation looks one panel ahead: the next panel's broadcast is
posted before the rest of the update); the Cmm panels come from the oracle's
covariance model on a check system; an indefinite Cmm (its failed pivot found
in a look-ahead step) stops every rank at the same step with the same column."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from moao_b200 import sharded as S


class NumpyOps:
    """The sharded build's tile operations on CPU tensors, in numpy."""

    @staticmethod
    def view(v, nrows, ncols):
        t, col, row = v
        return t.numpy()[col:col + ncols, row:row + nrows].T  # column-major block, writable

    def potrf_inv(self, v, n, Linv):
        Ablk = self.view(v, n, n)
        try:
            L = np.linalg.cholesky(np.tril(Ablk) + np.tril(Ablk, -1).T)
        except np.linalg.LinAlgError:
            d = np.diag(Ablk)
            return int(np.argmax(d <= 0)) + 1 if np.any(d <= 0) else 1
        lo = np.tril_indices(n)
        Ablk[lo] = L[lo]
        Linv.numpy()[:, :] = np.linalg.inv(L).T
        return 0

    def gemm(self, transB, lowerC, M, N, K, alpha, a, b, beta, c):
        A = self.view(a, M, K)
        B = self.view(b, N, K) if transB else self.view(b, K, N)
        Cb = self.view(c, M, N)
        P = alpha * (A @ (B.T if transB else B))
        if beta != 0.0:  # like the library: C is not read when beta is 0
            P = P + beta * Cb
        if lowerC:
            mask = np.tril(np.ones((M, N), dtype=bool))
            Cb[mask] = P[mask]
        else:
            Cb[:, :] = P

    def __init__(self, Cmm, Ctm):
        self.Cmm, self.Ctm = Cmm, Ctm

    def matcov(self, tomo, v, nrows, ncols, xoff, yoff, type_mat):
        src = self.Cmm if type_mat == 1 else self.Ctm
        blk = src[xoff:xoff + nrows, yoff:yoff + ncols]
        out = self.view(v, nrows, ncols)
        if type_mat == 1:
            gi = np.arange(nrows)[:, None] + xoff
            gj = np.arange(ncols)[None, :] + yoff
            out[gi >= gj] = blk[gi >= gj]
        else:
            out[:, :] = blk


def _problem(kind, n, m, seed):
    rng = np.random.default_rng(seed)
    if kind == "random":
        X = rng.standard_normal((n, n + 5))
        Cmm = X @ X.T / n + np.eye(n)
        Ctm = rng.standard_normal((m, n))
    elif kind == "indefinite":
        Cmm = np.eye(n)
        Cmm[n - 3, n - 3] = -1.0
        Ctm = rng.standard_normal((m, n))
    elif kind == "indefinite_mid":  # the failed pivot in panel 2 of 64-wide panels
        Cmm = np.eye(n)
        Cmm[150, 150] = -1.0
        Ctm = rng.standard_normal((m, n))
    else:  # the oracle's covariance model on a check system
        import oracle as O
        import systems
        import moao_b200 as M
        sf, af = systems.files(kind)
        g = O.Geometry.from_tomo(M.Tomo(sf, af))
        n, m = g.nmeas, g.nmeasts
        Cmm = O.matcov(g, n, n, 0, 0, 1, nthreads=4)
        Cmm = np.tril(Cmm) + np.tril(Cmm, -1).T
        Ctm = O.matcov(g, m, n, 0, 0, 3, nthreads=4)
    return Cmm, Ctm


def _run(rank, world, port, kind, n, m, nb, q):
    import datetime
    import torch
    import torch.distributed as dist
    torch.set_num_threads(1)
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
    Cmm, Ctm = _problem(kind, n, m, 5)
    n, m = Cmm.shape[0], Ctm.shape[0]
    lay = S.Layout(n, m, nb, world, rank)
    ops = NumpyOps(Cmm, Ctm)
    A = torch.zeros((lay.local_cols, n), dtype=torch.float64)
    B = torch.zeros((lay.local_cols, m), dtype=torch.float64)
    S.generate(lay, A, B, ops, None)
    d = dist if world > 1 else None
    info = S.factor_and_solve(lay, A, B, ops, d)
    R = S.gather_R(lay, B, d) if info == 0 else None
    out = {"rank": rank, "info": info, "owned": lay.owned,
           "R": None if R is None else R.numpy().T.copy()}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    q.put(out)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _launch(world, kind, n, m, nb):
    if world == 1:
        import queue
        q = queue.Queue()
        _run(0, 1, 0, kind, n, m, nb, q)
        return [q.get()]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_run, args=(r, world, port, kind, n, m, nb, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


@pytest.mark.parametrize("world,n,m,nb", [(1, 300, 40, 64), (2, 300, 40, 64), (3, 517, 61, 64),
                                          (2, 200, 0, 64), (3, 130, 17, 128), (4, 700, 30, 64)])
def test_sharded_schedule_builds_R(world, n, m, nb):
    res = _launch(world, "random", n, m, nb)
    Cmm, Ctm = _problem("random", n, m, 5)
    assert all(r["info"] == 0 for r in res)
    owned = sorted(sum((r["owned"] for r in res), []))
    assert owned == list(range((n + nb - 1) // nb))
    if m:
        R_ref = np.linalg.solve(Cmm, Ctm.T).T
        err = np.linalg.norm(res[0]["R"] - R_ref) / np.linalg.norm(R_ref)
        assert err < 1e-11, err


def test_sharded_schedule_on_a_check_system():
    res = _launch(2, "check2", 0, 0, 128)
    Cmm, Ctm = _problem("check2", 0, 0, 5)
    R_ref = np.linalg.solve(Cmm, Ctm.T).T
    kappa = np.linalg.cond(Cmm)
    err = np.linalg.norm(res[0]["R"] - R_ref) / np.linalg.norm(R_ref)
    assert err <= max(1e-10, 50 * kappa * np.finfo(float).eps), (err, kappa)


def test_sharded_failure_stops_every_rank_at_the_same_column():
    res = _launch(2, "indefinite", 300, 20, 64)
    assert [r["info"] for r in res] == [298, 298]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_failure_in_a_lookahead_step(world):
    """A non-positive pivot in panel 2 is found by panel 2's owner while it looks
    ahead during step 1; every rank reads it from that panel's broadcast at
    step 2 and stops with the same column."""
    res = _launch(world, "indefinite_mid", 300, 20, 64)
    assert [r["info"] for r in res] == [151] * world

