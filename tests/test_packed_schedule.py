"""The persistent tile-task kernel's schedule, replayed on the host (no GPU).

moao_packed_task_list returns the task list in the order the kernel's CTAs
claim it. This test restates the kernel's rules in numpy: every task waits until
the version counters of the tiles it reads and writes reach its step (a(i,j) of
Cmm's tiles, w(r,c) of Ctm's), runs its 64 x 64 tile operation and publishes the
next version. Checked here:
- run in claim order, every task finds its waits already satisfied (each task
  it depends on sits earlier in the list: the kernel's progress argument);
- the replay computes R = Ctm Cmm^-1 and the Cholesky factor, for ragged sizes
  (nmeas and nmeasts not multiples of 64, one-tile systems, nmeasts = 0);
- a simulated concurrent run (P workers claiming in order, random task
  durations, a task starting only when its waits hold) always completes;
- the list holds exactly the tile algorithm's tasks.
The tile operations follow the reference's dpotrf + two dtrsm
(lapack/compute/reconstructor.cpp:48-70) in tile form."""
import heapq

import numpy as np
import pytest

from moao_b200 import batch as B

T = 64
POTRF, TRSM, UPDATE, FUPD, FDIAG, BUPD, BDIAG = range(7)


def spd(n, rng):
    X = rng.standard_normal((n, n + 8))
    return X @ X.T / n + np.eye(n)


class Replay:
    """One instance's tiles and counters, with the kernel's wait rules."""

    def __init__(self, A, Ct):
        self.n, self.m = A.shape[0], Ct.shape[0]
        self.nt, self.mt = -(-self.n // T), -(-self.m // T)
        self.A = np.tril(A).copy()
        self.C = Ct.copy()
        self.Linv = [None] * self.nt
        self.a = np.zeros((self.nt, self.nt), dtype=np.int64)
        self.w = np.zeros((self.mt, self.nt), dtype=np.int64)

    def sa(self, q):
        return slice(q * T, min(self.n, (q + 1) * T))

    def sc(self, q):
        return slice(q * T, min(self.m, (q + 1) * T))

    def waits(self, t):
        """[(counter array, index, value)] and the published (array, index, value)."""
        _, ty, i, j, k = t
        nt = self.nt
        a, w = self.a, self.w
        if ty == POTRF:
            return [(a, (k, k), k)], (a, (k, k), k + 1)
        if ty == TRSM:
            return [(a, (k, k), k + 1), (a, (i, k), k)], (a, (i, k), k + 1)
        if ty == UPDATE:
            return [(a, (i, k), k + 1), (a, (j, k), k + 1), (a, (i, j), k)], (a, (i, j), k + 1)
        if ty == FUPD:
            return [(w, (i, k), k + 1), (a, (j, k), k + 1), (w, (i, j), k)], (w, (i, j), k + 1)
        if ty == FDIAG:
            return [(w, (i, k), k), (a, (k, k), k + 1)], (w, (i, k), k + 1)
        if ty == BUPD:
            return [(w, (i, k), nt + 1), (w, (i, j), j + nt - k)], (w, (i, j), j + 1 + nt - k)
        return [(w, (i, k), nt)], (w, (i, k), nt + 1)

    def ready(self, t):
        return all(arr[ix] >= v for arr, ix, v in self.waits(t)[0])

    def run(self, t):
        _, ty, i, j, k = t
        A, C, sa, sc = self.A, self.C, self.sa, self.sc
        if ty == POTRF:
            L = np.linalg.cholesky(A[sa(k), sa(k)])
            A[sa(k), sa(k)] = L
            self.Linv[k] = np.linalg.inv(L)
        elif ty == TRSM:
            A[sa(i), sa(k)] = A[sa(i), sa(k)] @ self.Linv[k].T
        elif ty == UPDATE:
            U = A[sa(i), sa(k)] @ A[sa(j), sa(k)].T
            A[sa(i), sa(j)] -= np.tril(U) if i == j else U
        elif ty == FUPD:
            C[sc(i), sa(j)] -= C[sc(i), sa(k)] @ A[sa(j), sa(k)].T
        elif ty == FDIAG:
            C[sc(i), sa(k)] = C[sc(i), sa(k)] @ self.Linv[k].T
        elif ty == BUPD:
            C[sc(i), sa(j)] -= C[sc(i), sa(k)] @ A[sa(k), sa(j)]
        else:
            C[sc(i), sa(k)] = C[sc(i), sa(k)] @ self.Linv[k]
        arr, ix, v = self.waits(t)[1]
        arr[ix] = v


SIZES = [[(100, 30)], [(64, 64)], [(40, 0)], [(300, 70), (129, 5), (64, 1), (200, 130)]]


@pytest.mark.parametrize("sizes", SIZES)
def test_claim_order_replay_builds_R(built, sizes):
    rng = np.random.default_rng(len(sizes))
    tasks, levels = B.packed_task_list([n for n, _ in sizes], [m for _, m in sizes])
    assert levels > 0 and len(tasks) > 0
    inst, want = [], []
    for n, m in sizes:
        A = spd(n, rng)
        Ct = rng.standard_normal((m, n))
        inst.append(Replay(A, Ct))
        want.append((np.linalg.cholesky(A), np.linalg.solve(A, Ct.T).T))
    for t in tasks:
        r = inst[t[0]]
        assert r.ready(t), ("a task's input is produced later in the list", t)
        r.run(t)
    for r, (L, R) in zip(inst, want):
        assert np.allclose(np.tril(r.A), L, rtol=0, atol=1e-10 * np.abs(L).max())
        if r.m:
            assert np.abs(r.C - R).max() <= 1e-9 * max(np.abs(R).max(), 1.0)


def test_task_counts_are_the_tile_algorithm(built):
    n, m = 300, 70  # nt = 5, mt = 2
    tasks, _ = B.packed_task_list([n], [m])
    nt, mt = 5, 2
    counts = np.bincount(tasks[:, 1], minlength=7)
    assert counts[POTRF] == nt and counts[TRSM] == nt * (nt - 1) // 2
    assert counts[UPDATE] == sum((nt - k - 1) * (nt - k) // 2 for k in range(nt))
    assert counts[FUPD] == counts[BUPD] == mt * nt * (nt - 1) // 2
    assert counts[FDIAG] == counts[BDIAG] == mt * nt
    assert len({tuple(t) for t in tasks}) == len(tasks)


@pytest.mark.parametrize("workers,seed", [(3, 1), (16, 2), (300, 3)])
def test_concurrent_claims_always_complete(built, workers, seed):
    """P workers (CTAs) claim tasks in list order; a claimed task starts once its
    waits hold and takes a random time; as in the kernel, a worker claims its next
    task as soon as its current one starts (one task queued behind the running
    one). The event simulation must finish every task."""
    rng = np.random.default_rng(seed)
    sizes = [(200, 70), (129, 64), (333, 10)]
    tasks, _ = B.packed_task_list([n for n, _ in sizes], [m for _, m in sizes])
    tasks = [tuple(int(x) for x in t) for t in tasks]
    inst = [Replay(spd(n, rng), rng.standard_normal((m, n))) for n, m in sizes]
    nxt, done, now = 0, 0, 0.0
    cur = [None] * workers      # claimed task waiting for its inputs, or None
    busy = [False] * workers    # running (its task is in the heap)
    queued = [None] * workers   # claimed behind the running task
    running = []                # heap of (finish time, seq, worker, task)
    seq = 0

    def claim():
        nonlocal nxt
        if nxt < len(tasks):
            nxt += 1
            return tasks[nxt - 1]
        return None

    for w in range(workers):
        cur[w] = claim()
    while done < len(tasks):
        started = True
        while started:
            started = False
            for w in range(workers):
                t = cur[w]
                if t is not None and not busy[w] and inst[t[0]].ready(t):
                    busy[w] = True
                    heapq.heappush(running, (now + rng.exponential(1.0), seq, w, t))
                    seq += 1
                    queued[w] = claim()  # claim-ahead once the current task runs
                    started = True
        assert running, "no claimed task can start: the schedule would deadlock"
        now, _, w, t = heapq.heappop(running)
        inst[t[0]].run(t)
        done += 1
        busy[w] = False
        cur[w], queued[w] = queued[w], None
    assert nxt == len(tasks) and all(c is None for c in cur)
