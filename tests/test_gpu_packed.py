"""Batched instances packed into the persistent tile-task kernel (packed.cu):
R of every packed instance against the direct FP64 API (a different blocking
of the same factorisation: agreement to max(1e-10, 50 kappa eps) relative, the
FP64 parity bound), packed and graph instances in one batch, a Cholesky failure
of one packed instance leaving the others intact, and a bounded wait that runs
out (wait limit of one poll) reporting MOAO_ERR_TIMEOUT with the context usable
afterwards."""
import numpy as np
import pytest

import moao_b200 as M
from moao_b200 import batch as B

from test_gpu_batch import direct, instances

pytestmark = pytest.mark.gpu


def cond_cmm(ctx, t):
    import torch
    nm = t.getNMeas()
    C = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
    M.matcov_tile(C, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
    A = C.cpu().numpy()
    A = np.tril(A) + np.tril(A, -1).T
    w = np.linalg.eigvalsh(A)
    return w[-1] / w[0]


def check_against_direct(ctx, tomos, outs, per):
    import torch
    for t, o, p in zip(tomos, outs, per):
        assert p["status"] == 0, p
        want = direct(ctx, t, "fp64", 256)
        err = (torch.max(torch.abs(o - want)) / torch.max(torch.abs(want))).item()
        bound = max(1e-10, 50 * cond_cmm(ctx, t) * np.finfo(float).eps)
        assert err <= bound, (p, err, bound)


def test_packed_equals_direct(tmp_path, built, cuda):
    import torch
    ctx = M.Context(0)
    tomos = instances(tmp_path, 8, 11, nssp_range=(6, 16))
    outs = [torch.zeros(t.getNMeas() * t.getNMeasTS(), dtype=torch.float64, device="cuda")
            for t in tomos]
    per, run = B.batch_reconstructors(tomos, outs, prec="fp64", packed_max=100000, ctx=ctx)
    assert run["packed_count"] == len(tomos) and run["streams_used"] == 0 and run["failed"] == 0
    assert all(p["packed"] for p in per) and run["packed_tasks"] > 0
    check_against_direct(ctx, tomos, outs, per)
    ctx.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_packed_beside_graph_instances(tmp_path, built, cuda, prec):
    """The smaller half packed, the rest on the graph's streams, one launch."""
    import torch
    ctx = M.Context(0)
    tomos = instances(tmp_path, 8, 12, nssp_range=(6, 20))
    ns = sorted(t.getNMeas() for t in tomos)
    bound = ns[len(ns) // 2 - 1]
    outs = [torch.zeros(t.getNMeas() * t.getNMeasTS(), dtype=torch.float64, device="cuda")
            for t in tomos]
    per, run = B.batch_reconstructors(tomos, outs, prec=prec, streams=2, packed_max=bound, ctx=ctx)
    assert run["failed"] == 0 and run["packed_count"] == sum(n <= bound for n in ns)
    for t, o, p in zip(tomos, outs, per):
        assert p["packed"] == (t.getNMeas() <= bound), p
        if p["packed"]:
            check_against_direct(ctx, [t], [o], [p])
        else:
            want = direct(ctx, t, prec, p["nb"])
            err = (torch.max(torch.abs(o - want)) / torch.max(torch.abs(want))).item()
            assert err <= 1e-12, (p, err)
    ctx.close()


def test_packed_reports_not_spd(tmp_path, built, cuda):
    ctx = M.Context(0)
    tomos = instances(tmp_path, 3, 9)
    tomos[1].set_profile(np.array([-50.0]), np.zeros(1), np.full(1, 25.0))
    per, run = B.batch_reconstructors(tomos, None, prec="fp64", packed_max=100000, ctx=ctx)
    assert per[0]["status"] == 0 and per[2]["status"] == 0, per
    assert per[1]["status_name"] == "MOAO_ERR_NOT_SPD" and per[1]["info"] > 0, per
    assert run["failed"] == 1
    ctx.close()


def test_packed_wait_limit_runs_out_then_recovers(tmp_path, built, cuda):
    """One poll per dependency wait: tasks claimed while their inputs are still
    being computed give up at once, the kernel stops and the batch reports
    MOAO_ERR_TIMEOUT for its packed instances; the same context then builds them
    correctly with the default limit."""
    import torch
    ctx = M.Context(0)
    tomos = instances(tmp_path, 4, 13, nssp_range=(14, 20))
    ctx.set_wait_limit(1)
    per, run = B.batch_reconstructors(tomos, None, prec="fp64", packed_max=100000, ctx=ctx)
    assert all(p["status_name"] == "MOAO_ERR_TIMEOUT" for p in per), per
    ctx.set_wait_limit(0)
    outs = [torch.zeros(t.getNMeas() * t.getNMeasTS(), dtype=torch.float64, device="cuda")
            for t in tomos]
    per, run = B.batch_reconstructors(tomos, outs, prec="fp64", packed_max=100000, ctx=ctx)
    check_against_direct(ctx, tomos, outs, per)
    ctx.close()
