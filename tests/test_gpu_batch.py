"""Batched builds in one CUDA graph launch: every instance's R equals the direct
API's with the same panel width (relative max error <= 1e-12; same kernels, same
order), for uneven instances on several streams, FP64 and mixed; the autotuner
fills its table and the table survives a save / load."""
import os

import numpy as np
import pytest

import moao_b200 as M
from moao_b200 import batch as B
from moao_b200 import params as P

pytestmark = pytest.mark.gpu


def instances(tmp_path, count, seed, nssp_range=(8, 20)):
    rng = np.random.default_rng(seed)
    tomos = []
    for i in range(count):
        s, a = P.config_random(rng, nssp_range=nssp_range, nwfs_range=(2, 5), nlayer_range=(1, 8))
        d = str(tmp_path / f"inst{i}")
        P.write_system(d, s, a)
        tomos.append(M.Tomo(os.path.join(d, "sys-params.txt"), os.path.join(d, "prof-1-atmos-night0.txt")))
    return tomos


def direct(ctx, t, prec, nb):
    import torch
    nm, nts = t.getNMeas(), t.getNMeasTS()
    ctx.set_block(nb)
    if prec == "mixed":
        ctx.set_mixed(final_residual=False)
        ctx.set_offsets_from_tomo(t)
    C = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
    T = torch.empty((nm, nts), dtype=torch.float64, device="cuda")
    M.matcov_tile(C, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
    M.matcov_tile(T, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
    M.reconstructor(nm, nts, C, nm, T, nts, 1, prec=prec, ctx=ctx)
    ctx.set_block(256)
    ctx.set_offsets([], [], [])
    return T.reshape(-1)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_equals_direct(tmp_path, built, cuda, prec):
    import torch
    ctx = M.Context(0)
    tomos = instances(tmp_path, 10, 7)
    outs = [torch.zeros(t.getNMeas() * t.getNMeasTS(), dtype=torch.float64, device="cuda")
            for t in tomos]
    per, run = B.batch_reconstructors(tomos, outs, prec=prec, streams=3, ctx=ctx)
    assert run["failed"] == 0 and run["streams_used"] == 3 and run["graph_nodes"] > len(tomos)
    assert {p["stream"] for p in per} == {0, 1, 2}
    for t, o, p in zip(tomos, outs, per):
        assert p["status"] == 0, p
        want = direct(ctx, t, prec, p["nb"])
        err = (torch.max(torch.abs(o - want)) / torch.max(torch.abs(want))).item()
        assert err <= 1e-12, (prec, p, err)
    ctx.close()


def test_batch_reports_not_spd(tmp_path, built, cuda):
    """An instance whose Cmm is indefinite (a negative turbulence strength) reports
    its Cholesky failure after the graph ran; the others in the same graph are
    unaffected."""
    ctx = M.Context(0)
    tomos = instances(tmp_path, 3, 9)
    tomos[1].set_profile(np.array([-50.0]), np.zeros(1), np.full(1, 25.0))
    for prec in ("fp64", "mixed"):
        per, run = B.batch_reconstructors(tomos, None, prec=prec, streams=2, ctx=ctx)
        assert per[0]["status"] == 0 and per[2]["status"] == 0, per
        assert per[1]["status_name"] == "MOAO_ERR_NOT_SPD" and per[1]["info"] > 0, per
        assert run["failed"] == 1
    ctx.close()


def test_autotune_and_table_round_trip(tmp_path, built, cuda):
    ctx = M.Context(0)
    tomos = instances(tmp_path, 3, 3, nssp_range=(10, 16))
    tab = B.autotune(tomos, "fp64", candidates=[64, 128, 256], ctx=ctx)
    assert tab["streams"] in (2, 4, 8)
    assert all(v % 64 == 0 for v in tab["nb"].values())
    p = str(tmp_path / "tune.txt")
    B.tuning_save(p, ctx=ctx)
    ctx2 = M.Context(0)
    B.tuning_load(p, ctx=ctx2)
    assert B.tuning("fp64", ctx=ctx2) == tab
    with open(p, "a") as f:
        f.write("nb 0 0 100\n")
    with pytest.raises(M.MoaoError):
        B.tuning_load(p, ctx=ctx2)
    ctx.close()
    ctx2.close()
