"""The FP64 tile configurations of the large products (moao_ctx_set_gemm_tile)
change the K depth per pipeline stage and the cp.async ring only: every
accumulator still sums its k16 slices in order, so the FP64 reconstructor's R
is bitwise the same under each of them. Invalid configurations are refused."""
import os

import numpy as np
import pytest

import moao_b200 as M
from moao_b200 import params as P

pytestmark = pytest.mark.gpu


def test_gemm_tile_configs_give_identical_R(tmp_path, built, cuda):
    import torch
    s, a = P.config_scaled(24, 6)
    P.write_system(str(tmp_path), s, a)
    t = M.Tomo(os.path.join(tmp_path, "sys-params.txt"), os.path.join(tmp_path, "prof-1-atmos-night0.txt"))
    nm, nts = t.getNMeas(), t.getNMeasTS()
    ctx = M.Context(0)
    ctx.set_block(512)
    out = []
    for cfg in range(4):
        ctx.set_gemm_tile(cfg)
        C = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
        T = torch.empty((nm, nts), dtype=torch.float64, device="cuda")
        M.matcov_tile(C, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
        M.matcov_tile(T, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
        M.reconstructor(nm, nts, C, nm, T, nts, 1, prec="fp64", ctx=ctx)
        out.append(T.cpu().numpy())
    for cfg in range(1, 4):
        assert np.array_equal(out[0], out[cfg]), cfg
    with pytest.raises(M.MoaoError):
        ctx.set_gemm_tile(4)
    ctx.close()
