"""The sharded build on the GPU with one rank (the schedule of
tests/test_sharded_gloo.py with the library's kernels: covariance panels,
dense_potrf_inv, dense_gemm): R equals the single-GPU FP64 reconstructor's with
the same panel width to 1e-12 relative, and the dense building blocks check
their arguments."""
import os

import numpy as np
import pytest

import moao_b200 as M
from moao_b200 import params as P
from moao_b200 import sharded as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nssp,nb", [(16, 256), (20, 512)])
def test_sharded_one_rank_equals_fp64_path(tmp_path, built, cuda, nssp, nb):
    import torch
    s, a = P.config_scaled(nssp, 4)
    P.write_system(str(tmp_path), s, a)
    t = M.Tomo(os.path.join(tmp_path, "sys-params.txt"), os.path.join(tmp_path, "prof-1-atmos-night0.txt"))
    nm, nts = t.getNMeas(), t.getNMeasTS()
    ctx = M.Context(0)
    R, lay, _ = S.sharded_reconstructor(t, nb=nb, ctx=ctx)
    torch.cuda.synchronize()
    ctx.set_block(nb)
    C = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
    T = torch.empty((nm, nts), dtype=torch.float64, device="cuda")
    M.matcov_tile(C, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
    M.matcov_tile(T, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
    M.reconstructor(nm, nts, C, nm, T, nts, 1, prec="fp64", ctx=ctx)
    ctx.synchronize()
    err = (torch.linalg.norm(R - T) / torch.linalg.norm(T)).item()
    assert lay.owned == list(range(lay.nt)) and err <= 1e-12, err
    ctx.close()


def test_dense_blocks_check_arguments(built, cuda):
    import ctypes as C
    from moao_b200._lib import lib
    ctx = M.Context(0)
    info = C.c_int()
    assert lib().moao_dense_potrf_inv(ctx.handle, 4, None, 4, None, 4, C.byref(info)) == 1
    assert lib().moao_dense_gemm(ctx.handle, 0, 0, -1, 1, 1, 1.0, None, 1, None, 1, 0.0, None, 1) == 1
    ctx.close()
