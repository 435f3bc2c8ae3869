"""Batched reconstructor builds in one CUDA graph launch, and the autotuner of
their panel width and stream count (see moao_batch_reconstructors and
moao_autotune in include/moao_b200.h). No reference counterpart: the
reference builds one reconstructor per driver call."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from ._lib import PREC, STATUS, BatchItem, BatchOpts, check, lib
from .api import Context, Tomo, _TorchOrder, default_context


def batch_reconstructors(tomos: Sequence[Tomo], outputs=None, prec: str = "fp64",
                         streams: int = 0, nb: Optional[Sequence[int]] = None,
                         packed_max: int = 0, ctx: Optional[Context] = None):
    """Builds R for every tomo (its current profile and target) in one graph.
    outputs: CUDA float64 tensors of nmeasts*nmeas elements (R column-major,
    ld nmeasts) or None. packed_max: instances with nmeas <= it are built (FP64)
    by the persistent tile-task kernel (0: the tuned bound, < 0: none).
    Returns (per-instance dicts, run dict)."""
    ctx = ctx or default_context()
    n = len(tomos)
    items = (BatchItem * max(n, 1))()
    for i, t in enumerate(tomos):
        items[i].tomo = t.handle.value
        out = None if outputs is None else outputs[i]
        if out is not None:
            import torch
            if out.dtype != torch.float64 or not out.is_cuda or out.numel() < t.getNMeas() * t.getNMeasTS():
                raise TypeError("batch output: CUDA float64 tensor of nmeasts*nmeas elements expected")
            items[i].d_R = out.data_ptr()
        items[i].nb = 0 if nb is None else int(nb[i])
    opts = BatchOpts()
    opts.prec = PREC[prec]
    opts.streams = streams
    opts.packed_max = int(packed_max)
    with _TorchOrder(ctx, outputs is not None):
        check(lib().moao_batch_reconstructors(ctx.handle, n, C.cast(items, C.c_void_p), C.byref(opts)),
              "moao_batch_reconstructors")
    per = [{"status": items[i].status, "status_name": STATUS.get(items[i].status),
            "info": items[i].info, "nb": items[i].nb_used, "stream": items[i].stream,
            "packed": bool(items[i].packed)}
           for i in range(n)]
    run = {k: getattr(opts, k) for k, _ in BatchOpts._fields_
           if k not in ("prec", "streams", "hbm_budget_gb", "packed_max", "gemm_tile")}
    return per, run


def autotune(samples: Sequence[Tomo], prec: str = "fp64", candidates=None,
             ctx: Optional[Context] = None) -> dict:
    ctx = ctx or default_context()
    arr = (C.c_void_p * len(samples))(*[t.handle.value if hasattr(t.handle, "value") else t.handle
                                       for t in samples])
    cand = None if candidates is None else np.ascontiguousarray(candidates, dtype=np.int32)
    check(lib().moao_autotune(ctx.handle, len(samples), C.cast(arr, C.c_void_p), PREC[prec],
                              None if cand is None else cand.ctypes.data,
                              0 if cand is None else len(cand)), "moao_autotune")
    return tuning(prec, ctx)


def tuning(prec: str = "fp64", ctx: Optional[Context] = None) -> dict:
    ctx = ctx or default_context()
    nbs = (C.c_int * 6)()
    s = C.c_int()
    check(lib().moao_tuning_get(ctx.handle, PREC[prec], C.cast(nbs, C.c_void_p), C.byref(s)),
          "moao_tuning_get")
    classes = ["<2k", "2k-4k", "4k-8k", "8k-16k", "16k-32k", ">=32k"]
    pm = C.c_long()
    check(lib().moao_tuning_get_packed(ctx.handle, PREC[prec], C.byref(pm)), "moao_tuning_get_packed")
    g = (C.c_int * 6)()
    check(lib().moao_tuning_get_gemm(ctx.handle, PREC[prec], C.cast(g, C.c_void_p)), "moao_tuning_get_gemm")
    return {"nb": dict(zip(classes, list(nbs))), "streams": s.value, "packed_max": pm.value,
            "gemm_tile": dict(zip(classes, list(g)))}


def tuning_save(path: str, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    check(lib().moao_tuning_save(ctx.handle, path.encode()), "moao_tuning_save")


def tuning_load(path: str, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    check(lib().moao_tuning_load(ctx.handle, path.encode()), "moao_tuning_load")


def packed_task_list(nmeas: Sequence[int], nmeasts: Sequence[int]):
    """The persistent tile-task kernel's task list for instances of these sizes
    (host only): an (ntasks, 5) int32 array of (instance, type, i, j, k) in claim
    order, and the number of DAG levels."""
    n = np.ascontiguousarray(nmeas, dtype=np.int64)
    m = np.ascontiguousarray(nmeasts, dtype=np.int64)
    cnt, lev = C.c_long(), C.c_int()
    check(lib().moao_packed_task_list(len(n), n.ctypes.data, m.ctypes.data, None, 0, C.byref(cnt),
                                      C.byref(lev)), "moao_packed_task_list")
    out = np.zeros((cnt.value, 5), dtype=np.int32)
    check(lib().moao_packed_task_list(len(n), n.ctypes.data, m.ctypes.data, out.ctypes.data,
                                      cnt.value, C.byref(cnt), C.byref(lev)), "moao_packed_task_list")
    return out, lev.value
