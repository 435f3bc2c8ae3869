"""Host-side mirror of the reference's operator interface for the reconstructor path.

Names, argument order and meaning follow the reference so code written against
it reads the same:

=======================  ==================================================
this module              reference
=======================  ==================================================
``Tomo``                 ``Tomo_struct<T>`` (common/tomo_struct/tomo_struct.hpp:9)
``matcov_tile``          ``MOAO_COMMON::matcov_tile`` (common/compute/matcov.cpp:17)
``reconstructor``        ``MOAO_LAPACK::reconstructor`` (lapack/compute/reconstructor.cpp:32)
``Cee_Cvv``              ``MOAO_LAPACK::Cee_Cvv`` (lapack/compute/cee_cvv.cpp:50)
``Intersample``          ``intersample_prepare/_init/_process/_free``
                         (common/tomo_struct/intersample.cpp:74-333)
=======================  ==================================================

Matrices are column-major with an explicit leading dimension, as in the
reference. A matrix argument is either a CUDA ``torch.Tensor`` of float64
(device path, asynchronous on the context stream, ordered after the work
already queued on torch's current stream and before the work queued there
afterwards, so tensors flow between torch and this library without explicit
synchronisation) or a writable float64
``numpy.ndarray`` (host path: copied to the GPU, computed there, copied back,
keeping the reference's in-place contracts). Every computation runs in the
CUDA library; there is no CPU implementation in this package.

Error behaviour: an unknown ``type_mat`` (the reference exits) raises
``MoaoError``; a non-positive Cholesky pivot (the reference prints and returns
without solving) raises ``NotSPDError`` carrying the 1-based column, after Cmm
has been partially overwritten and Ctm left untouched, as in the reference.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import Optional

import numpy as np

from ._lib import (IsampleInfo, MoaoError, NotSPDError, PREC, SolveReport, TomoInfo, check,
                   lib)

__all__ = ["Context", "Tomo", "matcov_tile", "reconstructor", "Cee_Cvv", "Intersample",
           "default_context", "MoaoError", "NotSPDError"]


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x, what: str) -> int:
    """Address of a float64 matrix argument plus a flag telling host or device."""
    if _is_torch(x):
        import torch
        if x.dtype != torch.float64:
            raise TypeError(f"{what}: expected float64, got {x.dtype}")
        if not x.is_cuda:
            raise TypeError(f"{what}: CPU torch tensors are not accepted; pass a CUDA tensor or a numpy array")
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        if x.dtype != np.float64:
            raise TypeError(f"{what}: expected float64, got {x.dtype}")
        if not (x.flags.c_contiguous or x.flags.f_contiguous):
            raise ValueError(f"{what}: array must be contiguous")
        return x.ctypes.data
    raise TypeError(f"{what}: expected a CUDA torch.Tensor or a numpy.ndarray, got {type(x)}")


class _TorchOrder:
    """Stream ordering of a device call against torch's current stream.

    On entry the context's stream waits for the work already queued on torch's
    current stream (the producer of the inputs); on exit torch's current stream
    waits for the context's work (so later torch kernels, and the caching
    allocator's reuse of freed blocks, come after the call). No host
    synchronisation; a no-op when both are the same stream."""

    def __init__(self, ctx: "Context", active: bool):
        self.active = active
        self.ctx = ctx

    def __enter__(self):
        if not self.active:
            return self
        import torch
        self.cur = torch.cuda.current_stream(self.ctx.device)
        handle = self.ctx.stream
        self.same = handle == self.cur.cuda_stream
        if not self.same:
            self.ext = torch.cuda.ExternalStream(handle, device=self.ctx.device)
            self.ext.wait_stream(self.cur)
        return self

    def __exit__(self, *exc):
        if self.active and not self.same:
            self.cur.wait_stream(self.ext)
        return False


def _on_device(*xs) -> bool:
    kinds = {_is_torch(x) for x in xs if x is not None}
    if len(kinds) > 1:
        raise TypeError("mixing device tensors and host arrays in one call is not supported")
    return kinds == {True}


class Context:
    """One device context: stream, cached device geometry, workspaces."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        check(lib().moao_ctx_create(device, C.byref(h)), "moao_ctx_create")
        self._h = h
        self.device = device
        if stream is not None:
            self.set_stream(stream)

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream: Optional[int]):
        """Run on an external cudaStream_t given as an int handle, e.g. torch's
        ``torch.cuda.current_stream().cuda_stream`` (0 is the legacy default
        stream); None returns to the context's own stream."""
        if stream is None:
            check(lib().moao_ctx_use_own_stream(self._h), "moao_ctx_use_own_stream")
        else:
            check(lib().moao_ctx_set_stream(self._h, C.c_void_p(stream)), "moao_ctx_set_stream")

    @property
    def stream(self) -> int:
        return lib().moao_ctx_stream(self._h) or 0

    def synchronize(self):
        check(lib().moao_ctx_synchronize(self._h), "moao_ctx_synchronize")

    @property
    def launches(self) -> int:
        return int(lib().moao_ctx_launch_count(self._h))

    def set_block(self, nb: int):
        check(lib().moao_ctx_set_block(self._h, nb), "moao_ctx_set_block")

    def set_mixed(self, bf16_slices: int = 3, ozaki_slices: int = 5, max_refine: int = 1,
                  tol: float = 0.0, final_residual: bool = False, corr_slices: int = 0):
        """Options of the mixed-precision reconstructor (see moao_ctx_set_mixed):
        bf16 slices of the bf16x3 format, int8 slices of the refinement residual,
        refinement corrections, stop tolerance, a last residual evaluation, and
        the factor slices of the correction solves (0: 1 for fp16x2, 2 for bf16x3)."""
        check(lib().moao_ctx_set_mixed(self._h, bf16_slices, corr_slices, ozaki_slices,
                                       max_refine, tol, int(final_residual)),
              "moao_ctx_set_mixed")

    def set_factor_format(self, fmt: str):
        """'bf16x3' (3 bf16 slices, 6 products) or 'f16x2' (2 fp16 slices scaled
        per row, 3 products) for the mixed path's tensor-core operands."""
        code = {"bf16x3": 0, "f16x2": 1}[fmt]
        check(lib().moao_ctx_set_factor_format(self._h, code), "moao_ctx_set_factor_format")

    def set_lookahead(self, sms=8):
        """Mixed factorisation: factor the next diagonal block on a side stream
        beside the trailing update, which leaves it `sms` SMs (default 8;
        0 or False turns the lookahead off; True means 8). Same results."""
        n = 8 if sms is True else int(sms)
        check(lib().moao_ctx_set_lookahead(self._h, n), "moao_ctx_set_lookahead")

    def set_offsets(self, begin, end, value):
        """Block-constant offsets of Cmm for the mixed path (see moao_ctx_set_offsets);
        empty sequences clear them."""
        b = np.ascontiguousarray(begin, dtype=np.int32)
        e = np.ascontiguousarray(end, dtype=np.int32)
        v = np.ascontiguousarray(value, dtype=np.float64)
        if not (len(b) == len(e) == len(v)):
            raise ValueError("set_offsets: begin, end and value differ in length")
        check(lib().moao_ctx_set_offsets(self._h, len(b), b.ctypes.data, e.ctypes.data,
                                         v.ctypes.data), "moao_ctx_set_offsets")

    def set_offsets_from_tomo(self, tomo: "Tomo"):
        """Declare the LGS constant blocks of the tomo's covariance model."""
        check(lib().moao_ctx_set_offsets_from_tomo(self._h, tomo.handle),
              "moao_ctx_set_offsets_from_tomo")

    def set_host_cache(self, on: bool = True):
        """Host-buffer cache of the drop-in path (see moao_ctx_set_host_cache):
        the caller promises not to modify the host Cmm / Ctm between
        matcov_tile on host buffers and reconstructor on host buffers."""
        check(lib().moao_ctx_set_host_cache(self._h, int(bool(on))), "moao_ctx_set_host_cache")

    def set_gemm_tile(self, cfg: int = 1):
        """Tile configuration of the large FP64 products (see
        moao_ctx_set_gemm_tile); same results."""
        check(lib().moao_ctx_set_gemm_tile(self._h, int(cfg)), "moao_ctx_set_gemm_tile")

    def set_residual_scheme(self, scheme: str = "crt"):
        """Refinement residual of the mixed path: 'crt' (exact products of the
        sliced operands by the Chinese remainder theorem, the default) or
        'slices' (int8 slice products); moao_ctx_set_residual."""
        code = {"slices": 0, "crt": 1}[scheme]
        check(lib().moao_ctx_set_residual(self._h, code), "moao_ctx_set_residual")

    def set_tc_pair(self, on: bool = True):
        """Tensor-core products of the mixed path on CTA pairs (256 x 256 tiles)
        or single CTAs (the default; moao_ctx_set_tc_pair); same results."""
        check(lib().moao_ctx_set_tc_pair(self._h, int(bool(on))), "moao_ctx_set_tc_pair")

    def set_lookahead_max(self, sms: int = 8):
        """SMs left to the next diagonal block in the last panels (see
        moao_ctx_set_lookahead_max)."""
        check(lib().moao_ctx_set_lookahead_max(self._h, int(sms)), "moao_ctx_set_lookahead_max")

    def set_accuracy(self, target: float = 0.0):
        """Accuracy target of the mixed reconstructor (0: off); a miss makes the
        FP64 path compute R (report fallback = 1). See moao_ctx_set_accuracy."""
        check(lib().moao_ctx_set_accuracy(self._h, float(target)), "moao_ctx_set_accuracy")

    def set_wait_limit(self, polls: int = 0):
        """Bound of the tensor-core kernel's waits in polls (0: the default);
        see moao_ctx_set_wait_limit."""
        check(lib().moao_ctx_set_wait_limit(self._h, int(polls)), "moao_ctx_set_wait_limit")

    def set_kernel_timing(self, enable: bool):
        check(lib().moao_ctx_set_kernel_timing(self._h, int(enable)), "moao_ctx_set_kernel_timing")

    def kernel_stats(self, family: str) -> dict:
        n, ms, work = C.c_longlong(), C.c_double(), C.c_double()
        check(lib().moao_ctx_kernel_stats(self._h, family.encode(), C.byref(n), C.byref(ms),
                                          C.byref(work)), "moao_ctx_kernel_stats")
        return {"launches": n.value, "ms": ms.value, "work": work.value}

    def reset_kernel_stats(self):
        check(lib().moao_ctx_reset_kernel_stats(self._h), "moao_ctx_reset_kernel_stats")

    def close(self):
        if self._h:
            lib().moao_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_ctx_lock = threading.Lock()
_default: dict = {}


def default_context(device: Optional[int] = None) -> Context:
    if device is None:
        try:
            import torch
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        except Exception:
            device = 0
    with _ctx_lock:
        if device not in _default:
            _default[device] = Context(device)
        return _default[device]


class Tomo:
    """The system model (``Tomo_struct``): parameter files, valid subapertures,
    LGS elongation, projected subapertures per layer and WFS noise."""

    def __init__(self, sys_file: str, atm_file: str):
        h = C.c_void_p()
        check(lib().moao_tomo_create(os.fsencode(sys_file), os.fsencode(atm_file), C.byref(h)),
              "moao_tomo_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def updateAtm(self, atm_file: str):
        check(lib().moao_tomo_update_atm(self._h, os.fsencode(atm_file)), "moao_tomo_update_atm")

    def set_profile(self, cn2, h, L0):
        cn2 = np.ascontiguousarray(cn2, dtype=np.float64)
        hh = np.ascontiguousarray(h, dtype=np.float64)
        L0 = np.ascontiguousarray(np.broadcast_to(L0, cn2.shape), dtype=np.float64)
        check(lib().moao_tomo_set_profile(self._h, len(cn2), cn2.ctypes.data, hh.ctypes.data,
                                          L0.ctypes.data), "moao_tomo_set_profile")

    def setTarget(self, idx: int):
        check(lib().moao_tomo_set_target(self._h, idx), "moao_tomo_set_target")

    @property
    def info(self) -> TomoInfo:
        i = TomoInfo()
        check(lib().moao_tomo_get_info(self._h, C.byref(i)), "moao_tomo_get_info")
        return i

    def getNMeas(self) -> int:
        return int(self.info.nmeas)

    def getNMeasTS(self) -> int:
        return int(self.info.nmeasts)

    def table(self, name: str) -> np.ndarray:
        n = lib().moao_tomo_table(self._h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        lib().moao_tomo_table(self._h, name.encode(), out.ctypes.data, n)
        return out

    def close(self):
        if self._h:
            lib().moao_tomo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def matcov_tile(data, nrows: int, ncols: int, xoffset: int, yoffset: int, lda: int, tomo: Tomo,
                type_mat: int, ctx: Optional[Context] = None):
    """Fill a tile of a covariance matrix (column-major, leading dimension lda).

    type_mat 1: Cmm, lower triangle only (uplo='l'); 3: Ctm (truth sensor rows);
    4: Ctt; 2: Cmt (truth sensor columns); 5: Cmm with both triangles."""
    ctx = ctx or default_context()
    p = _ptr(data, "matcov_tile data")
    if _on_device(data):
        with _TorchOrder(ctx, True):
            check(lib().moao_matcov_tile(ctx.handle, tomo.handle, p, nrows, ncols, xoffset,
                                         yoffset, lda, type_mat), "moao_matcov_tile")
    else:
        check(lib().moao_matcov_tile_host(ctx.handle, tomo.handle, p, nrows, ncols, xoffset,
                                          yoffset, lda, type_mat), "moao_matcov_tile_host")


def reconstructor(nmeas: int, nmeasts: int, Cmm, ldCmm: int, Ctm, ldCtm: int, ngal: int = 1,
                  prec: str = "fp64", ctx: Optional[Context] = None) -> dict:
    """R = Ctm Cmm^-1 in place in Ctm; Cmm is overwritten by its lower Cholesky
    factor. Returns the solve report as a dict."""
    ctx = ctx or default_context()
    rep = SolveReport()
    pc, pt = _ptr(Cmm, "Cmm"), _ptr(Ctm, "Ctm")
    if _on_device(Cmm, Ctm):
        with _TorchOrder(ctx, True):
            st = lib().moao_reconstructor(ctx.handle, nmeas, nmeasts, pc, ldCmm, pt, ldCtm, ngal,
                                          PREC[prec], C.byref(rep))
    else:
        # host buffers: the drop-in entry point, in the precision asked for
        check(lib().moao_ctx_set_host_precision(ctx.handle, PREC[prec]),
              "moao_ctx_set_host_precision")
        st = lib().moao_reconstructor_host(ctx.handle, nmeas, nmeasts, pc, ldCmm, pt, ldCtm, ngal,
                                           C.byref(rep))
    check(st, "reconstructor", column=rep.info) if st == 2 else check(st, "reconstructor")
    return {k: getattr(rep, k) for k, _ in SolveReport._fields_}


def Cee_Cvv(nmeas, nmeasts, nact, Cmm, ldCmm, Cpp, ldCpp, Cpm, ldCpm, R, ldR, Dx, ldDx, Cee,
            ldCee, Cvv, ldCvv, Tmp, ldTmp, prec: str = "fp64", ctx: Optional[Context] = None):
    """Cee = Ctt - Ctm R^T - R Ctm^T + R Cmm R^T ; Cvv = Dx Cee Dx^T (Cpp and Cpm
    are destroyed, Tmp is scratch), exactly the reference's in-place contract.
    prec "mixed" (device buffers) evaluates Cee = Ctt - R Ctm^T - E R^T with the
    residual E = Ctm - R Cmm on the int8 tensor cores (moao_cee_cvv_prec); Cpm
    then ends as R Cmm and Cpp is left as given."""
    ctx = ctx or default_context()
    mats = [Cmm, Cpp, Cpm, R, Dx, Cee, Cvv, Tmp]
    names = ["Cmm", "Cpp", "Cpm", "R", "Dx", "Cee", "Cvv", "Tmp"]
    lds = [ldCmm, ldCpp, ldCpm, ldR, ldDx, ldCee, ldCvv, ldTmp]
    args = []
    for m, n, ld in zip(mats, names, lds):
        args += [_ptr(m, n), ld]
    dev = _on_device(*mats)
    with _TorchOrder(ctx, dev):
        if dev:
            st = lib().moao_cee_cvv_prec(ctx.handle, nmeas, nmeasts, nact, *args, PREC[prec])
        else:
            check(lib().moao_ctx_set_host_precision(ctx.handle, PREC[prec]),
                  "moao_ctx_set_host_precision")
            st = lib().moao_cee_cvv_host(ctx.handle, nmeas, nmeasts, nact, *args)
        check(st, "Cee_Cvv")


def intersample_inputs(nssp: int, Dtel: float, obs: float, coupling: float = 0.2,
                       tables: bool = True, ctx: Optional[Context] = None):
    """The intersample tables without files or Python tooling (moao_intersample_inputs):
    returns (nact, N, idx, abs2fi, otf_tel); idx is exact host work, abs2fi and
    otf_tel are computed on the device (None when tables is False)."""
    na, N = C.c_long(), C.c_long()
    check(lib().moao_intersample_inputs(None, nssp, Dtel, obs, coupling, C.byref(na), C.byref(N),
                                        None, None, None), "moao_intersample_inputs")
    idx = np.zeros(na.value * na.value, dtype=np.int64)
    a = o = None
    if tables:
        ctx = ctx or default_context()
        a = np.zeros((N.value, N.value))
        o = np.zeros((N.value, N.value))
    check(lib().moao_intersample_inputs(ctx.handle if tables else None, nssp, Dtel, obs, coupling,
                                        C.byref(na), C.byref(N), idx.ctypes.data,
                                        a.ctypes.data if tables else None,
                                        o.ctypes.data if tables else None),
          "moao_intersample_inputs")
    return na.value, N.value, idx, a, o


class Intersample:
    """PSF from Cvv; the three input tables (idx, abs2fi, otf_tel) are given as
    arrays instead of the reference's idx.fits / abs2fi.fits / otftel.fits."""

    def __init__(self, nidx: int, np_: int, Dtel: float, idx, abs2fi, otf_tel,
                 ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        abs2fi = np.ascontiguousarray(abs2fi, dtype=np.float64)
        otf_tel = np.ascontiguousarray(otf_tel, dtype=np.float64)
        h = C.c_void_p()
        check(lib().moao_intersample_create(self.ctx.handle, nidx, np_, Dtel, idx.ctypes.data,
                                            abs2fi.ctypes.data, otf_tel.ctypes.data, C.byref(h)),
              "moao_intersample_create")
        self._h = h
        info = IsampleInfo()
        check(lib().moao_intersample_get_info(h, C.byref(info)), "moao_intersample_get_info")
        self.N, self.np, self.nidx = int(info.N), int(info.np), int(info.nidx)
        self.dactupix = float(info.dactupix)
        self.lam = float(info.lambda_)

    def process(self, Cvv, out=None):
        """PSF (N x N, FFTW-unnormalised) of a Cvv given as a CUDA tensor (result
        is a CUDA tensor) or a numpy array (result is a numpy array)."""
        if _is_torch(Cvv):
            import torch
            if out is None:
                out = torch.empty((self.N, self.N), dtype=torch.float64, device=Cvv.device)
            with _TorchOrder(self.ctx, True):
                check(lib().moao_intersample_process(self._h, _ptr(Cvv, "Cvv"),
                                                     _ptr(out, "psf")), "moao_intersample_process")
            return out
        cvv = np.ascontiguousarray(Cvv, dtype=np.float64)
        if out is None:
            out = np.empty((self.N, self.N), dtype=np.float64)
        check(lib().moao_intersample_process_host(self._h, cvv.ctypes.data, _ptr(out, "psf")),
              "moao_intersample_process_host")
        return out

    def close(self):
        if self._h:
            lib().moao_intersample_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
