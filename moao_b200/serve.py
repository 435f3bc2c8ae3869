"""Serving loop: reconstructor requests against registered systems, admitted
onto device slots by HBM footprint as they arrive (see moao_server_* in
include/moao_b200.h). No reference counterpart: the reference runs one
synchronous driver loop (lapack/moao_lapack.cpp:95-190).

    srv = Server(slots=3)
    sid = srv.add_system(sys_file, atm_file, Dx=Dx, idx=idx, abs2fi=a, otf=o)
    rid = srv.submit(sid, cn2, h, L0, prec="mixed", R=R_out, psf=psf_out)
    res = srv.wait(rid)          # dict: status, latency_ms, queue_ms, ...
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._lib import (PREC, STATUS, MoaoError, Request, RequestResult, ServerOpts, ServerStats,
                   check, lib)

BUSY, CANCELLED = 8, 9


def _out(a, n, what):
    if a is None:
        return None
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.writeable or a.size < n:
        raise TypeError(f"{what}: writable float64 array of at least {n} elements expected")
    if not (a.flags.c_contiguous or a.flags.f_contiguous):
        raise ValueError(f"{what}: array must be contiguous")
    return a


def _result(r: RequestResult) -> dict:
    d = {k: getattr(r, k) for k, _ in RequestResult._fields_ if k != "message"}
    d["message"] = r.message.decode(errors="replace")
    d["status_name"] = STATUS.get(r.status, str(r.status))
    return d


class Server:
    def __init__(self, device: int = 0, slots: int = 3, hbm_budget_gb: float = 0.0,
                 queue_capacity: int = 0, nb: int = 0, dry_run: bool = False):
        o = ServerOpts(device, slots, hbm_budget_gb, queue_capacity, nb, int(dry_run))
        h = C.c_void_p()
        check(lib().moao_server_create(C.byref(o), C.byref(h)), "moao_server_create")
        self._h = h
        self._keep = {}  # id -> arrays the request writes or reads

    def add_system(self, sys_file: str, atm_file: str, Dx=None, idx=None, abs2fi=None,
                   otf=None) -> int:
        """Registers a system; Dx (nact x nmeasts) enables Cvv, the intersample
        tables (idx, abs2fi, otf) enable the PSF."""
        keep = []
        nact = 0
        dxp = ip = ap = op = None
        if Dx is not None:
            Dx = np.asfortranarray(Dx, dtype=np.float64)
            nact = Dx.shape[0]
            keep.append(Dx)
            dxp = Dx.ctypes.data
        if idx is not None:
            idx = np.ascontiguousarray(idx, dtype=np.int64)
            abs2fi = np.ascontiguousarray(abs2fi, dtype=np.float64)
            otf = np.ascontiguousarray(otf, dtype=np.float64)
            keep += [idx, abs2fi, otf]
            ip, ap, op = idx.ctypes.data, abs2fi.ctypes.data, otf.ctypes.data
        sid = C.c_int()
        check(lib().moao_server_add_system(self._h, sys_file.encode(), atm_file.encode(), nact,
                                           dxp, ip, ap, op, C.byref(sid)), "moao_server_add_system")
        return int(sid.value)

    def add_system_synth(self, sys_file: str, atm_file: str, Dx, coupling: float = 0.2) -> int:
        """Registers a system whose PSF tables the library synthesises itself for
        the truth sensor (moao_server_add_system_synth); Dx is nact x nmeasts with
        nact the synthesised DM's actuator count (moao_b200.intersample_inputs)."""
        Dx = np.asfortranarray(Dx, dtype=np.float64)
        sid = C.c_int()
        check(lib().moao_server_add_system_synth(self._h, sys_file.encode(), atm_file.encode(),
                                                 Dx.shape[0], Dx.ctypes.data, coupling,
                                                 C.byref(sid)), "moao_server_add_system_synth")
        return int(sid.value)

    def system_info(self, system: int) -> dict:
        v = [C.c_long() for _ in range(4)]
        check(lib().moao_server_system_info(self._h, system, *[C.byref(x) for x in v]),
              "moao_server_system_info")
        return dict(zip(("nmeas", "nmeasts", "nact", "psf_n"), [int(x.value) for x in v]))

    def submit(self, system: int, cn2, h, L0, target: int = 0, prec: str = "fp64", R=None,
               Cvv=None, psf=None, dry_run_ms: float = 0.0) -> int:
        cn2 = np.ascontiguousarray(cn2, dtype=np.float64)
        h = np.ascontiguousarray(h, dtype=np.float64)
        L0 = np.ascontiguousarray(L0, dtype=np.float64)
        if not (len(cn2) == len(h) == len(L0)):
            raise ValueError("submit: cn2, h and L0 differ in length")
        info = self.system_info(system)
        R = _out(R, info["nmeas"] * info["nmeasts"], "R")
        Cvv = _out(Cvv, info["nact"] ** 2, "Cvv")
        psf = _out(psf, info["psf_n"] ** 2, "psf")
        req = Request(system, len(cn2), cn2.ctypes.data, h.ctypes.data, L0.ctypes.data, target,
                      PREC[prec], None if R is None else R.ctypes.data,
                      None if Cvv is None else Cvv.ctypes.data,
                      None if psf is None else psf.ctypes.data, dry_run_ms)
        rid = C.c_longlong()
        check(lib().moao_serve_submit(self._h, C.byref(req), C.byref(rid)), "moao_serve_submit")
        self._keep[int(rid.value)] = (R, Cvv, psf)
        return int(rid.value)

    def poll(self, rid: int) -> dict:
        r = RequestResult()
        check(lib().moao_serve_poll(self._h, rid, C.byref(r)), "moao_serve_poll")
        return _result(r)

    def wait(self, rid: int, timeout: float = -1.0) -> dict:
        r = RequestResult()
        check(lib().moao_serve_wait(self._h, rid, timeout, C.byref(r)), "moao_serve_wait")
        self._keep.pop(rid, None)
        return _result(r)

    def cancel(self, rid: int):
        check(lib().moao_serve_cancel(self._h, rid), "moao_serve_cancel")

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().moao_server_get_stats(self._h, C.byref(s)), "moao_server_get_stats")
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self._h:
            lib().moao_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
