#!/usr/bin/env python
"""Reconstructor builds per second on B200 (ELT-scale system).

One step = one tomographic reconstructor build for the ELT-scale system
(39 m, 64x64 subapertures, 6 LGS + 2 NGS + truth sensor, 35 layers;
nmeas 47,552, nmeasts 5,944): covariance generation of Cmm and Ctm on the GPU,
tiled Cholesky of Cmm and the two triangular solves giving R = Ctm Cmm^-1.

    python bench.py [--gpus N --steps K --warmup W] [--path fp64|mixed]
    python bench.py --impl reference ...     # the reference's CPU path
    python bench.py --probe STAGE --nssp S   # one stage once (profiling captures)

Printed on rank 0: one JSON line. ``value`` is whole-job builds/s with the
system tables resident in HBM. ``e2e`` is the same metric through the
reference-shaped host-buffer entry points of the C ABI (moao_matcov_tile_host
for Cmm and Ctm, then moao_reconstructor_host), host<->device copies inside the
timed region, from and into pinned host memory. Beside them: the error
covariances Cee and Cvv and the PSF Strehl ratio of the mixed path against the
FP64 path at ELT size, their stage times, and full builds of two systems the
CPU finishes, timed on the reference's own CPU code and on the GPU. Multi-GPU
runs are independent replicas (one reconstructor per GPU, no collective on the
data path). The CPU baseline / reference arm runs the reference's own code
(oracle/_ref, compiled from the reference sources: covariance generation, and
LAPACK through scipy's OpenBLAS) on a bounded sample of the ELT workload,
extrapolated by element and flop counts and marked as such.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "R builds/s (ELT-scale reconstructor: matcov Cmm+Ctm, Cholesky, 2 triangular solves)"
UNIT = "builds/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="moao", choices=["moao", "reference"])
    p.add_argument("--path", default="mixed", choices=["fp64", "mixed"])
    p.add_argument("--nb", type=int, default=0,
                   help="panel width (0: 1024, the fastest for both paths)")
    p.add_argument("--nb-fp64", type=int, default=1024, help="panel width of the FP64 comparison arm")
    p.add_argument("--config", default="elt", choices=["elt", "small"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--serving", action="store_true",
                   help="serving-loop benchmark (Poisson arrivals, p50/p99) instead of the build loop")
    p.add_argument("--serve-requests", type=int, default=120)
    p.add_argument("--batch", action="store_true",
                   help="batched uneven instances in one graph launch instead of the build loop")
    p.add_argument("--batch-count", type=int, default=256)
    p.add_argument("--batch-outputs", action="store_true", help="batch: copy every R out")
    p.add_argument("--batch-nssp", default="20,50",
                   help="batch: range of subapertures across the instances (lo,hi)")
    p.add_argument("--batch-no-tune", action="store_true",
                   help="batch: default panel widths and streams instead of the autotuner")
    p.add_argument("--batch-packed", type=int, default=0,
                   help="batch: nmeas bound of the instances packed into the tile-task kernel "
                        "(0: autotuned, -1: none)")
    p.add_argument("--serve-slots", type=int, default=3)
    p.add_argument("--sharded", action="store_true",
                   help="one ELT system's FP64 build with Cmm spread over the ranks (torchrun, "
                        "one GPU each) instead of one build per rank")
    p.add_argument("--no-compare", action="store_true",
                   help="mixed path: skip timing the FP64 path beside it")
    p.add_argument("--no-cee", action="store_true", help="skip the Cee/Cvv/PSF stage at ELT size")
    p.add_argument("--no-pairs", action="store_true",
                   help="skip the measured CPU-vs-GPU full builds of the small systems")
    p.add_argument("--e2e-steps", type=int, default=5, help="builds timed through the host path")
    p.add_argument("--tc-pair", type=int, default=-1, choices=[-1, 0, 1],
                   help="tensor-core products on CTA pairs (1) or single CTAs (0); "
                        "-1: the library's default")
    p.add_argument("--probe", default=None,
                   choices=["matcov_ctm", "build_fp64", "build_mixed", "cee_fp64", "cee_mixed",
                            "gemm_tiles"],
                   help="run one stage once on the ELT geometry at --nssp subapertures (for ncu)")
    p.add_argument("--nssp", type=int, default=37, help="probe: subapertures across (64 = ELT)")
    return p.parse_args()


def system(config):
    from moao_b200 import params as P
    s, a = P.config_elt() if config == "elt" else P.config_small()
    d = tempfile.mkdtemp(prefix="moao_bench_")
    P.write_system(d, s, a)
    return os.path.join(d, "sys-params.txt"), os.path.join(d, "prof-1-atmos-night0.txt"), s, a


def workload_name(config, nm, nts, nl):
    if config == "elt":
        return (f"ELT-scale reconstructor build: 39 m, 64x64 subapertures, 6 LGS + 2 NGS + TS, "
                f"{nl} layers (nmeas {nm}, nmeasts {nts})")
    return f"8 m reconstructor build: 10x10, 3 LGS + 1 NGS + TS, {nl} layers (nmeas {nm}, nmeasts {nts})"


# ----------------------------------------------------------------------------- clocks
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="moao_clocks_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def cpu_reference_sample(sf, af, nm, nts, budget_s=20.0):
    """Times the reference's CPU path on a bounded sample of the build and
    extrapolates it to the whole build; returns (builds/s, info)."""
    import numpy as np
    import scipy.linalg.blas as blas
    import scipy.linalg.lapack as lapack
    O = _oracle()

    cores = os.cpu_count() or 1
    kind = "reference" if O.RefTomo.available() else "port"
    # (1) covariance generation: rows of Ctm (type 3) with every core; per-element
    # cost applies to Cmm too (same layer loop and stencils per element).
    if kind == "reference":
        t = O.RefTomo(sf, af)
        t.setTarget(0)
        run = lambda rows: t.matcov_full(rows, nm, 3, nthreads=cores, ts=max(1, rows // cores + 1))
    else:
        import moao_b200 as M
        g = O.Geometry.from_tomo(M.Tomo(sf, af))
        run = lambda rows: O.matcov(g, rows, nm, 0, 0, 3, nthreads=cores)
    rows, el_time = 2, None
    while True:
        t0 = time.perf_counter()
        run(rows)
        dt = time.perf_counter() - t0
        if dt > budget_s / 3 or rows >= nts:
            el_time = dt / (rows * nm)
            break
        rows = min(nts, rows * 4 if dt < budget_s / 30 else rows * 2)
    n_el = nm * (nm + 1) / 2 + nts * nm
    t_matcov = el_time * n_el
    # (2) LAPACK (scipy's OpenBLAS, all cores): dpotrf + two dtrsm at a reduced size
    rng = np.random.default_rng(0)
    n = 4096
    while True:
        A = rng.standard_normal((n, n))
        C = np.asfortranarray(A + A.T + 4.0 * n * np.eye(n))  # SPD: diagonally dominant
        T = np.asfortranarray(rng.standard_normal((max(n // 8, 1), n)))
        t0 = time.perf_counter()
        L, info = lapack.dpotrf(C, lower=1, clean=0, overwrite_a=1)
        t1 = time.perf_counter()
        X = blas.dtrsm(1.0, L, T, side=1, lower=1, trans_a=1)
        blas.dtrsm(1.0, L, X, side=1, lower=1, trans_a=0)
        t2 = time.perf_counter()
        if t2 - t0 > budget_s / 6 or n >= 16384:
            break
        n *= 2
    rate_potrf = (n ** 3 / 3) / (t1 - t0)
    rate_trsm = (2 * T.shape[0] * n ** 2) / (t2 - t1)
    t_lapack = (nm ** 3 / 3) / rate_potrf + (2 * nts * nm ** 2) / rate_trsm
    total = t_matcov + t_lapack
    info = {
        "cores": cores, "kind": kind, "extrapolated": True,
        "sample": (f"covariance: {rows} Ctm rows x {nm} columns through the reference's matcov_tile "
                   f"({'oracle/_ref' if kind == 'reference' else 'C port'}, {cores} threads), "
                   f"{el_time * 1e6:.2f} us/element scaled to {n_el:.3e} elements; LAPACK: "
                   f"dpotrf n={n} + 2 dtrsm ({T.shape[0]} rows) with scipy OpenBLAS, "
                   f"{rate_potrf / 1e9:.1f} / {rate_trsm / 1e9:.1f} GFLOP/s scaled to nmeas {nm}; "
                   f"extrapolated build {total:.0f} s"),
        "seconds_per_build": total,
    }
    return 1.0 / total, info


PAIR_SYSTEMS = ("small", "nx5120_nLayers10_wfs8_Nssp29")


def pair_system(name):
    """(label, sys file, atm file) of a system the CPU builds in full: the 8 m
    small system, or a check system of the reference (datafile/check, parsed
    into tests/golden/check_sets.json)."""
    from moao_b200 import params as P
    if name == "small":
        sp, ap = P.config_small()
        label = "8 m, 10x10, 3 LGS + 1 NGS + TS, 3 layers"
    else:
        with open(os.path.join(ROOT, "tests", "golden", "check_sets.json")) as f:
            d = json.load(f)[name]
        sp, ap = P.SysParams(**d["sys"]), P.AtmParams(**d["atm"])
        label = (f"reference check system {name} ({sp.diam:g} m, {sp.nssp}x{sp.nssp}, {sp.nLgs} LGS + "
                 f"{sp.nW - sp.nLgs - 1} NGS + TS, {ap.nLayer} layers)")
    d = tempfile.mkdtemp(prefix="moao_pair_")
    P.write_system(d, sp, ap)
    return label, os.path.join(d, "sys-params.txt"), os.path.join(d, "prof-1-atmos-night0.txt")


def cpu_full_build(sf, af):
    """One full FP64 build on the host cores with the reference's own code:
    matcov_tile of Cmm and Ctm (oracle/_ref, all cores on independent tiles),
    then MOAO_LAPACK::reconstructor (oracle/_ref, scipy's OpenBLAS threads).
    Returns (seconds, R, nmeas, nmeasts, cores)."""
    O = _oracle()
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    t = O.RefTomo(sf, af)
    nm, nts = t.info.nmeas, t.info.nmeasts
    t.setTarget(0)
    Cmm = t.matcov_full(nm, nm, 1, nthreads=cores)
    Ctm = t.matcov_full(nts, nm, 3, nthreads=cores)
    if O.RefDense.available():
        _, R = O.RefDense.reconstructor(Cmm, Ctm)
    else:
        _, R, _ = O.reconstructor(Cmm, Ctm)
    return time.perf_counter() - t0, R, nm, nts, cores


def cpu_reference_pairs():
    """The reference's CPU path, full builds of the pair systems (seconds each)."""
    out = []
    for name in PAIR_SYSTEMS:
        label, sf, af = pair_system(name)
        sec, _, nm, nts, cores = cpu_full_build(sf, af)
        out.append({"system": label, "nmeas": nm, "nmeasts": nts, "cpu_s": sec, "cores": cores})
    return out


# ----------------------------------------------------------------------------- GPU
def fp64_peak_tflops(torch):
    """cuBLAS DGEMM (torch.matmul float64, 8192^3), best of 5: the measured FP64
    tensor-pipe ceiling the FP64 kernels are reported against."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / best / 1e9


def lower_panel_bytes(nrows, ncols, d, corner_only, w=512):
    """Bytes moved by the host entry points' lower-part copies (the column-panel
    copies of moao_matcov_tile_host / moao_reconstructor_host)."""
    total = 0
    for c0 in range(0, ncols, w):
        c1 = min(ncols, c0 + w)
        r0 = max(0, c0 - d)
        if r0 >= nrows:
            break
        r1 = min(nrows, max(r0, c1 - d)) if corner_only else nrows
        total += 8 * (r1 - r0) * (c1 - c0)
    return total


def gpu_build_device(M, torch, ctx, t, nm, nts, prec, rep_out=None, reps=5):
    """Median device ms of full builds (matcov Cmm + Ctm, reconstructor) through
    the device API, and the R of the last one (its solve report into rep_out)."""
    Cmm = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
    Ctm = torch.empty((nm, nts), dtype=torch.float64, device="cuda")
    ms = []
    for k in range(reps + 2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        M.matcov_tile(Cmm, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
        M.matcov_tile(Ctm, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
        rep = M.reconstructor(nm, nts, Cmm, nm, Ctm, nts, 1, prec=prec, ctx=ctx)
        e1.record()
        torch.cuda.synchronize()
        if k >= 2:
            ms.append(e0.elapsed_time(e1))
        if rep_out is not None:
            rep_out.update(rep)
    import numpy as np
    R = Ctm.cpu().numpy().T.copy(order="F")
    return float(np.median(ms)), R


def gpu_build_host(M, t, nm, nts, prec, ctx, reps=3):
    """Median wall ms of full builds through the host-buffer (drop-in) entry
    points: moao_matcov_tile_host for Cmm and Ctm, moao_reconstructor_host."""
    import numpy as np
    Cmm = np.zeros((nm, nm), order="F")
    Ctm = np.zeros((nts, nm), order="F")
    ms = []
    for k in range(reps + 1):
        t0 = time.perf_counter()
        M.matcov_tile(Cmm, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
        M.matcov_tile(Ctm, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
        M.reconstructor(nm, nts, Cmm, nm, Ctm, nts, 1, prec=prec, ctx=ctx)
        if k >= 1:
            ms.append(1000.0 * (time.perf_counter() - t0))
    return float(np.median(ms))


def measured_pairs(M, torch, ctx):
    """Full builds of the pair systems on the reference's CPU code and on the
    GPU (device API FP64 and mixed, and the drop-in host path FP64), with the
    agreement of the GPU FP64 R with the CPU R."""
    O = _oracle()
    out = []
    for name in PAIR_SYSTEMS:
        label, sf, af = pair_system(name)
        t = M.Tomo(sf, af)
        t.setTarget(0)
        nm, nts = t.getNMeas(), t.getNMeasTS()
        ms64, R64 = gpu_build_device(M, torch, ctx, t, nm, nts, "fp64")
        ctx.set_offsets_from_tomo(t)
        ctx.set_accuracy(1e-5)  # ill-conditioned systems fall back to FP64
        rep = {}
        msmx, Rmx = gpu_build_device(M, torch, ctx, t, nm, nts, "mixed", rep)
        ctx.set_accuracy(0)
        ms_host = gpu_build_host(M, t, nm, nts, "fp64", ctx)
        cpu_s, Rc, _, _, cores = cpu_full_build(sf, af)
        out.append({
            "system": label, "nmeas": nm, "nmeasts": nts,
            "cpu_reference_s": cpu_s, "cpu_cores": cores,
            "cpu_kind": "reference" if O.RefDense.available() else "reference matcov + oracle LAPACK",
            "gpu_fp64_ms": ms64, "gpu_mixed_ms": msmx, "gpu_fp64_dropin_host_ms": ms_host,
            "speedup_fp64": cpu_s * 1000.0 / ms64, "speedup_mixed": cpu_s * 1000.0 / msmx,
            "speedup_fp64_dropin": cpu_s * 1000.0 / ms_host,
            "rel_fro_R_gpu_fp64_vs_cpu": O.rel_fro(R64, Rc), "rel_fro_R_gpu_mixed_vs_cpu": O.rel_fro(Rmx, Rc),
            "mixed_accuracy_target": 1e-5, "mixed_fell_back_to_fp64": bool(rep.get("fallback")),
            "mixed_est_error": rep.get("est_error"),
        })
    ctx.set_offsets([], [], [])
    return out


def cee_stage(M, torch, ctx, t, nm, nts, Cmm, R_fp64, R_mixed):
    """Cee, Cvv and the PSF at ELT size from the FP64 R through the FP64 chain
    and from the mixed R through the mixed chain: stage times (second call of
    each; CUDA events on the context stream) and the relative Frobenius errors
    and Strehl-ratio difference of the mixed results against the FP64 ones."""
    import numpy as np
    from moao_b200 import inputs as I
    x = I.intersample_inputs(t.info.nssp_ts, t.info.diam, t.info.obs)
    nact = x.nact
    Dx = torch.from_numpy(np.ascontiguousarray(I.make_dx(nact, nts).T)).cuda()
    Ctm2 = torch.empty((nm, nts), dtype=torch.float64, device="cuda")
    Ctt = torch.empty((nts, nts), dtype=torch.float64, device="cuda")
    Cee = torch.empty((nts, nts), dtype=torch.float64, device="cuda")
    Cvv = torch.empty((nact, nact), dtype=torch.float64, device="cuda")
    Tmp = torch.empty((nts, nact), dtype=torch.float64, device="cuda")
    res = {}
    for prec, R in (("fp64", R_fp64), ("mixed", R_mixed)):
        for k in range(2):  # the first call sizes the workspaces
            M.matcov_tile(Cmm, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
            M.matcov_tile(Ctm2, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
            M.matcov_tile(Ctt, nts, nts, 0, 0, nts, t, 4, ctx=ctx)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            M.Cee_Cvv(nm, nts, nact, Cmm, nm, Ctt, nts, Ctm2, nts, R, nts, Dx, nact, Cee, nts, Cvv,
                      nact, Tmp, nact, prec=prec, ctx=ctx)
            e1.record()
            torch.cuda.synchronize()
        res[prec] = (Cee.clone(), Cvv.clone(), e0.elapsed_time(e1))
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    isx = M.Intersample(nact * nact, x.np_, t.info.diam, x.idx, x.abs2fi, x.otf, ctx=ctx)
    psf0 = isx.process(torch.zeros((nact, nact), dtype=torch.float64, device="cuda"))
    peak0 = float(psf0.max())
    strehl = lambda C, c: float(isx.process(c * C).max()) / peak0
    # The seeded N(0, 1) Dx gives phase variances whose PSF is all halo (Strehl
    # ~1e-5): both Cvv are scaled by the one factor that puts the FP64 Strehl at
    # 0.5 (bisection in log c; Cvv is quadratic in Dx, so this is Dx scaled).
    lo, hi = -40.0, 10.0
    for _ in range(48):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if strehl(res["fp64"][1], 10.0 ** mid) > 0.5 else (lo, mid)
    c = 10.0 ** (0.5 * (lo + hi))
    s_raw = strehl(res["fp64"][1], 1.0)
    s64 = strehl(res["fp64"][1], c)
    smx = strehl(res["mixed"][1], c)
    isx.close()
    out = {"nact": nact, "ms_fp64_chain": res["fp64"][2], "ms_mixed_chain": res["mixed"][2],
           "rel_fro_err_Cee_vs_fp64": rel(res["mixed"][0], res["fp64"][0]),
           "rel_fro_err_Cvv_vs_fp64": rel(res["mixed"][1], res["fp64"][1]),
           "strehl_fp64": s64, "strehl_mixed": smx, "strehl_delta": abs(smx - s64),
           "strehl_cvv_scale": c, "strehl_fp64_unscaled_dx": s_raw,
           "note": ("Cee/Cvv from the FP64 R by the FP64 chain against those from the mixed R by "
                    "the mixed chain (int8 Ozaki products); Strehl = PSF peak / telescope-only peak, "
                    "512^2 PSF on the truth direction, both Cvv scaled by strehl_cvv_scale so that the "
                    "FP64 Strehl is 0.5")}
    del Ctm2, Ctt, Cee, Cvv, Tmp, Dx, res
    torch.cuda.empty_cache()
    return out


def e2e_dropin(M, torch, ctx, t, nm, nts, prec, steps, set_profile, cache=False):
    """Builds through the reference-shaped host-buffer entry points of the C
    ABI (moao_matcov_tile_host of Cmm and Ctm, then moao_reconstructor_host),
    host buffers in pinned memory, every copy inside the timed region. With
    cache, moao_ctx_set_host_cache is on: the reconstructor reuses the device
    copies of the Cmm and Ctm that matcov_tile just wrote to those buffers."""
    ctx.set_host_cache(cache)
    Cmm_h = torch.empty((nm, nm), dtype=torch.float64, pin_memory=True).numpy().T
    Ctm_h = torch.empty((nm, nts), dtype=torch.float64, pin_memory=True).numpy().T

    def one():
        set_profile()
        M.matcov_tile(Cmm_h, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
        M.matcov_tile(Ctm_h, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
        M.reconstructor(nm, nts, Cmm_h, nm, Ctm_h, nts, 1, prec=prec, ctx=ctx)
    one()  # sizes the host-path workspaces
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    ctx.set_host_cache(False)
    R = Ctm_h.copy(order="F")
    if cache:  # the diagonal blocks of the panels go down twice, nothing else
        h2d = 2 * lower_panel_bytes(nm, nm, 0, True)
    else:
        h2d = (lower_panel_bytes(nm, nm, 0, True) + lower_panel_bytes(nm, nm, 0, False) +
               8 * nm * nts)
    d2h = 2 * lower_panel_bytes(nm, nm, 0, False) + 2 * 8 * nm * nts
    del Cmm_h, Ctm_h
    return sec, h2d, d2h, R


def read_traffic_ratio(name, key="dram_bytes_per_work"):
    """A figure from a committed ncu summary (line 'key: X'), by default the
    bytes of DRAM traffic per unit of work of the kernel, or None."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith(key + ":"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


# ----------------------------------------------------------------------------- serving
SERVING_METRIC = "serving: reconstructor requests/s (R + Cvv + 512^2 PSF each) and p50/p99 latency"


def serving_main(args):
    """Poisson-arrival reconstructor requests on the serving loop (mixed path,
    several slots) against the same requests run back to back on the FP64 path
    with one slot. Sizes are log-uniform in nmeas (ELT geometry at several grid
    sizes), each request has its own seeded 35-layer profile (exp(-h/5 km) x
    LogNormal(0, 0.2) fractions, r0 0.129 m, L0 25 m) and asks for R, Cvv and
    the PSF on the truth direction."""
    import numpy as np
    import torch
    from moao_b200 import inputs as I
    from moao_b200 import params as P
    import moao_b200 as M
    from moao_b200.serve import Server

    torch.cuda.init()
    rng = np.random.default_rng(2024)
    nssps = [10, 14, 20, 28, 40, 52, 64]
    systems = []
    for nssp in nssps:
        sp, ap = P.config_elt() if nssp == 64 else P.config_scaled(nssp, 35)
        d = tempfile.mkdtemp(prefix=f"moao_serve_{nssp}_")
        P.write_system(d, sp, ap)
        systems.append(dict(nssp=nssp, dir=d, sys=sp))
    n_req = args.serve_requests

    def profile(r):
        h = np.linspace(0.0, 20000.0, 35)
        f = np.exp(-h / 5000.0) * r.lognormal(0.0, 0.2, 35)
        f /= f.sum()
        return f * 0.129 ** (-5.0 / 3.0), h, np.full(35, 25.0)

    def make_server(slots):
        srv = Server(device=0, slots=slots, nb=args.nb or 1024)
        ids, infos = [], []
        for y in systems:
            sf, af = os.path.join(y["dir"], "sys-params.txt"), os.path.join(y["dir"], "prof-1-atmos-night0.txt")
            tm = M.Tomo(sf, af)
            # the PSF tables are synthesised by the library (C++/CUDA) for the truth sensor
            nact, *_ = M.intersample_inputs(tm.info.nssp_ts, tm.info.diam, tm.info.obs, tables=False)
            Dx = I.make_dx(nact, tm.getNMeasTS(), seed=y["nssp"])
            sid = srv.add_system_synth(sf, af, Dx)
            ids.append(sid)
            infos.append(srv.system_info(sid))
        return srv, ids, infos

    # request list: log-uniform nmeas in [1000, 48000], nearest grid size
    srv, ids, infos = make_server(1)
    logn = np.log([i["nmeas"] for i in infos])
    reqs = []
    for k in range(n_req):
        target = rng.uniform(np.log(1000.0), np.log(48000.0))
        j = int(np.argmin(np.abs(logn - target)))
        reqs.append((j, profile(np.random.default_rng(1000 + k))))

    def submit(srv, ids, infos, j, prof, prec):
        i = infos[j]
        R = np.empty(i["nmeas"] * i["nmeasts"])
        Cvv = np.empty(i["nact"] ** 2)
        psf = np.empty(i["psf_n"] ** 2)
        return srv.submit(ids[j], *prof, prec=prec, R=R, Cvv=Cvv, psf=psf)

    def closed_loop(srv, ids, infos, prec, parallel):
        # warm the slots once per system size
        for j in range(len(ids)):
            srv.wait(submit(srv, ids, infos, j, reqs[0][1], prec))
        t0 = time.perf_counter()
        if parallel:
            rid = [submit(srv, ids, infos, j, p, prec) for j, p in reqs]
            res = [srv.wait(r) for r in rid]
        else:
            res = [srv.wait(submit(srv, ids, infos, j, p, prec)) for j, p in reqs]
        wall = time.perf_counter() - t0
        lat = [r["latency_ms"] for r in res]
        assert all(r["status"] == 0 for r in res), [r for r in res if r["status"]][:1]
        return {"requests_per_s": len(res) / wall, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "wall_s": wall}

    base = closed_loop(srv, ids, infos, "fp64", parallel=False)
    srv.close()
    srv, ids, infos = make_server(args.serve_slots)
    sat = closed_loop(srv, ids, infos, "mixed", parallel=True)
    sweep = []
    for frac in (0.5, 0.75, 0.9):
        lam = frac * sat["requests_per_s"]
        arr = np.cumsum(np.random.default_rng(int(frac * 100)).exponential(1.0 / lam, n_req))
        t0 = time.perf_counter()
        rid = []
        for (j, p), ta in zip(reqs, arr):
            dt = ta - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            rid.append(submit(srv, ids, infos, j, p, "mixed"))
        res = [srv.wait(r) for r in rid]
        wall = time.perf_counter() - t0
        lat = [r["latency_ms"] for r in res]
        sweep.append({"rate_requests_per_s": lam, "throughput_requests_per_s": len(res) / wall,
                      "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                      "mean_queue_ms": float(np.mean([r["queue_ms"] for r in res]))})
    st = srv.stats()
    srv.close()
    sustained = max((x for x in sweep if x["throughput_requests_per_s"] >= 0.9 * x["rate_requests_per_s"]),
                    key=lambda x: x["rate_requests_per_s"], default=sweep[0])
    line = {
        "metric": SERVING_METRIC, "value": sustained["throughput_requests_per_s"],
        "unit": "requests/s", "n_gpus": 1, "higher_is_better": True,
        "latency_ms": {"p50": sustained["p50_ms"], "p99": sustained["p99_ms"],
                       "at_rate_requests_per_s": sustained["rate_requests_per_s"]},
        "config": {"workload": (f"{n_req} requests, nmeas log-uniform 1000-48000 over grids "
                                f"{nssps} (ELT geometry), 35-layer seeded profiles, R + Cvv + PSF each"),
                   "slots": args.serve_slots, "path": "mixed", "panel_nb": args.nb or 1024},
        "saturation_closed_loop": sat, "sweep": sweep,
        "baseline_sequential_fp64": base,
        "speedup_vs_sequential_fp64": sat["requests_per_s"] / base["requests_per_s"],
        "server_stats": st, "data": "synthetic",
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- batch
BATCH_METRIC = "batched uneven instances: reconstructor builds/s in one graph launch"


def batch_main(args):
    """256 uneven instances (grids 20x20 to 50x50, 2-8 WFS + truth sensor, 1-20
    layers at U(0, 20 km), Dirichlet(1) fractions, r0 U(0.08, 0.2) m, L0 U(10, 50)
    m, seeded) built in one CUDA graph launch with autotuned panel widths, stream
    count and packed-instance bound (the small instances in the persistent
    tile-task kernel), against the same instances built one after the other
    through the direct API (FP64 path)."""
    import numpy as np
    import torch
    import moao_b200 as M
    from moao_b200 import batch as B
    from moao_b200 import params as P

    torch.cuda.init()
    rng = np.random.default_rng(4096)
    lo, hi = (int(x) for x in args.batch_nssp.split(","))
    tomos = []
    for i in range(args.batch_count):
        sp, ap = P.config_random(rng, nssp_range=(lo, hi))
        d = tempfile.mkdtemp(prefix=f"moao_batch_{i}_")
        P.write_system(d, sp, ap)
        tomos.append(M.Tomo(os.path.join(d, "sys-params.txt"), os.path.join(d, "prof-1-atmos-night0.txt")))
    nmeas = np.array([t.getNMeas() for t in tomos])
    ctx = M.Context(0)
    prec = args.path
    # autotune on one sample per size class present
    classes = {}
    for t in tomos:
        classes.setdefault(int(np.log2(max(t.getNMeas(), 1024) / 1024)), t)
    tune = B.tuning(prec, ctx=ctx) if args.batch_no_tune else \
        B.autotune(list(classes.values()), prec, ctx=ctx)
    outs = [torch.empty(t.getNMeas() * t.getNMeasTS(), dtype=torch.float64, device="cuda")
            for t in tomos] if args.batch_outputs else None
    pm = args.batch_packed
    B.batch_reconstructors(tomos, outs, prec=prec, packed_max=pm, ctx=ctx)  # warm-up
    runs = []
    for _ in range(max(1, args.steps)):
        per, run = B.batch_reconstructors(tomos, outs, prec=prec, packed_max=pm, ctx=ctx)
        runs.append(run)
    ms = float(np.median([r["ms_device"] for r in runs]))
    # sequential direct API on the same instances (FP64, default panel width), device time
    run_last = runs[-1]
    ctx.close()  # frees the batch streams' workspaces before the comparison
    seq_ms = None
    if not args.no_compare:
        ctx2 = M.Context(0)
        ctx2.set_stream(torch.cuda.current_stream().cuda_stream)
        nmax = int(nmeas.max())
        tsmax = max(t.getNMeasTS() for t in tomos)
        Cbuf = torch.empty(nmax * nmax, dtype=torch.float64, device="cuda")
        Tbuf = torch.empty(nmax * tsmax, dtype=torch.float64, device="cuda")

        def one(t):
            nm, nts = t.getNMeas(), t.getNMeasTS()
            C, T = Cbuf[:nm * nm], Tbuf[:nm * nts]
            M.matcov_tile(C, nm, nm, 0, 0, nm, t, 1, ctx=ctx2)
            M.matcov_tile(T, nts, nm, 0, 0, nts, t, 3, ctx=ctx2)
            M.reconstructor(nm, nts, C, nm, T, nts, 1, prec="fp64", ctx=ctx2)
        for t in tomos[:4]:
            one(t)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for t in tomos:
            one(t)
        e1.record()
        torch.cuda.synchronize()
        seq_ms = e0.elapsed_time(e1)
        ctx2.close()
    nts_all = np.array([t.getNMeasTS() for t in tomos], dtype=np.float64)
    n_all = nmeas.astype(np.float64)
    flop = float(np.sum(n_all ** 3 / 3 + 2 * nts_all * n_all ** 2))  # POTRF + 2 TRSM per instance
    line = {
        "metric": BATCH_METRIC, "value": len(tomos) / (ms / 1000.0), "unit": "builds/s",
        "fp64_flop_per_batch": flop, "fp64_equivalent_tflops": flop / (ms * 1e9),
        "n_gpus": 1, "higher_is_better": True, "ms_per_batch": ms,
        "config": {"workload": (f"{len(tomos)} uneven instances: grids {lo}-{hi}, 2-8 WFS, 1-20 layers "
                                f"(nmeas {int(nmeas.min())}-{int(nmeas.max())}, median {int(np.median(nmeas))})"),
                   "path": prec, "streams": run_last["streams_used"]},
        "graph_nodes": run_last["graph_nodes"], "graph_build_ms": run_last["ms_build"],
        "packed": {"count": run_last["packed_count"], "tasks": run_last["packed_tasks"],
                   "nmeas_bound": pm if pm else tune.get("packed_max")},
        "device_gb": run_last["device_gb"], "failed": run_last["failed"], "tuning": tune,
        "sequential_fp64_direct": None if seq_ms is None else {
            "ms": seq_ms, "builds_per_s": len(tomos) / (seq_ms / 1000.0),
            "batch_speedup": seq_ms / ms},
        "data": "synthetic",
    }
    print(json.dumps(line), flush=True)
    return 0


def sharded_main(args):
    """The ELT build (matcov of each rank's panels, FP64 factorisation and both
    solves, R left distributed) with Cmm's column panels spread over the ranks:
    one build per step for the whole job, panels broadcast over NCCL."""
    import numpy as np
    import torch
    import moao_b200 as M
    from moao_b200 import sharded as S
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from moao_b200.replicas import max_over_ranks
    sf, af, sysp, atm = system(args.config)
    t = M.Tomo(sf, af)
    nm, nts = t.getNMeas(), t.getNMeasTS()
    ctx = M.Context(local)
    nb = args.nb or 1024

    def one():
        R, lay, B = S.sharded_reconstructor(t, nb=nb, ctx=ctx, dist=dist, gather=False)
        return B

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        one()
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, "cuda")
    if rank == 0:
        print(json.dumps({
            "metric": "R builds/s, one ELT system sharded over the ranks (FP64)", "value": 1000.0 / ms,
            "unit": "builds/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "dtype": "f64",
            "config": {"workload": workload_name(args.config, nm, nts, atm.nLayer), "panel_nb": nb,
                       "parallelism": f"column panels cyclic over {world} ranks"},
            "data": "synthetic"}), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def probe_main(args):
    """One stage, once, on the ELT geometry scaled to args.nssp subapertures
    across (35 layers; 64 gives the ELT system itself). For profiler captures:
    the ncu commands in profiles/ run this."""
    import numpy as np
    import torch
    import moao_b200 as M
    from moao_b200 import params as P
    from moao_b200 import inputs as I
    sp, ap = P.config_elt() if args.nssp == 64 else P.config_scaled(args.nssp, 35)
    d = tempfile.mkdtemp(prefix="moao_probe_")
    P.write_system(d, sp, ap)
    torch.cuda.set_device(0)
    ctx = M.Context(0)
    if args.tc_pair >= 0:
        ctx.set_tc_pair(args.tc_pair)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.set_block(args.nb or 1024)
    t = M.Tomo(os.path.join(d, "sys-params.txt"), os.path.join(d, "prof-1-atmos-night0.txt"))
    t.setTarget(0)
    nm, nts = t.getNMeas(), t.getNMeasTS()
    Ctm = torch.empty((nm, nts), dtype=torch.float64, device="cuda")
    t0 = time.perf_counter()
    if args.probe == "gemm_tiles":
        # FP64 builds with each tile configuration of the large products: the
        # gemm_f64 family's rate (kernel timing) against cuBLAS DGEMM
        Cmm = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
        peak = fp64_peak_tflops(torch)
        res = []
        for cfg in range(4):
            ctx.set_gemm_tile(cfg)
            rates, builds, leaf_us = [], [], []
            for rep in range(4):
                M.matcov_tile(Cmm, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
                M.matcov_tile(Ctm, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
                torch.cuda.synchronize()
                ctx.set_kernel_timing(True)
                ctx.reset_kernel_stats()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                M.reconstructor(nm, nts, Cmm, nm, Ctm, nts, 1, prec="fp64", ctx=ctx)
                e1.record()
                torch.cuda.synchronize()
                st = ctx.kernel_stats("gemm_f64")
                lf = ctx.kernel_stats("potrf_leaf")
                ctx.set_kernel_timing(False)
                if rep:
                    rates.append(st["work"] / st["ms"] / 1e9)
                    builds.append(e0.elapsed_time(e1))
                    leaf_us.append(1000.0 * lf["ms"] / max(lf["launches"], 1))
            res.append({"cfg": cfg, "gemm_tflops": float(np.median(rates)),
                        "of_cublas": float(np.median(rates)) / peak,
                        "build_ms": float(np.median(builds)),
                        "leaf_us_per_launch": float(np.median(leaf_us))})
        ctx.set_gemm_tile(1)
        print(json.dumps({"probe": "gemm_tiles", "nssp": args.nssp, "nmeas": nm,
                          "cublas_dgemm_tflops": peak, "configs": res}), flush=True)
        return 0
    if args.probe == "matcov_ctm":
        M.matcov_tile(Ctm, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
    else:
        prec = "mixed" if args.probe.endswith("mixed") else "fp64"
        if prec == "mixed":
            ctx.set_offsets_from_tomo(t)
        Cmm = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
        M.matcov_tile(Cmm, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
        M.matcov_tile(Ctm, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
        M.reconstructor(nm, nts, Cmm, nm, Ctm, nts, 1, prec=prec, ctx=ctx)
        if args.probe.startswith("cee"):
            nact = I.make_dm(t.info.nssp_ts, 0.2, t.info.obs).nactu
            Dx = torch.from_numpy(np.ascontiguousarray(I.make_dx(nact, nts).T)).cuda()
            Ctm2 = torch.empty((nm, nts), dtype=torch.float64, device="cuda")
            Ctt = torch.empty((nts, nts), dtype=torch.float64, device="cuda")
            Cee = torch.empty((nts, nts), dtype=torch.float64, device="cuda")
            Cvv = torch.empty((nact, nact), dtype=torch.float64, device="cuda")
            Tmp = torch.empty((nts, nact), dtype=torch.float64, device="cuda")
            M.matcov_tile(Cmm, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
            M.matcov_tile(Ctm2, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
            M.matcov_tile(Ctt, nts, nts, 0, 0, nts, t, 4, ctx=ctx)
            M.Cee_Cvv(nm, nts, nact, Cmm, nm, Ctt, nts, Ctm2, nts, Ctm, nts, Dx, nact, Cee, nts,
                      Cvv, nact, Tmp, nact, prec=prec, ctx=ctx)
    torch.cuda.synchronize()
    print(json.dumps({"probe": args.probe, "nssp": args.nssp, "nmeas": nm, "nmeasts": nts,
                      "wall_s": time.perf_counter() - t0, "launches": ctx.launches}), flush=True)
    return 0


def main():
    args = parse()
    if args.probe:
        return probe_main(args)
    if args.serving:
        return serving_main(args)
    if args.batch:
        return batch_main(args)
    if args.sharded:
        return sharded_main(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    sf, af, sysp, atm = system(args.config)

    if args.impl == "reference":
        if rank != 0:
            return 0
        # sizes from the reference's own Tomo_struct (oracle/_ref): nothing of
        # this repository's library is loaded on this arm
        O = _oracle()
        if O.RefTomo.available():
            ri = O.RefTomo(sf, af).info
            nm, nts = ri.nmeas, ri.nmeasts
        else:
            import moao_b200 as M
            t = M.Tomo(sf, af)
            nm, nts = t.getNMeas(), t.getNMeasTS()
        vals, walls = [], []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            v, info = cpu_reference_sample(sf, af, nm, nts, budget_s=3.0)
            if i >= args.warmup:
                vals.append(v)
                walls.append(time.perf_counter() - t0)
        value = statistics.median(vals)
        pairs = None if args.no_pairs else cpu_reference_pairs()
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
            "extrapolated": True,
            "sample_wall_s_per_step": statistics.median(walls),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded ELT-scale system)",
            "config": {"workload": workload_name(args.config, nm, nts, atm.nLayer),
                       "path": "reference CPU (matcov_tile + LAPACK)", "parallelism": "host cores"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                             "extrapolated": True, "sample": info["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "measured_full_builds": pairs,
            "note": ("value: each step times a bounded sample of the ELT build (Ctm rows through the "
                     "reference's matcov_tile, dpotrf/dtrsm at a reduced size) and extrapolates it to the "
                     "whole build by element and flop counts; measured_full_builds: whole builds of two "
                     "smaller systems, timed end to end"),
        }
        print(json.dumps(line), flush=True)
        return 0

    import numpy as np
    import torch

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    import moao_b200 as M
    from moao_b200.replicas import max_over_ranks

    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = M.Context(dev)
    if args.tc_pair >= 0:
        ctx.set_tc_pair(args.tc_pair)
    ctx.set_stream(stream.cuda_stream)
    nb_main = args.nb or 1024
    ctx.set_block(nb_main)
    t = M.Tomo(sf, af)
    nm, nts = t.getNMeas(), t.getNMeasTS()
    Cmm = torch.empty((nm, nm), dtype=torch.float64, device="cuda")   # column-major nm x nm
    Ctm = torch.empty((nm, nts), dtype=torch.float64, device="cuda")  # column-major nts x nm

    cn2_p = np.array(atm.cn2, dtype=np.float64)
    h_p, L0_p = np.array(atm.h, dtype=np.float64), np.array(atm.L0, dtype=np.float64)

    if args.path == "mixed":
        # defaults of the mixed path; the LGS constant blocks of the covariance
        # model are declared so the factorisation works on Cmm without them
        ctx.set_mixed()
        ctx.set_offsets_from_tomo(t)

    def step(path):
        # every build starts from the turbulence profile: projected geometry,
        # offset tables and both covariance matrices are recomputed
        t.set_profile(cn2_p, h_p, L0_p)
        M.matcov_tile(Cmm, nm, nm, 0, 0, nm, t, 1, ctx=ctx)
        M.matcov_tile(Ctm, nts, nm, 0, 0, nts, t, 3, ctx=ctx)
        return M.reconstructor(nm, nts, Cmm, nm, Ctm, nts, 1, prec=path, ctx=ctx)

    def timed(path, steps, warmup, measure):
        """Device time of `steps` builds after `warmup` untimed ones (CUDA events
        on the launching stream, barriers on both sides)."""
        for _ in range(warmup):
            step(path)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        if measure:
            ctx.reset_kernel_stats()
            ctx.set_kernel_timing(True)
            clocks = Clocks(dev)
            clocks.start()
        launches0 = ctx.launches
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        ev[0].record()
        for k in range(steps):
            step(path)
            ev[k + 1].record()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        out = {"launches": ctx.launches - launches0}
        if measure:
            out["clocks"] = clocks.stop()
            ctx.set_kernel_timing(False)
        out["per_step"] = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
        total = max_over_ranks(ev[0].elapsed_time(ev[-1]), dist, "cuda")
        out["total_ms"] = total
        return out

    main_run = timed(args.path, args.steps, max(3, args.warmup), True)
    total_ms, per_step, launches, clk = (main_run["total_ms"], main_run["per_step"],
                                         main_run["launches"], main_run["clocks"])
    value = world * args.steps / (total_ms / 1000.0)
    stats = {f: ctx.kernel_stats(f) for f in ("gemm_f64", "matcov", "matcov_table", "potrf_leaf",
                                              "tc_split", "tc_int8")}

    # The mixed path is reported beside the FP64 path of the same build: its
    # builds/s in this run and the relative Frobenius error of R between them.
    rel_err, fp64_arm, cee = None, None, None
    if args.path == "mixed":
        R_mixed = Ctm.clone()
        ctx.set_block(args.nb_fp64)
        if args.no_compare:
            step("fp64")
            torch.cuda.synchronize()
        else:
            arm = timed("fp64", args.steps, 1, False)
            v64 = world * args.steps / (arm["total_ms"] / 1000.0)
            fp64_arm = {"value": v64, "unit": UNIT, "ms_per_step": arm["total_ms"] / args.steps,
                        "latency_ms": {"p50": float(np.percentile(arm["per_step"], 50)),
                                       "p99": float(np.percentile(arm["per_step"], 99))},
                        "panel_nb": args.nb_fp64, "mixed_over_fp64": value / v64}
        rel_err = float(torch.linalg.norm(R_mixed - Ctm) / torch.linalg.norm(Ctm))
        # ---- Cee, Cvv and the PSF from both R (Ctm holds the FP64 R now)
        if not args.no_cee:
            cee = cee_stage(M, torch, ctx, t, nm, nts, Cmm, Ctm, R_mixed)
        del R_mixed
        torch.cuda.empty_cache()
        ctx.set_block(nb_main)

    def set_profile():
        t.set_profile(cn2_p, h_p, L0_p)

    geom_bytes = 8 * (2 * atm.nLayer * (nm // 2 + nts // 2) + 5 * (nm // 2 + nts // 2) +
                      sysp.nW * atm.nLayer + 3 * atm.nLayer + sysp.nW)
    # ---- e2e through the drop-in host-buffer entry points of the C ABI
    e2e, e2e_api, e2e_cache = None, None, None
    if not args.no_e2e:
        del Cmm
        torch.cuda.empty_cache()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ksteps = max(1, min(args.steps, args.e2e_steps))
        sec, h2d, d2h, R_dropin = e2e_dropin(M, torch, ctx, t, nm, nts, args.path, ksteps,
                                             set_profile)
        e2e_s = max_over_ranks(sec, dist, "cuda")
        e2e = {"value": world * ksteps / e2e_s, "unit": UNIT, "steps": ksteps,
               "h2d_bytes_per_step": int(h2d + geom_bytes), "d2h_bytes_per_step": int(d2h),
               "path": ("C ABI host-buffer entry points, as the reference's driver calls them: "
                        "moao_matcov_tile_host (Cmm, Ctm) then moao_reconstructor_host; pinned host "
                        "buffers; only the lower part of Cmm crosses PCIe"),
               "rel_fro_R_vs_device_path": float(np.linalg.norm(R_dropin - Ctm.cpu().numpy().T) /
                                                 np.linalg.norm(R_dropin)) if args.path == "fp64"
               else None}
        sec_c, h2d_c, d2h_c, R_cache = e2e_dropin(M, torch, ctx, t, nm, nts, args.path, ksteps,
                                                  set_profile, cache=True)
        e2e_c_s = max_over_ranks(sec_c, dist, "cuda")
        e2e_cache = {"value": world * ksteps / e2e_c_s, "unit": UNIT, "steps": ksteps,
                     "h2d_bytes_per_step": int(h2d_c + geom_bytes), "d2h_bytes_per_step": int(d2h_c),
                     "path": ("as e2e with moao_ctx_set_host_cache on (the caller promises not to "
                              "modify the host Cmm / Ctm between matcov_tile and reconstructor, as "
                              "the reference's driver does): the reconstructor reuses their device "
                              "copies; every output still lands in the host buffers"),
                     "R_equal_to_e2e": bool(np.array_equal(R_cache, R_dropin))}
        del R_dropin, R_cache
        Cmm = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
        # the public device API with the profile set from host memory every step and
        # R read back to pinned memory (the serving loop's flow)
        R_host = torch.empty((nm, nts), dtype=torch.float64, pin_memory=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(ksteps):
            step(args.path)             # host profile -> geometry recomputed and re-uploaded
            R_host.copy_(Ctm, non_blocking=True)
            torch.cuda.synchronize()
        api_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        e2e_api = {"value": world * ksteps / api_s, "unit": UNIT, "steps": ksteps,
                   "h2d_bytes_per_step": int(geom_bytes), "d2h_bytes_per_step": int(nm * nts * 8),
                   "path": "device API: profile from host memory in, R out to pinned memory"}
        del R_host

    # ---- roofline of the dominant kernel family (largest share of device time),
    # and of the largest tensor-core family beside it
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak_src = "of measured" if peaks else "of fallback"

    def roofline_of(fam):
        s = stats[fam]
        if s["ms"] <= 0 or s["launches"] <= 0:
            return None
        share = round(s["ms"] / total_ms, 4)
        if fam == "gemm_f64":
            peak = fp64_peak_tflops(torch)
            achieved = s["work"] / (s["ms"] / 1000.0) / 1e12
            ratio = read_traffic_ratio("gemm_f64_elt.txt")
            return {"kernel": "gemm_f64_kernel (FP64 DMMA m16n8k16)", "bound": "tensor",
                    "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": "TFLOP/s",
                    "frac": round(achieved / peak, 4),
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure in MEASURED_PEAKS.json)",
                    "traffic": (ratio * s["work"] / s["launches"]) if ratio else None,
                    "launches": s["launches"], "share": share}
        if fam in ("tc_split", "tc_int8"):
            # timed inside a seconds-long build: the sustained (power-capped) peak
            bf16 = float(peaks.get("bf16_tflops_sustained", 1400.0))
            peak = bf16 * (2.0 if fam == "tc_int8" else 1.0)
            achieved = s["work"] / (s["ms"] / 1000.0) / 1e12
            what = "int8" if fam == "tc_int8" else "fp16/bf16 split"
            ratio = read_traffic_ratio("tc_gemm_int8_crt_nmeas15936.txt" if fam == "tc_int8"
                                       else "tc_gemm_f16_trailing_nmeas15936.txt")
            return {"kernel": f"tc_gemm_kernel ({what} tcgen05, TMA, TMEM)", "bound": "tensor",
                    "achieved": round(achieved, 3), "peak": round(peak, 3),
                    "unit": "TFLOP/s" if fam == "tc_split" else "TOP/s",
                    "frac": round(achieved / peak, 4),
                    "peak_source": (f"bf16_tflops_sustained {peak_src}" if fam == "tc_split" else
                                    f"2 x bf16_tflops_sustained {peak_src} (the dense int8 rate is "
                                    "twice bf16)"),
                    "traffic": (ratio * s["work"] / s["launches"]) if ratio else None,
                    "launches": s["launches"], "share": share}
        if fam == "matcov":
            # HBM framing (bytes stored); the kernel itself is bound by its FP64 pipe
            hbm = float(peaks.get("hbm_gbs", 6650.0))
            bytes_alg = 8.0 * s["work"]
            achieved = bytes_alg / (s["ms"] / 1000.0) / 1e9
            ratio = read_traffic_ratio("matcov_edge_ctm_nmeas15936.txt")
            pipe = read_traffic_ratio("matcov_edge_ctm_nmeas15936.txt", "fp64_pipe_active")
            return {"kernel": "matcov_edge_kernel + matcov_block_kernel (covariance generation, FP64)",
                    "bound": "hbm",
                    "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                    "frac": round(achieved / hbm, 5), "peak_source": f"hbm_gbs {peak_src}",
                    "traffic": (8.0 * s["work"] / s["launches"]),
                    "traffic_note": ("bytes stored per launch; at ELT size Cmm (18 GB) exceeds L2 so "
                                     "DRAM writes equal them (ncu on a small case: "
                                     f"{ratio} B per element, the rest still in L2)"),
                    "real_bound": "FP64 pipe", "fp64_pipe_active": pipe,
                    "launches": s["launches"], "share": share}
        return {"kernel": fam, "ms": s["ms"], "share": share}

    def roofline_tc_kernel():
        """tc_gemm_kernel as one kernel: its fp16 launches (tc_split) and its int8
        launches (tc_int8) together, in bf16-equivalent flop (an int8 op counts
        half, the dense int8 rate being twice bf16's) against the sustained bf16
        peak; beside it the FP64-equivalent rate: the build's algorithmic FP64
        flop (POTRF nmeas^3/3, the two triangular solves 2 nmeasts nmeas^2, and per
        refinement step the residual and the correction solve, 2 nmeasts nmeas^2
        each) over the kernel's time."""
        a, b = stats["tc_split"], stats["tc_int8"]
        ms = a["ms"] + b["ms"]
        if ms <= 0:
            return None
        bf16 = float(peaks.get("bf16_tflops_sustained", 1400.0))
        achieved = (a["work"] + 0.5 * b["work"]) / (ms / 1000.0) / 1e12
        ra = read_traffic_ratio("tc_gemm_f16_trailing_nmeas15936.txt")
        rb = read_traffic_ratio("tc_gemm_int8_crt_nmeas15936.txt")
        traffic = None
        if ra and rb:
            traffic = (ra * a["work"] + rb * b["work"]) / max(1, a["launches"] + b["launches"])
        refine = 1 if args.path == "mixed" else 0
        fp64_flop = (nm ** 3 / 3.0 + 2.0 * nts * nm * nm * (1 + 2 * refine)) * args.steps
        fp64_equiv = fp64_flop / (ms / 1000.0) / 1e12
        return {"kernel": "tc_gemm_kernel (tcgen05 kind::f16 fp16-split products and kind::i8 exact "
                          "CRT residual products; TMA, TMEM)", "bound": "tensor",
                "achieved": round(achieved, 3), "peak": round(bf16, 3), "unit": "TFLOP/s",
                "frac": round(achieved / bf16, 4),
                "peak_source": (f"bf16_tflops_sustained {peak_src} (the kernel runs inside a "
                                "seconds-long build); int8 ops counted at half weight"),
                "fp64_equivalent_achieved": round(fp64_equiv, 3),
                "frac_fp64_equivalent": round(fp64_equiv / bf16, 4),
                "fp64_equivalent_note": ("algorithmic FP64 flop of the build over this kernel's time: "
                                         "the split products multiply the tensor work (3 fp16 products "
                                         "per update, one int8 product per CRT modulus, 11 at nmeas "
                                         "47,552, per residual)"),
                "traffic": traffic,
                "traffic_note": ("DRAM bytes per launch: each family's bytes per unit of work from its "
                                 "ncu capture in profiles/ (nmeas 15,936) times the work of this run's "
                                 "launches"),
                "launches": a["launches"] + b["launches"], "share": round(ms / total_ms, 4),
                "families": {"tc_split": roofline_of("tc_split"), "tc_int8": roofline_of("tc_int8")}}

    # the dominant kernel by device time: tc_gemm_kernel (both of its families) or a family
    # of another kernel
    tc_ms = stats["tc_split"]["ms"] + stats["tc_int8"]["ms"]
    others = [f for f in stats if f not in ("tc_split", "tc_int8")]
    top_other = max(others, key=lambda f: stats[f]["ms"])
    if tc_ms >= stats[top_other]["ms"]:
        roof, roof_tensor = roofline_tc_kernel(), roofline_of(top_other)
    else:
        roof, roof_tensor = roofline_of(top_other), roofline_tc_kernel()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps,
        "latency_ms": {"p50": float(np.percentile(per_step, 50)), "p99": float(np.percentile(per_step, 99))},
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.path == "fp64" else
                 ("fp16x2 row-scaled split (fp32 accumulate) tensor-core updates + f64 diagonal blocks "
                  "+ exact int8 CRT products for the f64 residual"),
        "data": "synthetic (seeded ELT-scale system; reference parameter-file format)",
        "config": {"workload": workload_name(args.config, nm, nts, atm.nLayer), "path": args.path,
                   "nmeas": nm, "nmeasts": nts, "layers": atm.nLayer, "panel_nb": nb_main,
                   "l2": f"inputs larger than L2 (Cmm {nm * nm * 8 / 1e9:.1f} GB regenerated every step)",
                   "parallelism": f"replicas x{world}"},
        "stages_ms_per_step": {f: stats[f]["ms"] / args.steps for f in stats},
        "rel_fro_err_R_vs_fp64": rel_err,
        "fp64_path": fp64_arm,
        "roofline": roof,
        "roofline_next": roof_tensor,
        "gpu_launches": int(launches),
        "clocks": clk,
        "e2e": e2e,
        "e2e_device_api": e2e_api,
        "e2e_host_cache": e2e_cache,
        "cee_cvv_psf": cee,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, info = cpu_reference_sample(sf, af, nm, nts)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                                "extrapolated": True, "sample": info["sample"]}
    if rank == 0 and world == 1 and not args.no_pairs:
        del Cmm, Ctm
        torch.cuda.empty_cache()
        line["measured_full_builds"] = measured_pairs(M, torch, ctx)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
