"""Serving loop scheduling on the host (dry-run slots: same footprints and
admission as on a GPU, each request waits its dry_run_ms instead of computing):
continuous batching, HBM-budget admission, arrival order, cancellation and the
error contract."""
import time

import numpy as np
import pytest

import systems
import moao_b200 as M
from moao_b200.serve import BUSY, CANCELLED, Server

PROF = (np.array([0.7, 0.3]), np.array([0.0, 8000.0]), np.array([25.0, 25.0]))


def add(srv, name):
    return srv.add_system(*systems.files(name))


def footprint_gb(name, prec="fp64"):
    with Server(slots=1, hbm_budget_gb=1000.0, dry_run=True) as srv:
        sid = add(srv, name)
        r = srv.wait(srv.submit(sid, *PROF, prec=prec, dry_run_ms=1))
        return r["footprint_gb"]


def test_footprint_grows_with_size_and_precision(built):
    small, big = footprint_gb("small"), footprint_gb("elt16")
    assert 0 < small < big
    assert footprint_gb("elt16", "mixed") > big


def test_continuous_batching(built):
    """A request queued behind two running ones starts when the shorter one ends,
    not when both have drained."""
    with Server(slots=2, hbm_budget_gb=100.0, dry_run=True) as srv:
        sid = add(srv, "small")
        a = srv.submit(sid, *PROF, dry_run_ms=400)
        b = srv.submit(sid, *PROF, dry_run_ms=60)
        c = srv.submit(sid, *PROF, dry_run_ms=60)
        ra, rb, rc = srv.wait(a), srv.wait(b), srv.wait(c)
        assert all(r["status"] == 0 for r in (ra, rb, rc))
        assert rc["slot"] == rb["slot"] != ra["slot"]
        assert rc["queue_ms"] < ra["latency_ms"] - 150, (rc, ra)
        assert srv.stats()["max_in_flight"] == 2


def test_admission_respects_hbm_budget(built):
    f = footprint_gb("elt16")
    with Server(slots=4, hbm_budget_gb=2.5 * f, dry_run=True) as srv:
        sid = add(srv, "elt16")
        t0 = time.perf_counter()
        ids = [srv.submit(sid, *PROF, dry_run_ms=80) for _ in range(6)]
        res = [srv.wait(i) for i in ids]
        wall = time.perf_counter() - t0
        st = srv.stats()
        assert all(r["status"] == 0 for r in res)
        assert st["max_in_flight"] == 2            # a third would exceed the budget
        assert st["peak_admitted_gb"] <= st["budget_gb"] + 1e-9
        assert wall >= 3 * 0.08 * 0.95               # three waves of two


def test_arrival_order_is_kept(built):
    """The queue head is never bypassed: a small request behind a large one that
    does not fit yet waits for it."""
    fb = footprint_gb("elt16")
    with Server(slots=3, hbm_budget_gb=1.5 * fb, dry_run=True) as srv:
        big, small = add(srv, "elt16"), add(srv, "small")
        b1 = srv.submit(big, *PROF, dry_run_ms=250)
        time.sleep(0.02)
        b2 = srv.submit(big, *PROF, dry_run_ms=50)
        s1 = srv.submit(small, *PROF, dry_run_ms=10)
        r1, r2, r3 = srv.wait(b1), srv.wait(b2), srv.wait(s1)
        assert r2["start_ms"] >= r1["end_ms"] - 1.0            # b2 waited for b1's memory
        assert r3["start_ms"] >= r2["start_ms"]                # s1 started no earlier than b2


def test_cancel_and_error_contract(built):
    f = footprint_gb("small")
    with Server(slots=1, hbm_budget_gb=100 * f, queue_capacity=2, dry_run=True) as srv:
        sid = add(srv, "small")
        running = srv.submit(sid, *PROF, dry_run_ms=300)
        queued = srv.submit(sid, *PROF, dry_run_ms=10)
        time.sleep(0.05)
        assert srv.poll(queued)["status"] == BUSY
        srv.cancel(queued)
        assert srv.poll(queued)["status"] == CANCELLED
        with pytest.raises(M.MoaoError) as e:
            srv.cancel(running)                      # already started
        assert e.value.name == "MOAO_ERR_BUSY"
        with pytest.raises(M.MoaoError) as e:
            srv.wait(running, timeout=0.01)
        assert e.value.name == "MOAO_ERR_TIMEOUT"
        more = [srv.submit(sid, *PROF, dry_run_ms=10) for _ in range(2)]
        with pytest.raises(M.MoaoError) as e:
            srv.submit(sid, *PROF, dry_run_ms=10)      # queue of 2 is full
        assert e.value.name == "MOAO_ERR_BUSY"
        assert srv.wait(running)["status"] == 0
        for i in more:
            assert srv.wait(i)["status"] == 0
        with pytest.raises(M.MoaoError) as e:
            srv.submit(7, *PROF)
        assert e.value.name == "MOAO_ERR_BAD_ARG"
        with pytest.raises(M.MoaoError) as e:
            srv.submit(sid, *PROF, Cvv=np.zeros(10))   # system registered without Dx
        assert e.value.name == "MOAO_ERR_BAD_ARG"
    with Server(slots=1, hbm_budget_gb=0.5 * f, dry_run=True) as srv:
        sid = add(srv, "small")
        with pytest.raises(M.MoaoError) as e:
            srv.submit(sid, *PROF)
        assert e.value.name == "MOAO_ERR_OOM"
        assert srv.stats()["rejected"] == 1


def test_system_with_synthesised_psf_tables(built):
    """A system registered with moao_server_add_system_synth carries PSF tables
    built by the library for its truth sensor; Dx must have the synthesised DM's
    actuator count (dry run: idx synthesised, no GPU)."""
    t = M.Tomo(*systems.files("small"))
    na, N, _, _, _ = M.intersample_inputs(t.info.nssp_ts, t.info.diam, t.info.obs, tables=False)
    Dx = np.zeros((na, t.getNMeasTS()), order="F")
    with Server(slots=1, hbm_budget_gb=100.0, dry_run=True) as srv:
        sid = srv.add_system_synth(*systems.files("small"), Dx)
        info = srv.system_info(sid)
        assert info["nact"] == na and info["psf_n"] == N
        with pytest.raises(M.MoaoError) as e:
            srv.add_system_synth(*systems.files("small"), Dx[:-1])
        assert e.value.name == "MOAO_ERR_BAD_ARG" and str(na) in str(e.value)
