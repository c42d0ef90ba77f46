"""The continuous-batching job server (sym_server_*).

A job's result must be the one it gets alone: jobs that arrive while others
run are admitted into the running batch, and each job's steps, stop-rule
readings and breakup step equal those of the same job served by itself
(bit for bit: a batch step equals a single-domain step, and checks fall on
the job's own multiples of check_every).  The server's stop rule is checked
against an independent reading through the per-handle entry points, and
admission against the footprint budget and the slot count.
"""
import math

import numpy as np
import pytest

from symmetry_b200 import configs
from symmetry_b200.lib import (DEV_TIMEOUT, Lattice, Server, footprint, job_spec, selftest_wait_timeout,
                              setup_workload)

pytestmark = pytest.mark.gpu


def small_jobs(storage):
    """Three uneven jobs: a periodic thread, a thread with a sphere, one with walls."""
    a = configs.c1_thread(nx=20, ny=20, nz=48, radius=4.0, storage=storage)
    rng = np.random.default_rng(11)
    b = configs._c4_domain(rng, "sphere", 77, storage, 0)
    while not b.params.par:
        b = configs._c4_domain(rng, "sphere", 77, storage, 0)
    b.params.nz = min(b.params.nz, 64)
    b.gen["wavelength"] = float(b.params.nz)
    b.particles[0]["center"][2] = b.params.nz / 2.0
    c = configs._c4_domain(np.random.default_rng(3), "walls", 78, storage, 0, wall_cita_deg=120.0)
    c.params.nz = min(c.params.nz, 64)
    c.gen["wavelength"] = float(c.params.nz)
    if c.params.par:
        c.particles[0]["center"][2] = c.params.nz / 2.0
    return [a, b, c]


def serve_alone(w, steps):
    S = Server(slots=4, check_every=10)
    i = S.submit(job_spec(w, steps))
    S.run_until_idle()
    r = S.result(i)
    S.close()
    return r


@pytest.mark.parametrize("storage", ["fp64", "fp16"])
def test_job_result_same_alone_and_in_mix(storage):
    ws = small_jobs(storage)
    limits = [60, 45, 70]
    S = Server(slots=8, check_every=10)
    ids = [S.submit(job_spec(ws[0], limits[0]))]
    S.tick()
    S.tick()   # job 0 runs; the others arrive while it is on the device
    ids.append(S.submit(job_spec(ws[1], limits[1])))
    S.tick()
    ids.append(S.submit(job_spec(ws[2], limits[2])))
    S.run_until_idle()
    mixed = [S.result(i) for i in ids]
    st = S.stats()
    S.close()
    assert st["done"] == 3 and st["failed"] == 0
    # the later jobs were admitted while job 0 was running
    assert mixed[1].t_admit < mixed[0].t_done and mixed[2].t_admit < mixed[0].t_done
    for w, n, m in zip(ws, limits, mixed):
        a = serve_alone(w, n)
        assert m.status == a.status == 3 and m.steps == a.steps == n, (w.name, m.as_dict(), a.as_dict())
        assert m.rmin == a.rmin, (w.name, m.rmin, a.rmin)
        assert m.node_updates == w.nodes * n


def test_breakup_detection_matches_independent_reading():
    """Thin viscous thread that breaks within a few thousand steps; the
    server's interpolated breakup step equals the one computed from readings
    through sym_neck_radius every 10 steps on a handle stepped alone."""
    w = configs.c1_thread(nx=24, ny=24, nz=64, radius=3.2, storage="fp64")
    w.params.sigma = 2e-2
    w.gen["wavelength"] = 32.0
    w.gen["amp"] = 0.1
    limit = 6000
    r = serve_alone(w, limit)
    assert r.status == 2, r.as_dict()
    # independent: step 10 at a time, read the neck through the handle
    L = setup_workload(w)
    prev_s, prev_r = 0, L.neck_radius()   # the initial phase field
    t_b = None
    for k in range(1, limit // 10 + 1):
        L.step(10)
        _ = L.get("rho_N")        # export: the reading below reduces the canonical rho_N
        rr = L.neck_radius()      # exported phi: the state after 10k-1 steps
        s = 10 * k - 1
        if rr < 1.0:
            f = (prev_r - 1.0) / (prev_r - rr)
            t_b = prev_s + f * (s - prev_s)
            break
        prev_s, prev_r = s, rr
    assert t_b is not None
    assert abs(r.breakup_step - t_b) <= 1e-6 * t_b, (r.breakup_step, t_b)
    assert r.steps == 10 * k


def test_admission_by_budget_and_slots():
    ws = small_jobs("fp16")[:1] * 3
    f = footprint(ws[0].params)
    # room for two jobs: the third waits until one retires (first come first served)
    S = Server(budget_bytes=2 * f + f // 2, slots=8, check_every=10)
    ids = [S.submit(job_spec(w, 30 + 10 * k)) for k, w in enumerate(ws)]
    r, p = S.tick()
    assert (r, p) == (2, 1)
    S.run_until_idle()
    res = [S.result(i) for i in ids]
    assert all(x.status == 3 for x in res)
    assert res[2].t_admit >= res[0].t_done
    S.close()
    # one slot: strictly one job after another
    S = Server(slots=1, check_every=10)
    ids = [S.submit(job_spec(w, 20)) for w in ws]
    r, p = S.tick()
    assert (r, p) == (1, 2)
    S.run_until_idle()
    res = [S.result(i) for i in ids]
    assert res[1].t_admit >= res[0].t_done and res[2].t_admit >= res[1].t_done
    S.close()


def test_oversized_job_fails_and_bad_specs_are_refused():
    w = configs.c1_thread(nx=16, ny=16, nz=32, radius=4.0, storage="fp16")
    S = Server(budget_bytes=footprint(w.params) // 2, slots=2)
    i = S.submit(job_spec(w, 10))
    S.run_until_idle()
    r = S.result(i)
    assert r.status == 4 and r.error == 2     # SYM_ERR_OOM: can never fit the budget
    bad = job_spec(w, 0)
    with pytest.raises(Exception):
        S.submit(bad)
    S.close()


def test_unstable_job_fails_with_nan():
    """A served job whose state diverges is retired as failed (SYM_ERR_NAN)
    and the server keeps serving the others.  The diverging job is one of the
    served stream: a light sphere of radius 2.1 on the thread axis at
    tau = 0.61 (c5_0090), whose lateral velocity grows exponentially until the
    coupling explodes near step 120 -- the CPU oracle of the reference
    algorithm diverges the same way."""
    jobs = {j.workload.name: j.workload for j in configs.c5_jobs(duration=5.0, storage="fp64")}
    w = jobs["c5_0090"]
    ok = configs.c1_thread(nx=16, ny=16, nz=32, radius=4.0, storage="fp64")
    S = Server(slots=4, check_every=10)
    i = S.submit(job_spec(w, 300))
    j = S.submit(job_spec(ok, 100))
    S.run_until_idle()
    r, q = S.result(i), S.result(j)
    assert r.status == 4 and r.error == 4, r.as_dict()
    assert 100 <= r.steps <= 300
    assert q.status == 3 and math.isfinite(q.rmin)
    S.close()


def test_drift_and_wall_budget_retire_jobs():
    """Failure detection beyond non-finite readings: a red-volume drift over the
    job's tolerance retires it with SYM_ERR_DRIFT, a resident time over its
    wall budget with SYM_ERR_TIMEOUT; a job without limits runs to its step cap
    beside them."""
    w = configs.c1_thread(nx=20, ny=20, nz=48, radius=4.0)
    S = Server(slots=4, check_every=10)
    a = S.submit(job_spec(w, 60, drift_tol=1e-14))
    b = S.submit(job_spec(w, 60, wall_budget_s=1e-9))
    c = S.submit(job_spec(w, 60))
    S.run_until_idle()
    ra, rb, rc = S.result(a), S.result(b), S.result(c)
    S.close()
    assert ra.status == 4 and ra.error == 9, ra.as_dict()
    assert rb.status == 4 and rb.error == 5, rb.as_dict()
    assert rc.status == 3 and rc.steps == 60, rc.as_dict()


def test_bounded_tile_wait_times_out():
    """The bounded mbarrier wait of the fused kernels' tile loads gives up on a
    barrier that nothing arrives on and reports the timeout flag instead of
    hanging; a completed barrier is seen at once.  The full poll limit of the
    kernels (2^22 polls) must end within seconds.  A run without faults
    records no flag."""
    f1, ms1 = selftest_wait_timeout(256)
    f2, ms2 = selftest_wait_timeout(4096)
    assert f1 == DEV_TIMEOUT and f2 == DEV_TIMEOUT, (f1, f2)
    per_poll_ms = max(ms2 - ms1, 1e-6) / (4096 - 256)
    assert per_poll_ms * 2 ** 22 < 30_000.0, per_poll_ms
    L = setup_workload(configs.c1_thread(nx=16, ny=16, nz=32, radius=4.0, storage="fp64"))
    L.step(20)
    assert L.device_status() == 0
