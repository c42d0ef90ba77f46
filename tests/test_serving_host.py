"""Host-side pieces of serving: the job structs match the C header layout and
the served-job stream is a frozen function of its seed."""
import ctypes

import numpy as np

from symmetry_b200 import configs
from symmetry_b200.lib import job_spec
from symmetry_b200.params import SymJobResult, SymJobSpec, SymParams


def test_job_struct_layout():
    # sym_job_spec: sym_params + 2 int32 + 5 doubles + uint64 + 10 doubles
    assert ctypes.sizeof(SymJobSpec) == ctypes.sizeof(SymParams) + 2 * 4 + 5 * 8 + 8 + 10 * 8
    # sym_job_result: 4 int32 + 5 doubles + int64
    assert ctypes.sizeof(SymJobResult) == 4 * 4 + 5 * 8 + 8


def test_served_stream_is_frozen_and_matches_its_distribution():
    a = configs.c5_jobs(duration=30.0)
    b = configs.c5_jobs(duration=30.0)
    assert [j.t_arrival for j in a] == [j.t_arrival for j in b]
    assert [j.workload.params.nz for j in a] == [j.workload.params.nz for j in b]
    n = len(a)
    assert 480 <= n <= 720                      # Poisson(600)
    t = np.array([j.t_arrival for j in a])
    assert np.all(np.diff(t) > 0) and t[-1] < 30.0
    big = [j for j in a if j.workload.params.nx == 128]
    assert 0.05 < len(big) / n < 0.15
    walls = [j for j in a if j.cita_deg is not None]
    assert 0.24 < len(walls) / n < 0.36
    assert all(30.0 <= j.cita_deg <= 150.0 and j.workload.params.wall_x == 1 for j in walls)
    for j in a:
        p = j.workload.params
        assert p.nx == p.ny and (p.nx == 128 or 24 <= p.nx <= 64)
        assert j.workload.gen["seed"] >= 1005000


def test_job_spec_carries_the_workload():
    w = [j.workload for j in configs.c5_jobs(duration=5.0) if j.workload.params.par][0]
    s = job_spec(w, 300, 1.0, 2.5)
    assert s.max_steps == 300 and s.kind == 0 and s.t_arrival == 2.5
    assert s.gen[0] == w.gen["radius"] and s.gen[2] == w.gen["wavelength"] and s.seed == w.gen["seed"]
    assert list(s.center) == w.particles[0]["center"]
    assert s.p.nx == w.params.nx and s.p.par == 1


def test_batched_mix_manifest_is_unchanged():
    ws = configs.c4_manifest()
    assert len(ws) == 96 and sum(w.nodes for w in ws) == 45025781
    assert sum(1 for w in ws if w.params.par) == 48
