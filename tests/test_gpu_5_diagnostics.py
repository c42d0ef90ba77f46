"""Checkpoint/restart of the stepping state, and the diagnostics of the
reference's output steps.

A run that is checkpointed, torn down and resumed in a new handle must end
bit for bit where the uninterrupted run ends: in the fused state (FP64 and
16-bit storage, with walls and a moving particle) and in the canonical state
(the reference geometry stepped by the reference-structured kernels).  The
energy sums of output4 and the field dump of output_results are compared with
the oracle; the particle, energy and neck logs with the values they record.
"""
import numpy as np
import pytest

from symmetry_b200 import configs, params
from symmetry_b200.lib import Lattice, SymError, setup_workload
from symmetry_b200.params import particles_get

pytestmark = pytest.mark.gpu


def particle_state(L):
    s = L.particles()
    return np.array([particles_get(s, k, L.p.par) for k in ("center", "up", "rp")]) if L.p.par else None


@pytest.mark.parametrize("storage", ["fp64", "fp16"])
def test_checkpoint_resume_is_bit_exact_fused(storage, tmp_path):
    w = configs.c2_wall_particle(nx=24, ny=24, nz=48, rad=4.0, centre=(12.0, 12.0, 16.0), z0=16.0, z1=32.0)
    w.params.storage = {"fp64": 0, "fp16": 2}[storage]
    a = setup_workload(w)
    a.step(40)
    b = setup_workload(w)
    b.step(25)
    path = str(tmp_path / "ck.bin")
    b.save(path)
    b.close()
    c = setup_workload(w)
    c.step(3)   # its own state is replaced by the checkpoint
    c.load(path)
    c.step(15)
    assert np.array_equal(a.get("ri"), c.get("ri")) and np.array_equal(a.get("bi"), c.get("bi"))
    assert np.array_equal(a.get("walls_all"), c.get("walls_all"))
    assert np.array_equal(particle_state(a), particle_state(c))


def test_checkpoint_resume_is_bit_exact_canonical(tmp_path):
    p = params.reference_params(48, 88, 48)
    def fresh():
        L = Lattice(p)
        L.initia_center()
        L.call("set_walls")
        L.initialization()
        L.call("derivatives")
        return L
    a = fresh()
    a.step(12)
    b = fresh()
    b.step(5)
    path = str(tmp_path / "ck_ref.bin")
    b.save(path)
    c = Lattice(p)
    c.load(path)
    c.step(7)
    for f in ("ri", "bi", "rho_N", "walls_all"):
        assert np.array_equal(a.get(f), c.get(f)), f
    assert np.array_equal(particle_state(a), particle_state(c))


def test_checkpoint_refuses_other_parameters(tmp_path):
    w = configs.c1_thread(nx=16, ny=16, nz=32, radius=4.0)
    a = setup_workload(w)
    a.step(2)
    path = str(tmp_path / "ck1.bin")
    a.save(path)
    w2 = configs.c1_thread(nx=16, ny=16, nz=48, radius=4.0)
    c = setup_workload(w2)
    with pytest.raises(SymError):
        c.load(path)


# ---- diagnostics of the reference's output steps (Source1.f90:218-234) ----------

def _c2_small(storage="fp64"):
    w = configs.c2_wall_particle(nx=24, ny=24, nz=48, rad=4.0, centre=(12.0, 12.0, 16.0), z0=16.0, z1=32.0)
    w.params.storage = {"fp64": 0, "fp16": 2}[storage]
    return w


def test_energy_sums_match_oracle():
    """output4's field sums (typos fixed) and particle terms against the oracle."""
    from oracle.oracle import setup_workload as orc_setup
    w = _c2_small()
    L = setup_workload(w)
    o = orc_setup(w)
    L.step(30)
    o.step(30)
    o.call("calmacros")
    e = L.energy()
    ref = o.energy()
    assert abs(e[0] - ref[0]) <= 1e-10 * max(abs(ref[0]), 1e-30), (e, ref)
    assert abs(e[1] - ref[1]) <= 1e-10 * max(abs(ref[1]), 1e-30), (e, ref)
    assert e[2] == ref[2], (e, ref)
    s = o.particles
    p = w.params
    up = np.array(particles_get(s, "up", 1))[0]
    rp = np.array(particles_get(s, "rp", 1))[0]
    ten = np.array(particles_get(s, "tension", 1))[0]
    tt = np.array(particles_get(s, "tension_t", 1))[0]
    emp = 0.5 * p.mass * up @ up + 0.5 * p.inertia * rp @ rp
    assert p.mass > 0 and abs(e[3] - emp) <= 1e-9 * max(abs(emp), 1e-30)
    assert abs(e[4] - (ten @ up + tt @ rp)) <= 1e-9 * max(abs(ten @ up + tt @ rp), 1e-20)
    assert abs(e[5] - s.shb[0]) <= 1e-9 * max(abs(s.shb[0]), 1e-30)


def test_output_results_file_matches_oracle_fields(tmp_path):
    """The Tecplot field dump of output_results: header, point order (x fastest,
    1-based) and F12.8 values of calmacros against the oracle's."""
    from oracle.oracle import setup_workload as orc_setup
    w = _c2_small()
    L = setup_workload(w)
    o = orc_setup(w)
    L.step(20)
    o.step(20)
    o.call("calmacros")
    path = str(tmp_path / "OUT_20.dat")
    L.output_results(path)
    lines = open(path).read().splitlines()
    assert lines[0].strip() == 'TITLE="Contact_Angles"'
    assert lines[1].strip() == "VARIABLES=X,Y,Z,WALL,RHO_N,U,V,W,RHO"
    zone = lines[2].split()
    assert zone[:2] == ["ZONE", "F=POINT"] and int(zone[3]) == 24 and int(zone[5]) == 24 and int(zone[7]) == 48
    data = np.loadtxt(lines[3:])
    nx, ny, nz = 24, 24, 48
    assert data.shape == (nx * ny * nz, 9)
    x, y, z = (data[:, k].astype(int) - 1 for k in range(3))
    assert x[1] == 1 and y[nx] == 1 and z[nx * ny] == 1   # x fastest, then y, then z
    wa = o.arr("walls_all")[x, y, z]
    assert np.array_equal(data[:, 3].astype(int), wa)
    for col, name in zip(range(4, 9), ("rho_N", "ux", "uy", "uz", "rho")):
        ref = o.arr(name)[x, y, z]
        assert np.abs(data[:, col] - ref).max() <= 1.1e-8, name


def test_particle_energy_and_neck_logs(tmp_path):
    w = _c2_small()
    L = setup_workload(w)
    prefix = str(tmp_path) + "/"
    wcap = 0.0
    for t in (0, 10, 20):
        if t:
            L.step(10)
        L.output_result2(prefix, t, 100.0)
        wcap = L.output4(str(tmp_path / "Energy.dat"), t, 100.0, 8.0, wcap)
    plog = open(prefix + "P_1.dat").read().splitlines()
    assert plog[0].strip().startswith("VARIABLES=t,t*,cx,cy,cz") and len(plog) == 4
    last = np.array(plog[-1].split(), dtype=float)
    s = L.particles()
    assert int(last[0]) == 20 and abs(last[1] - 0.2) < 1e-12
    assert np.allclose(last[2:5], np.array(particles_get(s, "center", 1))[0], atol=1e-6)
    assert np.allclose(last[5:8], np.array(particles_get(s, "up", 1))[0], atol=1e-6)
    elog = open(tmp_path / "Energy.dat").read().splitlines()
    assert elog[0].strip() == "VARIABLES=t,t*,Esur,Shb,Efree,Emov,Wcap,Emov_p,Esum" and len(elog) == 4
    assert all(np.isfinite(np.array(r.split(), dtype=float)).all() for r in elog[1:])


def test_neck_log_reference_geometry(tmp_path):
    p = params.reference_params(48, 88, 48)
    L = Lattice(p)
    L.initia_center()
    L.call("set_walls")
    L.initialization()
    L.call("derivatives")
    L.call("calmacros")
    L.output3_write(str(tmp_path / "hmin.dat"), 0, 164.3, 30.0, 172.0)
    h0, y0 = L.output3()
    rows = open(tmp_path / "hmin.dat").read().splitlines()
    assert rows[0].strip() == "VARIABLES=t,t*,h,y0"
    v = np.array(rows[1].split(), dtype=float)
    assert int(v[0]) == 0 and abs(v[2] - h0 / 30.0) < 1e-6 and abs(v[3] - y0 / 172.0) < 1e-6


@pytest.mark.parametrize("storage", ["fp64", "fp16"])
def test_get_macros_fused_and_exported_agree(storage):
    """sym_get_macros reads the fused populations while they are current and
    the canonical ones after an export; on a periodic handle without
    particles the canonical path allocates its calmacros arrays on first use.
    Both readings of the same state agree (FP64 export is exact; the 16-bit
    decode is the same function in both)."""
    w = configs.c1_thread(nx=16, ny=16, nz=32, radius=4.0, storage=storage)
    L = setup_workload(w)
    m0 = L.macros()                      # before any step: canonical path
    assert np.isfinite(m0["rho"]).all()
    L.step(12)
    fused = {k: v.copy() for k, v in L.macros().items()}
    L.mass_momentum()                    # exports: the canonical arrays become current
    exported = L.macros()
    for k in ("rho", "ux", "uy", "uz", "rho_N"):
        a, b = exported[k], fused[k]
        assert np.abs(a - b).max() <= 1e-13 * max(1.0, np.abs(b).max()), k
    L.close()
