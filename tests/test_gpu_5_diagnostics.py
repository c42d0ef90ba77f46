"""Checkpoint/restart of the stepping state.

A run that is checkpointed, torn down and resumed in a new handle must end
bit for bit where the uninterrupted run ends: in the fused state (FP64 and
16-bit storage, with walls and a moving particle) and in the canonical state
(the reference geometry stepped by the reference-structured kernels).
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
