"""CPU checks of the oracle and the compiled constants: pinned against the
golden tables parsed from the reference source, code-derived invariants, and
a second independent numpy restatement."""
import ctypes
import json
import os

import numpy as np
import pytest

from oracle import oracle as orc
from oracle.np_oracle import NpLattice
from symmetry_b200 import configs
from symmetry_b200 import lib as symlib
from symmetry_b200.params import config_params

G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_constants.json")))
TABLES = ["cix", "ciy", "ciz", "opc", "symx", "symy", "symz"]


def test_oracle_moment_matrix_matches_data_statement():
    o = orc.Oracle(config_params(4, 4, 4))
    M, Mi = o.matrices()
    assert (M == np.array(G["M"], dtype=float)).all()
    assert np.abs(M @ Mi - np.eye(19)).max() < 1e-15
    Mg = np.array(G["M"], dtype=float)
    assert np.array_equal(Mi, (Mg / (Mg * Mg).sum(1, keepdims=True)).T)


def test_oracle_and_library_tables_match_reference():
    t = np.zeros(7 * 19, dtype=np.int32); w = np.zeros(19)
    orc.lib().orc_tables(t.ctypes.data_as(ctypes.c_void_p), w.ctypes.data_as(ctypes.c_void_p))
    tl = np.zeros(7 * 19, dtype=np.int32); wl = np.zeros(19); ml = np.zeros(361)
    symlib.lib().sym_lattice_tables(tl.ctypes.data_as(ctypes.c_void_p), wl.ctypes.data_as(ctypes.c_void_p),
                                    ml.ctypes.data_as(ctypes.c_void_p))
    for k, name in enumerate(TABLES):
        assert list(t[19 * k:19 * k + 19]) == G[name], name
        assert list(tl[19 * k:19 * k + 19]) == G[name], name
    assert np.array_equal(w, np.array(G["wi"])) and np.array_equal(wl, np.array(G["wi"]))
    assert np.array_equal(ml.reshape(19, 19), np.array(G["M"], dtype=float))


def test_mass_conserved_per_colour():
    w = configs.c1_thread(nx=16, ny=16, nz=32, radius=4.0)
    o = orc.setup_workload(w)
    m0 = o.arr("ri").sum(), o.arr("bi").sum()
    o.step(100)
    m1 = o.arr("ri").sum(), o.arr("bi").sum()
    assert abs(m1[0] - m0[0]) <= 1e-13 * m0[0] and abs(m1[1] - m0[1]) <= 1e-13 * m0[1]


def test_uniform_phase_at_rest_is_fixed_point():
    p = config_params(8, 8, 8, tau_r=0.9)
    o = orc.Oracle(p)
    o.call("set_walls")
    o.init_phase(np.ones((8, 8, 8)), np.ones((8, 8, 8)))
    o.call("derivatives")
    r0 = o.arr("ri").copy()
    o.step(20)
    assert np.abs(o.arr("ri") - r0).max() < 1e-15
    assert np.abs(o.arr("bi")).max() == 0.0


def test_mirror_symmetric_thread_stays_symmetric():
    w = configs.c1_thread(nx=16, ny=16, nz=32, radius=4.0)
    w.gen["noise"] = 0.0
    o = orc.setup_workload(w)
    o.step(50)
    o.call("calmacros")
    phi = o.arr("rho_N")
    assert np.abs(phi - phi[::-1, :, :]).max() < 1e-12
    assert np.abs(phi - phi.transpose(1, 0, 2)).max() < 1e-12


@pytest.mark.parametrize("walls", [False, True])
def test_numpy_restatement_agrees(walls):
    if walls:
        w = configs.c2_wall_particle(nx=12, ny=10, nz=24, z0=6.0, z1=15.0)
        w.params.par = 0
        w.particles = []
    else:
        w = configs.c1_thread(nx=12, ny=12, nz=24, radius=3.5)
    phi, rho = w.phase()
    o = orc.setup_workload(w)
    n = NpLattice(w.params, phi, rho)
    for _ in range(20):
        o.step(1)
        n.step(1)
    o.call("calmacros")
    n.calmacros()
    fluid = o.arr("walls_all") == 0
    for a, b in [(n.rhoN, o.arr("rho_N")), (n.u[2], o.arr("uz")), (n.u[0], o.arr("ux")), (n.rho, o.arr("rho"))]:
        err = np.abs(np.where(fluid, a - b, 0)).max() / max(np.abs(b).max(), 1e-30)
        assert err < 1e-12, err
