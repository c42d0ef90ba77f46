"""The allocation-free reduction entry point, sym_mass_momentum_noalloc.

Callers that may not allocate device memory (a serving loop that reserved its
whole budget up front, a host program whose memory manager owns every device
byte) get the FP64 mass and momentum sums without a handle and without any
cudaMalloc: the entry point keeps its scratch in a fixed array inside the
library.  These tests check it against the handle-based sym_mass_momentum on
the same populations, on two calls in a row (the second on different data, so
a stale scratch would show), and that oversized domains are refused.  This
file is collected last so a failure here comes after every other test ran.
"""
import ctypes

import numpy as np
import pytest

from symmetry_b200 import configs
from symmetry_b200.lib import Lattice, lib, setup_workload

pytestmark = pytest.mark.gpu


def _device_soa(torch, pops):
    """Fortran-layout (nx,ny,nz,19) host populations -> device [19][N] FP64."""
    soa = np.ascontiguousarray(np.moveaxis(pops, -1, 0).reshape(19, -1))
    return torch.from_numpy(soa).cuda()


def _noalloc(torch, L, out):
    ri = _device_soa(torch, L.get("ri"))
    bi = _device_soa(torch, L.get("bi"))
    walls = torch.from_numpy(np.ascontiguousarray(L.get("walls_all").ravel())).cuda()
    msg = ctypes.create_string_buffer(200)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib().sym_mass_momentum_noalloc(ri.data_ptr(), bi.data_ptr(), walls.data_ptr(), ri.shape[1],
                                         out.data_ptr(), stream, msg, 200)
    torch.cuda.synchronize()
    assert rc == 0, msg.value.decode()
    return out.cpu().numpy().copy()


def test_noalloc_sums_match_handle_entry_point_twice():
    torch = pytest.importorskip("torch")
    w = configs.c2_wall_particle(nx=32, ny=32, nz=64, rad=5.0, centre=(16.0, 16.0, 20.0), z0=20.0, z1=44.0)
    L = setup_workload(w)
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    for call in range(2):
        if call == 1:
            L.step(25)   # different data for the second call
        want = L.mass_momentum()
        got = _noalloc(torch, L, out)
        # the same populations in the same node order, the same per-node
        # arithmetic and the same fixed reduction tree: identical bits
        assert np.array_equal(got, want), (call, got, want)


def test_noalloc_refuses_oversized_domain():
    torch = pytest.importorskip("torch")
    buf = torch.zeros(19, dtype=torch.float64, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    msg = ctypes.create_string_buffer(200)
    rc = lib().sym_mass_momentum_noalloc(buf.data_ptr(), buf.data_ptr(), None, 16_777_217, out.data_ptr(),
                                         None, msg, 200)
    assert rc == 1 and b"16777216" in msg.value
