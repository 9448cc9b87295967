"""emu_deposit_noalloc: the deposit for host programs that cannot let a
library allocate device memory (one that gives all device memory to its own
pool at start-up, or a step loop that must not pay for cudaMalloc/cudaFree,
which synchronise the device).  Its scratch is a fixed array inside the
library, so this test checks, through the C ABI, that two calls in a row
give the same mesh as the allocating path (emu_load_particles +
emu_get_mesh) within the FP64 deposit tolerance of the other GPU tests
(1e-13 of the summed |contributions| per component; the two paths add in
different orders), also when the records come in a random order, that
rho/T/Ye are filled, and that a mesh larger than the fixed scratch is
refused.  The test allocates its own input and output buffers with torch;
the entry point itself allocates nothing.

The file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from emu_b200 import api
from emu_b200 import workloads as W
from oracle.oracle import Oracle
from tests.helpers import magnitude_mesh, mesh_rel_mag

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _cases():
    a = W.c2_fast_flavor_1d(ncell_z=32, ndirs=12)
    b = W.c5_3d(n=6, ndirs=5, mixed=False)
    c = W.ci_msw()
    return [("fast_flavor_1d_nf2", a, False), ("3d_nf3", b, False), ("msw_one_cell", c, False),
            ("3d_nf3_unsorted_records", W.c5_3d(n=6, ndirs=5, mixed=False), True),
            ("fast_flavor_1d_nf2_unsorted_records", W.c2_fast_flavor_1d(ncell_z=32, ndirs=12), True)]


@pytest.mark.parametrize("name,p,shuffle", _cases(), ids=[c[0] for c in _cases()])
def test_deposit_noalloc_matches_allocating_path(name, p, shuffle):
    import torch
    lib = api.load_library()
    parts = api.init_particles(p)
    if shuffle:
        # moved particles: positions off the cell centres, records in a
        # random order (the allocating path sorts them at load)
        rng = np.random.default_rng(7)
        L = np.array([p.Lx, p.Ly, p.Lz])
        parts[:, 0:3] = (parts[:, 0:3] + rng.uniform(-1.5, 1.5, (len(parts), 3)) * L / np.array(list(p.ncell))) % L
        parts[:, 4:7] = parts[:, 0:3]
        parts = parts[rng.permutation(len(parts))].copy()
    nf = p.nflavors
    ncomp = api.ncomp(nf)
    ncells = p.ncell[0] * p.ncell[1] * p.ncell[2]
    with api.Context(p) as c:
        c.load_particles(parts)
        ref = c.get_mesh()
    mag = magnitude_mesh(Oracle(p), parts)
    d_in = torch.from_numpy(parts).cuda()
    d_out = torch.full((ncomp * ncells,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        code = lib.emu_deposit_noalloc(ctypes.byref(p), ctypes.c_void_p(d_in.data_ptr()), parts.shape[0],
                                       ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream))
        assert code == api.EMU_OK, api.last_error()
        torch.cuda.synchronize()
        out = d_out.cpu().numpy()
        assert np.isfinite(out).all()
        assert np.array_equal(out[:3 * ncells], ref[:3 * ncells])
        assert mesh_rel_mag(out, ref, mag, ncomp) < TOL


def test_deposit_noalloc_rejects_meshes_beyond_the_scratch():
    import torch
    lib = api.load_library()
    p = W.c5_3d(n=40, ndirs=1, mixed=False)     # 64000 cells x 72 > 2^19
    parts = api.init_particles(W.c5_3d(n=4, ndirs=1, mixed=False))
    d_in = torch.from_numpy(parts).cuda()
    d_out = torch.zeros(8, dtype=torch.float64, device="cuda")
    code = lib.emu_deposit_noalloc(ctypes.byref(p), ctypes.c_void_p(d_in.data_ptr()), parts.shape[0],
                                   ctypes.c_void_p(d_out.data_ptr()), None)
    assert code == api.EMU_ERR_LIMIT
    assert "exceeds the fixed scratch" in api.last_error()
    torch.cuda.synchronize()
    assert (d_out.cpu().numpy() == 0).all()
