"""emu_deposit_noalloc: the deposit for callers that cannot allocate device
memory (work captured into a CUDA graph, a fixed memory pool, a loop that
must not touch the allocator).  Its scratch is a fixed array inside the
library, so this test checks, through the C ABI, that two calls in a row
give the same mesh as the allocating path (emu_load_particles +
emu_get_mesh) within the FP64 deposit tolerance of the other GPU tests
(1e-13 of the summed |contributions| per component; the two paths add in
different orders), that rho/T/Ye are filled, and that a mesh larger than the
fixed scratch is refused.  The test allocates its own input and output
buffers with torch; the entry point itself allocates nothing.

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
    return [("fast_flavor_1d_nf2", a), ("3d_nf3", b), ("msw_one_cell", c)]


@pytest.mark.parametrize("name,p", _cases(), ids=[c[0] for c in _cases()])
def test_deposit_noalloc_matches_allocating_path(name, p):
    import torch
    lib = api.load_library()
    parts = api.init_particles(p)
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
