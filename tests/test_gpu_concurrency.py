"""Several contexts driven at once from host threads, each on its own CUDA
stream (the pattern of a serving process and of the end-to-end benchmark):
every context must give the result of a context used alone.

Tolerances: the mixed path's mesh sums are integers and its run sums follow
the cell-sorted order, so its results are bit-identical; the FP64 path adds
deposits with floating-point atomics in scheduling order, 1e-12 normwise
relative per attribute.
"""
import threading

import numpy as np
import pytest
import torch

from emu_b200 import api
from emu_b200 import workloads as W
from tests.helpers import colwise_rel

pytestmark = pytest.mark.gpu


def _params(mixed):
    if mixed:
        p = W.c3_three_flavor_1d(ncell_z=32, nphi_equator=4, mixed=True)
        p.precision = api.PREC_MIXED
    else:
        p = W.c2_fast_flavor_1d(ncell_z=16, ndirs=12)
    return p


def _run(p, recs, nsteps, stream=None):
    with api.Context(p) as c:
        if stream is not None:
            c.set_stream(stream.cuda_stream)
        c.load_particles(recs)
        info = c.evolve(nsteps)
        assert info.status == 0 and info.steps_done == nsteps
        return c.get_particles()


@pytest.mark.parametrize("mixed", [False, True])
def test_threads_with_own_contexts_match_a_single_context(mixed):
    p = _params(mixed)
    recs = api.init_particles(p)
    nsteps, nthreads, repeats = 6, 4, 3
    ref = _run(p, recs, nsteps)
    out = [[None] * repeats for _ in range(nthreads)]
    errors = []

    def worker(t):
        try:
            stream = torch.cuda.Stream()
            for r in range(repeats):
                out[t][r] = _run(p, recs, nsteps, stream)
        except Exception as e:  # reported by the main thread
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(nthreads)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    for t in range(nthreads):
        for r in range(repeats):
            got = out[t][r]
            assert got.shape == ref.shape
            if mixed:
                assert np.array_equal(got, ref), (t, r)
            else:
                assert colwise_rel(got, ref) < 1e-12, (t, r)
