"""cp_averages_noalloc: the volume averages without any device allocation.

Some callers of this library cannot call cudaMalloc: FE host codes that hand
the GPU's memory to their own pool allocator at start-up, and per-increment
callbacks that must not take cudaMalloc's device-wide synchronisation.  For
them cp_averages_noalloc reduces into a device array compiled into the
library instead of a buffer it allocates.  This test calls it through the C ABI
twice in a row and checks both results against cp_averages (same kernels and
summation order, so the tolerance is tight), then again after a new update so
a stale result from the shared array would show.
"""
import ctypes

import numpy as np
import pytest

from plasticity_b200 import harness as H
from plasticity_b200 import materials as M
from plasticity_b200.capi import CP_OK, CpHandle

pytestmark = pytest.mark.gpu


def _noalloc(gh):
    out = np.empty(22)
    rc = gh.lib.cp_averages_noalloc(gh.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == CP_OK, gh.lib.cp_last_error(gh.h)
    return out


def test_averages_noalloc_matches_cp_averages(cuda_lib):
    mesh = H.StructuredMesh((6, 6, 6))
    rng = np.random.default_rng(17)
    cl = (np.arange(mesh.n_cells) % 2).astype(np.int32)
    lid = np.repeat(cl, 8)
    rod = np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0)
    gh = CpHandle([M.fcc_cu(), M.hcp_mg()])
    gh.bind_qps(lid, rod)
    gh.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    du = (mesh.node_xyz @ (3e-4 * rng.standard_normal((3, 3))).T).ravel()
    tol = dict(rtol=1e-12, atol=1e-15)
    for k in (1, 2):
        gh.update(mesh.deformation_gradients(k * du), 0)
        ref = gh.averages()
        first = _noalloc(gh)
        second = _noalloc(gh)
        assert np.allclose(first, ref, **tol), (k, first - ref)
        assert np.allclose(second, ref, **tol), (k, second - ref)
        assert abs(ref[21] - 1.0) < 1e-12  # unit-cube volume
        if k == 1:
            prev = ref
    assert not np.allclose(prev[9:18], ref[9:18])  # the second update changed the stresses
    gh.close()
