"""cp_averages_noalloc: the volume averages without any device allocation.

Some callers of this library cannot call cudaMalloc: FE host codes that hand
the GPU's memory to their own pool allocator at start-up, and per-increment
callbacks that must not take cudaMalloc's device-wide synchronisation.  For
them cp_averages_noalloc reduces into a device array compiled into the
library instead of a buffer it allocates.  This test calls it through the C ABI
twice in a row and checks both results against cp_averages (same kernels and
summation order, so the tolerance is tight), then again after a new update so
a stale result from the shared array would show.  It also checks that the
first call on a fresh handle leaves the device's free memory unchanged (it
allocates nothing), and that a handle above the array's qp limit gets
CP_E_ARG with a message naming the limit.
"""
import ctypes

import numpy as np
import pytest

from plasticity_b200 import harness as H
from plasticity_b200 import materials as M
from plasticity_b200.capi import CP_E_ARG, CP_OK, CpHandle

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


def _loaded(mesh, rng):
    cl = (np.arange(mesh.n_cells) % 2).astype(np.int32)
    gh = CpHandle([M.fcc_cu(), M.hcp_mg()])
    gh.bind_qps(np.repeat(cl, 8), np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0))
    gh.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    gh.update(mesh.deformation_gradients((mesh.node_xyz @ (3e-4 * rng.standard_normal((3, 3))).T).ravel()), 0)
    return gh


def test_first_call_on_a_fresh_handle_allocates_nothing(cuda_lib):
    import torch
    mesh = H.StructuredMesh((4, 4, 4))
    rng = np.random.default_rng(5)
    warm = _loaded(mesh, rng)  # loads the averaging kernels into the context
    warm.averages()
    _noalloc(warm)
    warm.close()
    gh = _loaded(mesh, rng)
    gh.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    first = _noalloc(gh)  # this handle's first averages call of any kind
    gh.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    assert np.allclose(first, gh.averages(), rtol=1e-12, atol=1e-15)
    gh.close()


def test_above_the_limit_is_an_argument_error(cuda_lib):
    limit = 1 << 22  # CP_NOALLOC_AVG_MAX_QPS in include/cp_gpu.h
    n_cells = limit // 8 + 1  # one cell past the CP_NOALLOC_AVG_MAX_QPS qps of the array
    mesh_grad = H.StructuredMesh((1, 1, 1))
    gh = CpHandle([M.fcc_cu()])
    gh.bind_qps(np.zeros(8 * n_cells, np.int32), np.zeros((8 * n_cells, 3)))
    gh.bind_mesh(n_cells, mesh_grad.grad_N, mesh_grad.JxW, True)
    gh.update(np.tile(np.eye(3).ravel(), (8 * n_cells, 1)), 0, want_T=False)
    out = np.empty(22)
    rc = gh.lib.cp_averages_noalloc(gh.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == CP_E_ARG
    assert "CP_NOALLOC_AVG_MAX_QPS" in gh.lib.cp_last_error(gh.h).decode()
    assert np.isfinite(gh.averages()).all()  # the allocating call still serves it
    gh.close()
