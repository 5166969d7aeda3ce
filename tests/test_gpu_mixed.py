"""The mixed-precision path: the split-BF16 tensor-core element contraction
(cp_assemble_mixed: FP32 Ke, FP64 Re) against the FP64 contraction and the
oracle, and the mixed-precision Newton step (FP32 Jacobi BiCG inside FP64
residual refinement) against the FP64 device loop.  Each comparison reports
the error against its FP64 counterpart and bounds it."""
import numpy as np
import pytest

from plasticity_b200 import harness as H
from plasticity_b200 import materials as M
from plasticity_b200.capi import CP_PRECISION_MIXED, CpHandle, default_options, default_solver

pytestmark = pytest.mark.gpu

KE_TOL = 2e-6  # split-BF16 (3 terms, 6 products) with FP32 accumulation, relative to the cell's largest |Ke|


def ke_rel_err(a, b):
    """max over cells of max|a - b| / max|b| (per cell)."""
    a = np.asarray(a, np.float64).reshape(len(a), -1)
    b = np.asarray(b, np.float64).reshape(len(b), -1)
    return float((np.abs(a - b).max(axis=1) / np.abs(b).max(axis=1)).max())


def _loaded_pair(shape, lattices, seed, increments=5):
    """An FP64-assembly handle and a mixed-assembly handle with the same
    committed history (increments of macroscopic stretch plus nodal noise)."""
    mesh = H.StructuredMesh(shape)
    rng = np.random.default_rng(seed)
    lid = np.repeat(rng.choice(len(lattices), size=mesh.n_cells), 8).astype(np.int32)
    rod = np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0)
    hs = []
    for _ in range(2):
        h = CpHandle(lattices, default_options())
        h.bind_qps(lid, rod)
        h.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
        hs.append(h)
    u = np.zeros(mesh.n_dofs)
    for _ in range(increments):
        u = u + (mesh.node_xyz @ (1e-3 * np.diag([1.0, -0.3, -0.3]) + 2e-4 * rng.standard_normal((3, 3))).T).ravel()
        for h in hs:
            h.assemble(u[mesh.cell_dofs])
            h.commit()
    u = u + (mesh.node_xyz @ (1e-3 * np.diag([1.0, -0.3, -0.3])).T).ravel() + 1e-5 * rng.standard_normal(mesh.n_dofs)
    return mesh, hs[0], hs[1], u[mesh.cell_dofs]


@pytest.mark.parametrize("shape", [(6, 6, 6), (16, 16, 16)])
def test_tensor_core_contraction_matches_fp64(cuda_lib, shape):
    """6^3: 216 cells = 15 full 14-cell tiles and a partial one; 16^3: 4096
    cells = 293 tiles over at most 148 persistent CTAs (each loops, the next
    tile's bulk copy in flight during the current one)."""
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    mesh, h64, hmx, Ul = _loaded_pair(shape, mats, seed=int(np.prod(shape)))
    K64, R64, s64 = h64.assemble(Ul)
    Kmx, Rmx, smx = hmx.assemble_mixed(Ul)
    assert Kmx.dtype == np.float32
    err = ke_rel_err(Kmx, K64)
    print(f"Ke split-BF16 vs FP64: {err:.2e} (cells {mesh.n_cells})")
    assert err < KE_TOL, err
    assert np.array_equal(Rmx, R64), "Re must be the FP64 contraction's"
    assert np.array_equal(smx, s64)
    assert (h64.stats()[:, 1] > 0).mean() > 0.3  # plastic tangents, not only elastic ones
    # the repeat (graph replay of the captured call) gives the same bits
    Kmx2, Rmx2, _ = hmx.assemble_mixed(Ul)
    assert np.array_equal(Kmx2, Kmx) and np.array_equal(Rmx2, Rmx)
    h64.close()
    hmx.close()


def test_tensor_core_contraction_vs_oracle(oracle_lib, cuda_lib):
    """Against the CPU oracle's FP64 getElementalValues on the same history."""
    from tests._parity import copy_state
    mats = [M.fcc_cu(), M.hcp_mg()]
    mesh = H.StructuredMesh((3, 3, 3))
    rng = np.random.default_rng(31)
    lid = np.repeat(rng.choice(2, size=mesh.n_cells), 8).astype(np.int32)
    rod = np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0)
    ob = oracle_lib.OracleBackend(mats, default_options(), nthreads=0)
    ob.bind_qps(lid, rod)
    ob.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    u = np.zeros(mesh.n_dofs)
    for _ in range(3):
        u = u + (mesh.node_xyz @ (4e-4 * np.diag([1.0, -0.3, -0.3]) + 1e-4 * rng.standard_normal((3, 3))).T).ravel()
        ob.assemble(u[mesh.cell_dofs])
        ob.commit()
    gh = CpHandle(mats, default_options())
    gh.bind_qps(lid, rod)
    gh.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    copy_state(ob, gh)
    u = u + (mesh.node_xyz @ (4e-4 * np.diag([1.0, -0.3, -0.3])).T).ravel()
    Ko, Ro, _ = ob.assemble(u[mesh.cell_dofs])
    Kg, Rg, _ = gh.assemble_mixed(u[mesh.cell_dofs])
    cells = ((gh.stats()[:, 7] <= 12) & (ob.stats()[:, 7] <= 12)).reshape(-1, 8).all(axis=1)
    assert cells.sum() >= 10 and (gh.stats()[:, 1] > 0).mean() > 0.3
    err = ke_rel_err(Kg[cells], Ko[cells])
    print(f"Ke split-BF16 vs oracle: {err:.2e}")
    assert err < KE_TOL, err
    assert ke_rel_err(Rg[cells], Ro[cells]) < 1e-10
    gh.close()


def _rve_handle(mesh, rod, bc, precision, n_inc, total_strain=0.02):
    be = CpHandle([M.fcc_cu()], default_options())
    be.bind_qps(np.zeros(mesh.n_cells * 8, np.int32), rod)
    bc = np.array(bc, float)
    bc[-1, 2] = total_strain
    h = H.NewtonHarness(be, mesh, bc, 20, 4, device_system=True,
                        solver=default_solver(precision=precision, kernel_mode=1))
    h.run(n_inc)
    return be, h


RVE_BC = [[1, 1, 0.0], [1, 2, 0.0], [1, 3, 0.0], [2, 1, 0.02]]


def test_mixed_newton_step_matches_fp64(cuda_lib):
    """One Newton iteration of the 8^3 FCC RVE from the same plastic state
    (3 increments into the run): the mixed-precision step (FP32 tensor-core
    Ke, FP32 inner BiCG, FP64 refinement to ||r|| <= 1e-10 ||b||) against the
    FP64 step.  Their du differ only through K's FP32 rounding."""
    mesh = H.StructuredMesh((8, 8, 8))
    rod = np.repeat(M.random_rodrigues(np.random.default_rng(0), mesh.n_cells), 8, axis=0)
    be, h = _rve_handle(mesh, rod, RVE_BC, 0, 3)
    u0 = be.get_displacement()
    state = {f + suf: be.get_state(f + suf) for f in ("Fp", "Fe", "s", "W", "rot", "rotnew", "twinfrac",
                                                      "slipfrac", "twin") for suf in ("_conv", "_iter")}
    info64 = be.newton_iteration(None, h.F_e, h.F_r, default_solver(kernel_mode=1))
    du64 = be.get_displacement() - u0
    bm = CpHandle([M.fcc_cu()], default_options())
    bm.bind_qps(np.zeros(mesh.n_cells * 8, np.int32), rod)
    bm.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    bm.bind_dofs(mesh.n_dofs, mesh.cell_dofs, h.cdofs)
    for k, v in state.items():
        bm.set_state(k, v)
    bm.set_displacement(u0)
    infomx = bm.newton_iteration(None, h.F_e, h.F_r, default_solver(precision=CP_PRECISION_MIXED))
    dumx = bm.get_displacement() - u0
    assert infomx["converged"] and infomx["residual_norm"] <= 1e-10 * infomx["rhs_norm"], infomx
    assert infomx["refinements"] >= 1
    err = float(np.abs(dumx - du64).max() / np.abs(du64).max())
    print(f"one Newton step, mixed vs FP64: du {err:.2e}; iterations {infomx['iterations']} "
          f"({infomx['refinements']} refinements) vs {info64['iterations']}")
    assert err < 1e-4, err
    be.close()
    bm.close()


def test_mixed_newton_loop_elastic_range(cuda_lib):
    """The 8^3 FCC RVE pulled to 2e-4 in 20 increments: the first 3 stay
    elastic (no active-set solve, so no rounding-determined result), and the
    mixed-precision device loop matches the FP64 one there to 1e-6 in
    stress and displacement."""
    mesh = H.StructuredMesh((8, 8, 8))
    rod = np.repeat(M.random_rodrigues(np.random.default_rng(0), mesh.n_cells), 8, axis=0)
    out = []
    for prec in (0, CP_PRECISION_MIXED):
        be, h = _rve_handle(mesh, rod, RVE_BC, prec, 3, total_strain=2e-4)
        assert (be.stats()[:, 0] == 0).all()  # elastic: no potentially active system
        out.append((np.array(h.rows), be.get_displacement(), h.solve_info))
        be.close()
    (r64, u64, _), (rmx, umx, imx) = out
    assert all(i["converged"] for i in imx)
    s_err = float(np.abs(rmx[:, 6:12] - r64[:, 6:12]).max() / np.abs(r64[:, 6:12]).max())
    u_err = float(np.abs(umx - u64).max() / np.abs(u64).max())
    print(f"elastic RVE, mixed vs FP64: stress {s_err:.2e}, u {u_err:.2e}")
    assert s_err < 1e-6 and u_err < 1e-6, (s_err, u_err)


def test_mixed_inner_solve_ignores_stale_device_memory(cuda_lib):
    """The FP32 inner solve's vectors are allocated on a handle's first mixed
    Newton step.  Nothing that memory held before may reach the solve: the
    vectors start as zeros and the first direction of every pass is z itself
    (0 * NaN would otherwise turn every FP32 pass into NaN and hand the whole
    run to the FP64 fallback).  Device memory filled with NaN is released just
    before the handle is made, so that stale values are likely (not certain)
    to land in its buffers; on the elastic 8^3 RVE every Newton step must then
    converge with FP32 passes alone."""
    import torch
    junk = torch.full((1 << 30,), float("nan"), dtype=torch.float32, device="cuda")  # 4 GB of NaN
    torch.cuda.synchronize()
    del junk
    torch.cuda.empty_cache()
    mesh = H.StructuredMesh((8, 8, 8))
    rod = np.repeat(M.random_rodrigues(np.random.default_rng(0), mesh.n_cells), 8, axis=0)
    be, h = _rve_handle(mesh, rod, RVE_BC, CP_PRECISION_MIXED, 3, total_strain=2e-4)
    info = h.solve_info
    assert info and all(i["converged"] for i in info), info
    assert all(i["fp64_iterations"] == 0 for i in info), [i["fp64_iterations"] for i in info]
    be.close()
