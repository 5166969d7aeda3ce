"""The Newton step's global system on the GPU (cp_bind_dofs /
cp_newton_iteration / cp_update_from_displacement): the device scatter of
Ke/Re into CSR, the Dirichlet condensation and the Jacobi-preconditioned
Krylov solve against the host harness's direct sparse solve of the same
Newton loop, and the reference's golden curve."""
import numpy as np
import pytest

from plasticity_b200 import harness as H
from plasticity_b200 import materials as M
from plasticity_b200.capi import (CP_SOLVER_BICG, CP_SOLVER_BICGSTAB, CpError, CpHandle, default_options,
                                  default_solver)
from tests._parity import rel_err

pytestmark = pytest.mark.gpu

KAT = "tests/golden/kat_fcc_simpleTension.npz"


def _gpu_factory(mats, d):
    return CpHandle(mats, default_options(stress_tolerance=float(d["tol"])))


@pytest.mark.parametrize("kind", [CP_SOLVER_BICG, CP_SOLVER_BICGSTAB])
def test_device_newton_matches_host_direct_solve(cuda_lib, kind):
    """fcc/simpleTension deck, first 10 increments (through first yield):
    the device system (iterative, ||r|| <= 1e-10 ||b||) against the host
    direct solve; same rows to 1e-6, same displacements, golden curve."""
    n_inc = 10
    hh, d = H.kat_setup(KAT, _gpu_factory, M.material_from_deck)
    hd, _ = H.kat_setup(KAT, _gpu_factory, M.material_from_deck, device_system=True,
                        solver=default_solver(kind=kind))
    rh = hh.run(n_inc)
    rd = hd.run(n_inc)
    assert all(i["converged"] and not i["breakdown"] for i in hd.solve_info), hd.solve_info[:3]
    assert all(i["residual_norm"] <= 1e-10 * i["rhs_norm"] for i in hd.solve_info)
    assert rel_err(rd[:, :12], rh[:, :12]) < 1e-6
    assert np.abs(hd.u - hh.u).max() <= 1e-7 * np.abs(hh.u).max()
    err = H.golden_errors(rd, d["golden"], n_inc)
    assert err["stress"] < 1e-4 and err["strain"] < 1e-4, err
    hh.be.close()
    hd.be.close()


def test_device_newton_mixed_lattices_and_precond_norm(cuda_lib):
    """A 4x4x4 mesh whose cells alternate FCC and HCP grains under the deck's
    tension BCs; the device loop with PETSc's preconditioned-residual test
    against the host direct solve."""
    mesh = H.StructuredMesh((4, 4, 4))
    rng = np.random.default_rng(23)
    cl = (np.arange(mesh.n_cells) % 2).astype(np.int32)
    rod = np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0)
    # faces 1/3/5 (x=0, y=0, z=0) held in x/y/z, face 2 (x=1) pulled to u_x = 0.004 over 8 increments
    bc = np.array([[1, 1, 0.0], [3, 2, 0.0], [5, 3, 0.0], [2, 1, 0.004]])
    runs = []
    for dev in (False, True):
        be = CpHandle([M.fcc_cu(), M.hcp_mg()])
        be.bind_qps(np.repeat(cl, 8), rod)
        h = H.NewtonHarness(be, mesh, bc, 8, 4, device_system=dev,
                            solver=default_solver(precond_norm=1) if dev else None)
        runs.append((h, h.run(4)))
    (hh, rh), (hd, rd) = runs
    assert all(i["converged"] for i in hd.solve_info)
    assert np.abs(rh[:, 6:12]).max() > 20.0  # MPa: past the 5-16 MPa critical resolved shear stresses
    assert rel_err(rd[:, :12], rh[:, :12]) < 1e-4
    hh.be.close()
    hd.be.close()


def test_device_system_errors(cuda_lib):
    mesh = H.StructuredMesh((2, 2, 2))
    be = CpHandle([M.fcc_cu()])
    be.bind_qps(np.zeros(mesh.n_cells * 8, np.int32), np.zeros((mesh.n_cells * 8, 3)))
    with pytest.raises(CpError):
        be.newton_iteration()  # no mesh, no dofs
    be.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    with pytest.raises(CpError):
        be.newton_iteration()  # no dofs bound
    bad = mesh.cell_dofs.copy()
    bad[0, 0] = mesh.n_dofs
    with pytest.raises(CpError):
        be.bind_dofs(mesh.n_dofs, bad, [0])  # dof out of range
    bad = mesh.cell_dofs.copy()
    bad[0, 1] = bad[0, 0]
    with pytest.raises(CpError):
        be.bind_dofs(mesh.n_dofs, bad, [0])  # repeated dof in a cell
    with pytest.raises(CpError):
        be.bind_dofs(mesh.n_dofs, mesh.cell_dofs, [0, 0])  # constrained twice
    be.bind_dofs(mesh.n_dofs, mesh.cell_dofs, [0, 1, 2])
    with pytest.raises(CpError):
        be.newton_iteration(solver=default_solver(max_iterations=0))
    # an unloaded mesh: zero right-hand side, du = 0 with no iterations
    info = be.newton_iteration(np.zeros(3))
    assert info["converged"] and info["iterations"] == 0
    assert np.abs(be.get_displacement()).max() == 0.0
    be.close()
