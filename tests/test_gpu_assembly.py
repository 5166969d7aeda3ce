"""Fused element assembly (getElementalValues) and the Newton drop-in on the
GPU against the oracle, plus the reference's golden curve through the GPU."""
import numpy as np
import pytest

from plasticity_b200 import harness as H
from plasticity_b200 import materials as M
from plasticity_b200.capi import CpHandle, default_options
from tests._parity import TOL, copy_state, evolve, rel_err, well_posed

pytestmark = pytest.mark.gpu


def _mesh_pair(oracle_lib, mats, cell_lattice, seed, steps, amp=2e-4):
    """GPU handle and oracle with the same history, built by the oracle from
    'steps' committed increments of a mesh displacement field
    u_k = k (x L^T + noise): consistent, small strain increments."""
    mesh = H.StructuredMesh((4, 4, 4))
    rng = np.random.default_rng(seed)
    lid = np.repeat(np.asarray(cell_lattice, np.int32), 8)
    rod = np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0)
    ob = oracle_lib.OracleBackend(mats)
    ob.bind_qps(lid, rod)
    L = amp * rng.standard_normal((3, 3))
    du = (mesh.node_xyz @ L.T).ravel() + 0.1 * amp * rng.standard_normal(mesh.n_dofs)
    for k in range(1, steps + 1):
        ob.update(mesh.deformation_gradients(k * du), 0)
        ob.commit()
    gh = CpHandle(mats)
    gh.bind_qps(lid, rod)
    copy_state(ob, gh)
    for be in (gh, ob):
        be.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    return mesh, gh, ob, (steps + 1) * du


@pytest.mark.parametrize("mix", ["fcc", "bcc_hcp"])
def test_assemble_parity(oracle_lib, cuda_lib, mix):
    if mix == "fcc":
        mats, cl = [M.fcc_cu()], np.zeros(64, np.int32)
    else:
        mats = [M.bcc_48(), M.hcp_mg()]
        cl = (np.arange(64) % 3 == 0).astype(np.int32)
    mesh, gh, ob, u = _mesh_pair(oracle_lib, mats, cl, seed=3, steps=6)
    U = u[mesh.cell_dofs]
    Kg, Rg, sg = gh.assemble(U)
    Ko, Ro, so = ob.assemble(U)
    ok = well_posed(gh.stats(), ob.stats())
    cells = ok.reshape(-1, 8).all(axis=1)
    assert cells.mean() > 0.75
    assert (ob.stats()[:, 1] > 0).mean() > 0.3  # plastic flow in the increment
    assert np.array_equal(gh.stats()[ok, 1], ob.stats()[ok, 1])
    assert rel_err(Kg[cells], Ko[cells]) < TOL
    assert rel_err(Rg[cells], Ro[cells]) < TOL
    for f in ("Fp_iter", "s_iter"):
        assert rel_err(gh.get_state(f)[ok], ob.get_state(f)[ok]) < TOL
    gh.close()


def test_newton_dropin_matches_oracle_and_golden(oracle_lib, cuda_lib):
    """The reference's fcc/simpleTension deck through the GPU drop-in: every
    stress-strain row equals the oracle harness's and the golden curve."""
    n_inc = 12

    def gpu_factory(mats, d):
        return CpHandle(mats, default_options(stress_tolerance=float(d["tol"])))

    def cpu_factory(mats, d):
        return oracle_lib.OracleBackend(mats, default_options(stress_tolerance=float(d["tol"])))

    hg, d = H.kat_setup("tests/golden/kat_fcc_simpleTension.npz", gpu_factory, M.material_from_deck)
    ho, _ = H.kat_setup("tests/golden/kat_fcc_simpleTension.npz", cpu_factory, M.material_from_deck)
    rg = hg.run(n_inc)
    ro = ho.run(n_inc)
    assert rel_err(rg[:, :12], ro[:, :12]) < 1e-8
    err = H.golden_errors(rg, d["golden"], n_inc)
    assert err["stress"] < 1e-4 and err["strain"] < 1e-4 and err["slip"] < 1e-2, err
    hg.be.close()


def test_averages_match_oracle(oracle_lib, cuda_lib):
    mesh, gh, ob, u = _mesh_pair(oracle_lib, [M.hcp_mg()], np.zeros(64, np.int32), seed=9, steps=5)
    F = mesh.deformation_gradients(u)
    gh.update(F, 0)
    ob.update(F, 0)
    assert well_posed(gh.stats(), ob.stats()).all()
    a, b = gh.averages(), ob.averages()
    assert np.allclose(a, b, rtol=1e-10, atol=1e-13 * np.abs(b).max())
    gh.close()


def test_chunked_host_assembly_matches_device_assembly(cuda_lib):
    """cp_assemble with host buffers runs in caller-order chunks of cells
    (2 above 2^18 qps) with overlapped copies; every cell is independent, so
    Ke, Re and status must equal the unchunked device-pointer call's."""
    import torch
    mesh = H.StructuredMesh((32, 32, 33))  # 33,792 cells, 270,336 qps
    rng = np.random.default_rng(41)
    cl = (np.arange(mesh.n_cells) % 3).astype(np.int32)
    gh = CpHandle([M.fcc_cu(), M.bcc_48(), M.hcp_mg()])
    gh.bind_qps(np.repeat(cl, 8), np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0))
    gh.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    u = (mesh.node_xyz @ (2e-3 * rng.standard_normal((3, 3))).T).ravel()
    U = np.ascontiguousarray(u[mesh.cell_dofs])
    Ke, Re, st = gh.assemble(U)
    dev = torch.device("cuda", 0)
    Ud = torch.from_numpy(U).to(dev)
    Ked = torch.empty(mesh.n_cells, 24, 24, dtype=torch.float64, device=dev)
    Red = torch.empty(mesh.n_cells, 24, dtype=torch.float64, device=dev)
    Sd = torch.empty(mesh.n_cells * 8, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    gh.assemble_device(Ud.data_ptr(), 0.0, 0.0, Ked.data_ptr(), Red.data_ptr(), Sd.data_ptr())
    gh.synchronize()
    assert np.array_equal(Ke, Ked.cpu().numpy())
    assert np.array_equal(Re, Red.cpu().numpy())
    assert np.array_equal(st, Sd.cpu().numpy())
    assert (gh.stats()[:, 1] > 0).mean() > 0.3  # plastic
    gh.close()
