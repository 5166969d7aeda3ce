"""plasticity_b200.decks on a small deck written in the reference's formats
(deal.II parameter file, slip/twin tables, latent-hardening matrix, voxel
grain map, orientation table, BC table), and the oracle harness run from it.
(The reader reproduces the committed tests/golden/kat_*.npz fixtures from the
reference's own decks: tests/golden/make_fixtures.py uses it.)"""
import numpy as np
import pytest

from plasticity_b200 import decks, harness as H, materials as M
from plasticity_b200.capi import default_options

PRM = """# test deck
set Number of Slip Systems = 12
set Twinning enabled = false
set Number of Twin Systems = 0
set Elastic Stiffness row 1 = 170.0e3, 124.0e3, 124.0e3, 0, 0, 0
set Elastic Stiffness row 2 = 124.0e3, 170.0e3, 124.0e3, 0, 0, 0
set Elastic Stiffness row 3 = 124.0e3, 124.0e3, 170.0e3, 0, 0, 0
set Elastic Stiffness row 4 = 0, 0, 0, 75.0e3, 0, 0
set Elastic Stiffness row 5 = 0, 0, 0, 0, 75.0e3, 0
set Elastic Stiffness row 6 = 0, 0, 0, 0, 0, 75.0e3
set Slip Normals File = slipNormals.txt
set Slip Directions File = slipDirections.txt
set Latent Hardening Ratio filename = latent.txt
set Initial Slip Resistance = 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16
set Initial Hardening Modulus = 180, 180, 180, 180, 180, 180, 180, 180, 180, 180, 180, 180
set Saturation Stress = 148, 148, 148, 148, 148, 148, 148, 148, 148, 148, 148, 148
set Power Law Exponent = 2.25, 2.25, 2.25, 2.25, 2.25, 2.25, 2.25, 2.25, 2.25, 2.25, 2.25, 2.25
set Stress Tolerance = 1.0e-9
set Max Slip Search Iterations = 1
set Max Solver Iterations = 1
set Maximum non linear iterations = 4
set Maximum linear solver iterations = 50000
set Relative linear solver tolerance = 1.0e-10
set Time increments = 0.1
set Total time = 0.3
set Subdivisions X = 1
set Subdivisions Y = 1
set Subdivisions Z = 1
set Refine factor = 2
set Domain size X = 1.0
set Domain size Y = 1.0
set Domain size Z = 1.0
set Voxels in X direction = 2
set Voxels in Y direction = 2
set Voxels in Z direction = 2
set Grain ID file name = grainID.txt
set Header Lines GrainID File = 1
set Orientations file name = orientations.txt
set Boundary condition filename = BCinfo.txt
set BC file number of header lines = 1
set Number of boundary conditions = 4
"""


def _write_deck(tmp_path):
    mat = M.fcc_cu()
    n = np.array(mat.slip_normal).reshape(-1, 3)[:12]
    m = np.array(mat.slip_direction).reshape(-1, 3)[:12]
    (tmp_path / "prm.prm").write_text(PRM)
    (tmp_path / "slipNormals.txt").write_text("\n".join(" ".join(f"{v:.17g}" for v in r) for r in n))
    (tmp_path / "slipDirections.txt").write_text("\n".join(" ".join(f"{v:.17g}" for v in r) for r in m))
    q = np.array(mat.latent_hardening).reshape(64, 64)[:12, :12]
    (tmp_path / "latent.txt").write_text("\n".join(" ".join(f"{v:g}" for v in r) for r in q))
    # voxels: x outer, y middle (one line per (x, y)), z inner; grain = 1 + x + 2y + 4z
    lines = ["header"] + [" ".join(str(1 + x + 2 * y + 4 * z) for z in range(2)) for x in range(2) for y in range(2)]
    (tmp_path / "grainID.txt").write_text("\n".join(lines))
    rng = np.random.default_rng(3)
    rod = M.random_rodrigues(rng, 8)
    (tmp_path / "orientations.txt").write_text(
        "id r1 r2 r3\n" + "\n".join(f"{g + 1} {r[0]:.17g} {r[1]:.17g} {r[2]:.17g}" for g, r in enumerate(rod)))
    (tmp_path / "BCinfo.txt").write_text("face dof value\n1 1 0\n1 2 0\n1 3 0\n2 1 0.003\n")
    return rod, n, m, q


def test_load_deck_reads_every_part(tmp_path):
    rod, n, m, q = _write_deck(tmp_path)
    d = decks.load_deck(str(tmp_path))
    assert d["C6"][0, 1] == 124.0e3 and d["C6"][3, 3] == 75.0e3
    assert np.array_equal(d["slip_normals"], n) and np.array_equal(d["slip_dirs"], m)
    assert np.array_equal(d["q"], q)
    assert list(d["n_elem"]) == [4, 4, 4] and d["n_grains"] == 8
    assert d["max_newton"] == 4 and d["tol"] == 1e-9 and d["rel_linear_tol"] == 1e-10
    # cell (kx, ky, kz) of the 4^3 mesh lies in voxel (kx // 2, ky // 2, kz // 2)
    for kz in range(4):
        for ky in range(4):
            for kx in range(4):
                g = 1 + kx // 2 + 2 * (ky // 2) + 4 * (kz // 2)
                assert np.array_equal(d["cell_rodrigues"][kx + 4 * (ky + 4 * kz)], rod[g - 1])
    assert d["bc"].tolist() == [[1, 1, 0.0], [1, 2, 0.0], [1, 3, 0.0], [2, 1, 0.003]]


def test_nearest_voxel_ties_go_to_the_lower_voxel():
    # centres of 2 voxels on [0, 1]: 0.25, 0.75; 0.5 is a tie
    assert decks.nearest_index(0.5, 2) == 0
    assert decks.nearest_index(0.5000001, 2) == 1
    assert decks.nearest_index(0.0, 2) == 0 and decks.nearest_index(1.0, 2) == 1


def test_deck_runs_through_the_oracle_harness(tmp_path, oracle_lib):
    _write_deck(tmp_path)
    d = decks.load_deck(str(tmp_path))
    h, _ = H.deck_setup(d, lambda mats, dd: oracle_lib.OracleBackend(mats, default_options()),
                        M.material_from_deck)
    rows = h.run()
    assert rows.shape == (3, 15)
    assert rows[-1, 0] == pytest.approx(0.003, rel=0.05)  # mean E_xx follows the prescribed stretch
    assert rows[-1, 6] > rows[0, 6] > 0.0
