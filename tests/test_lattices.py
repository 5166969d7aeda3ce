"""Slip/twin tables generated from Miller(-Bravais) indices."""
import numpy as np
import pytest

from plasticity_b200 import materials as M


def _check(n, m):
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-15)
    assert np.allclose(np.linalg.norm(m, axis=1), 1.0, atol=1e-15)
    assert np.allclose(np.sum(n * m, axis=1), 0.0, atol=1e-14)
    pairs = {(tuple(np.round(a, 9)), tuple(np.round(b, 9))) for a, b in zip(n, m)}
    neg = {(tuple(np.round(-a, 9)), tuple(np.round(-b, 9))) for a, b in zip(n, m)}
    assert len(pairs) == len(n)
    assert not (pairs & neg) or len(n) == len(pairs)


def test_fcc_matches_reference_deck():
    n, m = M.fcc_systems()
    _check(n, m)
    d = np.load("tests/golden/kat_fcc_simpleTension.npz")
    assert np.allclose(n, M.normalise_rows(d["slip_normals"]), atol=1e-3)
    assert np.allclose(m, M.normalise_rows(d["slip_dirs"]), atol=1e-3)


def test_bcc48():
    n, m = M.bcc_systems()
    assert len(n) == 48
    _check(n, m)
    # the 12 {110} systems span the same set as the reference's bcc deck
    d = np.load("tests/golden/kat_bcc_simpleTension.npz")
    ref = {(tuple(np.round(a, 6)), tuple(np.round(b, 6))) for a, b in
           zip(M.normalise_rows(d["slip_normals"]), M.normalise_rows(d["slip_dirs"]))}
    ours = set()
    for a, b in zip(n[:12], m[:12]):
        for s1 in (1, -1):
            for s2 in (1, -1):
                ours.add((tuple(np.round(s1 * a, 6)), tuple(np.round(s2 * b, 6))))
    assert all(r in ours for r in ref)


def test_hcp30():
    n, m, groups = M.hcp_systems()
    assert len(n) == 30
    _check(n, m)
    assert [groups.count(g) for g in ("basal", "prism", "pyr_a", "pyr_ca", "twin")] == [3, 3, 6, 12, 6]
    tw = [i for i, g in enumerate(groups) if g == "twin"]
    # tension twins: positive resolved shear under c-axis tension
    for i in tw:
        assert m[i][2] * n[i][2] > 0
    # c/a from the pyramidal <c+a> direction: |c| = 1.624 a
    ca = [i for i, g in enumerate(groups) if g == "pyr_ca"]
    for i in ca:
        assert abs(m[i][2]) > 0.5


def test_materials_build():
    for mat in (M.fcc_cu(), M.bcc_48(), M.hcp_mg()):
        a = M.material_arrays(mat)
        n = mat.n_total
        assert a["n"].shape == (n, 3)
        if not mat.twinning_enabled:
            # dummy twin: zero latent-hardening row and column, CRSS 10e14
            assert np.all(a["q"][-1] == 0) and np.all(a["q"][:, -1] == 0)
            assert a["s0"][-1] == 10e14
    assert M.fcc_cu().n_total == 13 and M.bcc_48().n_total == 49 and M.hcp_mg().n_total == 30


def test_random_rodrigues_uniform():
    rng = np.random.default_rng(0)
    r = M.random_rodrigues(rng, 20000)
    q0 = 1 / np.sqrt(1 + np.sum(r * r, axis=1))
    # for uniform rotations q0 = cos(theta/2) has density (4/pi) sqrt(1-q0^2) on [0,1]
    assert abs(np.mean(q0) - 4 / (3 * np.pi)) < 0.01
