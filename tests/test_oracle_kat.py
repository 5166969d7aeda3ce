"""Pin the oracle to the reference's own known answers: the golden
stress-strain curves of tests/compile_tests/*/correct_stressstrain.txt,
reproduced through the Newton harness and judged with the reference's
criterion (run_compile_tests.py:43-60, relative error < 1e-2 on von Mises
strain, von Mises stress and total slip)."""
import numpy as np
import pytest

from plasticity_b200 import harness as H
from plasticity_b200 import materials as M
from plasticity_b200.capi import default_options


def _run(oracle_lib, case, n_inc):
    def factory(mats, d):
        opts = default_options(stress_tolerance=float(d["tol"]),
                               max_slip_search_iterations=int(d["max_slip_search"]),
                               max_solver_iterations=int(d["max_solver"]))
        return oracle_lib.OracleBackend(mats, opts, nthreads=0)

    h, d = H.kat_setup(f"tests/golden/kat_{case}.npz", factory, M.material_from_deck)
    rows = h.run(n_inc)
    return rows, d


@pytest.mark.parametrize("case,n_inc,tight,plastic", [("fcc_simpleTension", 30, 2e-3, True),
                                                     ("bcc_simpleTension", 12, 2e-3, False)])
def test_golden_curve_prefix(oracle_lib, case, n_inc, tight, plastic):
    """The first increments (elastic range, first yield and early hardening)
    must match far inside the reference's 1e-2 tolerance."""
    rows, d = _run(oracle_lib, case, n_inc)
    err = H.golden_errors(rows, d["golden"], n_inc)
    assert err["stress"] < tight and err["strain"] < tight, err
    assert err["slip"] < 1e-2, err
    # fcc: plastic flow has started inside the window (bcc's CRSS of 200 MPa
    # is reached only after ~140 increments: its prefix checks the elastic path)
    assert (rows[-1, 14] > 0) == plastic


def test_golden_curve_hcp_twin_prefix(oracle_lib):
    rows, d = _run(oracle_lib, "hcp_simpleTension", 25)
    err = H.golden_errors(rows, d["golden"], 25)
    assert err["stress"] < 1e-2 and err["strain"] < 1e-2 and err["slip"] < 1e-2, err


@pytest.mark.parametrize("case", ["fcc_DeformationGraidientBCs", "fcc_tabularSimpleCompression",
                                  "fcc_CyclicLoading", "fcc_RandomOrientationBlock"])
def test_golden_curve_prefix_loading_modes(oracle_lib, case):
    """The other loading modes and meshes of the reference's compile tests:
    the velocity-gradient boundary condition on the whole surface, tabular
    (piecewise-linear in time) face displacements, cyclic loading with
    kinematic hardening (backstress), and a 5x8x10 block of one grain per
    element.  The first 30 increments reach plastic flow in every case."""
    rows, d = _run(oracle_lib, case, 30)
    err = H.golden_errors(rows, d["golden"], 30)
    assert err["stress"] < 2e-3 and err["strain"] < 2e-3 and err["slip"] < 1e-2, err
    assert rows[-1, 14] > 0


@pytest.mark.slow
@pytest.mark.parametrize("case", ["fcc_simpleTension", "bcc_simpleTension", "hcp_simpleTension",
                                  "hcp_compression", "fcc_compression", "fcc_DeformationGraidientBCs",
                                  "fcc_tabularSimpleCompression", "fcc_RandomOrientationBlock"])
def test_golden_curve_full(oracle_lib, case):
    d = np.load(f"tests/golden/kat_{case}.npz")
    n = int(d["check_rows"]) + 1
    rows, d = _run(oracle_lib, case, n)
    err = H.golden_errors(rows, d["golden"], int(d["check_rows"]))
    assert err["stress"] < 1e-2 and err["strain"] < 1e-2 and err["slip"] < 1e-2, err


@pytest.mark.slow
def test_golden_curve_cyclic_full(oracle_lib):
    """fcc/CyclicLoading (backstress C1 = 200, C2 = 1, nearly no isotropic
    hardening) over the 999 checked rows: strain and total slip within the
    reference's 1e-2 everywhere, von Mises stress within 1e-2 over the first
    400 rows.  Beyond them the stress path is set by rounding: the oracle, the
    GPU update with a host direct solve and the GPU device loop, three orderings
    of the same arithmetic, differ from each other by up to 3.2 % in rows
    450-650 and each wanders around the golden curve (the device loop meets
    it to 1e-4 at row 561, where the oracle is 2.9 % off), so no bound tighter
    than a few percent holds for any implementation but the reference's own."""
    rows, d = _run(oracle_lib, "fcc_CyclicLoading", 999)
    err = H.golden_errors(rows, d["golden"], 999)
    assert err["strain"] < 1e-2 and err["slip"] < 1e-2, err
    assert H.golden_errors(rows, d["golden"], 400)["stress"] < 1e-2
    assert err["stress"] < 5e-2, err


@pytest.mark.slow
def test_cyclic_stress_beyond_row_400_is_set_by_rounding(oracle_lib):
    """Why the cyclic deck's stress is bounded only over its first 400 rows:
    the oracle as written and the oracle compiled with fused multiply-adds
    (two equally valid roundings of the same arithmetic) stay within the
    reference's 1e-2 of each other in von Mises stress over the first 400 rows
    (measured 1.4e-3 over the first 100, 4.0e-3 over 400) and part by more
    than that beyond (3.0e-2 at row 587): the same size as every
    implementation's distance from the golden curve there."""
    rows_a, _ = _run(oracle_lib, "fcc_CyclicLoading", 999)
    prev = oracle_lib.use_library(oracle_lib.build_fma())
    try:
        rows_b, _ = _run(oracle_lib, "fcc_CyclicLoading", 999)
    finally:
        oracle_lib.restore_library(prev)
    _, sa = H.von_mises_rows(rows_a)
    _, sb = H.von_mises_rows(rows_b)
    rel = np.abs(sa - sb) / np.abs(sa)
    print(f"cyclic deck, oracle vs its FMA build: von Mises stress {rel[:100].max():.1e} over rows < 100, "
          f"{rel[:400].max():.1e} over rows < 400, {rel[400:].max():.1e} beyond (row {400 + int(rel[400:].argmax())})")
    assert rel[:400].max() < 1e-2
    assert rel[400:].max() > 1e-2
