"""Generate the known-answer fixtures tests/golden/kat_*.npz from the
reference's own input decks and golden stress-strain curves.

Run where a reference checkout exists (its path is a required argument):
    python tests/golden/make_fixtures.py <reference checkout> [case ...]

For each case it stores what plasticity_b200.decks.load_deck reads from the
deck (derived as the reference derives it):
  * material constants from prm.prm (userInputParameters.cc:255-323), slip /
    twin vectors from the data files (normalised on load, init.cc:72-176), the
    latent-hardening matrix (init.cc:49-65);
  * the 8x8x8 mesh's per-cell Rodrigues vector: the grain of the voxel nearest
    to the cell centre, ties to the lower voxel (crystalOrientationsIO.cc:66-194,
    loadOrientations.cc:4-31), then the grain's row of orientations.txt;
  * the BCinfo face/dof/total-displacement table (ellipticBVP/init.cc:326-343),
    or the velocity gradient of a velocity-gradient deck;
  * the golden rows tests/compile_tests/<case>/correct_stressstrain.txt and
    the number of rows run_compile_tests.py checks (599 or 999).
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
from plasticity_b200.decks import load_deck  # noqa: E402

CASES = {
    "fcc_simpleTension": "fcc/simpleTension",
    "fcc_compression": "fcc/compression",
    "bcc_simpleTension": "bcc/simpleTension",
    "hcp_simpleTension": "hcp/simpleTension",
    "hcp_compression": "hcp/compression",
    "fcc_DeformationGraidientBCs": "fcc/DeformationGraidientBCs",
    "fcc_tabularSimpleCompression": "fcc/tabularSimpleCompression",
    "fcc_CyclicLoading": "fcc/CyclicLoading",
    "fcc_RandomOrientationBlock": "fcc/FCC_RandomOrientationBlock",
    "fcc_simpleCompression_Multiphase": "fcc/simpleCompression_Multiphase",
}
CHECK_ROWS = {"hcp_simpleTension": 599, "hcp_compression": 599}


def main(ref_root, only=None):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, sub in CASES.items():
        if only and name not in only:
            continue
        app = os.path.join(ref_root, "applications/crystalPlasticity", sub)
        d = load_deck(app, golden=os.path.join(ref_root, "tests/compile_tests", sub, "correct_stressstrain.txt"))
        for k in ("n_grains", "max_linear", "rel_linear_tol"):
            d.pop(k, None)
        d["check_rows"] = CHECK_ROWS.get(name, 999)
        out = os.path.join(here, f"kat_{name}.npz")
        np.savez_compressed(out, **d)
        print(f"{name}: mesh {d['n_elem']}, golden {d['golden'].shape} -> {out}")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_fixtures.py <reference checkout> [case ...]")
    main(sys.argv[1], sys.argv[2:])
