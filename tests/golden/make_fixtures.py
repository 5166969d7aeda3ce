"""Generate the known-answer fixtures tests/golden/kat_*.npz from the
reference's own input decks and golden stress-strain curves.

Run in a container where the reference checkout exists:
    python tests/golden/make_fixtures.py /root/reference

For each case it stores what the Newton harness needs, derived exactly as the
reference derives it:
  * material constants from prm.prm (userInputParameters.cc:255-323), slip /
    twin vectors from the data files (normalised on load, init.cc:72-176), the
    latent-hardening matrix (init.cc:49-65);
  * the 8x8x8 mesh's per-cell Rodrigues vector: the grain of the voxel nearest
    to the cell centre, ties to the lower voxel (crystalOrientationsIO.cc:66-194,
    loadOrientations.cc:4-31), then the grain's row of orientations.txt;
  * the BCinfo face/dof/total-displacement table (ellipticBVP/init.cc:326-343);
  * the golden rows tests/compile_tests/<case>/correct_stressstrain.txt and
    the number of rows run_compile_tests.py checks (599 or 999).
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

CASES = {
    "fcc_simpleTension": "fcc/simpleTension",
    "fcc_compression": "fcc/compression",
    "bcc_simpleTension": "bcc/simpleTension",
    "hcp_simpleTension": "hcp/simpleTension",
    "hcp_compression": "hcp/compression",
}
CHECK_ROWS = {"hcp_simpleTension": 599, "hcp_compression": 599}


def parse_prm(path):
    out = {}
    for line in open(path):
        line = line.split("#", 1)[0].strip()
        m = re.match(r"set\s+(.+?)\s*=\s*(.*)$", line)
        if m:
            out[m.group(1).strip()] = m.group(2).strip()
    return out


def floats(s):
    return np.array([float(x) for x in re.split(r"[,\s]+", s.strip()) if x], dtype=np.float64)


def read_vectors(path, count):
    rows = []
    for line in open(path):
        f = line.split()
        if len(f) >= 3:
            rows.append([float(f[0]), float(f[1]), float(f[2])])
        if len(rows) == count:
            break
    return np.array(rows)


def read_q(path, n):
    q = np.zeros((n, n))
    r = 0
    for line in open(path):
        f = line.split()
        if not f:
            continue
        q[r, :] = [float(x) for x in f[:n]]
        r += 1
        if r == n:
            break
    return q


def nearest_index(coord, n_pts, span=1.0):
    """Nearest voxel centre (x*stencil + stencil/2), ties to the lower one."""
    st = span / n_pts
    centres = np.arange(n_pts) * st + st / 2
    up = np.searchsorted(centres, coord, side="left")  # std::map::lower_bound
    if up == n_pts:
        return n_pts - 1
    if up == 0:
        return 0
    lo = up - 1
    return lo if abs(centres[up] - coord) >= abs(centres[lo] - coord) else up


def main(ref_root):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, sub in CASES.items():
        app = os.path.join(ref_root, "applications/crystalPlasticity", sub)
        prm = parse_prm(os.path.join(app, "prm.prm"))
        ns = int(prm["Number of Slip Systems"])
        twinning = prm.get("Twinning enabled", "false").lower() == "true"
        nw = int(prm["Number of Twin Systems"]) if twinning else 0
        C6 = np.vstack([floats(prm[f"Elastic Stiffness row {i}"]) for i in range(1, 7)])
        sn = read_vectors(os.path.join(app, prm["Slip Normals File"]), ns)
        sd = read_vectors(os.path.join(app, prm["Slip Directions File"]), ns)
        n_real = ns + nw
        q = read_q(os.path.join(app, prm["Latent Hardening Ratio filename"]), n_real)
        d = dict(C6=C6, slip_normals=sn, slip_dirs=sd, q=q,
                 s0=floats(prm["Initial Slip Resistance"]), h0=floats(prm["Initial Hardening Modulus"]),
                 s_s=floats(prm["Saturation Stress"]), a=floats(prm["Power Law Exponent"]),
                 twinning=np.int32(twinning),
                 tol=float(prm["Stress Tolerance"]),
                 max_slip_search=int(prm["Max Slip Search Iterations"]),
                 max_solver=int(prm["Max Solver Iterations"]),
                 max_newton=int(prm["Maximum non linear iterations"]),
                 delT=float(prm["Time increments"]), total_T=float(prm["Total time"]))
        if twinning:
            d.update(twin_normals=read_vectors(os.path.join(app, prm["Twin Normals File"]), nw),
                     twin_dirs=read_vectors(os.path.join(app, prm["Twin Directions File"]), nw),
                     twin_s0=floats(prm["Initial Slip Resistance Twin"]),
                     twin_h0=floats(prm["Initial Hardening Modulus Twin"]),
                     twin_s_s=floats(prm["Saturation Stress Twin"]),
                     twin_a=floats(prm["Power Law Exponent Twin"]),
                     twin_threshold=float(prm["Twin Threshold Fraction"]),
                     twin_saturation=float(prm["Twin Saturation Factor"]),
                     twin_shear=float(prm["Characteristic Twin Shear"]))
        # mesh: subdivided unit cube refined 'Refine factor' times
        subdiv = [int(prm[f"Subdivisions {a}"]) for a in "XYZ"]
        span = [float(prm[f"Domain size {a}"]) for a in "XYZ"]
        refine = int(prm["Refine factor"])
        ne = [s * 2 ** refine for s in subdiv]
        assert span == [1.0, 1.0, 1.0]
        # voxel grain ids: x outer, y middle (one line per (x,y)), z inner
        npts = [int(float(prm[f"Voxels in {a} direction"])) for a in "XYZ"]
        lines = open(os.path.join(app, prm["Grain ID file name"])).read().splitlines()
        hdr = int(prm["Header Lines GrainID File"])
        data = lines[hdr: hdr + npts[0] * npts[1]]
        vox = np.array([[int(float(x)) for x in l.split()[: npts[2]]] for l in data]).reshape(npts[0], npts[1], npts[2])
        orient = {}
        for l in open(os.path.join(app, prm["Orientations file name"])).read().splitlines()[1:]:
            f = l.split()
            if len(f) >= 4:
                orient[int(f[0])] = [float(f[1]), float(f[2]), float(f[3])]
        # cells in lexicographic order (x fastest); order is irrelevant to the averages
        rod = np.zeros((ne[0] * ne[1] * ne[2], 3))
        for kz in range(ne[2]):
            for ky in range(ne[1]):
                for kx in range(ne[0]):
                    c = [(kx + 0.5) / ne[0], (ky + 0.5) / ne[1], (kz + 0.5) / ne[2]]
                    vi = [nearest_index(c[a], npts[a]) for a in range(3)]
                    gid = vox[vi[0], vi[1], vi[2]]
                    rod[kx + ne[0] * (ky + ne[1] * kz)] = orient[gid]
        bc = []
        bl = open(os.path.join(app, prm["Boundary condition filename"])).read().splitlines()
        nh = int(prm["BC file number of header lines"])
        for l in bl[nh: nh + int(prm["Number of boundary conditions"])]:
            f = l.split()
            bc.append([int(f[0]), int(f[1]), float(f[2])])
        golden = np.loadtxt(os.path.join(ref_root, "tests/compile_tests", sub, "correct_stressstrain.txt"),
                            skiprows=1)
        d.update(n_elem=np.array(ne), cell_rodrigues=rod, bc=np.array(bc), golden=golden,
                 check_rows=CHECK_ROWS.get(name, 999))
        out = os.path.join(here, f"kat_{name}.npz")
        np.savez_compressed(out, **d)
        print(f"{name}: {ns} slip + {nw} twin, mesh {ne}, {len(orient)} grains, golden {golden.shape} -> {out}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
