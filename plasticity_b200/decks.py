"""Reference input decks -> the library's inputs.

Reads an application directory of PRISMS-Plasticity's crystalPlasticity
model (the ``prm.prm`` parameter file and the files it names) into the values
the library and the Newton harness need, derived as the reference derives
them:

* material constants from the parameter file (userInputParameters.cc:255-323);
  slip / twin normals and directions from their files, normalised on use
  (init.cc:72-176); the latent-hardening matrix (init.cc:49-65);
* the mesh (subdivided unit cube refined ``Refine factor`` times) and, per
  cell, the Rodrigues vector of the grain of the voxel nearest to the cell
  centre, ties to the lower voxel (crystalOrientationsIO.cc:66-194,
  loadOrientations.cc:4-31);
* the boundary-condition table face / dof / total displacement
  (ellipticBVP/init.cc:326-343) with the cyclic-loading face, direction and
  quarter-cycle time, the tabular table and its times, or the velocity
  gradient of the velocity-gradient boundary condition;
* the solver settings (tolerances, caps, Newton iterations, increments).

``load_deck`` returns a plain dict (the layout of tests/golden/kat_*.npz);
``materials.material_from_deck`` turns it into a ``CpMaterial`` and
``harness.kat_setup`` into a ready Newton harness.
"""
from __future__ import annotations

import os
import re

import numpy as np


def parse_prm(path):
    """``set Name = value`` lines of a deal.II parameter file ('#' comments)."""
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
    """The first ``count`` rows of three numbers of a slip/twin table."""
    rows = []
    for line in open(path):
        f = line.split()
        if len(f) >= 3:
            rows.append([float(f[0]), float(f[1]), float(f[2])])
        if len(rows) == count:
            break
    if len(rows) < count:
        raise ValueError(f"{path}: {len(rows)} vectors, {count} expected")
    return np.array(rows)


def read_q(path, n):
    """The leading n x n block of a latent-hardening matrix file."""
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
    if r < n:
        raise ValueError(f"{path}: {r} rows, {n} expected")
    return q


def nearest_index(coord, n_pts, span=1.0):
    """Nearest voxel centre (x*stencil + stencil/2) to a coordinate, ties to
    the lower one, as a std::map::lower_bound search does."""
    st = span / n_pts
    centres = np.arange(n_pts) * st + st / 2
    up = int(np.searchsorted(centres, coord, side="left"))
    if up == n_pts:
        return n_pts - 1
    if up == 0:
        return 0
    lo = up - 1
    return lo if abs(centres[up] - coord) >= abs(centres[lo] - coord) else up


def _material(prm, f, sfx=""):
    """Material constants of one phase: the unsuffixed keys for phase 1, the
    keys with " 2", " 3", ... for the other phases of a multiphase deck
    (userInputParameters.cc:255-323 and its copies per phase)."""
    ns = int(prm[f"Number of Slip Systems{sfx}"])
    twinning = prm.get(f"Twinning enabled{sfx}", "false").lower() == "true"
    nw = int(prm[f"Number of Twin Systems{sfx}"]) if twinning else 0
    C6 = np.vstack([floats(prm[f"Elastic Stiffness{sfx} row {i}"]) for i in range(1, 7)])
    d = dict(C6=C6, slip_normals=read_vectors(f(f"Slip Normals File{sfx}"), ns),
             slip_dirs=read_vectors(f(f"Slip Directions File{sfx}"), ns),
             q=read_q(f(f"Latent Hardening Ratio filename{sfx}"), ns + nw),
             s0=floats(prm[f"Initial Slip Resistance{sfx}"]), h0=floats(prm[f"Initial Hardening Modulus{sfx}"]),
             s_s=floats(prm[f"Saturation Stress{sfx}"]), a=floats(prm[f"Power Law Exponent{sfx}"]),
             twinning=np.int32(twinning))
    if prm.get(f"Enable Kinematic Hardening{sfx}", "false").lower() == "true":
        # backstress constants (userInputParameters.cc:274-296)
        d["c1"] = floats(prm[f"C_1 Slip Kinematic Hardening{sfx}"])
        d["c2"] = floats(prm[f"C_2 Slip Kinematic Hardening{sfx}"])
        if twinning:
            d["c1_twin"] = floats(prm[f"C_1 Twin Kinematic Hardening{sfx}"])
            d["c2_twin"] = floats(prm[f"C_2 Twin Kinematic Hardening{sfx}"])
    if twinning:
        d.update(twin_normals=read_vectors(f(f"Twin Normals File{sfx}"), nw),
                 twin_dirs=read_vectors(f(f"Twin Directions File{sfx}"), nw),
                 twin_s0=floats(prm[f"Initial Slip Resistance Twin{sfx}"]),
                 twin_h0=floats(prm[f"Initial Hardening Modulus Twin{sfx}"]),
                 twin_s_s=floats(prm[f"Saturation Stress Twin{sfx}"]),
                 twin_a=floats(prm[f"Power Law Exponent Twin{sfx}"]),
                 twin_threshold=float(prm[f"Twin Threshold Fraction{sfx}"]),
                 twin_saturation=float(prm[f"Twin Saturation Factor{sfx}"]),
                 twin_shear=float(prm[f"Characteristic Twin Shear{sfx}"]))
    return d


def load_deck(app_dir, golden=None):
    """Everything the harness needs from one application directory.
    ``golden``: optional path of a stress-strain file to attach as 'golden'.
    A multiphase deck's phases 2.. are stored under the prefixes 'ph2_',
    'ph3_', ..., with 'cell_phase' (1-based, per cell) from the fifth column
    of the orientations file (crystalPlasticity/init.cc:210-233)."""
    prm = parse_prm(os.path.join(app_dir, "prm.prm"))
    f = lambda key: os.path.join(app_dir, prm[key])
    d = _material(prm, f)
    d.update(tol=float(prm["Stress Tolerance"]),
             max_slip_search=int(prm["Max Slip Search Iterations"]),
             max_solver=int(prm["Max Solver Iterations"]),
             max_newton=int(prm["Maximum non linear iterations"]),
             delT=float(prm["Time increments"]), total_T=float(prm["Total time"]))
    n_phases = 1
    if prm.get("Enable Multiphase", "false").lower() == "true":
        n_phases = int(prm["Number of Phases"])
        d["multiphase"] = np.int32(1)
        for k in range(2, n_phases + 1):
            for key, v in _material(prm, f, f" {k}").items():
                d[f"ph{k}_{key}"] = v
    if "Maximum linear solver iterations" in prm:
        d["max_linear"] = int(prm["Maximum linear solver iterations"])
    if "Relative linear solver tolerance" in prm:
        d["rel_linear_tol"] = float(prm["Relative linear solver tolerance"])
    # mesh: the subdivided unit cube, refined 'Refine factor' times
    subdiv = [int(prm[f"Subdivisions {a}"]) for a in "XYZ"]
    span = [float(prm[f"Domain size {a}"]) for a in "XYZ"]
    if span != [1.0, 1.0, 1.0]:
        raise ValueError("only the unit-cube domain is supported")
    ne = [s * 2 ** int(prm["Refine factor"]) for s in subdiv]
    # voxel grain ids: x outer, y middle (one line per (x, y)), z inner
    npts = [int(float(prm[f"Voxels in {a} direction"])) for a in "XYZ"]
    lines = open(f("Grain ID file name")).read().splitlines()
    hdr = int(prm["Header Lines GrainID File"])
    data = lines[hdr: hdr + npts[0] * npts[1]]
    vox = np.array([[int(float(x)) for x in ln.split()[: npts[2]]] for ln in data]).reshape(npts)
    orient, phase_of = {}, {}
    for ln in open(f("Orientations file name")).read().splitlines()[1:]:
        g = ln.split()
        if len(g) >= 4:
            orient[int(g[0])] = [float(g[1]), float(g[2]), float(g[3])]
            phase_of[int(g[0])] = int(float(g[4])) if (n_phases > 1 and len(g) >= 5) else 1
    # cells in lexicographic order, x fastest
    rod = np.zeros((ne[0] * ne[1] * ne[2], 3))
    cell_phase = np.ones(ne[0] * ne[1] * ne[2], dtype=np.int32)
    for kz in range(ne[2]):
        for ky in range(ne[1]):
            for kx in range(ne[0]):
                c = [(kx + 0.5) / ne[0], (ky + 0.5) / ne[1], (kz + 0.5) / ne[2]]
                vi = [nearest_index(c[a], npts[a]) for a in range(3)]
                gid = int(vox[vi[0], vi[1], vi[2]])
                rod[kx + ne[0] * (ky + ne[1] * kz)] = orient[gid]
                cell_phase[kx + ne[0] * (ky + ne[1] * kz)] = phase_of[gid]
    d.update(n_elem=np.array(ne), cell_rodrigues=rod, n_grains=len(orient))
    if n_phases > 1:
        d["cell_phase"] = cell_phase
    flag = lambda key, default="false": prm.get(key, default).lower() == "true"
    if flag("Use velocity gradient BC"):
        # the whole boundary follows (I - L dt)^-1 per increment
        # (userInputParameters.cc:80-82, updateBeforeIncrement.cc:10-30)
        d["vel_grad"] = np.vstack([floats(prm[f"Velocity gradient row {i}"]) for i in range(1, 4)])
    elif flag("Use Tabular BCs"):
        # rows: face, dof, displacement at each time of the table
        # (ellipticBVP/init.cc:388-408)
        nt = int(prm["Number of time data for Tabular BCs"])
        rows = []
        for ln in open(f("Tabular Boundary condition filename")).read().splitlines():
            g = ln.split()
            if len(rows) == int(prm["Number of tabular boundary conditions"]):
                break
            if len(g) >= 2 + nt:
                rows.append([float(x) for x in g[: 2 + nt]])
        d["tab_bc"] = np.array(rows)
        d["tab_times"] = floats(prm["Tabular Time Table"])
    else:
        bl = open(f("Boundary condition filename")).read().splitlines()
        nh = int(prm["BC file number of header lines"])
        bc = [[int(g[0]), int(g[1]), float(g[2])] for g in (ln.split() for ln in bl[nh: nh + int(
            prm["Number of boundary conditions"])])]
        d["bc"] = np.array(bc)
        if flag("Enable cyclic loading"):
            d["cyclic"] = np.array([float(prm["Cyclic loading face"]), float(prm["Cyclic loading direction"]),
                                    float(prm["Quarter cycle time"])])
    if golden is not None:
        d["golden"] = np.loadtxt(golden, skiprows=1)
    return d
