"""Lattice tables and material constants (host side).

The reference reads slip/twin normals and directions from text files and
normalises each vector on load (src/materialModels/crystalPlasticity/
init.cc:72-176), reads the latent-hardening matrix for the real systems only
(init.cc:49-65) and, with twinning off, appends one dummy twin system
(init.cc:37-41,178-185; userInputParameters.cc:303-311).  ``build_material``
does the same from arrays; the tables here are generated from Miller /
Miller-Bravais indices (crystallography, not copied data):

* FCC  12 {111}<110>                       (ordered as the reference's fcc decks)
* BCC  48 = 12 {110}<111> + 12 {112}<111> + 24 {123}<111>
* HCP  30 = 3 basal + 3 prismatic + 6 pyramidal<a> + 12 pyramidal<c+a>
           + 6 {10-12}<-1011> tension twins (c/a = 1.624)
"""
from __future__ import annotations

import itertools

import numpy as np

from .capi import CP_MAX_SYSTEMS, CpMaterial


def _unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.sqrt(np.sum(v * v))


def normalise_rows(a):
    """init.cc:82-90: n <- n / sqrt(n0^2 + n1^2 + n2^2), accumulated in order."""
    a = np.asarray(a, dtype=np.float64).copy()
    for r in a:
        s = 0.0
        s = s + r[0] * r[0]
        s = s + r[1] * r[1]
        s = s + r[2] * r[2]
        s = np.sqrt(s)
        r[:] = r / s
    return a


# ---------------------------------------------------------------------------
# FCC {111}<110>, ordered plane by plane as in the reference's fcc decks
def fcc_systems():
    planes = [(1, 1, 1), (-1, -1, 1), (-1, 1, 1), (1, -1, 1)]
    dirs = [
        [(0, 1, -1), (-1, 0, 1), (1, -1, 0)],
        [(0, -1, -1), (1, 0, 1), (-1, 1, 0)],
        [(0, 1, -1), (1, 0, 1), (-1, -1, 0)],
        [(0, -1, -1), (-1, 0, 1), (1, 1, 0)],
    ]
    n, m = [], []
    for p, ds in zip(planes, dirs):
        for d in ds:
            assert np.dot(p, d) == 0
            n.append(p)
            m.append(d)
    return normalise_rows(n), normalise_rows(m)


def _signed_perms(v):
    out = set()
    for p in itertools.permutations(v):
        for s in itertools.product((1, -1), repeat=3):
            out.add(tuple(int(a * b) for a, b in zip(p, s)))
    return sorted(out)


def _canon(v):
    """Representative of +-v: first nonzero component positive."""
    v = tuple(v)
    for c in v:
        if c != 0:
            return v if c > 0 else tuple(-x for x in v)
    return v


def bcc_systems():
    """48 systems: {110}<111>, {112}<111>, {123}<111> (plane, direction) pairs
    with n.d = 0, each plane/direction pair counted once up to a common sign."""
    dirs = sorted({_canon(d) for d in _signed_perms((1, 1, 1))})
    n, m = [], []
    for fam in [(1, 1, 0), (1, 1, 2), (1, 2, 3)]:
        planes = sorted({_canon(p) for p in _signed_perms(fam)})
        for p in planes:
            for d in dirs:
                if np.dot(p, d) == 0:
                    n.append(p)
                    m.append(d)
    assert len(n) == 48, len(n)
    return normalise_rows(n), normalise_rows(m)


# ---------------------------------------------------------------------------
# HCP via Miller-Bravais indices
def hex_dir(uvtw, c_over_a):
    u, v, t, w = uvtw
    a1 = np.array([1.0, 0.0, 0.0])
    a2 = np.array([-0.5, np.sqrt(3.0) / 2.0, 0.0])
    a3 = -(a1 + a2)
    c = np.array([0.0, 0.0, c_over_a])
    return u * a1 + v * a2 + t * a3 + w * c


def hex_plane(hkil, c_over_a):
    h, k, i, l = hkil
    assert h + k + i == 0
    a1s = np.array([1.0, 1.0 / np.sqrt(3.0), 0.0])
    a2s = np.array([0.0, 2.0 / np.sqrt(3.0), 0.0])
    cs = np.array([0.0, 0.0, 1.0 / c_over_a])
    return h * a1s + k * a2s + l * cs


def _hex_family(base, with_l_sign=True):
    """All (h,k,i,l) obtained by permuting the first three indices and
    flipping signs consistently (hexagonal point group 6/mmm)."""
    h, k, i, l = base
    out = set()
    for p in itertools.permutations((h, k, i)):
        for s in (1, -1):
            for sl in ((1, -1) if with_l_sign else (1,)):
                out.add((s * p[0], s * p[1], s * p[2], sl * l))
    return sorted(out)


def hcp_systems(c_over_a=1.624):
    """Returns normals, directions (unit) and group labels
    basal(3) prism(3) pyr<a>(6) pyr<c+a>(12) twin(6)."""
    systems = []

    def add(group, plane_fam, dir_fam, unique_dir_sign=True, twin=False):
        planes = _hex_family(plane_fam)
        dirs = _hex_family(dir_fam)
        got = []
        seen = set()
        for p in planes:
            np_ = hex_plane(p, c_over_a)
            if np_[2] < -1e-12 or (abs(np_[2]) < 1e-12 and _canon(tuple(np.round(np_, 9))) != tuple(np.round(np_, 9))):
                continue  # one representative per plane (upper half space)
            for d in dirs:
                dv = hex_dir(d, c_over_a)
                if abs(np.dot(np_, dv)) > 1e-9:
                    continue
                if twin:
                    # twinning shear is one-directional: keep the sense giving c-axis extension
                    if dv[2] * np_[2] <= 0:
                        continue
                elif unique_dir_sign:
                    cd = _canon(tuple(np.round(dv, 9)))
                    if cd != tuple(np.round(dv, 9)):
                        continue
                key = (tuple(np.round(_unit(np_), 9)), tuple(np.round(_unit(dv), 9)))
                if key in seen:
                    continue
                seen.add(key)
                got.append((np_, dv))
        got.sort(key=lambda t: (round(-_unit(t[0])[2], 6), round(np.arctan2(t[0][1], t[0][0]), 6),
                                round(np.arctan2(t[1][1], t[1][0]), 6), round(t[1][2], 6)))
        for np_, dv in got:
            systems.append((group, _unit(np_), _unit(dv)))
        return len(got)

    nb = add("basal", (0, 0, 0, 1), (2, -1, -1, 0))
    npr = add("prism", (1, 0, -1, 0), (1, 1, -2, 0))
    npa = add("pyr_a", (1, 0, -1, 1), (1, 1, -2, 0))
    npc = add("pyr_ca", (1, 0, -1, 1), (1, 1, -2, 3))
    ntw = add("twin", (1, 0, -1, 2), (-1, 0, 1, 1), twin=True)
    assert (nb, npr, npa, npc, ntw) == (3, 3, 6, 12, 6), (nb, npr, npa, npc, ntw)
    groups = [s[0] for s in systems]
    n = normalise_rows([s[1] for s in systems])
    m = normalise_rows([s[2] for s in systems])
    return n, m, groups


def coplanar_latent_matrix(normals, self_ratio=1.0, latent_ratio=1.4):
    """q = 1 between systems sharing a slip plane and 1.4 otherwise, as in the
    reference's fcc LatentHardeningRatio.txt."""
    n = len(normals)
    q = np.full((n, n), latent_ratio)
    for a in range(n):
        for b in range(n):
            if abs(abs(np.dot(normals[a], normals[b])) - 1.0) < 1e-9:
                q[a, b] = self_ratio
    return q


def cubic_stiffness(c11, c12, c44):
    C = np.zeros((6, 6))
    C[:3, :3] = c12
    np.fill_diagonal(C[:3, :3], c11)
    C[3, 3] = C[4, 4] = C[5, 5] = c44
    return C


def hex_stiffness(c11, c12, c13, c33, c44, c66):
    C = np.zeros((6, 6))
    C[0, 0] = C[1, 1] = c11
    C[2, 2] = c33
    C[0, 1] = C[1, 0] = c12
    C[0, 2] = C[2, 0] = C[1, 2] = C[2, 1] = c13
    C[3, 3] = C[4, 4] = c44
    C[5, 5] = c66
    return C


def build_material(C6, slip_normals, slip_dirs, q, s0, h0, s_s, a, *, twin_normals=None,
                   twin_dirs=None, twin_s0=None, twin_h0=None, twin_s_s=None, twin_a=None,
                   q_full=None, twin_threshold=0.0, twin_saturation=0.0, twin_shear=1.0,
                   c1=None, c2=None, normalise=True) -> CpMaterial:
    """Fill a cp_material_t the way init.cc / userInputParameters.cc do.

    ``q`` is the n_slip x n_slip (or, with twins, the full real-system)
    latent-hardening matrix; with twinning off the dummy twin row/column is 0.
    """
    mat = CpMaterial()
    ns = len(slip_normals)
    sn = normalise_rows(slip_normals) if normalise else np.asarray(slip_normals, float)
    sd = normalise_rows(slip_dirs) if normalise else np.asarray(slip_dirs, float)
    twinning = twin_normals is not None
    if twinning:
        nw = len(twin_normals)
        tn = normalise_rows(twin_normals) if normalise else np.asarray(twin_normals, float)
        td = normalise_rows(twin_dirs) if normalise else np.asarray(twin_dirs, float)
    else:
        nw = 1
        tn = np.array([[1.0, 0.0, 0.0]])
        td = np.array([[0.0, 1.0, 0.0]])
    n = ns + nw
    assert n <= CP_MAX_SYSTEMS
    mat.n_slip = ns
    mat.n_twin = nw
    mat.twinning_enabled = 1 if twinning else 0
    C6 = np.asarray(C6, float).reshape(6, 6)
    for i in range(36):
        mat.elastic_stiffness[i] = C6.flat[i]
    allN = np.vstack([sn, tn])
    allM = np.vstack([sd, td])
    for i in range(n):
        for j in range(3):
            mat.slip_normal[3 * i + j] = allN[i, j]
            mat.slip_direction[3 * i + j] = allM[i, j]
    qq = np.zeros((n, n))
    qin = np.asarray(q_full if q_full is not None else q, float)
    n_real = n if twinning else ns
    qq[:n_real, :n_real] = qin[:n_real, :n_real]
    for i in range(n):
        for j in range(n):
            mat.latent_hardening[i * CP_MAX_SYSTEMS + j] = qq[i, j]

    def vec(x, k):
        x = np.broadcast_to(np.asarray(x, float), (k,))
        return x

    s0v, h0v, ssv, av = vec(s0, ns), vec(h0, ns), vec(s_s, ns), vec(a, ns)
    if twinning:
        ts0, th0, tss, ta = vec(twin_s0, nw), vec(twin_h0, nw), vec(twin_s_s, nw), vec(twin_a, nw)
    else:
        # userInputParameters.cc:303-311
        ts0, th0, tss, ta = [10e14], [1.0], [10e15], [0.0]
    for i in range(ns):
        mat.initial_slip_resistance[i] = s0v[i]
        mat.initial_hardening_modulus[i] = h0v[i]
        mat.saturation_stress[i] = ssv[i]
        mat.power_law_exponent[i] = av[i]
    for i in range(nw):
        mat.initial_slip_resistance[ns + i] = ts0[i]
        mat.initial_hardening_modulus[ns + i] = th0[i]
        mat.saturation_stress[ns + i] = tss[i]
        mat.power_law_exponent[ns + i] = ta[i]
    if c1 is not None:
        c1v, c2v = vec(c1, n), vec(c2, n)
        for i in range(n):
            mat.kinematic_c1[i] = c1v[i]
            mat.kinematic_c2[i] = c2v[i]
    mat.twin_threshold_fraction = twin_threshold
    mat.twin_saturation_factor = twin_saturation
    mat.twin_shear = twin_shear
    return mat


def material_arrays(mat: CpMaterial):
    """numpy views of a material (for host-side checks)."""
    n = mat.n_total
    N = np.ctypeslib.as_array(mat.slip_normal)[: 3 * n].reshape(n, 3)
    M = np.ctypeslib.as_array(mat.slip_direction)[: 3 * n].reshape(n, 3)
    q = np.ctypeslib.as_array(mat.latent_hardening).reshape(CP_MAX_SYSTEMS, CP_MAX_SYSTEMS)[:n, :n]
    s0 = np.ctypeslib.as_array(mat.initial_slip_resistance)[:n]
    return {"n": N, "m": M, "q": q, "s0": s0,
            "C": np.ctypeslib.as_array(mat.elastic_stiffness).reshape(6, 6)}


# ---------------------------------------------------------------------------
# the benchmark lattices (FCC Cu, BCC, HCP Mg-like)
def fcc_cu():
    """FCC Cu: C11/C12/C44 = 170/124/75 GPa, s0 16, h0 180, s_s 148, a 2.25 MPa,
    q 1.4 / 1 coplanar, twinning off (dummy twin appended)."""
    n, m = fcc_systems()
    q = coplanar_latent_matrix(n)
    return build_material(cubic_stiffness(170.0e3, 124.0e3, 75.0e3), n, m, q, 16.0, 180.0, 148.0, 2.25)


def bcc_48():
    """BCC, 48 systems: C11/C12/C44 = 231.4/134.7/116.4 GPa, CRSS 50 MPa,
    h0/s_s/a as FCC (180/148/2.25), q 1.4 / 1 coplanar, twinning off."""
    n, m = bcc_systems()
    q = coplanar_latent_matrix(n)
    return build_material(cubic_stiffness(231.4e3, 134.7e3, 116.4e3), n, m, q, 50.0, 180.0, 148.0, 2.25)


HCP_GROUP_S0 = {"basal": 5.0, "prism": 40.0, "pyr_a": 40.0, "pyr_ca": 80.0, "twin": 15.0}
HCP_GROUP_SS = {"basal": 95.0, "prism": 135.0, "pyr_a": 135.0, "pyr_ca": 420.0, "twin": 220.0}
HCP_GROUP_A = {"basal": 0.0, "prism": 6.0, "pyr_a": 6.0, "pyr_ca": 6.0, "twin": 0.75}
HCP_GROUP_H0 = {"basal": 150.0, "prism": 150.0, "pyr_a": 150.0, "pyr_ca": 150.0, "twin": 10.0}


def hcp_mg(twin_threshold=0.7, twin_saturation=0.0):
    """HCP Mg-like, 24 slip + 6 twins (c/a 1.624), Mg elastic constants and
    hardening from the reference's hcp/simpleTension deck; CRSS 5/40/40/80/15."""
    n, m, groups = hcp_systems()
    slip = [i for i, g in enumerate(groups) if g != "twin"]
    twin = [i for i, g in enumerate(groups) if g == "twin"]
    q = coplanar_latent_matrix(n)
    gs = [groups[i] for i in slip]
    gt = [groups[i] for i in twin]
    return build_material(
        hex_stiffness(59.3e3, 25.7e3, 21.4e3, 61.5e3, 16.4e3, 16.8e3),
        n[slip], m[slip], None,
        [HCP_GROUP_S0[g] for g in gs], [HCP_GROUP_H0[g] for g in gs],
        [HCP_GROUP_SS[g] for g in gs], [HCP_GROUP_A[g] for g in gs],
        twin_normals=n[twin], twin_dirs=m[twin],
        twin_s0=[HCP_GROUP_S0[g] for g in gt], twin_h0=[HCP_GROUP_H0[g] for g in gt],
        twin_s_s=[HCP_GROUP_SS[g] for g in gt], twin_a=[HCP_GROUP_A[g] for g in gt],
        q_full=q, twin_threshold=twin_threshold, twin_saturation=twin_saturation, twin_shear=0.129)


def random_rodrigues(rng: np.random.Generator, count: int):
    """Uniform random orientations: normalised N(0, I4) quaternion with
    q0 >= 0, converted to Rodrigues r = q[1:4]/q0 (the quat2rod clamp
    |q0| >= 1e-4 of updateAfterIncrement.cc:813-815 applied)."""
    q = rng.standard_normal((count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q[q[:, 0] < 0] *= -1.0
    q0 = np.where(np.abs(q[:, 0]) < 1e-4, 1e-4, q[:, 0])
    return q[:, 1:] / q0[:, None]


def material_from_deck(d, phase: int = 1) -> CpMaterial:
    """A material from a parsed reference input deck (the dict stored in
    tests/golden/kat_*.npz: prm values plus slip/twin/q tables); phase k > 1
    of a multiphase deck reads the keys stored under the prefix 'ph<k>_'."""
    if phase > 1:
        pre = f"ph{phase}_"
        d = {k[len(pre):]: v for k, v in d.items() if k.startswith(pre)}
    kw = {}
    if int(d["twinning"]):
        kw = dict(twin_normals=d["twin_normals"], twin_dirs=d["twin_dirs"], twin_s0=d["twin_s0"],
                  twin_h0=d["twin_h0"], twin_s_s=d["twin_s_s"], twin_a=d["twin_a"],
                  q_full=d["q"], twin_threshold=float(d["twin_threshold"]),
                  twin_saturation=float(d["twin_saturation"]), twin_shear=float(d["twin_shear"]))
    if "c1" in d:
        # backstress constants of the slip systems, then of the twins (0 for the
        # dummy twin of twinning off, userInputParameters.cc:303-311)
        nw = len(d["twin_normals"]) if int(d["twinning"]) else 1
        tw1 = d["c1_twin"] if "c1_twin" in d else np.zeros(nw)
        tw2 = d["c2_twin"] if "c2_twin" in d else np.zeros(nw)
        kw.update(c1=np.concatenate([d["c1"], tw1]), c2=np.concatenate([d["c2"], tw2]))
    return build_material(d["C6"], d["slip_normals"], d["slip_dirs"], d["q"], d["s0"], d["h0"],
                          d["s_s"], d["a"], **kw)
