"""Host Newton harness: a minimal restatement of the reference's ellipticBVP
driver around the qp hot path.

It plays the part of the deal.II caller of the C ABI.  Reference pieces it
restates (paths under src/):

* mesh: subdivided unit cube refined ``r`` times -> n x n x n Q1 hexahedra
  (ellipticBVP/mesh.cc:32,101), QGauss(2) -> 8 qps per cell, FESystem dof
  ordering (local dof d = 3*vertex + component, vertices lexicographic);
* Dirichlet BCs from a (face, dof, total displacement) table
  (ellipticBVP/boundaryConditions.cc:79-118): the value is applied at Newton
  iteration 0 only, 0 afterwards (boundaryConditions.cc:485-490), with
  deluConstraint = totalU / totalIncrements (ellipticBVP/init.cc:326-343);
* exactly ``max_newton`` assemble+solve passes per increment, no convergence
  test (ellipticBVP/solveNonLinearSystem.cc:14-81);
* the increment commit of updateAfterIncrement.cc: post-pass update with
  StiffnessCalFlag 0 (:105), volume averages (:119-126,218-235,710-722),
  reorient (:291), *_iter -> *_conv (:298-305), and the stressstrain.txt
  row (:733-771).

The Newton-step linear system is solved directly (sparse LU) on the host; the
reference uses PETSc BiCG + Jacobi to 1e-10 relative residual
(ellipticBVP/solveLinearSystem.cc:14-16).

The backend is any object with the CpHandle method set (the GPU library, or
in tests the CPU oracle).
"""
from __future__ import annotations

import dataclasses

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

GAUSS = (0.5 - 0.5 / np.sqrt(3.0), 0.5 + 0.5 / np.sqrt(3.0))


def q1_reference_gradients():
    """d N_a / d xi at the 8 Gauss points of the unit reference cube:
    array [q][a][3], q and a lexicographic (x fastest)."""
    g = np.zeros((8, 8, 3))
    for q in range(8):
        xi = (GAUSS[q & 1], GAUSS[(q >> 1) & 1], GAUSS[(q >> 2) & 1])
        for a in range(8):
            bits = (a & 1, (a >> 1) & 1, (a >> 2) & 1)
            f = [xi[d] if bits[d] else 1.0 - xi[d] for d in range(3)]
            df = [1.0 if bits[d] else -1.0 for d in range(3)]
            g[q, a, 0] = df[0] * f[1] * f[2]
            g[q, a, 1] = f[0] * df[1] * f[2]
            g[q, a, 2] = f[0] * f[1] * df[2]
    return g


@dataclasses.dataclass
class StructuredMesh:
    """n[0] x n[1] x n[2] uniform Q1 cells on [0,1]^3."""

    n: tuple

    def __post_init__(self):
        nx, ny, nz = self.n
        self.h = np.array([1.0 / nx, 1.0 / ny, 1.0 / nz])
        self.n_nodes = (nx + 1) * (ny + 1) * (nz + 1)
        self.n_dofs = 3 * self.n_nodes
        self.n_cells = nx * ny * nz
        ix, iy, iz = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
        node_id = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)
        self.node_xyz = np.zeros((self.n_nodes, 3))
        nid = node_id(ix, iy, iz)
        self.node_xyz[nid.ravel(), 0] = ix.ravel() * self.h[0]
        self.node_xyz[nid.ravel(), 1] = iy.ravel() * self.h[1]
        self.node_xyz[nid.ravel(), 2] = iz.ravel() * self.h[2]
        cells = []
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    cells.append([node_id(i + (a & 1), j + ((a >> 1) & 1), k + ((a >> 2) & 1)) for a in range(8)])
        self.cell_nodes = np.array(cells, dtype=np.int64)
        self.cell_dofs = (3 * self.cell_nodes[:, :, None] + np.arange(3)).reshape(self.n_cells, 24)
        gref = q1_reference_gradients()
        self.grad_N = gref / self.h  # uniform mesh: [q][a][3]
        self.JxW = np.full(8, np.prod(self.h) / 8.0)
        self._pattern = False  # the host CSR pattern, built on first use (the device system needs none)

    def cell_centres(self):
        return self.node_xyz[self.cell_nodes].mean(axis=1)

    def _build_pattern(self):
        if self._pattern:
            return
        self._pattern = True
        rows = np.repeat(self.cell_dofs, 24, axis=1).ravel()
        cols = np.tile(self.cell_dofs, (1, 24)).ravel()
        lin = rows * self.n_dofs + cols
        uniq, inv = np.unique(lin, return_inverse=True)
        self._pos = inv
        self._nnz = len(uniq)
        r = uniq // self.n_dofs
        c = uniq % self.n_dofs
        self._indptr = np.searchsorted(r, np.arange(self.n_dofs + 1))
        self._indices = c.astype(np.int32)
        self._rows = r

    def assemble_matrix(self, Ke):
        self._build_pattern()
        data = np.bincount(self._pos, weights=np.asarray(Ke).ravel(), minlength=self._nnz)
        return sp.csr_matrix((data, self._indices, self._indptr), shape=(self.n_dofs, self.n_dofs))

    def assemble_vector(self, Re):
        return np.bincount(self.cell_dofs.ravel(), weights=np.asarray(Re).ravel(), minlength=self.n_dofs)

    def deformation_gradients(self, u):
        """F = I + sum_d U_d grad N_d at every qp (getElementalValues.cc:129-138);
        returns [cell*8 + q][9]."""
        Ul = u[self.cell_dofs].reshape(self.n_cells, 8, 3)  # [cell][a][comp]
        F = np.einsum("cai,qaj->cqij", Ul, self.grad_N)
        F += np.eye(3)
        return F.reshape(-1, 9)


def face_nodes(mesh: StructuredMesh, face: int, eps: float = 1e-5):
    """Faces 1..6 = x=0, x=1, y=0, y=1, z=0, z=1 (boundaryConditions.cc:84-111)."""
    axis = (face - 1) // 2
    x = mesh.node_xyz[:, axis]
    return np.nonzero(x <= eps)[0] if face % 2 == 1 else np.nonzero(x >= 1.0 - eps)[0]


def dirichlet_increments(mesh: StructuredMesh, bc_table, n_increments: int):
    """Constrained dofs and their per-increment values.  A node on several
    constrained faces takes the value of the lowest face id, as the early
    return in setBoundaryValues does (boundaryConditions.cc:79-113)."""
    constrained = {}
    rows = sorted([(int(f), int(d), float(u)) for f, d, u in bc_table])
    for face in range(1, 7):
        for f, dof, total in rows:
            if f != face:
                continue
            for nd in face_nodes(mesh, face):
                gd = 3 * nd + (dof - 1)
                if gd not in constrained:
                    constrained[gd] = total / n_increments
    dofs = np.array(sorted(constrained), dtype=np.int64)
    vals = np.array([constrained[d] for d in dofs])
    return dofs, vals


def face_precedence(mesh: StructuredMesh, pairs):
    """Constrained dof -> the (face, dof) entry that sets it: a node on several
    constrained faces takes the lowest face id, as the early return in
    setBoundaryValues does (boundaryConditions.cc:79-113, :148-246)."""
    owner = {}
    for face in range(1, 7):
        for f, dof in sorted(set((int(f), int(d)) for f, d in pairs)):
            if f != face:
                continue
            for nd in face_nodes(mesh, face):
                owner.setdefault(3 * nd + (dof - 1), (f, dof))
    dofs = np.array(sorted(owner), dtype=np.int64)
    return dofs, [owner[d] for d in dofs]


class CyclicLoading:
    """Simple face BCs plus one cyclic (face, dof): its nodes move by
    +-du_c per increment, du_c = U_total dt / t_quarter, positive while
    fmod(k dt, 4 t_quarter) < t_quarter or >= 3 t_quarter, negative between
    (boundaryConditions.cc:15-77; ellipticBVP/init.cc:326-346; cycle time
    ellipticBVP.cc:39).  The cyclic dof is checked before the face table, so
    its nodes take it whatever other face they lie on."""

    def __init__(self, mesh, bc_table, n_increments, delT, face, dof, quarter):
        self.k = 0
        self.delT, self.quarter = float(delT), float(quarter)
        total = {(int(f), int(d)): float(u) for f, d, u in bc_table}
        cyc = set(3 * face_nodes(mesh, int(face)) + (int(dof) - 1))
        base_dofs, base_vals = dirichlet_increments(mesh, bc_table, n_increments)
        vals = {int(g): v for g, v in zip(base_dofs, base_vals)}
        self.du_c = total.get((int(face), int(dof)), 0.0) / n_increments * n_increments * self.delT / self.quarter
        self.dofs = np.array(sorted(set(vals) | cyc), dtype=np.int64)
        self.is_cyc = np.array([g in cyc for g in self.dofs])
        self.base = np.array([0.0 if g in cyc else vals[g] for g in self.dofs])

    def next_values(self, mesh, dofs):
        r = math.fmod(self.k * self.delT, 4 * self.quarter)
        sign = 1.0 if r < self.quarter else (-1.0 if r < 3 * self.quarter else 1.0)
        self.k += 1
        return np.where(self.is_cyc, sign * self.du_c, self.base)


class TabularLoading:
    """Piecewise-linear face displacements: rows (face, dof, U at the times of
    the time table); in increment k (time (k+1) dt) a constrained dof moves by
    dt times the slope of its row on the current time interval, the interval
    advancing once the time passes its end (boundaryConditions.cc:148-246;
    ellipticBVP/init.cc:388-408)."""

    def __init__(self, mesh, rows, times, delT):
        self.rows = {(int(r[0]), int(r[1])): np.asarray(r[2:], float) for r in rows}
        self.times = np.asarray(times, float)
        self.delT = float(delT)
        self.k = 0
        self.tc = 1
        self.dofs, owners = face_precedence(mesh, list(self.rows))
        self.owners = owners

    def next_values(self, mesh, dofs):
        t = self.delT * (self.k + 1)
        if self.k == 0:
            self.tc = 1
        while self.tc + 1 < len(self.times) and t > self.times[self.tc]:
            self.tc += 1
        self.k += 1
        tc, T = self.tc, self.times
        slope = {key: (u[tc] - u[tc - 1]) / (T[tc] - T[tc - 1]) * self.delT for key, u in self.rows.items()}
        return np.array([slope[o] for o in self.owners])


def boundary_dofs(mesh: StructuredMesh, eps: float = 1e-5):
    """Every dof of every node on the cube's surface: the velocity-gradient
    boundary condition sets all of them (setBoundaryValues,
    boundaryConditions.cc:269-274, which applyDirichletBCs calls for each dof
    of each boundary face, :453-497)."""
    x = mesh.node_xyz
    nodes = np.nonzero(((x <= eps) | (x >= 1.0 - eps)).any(axis=1))[0]
    return (3 * nodes[:, None] + np.arange(3)[None, :]).ravel().astype(np.int64)


class VelocityGradientLoading:
    """Macroscopic velocity gradient L applied in steps dt: before increment k,
    F_k = (I - L dt)^-1 F_{k-1} with F_0 = I (updateBeforeIncrement.cc:10-30,
    ellipticBVP/init.cc:551), and the boundary node at X moves by
    (F_k - F_{k-1}) X in the increment's first Newton pass
    (boundaryConditions.cc:269-274)."""

    def __init__(self, L, dt):
        self.L = np.asarray(L, dtype=np.float64).reshape(3, 3)
        self.dt = float(dt)
        self.F = np.eye(3)

    def next_values(self, mesh: StructuredMesh, dofs):
        F_new = np.linalg.inv(np.eye(3) - self.L * self.dt) @ self.F
        dF = F_new - self.F
        self.F = F_new
        X = mesh.node_xyz[dofs // 3]
        return (X @ dF.T)[np.arange(len(dofs)), dofs % 3]


def von_mises_rows(rows):
    """run_compile_tests.py:45-48 on stressstrain rows."""
    r = np.asarray(rows)
    e = np.sqrt(0.5 * ((r[:, 0] - r[:, 1]) ** 2 + (r[:, 1] - r[:, 2]) ** 2 + (r[:, 2] - r[:, 0]) ** 2
                       + 6 * (r[:, 3] ** 2 + r[:, 4] ** 2 + r[:, 5] ** 2)))
    s = np.sqrt(0.5 * ((r[:, 6] - r[:, 7]) ** 2 + (r[:, 7] - r[:, 8]) ** 2 + (r[:, 8] - r[:, 6]) ** 2
                       + 6 * (r[:, 9] ** 2 + r[:, 10] ** 2 + r[:, 11] ** 2)))
    return e, s


def golden_errors(new_rows, old_rows, check_rows):
    """The reference's pass criterion (run_compile_tests.py:55-60): max relative
    error of von Mises strain, von Mises stress and SlipTotal over the first
    ``check_rows`` rows, nan -> 0 and inf -> max float as np.nan_to_num does."""
    n = min(check_rows, len(new_rows), len(old_rows))
    oe, os_ = von_mises_rows(old_rows[:n])
    ne, ns = von_mises_rows(new_rows[:n])
    with np.errstate(divide="ignore", invalid="ignore"):
        err = lambda a, b: float(np.max(np.nan_to_num(np.abs((a - b) / a))))
        return {"strain": err(oe, ne), "stress": err(os_, ns),
                "slip": err(np.asarray(old_rows)[:n, 14], np.asarray(new_rows)[:n, 14]),
                "twin": err(np.asarray(old_rows)[:n, 13], np.asarray(new_rows)[:n, 13]), "rows": n}


class NewtonHarness:
    """Fixed-iteration Newton loop over a structured Q1 mesh."""

    def __init__(self, backend, mesh: StructuredMesh, bc_table, n_increments: int, max_newton: int = 4,
                 multiphase: bool = False, device_system: bool = False, solver=None, vel_grad=None, delT=None,
                 cyclic=None, tabular=None):
        """device_system: run the global system on the GPU (cp_bind_dofs /
        cp_newton_iteration / cp_update_from_displacement) with 'solver'
        (capi.CpSolver, default BiCG 1e-10); otherwise assemble on the
        backend and solve on the host with a sparse LU.  Boundary conditions:
        bc_table (face, dof, total displacement), plus cyclic = (face, dof,
        quarter-cycle time) for cyclic loading; or tabular = (rows, times);
        or vel_grad (3x3); delT is the time step of the last three."""
        self.be = backend
        self.device_system = device_system
        self.solver = solver
        self.solve_info = []
        self.mesh = mesh
        self.n_increments = n_increments
        self.max_newton = max_newton
        self.multiphase = multiphase
        if vel_grad is not None:
            self.loading = VelocityGradientLoading(vel_grad, delT)
            self.cdofs = boundary_dofs(mesh)
            self.cvals = np.zeros(len(self.cdofs))
        elif tabular is not None:
            self.loading = TabularLoading(mesh, tabular[0], tabular[1], delT)
            self.cdofs = self.loading.dofs
            self.cvals = np.zeros(len(self.cdofs))
        elif cyclic is not None:
            self.loading = CyclicLoading(mesh, bc_table, n_increments, delT, *cyclic)
            self.cdofs = self.loading.dofs
            self.cvals = np.zeros(len(self.cdofs))
        else:
            self.loading = None
            self.cdofs, self.cvals = dirichlet_increments(mesh, bc_table, n_increments)
        self.u = np.zeros(mesh.n_dofs)
        self.F_e = 0.0
        self.F_r = 0.0
        self.rows = []
        mask = np.zeros(mesh.n_dofs, dtype=bool)
        mask[self.cdofs] = True
        self.cmask = mask
        self._zero_entries = None  # host condensation mask, built on first host solve
        self._diag = None
        backend.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
        if device_system:
            backend.bind_dofs(mesh.n_dofs, mesh.cell_dofs, self.cdofs)

    def _solve(self, K, R, duc):
        """K du = R with du[c] = duc (constraints condensed as deal.II's
        distribute_local_to_global with inhomogeneities does)."""
        du_full = np.zeros(self.mesh.n_dofs)
        du_full[self.cdofs] = duc
        rhs = R - K @ du_full
        if self._zero_entries is None:
            self.mesh._build_pattern()
            self._zero_entries = self.cmask[self.mesh._rows] | self.cmask[self.mesh._indices]
        K = K.copy()
        K.data[self._zero_entries] = 0.0
        K = K + sp.diags(self.cmask.astype(float))
        rhs[self.cdofs] = duc
        return spla.splu(K.tocsc()).solve(rhs)

    def begin_increment(self):
        """The increment's prescribed boundary values (moving boundaries)."""
        if self.loading is not None:
            self.cvals = self.loading.next_values(self.mesh, self.cdofs)

    def constrained_increment(self, it):
        """What Newton pass 'it' prescribes on the constrained dofs (the whole
        increment on the first pass, nothing after)."""
        return self.cvals if it == 0 else None

    def step(self):
        """One increment: max_newton assemble+solve passes, then the commit."""
        mesh = self.mesh
        self.begin_increment()
        if self.device_system:
            for it in range(self.max_newton):
                self.solve_info.append(self.be.newton_iteration(self.constrained_increment(it), self.F_e, self.F_r,
                                                                self.solver))
            self.be.update_from_displacement(self.F_e, self.F_r)
            return self.finish_increment()
        else:
            for it in range(self.max_newton):
                Ke, Re, st = self.be.assemble(self.u[mesh.cell_dofs], self.F_e, self.F_r)
                K = mesh.assemble_matrix(Ke)
                R = mesh.assemble_vector(Re)
                duc = self.cvals if it == 0 else np.zeros_like(self.cvals)
                self.u += self._solve(K, R, duc)
            F = mesh.deformation_gradients(self.u)
            self.be.update(F, 0, self.F_e, self.F_r)
        return self.finish_increment()

    def finish_increment(self):
        """After the post-pass update: the volume averages, reorientation,
        commit, the twin-rule scalars for the next increment and the
        stress-strain row (updateAfterIncrement.cc)."""
        if self.device_system:
            self.u = self.be.get_displacement()
        avg = self.be.averages()
        self.be.reorient()
        self.be.commit()
        # a multiphase run keeps F_r = F_e = F_s = 0, in the twin rule and in
        # the output row (updateAfterIncrement.cc:718-725, :755)
        twin_cols = [0.0, 0.0, 0.0] if self.multiphase else [avg[18], avg[19], avg[20]]
        if self.multiphase:
            self.F_e = self.F_r = 0.0
        else:
            self.F_r, self.F_e = float(avg[18]), float(avg[19])
        E = avg[0:9].reshape(3, 3)
        T = avg[9:18].reshape(3, 3)
        row = [E[0, 0], E[1, 1], E[2, 2], E[1, 2], E[0, 2], E[0, 1],
               T[0, 0], T[1, 1], T[2, 2], T[1, 2], T[0, 2], T[0, 1]] + twin_cols
        self.rows.append(row)
        return row

    def run(self, n_steps=None, callback=None):
        n_steps = self.n_increments if n_steps is None else n_steps
        for i in range(n_steps):
            row = self.step()
            if callback:
                callback(i, row)
        return np.array(self.rows)


def deck_setup(d, backend_factory, material_from_fixture, **harness_kw):
    """Build mesh/backend/harness from a parsed deck (decks.load_deck, or a
    tests/golden/kat_*.npz fixture's dict); harness_kw: NewtonHarness options
    such as device_system, solver."""
    mesh = StructuredMesh(tuple(int(x) for x in d["n_elem"]))
    n_phases = 1 + sum(1 for k in d if k.startswith("ph") and k.endswith("_C6"))
    mats = [material_from_fixture(d)] + [material_from_fixture(d, phase=k) for k in range(2, n_phases + 1)]
    n_inc = int(round(float(d["total_T"]) / float(d["delT"])))
    be = backend_factory(mats, d)
    rod = np.repeat(d["cell_rodrigues"], 8, axis=0)
    lid = np.repeat(np.asarray(d["cell_phase"], np.int32) - 1, 8) if "cell_phase" in d else \
        np.zeros(mesh.n_cells * 8, np.int32)
    be.bind_qps(lid, rod)
    harness_kw.setdefault("multiphase", bool(int(d.get("multiphase", 0))))
    tab = (d["tab_bc"], d["tab_times"]) if "tab_bc" in d else None
    cyc = tuple(d["cyclic"]) if "cyclic" in d else None
    h = NewtonHarness(be, mesh, d.get("bc"), n_inc, int(d["max_newton"]), vel_grad=d.get("vel_grad"),
                      delT=float(d["delT"]), cyclic=cyc, tabular=tab, **harness_kw)
    return h, d


def kat_setup(fixture, backend_factory, material_from_fixture, **harness_kw):
    """deck_setup for a tests/golden/kat_*.npz fixture."""
    return deck_setup(dict(np.load(fixture)), backend_factory, material_from_fixture, **harness_kw)
