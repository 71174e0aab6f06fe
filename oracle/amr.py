"""Heat operator on a two-level box mesh with hanging-node constraints (TEST INFRASTRUCTURE ONLY).

A CPU restatement of what MeltPoolDG's heat path does on an adaptively refined mesh. The heat
application refines its triangulation with ``refine_grid`` (``source/utilities/amr.cpp:18-41``,
called from ``applications/mp-heat-transfer/heat_transfer_application.cpp:363-453``) and builds
the heat DoFs' constraints with deal.II's ``DoFTools::make_hanging_node_constraints``, merged into
the Dirichlet constraints (``include/meltpooldg/utilities/constraints.hpp:111-132``, ``:256-269``).
deal.II is not vendored with the reference; its published rule is restated here: a node of a
refined cell that lies on a face or an edge of an unrefined neighbour, and is not one of the
neighbour's nodes, is constrained to the neighbour's FE_Q(p) interpolant at that point,
``u_h = sum_c phi_c(x_h) u_c`` over the neighbour's nodes (the continuous FE space on a mesh with
one level of refinement difference).

The mesh is a structured box of ``cells`` coarse cells in which any set of coarse cells is
refined once (each into 8 children). The operator is the heat tangent of the structured oracle
(``mpdg_oracle.c``: ``rho_cp/dt M + K_k`` with ``k = k0 + k1 T_lin`` and the ``k1 grad(T_lin) u``
term of the linear law, ``heat_diffuse_operator.cpp:1029-1078``), assembled from element
matrices on the active cells and condensed as ``C^T A C`` with the hanging-node matrix ``C``.
Dirichlet DoFs follow the deal.II conventions of the structured oracle: read as zero, zero rows.

Only tests use this module; the product never imports it.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

FACES = {"x-": (0, 0), "x+": (0, 1), "y-": (1, 0), "y+": (1, 1), "z-": (2, 0), "z+": (2, 1)}


def gauss_lobatto(p: int) -> np.ndarray:
    """The p+1 Gauss-Lobatto points on [0, 1]: the ends and the roots of P_p' (Newton-polished)."""
    if p == 1:
        return np.array([0.0, 1.0])
    dP = np.polynomial.legendre.Legendre.basis(p).deriv()
    x = np.sort(dP.roots().real)
    d2P = dP.deriv()
    for _ in range(3):
        x = x - dP(x) / d2P(x)
    return (np.concatenate([[-1.0], x, [1.0]]) + 1.0) / 2.0


def gauss(n: int):
    """n-point Gauss-Legendre rule on [0, 1]."""
    x, w = np.polynomial.legendre.leggauss(n)
    return (x + 1.0) / 2.0, w / 2.0


def lagrange(nodes: np.ndarray, x: np.ndarray):
    """Values V[q, i] = l_i(x_q) and derivatives D[q, i] of the Lagrange basis on `nodes`."""
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    n = len(nodes)
    V = np.ones((len(x), n))
    D = np.zeros((len(x), n))
    for i in range(n):
        others = [j for j in range(n) if j != i]
        den = np.prod([nodes[i] - nodes[j] for j in others])
        for j in others:
            V[:, i] *= (x - nodes[j])
        for m in others:
            term = np.ones(len(x))
            for j in others:
                if j != m:
                    term *= (x - nodes[j])
            D[:, i] += term
        V[:, i] /= den
        D[:, i] /= den
    return V, D


class TwoLevelBoxMesh:
    """FE_Q(p) heat operator on a box of coarse cells, the cells in `refine` split once.

    refine: iterable of coarse cell indices (ix, iy, iz), or a boolean array [mz][my][mx].
    DoFs are the nodes that are not hanging, numbered by position (z, y, x lexicographic).
    constrain_hanging=False leaves the hanging nodes free (a nonconforming space): a planted
    mistake for the tests that check the constraints matter.
    """

    def __init__(self, degree, cells, refine=(), lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                 dirichlet=("x-", "x+", "y-", "y+", "z-", "z+"), constrain_hanging=True):
        self.p = p = int(degree)
        self.n = n = p + 1
        self.m = m = tuple(int(c) for c in cells)
        self.lo = np.asarray(lo, dtype=np.float64)
        self.h = (np.asarray(hi, dtype=np.float64) - self.lo) / np.asarray(m)
        ref = np.zeros((m[2], m[1], m[0]), dtype=bool)
        if isinstance(refine, np.ndarray) and refine.dtype == bool:
            ref[...] = refine
        else:
            for ix, iy, iz in refine:
                ref[iz, iy, ix] = True
        self.refined = ref
        self.xi = gauss_lobatto(p)
        # active cells: origin and size in coarse-cell units
        origins, sizes, parents = [], [], []
        for iz in range(m[2]):
            for iy in range(m[1]):
                for ix in range(m[0]):
                    if ref[iz, iy, ix]:
                        for sz in (0, 1):
                            for sy in (0, 1):
                                for sx in (0, 1):
                                    origins.append((ix + 0.5 * sx, iy + 0.5 * sy, iz + 0.5 * sz))
                                    sizes.append(0.5)
                                    parents.append((ix, iy, iz))
                    else:
                        origins.append((ix, iy, iz))
                        sizes.append(1.0)
                        parents.append((ix, iy, iz))
        self.origins = np.asarray(origins, dtype=np.float64)
        self.sizes = np.asarray(sizes, dtype=np.float64)
        self.parents = np.asarray(parents, dtype=np.int64)
        # child position (s_x, s_y, s_z) of a refined cell in its parent
        self.child = np.rint((self.origins - self.parents) * 2.0).astype(np.int64)
        self.n_cells = len(sizes)
        # local node offsets in the unit cell, x fastest
        lx = np.array([(self.xi[i], self.xi[j], self.xi[k])
                       for k in range(n) for j in range(n) for i in range(n)])
        self._local = lx
        pos = self.origins[:, None, :] + self.sizes[:, None, None] * lx[None, :, :]
        keys = np.round(pos.reshape(-1, 3) * (1 << 26)).astype(np.int64)
        uniq, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
        self.cell_nodes = inv.reshape(self.n_cells, n ** 3)
        self.node_pos = pos.reshape(-1, 3)[first]  # coarse-cell units (the key only matches)
        n_nodes = len(uniq)
        # hanging nodes: nodes of refined cells that lie on the closed box of an unrefined
        # coarse cell without being one of its nodes; constrained to its interpolant there
        coarse_cells = [c for c in range(self.n_cells) if self.sizes[c] == 1.0]
        is_coarse_node = np.zeros(n_nodes, dtype=bool)
        for c in coarse_cells:
            is_coarse_node[self.cell_nodes[c]] = True
        fine_nodes = np.unique(self.cell_nodes[self.sizes == 0.5]) if np.any(
            self.sizes == 0.5) else np.zeros(0, dtype=np.int64)
        candidates = [v for v in fine_nodes if not is_coarse_node[v]] if constrain_hanging else []
        cons = {}
        tol = 1e-9
        coarse_origin = {tuple(self.origins[c].astype(int)): c for c in coarse_cells}
        for v in candidates:
            x = self.node_pos[v]
            # unrefined coarse cells whose closed box holds x
            base = np.floor(x + tol).astype(int)
            owner = None
            for dz in (0, -1):
                for dy in (0, -1):
                    for dx in (0, -1):
                        c0 = (base[0] + dx, base[1] + dy, base[2] + dz)
                        if c0 in coarse_origin:
                            o = np.asarray(c0, dtype=np.float64)
                            if np.all(x >= o - tol) and np.all(x <= o + 1.0 + tol):
                                owner = coarse_origin[c0]
                                break
                    if owner is not None:
                        break
                if owner is not None:
                    break
            if owner is None:
                continue  # interior of the refined region: a regular node
            loc = np.clip(x - self.origins[owner], 0.0, 1.0)
            w = self._tensor_basis(loc)
            nz = np.abs(w) > 1e-14
            cons[v] = (self.cell_nodes[owner][nz], w[nz])
        self._finish(cons, dirichlet)

    def _finish(self, cons, dirichlet):
        """DoF numbering, the constraint matrix, the Dirichlet mask and the reference tables,
        given the hanging nodes' constraints {node: (nodes, weights)}."""
        n, m = self.n, self.m
        n_nodes = len(self.node_pos)
        self.hanging = np.zeros(n_nodes, dtype=bool)
        self.hanging[list(cons)] = True
        # DoFs: the regular nodes, in position order (z, y, x)
        regular = np.flatnonzero(~self.hanging)
        order = np.lexsort((self.node_pos[regular, 0], self.node_pos[regular, 1],
                            self.node_pos[regular, 2]))
        regular = regular[order]
        self.dof_of_node = -np.ones(n_nodes, dtype=np.int64)
        self.dof_of_node[regular] = np.arange(len(regular))
        self.n_dofs = len(regular)
        self.node_of_dof = regular
        rows, cols, vals = [], [], []
        for v in regular:
            rows.append(v)
            cols.append(self.dof_of_node[v])
            vals.append(1.0)
        for v, (cn, w) in cons.items():
            for c, wc in zip(cn, w):
                d = self.dof_of_node[c]
                assert d >= 0, "a hanging node depends on another hanging node"
                rows.append(v)
                cols.append(d)
                vals.append(wc)
        self.C = sp.csr_matrix((vals, (rows, cols)), shape=(n_nodes, self.n_dofs))
        # Dirichlet DoFs: regular nodes on the flagged faces of the box
        mask = np.zeros(self.n_dofs, dtype=bool)
        P = self.node_pos[regular]
        for f in dirichlet:
            d, side = FACES[f]
            mask |= np.abs(P[:, d] - (m[d] if side else 0)) < 1e-9
        self.mask = mask
        # reference-cell tables: QGauss(p+1), FE_Q(p) on Gauss-Lobatto points
        xq, wq = gauss(n)
        V1, D1 = lagrange(self.xi, xq)
        self._N = np.kron(V1, np.kron(V1, V1))
        self._G = [np.kron(V1, np.kron(V1, D1)), np.kron(V1, np.kron(D1, V1)),
                   np.kron(D1, np.kron(V1, V1))]
        self._w = np.kron(wq, np.kron(wq, wq))
        self._xq = np.array([(xq[i], xq[j], xq[k]) for k in range(n) for j in range(n)
                             for i in range(n)])

    def _tensor_basis(self, loc):
        vx = lagrange(self.xi, [loc[0]])[0][0]
        vy = lagrange(self.xi, [loc[1]])[0][0]
        vz = lagrange(self.xi, [loc[2]])[0][0]
        return np.kron(vz, np.kron(vy, vx))

    # ------------------------------------------------------------------------------------
    def support_points(self) -> np.ndarray:
        """Physical coordinates of the DoFs, shape (n_dofs, 3)."""
        return self.lo + self.node_pos[self.node_of_dof] * self.h

    def quadrature_points(self, cell: int) -> np.ndarray:
        return self.lo + (self.origins[cell] + self.sizes[cell] * self._xq) * self.h

    def node_values(self, u_dofs: np.ndarray) -> np.ndarray:
        """All nodal values (hanging nodes from their constraints)."""
        return self.C @ u_dofs

    def _cell_factors(self, cell):
        hs = self.sizes[cell] * self.h
        jxw = self._w * np.prod(hs)
        G = [self._G[d] / hs[d] for d in range(3)]
        return jxw, G

    def _element_matrix(self, c, rho_cp, dt, k0, k1, te):
        """Cell matrix of rho_cp/dt M + K_k (+ k1 grad(T_lin) u) with te the cell's T_lin."""
        jxw, G = self._cell_factors(c)
        N = self._N
        A = (rho_cp / dt) * (N.T * jxw) @ N
        if te is None:
            kq = np.full(len(jxw), k0)
            gT = None
        else:
            kq = k0 + k1 * (N @ te)
            gT = [Gd @ te for Gd in G]
        for d in range(3):
            A += (G[d].T * (jxw * kq)) @ G[d]
            if gT is not None:
                A += (G[d].T * (jxw * k1 * gT[d])) @ N
        return A

    def assemble(self, rho_cp=1.0, dt=1.0, k0=1.0, k1=0.0, T_lin=None) -> sp.csr_matrix:
        """C^T A C of the tangent rho_cp/dt M + K_k(T_lin) (+ k1 grad(T_lin) u), on all DoFs."""
        n3 = self.n ** 3
        Tn = None if T_lin is None or k1 == 0.0 else self.node_values(T_lin)
        rows = np.repeat(self.cell_nodes, n3, axis=1).ravel()
        cols = np.tile(self.cell_nodes, (1, n3)).ravel()
        data = np.empty((self.n_cells, n3, n3))
        for c in range(self.n_cells):
            te = None if Tn is None else Tn[self.cell_nodes[c]]
            data[c] = self._element_matrix(c, rho_cp, dt, k0, k1, te)
        An = sp.csr_matrix((data.ravel(), (rows, cols)),
                           shape=(len(self.node_pos), len(self.node_pos)))
        return (self.C.T @ An @ self.C).tocsr()

    def vmult(self, src, **coef) -> np.ndarray:
        """dst = J src with Dirichlet DoFs read as zero and their rows zero."""
        s = np.where(self.mask, 0.0, src)
        y = self.assemble(**coef) @ s
        y[self.mask] = 0.0
        return y

    def load_vector(self, f) -> np.ndarray:
        """C^T of the element integrals of f(x) phi_i (f evaluated at the q-points)."""
        b = np.zeros(len(self.node_pos))
        for c in range(self.n_cells):
            jxw, _ = self._cell_factors(c)
            fq = f(self.quadrature_points(c))
            np.add.at(b, self.cell_nodes[c], self._N.T @ (jxw * fq))
        return self.C.T @ b

    def solve(self, b, **coef) -> np.ndarray:
        """Solve J x = b on the free DoFs (direct), x = 0 on the Dirichlet DoFs."""
        A = self.assemble(**coef)
        free = np.flatnonzero(~self.mask)
        x = np.zeros(self.n_dofs)
        x[free] = spla.spsolve(A[free][:, free].tocsc(), b[free])
        return x

    # ------------------------------------------------------------------------------------
    # second form: the constraints applied inside each cell, as a cell kernel applies them
    def _coarse_unrefined(self, q):
        m = self.m
        if not all(0 <= q[d] < m[d] for d in range(3)):
            return None
        if self.refined[q[2], q[1], q[0]]:
            return None
        return q

    def hanging_code(self, c) -> int:
        """9-bit code of a cell's hanging faces and edges: bits 0-2 its child position
        (s_x, s_y, s_z) in the parent, bit 3+d a hanging face normal to direction d (at side
        s_d), bit 6+d a hanging edge parallel to d (at the sides s of the two other directions)
        whose two adjacent faces do not hang. 0 for a cell without hanging nodes."""
        if self.sizes[c] == 1.0 or not self.hanging.any():
            return 0
        par, sv = self.parents[c], self.child[c]
        step = np.where(sv == 0, -1, 1)
        face = [self._coarse_unrefined(par + step[d] * np.eye(3, dtype=np.int64)[d]) is not None
                for d in range(3)]
        edge = []
        for d in range(3):
            d1, d2 = [e for e in range(3) if e != d]
            off = np.zeros(3, dtype=np.int64)
            off[d1], off[d2] = step[d1], step[d2]
            edge.append(self._coarse_unrefined(par + off) is not None and not face[d1]
                        and not face[d2])
        code = sum(int(face[d]) << (3 + d) for d in range(3)) + \
            sum(int(edge[d]) << (6 + d) for d in range(3))
        if code == 0:
            return 0
        return code | int(sv[0]) | (int(sv[1]) << 1) | (int(sv[2]) << 2)

    def child_interpolation(self, s: int) -> np.ndarray:
        """I[j, a] = l_a((s + xi_j) / 2): the coarse 1D basis at the nodes of child s."""
        return lagrange(self.xi, (s + self.xi) / 2.0)[0]

    def cell_map(self, c):
        """Gathered DoF indices of cell c and the matrix F with local = F gathered: the nodes
        of a hanging face or edge gather the coarse neighbour's face or edge DoFs of the same
        indices, and F interpolates them with the 1D child matrices, one direction at a time."""
        n, n3 = self.n, self.n ** 3
        idx = self.dof_of_node[self.cell_nodes[c]].copy()
        code = self.hanging_code(c)
        if code == 0:
            return idx, None
        sv = [(code >> d) & 1 for d in range(3)]
        par = self.parents[c]
        step = [(-1 if sv[d] == 0 else 1) for d in range(3)]
        own = [0 if sv[d] == 0 else n - 1 for d in range(3)]   # the cell's side
        other = [n - 1 - own[d] for d in range(3)]             # the neighbour's side
        lin = lambda i, j, k: i + n * (j + n * k)
        lines = {0: [], 1: [], 2: []}  # lines along d to interpolate: fixed (index, index)
        for d in range(3):
            if not (code >> (3 + d)) & 1:
                continue
            q = par.copy()
            q[d] += step[d]
            nb = self._neighbour(c, q)
            for a in range(n):
                for b in range(n):
                    i = [0, 0, 0]
                    d1, d2 = [e for e in range(3) if e != d]
                    i[d], i[d1], i[d2] = own[d], a, b
                    jn = list(i)
                    jn[d] = other[d]
                    idx[lin(*i)] = self.dof_of_node[self.cell_nodes[nb][lin(*jn)]]
            for e in range(3):
                if e != d:
                    lines[e].append((d, own[d]))
        for d in range(3):
            if not (code >> (6 + d)) & 1:
                continue
            d1, d2 = [e for e in range(3) if e != d]
            q = par.copy()
            q[d1] += step[d1]
            q[d2] += step[d2]
            nb = self._neighbour(c, q)
            for a in range(n):
                i = [0, 0, 0]
                i[d], i[d1], i[d2] = a, own[d1], own[d2]
                jn = list(i)
                jn[d1], jn[d2] = other[d1], other[d2]
                idx[lin(*i)] = self.dof_of_node[self.cell_nodes[nb][lin(*jn)]]
            lines[d].append(((d1, own[d1]), (d2, own[d2])))
        F = np.eye(n3)
        for d in range(3):
            I = self.child_interpolation(sv[d])
            Fd = np.eye(n3)
            done = set()
            for spec in lines[d]:
                fixed = [spec] if isinstance(spec[0], int) else list(spec)
                d1, d2 = [e for e in range(3) if e != d]
                for a in range(n):
                    for b in range(n):
                        i = [0, 0, 0]
                        i[d1], i[d2] = a, b
                        if any(i[fd] != fv for fd, fv in fixed) or (a, b) in done:
                            continue
                        done.add((a, b))
                        nodes = []
                        for t in range(n):
                            i[d] = t
                            nodes.append(lin(*i))
                        Fd[np.ix_(nodes, nodes)] = I
            F = Fd @ F
        assert (idx >= 0).all(), "a hanging node left ungathered"
        return idx, F

    def _neighbour(self, c, q):
        """The unrefined neighbour of cell c's parent at coarse index q."""
        return self._coarse_cell(q)

    def _coarse_cell(self, q):
        ox = np.asarray(q, dtype=np.float64)
        hit = np.flatnonzero((self.sizes == 1.0) & np.all(self.origins == ox, axis=1))
        return int(hit[0])

    def vmult_cellwise(self, src, rho_cp=1.0, dt=1.0, k0=1.0, k1=0.0, T_lin=None) -> np.ndarray:
        """The operator of vmult with the constraints applied per cell (gather, F, cell matrix,
        F^T, scatter), as a matrix-free cell kernel applies them."""
        s = np.where(self.mask, 0.0, src)
        y = np.zeros(self.n_dofs)
        for c in range(self.n_cells):
            idx, F = self.cell_map(c)
            ul = s[idx] if F is None else F @ s[idx]
            te = None
            if T_lin is not None and k1 != 0.0:
                te = T_lin[idx] if F is None else F @ T_lin[idx]
            yl = self._element_matrix(c, rho_cp, dt, k0, k1, te) @ ul
            np.add.at(y, idx, yl if F is None else F.T @ yl)
        y[self.mask] = 0.0
        return y

    # ------------------------------------------------------------------------------------
    # residual and implicit step (the rest of the path on the refined mesh)
    def create_rhs(self, T, T_old, heat_source=None, dst=None, rho_cp=1.0, dt=1.0, k0=1.0,
                   k1=0.0) -> np.ndarray:
        """dst += -R(T) (create_rhs, heat_diffuse_operator.cpp:393-529): per q-point
        -(rho_cp/dt (T - T_old) - q_h) against v and -k(T) grad(T) against grad(v), with q_h the
        FE interpolant of the nodal source; T, T_old and the source are read plain, the
        Dirichlet rows are left untouched."""
        dst = np.zeros(self.n_dofs) if dst is None else dst
        Tn, Ton = self.node_values(T), self.node_values(T_old)
        qn = None if heat_source is None else self.node_values(heat_source)
        b = np.zeros(len(self.node_pos))
        N = self._N
        for c in range(self.n_cells):
            jxw, G = self._cell_factors(c)
            nodes = self.cell_nodes[c]
            Tq = N @ Tn[nodes]
            val = rho_cp / dt * (Tq - N @ Ton[nodes])
            if qn is not None:
                val = val - N @ qn[nodes]
            kq = k0 + k1 * Tq
            r = N.T @ (jxw * val)
            for d in range(3):
                r += G[d].T @ (jxw * kq * (G[d] @ Tn[nodes]))
            np.add.at(b, nodes, -r)
        r = self.C.T @ b
        dst[~self.mask] += r[~self.mask]
        return dst

    def time_step_newton(self, T_cur, T_old, dt, dt_old, heat_source=None, rho_cp=1.0, k0=1.0,
                         k1=0.0, newton_max_it=10, res_tol=1e-9, corr_tol=1e-10):
        """HeatDiffuseOperation::solve on the refined mesh, in place: linear predictor
        (predictor_linear.cpp:74-96), history commit T_old <- T, Dirichlet values (zero), then
        Newton (newton_raphson_solver.cpp:22-68) with exact linear solves; converged when
        |rhs| < res_tol and |delta| < corr_tol (the converged update is not applied).
        Returns the number of Newton iterations."""
        r = dt / dt_old if abs(dt_old) >= 1e-12 else 0.0
        pred = (1.0 + r) * T_cur - r * T_old
        T_old[:] = T_cur
        T_cur[:] = np.where(self.mask, 0.0, pred)
        for it in range(newton_max_it):
            rhs = self.create_rhs(T_cur, T_old, heat_source, rho_cp=rho_cp, dt=dt, k0=k0, k1=k1)
            delta = self.solve(rhs, rho_cp=rho_cp, dt=dt, k0=k0, k1=k1,
                               T_lin=T_cur if k1 != 0.0 else None)
            if np.linalg.norm(rhs) < res_tol and np.linalg.norm(delta) < corr_tol:
                return it + 1
            T_cur += delta
        raise RuntimeError("Newton-Raphson did not converge")

    # ------------------------------------------------------------------------------------
    # the inverse diagonal and the residual in the cell-wise form (what the GPU path needs
    # next: a refined cell on an interface has no closed-form diagonal, F^T A F is applied to
    # its unit vectors instead)
    def inverse_diagonal(self, **coef) -> np.ndarray:
        """1/diag(C^T A C) with the reference's rule |d| > 1e-10 ? 1/d : 1
        (heat_diffuse_operator.cpp:282-283); Dirichlet DoFs 1."""
        d = self.assemble(**coef).diagonal().copy()
        d[self.mask] = 0.0
        return np.where(np.abs(d) > 1e-10, 1.0 / np.where(d == 0.0, 1.0, d), 1.0)

    def inverse_diagonal_cellwise(self, rho_cp=1.0, dt=1.0, k0=1.0, k1=0.0, T_lin=None):
        """The same diagonal accumulated cell by cell: diag(F^T A_e F) at the gathered DoFs
        (the gathered DoFs of a cell are distinct, so the local diagonal is the contribution)."""
        d = np.zeros(self.n_dofs)
        for c in range(self.n_cells):
            idx, F = self.cell_map(c)
            te = None
            if T_lin is not None and k1 != 0.0:
                te = T_lin[idx] if F is None else F @ T_lin[idx]
            A = self._element_matrix(c, rho_cp, dt, k0, k1, te)
            loc = np.diag(A) if F is None else np.einsum("il,ij,jl->l", F, A, F)
            np.add.at(d, idx, loc)
        d[self.mask] = 0.0
        return np.where(np.abs(d) > 1e-10, 1.0 / np.where(d == 0.0, 1.0, d), 1.0)

    def create_rhs_cellwise(self, T, T_old, heat_source=None, dst=None, rho_cp=1.0, dt=1.0,
                            k0=1.0, k1=0.0) -> np.ndarray:
        """create_rhs with the constraints applied per cell: T, T_old and the source gathered
        and interpolated by F, the residual integrated, F^T in the scatter."""
        dst = np.zeros(self.n_dofs) if dst is None else dst
        N = self._N
        y = np.zeros(self.n_dofs)
        for c in range(self.n_cells):
            idx, F = self.cell_map(c)
            loc = (lambda v: v[idx]) if F is None else (lambda v: F @ v[idx])
            te, to = loc(T), loc(T_old)
            jxw, G = self._cell_factors(c)
            Tq = N @ te
            val = rho_cp / dt * (Tq - N @ to)
            if heat_source is not None:
                val = val - N @ loc(heat_source)
            kq = k0 + k1 * Tq
            r = N.T @ (jxw * val)
            for d in range(3):
                r += G[d].T @ (jxw * kq * (G[d] @ te))
            np.add.at(y, idx, -(r if F is None else F.T @ r))
        dst[~self.mask] += y[~self.mask]
        return dst


class MultiLevelBoxMesh(TwoLevelBoxMesh):
    """The box with each coarse cell refined uniformly `levels[iz][iy][ix]` times, neighbouring
    coarse cells (across faces, edges and vertices) differing by one level at most: the 2:1
    balance p4est keeps for MeltPoolDG's adaptive meshes. A node hangs when the coarsest cells
    whose closed boxes hold it (level l_min) do not have it as a node; it is constrained to such
    a cell's interpolant. Under the balance the constraining nodes never hang, so the rule of
    the two-level mesh applies unchanged at every interface. The operator, the residual, the
    solve and the cell-wise form are those of TwoLevelBoxMesh."""

    def __init__(self, degree, cells, levels, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                 dirichlet=("x-", "x+", "y-", "y+", "z-", "z+")):
        self.p = p = int(degree)
        self.n = n = p + 1
        self.m = m = tuple(int(c) for c in cells)
        self.lo = np.asarray(lo, dtype=np.float64)
        self.h = (np.asarray(hi, dtype=np.float64) - self.lo) / np.asarray(m)
        lev = np.asarray(levels, dtype=np.int64).reshape(m[2], m[1], m[0])
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    a = lev[max(dz, 0):m[2] + min(dz, 0), max(dy, 0):m[1] + min(dy, 0),
                            max(dx, 0):m[0] + min(dx, 0)]
                    b = lev[max(-dz, 0):m[2] + min(-dz, 0), max(-dy, 0):m[1] + min(-dy, 0),
                            max(-dx, 0):m[0] + min(-dx, 0)]
                    if a.size and np.abs(a - b).max() > 1:
                        raise ValueError("neighbouring coarse cells differ by more than one level")
        self.levels = lev
        self.refined = lev > 0
        self.xi = gauss_lobatto(p)
        origins, sizes, parents, lvl, gidx = [], [], [], [], []
        for iz in range(m[2]):
            for iy in range(m[1]):
                for ix in range(m[0]):
                    L = int(lev[iz, iy, ix])
                    k = 1 << L
                    for sz in range(k):
                        for sy in range(k):
                            for sx in range(k):
                                origins.append((ix + sx / k, iy + sy / k, iz + sz / k))
                                sizes.append(1.0 / k)
                                lvl.append(L)
                                g = (ix * k + sx, iy * k + sy, iz * k + sz)
                                gidx.append(g)
                                parents.append(tuple(v // 2 for v in g))
        self.origins = np.asarray(origins, dtype=np.float64)
        self.sizes = np.asarray(sizes, dtype=np.float64)
        self.cell_level = np.asarray(lvl, dtype=np.int64)
        self.gidx = np.asarray(gidx, dtype=np.int64)        # index on its level's lattice
        self.parents = np.asarray(parents, dtype=np.int64)  # index on the level below
        self.child = self.gidx % 2
        self.n_cells = len(sizes)
        self._cell_at = {(int(lvl[c]),) + tuple(int(v) for v in gidx[c]): c
                         for c in range(self.n_cells)}
        lx = np.array([(self.xi[i], self.xi[j], self.xi[k])
                       for k in range(n) for j in range(n) for i in range(n)])
        self._local = lx
        pos = self.origins[:, None, :] + self.sizes[:, None, None] * lx[None, :, :]
        keys = np.round(pos.reshape(-1, 3) * (1 << 26)).astype(np.int64)
        uniq, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
        self.cell_nodes = inv.reshape(self.n_cells, n ** 3)
        self.node_pos = pos.reshape(-1, 3)[first]
        n_nodes = len(uniq)
        node_of_level = {}
        for L in np.unique(self.cell_level):
            f = np.zeros(n_nodes, dtype=bool)
            f[self.cell_nodes[self.cell_level == L].ravel()] = True
            node_of_level[int(L)] = f
        tol = 1e-9
        cons = {}
        for v in range(n_nodes):
            x = self.node_pos[v]
            base = np.floor(x + tol).astype(int)
            holders = []
            for dz in (0, -1):
                for dy in (0, -1):
                    for dx in (0, -1):
                        c0 = (base[0] + dx, base[1] + dy, base[2] + dz)
                        if all(0 <= c0[d] < m[d] for d in range(3)):
                            o = np.asarray(c0, dtype=np.float64)
                            if np.all(x >= o - tol) and np.all(x <= o + 1.0 + tol):
                                holders.append(c0)
            lmin = min(int(lev[c[2], c[1], c[0]]) for c in holders)
            if node_of_level[lmin][v]:
                continue
            c0 = next(c for c in holders if lev[c[2], c[1], c[0]] == lmin)
            k = 1 << lmin
            sub = np.clip(np.floor((x - np.asarray(c0)) * k + tol).astype(int), 0, k - 1)
            g = tuple(int(c0[d] * k + sub[d]) for d in range(3))
            owner = self._cell_at[(lmin,) + g]
            loc = np.clip((x - self.origins[owner]) / self.sizes[owner], 0.0, 1.0)
            w = self._tensor_basis(loc)
            nz = np.abs(w) > 1e-14
            cons[v] = (self.cell_nodes[owner][nz], w[nz])
        self._finish(cons, dirichlet)

    def _neighbour(self, c, q):
        return self._coarse_unrefined_at(c, q)

    # neighbour lookups on the level below the cell: the coarse cell of the two-level mesh
    def _coarse_unrefined_at(self, c, q):
        L = int(self.cell_level[c]) - 1
        return self._cell_at.get((L,) + tuple(int(v) for v in q))

    def hanging_code(self, c) -> int:
        if self.cell_level[c] == 0 or not self.hanging.any():
            return 0
        par, sv = self.parents[c], self.child[c]
        step = np.where(sv == 0, -1, 1)
        e = np.eye(3, dtype=np.int64)
        face = [self._coarse_unrefined_at(c, par + step[d] * e[d]) is not None for d in range(3)]
        edge = []
        for d in range(3):
            d1, d2 = [x for x in range(3) if x != d]
            off = np.zeros(3, dtype=np.int64)
            off[d1], off[d2] = step[d1], step[d2]
            edge.append(self._coarse_unrefined_at(c, par + off) is not None and not face[d1]
                        and not face[d2])
        code = sum(int(face[d]) << (3 + d) for d in range(3)) + \
            sum(int(edge[d]) << (6 + d) for d in range(3))
        if code == 0:
            return 0
        return code | int(sv[0]) | (int(sv[1]) << 1) | (int(sv[2]) << 2)
