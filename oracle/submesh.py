"""CPU restatement of the [mesh] selection path (numpy / scipy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of
icarat_ctx_create_selection; the product (icarat2_b200) never imports it.

It restates, on the kept mesh of a voxel box:
  - MeshIcarat::modifyMesh (src/io/mesh_icarat.hpp:636-755): nodes inside a
    selection box widened by 1e-7, elements whose centroid (running sum of
    x / ne over the local nodes) is inside one, both renumbered in ascending
    box order; a kept element with a removed node is an error;
  - BCIcarat::input_dirich + countDOF (boundary_condition_icarat.hpp:73-148,
    boundary_condition_base.hpp:19-95) over the kept nodes, and the point
    loads of input_neumann (boundary_condition_icarat.hpp:380-396);
  - LinearAnalysis::solve (src/analysis/linear.hpp:55-104) as triplet
    assembly of K_ff (assembling.hpp:19-39; duplicates summed as
    setFromTriplets does) and a direct sparse solve;
  - divideValIntoNode (analysis_utility.hpp:9-31), the driver sensitivity
    (opt_macro_oc.cpp:182-212) and the loop body of opt_macro_oc.cpp:83-172 /
    opt_macro_mma_nondesign.cpp:90-178 with the radius Filter of the kept
    elements (oracle.Filter over their centroids: preNeighbour, filter.hpp:
    254-297), OC (oracle.oc_update) and MMA (oracle.MMA).
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import oracle as O

TOL = 1.0e-7


def box_mesh(nx, ny, nz, lx, ly, lz):
    """node coordinates (numnp x 3) and hexa8 connectivity (nelx x 8) of the
    box mesher (the C restatement's or_mesh_box)."""
    numnp, nelx = (nx + 1) * (ny + 1) * (nz + 1), nx * ny * nz
    xyz = np.zeros(3 * numnp)
    conn = np.zeros(8 * nelx, np.int32)
    O.lib.or_mesh_box(nx, ny, nz, lx, ly, lz, xyz, conn)
    return xyz.reshape(-1, 3), conn.reshape(-1, 8)


def modify_mesh(xyz, conn, boxes):
    """(kept node ids, kept element ids, connectivity in kept node numbers)."""
    numnp, nelx = xyz.shape[0], conn.shape[0]
    node_in = np.zeros(numnp, bool)
    elem_in = np.zeros(nelx, bool)
    cen = np.zeros((nelx, 3))
    for e in range(nelx):
        s = [0.0, 0.0, 0.0]
        for a in range(conn.shape[1]):
            for d in range(3):
                s[d] += float(xyz[conn[e, a], d]) / conn.shape[1]
        cen[e] = s
    for b in boxes:
        b = np.asarray(b, float).reshape(3, 2)
        lo, hi = b[:, 0] - TOL, b[:, 1] + TOL
        node_in |= np.all((xyz >= lo) & (xyz <= hi), axis=1)
        elem_in |= np.all((cen >= lo) & (cen <= hi), axis=1)
    nodes = np.flatnonzero(node_in)
    elems = np.flatnonzero(elem_in)
    new_id = np.full(numnp, -1, np.int64)
    new_id[nodes] = np.arange(nodes.size)
    kconn = new_id[conn[elems]]
    if np.any(kconn < 0):
        raise ValueError("error in mesh_icarat: a kept element has a removed node")
    return nodes, elems, kconn.astype(np.int64)


def count_dof(xyz, dirichlet):
    """input_dirich + countDOF: (dof numbers numnp x 3, numeq, prescribed values)."""
    numnp = xyz.shape[0]
    has = np.zeros(numnp, bool)
    flag = np.zeros((numnp, 3), np.int64)
    val = np.zeros((numnp, 3))
    for fl, vl, bx in dirichlet:
        bx = np.asarray(bx, float).reshape(3, 2)
        inside = np.all((xyz >= bx[:, 0] - TOL) & (xyz <= bx[:, 1] + TOL), axis=1)
        for n in np.flatnonzero(inside):
            has[n] = True
            for q in range(3):
                if flag[n, q] != 1:
                    flag[n, q] = fl[q]
                val[n, q] = vl[q]
    dof = np.zeros((numnp, 3), np.int64)
    counter = 0
    for n in range(numnp):
        for q in range(3):
            if not has[n] or flag[n, q] == 0:
                dof[n, q] = counter
                counter += 1
    numeq = counter
    uD = np.zeros((numnp, 3))
    for n in range(numnp):
        if has[n]:
            for q in range(3):
                if flag[n, q] != 0:
                    dof[n, q] = counter
                    counter += 1
                    if flag[n, q] == 1:
                        uD[n, q] = val[n, q]
    return dof, numeq, uD


class SelProblem:
    """The kept mesh of a box with its boundary conditions (point loads only)."""

    def __init__(self, nx, ny, nz, boxes, dirichlet, loads, lx=None, ly=None, lz=None,
                 E1=1e-9, E2=1.0, nu=0.3, penalty=3.0):
        lx = float(nx if lx is None else lx)
        ly = float(ny if ly is None else ly)
        lz = float(nz if lz is None else lz)
        bxyz, bconn = box_mesh(nx, ny, nz, lx, ly, lz)
        self.node_ids, self.elem_ids, self.conn = modify_mesh(bxyz, bconn, boxes)
        self.xyz = bxyz[self.node_ids]
        self.numnp, self.nelx = self.node_ids.size, self.elem_ids.size
        self.dof, self.numeq, uD = count_dof(self.xyz, dirichlet)
        if np.any(uD != 0.0):
            raise ValueError("prescribed displacements are not restated here")
        self.fext = np.zeros(self.numeq)
        for vl, bx in loads:
            bx = np.asarray(bx, float).reshape(3, 2)
            if np.any(bx[:, 0] != bx[:, 1]):
                raise ValueError("only point loads are restated here")
            inside = np.all((self.xyz >= bx[:, 0] - TOL) & (self.xyz <= bx[:, 1] + TOL), axis=1)
            for n in np.flatnonzero(inside):
                for q in range(3):
                    if self.dof[n, q] < self.numeq:
                        self.fext[self.dof[n, q]] += vl[q]
        self.ke0, self.vol0 = O.hexa8_ke(bxyz[bconn[0]], 1.0, nu)
        self.E1, self.E2, self.pp = E1, E2, penalty
        edof = self.dof[self.conn].reshape(self.nelx, 24)  # 3 a + c order
        self.edof = edof
        ii = np.repeat(edof, 24, axis=1)
        jj = np.tile(edof, (1, 24))
        self._mask = (ii < self.numeq) & (jj < self.numeq)
        self._ii, self._jj = ii, jj
        cen = np.zeros((self.nelx, 3))
        for e in range(self.nelx):
            for d in range(3):
                s = 0.0
                for a in range(8):
                    s += float(self.xyz[self.conn[e, a], d]) / 8
                cen[e, d] = s
        self.centroids = cen

    def young(self, rho):
        rp = np.power(rho, self.pp)
        return (1.0 - rp) * self.E1 + rp * self.E2

    def K(self, rho):
        """K_ff from the element triplets (assembling, setFromTriplets)."""
        v = self.young(np.asarray(rho, float))[:, None] * self.ke0.ravel()[None, :]
        m = self._mask
        return sp.coo_matrix((v[m], (self._ii[m], self._jj[m])),
                             shape=(self.numeq, self.numeq)).tocsr()

    def solve(self, rho):
        return spla.spsolve(self.K(rho).tocsc(), self.fext)

    def node_values(self, val):
        nv = np.zeros((self.numnp, 3))
        free = self.dof < self.numeq
        nv[free] = val[self.dof[free]]
        nv[np.abs(nv) < 1e-15] = 0.0
        return nv

    def compliance(self, val):
        return float(val @ self.fext)

    def sensitivity(self, rho, node_val, dgds_scale=1.0):
        rho = np.asarray(rho, float)
        u = node_val[self.conn].reshape(self.nelx, 24)
        q = np.einsum("ei,ij,ej->e", u, self.ke0, u) * self.young(rho)
        dyoung = self.pp * np.power(rho, self.pp - 1.0) * (self.E2 - self.E1)
        return -(dyoung / self.young(rho)) * q, np.full(self.nelx, self.vol0 * dgds_scale)


class SelLoop:
    """One design iteration per step() on the kept mesh (no threshold)."""

    def __init__(self, P, radius, method="mma", x0=0.3, move=None, xmin=1e-4, xmax=1.0):
        self.P, self.method = P, method
        self.F = O.Filter(centroids=P.centroids, radius=radius)
        self.x = np.full(P.nelx, float(x0))
        self.xmin, self.xmax = np.full(P.nelx, xmin), np.full(P.nelx, xmax)
        self.move = move if move is not None else (0.2 if method == "mma" else 0.15)
        if method == "mma":
            self.M = O.MMA(P.nelx, 1)
            self.M.set_move_limit(self.move)
        self.optstep, self.V0 = 0, 0.0
        self.vol = np.full(P.nelx, P.vol0)

    def step(self):
        P = self.P
        self.optstep += 1
        xfil = self.F.density_filter(self.x)
        val = P.solve(xfil)
        nv = P.node_values(val)
        self.compliance = P.compliance(val)
        if self.optstep == 1:
            self.V0 = float(np.sum(xfil * self.vol))
            self.constraint = 0.0 if self.method == "mma" else self.V0
        elif self.method == "mma":
            self.constraint = float(np.sum(xfil * self.vol / self.V0)) - 1.0
        else:
            self.constraint = float(np.sum(xfil * self.vol))
        dfds, dgds = P.sensitivity(xfil, nv, 1.0 / self.V0 if self.method == "mma" else 1.0)
        self.dfds = self.F.density_filter(dfds, True)
        self.dgds = self.F.density_filter(dgds, True)
        if self.method == "mma":
            self.x = self.M.update(self.x, self.dfds, np.array([self.constraint]),
                                   self.dgds, self.xmin, self.xmax)
        else:
            def volume(xt):
                return float(np.sum(self.F.density_filter(xt) * self.vol))
            self.x, _ = O.oc_update(self.x, self.dfds, self.V0, self.dgds, self.xmin,
                                    self.xmax, volume, move=self.move)
        self.xfil = xfil
