"""CPU check of the multigrid's Galerkin coarse operators (numpy / scipy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of
ICARAT_COARSE_GALERKIN; the product (icarat2_b200) never imports it.

The reference has no multigrid (it solves with Eigen's Jacobi-PCG or a direct
solver, src/solver/solvers.cpp:63-91), so there is no reference code to
follow: this restates the definition the GPU hierarchy implements, from the
oracle's own CSR stiffness (Problem.csr, the reference's assembly):

  A_0     = K with the rows and columns of constrained components zero,
            over all 3 numnp components, component-major (c numnp + n);
  A_{l+1} = D_{l+1} P_l^T A_l P_l D_{l+1},

P_l the trilinear prolongation from level l + 1 (every axis halved) to level
l (weight 1 / 2^k for a fine node k half-steps off the coincident coarse
node, per component), D_{l+1} zeroing the components the coarse level
constrains: those whose coincident fine node has them constrained.
"""
import numpy as np
import scipy.sparse as sp


def dims(nx, ny, nz, level):
    s = 2 ** level
    return nx // s, ny // s, nz // s


def full_operator(P):
    """A_0 of an assembled oracle Problem (call P.assemble first) and the
    constrained mask (numnp x 3 bools)."""
    rp, col, val = P.csr()
    dof = P.dof()
    numnp, numeq = P.numnp, P.numeq
    free = dof < numeq
    # free dof number -> component-major index
    inv = np.zeros(numeq, np.int64)
    nodes, comps = np.nonzero(free)
    inv[dof[nodes, comps]] = comps * numnp + nodes
    rows = np.repeat(np.arange(numeq), np.diff(rp))
    A = sp.csr_matrix((val, (inv[rows], inv[col])), shape=(3 * numnp, 3 * numnp))
    return A, ~free


def prolongation(f, c):
    """P (3 numnp_f x 3 numnp_c) from coarse element counts c to fine f."""
    NXf, NYf, NZf = (d + 1 for d in f)
    NXc, NYc, NZc = (d + 1 for d in c)
    nf, nc = NXf * NYf * NZf, NXc * NYc * NZc
    rows, cols, vals = [], [], []
    for k in range(NZf):
        for j in range(NYf):
            for i in range(NXf):
                n = i + NXf * (j + NYf * k)
                for K in {k // 2, (k + 1) // 2}:
                    for J in {j // 2, (j + 1) // 2}:
                        for I in {i // 2, (i + 1) // 2}:
                            w = (1.0 if i == 2 * I else 0.5) * (1.0 if j == 2 * J else 0.5) * \
                                (1.0 if k == 2 * K else 0.5)
                            m = I + NXc * (J + NYc * K)
                            rows.append(n)
                            cols.append(m)
                            vals.append(w)
    P1 = sp.csr_matrix((vals, (rows, cols)), shape=(nf, nc))
    return sp.block_diag([P1, P1, P1], format="csr")


def coarse_mask(fixed_f, f, c):
    """constrained components of the coarse nodes (numnp_c x 3): those of the
    coincident fine node."""
    NXf, NYf = f[0] + 1, f[1] + 1
    NXc, NYc, NZc = (d + 1 for d in c)
    out = np.zeros((NXc * NYc * NZc, 3), bool)
    for K in range(NZc):
        for J in range(NYc):
            for I in range(NXc):
                out[I + NXc * (J + NYc * K)] = fixed_f[2 * I + NXf * (2 * J + NYf * 2 * K)]
    return out


def hierarchy(P, levels):
    """[(A_l, constrained_l)] for l = 0 .. levels - 1 of an assembled Problem."""
    A, fixed = full_operator(P)
    out = [(A, fixed)]
    for l in range(1, levels):
        f, c = dims(P.nx, P.ny, P.nz, l - 1), dims(P.nx, P.ny, P.nz, l)
        Pl = prolongation(f, c)
        fixed = coarse_mask(fixed, f, c)
        D = sp.diags((~fixed).T.ravel().astype(float))
        A = (D @ (Pl.T @ (A @ Pl)) @ D).tocsr()
        out.append((A, fixed))
    return out
