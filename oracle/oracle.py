"""ctypes wrapper of the CPU restatement in icarat_oracle.c.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product (icarat2_b200) never
imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_REFLIB = os.path.join(_HERE, "_ref", "libicarat_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_vp = C.c_void_p

VOLUME_FN = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p)
REF_VOLUME_FN = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_int, C.c_void_p)


def build(ref=False):
    """Compile liboracle.so (and, with ref=True, the reference MMA/OC)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    if ref:
        subprocess.check_call(["make", "-s", "-C", _HERE, "ref"])


class _OCParams(C.Structure):
    _fields_ = [("move", C.c_double), ("iota", C.c_double), ("lmin", C.c_double),
                ("lmax", C.c_double), ("leps", C.c_double), ("maxiter", C.c_int)]


def _load():
    if not os.path.exists(_LIB):
        build()
    L = C.CDLL(_LIB)
    sig = {
        "or_num_threads": (C.c_int, []),
        "or_set_threads": (None, [C.c_int]),
        "or_mesh_box": (None, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                               C.c_double, _dp, _ip]),
        "or_hexa8_ke": (None, [_dp, C.c_double, C.c_double, _dp, C.POINTER(C.c_double)]),
        "or_elastic_D": (None, [C.c_double, C.c_double, _dp]),
        "or_problem_create": (_vp, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_int, _ip, _dp, _dp, C.c_int, _dp,
                                    _dp, C.POINTER(C.c_int)]),
        "or_problem_destroy": (None, [_vp]),
        "or_problem_sizes": (None, [_vp, _ip]),
        "or_problem_nnz": (C.c_long, [_vp]),
        "or_problem_dof": (None, [_vp, _ip]),
        "or_problem_fext": (None, [_vp, _dp]),
        "or_problem_ke0": (None, [_vp, _dp, C.POINTER(C.c_double)]),
        "or_problem_xyz": (None, [_vp, _dp]),
        "or_problem_conn": (None, [_vp, _ip]),
        "or_problem_csr": (None, [_vp, _lp, _ip, _dp]),
        "or_assemble": (None, [_vp, _dp]),
        "or_apply_K": (None, [_vp, _dp, _dp]),
        "or_pcg": (C.c_int, [_vp, _dp, _dp, C.c_double, C.c_int, C.POINTER(C.c_int),
                             C.POINTER(C.c_double)]),
        "or_linear_solve": (C.c_int, [_vp, _dp, C.c_double, C.c_int, _dp,
                                      C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        "or_node_values": (None, [_vp, _dp, _dp]),
        "or_compliance": (C.c_double, [_vp, _dp]),
        "or_sensitivity": (None, [_vp, _dp, _dp, C.c_double, _dp, _dp]),
        "or_filter_create": (_vp, [_vp, C.c_double, C.c_int]),
        "or_filter_create_centroids": (_vp, [C.c_int, _dp, C.c_double]),
        "or_filter_destroy": (None, [_vp]),
        "or_filter_nnz": (C.c_long, [_vp]),
        "or_filter_lists": (None, [_vp, _lp, _ip, _dp]),
        "or_filter_density": (C.c_int, [_vp, _dp, _dp, C.c_int]),
        "or_filter_sensitivity": (None, [_vp, _dp, _dp, _dp, _dp]),
        "or_threshold": (None, [C.c_int, _dp, C.c_double, C.c_double, _dp]),
        "or_helmholtz_filter": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                          C.c_double, C.c_double, _dp, _dp, C.c_int,
                                          C.c_double, C.c_int, C.POINTER(C.c_int)]),
        "or_threshold_deriv": (None, [C.c_int, _dp, C.c_double, C.c_double, _dp]),
        "or_oc_update": (C.c_int, [C.c_int, _dp, _dp, C.c_double, _dp, _dp, _dp,
                                   C.POINTER(_OCParams), VOLUME_FN, C.c_void_p,
                                   C.POINTER(C.c_int)]),
        "or_mma_create": (_vp, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]),
        "or_mma_destroy": (None, [_vp]),
        "or_mma_set_move": (None, [_vp, C.c_double]),
        "or_mma_set_asymptotes": (None, [_vp, C.c_double, C.c_double, C.c_double]),
        "or_mma_set_oscillation": (None, [_vp, C.c_double]),
        "or_mma_update": (None, [_vp, _dp, _dp, _dp, _dp, _dp, _dp]),
        "or_mma_outloops": (C.c_int, [_vp]),
        "or_mma_inner_total": (C.c_int, [_vp]),
        "or_mma_state": (None, [_vp, _dp, _dp, _dp, _dp]),
        "or_loop_set_helmholtz": (None, [_vp, C.c_double, C.c_double]),
        "or_loop_create": (_vp, [_vp, _vp, C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_int, _dp]),
        "or_loop_destroy": (None, [_vp]),
        "or_loop_step": (C.c_int, [_vp]),
        "or_loop_get": (None, [_vp, C.c_int, _dp]),
        "or_loop_scalars": (None, [_vp, _dp, _ip]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


lib = _load()


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def hexa8_ke(X, E=1.0, nu=0.3):
    """24x24 element stiffness and volume of a hexa8 with nodes X (8x3)."""
    ke = np.zeros(576)
    vol = C.c_double()
    lib.or_hexa8_ke(_f64(X).ravel(), E, nu, ke, C.byref(vol))
    return ke.reshape(24, 24), vol.value


def box_bc(dirichlet=(), loads=()):
    """Pack Dirichlet boxes [(flag3, val3, box3x2)] and point loads [(val3, box3x2)]."""
    nd = len(dirichlet)
    df = np.zeros(max(nd, 1) * 3, np.int32)
    dv = np.zeros(max(nd, 1) * 3)
    db = np.zeros(max(nd, 1) * 6)
    for i, (fl, vl, bx) in enumerate(dirichlet):
        df[3 * i:3 * i + 3] = fl
        dv[3 * i:3 * i + 3] = vl
        db[6 * i:6 * i + 6] = np.asarray(bx, float).ravel()
    nl = len(loads)
    lv = np.zeros(max(nl, 1) * 3)
    lb = np.zeros(max(nl, 1) * 6)
    for i, (vl, bx) in enumerate(loads):
        lv[3 * i:3 * i + 3] = vl
        lb[6 * i:6 * i + 6] = np.asarray(bx, float).ravel()
    return nd, df, dv, db, nl, lv, lb


def cantilever_bc(nx, ny, nz, lx=None, ly=None, lz=None, load_node=None):
    """x = 0 face clamped; unit load (0,0,-1) at node (nx, ny/2, 0) by default."""
    lx = float(nx if lx is None else lx)
    ly = float(ny if ly is None else ly)
    lz = float(nz if lz is None else lz)
    if load_node is None:
        load_node = (nx, ny // 2, 0)
    p = (load_node[0] * lx / nx, load_node[1] * ly / ny, load_node[2] * lz / nz)
    dirichlet = [((1, 1, 1), (0.0, 0.0, 0.0), ((0.0, 0.0), (0.0, ly), (0.0, lz)))]
    loads = [((0.0, 0.0, -1.0), ((p[0], p[0]), (p[1], p[1]), (p[2], p[2])))]
    return dirichlet, loads


class Problem:
    """Mesh + boundary conditions + CSR K_ff of the CPU restatement."""

    def __init__(self, nx, ny, nz, lx=None, ly=None, lz=None, E1=1e-9, E2=1.0,
                 nu=0.3, penal=3.0, dirichlet=None, loads=None):
        lx = float(nx if lx is None else lx)
        ly = float(ny if ly is None else ly)
        lz = float(nz if lz is None else lz)
        if dirichlet is None and loads is None:
            dirichlet, loads = cantilever_bc(nx, ny, nz, lx, ly, lz)
        nd, df, dv, db, nl, lv, lb = box_bc(dirichlet or (), loads or ())
        st = C.c_int()
        self.h = lib.or_problem_create(nx, ny, nz, lx, ly, lz, E1, E2, nu, penal,
                                       nd, df, dv, db, nl, lv, lb, C.byref(st))
        if not self.h:
            raise ValueError("or_problem_create failed: %d" % st.value)
        s = np.zeros(4, np.int32)
        lib.or_problem_sizes(self.h, s)
        self.numnp, self.nelx, self.neq, self.numeq = (int(v) for v in s)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.penal, self.E1, self.E2, self.nu = penal, E1, E2, nu

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_problem_destroy(self.h)
            self.h = None

    def dof(self):
        d = np.zeros(3 * self.numnp, np.int32)
        lib.or_problem_dof(self.h, d)
        return d.reshape(-1, 3)

    def fext(self):
        f = np.zeros(max(self.numeq, 1))
        lib.or_problem_fext(self.h, f)
        return f[:self.numeq]

    def ke0(self):
        k = np.zeros(576)
        v = C.c_double()
        lib.or_problem_ke0(self.h, k, C.byref(v))
        return k.reshape(24, 24), v.value

    def xyz(self):
        x = np.zeros(3 * self.numnp)
        lib.or_problem_xyz(self.h, x)
        return x.reshape(-1, 3)

    def conn(self):
        c = np.zeros(8 * self.nelx, np.int32)
        lib.or_problem_conn(self.h, c)
        return c.reshape(-1, 8)

    def assemble(self, design_s):
        lib.or_assemble(self.h, _f64(design_s))

    def csr(self):
        nnz = lib.or_problem_nnz(self.h)
        rp = np.zeros(self.numeq + 1, np.int64)
        col = np.zeros(max(nnz, 1), np.int32)
        val = np.zeros(max(nnz, 1))
        lib.or_problem_csr(self.h, rp, col, val)
        return rp, col[:nnz], val[:nnz]

    def apply_K(self, u):
        y = np.zeros(self.numeq)
        lib.or_apply_K(self.h, _f64(u), y)
        return y

    def pcg(self, rhs, tol=1e-10, maxit=10000):
        sol = np.zeros(self.numeq)
        it = C.c_int()
        rr = C.c_double()
        lib.or_pcg(self.h, _f64(rhs), sol, tol, maxit, C.byref(it), C.byref(rr))
        return sol, it.value, rr.value

    def solve(self, design_s, tol=1e-10, maxit=10000):
        """LinearAnalysis::solve: returns (value.val, iterations, rel. residual)."""
        val = np.zeros(max(self.numeq, 1))
        it = C.c_int()
        rr = C.c_double()
        lib.or_linear_solve(self.h, _f64(design_s), tol, maxit, val, C.byref(it),
                            C.byref(rr))
        return val[:self.numeq], it.value, rr.value

    def node_values(self, val):
        nv = np.zeros(3 * self.numnp)
        lib.or_node_values(self.h, _f64(val), nv)
        return nv.reshape(-1, 3)

    def compliance(self, val):
        return lib.or_compliance(self.h, _f64(val))

    def sensitivity(self, design_s, node_val, dgds_scale=1.0):
        dfds = np.zeros(self.nelx)
        dgds = np.zeros(self.nelx)
        lib.or_sensitivity(self.h, _f64(design_s), _f64(node_val).ravel(), dgds_scale,
                           dfds, dgds)
        return dfds, dgds


class Filter:
    """Filter<E,N> restatement (radius density filter)."""

    def __init__(self, problem=None, radius=1.5, faithful=False, centroids=None):
        if centroids is not None:
            cen = _f64(centroids).reshape(-1, 3)
            self.n = cen.shape[0]
            self.h = lib.or_filter_create_centroids(self.n, cen.ravel(), radius)
        else:
            self.n = problem.nelx
            self.h = lib.or_filter_create(problem.h, radius, 1 if faithful else 0)
        self.radius = radius

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_filter_destroy(self.h)
            self.h = None

    def lists(self):
        nnz = lib.or_filter_nnz(self.h)
        ptr = np.zeros(self.n + 1, np.int64)
        ids = np.zeros(max(nnz, 1), np.int32)
        dis = np.zeros(max(nnz, 1))
        lib.or_filter_lists(self.h, ptr, ids, dis)
        return ptr, ids[:nnz], dis[:nnz]

    def density_filter(self, x, is_sens=False):
        out = np.zeros(self.n)
        st = lib.or_filter_density(self.h, _f64(x), out, 1 if is_sens else 0)
        if st != 0:
            raise RuntimeError("or_filter_density: status %d" % st)
        return out

    def sensitivity_filter(self, design_s, dfds, volume):
        out = np.zeros(self.n)
        lib.or_filter_sensitivity(self.h, _f64(design_s), _f64(dfds), _f64(volume), out)
        return out


def helmholtz_filter(nx, ny, nz, R, x, is_sens=False, tol=1e-14, lx=None, ly=None, lz=None,
                     maxit=100000):
    """FilterHelmholtz::densityFilter (filter_helm.hpp:76-138) on the box;
    returns (filtered, PCG iterations)."""
    x = _f64(x)
    out = np.zeros(nx * ny * nz)
    it = C.c_int()
    st = lib.or_helmholtz_filter(nx, ny, nz, float(nx if lx is None else lx),
                                 float(ny if ly is None else ly),
                                 float(nz if lz is None else lz), R, x, out,
                                 1 if is_sens else 0, tol, maxit, C.byref(it))
    if st != 0:
        raise RuntimeError("or_helmholtz_filter: status %d" % st)
    return out, it.value


def threshold(x, beta, T):
    x = _f64(x)
    out = np.zeros_like(x)
    lib.or_threshold(x.size, x, beta, T, out)
    return out


def threshold_derivative(x, beta, T):
    x = _f64(x)
    out = np.zeros_like(x)
    lib.or_threshold_deriv(x.size, x, beta, T, out)
    return out


def oc_update(x, dfdx, g, dgdx, xmin, xmax, volume_fn, move=0.15, iota=0.5,
              lmin=0.0, lmax=1.0e4, leps=1.0e-5, maxiter=100):
    """OC::UpdateVariables with a Python volume functor g(x)."""
    x = _f64(x).copy()
    n = x.size

    def cb(ptr, user):
        return float(volume_fn(np.ctypeslib.as_array(ptr, shape=(n,)).copy()))

    fn = VOLUME_FN(cb)
    prm = _OCParams(move, iota, lmin, lmax, leps, maxiter)
    steps = C.c_int()
    lib.or_oc_update(n, x, _f64(dfdx), g, _f64(dgdx), _f64(xmin), _f64(xmax),
                     C.byref(prm), fn, None, C.byref(steps))
    return x, steps.value


class MMA:
    """MMASolver restatement (Svanberg MMA, dual interior point)."""

    def __init__(self, n, m, a=0.0, c=100000.0, d=0.0):
        self.n, self.m = n, m
        self.h = lib.or_mma_create(n, m, a, c, d)

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_mma_destroy(self.h)
            self.h = None

    def set_move_limit(self, m):
        lib.or_mma_set_move(self.h, m)

    def set_asymptotes(self, init, dec, inc):
        lib.or_mma_set_asymptotes(self.h, init, dec, inc)

    def set_oscillation(self, a):
        lib.or_mma_set_oscillation(self.h, a)

    def update(self, x, dfdx, gx, dgdx, xmin, xmax):
        x = _f64(x).copy()
        lib.or_mma_update(self.h, x, _f64(dfdx), _f64(np.atleast_1d(gx)),
                          _f64(dgdx).ravel(), _f64(xmin), _f64(xmax))
        return x

    def outloops(self):
        return lib.or_mma_outloops(self.h)

    def state(self):
        a = [np.zeros(self.n) for _ in range(4)]
        lib.or_mma_state(self.h, *a)
        return dict(low=a[0], upp=a[1], xold1=a[2], xold2=a[3])


class Loop:
    """One design iteration per step() of the sample drivers (OC / MMA)."""

    def __init__(self, problem, filt, method="mma", x0=0.3, move=None,
                 use_threshold=False, xmin=1e-4, xmax=1.0, cg_tol=1e-10,
                 cg_maxit=10000, helmholtz_R=None, helmholtz_tol=1e-10):
        """filt: a radius Filter, or None with helmholtz_R: the Helmholtz
        filter of radius helmholtz_R solved to helmholtz_tol."""
        self.P, self.F = problem, filt
        if move is None:
            move = 0.15
        x0 = np.full(problem.nelx, x0) if np.isscalar(x0) else _f64(x0)
        self.h = lib.or_loop_create(problem.h, filt.h if filt is not None else None,
                                    1 if method == "mma" else 0,
                                    1 if use_threshold else 0, move, xmin, xmax,
                                    cg_tol, cg_maxit, _f64(x0))
        if helmholtz_R is not None:
            lib.or_loop_set_helmholtz(self.h, helmholtz_R, helmholtz_tol)

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_loop_destroy(self.h)
            self.h = None

    def step(self):
        st = lib.or_loop_step(self.h)
        if st != 0:
            raise RuntimeError("or_loop_step: status %d" % st)

    def get(self, which):
        idx = {"x": 0, "xfil": 1, "xthr": 2, "dfds": 3, "dgds": 4, "val": 5,
               "node_val": 6}[which]
        n = {5: self.P.numeq, 6: 3 * self.P.numnp}.get(idx, self.P.nelx)
        out = np.zeros(max(n, 1))
        lib.or_loop_get(self.h, idx, out)
        return out[:n]

    def scalars(self):
        d = np.zeros(9)
        iv = np.zeros(4, np.int32)
        lib.or_loop_scalars(self.h, d, iv)
        keys = ["compliance", "constraint", "V0", "cg_relres", "t_filter", "t_solve",
                "t_sens", "t_update", "t_pcg"]
        out = {k: float(v) for k, v in zip(keys, d)}
        out.update(optstep=int(iv[0]), cg_iters=int(iv[1]), oc_steps=int(iv[2]),
                   mma_outloops=int(iv[3]))
        return out


class CaseLoop:
    """MMA design loop over several load cases with design / non-design
    element IDs, composed from the primitives above (test infrastructure):
    the loop body of sample/software/opt-multi-load/opt_multi_load.cpp:100-200
    (per case: solve, object_f += u.f, dfds += -(E'/E) u Ke u; volume
    constraint over the design IDs, V0 on step 1) and of
    sample/algorithm/opt-macro-mma-nondesign/opt_macro_mma_nondesign.cpp:
    90-178 (threshold, filter^T, sensitivities zeroed on the non-design IDs
    :161-166, MMA).  problems: one Problem per load case (same mesh and
    Dirichlet boxes); filt: a radius Filter, or None with helmholtz_R."""

    def __init__(self, problems, filt=None, helmholtz_R=None, x0=0.3, design_ids=None,
                 nondesign_ids=(), use_threshold=True, move=0.2, xmin=1e-4, xmax=1.0,
                 cg_tol=1e-12, helmholtz_tol=1e-10):
        self.P = problems
        self.F, self.R, self.htol = filt, helmholtz_R, helmholtz_tol
        n = problems[0].nelx
        self.x = np.full(n, x0) if np.isscalar(x0) else _f64(x0).copy()
        self.design = np.arange(n) if design_ids is None else np.asarray(design_ids)
        self.nondesign = np.asarray(nondesign_ids, dtype=np.int64)
        self.use_thr, self.cg_tol = use_threshold, cg_tol
        self.xmin, self.xmax = np.full(n, xmin), np.full(n, xmax)
        self.mma = MMA(n, 1)
        self.mma.set_move_limit(move)
        self.vol = problems[0].ke0()[1]
        self.optstep, self.V0 = 0, 0.0

    def _filter(self, v, sens):
        if self.R is not None:
            P = self.P[0]
            return helmholtz_filter(P.nx, P.ny, P.nz, self.R, v, is_sens=sens, tol=self.htol,
                                    lx=self.lx, ly=self.ly, lz=self.lz)[0]
        return self.F.density_filter(v, sens)

    lx = ly = lz = None

    def step(self):
        self.optstep += 1
        xfil = self._filter(self.x, False)
        beta = min(2.0 ** int(self.optstep / 40), 16.0)
        if self.use_thr:
            thr, thrd = threshold(xfil, beta, 0.5), threshold_derivative(xfil, beta, 0.5)
        else:
            thr, thrd = xfil.copy(), np.ones_like(xfil)
        const = 0.0
        if self.optstep == 1:
            self.V0 = 0.0
            for e in self.design:
                self.V0 += thr[e] * self.vol
        else:
            for e in self.design:
                const += thr[e] * self.vol / self.V0
            const += -1.0
        comp, dfds, dgds, its = 0.0, np.zeros_like(xfil), None, 0
        for P in self.P:
            val, it, _ = P.solve(thr, tol=self.cg_tol)
            its += it
            comp += P.compliance(val)
            df, dgds = P.sensitivity(thr, P.node_values(val), 1.0 / self.V0)
            dfds += df
        dfds, dgds = dfds * thrd, dgds * thrd
        dfds, dgds = self._filter(dfds, True), self._filter(dgds, True)
        dfds[self.nondesign] = 0.0
        dgds[self.nondesign] = 0.0
        self.x = self.mma.update(self.x, dfds, [const], dgds, self.xmin, self.xmax)
        self.xfil, self.dfds, self.dgds = xfil, dfds, dgds
        return comp, const, its


def hexa8_gauss_B(h):
    """Voigt B (6 x 24) at the 8 Gauss points of an h[0] x h[1] x h[2] voxel
    (src/basis/bmatrix.hpp:125-140 with shape_function.cpp:422-447 and the
    Gauss8Cubic order of gauss_integration.cpp:268-289), and det J."""
    corner = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1),
              (0, 1, 1)]
    g = 1.0 / np.sqrt(3.0)
    Bs = []
    for sx, sy, sz in [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (-1, -1, 1),
                       (1, -1, 1), (1, 1, 1), (-1, 1, 1)]:
        r = np.array([sx, sy, sz]) * g
        B = np.zeros((6, 24))
        for a, c in enumerate(corner):
            s = [1.0 if v else -1.0 for v in c]
            f = [1 + s[d] * r[d] for d in range(3)]
            dx = 0.125 * s[0] * f[1] * f[2] * 2.0 / h[0]
            dy = 0.125 * s[1] * f[0] * f[2] * 2.0 / h[1]
            dz = 0.125 * s[2] * f[0] * f[1] * 2.0 / h[2]
            B[0, 3 * a], B[1, 3 * a + 1], B[2, 3 * a + 2] = dx, dy, dz
            B[3, 3 * a], B[3, 3 * a + 1] = dy, dx
            B[4, 3 * a + 1], B[4, 3 * a + 2] = dz, dy
            B[5, 3 * a], B[5, 3 * a + 2] = dz, dx
        Bs.append(B)
    return Bs


def mises(P, design_s, node_val, lx=None, ly=None, lz=None):
    """Elastic::makeMisesStress (src/problem/elasticity.cpp:166-207) per
    element: stress = sum_ip De B(ip) u_e / ipmax with De of E(rho) (SIMP)
    and the truncated nodal values, mises = sqrt(stress^T V stress)."""
    h = [(lx or P.nx) / P.nx, (ly or P.ny) / P.ny, (lz or P.nz) / P.nz]
    Bs = hexa8_gauss_B(h)
    nu = P.nu
    lam = nu / ((1 + nu) * (1 - 2 * nu))
    mu = 1.0 / (2 * (1 + nu))
    D0 = np.zeros((6, 6))
    D0[:3, :3] = lam
    D0[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
    D0[[3, 4, 5], [3, 4, 5]] = mu
    V = np.array([[1, -.5, -.5, 0, 0, 0], [-.5, 1, -.5, 0, 0, 0], [-.5, -.5, 1, 0, 0, 0],
                  [0, 0, 0, 3, 0, 0], [0, 0, 0, 0, 3, 0], [0, 0, 0, 0, 0, 3]])
    conn = P.conn()
    nv = np.asarray(node_val).reshape(-1, 3)
    rho = np.asarray(design_s)
    E = (1 - rho ** P.penal) * P.E1 + rho ** P.penal * P.E2
    out = np.zeros(P.nelx)
    for e in range(P.nelx):
        ue = nv[conn[e]].ravel()
        st = sum((E[e] * D0) @ (B @ ue) for B in Bs) / 8.0
        out[e] = np.sqrt(max(st @ V @ st, 0.0))
    return out


def vtk_ascii(nx, ny, nz, node_val=None, density=None, mises=None, lx=None, ly=None, lz=None):
    """The bytes the reference's sample output() writes for the box
    (src/io/export_vtk.hpp: makeHeaderVTK :47-53, setPointVTK :67-79,
    setElementVTK :82-101, setElementTypeVTK :104-112, addPointVectorVTK
    :134-151, addElementScalarVTK :153-170); numbers through an ostream's
    default formatting, which is printf %g."""
    lx = float(nx if lx is None else lx)
    ly = float(ny if ly is None else ly)
    lz = float(nz if lz is None else lz)
    xyz = np.zeros(3 * (nx + 1) * (ny + 1) * (nz + 1))
    conn = np.zeros(8 * nx * ny * nz, np.int32)
    lib.or_mesh_box(nx, ny, nz, lx, ly, lz, xyz, conn)
    xyz, conn = xyz.reshape(-1, 3), conn.reshape(-1, 8)
    out = ["# vtk DataFile Version 4.1\nvtk output\nASCII\nDATASET UNSTRUCTURED_GRID\n"]
    out.append("\nPOINTS\t%d\tfloat\n" % len(xyz))
    out += ["".join("%g\t" % v for v in p) + "\n" for p in xyz]
    out.append("\nCELLS %d\t%d\n" % (len(conn), 9 * len(conn)))
    out += ["8\t" + "".join("%d\t" % v for v in c) + "\n" for c in conn]
    out.append("\nCELL_TYPES\t%d\n" % len(conn))
    out += ["12\n"] * len(conn)
    if node_val is not None:
        out.append("\nPOINT_DATA\t%d\nVECTORS displacement float\n" % len(xyz))
        out += ["".join("%g\t" % v for v in p) + "\n" for p in np.asarray(node_val).reshape(-1, 3)]
    first = True
    for name, f in (("density", density), ("mises", mises)):
        if f is None:
            continue
        if first:
            out.append("\nCELL_DATA\t%d\n" % len(conn))
            first = False
        out.append("SCALARS %s float\nLOOKUP_TABLE default\n" % name)
        out += ["%g\n" % v for v in f]
    return "".join(out).encode()


def voxelize(tri, dims, origin, pitch):
    """Ray-parity voxelisation along +z (test infrastructure, the algorithm of
    the library's voxel.cu restated in numpy): per column centre, crossings
    with counter-clockwise-normalised projected triangles under a top-left
    rule, edge functions from the smaller endpoint; odd crossings below a
    centre = inside."""
    tri = np.asarray(tri, dtype=np.float64).reshape(-1, 3, 3)
    nx, ny, nz = dims
    ox, oy, oz = origin
    px, py, pz = pitch

    def efn(ax, ay, bx, by, x, y):
        return (bx - ax) * (y - ay) - (by - ay) * (x - ax)

    def canon(ax, ay, bx, by, x, y):
        sw = (bx < ax) | ((bx == ax) & (by < ay))
        return np.where(sw, -efn(bx, by, ax, ay, x, y), efn(ax, ay, bx, by, x, y))

    def tl(ax, ay, bx, by):
        return ((ay == by) & (bx < ax)) | (by < ay)

    a, b, c = tri[:, 0].copy(), tri[:, 1].copy(), tri[:, 2].copy()
    area = efn(a[:, 0], a[:, 1], b[:, 0], b[:, 1], c[:, 0], c[:, 1])
    keep = area != 0
    a, b, c, area = a[keep], b[keep], c[keep], area[keep]
    neg = area < 0
    b[neg], c[neg] = c[neg].copy(), b[neg].copy()
    area = np.abs(area)
    t0, t1, t2 = tl(b[:, 0], b[:, 1], c[:, 0], c[:, 1]), tl(c[:, 0], c[:, 1], a[:, 0], a[:, 1]), \
        tl(a[:, 0], a[:, 1], b[:, 0], b[:, 1])
    zc = oz + (np.arange(nz) + 0.5) * pz
    mask = np.zeros((nz, ny, nx), np.uint8)
    for j in range(ny):
        for i in range(nx):
            x, y = ox + (i + 0.5) * px, oy + (j + 0.5) * py
            w0 = canon(b[:, 0], b[:, 1], c[:, 0], c[:, 1], x, y)
            w1 = canon(c[:, 0], c[:, 1], a[:, 0], a[:, 1], x, y)
            w2 = canon(a[:, 0], a[:, 1], b[:, 0], b[:, 1], x, y)
            ins = ((w0 > 0) | ((w0 == 0) & t0)) & ((w1 > 0) | ((w1 == 0) & t1)) & \
                  ((w2 > 0) | ((w2 == 0) & t2))
            z = (w0 * a[:, 2] + w1 * b[:, 2] + w2 * c[:, 2])[ins] / area[ins]
            below = np.searchsorted(np.sort(z), zc, side="left")
            mask[:, j, i] = below & 1
    return mask.ravel()


def ref_available():
    return os.path.exists(_REFLIB)


class RefMMA:
    """The reference's own MMASolver (oracle/_ref, compiled from its sources)."""

    _lib = None

    @classmethod
    def _get(cls):
        if cls._lib is None:
            L = C.CDLL(_REFLIB)
            L.ref_mma_create.restype = _vp
            L.ref_mma_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double,
                                         C.c_double]
            L.ref_mma_destroy.argtypes = [_vp]
            L.ref_mma_set_move.argtypes = [_vp, C.c_double]
            L.ref_mma_set_asymptotes.argtypes = [_vp, C.c_double, C.c_double, C.c_double]
            L.ref_mma_set_oscillation.argtypes = [_vp, C.c_double]
            L.ref_mma_update.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp, _dp]
            L.ref_oc_update.argtypes = [C.c_int, _dp, _dp, C.c_double, _dp, _dp, _dp,
                                        C.c_double, REF_VOLUME_FN, C.c_void_p]
            cls._lib = L
        return cls._lib

    def __init__(self, n, m, a=0.0, c=100000.0, d=0.0):
        self.L = self._get()
        self.h = self.L.ref_mma_create(n, m, a, c, d)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_mma_destroy(self.h)
            self.h = None

    def set_move_limit(self, m):
        self.L.ref_mma_set_move(self.h, m)

    def set_asymptotes(self, init, dec, inc):
        self.L.ref_mma_set_asymptotes(self.h, init, dec, inc)

    def set_oscillation(self, a):
        self.L.ref_mma_set_oscillation(self.h, a)

    def update(self, x, dfdx, gx, dgdx, xmin, xmax):
        x = _f64(x).copy()
        self.L.ref_mma_update(self.h, x, _f64(dfdx), _f64(np.atleast_1d(gx)),
                              _f64(dgdx).ravel(), _f64(xmin), _f64(xmax))
        return x


def ref_oc_update(x, dfdx, g, dgdx, xmin, xmax, volume_fn, move=0.15):
    """The reference's own OC::UpdateVariables (oracle/_ref)."""
    L = RefMMA._get()
    x = _f64(x).copy()
    n = x.size

    def cb(ptr, nn, user):
        return float(volume_fn(np.ctypeslib.as_array(ptr, shape=(nn,)).copy()))

    fn = REF_VOLUME_FN(cb)
    L.ref_oc_update(n, x, _f64(dfdx).copy(), g, _f64(dgdx).copy(), _f64(xmin),
                    _f64(xmax), move, fn, None)
    return x


class Convergence:
    """Optimize::isConvergence (src/optimization/opt_base.hpp:28-43): is_convergence
    returns 0 when |object_old - object_f| / object_f < epsilon and optstep >
    minstep, else 1 with object_old = object_f.  object_old starts at 0 (the
    reference leaves it uninitialised)."""

    def __init__(self):
        self.object_old = 0.0

    def is_convergence(self, object_f, optstep, epsilon, minstep):
        old, f = float(self.object_old), float(object_f)
        diff = abs(old - f)
        if f != 0.0:
            ratio = diff / f
        else:
            ratio = float("nan") if diff == 0.0 else float("inf")
        if ratio < epsilon and optstep > minstep:
            return 0
        self.object_old = f
        return 1
