"""icarat2_b200 -- B200 (sm_100a) implementation of ICARAT's linear-static
SIMP topology-optimisation inner loop behind a C ABI (include/icarat_gpu.h).

This module is the Python host side over that ABI.  Its classes mirror the
reference call surface for the path:

    Context            MeshIcarat + BCIcarat + device state
    LinearAnalysis     src/analysis/linear.hpp:15-41   (solve)
    Filter             src/optimization/filter.hpp:17-61
    OC                 src/optimization/opt-solver/OCSolver.hpp:13-80
    MMASolver          src/optimization/opt-solver/MMASolver.hpp:62-116

Every call runs on the GPU through libicarat_gpu.so; there is no CPU path.
Importing fails loudly when the library has not been built
(``python -m icarat2_b200.build``).
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libicarat_gpu.so")

OK = 0
WARN_MAXITER = 1
WARN_STAGNATION = 2
ERR_ARG = -1
ERR_CUDA = -2
ERR_NAN = -4
ERR_STATE = -5
ERR_FILTER = -6
ERR_UNSUPPORTED = -7
ERR_NOMEM = -8

JACOBI_PCG = 0
MG_PCG = 1
MIXED_IR = 2
LEARNED_FPCG = 3

COARSE_REDISCRETISED = 0  # ICARAT_COARSE_*: coarse multigrid operators
COARSE_GALERKIN = 1
OP_FP64 = 0
OP_FP32 = 1
OP_TC_BF16X3 = 2
OP_TC_BF16 = 3
OP_TC_FP64 = 4


class IcaratError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d)" % (msg, status))
        self.status = status


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double)]


class Material(C.Structure):
    _fields_ = [("young_min", C.c_double), ("young_max", C.c_double),
                ("poisson", C.c_double), ("penalty", C.c_double)]


class Dirichlet(C.Structure):
    _fields_ = [("flag", C.c_int * 3), ("val", C.c_double * 3),
                ("box", (C.c_double * 2) * 3)]


class Load(C.Structure):
    _fields_ = [("val", C.c_double * 3), ("box", (C.c_double * 2) * 3)]


class BC(C.Structure):
    _fields_ = [("n_dirichlet", C.c_int), ("dirichlet", C.POINTER(Dirichlet)),
                ("n_loads", C.c_int), ("loads", C.POINTER(Load))]


class SolveOpts(C.Structure):
    _fields_ = [("method", C.c_int), ("rtol", C.c_double), ("maxit", C.c_int),
                ("mg_levels", C.c_int), ("mg_smooth", C.c_int), ("chunk", C.c_int),
                ("refresh", C.c_double), ("fine_op", C.c_int), ("krylov_op", C.c_int),
                ("warm_start", C.c_int), ("fp64_tc", C.c_int), ("coarse_lag", C.c_int),
                ("coarse_op", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("rel_residual", C.c_double),
                ("status", C.c_int), ("refreshes", C.c_int),
                ("learned_iterations", C.c_int)]


class OcOpts(C.Structure):
    _fields_ = [("move", C.c_double), ("iota", C.c_double), ("lambda_min", C.c_double),
                ("lambda_max", C.c_double), ("lambda_eps", C.c_double),
                ("maxiter", C.c_int), ("use_threshold", C.c_int), ("beta", C.c_double),
                ("T", C.c_double), ("filter_kind", C.c_int)]


class LoopOpts(C.Structure):
    _fields_ = [("method", C.c_int), ("use_threshold", C.c_int), ("T", C.c_double),
                ("move", C.c_double), ("xmin", C.c_double), ("xmax", C.c_double),
                ("filter_radius", C.c_double), ("solve", SolveOpts),
                ("filter_kind", C.c_int)]


class BatchOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("maxit", C.c_int), ("refresh", C.c_double),
                ("tile", C.c_int), ("blocks_per_sm", C.c_int), ("method", C.c_int),
                ("mg_levels", C.c_int), ("chunk", C.c_int), ("warm_start", C.c_int)]


class StepInfo(C.Structure):
    _fields_ = [("step", C.c_int), ("compliance", C.c_double),
                ("constraint", C.c_double), ("cg_iterations", C.c_int),
                ("cg_rel_residual", C.c_double), ("update_steps", C.c_int),
                ("status", C.c_int)]


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = C.c_void_p
# ICARAT_ABI_VERSION of include/icarat_gpu.h that the structs below mirror
ABI_VERSION = 10300

_i = C.c_int
_d = C.c_double
_P = C.POINTER

# every symbol of include/icarat_gpu.h with its ctypes signature
SIGNATURES = {
    "icarat_version": (_i, []),
    "icarat_status_string": (C.c_char_p, [_i]),
    "icarat_last_error": (C.c_char_p, []),
    "icarat_ctx_create": (_i, [_P(Grid), _P(Material), _P(BC), _i, _P(_vp)]),
    "icarat_ctx_destroy": (_i, [_vp]),
    "icarat_sizes": (_i, [_vp, _P(_i), _P(_i), _P(_i), _P(_i)]),
    "icarat_stream": (_i, [_vp, _P(_vp)]),
    "icarat_synchronize": (_i, [_vp]),
    "icarat_dof_map": (_i, [_vp, _ip]),
    "icarat_fext": (_i, [_vp, _dp]),
    "icarat_element_stiffness": (_i, [_vp, _dp, _P(_d)]),
    "icarat_set_design": (_i, [_vp, _dp]),
    "icarat_set_design_dev": (_i, [_vp, _vp]),
    "icarat_apply_K": (_i, [_vp, _dp, _dp]),
    "icarat_apply_K_dev": (_i, [_vp, _vp, _vp]),
    "icarat_solve": (_i, [_vp, _P(SolveOpts), _vp, _P(SolveInfo)]),
    "icarat_solve_rhs": (_i, [_vp, _P(SolveOpts), _dp, _vp, _P(SolveInfo)]),
    "icarat_node_values": (_i, [_vp, _dp]),
    "icarat_compliance": (_i, [_vp, _P(_d)]),
    "icarat_sensitivity": (_i, [_vp, _d, _vp, _vp]),
    "icarat_sensitivity_dev": (_i, [_vp, _d, _vp, _vp]),
    "icarat_filter_setup": (_i, [_vp, _d]),
    "icarat_density_filter": (_i, [_vp, _dp, _dp, _i]),
    "icarat_density_filter_dev": (_i, [_vp, _vp, _vp, _i]),
    "icarat_sensitivity_filter": (_i, [_vp, _dp, _dp, _dp]),
    "icarat_set_load_cases": (_i, [_vp, _i, _vp]),
    "icarat_mises": (_i, [_vp, _dp]),
    "icarat_mises_dev": (_i, [_vp, _vp]),
    "icarat_write_vtk": (_i, [_vp, C.c_char_p, _i]),
    "icarat_voxelize": (_i, [_i, _dp, _i, _i, _i, _i, _dp, _dp, _vp]),
    "icarat_write_vtk_arrays": (_i, [C.c_char_p, _i, _i, _i, _i, _d, _d, _d, _vp, _vp, _vp]),
    "icarat_loop_set_domains": (_i, [_vp, _vp, _i, _vp, _i]),
    "icarat_helmholtz_setup": (_i, [_vp, _d]),
    "icarat_helmholtz_filter": (_i, [_vp, _dp, _dp, _i, _d, _i, _P(SolveInfo)]),
    "icarat_helmholtz_filter_dev": (_i, [_vp, _vp, _vp, _i, _d, _i, _P(SolveInfo)]),
    "icarat_threshold": (_i, [_vp, _dp, _d, _d, _dp]),
    "icarat_threshold_derivative": (_i, [_vp, _dp, _d, _d, _dp]),
    "icarat_oc_update": (_i, [_vp, _dp, _dp, _d, _dp, _dp, _dp, _P(OcOpts), _P(_i)]),
    "icarat_oc_update_dev": (_i, [_vp, _vp, _vp, _d, _vp, _vp, _vp, _P(OcOpts),
                                  _P(_i)]),
    "icarat_mma_create": (_i, [_i, _i, _i, _d, _d, _d, _P(_vp)]),
    "icarat_mma_destroy": (_i, [_vp]),
    "icarat_mma_set_move_limit": (_i, [_vp, _d]),
    "icarat_mma_set_asymptotes": (_i, [_vp, _d, _d, _d]),
    "icarat_mma_set_oscillation": (_i, [_vp, _d]),
    "icarat_mma_update": (_i, [_vp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "icarat_mma_update_dev": (_i, [_vp, _vp, _vp, _dp, _vp, _vp, _vp]),
    "icarat_mma_last_loops": (_i, [_vp, _P(_i), _P(_i)]),
    "icarat_solve_noalloc": (_i, [_vp, _P(SolveOpts), _vp, _vp, _P(SolveInfo)]),
    "icarat_kernel_launches": (_i, [_P(C.c_ulonglong)]),
    "icarat_time_operator": (_i, [_vp, _i, _P(_d)]),
    "icarat_apply_K_op": (_i, [_vp, _i, _dp, _dp]),
    "icarat_net_create": (_i, [_i, C.c_ulonglong, _P(_vp)]),
    "icarat_net_destroy": (_i, [_vp]),
    "icarat_net_num_params": (_i, [_vp, _P(C.c_longlong)]),
    "icarat_net_get_params": (_i, [_vp, _vp]),
    "icarat_net_set_params": (_i, [_vp, _vp]),
    "icarat_net_train_step": (_i, [_vp, _vp, _dp, _dp, _dp, _d, _P(_d)]),
    "icarat_net_get_grads": (_i, [_vp, _vp]),
    "icarat_net_infer": (_i, [_vp, _vp, _dp, _dp]),
    "icarat_net_infer_dev": (_i, [_vp, _vp, _vp, _vp]),
    "icarat_ctx_set_net": (_i, [_vp, _vp]),
    "icarat_batch_create": (_i, [_vp, _vp, _i, _P(Material), _i, _P(_vp)]),
    "icarat_batch_destroy": (_i, [_vp]),
    "icarat_batch_ctx": (_i, [_vp, _i, _P(_vp)]),
    "icarat_batch_autotune": (_i, [_vp, _P(_i), _P(_i), _P(_d)]),
    "icarat_batch_autotune_mg": (_i, [_vp, _i, _P(_i), _P(_i), _P(_d)]),
    "icarat_batch_solve": (_i, [_vp, _P(BatchOpts), _vp]),
    "icarat_batch_solution": (_i, [_vp, _i, _dp]),
    "icarat_batch_loop_step": (_i, [_vp, _P(BatchOpts), _vp]),
    "icarat_time_operator_op": (_i, [_vp, _i, _i, _P(_d)]),
    "icarat_mg_coarse_check": (_i, [_vp, _i, _P(_d), _P(_i)]),
    "icarat_mg_level_apply": (_i, [_vp, _P(SolveOpts), _i, _dp, _dp]),
    "icarat_loop_init": (_i, [_vp, _P(LoopOpts), _dp]),
    "icarat_loop_step": (_i, [_vp, _P(StepInfo)]),
    "icarat_loop_get": (_i, [_vp, _i, _dp]),
    "icarat_loop_is_convergence": (_i, [_vp, _d, _d, _P(_i)]),
    "icarat_loop_save": (_i, [_vp, C.c_char_p]),
    "icarat_loop_load": (_i, [_vp, C.c_char_p]),
    "icarat_ctx_create_selection": (_i, [_P(Grid), _P(Material), _P(BC), _i, _dp, _i,
                                         _P(_vp)]),
    "icarat_selection_ids": (_i, [_vp, _vp, _vp]),
}

_lib = None


def load_library(path=LIBPATH):
    """Load libicarat_gpu.so (raises if it is missing: no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libicarat_gpu.so not built; run python -m icarat2_b200.build")
    L = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.icarat_version() != ABI_VERSION:
        raise ImportError("libicarat_gpu.so has ABI %d, these bindings %d: rebuild with "
                          "python -m icarat2_b200.build" % (L.icarat_version(), ABI_VERSION))
    _lib = L
    return L


def _check(status, what):
    if status < 0:
        msg = _lib.icarat_last_error().decode() or _lib.icarat_status_string(status).decode()
        raise IcaratError(status, "%s: %s" % (what, msg))
    return status


def _out(a, n):
    """A caller's output array: contiguous float64 with at least n entries."""
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
            and a.size >= max(n, 1)):
        raise ValueError("out must be a contiguous float64 array of %d entries" % n)
    return a


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _box(b):
    arr = ((C.c_double * 2) * 3)()
    for a in range(3):
        arr[a][0], arr[a][1] = float(b[a][0]), float(b[a][1])
    return arr


def nondesign_boxes(nx, ny, nz, boxes, designs_0, lx=None, ly=None, lz=None):
    """getDesignNonDesignIDs of opt_macro_mma_nondesign.cpp:247-317 on the
    voxel box: boxes is a list of (value, ((x0, x1), (y0, y1), (z0, z1))); an
    element whose centroid lies strictly inside a box is non-design and
    starts at that box's value.  As in the reference, each box adds every
    element outside it to the design IDs, so with two or more disjoint boxes
    every element counts in the volume.  Returns (x0, design_ids,
    nondesign_ids)."""
    lx = float(nx if lx is None else lx)
    ly = float(ny if ly is None else ly)
    lz = float(nz if lz is None else lz)
    hx, hy, hz = lx / nx, ly / ny, lz / nz
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    # centroid as the mean of the 8 corner coordinates, corner by corner
    cx = sum(((i + a) * hx) / 8.0 for a in (0, 1, 1, 0, 0, 1, 1, 0)).ravel()
    cy = sum(((j + b) * hy) / 8.0 for b in (0, 0, 1, 1, 0, 0, 1, 1)).ravel()
    cz = sum(((k + c) * hz) / 8.0 for c in (0, 0, 0, 0, 1, 1, 1, 1)).ravel()
    x0 = np.full(nx * ny * nz, float(designs_0))
    design, nondesign = [], []
    for value, ((x_0, x_1), (y_0, y_1), (z_0, z_1)) in boxes:
        inside = (x_0 < cx) & (cx < x_1) & (y_0 < cy) & (cy < y_1) & (z_0 < cz) & (cz < z_1)
        nondesign.append(np.nonzero(inside)[0])
        design.append(np.nonzero(~inside)[0])
        x0[inside] = value
    if not boxes:
        design = [np.arange(nx * ny * nz)]
    d = np.unique(np.concatenate(design)) if design else np.zeros(0, np.int64)
    nd = np.unique(np.concatenate(nondesign)) if nondesign else np.zeros(0, np.int64)
    return x0, d.astype(np.int32), nd.astype(np.int32)


def write_vtk_arrays(path, nx, ny, nz, node_val=None, density=None, mises=None, binary=False,
                     lx=None, ly=None, lz=None):
    """icarat_write_vtk_arrays: the VTK writer on host arrays (no GPU work)."""
    L = load_library()
    lx = float(nx if lx is None else lx)
    ly = float(ny if ly is None else ly)
    lz = float(nz if lz is None else lz)
    keep = []

    def ptr(a, n):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        if a.size != n:
            raise ValueError("array of %d values expected" % n)
        keep.append(a)
        return a.ctypes.data

    numnp, nelx = (nx + 1) * (ny + 1) * (nz + 1), nx * ny * nz
    _check(L.icarat_write_vtk_arrays(os.fsencode(path), 1 if binary else 0, nx, ny, nz, lx, ly,
                                     lz, ptr(node_val, 3 * numnp), ptr(density, nelx),
                                     ptr(mises, nelx)), "write_vtk_arrays")


def read_stl(path):
    """Triangles of a binary or ASCII STL file as an (ntri, 9) float64 array
    (three xyz vertices per row)."""
    data = open(path, "rb").read()
    if len(data) >= 84:
        n = int(np.frombuffer(data[80:84], "<u4")[0])
        if len(data) == 84 + 50 * n:
            rec = np.frombuffer(data[84:], np.dtype([("n", "<f4", 3), ("v", "<f4", 9),
                                                     ("a", "<u2")]), count=n)
            return rec["v"].astype(np.float64)
    verts = [list(map(float, ln.split()[1:4])) for ln in data.decode(errors="replace").splitlines()
             if ln.strip().startswith("vertex")]
    if not verts or len(verts) % 3:
        raise ValueError("%s: not an STL file" % path)
    return np.array(verts, dtype=np.float64).reshape(-1, 9)


def voxelize(tri, dims, origin, pitch, device=0):
    """icarat_voxelize: inside (1) / outside (0) of the closed surface tri
    for the voxel centres of the grid; flat uint8 array, x fastest."""
    L = load_library()
    tri = np.ascontiguousarray(tri, dtype=np.float64).reshape(-1, 9)
    nx, ny, nz = (int(v) for v in dims)
    mask = np.zeros(nx * ny * nz, np.uint8)
    _check(L.icarat_voxelize(device, tri.ravel(), tri.shape[0], nx, ny, nz,
                             _f64(origin), _f64(pitch), mask.ctypes.data), "voxelize")
    return mask


def voxelize_stl(stl, mesh_size=100, cubic=False, device=0):
    """The grid of scripts/stl_to_vtk_voxel.py: mesh_size cells per axis over
    the surface's bounding box, pitch (max - min) / mesh_size per axis
    ("rect") or the largest extent / mesh_size on every axis ("cubic"); stl
    is a path or an (ntri, 9) array.  Returns (mask, dims, origin, pitch)."""
    tri = read_stl(stl) if isinstance(stl, (str, bytes, os.PathLike)) else np.asarray(stl)
    v = tri.reshape(-1, 3)
    lo, hi = v.min(axis=0), v.max(axis=0)
    ext = hi - lo
    pitch = np.full(3, ext.max() / mesh_size) if cubic else ext / mesh_size
    dims = (mesh_size, mesh_size, mesh_size)
    return voxelize(tri, dims, lo, pitch, device), dims, lo, pitch


def design_nondesign_ids(nelx, nondesign_ids):
    """getDesignNonDesignIDs of src/misc/non_design_domain.hpp:9-53 from
    element ID lists: (all minus the sorted unique non-design IDs, those IDs)."""
    nd = np.unique(np.asarray(nondesign_ids, dtype=np.int64))
    d = np.setdiff1d(np.arange(nelx), nd)
    return d.astype(np.int32), nd.astype(np.int32)


def cantilever_bc(nx, ny, nz, lx=None, ly=None, lz=None, load_node=None, load=(0.0, 0.0, -1.0)):
    """x = 0 face clamped; point load at node (nx, ny/2, 0) by default."""
    lx = float(nx if lx is None else lx)
    ly = float(ny if ly is None else ly)
    lz = float(nz if lz is None else lz)
    if load_node is None:
        load_node = (nx, ny // 2, 0)
    p = (load_node[0] * lx / nx, load_node[1] * ly / ny, load_node[2] * lz / nz)
    dirichlet = [((1, 1, 1), (0.0, 0.0, 0.0), ((0.0, 0.0), (0.0, ly), (0.0, lz)))]
    loads = [(tuple(load), ((p[0], p[0]), (p[1], p[1]), (p[2], p[2])))]
    return dirichlet, loads


def _bc_struct(dirichlet, loads):
    dirichlet = list(dirichlet or [])
    loads = list(loads or [])
    d = (Dirichlet * max(1, len(dirichlet)))()
    for i, (fl, vl, bx) in enumerate(dirichlet):
        d[i].flag = (C.c_int * 3)(*fl)
        d[i].val = (C.c_double * 3)(*vl)
        d[i].box = _box(bx)
    lo = (Load * max(1, len(loads)))()
    for i, (vl, bx) in enumerate(loads):
        lo[i].val = (C.c_double * 3)(*vl)
        lo[i].box = _box(bx)
    return BC(len(dirichlet), d, len(loads), lo), d, lo


def solve_opts(method=JACOBI_PCG, rtol=1e-10, maxit=10000, mg_levels=4, mg_smooth=2,
               chunk=0, refresh=0.0, fine_op=0, krylov_op=0, warm_start=0, fp64_tc=0,
               coarse_lag=0, coarse_op=COARSE_REDISCRETISED):
    """fp64_tc (JACOBI_PCG, MG_PCG): FP64 products by the node stencil (0,
    the default, and -1; the faster operator at every measured size) or on
    the FP64 tensor cores on every level of 32k nodes and more (1).
    coarse_lag (MG_PCG, MIXED_IR): keep the previous design's coarsest factor
    while this design's is computed on a second stream.  coarse_op (MG_PCG,
    MIXED_IR): COARSE_REDISCRETISED (default) or COARSE_GALERKIN coarse
    operators."""
    return SolveOpts(method, rtol, maxit, mg_levels, mg_smooth, chunk, refresh, fine_op,
                     krylov_op, warm_start, int(fp64_tc), int(bool(coarse_lag)),
                     int(coarse_op))


class Context:
    """A hexa8 voxel box with its boundary conditions, resident on one GPU."""

    def __init__(self, nx, ny, nz, lx=None, ly=None, lz=None, young=(1e-9, 1.0),
                 poisson=0.3, penalty=3.0, dirichlet=None, loads=None, device=0,
                 selection=None):
        """selection: the [mesh] selection boxes, ((x0, x1), (y0, y1), (z0, z1))
        each (MeshIcarat::modifyMesh); sizes, element and node vectors are then
        those of the kept mesh."""
        L = load_library()
        lx = float(nx if lx is None else lx)
        ly = float(ny if ly is None else ly)
        lz = float(nz if lz is None else lz)
        if dirichlet is None and loads is None:
            dirichlet, loads = cantilever_bc(nx, ny, nz, lx, ly, lz)
        dirichlet = list(dirichlet or [])
        loads = list(loads or [])
        bc, self._dir, self._loads = _bc_struct(dirichlet, loads)
        grid = Grid(nx, ny, nz, lx, ly, lz)
        mat = Material(young[0], young[1], poisson, penalty)
        h = C.c_void_p()
        if selection is None:
            _check(L.icarat_ctx_create(C.byref(grid), C.byref(mat), C.byref(bc), device,
                                       C.byref(h)), "icarat_ctx_create")
        else:
            boxes = np.ascontiguousarray(np.asarray(selection, dtype=np.float64).reshape(-1, 6))
            _check(L.icarat_ctx_create_selection(C.byref(grid), C.byref(mat), C.byref(bc),
                                                 boxes.shape[0], boxes.ravel(), device,
                                                 C.byref(h)), "icarat_ctx_create_selection")
        self._adopt(h, L, (nx, ny, nz), young, poisson, penalty, owned=True)

    def selection_ids(self):
        """(box node id of every node, box element id of every element)"""
        nodes = np.zeros(max(self.numnp, 1), np.int32)
        elems = np.zeros(max(self.nelx, 1), np.int32)
        _check(self.lib.icarat_selection_ids(self.h, nodes.ctypes.data, elems.ctypes.data),
               "selection_ids")
        return nodes[:self.numnp], elems[:self.nelx]

    def _adopt(self, h, L, dims, young, poisson, penalty, owned):
        self.h = h
        self.lib = L
        self._owned = owned
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(L.icarat_sizes(h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)), "sizes")
        self.numnp, self.nelx, self.neq, self.numeq = a.value, b.value, c.value, d.value
        self.nx, self.ny, self.nz = dims
        self.young, self.poisson, self.penalty = young, poisson, penalty

    @classmethod
    def _member(cls, h, L, dims, young, poisson, penalty):
        """A context owned by a Batch (not destroyed by this object)."""
        obj = cls.__new__(cls)
        obj._adopt(h, L, dims, young, poisson, penalty, owned=False)
        return obj

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.lib.icarat_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- mesh / BC -----------------------------------------------------------
    def stream_ptr(self):
        s = C.c_void_p()
        _check(self.lib.icarat_stream(self.h, C.byref(s)), "stream")
        return s.value or 0

    def synchronize(self):
        _check(self.lib.icarat_synchronize(self.h), "synchronize")

    def dof_map(self):
        d = np.zeros(3 * self.numnp, np.int32)
        _check(self.lib.icarat_dof_map(self.h, d), "dof_map")
        return d.reshape(-1, 3)

    def fext(self):
        f = np.zeros(max(self.numeq, 1))
        _check(self.lib.icarat_fext(self.h, f), "fext")
        return f[:self.numeq]

    def element_stiffness(self):
        k = np.zeros(576)
        v = C.c_double()
        _check(self.lib.icarat_element_stiffness(self.h, k, C.byref(v)), "element_stiffness")
        return k.reshape(24, 24), v.value

    # --- analysis ------------------------------------------------------------
    def set_design(self, design_s):
        _check(self.lib.icarat_set_design(self.h, _f64(design_s)), "set_design")

    def set_design_dev(self, ptr):
        _check(self.lib.icarat_set_design_dev(self.h, C.c_void_p(ptr)), "set_design_dev")

    def apply_K(self, u):
        y = np.zeros(max(self.numeq, 1))
        _check(self.lib.icarat_apply_K(self.h, _f64(u), y), "apply_K")
        return y[:self.numeq]

    def apply_K_dev(self, uptr, yptr):
        _check(self.lib.icarat_apply_K_dev(self.h, C.c_void_p(uptr), C.c_void_p(yptr)),
               "apply_K_dev")

    def solve(self, opts=None, want_val=True, out=None):
        """LinearAnalysis::solve: returns (value.val, SolveInfo); out: an
        optional float64 array of numeq entries (e.g. in pinned memory) that
        receives value.val."""
        info = SolveInfo()
        val = (_out(out, self.numeq) if out is not None else np.zeros(max(self.numeq, 1))) \
            if want_val else None
        st = self.lib.icarat_solve(self.h, C.byref(opts) if opts is not None else None,
                                   val.ctypes.data if want_val else None, C.byref(info))
        _check(st, "solve")
        return (val[:self.numeq] if want_val else None), info

    def solve_rhs(self, f, opts=None):
        info = SolveInfo()
        u = np.zeros(max(self.numeq, 1))
        st = self.lib.icarat_solve_rhs(self.h, C.byref(opts) if opts is not None else None,
                                       _f64(f), u.ctypes.data, C.byref(info))
        _check(st, "solve_rhs")
        return u[:self.numeq], info

    def solve_noalloc(self, f_ptr, u_ptr, opts=None):
        """Jacobi-PCG solve on device pointers that allocates no device memory
        (work vectors in the library's static buffer); returns SolveInfo."""
        info = SolveInfo()
        st = self.lib.icarat_solve_noalloc(self.h, C.byref(opts) if opts is not None else None,
                                           C.c_void_p(f_ptr), C.c_void_p(u_ptr),
                                           C.byref(info))
        _check(st, "solve_noalloc")
        return info

    def node_values(self):
        v = np.zeros(3 * self.numnp)
        _check(self.lib.icarat_node_values(self.h, v), "node_values")
        return v.reshape(-1, 3)

    def compliance(self):
        c = C.c_double()
        _check(self.lib.icarat_compliance(self.h, C.byref(c)), "compliance")
        return c.value

    def sensitivity(self, dgds_scale=1.0, out=None):
        """(dfds, dgds); out: an optional pair of float64 arrays of nelx
        entries that receive them."""
        dfds = _out(out[0], self.nelx) if out is not None else np.zeros(self.nelx)
        dgds = _out(out[1], self.nelx) if out is not None else np.zeros(self.nelx)
        _check(self.lib.icarat_sensitivity(self.h, dgds_scale, dfds.ctypes.data,
                                           dgds.ctypes.data), "sensitivity")
        return dfds, dgds

    # --- filter ----------------------------------------------------------------
    def filter_setup(self, radius):
        _check(self.lib.icarat_filter_setup(self.h, radius), "filter_setup")

    def density_filter(self, x, is_sens=False, out=None):
        out = _out(out, self.nelx) if out is not None else np.zeros(self.nelx)
        _check(self.lib.icarat_density_filter(self.h, _f64(x), out, 1 if is_sens else 0),
               "density_filter")
        return out

    def helmholtz_setup(self, radius):
        _check(self.lib.icarat_helmholtz_setup(self.h, radius), "helmholtz_setup")

    def helmholtz_filter(self, x, is_sens=False, rtol=0.0, maxit=0, out=None):
        """FilterHelmholtz::densityFilter: returns (filtered, SolveInfo of the
        nodal CG); rtol <= 0 / maxit <= 0 take 1e-10 / 10000."""
        out = _out(out, self.nelx) if out is not None else np.zeros(self.nelx)
        info = SolveInfo()
        _check(self.lib.icarat_helmholtz_filter(self.h, _f64(x), out, 1 if is_sens else 0,
                                                rtol, maxit, C.byref(info)),
               "helmholtz_filter")
        return out, info

    def helmholtz_filter_dev(self, in_ptr, out_ptr, is_sens=False, rtol=0.0, maxit=0):
        info = SolveInfo()
        _check(self.lib.icarat_helmholtz_filter_dev(self.h, C.c_void_p(in_ptr),
                                                    C.c_void_p(out_ptr), 1 if is_sens else 0,
                                                    rtol, maxit, C.byref(info)),
               "helmholtz_filter_dev")
        return info

    def sensitivity_filter(self, design_s, dfds):
        out = np.zeros(self.nelx)
        _check(self.lib.icarat_sensitivity_filter(self.h, _f64(design_s), _f64(dfds), out),
               "sensitivity_filter")
        return out

    def threshold(self, x, beta, T):
        out = np.zeros(self.nelx)
        _check(self.lib.icarat_threshold(self.h, _f64(x), beta, T, out), "threshold")
        return out

    def threshold_derivative(self, x, beta, T):
        out = np.zeros(self.nelx)
        _check(self.lib.icarat_threshold_derivative(self.h, _f64(x), beta, T, out),
               "threshold_derivative")
        return out

    def oc_update(self, x, dfdx, g, dgdx, xmin, xmax, move=0.15, iota=0.5,
                  lambda_min=0.0, lambda_max=1.0e4, lambda_eps=1.0e-5, maxiter=100,
                  use_threshold=False, beta=1.0, T=0.5, filter="radius"):
        """OC::UpdateVariables with the drivers' volume functor over the
        context's radius filter or (filter="helmholtz") its Helmholtz filter"""
        if filter not in ("radius", "helmholtz"):
            raise ValueError("filter must be 'radius' or 'helmholtz'")
        x = _f64(x).copy()
        o = OcOpts(move, iota, lambda_min, lambda_max, lambda_eps, maxiter,
                   1 if use_threshold else 0, beta, T, 1 if filter == "helmholtz" else 0)
        steps = C.c_int()
        _check(self.lib.icarat_oc_update(self.h, x, _f64(dfdx), g, _f64(dgdx), _f64(xmin),
                                         _f64(xmax), C.byref(o), C.byref(steps)),
               "oc_update")
        return x, steps.value

    # --- design loop -------------------------------------------------------------
    def loop_init(self, x0, method="mma", filter_radius=1.5, move=None, xmin=1e-4,
                  xmax=1.0, use_threshold=False, T=0.5, solve=None, filter="radius"):
        """filter: "radius" (Filter, filter.hpp) or "helmholtz" (FilterHelmholtz,
        filter_helm.hpp, as opt_macro_oc.cpp / opt_mma_Helmholtz.cpp use)."""
        if filter not in ("radius", "helmholtz"):
            raise ValueError("filter must be 'radius' or 'helmholtz'")
        if move is None:
            move = 0.2 if method == "mma" else 0.15
        if np.isscalar(x0):
            x0 = np.full(self.nelx, float(x0))
        o = LoopOpts(1 if method == "mma" else 0, 1 if use_threshold else 0, T, move, xmin,
                     xmax, filter_radius, solve if solve is not None else solve_opts(),
                     1 if filter == "helmholtz" else 0)
        _check(self.lib.icarat_loop_init(self.h, C.byref(o), _f64(x0)), "loop_init")

    def mg_level_apply(self, level, x, opts=None):
        """y = A_level x for the V-cycle of opts (mg_levels, coarse_op) on the
        current design; x and y component-major over the level's nodes."""
        o = opts if opts is not None else solve_opts(MG_PCG)
        xx = np.ascontiguousarray(x, dtype=np.float64)
        s = 2 ** int(level)
        n = 3 * (self.nx // s + 1) * (self.ny // s + 1) * (self.nz // s + 1)
        if xx.size != n:
            raise ValueError("x must hold %d entries on level %d" % (n, level))
        y = np.zeros_like(xx)
        _check(self.lib.icarat_mg_level_apply(self.h, C.byref(o), int(level), xx, y),
               "icarat_mg_level_apply")
        return y

    def coarse_check(self, mg_levels=4):
        """(||b - K_c x|| / ||b||, unknowns) of the multigrid's coarsest dense
        solve on the current design."""
        r, n = C.c_double(), C.c_int()
        _check(self.lib.icarat_mg_coarse_check(self.h, mg_levels, C.byref(r), C.byref(n)),
               "icarat_mg_coarse_check")
        return r.value, n.value

    def time_operator(self, reps=20, op=OP_FP64):
        ms = C.c_double()
        _check(self.lib.icarat_time_operator_op(self.h, op, reps, C.byref(ms)),
               "time_operator")
        return ms.value

    def set_net(self, net):
        """attach a Net for the LEARNED_FPCG solver (None detaches)"""
        _check(self.lib.icarat_ctx_set_net(self.h, net.h if net is not None else None),
               "icarat_ctx_set_net")
        self._net = net

    def apply_K_op(self, u, op):
        """y = K u with operator `op` (OP_FP64 node stencil, OP_FP32, OP_TC_BF16X3,
        OP_TC_BF16, OP_TC_FP64)."""
        y = np.zeros(max(self.numeq, 1))
        _check(self.lib.icarat_apply_K_op(self.h, op, _f64(u), y), "apply_K_op")
        return y[:self.numeq]

    def loop_step(self):
        info = StepInfo()
        _check(self.lib.icarat_loop_step(self.h, C.byref(info)), "loop_step")
        return info

    def mises(self):
        """element von Mises stress of the last solve (nelx)"""
        out = np.zeros(max(self.nelx, 1))
        _check(self.lib.icarat_mises(self.h, out), "mises")
        return out[:self.nelx]

    def write_vtk(self, path, binary=False):
        """the sample drivers' output(): displacement, density, mises"""
        _check(self.lib.icarat_write_vtk(self.h, os.fsencode(path), 1 if binary else 0),
               "write_vtk")

    def set_load_cases(self, fext_cases):
        """the load cases of a multi-load loop: an (ncases, numeq) array of
        icarat_fext-layout vectors; None or an empty array returns to the
        context's own load"""
        if fext_cases is None or len(fext_cases) == 0:
            _check(self.lib.icarat_set_load_cases(self.h, 0, None), "set_load_cases")
            return
        F = np.ascontiguousarray(fext_cases, dtype=np.float64)
        if F.ndim != 2 or F.shape[1] != self.numeq:
            raise ValueError("load cases must be (ncases, %d)" % self.numeq)
        _check(self.lib.icarat_set_load_cases(self.h, F.shape[0], F.ctypes.data),
               "set_load_cases")

    def loop_set_domains(self, design_ids=None, nondesign_ids=()):
        """volume over design_ids (None: all elements), sensitivities zeroed on
        nondesign_ids; after loop_init"""
        nd = np.ascontiguousarray(nondesign_ids, dtype=np.int32)
        if design_ids is None:
            dp, dn = None, 0
        else:
            d = np.ascontiguousarray(design_ids, dtype=np.int32)
            dp, dn = d.ctypes.data, d.size
        _check(self.lib.icarat_loop_set_domains(self.h, dp, dn, nd.ctypes.data if nd.size
                                                else None, nd.size), "loop_set_domains")

    def loop_is_convergence(self, epsilon=1.0e-5, minstep=50):
        """Optimize::isConvergence on the device loop's objective
        (opt_base.hpp:28-43): 0 when the last step's compliance changed by less
        than epsilon relative to the one kept at the previous call and the step
        count exceeds minstep, else 1 (and the compliance is kept)."""
        conv = C.c_int()
        _check(self.lib.icarat_loop_is_convergence(self.h, epsilon, minstep, C.byref(conv)),
               "loop_is_convergence")
        return conv.value

    def loop_save(self, path):
        """checkpoint of the device loop (icarat_loop_save)"""
        _check(self.lib.icarat_loop_save(self.h, os.fsencode(path)), "loop_save")

    def loop_load(self, path):
        """resume a device loop from a checkpoint (icarat_loop_load)"""
        _check(self.lib.icarat_loop_load(self.h, os.fsencode(path)), "loop_load")

    def loop_get(self, which):
        idx = {"x": 0, "xfil": 1, "xthr": 2, "dfds": 3, "dgds": 4}[which]
        out = np.zeros(self.nelx)
        _check(self.lib.icarat_loop_get(self.h, idx, out), "loop_get")
        return out


# ---- reference-named mirrors ------------------------------------------------------
_SOLVER_NAMES = {"Eigen_CG": JACOBI_PCG, "Scaling_CG": JACOBI_PCG, "MG_CG": MG_PCG,
                 "Mixed_MG_CG": MIXED_IR,
                 # the reference's other names (Solvers::solve, solvers.cpp:27-61):
                 # plain CG as Jacobi-PCG, the other preconditioned Krylov
                 # solvers as MG-PCG (same solution to the tolerance, other
                 # iteration counts), the direct solvers as MG-PCG to 1e-12
                 "CG": JACOBI_PCG, "ICCG": MG_PCG, "Eigen_ICCG": MG_PCG,
                 "Eigen_BiCGSTAB": MG_PCG, "Eigen_SparseLU": MG_PCG, "Eigen_LDLT": MG_PCG,
                 "Pardiso_LDLT": MG_PCG, "Pardiso_LLT": MG_PCG, "Pardiso_LU": MG_PCG}
_DIRECT_NAMES = ("Eigen_SparseLU", "Eigen_LDLT", "Pardiso_LDLT", "Pardiso_LLT", "Pardiso_LU")


class LinearAnalysis:
    """LinearAnalysis<LinearElastic, Node> (src/analysis/linear.hpp:15-41)."""

    def __init__(self, ctx, rtol=1e-10, maxit=10000, mg_levels=4, mg_smooth=2):
        self.ctx = ctx
        self.rtol, self.maxit = rtol, maxit
        self.mg_levels, self.mg_smooth = mg_levels, mg_smooth
        self.info = None
        self.val = None

    def solve(self, solvName="Eigen_CG", log=False):
        if solvName not in _SOLVER_NAMES:
            # Solvers::solve exits on an unknown name (solvers.cpp:56-60)
            raise IcaratError(ERR_UNSUPPORTED, "Solver type name is wrong: %s" % solvName)
        rtol = min(self.rtol, 1e-12) if solvName in _DIRECT_NAMES else self.rtol
        o = solve_opts(_SOLVER_NAMES[solvName], rtol, self.maxit, self.mg_levels,
                       self.mg_smooth)
        self.val, self.info = self.ctx.solve(o)
        if log:
            print("iteration: %d\nresidual: %g" % (self.info.iterations,
                                                    self.info.rel_residual))
        return self.val


class Filter:
    """Filter<E,N> (src/optimization/filter.hpp:17-61) on the voxel grid."""

    def __init__(self, ctx, radius):
        self.ctx = ctx
        ctx.filter_setup(radius)

    def densityFilter(self, design_s, isSens):
        return self.ctx.density_filter(design_s, isSens)

    def sensitivityFilter(self, design_s, dfds):
        return self.ctx.sensitivity_filter(design_s, dfds)

    def threshold(self, d, beta, T):
        return self.ctx.threshold(d, beta, T)

    def thresholdDerivative(self, d, beta, T):
        return self.ctx.threshold_derivative(d, beta, T)


class FilterHelmholtz:
    """FilterHelmholtz<E,N> (src/optimization/filter_helm.hpp:16-65) on the
    voxel grid: densityFilter (:75-138) solves the nodal Helmholtz system on
    the GPU; "Eigen_CG" is the solver the samples name."""

    def __init__(self, ctx, radious):
        self.ctx = ctx
        ctx.helmholtz_setup(radious)
        self.info = None

    def densityFilter(self, design_s, solvName="Eigen_CG", log=0, sensFlag=False):
        if solvName not in _SOLVER_NAMES:
            # Solvers::solve exits on an unknown name (solvers.cpp:56-60)
            raise IcaratError(ERR_UNSUPPORTED, "Solver type name is wrong: %s" % solvName)
        out, self.info = self.ctx.helmholtz_filter(design_s, is_sens=sensFlag)
        if log == 1:
            print("Helmholtz filtering...")
            print("#iterations:     %d" % self.info.iterations)
            print("estimated error: %g" % self.info.rel_residual)
        return out

    def threshold(self, design_filtered, beta, T):
        return self.ctx.threshold(design_filtered, beta, T)

    def thresholdDerivative(self, design_filtered, beta, T):
        return self.ctx.threshold_derivative(design_filtered, beta, T)


class Optimize:
    """Optimize (src/optimization/opt_base.hpp:14-76): the design state of a
    host-composed loop and its convergence test."""

    def __init__(self, design, constraint, xmin, xmax):
        self.design_s = np.zeros(design)
        self.const_h = np.zeros(constraint)
        self.dfds = np.zeros(design)
        self.dgds = np.zeros(constraint * design)
        self.xmin = np.full(design, float(xmin))
        self.xmax = np.full(design, float(xmax))
        self.optstep = 0
        self.object_f = 0.0
        # uninitialised in the reference; 0 here (the first test then sees a
        # relative change of 1)
        self._object_old = 0.0

    def isConvergence(self, epsilon, minstep):
        """0 when |object_old - object_f| / object_f < epsilon and optstep >
        minstep, else 1 with object_old = object_f (opt_base.hpp:28-43)."""
        with np.errstate(divide="ignore", invalid="ignore"):
            change = np.float64(abs(self._object_old - self.object_f)) / np.float64(self.object_f)
        if change < epsilon and self.optstep > minstep:
            return 0
        self._object_old = self.object_f
        return 1


class OC:
    """OC (OCSolver.hpp:13-80); the volume functor is the drivers' filtered
    volume, evaluated on the GPU with the context's radius filter or, with
    filter="helmholtz", its Helmholtz filter (opt_macro_oc.cpp:153-164)."""

    def __init__(self, ctx, use_threshold=False, beta=1.0, T=0.5, filter="radius"):
        self.ctx = ctx
        self.movelimit = 0.15
        self.use_threshold, self.beta, self.T = use_threshold, beta, T
        self.filter = filter
        self.steps = 0

    def setMoveLimit(self, m):
        self.movelimit = m

    def UpdateVariables(self, xk, dfdx, g, dgdx, xmin, xmax):
        x, self.steps = self.ctx.oc_update(xk, dfdx, g, dgdx, xmin, xmax,
                                           move=self.movelimit,
                                           use_threshold=self.use_threshold,
                                           beta=self.beta, T=self.T, filter=self.filter)
        xk[:] = x
        return xk


class MMASolver:
    """MMASolver(n, m, a, c, d) (MMASolver.hpp:62-116) on the GPU."""

    def __init__(self, n, m, a=0.0, c=100000.0, d=0.0, device=0):
        L = load_library()
        h = C.c_void_p()
        _check(L.icarat_mma_create(device, n, m, a, c, d, C.byref(h)), "mma_create")
        self.h, self.lib, self.n, self.m = h, L, n, m

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.icarat_mma_destroy(self.h)
            self.h = None

    def SetMoveLimit(self, m):
        _check(self.lib.icarat_mma_set_move_limit(self.h, m), "SetMoveLimit")

    def SetAsymptotes(self, init, decrease, increase):
        _check(self.lib.icarat_mma_set_asymptotes(self.h, init, decrease, increase),
               "SetAsymptotes")

    def SetOscillation(self, a):
        _check(self.lib.icarat_mma_set_oscillation(self.h, a), "SetOscillation")

    def Update(self, xval, dfdx, gx, dgdx, xmin, xmax):
        """In place on xval (a float64 numpy array), like the reference."""
        assert xval.dtype == np.float64 and xval.flags.c_contiguous
        _check(self.lib.icarat_mma_update(self.h, xval, _f64(dfdx),
                                          _f64(np.atleast_1d(gx)), _f64(dgdx).ravel(),
                                          _f64(xmin), _f64(xmax)), "Update")
        return xval

    def last_loops(self):
        a, b = C.c_int(), C.c_int()
        _check(self.lib.icarat_mma_last_loops(self.h, C.byref(a), C.byref(b)), "loops")
        return a.value, b.value


def kernel_launches():
    """Kernels launched so far by libicarat_gpu.so in this process."""
    L = load_library()
    n = C.c_ulonglong()
    _check(L.icarat_kernel_launches(C.byref(n)), "kernel_launches")
    return n.value


class Batch:
    """Many independent designs solved together (icarat_batch_*).

    problems: list of (nx, ny, nz) or (nx, ny, nz, dirichlet, loads); unit
    cubes (length = division) unless lengths are given as (nx, ny, nz, lx, ly,
    lz, dirichlet, loads).  Every member is a Context (``batch[i]``) for the
    per-design calls."""

    def __init__(self, problems, young=(1e-9, 1.0), poisson=0.3, penalty=3.0, device=0):
        L = load_library()
        n = len(problems)
        grids = (Grid * n)()
        bcs = (BC * n)()
        self._keep = []
        dims = []
        for i, pr in enumerate(problems):
            pr = tuple(pr)
            nx, ny, nz = pr[:3]
            if len(pr) >= 8:
                lx, ly, lz, dirichlet, loads = pr[3:8]
            else:
                lx, ly, lz = float(nx), float(ny), float(nz)
                dirichlet, loads = pr[3:5] if len(pr) >= 5 else cantilever_bc(nx, ny, nz)
            grids[i] = Grid(nx, ny, nz, lx, ly, lz)
            bc, d, lo = _bc_struct(dirichlet, loads)
            bcs[i] = bc
            self._keep += [d, lo]
            dims.append((nx, ny, nz))
        mat = Material(young[0], young[1], poisson, penalty)
        h = C.c_void_p()
        _check(L.icarat_batch_create(C.cast(grids, C.c_void_p), C.cast(bcs, C.c_void_p), n,
                                     C.byref(mat), device, C.byref(h)), "icarat_batch_create")
        self.h, self.lib = h, L
        self.ctx = []
        for i in range(n):
            c = C.c_void_p()
            _check(L.icarat_batch_ctx(h, i, C.byref(c)), "icarat_batch_ctx")
            self.ctx.append(Context._member(c, L, dims[i], young, poisson, penalty))

    def __len__(self):
        return len(self.ctx)

    def __getitem__(self, i):
        return self.ctx[i]

    def close(self):
        if getattr(self, "h", None):
            for c in self.ctx:
                c.h = None
            self.lib.icarat_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @staticmethod
    def opts(rtol=1e-8, maxit=10000, refresh=0.0, tile=0, blocks_per_sm=0, method=0,
             mg_levels=0, chunk=0, warm_start=False):
        """method 0: one persistent Jacobi launch for all designs;
        MG_PCG: one persistent multigrid-PCG launch for all designs (every
        design's own hierarchy, the V-cycles of all designs phase by phase);
        MIXED_IR: each design's own mixed-precision multigrid solve,
        interleaved on the designs' streams."""
        return BatchOpts(rtol, maxit, refresh, tile, blocks_per_sm, method, mg_levels, chunk,
                         int(bool(warm_start)))

    def autotune(self):
        t, b, ms = C.c_int(), C.c_int(), C.c_double()
        _check(self.lib.icarat_batch_autotune(self.h, C.byref(t), C.byref(b), C.byref(ms)),
               "icarat_batch_autotune")
        return t.value, b.value, ms.value

    def autotune_mg(self, mg_levels=0):
        """(tile, CTAs per SM, ms per iteration) of the persistent multigrid
        launch (method MG_PCG), kept for later MG_PCG solves"""
        t, b, ms = C.c_int(), C.c_int(), C.c_double()
        _check(self.lib.icarat_batch_autotune_mg(self.h, mg_levels, C.byref(t), C.byref(b),
                                                 C.byref(ms)), "icarat_batch_autotune_mg")
        return t.value, b.value, ms.value

    def solve(self, opts=None):
        infos = (SolveInfo * len(self.ctx))()
        st = self.lib.icarat_batch_solve(self.h, C.byref(opts) if opts is not None else None,
                                         C.cast(infos, C.c_void_p))
        _check(st, "icarat_batch_solve")
        return list(infos)

    def solution(self, i):
        u = np.zeros(max(self.ctx[i].numeq, 1))
        _check(self.lib.icarat_batch_solution(self.h, i, u), "icarat_batch_solution")
        return u[:self.ctx[i].numeq]

    def loop_step(self, opts=None):
        infos = (StepInfo * len(self.ctx))()
        st = self.lib.icarat_batch_loop_step(self.h, C.byref(opts) if opts is not None
                                             else None, C.cast(infos, C.c_void_p))
        _check(st, "icarat_batch_loop_step")
        return list(infos)


class Net:
    """The learned preconditioner (icarat_net_*): a 4-level, 16-channel 3-D
    U-net with BF16 weights and activations, trained by the library's own
    kernels."""

    def __init__(self, seed=0, device=0):
        L = load_library()
        h = C.c_void_p()
        _check(L.icarat_net_create(device, seed, C.byref(h)), "icarat_net_create")
        self.h, self.lib = h, L
        n = C.c_longlong()
        _check(L.icarat_net_num_params(h, C.byref(n)), "icarat_net_num_params")
        self.n = n.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.icarat_net_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def params(self):
        w = np.zeros(self.n, dtype=np.float32)
        _check(self.lib.icarat_net_get_params(self.h, w.ctypes.data), "get_params")
        return w

    def set_params(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == self.n
        _check(self.lib.icarat_net_set_params(self.h, w.ctypes.data), "set_params")

    def grads(self):
        g = np.zeros(self.n, dtype=np.float32)
        _check(self.lib.icarat_net_get_grads(self.h, g.ctypes.data), "get_grads")
        return g

    def train_step(self, ctx, rho, f, u, lr):
        loss = C.c_double()
        _check(self.lib.icarat_net_train_step(self.h, ctx.h, _f64(rho), _f64(f), _f64(u), lr,
                                              C.byref(loss)), "train_step")
        return loss.value

    def infer(self, ctx, f):
        u = np.zeros(max(ctx.numeq, 1))
        _check(self.lib.icarat_net_infer(self.h, ctx.h, _f64(f), u), "infer")
        return u[:ctx.numeq]

    def infer_dev(self, ctx, f_ptr, u_ptr):
        """infer() on device pointers (numeq doubles each, e.g. torch
        tensors' data_ptr()), enqueued on the context's stream."""
        _check(self.lib.icarat_net_infer_dev(self.h, ctx.h, C.c_void_p(f_ptr), C.c_void_p(u_ptr)),
               "infer_dev")
