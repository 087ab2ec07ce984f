"""B200 (sm_100a) implementation of the per-design-iteration hot path of
natashahirt/AlgorithmEngineering_AltProject (`top3d_xl_cli GLOBAL`).

The compute lives in the in-tree CUDA library ``libt3d_b200.so`` (C-ABI: include/t3d_b200.h).
This module is a thin ctypes binding that mirrors the reference's operator API
(cpp/include/fea.hpp, solver.hpp, multigrid/multigrid.hpp, filter.hpp, driver.hpp) with the
reference's array layouts.  There is no Python or CPU fallback: importing works without a GPU,
but every compute call needs the native library and a CUDA device and raises otherwise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = ["Problem", "Batch", "T3DError", "library", "IterRecord", "Params", "LIB_PATH", "HEADER_PATH"]

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libt3d_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(PKG_DIR), "include", "t3d_b200.h")

T3D_OK, T3D_ERR_INVALID, T3D_ERR_CUDA, T3D_ERR_OOM, T3D_ERR_NO_DEVICE, T3D_ERR_UNSUPPORTED, T3D_ERR_NUMERIC = range(7)
T3D_SUM_REFERENCE, T3D_SUM_FP64 = 0, 1
T3D_FP64, T3D_MIXED = 0, 1
T3D_MATVEC32_AUTO, T3D_MATVEC32_DENSE = 0, 1
T3D_COARSE_REFERENCE, T3D_COARSE_FULL = 0, 1
T3D_MATVEC64_AUTO, T3D_MATVEC64_NODES = 0, 1
T3D_VCYCLE_ADAPTED, T3D_VCYCLE_STANDARD = 0, 1

_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class T3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("t3d error %d: %s" % (code, msg))
        self.code = code


class Params(C.Structure):
    _fields_ = [("E0", C.c_float), ("Emin", C.c_float), ("nu", C.c_float), ("penal", C.c_float),
                ("cg_tol", C.c_float), ("cg_max_it", C.c_int), ("mg_nondyadic", C.c_int),
                ("mg_max_levels", C.c_int), ("mg_weight", C.c_float), ("filter_rmin", C.c_float),
                ("oc_sum_order", C.c_int), ("precision", C.c_int), ("device", C.c_int),
                ("matvec32_form", C.c_int), ("mg_coarse_assembly", C.c_int), ("matvec64_form", C.c_int),
                ("mg_vcycle", C.c_int), ("mg_standard_weight", C.c_float),
                ("mg_rebuild_period", C.c_int), ("matvec32_tile", C.c_int)]


T3D_LOAD_TIP_LINE, T3D_LOAD_TOP_TRACTION, T3D_LOAD_TORSION = 0, 1, 2
T3D_MAX_VOIDS = 4


class ProblemSpec(C.Structure):
    """t3d_problem: load case and passive-void ellipsoids (centre ex,ey,ez and radii rx,ry,rz in element
    units of the reference's element coordinates)."""
    _fields_ = [("load_case", C.c_int), ("num_voids", C.c_int), ("voids", (C.c_double * 6) * T3D_MAX_VOIDS)]

    @classmethod
    def make(cls, load_case=T3D_LOAD_TIP_LINE, voids=()):
        p = cls()
        p.load_case = load_case
        p.num_voids = len(voids)
        for k, v in enumerate(voids):
            for d in range(6):
                p.voids[k][d] = float(v[d])
        return p


class Info(C.Structure):
    _fields_ = [("res", C.c_int64 * 3), ("orig", C.c_int64 * 3), ("num_elements", C.c_int64),
                ("num_nodes", C.c_int64), ("num_free", C.c_int64), ("num_levels", C.c_int64),
                ("levels", (C.c_int64 * 4) * 8), ("coarse_n", C.c_int64), ("coarse_cholesky_ok", C.c_int64),
                ("device_bytes", C.c_int64), ("kernel_launches", C.c_int64), ("matvec32_modal", C.c_int64),
                ("matvec32_tile", C.c_int64 * 4), ("matvec64_kernel", C.c_int64),
                ("matvec32_variant", C.c_int64), ("last_outer_passes", C.c_int64)]


class IterRecord(C.Structure):
    _fields_ = [("loop", C.c_int), ("pcg_iters", C.c_int), ("obj", C.c_double), ("vol", C.c_float),
                ("sharp", C.c_float), ("cons", C.c_float), ("change", C.c_float), ("lmid", C.c_float),
                ("bisections", C.c_int), ("t_total", C.c_double), ("t_cg", C.c_double), ("t_opt", C.c_double),
                ("t_filter", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_CTX = C.c_void_p
_BATCH = C.c_void_p
# name -> (restype, argtypes); every function declared in include/t3d_b200.h
_SIGS = {
    "t3d_params_default": (C.c_int, [C.POINTER(Params)]),
    "t3d_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(Params), C.POINTER(_CTX)]),
    "t3d_create_problem": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(Params), C.POINTER(ProblemSpec),
                                     C.POINTER(_CTX)]),
    "t3d_topvoxel_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64)]),
    "t3d_create_from_topvoxel": (C.c_int, [C.c_char_p, C.POINTER(Params), C.POINTER(_CTX)]),
    "t3d_destroy": (C.c_int, [_CTX]),
    "t3d_get_info": (C.c_int, [_CTX, C.POINTER(Info)]),
    "t3d_last_error": (C.c_char_p, []),
    "t3d_voxel_ke": (C.c_int, [C.c_double, C.c_double, _f64p]),
    "t3d_get_ke": (C.c_int, [_CTX, _f64p]),
    "t3d_set_ke": (C.c_int, [_CTX, _f64p]),
    "t3d_get_element_map": (C.c_int, [_CTX, _i32p]),
    "t3d_get_free_dofs": (C.c_int, [_CTX, _i32p]),
    "t3d_get_load": (C.c_int, [_CTX, _f64p]),
    "t3d_matvec": (C.c_int, [_CTX, _f64p, _f64p, _f64p]),
    "t3d_matvec32": (C.c_int, [_CTX, _f64p, _f64p, _f64p]),
    "t3d_mg_setup": (C.c_int, [_CTX, _f64p]),
    "t3d_vcycle": (C.c_int, [_CTX, _f64p, _f64p]),
    "t3d_vcycle32": (C.c_int, [_CTX, _f64p, _f64p]),
    "t3d_pcg": (C.c_int, [_CTX, _f64p, _f64p, _f64p, C.c_double, C.c_int, C.POINTER(C.c_int)]),
    "t3d_compliance": (C.c_int, [_CTX, _f64p, _f64p, _f64p, C.POINTER(C.c_double)]),
    "t3d_mg_get_diag": (C.c_int, [_CTX, C.c_int, _f64p]),
    "t3d_mg_get_mask": (C.c_int, [_CTX, C.c_int, _u8p]),
    "t3d_mg_coarse_matrix": (C.c_int, [_CTX, _f64p, _f64p]),
    "t3d_filter_apply": (C.c_int, [_CTX, _f32p, _f32p]),
    "t3d_filter_setup": (C.c_int, [_CTX, C.c_float]),
    "t3d_filter_get_state": (C.c_int, [_CTX, _f64p, _f64p, _f64p]),
    "t3d_filter_set_state": (C.c_int, [_CTX, _f64p, _f64p]),
    "t3d_simp": (C.c_int, [_CTX, _f32p, _f64p]),
    "t3d_sensitivity": (C.c_int, [_CTX, _f32p, _f64p, C.c_double, _f32p]),
    "t3d_dc_scale": (C.c_int, [_CTX, _f32p, _f32p, _f32p]),
    "t3d_oc_update": (C.c_int, [_CTX, _f32p, _f32p, C.c_float, _f32p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                C.POINTER(C.c_int)]),
    "t3d_design_init": (C.c_int, [_CTX, C.c_float, C.POINTER(C.c_double)]),
    "t3d_design_step": (C.c_int, [_CTX, C.POINTER(IterRecord)]),
    "t3d_design_step_host": (C.c_int, [_CTX, _f32p, _f32p, C.POINTER(IterRecord)]),
    "t3d_get_density": (C.c_int, [_CTX, _f32p]),
    "t3d_set_density": (C.c_int, [_CTX, _f32p]),
    "t3d_get_displacement": (C.c_int, [_CTX, _f64p]),
    "t3d_run_global": (C.c_int, [_CTX, C.c_float, C.c_int, C.POINTER(C.c_double), C.POINTER(IterRecord),
                                 C.POINTER(C.c_int), _f32p]),
    "t3d_synchronize": (C.c_int, [_CTX]),
    "t3d_export_stl": (C.c_int, [_CTX, C.c_void_p, C.c_float, C.c_char_p, C.POINTER(C.c_int64)]),
    "t3d_profile": (C.c_int, [_CTX, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "t3d_compliance_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, _f64p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]),
    "t3d_batch_create": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(Params), C.POINTER(ProblemSpec),
                                   C.POINTER(_BATCH)]),
    "t3d_batch_member": (C.c_int, [_BATCH, C.c_int, C.POINTER(_CTX)]),
    "t3d_batch_open": (C.c_int, [C.c_int, C.POINTER(_BATCH)]),
    "t3d_batch_adopt": (C.c_int, [_BATCH, _CTX]),
    "t3d_batch_release": (C.c_int, [_BATCH, C.c_int, C.POINTER(_CTX)]),
    "t3d_batch_design_init": (C.c_int, [_BATCH, _f32p, _f64p]),
    "t3d_batch_design_step": (C.c_int, [_BATCH, C.POINTER(IterRecord)]),
    "t3d_batch_run": (C.c_int, [_BATCH, C.POINTER(C.c_int), C.POINTER(IterRecord)]),
    "t3d_batch_submit": (C.c_int, [_BATCH, _CTX, C.c_int]),
    "t3d_batch_collect": (C.c_int, [_BATCH, C.c_int, C.POINTER(_CTX), C.POINTER(IterRecord), C.c_int,
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "t3d_batch_info": (C.c_int, [_BATCH, C.POINTER(C.c_int64)]),
    "t3d_batch_destroy": (C.c_int, [_BATCH]),
}
T3D_BATCH_TILE = 7
T3D_PROFILE_MATVEC, T3D_PROFILE_VCYCLE, T3D_PROFILE_MATVEC32, T3D_PROFILE_VCYCLE32 = 0, 1, 2, 3

_lib = None


def library():
    """Load libt3d_b200.so (raises if it has not been built; there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise T3DError(T3D_ERR_UNSUPPORTED, "native library %s not built; run "
                           "`python -m algorithmengineering_altproject_b200._build`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != T3D_OK:
        raise T3DError(rc, library().t3d_last_error().decode())


def topvoxel_info(path):
    """Parses a TopVoxel file (no GPU needed) and returns its sizes."""
    v = (C.c_int64 * 8)()
    _check(library().t3d_topvoxel_info(os.fsencode(path), v))
    keys = ("nelx", "nely", "nelz", "solid", "passive", "fixed_nodes", "loaded_nodes", "additional_load_cases")
    return dict(zip(keys, (int(x) for x in v)))


def ComputeVoxelKe(nu=0.3, cellSize=1.0):
    """The reference's ComputeVoxelKe (fea.hpp:37): unit-modulus hex8 stiffness, 24x24 (host only)."""
    Ke = np.zeros(576)
    _check(library().t3d_voxel_ke(float(nu), float(cellSize), Ke))
    return Ke.reshape(24, 24)


def default_params(**kw):
    p = Params()
    _check(library().t3d_params_default(C.byref(p)))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Problem:
    """One cantilever design on one GPU: the reference's `Problem` + MG hierarchy + PDE filter.

    Constructed like ``CreateVoxelFEAmodel_Cuboid(pb, nely, nelx, nelz); ApplyBoundaryConditions(pb);
    mg::build_static_once(...); SetupPDEFilter(pb, rMin)`` (fea.cpp:181-447, preconditioner.cpp:19,
    filter.cpp:9).  Methods keep the reference's names and array layouts.
    """

    def __init__(self, nely, nelx, nelz, problem=None, **params):
        """`problem`: optional ProblemSpec (load case, passive voids); None = the reference cantilever."""
        self._lib = library()
        self.params = default_params(**params)
        h = _CTX()
        if problem is None:
            _check(self._lib.t3d_create(nely, nelx, nelz, C.byref(self.params), C.byref(h)))
        else:
            _check(self._lib.t3d_create_problem(nely, nelx, nelz, C.byref(self.params), C.byref(problem),
                                                C.byref(h)))
        self._attach(h)

    @classmethod
    def from_topvoxel(cls, path, **params):
        """An external design domain from a TopVoxel file (the MATLAB original's CreateVoxelFEAmodel,
        TOP3D_XL.m:458-586): its solid voxels, passive elements, fixations and loads replace the built-in
        cantilever.  Element arrays cover the solid voxels in Morton order."""
        self = cls.__new__(cls)
        self._lib = library()
        self.params = default_params(**params)
        h = _CTX()
        _check(self._lib.t3d_create_from_topvoxel(os.fsencode(path), C.byref(self.params), C.byref(h)))
        self._attach(h)
        return self

    def _attach(self, h):
        self._h = h
        info = Info()
        _check(self._lib.t3d_get_info(self._h, C.byref(info)))
        self.res = tuple(int(v) for v in info.res)
        self.ne = int(info.num_elements)
        self.nn = int(info.num_nodes)
        self.nf = int(info.num_free)
        self.nlev = int(info.num_levels)
        self.levels = [tuple(int(v) for v in info.levels[l]) for l in range(self.nlev)]
        self.coarse_n = int(info.coarse_n)
        self.device_bytes = int(info.device_bytes)

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                self._lib.t3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        info = Info()
        _check(self._lib.t3d_get_info(self._h, C.byref(info)))
        return info

    def level_nodes(self, l):
        nx, ny, nz, _ = self.levels[l]
        return (nx + 1) * (ny + 1) * (nz + 1)

    # ---- model data
    def ke(self):
        out = np.zeros(576)
        _check(self._lib.t3d_get_ke(self._h, out))
        return out.reshape(24, 24)

    def set_ke(self, Ke):
        _check(self._lib.t3d_set_ke(self._h, _f64(Ke).ravel()))

    def ele_map_back(self):
        out = np.zeros(self.ne, dtype=np.int32)
        _check(self._lib.t3d_get_element_map(self._h, out))
        return out

    def free_dofs(self):
        out = np.zeros(self.nf, dtype=np.int32)
        _check(self._lib.t3d_get_free_dofs(self._h, out))
        return out

    def bfree(self):
        out = np.zeros(self.nf)
        _check(self._lib.t3d_get_load(self._h, out))
        return out

    # ---- operators (reference names)
    def K_times_u_finest(self, eleE, uFree):
        y = np.zeros(self.nf)
        _check(self._lib.t3d_matvec(self._h, _f64(eleE), _f64(uFree), y))
        return y

    def K_times_u_finest32(self, eleE, uFree):
        """the FP32 K(E)u of the mixed-precision inner solve (mixed contexts only), widened to FP64"""
        y = np.zeros(self.nf)
        _check(self._lib.t3d_matvec32(self._h, _f64(eleE), _f64(uFree), y))
        return y

    def make_diagonal_preconditioner_from_static(self, eleE):
        _check(self._lib.t3d_mg_setup(self._h, _f64(eleE)))

    def vcycle(self, rFree):
        z = np.zeros(self.nf)
        _check(self._lib.t3d_vcycle(self._h, _f64(rFree), z))
        return z

    def export_stl(self, path, iso=0.3, xPhys=None):
        """export_surface_stl (io.cpp:80-87): binary STL of the current design (or of xPhys, reference element
        order) at threshold iso; returns the triangle count"""
        n = C.c_int64(0)
        xp = None if xPhys is None else _f32(xPhys)
        _check(self._lib.t3d_export_stl(self._h, None if xp is None else xp.ctypes.data_as(C.c_void_p),
                                        C.c_float(iso), str(path).encode(), C.byref(n)))
        return int(n.value)

    def vcycle32(self, rFree):
        """the FP32 V-cycle of the mixed-precision inner solve (mixed contexts only), widened to FP64"""
        z = np.zeros(self.nf)
        _check(self._lib.t3d_vcycle32(self._h, _f64(rFree), z))
        return z

    def PCG_free(self, eleE, bFree, xFree, tol=None, maxIt=800):
        tol = float(np.float32(1e-3)) if tol is None else float(tol)
        x = np.array(xFree, dtype=np.float64, copy=True)
        its = C.c_int()
        _check(self._lib.t3d_pcg(self._h, _f64(eleE), _f64(bFree), x, C.c_double(tol), int(maxIt), C.byref(its)))
        return x, int(its.value)

    def ComputeCompliance(self, eleE, uFree):
        ce = np.zeros(self.ne)
        Cv = C.c_double()
        _check(self._lib.t3d_compliance(self._h, _f64(eleE), _f64(uFree), ce, C.byref(Cv)))
        return float(Cv.value), ce

    def mg_diag(self, level):
        out = np.zeros(3 * self.level_nodes(level))
        _check(self._lib.t3d_mg_get_diag(self._h, level, out))
        return out

    def mg_mask(self, level):
        out = np.zeros(3 * self.level_nodes(level), dtype=np.uint8)
        _check(self._lib.t3d_mg_get_mask(self._h, level, out))
        return out

    def coarse_matrix(self, eleE):
        n = self.coarse_n
        out = np.zeros(n * n)
        _check(self._lib.t3d_mg_coarse_matrix(self._h, _f64(eleE), out))
        return out.reshape(n, n)

    def ApplyPDEFilter(self, src):
        dst = np.zeros(self.ne, dtype=np.float32)
        _check(self._lib.t3d_filter_apply(self._h, _f32(src), dst))
        return dst

    def SetupPDEFilter(self, filterRadius):
        """SetupPDEFilter (filter.hpp:17) for another radius; resets the filter's warm start."""
        _check(self._lib.t3d_filter_setup(self._h, float(filterRadius)))

    def filter_state(self):
        lx, lr, dg = np.zeros(self.nn), np.zeros(self.nn), np.zeros(self.nn)
        _check(self._lib.t3d_filter_get_state(self._h, lx, lr, dg))
        return lx, lr, dg

    def filter_set_state(self, lastx, lastrhs):
        _check(self._lib.t3d_filter_set_state(self._h, _f64(lastx), _f64(lastrhs)))

    def simp(self, xPhys):
        E = np.zeros(self.ne)
        _check(self._lib.t3d_simp(self._h, _f32(xPhys), E))
        return E

    def sensitivity(self, xPhys, ce, csolid):
        dc = np.zeros(self.ne, dtype=np.float32)
        _check(self._lib.t3d_sensitivity(self._h, _f32(xPhys), _f64(ce), C.c_double(csolid), dc))
        return dc

    def dc_scale(self, dcf, x):
        dc = np.zeros(self.ne, dtype=np.float32)
        _check(self._lib.t3d_dc_scale(self._h, _f32(dcf), _f32(x), dc))
        return dc

    def oc_update(self, x, dc, V0):
        xn = np.zeros(self.ne, dtype=np.float32)
        ch, lm, nb = C.c_float(), C.c_float(), C.c_int()
        _check(self._lib.t3d_oc_update(self._h, _f32(x), _f32(dc), C.c_float(V0), xn, C.byref(ch), C.byref(lm),
                                       C.byref(nb)))
        return xn, float(ch.value), float(lm.value), int(nb.value)

    # ---- design loop
    def design_init(self, V0):
        cs = C.c_double()
        _check(self._lib.t3d_design_init(self._h, C.c_float(V0), C.byref(cs)))
        return float(cs.value)

    def design_step(self):
        rec = IterRecord()
        _check(self._lib.t3d_design_step(self._h, C.byref(rec)))
        return rec.as_dict()

    def design_step_host(self, x_in, out=None):
        """One design iteration with the design field passed through host memory: x_in (reference element
        order) in, the updated field out.  `out`, when given, is a caller-owned float32 array of ne values
        (e.g. pinned memory reused across iterations) that receives the result; else a new array does."""
        rec = IterRecord()
        if out is None:
            out = np.zeros(self.ne, dtype=np.float32)
        elif out.dtype != np.float32 or out.shape != (self.ne,) or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 array of %d values" % self.ne)
        _check(self._lib.t3d_design_step_host(self._h, _f32(x_in), out, C.byref(rec)))
        return out, rec.as_dict()

    def density(self):
        x = np.zeros(self.ne, dtype=np.float32)
        _check(self._lib.t3d_get_density(self._h, x))
        return x

    def set_density(self, x):
        _check(self._lib.t3d_set_density(self._h, _f32(x)))

    def displacement(self):
        """the design loop's displacement on the free DOFs (reference order)"""
        u = np.zeros(self.nf)
        _check(self._lib.t3d_get_displacement(self._h, u))
        return u

    def run_global(self, V0, nLoop):
        """TOP3D_XL_GLOBAL for one simulation (driver.cpp:23-218): (Csolid, records, final x)."""
        recs = (IterRecord * max(1, nLoop))()
        n = C.c_int()
        cs = C.c_double()
        x = np.zeros(self.ne, dtype=np.float32)
        _check(self._lib.t3d_run_global(self._h, C.c_float(V0), int(nLoop), C.byref(cs), recs, C.byref(n), x))
        return float(cs.value), [recs[i].as_dict() for i in range(n.value)], x

    def synchronize(self):
        _check(self._lib.t3d_synchronize(self._h))

    def profile(self, what, reps):
        """mean ms per launch of the FP64 matvec (what=0) or V-cycle (what=1), or of their FP32 forms
        (2, 3; precision T3D_MIXED only), CUDA events on the library stream"""
        ms = C.c_double()
        _check(self._lib.t3d_profile(self._h, int(what), int(reps), C.byref(ms)))
        return float(ms.value)

    def kernel_launches(self):
        return int(self.info().kernel_launches)


class Batch:
    """Many designs of uneven grid size stepping together (t3d_batch_*; no reference counterpart -- the
    reference runs one design per process, driver.cpp:23).  Members share one device arena; every kernel of
    their inner FP32 MG-PCG iteration is one persistent launch over an (instance, block) work list with
    per-instance convergence masks, and each member's results equal those of a Problem created alone with
    the same parameters and ``matvec32_tile=T3D_BATCH_TILE``.

    dims: [(nely, nelx, nelz), ...]; problems: ProblemSpec per member or None (the reference cantilever);
    params: common keyword parameters (precision is T3D_MIXED), or ``member_params``: one dict per member.
    ``members[i]`` is a Problem view of member i (queries only; the batch owns it).
    """

    def __init__(self, dims, problems=None, member_params=None, **params):
        self._lib = library()
        n = len(dims)
        P = (Params * n)()
        for i in range(n):
            kw = dict(params, precision=T3D_MIXED)
            if member_params is not None:
                kw.update(member_params[i])
            P[i] = default_params(**kw)
        D = (C.c_int * (3 * n))(*[int(v) for d in dims for v in d])
        Q = None
        if problems is not None:
            Q = (ProblemSpec * n)()
            for i, q in enumerate(problems):
                Q[i] = q if q is not None else ProblemSpec.make()
        h = _BATCH()
        _check(self._lib.t3d_batch_create(n, D, P, Q, C.byref(h)))
        self._h = h
        self.n = n
        self.members = []
        for i in range(n):
            c = _CTX()
            _check(self._lib.t3d_batch_member(self._h, i, C.byref(c)))
            m = Problem.__new__(Problem)
            m._lib = self._lib
            m.params = P[i]
            m._owned = False
            m._attach(c)
            self.members.append(m)

    @classmethod
    def open(cls, device=0):
        """An empty batch for continuous batching: members join with adopt() and leave with release()."""
        self = cls.__new__(cls)
        self._lib = library()
        h = _BATCH()
        _check(self._lib.t3d_batch_open(int(device), C.byref(h)))
        self._h = h
        self.n = 0
        self.members = []
        return self

    def adopt(self, problem):
        """Moves a Problem created alone (precision T3D_MIXED, matvec32_tile=T3D_BATCH_TILE, one load case,
        design_init done) into the batch as its last member; the batch owns it until release()."""
        _check(self._lib.t3d_batch_adopt(self._h, problem._h))
        problem._owned = False
        self.members.append(problem)
        self.n += 1

    def release(self, i):
        """Takes member i out of the batch (later members move down) and returns it; the caller closes it."""
        c = _CTX()
        _check(self._lib.t3d_batch_release(self._h, int(i), C.byref(c)))
        p = self.members.pop(i)
        p._owned = True
        self.n -= 1
        return p

    def design_init(self, V0):
        """t3d_design_init of every member; V0: one value per member; returns the solid compliances"""
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(V0, dtype=np.float32), (self.n,)))
        cs = np.zeros(self.n)
        _check(self._lib.t3d_batch_design_init(self._h, v, cs))
        return cs

    def design_step(self):
        """one design iteration of every member; returns their records"""
        recs = (IterRecord * self.n)()
        _check(self._lib.t3d_batch_design_step(self._h, recs))
        return [recs[i].as_dict() for i in range(self.n)]

    def run(self, steps):
        """steps[i] design iterations of member i, members advancing independently (only their inner solves
        share the batched launches); returns each member's list of records"""
        steps = [int(k) for k in steps]
        st = (C.c_int * self.n)(*steps)
        recs = (IterRecord * max(1, sum(steps)))()
        _check(self._lib.t3d_batch_run(self._h, st, recs))
        out, k = [], 0
        for n in steps:
            out.append([recs[k + j].as_dict() for j in range(n)])
            k += n
        return out

    def submit(self, problem, steps):
        """Submitted work (a batch from Batch.open()): `problem` (created alone with precision T3D_MIXED and
        matvec32_tile=T3D_BATCH_TILE, design_init done) runs `steps` design iterations in the batch from now
        on; collect() hands it back when done."""
        _check(self._lib.t3d_batch_submit(self._h, problem._h, int(steps)))
        problem._owned = False
        self._submitted = getattr(self, "_submitted", {})
        self._submitted[problem._h.value if hasattr(problem._h, "value") else problem._h] = (problem, int(steps))

    def collect(self, timeout_ms=100):
        """(problem, records, error or None) of a finished submission, or None when none finished within the
        timeout; the problem is the caller's again (close it)."""
        c = _CTX()
        nrec, status = C.c_int(), C.c_int()
        pending = getattr(self, "_submitted", {})
        cap = max([k for _, k in pending.values()] + [1])
        recs = (IterRecord * cap)()
        _check(self._lib.t3d_batch_collect(self._h, int(timeout_ms), C.byref(c), recs, cap, C.byref(nrec),
                                           C.byref(status)))
        if not c.value:
            return None
        problem, _ = pending.pop(c.value)
        problem._owned = True
        err = None if status.value == T3D_OK else self._lib.t3d_last_error().decode()
        return problem, [recs[i].as_dict() for i in range(nrec.value)], err

    def info(self):
        v = (C.c_int64 * 6)()
        _check(self._lib.t3d_batch_info(self._h, v))
        keys = ("arena_bytes", "members", "batched_launches", "kernels_per_iteration", "blocks_per_iteration",
                "member_launches")
        return {k: int(v[i]) for i, k in enumerate(keys)}

    def close(self):
        if getattr(self, "_h", None):
            for m in self.members:
                m._h = None
            for p, _ in getattr(self, "_submitted", {}).values():   # destroyed with the batch
                p._h = None
            self._lib.t3d_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
