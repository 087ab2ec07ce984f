"""Test infrastructure only: ctypes bindings for the CPU oracle and the reference harness.

* ``Oracle``    -> oracle/_build/libt3d_oracle.so   (C restatement, oracle/t3d_oracle.c)
* ``Reference`` -> oracle/_ref/libt3d_ref.so        (unmodified reference sources +
                                                    oracle/ref_harness.cpp, see oracle/Makefile)

Used by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg as the checker.
Both share one Python API; arrays use the reference's layouts (Morton element order, free-DOF
vectors, lexicographic nodes).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libt3d_oracle.so")
# T3D_REF_SO selects another build of the same reference sources (the fixture scripts use the build
# without -ffast-math, oracle/_ref/nofm, to measure the reference's build-to-build drift)
REF_SO = os.environ.get("T3D_REF_SO") or os.path.join(HERE, "_ref", "libt3d_ref.so")

_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class OrcParams(C.Structure):
    _fields_ = [("E0", C.c_float), ("Emin", C.c_float), ("nu", C.c_float), ("penal", C.c_float),
                ("cg_tol", C.c_float), ("cg_max_it", C.c_int), ("mg_nondyadic", C.c_int),
                ("mg_max_levels", C.c_int), ("mg_weight", C.c_float), ("pow_mode", C.c_int),
                ("vol_mode", C.c_int), ("approx_mode", C.c_int), ("red_mode", C.c_int), ("coarse_full", C.c_int)]


class OrcIterRecord(C.Structure):
    _fields_ = [("loop", C.c_int), ("pcg_iters", C.c_int), ("obj", C.c_double), ("vol", C.c_float),
                ("sharp", C.c_float), ("cons", C.c_float), ("change", C.c_float), ("lmid", C.c_float),
                ("bisections", C.c_int)]


def build_oracle() -> str:
    """Compile the oracle restatement if needed (gcc only; no reference sources involved)."""
    src = os.path.join(HERE, "t3d_oracle.c")
    if (not os.path.exists(ORACLE_SO)) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return ORACLE_SO


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class _Common:
    """Shared shape helpers; subclasses bind the C entry points."""

    def _setup_info(self):
        info = np.zeros(64, dtype=np.int64)
        self._info(self.h, info)
        self.res = tuple(int(v) for v in info[0:3])          # (resX, resY, resZ)
        self.ne = int(info[3])
        self.nn = int(info[4])
        self.nf = int(info[5])
        self.nlev = int(info[6])
        self.levels = [tuple(int(v) for v in info[7 + 4 * l:11 + 4 * l]) for l in range(self.nlev)]

    def level_nodes(self, l):
        nx, ny, nz, _ = self.levels[l]
        return (nx + 1) * (ny + 1) * (nz + 1)

    def ele_map_back(self):
        out = np.zeros(self.ne, dtype=np.int32)
        self._emb(self.h, out)
        return out

    def free_dofs(self):
        out = np.zeros(self.nf, dtype=np.int32)
        self._fd(self.h, out)
        return out

    def bfree(self):
        out = np.zeros(self.nf)
        self._bf(self.h, out)
        return out

    def ke(self):
        out = np.zeros(576)
        self._ke(self.h, out)
        return out.reshape(24, 24)

    def matvec(self, E, u):
        y = np.zeros(self.nf)
        self._mv(self.h, np.ascontiguousarray(E, np.float64), np.ascontiguousarray(u, np.float64), y)
        return y

    def mg_build(self, E):
        self._mgb(self.h, np.ascontiguousarray(E, np.float64))

    def vcycle(self, r):
        z = np.zeros(self.nf)
        self._vc(self.h, np.ascontiguousarray(r, np.float64), z)
        return z

    def pcg(self, E, b, x0, tol=None, maxit=800):
        tol = float(np.float32(1e-3)) if tol is None else tol
        x = np.array(x0, dtype=np.float64, copy=True)
        it = self._pcg(self.h, np.ascontiguousarray(E, np.float64), np.ascontiguousarray(b, np.float64), x,
                       C.c_double(tol), maxit)
        return x, int(it)

    def compliance(self, E, u):
        ce = np.zeros(self.ne)
        Cv = self._cc(self.h, np.ascontiguousarray(E, np.float64), np.ascontiguousarray(u, np.float64), ce)
        return float(Cv), ce

    def mg_diag(self, level, E=None):
        out = np.zeros(3 * self.level_nodes(level))
        if E is None:
            self._mgd(self.h, level, out)
        else:
            self._mgd(self.h, np.ascontiguousarray(E, np.float64), level, out)
        return out

    def mg_mask(self, level):
        out = np.zeros(3 * self.level_nodes(level), dtype=np.uint8)
        self._mgm(self.h, level, out)
        return out

    def coarse_matrix(self, E):
        n = 3 * self.level_nodes(self.nlev - 1)
        out = np.zeros(n * n)
        N = self._ckc(self.h, np.ascontiguousarray(E, np.float64), out)
        return out.reshape(n, n) if N else None

    def filter_setup(self, rmin=float(np.sqrt(np.float32(3.0)))):
        self._fs(self.h, C.c_float(rmin))

    def filter_apply(self, src):
        dst = np.zeros(self.ne, dtype=np.float32)
        self._fa(self.h, np.ascontiguousarray(src, np.float32), dst)
        return dst

    def filter_state(self):
        lx, lr, dg = np.zeros(self.nn), np.zeros(self.nn), np.zeros(self.nn)
        self._fst(self.h, lx, lr, dg)
        return lx, lr, dg

    def filter_set_state(self, lastx, lastrhs):
        self._fss(self.h, np.ascontiguousarray(lastx, np.float64), np.ascontiguousarray(lastrhs, np.float64))


def voxel_model_from_rows(nelx, nely, nelz, solid, passive=(), fixations=(), load_cases=((),),
                          loaded_nodes_free=True):
    """The arrays of an external model for `Oracle(..., voxel_model=...)` from 0-based rows: solid and passive
    voxels (x, y, z), fixations (x, y, z, fx, fy, fz) with 0/1 flags, load cases of (x, y, z, Fx, Fy, Fz).
    As in the MATLAB reader (TOP3D_XL.m:529-545): duplicate nodes keep their first row, nodes ascending;
    all-zero fixation rows fix nothing.  With loaded_nodes_free (a TopVoxel file, FEA_ApplyBoundaryCondition
    TOP3D_XL.m:1326-1331) a node that any load case loads loses its fixation row; without it (the restatement
    of a built-in problem spec) fixations stay and loads on fixed DOFs are dropped."""
    vox = np.zeros(nelx * nely * nelz, dtype=np.uint8)
    for x, y, z in solid:
        vox[y + nely * (x + nelx * z)] = 1
    for x, y, z in passive:
        vox[y + nely * (x + nelx * z)] = 2
    node = lambda x, y, z: y + (nely + 1) * (x + (nelx + 1) * z)
    fix = {}
    for x, y, z, fx, fy, fz in fixations:
        fix.setdefault(node(x, y, z), (1 if fx else 0) | (2 if fy else 0) | (4 if fz else 0))
    fix = {k: v for k, v in fix.items() if v}
    nodes, forces, counts = [], [], []
    for case in load_cases:
        rows = {}
        for x, y, z, fx, fy, fz in case:
            rows.setdefault(node(x, y, z), (fx, fy, fz))
        keys = sorted(rows)
        nodes += keys
        forces += [v for k in keys for v in rows[k]]
        counts.append(len(keys))
    if loaded_nodes_free:
        for k in nodes:
            fix.pop(k, None)
    keys = sorted(fix)
    return {"voxel": vox, "fix_node": np.array(keys, dtype=np.int64), "fix_bits": np.array([fix[k] for k in keys],
            dtype=np.uint8), "case_n": np.array(counts, dtype=np.int32), "load_node": np.array(nodes, dtype=np.int64),
            "load_f": np.array(forces, dtype=np.float64)}


class Oracle(_Common):
    """The C restatement (oracle/t3d_oracle.c)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = C.CDLL(build_oracle())
            L.orc_create.restype = C.c_void_p
            L.orc_create_voxel.restype = C.c_void_p
            L.orc_create_voxel.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams), C.c_void_p, C.c_int,
                                           C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
            L.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams)]
            L.orc_destroy.argtypes = [C.c_void_p]
            L.orc_params_default.argtypes = [C.POINTER(OrcParams)]
            L.orc_info.argtypes = [C.c_void_p, _i64p]
            L.orc_ele_map_back.argtypes = [C.c_void_p, _i32p]
            L.orc_free_dofs.argtypes = [C.c_void_p, _i32p]
            L.orc_bfree.argtypes = [C.c_void_p, _f64p]
            L.orc_ke.argtypes = [C.c_void_p, _f64p]
            L.orc_set_ke.argtypes = [C.c_void_p, _f64p]
            L.orc_matvec.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
            L.orc_mg_build.argtypes = [C.c_void_p, _f64p]
            L.orc_mg_coarse_n.argtypes = [C.c_void_p]
            L.orc_mg_coarse_n.restype = C.c_int
            L.orc_mg_diag.argtypes = [C.c_void_p, C.c_int, _f64p]
            L.orc_mg_mask.argtypes = [C.c_void_p, C.c_int, _u8p]
            L.orc_coarse_matrix.argtypes = [C.c_void_p, _f64p, _f64p]
            L.orc_coarse_matrix.restype = C.c_int
            L.orc_vcycle.argtypes = [C.c_void_p, _f64p, _f64p]
            L.orc_pcg.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, C.c_double, C.c_int]
            L.orc_pcg.restype = C.c_int
            L.orc_compliance.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
            L.orc_compliance.restype = C.c_double
            L.orc_objective.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double]
            L.orc_objective.restype = C.c_double
            L.orc_filter_setup.argtypes = [C.c_void_p, C.c_float]
            L.orc_filter_apply.argtypes = [C.c_void_p, _f32p, _f32p]
            L.orc_filter_state.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
            L.orc_filter_set_state.argtypes = [C.c_void_p, _f64p, _f64p]
            L.orc_simp.argtypes = [C.c_void_p, _f32p, _f64p]
            L.orc_sens.argtypes = [C.c_void_p, _f32p, _f64p, C.c_double, _f32p]
            L.orc_dc_scale.argtypes = [C.c_void_p, _f32p, _f32p, _f32p]
            L.orc_oc.argtypes = [C.c_void_p, _f32p, _f32p, C.c_float, _f32p, C.POINTER(C.c_float),
                                 C.POINTER(C.c_float)]
            L.orc_oc.restype = C.c_int
            L.orc_vol_sum.argtypes = [C.c_void_p, _f32p, C.c_int]
            L.orc_vol_sum.restype = C.c_float
            L.orc_sharpness.argtypes = [C.c_void_p, _f32p, C.c_int]
            L.orc_sharpness.restype = C.c_float
            L.orc_export_stl.argtypes = [C.c_void_p, _f32p, C.c_char_p, C.c_float]
            L.orc_export_stl.restype = C.c_int64
            L.orc_design_loop.argtypes = [C.c_void_p, C.c_float, C.c_int, C.c_float, C.POINTER(C.c_double),
                                          C.POINTER(OrcIterRecord), _f32p]
            L.orc_design_loop.restype = C.c_int
            cls._lib = L
        return cls._lib

    def __init__(self, nely, nelx, nelz, emin=None, max_levels=5, pow_mode=0, vol_mode=0, approx_mode=0, red_mode=0,
                 penal=None, coarse_full=0, voxel_model=None):
        """voxel_model: an external (TopVoxel) model from `voxel_model_from_rows`, else the cantilever."""
        L = self.lib()
        p = OrcParams()
        L.orc_params_default(C.byref(p))
        if emin is not None:
            p.Emin = emin
        if penal is not None:
            p.penal = penal
        p.mg_max_levels = max_levels
        p.pow_mode = pow_mode
        p.vol_mode = vol_mode
        p.approx_mode = approx_mode
        p.red_mode = red_mode
        p.coarse_full = coarse_full
        self.params = p
        if voxel_model is None:
            self.h = C.c_void_p(L.orc_create(nely, nelx, nelz, C.byref(p)))
        else:
            self._vm = vm = voxel_model        # the C side keeps pointers into these arrays
            ptr = lambda a: a.ctypes.data_as(C.c_void_p)
            self.h = C.c_void_p(L.orc_create_voxel(nely, nelx, nelz, C.byref(p), ptr(vm["voxel"]), len(vm["fix_node"]),
                                                   ptr(vm["fix_node"]), ptr(vm["fix_bits"]), len(vm["case_n"]),
                                                   ptr(vm["case_n"]), ptr(vm["load_node"]), ptr(vm["load_f"])))
        self._info = L.orc_info
        self._emb, self._fd, self._bf, self._ke = L.orc_ele_map_back, L.orc_free_dofs, L.orc_bfree, L.orc_ke
        self._mv, self._mgb, self._vc, self._pcg, self._cc = (L.orc_matvec, L.orc_mg_build, L.orc_vcycle,
                                                              L.orc_pcg, L.orc_compliance)
        self._mgd, self._mgm, self._ckc = L.orc_mg_diag, L.orc_mg_mask, L.orc_coarse_matrix
        self._fs, self._fa, self._fst, self._fss = (L.orc_filter_setup, L.orc_filter_apply, L.orc_filter_state,
                                                    L.orc_filter_set_state)
        self._setup_info()

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().orc_destroy(self.h)
            self.h = None

    def set_ke(self, Ke):
        self.lib().orc_set_ke(self.h, np.ascontiguousarray(Ke, np.float64).ravel())

    def mg_diag(self, level, E=None):
        out = np.zeros(3 * self.level_nodes(level))
        self.lib().orc_mg_diag(self.h, level, out)
        return out

    def coarse_n(self):
        return int(self.lib().orc_mg_coarse_n(self.h))

    def simp(self, xphys):
        E = np.zeros(self.ne)
        self.lib().orc_simp(self.h, np.ascontiguousarray(xphys, np.float32), E)
        return E

    def sens(self, xphys, ce, csolid):
        dc = np.zeros(self.ne, dtype=np.float32)
        self.lib().orc_sens(self.h, np.ascontiguousarray(xphys, np.float32), np.ascontiguousarray(ce, np.float64),
                            C.c_double(csolid), dc)
        return dc

    def oc(self, x, dc, V0):
        xnew = np.zeros(self.ne, dtype=np.float32)
        ch, lm = C.c_float(), C.c_float()
        n = self.lib().orc_oc(self.h, np.ascontiguousarray(x, np.float32), np.ascontiguousarray(dc, np.float32),
                              C.c_float(V0), xnew, C.byref(ch), C.byref(lm))
        return xnew, float(ch.value), float(lm.value), int(n)

    def objective(self, E, ce, csolid):
        return float(self.lib().orc_objective(self.h, np.ascontiguousarray(E, np.float64),
                                              np.ascontiguousarray(ce, np.float64), C.c_double(csolid)))

    def dc_scale(self, dcf, x):
        dc = np.zeros(self.ne, dtype=np.float32)
        self.lib().orc_dc_scale(self.h, np.ascontiguousarray(dcf, np.float32), np.ascontiguousarray(x, np.float32), dc)
        return dc

    def export_stl(self, xphys, path, iso=0.3):
        """restated export_surface_stl (io.cpp:80-87); returns the triangle count"""
        n = self.lib().orc_export_stl(self.h, np.ascontiguousarray(xphys, np.float32), path.encode(), C.c_float(iso))
        if n < 0:
            raise OSError("cannot write %s" % path)
        return int(n)

    def vol_sum(self, x):
        return float(self.lib().orc_vol_sum(self.h, np.ascontiguousarray(x, np.float32), len(x)))

    def sharpness(self, x):
        return float(self.lib().orc_sharpness(self.h, np.ascontiguousarray(x, np.float32), len(x)))

    def design_loop(self, V0, nloop, rmin=float(np.sqrt(np.float32(3.0)))):
        recs = (OrcIterRecord * max(1, nloop))()
        xf = np.zeros(self.ne, dtype=np.float32)
        cs = C.c_double()
        n = self.lib().orc_design_loop(self.h, C.c_float(V0), nloop, C.c_float(rmin), C.byref(cs), recs, xf)
        out = [dict(loop=r.loop, pcg_iters=r.pcg_iters, obj=r.obj, vol=r.vol, sharp=r.sharp, cons=r.cons,
                    change=r.change, lmid=r.lmid, bisections=r.bisections) for r in recs[:n]]
        return float(cs.value), out, xf


class Reference(_Common):
    """The unmodified reference sources behind oracle/ref_harness.cpp (oracle/_ref/libt3d_ref.so)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not reference_available():
                raise FileNotFoundError(REF_SO)
            L = C.CDLL(REF_SO)
            L.ref_create.restype = C.c_void_p
            L.ref_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_float]
            L.ref_destroy.argtypes = [C.c_void_p]
            L.ref_info.argtypes = [C.c_void_p, _i64p]
            L.ref_ele_map_back.argtypes = [C.c_void_p, _i32p]
            L.ref_free_dofs.argtypes = [C.c_void_p, _i32p]
            L.ref_bfree.argtypes = [C.c_void_p, _f64p]
            L.ref_ke.argtypes = [C.c_void_p, _f64p]
            L.ref_matvec.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
            L.ref_mg_build.argtypes = [C.c_void_p, _f64p]
            L.ref_vcycle.argtypes = [C.c_void_p, _f64p, _f64p]
            L.ref_pcg.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, C.c_double, C.c_int]
            L.ref_pcg.restype = C.c_int
            L.ref_compliance.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
            L.ref_compliance.restype = C.c_double
            L.ref_mg_diag.argtypes = [C.c_void_p, _f64p, C.c_int, _f64p]
            L.ref_mg_mask.argtypes = [C.c_void_p, C.c_int, _u8p]
            L.ref_coarse_matrix.argtypes = [C.c_void_p, _f64p, _f64p]
            L.ref_coarse_matrix.restype = C.c_int
            L.ref_filter_setup.argtypes = [C.c_void_p, C.c_float]
            L.ref_filter_apply.argtypes = [C.c_void_p, _f32p, _f32p]
            L.ref_filter_state.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
            L.ref_filter_set_state.argtypes = [C.c_void_p, _f64p, _f64p]
            L.ref_set_threads.argtypes = [C.c_int]
            L.ref_max_threads.restype = C.c_int
            L.ref_sample_iteration.argtypes = [C.c_void_p, C.c_float, C.c_int, C.c_int, _f64p]
            L.ref_sample_iteration.restype = C.c_int
            L.ref_run_global.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_float, C.c_char_p]
            L.ref_export_stl.argtypes = [C.c_void_p, _f32p, C.c_char_p, C.c_float]
            cls._lib = L
        return cls._lib

    @classmethod
    def set_threads(cls, n):
        cls.lib().ref_set_threads(int(n))

    @classmethod
    def run_global(cls, nely, nelx, nelz, V0, nloop, capdir, rmin=float(np.sqrt(np.float32(3.0)))):
        cls.lib().ref_run_global(nely, nelx, nelz, C.c_float(V0), nloop, C.c_float(rmin),
                                 capdir.encode() if capdir else b"")

    def export_stl(self, xphys, path, iso=0.3):
        """the reference's export_surface_stl (io.cpp:80-87) of densities in Morton order"""
        self.lib().ref_export_stl(self.h, np.ascontiguousarray(xphys, np.float32), path.encode(), C.c_float(iso))

    def __init__(self, nely, nelx, nelz, emin=None, max_levels=5):
        L = self.lib()
        self.h = C.c_void_p(L.ref_create(nely, nelx, nelz, max_levels, C.c_float(emin if emin else 0.0)))
        self._info = L.ref_info
        self._emb, self._fd, self._bf, self._ke = L.ref_ele_map_back, L.ref_free_dofs, L.ref_bfree, L.ref_ke
        self._mv, self._mgb, self._vc, self._pcg, self._cc = (L.ref_matvec, L.ref_mg_build, L.ref_vcycle,
                                                              L.ref_pcg, L.ref_compliance)
        self._mgd, self._mgm, self._ckc = L.ref_mg_diag, L.ref_mg_mask, L.ref_coarse_matrix
        self._fs, self._fa, self._fst, self._fss = (L.ref_filter_setup, L.ref_filter_apply, L.ref_filter_state,
                                                    L.ref_filter_set_state)
        self._setup_info()

    def sample_iteration(self, V0, pcg_max, rebuild_mg):
        """one reference design iteration with PCG capped at pcg_max; returns (iters, times[6])"""
        t = np.zeros(6)
        it = self.lib().ref_sample_iteration(self.h, C.c_float(V0), int(pcg_max), int(bool(rebuild_mg)), t)
        return int(it), t

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().ref_destroy(self.h)
            self.h = None
