"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the UNMODIFIED reference sources (oracle/_ref/libt3d_ref.so, built by
``make -C oracle ref``) single-threaded and records:

* ``struct_<nely>_<nelx>_<nelz>.npz`` -- model structure: padded dims, MG levels, Morton element
  map (eleMapBack), free-DOF list, load vector, Ke, per-level BC masks (full arrays for the small
  grids, SHA-256 digests for the config-0 grid);
* ``ops_<dims>.npz`` -- single-call operator vectors on seeded inputs: K(E)u (fea.cpp:763),
  MG diagonals and coarsest Galerkin matrix (diagonal.cpp:140, coarsest.cpp:138), one V-cycle
  application (preconditioner.cpp:88), 50 PCG iterations (solver.cpp:87), compliance
  (fea.cpp:851) and one PDE-filter application (filter.cpp:175);
* ``traj_<dims>.npz`` -- a capture of the reference driver TOP3D_XL_GLOBAL (driver.cpp:23) for a
  few design iterations: per iteration the SIMP moduli, PCG warm start/result/iteration count,
  element compliances, filter input/output and warm-start state, and the final densities.

Usage:  python tests/golden/make_golden.py   (needs the reference build oracle/_ref:
        make -C oracle ref REF=<reference root>)
"""
import hashlib
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.bindings import Reference  # noqa: E402

SMALL = [(6, 12, 6), (10, 20, 10)]
CONFIG0 = (30, 60, 30)
TRAJ = ((10, 20, 10), 0.12, 4)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def structure(dims, full):
    r = Reference(*dims)
    d = dict(res=np.array(r.res), ne=r.ne, nn=r.nn, nf=r.nf, levels=np.array(r.levels), ke=r.ke())
    arrays = dict(ele_map_back=r.ele_map_back(), free_dofs=r.free_dofs(), bfree=r.bfree())
    for l in range(r.nlev):
        arrays["mask%d" % l] = r.mg_mask(l)
    for k, v in arrays.items():
        d["sha_" + k] = sha(v)
        if full:
            d[k] = v
    np.savez_compressed(os.path.join(HERE, "struct_%d_%d_%d.npz" % dims), **d)


def ops(dims):
    r = Reference(*dims)
    rng = np.random.default_rng(20251203)
    E = rng.uniform(1e-6, 1.0, r.ne)
    u = rng.standard_normal(r.nf)
    d = dict(E=E, u=u, Ku=r.matvec(E, u))
    for l in range(r.nlev):
        d["diag%d" % l] = r.mg_diag(l, E)
    Kc = r.coarse_matrix(E)
    if Kc is not None:
        d["Kc"] = Kc
    r.mg_build(E)
    rv = rng.standard_normal(r.nf)
    d["vc_r"] = rv
    d["vc_z"] = r.vcycle(rv)
    b = r.bfree()
    x, it = r.pcg(E, b, np.zeros(r.nf), maxit=50)
    d["pcg50_x"] = x
    d["pcg50_iters"] = it
    C, ce = r.compliance(E, x)
    d["C"] = C
    d["ce"] = ce
    r.filter_setup()
    src = (-rng.uniform(0.0, 0.5, r.ne)).astype(np.float32)
    d["filt_src"] = src
    d["filt_dst"] = r.filter_apply(src)
    d["filt_diag"] = r.filter_state()[2]
    np.savez_compressed(os.path.join(HERE, "ops_%d_%d_%d.npz" % dims), **d)


def trajectory(dims, V0, nloop):
    cap = tempfile.mkdtemp(prefix="t3dcap_")
    cwd = os.getcwd()
    try:
        os.chdir(cap)
        Reference.run_global(*dims, V0, nloop, cap)
    finally:
        os.chdir(cwd)

    def rd(name, dt):
        return np.fromfile(os.path.join(cap, name), dtype=dt)

    d = dict(V0=V0, nloop=nloop, Csolid=rd("cc_000_C.bin", np.float64)[0],
             solid_iters=rd("pcg_000_iters.bin", np.int32)[0], solid_u=rd("pcg_000_x1.bin", np.float64))
    for k in range(1, nloop + 1):
        d["E%d" % k] = rd("pcg_%03d_E.bin" % k, np.float64)
        d["u0_%d" % k] = rd("pcg_%03d_x0.bin" % k, np.float64)
        d["u1_%d" % k] = rd("pcg_%03d_x1.bin" % k, np.float64)
        d["iters%d" % k] = rd("pcg_%03d_iters.bin" % k, np.int32)[0]
        d["ce%d" % k] = rd("cc_%03d_ce.bin" % k, np.float64)
        d["C%d" % k] = rd("cc_%03d_C.bin" % k, np.float64)[0]
        d["fsrc%d" % k] = rd("filt_%03d_src.bin" % (k - 1), np.float32)
        d["fdst%d" % k] = rd("filt_%03d_dst.bin" % (k - 1), np.float32)
        d["flastx%d" % k] = rd("filt_%03d_lastx0.bin" % (k - 1), np.float64)
        d["flastrhs%d" % k] = rd("filt_%03d_lastrhs0.bin" % (k - 1), np.float64)
    d["xfinal"] = rd("xphys_final.bin", np.float32)
    shutil.rmtree(cap, ignore_errors=True)
    np.savez_compressed(os.path.join(HERE, "traj_%d_%d_%d.npz" % dims), **d)


def main():
    Reference.set_threads(1)
    for dims in SMALL:
        structure(dims, True)
        ops(dims)
    structure(CONFIG0, False)
    trajectory(*TRAJ)


if __name__ == "__main__":
    main()
