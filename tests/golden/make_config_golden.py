"""Generate the golden fixtures of the benchmark configurations (tests/golden/cfg*.npz).

The CUDA path matches the oracle's canonical mode bit for bit, so for the large grids the fixtures keep
SHA-256 digests of the oracle's outputs (plus norms for a readable failure message) instead of the
vectors; against the reference they keep seeded samples of its outputs.  Inputs are regenerated in the
tests from the same seeds (numpy's default_rng, one seed per input).

* ``cfg0_traj.npz`` -- the reference CLI demo ``GLOBAL 30 60 30 0.12 30`` (driver.cpp:23-280): the
  canonical oracle's whole 30-iteration trajectory (solid compliance; per iteration PCG count, objective,
  volume, sharpness, change, bisection passes; final densities), the reference's own run (one thread,
  captured through oracle/ref_harness.cpp: solid compliance, per-iteration compliance and PCG count, the
  printed ``It.:`` lines, final densities) and the same run of the reference built without -ffast-math
  (oracle/Makefile ``ref-nofm``): the reference's build-to-build drift, the floor for comparing free-
  running trajectories;
* ``cfg1_ops.npz`` -- single-call operators at 96x192x96 (5,419,584 free DOFs) on seeded inputs:
  canonical-oracle digests of K(E)u, MG diagonals, one V-cycle, 50 PCG iterations, compliance, the PDE
  filter, SIMP, sensitivities, dc scaling and the OC update; reference samples of the same vectors;
* ``cfg1_traj.npz`` -- the first three design iterations of the reference at 96x192x96 (fast-math and
  without it, eight threads): solid compliance, per-iteration compliance and PCG count, samples of the
  displacement and moduli, final densities;
* ``cfg2_ops.npz`` -- FP64 K(E)u and one V-cycle (6 levels) at 256x512x256 (101,451,264 free DOFs):
  canonical-oracle digests.

Usage:  python tests/golden/make_config_golden.py cfg0|cfg1|cfg2 ...
        (needs oracle/_ref and oracle/_ref/nofm: make -C oracle ref ref-nofm REF=<reference root>)
"""
import hashlib
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
from oracle.bindings import Oracle, Reference  # noqa: E402
from seeded import NSAMPLE, config_inputs, sample_indices  # noqa: E402

NOFM_SO = os.path.join(ROOT, "oracle", "_ref", "nofm", "libt3d_ref.so")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def canon(dims, **kw):
    return Oracle(*dims, red_mode=1, pow_mode=0, vol_mode=0, approx_mode=0, **kw)


def inputs(seed, ne, nf):
    """The seeded inputs of the single-call checks (the tests draw the same arrays)."""
    return config_inputs(seed, ne, nf)


# ---------------------------------------------------------------- reference runs (one process per build)
def run_reference_global(dims, V0, nloop, threads, so=None):
    """TOP3D_XL_GLOBAL of the reference build `so` in a child process: returns its captured arrays and the
    parsed It.: lines."""
    work = tempfile.mkdtemp(prefix="t3dref_")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    if so:
        env["T3D_REF_SO"] = so
    cmd = [sys.executable, os.path.abspath(__file__), "_refrun", json.dumps([list(dims), V0, nloop, threads]), work]
    with open(os.path.join(work, "stdout.txt"), "w") as out:
        subprocess.run(cmd, check=True, env=env, stdout=out, cwd=work)
    text = open(os.path.join(work, "stdout.txt")).read()
    lines = re.findall(r"It\.:\s*(\d+) Obj\.:\s*(\S+) Vol\.:\s*(\S+) Sharp\.:\s*(\S+) Cons\.:\s*(\S+) Ch\.:\s*(\S+)",
                       text)
    rd = lambda name, dt: np.fromfile(os.path.join(work, name), dtype=dt)
    res = dict(csolid=rd("cc_000_C.bin", np.float64)[0], n=len(lines),
               obj_printed=np.array([float(l[1]) for l in lines]), change_printed=np.array([float(l[5]) for l in lines]),
               sharp_printed=np.array([float(l[3]) for l in lines]), vol_printed=np.array([float(l[2]) for l in lines]),
               C=np.array([rd("cc_%03d_C.bin" % k, np.float64)[0] for k in range(1, len(lines) + 1)]),
               iters=np.array([rd("pcg_%03d_iters.bin" % k, np.int32)[0] for k in range(1, len(lines) + 1)]),
               xfinal=rd("xphys_final.bin", np.float32), work=work)
    return res


def _refrun(spec, work):
    dims, V0, nloop, threads = json.loads(spec)
    Reference.set_threads(threads)
    Reference.run_global(*dims, V0, nloop, work)
    import ctypes
    ctypes.CDLL(None).fflush(None)


# ---------------------------------------------------------------- config 0: the CLI demo, whole trajectory
def cfg0():
    dims, V0, nloop = (30, 60, 30), 0.12, 30
    O = canon(dims)
    cs, recs, xf = O.design_loop(V0, nloop)
    d = dict(V0=V0, nloop=nloop, orc_csolid=cs, orc_xfinal=xf)
    for k in ("pcg_iters", "obj", "vol", "sharp", "change", "bisections"):
        d["orc_" + k] = np.array([r[k] for r in recs])
    for tag, so in (("ref", None), ("nofm", NOFM_SO)):
        r = run_reference_global(dims, V0, nloop, 1, so)
        shutil.rmtree(r.pop("work"), ignore_errors=True)
        for k, v in r.items():
            d["%s_%s" % (tag, k)] = v
    np.savez_compressed(os.path.join(HERE, "cfg0_traj.npz"), **d)
    print("cfg0: oracle obj[0]=%.9e ref obj[0]=%.9e nofm obj[0]=%.9e; it.30 ref %.9e nofm %.9e oracle %.9e"
          % (d["orc_obj"][0], d["ref_C"][0], d["nofm_C"][0], d["ref_C"][-1], d["nofm_C"][-1], d["orc_obj"][-1]))


# ---------------------------------------------------------------- config 1: single-call operators
def cfg1_ops():
    dims, seed = (96, 192, 96), 20251203
    O = canon(dims)
    I = inputs(seed, O.ne, O.nf)
    d = dict(seed=seed, idx_f=I["idx_f"], idx_e=I["idx_e"])

    f, e = I["idx_f"], I["idx_e"]

    def put(name, a, idx=None):
        a = np.ascontiguousarray(a)
        d["sha_" + name] = sha(a)
        d["norm_" + name] = float(np.linalg.norm(a.astype(np.float64)))
        if idx is not None:
            d["orc_" + name] = a[idx]

    put("Ku", O.matvec(I["E"], I["u"]), f)
    O.mg_build(I["E"])
    for l in range(O.nlev):
        put("diag%d" % l, O.mg_diag(l))
    put("vc_z", O.vcycle(I["r"]), f)
    b = O.bfree()
    x, it = O.pcg(I["E"], b, np.zeros(O.nf), maxit=50)
    put("pcg50_x", x, f)
    d["orc_pcg50_iters"] = it
    C, ce = O.compliance(I["E"], x)
    put("ce", ce, e)
    d["orc_C"] = C
    O.filter_setup()
    put("filt_dst", O.filter_apply(I["fsrc"]), e)
    put("simp", O.simp(I["x"]))
    dc = O.sens(I["x"], I["ce"], 1.7)
    put("sens", dc)
    dcs = O.dc_scale(I["fsrc"], I["x"])
    put("dc_scale", dcs)
    xn, ch, lm, nb = O.oc(I["x"], dcs, 0.12)
    put("oc_x", xn)
    d.update(orc_oc_change=ch, orc_oc_lmid=lm, orc_oc_bisections=nb)
    del O
    # the reference (fast-math build, eight threads) on the same inputs: samples
    Reference.set_threads(8)
    R = Reference(*dims)
    d["ref_Ku"] = R.matvec(I["E"], I["u"])[f]
    R.mg_build(I["E"])
    d["ref_vc_z"] = R.vcycle(I["r"])[f]
    xr, itr = R.pcg(I["E"], b, np.zeros(R.nf), maxit=50)
    d["ref_pcg50_x"] = xr[f]
    d["ref_pcg50_iters"] = itr
    Cr, cer = R.compliance(I["E"], xr)
    d["ref_C"] = Cr
    d["ref_ce"] = cer[e]
    R.filter_setup()
    d["ref_filt_dst"] = R.filter_apply(I["fsrc"])[e]
    np.savez_compressed(os.path.join(HERE, "cfg1_ops.npz"), **d)
    rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())
    print("cfg1 ops: pcg50 oracle %d ref %d; C oracle %.15e ref %.15e" % (it, itr, C, Cr))
    print("cfg1 ops: oracle vs reference samples:", {k: rel(d["orc_" + k], d["ref_" + k])
                                                      for k in ("Ku", "vc_z", "pcg50_x", "ce", "filt_dst")})


# ---------------------------------------------------------------- config 1: first design iterations
def cfg1_traj():
    dims, V0, nloop = (96, 192, 96), 0.12, 3
    seed = 20251203
    d = dict(V0=V0, nloop=nloop)
    for tag, so in (("ref", None), ("nofm", NOFM_SO)):
        r = run_reference_global(dims, V0, nloop, 8, so)
        work = r.pop("work")
        nf = len(np.fromfile(os.path.join(work, "pcg_001_x1.bin"), dtype=np.float64))
        idx = sample_indices(seed, 9, nf)
        d["idx_u"] = idx
        for k in range(1, nloop + 1):
            d["%s_u%d" % (tag, k)] = np.fromfile(os.path.join(work, "pcg_%03d_x1.bin" % k), dtype=np.float64)[idx]
        shutil.rmtree(work, ignore_errors=True)
        for k, v in r.items():
            d["%s_%s" % (tag, k)] = v
    # final densities: the full-field build-to-build drift and seeded samples of both builds
    idx = sample_indices(seed, 10, len(d["ref_xfinal"]))
    d["idx_x"] = idx
    d["xdrift_full"] = float(np.abs(d["ref_xfinal"] - d["nofm_xfinal"]).max())
    d["ref_xfinal"], d["nofm_xfinal"] = d["ref_xfinal"][idx], d["nofm_xfinal"][idx]
    np.savez_compressed(os.path.join(HERE, "cfg1_traj.npz"), **d)
    print("cfg1 traj: ref C", d["ref_C"], "nofm C", d["nofm_C"], "iters", d["ref_iters"])


# ---------------------------------------------------------------- config 2: FP64 single-call operators
def cfg2_ops():
    dims, seed = (256, 512, 256), 20251204
    O = canon(dims, max_levels=6)
    g = lambda k: np.random.default_rng([seed, k])
    E = g(1).uniform(1e-6, 1.0, O.ne)
    u = g(2).standard_normal(O.nf)
    d = dict(seed=seed)
    Ku = O.matvec(E, u)
    d.update(sha_Ku=sha(Ku), norm_Ku=float(np.linalg.norm(Ku)))
    del Ku, u
    O.mg_build(E)
    r = g(3).standard_normal(O.nf)
    z = O.vcycle(r)
    d.update(sha_vc_z=sha(z), norm_vc_z=float(np.linalg.norm(z)), nlev=O.nlev, coarse_n=O.coarse_n())
    np.savez_compressed(os.path.join(HERE, "cfg2_ops.npz"), **d)
    print("cfg2 ops:", {k: v for k, v in d.items() if k.startswith("norm")})


def main(argv):
    if argv[:1] == ["_refrun"]:
        return _refrun(argv[1], argv[2])
    jobs = {"cfg0": cfg0, "cfg1": lambda: (cfg1_ops(), cfg1_traj()), "cfg1_ops": cfg1_ops, "cfg1_traj": cfg1_traj,
            "cfg2": cfg2_ops}
    for a in argv or ["cfg0", "cfg1", "cfg2"]:
        jobs[a]()


if __name__ == "__main__":
    main(sys.argv[1:])
