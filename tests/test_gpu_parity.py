"""Parity of the CUDA path (through the C-ABI) with the CPU oracle and with the reference.

Two oracles are used:
* the C restatement in its canonical-order mode (red_mode=1: the CUDA path's deterministic
  reduction order; IEEE sqrt/division; correctly rounded powf).  Against it every result is
  compared BIT FOR BIT -- operator outputs, PCG iteration counts and iterates, and whole design
  trajectories;
* the reference itself, through the golden fixtures made from its unmodified build
  (tests/golden/make_golden.py).  Against these the tolerances are the reference build's own
  rounding (fast-math reassociated sums): 1e-15..1e-12 relative for operators, iteration counts
  equal, float design quantities within one float ulp where the reference uses x86 approximate
  rsqrt/rcp (driver.cpp:166,176).
"""
import numpy as np
import pytest

from conftest import golden
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu

SMALL = [(6, 12, 6), (10, 20, 10)]


def gpu_problem(dims, **kw):
    import algorithmengineering_altproject_b200 as t3d
    return t3d.Problem(*dims, **kw)


def canon_oracle(dims, **kw):
    return Oracle(*dims, red_mode=1, pow_mode=0, vol_mode=0, approx_mode=0, **kw)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def same_bits(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape
    return bool(np.array_equal(a.view(np.uint8), b.view(np.uint8)))


@pytest.mark.parametrize("dims", SMALL + [(30, 60, 30)])
def test_structure_matches_reference(dims):
    import hashlib
    g = golden("struct_%d_%d_%d.npz" % dims)
    P = gpu_problem(dims)
    assert P.res == tuple(g["res"])
    assert P.ne == int(g["ne"]) and P.nn == int(g["nn"]) and P.nf == int(g["nf"])
    assert P.levels == [tuple(l) for l in g["levels"]]
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    assert sha(P.ele_map_back()) == str(g["sha_ele_map_back"])
    assert sha(P.free_dofs()) == str(g["sha_free_dofs"])
    assert sha(P.bfree()) == str(g["sha_bfree"])
    for l in range(P.nlev):
        assert sha(P.mg_mask(l)) == str(g["sha_mask%d" % l])
    assert np.abs(P.ke() - g["ke"]).max() < 1e-16


@pytest.mark.parametrize("dims", SMALL)
def test_operators_bit_exact_with_oracle(dims):
    P = gpu_problem(dims)
    O = canon_oracle(dims)
    assert same_bits(P.ke(), O.ke())
    rng = np.random.default_rng(11)
    E = rng.uniform(1e-6, 1.0, P.ne)
    u = rng.standard_normal(P.nf)
    assert same_bits(P.K_times_u_finest(E, u), O.matvec(E, u))
    P.make_diagonal_preconditioner_from_static(E)
    O.mg_build(E)
    for l in range(P.nlev):
        assert same_bits(P.mg_diag(l), O.mg_diag(l)), l
    if P.coarse_n:
        assert same_bits(P.coarse_matrix(E), O.coarse_matrix(E))
        P.make_diagonal_preconditioner_from_static(E)
    r = rng.standard_normal(P.nf)
    assert same_bits(P.vcycle(r), O.vcycle(r))
    b = P.bfree()
    xg, ig = P.PCG_free(E, b, np.zeros(P.nf))
    xo, io = O.pcg(E, b, np.zeros(P.nf))
    assert ig == io
    assert same_bits(xg, xo)
    Cg, ceg = P.ComputeCompliance(E, xg)
    Co, ceo = O.compliance(E, xo)
    assert same_bits(ceg, ceo) and Cg == Co


@pytest.mark.parametrize("dims", SMALL)
def test_operators_match_reference_golden(dims):
    g = golden("ops_%d_%d_%d.npz" % dims)
    P = gpu_problem(dims)
    P.set_ke(golden("struct_%d_%d_%d.npz" % dims)["ke"])
    E = g["E"]
    assert rel(P.K_times_u_finest(E, g["u"]), g["Ku"]) < 1e-15
    P.make_diagonal_preconditioner_from_static(E)
    for l in range(P.nlev):
        assert rel(P.mg_diag(l), g["diag%d" % l]) < 1e-15
    if "Kc" in g:
        assert rel(P.coarse_matrix(E), g["Kc"]) < 1e-14
        P.make_diagonal_preconditioner_from_static(E)
    assert rel(P.vcycle(g["vc_r"]), g["vc_z"]) < 1e-13
    x, it = P.PCG_free(E, P.bfree(), np.zeros(P.nf), maxIt=50)
    assert it == int(g["pcg50_iters"])
    assert np.linalg.norm(x - g["pcg50_x"]) / np.linalg.norm(g["pcg50_x"]) < 1e-12
    C, ce = P.ComputeCompliance(E, g["pcg50_x"])
    assert abs(C - float(g["C"])) / abs(float(g["C"])) < 1e-13
    assert rel(ce, g["ce"]) < 1e-12
    assert rel(P.filter_state()[2], g["filt_diag"]) < 1e-15
    np.testing.assert_array_equal(P.ApplyPDEFilter(g["filt_src"]), g["filt_dst"])


def test_design_quantities_bit_exact_with_oracle():
    dims = (10, 20, 10)
    P = gpu_problem(dims)
    O = canon_oracle(dims)
    rng = np.random.default_rng(5)
    x = rng.uniform(1e-3, 1.0, P.ne).astype(np.float32)
    assert same_bits(P.simp(x), O.simp(x))
    ce = rng.uniform(0.0, 2.0, P.ne)
    dc = P.sensitivity(x, ce, 1.7)
    assert same_bits(dc, O.sens(x, ce, 1.7))
    src = (x * dc).astype(np.float32)
    O.filter_setup()
    assert same_bits(P.ApplyPDEFilter(src), O.filter_apply(src))
    dcs = P.dc_scale(src, x)
    assert same_bits(dcs, O.dc_scale(src, x))
    xg, chg, lmg, nbg = P.oc_update(x, dcs, 0.12)
    xo, cho, lmo, nbo = O.oc(x, dcs, 0.12)
    assert nbg == nbo and lmg == lmo and chg == cho
    assert same_bits(xg, xo)


@pytest.mark.parametrize("dims,nloop", [((6, 12, 6), 6), ((10, 20, 10), 5)])
def test_design_loop_bit_exact_with_oracle(dims, nloop):
    P = gpu_problem(dims)
    O = canon_oracle(dims)
    csg, recg, xg = P.run_global(0.12, nloop)
    cso, reco, xo = O.design_loop(0.12, nloop)
    assert csg == cso
    assert len(recg) == len(reco)
    for a, b in zip(recg, reco):
        assert a["pcg_iters"] == b["pcg_iters"]
        assert a["obj"] == b["obj"]
        assert a["change"] == b["change"] and a["sharp"] == b["sharp"] and a["vol"] == b["vol"]
        assert a["bisections"] == b["bisections"]
    assert same_bits(xg, xo)


def test_replay_against_reference_capture():
    """Each design iteration of the captured reference run replayed on the GPU from the reference's
    own state: PCG iteration counts equal, converged displacements within 1e-10, compliance within
    1e-12, filter outputs bit-identical, OC densities within one float ulp of the reference (whose
    build evaluates sqrt and the dc division with x86 approximate rsqrt/rcp + one Newton step)."""
    t = golden("traj_10_20_10.npz")
    dims = (10, 20, 10)
    P = gpu_problem(dims)
    P.set_ke(golden("struct_10_20_10.npz")["ke"])
    b = P.bfree()
    V0 = float(t["V0"])
    x = np.full(P.ne, np.float32(V0), np.float32)
    for k in range(1, int(t["nloop"]) + 1):
        pk = 1 if k < 5 else (k // 5) * 5
        P.make_diagonal_preconditioner_from_static(t["E%d" % pk])
        u, it = P.PCG_free(t["E%d" % k], b, t["u0_%d" % k])
        assert it == int(t["iters%d" % k])
        if it < 800:
            assert np.linalg.norm(u - t["u1_%d" % k]) / np.linalg.norm(t["u1_%d" % k]) < 1e-10
        C, ce = P.ComputeCompliance(t["E%d" % k], t["u1_%d" % k])
        assert abs(C - float(t["C%d" % k])) / float(t["C%d" % k]) < 1e-12
        P.filter_set_state(t["flastx%d" % k], t["flastrhs%d" % k])
        np.testing.assert_array_equal(P.ApplyPDEFilter(t["fsrc%d" % k]), t["fdst%d" % k])
        if k == 1:
            np.testing.assert_array_equal(P.simp(x), t["E1"])
    # whole chain from the captured filter outputs: densities within one float ulp of the reference
    x = np.full(P.ne, np.float32(V0), np.float32)
    for k in range(1, int(t["nloop"]) + 1):
        dcs = P.dc_scale(t["fdst%d" % k], x)
        x, _, _, _ = P.oc_update(x, dcs, V0)
        if k < int(t["nloop"]):
            Eg = P.simp(x)
            assert rel(Eg, t["E%d" % (k + 1)]) < 1e-6
    assert np.abs(x - t["xfinal"]).max() <= 1.2e-7


def test_published_reference_values_50x100x50():
    """The reference's published run (out/log/GLOBAL_latest.log:53,56): compliance of the solid
    domain 6.365655e-01 and iteration-1 objective 3.68170629e+02 at 50x100x50, V0 = 0.12."""
    P = gpu_problem((50, 100, 50))
    cs = P.design_init(0.12)
    assert "%.6e" % cs == "6.365655e-01"
    rec = P.design_step()
    assert "%.8e" % rec["obj"] == "3.68170629e+02"
