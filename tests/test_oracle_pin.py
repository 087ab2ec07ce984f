"""Pins the CPU oracle (oracle/t3d_oracle.c) to the reference.

Golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the unmodified reference
build) are always checked; the live reference build (oracle/_ref) is used when present.
Tolerances: structure, masks, loads and every float32 design quantity are exact; double-precision
operator outputs agree to a few ulps (the reference build reassociates sums under -ffast-math).
"""
import hashlib

import numpy as np
import pytest

from conftest import golden
from oracle.bindings import Oracle

SMALL = [(6, 12, 6), (10, 20, 10)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.mark.parametrize("dims", SMALL + [(30, 60, 30)])
def test_structure_matches_reference(dims):
    g = golden("struct_%d_%d_%d.npz" % dims)
    o = Oracle(*dims)
    assert tuple(g["res"]) == o.res
    assert int(g["ne"]) == o.ne and int(g["nn"]) == o.nn and int(g["nf"]) == o.nf
    assert [tuple(l) for l in g["levels"]] == o.levels
    assert sha(o.ele_map_back()) == str(g["sha_ele_map_back"])
    assert sha(o.free_dofs()) == str(g["sha_free_dofs"])
    assert sha(o.bfree()) == str(g["sha_bfree"])
    for l in range(o.nlev):
        assert sha(o.mg_mask(l)) == str(g["sha_mask%d" % l]), l
    assert np.abs(o.ke() - g["ke"]).max() < 1e-16


@pytest.mark.parametrize("dims", SMALL)
def test_single_call_operators_match_reference(dims):
    g = golden("ops_%d_%d_%d.npz" % dims)
    s = golden("struct_%d_%d_%d.npz" % dims)
    o = Oracle(*dims)
    o.set_ke(s["ke"])
    E, u = g["E"], g["u"]
    assert rel(o.matvec(E, u), g["Ku"]) < 1e-15
    o.mg_build(E)
    for l in range(o.nlev):
        assert rel(o.mg_diag(l), g["diag%d" % l]) < 1e-15, l
    if "Kc" in g:
        assert rel(o.coarse_matrix(E), g["Kc"]) < 1e-14
    assert rel(o.vcycle(g["vc_r"]), g["vc_z"]) < 1e-13
    x, it = o.pcg(E, o.bfree(), np.zeros(o.nf), maxit=50)
    assert it == int(g["pcg50_iters"])
    assert np.linalg.norm(x - g["pcg50_x"]) / np.linalg.norm(g["pcg50_x"]) < 1e-12
    C, ce = o.compliance(E, g["pcg50_x"])
    assert abs(C - float(g["C"])) / abs(float(g["C"])) < 1e-13
    assert rel(ce, g["ce"]) < 1e-12
    o.filter_setup()
    assert rel(o.filter_state()[2], g["filt_diag"]) < 1e-15
    np.testing.assert_array_equal(o.filter_apply(g["filt_src"]), g["filt_dst"])


def test_design_iterations_replay_bit_exact():
    """Replay of the captured reference driver: with the reference build's x86 approximations
    emulated (approx_mode=1, libmvec powf), SIMP, sensitivities, filter, dc scaling and OC
    reproduce the reference bit for bit at every iteration; PCG iteration counts are identical."""
    t = golden("traj_10_20_10.npz")
    dims = (10, 20, 10)
    s = golden("struct_%d_%d_%d.npz" % dims)
    o = Oracle(*dims, pow_mode=1, vol_mode=0, approx_mode=1)
    o.set_ke(s["ke"])
    b = o.bfree()
    V0 = float(t["V0"])
    Cs = float(t["Csolid"])
    x = np.full(o.ne, np.float32(V0), np.float32)
    nloop = int(t["nloop"])
    for k in range(1, nloop + 1):
        np.testing.assert_array_equal(o.simp(x), t["E%d" % k])
        pk = 1 if k < 5 else (k // 5) * 5
        o.mg_build(t["E%d" % pk])
        u, it = o.pcg(t["E%d" % k], b, t["u0_%d" % k])
        assert it == int(t["iters%d" % k])
        if it < 800:
            assert np.linalg.norm(u - t["u1_%d" % k]) / np.linalg.norm(t["u1_%d" % k]) < 1e-10
        C, ce = o.compliance(t["E%d" % k], t["u1_%d" % k])
        assert abs(C - float(t["C%d" % k])) / float(t["C%d" % k]) < 1e-12
        dc = o.sens(x, t["ce%d" % k], Cs)
        np.testing.assert_array_equal((x * dc).astype(np.float32), t["fsrc%d" % k])
        o.filter_setup()
        o.filter_set_state(t["flastx%d" % k], t["flastrhs%d" % k])
        np.testing.assert_array_equal(o.filter_apply(t["fsrc%d" % k]), t["fdst%d" % k])
        dcs = o.dc_scale(t["fdst%d" % k], x)
        x, ch, lm, nb = o.oc(x, dcs, V0)
    np.testing.assert_array_equal(x, t["xfinal"])


def test_solid_solve_matches_reference():
    t = golden("traj_10_20_10.npz")
    o = Oracle(10, 20, 10)
    o.set_ke(golden("struct_10_20_10.npz")["ke"])
    E = np.ones(o.ne)
    o.mg_build(E)
    u, it = o.pcg(E, o.bfree(), np.zeros(o.nf))
    assert it == int(t["solid_iters"])
    C, _ = o.compliance(E, u)
    assert abs(C - float(t["Csolid"])) / float(t["Csolid"]) < 1e-12


def test_live_reference_single_calls(ref_or_skip):
    Reference = ref_or_skip
    dims = (6, 12, 6)
    r = Reference(*dims)
    o = Oracle(*dims)
    o.set_ke(r.ke())
    rng = np.random.default_rng(7)
    E = rng.uniform(1e-3, 1.0, o.ne)
    u = rng.standard_normal(o.nf)
    assert rel(o.matvec(E, u), r.matvec(E, u)) < 1e-15
    o.mg_build(E)
    r.mg_build(E)
    rv = rng.standard_normal(o.nf)
    assert rel(o.vcycle(rv), r.vcycle(rv)) < 1e-13
