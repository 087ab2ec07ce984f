"""The two FP64 K(E)u kernels against each other, bit for bit.

The element-streaming kernel (the default) runs the same FMA chains as the node-centric gather
kernel, in the same order, and folds each node's eight element contributions in the reference's
colour order (fea.cpp:300, fea.cpp:763-837); only where each chain runs differs.  So the two forms
must agree in every bit, including the signs of zeros, on any grid (tiles and slabs that do not
divide it), with skipped elements (E <= 1e-16, voids) and through whole PCG solves and design steps.
Agreement with the oracle and the reference is covered by the parity tests, which run the default
(streaming) form.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64)).view(np.int64)


def pair(dims, **kw):
    import algorithmengineering_altproject_b200 as t3d
    S = t3d.Problem(*dims, **kw)
    N = t3d.Problem(*dims, matvec64_form=t3d.T3D_MATVEC64_NODES, **kw)
    return S, N


@pytest.mark.parametrize("dims", [(6, 12, 6), (10, 20, 10), (17, 40, 23), (30, 60, 30), (9, 70, 5)])
def test_streaming_matvec_is_bit_identical(dims):
    S, N = pair(dims)
    rng = np.random.default_rng(21)
    for trial in range(3):
        E = rng.uniform(1e-3, 1.0, S.ne)
        if trial == 1:    # design-like: many elements at Emin, some skipped (E <= 1e-16)
            E = np.where(rng.random(S.ne) < 0.6, 1e-9, 1.0)
            E[rng.random(S.ne) < 0.1] = 1e-17
        if trial == 2:
            E[rng.random(S.ne) < 0.3] = 0.0
        u = rng.standard_normal(S.nf)
        np.testing.assert_array_equal(bits(S.K_times_u_finest(E, u)), bits(N.K_times_u_finest(E, u)))
    S.close()
    N.close()


def test_streaming_matvec_with_voids_and_load_cases():
    import algorithmengineering_altproject_b200 as t3d
    spec = t3d.ProblemSpec.make(t3d.T3D_LOAD_TORSION, [(6.0, 3.0, 3.0, 2.5, 2.0, 2.0)])
    S, N = pair((6, 12, 6), problem=spec)
    rng = np.random.default_rng(8)
    E = rng.uniform(1e-3, 1.0, S.ne)
    u = rng.standard_normal(S.nf)
    np.testing.assert_array_equal(bits(S.K_times_u_finest(E, u)), bits(N.K_times_u_finest(E, u)))
    S.close()
    N.close()


@pytest.mark.parametrize("dims", [(10, 20, 10), (17, 40, 23)])
def test_pcg_and_design_steps_identical_across_forms(dims):
    S, N = pair(dims, cg_max_it=300)
    rng = np.random.default_rng(2)
    E = rng.uniform(1e-3, 1.0, S.ne)
    b = S.bfree()
    out = []
    for P in (S, N):
        P.make_diagonal_preconditioner_from_static(E)
        out.append(P.PCG_free(E, b, np.zeros(P.nf), tol=1e-10))
    (x_s, it_s), (x_n, it_n) = out[0], out[1]
    assert it_s == it_n
    np.testing.assert_array_equal(bits(x_s), bits(x_n))
    recs = []
    for P in (S, N):
        P.design_init(0.3)
        recs.append([P.design_step() for _ in range(2)])
    for rs, rn in zip(*recs):
        assert rs["obj"] == rn["obj"] and rs["pcg_iters"] == rn["pcg_iters"], (rs, rn)
    np.testing.assert_array_equal(S.density(), N.density())
    S.close()
    N.close()


@pytest.mark.parametrize("precision", [0, 1])   # T3D_FP64, T3D_MIXED
def test_set_ke_reaches_captured_pcg_iterations(precision):
    # the captured PCG iterations carry Ke (FP64 streaming kernel) and the modal FP32 coefficients by
    # value: after t3d_set_ke a context that has already solved must give what a fresh one gives
    import algorithmengineering_altproject_b200 as t3d
    A = t3d.Problem(10, 20, 10, precision=precision)
    B = t3d.Problem(10, 20, 10, precision=precision)
    K2 = 2.0 * A.ke()
    c1 = A.design_init(0.3)
    A.set_ke(K2)
    B.set_ke(K2)
    ca, cb = A.design_init(0.3), B.design_init(0.3)
    # and the stiffer Ke is in effect: about half the compliance (not exactly: the coarsest operator's
    # Emin floor and the stopping test do not scale with Ke)
    assert ca == cb and abs(ca - 0.5 * c1) <= 1e-3 * c1, (c1, ca, cb)
    A.close()
    B.close()


def test_kernel_forms_follow_ke():
    # the built-in Ke runs the register-operand form (2); any other Ke the constant-bank form (1); both
    # agree bit for bit with the node-centric kernel (0)
    import algorithmengineering_altproject_b200 as t3d
    S, N = pair((10, 20, 10))
    assert S.info().matvec64_kernel == 2 and N.info().matvec64_kernel == 0
    rng = np.random.default_rng(13)
    E = rng.uniform(1e-3, 1.0, S.ne)
    u = rng.standard_normal(S.nf)
    Ke = S.ke()
    A = rng.standard_normal((24, 24)) * 1e-3
    K2 = Ke + (A + A.T)
    for P in (S, N):
        P.set_ke(K2)
    assert S.info().matvec64_kernel == 1
    np.testing.assert_array_equal(bits(S.K_times_u_finest(E, u)), bits(N.K_times_u_finest(E, u)))
    for P in (S, N):
        P.set_ke(Ke)
    assert S.info().matvec64_kernel == 2
    np.testing.assert_array_equal(bits(S.K_times_u_finest(E, u)), bits(N.K_times_u_finest(E, u)))
    S.close()
    N.close()
