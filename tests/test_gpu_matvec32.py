"""The FP32 K(E)u of the mixed-precision inner solve against the FP64 operator.

Two FP32 forms exist: the modal (corner-Hadamard) kernel, used whenever Ke is the stiffness of an
axis-aligned cubic isotropic voxel, and the dense 24x24 gather kernel.  Both compute the reference's
K_times_u_finest (fea.cpp:763-837) with FP32 inputs, so each must agree with the FP64 product to
FP32 accuracy: ||y32 - y64|| <= 2e-6 ||y64|| on random moduli and displacements.  The grids cover a
padded one (30x60x30 -> 64x32x32 elements) and ones that do not divide the kernel's node tiles.
The FP32 V-cycle of the same inner solve is checked against the FP64 V-cycle the same way (1e-5).
Every tile shape of the modal kernel -- per-thread cp.async staging and TMA bulk-tensor staging alike -- runs
the same arithmetic in the same order, so all shapes must give bit-identical products.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2e-6


@pytest.mark.parametrize("dims", [(6, 12, 6), (10, 20, 10), (30, 60, 30), (17, 40, 23)])
def test_fp32_matvec_forms_match_fp64(dims):
    import algorithmengineering_altproject_b200 as t3d
    P = t3d.Problem(*dims, precision=t3d.T3D_MIXED)
    D = t3d.Problem(*dims, precision=t3d.T3D_MIXED, matvec32_form=t3d.T3D_MATVEC32_DENSE)
    assert P.info().matvec32_modal == 1 and D.info().matvec32_modal == 0
    rng = np.random.default_rng(11)
    for trial in range(2):
        E = rng.uniform(1e-6, 1.0, P.ne)
        if trial == 1:   # design-like field: many elements at Emin
            E = np.where(rng.random(P.ne) < 0.7, 1e-9, 1.0)
        u = rng.standard_normal(P.nf)
        y64 = P.K_times_u_finest(E, u)
        # the FP64 reference of the FP32 operator sees the FP32-rounded inputs
        y64r = P.K_times_u_finest(E.astype(np.float32).astype(np.float64), u.astype(np.float32).astype(np.float64))
        ym = P.K_times_u_finest32(E, u)
        yd = D.K_times_u_finest32(E, u)
        n = np.linalg.norm(y64r)
        assert np.linalg.norm(ym - y64r) <= TOL * n, (trial, np.linalg.norm(ym - y64r) / n)
        assert np.linalg.norm(yd - y64r) <= TOL * n, (trial, np.linalg.norm(yd - y64r) / n)
        assert np.linalg.norm(ym - y64) <= 1e-6 * np.linalg.norm(y64) + TOL * n
    P.close()
    D.close()


def test_modal_form_follows_set_ke():
    import algorithmengineering_altproject_b200 as t3d
    P = t3d.Problem(10, 20, 10, precision=t3d.T3D_MIXED)
    Ke = P.ke()
    rng = np.random.default_rng(5)
    S = rng.standard_normal((24, 24)) * 1e-3
    P.set_ke(Ke + (S + S.T))          # not a cubic-voxel stiffness: the dense FP32 form takes over
    assert P.info().matvec32_modal == 0
    E = rng.uniform(0.1, 1.0, P.ne)
    u = rng.standard_normal(P.nf)
    y64 = P.K_times_u_finest(E.astype(np.float32).astype(np.float64), u.astype(np.float32).astype(np.float64))
    y32 = P.K_times_u_finest32(E, u)
    assert np.linalg.norm(y32 - y64) <= TOL * np.linalg.norm(y64)
    P.set_ke(Ke)
    assert P.info().matvec32_modal == 1
    P.close()


def test_modal_matvec_p_dot_ap_is_deterministic():
    import algorithmengineering_altproject_b200 as t3d
    P = t3d.Problem(30, 60, 30, precision=t3d.T3D_MIXED)
    rng = np.random.default_rng(3)
    E = rng.uniform(1e-3, 1.0, P.ne)
    u = rng.standard_normal(P.nf)
    a = P.K_times_u_finest32(E, u)
    b = P.K_times_u_finest32(E, u)
    np.testing.assert_array_equal(a, b)
    P.close()


@pytest.mark.parametrize("dims", [(6, 12, 6), (30, 60, 30), (17, 40, 23)])
def test_fp32_vcycle_matches_fp64(dims):
    # the FP32 V-cycle (transfers, smoother, FP64 coarsest solve on the FP32 residual) against the FP64 one on
    # the same FP32-rounded residual: ||z32 - z64|| <= 1e-5 ||z64||
    import algorithmengineering_altproject_b200 as t3d
    P = t3d.Problem(*dims, precision=t3d.T3D_MIXED)
    rng = np.random.default_rng(9)
    E = rng.uniform(1e-3, 1.0, P.ne)
    P.make_diagonal_preconditioner_from_static(E)
    r = rng.standard_normal(P.nf).astype(np.float32).astype(np.float64)
    z64 = P.vcycle(r)
    z32 = P.vcycle32(r)
    assert np.linalg.norm(z32 - z64) <= 1e-5 * np.linalg.norm(z64), np.linalg.norm(z32 - z64) / np.linalg.norm(z64)
    P.close()


@pytest.mark.parametrize("dims", [(6, 12, 6), (17, 40, 23), (30, 60, 30)])
def test_every_modal_tile_shape_gives_identical_results(dims):
    import algorithmengineering_altproject_b200 as t3d
    rng = np.random.default_rng(21)
    ref = None
    shapes = []
    for v in range(64):
        try:
            P = t3d.Problem(*dims, precision=t3d.T3D_MIXED, matvec32_tile=v + 1)
        except t3d.T3DError:
            break
        assert P.info().matvec32_variant == v
        shapes.append(tuple(P.info().matvec32_tile))
        if ref is None:
            E = np.where(rng.random(P.ne) < 0.5, 1e-9, rng.uniform(0.01, 1.0, P.ne))
            u = rng.standard_normal(P.nf)
        y = P.K_times_u_finest32(E, u)
        if ref is None:
            ref = y
        np.testing.assert_array_equal(y, ref, err_msg="tile shape %d %s" % (v, shapes[-1]))
        P.close()
    assert len(shapes) >= 6 and any(s[3] == 2 for s in shapes), shapes   # the TMA-staged shapes are among them


@pytest.mark.parametrize("dims", [(17, 40, 23), (30, 60, 30)])
def test_every_tma_tile_shape_gives_the_same_standard_vcycle(dims):
    """The Standard V-cycle fuses its level-0 residual and correction into the TMA-staged K(E)u (epilogue modes
    1 and 2): every TMA shape gives the same z bit for bit."""
    import algorithmengineering_altproject_b200 as t3d
    rng = np.random.default_rng(5)
    ref, seen = None, 0
    for v in range(64):
        try:
            P = t3d.Problem(*dims, precision=t3d.T3D_MIXED, mg_vcycle=t3d.T3D_VCYCLE_STANDARD, matvec32_tile=v + 1)
        except t3d.T3DError:
            break
        if P.info().matvec32_tile[3] < 2:
            P.close()
            continue
        if ref is None:
            E = np.where(rng.random(P.ne) < 0.5, 1e-9, rng.uniform(0.01, 1.0, P.ne))
            r = rng.standard_normal(P.nf)
        P.make_diagonal_preconditioner_from_static(E)
        z = P.vcycle32(r)
        if ref is None:
            ref = z
        np.testing.assert_array_equal(z, ref, err_msg="tile shape %d" % v)
        seen += 1
        P.close()
    assert seen >= 4
