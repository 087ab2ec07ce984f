"""Mixed-precision design loop (precision T3D_MIXED): FP32 inner MG-preconditioned PCG inside an
FP64 defect-correction loop on the true residual.

The FP32 form is not bit-comparable with the FP64 oracle, so its checks are:
  * solved to a tight tolerance, the defect correction reaches the FP64 solution (compliance and
    displacement agree with the plain FP64 form to the tolerances written below);
  * at the reference's defaults (tol 1e-3, 800 iterations) each design iteration, started from the
    FP64 form's density, stays within the distance that the tolerance itself allows;
  * the FP32 kernels are the ones that run (FP32 profile kinds exist only on a mixed context).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(dims, **kw):
    import algorithmengineering_altproject_b200 as t3d
    F = t3d.Problem(*dims, precision=t3d.T3D_FP64, oc_sum_order=t3d.T3D_SUM_FP64, **kw)
    M = t3d.Problem(*dims, precision=t3d.T3D_MIXED, oc_sum_order=t3d.T3D_SUM_FP64, **kw)
    return F, M


@pytest.mark.parametrize("dims", [(6, 12, 6), (30, 60, 30)])
def test_defect_correction_reaches_fp64_solution(dims):
    # |r| < 1e-9 |b| on the true (FP64) residual in both forms
    F, M = _pair(dims, cg_tol=1e-9, cg_max_it=20000)
    csF, csM = F.design_init(0.12), M.design_init(0.12)
    assert abs(csM - csF) <= 1e-8 * abs(csF), (csF, csM)
    uF, uM = F.displacement(), M.displacement()
    assert np.linalg.norm(uM - uF) <= 1e-6 * np.linalg.norm(uF)
    rF, rM = F.design_step(), M.design_step()
    assert rM["pcg_iters"] < 20000 and rF["pcg_iters"] < 20000
    assert abs(rM["obj"] - rF["obj"]) <= 1e-8 * abs(rF["obj"]), (rF["obj"], rM["obj"])
    F.close()
    M.close()


def test_reference_defaults_stay_within_solver_tolerance():
    # 30x60x30 at tol 1e-3: the first solves converge (~430 iterations), later ones hit the 800 cap
    F, M = _pair((30, 60, 30))
    csF, csM = F.design_init(0.12), M.design_init(0.12)
    assert abs(csM - csF) <= 1e-2 * abs(csF)
    for _ in range(3):
        M.set_density(F.density())
        rF, rM = F.design_step(), M.design_step()
        assert abs(rM["obj"] - rF["obj"]) <= 1e-2 * abs(rF["obj"]), (rF, rM)
        assert np.max(np.abs(M.density().astype(np.float64) - F.density())) <= 0.2   # OC move limit
        assert abs(rM["vol"] - rF["vol"]) <= 1e-4
    F.close()
    M.close()


def test_fp32_kernels_run_only_on_mixed_contexts():
    import algorithmengineering_altproject_b200 as t3d
    F, M = _pair((10, 20, 10))
    E = np.full(M.ne, 0.5)
    for P in (F, M):
        P.make_diagonal_preconditioner_from_static(E)
    assert M.profile(t3d.T3D_PROFILE_MATVEC32, 2) > 0
    assert M.profile(t3d.T3D_PROFILE_VCYCLE32, 2) > 0
    with pytest.raises(t3d.T3DError) as e:
        F.profile(t3d.T3D_PROFILE_MATVEC32, 2)
    assert e.value.code == t3d.T3D_ERR_INVALID
    F.close()
    M.close()


def test_mixed_design_loop_is_deterministic():
    F, M = _pair((10, 20, 10))
    _, M2 = _pair((10, 20, 10))
    M.design_init(0.12)
    M2.design_init(0.12)
    for _ in range(3):
        a, b = M.design_step(), M2.design_step()
        assert a["obj"] == b["obj"] and a["pcg_iters"] == b["pcg_iters"]
    np.testing.assert_array_equal(M.density(), M2.density())
    for P in (F, M, M2):
        P.close()


@pytest.mark.parametrize("dims", [(30, 60, 30), (24, 88, 40)])
def test_full_galerkin_coarsest_matches_oracle(dims):
    # T3D_COARSE_FULL samples every fine element of each coarsest element (span = product of the level spans)
    # instead of the reference's corner sub-block; bit-identical to the oracle's restatement of the same assembly
    import algorithmengineering_altproject_b200 as t3d
    from oracle.bindings import Oracle
    P = t3d.Problem(*dims, mg_coarse_assembly=t3d.T3D_COARSE_FULL)
    O = Oracle(*dims, red_mode=1, coarse_full=1)
    rng = np.random.default_rng(6)
    E = rng.uniform(1e-3, 1.0, P.ne)
    assert np.array_equal(P.coarse_matrix(E), O.coarse_matrix(E))
    P.close()


def test_full_galerkin_coarsest_repairs_a_stalling_grid():
    # 24x88x40 (levels 88x24x40 / 22x6x10 / 11x3x5): with the reference's assembly PCG on the solid domain is
    # still at half the initial residual after 800 iterations; with the full Galerkin operator it gets within
    # 1e-2 of the tolerance (oracle: 0.505 vs 0.00146)
    import algorithmengineering_altproject_b200 as t3d
    res = {}
    for mode in (t3d.T3D_COARSE_REFERENCE, t3d.T3D_COARSE_FULL):
        P = t3d.Problem(24, 88, 40, mg_coarse_assembly=mode)
        b = P.bfree()
        E1 = np.ones(P.ne)
        P.make_diagonal_preconditioner_from_static(E1)
        x, its = P.PCG_free(E1, b, np.zeros(P.nf), tol=1e-3, maxIt=800)
        res[mode] = np.linalg.norm(b - P.K_times_u_finest(E1, x)) / np.linalg.norm(b)
        P.close()
    assert res[t3d.T3D_COARSE_FULL] < 1e-2 < 0.1 < res[t3d.T3D_COARSE_REFERENCE], res


def test_fp32_breakdown_stops_the_inner_solve_without_nan():
    # 16x72x24 with the reference's coarsest assembly: the preconditioner is not positive definite and the
    # FP32 recurrence breaks down; the inner solve stops at the breakdown and the FP64 outer loop restarts,
    # so the design iteration stays finite
    import algorithmengineering_altproject_b200 as t3d
    M = t3d.Problem(16, 72, 24, precision=t3d.T3D_MIXED, oc_sum_order=t3d.T3D_SUM_FP64)
    cs = M.design_init(0.2)
    r = M.design_step()
    assert np.isfinite(cs) and np.isfinite(r["obj"])
    M.close()


def test_host_buffer_design_step_matches_the_resident_one():
    # t3d_design_step_host (the design field through host memory, as a caller without device buffers uses
    # it) gives the resident design step's result bit for bit, into a caller-owned output buffer reused
    # across iterations
    import algorithmengineering_altproject_b200 as t3d
    A = t3d.Problem(10, 20, 10, precision=t3d.T3D_MIXED)
    B = t3d.Problem(10, 20, 10, precision=t3d.T3D_MIXED)
    assert A.design_init(0.3) == B.design_init(0.3)
    x, out = A.density(), np.empty(A.ne, dtype=np.float32)
    for _ in range(3):
        xo, ra = A.design_step_host(x, out=out)
        rb = B.design_step()
        assert xo is out
        np.testing.assert_array_equal(out, B.density())
        assert ra["obj"] == rb["obj"] and ra["pcg_iters"] == rb["pcg_iters"], (ra, rb)
        x = out.copy()
    with pytest.raises(ValueError):
        A.design_step_host(x, out=np.empty(A.ne, dtype=np.float64))
    A.close()
    B.close()
