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
