"""Problem specs beyond the reference's cantilever: load cases and passive-void ellipsoids.

The reference has no such cases (its driver builds one cuboid with one tip-line load,
fea.cpp:181-447), so parity here is against restatements written in numpy in this file:
  * the solid element set: an element is absent when its centre lies inside a void ellipsoid;
  * the operator: K(E)u = sum_e E_e Ke u_e over the solid elements, assembled element by element
    from the context's Ke and layouts (free-DOF order, Morton element order), FP64 to 1e-13 and the
    FP32 modal kernel to 2e-6 relative;
  * the loads: totals and torque of each load case on the free DOFs;
  * the design loop runs on each case in both precisions and keeps the volume fraction.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CORNER_D = [(0, 1, 0), (1, 1, 0), (1, 0, 0), (0, 0, 0), (0, 1, 1), (1, 1, 1), (1, 0, 1), (0, 0, 1)]


def solid_elements(nely, nelx, nelz, voids):
    ex, ey, ez = np.meshgrid(np.arange(nelx), np.arange(nely), np.arange(nelz), indexing="ij")
    keep = np.ones(ex.shape, dtype=bool)
    for cx, cy, cz, rx, ry, rz in voids:
        d = ((ex + 0.5 - cx) / rx) ** 2 + ((ey + 0.5 - cy) / ry) ** 2 + ((ez + 0.5 - cz) / rz) ** 2
        keep &= d > 1.0
    return int(keep.sum())


def numpy_matvec(P, E, u_free):
    nx, ny, nz = P.res
    nnx, nny = nx + 1, ny + 1
    NN = (nx + 1) * (ny + 1) * (nz + 1)
    fd = P.free_dofs().astype(np.int64)
    u = np.zeros(3 * NN)
    u[fd] = u_free
    Ke = P.ke()
    y = np.zeros(3 * NN)
    full = P.ele_map_back().astype(np.int64)
    cz, rem = np.divmod(full, nx * ny)
    cx, cy = np.divmod(rem, ny)
    dofs = np.zeros((len(full), 24), dtype=np.int64)
    for a, (dx, dy, dz) in enumerate(CORNER_D):
        n = ((cz + dz) * nny + (cy + dy)) * nnx + (cx + dx)
        for c in range(3):
            dofs[:, 3 * a + c] = 3 * n + c
    ye = (u[dofs] @ Ke.T) * E[:, None]
    np.add.at(y, dofs.ravel(), ye.ravel())
    return y[fd]


VOIDS = [(6.0, 3.0, 3.0, 2.5, 2.0, 2.0)]


@pytest.mark.parametrize("load_case", [0, 1, 2])
def test_void_domain_operator_and_layouts(load_case):
    import algorithmengineering_altproject_b200 as t3d
    dims = (6, 12, 6)
    spec = t3d.ProblemSpec.make(load_case, VOIDS)
    P = t3d.Problem(*dims, problem=spec, precision=t3d.T3D_MIXED)
    assert P.ne == solid_elements(*dims, VOIDS) < 6 * 12 * 6
    assert len(np.unique(P.ele_map_back())) == P.ne
    rng = np.random.default_rng(4)
    E = rng.uniform(1e-3, 1.0, P.ne)
    u = rng.standard_normal(P.nf)
    ref = numpy_matvec(P, E, u)
    y64 = P.K_times_u_finest(E, u)
    assert np.linalg.norm(y64 - ref) <= 1e-13 * np.linalg.norm(ref)
    Er = E.astype(np.float32).astype(np.float64)
    ur = u.astype(np.float32).astype(np.float64)
    y32 = P.K_times_u_finest32(E, u)
    ref32 = numpy_matvec(P, Er, ur)
    assert np.linalg.norm(y32 - ref32) <= 2e-6 * np.linalg.norm(ref32)
    P.close()


def test_load_cases_totals():
    import algorithmengineering_altproject_b200 as t3d
    nely, nelx, nelz = 8, 16, 8
    for lc in (1, 2):
        P = t3d.Problem(nely, nelx, nelz, problem=t3d.ProblemSpec.make(lc))
        nx, ny, nz = P.res
        NN = (nx + 1) * (ny + 1) * (nz + 1)
        fd = P.free_dofs().astype(np.int64)
        b = np.zeros(3 * NN)
        b[fd] = P.bfree()
        fx, fy, fz = b[0::3], b[1::3], b[2::3]
        iz = np.arange(NN) // ((nx + 1) * (ny + 1))
        if lc == 1:   # top traction: the x = 0 column of the top face is fixed, the rest carries -1 in total
            assert abs(fz.sum() + nelx / (nelx + 1)) < 1e-12
            assert np.all(fz[iz != nelz] == 0) and fx.sum() == 0 and fy.sum() == 0
        else:         # torsion couple: zero net force, torque 1 * nelz about x
            assert abs(fy.sum()) < 1e-12 and fz.sum() == 0
            assert abs((fy * iz).sum() - nelz) < 1e-9
        P.close()


@pytest.mark.parametrize("load_case", [0, 1, 2])
def test_design_loop_runs_on_each_case(load_case):
    import algorithmengineering_altproject_b200 as t3d
    spec = t3d.ProblemSpec.make(load_case, VOIDS)
    out = {}
    for prec in (t3d.T3D_FP64, t3d.T3D_MIXED):
        P = t3d.Problem(6, 12, 6, problem=spec, precision=prec, oc_sum_order=t3d.T3D_SUM_FP64,
                        cg_tol=1e-9, cg_max_it=5000)
        cs = P.design_init(0.2)
        recs = [P.design_step() for _ in range(3)]
        assert cs > 0 and all(np.isfinite(r["obj"]) and r["obj"] > 0 for r in recs)
        assert all(abs(r["vol"] - 0.2) < 1e-3 for r in recs)
        out[prec] = (cs, [r["obj"] for r in recs])
        P.close()
    (c64, o64), (c32, o32) = out[t3d.T3D_FP64], out[t3d.T3D_MIXED]
    assert abs(c32 - c64) <= 1e-8 * c64
    assert abs(o32[0] - o64[0]) <= 1e-8 * o64[0]


def test_degenerate_and_oversized_problems_are_errors():
    import algorithmengineering_altproject_b200 as t3d
    with pytest.raises(t3d.T3DError) as e:   # a void that swallows the whole cuboid
        t3d.Problem(6, 12, 6, problem=t3d.ProblemSpec.make(0, [(6.0, 3.0, 3.0, 50.0, 50.0, 50.0)]))
    assert e.value.code == t3d.T3D_ERR_INVALID and "every element" in str(e.value)
    with pytest.raises(t3d.T3DError) as e:   # 3 x nodes beyond 32-bit DOF indices: refused before any allocation
        t3d.Problem(896, 1024, 896)
    assert e.value.code == t3d.T3D_ERR_UNSUPPORTED


def spec_as_voxel_model(P, nely, nelx, nelz, load_case, voids):
    """The problem spec as the oracle's external model: cuboid minus the voids, the x = 0 face fixed, and the
    load case's forces on the reference's nodes (file coordinates: element / node (x, y, z) of the reference,
    y = the reference's row index)."""
    from oracle.bindings import voxel_model_from_rows
    nx, ny, nz = P.res
    solid = [(x, y, z) for z in range(nelz) for x in range(nelx) for y in range(nely)
             if all(((x + 0.5 - cx) / rx) ** 2 + ((y + 0.5 - cy) / ry) ** 2 + ((z + 0.5 - cz) / rz) ** 2 > 1.0
                    for cx, cy, cz, rx, ry, rz in voids)]
    fix = [(0, y, z, 1, 1, 1) for z in range(nelz + 1) for y in range(nely + 1)]
    if load_case == 0:     # tip line: -1/count over the padded grid's rows, z <= max(1, nz // 6)
        iz_max = max(1, nz // 6)
        count = (iz_max + 1) * (ny + 1)
        loads = [(nelx, y, z, 0.0, 0.0, -1.0 / count) for z in range(min(iz_max, nelz) + 1) for y in range(nely + 1)]
    elif load_case == 1:   # top traction on the z = nelz face
        f = -1.0 / ((nelx + 1) * (nely + 1))
        loads = [(x, y, nelz, 0.0, 0.0, f) for x in range(nelx + 1) for y in range(nely + 1)]
    else:                  # torsion couple at x = nelx: +f on the top edge, -f on the bottom edge
        f = 1.0 / (nely + 1)
        loads = [(nelx, y, nelz, 0.0, f, 0.0) for y in range(nely + 1)] + \
                [(nelx, y, 0, 0.0, -f, 0.0) for y in range(nely + 1)]
    return voxel_model_from_rows(nelx, nely, nelz, solid, fixations=fix, load_cases=[loads], loaded_nodes_free=False)


@pytest.mark.parametrize("load_case", [0, 1, 2])
def test_problem_spec_design_loop_matches_the_oracle(load_case):
    # the problem-spec path (load cases, voids) against the oracle's external-model restatement, bit for bit
    import algorithmengineering_altproject_b200 as t3d
    from oracle.bindings import Oracle
    dims = (6, 12, 6)
    P = t3d.Problem(*dims, problem=t3d.ProblemSpec.make(load_case, VOIDS))
    vm = spec_as_voxel_model(P, *dims, load_case, VOIDS)
    O = Oracle(*dims, voxel_model=vm, red_mode=1, pow_mode=0, vol_mode=0, approx_mode=0)
    np.testing.assert_array_equal(P.ele_map_back(), O.ele_map_back())
    np.testing.assert_array_equal(P.free_dofs(), O.free_dofs())
    np.testing.assert_array_equal(P.bfree(), O.bfree())
    csg, recg, xg = P.run_global(0.2, 3)
    P.close()
    cso, reco, xo = O.design_loop(0.2, 3)
    assert csg == cso
    for a, b in zip(recg, reco):
        assert a["obj"] == b["obj"] and a["pcg_iters"] == b["pcg_iters"] and a["change"] == b["change"], (a, b)
    np.testing.assert_array_equal(xg, xo)
