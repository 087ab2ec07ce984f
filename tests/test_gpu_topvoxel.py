"""External design domains from TopVoxel files (TOP3D_XL.m:458-586) on the GPU.

* The reference cantilever written as a TopVoxel file (full cuboid, x = 0 face fixed, tip-line load,
  fea.cpp:374-403) must give exactly the built-in problem: same free DOFs, element order and load, and a
  bit-identical design trajectory (FP64 form; the mixed form is compared the same way).
* An L-shaped domain with passive elements, its own fixations and a load vector: the element set, free
  DOFs and load match a numpy restatement of the file's meaning (file node (x, y, z) is reference node
  (x, y, z); the operator is checked against the element-by-element assembly of the problem-spec tests),
  passive elements stay at density 1 after every OC update (TOP3D_XL.m:152,166) and count in the volume.
* Several load cases (TOP3D_XL.m:105,125,605-621): each solved from its own previous displacement, the
  element compliance averaged.  Two identical cases must reproduce the single-case design bit for bit
  (weights 1/2 are exact) with twice the PCG iterations; two different cases give the mean of the
  single-case solid compliances.
* The whole design loop on an external domain with passive elements and two load cases matches the
  oracle's restatement (oracle/t3d_oracle.c, external-model path) bit for bit: solid compliance, every
  iteration's objective, PCG count and change, and the final densities.
  A variant whose fixation list also fixes loaded nodes (of either load case) checks the MATLAB rule that a
  loaded node loses its fixation (FEA_ApplyBoundaryCondition, TOP3D_XL.m:1326-1331) on both sides.
* Files the design loop cannot run are refused: no fixation, no load.
"""
import numpy as np
import pytest

from test_gpu_problems import numpy_matvec

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.int64 if np.asarray(a).dtype == np.float64 else np.int32)


@pytest.mark.parametrize("dims", [(6, 12, 6), (9, 20, 7)])
@pytest.mark.parametrize("precision", [0, 1])
def test_cantilever_file_reproduces_the_builtin_problem(tmp_path, dims, precision):
    import algorithmengineering_altproject_b200 as t3d
    from algorithmengineering_altproject_b200.topvoxel import cantilever_topvoxel
    kw = dict(precision=precision, oc_sum_order=t3d.T3D_SUM_FP64)
    P = t3d.Problem(*dims, **kw)
    path = str(tmp_path / "c.TopVoxel")
    cantilever_topvoxel(path, *dims, P.res)
    Q = t3d.Problem.from_topvoxel(path, **kw)
    assert Q.res == P.res and Q.ne == P.ne and Q.nf == P.nf
    np.testing.assert_array_equal(Q.free_dofs(), P.free_dofs())
    np.testing.assert_array_equal(Q.ele_map_back(), P.ele_map_back())
    np.testing.assert_array_equal(bits(Q.bfree()), bits(P.bfree()))
    assert Q.design_init(0.2) == P.design_init(0.2)
    for _ in range(2):
        rq, rp = Q.design_step(), P.design_step()
        assert rq["obj"] == rp["obj"] and rq["vol"] == rp["vol"] and rq["pcg_iters"] == rp["pcg_iters"]
    np.testing.assert_array_equal(Q.density(), P.density())
    P.close()
    Q.close()


def l_domain(nelx, nely, nelz):
    solid = [(x, y, z) for z in range(nelz) for x in range(nelx) for y in range(nely)
             if not (x >= nelx // 2 and z >= nelz // 2)]
    passive = [(x, y, 0) for x in range(nelx - 2, nelx) for y in range(nely)]            # a pad under the load
    fix = [(0, y, z, 1, 1, 1) for z in range(nelz + 1) for y in range(nely + 1)]
    fix += [(nelx // 2, y, nelz, 0, 0, 1) for y in range(nely + 1)]                      # a roller line on top
    rng = np.random.default_rng(3)
    loads = [(nelx, y, 0, 0.0, rng.uniform(-0.1, 0.1), -1.0 / (nely + 1)) for y in range(nely + 1)]
    return solid, passive, fix, loads


def test_l_domain_with_passive_elements(tmp_path):
    import algorithmengineering_altproject_b200 as t3d
    from algorithmengineering_altproject_b200.topvoxel import write_topvoxel
    nelx, nely, nelz = 12, 6, 8
    solid, passive, fix, loads = l_domain(nelx, nely, nelz)
    path = str(tmp_path / "l.TopVoxel")
    write_topvoxel(path, nelx, nely, nelz, solid, passive=passive, fixations=fix, loads=loads)
    Q = t3d.Problem.from_topvoxel(path, oc_sum_order=t3d.T3D_SUM_FP64, cg_tol=1e-9, cg_max_it=5000)
    nx, ny, nz = Q.res
    assert Q.ne == len(solid)
    # element set in the reference's full index (row + ny*x + ny*nx*z of the padded grid, row = ny-1-y:
    # the reference's grid rows run opposite to the file's y, fea.cpp:222)
    full = np.sort(Q.ele_map_back().astype(np.int64))
    want = np.sort(np.array([(ny - 1 - y) + ny * x + ny * nx * z for x, y, z in solid], dtype=np.int64))
    np.testing.assert_array_equal(full, want)
    # free DOFs and load: file node (x, y, z) is grid node (x, ny - y, z)
    nnx, nny = nx + 1, ny + 1
    NN = nnx * nny * (nz + 1)
    touched = np.zeros(NN, dtype=bool)
    for x, y, z in solid:
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    touched[((z + dz) * nny + (ny - (y + dy))) * nnx + (x + dx)] = True
    fixed = np.repeat(~touched, 3)
    for x, y, z, fx, fy, fz in fix:
        n = (z * nny + (ny - y)) * nnx + x
        fixed[3 * n:3 * n + 3] |= np.array([fx, fy, fz], dtype=bool)
    np.testing.assert_array_equal(Q.free_dofs(), np.flatnonzero(~fixed))
    b = np.zeros(3 * NN)
    for x, y, z, fx, fy, fz in loads:
        n = (z * nny + (ny - y)) * nnx + x
        b[3 * n:3 * n + 3] = (fx, fy, fz)
    np.testing.assert_array_equal(Q.bfree(), b[~fixed])
    # the operator on this element set
    rng = np.random.default_rng(5)
    E = rng.uniform(1e-3, 1.0, Q.ne)
    u = rng.standard_normal(Q.nf)
    ref = numpy_matvec(Q, E, u)
    assert np.linalg.norm(Q.K_times_u_finest(E, u) - ref) <= 1e-13 * np.linalg.norm(ref)
    # design loop: passive elements at 1 after each OC update, volume fraction kept
    emap = Q.ele_map_back().astype(np.int64)
    pas = np.isin(emap, np.array([(ny - 1 - y) + ny * x + ny * nx * z for x, y, z in passive], dtype=np.int64))
    assert pas.sum() == len(passive)
    Q.design_init(0.3)
    for _ in range(3):
        r = Q.design_step()
        x = Q.density()
        assert np.all(x[pas] == 1.0) and np.isfinite(r["obj"]) and r["obj"] > 0
        assert abs(r["vol"] - 0.3) < 1e-3 and abs(x.mean() - 0.3) < 2e-3
    Q.close()


def test_unrunnable_files_are_refused(tmp_path):
    import algorithmengineering_altproject_b200 as t3d
    from algorithmengineering_altproject_b200.topvoxel import write_topvoxel
    solid, passive, fix, loads = l_domain(8, 4, 4)
    cases = {
        "nofix": (dict(fixations=[], loads=loads), t3d.T3D_ERR_INVALID, "singular"),
        "noload": (dict(fixations=fix, loads=[]), t3d.T3D_ERR_INVALID, "no loads"),
    }
    for name, (kw, code, fragment) in cases.items():
        path = str(tmp_path / (name + ".TopVoxel"))
        write_topvoxel(path, 8, 4, 4, solid, **kw)
        with pytest.raises(t3d.T3DError) as e:
            t3d.Problem.from_topvoxel(path)
        assert e.value.code == code and fragment in str(e.value), (name, str(e.value))


def test_identical_load_cases_reproduce_the_single_case(tmp_path):
    import algorithmengineering_altproject_b200 as t3d
    from algorithmengineering_altproject_b200.topvoxel import write_topvoxel
    solid, passive, fix, loads = l_domain(12, 6, 8)
    one, two = str(tmp_path / "one.TopVoxel"), str(tmp_path / "two.TopVoxel")
    write_topvoxel(one, 12, 6, 8, solid, passive=passive, fixations=fix, loads=loads)
    write_topvoxel(two, 12, 6, 8, solid, passive=passive, fixations=fix, loads=loads, extra_load_cases=[loads])
    assert t3d.topvoxel_info(two)["additional_load_cases"] == 1
    kw = dict(oc_sum_order=t3d.T3D_SUM_FP64)
    A, B = t3d.Problem.from_topvoxel(one, **kw), t3d.Problem.from_topvoxel(two, **kw)
    assert A.design_init(0.3) == B.design_init(0.3)
    for _ in range(2):
        ra, rb = A.design_step(), B.design_step()
        assert ra["obj"] == rb["obj"] and rb["pcg_iters"] == 2 * ra["pcg_iters"], (ra, rb)
    np.testing.assert_array_equal(A.density(), B.density())
    np.testing.assert_array_equal(bits(A.bfree()), bits(B.bfree()))   # the context's load is case 1
    A.close()
    B.close()


def test_two_load_cases_average_the_compliance(tmp_path):
    import algorithmengineering_altproject_b200 as t3d
    from algorithmengineering_altproject_b200.topvoxel import write_topvoxel
    nelx, nely, nelz = 12, 6, 8
    solid, passive, fix, loads = l_domain(nelx, nely, nelz)
    side = [(nelx, y, 2, 0.0, 1.0 / (nely + 1), 0.0) for y in range(nely + 1)]   # a lateral case
    paths = [str(tmp_path / n) for n in ("a.TopVoxel", "b.TopVoxel", "ab.TopVoxel")]
    write_topvoxel(paths[0], nelx, nely, nelz, solid, fixations=fix, loads=loads)
    write_topvoxel(paths[1], nelx, nely, nelz, solid, fixations=fix, loads=side)
    write_topvoxel(paths[2], nelx, nely, nelz, solid, fixations=fix, loads=loads, extra_load_cases=[side])
    kw = dict(cg_tol=1e-10, cg_max_it=5000)
    cs = [t3d.Problem.from_topvoxel(p, **kw).design_init(0.3) for p in paths]
    assert abs(cs[2] - 0.5 * (cs[0] + cs[1])) <= 1e-12 * cs[2], cs


@pytest.mark.parametrize("two_cases, fix_loaded", [(False, False), (True, False), (True, True)])
def test_external_design_loop_matches_the_oracle(tmp_path, two_cases, fix_loaded):
    import algorithmengineering_altproject_b200 as t3d
    from algorithmengineering_altproject_b200.topvoxel import write_topvoxel
    from oracle.bindings import Oracle, voxel_model_from_rows
    nelx, nely, nelz = 12, 6, 8
    solid, passive, fix, loads = l_domain(nelx, nely, nelz)
    side = [(nelx, y, 2, 0.0, 1.0 / (nely + 1), 0.0) for y in range(nely + 1)]
    cases = [loads, side] if two_cases else [loads]
    if fix_loaded:   # fixations on a node of each load case: both rows must be dropped
        fix = fix + [(nelx, 1, 0, 1, 1, 1), (nelx, 2, 2, 0, 1, 0)]
    path = str(tmp_path / "l.TopVoxel")
    write_topvoxel(path, nelx, nely, nelz, solid, passive=passive, fixations=fix, loads=loads,
                   extra_load_cases=cases[1:])
    P = t3d.Problem.from_topvoxel(path)
    csg, recg, xg = P.run_global(0.3, 3)
    P.close()
    vm = voxel_model_from_rows(nelx, nely, nelz, solid, passive=passive, fixations=fix, load_cases=cases)
    O = Oracle(nely, nelx, nelz, voxel_model=vm, red_mode=1, pow_mode=0, vol_mode=0, approx_mode=0)
    cso, reco, xo = O.design_loop(0.3, 3)
    assert csg == cso, (csg, cso)
    assert len(recg) == len(reco)
    for a, b in zip(recg, reco):
        assert a["obj"] == b["obj"] and a["pcg_iters"] == b["pcg_iters"] and a["change"] == b["change"], (a, b)
    np.testing.assert_array_equal(xg, xo)
