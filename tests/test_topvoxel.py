"""TopVoxel reader (the MATLAB original's CreateVoxelFEAmodel, TOP3D_XL.m:458-586), parse only, on CPU.

Files are written with `algorithmengineering_altproject_b200.topvoxel`; `t3d_topvoxel_info` parses them
without a device.  Checked: the sizes it reports (solid voxels, passive elements, fixed and loaded nodes
after dropping all-zero fixation rows and duplicate nodes, as MATLAB's unique() does), the optional
density column, further load cases ("Loads: n idx" blocks, idx = 2..K+1), and that every malformed
file is an error with a message, never a crash.
"""
import pytest

import algorithmengineering_altproject_b200 as t3d
from algorithmengineering_altproject_b200.topvoxel import cantilever_topvoxel, write_topvoxel


def test_cantilever_file_sizes(tmp_path):
    p = str(tmp_path / "cantilever.TopVoxel")
    cantilever_topvoxel(p, 6, 12, 6, (16, 8, 8))
    info = t3d.topvoxel_info(p)
    assert info == {"nelx": 12, "nely": 6, "nelz": 6, "solid": 432, "passive": 0, "fixed_nodes": 49,
                    "loaded_nodes": 14, "additional_load_cases": 0}


def test_duplicates_zero_rows_passive_and_extra_cases(tmp_path):
    p = str(tmp_path / "l.TopVoxel")
    solid = [(x, y, z) for z in range(3) for x in range(4) for y in range(2) if not (x >= 2 and z >= 1)]
    fix = [(0, 0, 0, 1, 1, 1), (0, 0, 0, 0, 0, 1), (0, 1, 0, 0, 0, 0), (0, 2, 1, 1, 0, 0)]
    loads = [(4, 0, 0, 0.0, 0.0, -1.0), (4, 0, 0, 5.0, 5.0, 5.0), (4, 2, 0, 0.0, 0.0, -1.0)]
    write_topvoxel(p, 4, 2, 3, solid, passive=[(0, 0, 0), (1, 1, 2)], fixations=fix, loads=loads,
                   extra_load_cases=[[(4, 1, 1, 1.0, 0.0, 0.0)]])
    info = t3d.topvoxel_info(p)
    assert info["solid"] == len(solid) and info["passive"] == 2
    assert info["fixed_nodes"] == 2            # duplicate keeps its first row; the all-zero row fixes nothing
    assert info["loaded_nodes"] == 2
    assert info["additional_load_cases"] == 1


def test_loaded_nodes_lose_their_fixation(tmp_path):
    """FEA_ApplyBoundaryCondition (TOP3D_XL.m:1326-1331) drops, for every load case, the fixation rows of the
    nodes that case loads: a node both fixed and loaded ends up loaded and free."""
    p = str(tmp_path / "fl.TopVoxel")
    solid = [(x, y, z) for z in range(2) for x in range(4) for y in range(2)]
    fix = [(0, y, z, 1, 1, 1) for z in range(3) for y in range(3)] + [(4, 0, 0, 1, 1, 1), (4, 1, 2, 0, 1, 0)]
    loads = [(4, 0, 0, 0.0, 0.0, -1.0), (4, 2, 0, 0.0, 0.0, -1.0)]
    write_topvoxel(p, 4, 2, 2, solid, fixations=fix, loads=loads, extra_load_cases=[[(4, 1, 2, 0.0, 1.0, 0.0)]])
    info = t3d.topvoxel_info(p)
    assert info["fixed_nodes"] == 9            # the x = 0 face only: both loaded nodes lost their rows
    assert info["loaded_nodes"] == 2


def test_density_column_is_read(tmp_path):
    p = tmp_path / "d.TopVoxel"
    p.write_text("# TopVoxel design domain\nVersion: 1.0\nResolution: 2 2 2\nDensity values: 1\n"
                 "Solid voxels: 2\n1 0.5\n8 1e-3\nPassive elements: 0\nFixations: 1\n1 1 1 1\n"
                 "Loads: 1\n27 0 0 -1\nAdditional loads: 0\n")
    assert t3d.topvoxel_info(str(p))["solid"] == 2


GOOD = ("# TopVoxel design domain\nVersion: 1.0\nResolution: 2 2 2\nDensity values: 0\nSolid voxels: 2\n1\n8\n"
        "Passive elements: 1\n8\nFixations: 1\n1 1 1 1\nLoads: 1\n27 0 0 -1\nAdditional loads: 0\n")


@pytest.mark.parametrize("bad, fragment", [
    (GOOD.replace("Version: 1.0", "Version: 2.0"), "version"),
    (GOOD.replace("Resolution:", "Res:"), "Resolution:"),
    (GOOD.replace("Resolution: 2 2 2", "Resolution: 2 0 2"), "resolution"),
    (GOOD.replace("Resolution: 2 2 2", "Resolution: 1048576 1048576 8"), "resolution"),
    (GOOD.replace("Solid voxels: 2\n1\n8", "Solid voxels: 2\n1\n9"), "voxel index"),
    (GOOD.replace("Passive elements: 1\n8", "Passive elements: 1\n2"), "not a solid voxel"),
    (GOOD.replace("Passive elements", "Active elements"), "Passive"),
    (GOOD.replace("Fixations: 1\n1 1 1 1", "Fixations: 1\n28 1 1 1"), "node index"),
    (GOOD.replace("27 0 0 -1", "27 0 x -1"), "bad number"),
    (GOOD.replace("Loads: 1", "Loads: -1"), "negative"),
    (GOOD[: GOOD.index("Loads:")], "end of file"),
    (GOOD.replace("Additional loads: 0", "Additional loads: 1\nLoads: 1 3\n27 0 0 -1"), "load case indices"),
])
def test_malformed_files_are_errors(tmp_path, bad, fragment):
    p = tmp_path / "bad.TopVoxel"
    p.write_text(bad)
    with pytest.raises(t3d.T3DError) as e:
        t3d.topvoxel_info(str(p))
    assert e.value.code == t3d.T3D_ERR_INVALID and fragment in str(e.value), str(e.value)


def test_missing_file_is_an_error(tmp_path):
    with pytest.raises(t3d.T3DError) as e:
        t3d.topvoxel_info(str(tmp_path / "absent.TopVoxel"))
    assert e.value.code == t3d.T3D_ERR_INVALID and "cannot open" in str(e.value)


def test_oracle_voxel_model_reproduces_the_builtin_cantilever():
    # the oracle's external-model path (test infrastructure for the GPU TopVoxel tests) against its own
    # built-in cantilever: same element order, free DOFs, load and a bit-identical design loop
    import numpy as np
    from oracle.bindings import Oracle, voxel_model_from_rows
    nely, nelx, nelz = 6, 12, 6
    kw = dict(red_mode=1, pow_mode=0, vol_mode=0, approx_mode=0)
    A = Oracle(nely, nelx, nelz, **kw)
    nx, ny, nz = A.res
    iz_max = max(1, nz // 6)
    count = (iz_max + 1) * (ny + 1)
    solid = [(x, y, z) for z in range(nelz) for x in range(nelx) for y in range(nely)]
    fix = [(0, y, z, 1, 1, 1) for z in range(nelz + 1) for y in range(nely + 1)]
    loads = [(nelx, y, z, 0.0, 0.0, -1.0 / count) for z in range(min(iz_max, nelz) + 1) for y in range(nely + 1)]
    B = Oracle(nely, nelx, nelz, voxel_model=voxel_model_from_rows(nelx, nely, nelz, solid, fixations=fix,
                                                                   load_cases=[loads]), **kw)
    np.testing.assert_array_equal(A.ele_map_back(), B.ele_map_back())
    np.testing.assert_array_equal(A.free_dofs(), B.free_dofs())
    np.testing.assert_array_equal(A.bfree(), B.bfree())
    ca, ra, xa = A.design_loop(0.12, 2)
    cb, rb, xb = B.design_loop(0.12, 2)
    assert ca == cb and [r["obj"] for r in ra] == [r["obj"] for r in rb]
    np.testing.assert_array_equal(xa, xb)
