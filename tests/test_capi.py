"""C-ABI boundary checks that need no GPU: the library builds, loads and exports every entry point
declared in include/t3d_b200.h; the Python binding covers the same set; without a device the
library refuses to run (there is no CPU path)."""
import ctypes as C
import re
import subprocess

import pytest

import algorithmengineering_altproject_b200 as t3d


def header_functions():
    src = open(t3d.HEADER_PATH).read()
    return sorted(set(re.findall(r"\b(t3d_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_operator_api():
    names = header_functions()
    for required in ["t3d_matvec", "t3d_mg_setup", "t3d_vcycle", "t3d_pcg", "t3d_compliance", "t3d_filter_apply",
                     "t3d_oc_update", "t3d_design_step", "t3d_run_global"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = t3d.library()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", t3d.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (t3d_[a-z0-9_]+)", out))
    assert set(header_functions()) <= exported


def test_binding_covers_header():
    assert set(header_functions()) == set(t3d._SIGS)


def test_library_is_built_for_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", t3d.LIB_PATH], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_defaults_match_reference_globalparams():
    p = t3d.default_params()
    assert p.E0 == 1.0 and abs(p.Emin - 1e-6) < 1e-12 and p.penal == 3.0
    assert p.cg_max_it == 800 and abs(p.cg_tol - 1e-3) < 1e-9
    assert p.mg_max_levels == 5 and p.mg_nondyadic == 1 and abs(p.mg_weight - 0.6) < 1e-7
    assert abs(p.filter_rmin - 3 ** 0.5) < 1e-6


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(t3d.T3DError) as e:
        t3d.Problem(6, 12, 6)
    assert e.value.code == t3d.T3D_ERR_NO_DEVICE


@pytest.mark.parametrize("dims", [(0, 12, 6), (6, 0, 6), (6, 12, -1)])
def test_empty_grids_are_rejected_before_any_device_work(dims):
    with pytest.raises(t3d.T3DError) as e:
        t3d.Problem(*dims)
    assert e.value.code == t3d.T3D_ERR_INVALID


@pytest.mark.parametrize("spec,msg", [
    (dict(load_case=3), "load case"),
    (dict(load_case=-1), "load case"),
    (dict(voids=[(1, 1, 1, 0.0, 1, 1)]), "radii"),
    (dict(voids=[(1, 1, 1, 1, 1, 1)] * 4, extra=True), "num_voids"),
])
def test_bad_problem_specs_are_rejected(spec, msg):
    extra = spec.pop("extra", False)
    p = t3d.ProblemSpec.make(**spec)
    if extra:
        p.num_voids = t3d.T3D_MAX_VOIDS + 1
    with pytest.raises(t3d.T3DError) as e:
        t3d.Problem(6, 12, 6, problem=p)
    assert e.value.code == t3d.T3D_ERR_INVALID and msg in str(e.value)


def test_null_arguments_are_errors():
    lib = t3d.library()
    assert lib.t3d_create(6, 12, 6, None, None) == t3d.T3D_ERR_INVALID
    assert lib.t3d_get_info(None, None) == t3d.T3D_ERR_INVALID
    assert lib.t3d_destroy(None) == t3d.T3D_OK


def test_batch_arguments_are_checked_before_any_device_work():
    import ctypes as C
    lib = t3d.library()
    h = C.c_void_p()
    dims = (C.c_int * 3)(8, 16, 8)
    assert lib.t3d_batch_create(0, dims, None, None, C.byref(h)) == t3d.T3D_ERR_INVALID
    assert lib.t3d_batch_create(1, None, None, None, C.byref(h)) == t3d.T3D_ERR_INVALID
    assert lib.t3d_batch_create(1, dims, None, None, None) == t3d.T3D_ERR_INVALID
    assert lib.t3d_batch_design_step(None, None) == t3d.T3D_ERR_INVALID
    assert lib.t3d_batch_info(None, None) == t3d.T3D_ERR_INVALID
    assert lib.t3d_batch_destroy(None) == t3d.T3D_OK
