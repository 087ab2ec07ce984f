"""Surface export (io.cpp:80-87 -> voxel_surface.hpp:12-93 -> export_stl.hpp:14-33).

CPU: the oracle's restatement writes the same bytes as the reference's own export_surface_stl (built
from the unmodified sources in oracle/_ref) on random and thresholded density fields, padded grids
included.  GPU (tests/test_gpu_parity.py-style, marked gpu): the device exporter writes the same bytes
as both, on a design produced by the GPU loop.
"""
import os

import numpy as np
import pytest

from oracle.bindings import Oracle


def _bytes(path):
    with open(path, "rb") as f:
        return f.read()


@pytest.mark.parametrize("dims", [(6, 12, 6), (10, 20, 10), (17, 40, 23)])
def test_oracle_stl_matches_reference(tmp_path, ref_or_skip, dims):
    O = Oracle(*dims)
    R = ref_or_skip(*dims)
    rng = np.random.default_rng(3)
    for k, x in enumerate([rng.random(O.ne).astype(np.float32),
                           np.where(rng.random(O.ne) < 0.4, 1.0, 1e-3).astype(np.float32)]):
        po, pr = str(tmp_path / ("o%d.stl" % k)), str(tmp_path / ("r%d.stl" % k))
        n = O.export_stl(x, po, 0.3)
        R.export_stl(x, pr, 0.3)
        bo, br = _bytes(po), _bytes(pr)
        assert len(bo) == 84 + 50 * n and n > 0
        assert bo == br


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(6, 12, 6), (17, 40, 23)])
def test_device_stl_matches_oracle_and_reference(tmp_path, dims):
    import algorithmengineering_altproject_b200 as t3d
    from oracle.bindings import Reference, reference_available
    P = t3d.Problem(*dims)
    P.design_init(0.3)
    for _ in range(2):
        P.design_step()
    x = P.density()
    pg, po = str(tmp_path / "g.stl"), str(tmp_path / "o.stl")
    n = P.export_stl(pg, 0.3)
    assert n == Oracle(*dims).export_stl(x, po, 0.3)
    assert _bytes(pg) == _bytes(po)
    if reference_available():
        pr = str(tmp_path / "r.stl")
        Reference(*dims).export_stl(x, pr, 0.3)
        assert _bytes(pg) == _bytes(pr)
    P.close()
