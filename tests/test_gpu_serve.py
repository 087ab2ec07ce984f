"""Continuous batching on the GPU: three design requests (different sizes, load cases and voids) give
the same results when each runs alone and when all three are admitted together and their kernels
overlap on the device.  Stated tolerance: exact equality of every compliance and PCG iteration count
and of the final densities.  Each request has its own context and stream and every kernel is
deterministic for a given grid (the modal tile shape is chosen once per grid size per process), so
the mix changes timing only."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from algorithmengineering_altproject_b200.serve import DesignRequest
    return [DesignRequest(8, 16, 8, 0.12, load_case=0, iters=3, rid=0, keep_density=True),
            DesignRequest(16, 32, 16, 0.2, load_case=1, voids=[(16.0, 8.0, 8.0, 3.0, 3.0, 3.0)], iters=3, rid=1,
                          keep_density=True),
            DesignRequest(16, 24, 8, 0.3, load_case=2, voids=[(6.0, 4.0, 4.0, 2.0, 3.0, 2.0)], iters=3, rid=2,
                          keep_density=True)]


def test_results_alone_equal_results_in_the_mix():
    from algorithmengineering_altproject_b200.serve import DesignServer
    alone = []
    with DesignServer(max_active=1) as srv:
        for req in _requests():
            alone.append(srv.submit(req).result())
    with DesignServer(max_active=3) as srv:
        futs = [srv.submit(req) for req in _requests()]
        mixed = [f.result() for f in futs]
    for a, m in zip(alone, mixed):
        assert a.error is None and m.error is None, (a.error, m.error)
        assert a.c_solid == m.c_solid
        assert a.objectives == m.objectives and a.pcg_iters == m.pcg_iters
        np.testing.assert_array_equal(a.density, m.density)


def test_topvoxel_requests_in_the_mix(tmp_path):
    # an external domain with two load cases served next to built-in requests: same results alone and mixed
    from algorithmengineering_altproject_b200.serve import DesignRequest, DesignServer
    from algorithmengineering_altproject_b200.topvoxel import write_topvoxel
    solid = [(x, y, z) for z in range(8) for x in range(16) for y in range(8) if not (x >= 8 and z >= 4)]
    fix = [(0, y, z, 1, 1, 1) for z in range(9) for y in range(9)]
    down = [(16, y, 0, 0.0, 0.0, -1.0 / 9) for y in range(9)]
    side = [(16, y, 2, 0.0, 1.0 / 9, 0.0) for y in range(9)]
    path = str(tmp_path / "l.TopVoxel")
    write_topvoxel(path, 16, 8, 8, solid, passive=[(15, y, 0) for y in range(8)], fixations=fix, loads=down,
                   extra_load_cases=[side])

    def reqs():
        return [DesignRequest.from_topvoxel(path, 0.3, iters=3, rid="tv", keep_density=True)] + _requests()[:2]

    with DesignServer(max_active=1) as srv:
        alone = [srv.submit(r).result() for r in reqs()]
    with DesignServer(max_active=3) as srv:
        futs = [srv.submit(r) for r in reqs()]
        mixed = [f.result() for f in futs]
    for a, m in zip(alone, mixed):
        assert a.error is None and m.error is None, (a.error, m.error)
        assert a.c_solid == m.c_solid and a.objectives == m.objectives and a.pcg_iters == m.pcg_iters
        np.testing.assert_array_equal(a.density, m.density)
    assert len(alone[0].objectives) == 3 and all(np.isfinite(alone[0].objectives))


def test_batched_engine_results_equal_results_alone():
    """The batched engine (requests initialised alone, then stepped together in one t3d batch, joining and
    leaving between design iterations): every request's results equal its run alone with the batch's tile
    shape, exactly.  A two-load-case TopVoxel request, which the batch does not take, runs beside it alone."""
    from algorithmengineering_altproject_b200 import T3D_BATCH_TILE
    from algorithmengineering_altproject_b200.serve import DesignRequest, DesignServer

    def reqs():
        r = _requests()
        r[0].iters, r[2].iters = 5, 2     # leave the batch at different steps
        r.append(DesignRequest(8, 32, 8, 0.15, load_case=2, iters=4, rid=3, keep_density=True))
        return r

    with DesignServer(max_active=1, matvec32_tile=T3D_BATCH_TILE) as srv:
        alone = [srv.submit(r).result() for r in reqs()]
    with DesignServer(max_active=4, engine="batched") as srv:
        futs = [srv.submit(r) for r in reqs()]
        mixed = [f.result() for f in futs]
    for a, m in zip(alone, mixed):
        assert a.error is None and m.error is None, (a.error, m.error)
        assert a.c_solid == m.c_solid
        assert a.objectives == m.objectives and a.pcg_iters == m.pcg_iters
        assert len(m.objectives) == m.request.iters
        np.testing.assert_array_equal(a.density, m.density)
