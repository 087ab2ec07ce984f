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
