"""Admission logic of the design server, on the CPU: requests are admitted in arrival order while a
slot and the HBM budget allow, never more at once than either limit, and a request that alone exceeds
the budget is rejected.  The device work is replaced by a timed sleep (the GPU path is covered by
tests/test_gpu_serve.py)."""
import threading
import time

import algorithmengineering_altproject_b200.serve as serve


class FakeServer(serve.DesignServer):
    def __init__(self, *a, **kw):
        self.log = []
        self.peak_active = 0
        self.peak_bytes = 0.0
        self._lk = threading.Lock()
        super().__init__(*a, **kw)

    def _warm_up(self):
        self._warm = True

    def _execute(self, req, res):
        with self._lk:
            self.log.append(req.rid)
            self.peak_active = max(self.peak_active, self._active)
            self.peak_bytes = max(self.peak_bytes, self._reserved)
        time.sleep(0.05)
        res.objectives = [float(req.rid)]


def test_admission_respects_slots_budget_and_order():
    reqs = [serve.DesignRequest(8, 16, 8, 0.1, rid=k, iters=1) for k in range(12)]
    one = FakeServer(hbm_budget=1e18).projected_bytes(reqs[0])
    srv = FakeServer(hbm_budget=3.5 * one, max_active=8)   # the budget, not the slots, limits to 3
    futs = [srv.submit(r) for r in reqs]
    res = [f.result() for f in futs]
    srv.close()
    assert [r.objectives[0] for r in res] == list(range(12))
    assert srv.log == list(range(12))            # admitted in arrival order
    assert srv.peak_active <= 3 and srv.peak_bytes <= 3.5 * one
    assert all(r.latency >= 0.05 for r in res)


def test_slots_limit_and_oversized_rejection():
    srv = FakeServer(hbm_budget=1e18, max_active=2)
    futs = [srv.submit(serve.DesignRequest(8, 16, 8, 0.1, rid=k, iters=1)) for k in range(6)]
    [f.result() for f in futs]
    assert srv.peak_active <= 2
    srv.close()
    small = FakeServer(hbm_budget=1e6, max_active=2)
    r = small.submit(serve.DesignRequest(64, 128, 64, 0.1, rid=0)).result()
    small.close()
    assert r.error and "budget" in r.error


def test_workload_generators_follow_the_batched_distributions():
    import numpy as np
    rng = np.random.default_rng(20251203)
    for _ in range(200):
        q = serve.draw_instance(rng)
        assert q.nelx % 8 == 0 and q.nely % 8 == 0 and q.nelz % 8 == 0
        assert 32 <= q.nelx <= 192 and 0.06 <= q.V0 <= 0.30 and q.load_case in (0, 1, 2)
        assert len(q.voids) <= 3
        short = min(q.nelx, q.nely, q.nelz)
        assert all(0.10 * short <= v[3 + d] <= 0.25 * short for v in q.voids for d in range(3))
    for _ in range(200):
        q = serve.draw_served(rng)
        ne = q.nelx * q.nely * q.nelz
        assert 8 * 8 * 8 <= ne <= 2.2 * 16e6


def test_topvoxel_requests_are_sized_from_the_file(tmp_path):
    from algorithmengineering_altproject_b200.topvoxel import write_topvoxel
    solid = [(x, y, z) for z in range(6) for x in range(10) for y in range(4)]
    fix = [(0, y, z, 1, 1, 1) for z in range(7) for y in range(5)]
    loads = [(10, y, 0, 0.0, 0.0, -0.2) for y in range(5)]
    one, two = str(tmp_path / "one.TopVoxel"), str(tmp_path / "two.TopVoxel")
    write_topvoxel(one, 10, 4, 6, solid, fixations=fix, loads=loads)
    write_topvoxel(two, 10, 4, 6, solid, fixations=fix, loads=loads, extra_load_cases=[loads])
    a = serve.DesignRequest.from_topvoxel(one, 0.3, rid=0)
    b = serve.DesignRequest.from_topvoxel(two, 0.3, rid=1)
    assert (a.nely, a.nelx, a.nelz, a.load_cases, b.load_cases) == (4, 10, 6, 1, 2)
    assert a.as_dict()["topvoxel"] == one and b.as_dict()["load_cases"] == 2
    srv = FakeServer(hbm_budget=1e18)
    assert srv.projected_bytes(b) > srv.projected_bytes(a) == srv.projected_bytes(serve.DesignRequest(4, 10, 6, 0.3))
    futs = [srv.submit(r) for r in (a, b)]
    [f.result() for f in futs]
    srv.close()
    assert srv.log == [0, 1]


def test_projection_uses_the_reference_padding():
    """Admission sizes a request by the padded grid of padding.hpp:23-53, not by its raw sides: sides that are
    not multiples of 2^L grow, and grids of 25.6M voxels or more pad to multiples of 16 (L = 4)."""
    assert serve.padded_dims(60, 30, 30) == (64, 32, 32)          # the reference CLI demo's grid
    assert serve.padded_dims(10, 4, 6) == (16, 8, 8)
    assert serve.padded_dims(512, 256, 256) == (512, 256, 256)
    assert serve.padded_dims(500, 250, 250) == (512, 256, 256)    # L = 4: multiples of 16
    assert serve.padded_dims(200, 100, 100) == (200, 104, 104)    # 2.0M voxels: L = 3
    assert serve.padded_dims(292, 300, 300) == (304, 304, 304)    # 26M voxels: L = 4, multiples of 16
    assert serve.padded_dims(292, 300, 300, solid=20_000_000) == (296, 304, 304)   # L = 3 from the solid count
    r = serve.DesignRequest(4, 10, 6, 0.3)
    assert r.padded_nodes() == 17 * 9 * 9


def test_unexpected_failures_are_reported_on_the_request():
    class Failing(FakeServer):
        def _execute(self, req, res):
            raise ValueError("boom %s" % req.rid)
    srv = Failing(hbm_budget=1e18)
    r = srv.submit(serve.DesignRequest(8, 16, 8, 0.1, rid=7)).result()
    srv.close()
    assert r.error == "ValueError: boom 7"
