"""Continuous-batching design server on one GPU.

Requests (grid dims, volume fraction, load case, passive voids, OC iteration count; or a TopVoxel design
domain, `DesignRequest.from_topvoxel`) are admitted in arrival order as soon as a slot and the HBM budget
allow: each admitted request gets its own device context (model, MG hierarchy, density, warm-start
displacement and filter state stay resident for all its OC iterations).  With the batched engine (the
default of the command line) an admitted request is initialised on a worker thread and then joins the
one t3d batch that steps every request in flight together -- each kernel of the inner PCG iteration one
launch for all of them -- leaving it when its iterations are done; with the streams engine each request
runs its own loop on its own stream and the kernels of all admitted requests overlap on the device.  The projected footprint of a
request is bytes-per-node (learned from the contexts created so far, per precision) times its padded
node count, with a margin; a request that alone exceeds the budget is rejected.

The reference has no batching or serving (its driver runs one cuboid design per process,
driver.cpp:23-280); this module is the request loop around the same design iteration.

    python -m algorithmengineering_altproject_b200.serve --rate 2 --requests 24 --iters 10
"""
from __future__ import annotations

import argparse
import json
import math
import os
import threading
import time
from concurrent.futures import Future

import numpy as np

# Load every kernel of the library when the CUDA context is created instead of at first launch: many
# request threads start at once, and their first launches should not race the module loader.
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")

from . import (T3D_BATCH_TILE, T3D_COARSE_FULL, T3D_FP64, T3D_MIXED, T3D_SUM_FP64, Batch, Problem,  # noqa: E402
               ProblemSpec, T3DError, topvoxel_info)

# bytes per padded grid node of a context, before the first context of a precision is measured
DEFAULT_BYTES_PER_NODE = {T3D_FP64: 900.0, T3D_MIXED: 1100.0}
MARGIN = 1.15


def padded_dims(nelx, nely, nelz, solid=None):
    """The reference's padded grid (padding.hpp:23-53): L = number of times the solid voxel count (the whole
    cuboid unless `solid` is given, as for a TopVoxel domain, TOP3D_XL.m:1765-1774), while at least 50,000, is
    divided by 8 (rounding to nearest), at least 3; each side rounded up to a multiple of 2^L."""
    nvox, L = (nelx * nely * nelz if solid is None else solid), 0
    while nvox >= 50000:
        L += 1
        nvox = (nvox + 4) // 8
    step = 1 << max(L, 3)
    return tuple((n + step - 1) // step * step for n in (nelx, nely, nelz))


class DesignRequest:
    def __init__(self, nely, nelx, nelz, V0, load_case=0, voids=(), iters=40, rid=None, keep_density=False):
        self.nely, self.nelx, self.nelz = int(nely), int(nelx), int(nelz)
        self.V0 = float(V0)
        self.load_case = int(load_case)
        self.voids = [tuple(float(x) for x in v) for v in voids]
        self.iters = int(iters)
        self.rid = rid
        self.keep_density = keep_density
        self.arrival = None
        self.topvoxel = None        # path of a TopVoxel design domain (replaces dims, load case and voids)
        self.load_cases = 1
        self.solid = None           # solid voxels of a TopVoxel domain (they set its padding)

    @classmethod
    def from_topvoxel(cls, path, V0, iters=40, rid=None, keep_density=False):
        """A request for an external design domain (TopVoxel file); its size is read without a device."""
        info = topvoxel_info(path)
        req = cls(info["nely"], info["nelx"], info["nelz"], V0, iters=iters, rid=rid, keep_density=keep_density)
        req.topvoxel = str(path)
        req.load_cases = 1 + info["additional_load_cases"]
        req.solid = info["solid"]
        return req

    def padded_nodes(self):
        nx, ny, nz = padded_dims(self.nelx, self.nely, self.nelz, self.solid)
        return (nx + 1) * (ny + 1) * (nz + 1)

    def spec(self):
        return ProblemSpec.make(self.load_case, self.voids)

    def as_dict(self):
        d = {"rid": self.rid, "dims": [self.nely, self.nelx, self.nelz], "V0": self.V0,
             "load_case": self.load_case, "voids": len(self.voids), "iters": self.iters}
        if self.topvoxel:
            d.update(topvoxel=self.topvoxel, load_cases=self.load_cases)
        return d


class DesignResult:
    def __init__(self, req):
        self.request = req
        self.c_solid = None
        self.objectives = []
        self.pcg_iters = []
        self.density = None
        self.error = None
        self.admitted = None
        self.finished = None

    @property
    def latency(self):
        return self.finished - self.request.arrival


class DesignServer:
    """Admits DesignRequests against an HBM budget and runs them concurrently on one GPU."""

    def __init__(self, device=0, hbm_budget=160e9, max_active=8, precision=T3D_MIXED, engine="streams", **params):
        """engine "streams": every admitted request runs its own design loop on its own context and stream;
        "batched" (mixed precision): admitted requests are initialised alone, then join one t3d batch that
        steps all of them together -- one launch per kernel of the inner PCG iteration for every request in
        flight -- and leave it when their iterations are done (requests with several load cases, which the
        batch does not take, run alone)."""
        if engine not in ("streams", "batched"):
            raise ValueError("engine must be 'streams' or 'batched'")
        if engine == "batched" and precision != T3D_MIXED:
            raise ValueError("the batched engine runs the mixed-precision form")
        self.device = device
        self.budget = float(hbm_budget)
        self.max_active = int(max_active)
        self.precision = precision
        self.engine = engine
        self.params = dict(params)
        if engine == "batched":
            self.params["matvec32_tile"] = T3D_BATCH_TILE
        # arbitrary request grids: the full Galerkin coarsest operator (the reference's corner-sub-block
        # assembly is kept only for its own cantilever, where it is the parity target)
        self.params.setdefault("mg_coarse_assembly", T3D_COARSE_FULL)
        self._cv = threading.Condition()
        self._queue = []            # (request, future) in arrival order
        self._active = 0
        self._reserved = 0.0
        self._bpn = dict(DEFAULT_BYTES_PER_NODE)
        self._closed = False
        self._threads = []
        self._create_lock = threading.Lock()   # context creation (allocations, tile autotuning) one at a time
        # first solves one at a time: run concurrently they occasionally gave one context a zero solid-domain
        # compliance (cause not found); their design iterations still overlap
        self._init_lock = threading.Lock()
        self._warm = False
        self._joining = []          # batched engine: initialised requests waiting to join the batch
        self._engine_closed = False
        self._engine_thread = None
        if engine == "batched":
            self._engine_thread = threading.Thread(target=self._engine, daemon=True)
            self._engine_thread.start()
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._dispatcher.start()

    # ---- public API
    def submit(self, req: DesignRequest) -> Future:
        fut = Future()
        req.arrival = time.perf_counter() if req.arrival is None else req.arrival
        if self.projected_bytes(req) > self.budget:
            res = DesignResult(req)
            res.error = "projected footprint %.3g B exceeds the HBM budget" % self.projected_bytes(req)
            res.finished = time.perf_counter()
            fut.set_result(res)
            return fut
        with self._cv:
            self._queue.append((req, fut))
            self._cv.notify_all()
        return fut

    def projected_bytes(self, req):
        # several load cases keep a load and a displacement (3 doubles each) per node per case
        extra = 48.0 * req.load_cases if req.load_cases > 1 else 0.0
        return MARGIN * (self._bpn[self.precision] + extra) * req.padded_nodes()

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        self._dispatcher.join()
        for t in self._threads:
            t.join()
        if self._engine_thread is not None:   # after the workers: every request has joined the batch or ended
            with self._cv:
                self._engine_closed = True
                self._cv.notify_all()
            self._engine_thread.join()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- internals
    def _warm_up(self):
        """One small design before the first admission, so that every kernel and the tile autotuner have run
        once before request threads overlap."""
        try:
            self._execute(DesignRequest(8, 16, 8, 0.2, load_case=1, voids=[(8.0, 4.0, 4.0, 2.0, 2.0, 2.0)], iters=1),
                          DesignResult(None))
        except T3DError:
            pass
        self._warm = True

    def _dispatch(self):
        if not self._warm:
            self._warm_up()
        while True:
            with self._cv:
                while True:
                    if self._queue:
                        req, fut = self._queue[0]
                        need = self.projected_bytes(req)
                        if self._active < self.max_active and self._reserved + need <= self.budget:
                            self._queue.pop(0)
                            self._active += 1
                            self._reserved += need
                            break
                    elif self._closed:
                        return
                    self._cv.wait()
            t = threading.Thread(target=self._run, args=(req, fut, need), daemon=True)
            self._threads.append(t)
            t.start()

    def _run(self, req, fut, need):
        res = DesignResult(req)
        res.admitted = time.perf_counter()
        try:
            if self.engine == "batched" and getattr(req, "load_cases", 1) == 1 and req.iters > 0:
                P = self._create(req)
                try:
                    with self._init_lock:
                        res.c_solid = P.design_init(req.V0)
                except BaseException:
                    P.close()
                    raise
                with self._cv:                     # the engine steps it from here on and finishes the request
                    self._joining.append((P, req, res, fut, need))
                    self._cv.notify_all()
                return
            self._execute(req, res)
        except T3DError as e:
            res.error = str(e)
        except Exception as e:   # any other failure is reported on the request, never lost in the worker
            res.error = "%s: %s" % (type(e).__name__, e)
        self._finish(res, fut, need)

    def _finish(self, res, fut, need):
        res.finished = time.perf_counter()
        with self._cv:
            self._active -= 1
            self._reserved -= need
            self._cv.notify_all()
        fut.set_result(res)

    def _engine(self):
        """The batched engine: requests initialised on their worker threads are submitted to one t3d batch,
        where each advances on its own (host thread and stream) and only the inner PCG solves share the
        batched launches; finished ones come back through collect()."""
        B = Batch.open(self.device)
        live = {}                                  # problem handle -> (request, result, future, need)
        try:
            while True:
                with self._cv:
                    joining, self._joining = self._joining, []
                    closing = self._engine_closed
                for P, req, res, fut, need in joining:
                    try:
                        B.submit(P, req.iters)
                        live[P._h.value] = (req, res, fut, need)
                    except T3DError as e:
                        P.close()
                        res.error = str(e)
                        self._finish(res, fut, need)
                if not live:
                    if closing and not joining:
                        return
                    with self._cv:
                        self._cv.wait_for(lambda: self._joining or self._engine_closed, timeout=0.5)
                    continue
                got = B.collect(50)
                if got is None:
                    continue
                P, recs, err = got
                req, res, fut, need = live.pop(P._h.value)
                res.objectives = [r["obj"] for r in recs]
                res.pcg_iters = [r["pcg_iters"] for r in recs]
                res.error = err
                if req.keep_density and err is None:
                    res.density = P.density()
                P.close()
                self._finish(res, fut, need)
        finally:
            B.close()

    def _create(self, req):
        kw = dict(device=self.device, precision=self.precision, oc_sum_order=T3D_SUM_FP64, **self.params)
        with self._create_lock:
            if getattr(req, "topvoxel", None):
                P = Problem.from_topvoxel(req.topvoxel, **kw)
            else:
                P = Problem(req.nely, req.nelx, req.nelz, problem=req.spec(), **kw)
        with self._cv:   # learn the footprint per node from the real allocation (single-case problems)
            if getattr(req, "load_cases", 1) == 1:
                self._bpn[self.precision] = max(self._bpn[self.precision], P.device_bytes / P.nn)
        return P

    def _execute(self, req, res):
        """Runs one request to completion on its own context (and stream)."""
        P = self._create(req)
        try:
            with self._init_lock:
                res.c_solid = P.design_init(req.V0)
            for _ in range(req.iters):
                r = P.design_step()
                res.objectives.append(r["obj"])
                res.pcg_iters.append(r["pcg_iters"])
            if req.keep_density:
                res.density = P.density()
        finally:
            P.close()


# ---------------------------------------------------------------- workload generators
def _round8(v):
    return max(8, int(round(v / 8.0)) * 8)


def draw_instance(rng, nelx=None, iters=40):
    """One instance drawn as in the batched workload: nelx a multiple of 8 in [32, 192]; nely, nelz =
    nelx/2 scaled by U(0.5, 1.0), multiples of 8; V0 ~ U(0.06, 0.30); load case uniform over the three;
    0-3 void ellipsoids with radii 10-25 % of the shortest side at uniform centres."""
    if nelx is None:
        nelx = int(rng.integers(4, 25)) * 8
    nely = _round8(nelx / 2 * rng.uniform(0.5, 1.0))
    nelz = _round8(nelx / 2 * rng.uniform(0.5, 1.0))
    short = min(nelx, nely, nelz)
    voids = []
    for _ in range(int(rng.integers(0, 4))):
        r = [short * rng.uniform(0.10, 0.25) for _ in range(3)]
        c = [rng.uniform(0, nelx), rng.uniform(0, nely), rng.uniform(0, nelz)]
        voids.append(tuple(c + r))
    return DesignRequest(nely, nelx, nelz, rng.uniform(0.06, 0.30), int(rng.integers(0, 3)), voids, iters)


def draw_served(rng, iters=40, median=0.5e6, lo=30e3, hi=16e6):
    """A served request: element count lognormal (median 0.5M, clipped to [30k, 16M]); shape, V0, load
    case and voids as draw_instance."""
    ne = float(np.clip(rng.lognormal(math.log(median), 1.0), lo, hi))
    ay, az = rng.uniform(0.5, 1.0), rng.uniform(0.5, 1.0)
    nelx = _round8((ne / (0.25 * ay * az)) ** (1.0 / 3.0))
    req = draw_instance(rng, nelx=nelx, iters=iters)
    return req


def percentile(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def run_poisson(server, rng, rate, n, iters, median=0.5e6, hi=16e6):
    """Submits n served requests with Poisson arrivals at `rate` per second; returns the results."""
    futs = []
    t0 = time.perf_counter()
    t_next = t0
    for k in range(n):
        req = draw_served(rng, iters=iters, median=median, hi=hi)
        req.rid = k
        now = time.perf_counter()
        if t_next > now:
            time.sleep(t_next - now)
        req.arrival = time.perf_counter()
        futs.append(server.submit(req))
        t_next += rng.exponential(1.0 / rate)
    results = [f.result() for f in futs]
    return results, time.perf_counter() - t0


def summary(results, wall):
    ok = [r for r in results if r.error is None]
    lat = [r.latency for r in ok]
    return {"requests": len(results), "completed": len(ok), "errors": [r.error for r in results if r.error],
            "designs_per_s": len(ok) / wall if wall > 0 else None, "wall_s": wall,
            "latency_s": {"p50": percentile(lat, 50), "p95": percentile(lat, 95), "p99": percentile(lat, 99)}}


def run_batch(server, rng, n, iters):
    """The batched workload: n seed-drawn instances (draw_instance) all submitted at once."""
    reqs = [draw_instance(rng, iters=iters) for _ in range(n)]
    t0 = time.perf_counter()
    for k, q in enumerate(reqs):
        q.rid = k
        q.arrival = t0
    futs = [server.submit(q) for q in reqs]
    results = [f.result() for f in futs]
    return results, time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=0, help="submit this many seed-drawn instances at once instead")
    ap.add_argument("--rate", type=float, default=2.0)
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--max-active", type=int, default=8)
    ap.add_argument("--budget-gb", type=float, default=160.0)
    ap.add_argument("--median", type=float, default=0.5e6)
    ap.add_argument("--max-elements", type=float, default=16e6)
    ap.add_argument("--seed", type=int, default=20251203)
    ap.add_argument("--sequential-fp64", action="store_true", help="also run the same requests one at a time in FP64")
    ap.add_argument("--engine", default="batched", choices=["batched", "streams"],
                    help="batched: requests in flight stepped together in one t3d batch; streams: one context and "
                         "stream per request")
    a = ap.parse_args()
    def workload(srv):
        rng = np.random.default_rng(a.seed)
        if a.batch:
            return run_batch(srv, rng, a.batch, a.iters)
        return run_poisson(srv, rng, a.rate, a.requests, a.iters, a.median, a.max_elements)

    with DesignServer(hbm_budget=a.budget_gb * 1e9, max_active=a.max_active, precision=T3D_MIXED,
                      engine=a.engine) as srv:
        res, wall = workload(srv)
    out = {"mode": ("batch of %d instances" % a.batch) if a.batch else "Poisson arrivals", "engine": a.engine,
           "precision": "mixed", "rate_per_s": None if a.batch else a.rate, "iters": a.iters,
           "max_active": a.max_active, "budget_gb": a.budget_gb, **summary(res, wall)}
    if a.sequential_fp64:
        with DesignServer(hbm_budget=a.budget_gb * 1e9, max_active=1, precision=T3D_FP64) as srv:
            res2, wall2 = workload(srv)
        out["sequential_fp64"] = summary(res2, wall2)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
