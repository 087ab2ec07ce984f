"""Benchmark of the B200 design iteration (SIMP -> MG-preconditioned PCG -> compliance ->
sensitivities -> PDE filter -> OC) on the reference's cantilever.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--config c2]
                    [--precision mixed|fp64] [--regime converged|reference] [--compare-steps S]
                    [--kernels-only --reps R --tile T] [--batch N --batch-iters K]

`serving` (N=1, after the timed region) runs the request loop (serve.py) on Poisson arrivals at 0.5 and 8
requests/s and the same requests one at a time in FP64: designs/s and p50/p95/p99 latency.

Prints ONE JSON line (rank 0).  A step is one design iteration of 256x512x256 (101.6M DOF).  The default
form is the mixed-precision one (FP32 inner MG-PCG inside FP64 defect correction) in the "converged"
regime: every solve reaches |r| < 1e-6 |b| with the Standard V-cycle rebuilt every design iteration, so
mixed and FP64 approximate the same solution; `vs_fp64` runs S design iterations of both forms from the
same densities and reports the speed ratio and the compliance / displacement / density errors there, and
`reference_regime` the same for the reference CLI's own solver settings (Adapted cycle, tol 1e-3,
800-iteration cap, which both forms hit at this size).  `value` = design iterations/s over the whole job,
timed on the device (CUDA events recorded by the library on its stream; max over ranks); `e2e` = the same
metric through the host-buffer C-ABI call t3d_design_step_host (H2D of the design field, D2H of the updated
field, between two pinned host buffers, wall clock).  Multi-GPU runs are independent replicas (one design
per GPU, no collective on the data path).

--impl reference times the reference's own CPU implementation (oracle/_ref/libt3d_ref.so, the
unmodified reference sources) on this host's physical cores with a bounded sample of the same workload:
design iterations with PCG capped at 1 and 3 iterations, extrapolated to the 800 iterations its solves
take at this size.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
import warnings

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# workloads: element counts, V0, MG level cap (c2: 101.6M DOF, the headline; c0/c1: smaller parity cases)
CONFIGS = {
    "c0": dict(nely=30, nelx=60, nelz=30, V0=0.12, max_levels=5,
               name="cantilever 30x60x30 (54,000 elements, 172,980 free DOF)"),
    "c1": dict(nely=96, nelx=192, nelz=96, V0=0.12, max_levels=5,
               name="cantilever 96x192x96 (1,769,472 elements, 5,419,584 free DOF)"),
    "c2": dict(nely=256, nelx=512, nelz=256, V0=0.08, max_levels=6,
               name="cantilever 256x512x256 (33,554,432 elements, 101,451,264 free DOF)"),
    # kernel-capture size: vectors above L2, a few GB on the device
    "k1": dict(nely=160, nelx=320, nelz=160, V0=0.08, max_levels=5,
               name="cantilever 160x320x160 (8,192,000 elements)"),
    # DRAM-traffic capture size: FP32 node vectors 273 MB each, 2.2x the 126 MB L2
    "k2": dict(nely=224, nelx=448, nelz=224, V0=0.08, max_levels=6,
               name="cantilever 224x448x224 (22,478,848 elements)"),
}
DEFAULT_CONFIG = "c2"
METRIC = "design iterations/s"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_NOTE = os.path.join(ROOT, "profiles", "matvec_traffic.md")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default=DEFAULT_CONFIG, choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--regime", default="converged", choices=sorted(REGIMES),
                    help="converged: both forms solve to 1e-6 with the Standard V-cycle rebuilt every iteration; "
                         "reference: the reference CLI's Adapted cycle, tol 1e-3, 800-iteration cap")
    ap.add_argument("--compare-steps", type=int, default=5,
                    help="design iterations run by both forms from the same density (mixed vs FP64 errors)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="time the matvec and V-cycle alone on the config's grid (for ncu captures)")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--tile", type=int, default=0,
                    help="modal FP32 K(E)p tile shape: 0 = autotuned, k = shape k-1 (--kernels-only timing)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=8,
                    help="requests per arrival rate in the serving sample (0 = no serving sample)")
    ap.add_argument("--batch", type=int, default=0,
                    help="batched-designs mode: this many seed-drawn instances stepped together (t3d_batch), "
                         "against the same designs run one at a time in mixed precision and in plain FP64")
    ap.add_argument("--batch-iters", type=int, default=10, help="design iterations per instance in --batch mode")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


# ---------------------------------------------------------------- clocks sampling
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", "t3d_clocks_%d_%d.csv" % (os.getpid(), index))

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        busy = [s for s in sm if s > 600] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    try:
        d = json.load(open(MEASURED_PEAKS))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_launch(kernel):
    """dram read+write bytes per full-size launch of `kernel` from the committed ncu summary, if present."""
    try:
        m = re.search(kernel + r"_traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(TRAFFIC_NOTE).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


# ---------------------------------------------------------------- CPU baseline / reference arm
CPU_SAMPLES = 10   # PCG-cost samples in both the reference arm and the cpu_baseline leg


def setup_cpu_env():
    """OpenMP placement of the reference's own runs (run_cubic_test_top3d_GLOBAL.sbatch:54-56): threads bound
    close, one per physical core.  Must be set before the reference library (libgomp) is loaded."""
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")


def physical_cores():
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
    except Exception:
        n = None
    return int(n or os.cpu_count() or 1)


def reference_sample(cfg, samples, n_pcg, threads):
    """Bounded sample of the reference's CPU design iteration (the reference build of oracle/_ref): `samples`
    pairs of design iterations with PCG capped at 1 and 3 iterations give the per-PCG-iteration cost (their
    PCG-time difference / 2), extrapolated to n_pcg PCG iterations per design iteration, plus the measured
    SIMP / compliance / filter / OC time and 1/5 of an MG rebuild (the reference rebuilds at loop 1 and every
    5th, driver.cpp:132).  PCG_free, the MG preconditioner, ComputeCompliance and ApplyPDEFilter are the
    reference's own; SIMP, dc and OC are the harness's restatement of driver.cpp:117-183."""
    from oracle.bindings import Reference, reference_available
    if not reference_available():
        raise RuntimeError("reference build oracle/_ref/libt3d_ref.so is not present")
    Reference.set_threads(threads)
    r = Reference(cfg["nely"], cfg["nelx"], cfg["nelz"], max_levels=cfg["max_levels"])
    V0 = cfg["V0"]
    r.sample_iteration(V0, 1, True)   # warm-up: filter set-up, first MG build
    per_iter, rest = [], []
    for _ in range(samples):
        _, a = r.sample_iteration(V0, 1, False)
        _, b = r.sample_iteration(V0, 3, False)
        per_iter.append((b[2] - a[2]) / 2.0)
        rest.append(b[0] + b[3] + b[4] + b[5])
    _, mg = r.sample_iteration(V0, 1, True)
    t_iter = statistics.median(per_iter)
    t_design = max(t_iter, 0.0) * n_pcg + statistics.median(rest) + mg[1] / 5.0
    spread = {"min": min(per_iter), "median": t_iter, "max": max(per_iter)}
    return dict(value=1.0 / t_design, seconds_per_design_iteration=t_design, pcg_iteration_s=spread,
                kind="reference", cores=threads,
                sample="%d pairs of reference design iterations (%s) with PCG capped at 1 and 3 iterations: "
                       "per-PCG-iteration cost median %.3f s (min %.3f, max %.3f), extrapolated to %d PCG iterations "
                       "(cgMaxIt, core.hpp:36; the reference's Adapted-cycle solves hit it at this size), plus the "
                       "measured SIMP/compliance/filter/OC time and 1/5 of an MG rebuild; OpenMP %d threads on "
                       "physical cores (OMP_PROC_BIND=%s, OMP_PLACES=%s); PCG, MG, compliance and filter are the "
                       "reference's own code, SIMP/dc/OC the harness's restatement of driver.cpp:117-183"
                       % (samples, cfg["name"], t_iter, spread["min"], spread["max"], n_pcg, threads,
                          os.environ.get("OMP_PROC_BIND"), os.environ.get("OMP_PLACES")))


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    setup_cpu_env()
    cfg = CONFIGS[args.config]
    threads = physical_cores()
    n_pcg = 800   # cgMaxIt (core.hpp:36): the reference's solves hit the cap at these sizes
    t0 = time.time()
    s = reference_sample(cfg, CPU_SAMPLES, n_pcg, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": s["value"], "unit": "design iter/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * s["seconds_per_design_iteration"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (built-in cantilever load case)",
        "config": {"workload": cfg["name"], "V0": cfg["V0"], "mg_max_levels": cfg["max_levels"],
                   "precision": "fp64 (reference OpenMP CPU path)", "vcycle": "adapted (the reference's only cycle)",
                   "pcg_iterations_assumed": n_pcg},
        "cpu_baseline": {"value": s["value"], "unit": "design iter/s", "cores": s["cores"], "kind": s["kind"],
                         "sample": s["sample"], "pcg_iteration_s": s["pcg_iteration_s"]},
        "e2e": {"value": s["value"], "unit": "design iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.time() - t0,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- replicas (one independent design per GPU)
def max_over_ranks(values, world, device):
    """Each rank's timings -> the maximum over all ranks (the job's time is its slowest replica)."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_throughput(world, steps, seconds):
    """Whole-job design iterations/s: every replica runs `steps` iterations in at most `seconds`."""
    return world * steps / seconds


# ---------------------------------------------------------------- B200 arm
# Solver regimes of the design loop.  "converged": both forms solve every design iteration to |r| < 1e-6 |b| with
# the Standard V-cycle (the MATLAB original's 'Standard', TOP3D_XL.m:772-807) rebuilt every iteration -- the
# regime in which "compliance within 1e-6 of FP64" is a property of the solution; "reference": the reference
# CLI's algorithm (Adapted V-cycle, rebuilt at loop 1 and every 5th, tol 1e-3, 800-iteration cap), in which the
# solves stop at the cap unconverged at this size, as the reference's do.
REGIMES = {
    "converged": dict(mg_vcycle="standard", mg_rebuild_period=1, cg_tol=1e-6, cg_max_it=2000,
                      desc="converged: every solve to |r| < 1e-6 |b| (PCG cap 2000), Standard V-cycle rebuilt every "
                           "design iteration, both forms"),
    "reference": dict(mg_vcycle="adapted", mg_rebuild_period=5, cg_tol=1e-3, cg_max_it=800,
                      desc="reference: the reference CLI's solver (Adapted V-cycle rebuilt at loop 1 and every 5th, "
                           "tol 1e-3, 800-iteration cap; unconverged at the cap at this size)"),
}


# Serving sample: Poisson arrivals at the two ends of the 0.5-8 requests/s sweep, request sizes lognormal (median
# 0.5M elements, clipped to [30k, 16M]) with shapes, V0, load cases and voids drawn as in the batched workload,
# 40 OC iterations per request, 160 GB admission budget; the same seeded requests one at a time in plain FP64 as
# the baseline.
SERVE_RATES = (0.5, 8.0)
SERVE_SEED = 20251203
SERVE_ITERS = 40


def serving_sample(dev, n, regime):
    """designs/s and p50/p95/p99 end-to-end latency of the request loop (serve.DesignServer: admission by
    projected HBM footprint, concurrent contexts on their own streams) for n requests at each rate, and of the
    same requests served one at a time in FP64."""
    import algorithmengineering_altproject_b200 as t3d
    from algorithmengineering_altproject_b200 import serve

    def run(rate, precision, max_active, engine="streams"):
        with serve.DesignServer(device=dev, hbm_budget=160e9, max_active=max_active, precision=precision,
                                engine=engine, **regime_kw(t3d, regime)) as srv:
            res, wall = serve.run_poisson(srv, np.random.default_rng(SERVE_SEED), rate, n, SERVE_ITERS)
        s = serve.summary(res, wall)
        s["elements"] = int(sum(r.request.nelx * r.request.nely * r.request.nelz for r in res))
        return {"rate_per_s": rate, **s}

    out = {"requests_per_rate": n, "iters_per_request": SERVE_ITERS, "seed": SERVE_SEED, "budget_gb": 160,
           "max_active": 16, "precision": "mixed", "regime": REGIMES[regime]["desc"],
           "engine": "batched: requests in flight stepped together in one t3d batch, joining and leaving between "
                     "design iterations",
           "note": "p99 of %d requests is their maximum latency; latency = arrival to result" % n,
           "rates": [run(r, t3d.T3D_MIXED, 16, "batched") for r in SERVE_RATES]}
    out["streams_engine"] = run(SERVE_RATES[-1], t3d.T3D_MIXED, 8)
    out["sequential_fp64"] = run(SERVE_RATES[0], t3d.T3D_FP64, 1)
    return out


def run_batch_mode(args):
    """The batched workload: --batch instances drawn with the serving seed (nelx a multiple of 8 in [32, 192],
    nely and nelz nelx/2 scaled by U(0.5, 1), V0 ~ U(0.06, 0.30), the three load cases, 0-3 void ellipsoids),
    --batch-iters design iterations each, timed three ways on the same designs: all instances stepped
    together (t3d_batch: one launch per PCG kernel for all), one at a time in mixed precision (the same
    parameters, so the same results), and one at a time in plain FP64.  Times are wall clock around the design
    iterations (creation and the solid-domain solve excluded), synchronised; designs/s = design iterations/s
    divided by the 40 OC iterations of a design."""
    import torch
    import algorithmengineering_altproject_b200 as t3d
    from algorithmengineering_altproject_b200 import serve
    dev = dist_env()[2]
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(SERVE_SEED)
    reqs = [serve.draw_instance(rng, iters=args.batch_iters) for _ in range(args.batch)]
    dims = [(q.nely, q.nelx, q.nelz) for q in reqs]
    common = dict(device=dev, oc_sum_order=t3d.T3D_SUM_FP64, mg_coarse_assembly=t3d.T3D_COARSE_FULL,
                  **regime_kw(t3d, args.regime))
    K = args.batch_iters
    t0 = time.perf_counter()
    B = t3d.Batch(dims, problems=[q.spec() for q in reqs], **common)
    t_create = time.perf_counter() - t0
    bcs = B.design_init([q.V0 for q in reqs])
    torch.cuda.synchronize(dev)
    l0 = B.info()
    t0 = time.perf_counter()
    brecs = B.run([K] * len(reqs))          # every member K design iterations, advancing independently
    torch.cuda.synchronize(dev)
    t_batch = time.perf_counter() - t0
    info = B.info()
    bobj = np.array([[r["obj"] for r in brecs[i]] for i in range(len(reqs))])
    bits = np.array([[r["pcg_iters"] for r in brecs[i]] for i in range(len(reqs))])
    B.close()

    def alone(precision, **kw):
        total, objs, its, css = 0.0, [], [], []
        for q in reqs:
            P = t3d.Problem(q.nely, q.nelx, q.nelz, problem=q.spec(), precision=precision, **common, **kw)
            css.append(P.design_init(q.V0))
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            recs = [P.design_step() for _ in range(K)]
            torch.cuda.synchronize(dev)
            total += time.perf_counter() - t0
            objs.append([r["obj"] for r in recs])
            its.append([r["pcg_iters"] for r in recs])
            P.close()
        return total, np.array(objs), np.array(its), np.array(css)

    t_mixed, mobj, mits, mcs = alone(t3d.T3D_MIXED, matvec32_tile=t3d.T3D_BATCH_TILE)
    t_fp64, fobj, fits, _ = alone(t3d.T3D_FP64)
    # the same designs through the request loop's streams engine (one context and stream each, 12 in flight, all
    # submitted at once): wall time to the last result with K iterations each minus the same with none (creation
    # and the solid-domain solve), so that like the other arms it counts the design iterations only
    def streams(iters):
        with serve.DesignServer(device=dev, max_active=12, precision=t3d.T3D_MIXED, engine="streams",
                                **regime_kw(t3d, args.regime)) as srv:
            sreqs = [serve.DesignRequest(q.nely, q.nelx, q.nelz, q.V0, q.load_case, q.voids, iters, rid=k)
                     for k, q in enumerate(reqs)]
            t0 = time.perf_counter()
            sres = [f.result() for f in [srv.submit(q) for q in sreqs]]
            return time.perf_counter() - t0, [r.error for r in sres if r.error]

    t_setup, e0 = streams(0)
    t_full, e1 = streams(K)
    t_streams = max(1e-9, t_full - t_setup)
    serrors = e0 + e1
    its = len(reqs) * K
    rate = lambda t: its / t
    # bit-identity with the solo runs (NaN-aware), and the compliance error against FP64 per instance
    mismatch = [k for k in range(len(reqs)) if not np.array_equal(bobj[k], mobj[k], equal_nan=True)
                or bcs[k] != mcs[k]]
    mismatch_detail = [{"instance": k, "dims": list(dims[k]), "c_solid": [repr(bcs[k]), repr(mcs[k])],
                        "obj_batched": [repr(v) for v in bobj[k]], "obj_solo": [repr(v) for v in mobj[k]],
                        "pcg_batched": bits[k].tolist(), "pcg_solo": mits[k].tolist()} for k in mismatch]
    with np.errstate(divide="ignore", invalid="ignore"), warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)   # an all-NaN row (a singular domain) gives NaN
        rel = np.nanmax(np.abs(fobj - bobj) / np.abs(fobj), axis=1)
    capped = [k for k in range(len(reqs)) if (fits[k] >= REGIMES[args.regime]["cg_max_it"]).any()]
    # the error is stated over the instances whose FP64 solves all converged; an instance whose FP64 solve
    # stopped at the iteration cap (a singular domain) has no converged solution to compare with
    conv = np.array([k for k in range(len(reqs)) if k not in capped], dtype=np.int64)
    rc = rel[conv] if conv.size else np.array([np.nan])
    order = conv[np.argsort(-np.nan_to_num(rc, nan=np.inf))] if conv.size else conv
    worst = {"over": "instances whose FP64 solves converged", "instances": int(conv.size),
             "max": float(np.nanmax(rc)) if np.isfinite(rc).any() else None,
             "median": float(np.nanmedian(rc)) if np.isfinite(rc).any() else None,
             "instances_over_1e-6": int(np.sum(~(rc <= 1e-6))),
             "top": [{"instance": int(k), "dims": list(dims[k]), "rel_err": float(rel[k])} for k in order[:3]],
             "fp64_solves_at_the_iteration_cap": [{"instance": k, "dims": list(dims[k]),
                                                   "rel_err": None if not np.isfinite(rel[k]) else float(rel[k])}
                                                  for k in capped]}
    print(json.dumps({
        "mode": "batched designs", "instances": len(reqs), "design_iters_each": K,
        "elements_total": int(sum(a * b * c for a, b, c in dims)),
        "elements_median": float(np.median([a * b * c for a, b, c in dims])),
        "design_iters_per_s": {"batched": rate(t_batch), "sequential_mixed": rate(t_mixed),
                               "sequential_fp64": rate(t_fp64), "concurrent_streams": rate(t_streams)},
        "concurrent_streams_errors": serrors,
        "designs_per_s_at_40_iters": {"batched": rate(t_batch) / 40, "sequential_mixed": rate(t_mixed) / 40,
                                      "sequential_fp64": rate(t_fp64) / 40},
        "speedup_vs_sequential_fp64": t_fp64 / t_batch, "speedup_vs_sequential_mixed": t_mixed / t_batch,
        "batched_equals_solo_mixed": not mismatch, "instances_differing_from_solo": mismatch_detail,
        "compliance_rel_err_vs_fp64": worst,
        "batched_launches": info["batched_launches"] - l0["batched_launches"],
        "member_launches": info["member_launches"] - l0["member_launches"],
        "kernels_per_batched_pcg_iteration": info["kernels_per_iteration"],
        "logical_blocks_per_batched_pcg_iteration": info["blocks_per_iteration"],
        "arena_bytes": info["arena_bytes"], "create_s": t_create,
        "regime": REGIMES[args.regime]["desc"],
        "params": "mixed precision, full Galerkin coarsest, FP64 OC sum",
        "data": "synthetic (seed-drawn instances; no dataset involved)"}), flush=True)
    return 0


def regime_kw(t3d, regime):
    R = REGIMES[regime]
    return dict(mg_vcycle=t3d.T3D_VCYCLE_STANDARD if R["mg_vcycle"] == "standard" else t3d.T3D_VCYCLE_ADAPTED,
                mg_rebuild_period=R["mg_rebuild_period"], cg_tol=R["cg_tol"], cg_max_it=R["cg_max_it"])


def problem_kw(t3d, cfg, regime, precision, dev, tile=0):
    return dict(device=dev, mg_max_levels=cfg["max_levels"], oc_sum_order=t3d.T3D_SUM_FP64,
                precision=t3d.T3D_MIXED if precision == "mixed" else t3d.T3D_FP64, matvec32_tile=tile,
                **regime_kw(t3d, regime))


def matvec_roofline(P, mixed, mv_ms):
    """roofline of K(E)p (+ p.Ap): algorithmic bytes = w*(2 n_free + n_elements), w = 4 (FP32) or 8."""
    w = 4 if mixed else 8
    alg_bytes = w * (2 * P.nf + P.ne)
    achieved = alg_bytes / (mv_ms * 1e-3) / 1e9
    peak, peak_kind = hbm_peak()
    flops = 1152 * P.ne
    info = P.info()
    staging = {0: "per-thread cp.async", 1: "per-thread cp.async, packed FP32x2",
               2: "TMA bulk tensor copies, packed FP32x2"}.get(int(info.matvec32_tile[3]), "?")
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic_per_launch("matvec32" if mixed else "matvec64"), "peak_source": peak_kind,
            "kernel": (("k_matvec32_tma" if info.matvec32_tile[3] == 2 else "k_matvec32_modal"
                        if info.matvec32_modal else "k_matvec32") + " (FP32 K(E)p + FP64 p.Ap; %s)" % staging
                       if mixed else "k_matvec64_stream + k_dot_pcg (FP64 K(E)p, then p.Ap)"),
            "algorithmic_bytes_per_launch": alg_bytes, "flops_per_launch": flops,
            "tflops": flops / (mv_ms * 1e-3) / 1e12, "ms": mv_ms}


def throughput_fractions(P, mixed, vcycle, mv_ms, vc_ms, it_ms):
    """DOF-matvecs/s, V-cycles/s and PCG iterations/s with the HBM-roofline fraction of each, from algorithmic
    bytes per unit (n = free DOFs, N_e = elements, w = bytes per value of the inner solve, c = the coarse levels'
    3 * nodes):
      Adapted V-cycle   w * 4 (n + c)            (down: read r; up: read r and D, write z)
      Standard V-cycle  w * (22 n + 2 N_e + 8 c) + 2 k Σ N_l (level 0: Jacobi start r, D -> x; K x (2n + N_e);
                        residual r, Kx -> t; restriction reads t; prolongation x -> x; K x; correction r, t, x, D
                        -> x; r.z; each level l between the finest and the coarsest: two products with its N_l
                        stored Galerkin element matrices of k bytes each, 300 FP32 (symmetric-packed) or 576 FP64)
      PCG iteration     the V-cycle + w * (11 n + N_e) (K(E)p 2n + N_e, update 3n, direction and x update 6n)"""
    w = 4 if mixed else 8
    peak, _ = hbm_peak()
    coarse = sum(3 * (nx + 1) * (ny + 1) * (nz + 1) for nx, ny, nz, _ in P.levels[1:])
    n, ne = P.nf, P.ne
    kel = (300 * 4 if mixed else 576 * 8) * sum(nx * ny * nz for nx, ny, nz, _ in P.levels[1:-1])
    vc_bytes = w * (22 * n + 2 * ne + 8 * coarse) + 2 * kel if vcycle == "standard" else w * 4 * (n + coarse)
    it_bytes = vc_bytes + w * (11 * n + ne)
    out = {"dof_matvecs_per_s": n / (mv_ms * 1e-3), "vcycles_per_s": 1.0 / (vc_ms * 1e-3),
           "vcycle": vcycle, "vcycle_bytes": vc_bytes, "vcycle_gbs": vc_bytes / (vc_ms * 1e-3) / 1e9,
           "pcg_iteration_bytes": it_bytes}
    out["vcycle_frac"] = out["vcycle_gbs"] / peak
    if it_ms and it_ms > 0:
        out["pcg_iterations_per_s"] = 1.0 / (it_ms * 1e-3)
        out["pcg_iteration_gbs"] = it_bytes / (it_ms * 1e-3) / 1e9
        out["pcg_iteration_frac"] = out["pcg_iteration_gbs"] / peak
    return out


def run_kernels_only(args):
    """K(E)p and one V-cycle timed alone with CUDA events on a design-like state (E = SIMP of V0)."""
    import algorithmengineering_altproject_b200 as t3d
    cfg = CONFIGS[args.config]
    mixed = args.precision == "mixed"
    P = t3d.Problem(cfg["nely"], cfg["nelx"], cfg["nelz"], **problem_kw(t3d, cfg, args.regime, args.precision, 0,
                                                                       args.tile))
    rng = np.random.default_rng(7)
    E = np.full(P.ne, 1e-9 + cfg["V0"] ** 3 * (1.0 - 1e-9))
    P.make_diagonal_preconditioner_from_static(E)
    P.K_times_u_finest(E, rng.standard_normal(P.nf))     # leaves p on the device
    P.vcycle(rng.standard_normal(P.nf))                  # leaves r on the device
    mv = P.profile(t3d.T3D_PROFILE_MATVEC32 if mixed else t3d.T3D_PROFILE_MATVEC, args.reps)
    vc = P.profile(t3d.T3D_PROFILE_VCYCLE32 if mixed else t3d.T3D_PROFILE_VCYCLE, args.reps)
    print(json.dumps({"config": cfg["name"], "precision": args.precision, "regime": args.regime,
                      "matvec_ms": mv, "vcycle_ms": vc,
                      "matvec32_tile": list(P.info().matvec32_tile) if mixed else None,
                      "matvec32_variant": int(P.info().matvec32_variant) if mixed else None,
                      "roofline": matvec_roofline(P, mixed, mv)}), flush=True)
    P.close()
    return 0


def compare_forms(cfg, regime, dev, steps, warm=1):
    """Mixed vs plain FP64 on the same designs: both forms run `warm` untimed and `steps` compared design
    iterations, the mixed one starting each iteration from the FP64 one's density.  Returns speeds (device time
    of the compared iterations) and relative errors."""
    import algorithmengineering_altproject_b200 as t3d
    F = t3d.Problem(cfg["nely"], cfg["nelx"], cfg["nelz"], **problem_kw(t3d, cfg, regime, "fp64", dev))
    M = t3d.Problem(cfg["nely"], cfg["nelx"], cfg["nelz"], **problem_kw(t3d, cfg, regime, "mixed", dev))
    csF, csM = F.design_init(cfg["V0"]), M.design_init(cfg["V0"])
    out = {"regime": REGIMES[regime]["desc"], "c_solid_rel_err": abs(csM - csF) / abs(csF), "iterations": []}
    tF = tM = 0.0
    for k in range(warm + steps):
        M.set_density(F.density())
        rF, rM = F.design_step(), M.design_step()
        if k < warm:
            continue
        uF, uM = F.displacement(), M.displacement()
        xF, xM = F.density(), M.density()
        tF += rF["t_total"]
        tM += rM["t_total"]
        out["iterations"].append({
            "loop": rF["loop"], "pcg_iters_fp64": rF["pcg_iters"], "pcg_iters_mixed": rM["pcg_iters"],
            "outer_passes_mixed": int(M.info().last_outer_passes),
            "compliance_rel_err": abs(rM["obj"] - rF["obj"]) / abs(rF["obj"]),
            "displacement_rel_l2_err": float(np.linalg.norm(uM - uF) / np.linalg.norm(uF)),
            "density_max_abs_err": float(np.max(np.abs(xM.astype(np.float64) - xF))),
            "s_fp64": rF["t_total"], "s_mixed": rM["t_total"]})
    out["max_compliance_rel_err"] = max(i["compliance_rel_err"] for i in out["iterations"])
    out["fp64_design_iter_per_s"] = steps / tF
    out["mixed_design_iter_per_s"] = steps / tM
    out["speedup_mixed_vs_fp64"] = tF / tM
    F.close()
    M.close()
    return out


def run_b200(args):
    # the serving sample runs concurrent contexts in this process: load every kernel module at CUDA start-up
    os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")
    import torch
    import algorithmengineering_altproject_b200 as t3d

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local
    torch.cuda.set_device(dev)
    cfg = CONFIGS[args.config]
    mixed = args.precision == "mixed"
    regime = args.regime

    comparison = compare_forms(cfg, regime, dev, args.compare_steps) if (mixed and args.compare_steps > 0) else None
    # the other regime, briefly, for context (no FP64 comparison in the reference regime: 1 warm + 1 compared step)
    other = None
    if mixed and regime == "converged" and args.compare_steps > 0:
        other = compare_forms(cfg, "reference", dev, 1)

    P = t3d.Problem(cfg["nely"], cfg["nelx"], cfg["nelz"], **problem_kw(t3d, cfg, regime, args.precision, dev))
    P.design_init(cfg["V0"])
    for _ in range(args.warmup):
        P.design_step()

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()

    # One timed loop gives both numbers on the same design iterations: every iteration takes the design field
    # from pinned host memory and returns the updated one there (t3d_design_step_host; the two pinned buffers
    # trade roles), `value` sums the library's CUDA-event time of the iterations themselves (inputs resident in
    # HBM), `e2e` is the wall time of the loop with the host<->device copies inside.
    x = torch.empty(P.ne, dtype=torch.float32, pin_memory=True).numpy()
    xo = torch.empty(P.ne, dtype=torch.float32, pin_memory=True).numpy()
    x[:] = P.density()
    clocks = ClockSampler(dev)
    clocks.start()
    barrier()
    launches0 = P.kernel_launches()
    t_wall0 = time.perf_counter()
    recs = []
    for _ in range(args.steps):
        _, rec = P.design_step_host(x, out=xo)
        recs.append(rec)
        x, xo = xo, x
    barrier()
    t_wall = time.perf_counter() - t_wall0
    launches = P.kernel_launches() - launches0
    clk = clocks.stop()
    dev_time = sum(r["t_total"] for r in recs)
    e2e = None if args.no_e2e else t_wall

    # the dominant kernel (K(E)p with the fused p.Ap) and one V-cycle, CUDA events on the library stream
    mv_ms = P.profile(t3d.T3D_PROFILE_MATVEC32 if mixed else t3d.T3D_PROFILE_MATVEC, args.reps)
    vc_ms = P.profile(t3d.T3D_PROFILE_VCYCLE32 if mixed else t3d.T3D_PROFILE_VCYCLE, max(1, args.reps // 2))

    dev_time, t_wall, e2e = max_over_ranks([dev_time, t_wall, e2e if e2e is not None else 0.0], world, "cuda")

    if rank == 0:
        ne = P.ne
        pcg_its = [r["pcg_iters"] for r in recs]
        it_ms = 1000.0 * sum(r["t_cg"] for r in recs) / max(1, sum(pcg_its))
        R = REGIMES[regime]
        line = {
            "metric": METRIC, "value": job_throughput(world, args.steps, dev_time), "unit": "design iter/s",
            "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dev_time / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64 (mixed)" if mixed else "f64",
            "data": "synthetic (the reference's built-in cantilever load case; no dataset involved)",
            "config": {"workload": cfg["name"], "V0": cfg["V0"], "mg_max_levels": cfg["max_levels"],
                       "mg_levels": P.nlev, "coarse_dofs": P.coarse_n, "regime": R["desc"],
                       "precision": ("mixed: FP32 inner MG-PCG in FP64 defect correction" if mixed
                                     else "fp64 (plain GPU form)"),
                       "oc_volume_sum": "fp64", "parallelism": "replicas" if world > 1 else "single GPU",
                       "vcycle": R["mg_vcycle"] + ("" if R["mg_vcycle"] == "adapted" else
                                                  " (the MATLAB original's Standard cycle; the C++ reference has "
                                                  "only the Adapted one)"),
                       "mg_rebuild_period": R["mg_rebuild_period"], "cg_tol": R["cg_tol"],
                       "cg_max_it": R["cg_max_it"],
                       "l2": "inputs larger than L2 (node vectors %.0f MB each)" % (3 * P.nn * (4 if mixed else 8) / 1e6)},
            "pcg_iterations": pcg_its,
            "per_kernel_ms": {"matvec": mv_ms, "vcycle": vc_ms, "pcg_iteration": it_ms},
            "throughput": throughput_fractions(P, mixed, R["mg_vcycle"], mv_ms, vc_ms, it_ms),
            "roofline": matvec_roofline(P, mixed, mv_ms),
            "matvec32_tile": list(P.info().matvec32_tile) if mixed else None,
            "clocks": clk,
            "gpu_launches": launches,
            "wall_s_timed": t_wall,
        }
        if comparison is not None:
            line["vs_fp64"] = comparison
        if other is not None:
            line["reference_regime"] = other
        if e2e:
            line["e2e"] = {"value": job_throughput(world, args.steps, e2e), "unit": "design iter/s",
                           "h2d_bytes_per_step": 4 * ne, "d2h_bytes_per_step": 4 * ne + 64}
        if not args.no_cpu_baseline and world == 1:
            try:
                s = reference_sample(CONFIGS[args.config], CPU_SAMPLES, 800, physical_cores())
                line["cpu_baseline"] = {"value": s["value"], "unit": "design iter/s", "cores": s["cores"],
                                        "kind": s["kind"], "sample": s["sample"],
                                        "pcg_iteration_s": s["pcg_iteration_s"]}
            except Exception as e:  # baseline is reported, never required for the GPU number
                line["cpu_baseline"] = {"value": None, "unit": "design iter/s", "cores": 0, "kind": "reference",
                                        "sample": "unavailable: %s" % e}
    P.close()
    if rank == 0:
        if args.serve_requests > 0 and world == 1 and mixed:
            try:
                line["serving"] = serving_sample(dev, args.serve_requests, regime)
            except Exception as e:  # reported beside the headline, never required for it
                line["serving"] = {"unavailable": "%s: %s" % (type(e).__name__, e)}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    args = parse_args()
    setup_cpu_env()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.kernels_only:
        return run_kernels_only(args)
    if args.batch > 0:
        os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")
        return run_batch_mode(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
