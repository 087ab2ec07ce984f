"""Batched designs (t3d_batch_*): designs of uneven grid size stepping together, every kernel of the inner FP32
MG-PCG iteration one persistent launch over an (instance, block) work list with per-instance convergence
masks.  Each member's design iterations must equal, bit for bit, those of the same design run alone with the
same parameters (the batched launches give every instance the blocks, arithmetic and reduction order of its
own launches); the solo path itself is pinned to the oracle by the parity tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# uneven grids, all three load cases, voids (centre ex, ey, ez, radii rx, ry, rz in element units)
CASES = [
    dict(dims=(16, 48, 24), load_case=0, voids=(), V0=0.12),
    dict(dims=(24, 40, 16), load_case=1, voids=((20.0, 12.0, 8.0, 6.0, 5.0, 4.0),), V0=0.2),
    dict(dims=(32, 64, 32), load_case=2, voids=((40.0, 10.0, 16.0, 8.0, 6.0, 6.0), (12.0, 20.0, 10.0, 5.0, 5.0, 5.0)),
         V0=0.08),
    dict(dims=(8, 32, 16), load_case=0, voids=(), V0=0.3),
]
COMMON = dict(oc_sum_order=1, mg_coarse_assembly=1)


def spec(t3d, c):
    return t3d.ProblemSpec.make(c["load_case"], c["voids"])


def run_alone(t3d, c, steps, **extra):
    P = t3d.Problem(*c["dims"], problem=spec(t3d, c), precision=t3d.T3D_MIXED, matvec32_tile=t3d.T3D_BATCH_TILE,
                    **COMMON, **extra)
    cs = P.design_init(c["V0"])
    recs = [P.design_step() for _ in range(steps)]
    x, u = P.density(), P.displacement()
    P.close()
    return cs, recs, x, u


def same_records(a, b):
    for key in ("loop", "pcg_iters", "obj", "vol", "sharp", "change", "lmid", "bisections"):
        assert a[key] == b[key], (key, a[key], b[key])


# the reference's solver (Adapted V-cycle, tol 1e-3) and the converged regime (Standard V-cycle rebuilt every
# iteration, tol 1e-6)
REGIMES = {"adapted": dict(), "standard": dict(mg_vcycle=1, mg_rebuild_period=1, cg_tol=1e-6, cg_max_it=2000)}


@pytest.mark.parametrize("regime", sorted(REGIMES))
def test_batch_members_equal_their_solo_runs(regime):
    import algorithmengineering_altproject_b200 as t3d
    steps = 3
    R = REGIMES[regime]
    B = t3d.Batch([c["dims"] for c in CASES], problems=[spec(t3d, c) for c in CASES], **COMMON, **R)
    info = B.info()
    assert info["members"] == len(CASES) and info["arena_bytes"] > 0
    assert all(m.device_bytes > 0 for m in B.members)
    cs = B.design_init([c["V0"] for c in CASES])
    brecs = [B.design_step() for _ in range(steps)]
    bx = [m.density() for m in B.members]
    bu = [m.displacement() for m in B.members]
    info = B.info()
    B.close()
    # one launch per kernel of the PCG iteration for all members: far fewer than the members' own launches
    assert 5 <= info["kernels_per_iteration"] <= 40
    assert info["batched_launches"] > 0
    for i, c in enumerate(CASES):
        cs1, recs1, x1, u1 = run_alone(t3d, c, steps, **R)
        assert cs[i] == cs1
        for k in range(steps):
            same_records(brecs[k][i], recs1[k])
        np.testing.assert_array_equal(bx[i], x1)
        np.testing.assert_array_equal(bu[i], u1)


def test_batch_member_budgets_and_masks():
    """Members with their own iteration budgets (one far below its need, not a multiple of the graph chunk)
    stop on the device at their budget while the others go on; each still equals its solo run."""
    import algorithmengineering_altproject_b200 as t3d
    cases = CASES[:3]
    extra = [dict(cg_max_it=11), dict(), dict(cg_tol=1e-5)]
    B = t3d.Batch([c["dims"] for c in cases], problems=[spec(t3d, c) for c in cases], member_params=extra, **COMMON)
    B.design_init([c["V0"] for c in cases])
    brecs = [B.design_step() for _ in range(2)]
    bx = [m.density() for m in B.members]
    B.close()
    assert brecs[0][0]["pcg_iters"] <= 11   # its budget
    for i, c in enumerate(cases):
        _, recs1, x1, _ = run_alone(t3d, c, 2, **extra[i])
        for k in range(2):
            same_records(brecs[k][i], recs1[k])
        np.testing.assert_array_equal(bx[i], x1)


def test_batch_rejects_members_it_cannot_batch():
    import algorithmengineering_altproject_b200 as t3d
    with pytest.raises(t3d.T3DError, match="one V-cycle"):
        t3d.Batch([(16, 32, 16), (16, 32, 16)], member_params=[dict(), dict(mg_vcycle=t3d.T3D_VCYCLE_STANDARD)])
    with pytest.raises(t3d.T3DError, match="T3D_MIXED"):
        P = t3d.Problem(16, 32, 16, matvec32_tile=t3d.T3D_BATCH_TILE)   # FP64
        P.design_init(0.2)
        B = t3d.Batch.open()
        try:
            B.adopt(P)
        finally:
            B.close()
            P.close()


def test_members_join_and_leave_between_steps():
    """Continuous batching: contexts created and initialised alone join an open batch (adopt) and leave it
    (release) between design iterations; each still equals its solo run."""
    import algorithmengineering_altproject_b200 as t3d
    cases = CASES[:3]

    def make(c):
        P = t3d.Problem(*c["dims"], problem=spec(t3d, c), precision=t3d.T3D_MIXED,
                        matvec32_tile=t3d.T3D_BATCH_TILE, **COMMON)
        P.design_init(c["V0"])
        return P

    B = t3d.Batch.open()
    assert B.design_step() == []                     # an empty batch steps nothing
    got = {0: [], 1: [], 2: []}
    B.adopt(make(cases[0]))
    B.adopt(make(cases[1]))
    for r, k in zip(B.design_step(), (0, 1)):
        got[k].append(r)
    B.adopt(make(cases[2]))                           # joins at the second step
    for r, k in zip(B.design_step(), (0, 1, 2)):
        got[k].append(r)
    P0 = B.release(0)                                 # leaves after two steps
    x0 = P0.density()
    P0.close()
    for r, k in zip(B.design_step(), (1, 2)):
        got[k].append(r)
    x = {1: B.members[0].density(), 2: B.members[1].density(), 0: x0}
    B.close()
    for k, c in enumerate(cases):
        _, recs1, x1, _ = run_alone(t3d, c, len(got[k]))
        for a, b in zip(got[k], recs1):
            same_records(a, b)
        np.testing.assert_array_equal(x[k], x1)


def test_arena_members_cannot_be_released():
    import algorithmengineering_altproject_b200 as t3d
    B = t3d.Batch([CASES[3]["dims"]], **COMMON)
    with pytest.raises(t3d.T3DError, match="arena"):
        B.release(0)
    B.close()


def test_run_with_uneven_step_counts():
    """t3d_batch_run: members run different numbers of design iterations, each advancing on its own; every
    member equals its solo run."""
    import algorithmengineering_altproject_b200 as t3d
    cases = CASES[:3]
    steps = [2, 4, 1]
    R = REGIMES["standard"]
    B = t3d.Batch([c["dims"] for c in cases], problems=[spec(t3d, c) for c in cases], **COMMON, **R)
    B.design_init([c["V0"] for c in cases])
    recs = B.run(steps)
    x = [m.density() for m in B.members]
    B.close()
    for i, c in enumerate(cases):
        assert len(recs[i]) == steps[i]
        _, recs1, x1, _ = run_alone(t3d, c, steps[i], **R)
        for a, b in zip(recs[i], recs1):
            same_records(a, b)
        np.testing.assert_array_equal(x[i], x1)


def test_submitted_work_is_collected_with_solo_results():
    """Submitted work (the request loop's engine): contexts initialised alone are submitted with their own
    iteration counts and collected when done; results equal the solo runs."""
    import algorithmengineering_altproject_b200 as t3d
    cases = CASES
    steps = [3, 1, 2, 4]
    B = t3d.Batch.open()
    subs = {}
    for i, c in enumerate(cases):
        P = t3d.Problem(*c["dims"], problem=spec(t3d, c), precision=t3d.T3D_MIXED,
                        matvec32_tile=t3d.T3D_BATCH_TILE, **COMMON)
        P.design_init(c["V0"])
        B.submit(P, steps[i])
        subs[id(P)] = i
    got = {}
    while len(got) < len(cases):
        r = B.collect(1000)
        if r is None:
            continue
        P, recs, err = r
        assert err is None, err
        got[subs[id(P)]] = (recs, P.density())
        P.close()
    B.close()
    for i, c in enumerate(cases):
        recs, x = got[i]
        assert len(recs) == steps[i]
        _, recs1, x1, _ = run_alone(t3d, c, steps[i])
        for a, b in zip(recs, recs1):
            same_records(a, b)
        np.testing.assert_array_equal(x, x1)
