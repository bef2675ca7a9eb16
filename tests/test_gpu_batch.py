"""Batched solves on the GPU: every member's result equals its solve alone and in any mix.

A member of a batch runs on fewer CTAs than it would alone, so its reductions add partials in
a different order: the float32 fields agree with the solo solve to round-off of the pressure
tolerance, not bit for bit. The stated tolerance is 2e-5 absolute on the cell velocity
(freestream speed 1) with equal substep counts; the same member in two different mixes is
held to the same bound.
"""

import numpy as np
import pytest

from foilbench_b200 import workloads
from foilbench_b200.batch import StableFluidsBatch
from foilbench_b200.geometry import NacaFoil
from foilbench_b200.models import NumericalFailure
from foilbench_b200.solver import StableFluidsSolver

pytestmark = pytest.mark.gpu

TOL = 2.0e-5
STEPS = 3


def _cases():
    return {
        "a": workloads.single("a", 256, 128, "0012", 8.0, 1000.0),
        "b": workloads.single("b", 384, 192, "2412", 12.0, 300.0),
        "c": workloads.single("c", 512, 256, "4415", -3.0, 5000.0),
        "d": workloads.single("d", 768, 384, "0009", 18.0, 150.0),
    }


def _start(sc):
    s = StableFluidsSolver()
    s.initialize(sc, NacaFoil(sc.foil), 0)
    return s


def _alone(sc):
    s = _start(sc)
    subs = []
    for k in range(STEPS):
        subs.append(s.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt).substeps)
    return s.cell_velocity(), subs


def _batched(scs):
    solvers = [_start(sc) for sc in scs]
    batch = StableFluidsBatch(solvers)
    subs = [[] for _ in scs]
    for k in range(STEPS):
        reps = batch.advance([sc.control_at((k + 1) * sc.output_dt) for sc in scs], [sc.output_dt for sc in scs])
        for i, r in enumerate(reps):
            assert not isinstance(r, NumericalFailure), r
            subs[i].append(r.substeps)
            assert r.state_revision == k + 1
        assert min(batch.ctas()) >= 1 and sum(batch.ctas()) <= 148 * 4
    out = [s.cell_velocity() for s in solvers]
    batch.close()
    return out, subs


def test_batch_members_match_their_solo_solves():
    cases = _cases()
    names = ["a", "b", "c"]
    solo = {n: _alone(cases[n]) for n in names}
    vel, subs = _batched([cases[n] for n in names])
    for i, n in enumerate(names):
        assert subs[i] == solo[n][1], n
        np.testing.assert_allclose(vel[i], solo[n][0], rtol=0, atol=TOL, err_msg=n)


def test_member_result_does_not_depend_on_the_mix():
    cases = _cases()
    v1, s1 = _batched([cases["a"], cases["b"], cases["c"]])
    v2, s2 = _batched([cases["d"], cases["a"]])
    assert s1[0] == s2[1]
    np.testing.assert_allclose(v1[0], v2[1], rtol=0, atol=TOL)


def test_failing_member_rolls_back_alone():
    cases = _cases()
    bad = workloads.single("bad", 256, 128, "0012", 8.0, 1000.0, extra={"mac_maximum_divergence_linf": 1.0e-30})
    solvers = [_start(cases["a"]), _start(bad)]
    before = solvers[1].cell_velocity()
    batch = StableFluidsBatch(solvers)
    reps = batch.advance([cases["a"].control_at(cases["a"].output_dt), bad.control_at(bad.output_dt)],
                         [cases["a"].output_dt, bad.output_dt])
    batch.close()
    assert not isinstance(reps[0], NumericalFailure)
    assert isinstance(reps[1], NumericalFailure) and reps[1].reason == "postcondition_failure"
    assert solvers[1].state_revision == 0 and solvers[0].state_revision == 1
    np.testing.assert_array_equal(solvers[1].cell_velocity(), before)


def test_batch_rejects_unsupported_members():
    sc = workloads.single("f64", 256, 128, "0012", 8.0, 1000.0, precision="float64")
    s = _start(sc)
    with pytest.raises(Exception, match="float32"):
        StableFluidsBatch([s])


def test_served_requests_match_their_solo_solves():
    """Requests that arrive while others run join the next batched launch; each finished
    request's field equals its own solo solve of the same number of steps (same tolerance)."""
    from foilbench_b200.serving import ServedSolves
    from foilbench_b200.workloads import Request

    cases = _cases()
    tick = [0.0]
    reqs = [Request(0, 0.0, 4, cases["a"]), Request(1, 0.0, 3, cases["c"]), Request(2, 1.5, 2, cases["b"])]
    served = ServedSolves(max_members=8, clock=lambda: tick[0], keep_fields=True)

    def on_tick(n):
        tick[0] = float(n)

    stats = served.run(reqs, on_tick=on_tick)
    assert len(stats.completed) == 3 and not any(c.failed for c in stats.completed)
    assert stats.max_active == 3  # request 2 joined while 0 and 1 were still running
    for c in stats.completed:
        sc = reqs[c.rid].scenario
        s = _start(sc)
        for k in range(reqs[c.rid].steps):
            s.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
        np.testing.assert_allclose(c.velocity, s.cell_velocity(), rtol=0, atol=TOL, err_msg=str(c.rid))
    p = stats.latency_percentiles()
    assert p["p50_s"] <= p["p99_s"]


def test_serving_admission_binds_on_the_hbm_budget():
    """The device context's HBM budget is the admission rule: with room for two of these solves
    and member slots to spare, the other requests wait in the queue (counted as budget
    rejections) and are admitted, in arrival order, as finished solves free their memory.
    Every result equals its solo solve."""
    from dataclasses import replace

    from foilbench_b200 import _native as N
    from foilbench_b200.serving import ServedSolves
    from foilbench_b200.workloads import Request

    base = _cases()["a"]
    scs = [replace(base, id=f"budget-{k}", controls=(type(base.controls[0])(0.0, 4.0 + 3.0 * k),)) for k in range(4)]
    probe = N.Context(0, 0)
    s = StableFluidsSolver(context=probe)
    s.initialize(scs[0], NacaFoil(scs[0].foil), 0)
    per = probe.bytes_in_use()
    s.close()
    assert per > 0
    tick = [0.0]
    reqs = [Request(k, 0.0, 2 + (k % 2), scs[k]) for k in range(4)]
    served = ServedSolves(hbm_budget=int(2.5 * per), max_members=64, clock=lambda: tick[0], keep_fields=True)

    def on_tick(n):
        tick[0] = float(n)

    stats = served.run(reqs, on_tick=on_tick)
    assert len(stats.completed) == 4 and not any(c.failed for c in stats.completed)
    assert stats.max_active == 2 and stats.rejected_budget > 0
    by_id = {c.rid: c for c in stats.completed}
    # requests 2 and 3 were admitted only after an earlier request finished
    first_done = min(by_id[0].finished_s, by_id[1].finished_s)
    assert by_id[2].admitted_s >= first_done and by_id[3].admitted_s >= first_done
    assert by_id[2].admitted_s <= by_id[3].admitted_s
    for c in stats.completed:
        sc = reqs[c.rid].scenario
        solo = _start(sc)
        for k in range(reqs[c.rid].steps):
            solo.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
        np.testing.assert_allclose(c.velocity, solo.cell_velocity(), rtol=0, atol=TOL, err_msg=str(c.rid))
