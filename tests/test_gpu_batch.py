"""Batched and served forms on the GPU: many boxes of uneven sizes, flow parameters and
precisions advanced through one CUDA graph, the launch-shape autotuner, and the serving loop.

Bound: bit-identical.  A box's arithmetic does not depend on the other boxes, on the graph or
on the tick in which it runs, so results must equal those of the box advanced alone with the
same launch tuning, bit for bit.
"""
import numpy as np
import pytest

from conftest import channel_ini, requires_gpu

pytestmark = [pytest.mark.gpu, requires_gpu]

BOXES = [dict(nx=32, ny=24, nz=16, mach=1.5, precision=0),
         dict(nx=24, ny=16, nz=12, mach=0.6, re_bulk=2500.0, seed=3, precision=1),
         dict(nx=48, ny=32, nz=16, mach=1.9, re_bulk=5500.0, seed=5, precision=0),
         dict(nx=16, ny=16, nz=16, mach=0.9, sensor=-1.0, seed=7, precision=1)]


def make(tmp_path, i, kw):
    from streams_b200 import Case, Solver
    kw = dict(kw)
    prec = kw.pop("precision")
    d = tmp_path / f"box{i}"
    d.mkdir(exist_ok=True)
    case = Case(d, channel_ini(**kw))
    s = Solver.from_case(case, precision=prec)
    s.init_run()
    return s


@pytest.mark.parametrize("nsteps,spg", [(24, 10), (7, 3), (1, 4)])
def test_batch_equals_alone(tmp_path, nsteps, spg):
    from streams_b200 import Batch
    alone = []
    for i, kw in enumerate(BOXES):
        s = make(tmp_path, i, kw)
        s.advance(nsteps)
        alone.append((s.copy_to_field(), s.scalars()))
        s.close()
    solvers = [make(tmp_path, i, kw) for i, kw in enumerate(BOXES)]
    b = Batch(solvers, steps_per_graph=spg)
    assert b.groups() == (2, 4)  # the FP64 pair and the mixed pair share launches
    b.advance(nsteps)
    b.synchronize()
    replays, per = b.stats()
    if nsteps - 1 >= spg:
        assert replays >= 1 and per > 0
    for s, (w, sc) in zip(solvers, alone):
        assert np.array_equal(s.copy_to_field(), w)
        assert s.scalars() == sc
    b.close()


def test_shared_launches_equal_separate_branches(tmp_path):
    """A group's shared launches (one launch per kernel kind and stage for all its boxes) give
    the boxes' own results, with fewer launches per replay than a branch per box."""
    from streams_b200 import Batch
    boxes = BOXES + [dict(nx=64, ny=32, nz=24, mach=1.1, re_bulk=4000.0, seed=9, precision=0),
                     dict(nx=40, ny=24, nz=20, mach=0.5, seed=11, precision=1),
                     dict(nx=48, ny=32, nz=32, mach=1.3, seed=13, precision=0)]
    out = {}
    for shared in (0, 1, 2):
        solvers = [make(tmp_path, i, kw) for i, kw in enumerate(boxes)]
        b = Batch(solvers, steps_per_graph=5)
        b.set_shared_launches(shared)
        # 4 FP64 boxes, 3 mixed: one group per class, or the FP64 class in two groups of two
        # (equal cell counts: 64x32x24 with 32x24x16, 48x32x32 with 48x32x16)
        assert b.groups() == {0: (0, 0), 1: (2, 7), 2: (3, 7)}[shared]
        b.advance(16)
        b.synchronize()
        out[shared] = ([s.copy_to_field() for s in solvers], [s.scalars() for s in solvers], b.stats())
        b.close()
        for s in solvers:
            s.close()
    for shared in (1, 2):
        for wa, wb in zip(out[0][0], out[shared][0]):
            assert np.array_equal(wa, wb)
        assert out[0][1] == out[shared][1]
    (ra, pa), (rb, pb) = out[0][2], out[1][2]
    assert ra == rb == 3 and pb < pa / 2, (pa, pb)


def test_launch_form_tuning_keeps_the_results(tmp_path):
    """The launch-form tuner advances the live boxes through every form; they still equal their
    runs alone, and the batch is left in the fastest form."""
    from streams_b200 import Batch
    solvers = [make(tmp_path, i, kw) for i, kw in enumerate(BOXES)]
    b = Batch(solvers, steps_per_graph=3)
    form, done, times = b.tune_form(forms=(1, 0), replays=1)
    assert form in (1, 0) and set(times) == {1, 0} and done == 1 + 2 * 2 * 3
    b.advance(5)
    b.synchronize()
    total = done + 5
    for i, kw in enumerate(BOXES):
        s = make(tmp_path, 10 + i, kw)
        s.advance(total)
        assert np.array_equal(s.copy_to_field(), solvers[i].copy_to_field()), i
        s.close()
    b.close()


def test_a_box_outside_the_groups_keeps_its_branch(tmp_path):
    """A boundary-layer box (stored ghosts, recycling inflow, non-reflecting faces) advances on
    its own branch beside a group of channels; every box equals its run alone."""
    from streams_b200 import Batch, Case, Solver
    from streams_b200.cases import bl_ini

    def bl():
        d = tmp_path / "bl"
        d.mkdir(exist_ok=True)
        s = Solver.from_case(Case(d, bl_ini(nx=48, ny=40, nz=16)), precision=0)
        s.init_run()
        return s

    kws = [BOXES[0], BOXES[2]]
    alone = []
    for i, kw in enumerate(kws):
        s = make(tmp_path, i, kw)
        s.advance(9)
        alone.append(s.copy_to_field())
        s.close()
    s = bl()
    s.advance(9)
    alone.append(s.copy_to_field())
    s.close()
    solvers = [make(tmp_path, i, kw) for i, kw in enumerate(kws)] + [bl()]
    b = Batch(solvers, steps_per_graph=4)
    assert b.groups() == (1, 2)
    b.advance(9)
    b.synchronize()
    for s, w in zip(solvers, alone):
        assert np.array_equal(s.copy_to_field(), w)
    b.close()


def test_a_retuned_box_rebuilds_its_group(tmp_path):
    from streams_b200 import Batch
    kws = [BOXES[0], BOXES[2]]
    ref = []
    for i, kw in enumerate(kws):
        s = make(tmp_path, i, kw)
        s.advance(7)
        if i == 1:
            s.set_tuning(37888, 8)
        s.advance(8)
        ref.append(s.copy_to_field())
        s.close()
    solvers = [make(tmp_path, i, kw) for i, kw in enumerate(kws)]
    b = Batch(solvers, steps_per_graph=3)
    b.advance(7)
    solvers[1].set_tuning(37888, 8)
    b.advance(8)
    b.synchronize()
    assert b.groups() == (1, 2)
    for s, w in zip(solvers, ref):
        assert np.array_equal(s.copy_to_field(), w)
    b.close()


def test_batch_continues_and_recaptures_after_retuning(tmp_path):
    from streams_b200 import Batch
    a = [make(tmp_path, i, kw) for i, kw in enumerate(BOXES[:2])]
    for s in a:
        s.advance(6)
        s.set_tuning(37888, 8)
        s.advance(9)
    ref = [s.copy_to_field() for s in a]
    solvers = [make(tmp_path, i, kw) for i, kw in enumerate(BOXES[:2])]
    b = Batch(solvers, steps_per_graph=5)
    b.advance(6)
    for s in solvers:
        s.set_tuning(37888, 8)
    b.advance(9)
    for s, w in zip(solvers, ref):
        assert np.array_equal(s.copy_to_field(), w)
    b.close()


def test_batch_rejects_bad_arguments(tmp_path):
    from streams_b200 import Batch, BackendError
    s = make(tmp_path, 0, BOXES[0])
    with pytest.raises(BackendError):
        Batch([s, s])
    with pytest.raises(BackendError):
        Batch([s], steps_per_graph=5, dt_every=2)
    with pytest.raises(BackendError):
        s.set_tuning(100, 16)
    with pytest.raises(BackendError):
        s.set_tuning(151552, 2)


def test_autotune_picks_a_candidate_and_caches(tmp_path):
    from streams_b200 import Case
    from streams_b200.tune import CANDIDATES, autotune
    case = Case(tmp_path, channel_ini(nx=48, ny=32, nz=32))
    cache = {}
    t = autotune(case, precision=0, cache=cache)
    assert t in CANDIDATES
    assert autotune(case, precision=0, cache=cache) == t and len(cache) == 1


def test_serving_alone_equals_in_the_mix():
    from streams_b200.serve import Server
    reqs = [dict(rid=0, arrival=0.0, nx=32, ny=24, nz=16, mach=1.2, nsteps=23, precision=0, seed=1),
            dict(rid=1, arrival=0.05, nx=48, ny=32, nz=16, mach=2.0, nsteps=31, precision=1, seed=2),
            dict(rid=2, arrival=0.10, nx=24, ny=16, nz=16, mach=0.7, nsteps=12, precision=0, seed=3),
            dict(rid=3, arrival=0.12, nx=16, ny=16, nz=16, mach=0.9, nsteps=1, precision=1, seed=4)]
    cache = {}
    mix = Server(budget_bytes=1 << 34, tick_steps=5, keep_fields=True, tune_cache=cache).run(reqs)
    assert mix["completed"] == 4 and mix["p50_s"] is not None and mix["p99_s"] >= mix["p50_s"]
    for r in reqs:
        alone = Server(budget_bytes=1 << 34, tick_steps=5, keep_fields=True, tune_cache=cache).run([dict(r, arrival=0.0)])
        a, m = alone["solves"][r["rid"]], mix["solves"][r["rid"]]
        assert np.array_equal(a.result["w"], m.result["w"]), r["rid"]
        assert a.result["scalars"] == m.result["scalars"]


def test_serving_cohorts_share_launches_and_equal_alone():
    """Solves of one class resident together advance as a cohort (shared launches); each result
    equals the solve served alone, bit for bit, and the same mix served without cohorts."""
    from streams_b200.serve import Server
    # long enough (and untuned, so that admission is quick) for the solves to be resident together
    reqs = [dict(rid=0, arrival=0.0, nx=48, ny=32, nz=32, mach=1.2, nsteps=400, precision=0, seed=1),
            dict(rid=1, arrival=0.0, nx=32, ny=24, nz=16, mach=2.0, nsteps=270, precision=0, seed=2),
            dict(rid=2, arrival=0.0, nx=64, ny=32, nz=16, mach=0.7, nsteps=330, precision=0, seed=3),
            dict(rid=3, arrival=0.0, nx=32, ny=32, nz=16, mach=0.9, nsteps=350, precision=1, seed=4),
            dict(rid=4, arrival=0.0, nx=48, ny=24, nz=16, mach=1.4, nsteps=220, precision=1, seed=5),
            dict(rid=5, arrival=0.0, nx=32, ny=32, nz=32, mach=0.8, nsteps=300, precision=1, seed=6)]
    kw = dict(budget_bytes=1 << 34, tick_steps=5, keep_fields=True, tune=False)
    mix = Server(**kw).run(reqs)
    assert mix["completed"] == 6 and mix["cohort_ticks"] > 0 and mix["max_cohort"] >= 2, mix
    apart = Server(shared=False, **kw).run(reqs)
    assert apart["cohort_ticks"] == 0
    for r in reqs:
        alone = Server(**kw).run([r])
        a, m, p = alone["solves"][r["rid"]], mix["solves"][r["rid"]], apart["solves"][r["rid"]]
        assert np.array_equal(a.result["w"], m.result["w"]), r["rid"]
        assert np.array_equal(a.result["w"], p.result["w"]), r["rid"]
        assert a.result["scalars"] == m.result["scalars"]


def test_serving_admits_within_the_memory_budget():
    from streams_b200.serve import Server, footprint_of, prepare
    import tempfile
    reqs = [dict(rid=i, arrival=0.0, nx=32, ny=24, nz=16, mach=1.5, nsteps=8, precision=0, seed=i + 1)
            for i in range(3)]
    one = footprint_of(prepare(reqs[0], tempfile.mkdtemp()), 0)
    srv = Server(budget_bytes=int(one * 1.5), tick_steps=4, tune=False)
    out = srv.run(reqs)
    assert out["completed"] == 3 and out["max_resident"] == 1
    big = Server(budget_bytes=one // 2, tune=False).run(reqs[:1])
    assert big["rejected"] == [0] and big["completed"] == 0
