"""Host logic of the batched and served forms (no GPU): the request mixes and the serving
loop's admission and tick rules."""
import pytest

from streams_b200.cases import batch_mix, serve_mix, BATCH_NX, BATCH_NY, BATCH_NZ


def test_batch_mix_matches_the_workload():
    boxes = batch_mix()
    assert len(boxes) == 48
    for b in boxes:
        assert b["nx"] in BATCH_NX and b["ny"] in BATCH_NY and b["nz"] in BATCH_NZ
        assert 0.3 <= b["mach"] <= 2.0 and 2000 <= b["re_bulk"] <= 6000
    assert batch_mix() == boxes  # seeded


def test_serve_mix_is_a_poisson_stream():
    reqs = serve_mix(400, rate_per_s=2.0)
    gaps = [b["arrival"] - a["arrival"] for a, b in zip(reqs, reqs[1:])]
    assert all(g > 0 for g in gaps)
    assert sum(gaps) / len(gaps) == pytest.approx(0.5, rel=0.15)
    for r in reqs:
        assert 32 <= r["ny"] and r["nx"] % 16 == 0 and 0.5 <= r["mach"] <= 2.5
        assert 200 <= r["nsteps"] <= 2000 and r["precision"] in (0, 1)


def test_admission_is_fifo_by_footprint():
    from streams_b200.serve import admit_fifo
    assert admit_fifo([4, 4, 4], used=0, budget=10) == 2
    assert admit_fifo([8, 1, 1], used=4, budget=10) == 0  # the head does not fit: nobody overtakes
    assert admit_fifo([], used=0, budget=10) == 0
    assert admit_fifo([10], used=0, budget=10) == 1


def test_tick_never_overshoots_a_solve():
    from streams_b200.serve import tick_length
    assert tick_length([100, 7, 50], 10) == 7
    assert tick_length([100, 50], 10) == 10
    assert tick_length([1], 10) == 1
