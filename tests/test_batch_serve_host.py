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
    frac = sum(r["kind"] == "sbli" for r in reqs) / len(reqs)
    assert 0.2 < frac < 0.4


def test_shock_angle_gives_the_deflection():
    import math
    from streams_b200.cases import shock_angle_for
    for m in (1.8, 2.0, 2.28, 2.5):
        b = math.radians(shock_angle_for(m))
        th = math.atan(2.0 / math.tan(b) * (m * m * math.sin(b) ** 2 - 1.0) / (m * m * (1.4 + math.cos(2 * b)) + 2.0))
        assert abs(math.degrees(th) - 8.0) < 1e-6
    assert abs(shock_angle_for(2.28) - 32.6) < 0.5


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
