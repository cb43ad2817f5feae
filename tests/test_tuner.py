"""The batch autotuner's performance model and search (CPU: no GPU needed).

The model's per-algorithm counts follow the reference's model (model_coefficient.py:36-100:
[R, A additions, B additions, C updates]); the B200 constants and the search are this
project's own.  The search is exercised with a synthetic measure function."""
import math

import pytest

from fmm_gen_b200 import tuner


def test_counts_match_the_reference_model():
    # 222-1 (Strassen): 7 products, 5 extra A terms, 5 extra B terms, 12 C updates
    assert tuner.model_counts(tuner.plan_of("222-1")) == [7, 5, 5, 12]
    r, a, b, c = tuner.model_counts(tuner.plan_of("222-2"))
    assert r == 49 and c == 144


def test_model_prefers_classical_small_and_fmm_large():
    m = tuner.B200Model()
    assert tuner.rank_candidates(m, (256, 256, 256))[0][0] == "classical"
    best_big = tuner.rank_candidates(m, (16384, 16384, 16384))[0][0]
    assert best_big in ("222-1", "222-2")
    # FMM executes fewer flops: at 16384^3 the model's 222-1 time is near 7/8 of classical
    t_c = tuner.model_time(m, "classical", 16384, 16384, 16384)
    t_s = tuner.model_time(m, "222-1", 16384, 16384, 16384)
    assert 0.8 < t_s / t_c < 0.97


def test_partition_and_units_cover_fringes():
    m = tuner.B200Model()
    c = tuner.job_costs(m, "222-1", 1030, 1001, 777)
    assert c["units"] > 0 and c["sm_s"] > 0
    # classical and FMM agree on the flop scale for tiny shapes
    assert tuner.model_time(m, "classical", 1, 1, 1) > 0


def test_random_batch_shapes_are_seeded_and_in_range():
    a = tuner.random_batch_shapes(512, seed=0)
    b = tuner.random_batch_shapes(512, seed=0)
    assert a == b and len(a) == 512
    assert all(256 <= v <= 4096 for s in a for v in s)
    mean = sum(math.log(v) for s in a for v in s) / (3 * 512)
    assert abs(mean - (math.log(256) + math.log(4096)) / 2) < 0.1


def test_search_keeps_measured_improvements():
    shapes = [(4096, 4096, 4096)] * 4 + [(300, 300, 300)] * 4
    calls = []

    def measure(choices):  # a machine on which every FMM is slower than classical
        calls.append(list(choices))
        return sum(2.0 if c != "classical" else 1.0 for c in choices)

    rep = tuner.BatchTuner().tune(shapes, measure)
    assert rep.model_choices[0] != "classical"
    assert rep.choices == ["classical"] * len(shapes)
    assert rep.trials[0][0] == "model choice" and len(calls) >= 2


def test_search_without_measurement_returns_the_model_choice():
    shapes = tuner.random_batch_shapes(16, seed=1)
    rep = tuner.BatchTuner().tune(shapes)
    assert rep.choices == rep.model_choices


def test_sweep_families_match_the_reference_ranges():
    from fmm_gen_b200 import sweep

    assert sweep.shapes("square", [240, 480]) == [(240, 240, 240), (480, 480, 480)]
    assert sweep.shapes("rankk", [240]) == [(14400, 14400, 240)]
    assert sweep.shapes("fixk", [960]) == [(960, 960, 1024)]
    with pytest.raises(ValueError):
        sweep.shapes("cube", [1])
    m = tuner.B200Model()
    assert sweep.model_gflops("222-1", 8192, 8192, 8192, m) > sweep.model_gflops("classical", 8192, 8192, 8192, m)
