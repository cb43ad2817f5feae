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

    def measure(choices, tiles=None):  # a machine on which every FMM is slower than classical
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


def test_tile_work_counts_edge_fragments():
    assert tuner._tile_work(256, 384) == 6.0  # whole tiles
    # 40 rows past the last whole tile: 3 of 8 16-row fragments
    assert tuner._tile_work(128 + 40, 128) == 1.0 + 3 / 8
    # 40 columns past it: 2 of 4 32-column groups
    assert tuner._tile_work(128, 128 + 40) == 1.0 + 2 / 4
    # corner: the cheaper of the two edge forms
    assert tuner._tile_work(40, 40) == min(3 / 8, 2 / 4)
    assert tuner._tile_work(0, 128) == 0.0


# Single-problem times (ms) measured on B200 with this library's current kernels; the model's
# stated fit is 9 % RMS of the log ratio over these points.
MEASURED_MS = {
    ("222-1_333-1", 4000, 3840, 2000): 2.659, ("222-1_333-1", 4000, 8000, 2000): 5.264,
    ("222-1_333-1", 4096, 4096, 4096): 5.077, ("222-1_333-1", 3000, 3000, 3000): 2.122,
    ("222-1_333-1", 14400, 3840, 480): 3.807, ("222-1_333-1", 16384, 16384, 16384): 205.42,
    ("222-1_333-1", 4000, 16000, 2000): 9.65, ("222-1_333-1", 14400, 14400, 480): 12.76,
    ("222-1", 1024, 1024, 1024): 0.138, ("222-1", 2048, 2048, 2048): 0.64,
    ("222-1", 6000, 6000, 6000): 11.79, ("222-1", 16384, 16384, 16384): 219.7,
    ("222-2", 2048, 2048, 2048): 0.604, ("222-2", 3000, 3000, 3000): 1.874,
    ("classical", 3000, 3000, 3000): 1.67, ("classical", 16384, 16384, 16384): 249.1,
    ("classical", 2048, 2048, 2048): 0.577,
}


def test_single_problem_model_fits_the_measurements():
    m = tuner.B200Model()
    logs = [math.log(tuner.model_time_single(m, a, *s) * 1e3 / t) for (a, *s), t in MEASURED_MS.items()]
    rms = math.sqrt(sum(x * x for x in logs) / len(logs))
    assert rms < 0.10
    assert max(abs(x) for x in logs) < 0.25


def test_single_problem_view_adds_waves_and_launches():
    m = tuner.B200Model()
    # a small problem leaves SMs idle and pays launch latency: slower than its batch share
    assert tuner.model_time_single(m, "222-1", 1024, 1024, 1024) > 1.5 * tuner.model_time(m, "222-1", 1024, 1024, 1024)
    # a large one fills many waves: the two views agree closely
    a = tuner.model_time_single(m, "222-1", 16384, 16384, 16384)
    b = tuner.model_time(m, "222-1", 16384, 16384, 16384)
    assert abs(a / b - 1) < 0.05


def test_tile_refinement_keeps_64_row_tiles_only_where_measured_faster():
    """The tuner tries 64-row tiles for the problems with the longest, fewest units first and
    keeps a tile choice only when the measured batch gets faster."""
    shapes = [(256, 256, 4096)] * 2 + [(2048, 2048, 512)] * 38
    tn = tuner.BatchTuner()
    pressure = [tn.tile_pressure("classical", s) for s in shapes]
    assert min(pressure[:2]) > max(pressure[2:])  # deep, narrow problems rank first

    def measure(choices, tiles=None):  # 64-row tiles help the two deep problems only
        t = 100.0
        for i, tl in enumerate(tiles or [128] * len(choices)):
            if tl == 64:
                t += -3.0 if i < 2 else 1.0
        return t

    rep = tn.tune(shapes, measure)
    assert rep.tiles[:2] == [64, 64] and set(rep.tiles[2:]) == {128}
    assert rep.counts()["classical/64"] == 2

    rep2 = tn.tune(shapes, lambda c, tiles=None: 100.0 + sum(1.0 for x in (tiles or []) if x == 64))
    assert set(rep2.tiles) == {128}
