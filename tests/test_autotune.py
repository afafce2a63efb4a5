"""The launch-shape tuner (autotune.py) on the CPU: candidate shapes, the choice of the fastest
by a fake clock, and the JSON cache round trip."""

import autotune


def test_candidates_cover_radius_batches_and_group_sizes():
    c = autotune.candidates(12)
    assert {kb for kb, _ in c} == set(autotune.RADIUS_BATCHES)
    assert {u for _, u in c} == {12, 6, 3, 1}
    assert autotune.candidates(1) == [(kb, 1) for kb in autotune.RADIUS_BATCHES]


def test_tune_picks_the_fastest_shape_and_caches_it(tmp_path):
    cost = {(kb, u): 1.0 + abs(kb - 8) * 0.1 + (0.5 if u == 1 else 0.0) for kb, u in autotune.candidates(12)}
    now = [0.0]
    ran = []

    def run(kb, per_call):
        ran.append((kb, per_call))
        now[0] += cost[(kb, per_call)]

    best, ms = autotune.tune(run, lambda: None, 12, reps=2, clock=lambda: now[0])
    assert best[0] == 8 and best[1] != 1
    assert len(ms) == len(cost) and len(ran) == 3 * len(cost)

    path = str(tmp_path / "cache.json")
    key = autotune.shape_key("B200", 64, 2, 12, 44)
    got = autotune.tuned(key, run, lambda: None, 12, path=path, clock=lambda: now[0])
    assert got == best
    n = len(ran)
    assert autotune.tuned(key, run, lambda: None, 12, path=path, clock=lambda: now[0]) == best   # from the cache: nothing runs
    assert len(ran) == n
    autotune.store({"other": {"radius_batch": 4, "per_call": 1}}, path)
    assert key in autotune.load(path) and "other" in autotune.load(path)


def test_store_into_an_unwritable_place_keeps_nothing(tmp_path):
    path = str(tmp_path / "no_such_dir" / "cache.json")
    assert autotune.store({"k": {"radius_batch": 8, "per_call": 1}}, path) is False
    assert autotune.load(path) == {}
