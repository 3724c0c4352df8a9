"""Autotuner host logic (CPU): search, shape classes, the on-disk cache."""
import json

from vibespatial_b200 import autotune as at


def test_search_finds_the_minimum_of_a_separable_cost():
    target = {"blocks_per_sm": 6, "packets_per_grab": 2, "sort_levels": 10}
    calls = []

    def cost(o):
        calls.append(o)
        return sum((o[k] - target[k]) ** 2 for k in target) + 1.0

    best, ms, tried = at.search(cost)
    assert best == target and ms == 1.0
    # every candidate measured once; far fewer than the full grid
    assert len(calls) == len(tried) == len({tuple(sorted(c.items())) for c in calls})
    full = 1
    for v in at.SPACE.values():
        full *= len(v)
    assert len(calls) < full


def test_search_keeps_defaults_when_nothing_is_faster():
    best, ms, tried = at.search(lambda o: 5.0)
    assert best == at.DEFAULTS and ms == 5.0
    assert tried[0][0] == at.DEFAULTS


def test_shape_class_buckets():
    assert at.shape_class(256, 67_000_000, 1_500_000) == "j8-p17-g12"
    assert at.shape_class(1, 0, 0) == "j0-p0-g0"
    assert at.shape_class(256, 67_000_000, 1_500_000) == at.shape_class(300, 70_000_000, 1_600_000)
    assert at.shape_class(16, 1_000_000, 1000) != at.shape_class(256, 1_000_000, 1000)


def test_cache_round_trip(tmp_path):
    p = tmp_path / "sub" / "tune.json"
    key = at.cache_key("NVIDIA B200", 148, "j8-p17-g12", 2)
    assert at.lookup(key, p) is None
    at.store(key, {"blocks_per_sm": 6, "packets_per_grab": 8, "sort_levels": 10}, 12.5, p)
    at.store(at.cache_key("NVIDIA B200", 148, "j1-p10-g3", 2), at.DEFAULTS, 0.3, p)
    assert at.lookup(key, p) == {"blocks_per_sm": 6, "packets_per_grab": 8, "sort_levels": 10}
    data = json.loads(p.read_text())
    assert len(data) == 2 and data[key]["ms"] == 12.5


def test_cache_tolerates_garbage_and_partial_entries(tmp_path, monkeypatch):
    p = tmp_path / "tune.json"
    p.write_text("not json")
    assert at.load_cache(p) == {}
    p.write_text(json.dumps({"k": {"options": {"sort_levels": 12, "bogus": 1}}}))
    assert at.lookup("k", p) == {**at.DEFAULTS, "sort_levels": 12}
    monkeypatch.setenv(at.CACHE_ENV, str(p))
    assert at.cache_path() == p


def test_learned_space_and_keys(tmp_path):
    """The learned pipeline has its own defaults, search space and cache entries (the R-tree's stay apart)."""
    d, sp = at.space_for(at.METHOD_LEARNED)
    assert d == at.LEARNED_DEFAULTS and sp == at.LEARNED_SPACE
    assert all(d[k] in sp[k] for k in d)
    kr = at.cache_key("NVIDIA B200", 148, "j8-p17-g12", 2)
    kl = at.cache_key("NVIDIA B200", 148, "j8-p17-g12", 2, at.METHOD_LEARNED)
    assert kr != kl
    p = tmp_path / "tune.json"
    at.store(kl, {"learned_map_blocks_per_sm": 4, "learned_refine_blocks_per_sm": 5, "learned_grab": 64}, 3.4, p)
    assert at.lookup(kr, p) is None
    assert at.lookup(kl, p, at.METHOD_LEARNED) == {"learned_map_blocks_per_sm": 4, "learned_map_packets": 1,
                                                   "learned_refine_blocks_per_sm": 5, "learned_grab": 64}
    target = {"learned_map_blocks_per_sm": 4, "learned_map_packets": 2, "learned_refine_blocks_per_sm": 3,
              "learned_grab": 128}
    best, ms, _ = at.search(lambda o: sum((o[k] - target[k]) ** 2 for k in target), space=sp, start=d)
    assert best == target and ms == 0
