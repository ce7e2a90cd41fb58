"""The tile autotuner's host logic (CPU): candidates, the shared-memory bound, the JSON cache."""
from types import SimpleNamespace

from ggbtddft_b200 import autotune as AT


def test_stage_bound_matches_the_library_formula():
    # 8 W planes of 128 x 32 plus 12 x planes of bn x 32 per stage, within 200 KB, 2..8 stages
    assert [AT.max_stages(bn) for bn in (16, 32, 64)] == [5, 4, 3]


def test_candidates_stop_at_the_first_width_that_covers_the_columns():
    assert {bn for bn, _ in AT.candidates(9)} == {16}
    assert {bn for bn, _ in AT.candidates(30)} == {16, 32}
    assert {bn for bn, _ in AT.candidates(189)} == {16, 32, 64}
    assert all(2 <= st <= AT.max_stages(bn) for bn, st in AT.candidates(189))


def test_candidates_keep_one_radial_cta_per_sm():
    # each CTA holds all 512 tensor-memory columns of its SM: a tile small enough for two CTAs per
    # SM (<= 113 KB) would make the second wait in tcgen05.alloc
    assert AT.candidates(189) == [(16, 3), (16, 4), (16, 5), (32, 3), (32, 4), (64, 3)]
    assert all(2 * (AT.smem_bytes(bn, st) + 1024) > 228 * 1024 for bn, st in AT.candidates(189))
    # the library's built-in choice (the most stages that fit) is always among them
    assert all((bn, AT.max_stages(bn)) in AT.candidates(189) for bn in (16, 32, 64))


def test_tuning_is_timed_once_and_then_read_from_the_cache(tmp_path):
    runs = [SimpleNamespace(n_r=600, n_l=97, n_orb=9) for _ in range(16)] + \
           [SimpleNamespace(n_r=400, n_l=65, n_orb=1)]
    groups = [list(range(16)), [16]]
    calls = []

    def timer(rs, cand):
        calls.append((len(rs), cand))
        return 1.0 + abs(cand[0] - 32) + 0.1 * cand[1]      # fastest: bn 32, fewest stages

    path = str(tmp_path / "tune.json")
    t1 = AT.tuning_for(runs, groups, cache_file=path, timer=timer, device_name="B200")
    assert t1 == {0: (32, 3), 1: (16, 3)}
    n = len(calls)
    assert n == len(AT.candidates(144)) + len(AT.candidates(1))
    t2 = AT.tuning_for(runs, groups, cache_file=path, timer=timer, device_name="B200")
    assert t2 == t1 and len(calls) == n                      # no timing on a cache hit
    cache = AT.load_cache(path)
    key = AT.cache_key(600, 96, 144, "B200")
    assert key in cache and "ms" in cache[key]
    assert AT.library_version() in key                      # old kernels' tunings are not reused
    # another GPU model is tuned on its own
    AT.tuning_for(runs, groups, cache_file=path, timer=timer, device_name="other")
    assert len(calls) == 2 * n


def test_a_corrupt_cache_is_ignored(tmp_path):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    assert AT.load_cache(str(p)) == {}
