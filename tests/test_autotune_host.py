"""The autotuner's host logic without a GPU (no counterpart in the
reference): the shape bucket (keyed by the GPU's name), the choice of the
fastest candidate, the JSON cache (a cached bucket is applied without
timing, only on the GPU type that wrote it; buckets written by another tuner
are kept), on a fake generator whose Bellman-Ford time depends on the team
shape."""
import json

import pytest


class FakeGenerator:
    def __init__(self, nodes=300, layers=100, intra=10, times=None, auto=(57, 640), gpu="NVIDIA B200"):
        self.gpu = gpu
        self.info = {"nodes_per_layer": nodes, "layers": layers, "intra_edges_per_layer": intra}
        self.times = times or {}
        self.auto = auto
        self.shape = (0, 0)
        self.applied = []
        self.solves = 0

    def device_name(self):
        return self.gpu

    def graph_info(self):
        return dict(self.info)

    def set_team_shape(self, ctas, threads):
        self.shape = (int(ctas), int(threads))
        self.applied.append(self.shape)

    def generate(self):
        pass

    def solve_with_cost_time_ratio(self, name, k):
        assert name == "lawlergpu"
        self.solves += 1
        return True, 0.5, None

    def last_stats(self):
        return {"device_us": 1000.0 * self.times.get(self.shape, 10.0)}

    def last_profile(self):
        ctas, threads = self.shape
        return {"ctas": ctas or self.auto[0], "threads": threads or self.auto[1]}


def test_bucket_and_fastest_candidate(cpg, tmp_path):
    g = FakeGenerator(nodes=300, layers=100, intra=10, times={(0, 0): 5.0, (8, 320): 3.0, (16, 640): 4.0})
    e = cpg.autotune(g, 3, candidates=[(0, 0), (8, 320), (16, 640)], cache_path=str(tmp_path / "c.json"), repeats=2)
    assert e["bucket"] == "NVIDIA B200|n512-l128-k3-intra1" and not e["cached"]
    assert (e["ctas"], e["threads_per_cta"], e["bf_ms"]) == (8, 320, 3.0)
    assert g.shape == (8, 320) and g.solves == 6
    assert [c["bf_ms"] for c in e["candidates"]] == [5.0, 3.0, 4.0]
    assert e["candidates"][0]["team"] == [57, 640]


def test_default_candidates_follow_the_automatic_shape(cpg):
    g = FakeGenerator(times={(57, 480): 1.0}, auto=(57, 640))
    e = cpg.autotune(g, 2, repeats=1)
    assert [(c["ctas"], c["threads_per_cta"]) for c in e["candidates"]] == [(0, 0), (57, 320), (57, 480), (28, 640)]
    assert g.shape == (57, 480)


def test_cache_hit_applies_without_timing(cpg, tmp_path):
    cache = tmp_path / "c.json"
    g = FakeGenerator(times={(8, 320): 1.0})
    cpg.autotune(g, 3, candidates=[(0, 0), (8, 320)], cache_path=str(cache))
    g2 = FakeGenerator(nodes=400, layers=65, intra=1)  # the same bucket
    e = cpg.autotune(g2, 3, candidates=[(0, 0)], cache_path=str(cache))
    assert e["cached"] and e["bucket"] == "NVIDIA B200|n512-l128-k3-intra1"
    assert g2.solves == 0 and g2.applied == [(8, 320)]


def test_cache_of_another_gpu_type_is_not_applied(cpg, tmp_path):
    cache = tmp_path / "c.json"
    cpg.autotune(FakeGenerator(gpu="NVIDIA H100 80GB HBM3", times={(8, 320): 1.0}), 3,
                 candidates=[(0, 0), (8, 320)], cache_path=str(cache))
    g = FakeGenerator(times={(16, 640): 1.0})  # the same shape bucket on a B200
    e = cpg.autotune(g, 3, candidates=[(0, 0), (16, 640)], cache_path=str(cache))
    assert not e["cached"] and e["bucket"] == "NVIDIA B200|n512-l128-k3-intra1"
    assert g.solves == 4 and g.shape == (16, 640)
    assert set(json.loads(cache.read_text())) == {"NVIDIA H100 80GB HBM3|n512-l128-k3-intra1",
                                                  "NVIDIA B200|n512-l128-k3-intra1"}


def test_buckets_of_other_tuners_are_kept(cpg, tmp_path):
    cache = tmp_path / "c.json"
    a, b = FakeGenerator(), FakeGenerator(intra=0)
    cpg.autotune(a, 3, candidates=[(0, 0)], cache_path=str(cache))
    # another tuner adds a bucket after this one read the file
    other = json.loads(cache.read_text())
    other["NVIDIA B200|n8-l8-k1-intra0"] = {"ctas": 1, "threads_per_cta": 32, "bf_ms": 0.1, "candidates": []}
    cache.write_text(json.dumps(other))
    cpg.autotune(b, 3, candidates=[(0, 0)], cache_path=str(cache))
    keys = set(json.loads(cache.read_text()))
    assert keys == {"NVIDIA B200|n512-l128-k3-intra1", "NVIDIA B200|n512-l128-k3-intra0", "NVIDIA B200|n8-l8-k1-intra0"}
    assert sorted(p.name for p in tmp_path.iterdir()) == ["c.json"]


@pytest.mark.parametrize("n,want", [(1, 1), (2, 2), (3, 4), (32, 32), (33, 64), (89964, 131072)])
def test_bucket_rounds_up_to_powers_of_two(cpg, n, want):
    g = FakeGenerator(nodes=n, layers=n, intra=0)
    e = cpg.autotune(g, None, candidates=[(0, 0)], repeats=1)
    assert e["bucket"] == f"NVIDIA B200|n{want}-l{want}-kNone-intra0"
