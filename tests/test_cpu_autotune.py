"""The batched-launch autotuner's host logic (krans_b200/autotune.py): the
table file format and its checks, the device key, and the coordinate search,
with a stand-in for the GPU measurement."""
import json

import pytest

from krans_b200 import autotune as T


def test_device_key_and_path():
    assert T.device_key("NVIDIA B200", 148) == "NVIDIA_B200_148sm"
    assert T.table_path("NVIDIA B200", 148).endswith("tuning/NVIDIA_B200_148sm.json")


def test_search_keeps_only_clear_wins():
    # a stand-in speed model: clusters of 8 best, cluster_min 8192 3% faster,
    # pair_max 60000 1% faster (below the margin), lanes[1] = 4 5% faster
    def speed(k):
        v = 100.0
        v *= 1.0 if k["cluster_size"] == 8 else 0.8
        v *= 1.03 if k["cluster_min"] == 8192 else 1.0
        v *= 1.01 if k["pair_max"] == 60000 else 1.0
        v *= 1.05 if k["lanes"][1] == 4 else 1.0
        return v
    best, v, trials = T.search(speed, T.DEFAULTS)
    assert best == {"cluster_min": 8192, "pair_max": 120000, "cluster_size": 8, "lanes": [1, 4, 4, 8, 16, 32]}
    assert abs(v - 100 * 1.03 * 1.05) < 1e-9
    assert trials[0]["knobs"] == T.DEFAULTS
    assert len({json.dumps(t["knobs"], sort_keys=True) for t in trials}) == len(trials)  # no repeats
    assert T.DEFAULTS["lanes"] == [1, 2, 4, 8, 16, 32]  # the start point is not modified


def test_table_round_trip(tmp_path, monkeypatch):
    monkeypatch.setattr(T, "TABLE_DIR", str(tmp_path))
    table = {"device": "NVIDIA B200", "sms": 148, "library": "x", "knobs": dict(T.DEFAULTS, cluster_min=8192),
             "trials": []}
    p = T.save(table)
    t = T.load("NVIDIA B200", 148)
    assert p.endswith("NVIDIA_B200_148sm.json") and t["knobs"]["cluster_min"] == 8192
    assert T.load("Other GPU", 10) is None

    class FakeCtx:
        calls = []

        def set_batch_tuning(self, **kw):
            self.calls.append(kw)
    ctx = FakeCtx()
    T.apply(ctx, t["knobs"])
    assert ctx.calls == [{"cluster_min": 8192, "pair_max": 120000, "cluster_size": 8, "lanes": [1, 2, 4, 8, 16, 32]}]


@pytest.mark.parametrize("bad", [{"lanes": [1, 2, 3, 8, 16, 32]}, {"lanes": [1, 2]}, {"cluster_size": 17},
                                 {"cluster_min": 0}])
def test_table_checks(bad):
    with pytest.raises(ValueError):
        T.validate({"knobs": dict(T.DEFAULTS, **bad)})
