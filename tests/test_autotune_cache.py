"""Host logic of the launch-shape autotuner (walicxe3d_b200/autotune.py):
the workload key, the on-disk cache and its reuse, with a stand-in for the
context (no GPU)."""
import json

from walicxe3d_b200 import autotune, problems


class FakeContext:
    """Records what the tuner asks of a context; autotune() returns a fixed
    measurement as wx3d_autotune would."""

    def __init__(self, best=2, fused=False):
        self.best, self.fused = best, fused
        self.calls, self.zsplit, self.fusion = 0, None, None

    def autotune(self, reps):
        self.calls += 1
        return self.best, self.fused, {"1-fused": 1.5, "1": 1.4, "2": 1.2, "4": 1.3, "8": 1.9}

    def set_zsplit(self, z):
        self.zsplit = z

    def set_fusion(self, on):
        self.fusion = on


def test_signature_counts_blocks_per_level():
    prob = problems.blast_amr(nroot=3, maxlev=3, shell_radius=0.1, shell_width=0.02)
    levels = [prob.tree.level(int(b)) for b in prob.local_blocks]
    key = autotune.signature(prob.cfg, prob.nblocks, levels)
    hist = {l: levels.count(l) for l in set(levels)}
    assert key.endswith("lev" + ",".join(f"{l}:{hist[l]}" for l in sorted(hist)))
    assert f"nb{prob.nblocks}" in key and f"neq{prob.cfg.neqtot}" in key
    # a different level histogram with the same block count is another workload
    other = autotune.signature(prob.cfg, prob.nblocks, sorted(levels)[:-1] + [levels[0] + 5])
    assert other != key


def test_measured_choice_is_cached_and_reused(tmp_path):
    prob = problems.sedov(2)
    cache = tmp_path / "tuning.json"
    first = FakeContext(best=2, fused=False)
    rec = autotune.tune(first, prob, cache=cache, reps=1)
    assert first.calls == 1 and rec["cached"] is False
    assert (rec["zsplit"], rec["fused"]) == (2, False)
    table = json.loads(cache.read_text())
    assert table[rec["key"]]["zsplit"] == 2 and table[rec["key"]]["ms_per_pass"]["2"] == 1.2
    # a second context on the same workload takes the cached shape without measuring
    second = FakeContext(best=8, fused=True)
    rec2 = autotune.tune(second, prob, cache=cache, reps=1)
    assert second.calls == 0 and rec2["cached"] is True
    assert (second.zsplit, second.fusion) == (2, False)
    # force measures again and replaces the record
    third = FakeContext(best=4, fused=False)
    rec3 = autotune.tune(third, prob, cache=cache, reps=1, force=True)
    assert third.calls == 1 and rec3["zsplit"] == 4
    assert json.loads(cache.read_text())[rec3["key"]]["zsplit"] == 4


def test_unreadable_cache_is_measured_over(tmp_path):
    prob = problems.sedov(2)
    cache = tmp_path / "tuning.json"
    cache.write_text("{not json")
    ctx = FakeContext(best=1, fused=True)
    rec = autotune.tune(ctx, prob, cache=cache, reps=1)
    assert ctx.calls == 1 and rec["fused"] is True
    assert json.loads(cache.read_text())[rec["key"]]["fused"] is True


def test_no_cache_always_measures():
    prob = problems.sedov(2)
    ctx = FakeContext()
    autotune.tune(ctx, prob, cache=None, reps=1)
    autotune.tune(ctx, prob, cache=None, reps=1)
    assert ctx.calls == 2
