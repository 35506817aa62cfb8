"""The batched form's autotuner on the host (`lumenwright_b200/batch.py`): against a stand-in
context whose trial times are set per tuning, it times every candidate on the cut-down trial
batch, keeps the fastest, caches it per workload class and serves it from the cache afterwards.
CPU only: the stand-in launches nothing."""

import json

from lumenwright_b200 import batch as BT
from lumenwright_b200 import layout as L


class TrialContext:
    """Records what the tuner asks for; a batch run "takes" the time `cost` gives its tuning."""

    def __init__(self, cost):
        self.cost = cost
        self.tuning = {"threads": 128, "budget": 0, "sub": 0, "engine": 0, "paths": 0}
        self.prepared = []
        self.runs = 0
        self.last_ms = 0.0

    def set_tuning(self, **t):
        self.tuning.update(t)

    def get_tuning(self):
        return dict(self.tuning)

    def batch_prepare(self, jobs):
        self.prepared.append([spp for _, _, spp in jobs])

    def batch_run(self):
        self.runs += 1
        self.last_ms = self.cost(self.tuning)

    def stats(self):
        return {"kernel_ms": self.last_ms}


def jobs(sizes_spp):
    out = []
    for (w, h, bounces), spp in sizes_spp:
        p = L.new_params()
        p["frame"] = [w, h, 0, bounces]
        out.append((p, None, spp))
    return out


def key(t):
    return (t["engine"], t["threads"], t["budget"], t["sub"], t["paths"])


def test_the_fastest_trial_is_kept_and_cached(tmp_path):
    cands = BT.Autotuner.candidates()
    fastest = cands[7]
    cost = lambda t: 1.0 if key(t) == key(fastest) else 2.0 + 0.01 * t["threads"]  # noqa: E731
    ctx = TrialContext(cost)
    work = jobs([((320, 180, 4), 64), ((1920, 1080, 8), 16), ((640, 360, 6), 1)])
    tuner = BT.Autotuner(ctx, cache_dir=str(tmp_path), trial_fraction=1 / 32)
    best, entry = tuner.tune(work)
    assert best == fastest and ctx.get_tuning() == fastest
    # every candidate is tried once warm and once timed, on spp cut to 1/32 (at least 1)
    assert len(entry["trials"]) == len(cands) and ctx.runs == 2 * len(cands)
    assert ctx.prepared[0] == [2, 1, 1]
    table = json.load(open(tmp_path / "autotune.json"))
    h, k = BT.Autotuner.workload_class(work)
    assert table[h]["key"] == k and table[h]["tuning"] == fastest and table[h]["trial_ms"] == 1.0

    # A new tuner over the same cache serves the workload class without a trial and sets it.
    ctx2 = TrialContext(cost)
    best2, _ = BT.Autotuner(ctx2, cache_dir=str(tmp_path)).tune(work)
    assert best2 == fastest and ctx2.runs == 0 and ctx2.get_tuning() == fastest

    # force: the trials run again (here another candidate has become the fastest)
    other = cands[0]
    ctx3 = TrialContext(lambda t: 0.5 if key(t) == key(other) else 3.0)
    best3, _ = BT.Autotuner(ctx3, cache_dir=str(tmp_path)).tune(work, force=True)
    assert best3 == other and ctx3.runs == 2 * len(cands)


def test_workload_classes_follow_size_samples_and_bounces():
    a = jobs([((320, 180, 4), 64), ((640, 360, 8), 16)])
    same = jobs([((640, 360, 8), 16), ((320, 180, 4), 64)])  # the same cameras in another order
    more_spp = jobs([((320, 180, 4), 256), ((640, 360, 8), 64)])
    other_bounces = jobs([((320, 180, 4), 64), ((640, 360, 6), 16)])
    c = BT.Autotuner.workload_class
    assert c(a) == c(same)
    assert c(a)[0] != c(more_spp)[0] and c(a)[0] != c(other_bounces)[0]
