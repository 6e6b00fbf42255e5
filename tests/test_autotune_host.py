"""The autotuner's search and cache (no GPU)."""
import collections

from gpudbmetalcodegen_b200 import autotune as A


def test_coordinate_descent_finds_the_separable_minimum():
    space = {"a": [3, 1, 2, 4], "b": ["x", "y", "z"], "c": [0, 1]}
    cost = {"a": {1: 5, 2: 1, 3: 3, 4: 9}, "b": {"x": 4, "y": 1, "z": 2}, "c": {0: 1, 1: 0}}
    calls = []

    def measure(cfg):
        calls.append(dict(cfg))
        if cfg["b"] == "z" and cfg["c"] == 1:
            return None  # an invalid candidate is never chosen
        return sum(cost[k][v] for k, v in cfg.items()) + 10

    log = []
    best, t, t0 = A.coordinate_descent(space, measure, rounds=3, log=log)
    assert best == {"a": 2, "b": "y", "c": 1} and t == 12 and t0 == 3 + 4 + 1 + 10
    assert len(calls) == len({tuple(sorted(c.items())) for c in calls})  # nothing measured twice
    assert len(log) == len(calls) - 1


def test_noise_margin_keeps_the_default():
    best, t, t0 = A.coordinate_descent({"a": [1, 2]}, lambda c: 100.0 if c["a"] == 1 else 99.0)
    assert best == {"a": 1} and t == t0 == 100.0


def test_cache_round_trip_and_size_buckets(tmp_path):
    assert A.size_bucket(6_001_215) == A.size_bucket(10_000_000) != A.size_bucket(60_000_000)
    c = A.TuneCache(tmp_path / "dev.json")
    assert c.get("q1", 6_001_215) is None
    c.put("q1", 6_001_215, "bs=256;stages=2", 0.04, 0.05)
    again = A.TuneCache(tmp_path / "dev.json")
    assert again.get("q1", 7_000_000) == "bs=256;stages=2"
    assert again.get("q1", 100_000_000) is None


def test_seeds_reach_joint_moves():
    # only the joint move (a=1, b=1) is better: one parameter at a time never finds it
    space = {"a": [0, 1], "b": [0, 1]}
    t = {(0, 0): 10.0, (1, 0): 12.0, (0, 1): 12.0, (1, 1): 5.0}
    measure = lambda c: t[(c["a"], c["b"])]
    best, bt, t0 = A.coordinate_descent(space, measure)
    assert best == {"a": 0, "b": 0}
    best, bt, t0 = A.coordinate_descent(space, measure, seeds=[{"a": 1, "b": 1}, {"zzz": 3}])
    assert best == {"a": 1, "b": 1} and bt == 5.0 and t0 == 10.0


def test_every_tuning_the_tuner_can_try_is_a_valid_plan():
    """Each value of each searched parameter, and each seed, parses and
    plans and compiles for its template (no GPU needed)."""
    from gpudbmetalcodegen_b200 import autotune as A
    from gpudbmetalcodegen_b200 import engine
    specs = {"q1": "template=q1", "q6": "template=q6", "join_topk": "template=join_topk",
             "groupby": "template=groupby", "hashjoin": "template=hashjoin"}
    for tpl, space in A.SPACES.items():
        tunes = [f"{k}={v}" for k, vals in space.items() for v in vals]
        tunes += [";".join(f"{k}={v}" for k, v in seed.items()) for seed in A.SEEDS.get(tpl, [])]
        for t in tunes:
            if "layout=bucket8" in t and tpl == "join_topk":
                continue
            q = engine.Query(specs[tpl], t)
            assert "phase 0" in q.plan, (tpl, t)
            q.close()


def _writer(path, i):
    from gpudbmetalcodegen_b200 import autotune as A
    c = A.TuneCache(path)
    for j in range(100):
        c.put("q1", 1000, f"bs={32 * (i + 1)}", float(j), 2.0)
        c.put(f"own{i}", 1000, f"bs={32 * (i + 1)}", float(j), 2.0)


def test_replicas_writing_the_cache_at_once_leave_a_valid_file(tmp_path):
    """Ranks of a multi-GPU run tune concurrently and all write the same
    per-device cache: none may fail, and the file stays readable."""
    import json
    import multiprocessing as mp
    from gpudbmetalcodegen_b200 import autotune as A
    path = tmp_path / "dev.json"
    ps = [mp.get_context("spawn").Process(target=_writer, args=(path, i)) for i in range(4)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    assert [p.exitcode for p in ps] == [0, 0, 0, 0]
    data = json.loads(path.read_text())
    assert data[A.TuneCache.key("q1", 1000)]["tune"] in {f"bs={32 * (i + 1)}" for i in range(4)}
    # each writer's own entry survives the others' writes (merged, not overwritten)
    for i in range(4):
        assert data[A.TuneCache.key(f"own{i}", 1000)]["tune"] == f"bs={32 * (i + 1)}"
    assert not list(tmp_path.glob("*.tmp"))


# ---------------------------------------------------------------------------
# tune_query against a fake context: with a caller's `timer` (the bench hands
# it one that runs each candidate back to back over rotated input copies) the
# timer ranks the candidates, each runs once to check its answer and never
# for timing, and one whose answer differs from the default's is dropped
# however fast its timer says it is
# ---------------------------------------------------------------------------
class FakeQuery:
    def __init__(self, tune):
        self.tune = tune


class FakeResult:
    def __init__(self, rows):
        self.types = ["int64"]
        self.rows = rows


class FakeTiming:
    def __init__(self, ms):
        self.phase_ms = [ms]


class FakeContext:
    """Answers [[7]] ([[8]] for the tunes in `wrong`); each run's single
    phase takes `run_ms[tune]` ms (1 ms when absent)."""

    def __init__(self, wrong=(), run_ms=None):
        self.wrong = set(wrong)
        self.run_ms = run_ms or {}
        self.runs = collections.Counter()

    def prepare(self, spec, tune):
        return FakeQuery(tune)

    def run(self, q, collect=True, **kw):
        self.runs[q.tune] += 1
        return FakeResult([[8]] if q.tune in self.wrong else [[7]]), FakeTiming(self.run_ms.get(q.tune, 1.0))


def test_timer_ranks_candidates_and_answers_still_gate_them():
    space = {"bs": ["512", "256"], "tile": ["0", "448", "512"]}
    # coordinate descent: bs first (256 beats 512 by more than its 2 %
    # margin), then the tile at bs=256
    times = {"bs=512;tile=0": 31.0, "bs=256;tile=0": 29.9, "bs=512;tile=448": 33.0, "bs=512;tile=512": 32.0,
             "bs=256;tile=448": 29.0, "bs=256;tile=512": 20.0}
    ctx = FakeContext(wrong={"bs=256;tile=512"})
    timed = []

    def timer(q):
        timed.append(q.tune)
        return times[q.tune]

    tune, best, default = A.tune_query(ctx, "template=fake_scan", 1000, space=space, rounds=2, timer=timer)
    # the fastest candidate returned a different answer: dropped, never timed
    assert "bs=256;tile=512" not in timed
    assert tune == "bs=256;tile=448" and best == 29.0 and default == 31.0
    # with a timer, every candidate but the default (which also warms the
    # clocks) runs exactly once: the answer check
    assert all(n == 1 for t, n in ctx.runs.items() if t != "bs=512;tile=0")


def test_without_a_timer_candidates_are_timed_by_their_own_runs():
    space = {"bs": ["512", "256", "128"]}
    ctx = FakeContext(run_ms={"bs=512": 2.0, "bs=256": 1.5, "bs=128": 1.0})
    flushes = []
    tune, best, default = A.tune_query(ctx, "template=fake_scan", 1000, space=space, rounds=1, reps=3,
                                       warmup=2, flush=lambda: flushes.append(1))
    assert (tune, best, default) == ("bs=128", 1.0, 2.0)
    # a non-default candidate: the answer check, 2 warm-ups, 3 timed runs,
    # each timed run after a flush
    assert ctx.runs["bs=256"] == ctx.runs["bs=128"] == 6
    assert len(flushes) == 3 * 3
