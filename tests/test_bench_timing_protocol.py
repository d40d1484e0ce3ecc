"""bench.py's timing protocol, checked on the CPU with a stand-in for the
simulation: each timed region (the K steps of a precision form, the K
end-to-end steps) opens with a drained solver stream and the ranks'
barrier before its start event and closes with its end event, a drained
stream and the barrier again; the region holds exactly K steps; its time
is the device time between the two events."""
import bench


class FakeStats:
    def __init__(self):
        self.pp_iters_total = 150
        self.pp_solves = 3
        self.helm_iters_total = 60
        self.guess_used = 0
        self.guess_evaluated = 0
        self.step_dt = 0.05
        self.cfl_adv = 0.4
        self.guess_r0 = 0.0
        self.extrap_r0 = 0.0
        self.lamb_iters = 3
        self.pp_outer_last = 2
        self.guess_cost_ms = 0.0
        self.guess_benefit_ms = 0.0


class FakeLib:
    def __init__(self, log):
        self.log = log
        self.marks = {}
        self.clock = 0.0

    def bbb_mark(self, i):
        self.log.append(("mark", i))
        self.marks[i] = self.clock

    def bbb_mark_elapsed(self, a, b):
        self.log.append(("elapsed", a, b))
        return self.marks[b] - self.marks[a]

    def bbb_kernel_launches(self):
        return 0

    def bbb_profile_reset(self):
        pass

    def bbb_profile_enable(self, on):
        pass

    def bbb_profile_get(self, ms, iters, byts):
        ms._obj.value, iters._obj.value, byts._obj.value = 1.0, 10, 1e9

    def bbb_profile_get_pass(self, k, ms, n, byts):
        ms._obj.value, n._obj.value, byts._obj.value = 1.0, 4, 1e9

    def bbb_part_state_pull(self):
        self.log.append(("pull",))

    def bbb_part_state_push(self):
        self.log.append(("push",))


class FakeDom:
    xn, yn, zn = 8, 8, 8


class FakeSim:
    def __init__(self, log):
        self.log = log
        self.lib = FakeLib(log)
        self.nparts = 0
        self.dom = FakeDom()

    def prepare(self):
        self.log.append(("prepare",))

    def step(self):
        self.log.append(("step",))
        self.lib.clock += 10.0       # device ms per step

    def stats(self):
        return FakeStats()

    def parts(self):
        return []

    def scalar(self, name):
        return 0.05

    def status(self):
        return 0

    def close(self):
        self.log.append(("close",))


def _run(monkeypatch, steps, warmup, e2e):
    import bluebottle_b200
    log = []
    monkeypatch.setattr(bluebottle_b200, "Sim", lambda wl, options=None: FakeSim(log))
    monkeypatch.setattr(bench, "workload", lambda name, prec: None)
    out = bench.run_form(1, steps, warmup, e2e_steps=e2e, profile=True,
                         learned=False, barrier=lambda: log.append(("barrier",)))
    return out, log


def _region(log, start, end):
    i0 = log.index(("mark", start))
    i1 = log.index(("mark", end))
    # drained stream and barrier just before the start event
    assert log[i0 - 3:i0] == [("mark", 5), ("elapsed", 5, 5), ("barrier",)]
    # drained stream and barrier just after the end event
    assert log[i1 + 1:i1 + 4] == [("mark", 5), ("elapsed", 5, 5), ("barrier",)]
    return log[i0 + 1:i1]


def test_timed_regions_are_bracketed(monkeypatch):
    out, log = _run(monkeypatch, steps=4, warmup=3, e2e=2)
    timed = _region(log, 0, 1)
    assert timed.count(("step",)) == 4
    assert out["ms"] == 40.0
    e2e = _region(log, 2, 3)
    assert e2e.count(("step",)) == 2
    assert e2e.count(("push",)) == 2 and e2e.count(("pull",)) == 2
    assert out["e2e_ms"] == 20.0
    # the warm-up and probe steps, and only they, come before the region
    assert log[:log.index(("mark", 0))].count(("step",)) == 3 + bench.PROBE_STEPS
    assert log.count(("barrier",)) == 4


def test_no_end_to_end_steps_still_pairs_barriers(monkeypatch):
    out, log = _run(monkeypatch, steps=2, warmup=3, e2e=0)
    assert _region(log, 2, 3) == []
    assert log.count(("barrier",)) == 4
    assert out["ms"] == 20.0
