"""The ensemble's output loop (Ensemble.run, main.cpp's loop for every
instance) on fake instances: outputs at every dtoutput up to tmax, a last
shorter interval, and instances that stop early (their step limit) no longer
hold the loop."""
from gaukuk_b200.ensemble import Ensemble


class FakeInstance:
    def __init__(self, stop_at=None):
        self.t = 0.0
        self.stop_at = stop_at
        self.is_continue = True

    def get_time(self):
        return self.t

    def advance(self, dtoutput):
        if not self.is_continue:
            return
        self.t += dtoutput
        if self.stop_at is not None and self.t >= self.stop_at - 1e-12:
            self.is_continue = False


def _ensemble(sims):
    e = Ensemble.__new__(Ensemble)  # no device: the loop only
    e.sims = sims
    e.calls = []

    def advance(dt):
        e.calls.append(dt)
        for s in sims:
            if abs(1.0 - s.t) > 1e-12 and s.is_continue:
                s.advance(dt)

    e.advance = advance
    return e


def test_outputs_every_interval_then_a_shorter_last_one():
    sims = [FakeInstance(), FakeInstance()]
    e = _ensemble(sims)
    e.run(1.0, 0.3)
    assert len(e.calls) == 4 and e.calls[:3] == [0.3] * 3
    assert abs(e.calls[3] - 0.1) < 1e-12
    assert all(abs(s.t - 1.0) < 1e-12 for s in sims)


def test_an_instance_that_stops_early_does_not_hold_the_loop():
    sims = [FakeInstance(stop_at=0.5), FakeInstance()]
    e = _ensemble(sims)
    e.run(1.0, 0.25)
    assert e.calls == [0.25] * 4
    assert sims[0].t == 0.5 and not sims[0].is_continue and sims[1].t == 1.0


def test_no_dtoutput_is_one_interval():
    sims = [FakeInstance()]
    e = _ensemble(sims)
    e.run(1.0)
    assert e.calls == [1.0]
