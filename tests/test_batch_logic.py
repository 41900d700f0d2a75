"""Host logic of the batched-realization measurement, without a device: with
tuning on, every shape is measured before the timed legs start, and both the
plain and the batched leg launch every job with the tuned choice at the
measured ring depth."""
import numpy as np
import pytest

from oidt_b200 import batch as B
from oidt_b200 import tune

SMALL = dict(nf=3, P=4, src_gap=2, port_gap=3, core_x_nm=120, core_y_nm=160)


def _configs(n, master_seed=0, steps=200):
    rng = np.random.default_rng(master_seed)
    return [dict(nx=int(rng.choice([20, 22])), ny=19, nz=int(rng.integers(40, 48)), sigma_nm=10.0, lc_nm=50.0,
                 seed=r, steps=steps) for r in range(n)]


class _Job:
    _next = 1

    def __init__(self, eng, spec):
        self.eng, self.spec, self.steps = eng, spec, 0
        self.id = _Job._next
        _Job._next += 1

    def advance(self, n):
        self.steps += n
        return self

    def run(self):
        return self.advance(self.spec.nt - self.steps)

    def sync(self, timeout_ms=-1):
        return self

    def port_power(self, port, minus=None, window=None):
        return np.full(self.spec.nf, 0.25 if minus is not None else 1.0 + port, complex)

    def release(self):
        pass


class _Engine:
    def __init__(self, log):
        self.log = log

    def submit(self, spec, **kw):
        self.log.append(("submit", kw))
        return _Job(self, spec)

    def batch_advance(self, jobs, n):
        for j in jobs:
            j.advance(n)


@pytest.mark.parametrize("ring", [32, 64])
def test_measure_tunes_first_and_both_legs_use_the_choice(monkeypatch, ring):
    log = []
    times = {"wave": 0.96, "vec": 0.95, "cell/rows4": 1.0, "cell/rows2": 1.1, "cell/rows8": 0.9, "sweep/depth-auto": 2.0,
             "sweep/depth16": 2.0}

    def fake_time(self, spec, choice, precision=None, arith="fast", ring_steps=32):
        log.append(("tune", ring_steps))
        return times[tune.label(choice)]

    monkeypatch.setattr(tune.Tuner, "time_choice", fake_time)
    monkeypatch.setattr(B.W, "batch_configs", lambda n=64, master_seed=0, steps=3000: _configs(n, master_seed))
    orig = B.realization_set
    monkeypatch.setattr(B, "realization_set", lambda configs, nf=41, **kw: orig(configs, **SMALL))
    out = B.measure(_Engine(log), n=5, steps=200, ring_steps=ring)
    first_submit = next(i for i, e in enumerate(log) if e[0] == "submit")
    assert all(e[0] == "submit" for e in log[first_submit:]), "tuning ran inside a timed leg"
    assert all(e[1] == ring for e in log if e[0] == "tune")
    subs = [e[1] for e in log if e[0] == "submit"]
    plain = [k for k in subs if k.get("graphs") is False]
    batched = [k for k in subs if "graphs" not in k]
    assert len(plain) == 2 * 5 and len(batched) == 5 + out["shared_incident_runs"]
    for k in subs:
        assert k["ring_steps"] == ring and k["variant"] == "cell" and k["rows"] == 8
    assert out["launch_tuning"]["choices"] == {"cell/rows8": len(batched)}
    assert out["max_abs_dS21_batched_vs_plain"] == 0.0
    assert set(out["s21_loss_db_percentiles"]) == {"0", "5", "25", "50", "75", "95", "100"}
