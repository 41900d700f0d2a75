"""Served mix on the GPU: every job's result served in the mix equals the
same job run alone (the served path advances jobs together in multi-job
graph launches), and a tight HBM budget delays admission without changing
results."""
import numpy as np
import pytest

from oidt_b200 import workloads as W
from oidt_b200.serve import Request, Server

pytestmark = pytest.mark.gpu


def _requests():
    specs = [
        W.slab2d(nx=300, ny=150, P=8, core_cells=10, src_x=20, ports=(40, 260), steps=600, nf=5, rough=True,
                 sigma_nm=10, lc_nm=40, seed=1, precision=np.float32),
        W.strip3d(nx=48, ny=40, nz=96, P=6, src_gap=3, port_gap=6, steps=500, nf=5, seed=2),
        W.slab2d(nx=360, ny=170, P=8, core_cells=10, src_x=20, ports=(40, 320), steps=700, nf=5, rough=True,
                 sigma_nm=12, lc_nm=60, seed=3, precision=np.float32),
        W.strip3d(nx=56, ny=48, nz=120, P=6, src_gap=3, port_gap=6, steps=640, nf=5, seed=4),
    ]
    return [Request(k, arrival=0.05 * k, spec=s) for k, s in enumerate(specs)]


def _solo(eng, spec):
    j = eng.submit(spec, precision=np.float32)
    j.run().sync(120000)
    nc = 4 if spec.mode == "yee3d" else 2
    out = {(p, c): j.dft(p, c) for p in (0, 1) for c in range(nc)}
    j.release()
    return out


# (budget, realtime): all requests at once in one mix; arrivals honoured on
# the wall clock; all at once with room for one job (admission must wait).
@pytest.mark.parametrize("budget_jobs,realtime", [(0, False), (0, True), (1, False)])
def test_served_equals_alone(budget_jobs, realtime):
    from oidt_b200.engine import Engine
    reqs = _requests()
    probe = Engine(0)
    sizes = [probe.job_bytes(r.spec, precision=np.float32) for r in reqs]
    alone = [_solo(probe, r.spec) for r in reqs]
    probe.close()
    budget = 0 if budget_jobs == 0 else max(sizes) + 1  # room for one job at a time
    eng = Engine(0, hbm_budget=budget)
    srv = Server(eng, tick=64, keep_dfts=True)
    res = srv.run(reqs, realtime=realtime, max_wall=120)
    eng.close()
    assert sorted(r.rid for r in res) == list(range(len(reqs)))
    for r in res:
        for k, v in alone[r.rid].items():
            np.testing.assert_array_equal(r.dfts[k], v)
    if budget_jobs:
        assert srv.refused > 0
