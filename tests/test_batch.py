"""Batched stepping of independent instances: every instance computes bit for
bit what its own handle computes alone, whatever the schedule (autotuned or
fixed concurrency and Arnoldi chunk length)."""
import numpy as np
import pytest

from cfdsfemmpi_b200 import Batch, Handle, meshgen

pytestmark = pytest.mark.gpu

KW = dict(restart=50, rtol=1e-10, pc="jacobi")


def _cases():
    sizes = [8, 20, 10, 16, 12, 14]
    res = [100.0, 400.0, 1000.0, 250.0, 2500.0, 150.0]
    return [(meshgen.cavity2d(n), meshgen.control_for(20, 0.05, 1.0 / re)) for n, re in zip(sizes, res)]


def _alone(cases, steps):
    out = []
    for mesh, ctrl in cases:
        h = Handle(mesh, ctrl, **KW)
        st = []
        t = ctrl.dt
        for _ in range(steps):
            st.append(h.step(t, min(t, 1.0)).as_dict())
            t += ctrl.dt
        out.append((h.get_solution(), st))
        h.close()
    return out


@pytest.mark.parametrize("schedule", [(0, 0, 0), (2, 3, 1), (1, 8, 2), (6, 4, 4)])
def test_batch_matches_single_instance_runs_bitwise(schedule):
    cases = _cases()
    steps = 6
    ref = _alone(cases, steps)
    b = Batch(cases, **KW)
    b.set_schedule(*schedule)
    t = np.full(len(cases), cases[0][1].dt)
    stats, lats = [], []
    for _ in range(steps):
        st, lat = b.step(t)
        stats.append([s.as_dict() for s in st])
        lats.append(lat)
        t = t + cases[0][1].dt
    sched = b.schedule()
    sols = [h.get_solution() for h in b.handles]
    b.close()
    for i, (sol, st_ref) in enumerate(ref):
        assert np.array_equal(sols[i], sol), i
        for k in range(steps):
            a, r = stats[k][i], st_ref[k]
            assert a["newton_iters"] == r["newton_iters"] and a["ksp_its"] == r["ksp_its"], (i, k)
            assert a["norms"] == r["norms"], (i, k)
    assert all(np.all(l > 0) for l in lats)
    if schedule == (0, 0, 0):
        # 6 instances: one concurrency candidate (6) x chunks (4, 8) x depths (1, 2, 4)
        assert sched["tuned"] and sched["concurrency"] == 6 and sched["chunk"] in (4, 8)
        assert sched["depth"] in (1, 2, 4)
    else:
        assert sched == {"concurrency": schedule[0], "chunk": schedule[1], "depth": schedule[2], "tuned": True}


def test_batch_reports_the_failing_instance():
    """An instance whose solve cannot converge (max_it 1) makes the batch step
    fail with that instance's error; the others are unaffected."""
    cases = _cases()[:3]
    b = Batch(cases, restart=50, rtol=1e-10, pc="jacobi", max_it=1)
    b.set_schedule(3, 8, 1)
    with pytest.raises(Exception) as e:
        b.step(np.full(3, 0.05))
    assert "instance 0" in str(e.value) and "KSP" in str(e.value)
    b.close()
