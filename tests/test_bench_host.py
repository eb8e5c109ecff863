"""Host-side logic of the benchmark and the guess training (no GPU): the
solver and training defaults per workload, the variant list, and the pooled
scales of the shared guess network."""
import sys

import numpy as np

import bench
from cfdsfemmpi_b200.surrogate import fit_scales, fit_scales_pooled


def _parse(*argv):
    old = sys.argv
    sys.argv = ["bench.py", *argv]
    try:
        return bench.parse()
    finally:
        sys.argv = old


def test_workload_defaults():
    a = _parse()
    assert (a.workload, a.solver, a.train_steps) == ("ldc3d_115", "bcgs-ilu0", 20)
    a = _parse("--method", "surrogate", "--workload", "cylinder_wake")
    assert (a.solver, a.train_steps) == ("bcgs-ilu3", 1000)
    a = _parse("--workload", "ldc3d_32", "--solver", "gmres-pbjacobi")
    assert bench.solver_options(a.workload, a.solver)["restart"] == 400


def test_pooled_scales_reduce_to_single_instance_scales():
    rng = np.random.default_rng(1)
    traj = [rng.standard_normal(30) for _ in range(6)]
    a_in, a_out = fit_scales(traj, 3)
    b_in, b_out = fit_scales_pooled([traj], 3)
    assert np.allclose(a_in, b_in, rtol=1e-6) and np.allclose(a_out, b_out, rtol=1e-6)
    # two instances of different sizes: the RMS over all their nodes and steps
    t2 = [rng.standard_normal(12) for _ in range(6)]
    c_in, _ = fit_scales_pooled([traj, t2], 3)
    U = np.concatenate([np.stack(traj[1:]).reshape(-1, 3), np.stack(t2[1:]).reshape(-1, 3)])
    assert np.allclose(c_in[:3], np.sqrt((U ** 2).mean(axis=0)), rtol=1e-6)


def test_labels_and_variants():
    opts = bench.solver_options("ldc3d_115", "bcgs-ilu0")
    assert bench.solver_label(opts) == "BiCGStab + block Jacobi, 1 block(s) of ILU(0), rtol 1e-10"
    assert bench.pc_label(bench.mixed_options(opts)) == "block Jacobi, 1 block(s) of ILU(0)"
    assert set(bench.DEFAULT_VARIANTS["cylinder_wake"]) <= set(bench.GUESS_VARIANTS)


class _FakeHandle:
    def __init__(self, n):
        self.n = n
        self.ndof = 3


class _FakeNet:
    """Stands in for the GPU network: records what train_shared asks of it."""
    made = []

    def __init__(self, handle, seed=0):
        self.handle = handle
        self.samples = []
        self.scales = None
        self.trained = 0
        _FakeNet.made.append(self)

    def set_scales(self, a, b):
        self.scales = (a, b)

    def add_sample(self, u_nm1, u_n, u_np1, handle=None, cond=None):
        self.samples.append((handle, cond, len(u_n)))

    def train(self, k, lr):
        self.trained += k
        return 1.0 / (1 + self.trained)

    def get_params(self):
        return np.zeros(4, np.float32)


def test_shared_training_pools_every_instance(monkeypatch):
    """train_shared puts the network on the instance with the most nodes,
    adds every instance's samples n = first..len-2 on that instance's own
    mesh with its own condition, and runs the requested Adam steps."""
    import cfdsfemmpi_b200.surrogate as sur
    _FakeNet.made.clear()
    monkeypatch.setattr(sur, "Mpnn", _FakeNet)
    hs = [_FakeHandle(12), _FakeHandle(30), _FakeHandle(21)]
    rng = np.random.default_rng(0)
    trajs = [[rng.standard_normal(h.n) for _ in range(6)] for h in hs]
    conds = [0.1, 0.2, 0.3]
    net, shared, losses = sur.train_shared(hs, trajs, conds, iters=40, first=2)
    assert net.handle is hs[1] and len(_FakeNet.made) == 1
    # 3 samples per instance (n = 2, 3, 4 of 6 states); the owner's own samples carry no handle
    assert len(net.samples) == 9
    for (h, c, n), k in zip(net.samples, [0, 0, 0, 1, 1, 1, 2, 2, 2]):
        assert c == conds[k] and n == hs[k].n
        assert (h is None) == (k == 1) and (h is None or h is hs[k])
    assert net.trained == 40 and len(losses) == 20
    assert shared[1] is net.scales[0] and shared[2] is net.scales[1]
