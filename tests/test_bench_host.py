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
