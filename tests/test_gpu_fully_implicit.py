"""The opt-in fully-implicit element formulation (the reference's
commented-out "Fully-implicit formulation" routines: SUPG + PSPG, LSIC in 3D,
full Newton tangent) on the GPU against the CPU oracle's restatement of the
same routines.

Tolerances as for the active formulation: element matrices normwise 1e-13,
tangent vs central differences 1e-7, fields after N steps 1e-8 relative L2.
"""
import dataclasses

import numpy as np
import pytest

import oracle
from cfdsfemmpi_b200 import Handle, meshgen

from test_gpu_parity import MESHES, _random_state, _run_gpu

pytestmark = pytest.mark.gpu

FI = "fully_implicit"


def _lsic(ctrl, c=1.0):
    return dataclasses.replace(ctrl, stab=(1.0, 1.0, c))


@pytest.mark.parametrize("kind", list(MESHES))
@pytest.mark.parametrize("tis", [0, 2])
def test_element_matrices_match_oracle(kind, tis):
    mesh = MESHES[kind]()
    ctrl = _lsic(meshgen.control_for(5, 0.1, 0.01, tis=tis))
    h = Handle(mesh, ctrl, formulation=FI)
    prev, cur, dot = _random_state(mesh.nNode * mesh.ndof, 13)
    h.set_element_state(prev, cur, dot)
    K, F = h.element_matrices(np.arange(mesh.nElem, dtype=np.int32))
    h.close()
    td = oracle.time_params(tis, ctrl.rhoInf, ctrl.dt)
    ed = ctrl.elem_data()
    ndof = mesh.ndof
    worstK = worstF = 0.0
    for e in range(mesh.nElem):
        nodes = mesh.conn[e]
        g = (nodes[:, None] * ndof + np.arange(ndof)).ravel()
        Kr, Fr, _, _ = oracle.element(mesh.elem_type, mesh.coords[nodes], prev[g], cur[g], dot[g], ed, td, form=FI)
        worstK = max(worstK, np.abs(K[e] - Kr).max() / np.abs(Kr).max())
        worstF = max(worstF, np.abs(F[e] - Fr).max() / np.abs(Fr).max())
    assert worstK < 1e-13, worstK
    assert worstF < 1e-13, worstF


@pytest.mark.parametrize("kind", list(MESHES))
def test_tangent_is_the_newton_derivative(kind):
    """K of the fully-implicit kernels equals -dF/dsoln (central differences
    through the generalised-alpha chain), LSIC active."""
    mesh = MESHES[kind]()
    ctrl = _lsic(meshgen.control_for(5, 0.1, 0.01, tis=2))
    td = oracle.time_params(2, 0.0, 0.1)
    n = mesh.nNode * mesh.ndof
    rng = np.random.default_rng(23)
    prev = 0.3 * rng.standard_normal(n)
    dotprev = 0.1 * rng.standard_normal(n)
    soln = 0.3 * rng.standard_normal(n)
    h = Handle(mesh, ctrl, formulation=FI)

    def KF(s):
        cur = td[2] * s + (1 - td[2]) * prev
        dot = td[9] * s + td[10] * prev + td[15] * dotprev
        dotcur = td[1] * dot + (1 - td[1]) * dotprev
        h.set_element_state(prev, cur, dotcur)
        return h.element_matrices(np.array([0], np.int32))

    K, _ = KF(soln)
    nodes = mesh.conn[0]
    ndof = mesh.ndof
    g = (nodes[:, None] * ndof + np.arange(ndof)).ravel()
    eps = 1e-6
    Kfd = np.zeros_like(K[0])
    for j, gj in enumerate(g):
        sp = soln.copy(); sm = soln.copy()
        sp[gj] += eps; sm[gj] -= eps
        Kfd[:, j] = -(KF(sp)[1][0] - KF(sm)[1][0]) / (2 * eps)
    h.close()
    assert np.abs(K[0] - Kfd).max() / np.abs(K[0]).max() < 1e-7


def test_ldc2d_matches_oracle_with_genuine_newton():
    """2D cavity (gen-alpha, dt 0.1, 20 steps, GMRES(50)+Jacobi rtol 1e-10),
    fully implicit on both sides: same fields, same Newton iteration counts,
    and Newton takes more than one correction on the nonlinear steps."""
    mesh, ctrl, _ = meshgen.CASES["ldc2d_10"]()
    ref = oracle.OracleFEM(mesh, ctrl, solver="gmres", restart=50, rtol=1e-10, pc="jacobi", form=FI)
    ref.solve()
    s, stats = _run_gpu(mesh, ctrl, restart=50, rtol=1e-10, pc="jacobi", formulation=FI)
    rel = np.linalg.norm(s - ref.soln) / np.linalg.norm(ref.soln)
    assert rel < 1e-8, rel
    assert len(stats) == 20 and all(st["converged"] for st in stats)
    assert [st["newton_iters"] for st in stats] == [len(st["norms"]) for st in ref.stats]
    assert max(st["newton_iters"] for st in stats) > 2


def test_ldc3d_matches_oracle_lu():
    """hex8 cavity 5^3, 2 steps, LSIC on: GMRES(200)+pbjacobi at rtol 1e-12
    against the oracle with a direct solve."""
    mesh, ctrl, _ = meshgen.case_hex(5, 2)
    ctrl = _lsic(ctrl)
    ref = oracle.OracleFEM(mesh, ctrl, solver="lu", form=FI)
    ref.solve()
    s, stats = _run_gpu(mesh, ctrl, restart=200, rtol=1e-12, pc="pbjacobi", formulation=FI)
    rel = np.linalg.norm(s - ref.soln) / np.linalg.norm(ref.soln)
    assert rel < 1e-8, rel
    assert all(st["converged"] for st in stats)


def test_mixed_precision_and_guess_with_fully_implicit():
    """Mixed precision and the extrapolation guess also run the fully-implicit
    formulation: every step converges to the 1e-8 Newton tolerance and the
    velocity agrees with the FP64 run; the guess is kept only where its
    re-assembled residual is lower."""
    mesh, ctrl, _ = meshgen.case_hex(8, 6)
    s64, st64 = _run_gpu(mesh, ctrl, restart=400, rtol=1e-10, pc="pbjacobi", formulation=FI)
    s32, st32 = _run_gpu(mesh, ctrl, restart=30, pc="pbjacobi", precision="mixed", inner_restart=20,
                         inner_rtol=1e-2, max_it=2000, formulation=FI, guess="extrapolation")
    assert all(st["converged"] for st in st64 + st32)
    for st in st32:
        assert st["guess_norm"] <= st["plain_norm"]
    assert any(st["guess_used"] for st in st32)
    a, b = s32.reshape(-1, 4), s64.reshape(-1, 4)
    d = np.linalg.norm(a[:, :3] - b[:, :3]) / np.linalg.norm(b[:, :3])
    assert d < 1e-4, d
