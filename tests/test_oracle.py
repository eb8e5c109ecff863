"""The CPU oracle against the reference's own known-answer tests.

The reference's test drivers (src/test-ldc-stru-nelem10.cpp,
src/test-ldc-stru-mesh2.cpp) run 10 steps with an LU solve and pass when
every node's (u, v, p) lies within 1e-4 of the shipped solution
(StabFEM::checkResult, src/base/StabFEM.cpp:501-554).  The oracle must pass
the same check; it reaches the files' print precision (5e-9).
"""
import os

import numpy as np
import pytest

import oracle
from cfdsfemmpi_b200 import io, meshgen


def _golden(golden_dir, case, mesh, ctrl, ref):
    d = os.path.join(golden_dir, case)
    m = io.read_mesh(os.path.join(d, mesh))
    c = io.read_control(os.path.join(d, ctrl))
    return m, c, os.path.join(d, ref)


def test_kat_ldc2dquad10(golden_dir):
    m, c, ref = _golden(golden_dir, "ldc2dquad10", "LDC2Dquad10", "control-parameters-ldc-Re100.dat",
                        "test-ldc-stru-nelem10-ref.dat")
    assert (m.nNode, m.nElem, m.nDBC) == (121, 100, 81)
    fem = oracle.OracleFEM(m, c, solver="lu")
    st = fem.solve()
    assert len(st) == 10
    assert io.check_result(ref, fem.solution(), m.nNode, 2) == 0
    diff = np.abs(io.read_result(ref) - fem.solution().reshape(-1, 3)).max()
    assert diff < 6e-9
    # every step converges in one linear solve plus one residual check
    assert all(s["converged"] and len(s["norms"]) == 2 for s in st)


@pytest.mark.slow
def test_kat_ldc2dquad_mesh2(golden_dir):
    m, c, ref = _golden(golden_dir, "ldc2dquad-mesh2", "LDC2Dquad-mesh2", "control-parameters-Re1000.dat",
                        "test-ldc-stru-mesh2-ref.dat")
    assert (m.nNode, m.nElem, m.nDBC) == (16641, 16384, 1033)
    fem = oracle.OracleFEM(m, c, solver="lu", threads=8)
    fem.solve()
    assert io.check_result(ref, fem.solution(), m.nNode, 2) == 0
    diff = np.abs(io.read_result(ref) - fem.solution().reshape(-1, 3)).max()
    assert diff < 6e-9


def test_check_result_detects_mismatch(golden_dir, tmp_path):
    m, c, ref = _golden(golden_dir, "ldc2dquad10", "LDC2Dquad10", "control-parameters-ldc-Re100.dat",
                        "test-ldc-stru-nelem10-ref.dat")
    s = io.read_result(ref).ravel().copy()
    assert io.check_result(ref, s, m.nNode, 2) == 0
    s[5 * 3 + 2] += 2e-4
    assert io.check_result(ref, s, m.nNode, 2) == -2
    assert io.check_result(ref, s[:-3], m.nNode - 1, 2) == -1


def test_gmres_matches_lu_2d():
    """The 2D cavity configuration (gen-alpha, GMRES(50)+Jacobi, 20 steps)."""
    m, c, _ = meshgen.CASES["ldc2d_10"]()
    a = oracle.OracleFEM(m, c, solver="gmres", restart=50, rtol=1e-10, pc="jacobi")
    a.solve()
    b = oracle.OracleFEM(m, c, solver="lu")
    b.solve()
    rel = np.linalg.norm(a.solution() - b.solution()) / np.linalg.norm(b.solution())
    assert rel < 1e-8
    assert len(a.stats) == 20
    its = [s["gmres_its"][0] for s in a.stats]
    assert 50 < min(its) and max(its) < 200


@pytest.mark.parametrize("form", ["semi_implicit", "fully_implicit"])
@pytest.mark.parametrize("et", [0, 1, 2, 3])
def test_tangent_matches_finite_difference(et, form):
    """diffStiffTest analogue (src/base/StabFEM.cpp:581-706): K = -dF/dsoln.

    solnCur = af*soln + (1-af)*solnPrev and solnDotCur = am*(td9*soln + ...)
    so dF/dsoln = af dF/dcur + am td9 dF/ddotcur; the element's acceFact td[8]
    equals am*td9 for gen-alpha, so K must match the chain-rule derivative.
    The fully-implicit routine is nonlinear in soln (convection, SUPG weight)
    and its K is the full Newton tangent, LSIC included (active here).
    """
    rng = np.random.default_rng(7 + et)
    ndim, npe, _ = oracle.ELEM_INFO[et]
    ndof = ndim + 1
    ref = {0: [[0, 0], [1, 0], [0, 1]], 1: [[0, 0], [1, 0], [1, 1], [0, 1]],
           2: [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]],
           3: [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]]}[et]
    X = 0.1 * np.array(ref, dtype=float) + 0.01 * rng.standard_normal((npe, ndim))
    td = oracle.time_params(2, 0.0, 0.1)
    ed = np.zeros(50); ed[0] = 1.0; ed[1] = 0.01
    ed[8:11] = (1.0, 1.0, 0.0) if form == "semi_implicit" else (1.0, 1.0, 1.0)
    prev = rng.standard_normal((npe, ndof)) * 0.3
    dotprev = rng.standard_normal((npe, ndof)) * 0.1
    soln = rng.standard_normal((npe, ndof)) * 0.3

    def F_of(s):
        cur = td[2] * s + (1 - td[2]) * prev
        dot = td[9] * s + td[10] * prev + td[15] * dotprev
        dotcur = td[1] * dot + (1 - td[1]) * dotprev
        K, F, info, rc = oracle.element(et, X, prev, cur, dotcur, ed, td, form=form)
        return K, F

    K, _ = F_of(soln)
    h = 1e-6
    n = npe * ndof
    Kfd = np.zeros((n, n))
    for j in range(n):
        sp = soln.copy().ravel(); sm = soln.copy().ravel()
        sp[j] += h; sm[j] -= h
        Kfd[:, j] = -(F_of(sp.reshape(npe, ndof))[1] - F_of(sm.reshape(npe, ndof))[1]) / (2 * h)
    assert np.abs(K - Kfd).max() / np.abs(K).max() < 1e-7
