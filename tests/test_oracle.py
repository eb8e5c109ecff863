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


def _dense_iluk(A, levels, blocks):
    """ILU(levels) of the block-diagonal part of dense A (blocks: row offsets),
    restated from the textbook definition (Saad, Iterative Methods for Sparse
    Linear Systems, ILU(p)): for each row, pivots p in increasing order whose
    level lev(i,p) is within the limit eliminate the whole row (updates reach
    every column), levels update as lev(i,j) = min(lev(i,j), lev(i,p) +
    lev(p,j) + 1) with A's entries at level 0, and entries whose final level
    exceeds the limit are dropped when the row is done."""
    n = A.shape[0]
    W = np.zeros_like(A)
    lev = np.full((n, n), 10 ** 9)
    for b in range(len(blocks) - 1):
        r0, r1 = blocks[b], blocks[b + 1]
        W[r0:r1, r0:r1] = A[r0:r1, r0:r1]
        sub = lev[r0:r1, r0:r1]
        sub[A[r0:r1, r0:r1] != 0] = 0
    for i in range(n):
        for p in range(i):
            if lev[i, p] > levels:
                continue
            W[i, p] /= W[p, p]
            for j in range(p + 1, n):
                if lev[p, j] > levels:
                    continue
                lev[i, j] = min(lev[i, j], lev[i, p] + lev[p, j] + 1)
                W[i, j] -= W[i, p] * W[p, j]
        W[i, lev[i] > levels] = 0.0
    return W, lev <= levels


@pytest.mark.parametrize("levels,blocks", [(0, 1), (1, 1), (2, 1), (1, 3)])
def test_ilu_matches_dense_definition(levels, blocks):
    """The oracle's block-Jacobi ILU(k) (PETSc PCBJACOBI + ILU(levels)) against
    a dense restatement of the level-of-fill definition."""
    import scipy.sparse as sp
    rng = np.random.default_rng(11 + levels)
    n = 40
    A = sp.random(n, n, density=0.12, random_state=rng).toarray()
    A += np.diag(4.0 + rng.random(n))
    Ac = sp.csr_matrix(A)
    Ac.sort_indices()
    rowptr = Ac.indptr.astype(np.int32)
    colidx = Ac.indices.astype(np.int32)
    vals = Ac.data.astype(np.float64)
    q, r = divmod(n, blocks)
    blk = np.array([b * q + min(b, r) for b in range(blocks + 1)], dtype=np.int32)
    L = oracle.lib()
    nnz = L.orc_ilu_symbolic(n, rowptr, colidx, blocks, blk, levels)
    fptr = np.zeros(n + 1, np.int32); fcol = np.zeros(nnz, np.int32); fdg = np.zeros(n, np.int32)
    L.orc_ilu_pattern(fptr.ctypes.data, fcol.ctypes.data, fdg.ctypes.data)
    assert L.orc_ilu_numeric(rowptr, colidx, vals, 1) == 0
    fv = np.zeros(nnz)
    L.orc_ilu_values(fv)
    W, keep = _dense_iluk(A, levels, blk)
    F = np.zeros((n, n))
    pattern = np.zeros((n, n), dtype=bool)
    for i in range(n):
        F[i, fcol[fptr[i]:fptr[i + 1]]] = fv[fptr[i]:fptr[i + 1]]
        pattern[i, fcol[fptr[i]:fptr[i + 1]]] = True
    assert np.array_equal(pattern, keep)
    assert np.abs(F - W).max() <= 1e-13 * np.abs(W).max()
    # applying the factors solves (L U) z = r, with any thread count
    rr = rng.standard_normal(n)
    Lf = np.tril(W, -1) + np.eye(n)
    Uf = np.triu(W)
    zs = []
    for threads in (1, 3):
        z = np.zeros(n)
        L.orc_ilu_apply(rr, z, threads)
        assert np.abs(Lf @ (Uf @ z) - rr).max() <= 1e-12 * np.abs(rr).max()
        zs.append(z)
    assert np.array_equal(zs[0], zs[1])


def test_complete_factorisation_is_a_direct_solve(golden_dir):
    """-ksp_type preonly -pc_type lu (the reference's test options) with the
    oracle's complete factorisation (ILU without a level limit) reproduces the
    10x10 golden like SuperLU does."""
    m, c, ref = _golden(golden_dir, "ldc2dquad10", "LDC2Dquad10", "control-parameters-ldc-Re100.dat",
                        "test-ldc-stru-nelem10-ref.dat")
    fem = oracle.OracleFEM(m, c, solver="preonly", pc="bjacobi", ilu_levels=10 ** 6)
    st = fem.solve()
    assert io.check_result(ref, fem.solution(), m.nNode, 2) == 0
    diff = np.abs(io.read_result(ref) - fem.solution().reshape(-1, 3)).max()
    assert diff < 6e-9
    assert all(s["converged"] and len(s["norms"]) == 2 for s in st)


@pytest.mark.parametrize("solver,levels", [("bcgs", 0), ("bcgs", 1), ("gmres", 1)])
def test_ilu_krylov_matches_lu_2d(solver, levels):
    """The 2D cavity with the reference's iterative option family (BiCGStab or
    GMRES(20) with ILU(k)) against the direct solve: 20 steps at rtol 1e-10."""
    m, c, _ = meshgen.CASES["ldc2d_10"]()
    a = oracle.OracleFEM(m, c, solver=solver, restart=20, rtol=1e-10, pc="bjacobi", ilu_levels=levels)
    a.solve()
    b = oracle.OracleFEM(m, c, solver="lu")
    b.solve()
    rel = np.linalg.norm(a.solution() - b.solution()) / np.linalg.norm(b.solution())
    assert rel < 1e-8
    assert all(s["converged"] for s in a.stats)
