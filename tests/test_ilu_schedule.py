"""Host-only checks of the block ILU(k) symbolic phase and of the schedules
the persistent factorisation and triangular-solve kernels run on.

Those kernels hand out rows (factorisation) or chains of rows (solves) from
an atomic ticket and let a task spin, with a bounded wait, until its inputs
are written.  They make progress only if every input of a task belongs to a
task handed out earlier.  These tests check that invariant, and the shape
of the chains, on the library's own host builder (cfdgpu_ilu_pattern_build),
for ILU(0), ILU(1), ILU(3), block Jacobi and the complete factorisation
(reverse Cuthill-McKee order), on 2D and 3D meshes, a randomly renumbered
mesh and the cylinder O-grid.  No GPU is needed.
"""
import numpy as np
import pytest

from cfdsfemmpi_b200 import io, meshgen, pattern_build
from cfdsfemmpi_b200._lib import ilu_pattern_build

CHAIN_MAX = 128


def _renumbered(mesh, seed):
    rng = np.random.default_rng(seed)
    p = rng.permutation(mesh.nNode)          # new id of old node
    coords = np.empty_like(mesh.coords)
    coords[p] = mesh.coords
    dbc = mesh.dbc.copy()
    dbc[:, 0] = p[mesh.dbc[:, 0].astype(int)]
    return io.Mesh(ndim=mesh.ndim, npElem=mesh.npElem, coords=coords, conn=p[mesh.conn].astype(np.int32), dbc=dbc,
                   output_nodes=mesh.output_nodes)


MESHES = {
    "quad4_9": lambda: meshgen.cavity2d(9),
    "hex8_5": lambda: meshgen.cavity3d(5),
    "hex8_4_renumbered": lambda: _renumbered(meshgen.cavity3d(4), 3),
    "ogrid_32x8": lambda: meshgen.cylinder_ogrid(nt=32, nr=8),
}


def _rows(d):
    rp, ci = d["rowptr"], d["colidx"]
    return [ci[rp[i]:rp[i + 1]] for i in range(len(rp) - 1)]


def _check_order(order, deps, n):
    assert sorted(order.tolist()) == list(range(n))
    pos = np.empty(n, np.int64)
    pos[order] = np.arange(n)
    for i in range(n):
        for p in deps[i]:
            assert pos[p] < pos[i], (i, p)


def _check_chains(chains, chain_order, deps, n, upper):
    # consecutive runs covering every row once, at most CHAIN_MAX rows each
    lo_sorted = chains[np.argsort(chains[:, 0])]
    assert lo_sorted[0, 0] == 0 and lo_sorted[-1, 1] == n
    assert np.all(lo_sorted[1:, 0] == lo_sorted[:-1, 1])
    assert np.all(lo_sorted[:, 1] > lo_sorted[:, 0]) and np.all(lo_sorted[:, 1] - lo_sorted[:, 0] <= CHAIN_MAX)
    chain_of = np.empty(n, np.int64)
    for c, (lo, hi) in enumerate(chains):
        chain_of[lo:hi] = c
        # each row of a chain depends on the row solved before it
        for i in range(lo, hi):
            prev = i + 1 if upper else i - 1
            if (upper and i < hi - 1) or (not upper and i > lo):
                assert prev in set(deps[i].tolist()), (lo, hi, i)
    # every input from another chain lies in a chain handed out earlier
    assert sorted(chain_order.tolist()) == list(range(len(chains)))
    pos = np.empty(len(chains), np.int64)
    pos[chain_order] = np.arange(len(chains))
    for i in range(n):
        for p in deps[i]:
            if chain_of[p] != chain_of[i]:
                assert pos[chain_of[p]] < pos[chain_of[i]], (i, p)


@pytest.mark.parametrize("kind", list(MESHES))
@pytest.mark.parametrize("levels,blocks", [(0, 1), (1, 1), (3, 1), (1, 3), (-1, 1)])
def test_schedules_hand_out_every_input_first(kind, levels, blocks):
    mesh = MESHES[kind]()
    d = ilu_pattern_build(mesh, levels, blocks)
    n = mesh.nNode
    rows = _rows(d)
    assert len(rows) == n
    for i, r in enumerate(rows):
        assert np.all(np.diff(r) > 0) and i in set(r.tolist()), i
    lower = [r[r < i] for i, r in enumerate(rows)]
    upper = [r[r > i] for i, r in enumerate(rows)]
    assert sorted(d["perm"].tolist()) == list(range(n))
    _check_order(d["lorder"], lower, n)
    _check_order(d["uorder"], upper, n)
    _check_chains(d["lchain"], d["lchain_order"], lower, n, upper=False)
    _check_chains(d["uchain"], d["uchain_order"], upper, n, upper=True)
    info = d["info"]
    assert info.nlev_l >= 1 and info.chain_levels_l >= 1 and info.nnzb == len(d["colidx"])


@pytest.mark.parametrize("kind", ["quad4_9", "hex8_5", "ogrid_32x8"])
def test_ilu0_keeps_the_matrix_pattern_and_fill_grows_with_levels(kind):
    """ILU(0) in natural order has the node graph's pattern (a node whose
    every dof is prescribed keeps only its diagonal); ILU(k) patterns nest
    and grow with k; the complete factorisation holds the most."""
    mesh = MESHES[kind]()
    a = pattern_build(mesh)
    arows = [set(a["colidx"][a["rowptr"][i]:a["rowptr"][i + 1]].tolist()) for i in range(mesh.nNode)]
    ndof = mesh.ndim + 1
    dofmap = a["dofmap"].reshape(-1, ndof)
    pats = {k: _rows(ilu_pattern_build(mesh, k, 1)) for k in (0, 1, 3)}
    for i in range(mesh.nNode):
        r0 = set(pats[0][i].tolist())
        if np.all(dofmap[i] < 0):
            assert r0 == {i}
        else:
            assert r0 <= arows[i]
            assert r0 == {j for j in arows[i] if not np.all(dofmap[j] < 0) or j == i}
        assert r0 <= set(pats[1][i].tolist()) <= set(pats[3][i].tolist())
    full = ilu_pattern_build(mesh, -1, 1)["info"].nnzb
    assert sum(len(r) for r in pats[0]) < sum(len(r) for r in pats[3]) <= full


def test_ogrid_numbering_keeps_the_dependency_depth_low():
    """The O-grid is numbered ray by ray: the natural-order ILU's lower DAG
    has about nr + 2 nt levels, not one level per node as ring-by-ring
    numbering (whose ring closure chains every row to the one before) gives."""
    nt, nr = 64, 16
    mesh = meshgen.cylinder_ogrid(nt=nt, nr=nr)
    info = ilu_pattern_build(mesh, 0, 1)["info"]
    assert info.nlev_l <= nr + 2 * nt + 8, info.nlev_l
    assert info.nlev_l < mesh.nNode // 4
