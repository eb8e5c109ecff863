"""Host-side checks that need no GPU: the C ABI library loads and exports
every symbol include/cfdgpu.h declares, and the host-built structures
(free-dof numbering, block pattern, Dirichlet sets, colouring, slot map)
match the oracle bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from cfdsfemmpi_b200 import _lib, io, meshgen, pattern_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cfdgpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char \*|cfdgpu_handle \*)\s*\*?\s*(cfdgpu_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(_lib.EXPORTS) == syms


def _meshes(golden_dir):
    yield "ldc2d10", meshgen.cavity2d(10)
    yield "ldc2d_graded", meshgen.cavity2d(7, pin_node=3, graded_beta=1.2)
    yield "ldc3d6", meshgen.cavity3d(6)
    yield "golden10", io.read_mesh(os.path.join(golden_dir, "ldc2dquad10", "LDC2Dquad10"))
    # unstructured-numbered golden mesh (16,641 nodes)
    yield "mesh2", io.read_mesh(os.path.join(golden_dir, "ldc2dquad-mesh2", "LDC2Dquad-mesh2"))
    # tri3 and tet4: split the structured meshes
    q = meshgen.cavity2d(5)
    tri = q.conn[:, [0, 1, 2]].tolist() + q.conn[:, [0, 2, 3]].tolist()
    yield "tri", io.Mesh(ndim=2, npElem=3, coords=q.coords, conn=np.array(tri, np.int32), dbc=q.dbc,
                         output_nodes=np.zeros(0, np.int32))
    h = meshgen.cavity3d(3)
    tets = []
    for c in h.conn:
        for t in ([0, 1, 3, 4], [1, 2, 3, 6], [1, 3, 4, 6], [1, 4, 5, 6], [3, 4, 6, 7]):
            tets.append(c[t])
    yield "tet", io.Mesh(ndim=3, npElem=4, coords=h.coords, conn=np.array(tets, np.int32), dbc=h.dbc,
                         output_nodes=np.zeros(0, np.int32))


def scalar_pattern_from_blocks(d, ndof):
    """Expand the BSR block pattern to the free-dof scalar pattern."""
    rowptr, colidx, dofmap = d["rowptr"], d["colidx"], d["dofmap"]
    nfree = int(d["info"].nfree)
    rp = [0]
    ci = []
    for n in range(len(rowptr) - 1):
        cols = colidx[rowptr[n]:rowptr[n + 1]]
        for a in range(ndof):
            if dofmap[n * ndof + a] < 0:
                continue
            for mm in cols:
                for b in range(ndof):
                    c = dofmap[mm * ndof + b]
                    if c >= 0:
                        ci.append(c)
            rp.append(len(ci))
    assert len(rp) == nfree + 1
    return np.array(rp, np.int32), np.array(ci, np.int32)


def test_pattern_and_sets_match_oracle(golden_dir):
    L = oracle.lib()
    for name, mesh in _meshes(golden_dir):
        d = pattern_build(mesh)
        ref = oracle.OracleFEM(mesh, io.Control(), solver="lu")
        # free-dof numbering and Dirichlet set (StabFEM2.cpp:57-81)
        assert np.array_equal(d["dofmap"], ref.dofmap), name
        assert np.array_equal(d["fixed_dofs"], np.unique(ref.dbc_index).astype(np.int32)), name
        assert d["info"].nfree == ref.ntot
        # scalar pattern with Dirichlet rows/columns deleted == reference pattern
        if mesh.nNode < 5000:
            rp, ci = scalar_pattern_from_blocks(d, mesh.ndof)
            assert np.array_equal(rp, ref.rowptr), name
            assert np.array_equal(ci, ref.colidx), name
        # colouring: same greedy rule as the oracle
        col = np.zeros(mesh.nElem, np.int32)
        nc = L.orc_color(mesh.nNode, mesh.nElem, mesh.npElem, np.ascontiguousarray(mesh.conn, np.int32), col)
        assert nc == d["info"].ncolors and np.array_equal(col, d["color"]), name


def test_colouring_and_slot_map_invariants(golden_dir):
    for name, mesh in _meshes(golden_dir):
        d = pattern_build(mesh)
        npe = mesh.npElem
        conn = mesh.conn
        color = d["color"]
        # no two elements of one colour share a node
        for c in range(d["info"].ncolors):
            els = np.nonzero(color == c)[0]
            nodes = conn[els].ravel()
            assert len(np.unique(nodes)) == len(nodes), (name, c)
        # colour-ordered element list
        ce, cp = d["color_elems"], d["color_ptr"]
        for c in range(d["info"].ncolors):
            seg = ce[cp[c]:cp[c + 1]]
            assert np.all(color[seg] == c) and np.all(np.diff(seg) > 0)
        # slot map points at block (conn[e][i], conn[e][j])
        slot = d["slot"].reshape(mesh.nElem, npe, npe)
        first = slot < 0
        s = np.where(first, -slot - 1, slot)
        rowptr, colidx = d["rowptr"], d["colidx"]
        assert np.array_equal(colidx[s], np.broadcast_to(conn[:, None, :], s.shape))
        row_of = np.repeat(np.arange(mesh.nNode), np.diff(rowptr))
        assert np.array_equal(row_of[s], np.broadcast_to(conn[:, :, None], s.shape))
        # every block has exactly one first writer, the earliest in launch order
        nnzb = int(d["info"].nnzb)
        assert np.bincount(s[first], minlength=nnzb).max() == 1
        assert np.bincount(s[first], minlength=nnzb).min() == 1
        order = np.empty(mesh.nElem, np.int64)
        order[ce] = np.arange(mesh.nElem)
        pos = np.broadcast_to(order[:, None, None], s.shape)
        earliest = np.full(nnzb, np.iinfo(np.int64).max)
        np.minimum.at(earliest, s.ravel(), pos.ravel())
        assert np.array_equal(earliest[s[first]], pos[first])


def test_pattern_sizes_3d32():
    """Sizes quoted for the 32^3 graded cube: 35,937 nodes, 912,673 blocks,
    18,439 prescribed dofs (walls x 3 + one pressure pin), 8 colours."""
    d = pattern_build(meshgen.cavity3d(32))
    pi = d["info"]
    assert (pi.nNode, pi.nElem, pi.nnzb, pi.nfixed, pi.ncolors) == (35937, 32768, 912673, 18439, 8)
    assert pi.nfree == 35937 * 4 - 18439


def test_create_fails_loudly_without_device():
    """No CPU fallback: without a GPU, cfdgpu_create returns an error."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("GPU present")
    m, c, _ = meshgen.CASES["ldc2d_10"]()
    with pytest.raises(_lib.CfdGpuError) as ei:
        _lib.Handle(m, c)
    assert ei.value.code in (_lib.ENODEV, _lib.ECUDA)


def test_batch_create_fails_loudly_without_device():
    """The batch runtime has no CPU fallback either: without a GPU the first
    instance's create error comes back with the instance named."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("GPU present")
    cases = [(meshgen.cavity2d(n), meshgen.control_for(5, 0.05, 0.01)) for n in (4, 6)]
    with pytest.raises(_lib.CfdGpuError) as ei:
        _lib.Batch(cases)
    assert ei.value.code in (_lib.ENODEV, _lib.ECUDA)
    assert "instance 0" in str(ei.value)


@pytest.mark.parametrize("case", ["empty", "node_out_of_range", "negative_node", "repeated_node", "bad_dbc_node",
                                  "bad_dbc_dof"])
def test_invalid_meshes_are_rejected(case):
    """Bad input comes back as CFDGPU_EINVAL from the host set-up (the same
    checks run in cfdgpu_create before anything reaches the device)."""
    m = meshgen.cavity2d(3)
    conn = m.conn.copy()
    dbc = m.dbc.copy()
    nNode = m.nNode
    if case == "empty":
        conn = conn[:0]
    elif case == "node_out_of_range":
        conn[2, 1] = nNode
    elif case == "negative_node":
        conn[0, 0] = -1
    elif case == "repeated_node":
        conn[1, 2] = conn[1, 0]
    elif case == "bad_dbc_node":
        dbc[0, 0] = nNode + 5
    elif case == "bad_dbc_dof":
        dbc[0, 1] = 3
    bad = io.Mesh(ndim=2, npElem=4, coords=m.coords, conn=conn, dbc=dbc, output_nodes=np.zeros(0, np.int32))
    with pytest.raises(_lib.CfdGpuError) as ei:
        pattern_build(bad)
    assert ei.value.code == _lib.EINVAL


def test_cylinder_ogrid_matches_its_description():
    """O-grid of the cylinder-wake configuration: 256 x 128 quads (33,024
    nodes), radial spacing 0.005 at r = 0.5 growing geometrically to r = 20,
    counter-clockwise elements, no-slip on the cylinder, inflow on the outer
    arc where x < 0, nothing prescribed where x >= 0; nodes numbered ray by
    ray (radial index fastest)."""
    m = meshgen.cylinder_ogrid()
    assert (m.nNode, m.nElem) == (33024, 32768)
    r = np.hypot(m.coords[:, 0], m.coords[:, 1]).reshape(256, 129)
    assert np.allclose(r[:, 0], 0.5) and np.allclose(r[:, -1], 20.0)
    assert abs((r[0, 1] - r[0, 0]) - 0.005) < 1e-12
    dr = np.diff(r[0])
    assert np.allclose(dr[1:] / dr[:-1], dr[1] / dr[0])
    th = np.arctan2(m.coords[:, 1], m.coords[:, 0]).reshape(256, 129)
    assert np.allclose(th[:, 0], th[:, -1]) and np.all(np.diff(np.unwrap(th[:, 0])) > 0)
    p = m.coords[m.conn]
    area2 = (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 3, 1] - p[:, 1, 1]) - (p[:, 2, 1] - p[:, 0, 1]) * (p[:, 3, 0] - p[:, 1, 0])
    assert np.all(area2 > 0)
    d = m.dbc
    on_cyl = d[:, 0].astype(int) % 129 == 0
    cyl = d[on_cyl]
    assert len(cyl) == 512 and np.all(cyl[:, 2] == 0.0)
    outer = d[~on_cyl]
    assert np.all(outer[:, 0].astype(int) % 129 == 128)
    assert np.all(m.coords[outer[:, 0].astype(int), 0] < 0)
    assert np.all(outer[outer[:, 1] == 0, 2] == 1.0) and np.all(outer[outer[:, 1] == 1, 2] == 0.0)
    assert not np.any(d[:, 1] == 2)
    u0 = meshgen.cylinder_initial_state(m)
    assert np.all(u0.reshape(-1, 3)[:, [0, 2]] == 0) and 0 < np.abs(u0).max() <= 1e-3


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_pattern_matches_oracle_on_renumbered_meshes(seed):
    """Ragged numbering: the cavity meshes with nodes and elements in random
    order (and a pressure pin moved with them) give the oracle's free-dof
    numbering, scalar pattern and colouring, bit for bit."""
    rng = np.random.default_rng(seed)
    for base in (meshgen.cavity2d(6), meshgen.cavity3d(3)):
        perm = rng.permutation(base.nNode)          # old -> new node id
        eorder = rng.permutation(base.nElem)
        coords = np.empty_like(base.coords)
        coords[perm] = base.coords
        conn = perm[base.conn[eorder]].astype(np.int32)
        dbc = base.dbc.copy()
        dbc[:, 0] = perm[dbc[:, 0].astype(int)]
        mesh = io.Mesh(ndim=base.ndim, npElem=base.npElem, coords=coords, conn=conn, dbc=dbc,
                       output_nodes=np.zeros(0, np.int32))
        d = pattern_build(mesh)
        ref = oracle.OracleFEM(mesh, io.Control(), solver="lu")
        assert np.array_equal(d["dofmap"], ref.dofmap)
        rp, ci = scalar_pattern_from_blocks(d, mesh.ndof)
        assert np.array_equal(rp, ref.rowptr) and np.array_equal(ci, ref.colidx)
        col = np.zeros(mesh.nElem, np.int32)
        nc = oracle.lib().orc_color(mesh.nNode, mesh.nElem, mesh.npElem, np.ascontiguousarray(mesh.conn, np.int32), col)
        assert nc == d["info"].ncolors and np.array_equal(col, d["color"])
