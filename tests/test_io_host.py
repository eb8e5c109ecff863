"""Reference-format input/output and the VTU writer, on the host: files
written by this package read back to the same data, in the layouts the
reference's readers and writers use."""
import os

import numpy as np
import pytest

from cfdsfemmpi_b200 import io, meshgen
from cfdsfemmpi_b200.vtu import read_vtu_point_data, write_vtu


@pytest.mark.parametrize("kind", ["quad4", "hex8"])
def test_case_files_round_trip(kind, tmp_path):
    mesh = meshgen.cavity2d(5) if kind == "quad4" else meshgen.cavity3d(3)
    ctrl = meshgen.control_for(7, 0.05, 0.002)
    opts = {"-ksp_type": "gmres", "-ksp_gmres_restart": "50", "-pc_type": "jacobi", "-ksp_rtol": "1.e-10"}
    mp, cp, op = meshgen.write_case(str(tmp_path), "case", mesh, ctrl, opts)
    m2 = io.read_mesh(mp)
    assert (m2.ndim, m2.npElem, m2.nNode, m2.nElem) == (mesh.ndim, mesh.npElem, mesh.nNode, mesh.nElem)
    assert np.allclose(m2.coords, mesh.coords, rtol=0, atol=1e-12)
    assert np.array_equal(m2.conn, mesh.conn)
    assert np.array_equal(m2.dbc[:, :2], mesh.dbc[:, :2]) and np.allclose(m2.dbc[:, 2], mesh.dbc[:, 2])
    c2 = io.read_control(cp)
    assert np.allclose(c2.elem_data(), ctrl.elem_data())
    assert (c2.tis, c2.dt, c2.stepsMax) == (ctrl.tis, ctrl.dt, ctrl.stepsMax)
    assert io.read_options(op) == opts


def test_result_file_round_trip_and_check(tmp_path):
    rng = np.random.default_rng(3)
    n = 121
    s = rng.uniform(-1, 1, n * 3)
    path = str(tmp_path / "res.dat")
    assert io.write_result(path, s, n, 3) == 0
    back = io.read_result(path)
    assert back.shape == (n, 3) and np.abs(back.ravel() - s).max() < 5e-9
    assert io.check_result(path, s, n, 2) == 0
    s2 = s.copy()
    s2[7] += 1e-3
    assert io.check_result(path, s2, n, 2) != 0


@pytest.mark.parametrize("kind,ctype", [("quad4", 9), ("hex8", 12), ("tri3", 5), ("tet4", 10)])
def test_vtu_writer_fields_and_cells(kind, ctype, tmp_path):
    if kind in ("quad4", "tri3"):
        mesh = meshgen.cavity2d(4)
        if kind == "tri3":
            c = mesh.conn
            mesh = io.Mesh(ndim=2, npElem=3, coords=mesh.coords,
                           conn=np.array(c[:, [0, 1, 2]].tolist() + c[:, [0, 2, 3]].tolist(), np.int32),
                           dbc=mesh.dbc, output_nodes=np.zeros(0, np.int32))
    else:
        mesh = meshgen.cavity3d(2)
        if kind == "tet4":
            tets = [c[t] for c in mesh.conn for t in ([0, 1, 3, 4], [1, 2, 3, 6], [1, 3, 4, 6], [1, 4, 5, 6], [3, 4, 6, 7])]
            mesh = io.Mesh(ndim=3, npElem=4, coords=mesh.coords, conn=np.array(tets, np.int32), dbc=mesh.dbc,
                           output_nodes=np.zeros(0, np.int32))
    ndof = mesh.ndim + 1
    s = np.random.default_rng(1).uniform(-2, 2, mesh.nNode * ndof)
    f = str(tmp_path / "out-000000.vtu")
    write_vtu(f, mesh, s, proc_id=0)
    d = read_vtu_point_data(f)
    s = s.reshape(-1, ndof)
    assert d["velocity"].shape == (mesh.nNode, 3)
    assert np.allclose(d["velocity"][:, :mesh.ndim], s[:, :mesh.ndim].astype(np.float32))
    if mesh.ndim == 2:
        assert np.all(d["velocity"][:, 2] == 0)
    assert np.allclose(d["pressure"], s[:, mesh.ndim].astype(np.float32))
    text = open(f).read()
    assert f'NumberOfPoints="{mesh.nNode}"' in text and f'NumberOfCells="{mesh.nElem}"' in text
    types = text.split('Name="types"')[1].split(">", 1)[1].split("<")[0].split()
    assert len(types) == mesh.nElem and set(types) == {str(ctype)}
