"""Headless VTK XML unstructured-grid (.vtu) writer.

Writes the fields of StabFEM::postProcess (src/base/StabFEM3.cpp:6-160):
point data ``velocity`` (3 components, w = 0 in 2D), ``pressure`` and
``procId``; cell data ``procId``; cells of VTK type triangle (5), quad (9),
tetra (10) or hexahedron (12) with the mesh's node order; file name
``<prefix>-%06d.vtu``.  Values are stored as Float32 like the reference's
vtkFloatArray.  No graphics library is involved.
"""
from __future__ import annotations

import numpy as np

_CELL_TYPE = {(2, 3): 5, (2, 4): 9, (3, 4): 10, (3, 8): 12}


def write_vtu(fname: str, mesh, soln: np.ndarray, proc_id: int = 0) -> None:
    nn, ne = mesh.nNode, mesh.nElem
    ndof = mesh.ndim + 1
    s = np.asarray(soln).reshape(nn, ndof)
    pts = np.zeros((nn, 3), dtype=np.float32)
    pts[:, :mesh.ndim] = mesh.coords
    vel = np.zeros((nn, 3), dtype=np.float32)
    vel[:, :mesh.ndim] = s[:, :mesh.ndim]
    pres = s[:, mesh.ndim].astype(np.float32)
    ctype = _CELL_TYPE[(mesh.ndim, mesh.npElem)]
    conn = np.asarray(mesh.conn, dtype=np.int64)
    offsets = np.arange(1, ne + 1, dtype=np.int64) * mesh.npElem
    f32 = lambda a: " ".join(f"{v:.9g}" for v in np.asarray(a, dtype=np.float32).ravel())
    ints = lambda a: " ".join(str(int(v)) for v in np.asarray(a).ravel())
    with open(fname, "w") as f:
        f.write('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">\n')
        f.write(f'<UnstructuredGrid>\n<Piece NumberOfPoints="{nn}" NumberOfCells="{ne}">\n')
        f.write('<PointData Scalars="pressure" Vectors="velocity">\n')
        f.write(f'<DataArray type="Float32" Name="pressure" format="ascii">\n{f32(pres)}\n</DataArray>\n')
        f.write(f'<DataArray type="Float32" Name="procId" format="ascii">\n{f32(np.full(nn, proc_id))}\n</DataArray>\n')
        f.write(f'<DataArray type="Float32" Name="velocity" NumberOfComponents="3" format="ascii">\n{f32(vel)}\n'
                '</DataArray>\n</PointData>\n')
        f.write('<CellData Scalars="procId">\n')
        f.write(f'<DataArray type="Float32" Name="procId" format="ascii">\n{f32(np.full(ne, proc_id))}\n</DataArray>\n'
                '</CellData>\n')
        f.write(f'<Points>\n<DataArray type="Float32" NumberOfComponents="3" format="ascii">\n{f32(pts)}\n'
                '</DataArray>\n</Points>\n')
        f.write('<Cells>\n')
        f.write(f'<DataArray type="Int64" Name="connectivity" format="ascii">\n{ints(conn)}\n</DataArray>\n')
        f.write(f'<DataArray type="Int64" Name="offsets" format="ascii">\n{ints(offsets)}\n</DataArray>\n')
        f.write(f'<DataArray type="UInt8" Name="types" format="ascii">\n{ints(np.full(ne, ctype))}\n</DataArray>\n')
        f.write('</Cells>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n')


def read_vtu_point_data(fname: str) -> dict:
    """Parse the ASCII arrays back (used by tests)."""
    import re
    text = open(fname).read()
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)" Name="(\w+)"(?: NumberOfComponents="(\d)")? format="ascii">\n(.*?)\n</DataArray>',
                         text, re.S):
        dt = np.float32 if m.group(1).startswith("Float") else np.int64
        arr = np.array(m.group(4).split(), dtype=dt)
        if m.group(3):
            arr = arr.reshape(-1, int(m.group(3)))
        out.setdefault(m.group(2), arr)
    return out
